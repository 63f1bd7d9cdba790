"""ctypes binding of libzlfft_cuda.so (the C ABI in include/zlfft.h).

The library is loaded from this package's lib/ directory. There is no
fallback: if the library is missing or fails to load, every entry point
raises, so a missing build can never silently turn into a CPU computation.
"""
from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libzlfft_cuda.so")

# constants mirrored from include/zlfft.h
OK = 0
ERR_INVALID_ARG = -1
ERR_UNSUPPORTED = -2
ERR_ALIGNMENT = -3
ERR_CUDA = -4
ERR_ALLOC = -5
ERR_DEVICE_TIMEOUT = -6

C2C, R2C = 0, 1
F32, F64 = 0, 1
AOS, SOA = 0, 1
FORWARD, BACKWARD, FORWARD_SQR_MAG = 0, 1, 2
MODE_PLAIN, MODE_TC_FP16, MODE_TUNED, MODE_FAST, MODE_HOST = 0, 1, 4, 5, 6
SCHED_PER_ORDER, SCHED_PERSISTENT, SCHED_GRAPH = 0, 1, 2


class Desc(ctypes.Structure):
    """zlfft_desc: one transform of a mixed batch (device pointers)."""
    _fields_ = [("kind", ctypes.c_int), ("precision", ctypes.c_int), ("order", ctypes.c_int), ("op", ctypes.c_int),
                ("in_", ctypes.c_void_p), ("out", ctypes.c_void_p)]


class Tuning(ctypes.Structure):
    """zlfft_tuning: the measured plan parameters of one transform size."""
    _fields_ = [("chunk_mb", ctypes.c_int), ("streams", ctypes.c_int), ("tma", ctypes.c_int), ("form", ctypes.c_int),
                ("split_fused", ctypes.c_int), ("store_tma", ctypes.c_int), ("gbs", ctypes.c_double),
                ("gbs_default", ctypes.c_double)]


# every symbol include/zlfft.h declares
EXPORTS = (
    "zlfft_plan_create",
    "zlfft_plan_create_hybrid",
    "zlfft_host_switch_order",
    "zlfft_plan_get_micro_order",
    "zlfft_plan_destroy",
    "zlfft_plan_get_size",
    "zlfft_plan_get_order",
    "zlfft_exec_host",
    "zlfft_exec_host_batched",
    "zlfft_exec_device",
    "zlfft_exec_device_noalloc",
    "zlfft_stft_device",
    "zlfft_istft_device",
    "zlfft_plan_take_launch_count",
    "zlfft_plan_copy_twiddles",
    "zlfft_plan_device_status",
    "zlfft_selftest_bounded_wait",
    "zlfft_selftest_tc_dft16",
    "zlfft_mixed_create",
    "zlfft_mixed_exec",
    "zlfft_mixed_take_launch_count",
    "zlfft_mixed_device_status",
    "zlfft_mixed_destroy",
    "zlfft_exec_mixed_device",
    "zlfft_autotune",
    "zlfft_tuning_get",
    "zlfft_tuning_save",
    "zlfft_tuning_load",
    "zlfft_tuning_clear",
    "zlfft_last_error",
    "zlfft_version",
)


class ZlfftError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"zlfft error {code}: {msg}")
        self.code = code


_lib = None
_lock = threading.Lock()


def lib() -> ctypes.CDLL:
    """Load and type the library (raises if it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"libzlfft_cuda.so not found at {LIB_PATH}; build it with `python -m zldsp_fft_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        sz, vp, i = ctypes.c_size_t, ctypes.c_void_p, ctypes.c_int
        L.zlfft_plan_create.argtypes = [ctypes.POINTER(vp), i, i, sz, i, i]
        L.zlfft_plan_create_hybrid.argtypes = [ctypes.POINTER(vp), i, i, sz, i, i, i]
        L.zlfft_host_switch_order.argtypes = [i, ctypes.POINTER(sz), ctypes.POINTER(sz)]
        L.zlfft_plan_get_micro_order.argtypes = [vp, ctypes.POINTER(i)]
        L.zlfft_plan_destroy.argtypes = [vp]
        L.zlfft_plan_get_size.argtypes = [vp, ctypes.POINTER(sz)]
        L.zlfft_plan_get_order.argtypes = [vp, ctypes.POINTER(sz)]
        L.zlfft_exec_host.argtypes = [vp, i, i, i, vp, vp, vp, vp]
        L.zlfft_exec_host_batched.argtypes = [vp, i, i, i, vp, vp, vp, vp, sz]
        L.zlfft_exec_device.argtypes = [vp, i, i, i, vp, vp, vp, vp, sz, sz, sz, vp]
        L.zlfft_exec_device_noalloc.argtypes = [vp, i, i, i, vp, vp, vp, vp, sz, sz, sz, vp]
        L.zlfft_stft_device.argtypes = [vp, i, i, vp, sz, vp, vp, vp, sz, sz, vp]
        L.zlfft_istft_device.argtypes = [vp, i, vp, vp, sz, vp, vp, sz, sz, vp, vp]
        L.zlfft_plan_take_launch_count.argtypes = [vp, ctypes.POINTER(sz)]
        L.zlfft_plan_copy_twiddles.argtypes = [vp, vp, sz, ctypes.POINTER(sz)]
        L.zlfft_plan_device_status.argtypes = [vp, ctypes.POINTER(i)]
        L.zlfft_selftest_bounded_wait.argtypes = [i, ctypes.POINTER(i)]
        L.zlfft_selftest_tc_dft16.argtypes = [i, vp, vp, ctypes.POINTER(i)]
        L.zlfft_mixed_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(Desc), sz, i]
        L.zlfft_mixed_exec.argtypes = [vp, i, vp]
        L.zlfft_mixed_take_launch_count.argtypes = [vp, ctypes.POINTER(sz)]
        L.zlfft_mixed_device_status.argtypes = [vp, ctypes.POINTER(i)]
        L.zlfft_mixed_destroy.argtypes = [vp]
        L.zlfft_exec_mixed_device.argtypes = [ctypes.POINTER(Desc), sz, vp]
        L.zlfft_autotune.argtypes = [i, i, i, sz, sz]
        L.zlfft_tuning_get.argtypes = [i, i, i, sz, ctypes.POINTER(Tuning)]
        L.zlfft_tuning_save.argtypes = [i, ctypes.c_char_p]
        L.zlfft_tuning_load.argtypes = [i, ctypes.c_char_p, ctypes.POINTER(sz)]
        L.zlfft_tuning_clear.argtypes = []
        L.zlfft_last_error.restype = ctypes.c_char_p
        L.zlfft_last_error.argtypes = []
        L.zlfft_version.restype = ctypes.c_char_p
        L.zlfft_version.argtypes = []
        for name in EXPORTS:
            getattr(L, name).restype = getattr(L, name).restype if name in ("zlfft_last_error", "zlfft_version") else i
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != OK:
        raise ZlfftError(rc, lib().zlfft_last_error().decode())


def last_error() -> str:
    return lib().zlfft_last_error().decode()


def version() -> str:
    return lib().zlfft_version().decode()
