"""Host-side mirror of the reference's operator interface.

``CFFT`` and ``RFFT`` have the constructors, getters and forward/backward
member functions of zldsp::fft::CFFT<F> (src/zldsp_fft_cfft.hpp:11-118) and
zldsp::fft::RFFT<F> (src/zldsp_fft_rfft.hpp:11-139), taking numpy host
buffers: an AoS complex buffer is a complex ndarray, a split-SoA buffer is a
pair ``(re, im)`` of real ndarrays, exactly the reference's
``std::complex<F>*`` / ``std::array<F*, 2>`` overloads. Calls are synchronous
and write into the caller's output buffers, like the reference.

``Plan`` is the batched device-pointer entry point (zlfft_exec_device) for
callers that keep data in GPU memory (raw pointers or torch CUDA tensors).

Everything runs on the GPU through libzlfft_cuda.so; there is no CPU path.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi as C


def _prec(dtype) -> int:
    dt = np.dtype(dtype)
    if dt in (np.float32, np.complex64):
        return C.F32
    if dt in (np.float64, np.complex128):
        return C.F64
    raise TypeError(f"unsupported dtype {dt}; the reference is instantiated for float and double")


def host_switch_order(dtype=np.float32):
    """(max_l1_order, switch_order) the reference computes from this host's
    caches (zlfft_host_switch_order; src/common/zldsp_fft_common_system.hpp:132-157)."""
    a, b = ctypes.c_size_t(), ctypes.c_size_t()
    C.check(C.lib().zlfft_host_switch_order(_prec(dtype), ctypes.byref(a), ctypes.byref(b)))
    return a.value, b.value


class Plan:
    """A zlfft plan (one transform size, kind, precision and form).

    ``switch=(max_l1_order, switch_order)`` makes a plain plan follow the
    reference's algorithm switch with those values (zlfft_plan_create_hybrid):
    orders at or above switch_order run the reference's macro DIF path."""

    def __init__(self, kind: int, order: int, dtype=np.float32, mode: int = C.MODE_PLAIN, device: int = -1,
                 switch=None):
        self._lib = C.lib()
        self.kind = kind
        self.order = int(order)
        self.prec = _prec(dtype)
        self.mode = mode
        h = ctypes.c_void_p()
        if switch is not None:
            C.check(self._lib.zlfft_plan_create_hybrid(ctypes.byref(h), kind, self.prec, self.order, int(switch[0]),
                                                       int(switch[1]), device))
        else:
            C.check(self._lib.zlfft_plan_create(ctypes.byref(h), kind, self.prec, self.order, mode, device))
        self.handle = h

    def micro_order(self) -> int:
        """Micro order of the plan's macro path, -1 on the micro-only path."""
        v = ctypes.c_int()
        C.check(self._lib.zlfft_plan_get_micro_order(self.handle, ctypes.byref(v)))
        return v.value

    @property
    def real_dtype(self):
        return np.float32 if self.prec == C.F32 else np.float64

    @property
    def complex_dtype(self):
        return np.complex64 if self.prec == C.F32 else np.complex128

    def close(self):
        if getattr(self, "handle", None) and self.handle.value:
            self._lib.zlfft_plan_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_size(self) -> int:
        v = ctypes.c_size_t()
        C.check(self._lib.zlfft_plan_get_size(self.handle, ctypes.byref(v)))
        return v.value

    def get_order(self) -> int:
        v = ctypes.c_size_t()
        C.check(self._lib.zlfft_plan_get_order(self.handle, ctypes.byref(v)))
        return v.value

    def exec_device(self, op, in_layout, out_layout, in0, in1, out0, out1, batch, in_stride=0, out_stride=0,
                    stream=0):
        """Batched transform on device pointers (ints), async on `stream` (cudaStream_t as int)."""
        C.check(self._lib.zlfft_exec_device(self.handle, op, in_layout, out_layout, in0, in1, out0, out1,
                                            int(batch), int(in_stride), int(out_stride), stream))

    def stft(self, op, out_layout, signal, hop, window, out0, out1, n_frames, out_stride=0, stream=0):
        """STFT frames of a device signal (zlfft_stft_device): frame f is
        signal[f*hop : f*hop + N] * window, through forward or forward_sqr_mag."""
        C.check(self._lib.zlfft_stft_device(self.handle, op, out_layout, signal, int(hop), window, out0, out1,
                                            int(n_frames), int(out_stride), stream))

    def istft(self, in_layout, in0, in1, hop, n_frames, signal, filter=None, window=None, in_stride=0, stream=0):
        """Inverse STFT with overlap-add of device bins (zlfft_istft_device):
        signal[f*hop + n] = sum over frames f, in order, of
        window[n] * backward(filter * bins_f)[n]; the signal holds
        (n_frames - 1) * hop + N reals and is written, not accumulated into."""
        C.check(self._lib.zlfft_istft_device(self.handle, in_layout, in0, in1, int(in_stride), filter, window, int(hop),
                                             int(n_frames), signal, stream))

    def exec_host(self, op, in_layout, out_layout, in0, in1, out0, out1, batch=1):
        C.check(self._lib.zlfft_exec_host_batched(self.handle, op, in_layout, out_layout, in0, in1, out0, out1,
                                                  int(batch)))

    def take_launch_count(self) -> int:
        v = ctypes.c_size_t()
        C.check(self._lib.zlfft_plan_take_launch_count(self.handle, ctypes.byref(v)))
        return v.value

    def device_status(self) -> int:
        """Synchronise, then read and clear the plan's device error word (0 = ok)."""
        v = ctypes.c_int()
        self._lib.zlfft_plan_device_status(self.handle, ctypes.byref(v))
        return v.value

    def twiddles(self) -> np.ndarray:
        """The device-generated unified twiddle table, copied to the host."""
        n = ctypes.c_size_t()
        C.check(self._lib.zlfft_plan_copy_twiddles(self.handle, None, 0, ctypes.byref(n)))
        out = np.zeros(max(n.value, 1), self.complex_dtype)
        C.check(self._lib.zlfft_plan_copy_twiddles(self.handle, out.ctypes.data, out.size, ctypes.byref(n)))
        return out[: n.value]


def _complex_arg(buf, n, cdt, rdt, name, writable):
    """(layout, ptr0, ptr1) for an AoS ndarray or an SoA (re, im) pair."""
    if isinstance(buf, (tuple, list)):
        if len(buf) != 2:
            raise ValueError(f"{name}: SoA buffer must be a (re, im) pair")
        re, im = buf
        for a in (re, im):
            if not isinstance(a, np.ndarray) or a.dtype != rdt or not a.flags.c_contiguous or a.size < n:
                raise ValueError(f"{name}: SoA parts must be contiguous {np.dtype(rdt)} arrays of >= {n} elements")
            if writable and not a.flags.writeable:
                raise ValueError(f"{name}: output is read-only")
        return C.SOA, re.ctypes.data, im.ctypes.data
    if not isinstance(buf, np.ndarray) or buf.dtype != cdt or not buf.flags.c_contiguous or buf.size < n:
        raise ValueError(f"{name}: AoS buffer must be a contiguous {np.dtype(cdt)} array of >= {n} elements")
    if writable and not buf.flags.writeable:
        raise ValueError(f"{name}: output is read-only")
    return C.AOS, buf.ctypes.data, None


def _real_arg(buf, n, rdt, name, writable):
    if not isinstance(buf, np.ndarray) or buf.dtype != rdt or not buf.flags.c_contiguous or buf.size < n:
        raise ValueError(f"{name}: must be a contiguous {np.dtype(rdt)} array of >= {n} elements")
    if writable and not buf.flags.writeable:
        raise ValueError(f"{name}: output is read-only")
    return buf.ctypes.data


class CFFT:
    """zldsp::fft::CFFT<F> on the GPU (src/zldsp_fft_cfft.hpp:11-118).

    forward/backward(in, out) accept the reference's four layout pairings:
    AoS->AoS, AoS->SoA, SoA->AoS, SoA->SoA. backward is the unnormalised
    inverse (backward(forward(x)) == N * x). By default the plan follows the
    reference's algorithm switch as this host's caches set it
    (MODE_HOST), so the results are the reference's on this host."""

    def __init__(self, order: int, dtype=np.float32, mode: int = C.MODE_HOST):
        self._plan = Plan(C.C2C, order, dtype, mode)
        self._n = 1 << int(order)

    def get_size(self) -> int:
        return self._plan.get_size()

    def get_order(self) -> int:
        return self._plan.get_order()

    def _exec(self, op, in_buffer, out_buffer):
        p = self._plan
        il, i0, i1 = _complex_arg(in_buffer, self._n, p.complex_dtype, p.real_dtype, "in_buffer", False)
        ol, o0, o1 = _complex_arg(out_buffer, self._n, p.complex_dtype, p.real_dtype, "out_buffer", True)
        p.exec_host(op, il, ol, i0, i1, o0, o1)

    def forward(self, in_buffer, out_buffer) -> None:
        self._exec(C.FORWARD, in_buffer, out_buffer)

    def backward(self, in_buffer, out_buffer) -> None:
        self._exec(C.BACKWARD, in_buffer, out_buffer)

    @property
    def plan(self) -> Plan:
        return self._plan


class RFFT:
    """zldsp::fft::RFFT<F> on the GPU (src/zldsp_fft_rfft.hpp:11-139).

    forward(real_in, out) writes N/2+1 bins (AoS ndarray or SoA pair);
    backward(in, real_out) is unnormalised (backward(forward(x)) == N/2 * x);
    forward_sqr_mag(real_in, out) writes N/2+1 squared magnitudes. Like CFFT,
    it follows the reference's algorithm switch of this host by default."""

    def __init__(self, order: int, dtype=np.float32, mode: int = C.MODE_HOST):
        self._plan = Plan(C.R2C, order, dtype, mode)
        self._n = 1 << int(order)
        self._nb = self._n // 2 + 1

    def get_size(self) -> int:
        return self._plan.get_size()

    def get_order(self) -> int:
        return self._plan.get_order()

    def forward(self, in_buffer, out_buffer) -> None:
        p = self._plan
        i0 = _real_arg(in_buffer, self._n, p.real_dtype, "in_buffer", False)
        ol, o0, o1 = _complex_arg(out_buffer, self._nb, p.complex_dtype, p.real_dtype, "out_buffer", True)
        p.exec_host(C.FORWARD, C.AOS, ol, i0, None, o0, o1)

    def backward(self, in_buffer, out_buffer) -> None:
        p = self._plan
        il, i0, i1 = _complex_arg(in_buffer, self._nb, p.complex_dtype, p.real_dtype, "in_buffer", False)
        o0 = _real_arg(out_buffer, self._n, p.real_dtype, "out_buffer", True)
        p.exec_host(C.BACKWARD, il, C.AOS, i0, i1, o0, None)

    def forward_sqr_mag(self, in_buffer, out_buffer) -> None:
        p = self._plan
        i0 = _real_arg(in_buffer, self._n, p.real_dtype, "in_buffer", False)
        o0 = _real_arg(out_buffer, self._nb, p.real_dtype, "out_buffer", True)
        p.exec_host(C.FORWARD_SQR_MAG, C.AOS, C.AOS, i0, None, o0, None)

    @property
    def plan(self) -> Plan:
        return self._plan


class MixedBatch:
    """Transforms of many orders and kinds in one call (zlfft_mixed_*).

    ``descs`` is a sequence of ``(kind, order, op, in_ptr, out_ptr)`` tuples
    (device pointers as ints, AoS buffers), all of precision ``dtype``, or of
    ``(kind, order, op, in_ptr, out_ptr, precision)`` to mix precisions.
    ``run(schedule)`` executes the whole batch on ``stream``; the schedules
    are SCHED_PER_ORDER (one batched launch per order group),
    SCHED_PERSISTENT (orders up to 2^11 complex in one persistent launch) and
    SCHED_GRAPH (the persistent schedule replayed from a CUDA graph).
    """

    def __init__(self, descs, dtype=np.float32, device: int = -1):
        self._lib = C.lib()
        prec = _prec(dtype)
        arr = (C.Desc * max(len(descs), 1))()
        for i, d in enumerate(descs):
            kind, order, op, ip, op_ptr = d[:5]
            arr[i] = C.Desc(kind, d[5] if len(d) > 5 else prec, int(order), op, int(ip), int(op_ptr))
        h = ctypes.c_void_p()
        C.check(self._lib.zlfft_mixed_create(ctypes.byref(h), arr, len(descs), device))
        self.handle = h
        self.size = len(descs)

    def run(self, schedule: int = C.SCHED_PERSISTENT, stream=0) -> None:
        C.check(self._lib.zlfft_mixed_exec(self.handle, schedule, stream))

    def take_launch_count(self) -> int:
        v = ctypes.c_size_t()
        C.check(self._lib.zlfft_mixed_take_launch_count(self.handle, ctypes.byref(v)))
        return v.value

    def device_status(self) -> int:
        v = ctypes.c_int()
        self._lib.zlfft_mixed_device_status(self.handle, ctypes.byref(v))
        return v.value

    def close(self):
        if getattr(self, "handle", None) and self.handle.value:
            self._lib.zlfft_mixed_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune(kind: int, order_lo: int, order_hi: int, dtype=np.float32, device: int = -1) -> None:
    """Measure the candidate plans of every order in [order_lo, order_hi] on the
    device and record the fastest (zlfft_autotune); later plans use them."""
    C.check(C.lib().zlfft_autotune(device, kind, _prec(dtype), int(order_lo), int(order_hi)))


def tuning(kind: int, order: int, dtype=np.float32, device: int = -1):
    """The tuning entry of a size as a dict, or None if it has none."""
    t = C.Tuning()
    rc = C.lib().zlfft_tuning_get(device, kind, _prec(dtype), int(order), ctypes.byref(t))
    if rc == C.ERR_UNSUPPORTED:
        return None
    C.check(rc)
    return {"chunk_mb": t.chunk_mb, "streams": t.streams, "tma": t.tma,
            "form": {C.MODE_TC_FP16: "tc_fp16", C.MODE_FAST: "fast"}.get(t.form, "plain"),
            "split_fused": t.split_fused,
            "store_tma": t.store_tma,
            "gbs": t.gbs, "gbs_default": t.gbs_default}


def tuning_save(path: str, device: int = -1) -> None:
    C.check(C.lib().zlfft_tuning_save(device, path.encode()))


def tuning_load(path: str, device: int = -1) -> int:
    n = ctypes.c_size_t()
    C.check(C.lib().zlfft_tuning_load(device, path.encode(), ctypes.byref(n)))
    return n.value


def tuning_clear() -> None:
    C.check(C.lib().zlfft_tuning_clear())
