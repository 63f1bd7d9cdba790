"""C ABI checks that need no GPU: the library loads, exports every symbol
include/zlfft.h declares, and rejects invalid arguments before touching CUDA
(the reference has no defined behaviour for these; the ABI reports them)."""
import ctypes
import os
import re

import pytest

import zldsp_fft_b200 as Z
from zldsp_fft_b200 import _capi as C

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "zlfft.h")).read()
    return sorted(set(re.findall(r"ZLFFT_API\s+(?:const\s+)?\w+\*?\s+\**(zlfft_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = C.lib()
    declared = _declared()
    assert declared, "no declarations parsed"
    assert sorted(C.EXPORTS) == declared
    for name in declared:
        assert hasattr(lib, name), name
    assert "sm_100a" in C.version()


def test_invalid_arguments_rejected_without_cuda():
    lib = C.lib()
    h = ctypes.c_void_p()
    assert lib.zlfft_plan_create(None, 0, 0, 4, 0, -1) == C.ERR_INVALID_ARG
    assert lib.zlfft_plan_create(ctypes.byref(h), 7, 0, 4, 0, -1) == C.ERR_INVALID_ARG
    assert lib.zlfft_plan_create(ctypes.byref(h), 0, 5, 4, 0, -1) == C.ERR_INVALID_ARG
    assert lib.zlfft_plan_create(ctypes.byref(h), 0, 0, 31, 0, -1) == C.ERR_INVALID_ARG
    # the reference's RFFT(0) underflows (src/zldsp_fft_rfft.hpp:26); the ABI refuses it
    assert lib.zlfft_plan_create(ctypes.byref(h), C.R2C, 0, 0, 0, -1) == C.ERR_INVALID_ARG
    assert "RFFT order" in C.last_error()
    assert lib.zlfft_exec_device(None, 0, 0, 0, None, None, None, None, 1, 0, 0, None) == C.ERR_INVALID_ARG
    assert lib.zlfft_plan_destroy(None) == C.OK
    sz = ctypes.c_size_t()
    assert lib.zlfft_plan_get_size(None, ctypes.byref(sz)) == C.ERR_INVALID_ARG


def test_tuning_arguments_rejected_without_cuda():
    lib = C.lib()
    assert lib.zlfft_autotune(0, 7, C.F32, 10, 12) == C.ERR_INVALID_ARG
    assert lib.zlfft_autotune(0, C.C2C, 9, 10, 12) == C.ERR_INVALID_ARG
    assert lib.zlfft_autotune(0, C.C2C, C.F32, 12, 10) == C.ERR_UNSUPPORTED
    assert lib.zlfft_autotune(0, C.R2C, C.F32, 0, 3) == C.ERR_UNSUPPORTED
    assert lib.zlfft_tuning_get(0, C.C2C, C.F32, 10, None) == C.ERR_INVALID_ARG
    assert lib.zlfft_tuning_save(0, None) == C.ERR_INVALID_ARG
    assert lib.zlfft_tuning_load(0, None, None) == C.ERR_INVALID_ARG
    assert lib.zlfft_tuning_clear() == C.OK


def test_mixed_batch_descriptors_rejected_without_cuda():
    """zlfft_mixed_create checks every descriptor before it touches CUDA."""
    lib = C.lib()
    h = ctypes.c_void_p()
    ok = dict(kind=C.C2C, precision=C.F32, order=10, op=C.FORWARD, in_=4096, out=8192)

    def one(**kw):
        d = dict(ok)
        d.update(kw)
        arr = (C.Desc * 2)(C.Desc(**ok), C.Desc(**d))
        return lib.zlfft_mixed_create(ctypes.byref(h), arr, 2, -1)

    assert lib.zlfft_mixed_create(None, None, 0, -1) == C.ERR_INVALID_ARG
    assert lib.zlfft_mixed_create(ctypes.byref(h), None, 3, -1) == C.ERR_INVALID_ARG
    assert one(kind=5) == C.ERR_INVALID_ARG and "descriptor 1" in C.last_error()
    assert one(precision=9) == C.ERR_INVALID_ARG
    assert one(order=27) == C.ERR_UNSUPPORTED  # above the three-pass maximum (26)
    assert one(kind=C.R2C, order=0) == C.ERR_UNSUPPORTED  # RFFT order 0 has no inner CFFT
    assert one(op=7) == C.ERR_INVALID_ARG
    assert one(op=C.FORWARD_SQR_MAG) == C.ERR_INVALID_ARG  # an RFFT operation
    assert one(in_=None) == C.ERR_INVALID_ARG
    assert one(out=8196) == C.ERR_ALIGNMENT  # complex64 output needs 8-byte alignment
    assert one(precision=C.F64, in_=4104) == C.ERR_ALIGNMENT  # complex128 needs 16
    assert lib.zlfft_mixed_exec(None, 1, None) == C.ERR_INVALID_ARG
    assert lib.zlfft_mixed_destroy(None) == C.OK


def test_mixed_batch_overlaps_rejected_without_cuda():
    """The transforms of a mixed batch run concurrently, so zlfft_mixed_create
    refuses outputs that overlap another transform's output or input (checked
    before it touches CUDA). Shared inputs and in place are accepted."""
    lib = C.lib()
    h = ctypes.c_void_p()
    mib = 1 << 20
    n10 = 8 << 10  # bytes of a CFFT<float> of order 10

    def create(*descs):
        arr = (C.Desc * len(descs))(*[C.Desc(kind=k, precision=C.F32, order=o, op=op, in_=i, out=out)
                                      for k, o, op, i, out in descs])
        rc = lib.zlfft_mixed_create(ctypes.byref(h), arr, len(descs), -1)
        if rc == C.OK:  # a GPU is present: the batch was built
            lib.zlfft_mixed_destroy(h)
        return rc

    a = (C.C2C, 10, C.FORWARD, 1 * mib, 2 * mib)
    # outputs overlap
    assert create(a, (C.C2C, 10, C.FORWARD, 3 * mib, 2 * mib + n10 - 8)) == C.ERR_INVALID_ARG
    assert "outputs overlap" in C.last_error()
    # the second transform reads the first one's output; the first overwrites the second's input in place
    assert create(a, (C.C2C, 10, C.FORWARD, 2 * mib, 4 * mib)) == C.ERR_INVALID_ARG
    assert "writes over the input" in C.last_error()
    assert create((C.C2C, 10, C.FORWARD, 1 * mib, 1 * mib), (C.C2C, 9, C.BACKWARD, 1 * mib + 64, 4 * mib)) \
        == C.ERR_INVALID_ARG
    # an RFFT forward output (N/2 + 1 bins) runs 8 bytes past its input into the next transform's input
    assert create((C.R2C, 10, C.FORWARD, 1 * mib, 1 * mib), (C.C2C, 4, C.FORWARD, 1 * mib + 4096, 4 * mib)) \
        == C.ERR_INVALID_ARG
    # accepted (then CUDA is needed): shared inputs, in place, a forward_sqr_mag output packed right
    # after another transform's
    ok = create(a, (C.C2C, 10, C.BACKWARD, 1 * mib, 3 * mib), (C.C2C, 8, C.FORWARD, 5 * mib, 5 * mib),
                (C.R2C, 10, C.FORWARD_SQR_MAG, 6 * mib, 2 * mib + n10))
    assert ok in (C.ERR_CUDA, C.OK), C.last_error()


def test_python_mirror_rejects_bad_buffers():
    from zldsp_fft_b200.fft import _complex_arg, _real_arg
    import numpy as np
    with pytest.raises(ValueError):
        _complex_arg(np.zeros(4, np.complex128), 8, np.complex64, np.float32, "in", False)
    with pytest.raises(ValueError):
        _complex_arg((np.zeros(8, np.float32),), 8, np.complex64, np.float32, "in", False)
    with pytest.raises(ValueError):
        _real_arg(np.zeros(3, np.float32), 8, np.float32, "in", False)
    ro = np.zeros(8, np.float32)
    ro.flags.writeable = False
    with pytest.raises(ValueError):
        _real_arg(ro, 8, np.float32, "out", True)
    with pytest.raises(TypeError):
        Z.fft._prec(np.int32)


def _build_dropin(tmp_path):
    import shutil
    import subprocess
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    exe = tmp_path / "dropin"
    cmd = ["g++", "-std=c++20", "-O2", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "dropin_example.cpp"),
           "-L", os.path.join(ROOT, "zldsp_fft_b200", "lib"), "-lzlfft_cuda", "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_cpp_dropin_headers_compile_and_link(tmp_path):
    """The reference's README usage compiles unchanged against the drop-in
    headers (include/zldsp_fft_cuda/) and links against libzlfft_cuda.so."""
    _build_dropin(tmp_path)


def test_host_switch_order_is_the_references():
    """zlfft_host_switch_order restates the reference's get_switch_order<F>
    (src/common/zldsp_fft_common_system.hpp:132-157) from the same cache
    queries: on this host it gives the reference's own values."""
    from oracle import oracle as O
    for prec, dt in (("f32", 0), ("f64", 1)):
        a, b = ctypes.c_size_t(), ctypes.c_size_t()
        assert C.lib().zlfft_host_switch_order(dt, ctypes.byref(a), ctypes.byref(b)) == C.OK
        if O.ref_available():
            assert (a.value, b.value) == O.ref_switch_order(prec)
        assert a.value >= 1 and b.value >= a.value + 4
    assert C.lib().zlfft_host_switch_order(7, ctypes.byref(a), ctypes.byref(b)) == C.ERR_INVALID_ARG
    assert C.lib().zlfft_plan_create_hybrid(None, 0, 0, 16, 10, 14, -1) == C.ERR_INVALID_ARG
    h = ctypes.c_void_p()
    assert C.lib().zlfft_plan_create_hybrid(ctypes.byref(h), 0, 0, 16, -3, 14, -1) == C.ERR_INVALID_ARG
