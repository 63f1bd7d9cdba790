"""Tensor-core split-precision form (tcgen05): building blocks and transforms
against the FP64 oracle."""
import ctypes

import numpy as np
import pytest

import zldsp_fft_b200 as Z

pytestmark = pytest.mark.gpu


def test_tc_dft16_selftest_matches_fp64():
    """128 independent DFT-16s on the tensor cores with split FP16 hi/lo
    operands and FP32 accumulation: FP32-level accuracy against FP64."""
    rng = np.random.default_rng(16)
    x = (rng.uniform(-1, 1, (128, 16)) + 1j * rng.uniform(-1, 1, (128, 16))).astype(np.complex64)
    out = np.zeros_like(x)
    st = ctypes.c_int(-1)
    rc = Z._capi.lib().zlfft_selftest_tc_dft16(0, x.ctypes.data, out.ctypes.data, ctypes.byref(st))
    assert rc == 0, Z._capi.last_error()
    assert st.value == 0
    ref = np.fft.fft(x.astype(np.complex128), axis=1)
    err = np.linalg.norm(out - ref, axis=1) / np.linalg.norm(ref, axis=1)
    # one radix-16 stage: 4 * log2(16) * 2^-24 is the per-transform FP32 bar
    assert err.max() <= 4 * 4 * 2.0 ** -24, err.max()
