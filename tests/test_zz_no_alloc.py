"""The allocation-free entry point, zlfft_exec_device_noalloc.

It exists for callers that cannot allocate device memory when they run a
transform: a real-time audio thread (an allocation may block for an unbounded
time, and a missed audio deadline is an audible glitch), or a host whose
device memory all belongs to its own pool. For orders 14 and up it passes the
intermediates between kernel passes through a scratch array built into the
library instead of allocating one.

This file is named so that pytest collects it last; it must pass on its own
in a fresh process as well as after the other GPU tests.
"""
import numpy as np
import pytest

import zldsp_fft_b200 as Z
from tests import gpu_util as G

pytestmark = pytest.mark.gpu


def _run_noalloc(plan, op, il, ol, i0, i1, o0, o1, batch, stream=None):
    lib = Z._capi.lib()
    return lib.zlfft_exec_device_noalloc(plan.handle, op, il, ol, i0, i1, o0, o1, int(batch), 0, 0, stream)


def test_noalloc_matches_exec_device_on_two_calls(oracle):
    """Same results as zlfft_exec_device (within the parity tolerance, and in
    fact bit-identical) for multi-pass orders that need scratch, two calls in
    a row so the second one runs on the scratch the first one left behind."""
    import torch
    rng = np.random.default_rng(2024)
    # order 16: more transforms than one scratch chunk (64); order 19: its two-pass form (512 | 1024 points)
    for order, batch in ((16, 70), (19, 5), (20, 3)):
        n = 1 << order
        plan = Z.Plan(Z.C2C, order, np.float32)
        tol = oracle.tolerance(order, "f32")
        for call in range(2):
            x = (rng.uniform(-1, 1, (batch, n)) + 1j * rng.uniform(-1, 1, (batch, n))).astype(np.complex64)
            ref = G.run_c2c(plan, x, True)  # the existing entry point
            ti = G.dev(x)
            to = torch.zeros((batch, n, 2), dtype=torch.float32, device="cuda")
            assert _run_noalloc(plan, Z.FORWARD, Z.AOS, Z.AOS, ti.data_ptr(), None, to.data_ptr(), None,
                                batch) == 0, Z._capi.last_error()
            torch.cuda.synchronize()
            y = to.cpu().numpy()
            y = (y[..., 0] + 1j * y[..., 1]).astype(np.complex64)
            assert oracle.rel_l2(y, ref).max() <= tol, (order, call)
            assert np.array_equal(y, ref), (order, call)
            assert oracle.rel_l2(y[:1], oracle.cfft_fp64(x[:1])).max() <= tol
        assert plan.device_status() == 0

    # RFFT order 16 (inner CFFT order 15, multi-pass): forward to split-SoA bins, twice
    plan = Z.Plan(Z.R2C, 16, np.float32)
    n, nb = 1 << 16, (1 << 15) + 1
    for call in range(2):
        x = rng.uniform(-1, 1, (4, n)).astype(np.float32)
        ref = G.run_r2c(plan, x, Z.SOA)
        ti = G.dev(x)
        re = torch.zeros((4, nb), dtype=torch.float32, device="cuda")
        im = torch.zeros((4, nb), dtype=torch.float32, device="cuda")
        assert _run_noalloc(plan, Z.FORWARD, Z.AOS, Z.SOA, ti.data_ptr(), None, re.data_ptr(), im.data_ptr(),
                            4) == 0, Z._capi.last_error()
        torch.cuda.synchronize()
        y = (re.cpu().numpy() + 1j * im.cpu().numpy()).astype(np.complex64)
        assert oracle.rel_l2(y, ref).max() <= oracle.tolerance(16, "f32"), call
        assert np.array_equal(y, ref), call


def test_noalloc_rejects_transforms_beyond_the_built_in_scratch():
    """A transform larger than one half of the built-in array (32 MiB) is
    refused with a clear message instead of running past it."""
    import torch
    plan = Z.Plan(Z.C2C, 23, np.float32)  # 2^23 complex64 = 64 MiB per transform
    x = torch.zeros((1 << 23, 2), dtype=torch.float32, device="cuda")
    y = torch.zeros_like(x)
    rc = _run_noalloc(plan, Z.FORWARD, Z.AOS, Z.AOS, x.data_ptr(), None, y.data_ptr(), None, 1)
    assert rc == Z._capi.ERR_UNSUPPORTED
    assert "allocation-free" in Z._capi.last_error()


def _cx_dev(x, layout):
    return G.complex_to_dev(x, layout)


def test_noalloc_backward_paths_and_tile_orders(oracle):
    """The paths of the allocation-free entry point beyond forward C2C, each
    against zlfft_exec_device on two calls in a row:
    - the RFFT backward (its pre-step writes the first half of the array and the
      passes run on the halves swapped), AoS and SoA bins;
    - FP64 C2C backward from split-SoA input with more transforms than one
      chunk of the array (64 of order 15), within the FP64 bar and bit-equal;
    - FP32 C2C order 14, which runs on one tile per transform and needs no
      scratch at all."""
    import torch
    rng = np.random.default_rng(2025)
    # RFFT order 16 backward (inner CFFT order 15: two passes)
    plan = Z.Plan(Z.R2C, 16, np.float32)
    n, nb = 1 << 16, (1 << 15) + 1
    for layout in (Z.AOS, Z.SOA):
        for call in range(2):
            X = (rng.uniform(-1, 1, (3, nb)) + 1j * rng.uniform(-1, 1, (3, nb))).astype(np.complex64)
            ref = G.run_c2r(plan, X, layout)
            i0, i1, keep = _cx_dev(X, layout)
            to = torch.zeros((3, n), dtype=torch.float32, device="cuda")
            assert _run_noalloc(plan, Z.BACKWARD, layout, Z.AOS, i0, i1, to.data_ptr(), None, 3) == 0, \
                Z._capi.last_error()
            torch.cuda.synchronize()
            y = to.cpu().numpy()
            assert np.array_equal(y, ref), (layout, call)
            assert oracle.rel_l2(y, oracle.rfft_backward_fp64(X)).max() <= oracle.tolerance(16, "f32")
    # FP64 C2C order 15 backward, SoA in, AoS out, 70 transforms (> 64 per chunk)
    plan = Z.Plan(Z.C2C, 15, np.float64)
    n, b = 1 << 15, 70
    for call in range(2):
        x = (rng.uniform(-1, 1, (b, n)) + 1j * rng.uniform(-1, 1, (b, n))).astype(np.complex128)
        ref = G.run_c2c(plan, x, False, Z.SOA, Z.AOS)
        i0, i1, keep = _cx_dev(x, Z.SOA)
        to = torch.zeros((b, n, 2), dtype=torch.float64, device="cuda")
        assert _run_noalloc(plan, Z.BACKWARD, Z.SOA, Z.AOS, i0, i1, to.data_ptr(), None, b) == 0, \
            Z._capi.last_error()
        torch.cuda.synchronize()
        y = to.cpu().numpy()
        y = y[..., 0] + 1j * y[..., 1]
        assert oracle.rel_l2(y, ref).max() <= oracle.tolerance(15, "f64"), call
        assert np.array_equal(y, ref), call
        assert oracle.rel_l2(y[:2], oracle.cfft_fp64(x[:2], False)).max() <= oracle.tolerance(15, "f64")
    # FP32 C2C order 14: the single-tile kernel, the same as zlfft_exec_device
    plan = Z.Plan(Z.C2C, 14, np.float32)
    n, b = 1 << 14, 40
    for call in range(2):
        x = (rng.uniform(-1, 1, (b, n)) + 1j * rng.uniform(-1, 1, (b, n))).astype(np.complex64)
        ref = G.run_c2c(plan, x, True)
        ti = G.dev(x)
        to = torch.zeros((b, n, 2), dtype=torch.float32, device="cuda")
        plan.take_launch_count()
        assert _run_noalloc(plan, Z.FORWARD, Z.AOS, Z.AOS, ti.data_ptr(), None, to.data_ptr(), None, b) == 0
        torch.cuda.synchronize()
        assert plan.take_launch_count() == 1  # one tile kernel launch, no passes
        y = to.cpu().numpy()
        assert np.array_equal((y[..., 0] + 1j * y[..., 1]).astype(np.complex64), ref), call
