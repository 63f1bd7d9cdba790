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


def _c2c(plan, x, forward=True):
    from tests import gpu_util as G
    return G.run_c2c(plan, x, forward)


@pytest.mark.parametrize("order", [14, 15, 16, 17, 18, 20])
def test_tc_fp16_cfft_within_fp32_tolerance(oracle, order):
    """CFFT<float> in the split-precision tensor-core form, forward and
    backward, against the FP64 oracle with the FP32 bar 4 log2(N) 2^-24; the
    form really runs (its results differ in rounding from the plain form's)."""
    rng = np.random.default_rng(600 + order)
    batch = 6 if order <= 16 else 2
    n = 1 << order
    x = (rng.uniform(-1, 1, (batch, n)) + 1j * rng.uniform(-1, 1, (batch, n))).astype(np.complex64)
    tc = Z.Plan(Z.C2C, order, np.float32, mode=Z.MODE_TC_FP16)
    plain = Z.Plan(Z.C2C, order, np.float32)
    tol = oracle.tolerance(order, "f32")
    y = _c2c(tc, x, True)
    err = oracle.rel_l2(y, oracle.cfft_fp64(x))
    assert err.max() <= tol, (err.max(), tol)
    yp = _c2c(plain, x, True)
    assert not np.array_equal(y, yp)
    z = _c2c(tc, y, False)
    err_b = oracle.rel_l2(z, oracle.cfft_fp64(y, False))
    assert err_b.max() <= tol, (err_b.max(), tol)
    assert tc.device_status() == 0


def test_tc_fp16_extreme_magnitudes_and_chunks(oracle):
    """Exact power-of-two scaling keeps the FP16 operands in range for inputs
    of any FP32 magnitude; batches larger than one scratch chunk (two chunk
    pipelines) and all-zero transforms come out right."""
    rng = np.random.default_rng(7)
    order, n = 14, 1 << 14
    tc = Z.Plan(Z.C2C, order, np.float32, mode=Z.MODE_TC_FP16)
    tol = oracle.tolerance(order, "f32")
    base = (rng.uniform(-1, 1, (4, n)) + 1j * rng.uniform(-1, 1, (4, n)))
    for scale in (1e-30, 1e-8, 1e12, 1e30):
        x = (base * scale).astype(np.complex64)
        y = _c2c(tc, x, True)
        assert np.isfinite(y).all(), scale
        assert oracle.rel_l2(y, oracle.cfft_fp64(x)).max() <= tol, scale
    # 400 transforms > one 48 MiB chunk (384 of order 14): both chunk pipelines
    x = (rng.uniform(-1, 1, (400, n)) + 1j * rng.uniform(-1, 1, (400, n))).astype(np.complex64)
    x[17] = 0
    y = _c2c(tc, x, True)
    assert np.all(y[17] == 0)
    keep = [i for i in range(400) if i != 17]
    assert oracle.rel_l2(y[keep], oracle.cfft_fp64(x[keep])).max() <= tol


def test_tc_mode_rejected_where_not_built():
    h = ctypes.c_void_p()
    lib = Z._capi.lib()
    assert lib.zlfft_plan_create(ctypes.byref(h), Z.R2C, Z.F32, 12, Z.MODE_TC_FP16, -1) == Z._capi.ERR_UNSUPPORTED
    assert lib.zlfft_plan_create(ctypes.byref(h), Z.C2C, Z.F64, 16, Z.MODE_TC_FP16, -1) == Z._capi.ERR_UNSUPPORTED
    assert lib.zlfft_plan_create(ctypes.byref(h), Z.C2C, Z.F32, 16, 2, -1) == Z._capi.ERR_UNSUPPORTED  # no such mode


@pytest.mark.parametrize("prec,ft,ct", [("f32", np.float32, np.complex64), ("f64", np.float64, np.complex128)])
@pytest.mark.parametrize("order", [14, 15, 16, 17, 20])
def test_fast_twiddle_form_within_tolerance(oracle, prec, ft, ct, order):
    """ZLFFT_MODE_FAST (multi-pass radix-16 groups with twiddles built from two
    table values): CFFT both directions, RFFT forward / sqr_mag / backward,
    within the FP bar of the FP64 oracle; the form really runs (its bits
    differ from the plain form's)."""
    from tests import gpu_util as G
    rng = np.random.default_rng(700 + order)
    n = 1 << order
    batch = 3 if order <= 17 else 1
    tol = oracle.tolerance(order, prec)
    x = (rng.uniform(-1, 1, (batch, n)) + 1j * rng.uniform(-1, 1, (batch, n))).astype(ct)
    fast = Z.Plan(Z.C2C, order, ft, mode=Z.MODE_FAST)
    y = G.run_c2c(fast, x, True)
    assert oracle.rel_l2(y, oracle.cfft_fp64(x)).max() <= tol
    assert not np.array_equal(y, G.run_c2c(Z.Plan(Z.C2C, order, ft), x, True))
    z = G.run_c2c(fast, y, False)
    assert oracle.rel_l2(z, oracle.cfft_fp64(y, False)).max() <= tol
    xr = rng.uniform(-1, 1, (batch, n)).astype(ft)
    rf = Z.Plan(Z.R2C, order, ft, mode=Z.MODE_FAST)
    X = G.run_r2c(rf, xr)
    assert oracle.rel_l2(X, oracle.rfft_fp64(xr)).max() <= tol
    Pw = G.run_r2c(rf, xr, sqr_mag=True)
    assert oracle.rel_l2(Pw, np.abs(oracle.rfft_fp64(xr)) ** 2).max() <= 2 * tol
    back = G.run_c2r(rf, X.astype(ct))
    assert oracle.rel_l2(back, oracle.rfft_backward_fp64(X.astype(ct))).max() <= tol
    assert fast.device_status() == 0 and rf.device_status() == 0


@pytest.mark.parametrize("order", [11, 12, 13])
def test_fast_twiddle_form_tile_orders(oracle, order):
    """The fast-twiddle form of the single-tile kernels' middle radix-16 groups
    (CFFT orders 11-13, RFFT orders 12-14): within the FP32 bar, and not the
    plain form's bits."""
    from tests import gpu_util as G
    rng = np.random.default_rng(800 + order)
    n = 1 << order
    x = (rng.uniform(-1, 1, (20, n)) + 1j * rng.uniform(-1, 1, (20, n))).astype(np.complex64)
    tol = oracle.tolerance(order, "f32")
    fast = Z.Plan(Z.C2C, order, np.float32, mode=Z.MODE_FAST)
    y = G.run_c2c(fast, x, True)
    assert oracle.rel_l2(y, oracle.cfft_fp64(x)).max() <= tol
    assert not np.array_equal(y, G.run_c2c(Z.Plan(Z.C2C, order, np.float32), x, True))
    assert oracle.rel_l2(G.run_c2c(fast, y, False), oracle.cfft_fp64(y, False)).max() <= tol
    xr = rng.uniform(-1, 1, (20, 2 * n)).astype(np.float32)
    rf = Z.Plan(Z.R2C, order + 1, np.float32, mode=Z.MODE_FAST)
    rtol = oracle.tolerance(order + 1, "f32")
    for ol in (Z.AOS, Z.SOA):
        X = G.run_r2c(rf, xr, ol)
        assert oracle.rel_l2(X, oracle.rfft_fp64(xr)).max() <= rtol
    Pw = G.run_r2c(rf, xr, sqr_mag=True)
    assert oracle.rel_l2(Pw, np.abs(oracle.rfft_fp64(xr)) ** 2).max() <= 2 * rtol


def test_pipelined_tc_kernel_equals_serial_kernel():
    """The warp-specialised pipelined tensor-core pass (ZLFFT_TC_PIPE=1, its own
    process since the switch is read once) computes the serial kernel's
    arithmetic in the same order: bit-identical outputs, orders 14, 16 and 20,
    forward and backward, several chunks."""
    import os
    import subprocess
    import sys
    code = r'''
import sys, numpy as np, torch
sys.path.insert(0, sys.argv[1])
import zldsp_fft_b200 as Z
rng = np.random.default_rng(31)
out = {}
for order, b in ((14, 700), (16, 150), (20, 7)):
    n = 1 << order
    x = (rng.uniform(-1, 1, (b, n)) + 1j * rng.uniform(-1, 1, (b, n))).astype(np.complex64)
    p = Z.Plan(Z.C2C, order, np.float32, Z.MODE_TC_FP16)
    ti = torch.from_numpy(x.view(np.float32).reshape(b, n, 2).copy()).cuda()
    f = torch.empty_like(ti); g = torch.empty_like(ti)
    p.exec_device(Z.FORWARD, Z.AOS, Z.AOS, ti.data_ptr(), None, f.data_ptr(), None, b)
    p.exec_device(Z.BACKWARD, Z.AOS, Z.AOS, f.data_ptr(), None, g.data_ptr(), None, b)
    torch.cuda.synchronize()
    assert p.device_status() == 0
    out[f"f{order}"] = f.cpu().numpy(); out[f"g{order}"] = g.cpu().numpy()
np.savez(sys.argv[2], **out)
'''
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    res = {}
    for flag in ("0", "1"):
        path = os.path.join(os.environ.get("TMPDIR", "/tmp"), f"zlfft_tcpipe_{flag}_{os.getpid()}.npz")
        env = dict(os.environ, ZLFFT_TC_PIPE=flag)
        r = subprocess.run([sys.executable, "-c", code, root, path], env=env, capture_output=True, text=True,
                           timeout=600)
        assert r.returncode == 0, r.stdout + r.stderr
        res[flag] = dict(np.load(path))
        os.remove(path)
    for k in res["0"]:
        assert np.array_equal(res["0"][k], res["1"][k]), k
