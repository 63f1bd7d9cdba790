"""GPU parity: the CUDA kernels, called through the C ABI on device buffers,
against the oracle on the same seeded inputs.

Tolerance: relative L2 <= 4*log2(N)*eps against the FP64 oracle
(eps = 2^-24 f32, 2^-53 f64). The plain form rebuilds the reference's own
arithmetic, so in f32 (where the device-generated twiddle table is bit-equal
to the reference's) the output must also be BIT-IDENTICAL to the oracle's C
restatement, which is itself bit-identical to the reference's code.
"""
import numpy as np
import pytest

import zldsp_fft_b200 as Z
from tests import gpu_util as G

pytestmark = pytest.mark.gpu

PRECS = [("f32", np.float32, np.complex64), ("f64", np.float64, np.complex128)]
TILE_ORDERS = list(range(0, 14))


def _cx(rng, b, n, ct):
    return (rng.uniform(-1, 1, (b, n)) + 1j * rng.uniform(-1, 1, (b, n))).astype(ct)


@pytest.mark.parametrize("prec,ft,ct", PRECS)
def test_device_twiddles_equal_reference_table(oracle, prec, ft, ct):
    for order in (2, 4, 7, 10, 13):
        plan = Z.Plan(Z.C2C, order, ft)
        T = plan.twiddles()
        ref = oracle.twiddles(order, prec)
        if prec == "f32":
            assert np.array_equal(T, ref), order
        else:  # the device's double cos/sin vs the host libm's: within a few ulp
            assert np.abs(T - ref).max() <= 4 * 2.0 ** -53, order


@pytest.mark.parametrize("prec,ft,ct", PRECS)
@pytest.mark.parametrize("order", TILE_ORDERS)
def test_cfft_all_layouts(oracle, prec, ft, ct, order):
    n = 1 << order
    rng = np.random.default_rng(1000 + order)
    b = 3 if order < 12 else 2
    x = _cx(rng, b, n, ct)
    plan = Z.Plan(Z.C2C, order, ft)
    tol = oracle.tolerance(order, prec)
    for forward in (True, False):
        port = oracle.cfft_port(x, forward)
        fp64 = oracle.cfft_fp64(x, forward)
        for il in (Z.AOS, Z.SOA):
            for ol in (Z.AOS, Z.SOA):
                y = G.run_c2c(plan, x, forward, il, ol)
                err = oracle.rel_l2(y, fp64).max()
                assert err <= tol, (order, forward, il, ol, err)
                if prec == "f32":
                    assert np.array_equal(y, port), (order, forward, il, ol)
                else:
                    assert oracle.rel_l2(y, port).max() <= tol


@pytest.mark.parametrize("prec,ft,ct", PRECS)
@pytest.mark.parametrize("order", list(range(1, 15)))
def test_rfft_forward_sqr_backward(oracle, prec, ft, ct, order):
    n = 1 << order
    rng = np.random.default_rng(2000 + order)
    b = 3
    x = rng.uniform(-1, 1, (b, n)).astype(ft)
    plan = Z.Plan(Z.R2C, order, ft)
    tol = oracle.tolerance(order, prec)
    port = oracle.rfft_forward_port(x)
    for ol in (Z.AOS, Z.SOA):
        X = G.run_r2c(plan, x, ol)
        assert oracle.rel_l2(X, oracle.rfft_fp64(x)).max() <= tol
        if prec == "f32":
            assert np.array_equal(X, port), (order, ol)
    P = G.run_r2c(plan, x, sqr_mag=True)
    assert oracle.rel_l2(P, np.abs(oracle.rfft_fp64(x)) ** 2).max() <= 2 * tol
    if prec == "f32":
        assert np.array_equal(P, oracle.rfft_forward_port(x, sqr_mag=True)), order
    Xin = _cx(rng, b, n // 2 + 1, ct)
    for il in (Z.AOS, Z.SOA):
        back = G.run_c2r(plan, Xin, il)
        assert oracle.rel_l2(back, oracle.rfft_backward_fp64(Xin)).max() <= tol
        if prec == "f32":
            assert np.array_equal(back, oracle.rfft_backward_port(Xin)), (order, il)


@pytest.mark.parametrize("prec,ft,ct", PRECS)
def test_golden_reference_outputs(prec, ft, ct):
    """The reference's own outputs (fixtures) reproduced on the GPU."""
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", f"reference_{prec}.npz"))
    for order in range(0, 11):
        plan = Z.Plan(Z.C2C, order, ft)
        x = g[f"c2c_{order}_in"]
        y = G.run_c2c(plan, x, True)
        yb = G.run_c2c(plan, x, False)
        if prec == "f32":
            assert np.array_equal(y, g[f"c2c_{order}_fwd"]) and np.array_equal(yb, g[f"c2c_{order}_bwd"]), order
    for order in range(1, 12):
        plan = Z.Plan(Z.R2C, order, ft)
        x = g[f"r2c_{order}_in"]
        X = G.run_r2c(plan, x)
        if prec == "f32":
            assert np.array_equal(X, g[f"r2c_{order}_fwd"]), order
            assert np.array_equal(G.run_r2c(plan, x, sqr_mag=True), g[f"r2c_{order}_sqr"]), order
            assert np.array_equal(G.run_c2r(plan, g[f"r2c_{order}_bins"]), g[f"r2c_{order}_bwd"]), order


def test_config1_order10_single_transform(oracle):
    """CFFT<float> order 10, one transform, AoS: forward then backward, through
    the reference-shaped host API (zldsp::fft::CFFT::forward/backward)."""
    rng = np.random.default_rng(1001)
    n = 1024
    x = (rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)).astype(np.complex64)
    cf = Z.CFFT(10)
    assert cf.get_size() == 1024 and cf.get_order() == 10
    y = np.zeros_like(x)
    cf.forward(x, y)
    back = np.zeros_like(x)
    cf.backward(y, back)
    assert np.array_equal(y, oracle.cfft_port(x, True))
    assert np.array_equal(back, oracle.cfft_port(y, False))
    assert oracle.rel_l2(y, oracle.cfft_fp64(x)).max() <= oracle.tolerance(10)
    assert oracle.rel_l2(back, 1024 * x.astype(np.complex128)).max() <= 2 * oracle.tolerance(10)
    # SoA overloads of the reference: (re, im) pairs
    re, im = np.zeros(n, np.float32), np.zeros(n, np.float32)
    cf.forward(x, (re, im))
    assert np.array_equal(re + 1j * im, y)
    out = np.zeros_like(x)
    cf.forward((np.ascontiguousarray(x.real), np.ascontiguousarray(x.imag)), out)
    assert np.array_equal(out, y)


def test_rfft_host_api_overloads(oracle):
    rng = np.random.default_rng(1002)
    for order in (1, 2, 5, 12):
        n = 1 << order
        x = rng.uniform(-1, 1, n).astype(np.float32)
        rf = Z.RFFT(order)
        assert rf.get_size() == n and rf.get_order() == order
        X = np.zeros(n // 2 + 1, np.complex64)
        rf.forward(x, X)
        assert np.array_equal(X, oracle.rfft_forward_port(x))
        re, im = np.zeros(n // 2 + 1, np.float32), np.zeros(n // 2 + 1, np.float32)
        rf.forward(x, (re, im))
        assert np.array_equal(re + 1j * im, X)
        P = np.zeros(n // 2 + 1, np.float32)
        rf.forward_sqr_mag(x, P)
        assert np.array_equal(P, oracle.rfft_forward_port(x, sqr_mag=True))
        back = np.zeros(n, np.float32)
        rf.backward(X, back)
        assert np.array_equal(back, oracle.rfft_backward_port(X))
        back2 = np.zeros(n, np.float32)
        rf.backward((re, im), back2)
        assert np.array_equal(back2, back)


def test_config2_rfft_order12_batch8192(oracle):
    """RFFT<float> order 12 x 8192 Hann-windowed frames (3 sinusoids + noise):
    full batch on the GPU, a sample of frames checked bit-exactly, every frame
    checked by size-independent properties."""
    import torch
    n, b = 4096, 8192
    rng = np.random.default_rng(1002)
    t = np.arange(n)
    f = rng.uniform(0, 0.5, (b, 3, 1))
    amp = rng.uniform(0.1, 1, (b, 3, 1))
    ph = rng.uniform(0, 2 * np.pi, (b, 3, 1))
    sig = (amp * np.sin(2 * np.pi * f * t + ph)).sum(1) + rng.normal(0, 0.1, (b, n))
    x = (sig * (0.5 - 0.5 * np.cos(2 * np.pi * t / n))).astype(np.float32)
    plan = Z.Plan(Z.R2C, 12, np.float32)
    X = G.run_r2c(plan, x)
    P = G.run_r2c(plan, x, sqr_mag=True)
    sample = rng.choice(b, 16, replace=False)
    assert np.array_equal(X[sample], oracle.rfft_forward_port(x[sample]))
    assert np.array_equal(P[sample], oracle.rfft_forward_port(x[sample], sqr_mag=True))
    # every frame: DC/Nyquist real, |X|^2 consistent with sqr_mag, round trip N/2
    assert np.all(X[:, 0].imag == 0) and np.all(X[:, -1].imag == 0)
    mag = X.real.astype(np.float64) ** 2 + X.imag.astype(np.float64) ** 2
    assert oracle.rel_l2(P, mag).max() <= 2 * oracle.tolerance(12)
    back = G.run_c2r(plan, X)
    assert oracle.rel_l2(back, (n / 2) * x.astype(np.float64)).max() <= 2 * oracle.tolerance(12)
    del torch


def test_batch_strides_inplace_and_edges(oracle):
    import torch
    rng = np.random.default_rng(7)
    order, n = 9, 512
    plan = Z.Plan(Z.C2C, order, np.float32)
    # ragged strides: transforms at stride n + 37 in, n + 5 out
    b, si, so = 5, n + 37, n + 5
    buf = (rng.uniform(-1, 1, (b * si)) + 1j * rng.uniform(-1, 1, (b * si))).astype(np.complex64)
    ti = G.dev(buf)
    to = torch.zeros((b * so, 2), dtype=torch.float32, device="cuda")
    plan.exec_device(Z.FORWARD, Z.AOS, Z.AOS, ti.data_ptr(), None, to.data_ptr(), None, b, si, so)
    torch.cuda.synchronize()
    out = G.host(to)
    out = out[:, 0] + 1j * out[:, 1]
    for i in range(b):
        assert np.array_equal(out[i * so: i * so + n].astype(np.complex64),
                              oracle.cfft_port(buf[i * si: i * si + n][None, :], True)[0])
    # in place
    x = (rng.uniform(-1, 1, (4, n)) + 1j * rng.uniform(-1, 1, (4, n))).astype(np.complex64)
    t = G.dev(x)
    plan.exec_device(Z.FORWARD, Z.AOS, Z.AOS, t.data_ptr(), None, t.data_ptr(), None, 4)
    torch.cuda.synchronize()
    assert np.array_equal(G.host(t), oracle.cfft_port(x, True))
    # batch 0 is a no-op; misaligned and null pointers are rejected
    plan.exec_device(Z.FORWARD, Z.AOS, Z.AOS, t.data_ptr(), None, t.data_ptr(), None, 0)
    with pytest.raises(Z.ZlfftError) as e:
        plan.exec_device(Z.FORWARD, Z.AOS, Z.AOS, t.data_ptr() + 4, None, to.data_ptr(), None, 1)
    assert e.value.code == Z._capi.ERR_ALIGNMENT
    with pytest.raises(Z.ZlfftError) as e:
        plan.exec_device(Z.FORWARD, Z.SOA, Z.AOS, t.data_ptr(), None, to.data_ptr(), None, 1)
    assert e.value.code == Z._capi.ERR_INVALID_ARG
    with pytest.raises(Z.ZlfftError):
        plan.exec_device(Z.FORWARD_SQR_MAG, Z.AOS, Z.AOS, t.data_ptr(), None, to.data_ptr(), None, 1)
    # large batch (grid-stride loop over more tiles than resident CTAs)
    big = (rng.uniform(-1, 1, (40000, 64)) + 1j * rng.uniform(-1, 1, (40000, 64))).astype(np.complex64)
    p6 = Z.Plan(Z.C2C, 6, np.float32)
    y = G.run_c2c(p6, big, True)
    idx = [0, 1, 12345, 39999]
    assert np.array_equal(y[idx], oracle.cfft_port(big[idx], True))


def test_launch_counter():
    import torch
    plan = Z.Plan(Z.C2C, 10, np.float32)
    plan.take_launch_count()
    x = torch.zeros((8, 1024, 2), device="cuda")
    for _ in range(3):
        plan.exec_device(Z.FORWARD, Z.AOS, Z.AOS, x.data_ptr(), None, x.data_ptr(), None, 8)
    torch.cuda.synchronize()
    assert plan.take_launch_count() == 3


def test_bounded_wait_reports_instead_of_hanging():
    """A device wait that can never complete gives up after its poll limit,
    sets the error word and returns; the context stays usable afterwards."""
    import ctypes
    lib = Z._capi.lib()
    st = ctypes.c_int(-1)
    Z._capi.check(lib.zlfft_selftest_bounded_wait(0, ctypes.byref(st)))
    assert st.value == 1
    plan = Z.Plan(Z.C2C, 8, np.float32)
    assert plan.device_status() == 0
    x = np.ones((2, 256), np.complex64)
    y = G.run_c2c(plan, x, True)
    assert y[0, 0] == 256


@pytest.mark.parametrize("prec,ft,ct", PRECS)
@pytest.mark.parametrize("order", [14, 15, 16, 17, 18, 19, 20, 23])
def test_multipass_cfft(oracle, prec, ft, ct, order):
    """Orders above one CTA: 2-3 Stockham passes through L2-resident scratch;
    the arithmetic is still the reference's, so f32 stays bit-exact. Orders 17,
    18 and 23 start with a 512- or 1024-point pass (64- / 32-byte unit rows)."""
    n = 1 << order
    rng = np.random.default_rng(3000 + order)
    b = 2
    x = _cx(rng, b, n, ct)
    plan = Z.Plan(Z.C2C, order, ft)
    tol = oracle.tolerance(order, prec)
    layouts = [(Z.AOS, Z.AOS), (Z.SOA, Z.SOA)] if order > 16 else [(i, o) for i in (Z.AOS, Z.SOA) for o in (Z.AOS, Z.SOA)]
    for forward in (True, False):
        port = oracle.cfft_port(x, forward)
        fp64 = oracle.cfft_fp64(x, forward)
        for il, ol in layouts:
            y = G.run_c2c(plan, x, forward, il, ol)
            assert oracle.rel_l2(y, fp64).max() <= tol, (order, forward, il, ol)
            if prec == "f32":
                assert np.array_equal(y, port), (order, forward, il, ol)


@pytest.mark.parametrize("prec,ft,ct", PRECS)
@pytest.mark.parametrize("order", [15, 16, 17, 18, 19])
def test_multipass_rfft(oracle, prec, ft, ct, order):
    n = 1 << order
    rng = np.random.default_rng(4000 + order)
    x = rng.uniform(-1, 1, (2, n)).astype(ft)
    plan = Z.Plan(Z.R2C, order, ft)
    tol = oracle.tolerance(order, prec)
    for ol in (Z.AOS, Z.SOA):
        X = G.run_r2c(plan, x, ol)
        assert oracle.rel_l2(X, oracle.rfft_fp64(x)).max() <= tol
        if prec == "f32":
            assert np.array_equal(X, oracle.rfft_forward_port(x)), (order, ol)
    P = G.run_r2c(plan, x, sqr_mag=True)
    if prec == "f32":
        assert np.array_equal(P, oracle.rfft_forward_port(x, sqr_mag=True))
    Xin = _cx(rng, 2, n // 2 + 1, ct)
    for il in (Z.AOS, Z.SOA):
        back = G.run_c2r(plan, Xin, il)
        assert oracle.rel_l2(back, oracle.rfft_backward_fp64(Xin)).max() <= tol
        if prec == "f32":
            assert np.array_equal(back, oracle.rfft_backward_port(Xin)), (order, il)


def test_multipass_chunks_strides_inplace(oracle):
    """More transforms than one scratch chunk, ragged strides, and in place."""
    import torch
    order, n = 16, 1 << 16
    plan = Z.Plan(Z.C2C, order, np.float32)
    rng = np.random.default_rng(11)
    b = 100  # chunks hold 48 transforms of 2^16 complex f32
    x = (rng.uniform(-1, 1, (b, n)) + 1j * rng.uniform(-1, 1, (b, n))).astype(np.complex64)
    y = G.run_c2c(plan, x, True)
    assert np.array_equal(y, oracle.cfft_port(x, True))  # every transform, across chunk boundaries
    idx = [0, 47, 48, 99]
    t = G.dev(x)
    plan.exec_device(Z.FORWARD, Z.AOS, Z.AOS, t.data_ptr(), None, t.data_ptr(), None, b)
    torch.cuda.synchronize()
    assert np.array_equal(G.host(t)[idx], y[idx])
    si, so = n + 24, n + 8
    buf = np.zeros(3 * si, np.complex64)
    for i in range(3):
        buf[i * si: i * si + n] = x[i]
    ti = G.dev(buf)
    to = torch.zeros((3 * so, 2), dtype=torch.float32, device="cuda")
    plan.exec_device(Z.BACKWARD, Z.AOS, Z.AOS, ti.data_ptr(), None, to.data_ptr(), None, 3, si, so)
    torch.cuda.synchronize()
    o = G.host(to)
    o = (o[:, 0] + 1j * o[:, 1]).astype(np.complex64)
    ref = oracle.cfft_port(x[:3], False)
    for i in range(3):
        assert np.array_equal(o[i * so: i * so + n], ref[i])


def test_cpp_dropin_runs(tmp_path):
    """The C++ drop-in classes (zldsp::fft::CFFT/RFFT over the C ABI) run the
    reference's README example on the GPU and round-trip within tolerance."""
    import os
    import subprocess
    from tests.test_capi_cpu import _build_dropin
    exe = _build_dropin(tmp_path)
    env = dict(os.environ)
    libdir = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "zldsp_fft_b200", "lib")
    env["LD_LIBRARY_PATH"] = libdir + ":" + env.get("LD_LIBRARY_PATH", "")
    r = subprocess.run([str(exe)], capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "rfft0_throws=1" in r.stdout
    n = 1024
    i = np.arange(n, dtype=np.float32)
    x = (np.sin(np.float32(0.1) * i) + 1j * np.cos(np.float32(0.3) * i)).astype(np.complex64)
    X = np.fft.fft(x.astype(np.complex128))
    got = r.stdout.split("X0=")[1].split()[0].split(",")
    assert abs(float(got[0]) - X[0].real) < 1e-3 and abs(float(got[1]) - X[0].imag) < 1e-3


@pytest.mark.parametrize("case", ["tile_r2c_order12", "multipass_c2c_order16"])
def test_repeated_runs_identical(oracle, case):
    """Large batches run three times give identical outputs everywhere, and a
    sample matches the oracle. Guards the TMA prefetch pipelines (a refill
    racing a read would corrupt different transforms on each run)."""
    import torch
    rng = np.random.default_rng(77)
    if case == "tile_r2c_order12":
        plan = Z.Plan(Z.R2C, 12, np.float32)
        x = rng.uniform(-1, 1, (4096, 4096)).astype(np.float32)
        runs = [G.run_r2c(plan, x) for _ in range(3)]
        ref_sample = oracle.rfft_forward_port(x[::97])
        got_sample = runs[0][::97]
    else:
        plan = Z.Plan(Z.C2C, 16, np.float32)
        x = (rng.uniform(-1, 1, (200, 1 << 16)) + 1j * rng.uniform(-1, 1, (200, 1 << 16))).astype(np.complex64)
        runs = [G.run_c2c(plan, x, True) for _ in range(3)]
        ref_sample = oracle.cfft_port(x[::13], True)
        got_sample = runs[0][::13]
    assert np.array_equal(runs[0], runs[1]) and np.array_equal(runs[0], runs[2])
    assert np.array_equal(got_sample, ref_sample)
    assert plan.device_status() == 0
    del torch


@pytest.mark.parametrize("case", ["c2c_f32_order16", "r2c_f32_order17", "c2r_f32_order17", "c2c_f64_order15"])
def test_host_batched_multichunk_equals_device(case):
    """zlfft_exec_host_batched over several staging chunks of a
    multi-pass order (the chunks alternate between two streams and share the
    plan's scratch), from pageable and from pinned host buffers, run three
    times: bit-identical to the device-pointer path on the same input."""
    import torch
    rng = np.random.default_rng(2024)
    if case == "c2c_f32_order16":
        plan, b, n = Z.Plan(Z.C2C, 16, np.float32), 160, 1 << 16
        x = (rng.uniform(-1, 1, (b, n)) + 1j * rng.uniform(-1, 1, (b, n))).astype(np.complex64)
        op, ref, out = Z.FORWARD, G.run_c2c(plan, x, True), np.zeros_like(x)
    elif case == "c2c_f64_order15":
        plan, b, n = Z.Plan(Z.C2C, 15, np.float64), 96, 1 << 15
        x = rng.uniform(-1, 1, (b, n)) + 1j * rng.uniform(-1, 1, (b, n))
        op, ref, out = Z.BACKWARD, G.run_c2c(plan, x, False), np.zeros_like(x)
    elif case == "r2c_f32_order17":
        plan, b, n = Z.Plan(Z.R2C, 17, np.float32), 96, 1 << 17
        x = rng.uniform(-1, 1, (b, n)).astype(np.float32)
        op, ref, out = Z.FORWARD, G.run_r2c(plan, x), np.zeros((b, n // 2 + 1), np.complex64)
    else:
        plan, b, n = Z.Plan(Z.R2C, 17, np.float32), 96, 1 << 17
        x = (rng.uniform(-1, 1, (b, n // 2 + 1)) + 1j * rng.uniform(-1, 1, (b, n // 2 + 1))).astype(np.complex64)
        x[:, 0] = x[:, 0].real
        x[:, -1] = x[:, -1].real
        op, ref, out = Z.BACKWARD, G.run_c2r(plan, x), np.zeros((b, n), np.float32)
    x = np.ascontiguousarray(x)
    for _ in range(3):  # pageable buffers: staged through the plan's pinned buffers
        out[...] = 0
        plan.exec_host(op, Z.AOS, Z.AOS, x.ctypes.data, None, out.ctypes.data, None, b)
        assert np.array_equal(out, ref), case
    hin = torch.from_numpy(x.view(np.uint8)).pin_memory()
    hout = torch.zeros(out.nbytes, dtype=torch.uint8).pin_memory()
    for _ in range(3):  # page-locked buffers: copied directly
        hout.zero_()
        plan.exec_host(op, Z.AOS, Z.AOS, hin.data_ptr(), None, hout.data_ptr(), None, b)
        assert np.array_equal(hout.numpy().view(out.dtype).reshape(out.shape), ref), case
    assert plan.device_status() == 0



def test_threads_share_plans():
    """Host threads share plans: two call one order-16 plan through the
    host-batched path (serialised on the plan's staging lock), and two call
    one order-12 plan (single-CTA tiles, no scratch) through the device path
    on their own streams, all at once. Every result equals the
    single-threaded one, and each plan's launch counter (atomic) counts every
    launch."""
    import threading
    import torch
    rng = np.random.default_rng(31)
    big, small = Z.Plan(Z.C2C, 16, np.float32), Z.Plan(Z.C2C, 12, np.float32)
    xb = [(rng.uniform(-1, 1, (64, 1 << 16)) + 1j * rng.uniform(-1, 1, (64, 1 << 16))).astype(np.complex64)
          for _ in range(2)]
    xs = [(rng.uniform(-1, 1, (512, 1 << 12)) + 1j * rng.uniform(-1, 1, (512, 1 << 12))).astype(np.complex64)
          for _ in range(2)]
    rb = [G.run_c2c(big, x, True) for x in xb]
    rs = [G.run_c2c(small, x, True) for x in xs]
    # launches of one call on each path, measured alone
    ob = np.zeros_like(xb[0])
    big.take_launch_count()
    big.exec_host(Z.FORWARD, Z.AOS, Z.AOS, xb[0].ctypes.data, None, ob.ctypes.data, None, 64)
    per_host = big.take_launch_count()
    small.take_launch_count()
    G.run_c2c(small, xs[0], True)
    per_dev = small.take_launch_count()
    reps, errors = 3, []
    tin = [G.dev(x) for x in xs]
    tout = [torch.zeros((512, 1 << 12, 2), dtype=torch.float32, device="cuda") for _ in xs]
    streams = [torch.cuda.Stream() for _ in xs]

    def host_worker(i):
        try:
            out = np.zeros_like(xb[i])
            for _ in range(reps):
                big.exec_host(Z.FORWARD, Z.AOS, Z.AOS, xb[i].ctypes.data, None, out.ctypes.data, None, 64)
                if not np.array_equal(out, rb[i]):
                    errors.append(("host", i))
        except Exception as e:  # noqa: BLE001 - reported by the assertion below
            errors.append(("host", i, repr(e)))

    def device_worker(i):
        try:
            for _ in range(reps):
                small.exec_device(Z.FORWARD, Z.AOS, Z.AOS, tin[i].data_ptr(), None, tout[i].data_ptr(), None, 512,
                                  stream=streams[i].cuda_stream)
                streams[i].synchronize()
                o = G.host(tout[i])
                if not np.array_equal((o[..., 0] + 1j * o[..., 1]).astype(np.complex64), rs[i]):
                    errors.append(("device", i))
        except Exception as e:  # noqa: BLE001 - reported by the assertion below
            errors.append(("device", i, repr(e)))

    ths = [threading.Thread(target=host_worker, args=(i,)) for i in range(2)]
    ths += [threading.Thread(target=device_worker, args=(i,)) for i in range(2)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    assert not errors, errors
    assert big.take_launch_count() == 2 * reps * per_host
    assert small.take_launch_count() == 2 * reps * per_dev
    assert big.device_status() == 0 and small.device_status() == 0


def test_padded_in_place_rfft_and_cross_transform_aliasing_refused():
    """The padded in-place RFFT (real stride N + 2 = two reals per bin, same
    start and byte stride as the bins) runs forward and backward on the tile
    and multi-pass paths, equal to the out-of-place results bit for bit.
    Overlaps that would let one transform's output overwrite another's input
    (dense in place RFFT, in place with different strides, a shifted output)
    are refused."""
    import torch
    for order in (12, 16):  # single-CTA tiles; multi-pass
        n, nb = 1 << order, (1 << order) // 2 + 1
        plan = Z.Plan(Z.R2C, order, np.float32)
        rng = np.random.default_rng(60 + order)
        b = 6
        x = rng.uniform(-1, 1, (b, n)).astype(np.float32)
        ref = G.run_r2c(plan, x)
        buf = torch.zeros((b, 2 * nb), dtype=torch.float32, device="cuda")
        buf[:, :n] = torch.from_numpy(x).cuda()
        plan.exec_device(Z.FORWARD, Z.AOS, Z.AOS, buf.data_ptr(), None, buf.data_ptr(), None, b, 2 * nb, nb)
        torch.cuda.synchronize()
        got = G.host(buf).reshape(b, nb, 2)
        assert np.array_equal(got[..., 0] + 1j * got[..., 1], ref), order
        back_ref = G.run_c2r(plan, ref)
        plan.exec_device(Z.BACKWARD, Z.AOS, Z.AOS, buf.data_ptr(), None, buf.data_ptr(), None, b, nb, 2 * nb)
        torch.cuda.synchronize()
        assert np.array_equal(G.host(buf)[:, :n], back_ref), order
        with pytest.raises(Z.ZlfftError) as e:  # dense: real stride N, bin stride N/2 + 1
            plan.exec_device(Z.FORWARD, Z.AOS, Z.AOS, buf.data_ptr(), None, buf.data_ptr(), None, b, n, nb)
        assert e.value.code == Z._capi.ERR_INVALID_ARG
        assert plan.device_status() == 0
    cplan = Z.Plan(Z.C2C, 9, np.float32)
    t = torch.zeros((8, 512, 2), dtype=torch.float32, device="cuda")
    with pytest.raises(Z.ZlfftError) as e:
        cplan.exec_device(Z.FORWARD, Z.AOS, Z.AOS, t.data_ptr(), None, t.data_ptr(), None, 4, 512, 520)
    assert e.value.code == Z._capi.ERR_INVALID_ARG
    with pytest.raises(Z.ZlfftError) as e:
        cplan.exec_device(Z.FORWARD, Z.AOS, Z.AOS, t.data_ptr(), None, t[1].data_ptr(), None, 4)
    assert e.value.code == Z._capi.ERR_INVALID_ARG


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_single_transform_host_path_equals_device_path(oracle, prec):
    """One small transform from host buffers runs on mapped page-locked
    buffers (one launch, one synchronisation); it must give the device path's
    bits in every layout, CFFT orders 0-13 and RFFT orders 1-14, in place too."""
    ft, ct = (np.float32, np.complex64) if prec == "f32" else (np.float64, np.complex128)
    rng = np.random.default_rng(1010)
    for order in range(0, 14):
        n = 1 << order
        x = (rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)).astype(ct)
        cf = Z.CFFT(order, ft)
        for fwd in (True, False):
            ref = G.run_c2c(cf.plan, x[None, :], fwd)[0]
            y = np.zeros_like(x)
            (cf.forward if fwd else cf.backward)(x, y)
            assert np.array_equal(y, ref), (order, fwd)
            re, im = np.zeros(n, ft), np.zeros(n, ft)
            (cf.forward if fwd else cf.backward)((np.ascontiguousarray(x.real), np.ascontiguousarray(x.imag)),
                                                 (re, im))
            assert np.array_equal(re + 1j * im, ref), (order, fwd)
            z = x.copy()
            (cf.forward if fwd else cf.backward)(z, z)  # in place
            assert np.array_equal(z, ref), (order, fwd)
    for order in range(1, 15):
        n = 1 << order
        xr = rng.uniform(-1, 1, n).astype(ft)
        rf = Z.RFFT(order, ft)
        X = np.zeros(n // 2 + 1, ct)
        rf.forward(xr, X)
        assert np.array_equal(X, G.run_r2c(rf.plan, xr[None, :])[0]), order
        P = np.zeros(n // 2 + 1, ft)
        rf.forward_sqr_mag(xr, P)
        assert np.array_equal(P, G.run_r2c(rf.plan, xr[None, :], sqr_mag=True)[0]), order
        back = np.zeros(n, ft)
        rf.backward(X, back)
        assert np.array_equal(back, G.run_c2r(rf.plan, X[None, :])[0]), order
        if prec == "f32":
            assert np.array_equal(X, oracle.rfft_forward_port(xr)), order


@pytest.mark.parametrize("prec,ft,ct", PRECS)
@pytest.mark.parametrize("order", [19, 20])
def test_multipass_fast_form_two_pass_orders(oracle, prec, ft, ct, order):
    """The fast-twiddle form at orders 19-20, which may run as two passes
    (512 | 1024 and 1024 | 1024 points): within the tolerance of the FP64 DFT,
    both directions, AoS and SoA, several chunks."""
    n = 1 << order
    rng = np.random.default_rng(3500 + order)
    b = 3
    x = _cx(rng, b, n, ct)
    plan = Z.Plan(Z.C2C, order, ft, mode=Z.MODE_FAST)
    tol = oracle.tolerance(order, prec)
    for forward in (True, False):
        fp64 = oracle.cfft_fp64(x, forward)
        for il, ol in ((Z.AOS, Z.AOS), (Z.SOA, Z.SOA)):
            y = G.run_c2c(plan, x, forward, il, ol)
            assert oracle.rel_l2(y, fp64).max() <= tol, (order, forward, il, ol)


def test_pass_schemes_agree_bitwise():
    """Orders 19 and 20 in three passes (ZLFFT_PASS_SCHEME=0) and in two
    (ZLFFT_PASS_SCHEME=1; a process each, since the switch is read once): the
    same butterflies and twiddles, so the plain form's outputs are
    bit-identical in both precisions, forward and backward, AoS and SoA."""
    import os
    import subprocess
    import sys
    code = r'''
import sys, numpy as np, torch
sys.path.insert(0, sys.argv[1])
import zldsp_fft_b200 as Z
rng = np.random.default_rng(37)
out = {}
for dt, ct in ((np.float32, np.complex64), (np.float64, np.complex128)):
    for order, b in ((19, 5), (20, 3)):
        n = 1 << order
        x = (rng.uniform(-1, 1, (b, n)) + 1j * rng.uniform(-1, 1, (b, n))).astype(ct)
        p = Z.Plan(Z.C2C, order, dt)
        ti = torch.from_numpy(x.view(dt).reshape(b, n, 2).copy()).cuda()
        f = torch.empty_like(ti); g = torch.empty_like(ti)
        p.exec_device(Z.FORWARD, Z.AOS, Z.AOS, ti.data_ptr(), None, f.data_ptr(), None, b)
        p.exec_device(Z.BACKWARD, Z.AOS, Z.AOS, f.data_ptr(), None, g.data_ptr(), None, b)
        re = torch.empty(b, n, dtype=ti.dtype, device="cuda"); im = torch.empty_like(re)
        p.exec_device(Z.FORWARD, Z.AOS, Z.SOA, ti.data_ptr(), None, re.data_ptr(), im.data_ptr(), b)
        torch.cuda.synchronize()
        assert p.device_status() == 0
        k = f"{np.dtype(dt).name}_{order}"
        out["f" + k] = f.cpu().numpy(); out["g" + k] = g.cpu().numpy()
        out["r" + k] = re.cpu().numpy(); out["i" + k] = im.cpu().numpy()
np.savez(sys.argv[2], **out)
'''
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    res = {}
    for flag in ("0", "1"):
        path = os.path.join(os.environ.get("TMPDIR", "/tmp"), f"zlfft_scheme_{flag}_{os.getpid()}.npz")
        env = dict(os.environ, ZLFFT_PASS_SCHEME=flag)
        r = subprocess.run([sys.executable, "-c", code, root, path], env=env, capture_output=True, text=True,
                           timeout=600)
        assert r.returncode == 0, r.stdout + r.stderr
        res[flag] = dict(np.load(path))
        os.remove(path)
    for k in res["0"]:
        assert np.array_equal(res["0"][k], res["1"][k]), k
