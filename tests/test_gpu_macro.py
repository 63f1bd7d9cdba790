"""The reference's macro DIF path on the GPU (zlfft_plan_create_hybrid).

On a host whose caches set its switch order low enough, the reference runs
large CFFTs as Cooley-Tukey DIF macro stages + per-segment Stockham + a
digit-reversed transposed store (src/common/zldsp_fft_common_execute.hpp:174-272).
These tests hold the GPU's macro form to that output:
  * FP32 bit for bit against the oracle's restatement of the macro path (itself
    bit-identical to the reference's macro build, tests/test_oracle.py), in every
    layout pairing, CFFT and RFFT, orders 14-22;
  * FP32 against the SHA-256 of the reference's own macro-path outputs
    (tests/golden/reference_macro_f32.npz), orders 14-22;
  * FP64 within 4*log2(N)*2^-53 of the FP64 oracle and of the restatement;
  * many chunks (two pipelines), strides, in place, and the allocation-free
    entry point; refusals.
The small-cache host of the fixtures has (max_l1_order, switch_order) =
(10, 14) for float and (9, 13) for double.
"""
import hashlib
import importlib.util
import os

import numpy as np
import pytest

import zldsp_fft_b200 as Z
from tests.gpu_util import host, run_c2c, run_c2r, run_r2c

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
HOST = {"f32": (10, 14), "f64": (9, 13)}
DT = {"f32": (np.float32, np.complex64), "f64": (np.float64, np.complex128)}


def _make_golden():
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    return mg


def _sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _cx(rng, b, n, ct):
    return (rng.uniform(-1, 1, (b, n)) + 1j * rng.uniform(-1, 1, (b, n))).astype(ct)


def test_macro_plan_micro_orders():
    """The plan takes the reference's micro order: max_l1, or max_l1 - 1 for an
    odd difference; below the switch it is the micro-only plan."""
    for prec, (ft, ct) in DT.items():
        l1, sw = HOST[prec]
        for order in range(sw - 2, sw + 5):
            p = Z.Plan(Z.C2C, order, ft, switch=(l1, sw))
            expect = -1 if order < sw else (l1 - 1 if (order - l1) % 2 else l1)
            assert p.micro_order() == expect, (prec, order)
            r = Z.Plan(Z.R2C, order + 1, ft, switch=(l1, sw))
            assert r.micro_order() == expect, (prec, order)


@pytest.mark.parametrize("order", [14, 15, 16, 17])
def test_macro_cfft_f32_all_layouts_bit_exact(oracle, order):
    rng = np.random.default_rng(4000 + order)
    n = 1 << order
    x = _cx(rng, 3, n, np.complex64)
    plan = Z.Plan(Z.C2C, order, np.float32, switch=HOST["f32"])
    with oracle.macro_host("f32"):
        ref = {fwd: oracle.cfft_port(x, fwd) for fwd in (True, False)}
    for fwd in (True, False):
        for il in (Z.AOS, Z.SOA):
            for ol in (Z.AOS, Z.SOA):
                y = run_c2c(plan, x, fwd, il, ol)
                assert np.array_equal(y, ref[fwd]), (order, fwd, il, ol)
    # and it is the macro path: the micro-only form rounds differently
    assert not np.array_equal(ref[True], oracle.cfft_port(x, True))


@pytest.mark.parametrize("order", [15, 16, 17, 21])
def test_macro_rfft_f32_bit_exact(oracle, order):
    rng = np.random.default_rng(4100 + order)
    n = 1 << order
    b = 2 if order < 20 else 1
    xr = rng.uniform(-1, 1, (b, n)).astype(np.float32)
    plan = Z.Plan(Z.R2C, order, np.float32, switch=HOST["f32"])
    assert plan.micro_order() > 0
    with oracle.macro_host("f32"):
        X = oracle.rfft_forward_port(xr)
        P = oracle.rfft_forward_port(xr, sqr_mag=True)
        back = oracle.rfft_backward_port(X)
    for ol in (Z.AOS, Z.SOA):
        assert np.array_equal(run_r2c(plan, xr, ol), X), (order, ol)
    assert np.array_equal(run_r2c(plan, xr, sqr_mag=True), P), order
    for il in (Z.AOS, Z.SOA):
        assert np.array_equal(run_c2r(plan, X, il), back), (order, il)


@pytest.mark.parametrize("order", [18, 20, 22])
def test_macro_cfft_f32_large_orders_bit_exact(oracle, order):
    """One and two DIF passes (order 22: six macro stages, 3 + 3)."""
    rng = np.random.default_rng(4200 + order)
    x = _cx(rng, 1, 1 << order, np.complex64)
    plan = Z.Plan(Z.C2C, order, np.float32, switch=HOST["f32"])
    with oracle.macro_host("f32"):
        for fwd in (True, False):
            assert np.array_equal(run_c2c(plan, x, fwd), oracle.cfft_port(x, fwd)), (order, fwd)
    assert oracle.rel_l2(run_c2c(plan, x, True), oracle.cfft_fp64(x, True)).max() <= oracle.tolerance(order)


def test_macro_f32_matches_reference_fixture_hashes():
    """The GPU's macro form reproduces the reference's own macro-path outputs
    (SHA-256 of the output bytes, tests/golden/make_golden.py), orders 14-22:
    CFFT forward and backward, RFFT forward, forward_sqr_mag and backward."""
    mg = _make_golden()
    g = np.load(os.path.join(GOLDEN, "reference_macro_f32.npz"))
    for order in mg.MACRO_ORDERS["f32"]:
        x, xr, X = mg.macro_inputs("f32", order)
        cp = Z.Plan(Z.C2C, order, np.float32, switch=HOST["f32"])
        rp = Z.Plan(Z.R2C, order + 1, np.float32, switch=HOST["f32"])
        got = [_sha(run_c2c(cp, x, True)), _sha(run_c2c(cp, x, False)), _sha(run_r2c(rp, xr)),
               _sha(run_r2c(rp, xr, sqr_mag=True)), _sha(run_c2r(rp, X))]
        assert got == list(g[f"sha_{order}"]), order
        del cp, rp


@pytest.mark.parametrize("order", [13, 14, 15, 16, 19, 21])
def test_macro_f64_within_tolerance(oracle, order):
    rng = np.random.default_rng(4300 + order)
    n = 1 << order
    b = 2 if order < 18 else 1
    x = _cx(rng, b, n, np.complex128)
    plan = Z.Plan(Z.C2C, order, np.float64, switch=HOST["f64"])
    assert plan.micro_order() > 0
    tol = oracle.tolerance(order, "f64")
    with oracle.macro_host("f64"):
        for fwd in (True, False):
            y = run_c2c(plan, x, fwd, Z.SOA if fwd else Z.AOS, Z.AOS)
            assert oracle.rel_l2(y, oracle.cfft_fp64(x, fwd)).max() <= tol, (order, fwd)
            assert oracle.rel_l2(y, oracle.cfft_port(x, fwd)).max() <= 2 * tol, (order, fwd)
        if order <= 16:
            xr = rng.uniform(-1, 1, (b, 2 * n)).astype(np.float64)
            rp = Z.Plan(Z.R2C, order + 1, np.float64, switch=HOST["f64"])
            X = run_r2c(rp, xr)
            assert oracle.rel_l2(X, oracle.rfft_fp64(xr)).max() <= oracle.tolerance(order + 1, "f64")
            back = run_c2r(rp, X)
            assert oracle.rel_l2(back, oracle.rfft_backward_fp64(X)).max() <= oracle.tolerance(order + 1, "f64")


def test_macro_many_chunks_strides_in_place(oracle):
    """More transforms than one scratch chunk (both pipelines), strided and
    in-place calls: the same bits as the oracle's per-transform results."""
    import torch
    order, b = 14, 900  # 128 KB per transform: 384 per 48 MiB chunk -> 3 chunks on 2 pipelines
    n = 1 << order
    rng = np.random.default_rng(4400)
    x = _cx(rng, b, n, np.complex64)
    plan = Z.Plan(Z.C2C, order, np.float32, switch=HOST["f32"])
    with oracle.macro_host("f32"):
        ref = oracle.cfft_port(x, True)
    assert np.array_equal(run_c2c(plan, x, True), ref)
    # strided: transforms 1.25 N apart in and 1.5 N apart out
    si, so = n + n // 4, n + n // 2
    xs = np.zeros((b, si), np.complex64)
    xs[:, :n] = x
    ti = torch.from_numpy(xs.view(np.float32).reshape(b, si, 2).copy()).cuda()
    to = torch.zeros((b, so, 2), dtype=torch.float32, device="cuda")
    plan.exec_device(Z.FORWARD, Z.AOS, Z.AOS, ti.data_ptr(), None, to.data_ptr(), None, b, si, so)
    torch.cuda.synchronize()
    y = host(to)[:, :n]
    assert np.array_equal((y[..., 0] + 1j * y[..., 1]).astype(np.complex64), ref)
    # in place
    t = torch.from_numpy(x.view(np.float32).reshape(b, n, 2).copy()).cuda()
    plan.exec_device(Z.FORWARD, Z.AOS, Z.AOS, t.data_ptr(), None, t.data_ptr(), None, b)
    torch.cuda.synchronize()
    y = host(t)
    assert np.array_equal((y[..., 0] + 1j * y[..., 1]).astype(np.complex64), ref)
    assert plan.device_status() == 0


def test_macro_noalloc_equals_device_path():
    """The allocation-free entry point runs macro plans through the built-in
    array: the same bits as zlfft_exec_device, two calls in a row."""
    import torch
    lib = Z._capi.lib()
    for order, b in ((14, 300), (20, 3)):
        n = 1 << order
        rng = np.random.default_rng(4500 + order)
        x = _cx(rng, b, n, np.complex64)
        plan = Z.Plan(Z.C2C, order, np.float32, switch=HOST["f32"])
        ti = torch.from_numpy(x.view(np.float32).reshape(b, n, 2).copy()).cuda()
        ref = torch.zeros_like(ti)
        plan.exec_device(Z.BACKWARD, Z.AOS, Z.AOS, ti.data_ptr(), None, ref.data_ptr(), None, b)
        for _ in range(2):
            out = torch.zeros_like(ti)
            Z._capi.check(lib.zlfft_exec_device_noalloc(plan.handle, Z.BACKWARD, Z.AOS, Z.AOS, ti.data_ptr(), None,
                                                        out.data_ptr(), None, b, 0, 0, None))
            torch.cuda.synchronize()
            assert torch.equal(out, ref), order


def test_macro_refusals():
    import torch
    l1, sw = HOST["f32"]
    # micro orders outside the built range
    with pytest.raises(Z.ZlfftError) as e:
        Z.Plan(Z.C2C, 16, np.float32, switch=(14, 14))
    assert e.value.code == Z._capi.ERR_UNSUPPORTED
    with pytest.raises(Z.ZlfftError):
        Z.Plan(Z.C2C, 16, np.float32, switch=(-1, 14))
    # the STFT entry points run the micro-only form and refuse macro plans
    rp = Z.Plan(Z.R2C, 15, np.float32, switch=(l1, sw))
    assert rp.micro_order() == l1
    sig = torch.zeros(1 << 16, dtype=torch.float32, device="cuda")
    out = torch.zeros((2, (1 << 14) + 1, 2), dtype=torch.float32, device="cuda")
    with pytest.raises(Z.ZlfftError) as e:
        rp.stft(Z.FORWARD, Z.AOS, sig.data_ptr(), 1 << 14, None, out.data_ptr(), None, 2)
    assert e.value.code == Z._capi.ERR_UNSUPPORTED
    with pytest.raises(Z.ZlfftError) as e:
        rp.istft(Z.AOS, out.data_ptr(), None, 1 << 13, 2, sig.data_ptr())
    assert e.value.code == Z._capi.ERR_UNSUPPORTED


def test_host_mode_follows_this_hosts_switch(oracle):
    """ZLFFT_MODE_HOST plans (the drop-in classes' default) take this host's
    switch: bit-identical to the oracle under the same switch."""
    for prec, (ft, ct) in DT.items():
        l1, sw = Z.host_switch_order(ft)
        for order in (12, min(sw, 22)):
            p = Z.Plan(Z.C2C, order, ft, Z.MODE_HOST)
            expect = -1 if order < sw else (l1 - 1 if (order - l1) % 2 else l1)
            assert p.micro_order() == expect, (prec, order)
            if prec == "f32":
                x = _cx(np.random.default_rng(order), 1, 1 << order, ct)
                with oracle.hybrid(prec, l1, sw):
                    assert np.array_equal(run_c2c(p, x, True), oracle.cfft_port(x, True)), order


def test_macro_cfft_f32_orders_24_and_26(oracle):
    """The largest macro orders (seven and eight DIF stages in two passes,
    micro order 10): order 24 forward bit-identical to the restatement; order
    26 (512 MiB per transform) round trip and Parseval within the FP32 bar,
    computed on the device."""
    import torch
    rng = np.random.default_rng(4600)
    x = _cx(rng, 1, 1 << 24, np.complex64)
    plan = Z.Plan(Z.C2C, 24, np.float32, switch=HOST["f32"])
    assert plan.micro_order() == 10
    with oracle.macro_host("f32"):
        assert np.array_equal(run_c2c(plan, x, True), oracle.cfft_port(x, True))
    del x
    n = 1 << 26
    plan = Z.Plan(Z.C2C, 26, np.float32, switch=HOST["f32"])
    g = torch.Generator(device="cuda")
    g.manual_seed(4601)
    a = (torch.rand((n, 2), generator=g, device="cuda") * 2 - 1).contiguous()
    y = torch.empty_like(a)
    z = torch.empty_like(a)
    plan.exec_device(Z.FORWARD, Z.AOS, Z.AOS, a.data_ptr(), None, y.data_ptr(), None, 1)
    plan.exec_device(Z.BACKWARD, Z.AOS, Z.AOS, y.data_ptr(), None, z.data_ptr(), None, 1)
    torch.cuda.synchronize()
    assert plan.device_status() == 0
    xd, yd, zd = (torch.view_as_complex(t.double()) for t in (a, y, z))
    bar = oracle.tolerance(26, "f32")
    nx = torch.linalg.vector_norm(xd)
    assert (torch.linalg.vector_norm(zd - n * xd) / (n * nx)).item() <= 2 * bar
    assert abs((torch.linalg.vector_norm(yd) ** 2 - n * nx ** 2).item()) / (n * nx.item() ** 2) <= 4 * bar
