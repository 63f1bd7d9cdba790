"""Autotuning (zlfft_autotune): measured plan choice per transform size.

The tuned parameters (scratch chunk, chunk pipelines, TMA staging) never change
a form's arithmetic, so a plain plan gives the same bits before and after
tuning; MODE_TUNED plans may take the tensor-core form, which stays within the
FP32 bar against the FP64 oracle."""
import numpy as np
import pytest

import zldsp_fft_b200 as Z
from tests import gpu_util as G

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _clean_table():
    Z.tuning_clear()
    yield
    Z.tuning_clear()


def test_autotune_records_entries_and_keeps_results(oracle):
    rng = np.random.default_rng(31)
    n = 1 << 14
    x = (rng.uniform(-1, 1, (40, n)) + 1j * rng.uniform(-1, 1, (40, n))).astype(np.complex64)
    before = G.run_c2c(Z.Plan(Z.C2C, 14, np.float32), x, True)
    Z.autotune(Z.C2C, 12, 14, np.float32)
    Z.autotune(Z.R2C, 15, 15, np.float32)
    for kind, order in ((Z.C2C, 12), (Z.C2C, 13), (Z.C2C, 14), (Z.R2C, 15)):
        t = Z.tuning(kind, order, np.float32)
        assert t is not None, (kind, order)
        assert t["gbs"] > 0 and t["gbs"] >= t["gbs_default"] > 0, t
        assert t["streams"] in (1, 2) and t["tma"] in (0, 1)
    assert Z.tuning(Z.C2C, 16, np.float32) is None
    t14 = Z.tuning(Z.C2C, 14, np.float32)
    assert t14["chunk_mb"] in (16, 32, 48, 96, 192)
    # a plain plan created after tuning (tuned chunk, pipelines, staging): same bits
    after = G.run_c2c(Z.Plan(Z.C2C, 14, np.float32), x, True)
    assert np.array_equal(before, after)
    # the tuned form: plain bits, or the fast-twiddle / tensor-core form within the FP32 bar
    tuned = G.run_c2c(Z.Plan(Z.C2C, 14, np.float32, mode=Z.MODE_TUNED), x, True)
    if t14["form"] == "plain":
        assert np.array_equal(tuned, before)
    assert oracle.rel_l2(tuned, oracle.cfft_fp64(x)).max() <= oracle.tolerance(14, "f32")
    # RFFT order 15 under its tuned plan: the reference's bits in the plain form
    xr = rng.uniform(-1, 1, (8, 1 << 15)).astype(np.float32)
    p = Z.Plan(Z.R2C, 15, np.float32, mode=Z.MODE_TUNED)
    t15 = Z.tuning(Z.R2C, 15, np.float32)
    assert t15["split_fused"] in (0, 1) and t15["form"] in ("plain", "fast")
    got = G.run_r2c(p, xr)
    if t15["form"] == "plain":
        assert np.array_equal(got, oracle.rfft_forward_port(xr))
    ref = np.fft.rfft(xr.astype(np.float64), axis=-1)
    err = np.linalg.norm(got - ref, axis=-1) / np.linalg.norm(ref, axis=-1)
    assert err.max() <= oracle.tolerance(15, "f32")


def test_tuning_file_round_trip(tmp_path):
    Z.autotune(Z.C2C, 13, 14, np.float32)
    want = {o: Z.tuning(Z.C2C, o, np.float32) for o in (13, 14)}
    path = str(tmp_path / "tune.txt")
    Z.tuning_save(path)
    Z.tuning_clear()
    assert Z.tuning(Z.C2C, 14, np.float32) is None
    assert Z.tuning_load(path) == 2
    for o in (13, 14):
        got = Z.tuning(Z.C2C, o, np.float32)
        for k in ("chunk_mb", "streams", "tma", "form", "split_fused", "store_tma"):
            assert got[k] == want[o][k], (o, k)
    # a file written on another GPU model is not applied here
    other = tmp_path / "other.txt"
    text = open(path).read().splitlines()
    other.write_text("\n".join("gpu Some_Other_GPU sms 7" if ln.startswith("gpu ") else ln for ln in text) + "\n")
    Z.tuning_clear()
    assert Z.tuning_load(str(other)) == 0
    assert Z.tuning(Z.C2C, 14, np.float32) is None


def _this_gpu():
    import torch
    prop = torch.cuda.get_device_properties(0)
    return prop.name.replace(" ", "_").replace("\t", "_"), prop.multi_processor_count


@pytest.mark.parametrize("prec,dt", [("f32", np.float32), ("f64", np.float64)])
def test_rfft_split_fused_into_last_pass(oracle, tmp_path, prec, dt):
    """A tuning file can select the RFFT forward whose split runs inside the
    last multi-pass pass (units paired with their mirrors in one CTA): same
    bits as the oracle in FP32 (AoS, SoA, squared magnitudes), within the bar
    in FP64, including batches of several chunks."""
    name, sms = _this_gpu()
    pv = 0 if dt == np.float32 else 1
    lines = [f"gpu {name} sms {sms}"] + [f"entry 1 {pv} {o} 48 2 1 0 1 -1 0 0" for o in (15, 16, 17)]
    path = tmp_path / "fused.txt"
    path.write_text("\n".join(lines) + "\n")
    assert Z.tuning_load(str(path)) == 3
    rng = np.random.default_rng(77)
    for order, batch in ((15, 3), (16, 2), (17, 1)):
        assert Z.tuning(Z.R2C, order, dt)["split_fused"] == 1
        n = 1 << order
        x = rng.uniform(-1, 1, (batch, n)).astype(dt)
        plan = Z.Plan(Z.R2C, order, dt)
        tol = oracle.tolerance(order, prec)
        for ol in (Z.AOS, Z.SOA):
            X = G.run_r2c(plan, x, ol)
            assert oracle.rel_l2(X, oracle.rfft_fp64(x)).max() <= tol, (order, ol)
            if prec == "f32":
                assert np.array_equal(X, oracle.rfft_forward_port(x)), (order, ol)
        P = G.run_r2c(plan, x, sqr_mag=True)
        if prec == "f32":
            assert np.array_equal(P, oracle.rfft_forward_port(x, sqr_mag=True)), order
        else:
            ref = np.abs(oracle.rfft_fp64(x)) ** 2
            assert oracle.rel_l2(P, ref).max() <= 2 * tol
    # 300 frames of order 16 at a 16 MiB chunk: many chunks on both pipelines
    path.write_text(f"gpu {name} sms {sms}\nentry 1 {pv} 16 16 2 1 0 1 -1 0 0\n")
    assert Z.tuning_load(str(path)) == 1
    x = rng.uniform(-1, 1, (300, 1 << 16)).astype(dt)
    X = G.run_r2c(Z.Plan(Z.R2C, 16, dt), x, Z.AOS)
    assert oracle.rel_l2(X, oracle.rfft_fp64(x)).max() <= oracle.tolerance(16, prec)


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_first_pass_tma_store_on_and_off_give_the_same_bits(oracle, tmp_path, dt):
    """The first multi-pass pass writes its output by TMA tensor stores of
    swizzled boxes or by the threads; both give the same bits (FP32: the
    oracle's), for pass radices 16 (order 20), 64 (14), 256 (16) and 512 (17)."""
    name, sms = _this_gpu()
    pv = 0 if dt == np.float32 else 1
    rng = np.random.default_rng(123)
    for order, batch in ((14, 33), (16, 9), (17, 3), (20, 1)):
        n = 1 << order
        x = (rng.uniform(-1, 1, (batch, n)) + 1j * rng.uniform(-1, 1, (batch, n))).astype(
            np.complex64 if dt == np.float32 else np.complex128)
        res = []
        for store in (0, 1):
            path = tmp_path / f"s{store}.txt"
            path.write_text(f"gpu {name} sms {sms}\nentry 0 {pv} {order} 16 2 1 0 0 {store} 0 0\n")
            Z.tuning_clear()
            assert Z.tuning_load(str(path)) == 1
            plan = Z.Plan(Z.C2C, order, dt)
            res.append((G.run_c2c(plan, x, True), G.run_c2c(plan, x, False)))
        assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1]), order
        if dt == np.float32:
            assert np.array_equal(res[1][0], oracle.cfft_port(x, True)), order
