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
    # the tuned form: plain bits, or the tensor-core form within the FP32 bar
    tuned = G.run_c2c(Z.Plan(Z.C2C, 14, np.float32, mode=Z.MODE_TUNED), x, True)
    if t14["form"] == "plain":
        assert np.array_equal(tuned, before)
    assert oracle.rel_l2(tuned, oracle.cfft_fp64(x)).max() <= oracle.tolerance(14, "f32")
    # RFFT order 15 under its tuned plan
    xr = rng.uniform(-1, 1, (8, 1 << 15)).astype(np.float32)
    p = Z.Plan(Z.R2C, 15, np.float32, mode=Z.MODE_TUNED)
    assert np.array_equal(G.run_r2c(p, xr), oracle.rfft_forward_port(xr))


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
        for k in ("chunk_mb", "streams", "tma", "form"):
            assert got[k] == want[o][k], (o, k)
    # a file written on another GPU model is not applied here
    other = tmp_path / "other.txt"
    text = open(path).read().splitlines()
    other.write_text("\n".join("gpu Some_Other_GPU sms 7" if ln.startswith("gpu ") else ln for ln in text) + "\n")
    Z.tuning_clear()
    assert Z.tuning_load(str(other)) == 0
    assert Z.tuning(Z.C2C, 14, np.float32) is None
