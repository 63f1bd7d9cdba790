"""Orders 25 and 26 (the reference's macro-path sizes above the multi-pass
kernels' earlier limit of 24): three Stockham passes, one transform of
32-64 M points. FP32 plain: the reference's bits (the oracle port); both
precisions within the bar of the FP64 oracle."""
import numpy as np
import pytest

import zldsp_fft_b200 as Z
from tests import gpu_util as G

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("order", [25, 26])
def test_cfft_f32_large(oracle, order):
    n = 1 << order
    rng = np.random.default_rng(5000 + order)
    x = (rng.uniform(-1, 1, (1, n)) + 1j * rng.uniform(-1, 1, (1, n))).astype(np.complex64)
    plan = Z.Plan(Z.C2C, order, np.float32)
    y = G.run_c2c(plan, x, True)
    assert np.array_equal(y, oracle.cfft_port(x, True))
    assert oracle.rel_l2(y, oracle.cfft_fp64(x)).max() <= oracle.tolerance(order, "f32")
    back = G.run_c2c(plan, y, False)  # unnormalised: N x
    assert oracle.rel_l2(back, n * x.astype(np.complex128)).max() <= 2 * oracle.tolerance(order, "f32")
    fast = G.run_c2c(Z.Plan(Z.C2C, order, np.float32, mode=Z.MODE_FAST), x, True)
    assert oracle.rel_l2(fast, oracle.cfft_fp64(x)).max() <= oracle.tolerance(order, "f32")


def test_cfft_f64_order25(oracle):
    order = 25
    n = 1 << order
    rng = np.random.default_rng(5100)
    x = rng.uniform(-1, 1, (1, n)) + 1j * rng.uniform(-1, 1, (1, n))
    y = G.run_c2c(Z.Plan(Z.C2C, order, np.float64), x, True)
    assert oracle.rel_l2(y, oracle.cfft_fp64(x)).max() <= oracle.tolerance(order, "f64")


def test_rfft_f32_order26(oracle):
    order = 26  # complex order 25 plus the split
    n = 1 << order
    rng = np.random.default_rng(5200)
    x = rng.uniform(-1, 1, (1, n)).astype(np.float32)
    plan = Z.Plan(Z.R2C, order, np.float32)
    X = G.run_r2c(plan, x)
    assert np.array_equal(X, oracle.rfft_forward_port(x))
    assert oracle.rel_l2(X, oracle.rfft_fp64(x)).max() <= oracle.tolerance(order, "f32")


def test_order_above_26_refused():
    with pytest.raises(Z.ZlfftError):
        Z.Plan(Z.C2C, 27, np.float32)
