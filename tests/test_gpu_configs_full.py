"""The benchmark configurations at their full stated shapes, checked on the GPU
through properties that hold at any size plus bit-exact / FP64 samples:

* CFFT<float> orders 14, 16 and 20, each batched to 2 GiB of complex64
  (16384 / 4096 / 256 transforms), forward then backward, plain form (the
  reference's arithmetic) and the tensor-core split form;
* CFFT<double> order 16 x 512 (1 GiB per direction), the FP64 path.

Properties on every transform of the batch: the round trip backward(forward(x))
equals N x within 2 * 4 log2(N) eps (relative L2, per transform, computed on the
device in FP64), and Parseval's identity sum |X|^2 = N sum |x|^2 holds within
twice that. Samples (first, middle and last transform): bit-identical to the
oracle's restatement (FP32 plain form), within 4 log2(N) eps of numpy's FP64
FFT (every form).
"""
import numpy as np
import pytest

import zldsp_fft_b200 as Z

pytestmark = pytest.mark.gpu


def _run_full(order, total, dtype, mode):
    import torch
    rdt = torch.float32 if dtype == np.float32 else torch.float64
    n = 1 << order
    b = total >> order
    g = torch.Generator(device="cuda")
    g.manual_seed(1003 + order)
    x = (torch.rand((b, n, 2), generator=g, device="cuda", dtype=rdt) * 2 - 1).contiguous()
    y = torch.empty_like(x)
    z = torch.empty_like(x)
    p = Z.Plan(Z.C2C, order, dtype, mode)
    p.exec_device(Z.FORWARD, Z.AOS, Z.AOS, x.data_ptr(), None, y.data_ptr(), None, b)
    p.exec_device(Z.BACKWARD, Z.AOS, Z.AOS, y.data_ptr(), None, z.data_ptr(), None, b)
    torch.cuda.synchronize()
    assert p.device_status() == 0
    return x, y, z, b, n


def _properties(x, y, z, n, bar):
    import torch
    xd = torch.view_as_complex(x.double()) if x.dtype == torch.float32 else torch.view_as_complex(x)
    yd = torch.view_as_complex(y.double()) if y.dtype == torch.float32 else torch.view_as_complex(y)
    zd = torch.view_as_complex(z.double()) if z.dtype == torch.float32 else torch.view_as_complex(z)
    nx = torch.linalg.vector_norm(xd, dim=-1)
    rt = torch.linalg.vector_norm(zd - n * xd, dim=-1) / (n * nx)
    assert rt.max().item() <= 2 * bar, rt.max().item()
    pars = (torch.linalg.vector_norm(yd, dim=-1) ** 2 - n * nx ** 2).abs() / (n * nx ** 2)
    assert pars.max().item() <= 4 * bar, pars.max().item()  # |X|^2 doubles the relative error


@pytest.mark.parametrize("order", [14, 16, 20])
@pytest.mark.parametrize("form", ["plain", "tc"])
def test_config3_full_2gib_batches(oracle, order, form):
    mode = Z.MODE_PLAIN if form == "plain" else Z.MODE_TC_FP16
    x, y, z, b, n = _run_full(order, 1 << 28, np.float32, mode)
    bar = oracle.tolerance(order, "f32")
    _properties(x, y, z, n, bar)
    for i in (0, b // 2, b - 1):
        xi = x[i].cpu().numpy().view(np.complex64)[:, 0]
        yi = y[i].cpu().numpy().view(np.complex64)[:, 0]
        assert oracle.rel_l2(yi[None], oracle.cfft_fp64(xi[None])).max() <= bar, (i, form)
        if form == "plain":
            assert np.array_equal(yi, oracle.cfft_port(xi[None], True)[0]), i
    del x, y, z


def test_config5_cfft_double_order16_batch512(oracle):
    x, y, z, b, n = _run_full(16, 512 << 16, np.float64, Z.MODE_PLAIN)
    assert b == 512
    bar = oracle.tolerance(16, "f64")
    _properties(x, y, z, n, bar)
    for i in (0, b // 2, b - 1):
        xi = x[i].cpu().numpy().view(np.complex128)[:, 0]
        yi = y[i].cpu().numpy().view(np.complex128)[:, 0]
        assert oracle.rel_l2(yi[None], oracle.cfft_fp64(xi[None])).max() <= bar, i
        assert oracle.rel_l2(yi[None], oracle.cfft_port(xi[None], True)).max() <= 2 * bar, i
