"""STFT front end (zlfft_stft_device): framing at a hop, window multiply,
RFFT forward / forward_sqr_mag in one launch, against the oracle applied to
frames cut and windowed on the host."""
import numpy as np
import pytest

import zldsp_fft_b200 as Z

pytestmark = pytest.mark.gpu


def _frames(sig, n, hop, nf, win):
    idx = np.arange(nf)[:, None] * hop + np.arange(n)[None, :]
    fr = sig[idx]
    return fr * win[None, :] if win is not None else fr


def _run(plan, sig, hop, win, nf, op, ol, out_stride=0):
    import torch
    n = 1 << plan.order
    nb = n // 2 + 1
    rdt = torch.float32 if sig.dtype == np.float32 else torch.float64
    ts = torch.from_numpy(sig).cuda()
    tw = torch.from_numpy(win).cuda() if win is not None else None
    stride = out_stride or nb
    if op == Z.FORWARD_SQR_MAG or ol == Z.SOA:
        o0 = torch.zeros((nf, stride), dtype=rdt, device="cuda")
        o1 = torch.zeros((nf, stride), dtype=rdt, device="cuda") if ol == Z.SOA else None
    else:
        o0 = torch.zeros((nf, stride, 2), dtype=rdt, device="cuda")
        o1 = None
    plan.stft(op, ol, ts.data_ptr(), hop, tw.data_ptr() if tw is not None else None, o0.data_ptr(),
              o1.data_ptr() if o1 is not None else None, nf, out_stride)
    torch.cuda.synchronize()
    a = o0.cpu().numpy()
    if op == Z.FORWARD_SQR_MAG:
        return a[:, :nb]
    if ol == Z.SOA:
        return (a + 1j * o1.cpu().numpy())[:, :nb]
    return (a[..., 0] + 1j * a[..., 1])[:, :nb]


@pytest.mark.parametrize("order,hop,nf", [(12, 1024, 40), (12, 6, 25), (8, 2, 300), (14, 4096, 9), (15, 8192, 6),
                                          (1, 2, 5)])
def test_stft_f32_bit_exact(oracle, order, hop, nf):
    n = 1 << order
    rng = np.random.default_rng(900 + order)
    sig = rng.uniform(-1, 1, (nf - 1) * hop + n).astype(np.float32)
    win = (0.5 - 0.5 * np.cos(2 * np.pi * np.arange(n) / n)).astype(np.float32)
    plan = Z.Plan(Z.R2C, order, np.float32)
    frames = _frames(sig, n, hop, nf, win)
    ref = oracle.rfft_forward_port(frames)
    for ol in (Z.AOS, Z.SOA):
        y = _run(plan, sig, hop, win, nf, Z.FORWARD, ol)
        assert np.array_equal(y, ref.astype(np.complex64)), (order, hop, ol)
    p = _run(plan, sig, hop, win, nf, Z.FORWARD_SQR_MAG, Z.AOS)
    assert np.array_equal(p, oracle.rfft_forward_port(frames, sqr_mag=True)), (order, hop)
    # rectangular window (NULL): plain framing
    y = _run(plan, sig, hop, None, nf, Z.FORWARD, Z.AOS)
    assert np.array_equal(y, oracle.rfft_forward_port(_frames(sig, n, hop, nf, None)))
    assert oracle.rel_l2(y, oracle.rfft_fp64(_frames(sig, n, hop, nf, None))).max() <= oracle.tolerance(order, "f32")


def test_stft_f64_and_strided_output(oracle):
    order, hop, nf = 11, 512, 12
    n = 1 << order
    rng = np.random.default_rng(5)
    sig = rng.uniform(-1, 1, (nf - 1) * hop + n)
    win = np.hanning(n + 1)[:n]
    plan = Z.Plan(Z.R2C, order, np.float64)
    y = _run(plan, sig, hop, win, nf, Z.FORWARD, Z.AOS, out_stride=(n // 2 + 1) + 7)
    assert oracle.rel_l2(y, oracle.rfft_fp64(_frames(sig, n, hop, nf, win))).max() <= oracle.tolerance(order, "f64")


def test_stft_rejects_bad_arguments():
    import torch
    lib = Z._capi.lib()
    sig = torch.zeros(1 << 16, device="cuda")
    out = torch.zeros(1 << 16, device="cuda")
    p = Z.Plan(Z.R2C, 10, np.float32)
    h = p.handle
    assert lib.zlfft_stft_device(h, Z.FORWARD, Z.AOS, sig.data_ptr(), 3, None, out.data_ptr(), None, 4, 0,
                                 None) == Z._capi.ERR_INVALID_ARG  # odd hop
    assert lib.zlfft_stft_device(h, Z.BACKWARD, Z.AOS, sig.data_ptr(), 4, None, out.data_ptr(), None, 4, 0,
                                 None) == Z._capi.ERR_INVALID_ARG
    assert lib.zlfft_stft_device(h, Z.FORWARD, Z.SOA, sig.data_ptr(), 4, None, out.data_ptr(), None, 4, 0,
                                 None) == Z._capi.ERR_INVALID_ARG  # SoA needs two outputs
    assert lib.zlfft_stft_device(Z.Plan(Z.C2C, 10).handle, Z.FORWARD, Z.AOS, sig.data_ptr(), 4, None,
                                 out.data_ptr(), None, 4, 0, None) == Z._capi.ERR_INVALID_ARG
    for order, dt in ((16, np.float32), (15, np.float64)):  # above the single-CTA frame orders
        assert lib.zlfft_stft_device(Z.Plan(Z.R2C, order, dt).handle, Z.FORWARD, Z.AOS, sig.data_ptr(), 4, None,
                                     out.data_ptr(), None, 1, 0, None) == Z._capi.ERR_UNSUPPORTED
    assert lib.zlfft_stft_device(h, Z.FORWARD, Z.AOS, sig.data_ptr() + 4, 4, None, out.data_ptr(), None, 4, 0,
                                 None) == Z._capi.ERR_ALIGNMENT
    assert lib.zlfft_stft_device(h, Z.FORWARD, Z.AOS, sig.data_ptr(), 4, None, out.data_ptr(), None, 0, 0,
                                 None) == 0  # no frames
