"""Inverse STFT / overlap-add (zlfft_istft_device): spectral filter, RFFT
backward, synthesis window and overlap-add of frames in ascending order, in one
launch, against the oracle's sequential loop over frames (FP32: bit for bit)
and the FP64 oracle (within the RFFT tolerance)."""
import numpy as np
import pytest

import zldsp_fft_b200 as Z
from tests import gpu_util as G

pytestmark = pytest.mark.gpu


def _bins(rng, nf, n, ct):
    nb = n // 2 + 1
    X = (rng.uniform(-1, 1, (nf, nb)) + 1j * rng.uniform(-1, 1, (nf, nb))).astype(ct)
    X[:, 0] = X[:, 0].real  # DC and Nyquist bins of a real signal's spectrum
    X[:, -1] = X[:, -1].real
    return X


def _run(plan, X, hop, filt=None, win=None, layout=Z.AOS, in_stride=0):
    import torch
    nf, nb = X.shape
    n = 1 << plan.order
    ft = np.float32 if X.dtype == np.complex64 else np.float64
    tdt = torch.float32 if ft == np.float32 else torch.float64
    stride = in_stride or nb
    if layout == Z.AOS:
        host = np.zeros((nf, stride, 2), ft)
        host[:, :nb, 0], host[:, :nb, 1] = X.real, X.imag
        b0, b1 = torch.from_numpy(host).cuda(), None
    else:
        re, im = np.zeros((nf, stride), ft), np.zeros((nf, stride), ft)
        re[:, :nb], im[:, :nb] = X.real, X.imag
        b0, b1 = torch.from_numpy(re).cuda(), torch.from_numpy(im).cuda()
    th = torch.from_numpy(np.stack([filt.real, filt.imag], -1).astype(ft)).cuda() if filt is not None else None
    tw = torch.from_numpy(np.asarray(win, ft)).cuda() if win is not None else None
    sig = torch.full(((nf - 1) * hop + n,), float("nan"), dtype=tdt, device="cuda")  # every real is written
    plan.istft(layout, b0.data_ptr(), b1.data_ptr() if b1 is not None else None, hop, nf, sig.data_ptr(),
               filter=th.data_ptr() if th is not None else None, window=tw.data_ptr() if tw is not None else None,
               in_stride=in_stride)
    torch.cuda.synchronize()
    assert plan.device_status() == 0
    return sig.cpu().numpy()


def _hann(n, ft):
    return (0.5 - 0.5 * np.cos(2 * np.pi * np.arange(n) / n)).astype(ft)


@pytest.mark.parametrize("order,hop,nf", [(12, 1024, 40), (12, 2048, 7), (12, 4096, 5), (10, 256, 300),
                                          (14, 4096, 9), (11, 2, 3), (13, 1024, 1), (10, 512, 2000)])
def test_istft_f32_bit_exact(oracle, order, hop, nf):
    n = 1 << order
    rng = np.random.default_rng(1200 + order + hop)
    X = _bins(rng, nf, n, np.complex64)
    H = _bins(rng, 1, n, np.complex64)[0]
    win = _hann(n, np.float32)
    plan = Z.Plan(Z.R2C, order, np.float32)
    for filt, w in ((None, None), (H, None), (None, win), (H, win)):
        want = oracle.istft_port(X, hop, filt, w)
        for layout in (Z.AOS, Z.SOA):
            got = _run(plan, X, hop, filt, w, layout)
            assert np.array_equal(got, want), (order, hop, nf, filt is not None, w is not None, layout)
    # against FP64: the per-frame RFFT bar, scaled by the frames that overlap
    ref = oracle.istft_fp64(X, hop, H, win)
    got = _run(plan, X, hop, H, win)
    k = n // hop
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert err <= k * oracle.tolerance(order, "f32"), err


@pytest.mark.parametrize("order,hop,nf", [(12, 1024, 33), (10, 1024, 4), (13, 2048, 20)])
def test_istft_f64(oracle, order, hop, nf):
    """FP64 (whose RFFT backward is held to the FP64 oracle's bar, not to the
    port's bits): the fused launch equals the library's own batched RFFT
    backward of the filtered bins, windowed and overlap-added frame by frame,
    bit for bit, and the FP64 oracle within the bar."""
    n = 1 << order
    rng = np.random.default_rng(1300 + order)
    X = _bins(rng, nf, n, np.complex128)
    H = _bins(rng, 1, n, np.complex128)[0]
    win = _hann(n, np.float64)
    plan = Z.Plan(Z.R2C, order, np.float64)
    Y = np.empty_like(X)
    Y.real = X.real * H.real - X.imag * H.imag
    Y.imag = X.real * H.imag + X.imag * H.real
    x = G.run_c2r(plan, Y) * win[None, :]
    want = np.zeros((nf - 1) * hop + n)
    for f in range(nf):
        want[f * hop:f * hop + n] += x[f]
    for layout in (Z.AOS, Z.SOA):
        assert np.array_equal(_run(plan, X, hop, H, win, layout), want), layout
    ref = oracle.istft_fp64(X, hop, H, win)
    err = np.linalg.norm(want - ref) / np.linalg.norm(ref)
    assert err <= (n // hop) * oracle.tolerance(order, "f64")


def test_istft_strided_bins(oracle):
    order, hop, nf = 11, 512, 23
    n = 1 << order
    rng = np.random.default_rng(1401)
    X = _bins(rng, nf, n, np.complex64)
    plan = Z.Plan(Z.R2C, order, np.float32)
    got = _run(plan, X, hop, None, _hann(n, np.float32), Z.AOS, in_stride=n // 2 + 9)
    assert np.array_equal(got, oracle.istft_port(X, hop, None, _hann(n, np.float32)))


def test_istft_inverts_stft(oracle):
    """STFT (Hann, hop N/4) then inverse STFT (Hann): the signal times
    (N/2) * sum of squared windows (= 3N/4 at hop N/4), away from the edges."""
    import torch
    order, hop, nf = 12, 1024, 64
    n = 1 << order
    rng = np.random.default_rng(1402)
    sig = rng.uniform(-1, 1, (nf - 1) * hop + n).astype(np.float32)
    win = _hann(n, np.float32)
    plan = Z.Plan(Z.R2C, order, np.float32)
    ts, tw = torch.from_numpy(sig).cuda(), torch.from_numpy(win).cuda()
    bins = torch.zeros((nf, n // 2 + 1, 2), dtype=torch.float32, device="cuda")
    plan.stft(Z.FORWARD, Z.AOS, ts.data_ptr(), hop, tw.data_ptr(), bins.data_ptr(), None, nf)
    out = torch.zeros_like(ts)
    plan.istft(Z.AOS, bins.data_ptr(), None, hop, nf, out.data_ptr(), window=tw.data_ptr())
    torch.cuda.synchronize()
    y = out.cpu().numpy()
    mid = slice(n, len(sig) - n)
    gain = (n / 2) * 1.5
    assert np.abs(y[mid] / gain - sig[mid]).max() < 1e-4


def test_istft_errors():
    import torch
    p = Z.Plan(Z.R2C, 12, np.float32)
    b = torch.zeros((4, 2049, 2), device="cuda")
    s = torch.zeros(8192, device="cuda")
    for hop in (0, 3, 1000, 8192):  # odd, not dividing N, larger than N
        with pytest.raises(Z.ZlfftError):
            p.istft(Z.AOS, b.data_ptr(), None, hop, 4, s.data_ptr())
    with pytest.raises(Z.ZlfftError):  # frame order 9: outside the kernel's range
        Z.Plan(Z.R2C, 9, np.float32).istft(Z.AOS, b.data_ptr(), None, 128, 4, s.data_ptr())
    with pytest.raises(Z.ZlfftError):  # a CFFT plan
        Z.Plan(Z.C2C, 12, np.float32).istft(Z.AOS, b.data_ptr(), None, 1024, 4, s.data_ptr())
    p.istft(Z.AOS, b.data_ptr(), None, 1024, 0, s.data_ptr())  # no frames: nothing to do


@pytest.mark.parametrize("order,hop,nf,slices", [(12, 1024, 1021, 8), (10, 128, 300, 7), (11, 2048, 50, 4),
                                                 (12, 512, 40, 13)])
def test_istft_slices_reassemble_bit_exact(order, hop, nf, slices):
    """Host-copy pipelining: slice [f0, f1) launched on frames
    [f0 - K + 1, f1) into its own buffer holds final sums for its blocks
    [f0, f1) (plus the tail, for the last slice). Copying only those back
    rebuilds the single launch's signal bit for bit, whatever the cuts."""
    import torch
    n = 1 << order
    k = n // hop
    rng = np.random.default_rng(1500 + order + hop)
    X = _bins(rng, nf, n, np.complex64)
    H = _bins(rng, 1, n, np.complex64)[0]
    win = _hann(n, np.float32)
    plan = Z.Plan(Z.R2C, order, np.float32)
    whole = _run(plan, X, hop, H, win)
    host = np.zeros((nf, n // 2 + 1, 2), np.float32)
    host[..., 0], host[..., 1] = X.real, X.imag
    tb = torch.from_numpy(host).cuda()
    th = torch.from_numpy(np.stack([H.real, H.imag], -1).astype(np.float32)).cuda()
    tw = torch.from_numpy(win).cuda()
    total = (nf - 1) * hop + n
    out = np.full(total, np.nan, np.float32)
    cuts = sorted(set([0, nf] + list(rng.integers(1, nf, slices - 1))))
    for f0, f1 in zip(cuts[:-1], cuts[1:]):
        g0 = max(0, f0 - k + 1)
        buf = torch.full(((f1 - g0 - 1) * hop + n,), float("nan"), dtype=torch.float32, device="cuda")
        plan.istft(Z.AOS, tb[g0].data_ptr(), None, hop, f1 - g0, buf.data_ptr(), filter=th.data_ptr(),
                   window=tw.data_ptr())
        torch.cuda.synchronize()
        a, b = f0 * hop, (total if f1 == nf else f1 * hop)
        out[a:b] = buf[a - g0 * hop:b - g0 * hop].cpu().numpy()
    assert plan.device_status() == 0
    assert np.array_equal(out, whole), (order, hop, cuts)
