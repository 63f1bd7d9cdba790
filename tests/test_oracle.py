"""Pins the oracle before anything is checked against it (CPU only).

1. The C restatement reproduces the reference's golden outputs bit for bit
   (fixtures made from the reference's own code, tests/golden/make_golden.py).
2. Where the shim-built reference library is present, the restatement equals
   it bit for bit on fresh seeded inputs, orders 0..18.
3. Both agree with an independent FP64 FFT (numpy) within 4*log2(N)*eps.
4. Analytic known answers: impulse, constant, single tone, round-trip scale,
   Hermitian symmetry and Parseval.
"""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PRECS = [("f32", np.float32, np.complex64), ("f64", np.float64, np.complex128)]


def _golden(prec):
    return np.load(os.path.join(GOLDEN, f"reference_{prec}.npz"))


@pytest.mark.parametrize("prec,ft,ct", PRECS)
def test_port_matches_reference_golden_cfft(oracle, prec, ft, ct):
    g = _golden(prec)
    for order in range(0, 11):
        x = g[f"c2c_{order}_in"]
        assert np.array_equal(oracle.cfft_port(x, True), g[f"c2c_{order}_fwd"]), order
        assert np.array_equal(oracle.cfft_port(x, False), g[f"c2c_{order}_bwd"]), order


@pytest.mark.parametrize("prec,ft,ct", PRECS)
def test_port_matches_reference_golden_rfft(oracle, prec, ft, ct):
    g = _golden(prec)
    for order in range(1, 12):
        x = g[f"r2c_{order}_in"]
        assert np.array_equal(oracle.rfft_forward_port(x), g[f"r2c_{order}_fwd"]), order
        assert np.array_equal(oracle.rfft_forward_port(x, sqr_mag=True), g[f"r2c_{order}_sqr"]), order
        assert np.array_equal(oracle.rfft_backward_port(g[f"r2c_{order}_bins"]), g[f"r2c_{order}_bwd"]), order


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(GOLDEN), "..", "oracle", "_ref",
                                                    "libzlref.so")), reason="shim-built reference not present")
@pytest.mark.parametrize("prec,ft,ct", PRECS)
def test_port_bitwise_equals_reference_library(oracle, prec, ft, ct):
    rng = np.random.default_rng(99)
    _, switch = oracle.ref_switch_order(prec)
    for order in range(0, 19):
        n = 1 << order
        b = 2 if order < 15 else 1
        x = (rng.uniform(-1, 1, (b, n)) + 1j * rng.uniform(-1, 1, (b, n))).astype(ct)
        if order < switch:  # the reference's micro-only path (its macro path rounds differently)
            plan = oracle.RefPlan("c2c", order, prec)
            for fwd in (True, False):
                assert np.array_equal(oracle.cfft_port(x, fwd), plan.cfft(x, fwd)), (order, fwd)
            # every layout pairing of the reference gives the same values
            re, im = np.ascontiguousarray(x.real), np.ascontiguousarray(x.imag)
            ref_aos = plan.cfft(x, True)
            for il, inp in ((oracle.AOS, x), (oracle.SOA, (re, im))):
                for ol in (oracle.AOS, oracle.SOA):
                    y = plan.cfft(inp, True, il, ol)
                    y = y if ol == oracle.AOS else (y[0] + 1j * y[1]).astype(ct)
                    assert np.array_equal(y, ref_aos), (order, il, ol)
            plan.close()
        if order >= 1 and order - 1 < switch:
            xr = rng.uniform(-1, 1, (b, n)).astype(ft)
            plan = oracle.RefPlan("r2c", order, prec)
            X = plan.rfft_forward(xr)
            assert np.array_equal(oracle.rfft_forward_port(xr), X), order
            assert np.array_equal(oracle.rfft_forward_port(xr, True), plan.rfft_forward(xr, sqr_mag=True)), order
            assert np.array_equal(oracle.rfft_backward_port(X), plan.rfft_backward(X)), order
            plan.close()


@pytest.mark.parametrize("prec,ft,ct", PRECS)
def test_port_within_fp64_tolerance(oracle, prec, ft, ct):
    rng = np.random.default_rng(5)
    for order in range(0, 17):
        n = 1 << order
        x = (rng.uniform(-1, 1, (2, n)) + 1j * rng.uniform(-1, 1, (2, n))).astype(ct)
        tol = oracle.tolerance(order, prec)
        for fwd in (True, False):
            err = oracle.rel_l2(oracle.cfft_port(x, fwd), oracle.cfft_fp64(x, fwd)).max()
            assert err <= tol, (order, fwd, err, tol)
        if order >= 1:
            xr = rng.uniform(-1, 1, (2, n)).astype(ft)
            X = oracle.rfft_forward_port(xr)
            assert oracle.rel_l2(X, oracle.rfft_fp64(xr)).max() <= tol
            P = oracle.rfft_forward_port(xr, sqr_mag=True)
            assert oracle.rel_l2(P, np.abs(oracle.rfft_fp64(xr)) ** 2).max() <= 2 * tol
            back = oracle.rfft_backward_port(X)
            assert oracle.rel_l2(back, oracle.rfft_backward_fp64(X)).max() <= tol


@pytest.mark.parametrize("prec,ft,ct", PRECS)
def test_known_answers(oracle, prec, ft, ct):
    for order in (0, 1, 2, 3, 4, 5, 8, 11):
        n = 1 << order
        # impulse -> constant 1
        x = np.zeros((1, n), ct)
        x[0, 0] = 1
        assert np.array_equal(oracle.cfft_port(x, True), np.ones((1, n), ct))
        # constant -> N at bin 0
        y = oracle.cfft_port(np.ones((1, n), ct), True)
        assert abs(y[0, 0] - n) <= 1e-6 * n and np.abs(y[0, 1:]).max(initial=0) <= 1e-5 * n
        # single tone at bin k -> N at k
        k = (3 * n) // 7 if n > 1 else 0
        t = np.exp(2j * np.pi * ((k * np.arange(n)) % n) / n).astype(ct)[None, :]  # exact phase reduction
        y = oracle.cfft_port(t, True)
        expect = np.zeros((1, n), np.complex128)
        expect[0, k] = n
        assert oracle.rel_l2(y, expect).max() <= 4 * oracle.tolerance(order, prec) + 1e-15
        # round trip: backward(forward(x)) = N x
        rng = np.random.default_rng(order)
        z = (rng.uniform(-1, 1, (1, n)) + 1j * rng.uniform(-1, 1, (1, n))).astype(ct)
        rt = oracle.cfft_port(oracle.cfft_port(z, True), False)
        assert oracle.rel_l2(rt, n * z.astype(np.complex128)).max() <= 2 * oracle.tolerance(order, prec)
        # Parseval: sum |X|^2 = N sum |x|^2
        X = oracle.cfft_port(z, True).astype(np.complex128)
        assert abs(np.sum(np.abs(X) ** 2) - n * np.sum(np.abs(z.astype(np.complex128)) ** 2)) <= \
            8 * oracle.tolerance(order, prec) * n * np.sum(np.abs(z) ** 2) + 1e-12
    for order in (1, 2, 3, 6, 9, 12):
        n = 1 << order
        rng = np.random.default_rng(order + 100)
        xr = rng.uniform(-1, 1, (1, n)).astype(ft)
        X = oracle.rfft_forward_port(xr)
        assert X[0, 0].imag == 0 and X[0, -1].imag == 0  # DC and Nyquist are real
        back = oracle.rfft_backward_port(X)  # RFFT round trip scales by N/2
        assert oracle.rel_l2(back, (n / 2) * xr.astype(np.float64)).max() <= 2 * oracle.tolerance(order, prec)
        # real input: the N/2+1 bins equal the first half of the complex FFT (Hermitian)
        full = oracle.cfft_fp64(xr.astype(np.complex128))
        assert oracle.rel_l2(X, full[:, : n // 2 + 1]).max() <= oracle.tolerance(order, prec)


def test_twiddle_table_matches_reference_formula(oracle):
    # T[t] = (F)cos(-2 pi t / N) etc., computed as the reference does (cos(a*pi) in double)
    for order in (2, 5, 10, 16):
        n = 1 << order
        t = np.arange(3 * n // 4)
        a = t * (-2.0 / n)
        for prec, ct in (("f32", np.complex64), ("f64", np.complex128)):
            T = oracle.twiddles(order, prec)
            expect = (np.cos(a * np.pi) + 1j * np.sin(a * np.pi)).astype(ct)
            assert np.array_equal(T, expect)


def test_istft_port_overlap_add(oracle):
    """The sequential inverse STFT: hop = N concatenates the frames' RFFT
    backward outputs; overlapping hops stay within the FP64 oracle's bar."""
    rng = np.random.default_rng(1501)
    order, nf = 9, 6
    n = 1 << order
    X = (rng.uniform(-1, 1, (nf, n // 2 + 1)) + 1j * rng.uniform(-1, 1, (nf, n // 2 + 1))).astype(np.complex64)
    X[:, 0], X[:, -1] = X[:, 0].real, X[:, -1].real
    y = oracle.istft_port(X, n)
    assert np.array_equal(y, oracle.rfft_backward_port(X).reshape(-1))
    win = (0.5 - 0.5 * np.cos(2 * np.pi * np.arange(n) / n)).astype(np.float32)
    H = X[0]
    for hop in (n // 2, n // 4, 2):
        y = oracle.istft_port(X, hop, H, win)
        ref = oracle.istft_fp64(X, hop, H, win)
        assert y.shape == ((nf - 1) * hop + n,)
        assert np.linalg.norm(y - ref) / np.linalg.norm(ref) <= (n // hop) * oracle.tolerance(order, "f32")


def test_istft_slicing_recipe_on_the_oracle(oracle):
    """The slicing recipe for pipelining host copies with the inverse STFT,
    on the oracle's sequential overlap-add: slice [f0, f1) runs frames
    [max(0, f0 - K + 1), f1) into its own signal; its samples
    [f0 * hop, f1 * hop) (to the end, for the last slice) are final and,
    reassembled, equal one run over all frames bit for bit."""
    rng = np.random.default_rng(1502)
    order, nf = 8, 37
    n = 1 << order
    X = (rng.uniform(-1, 1, (nf, n // 2 + 1)) + 1j * rng.uniform(-1, 1, (nf, n // 2 + 1))).astype(np.complex64)
    X[:, 0], X[:, -1] = X[:, 0].real, X[:, -1].real
    win = (0.5 - 0.5 * np.cos(2 * np.pi * np.arange(n) / n)).astype(np.float32)
    for hop in (n, n // 4, n // 8):
        k = n // hop
        whole = oracle.istft_port(X, hop, X[1], win)
        total = (nf - 1) * hop + n
        for cuts in ([0, nf], [0, 1, 2, nf], [0, 5, 6, 20, 33, nf], list(range(nf + 1))):
            out = np.full(total, np.nan, np.float32)
            for f0, f1 in zip(cuts[:-1], cuts[1:]):
                g0 = max(0, f0 - k + 1)
                part = oracle.istft_port(X[g0:f1], hop, X[1], win)
                a, b = f0 * hop, (total if f1 == nf else f1 * hop)
                out[a:b] = part[a - g0 * hop:b - g0 * hop]
            assert np.array_equal(out, whole), (hop, cuts)


# ---------------------------------------------------------------- the reference's macro DIF path
# On a host with small caches the reference runs CFFTs of order >= switch_order
# as Cooley-Tukey DIF macro stages + per-segment Stockham + a digit-reversed
# transposed store (src/common/zldsp_fft_common_execute.hpp:174-272). The
# restatement follows it inside oracle.hybrid(); these tests pin it.

def _macro_golden(prec):
    return np.load(os.path.join(GOLDEN, f"reference_macro_{prec}.npz"))


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_port_macro_matches_reference_golden(oracle, prec):
    """Full vectors at the smallest macro order, and SHA-256 of the reference's
    outputs for every macro order up to 22 (float) / 21 (double), made by
    tests/golden/make_golden.py from the macro-path build of the reference."""
    import hashlib
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    g = _macro_golden(prec)
    orders = mg.MACRO_ORDERS[prec]
    sha = lambda a: hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()  # noqa: E731
    with oracle.macro_host(prec):
        o0 = orders[0]
        x = g[f"c2c_{o0}_in"]
        assert np.array_equal(oracle.cfft_port(x, True), g[f"c2c_{o0}_fwd"])
        assert np.array_equal(oracle.cfft_port(x, False), g[f"c2c_{o0}_bwd"])
        for order in orders:
            assert oracle.micro_order(order, prec) > 0, order
            x, xr, X = mg.macro_inputs(prec, order)
            got = [sha(oracle.cfft_port(x, True)), sha(oracle.cfft_port(x, False)), sha(oracle.rfft_forward_port(xr)),
                   sha(oracle.rfft_forward_port(xr, sqr_mag=True)), sha(oracle.rfft_backward_port(X))]
            assert got == list(g[f"sha_{order}"]), order


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(GOLDEN), "..", "oracle", "_ref",
                                                    "libzlref_macro.so")), reason="macro-path reference build absent")
@pytest.mark.parametrize("prec,ft,ct", PRECS)
def test_port_macro_bitwise_equals_reference_macro_library(oracle, prec, ft, ct):
    """The restatement's macro path equals the reference's, bit for bit, in every
    layout pairing: CFFT orders from the switch to 19 (both micro-order
    parities), RFFT forward / forward_sqr_mag / backward in AoS and SoA."""
    l1, switch = oracle.ref_switch_order(prec, macro=True)
    assert (l1, switch) == oracle.MACRO_HOST[prec]
    rng = np.random.default_rng(1234)
    with oracle.macro_host(prec):
        for order in range(switch - 1, 20):
            n = 1 << order
            b = 2 if order < 17 else 1
            x = (rng.uniform(-1, 1, (b, n)) + 1j * rng.uniform(-1, 1, (b, n))).astype(ct)
            plan = oracle.RefPlan("c2c", order, prec, macro=True)
            for fwd in (True, False):
                assert np.array_equal(oracle.cfft_port(x, fwd), plan.cfft(x, fwd)), (order, fwd)
            re, im = np.ascontiguousarray(x.real), np.ascontiguousarray(x.imag)
            for fwd in (True, False):
                ref_aos = plan.cfft(x, fwd)
                for il, inp in ((oracle.AOS, x), (oracle.SOA, (re, im))):
                    for ol in (oracle.AOS, oracle.SOA):
                        y = plan.cfft(inp, fwd, il, ol)
                        y = y if ol == oracle.AOS else (y[0] + 1j * y[1]).astype(ct)
                        assert np.array_equal(y, ref_aos), (order, fwd, il, ol)
            plan.close()
            xr = rng.uniform(-1, 1, (b, 2 * n)).astype(ft)
            rp = oracle.RefPlan("r2c", order + 1, prec, macro=True)
            X = rp.rfft_forward(xr)
            assert np.array_equal(oracle.rfft_forward_port(xr), X), order
            s0, s1 = rp.rfft_forward(xr, layout=oracle.SOA)
            assert np.array_equal((s0 + 1j * s1).astype(ct), X), order
            assert np.array_equal(oracle.rfft_forward_port(xr, True), rp.rfft_forward(xr, sqr_mag=True)), order
            assert np.array_equal(oracle.rfft_backward_port(X), rp.rfft_backward(X)), order
            Xs = (np.ascontiguousarray(X.real), np.ascontiguousarray(X.imag))
            assert np.array_equal(oracle.rfft_backward_port(X), rp.rfft_backward(Xs, layout=oracle.SOA)), order
            rp.close()


@pytest.mark.parametrize("prec,ft,ct", PRECS)
def test_port_macro_within_fp64_tolerance(oracle, prec, ft, ct):
    """The macro path is as accurate as the micro-only one, and a different
    rounding of the same transform (the two differ in their bits)."""
    rng = np.random.default_rng(77)
    l1, switch = oracle.MACRO_HOST[prec]
    for order in range(switch, switch + 5):
        n = 1 << order
        x = (rng.uniform(-1, 1, (1, n)) + 1j * rng.uniform(-1, 1, (1, n))).astype(ct)
        micro_only = oracle.cfft_port(x, True)
        with oracle.hybrid(prec, l1, switch):
            ym = oracle.cfft_port(x, True)
            yb = oracle.cfft_port(x, False)
            xr = rng.uniform(-1, 1, (1, 2 * n)).astype(ft)
            X = oracle.rfft_forward_port(xr)
        tol = oracle.tolerance(order, prec)
        assert oracle.rel_l2(ym, oracle.cfft_fp64(x, True)).max() <= tol
        assert oracle.rel_l2(yb, oracle.cfft_fp64(x, False)).max() <= tol
        assert oracle.rel_l2(X, oracle.rfft_fp64(xr)).max() <= oracle.tolerance(order + 1, prec)
        assert not np.array_equal(ym, micro_only)
    assert oracle.micro_order(switch, prec) == -1  # outside hybrid(): micro-only again
