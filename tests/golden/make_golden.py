"""Generate the golden fixtures from the reference's own code.

Runs the reference headers (zldsp::fft::CFFT/RFFT, unchanged) compiled here
against the project's Highway-API shim (oracle/_ref/libzlref.so, built by
`make -C oracle ref`, which needs the reference sources) on seeded inputs and
stores inputs and outputs, so parity tests can pin the oracle and the GPU
kernels where the reference sources are not present.

    python tests/golden/make_golden.py

Inputs: complex re, im ~ U[-1, 1) and real frames ~ U[-1, 1), numpy PCG64
seeds 7000 + order. Outputs are exactly what the reference writes.

reference_macro_{f32,f64}.npz come from the same reference code linked with a
sysconf() stand-in that reports a small-cache host
(oracle/_ref/libzlref_macro.so), so that the reference takes its Cooley-Tukey
DIF macro path from CFFT order 14 (float) / 13 (double). They hold the full
vectors of the smallest macro order, and for every macro order up to 22 / 21
(CFFT forward and backward; RFFT forward, forward_sqr_mag and backward of the
RFFT whose inner CFFT has that order) the SHA-256 of the reference's output
bytes on inputs regenerated from the seeds 9000 + order (complex) and
9500 + order (real): one transform each, too large to store in full.
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402

CFFT_ORDERS = list(range(0, 11))
RFFT_ORDERS = list(range(1, 12))
BATCH = 2


MACRO_ORDERS = {"f32": list(range(14, 23)), "f64": list(range(13, 22))}


def macro_inputs(prec, order):
    """Seeded inputs of the macro fixtures for CFFT order `order`: a complex
    transform, a real frame of twice its length and a bin vector for the RFFT."""
    ft, ct = (np.float32, np.complex64) if prec == "f32" else (np.float64, np.complex128)
    n = 1 << order
    rng = np.random.default_rng(9000 + order)
    x = (rng.uniform(-1, 1, (1, n)) + 1j * rng.uniform(-1, 1, (1, n))).astype(ct)
    rng = np.random.default_rng(9500 + order)
    xr = rng.uniform(-1, 1, (1, 2 * n)).astype(ft)
    X = (rng.uniform(-1, 1, (1, n + 1)) + 1j * rng.uniform(-1, 1, (1, n + 1))).astype(ct)
    return x, xr, X


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def macro_main():
    for prec in ("f32", "f64"):
        data = {}
        for i, order in enumerate(MACRO_ORDERS[prec]):
            x, xr, X = macro_inputs(prec, order)
            plan = O.RefPlan("c2c", order, prec, macro=True)
            fwd, bwd = plan.cfft(x, True), plan.cfft(x, False)
            plan.close()
            rp = O.RefPlan("r2c", order + 1, prec, macro=True)
            rf, rs, rb = rp.rfft_forward(xr), rp.rfft_forward(xr, sqr_mag=True), rp.rfft_backward(X)
            rp.close()
            if i == 0:
                data[f"c2c_{order}_in"] = x
                data[f"c2c_{order}_fwd"] = fwd
                data[f"c2c_{order}_bwd"] = bwd
            data[f"sha_{order}"] = np.array([sha(fwd), sha(bwd), sha(rf), sha(rs), sha(rb)])
        path = os.path.join(HERE, f"reference_macro_{prec}.npz")
        np.savez_compressed(path, **data)
        print(path, os.path.getsize(path), "bytes")


def main():
    for prec, ft, ct in (("f32", np.float32, np.complex64), ("f64", np.float64, np.complex128)):
        data = {}
        for order in CFFT_ORDERS:
            n = 1 << order
            rng = np.random.default_rng(7000 + order)
            x = (rng.uniform(-1, 1, (BATCH, n)) + 1j * rng.uniform(-1, 1, (BATCH, n))).astype(ct)
            plan = O.RefPlan("c2c", order, prec)
            data[f"c2c_{order}_in"] = x
            data[f"c2c_{order}_fwd"] = plan.cfft(x, True)
            data[f"c2c_{order}_bwd"] = plan.cfft(x, False)
            plan.close()
        for order in RFFT_ORDERS:
            n = 1 << order
            rng = np.random.default_rng(8000 + order)
            x = rng.uniform(-1, 1, (BATCH, n)).astype(ft)
            X = (rng.uniform(-1, 1, (BATCH, n // 2 + 1)) + 1j * rng.uniform(-1, 1, (BATCH, n // 2 + 1))).astype(ct)
            plan = O.RefPlan("r2c", order, prec)
            data[f"r2c_{order}_in"] = x
            data[f"r2c_{order}_fwd"] = plan.rfft_forward(x)
            data[f"r2c_{order}_sqr"] = plan.rfft_forward(x, sqr_mag=True)
            data[f"r2c_{order}_bins"] = X
            data[f"r2c_{order}_bwd"] = plan.rfft_backward(X)
            plan.close()
        path = os.path.join(HERE, f"reference_{prec}.npz")
        np.savez_compressed(path, **data)
        print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
    macro_main()
