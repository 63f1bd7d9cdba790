"""Generate the golden fixtures from the reference's own code.

Runs the reference headers (zldsp::fft::CFFT/RFFT, unchanged) compiled here
against the project's Highway-API shim (oracle/_ref/libzlref.so, built by
`make -C oracle ref`, which needs the reference sources) on seeded inputs and
stores inputs and outputs, so parity tests can pin the oracle and the GPU
kernels where the reference sources are not present.

    python tests/golden/make_golden.py

Inputs: complex re, im ~ U[-1, 1) and real frames ~ U[-1, 1), numpy PCG64
seeds 7000 + order. Outputs are exactly what the reference writes.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402

CFFT_ORDERS = list(range(0, 11))
RFFT_ORDERS = list(range(1, 12))
BATCH = 2


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
