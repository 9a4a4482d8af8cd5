"""Generate the golden fixtures of the BorderedCR parity tests by running the
reference's own alglin::BorderedCR<double> (compiled from the unmodified
reference sources into oracle/_ref/libbcr_ref.so, see oracle/Makefile).

    python tests/golden/make_golden.py

Each fixture stores the seeded system (reference block layout), the
right-hand sides and the reference's solutions; the tests compare the C
oracle and the GPU path against them.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from alglin_b200 import synth  # noqa: E402
from oracle import pyoracle as po  # noqa: E402

CASES = {
    # name: (system factory, [(internal, last, last2)], rhs kind)
    "coverage6": (lambda: synth.stable_small(),
                  [(i, l, "NONE") for i in ("LU", "QR", "QRP")
                   for l in ("LU", "LUPQ", "QR", "QRP", "SVD", "LSS", "LSY", "PINV")], "xref"),
    "dominant37": (lambda: synth.dominant(37, 4, 2, 3, 2, 1, seed=2),
                   [("LU", "LU", "NONE"), ("QR", "QR", "NONE"), ("QRP", "LU", "NONE")], "xref"),
    "colloc_A": (lambda: synth.collocation(1000, 8, 0, 0, 2, 2, seed=0),
                 [("LU", "LU", "NONE"), ("QR", "LU", "NONE")], "randn"),
    "colloc_B257": (lambda: synth.collocation(257, 16, 2, 2, 4, 4, seed=3),
                    [("LU", "LU", "NONE"), ("QR", "QR", "NONE"), ("QRP", "LU", "NONE")], "randn"),
    "rect7b": (lambda: synth.dominant(4, 2, 10, 1, 0, 0, seed=7),
               [("LU", "PINV", "NONE"), ("LU", "QR", "NONE")], "xref"),
}


def main():
    if not po.ref_available():
        raise SystemExit("build oracle/_ref first: make -C oracle")
    for name, (make, combos, kind) in CASES.items():
        s = make()
        L = max(s.nrows, s.ncols)
        if kind == "xref":
            xref = 1.0 + (np.arange(s.ncols) % 100)
            A = s.to_dense()
            b = np.zeros((2, L))
            b[0, :s.nrows] = A @ xref
            b[1, :s.nrows] = A @ (2 * xref - 0.1)
        else:
            b = synth.rhs(s, nrhs=2, seed=11)
        xs, tags = [], []
        for (internal, last, last2) in combos:
            r = po.RefBCR(s, internal, last, last2)
            assert r.factorize(), r.last_error()
            x = r.solve(b)
            xs.append(x)
            tags.append(f"{internal}/{last}/{last2}")
        np.savez_compressed(
            os.path.join(HERE, f"{name}.npz"),
            dims=np.array(s.dims()), D=s.D, E=s.E, B=s.B, C=s.C, Cq=s.Cq, F=s.F, H=s.H,
            b=b, x=np.stack(xs), tags=np.array(tags))
        print(name, s.dims(), len(combos), "combos")


if __name__ == "__main__":
    main()
