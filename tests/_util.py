"""Shared helpers of the BorderedCR tests."""
import os

import numpy as np

from alglin_b200 import synth

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
GOLDEN_CASES = ["coverage6", "dominant37", "colloc_A", "colloc_B257", "rect7b"]


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    nb, n, qr, qx, nr, nx = [int(v) for v in z["dims"]]
    s = synth.BABD(nb, n, qr, qx, nr, nx, D=z["D"], E=z["E"], B=z["B"], C=z["C"], Cq=z["Cq"],
                   F=z["F"], H=z["H"])
    tags = [t.split("/") for t in z["tags"]]
    return s, z["b"], z["x"], tags


def rel_residual(A_mv, x, b, normA, nrows):
    """||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf)."""
    r = b[:nrows] - A_mv(x)[:nrows]
    return np.abs(r).max() / (normA * np.abs(x).max() + np.abs(b[:nrows]).max())


def dense_norm_inf(s):
    return np.abs(s.to_dense()).sum(axis=1).max()


def block_norm_inf(s):
    """||A||_inf from the block arrays (no dense matrix)."""
    return s.norm_inf()


def fwd_err(x, xref):
    return np.abs(x - xref).max() / max(np.abs(xref).max(), 1e-300)
