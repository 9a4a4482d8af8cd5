"""GPU parity tests: the CUDA BorderedCR path, called through the C ABI, against
the reference's own results (golden fixtures) and the CPU oracle.

Tolerances (floating point): forward error against the reference/oracle
solution <= 1e-10 on these well-conditioned systems, and relative residual
||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf) <= 1e-13 for the FP64 path.
"""
import numpy as np
import pytest

from alglin_b200 import bcr as B
from alglin_b200 import synth
from oracle import pyoracle as po
from tests._util import GOLDEN_CASES, block_norm_inf, fwd_err, load_golden

pytestmark = pytest.mark.gpu

DEVICE_LAST = ("LU", "LUPQ", "QR", "QRP", "SVD", "LSS", "LSY", "PINV")  # all on the device


def gpu_solver(s, internal="LU", last="LU", last2="NONE"):
    h = B.BorderedCR()
    h.load_system(s)
    h.select(internal)
    h.select_last(last)
    h.select_last2(last2)
    return h


def gpu_solve(h, b):
    X = np.array(b, dtype=np.float64, order="C", copy=True)
    if X.ndim == 1:
        assert h.solve(X), h.last_error()
    else:
        assert h.solve_n(X.shape[0], X, X.shape[1]), h.last_error()
    return X


def relres(o, s, x, b):
    r = b[:s.nrows] - o.mv(x[:s.ncols])
    return np.abs(r).max() / (block_norm_inf(s) * np.abs(x[:s.ncols]).max() + np.abs(b[:s.nrows]).max())


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_gpu_matches_reference_golden(name):
    s, b, X, tags = load_golden(name)
    ran = 0
    for (internal, last, last2), xg in zip(tags, X):
        if last not in DEVICE_LAST:
            continue
        h = gpu_solver(s, internal, last, last2)
        assert h.factorize(), h.last_error()
        x = gpu_solve(h, b)
        for c in range(b.shape[0]):
            assert fwd_err(x[c, :s.ncols], xg[c, :s.ncols]) < 1e-10, (name, internal, last, c)
        ran += 1
    assert ran > 0


SHAPES = [
    (1, 1, 0, 0, 0, 0), (1, 2, 0, 0, 1, 1), (2, 1, 0, 0, 1, 1), (3, 2, 1, 1, 1, 1),
    (5, 3, 0, 2, 2, 0), (8, 4, 2, 2, 3, 3), (33, 5, 1, 0, 0, 2), (100, 8, 0, 0, 2, 2),
    (127, 16, 2, 2, 4, 4), (64, 32, 0, 0, 8, 8), (257, 7, 3, 1, 2, 5), (1000, 2, 0, 0, 0, 0),
    (40, 20, 1, 1, 2, 2), (33, 24, 0, 0, 4, 4), (70, 32, 2, 1, 3, 4),
]


@pytest.mark.parametrize("dims", SHAPES)
@pytest.mark.parametrize("internal", ["LU", "QR", "QRP"])
def test_gpu_matches_oracle_random(dims, internal):
    s = synth.collocation(*dims, seed=sum(dims)) if dims[1] > 1 else synth.dominant(*dims, seed=1)
    b = synth.rhs(s, nrhs=2, seed=7)
    last = "LU" if s.Nr == s.Nc else ("QR" if s.Nr > s.Nc else "PINV")
    o = po.Oracle(s, internal, last)
    assert o.factorize(), o.last_error()
    xo = o.solve(b)
    h = gpu_solver(s, internal, last)
    assert h.factorize(), h.last_error()
    xg = gpu_solve(h, b)
    for c in range(2):
        assert fwd_err(xg[c, :s.ncols], xo[c, :s.ncols]) < 1e-10, (dims, internal, c)
        assert relres(o, s, xg[c], b[c]) < 1e-13
    # single right-hand side entry point
    x1 = gpu_solve(h, b[0])
    assert fwd_err(x1[:s.ncols], xo[0, :s.ncols]) < 1e-10


def test_gpu_many_rhs_chunks():
    s = synth.collocation(77, 6, 1, 1, 2, 2, seed=9)
    b = synth.rhs(s, nrhs=37, seed=3)
    o = po.Oracle(s, "LU", "LU"); assert o.factorize()
    h = gpu_solver(s); assert h.factorize(), h.last_error()
    xg = gpu_solve(h, b)
    xo = o.solve(b)
    assert fwd_err(xg[:, :s.ncols], xo[:, :s.ncols]) < 1e-10


def test_gpu_mv_matches_oracle():
    s = synth.collocation(513, 8, 2, 2, 3, 3, seed=4)
    x = np.random.default_rng(0).standard_normal(s.ncols)
    o = po.Oracle(s)
    h = gpu_solver(s)
    y = h.mv(x)
    yo = o.mv(x)
    assert np.abs(y[:s.nrows] - yo).max() < 1e-12 * np.abs(yo).max()
    r = np.ones(s.nrows)
    h.add_mv(-2.0, x, r)
    assert np.abs(r - (1 - 2 * yo)).max() < 1e-12 * np.abs(yo).max()


def test_gpu_manufactured_test7_style():
    """src_tests/test7-BorderedCR.cc:120-288 sizes and checks."""
    s = synth.dominant(10000, 8, 4, 4, 1, 1, seed=2)
    xref = 1.0 + (np.arange(s.ncols) % 100)
    h = gpu_solver(s)
    rhs = np.zeros(max(s.nrows, s.ncols))
    rhs[:s.nrows] = h.mv(xref)
    assert h.factorize(), h.last_error()
    x = rhs.copy()
    assert h.solve(x)
    assert np.abs(x[:s.ncols] - xref).max() < 1e-8
    assert np.abs(x[:s.ncols] - xref).sum() / s.ncols < 1e-8
    X = np.stack([rhs, rhs])
    assert h.solve_n(2, X, X.shape[1])
    assert np.abs(X[:, :s.ncols] - xref).max() < 1e-8
    res = h.mv(x[:s.ncols]) - rhs[:s.nrows]
    assert np.linalg.norm(res) < 1e-6 and np.abs(res).sum() < 1e-6


def test_gpu_singular_panel_fails_like_reference():
    s = synth.dominant(4, 3, 0, 0, 0, 0, seed=1)
    s.D[1] = 0.0
    s.E[0] = 0.0
    h = gpu_solver(s)
    assert not h.factorize()
    assert "getrf(M=6,N=3,A,LDA=6,iperm)::INFO = 1" in h.last_error()


def test_gpu_singular_last_block_without_fallback():
    s = synth._zeros(1, 1, 0, 0, 1, 1)
    s.D[0, 0, 0] = 1; s.H[1, 0] = 1; s.C[0, 0, 0] = 1; s.C[1, 0, 0] = 1
    h = gpu_solver(s, "LU", "LU", "NONE")
    assert not h.factorize()
    assert "load_and_factorize_last" in h.last_error()


def test_gpu_deterministic():
    s = synth.collocation(999, 16, 2, 2, 4, 4, seed=1)
    b = synth.rhs(s, 1, seed=2)[0]
    h = gpu_solver(s)
    assert h.factorize()
    x1 = gpu_solve(h, b)
    assert h.factorize()
    x2 = gpu_solve(h, b)
    assert np.array_equal(x1, x2)


def _reference_solution(s, b, internal="LU"):
    """The reference BorderedCR's own solution (oracle/_ref, its thread pool)
    and the object that keeps the unfactored matrix for its Mv."""
    import os
    th = os.cpu_count() or 1
    src = po.RefBCR(s, internal, "LU", "NONE", nthreads=th, npb=th)
    work = po.RefBCR(s, internal, "LU", "NONE", nthreads=th, npb=th)
    work.set_threads(True, True)
    _, x = work.time_factor_solve(src, b)
    return x, src


def _ref_relres(src, s, x, b):
    r = b[:s.nrows] - src.mv(x[:s.ncols])
    return np.abs(r).max() / (block_norm_inf(s) * np.abs(x[:s.ncols]).max() + np.abs(b[:s.nrows]).max())


@pytest.mark.parametrize("internal", ["LU", "QR"])
def test_gpu_full_size_config_B_vs_reference(internal):
    """n=16, nblock=100000, qr=qx=2, nr=nx=4, the same seeded system as the
    benchmark: forward error against the reference BorderedCR's solution
    <= 1e-10 and relative residual with the reference's Mv <= 1e-13 (FP64)."""
    if not po.ref_available():
        pytest.skip("oracle/_ref not built")
    s = synth.collocation(**synth.CONFIGS["B"], seed=0)
    b = synth.rhs(s, nrhs=1, seed=1)[0]
    xr, src = _reference_solution(s, b, internal)
    h = gpu_solver(s, internal, "LU")
    assert h.factorize(), h.last_error()
    x = gpu_solve(h, b)
    assert fwd_err(x[:s.ncols], xr[:s.ncols]) < 1e-10
    assert _ref_relres(src, s, x, b) < 1e-13


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gpu_full_size_config_E_vs_reference(precision):
    """n=128, nblock=8192, qr=qx=4, nr=nx=16 (the tensor-core configuration):
    the FP64 path to rel. residual <= 1e-13, the mixed path (tcgen05 FP32
    products + FP64 refinement) to <= 1e-12, both with the reference's Mv, and
    the forward error against the reference BorderedCR's solution (<= 1e-10
    FP64; the mixed path's stays within cond(A) * 1e-12 of it: <= 1e-6)."""
    if not po.ref_available():
        pytest.skip("oracle/_ref not built")
    s = synth.collocation(**synth.CONFIGS["E"], seed=0)
    b = synth.rhs(s, nrhs=1, seed=1)[0]
    xr, src = _reference_solution(s, b)
    h = gpu_solver(s)
    if precision == "mixed":
        h.set_precision(B.PRECISION_MIXED)
    assert h.factorize(), h.last_error()
    x = gpu_solve(h, b)
    rel = _ref_relres(src, s, x, b)
    fe = fwd_err(x[:s.ncols], xr[:s.ncols])
    if precision == "fp64":
        assert rel < 1e-13 and fe < 1e-10, (rel, fe)
    else:
        assert rel < 1e-12 and fe < 1e-6, (rel, fe)


@pytest.mark.parametrize("dims,internal,nrhs", [
    ((1000, 16, 2, 2, 4, 4), "LU", 1), ((1000, 16, 2, 2, 4, 4), "LU", 4),
    ((777, 8, 0, 0, 2, 2), "LU", 3), ((300, 16, 2, 2, 4, 4), "LU", 6),
    ((129, 16, 1, 1, 3, 2), "QR", 2), ((65, 5, 1, 1, 2, 2), "LU", 2)])
def test_gpu_factorize_solve_fused(dims, internal, nrhs):
    """factorize+solve in one pass (forward elimination fused into the pair
    kernel where it fits) gives the oracle's answer, and the stored factors
    still serve a later plain solve."""
    s = synth.collocation(*dims, seed=21)
    b = synth.rhs(s, nrhs=nrhs, seed=5)
    last = "LU" if s.Nr == s.Nc else "QR"
    o = po.Oracle(s, internal, last)
    assert o.factorize(), o.last_error()
    xo = o.solve(b)
    h = gpu_solver(s, internal, last)
    X = b.copy()
    assert h.factorize_solve(nrhs, X, X.shape[1]), h.last_error()
    assert fwd_err(X[:, :s.ncols], xo[:, :s.ncols]) < 1e-10
    x2 = gpu_solve(h, b)
    assert fwd_err(x2[:, :s.ncols], xo[:, :s.ncols]) < 1e-10


@pytest.mark.parametrize("dims", [(65, 32, 0, 0, 8, 8), (17, 48, 2, 3, 4, 1), (9, 64, 1, 1, 2, 2),
                                  (5, 128, 4, 4, 16, 16), (12, 40, 0, 0, 3, 3), (6, 100, 2, 2, 5, 5),
                                  (7, 27, 1, 1, 2, 2)])
@pytest.mark.parametrize("internal", ["LU", "QR", "QRP"])
def test_gpu_large_blocks(dims, internal):
    """n > 24 runs one CTA per pair with the work matrix in a global slab
    (blocked LU in panels of 32 columns; config C has n=32, config E n=128);
    n = 27, 40 and 100 leave a partial last panel block."""
    s = synth.collocation(*dims, seed=sum(dims))
    b = synth.rhs(s, nrhs=2, seed=3)
    last = "LU" if s.Nr == s.Nc else "QR"
    o = po.Oracle(s, internal, last)
    assert o.factorize(), o.last_error()
    xo = o.solve(b)
    h = gpu_solver(s, internal, last)
    assert h.factorize(), h.last_error()
    xg = gpu_solve(h, b)
    for c in range(2):
        assert fwd_err(xg[c, :s.ncols], xo[c, :s.ncols]) < 1e-9, (dims, internal, c)
        if s.nrows == s.ncols:  # rectangular last blocks are least-squares solves
            assert relres(o, s, xg[c], b[c]) < 1e-13


FAMILIES = {"tc": B.PAIR_TC, "grp": B.PAIR_GRP, "rows": B.PAIR_ROWS, "cta": B.PAIR_CTA, "smem": B.PAIR_SMEM}


@pytest.mark.parametrize("dims", [(129, 16, 2, 2, 4, 4), (97, 32, 0, 0, 8, 8), (64, 32, 2, 1, 3, 4),
                                  (33, 16, 0, 0, 8, 8), (50, 8, 0, 0, 2, 2)])
@pytest.mark.parametrize("family", list(FAMILIES))
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gpu_pair_kernel_families(dims, family, precision):
    """Every pair-kernel family, forced, gives the oracle's solution."""
    s = synth.collocation(*dims, seed=sum(dims) + 5)
    b = synth.rhs(s, nrhs=1, seed=3)
    o = po.Oracle(s, "LU", "LU")
    assert o.factorize(), o.last_error()
    xo = o.solve(b)
    h = gpu_solver(s, "LU", "LU")
    h.set_pair_kernel(FAMILIES[family])
    if precision == "mixed":
        h.set_precision(B.PRECISION_MIXED)
    assert h.factorize(), h.last_error()
    x = gpu_solve(h, b)
    assert fwd_err(x[0, :s.ncols], xo[0, :s.ncols]) < (1e-10 if precision == "fp64" else 1e-8)
    bar = 1e-13 if precision == "fp64" else 1e-12
    assert relres(o, s, x[0], b[0]) <= bar


@pytest.mark.parametrize("last", ["LU", "LUPQ", "QR", "QRP", "SVD", "LSS", "LSY", "PINV"])
@pytest.mark.parametrize("dims", [(40, 6, 1, 1, 2, 2), (17, 16, 2, 2, 4, 4), (9, 3, 0, 2, 1, 0)])
def test_gpu_last_block_solvers(dims, last):
    """Every last-block solver against the oracle (square, and the
    under-determined shape for the SVD family: minimum-norm solution)."""
    s = synth.collocation(*dims, seed=sum(dims) + 3)
    if s.Nr != s.Nc and last in ("LU", "LUPQ"):
        pytest.skip("LU and LUPQ need a square last block")
    if s.Nr < s.Nc and last in ("QR", "QRP"):
        pytest.skip("QR and QRP need Nr >= Nc")
    b = synth.rhs(s, nrhs=2, seed=4)
    o = po.Oracle(s, "LU", last)
    assert o.factorize(), o.last_error()
    xo = o.solve(b)
    h = gpu_solver(s, "LU", last)
    assert h.factorize(), h.last_error()
    xg = gpu_solve(h, b)
    for c in range(2):
        assert fwd_err(xg[c, :s.ncols], xo[c, :s.ncols]) < 1e-9, (last, c)


@pytest.mark.parametrize("last2", ["SVD", "LSS", "LSY", "PINV"])
def test_gpu_last_block_fallback(last2):
    """test18-BorderedCR-coverage.cc:1061-1098: a singular last block is
    solved by the select_last2 solver (minimum-norm solution)."""
    s = synth._zeros(1, 1, 0, 0, 1, 1)
    s.D[0, 0, 0] = 1; s.H[1, 0] = 1; s.C[0, 0, 0] = 1; s.C[1, 0, 0] = 1
    h = gpu_solver(s, "LU", "LU", last2)
    assert h.factorize(), h.last_error()
    o = po.Oracle(s, "LU", "LU", last2)
    assert o.factorize()
    xref = np.array([2.0, -1.0, 0.0])
    b = np.zeros((1, 3))
    b[0] = o.mv(xref)
    xg = gpu_solve(h, b)[0]
    xo = o.solve(b)[0]
    assert np.abs(xg - xo).max() < 1e-12
    assert np.abs(xg - xref).max() < 5e-9


def test_gpu_fallback_not_used_when_primary_succeeds():
    s = synth.collocation(33, 8, 0, 0, 2, 2, seed=8)
    b = synth.rhs(s, nrhs=1, seed=2)
    h1 = gpu_solver(s, "LU", "LU", "NONE")
    h2 = gpu_solver(s, "LU", "LU", "PINV")
    assert h1.factorize() and h2.factorize()
    assert np.array_equal(gpu_solve(h1, b), gpu_solve(h2, b))


@pytest.mark.parametrize("dims", [(6, 30, 2, 2, 1, 1), (6, 31, 1, 1, 1, 1), (9, 40, 3, 3, 4, 4),
                                  (5, 128, 4, 4, 16, 16)])
def test_gpu_blocked_last_block_lu(dims):
    """Last blocks of order 64 and above are factored by the blocked LU (rows
    left in place); 63 stays on the unblocked one: both against the oracle."""
    s = synth.collocation(*dims, seed=sum(dims) + 7)
    assert s.Nr == s.Nc
    b = synth.rhs(s, nrhs=2, seed=6)
    o = po.Oracle(s, "LU", "LU")
    assert o.factorize(), o.last_error()
    xo = o.solve(b)
    h = gpu_solver(s, "LU", "LU")
    assert h.factorize(), h.last_error()
    xg = gpu_solve(h, b)
    for c in range(2):
        assert fwd_err(xg[c, :s.ncols], xo[c, :s.ncols]) < 1e-10
        assert relres(o, s, xg[c], b[c]) <= 1e-13


def test_gpu_blocked_last_block_singular_falls_back():
    """A singular last block of order 66 (zero boundary rows): LU reports it, and
    with select_last2 the minimum-norm solution matches the oracle's."""
    s = synth.collocation(9, 32, 0, 0, 2, 2, seed=5)
    s.H[:] = 0.0
    assert s.Nr == 66
    h = gpu_solver(s, "LU", "LU", "NONE")
    assert not h.factorize()
    assert "load_and_factorize_last" in h.last_error()
    o = po.Oracle(s, "LU", "LU", "PINV")
    assert o.factorize(), o.last_error()
    xref = synth.rhs(s, nrhs=1, seed=9)[0][:s.ncols]
    b = np.zeros((1, s.nrows))
    b[0] = o.mv(xref)
    xo = o.solve(b)[0]
    h2 = gpu_solver(s, "LU", "LU", "PINV")
    assert h2.factorize(), h2.last_error()
    xg = gpu_solve(h2, b)[0]
    assert fwd_err(xg[:s.ncols], xo[:s.ncols]) < 1e-8


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gpu_singular_panel_large_blocks(precision):
    """A zero first column in the panel of pair (0, 1) at n=40: the blocked FP64
    kernel and the FP32 tensor-core kernel both stop with getrf's INFO = 1."""
    s = synth.collocation(6, 40, 0, 0, 2, 2, seed=1)
    s.E[0][0, :] = 0.0  # column 0 (blocks are held column by column)
    s.D[1][0, :] = 0.0
    h = gpu_solver(s)
    if precision == "mixed":
        h.set_precision(B.PRECISION_MIXED)
    assert not h.factorize()
    assert "getrf(M=80,N=40,A,LDA=80,iperm)::INFO = 1" in h.last_error()
    # the handle recovers: a regular system factors afterwards
    s2 = synth.collocation(6, 40, 0, 0, 2, 2, seed=2)
    h2 = gpu_solver(s2)
    if precision == "mixed":
        h2.set_precision(B.PRECISION_MIXED)
    assert h2.factorize(), h2.last_error()
