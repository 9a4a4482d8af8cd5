"""GPU tests of the mixed-precision path: FP32 factors and sweeps, FP64 loaded
matrix, FP64 border accumulator F and last block, FP64 iterative refinement.

Bars: after refinement the relative residual
||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf) is <= 1e-12 (computed with
the oracle's FP64 Mv as well as reported by the library), and the forward
error against the FP64 oracle solution is <= 1e-8 on these systems (the
refinement stops at the first residual under the bar, so the forward error is
about cond(A) * 1e-13 rather than the FP64 path's cond(A) * 1e-16).
"""
import numpy as np
import pytest

from alglin_b200 import bcr as B
from alglin_b200 import synth
from oracle import pyoracle as po
from tests._util import block_norm_inf, fwd_err

pytestmark = pytest.mark.gpu

RELRES_BAR = 1e-12
FWD_BAR = 1e-8


def mixed_solver(s, internal="LU", last="LU", tol=1e-12, max_iter=10):
    h = B.BorderedCR()
    h.load_system(s)
    h.select(internal)
    h.select_last(last)
    h.set_precision(B.PRECISION_MIXED)
    h.set_refinement(tol, max_iter)
    return h


def relres(o, s, x, b):
    r = b[:s.nrows] - o.mv(x[:s.ncols])
    return np.abs(r).max() / (block_norm_inf(s) * np.abs(x[:s.ncols]).max() + np.abs(b[:s.nrows]).max())


def oracle_solution(s, b, internal="LU", last="LU"):
    o = po.Oracle(s, internal, last)
    assert o.factorize(), o.last_error()
    return o, o.solve(b)


@pytest.mark.parametrize("kappa", [1.0, 10.0, 100.0])
def test_mixed_config_C_shape(kappa):
    # config C's block shape (n=32, nr=nx=8) at a size the oracle finishes quickly
    s = synth.collocation(2000, 32, 0, 0, 8, 8, kappa=kappa, seed=3)
    b = synth.rhs(s, nrhs=1, seed=11)
    o, xo = oracle_solution(s, b)
    h = mixed_solver(s)
    assert h.factorize(), h.last_error()
    x = np.array(b, copy=True)
    assert h.solve(x[0]), h.last_error()
    it, rr = h.refinement_info()
    assert 1 <= it <= 10
    assert rr <= RELRES_BAR, (kappa, it, rr)
    assert relres(o, s, x[0], b[0]) <= RELRES_BAR
    assert fwd_err(x[0, :s.ncols], xo[0, :s.ncols]) <= FWD_BAR


@pytest.mark.parametrize("dims", [(1, 1, 0, 0, 0, 0), (3, 2, 1, 1, 1, 1), (8, 4, 2, 2, 3, 3),
                                  (100, 8, 0, 0, 2, 2), (127, 16, 2, 2, 4, 4), (257, 7, 3, 3, 2, 2),
                                  (1000, 2, 0, 0, 0, 0), (65, 48, 1, 1, 4, 4)])
@pytest.mark.parametrize("internal", ["LU", "QR", "QRP"])
def test_mixed_matches_oracle(dims, internal):
    s = synth.collocation(*dims, seed=sum(dims)) if dims[1] > 1 else synth.dominant(*dims, seed=1)
    assert s.nrows == s.ncols
    b = synth.rhs(s, nrhs=2, seed=5)
    o, xo = oracle_solution(s, b, internal)
    h = mixed_solver(s, internal)
    assert h.factorize(), h.last_error()
    x = np.array(b, copy=True)
    assert h.solve_n(2, x, x.shape[1]), h.last_error()
    it, rr = h.refinement_info()
    assert rr <= RELRES_BAR, (dims, internal, it, rr)
    for c in range(2):
        assert relres(o, s, x[c], b[c]) <= RELRES_BAR
        assert fwd_err(x[c, :s.ncols], xo[c, :s.ncols]) <= FWD_BAR


def test_mixed_unrefined_is_fp32_accurate():
    """With no correction step the result is the plain FP32 solve."""
    s = synth.collocation(500, 16, 2, 2, 4, 4, seed=9)
    b = synth.rhs(s, nrhs=1, seed=1)
    o = po.Oracle(s, "LU", "LU")
    h = mixed_solver(s, max_iter=0)
    assert h.factorize(), h.last_error()
    x = np.array(b[0], copy=True)
    assert h.solve(x), h.last_error()
    it, rr = h.refinement_info()
    assert it == 0
    assert 1e-14 < rr < 1e-4
    assert abs(relres(o, s, x, b[0]) - rr) <= 0.05 * rr
    h.set_refinement(1e-12, 10)
    x2 = np.array(b[0], copy=True)
    assert h.solve(x2), h.last_error()
    it2, rr2 = h.refinement_info()
    assert it2 >= 1 and rr2 <= RELRES_BAR


def test_mixed_factorize_solve_and_graph_step():
    torch = pytest.importorskip("torch")
    s = synth.collocation(4097, 16, 2, 2, 4, 4, seed=21)
    b = synth.rhs(s, nrhs=1, seed=2)
    o, xo = oracle_solution(s, b)
    h = mixed_solver(s)
    x = np.array(b, copy=True)
    assert h.factorize_solve(1, x, x.shape[1]), h.last_error()
    it, rr = h.refinement_info()
    assert rr <= RELRES_BAR
    assert fwd_err(x[0, :s.ncols], xo[0, :s.ncols]) <= FWD_BAR
    L = s.nrows
    rhs = torch.tensor(b[0, :L], dtype=torch.float64, device="cuda")
    dx = torch.empty(L, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    h.graph_capture(B.GRAPH_STEP, 1, dx.data_ptr(), L, rhs.data_ptr())
    for _ in range(3):
        h.graph_launch(B.GRAPH_STEP)
    h.synchronize()
    it_g, rr_g = h.refinement_info()
    assert it_g == it and rr_g <= RELRES_BAR
    xg = dx.cpu().numpy()
    assert fwd_err(xg, xo[0, :s.ncols]) <= FWD_BAR
    assert np.array_equal(xg, x[0, :s.ncols])  # graph replay is bit-identical to the eager run


def test_mixed_rejects_non_square():
    s = synth.collocation(10, 4, 1, 0, 2, 2, seed=2)
    assert s.nrows != s.ncols
    h = mixed_solver(s, last="QR")
    with pytest.raises(B.BCRError, match="square"):
        h.factorize()


def test_mixed_switch_back_to_fp64():
    s = synth.collocation(300, 8, 0, 0, 2, 2, seed=4)
    b = synth.rhs(s, nrhs=1, seed=3)
    o, xo = oracle_solution(s, b)
    h = mixed_solver(s)
    assert h.factorize(), h.last_error()
    h.set_precision(B.PRECISION_FP64)
    x = np.array(b[0], copy=True)
    assert not h.solve(x)  # precision change drops the factorization
    assert h.factorize(), h.last_error()
    assert h.solve(x), h.last_error()
    assert h.refinement_info() == (0, 0.0)
    assert fwd_err(x[:s.ncols], xo[0, :s.ncols]) <= 1e-10


@pytest.mark.parametrize("kappa", [1.0, 100.0])
def test_mixed_full_size_config_C(kappa):
    """n=32, nblock=65536, nr=nx=8: residual property at full size."""
    s = synth.collocation(**synth.CONFIGS["C"], kappa=kappa, seed=0)
    b = synth.rhs(s, nrhs=1, seed=0)
    h = mixed_solver(s)
    x = np.array(b[0], copy=True)
    assert h.factorize_solve(1, x, x.shape[0]), h.last_error()
    it, rr = h.refinement_info()
    assert rr <= RELRES_BAR, (kappa, it, rr)
    o = po.Oracle(s, "LU", "LU")
    assert relres(o, s, x, b[0]) <= RELRES_BAR


# shapes of the FP32 large-block kernel with tcgen05 tensor-core products
# (33 <= n <= 128, nr <= 16, nx <= 16): one and two N chunks of the product
# (2n + nx above 256 at n = 128), K and N padding, n not a multiple of 32
UMMA_DIMS = [(5, 128, 4, 4, 16, 16), (33, 128, 4, 4, 16, 16), (17, 100, 2, 2, 16, 16),
             (9, 48, 1, 1, 4, 4), (8, 67, 0, 2, 5, 3), (6, 40, 0, 0, 0, 0), (12, 33, 1, 1, 2, 2),
             (7, 96, 3, 3, 8, 8)]


@pytest.mark.parametrize("dims", UMMA_DIMS)
def test_mixed_tensor_core_large_blocks(dims):
    """The tcgen05 3xTF32 pair kernel: its unrefined FP32 solve is FP32-accurate
    (within 100x of the CUDA-core FP32 kernel's residual), and refinement
    reaches the mixed bar with the forward error of the FP64 oracle."""
    s = synth.collocation(*dims, seed=sum(dims))
    assert s.nrows == s.ncols
    b = synth.rhs(s, nrhs=1, seed=4)
    o, xo = oracle_solution(s, b)
    unref = {}
    for pk in (B.PAIR_CTA, B.PAIR_UMMA):
        h = mixed_solver(s, max_iter=0)
        h.set_pair_kernel(pk)
        assert h.factorize(), h.last_error()
        x = np.array(b[0], copy=True)
        assert h.solve(x), h.last_error()
        unref[pk] = h.refinement_info()[1]
    assert unref[B.PAIR_UMMA] < 1e-5 and unref[B.PAIR_UMMA] <= 100 * unref[B.PAIR_CTA] + 1e-12, unref
    h = mixed_solver(s)
    assert h.factorize(), h.last_error()
    x = np.array(b[0], copy=True)
    assert h.solve(x), h.last_error()
    it, rr = h.refinement_info()
    assert it <= 3 and rr <= RELRES_BAR, (dims, it, rr)
    assert relres(o, s, x, b[0]) <= RELRES_BAR
    assert fwd_err(x[:s.ncols], xo[0, :s.ncols]) <= FWD_BAR


@pytest.mark.parametrize("n", [8, 16])
@pytest.mark.parametrize("nrhs", [1, 3, 5])
def test_mixed_factorize_solve_fused_first_solve(n, nrhs):
    """factorize_solve on the mixed path forms x0 with the FP32 factorization
    carrying the right-hand sides (at most 2n + nx + nrhs <= the pair kernel's
    trailing columns; 5 right-hand sides at n=16 take the separate solve), then
    refines every column to the bar."""
    s = synth.collocation(3001, n, 0, 0, 4, 4, seed=n + nrhs)
    b = synth.rhs(s, nrhs=nrhs, seed=7)
    o, xo = oracle_solution(s, b)
    h = mixed_solver(s)
    x = np.array(b, copy=True)
    assert h.factorize_solve(nrhs, x, x.shape[1]), h.last_error()
    it, rr = h.refinement_info()
    assert 1 <= it <= 10 and rr <= RELRES_BAR, (it, rr)
    for c in range(nrhs):
        assert relres(o, s, x[c], b[c]) <= RELRES_BAR
        assert fwd_err(x[c, :s.ncols], xo[c, :s.ncols]) <= FWD_BAR
    # the factors again, with a plain solve
    y = np.array(b, copy=True)
    assert h.solve_n(nrhs, y, y.shape[1]), h.last_error()
    for c in range(nrhs):
        assert relres(o, s, y[c], b[c]) <= RELRES_BAR
