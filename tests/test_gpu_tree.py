"""GPU tests of the tree bookkeeping of the n = 8 / 16 FP64 LU factorization:
the tree schedule (k_factor_tree_tc: the whole cyclic reduction of one system
in one launch) and the level-by-level launches that gather the border
updates instead of running fix-up launches (PAIR_TC_GATHER).

Every number of blocks whose tree has a ragged edge (odd counts, one above and
one below a power of two) is compared with the CPU oracle (forward error
<= 1e-10, relative residual <= 1e-13) and with the level-by-level launches of
the same pair kernel (agreement to 1e-12: the border sums are added in another
order), on the plain factorize + solve and on the fused factorize+solve path;
the tree's results are bit-identical run to run."""
import numpy as np
import pytest

from alglin_b200 import bcr as B
from alglin_b200 import synth
from oracle import pyoracle as po
from tests._util import block_norm_inf, fwd_err

pytestmark = pytest.mark.gpu

NBLOCKS = [2, 3, 4, 5, 7, 8, 9, 16, 17, 31, 33, 100, 255, 256, 257, 1000, 4097]
BORDERS = [(0, 0, 0, 0), (2, 2, 4, 4), (1, 0, 3, 1), (0, 2, 8, 8)]


def _last(s):
    return "LU" if s.Nr == s.Nc else ("QR" if s.Nr > s.Nc else "PINV")


def _solver(s, family):
    h = B.BorderedCR()
    h.load_system(s)
    h.select("LU")
    h.select_last(_last(s))
    h.set_pair_kernel(family)
    return h


def _solve(h, b):
    X = np.array(b, dtype=np.float64, order="C", copy=True)
    assert h.solve_n(X.shape[0], X, X.shape[1]), h.last_error()
    return X


@pytest.mark.parametrize("nb", NBLOCKS)
@pytest.mark.parametrize("n", [8, 16])
@pytest.mark.parametrize("border", BORDERS)
def test_tree_matches_oracle_and_level_schedule(nb, n, border):
    qr, qx, nr, nx = border
    s = synth.collocation(nb, n, qr, qx, nr, nx, seed=nb + n + nr)
    b = synth.rhs(s, nrhs=2, seed=3)
    o = po.Oracle(s, "LU", _last(s))
    assert o.factorize(), o.last_error()
    xo = o.solve(b)
    hl = _solver(s, B.PAIR_TC)
    assert hl.factorize(), hl.last_error()
    xl = _solve(hl, b)
    for fam in (B.PAIR_TREE, B.PAIR_TC_GATHER):
        ht = _solver(s, fam)
        assert ht.factorize(), ht.last_error()
        xt = _solve(ht, b)
        for c in range(2):
            assert fwd_err(xt[c, :s.ncols], xo[c, :s.ncols]) < 1e-10, (fam, nb, n, border, c)
            assert fwd_err(xt[c, :s.ncols], xl[c, :s.ncols]) < 1e-12, (fam, nb, n, border, c)
            if s.Nr == s.Nc:
                r = b[c, :s.nrows] - o.mv(xt[c, :s.ncols])
                rel = np.abs(r).max() / (block_norm_inf(s) * np.abs(xt[c, :s.ncols]).max() +
                                         np.abs(b[c, :s.nrows]).max())
                assert rel < 1e-13, (fam, nb, n, border, rel)
        # the same factors again, and the fused factorize+solve
        X = b.copy()
        assert ht.factorize_solve(2, X, X.shape[1]), ht.last_error()
        assert fwd_err(X[:, :s.ncols], xo[:, :s.ncols]) < 1e-10
        # bit-identical run to run
        assert ht.factorize(), ht.last_error()
        assert np.array_equal(_solve(ht, b), xt)


@pytest.mark.parametrize("nrhs", [1, 3])
def test_tree_fused_rhs_full_width(nrhs):
    """Fused forward elimination of several right-hand sides through the tree
    (the xb updates are summed up the tree)."""
    s = synth.collocation(3001, 16, 2, 2, 4, 4, seed=8)
    b = synth.rhs(s, nrhs=nrhs, seed=9)
    o = po.Oracle(s, "LU", "LU")
    assert o.factorize(), o.last_error()
    xo = o.solve(b)
    for fam in (B.PAIR_TREE, B.PAIR_TC_GATHER):
        h = _solver(s, fam)
        X = b.copy()
        assert h.factorize_solve(nrhs, X, X.shape[1]), h.last_error()
        assert fwd_err(X[:, :s.ncols], xo[:, :s.ncols]) < 1e-10


def test_tree_singular_panel_reports_like_reference():
    """An exactly-zero panel [E_0; D_1] at n=16: the tree finishes every other
    pair and the factorization fails with the reference's getrf message."""
    s = synth.collocation(64, 16, 0, 0, 2, 2, seed=1)
    s.D[1] = 0.0
    s.E[0] = 0.0
    h = _solver(s, B.PAIR_TREE)
    assert not h.factorize()
    assert "getrf(M=32,N=16,A,LDA=32,iperm)::INFO = 1" in h.last_error()
    # a good matrix on the same handle factors again (counters reset)
    s2 = synth.collocation(64, 16, 0, 0, 2, 2, seed=2)
    h2 = _solver(s2, B.PAIR_TREE)
    assert h2.factorize(), h2.last_error()


@pytest.mark.parametrize("dims", [(2048, 16, 2, 2, 4, 4), (5000, 8, 0, 0, 2, 2), (10001, 16, 1, 1, 3, 3),
                                  (33000, 16, 0, 0, 0, 0)])
@pytest.mark.parametrize("nrhs", [1, 2])
def test_chunked_upload_factorize_solve(dims, nrhs):
    """factorize_solve from host buffers uploads the matrix in chunks and
    factors each chunk's own levels while the next chunk is in flight: the
    oracle's answer, a second call on the same handle, the loaded matrix on the
    device afterwards (Mv), and a later plain solve with the stored factors."""
    s = synth.collocation(*dims, seed=sum(dims))
    b = synth.rhs(s, nrhs=nrhs, seed=4)
    o = po.Oracle(s, "LU", _last(s))
    assert o.factorize(), o.last_error()
    xo = o.solve(b)
    h = _solver(s, B.PAIR_AUTO)
    for _ in range(2):
        X = b.copy()
        assert h.factorize_solve(nrhs, X, X.shape[1]), h.last_error()
        assert fwd_err(X[:, :s.ncols], xo[:, :s.ncols]) < 1e-10
    xr = np.random.default_rng(1).standard_normal(s.ncols)
    assert np.abs(h.mv(xr)[:s.nrows] - o.mv(xr)).max() < 1e-12 * max(1.0, np.abs(o.mv(xr)).max())
    Y = _solve(h, b)
    assert fwd_err(Y[:, :s.ncols], xo[:, :s.ncols]) < 1e-10
