"""CPU tests of the oracle: pinned against the reference's own BorderedCR
(golden fixtures made by tests/golden/make_golden.py, and the compiled
reference when it is present) and against dense solves."""
import numpy as np
import pytest

from alglin_b200 import synth
from oracle import pyoracle as po
from tests._util import GOLDEN_CASES, fwd_err, load_golden


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_oracle_matches_reference_golden(name):
    s, b, X, tags = load_golden(name)
    for (internal, last, last2), xg in zip(tags, X):
        o = po.Oracle(s, internal, last, last2)
        assert o.factorize(), o.last_error()
        x = o.solve(b)
        for c in range(b.shape[0]):
            err = fwd_err(x[c, :s.ncols], xg[c, :s.ncols])
            assert err < 1e-11, (name, internal, last, c, err)


@pytest.mark.skipif(not po.ref_available(), reason="reference build (oracle/_ref) absent")
@pytest.mark.parametrize("npb", [1, 2, 3, 4, 7])
@pytest.mark.parametrize("internal", ["LU", "QR", "QRP"])
def test_oracle_matches_reference_chunked(npb, internal):
    """The reference's threaded schedule (chunks + reduced CR, cc:139-158,
    1175-1266) restated in the oracle gives the reference's answer."""
    s = synth.collocation(61, 5, 1, 2, 3, 2, seed=5)
    b = synth.rhs(s, nrhs=3, seed=2)
    o = po.Oracle(s, internal, "LU", npb=npb)
    assert o.factorize(), o.last_error()
    r = po.RefBCR(s, internal, "LU", nthreads=npb, npb=npb)
    assert r.factorize(), r.last_error()
    xo, xr = o.solve(b), r.solve(b)
    assert fwd_err(xo[:, :s.ncols], xr[:, :s.ncols]) < 1e-12


@pytest.mark.parametrize("dims", [(1, 1, 0, 0, 1, 1), (2, 3, 0, 0, 0, 0), (5, 2, 1, 1, 2, 1),
                                  (9, 4, 2, 0, 0, 2), (16, 3, 0, 3, 1, 0)])
@pytest.mark.parametrize("internal", ["LU", "QR", "QRP"])
def test_oracle_dense_crosscheck(dims, internal):
    s = synth.dominant(*dims, seed=sum(dims))
    A = s.to_dense()
    if s.nrows != s.ncols:
        pytest.skip("square systems only")
    rng = np.random.default_rng(0)
    xref = rng.standard_normal(s.ncols)
    b = A @ xref
    o = po.Oracle(s, internal, "LU")
    assert o.factorize(), o.last_error()
    x = o.solve(b)
    assert fwd_err(x, xref) < 1e-11
    assert np.abs(o.mv(xref) - b).max() < 1e-12 * np.abs(b).max()


def test_oracle_manufactured_test7_style():
    """src_tests/test7-BorderedCR.cc:223-288 checks: x_i = 1 + (i % 100)."""
    s = synth.dominant(2000, 8, 4, 4, 1, 1, seed=2)
    xref = 1.0 + (np.arange(s.ncols) % 100)
    b = np.zeros(max(s.nrows, s.ncols))
    o = po.Oracle(s, "LU", "LU")
    b[:s.nrows] = o.mv(xref)
    assert o.factorize()
    x = o.solve(b)
    assert np.abs(x[:s.ncols] - xref).max() < 1e-8
    assert np.abs(x[:s.ncols] - xref).sum() / s.ncols < 1e-8
    assert np.abs(o.mv(x[:s.ncols]) - b[:s.nrows]).max() < 1e-6


def test_oracle_last_block_fallback():
    """test18-BorderedCR-coverage.cc:1061-1098: singular last block."""
    s = synth._zeros(1, 1, 0, 0, 1, 1)
    s.D[0, 0, 0] = 1; s.H[1, 0] = 1; s.C[0, 0, 0] = 1; s.C[1, 0, 0] = 1
    o = po.Oracle(s, "LU", "LU", "NONE")
    assert not o.factorize()
    assert "load_and_factorize_last" in o.last_error()
    o = po.Oracle(s, "LU", "LU", "PINV")
    assert o.factorize()
    xref = np.array([2.0, -1.0, 0.0])
    b = o.mv(xref)
    x = o.solve(b)
    assert np.abs(x - xref).max() < 5e-9


def test_oracle_singular_panel_reports_getrf():
    s = synth.dominant(4, 3, 0, 0, 0, 0, seed=1)
    s.D[1] = 0.0
    s.E[0] = 0.0
    o = po.Oracle(s, "LU", "LU")
    assert not o.factorize()
    assert "getrf(M=6,N=3,A,LDA=6,iperm)::INFO = 1" in o.last_error()
