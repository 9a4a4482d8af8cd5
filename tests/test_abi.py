"""CPU tests of the C ABI library: it loads, exports every symbol declared in
include/alglin_b200.h, and its host-side logic (sizes, loaders, element access,
selection strings, info(), sparse export/import, check_matrix) behaves like the
reference (src_tests/test17-BorderedCR-regressions.cc, test18 :265-918).
No compute call is made here."""
import ctypes as ct
import os
import re

import numpy as np
import pytest

from alglin_b200 import bcr as B
from alglin_b200 import synth
from oracle import pyoracle as po

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "alglin_b200.h")).read()
    return sorted(set(re.findall(r"\b(bcr_[A-Za-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_header_symbol():
    L = B.lib()
    missing = [s for s in header_symbols() if not hasattr(L, s)]
    assert not missing, missing
    assert sorted(header_symbols()) == sorted(B.exported_symbols())


def test_sizes_and_selection_strings():
    h = B.BorderedCR(4, 1)
    h.allocate(6, 2, 1, 2, 3, 2)
    assert (h.number_of_blocks(), h.block_size(), h.dim_qr(), h.dim_qx(), h.dim_nr(), h.dim_nx()) == (6, 2, 1, 2, 3, 2)
    assert h.Nr() == 2 * 2 + 1 + 3 and h.Nc() == 2 * 2 + 2 + 2
    assert h.nrows() == 2 * 7 + 1 + 3 and h.ncols() == 2 * 7 + 2 + 2
    h.set_factorize_use_thread(False); h.set_solve_use_thread(False)
    assert not h.factorize_use_thread() and not h.solve_use_thread()
    for s, name in [("LU", "CyclicReduction+LU"), ("QR", "CyclicReduction+QR"), ("QRP", "CyclicReduction+QRP")]:
        h.select(s)
        assert h.info_algo_block() == name
    for s in ["LU", "LUPQ", "QR", "QRP", "SVD", "LSS", "LSY", "PINV"]:
        h.select_last(s)
        assert h.info_algo_last_block() == "LastBlock " + s
    for s in ["NONE", "SVD", "LSS", "LSY", "PINV"]:
        h.select_last2(s)
        assert h.info_algo_last_block2() == "LastBlock " + s
    # test18:342-346: 4 requested blocks on nblock=6 -> nblk:3
    h.set_num_parallel_block(4)
    info = h.info("  ")
    assert "nblk:3" in info and "CyclicReduction+QRP" in info and "LastBlock PINV" in info
    assert info.startswith("  rows")
    for bad in (lambda: h.select("BAD"), lambda: h.select_last("BAD"), lambda: h.select_last2("BAD")):
        with pytest.raises(B.BCRError):
            bad()
    assert "unknown/unsupported factorization type" in h.last_error()


def test_loaders_and_element_access():
    h = B.BorderedCR()
    nb, n, qr, qx, nr, nx = 5, 3, 2, 1, 2, 2
    h.allocate(nb, n, qr, qx, nr, nx)
    h.fill_zero()
    rng = np.random.default_rng(0)
    D = rng.standard_normal((n, n)); E = rng.standard_normal((n, n)); Bm = rng.standard_normal((n, nx))
    h.load_D(1, D); h.load_E(1, E); h.load_B(1, Bm)
    assert np.array_equal(h.D(1), D) and np.array_equal(h.E(1), E) and np.array_equal(h.B(1), Bm)
    DEB = rng.standard_normal((n, 2 * n + nx))
    h.load_DEB(2, DEB)
    assert np.array_equal(h.D(2), DEB[:, :n]) and np.array_equal(h.E(2), DEB[:, n:2 * n])
    assert np.array_equal(h.B(2), DEB[:, 2 * n:])
    h.add_to_B(2, Bm)
    assert np.allclose(h.B(2), DEB[:, 2 * n:] + Bm)
    C2F = rng.standard_normal((nr, 2 * n + nx))
    h.zero_C(); h.zero_F()
    h.add_to_C2F(3, C2F)                                   # test17:53-120
    assert np.allclose(h.C(3), C2F[:, :n]) and np.allclose(h.C(4), C2F[:, n:2 * n])
    assert np.allclose(h.F(), C2F[:, 2 * n:])
    m = n + qr
    H0, HN, Hq, Hp = (rng.standard_normal((m, c)) for c in (n, n, qx, nx))
    h.load_bottom(H0, HN, Hq, Hp)
    assert np.array_equal(h.H(), np.hstack([H0, HN, Hq, Hp]))
    P = rng.standard_normal((nr, h.Nc()))
    h.load_bottom2(P)                                       # load_bottom2(MatW) cc:430-447
    assert np.array_equal(h.C(0), P[:, :n]) and np.array_equal(h.C(nb), P[:, n:2 * n])
    assert np.array_equal(h.Cq(), P[:, 2 * n:2 * n + qx]) and np.array_equal(h.F(), P[:, 2 * n + qx:])
    with pytest.raises(B.BCRError):
        h.add_to_C(0, np.zeros((1, n)))  # ldC < nr
    assert "bad ldC" in h.last_error()
    with pytest.raises(B.BCRError):
        h.load_D(nb, D)  # block index out of range


def test_sparse_roundtrip_matches_dense():
    s = synth.dominant(7, 3, 2, 1, 2, 2, seed=4)
    h = B.BorderedCR()
    h.load_system(s)
    I, J = h.sparse_pattern(0)
    V = h.sparse_values()
    A = np.zeros((s.nrows, s.ncols))
    np.add.at(A, (I, J), V)
    assert np.array_equal(A, s.to_dense())
    assert h.sparse_nnz() == len(V)
    g = B.BorderedCR()
    g.allocate(*s.dims())
    g.sparse_load(V, I + 1, 1, J + 1, 1)
    I2, J2 = g.sparse_pattern(1)
    assert np.array_equal(g.sparse_values(), V) and np.array_equal(I2, I + 1)
    with pytest.raises(B.BCRError):
        g.sparse_load(np.array([1.0]), np.array([0]), 0, np.array([s.ncols - 1 - s.nx - 1]), 0)
    assert "out of pattern" in g.last_error()


@pytest.mark.parametrize("dims", [(7, 3, 2, 1, 2, 2), (5, 4, 0, 0, 0, 0), (6, 2, 1, 3, 0, 2),
                                  (4, 3, 0, 2, 3, 0), (9, 16, 2, 2, 4, 4)])
def test_sparse_export_bit_exact_vs_reference(dims):
    """sparse_pattern / sparse_values agree element by element (same order,
    same indices, same values) with the reference's own export
    (BABD_BorderedCR.cc:2316-2413, compiled in oracle/_ref)."""
    if not po.ref_available():
        pytest.skip("oracle/_ref not built (reference tree absent)")
    s = synth.dominant(*dims, seed=5)
    h = B.BorderedCR()
    h.load_system(s)
    I, J = h.sparse_pattern(0)
    V = h.sparse_values()
    Ir, Jr, Vr = po.RefBCR(s).sparse()
    assert h.sparse_nnz() == len(Vr)
    assert np.array_equal(I, Ir) and np.array_equal(J, Jr)
    assert np.array_equal(V, Vr)
    I1, J1 = h.sparse_pattern(1)
    assert np.array_equal(I1, Ir + 1) and np.array_equal(J1, Jr + 1)


def test_check_matrix_and_tsolve():
    s = synth.stable_small()
    h = B.BorderedCR()
    h.load_system(s)
    h.check_matrix()
    h.F()[0, 0] = np.nan
    with pytest.raises(B.BCRError):
        h.check_matrix()
    assert "check_matrix" in h.last_error() and "matrix F" in h.last_error()
    with pytest.raises(B.BCRError):
        h.t_solve(np.zeros(h.ncols()))
    assert "t_solve() not defined" in h.last_error()


def test_dup_copies_matrix():
    s = synth.dominant(9, 2, 1, 1, 1, 1, seed=3)
    a = B.BorderedCR(); a.load_system(s)
    b = B.BorderedCR(); b.dup(a)
    assert b.nrows() == a.nrows()
    assert np.array_equal(b.sparse_values(), a.sparse_values())


def test_compute_without_gpu_fails_loudly(has_gpu):
    if has_gpu:
        pytest.skip("a GPU is present")
    h = B.BorderedCR()
    h.load_system(synth.stable_small())
    with pytest.raises(B.BCRError):
        h.factorize()
    assert "no CUDA device" in h.last_error()
