"""ctypes front-ends for the test oracles.  TEST INFRASTRUCTURE ONLY: imported by
tests/, by the smoke check and by the benchmark's CPU-baseline / reference arm,
never by the product package.

* ``Oracle``  -- the plain-C restatement in bcr_oracle.c (always available);
* ``RefBCR``  -- the reference's own BorderedCR compiled from the unmodified
  reference sources (oracle/_ref/libbcr_ref.so, present when it was built).
"""
from __future__ import annotations

import ctypes as ct
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_ORACLE = os.path.join(HERE, "liboracle_bcr.so")
LIB_REF = os.path.join(HERE, "_ref", "libbcr_ref.so")

INTERNAL = {"LU": 0, "QR": 1, "QRP": 2}
LAST = {"LU": 0, "LUPQ": 1, "QR": 2, "QRP": 3, "SVD": 4, "LSS": 5, "LSY": 6, "PINV": 7}
LAST2 = {"NONE": 0, "SVD": 1, "LSS": 2, "LSY": 3, "PINV": 4}

_dp = ct.POINTER(ct.c_double)


_ip = ct.POINTER(ct.c_int)


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def _iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_ip)


def _load(path):
    if not os.path.exists(path):
        raise FileNotFoundError(path)
    return ct.CDLL(path)


_lib_o = None
_lib_r = None


def oracle_lib():
    global _lib_o
    if _lib_o is None:
        L = _load(LIB_ORACLE)
        L.orc_create.restype = ct.c_void_p
        L.orc_create.argtypes = [ct.c_int] * 6
        L.orc_destroy.argtypes = [ct.c_void_p]
        L.orc_load.argtypes = [ct.c_void_p] + [_dp] * 7
        L.orc_select.argtypes = [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int]
        L.orc_set_num_parallel_block.argtypes = [ct.c_void_p, ct.c_int]
        L.orc_used_parallel_block.argtypes = [ct.c_void_p]
        L.orc_factorize.argtypes = [ct.c_void_p]
        L.orc_solve.argtypes = [ct.c_void_p, ct.c_int, _dp, ct.c_int]
        L.orc_add_mv.argtypes = [ct.c_void_p, ct.c_double, _dp, ct.c_double, _dp]
        L.orc_last_error.restype = ct.c_char_p
        L.orc_last_error.argtypes = [ct.c_void_p]
        L.orc_nrows.argtypes = [ct.c_void_p]
        L.orc_ncols.argtypes = [ct.c_void_p]
        _lib_o = L
    return _lib_o


def ref_available() -> bool:
    return os.path.exists(LIB_REF)


def ref_lib():
    global _lib_r
    if _lib_r is None:
        L = _load(LIB_REF)
        L.ref_create.restype = ct.c_void_p
        L.ref_create.argtypes = [ct.c_int, ct.c_int]
        L.ref_destroy.argtypes = [ct.c_void_p]
        L.ref_allocate.argtypes = [ct.c_void_p] + [ct.c_int] * 6
        L.ref_load.argtypes = [ct.c_void_p] + [_dp] * 7
        L.ref_select.argtypes = [ct.c_void_p, ct.c_char_p, ct.c_char_p, ct.c_char_p]
        L.ref_set_threads.argtypes = [ct.c_void_p, ct.c_int, ct.c_int]
        L.ref_set_num_parallel_block.argtypes = [ct.c_void_p, ct.c_int]
        L.ref_factorize.argtypes = [ct.c_void_p]
        L.ref_solve.argtypes = [ct.c_void_p, _dp]
        L.ref_solve_n.argtypes = [ct.c_void_p, ct.c_int, _dp, ct.c_int]
        L.ref_mv.argtypes = [ct.c_void_p, _dp, _dp]
        L.ref_dup.argtypes = [ct.c_void_p, ct.c_void_p]
        L.ref_last_error.restype = ct.c_char_p
        L.ref_last_error.argtypes = [ct.c_void_p]
        L.ref_info.restype = ct.c_char_p
        L.ref_info.argtypes = [ct.c_void_p]
        L.ref_nrows.argtypes = [ct.c_void_p]
        L.ref_ncols.argtypes = [ct.c_void_p]
        L.ref_sparse_nnz.argtypes = [ct.c_void_p]
        L.ref_sparse_pattern.argtypes = [ct.c_void_p, _ip, _ip, ct.c_int]
        L.ref_sparse_values.argtypes = [ct.c_void_p, _dp]
        L.ref_f32_factor_solve.restype = ct.c_double
        L.ref_f32_factor_solve.argtypes = [ct.c_int] * 8 + [_dp] * 8 + [ct.POINTER(ct.c_int)]
        L.ref_time_factor_solve.restype = ct.c_double
        L.ref_time_factor_solve.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_int, _dp, ct.c_int,
                                            ct.POINTER(ct.c_int)]
        _lib_r = L
    return _lib_r


def _arrays(s):
    return [np.ascontiguousarray(getattr(s, k), dtype=np.float64)
            for k in ("D", "E", "B", "C", "Cq", "F", "H")]


class Oracle:
    """The C restatement (bcr_oracle.c)."""

    def __init__(self, s, internal="LU", last="LU", last2="NONE", npb=1):
        self.L = oracle_lib()
        self.s = s
        self.h = self.L.orc_create(*s.dims())
        self._keep = _arrays(s)
        self.L.orc_load(self.h, *[_ptr(a) for a in self._keep])
        self.L.orc_select(self.h, INTERNAL[internal], LAST[last], LAST2[last2])
        if npb != 1:
            self.L.orc_set_num_parallel_block(self.h, npb)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_destroy(self.h)
            self.h = None

    @property
    def npb(self):
        return self.L.orc_used_parallel_block(self.h)

    def factorize(self) -> bool:
        return bool(self.L.orc_factorize(self.h))

    def last_error(self) -> str:
        return self.L.orc_last_error(self.h).decode()

    def solve(self, b: np.ndarray) -> np.ndarray:
        """b: (nrhs, L) or (L,) right-hand sides, L >= max(nrows, ncols)."""
        x = np.array(b, dtype=np.float64, order="C", copy=True)
        one = x.ndim == 1
        X = x.reshape(1, -1) if one else x
        ok = self.L.orc_solve(self.h, X.shape[0], _ptr(X), X.shape[1])
        if not ok:
            raise RuntimeError("oracle solve failed: " + self.last_error())
        return X[0] if one else X

    def mv(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        res = np.zeros(max(self.s.nrows, self.s.ncols))
        self.L.orc_add_mv(self.h, 1.0, _ptr(x), 0.0, _ptr(res))
        return res[:self.s.nrows]


def ref_f32_factor_solve(s, b, nthreads=0, npb=0):
    """The reference's BorderedCR<float> (LU, last block LU) on system s with
    every entry rounded to float: returns (seconds of factorize + solve, x)
    with x converted back to double.  No refinement."""
    L = ref_lib()
    x = np.array(b, dtype=np.float64, order="C", copy=True)
    arrs = _arrays(s)
    ok = ct.c_int(0)
    t = L.ref_f32_factor_solve(nthreads, npb, *s.dims(), *[_ptr(a) for a in arrs], _ptr(x), ct.byref(ok))
    if not ok.value:
        raise RuntimeError("reference BorderedCR<float> factor/solve failed")
    return t, x


class RefBCR:
    """The reference alglin::BorderedCR<double>, compiled from its own sources."""

    def __init__(self, s, internal="LU", last="LU", last2="NONE", nthreads=0, npb=0):
        self.L = ref_lib()
        self.s = s
        self.h = self.L.ref_create(nthreads, npb)
        if not self.L.ref_allocate(self.h, *s.dims()):
            raise RuntimeError(self.last_error())
        self._keep = _arrays(s)
        if not self.L.ref_load(self.h, *[_ptr(a) for a in self._keep]):
            raise RuntimeError(self.last_error())
        if not self.L.ref_select(self.h, internal.encode(), last.encode(), last2.encode()):
            raise RuntimeError(self.last_error())

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ref_destroy(self.h)
            self.h = None

    def set_threads(self, fact: bool, solve: bool):
        self.L.ref_set_threads(self.h, int(fact), int(solve))

    def set_num_parallel_block(self, npb: int):
        self.L.ref_set_num_parallel_block(self.h, npb)

    def info(self) -> str:
        return self.L.ref_info(self.h).decode()

    def last_error(self) -> str:
        return self.L.ref_last_error(self.h).decode()

    def factorize(self) -> bool:
        return bool(self.L.ref_factorize(self.h))

    def solve(self, b: np.ndarray) -> np.ndarray:
        x = np.array(b, dtype=np.float64, order="C", copy=True)
        if x.ndim == 1:
            ok = self.L.ref_solve(self.h, _ptr(x))
        else:
            ok = self.L.ref_solve_n(self.h, x.shape[0], _ptr(x), x.shape[1])
        if not ok:
            raise RuntimeError("reference solve failed: " + self.last_error())
        return x

    def mv(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        res = np.zeros(max(self.s.nrows, self.s.ncols))
        self.L.ref_mv(self.h, _ptr(x), _ptr(res))
        return res[:self.s.nrows]

    def sparse(self):
        """(I, J, V) of the reference's sparse_pattern(offs=0) / sparse_values."""
        nnz = self.L.ref_sparse_nnz(self.h)
        I = np.zeros(nnz, dtype=np.int32)
        J = np.zeros(nnz, dtype=np.int32)
        V = np.zeros(nnz)
        if not self.L.ref_sparse_pattern(self.h, _iptr(I), _iptr(J), 0):
            raise RuntimeError(self.last_error())
        if not self.L.ref_sparse_values(self.h, _ptr(V)):
            raise RuntimeError(self.last_error())
        return I, J, V

    def time_factor_solve(self, src: "RefBCR", b: np.ndarray):
        """Factorize a fresh copy of ``src``'s matrix into this object and solve
        ``b`` in place; returns (seconds, x)."""
        x = np.array(b, dtype=np.float64, order="C", copy=True)
        ok = ct.c_int(0)
        nrhs = 1 if x.ndim == 1 else x.shape[0]
        ld = x.shape[-1]
        t = self.L.ref_time_factor_solve(self.h, src.h, nrhs, _ptr(x), ld, ct.byref(ok))
        if not ok.value:
            raise RuntimeError("reference factor/solve failed: " + self.last_error())
        return t, x
