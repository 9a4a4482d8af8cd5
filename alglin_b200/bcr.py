"""Python front-end of the B200 BorderedCR solver (ctypes over the C ABI of
libalglin_b200.so, declared in include/alglin_b200.h).

``BorderedCR`` mirrors the methods of the reference C++ class
``alglin::BorderedCR<double>`` (src/Alglin/BABD_BorderedCR.hxx): the same
names, argument meanings and error behaviour -- ``factorize``/``solve`` return
``False`` on a numerical failure with the reason in ``last_error()``, and bad
arguments raise (the reference throws ``Utils::Runtime_Error``).  Every
numerical step runs on the GPU; without the compiled library or without a GPU
the calls fail loudly -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as ct
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libalglin_b200.so")

BCR_OK, BCR_NUMERICAL, BCR_BAD_ARGUMENT, BCR_CUDA_ERROR, BCR_DEVICE_TIMEOUT = range(5)
PRECISION_FP64, PRECISION_MIXED = 0, 1
PAIR_AUTO, PAIR_TC, PAIR_GRP, PAIR_ROWS, PAIR_CTA, PAIR_SMEM, PAIR_UMMA, PAIR_TREE, PAIR_TC_GATHER = range(9)

_dp = ct.POINTER(ct.c_double)
_ip = ct.POINTER(ct.c_int)
_H = ct.c_void_p

# (name, argtypes, restype) of every exported entry point
_SIGS = [
    ("bcr_create", [ct.POINTER(_H), ct.c_int, ct.c_int], ct.c_int),
    ("bcr_destroy", [_H], ct.c_int),
    ("bcr_allocate", [_H] + [ct.c_int] * 6, ct.c_int),
    ("bcr_dup", [_H, _H], ct.c_int),
    ("bcr_nrows", [_H], ct.c_int), ("bcr_ncols", [_H], ct.c_int),
    ("bcr_number_of_blocks", [_H], ct.c_int), ("bcr_block_size", [_H], ct.c_int),
    ("bcr_dim_qr", [_H], ct.c_int), ("bcr_dim_qx", [_H], ct.c_int),
    ("bcr_dim_nr", [_H], ct.c_int), ("bcr_dim_nx", [_H], ct.c_int),
    ("bcr_Nr", [_H], ct.c_int), ("bcr_Nc", [_H], ct.c_int),
    ("bcr_zero_B", [_H], ct.c_int), ("bcr_zero_C", [_H], ct.c_int), ("bcr_zero_Cq", [_H], ct.c_int),
    ("bcr_zero_D", [_H], ct.c_int), ("bcr_zero_E", [_H], ct.c_int), ("bcr_zero_F", [_H], ct.c_int),
    ("bcr_zero_H", [_H], ct.c_int), ("bcr_fill_zero", [_H], ct.c_int),
    ("bcr_load_B", [_H, ct.c_int, _dp, ct.c_int], ct.c_int),
    ("bcr_add_to_B", [_H, ct.c_int, _dp, ct.c_int], ct.c_int),
    ("bcr_load_C", [_H, ct.c_int, _dp, ct.c_int], ct.c_int),
    ("bcr_add_to_C", [_H, ct.c_int, _dp, ct.c_int], ct.c_int),
    ("bcr_add_to_C2", [_H, ct.c_int, _dp, ct.c_int], ct.c_int),
    ("bcr_add_to_C2F", [_H, ct.c_int, _dp, ct.c_int], ct.c_int),
    ("bcr_load_D", [_H, ct.c_int, _dp, ct.c_int], ct.c_int),
    ("bcr_load_E", [_H, ct.c_int, _dp, ct.c_int], ct.c_int),
    ("bcr_load_DE", [_H, ct.c_int, _dp, ct.c_int], ct.c_int),
    ("bcr_load_DEB", [_H, ct.c_int, _dp, ct.c_int], ct.c_int),
    ("bcr_load_F", [_H, _dp, ct.c_int], ct.c_int),
    ("bcr_add_to_F", [_H, _dp, ct.c_int], ct.c_int),
    ("bcr_load_Cq", [_H, _dp, ct.c_int], ct.c_int),
    ("bcr_load_CqF", [_H, _dp, ct.c_int], ct.c_int),
    ("bcr_load_bottom", [_H, _dp, ct.c_int, _dp, ct.c_int, _dp, ct.c_int, _dp, ct.c_int], ct.c_int),
    ("bcr_load_bottom_H", [_H, _dp, ct.c_int], ct.c_int),
    ("bcr_load_bottom2", [_H, _dp, ct.c_int, _dp, ct.c_int, _dp, ct.c_int, _dp, ct.c_int], ct.c_int),
    ("bcr_load_bottom2_H", [_H, _dp, ct.c_int], ct.c_int),
    ("bcr_block_data", [_H, ct.c_char, ct.c_int], _dp),
    ("bcr_select", [_H, ct.c_char_p], ct.c_int),
    ("bcr_select_last", [_H, ct.c_char_p], ct.c_int),
    ("bcr_select_last2", [_H, ct.c_char_p], ct.c_int),
    ("bcr_selected", [_H, _ip, _ip, _ip], ct.c_int),
    ("bcr_set_factorize_use_thread", [_H, ct.c_int], ct.c_int),
    ("bcr_set_solve_use_thread", [_H, ct.c_int], ct.c_int),
    ("bcr_factorize_use_thread", [_H], ct.c_int),
    ("bcr_solve_use_thread", [_H], ct.c_int),
    ("bcr_set_num_parallel_block", [_H, ct.c_int], ct.c_int),
    ("bcr_set_precision", [_H, ct.c_int], ct.c_int),
    ("bcr_set_refinement", [_H, ct.c_double, ct.c_int], ct.c_int),
    ("bcr_set_pair_kernel", [_H, ct.c_int], ct.c_int),
    ("bcr_refinement_info", [_H, ct.POINTER(ct.c_int), _dp], ct.c_int),
    ("bcr_info", [_H, ct.c_char_p], ct.c_char_p),
    ("bcr_last_error", [_H], ct.c_char_p),
    ("bcr_set_debug", [_H, ct.c_int], ct.c_int),
    ("bcr_check_matrix", [_H], ct.c_int),
    ("bcr_factorize", [_H], ct.c_int),
    ("bcr_solve", [_H, _dp], ct.c_int),
    ("bcr_solve_n", [_H, ct.c_int, _dp, ct.c_int], ct.c_int),
    ("bcr_factorize_solve", [_H, ct.c_int, _dp, ct.c_int], ct.c_int),
    ("bcr_factorize_solve_device", [_H, ct.c_int, ct.c_void_p, ct.c_int], ct.c_int),
    ("bcr_t_solve", [_H, _dp], ct.c_int),
    ("bcr_t_solve_n", [_H, ct.c_int, _dp, ct.c_int], ct.c_int),
    ("bcr_mv", [_H, _dp, _dp], ct.c_int),
    ("bcr_add_mv", [_H, ct.c_double, _dp, _dp], ct.c_int),
    ("bcr_sparse_nnz", [_H], ct.c_int),
    ("bcr_sparse_pattern", [_H, _ip, _ip, ct.c_int], ct.c_int),
    ("bcr_sparse_values", [_H, _dp], ct.c_int),
    ("bcr_sparse_load", [_H, _dp, _ip, ct.c_int, _ip, ct.c_int, ct.c_int, ct.c_int], ct.c_int),
    ("bcr_set_stream", [_H, ct.c_void_p], ct.c_int),
    ("bcr_upload", [_H], ct.c_int),
    ("bcr_factorize_device", [_H], ct.c_int),
    ("bcr_factorize_async", [_H], ct.c_int),
    ("bcr_factorize_status", [_H], ct.c_int),
    ("bcr_solve_device", [_H, ct.c_int, ct.c_void_p, ct.c_int], ct.c_int),
    ("bcr_mv_device", [_H, ct.c_double, ct.c_void_p, ct.c_double, ct.c_void_p], ct.c_int),
    ("bcr_synchronize", [_H], ct.c_int),
    ("bcr_get_stream", [_H], ct.c_void_p),
    ("bcr_graph_capture", [_H, ct.c_int, ct.c_int, ct.c_void_p, ct.c_int, ct.c_void_p], ct.c_int),
    ("bcr_graph_launch", [_H, ct.c_int], ct.c_int),
    ("bcr_mv_noalloc", [ct.c_int] * 6 + [ct.c_void_p] * 7 + [ct.c_double, ct.c_void_p, ct.c_double,
                                                               ct.c_void_p, ct.c_void_p, ct.c_char_p,
                                                               ct.c_int], ct.c_int),
    ("bcr_batch_create", [ct.POINTER(ct.c_void_p)], ct.c_int),
    ("bcr_batch_destroy", [ct.c_void_p], ct.c_int),
    ("bcr_batch_add", [ct.c_void_p, _H], ct.c_int),
    ("bcr_batch_size", [ct.c_void_p], ct.c_int),
    ("bcr_batch_add_device", [ct.c_void_p] + [ct.c_int] * 6 + [ct.c_char_p], ct.c_int),
    ("bcr_batch_matrix", [ct.c_void_p, ct.c_int] + [ct.POINTER(ct.c_void_p)] * 7, ct.c_int),
    ("bcr_batch_system_size", [ct.c_void_p, ct.c_int, _ip, _ip], ct.c_int),
    ("bcr_batch_device_b", [ct.c_void_p, ct.c_int], ct.c_void_p),
    ("bcr_batch_load_device", [ct.c_void_p, ct.c_int] + [ct.c_void_p] * 7, ct.c_int),
    ("bcr_batch_prepare", [ct.c_void_p, ct.c_int], ct.c_int),
    ("bcr_batch_autotune", [ct.c_void_p], ct.c_int),
    ("bcr_batch_classes", [ct.c_void_p], ct.c_int),
    ("bcr_batch_class_info", [ct.c_void_p, ct.c_int, _ip, _ip, _ip, _ip], ct.c_int),
    ("bcr_batch_upload", [ct.c_void_p], ct.c_int),
    ("bcr_batch_factorize", [ct.c_void_p], ct.c_int),
    ("bcr_batch_status", [ct.c_void_p, _ip], ct.c_int),
    ("bcr_batch_solve", [ct.c_void_p, ct.POINTER(_dp)], ct.c_int),
    ("bcr_batch_factorize_solve", [ct.c_void_p, ct.POINTER(_dp)], ct.c_int),
    ("bcr_batch_set_rhs", [ct.c_void_p, ct.POINTER(_dp)], ct.c_int),
    ("bcr_batch_device_x", [ct.c_void_p, ct.c_int], ct.c_void_p),
    ("bcr_batch_get_x", [ct.c_void_p, ct.POINTER(_dp)], ct.c_int),
    ("bcr_batch_graph_capture", [ct.c_void_p], ct.c_int),
    ("bcr_batch_graph_launch", [ct.c_void_p], ct.c_int),
    ("bcr_batch_check_status", [ct.c_void_p], ct.c_int),
    ("bcr_batch_stream", [ct.c_void_p], ct.c_void_p),
    ("bcr_batch_synchronize", [ct.c_void_p], ct.c_int),
    ("bcr_batch_last_error", [ct.c_void_p], ct.c_char_p),
    ("bcr_batch_set_precision", [ct.c_void_p, ct.c_int], ct.c_int),
    ("bcr_batch_set_schedule", [ct.c_void_p, ct.c_int], ct.c_int),
    ("bcr_batch_set_refinement", [ct.c_void_p, ct.c_double, ct.c_int], ct.c_int),
    ("bcr_batch_refinement_info", [ct.c_void_p, ct.POINTER(ct.c_int), _dp], ct.c_int),
]

GRAPH_FACTORIZE, GRAPH_SOLVE, GRAPH_STEP = 1, 2, 3
BATCH_PERSISTENT, BATCH_LEVELS = 0, 1

_lib = None


def lib():
    """Load libalglin_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"alglin_b200: {LIB_PATH} is missing; run __graft_entry__.build()")
        L = ct.CDLL(LIB_PATH)
        for name, args, res in _SIGS:
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def mv_noalloc(dims, D, E, B, C, Cq, F, H, alpha, x, beta, res, stream=0):
    """Allocation-free res = alpha*A*x + beta*res on caller-owned device memory
    (every array argument is a device pointer, as an int).  Returns
    (status, message)."""
    buf = ct.create_string_buffer(256)
    rc = lib().bcr_mv_noalloc(*dims, D or None, E or None, B or None, C or None, Cq or None,
                              F or None, H or None, alpha, x or None, beta, res or None,
                              stream or None, buf, 256)
    return rc, buf.value.decode()


def exported_symbols():
    return [s[0] for s in _SIGS]


class BCRError(RuntimeError):
    pass


def _f64(a, shape=None) -> np.ndarray:
    """A column-major float64 view/copy of a 2-D matrix (math orientation)."""
    a = np.asarray(a, dtype=np.float64)
    if a.ndim == 1 and shape is not None:
        a = a.reshape(shape, order="F")
    return np.asfortranarray(a)


def _p(a: np.ndarray):
    return a.ctypes.data_as(_dp)


class BorderedCR:
    """Drop-in for ``alglin::BorderedCR<double>`` backed by the B200 kernels."""

    def __init__(self, num_threads: int = 0, num_parallel_block: int = 0):
        self.L = lib()
        self.h = _H()
        self._check(self.L.bcr_create(ct.byref(self.h), num_threads, num_parallel_block))

    def __del__(self):
        h = getattr(self, "h", None)
        if h is None or not h.value:
            return
        try:
            self.L.bcr_destroy(h)
            h.value = None
        except TypeError:
            pass  # interpreter shutdown: the library bindings are already gone

    # ------------------------------------------------------------- errors ---
    def last_error(self) -> str:
        return self.L.bcr_last_error(self.h).decode()

    def _check(self, rc: int, numerical_ok: bool = False):
        if rc == BCR_OK:
            return True
        if rc == BCR_NUMERICAL and numerical_ok:
            return False
        raise BCRError(f"alglin_b200 status {rc}: {self.last_error()}")

    # -------------------------------------------------------------- sizes ---
    def allocate(self, nblock, n, qr=0, qx=0, nr=0, nx=0):
        self._check(self.L.bcr_allocate(self.h, nblock, n, qr, qx, nr, nx))

    def dup(self, other: "BorderedCR"):
        self._check(self.L.bcr_dup(self.h, other.h))

    def nrows(self): return self.L.bcr_nrows(self.h)
    def ncols(self): return self.L.bcr_ncols(self.h)
    def number_of_blocks(self): return self.L.bcr_number_of_blocks(self.h)
    def block_size(self): return self.L.bcr_block_size(self.h)
    def dim_qr(self): return self.L.bcr_dim_qr(self.h)
    def dim_qx(self): return self.L.bcr_dim_qx(self.h)
    def dim_nr(self): return self.L.bcr_dim_nr(self.h)
    def dim_nx(self): return self.L.bcr_dim_nx(self.h)
    def Nr(self): return self.L.bcr_Nr(self.h)
    def Nc(self): return self.L.bcr_Nc(self.h)

    # ------------------------------------------------------------ zeroing ---
    def zero_B(self): self._check(self.L.bcr_zero_B(self.h))
    def zero_C(self): self._check(self.L.bcr_zero_C(self.h))
    def zero_Cq(self): self._check(self.L.bcr_zero_Cq(self.h))
    def zero_D(self): self._check(self.L.bcr_zero_D(self.h))
    def zero_E(self): self._check(self.L.bcr_zero_E(self.h))
    def zero_F(self): self._check(self.L.bcr_zero_F(self.h))
    def zero_H(self): self._check(self.L.bcr_zero_H(self.h))
    def fill_zero(self): self._check(self.L.bcr_fill_zero(self.h))

    # ------------------------------------------------------------ loaders ---
    def _blk(self, fn, nbl, M):
        M = _f64(M)
        self._check(fn(self.h, nbl, _p(M), max(M.shape[0], 1)))

    def load_B(self, nbl, B): self._blk(self.L.bcr_load_B, nbl, B)
    def add_to_B(self, nbl, B): self._blk(self.L.bcr_add_to_B, nbl, B)
    def load_C(self, nbl, C): self._blk(self.L.bcr_load_C, nbl, C)
    def add_to_C(self, nbl, C): self._blk(self.L.bcr_add_to_C, nbl, C)
    def add_to_C2(self, nbl, C): self._blk(self.L.bcr_add_to_C2, nbl, C)
    def add_to_C2F(self, nbl, C): self._blk(self.L.bcr_add_to_C2F, nbl, C)
    def load_D(self, nbl, D): self._blk(self.L.bcr_load_D, nbl, D)
    def load_E(self, nbl, E): self._blk(self.L.bcr_load_E, nbl, E)
    def load_DE(self, nbl, DE): self._blk(self.L.bcr_load_DE, nbl, DE)
    def load_DEB(self, nbl, DEB): self._blk(self.L.bcr_load_DEB, nbl, DEB)

    def _one(self, fn, M):
        M = _f64(M)
        self._check(fn(self.h, _p(M), max(M.shape[0], 1)))

    def load_F(self, F): self._one(self.L.bcr_load_F, F)
    def add_to_F(self, F): self._one(self.L.bcr_add_to_F, F)
    def load_Cq(self, Cq): self._one(self.L.bcr_load_Cq, Cq)
    def load_CqF(self, CqF): self._one(self.L.bcr_load_CqF, CqF)

    def load_bottom(self, H0, HN=None, Hq=None, Hp=None):
        if HN is None:  # the concatenated [H0 | HN | Hq | Hp]
            self._one(self.L.bcr_load_bottom_H, H0)
            return
        m = self.block_size() + self.dim_qr()
        mats = [_f64(M).reshape(m, -1, order="F") for M in (H0, HN, Hq, Hp)]
        args = []
        for M in mats:
            args += [_p(M), m]
        self._check(self.L.bcr_load_bottom(self.h, *args))

    def load_bottom2(self, C0, CN=None, Cq=None, F=None):
        if CN is None:
            self._one(self.L.bcr_load_bottom2_H, C0)
            return
        nr = max(self.dim_nr(), 1)
        mats = [_f64(M).reshape(nr, -1, order="F") for M in (C0, CN, Cq, F)]
        args = []
        for M in mats:
            args += [_p(M), nr]
        self._check(self.L.bcr_load_bottom2(self.h, *args))

    # whole-matrix load from reference-layout arrays (see alglin_b200.synth)
    def load_system(self, s):
        self.allocate(*s.dims())
        for which, arr in (("D", s.D), ("E", s.E), ("B", s.B), ("C", s.C), ("Q", s.Cq),
                           ("F", s.F), ("H", s.H)):
            a = np.ascontiguousarray(arr, dtype=np.float64)
            if a.size == 0:
                continue
            ptr = self.L.bcr_block_data(self.h, which.encode(), 0)
            ct.memmove(ptr, a.ctypes.data, a.nbytes)

    # element access: views of the host copy (reference accessors hxx:972-998)
    def _view(self, which, nbl, rows, cols):
        ptr = self.L.bcr_block_data(self.h, which.encode(), nbl)
        if not ptr or rows * cols == 0:
            return np.zeros((rows, cols))
        buf = np.ctypeslib.as_array(ptr, shape=(rows * cols,))
        return buf.reshape((rows, cols), order="F")

    def D(self, nbl): return self._view("D", nbl, self.block_size(), self.block_size())
    def E(self, nbl): return self._view("E", nbl, self.block_size(), self.block_size())
    def B(self, nbl): return self._view("B", nbl, self.block_size(), self.dim_nx())
    def C(self, nbl): return self._view("C", nbl, self.dim_nr(), self.block_size())
    def F(self): return self._view("F", 0, self.dim_nr(), self.dim_nx())
    def Cq(self): return self._view("Q", 0, self.dim_nr(), self.dim_qx())
    def H(self): return self._view("H", 0, self.block_size() + self.dim_qr(), self.Nc())

    # ---------------------------------------------------------- selection ---
    def select(self, s): self._check(self.L.bcr_select(self.h, s.encode()))
    def select_LU(self): self.select("LU")
    def select_QR(self): self.select("QR")
    def select_QRP(self): self.select("QRP")
    def select_last(self, s): self._check(self.L.bcr_select_last(self.h, s.encode()))
    def select_last2(self, s): self._check(self.L.bcr_select_last2(self.h, s.encode()))
    def set_factorize_use_thread(self, yes): self._check(self.L.bcr_set_factorize_use_thread(self.h, int(yes)))
    def set_solve_use_thread(self, yes): self._check(self.L.bcr_set_solve_use_thread(self.h, int(yes)))
    def factorize_use_thread(self): return bool(self.L.bcr_factorize_use_thread(self.h))
    def solve_use_thread(self): return bool(self.L.bcr_solve_use_thread(self.h))
    def set_num_parallel_block(self, npb): self._check(self.L.bcr_set_num_parallel_block(self.h, npb))
    def set_precision(self, p): self._check(self.L.bcr_set_precision(self.h, p))

    def set_pair_kernel(self, choice: int):
        """Force a pair-kernel family (PAIR_AUTO, PAIR_TC, PAIR_GRP, PAIR_ROWS, PAIR_CTA, PAIR_SMEM, PAIR_UMMA,
        PAIR_TREE)."""
        self._check(self.L.bcr_set_pair_kernel(self.h, int(choice)))

    def set_refinement(self, tol: float = 1e-12, max_iter: int = 10):
        """Stopping rule of the mixed path's iterative refinement."""
        self._check(self.L.bcr_set_refinement(self.h, float(tol), int(max_iter)))

    def refinement_info(self) -> tuple[int, float]:
        """(corrections applied, final |b-Ax|/(|A||x|+|b|)) of the last mixed solve."""
        it = ct.c_int(0)
        rr = ct.c_double(0.0)
        self._check(self.L.bcr_refinement_info(self.h, ct.byref(it), ct.byref(rr)))
        return it.value, rr.value
    def set_debug(self, yes): self._check(self.L.bcr_set_debug(self.h, int(yes)))
    def check_matrix(self): self._check(self.L.bcr_check_matrix(self.h))

    def info(self, indent: str = "") -> str:
        return self.L.bcr_info(self.h, indent.encode()).decode()

    def _names(self):
        a, b, c = ct.c_int(), ct.c_int(), ct.c_int()
        self.L.bcr_selected(self.h, ct.byref(a), ct.byref(b), ct.byref(c))
        return a.value, b.value, c.value

    def info_algo_block(self):
        return ["CyclicReduction+LU", "CyclicReduction+QR", "CyclicReduction+QRP"][self._names()[0]]

    def info_algo_last_block(self):
        return "LastBlock " + ["LU", "LUPQ", "QR", "QRP", "SVD", "LSS", "LSY", "PINV"][self._names()[1]]

    def info_algo_last_block2(self):
        return "LastBlock " + ["NONE", "SVD", "LSS", "LSY", "PINV"][self._names()[2]]

    # ------------------------------------------------------ factor / solve ---
    def factorize(self) -> bool:
        return self._check(self.L.bcr_factorize(self.h), numerical_ok=True)

    def solve(self, x: np.ndarray) -> bool:
        """In place on a float64 vector of length >= max(nrows, ncols)."""
        assert x.dtype == np.float64 and x.flags.c_contiguous and x.ndim == 1
        assert x.size >= max(self.nrows(), self.ncols())
        return self._check(self.L.bcr_solve(self.h, _p(x)), numerical_ok=True)

    def solve_n(self, nrhs: int, X: np.ndarray, ld: int) -> bool:
        """In place on a float64 buffer holding nrhs columns of stride ld."""
        assert X.dtype == np.float64 and X.flags.c_contiguous and X.size >= nrhs * ld
        return self._check(self.L.bcr_solve_n(self.h, nrhs, _p(X), ld), numerical_ok=True)

    def factorize_solve(self, nrhs: int, X: np.ndarray, ld: int) -> bool:
        """factorize() then solve_n(nrhs, X, ld) in one pass (in place on X)."""
        assert X.dtype == np.float64 and X.flags.c_contiguous and X.size >= nrhs * ld
        return self._check(self.L.bcr_factorize_solve(self.h, nrhs, _p(X), ld), numerical_ok=True)

    def factorize_solve_device(self, nrhs: int, d_x_ptr: int, ld: int):
        self._check(self.L.bcr_factorize_solve_device(self.h, nrhs, d_x_ptr, ld))

    def t_solve(self, x):
        return self._check(self.L.bcr_t_solve(self.h, _p(np.asarray(x, dtype=np.float64))))

    def mv(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        res = np.zeros(max(self.nrows(), 1))
        self._check(self.L.bcr_mv(self.h, _p(x), _p(res)))
        return res

    def add_mv(self, alpha: float, x: np.ndarray, res: np.ndarray):
        x = np.ascontiguousarray(x, dtype=np.float64)
        assert res.dtype == np.float64 and res.flags.c_contiguous
        self._check(self.L.bcr_add_mv(self.h, alpha, _p(x), _p(res)))

    # ------------------------------------------------------------- sparse ---
    def sparse_nnz(self): return self.L.bcr_sparse_nnz(self.h)

    def sparse_pattern(self, offs: int = 0):
        nnz = self.sparse_nnz()
        I = np.zeros(nnz, dtype=np.int32)
        J = np.zeros(nnz, dtype=np.int32)
        self._check(self.L.bcr_sparse_pattern(self.h, I.ctypes.data_as(_ip), J.ctypes.data_as(_ip), offs))
        return I, J

    def sparse_values(self):
        V = np.zeros(self.sparse_nnz())
        self._check(self.L.bcr_sparse_values(self.h, _p(V)))
        return V

    def sparse_load(self, V, I, r_offs, J, c_offs, do_error=True):
        V = np.ascontiguousarray(V, dtype=np.float64)
        I = np.ascontiguousarray(I, dtype=np.int32)
        J = np.ascontiguousarray(J, dtype=np.int32)
        self._check(self.L.bcr_sparse_load(self.h, _p(V), I.ctypes.data_as(_ip), r_offs,
                                           J.ctypes.data_as(_ip), c_offs, V.size, int(do_error)))

    # ---------------------------------------------------- device-resident ---
    def set_stream(self, stream_ptr: int): self._check(self.L.bcr_set_stream(self.h, stream_ptr))
    def upload(self): self._check(self.L.bcr_upload(self.h))

    def factorize_device(self) -> bool:
        return self._check(self.L.bcr_factorize_device(self.h), numerical_ok=True)

    def factorize_async(self):
        """Enqueue the factorization (graph-capturable); see factorize_status()."""
        self._check(self.L.bcr_factorize_async(self.h))

    def factorize_status(self) -> bool:
        return self._check(self.L.bcr_factorize_status(self.h), numerical_ok=True)

    def solve_device(self, nrhs: int, d_x_ptr: int, ld: int) -> bool:
        return self._check(self.L.bcr_solve_device(self.h, nrhs, d_x_ptr, ld), numerical_ok=True)

    def mv_device(self, alpha, d_x_ptr, beta, d_res_ptr):
        self._check(self.L.bcr_mv_device(self.h, alpha, d_x_ptr, beta, d_res_ptr))

    def synchronize(self): self._check(self.L.bcr_synchronize(self.h))

    def stream(self) -> int:
        """cudaStream_t (as an int) the handle enqueues on."""
        return self.L.bcr_get_stream(self.h) or 0

    def graph_capture(self, what: int, nrhs: int = 0, d_x_ptr: int = 0, ld: int = 0, d_rhs_ptr: int = 0):
        self._check(self.L.bcr_graph_capture(self.h, what, nrhs, d_x_ptr or None, ld, d_rhs_ptr or None))

    def graph_launch(self, what: int):
        self._check(self.L.bcr_graph_launch(self.h, what))


class Batch:
    """Many independent BorderedCR systems factored and solved together on the
    device (FP64, internal LU).  The BorderedCR objects must outlive the batch."""

    def __init__(self, systems=()):
        self.L = lib()
        self.b = ct.c_void_p()
        self._check(self.L.bcr_batch_create(ct.byref(self.b)))
        self.systems = []
        for h in systems:
            self.add(h)

    def __del__(self):
        b = getattr(self, "b", None)
        if b is None or not b.value:
            return
        try:
            self.L.bcr_batch_destroy(b)
            b.value = None
        except TypeError:
            pass  # interpreter shutdown

    def last_error(self) -> str:
        return self.L.bcr_batch_last_error(self.b).decode()

    def _check(self, rc: int, numerical_ok: bool = False):
        if rc == BCR_OK:
            return True
        if rc == BCR_NUMERICAL and numerical_ok:
            return False
        raise BCRError(f"alglin_b200 batch status {rc}: {self.last_error()}")

    def add(self, h: "BorderedCR"):
        self._check(self.L.bcr_batch_add(self.b, h.h))
        self.systems.append(h)

    def add_device(self, nblock, n, qr=0, qx=0, nr=0, nx=0, last="LU"):
        """A system whose blocks are written on the device (see matrix())."""
        self._check(self.L.bcr_batch_add_device(self.b, nblock, n, qr, qx, nr, nx, last.encode()))
        self.systems.append(None)

    def matrix(self, i: int) -> dict:
        """Device addresses of system i's blocks D, E, B, C, Cq, F, H (reference layout)."""
        v = [ct.c_void_p() for _ in range(7)]
        self._check(self.L.bcr_batch_matrix(self.b, i, *[ct.byref(x) for x in v]))
        return dict(zip("D E B C Cq F H".split(), [x.value or 0 for x in v]))

    def system_size(self, i: int):
        r, c = ct.c_int(), ct.c_int()
        self._check(self.L.bcr_batch_system_size(self.b, i, ct.byref(r), ct.byref(c)))
        return r.value, c.value

    def load_device(self, i: int, D=0, E=0, B=0, C=0, Cq=0, F=0, H=0):
        """Copy system i's blocks from device addresses (ints; 0 skips a block)."""
        self._check(self.L.bcr_batch_load_device(self.b, i, D or None, E or None, B or None, C or None,
                                                 Cq or None, F or None, H or None))

    def device_b(self, i: int) -> int:
        return self.L.bcr_batch_device_b(self.b, i) or 0

    def __len__(self):
        return self.L.bcr_batch_size(self.b)

    def set_precision(self, p: int):
        """PRECISION_FP64 or PRECISION_MIXED (FP32 factors + FP64 refinement); before prepare()."""
        self._check(self.L.bcr_batch_set_precision(self.b, int(p)))

    def set_refinement(self, tol: float = 1e-12, max_iter: int = 10):
        self._check(self.L.bcr_batch_set_refinement(self.b, float(tol), int(max_iter)))

    def set_schedule(self, schedule: int):
        """BATCH_LEVELS (default: one launch per level) or BATCH_PERSISTENT (one
        persistent launch per class with a per-system level schedule); before prepare()."""
        self._check(self.L.bcr_batch_set_schedule(self.b, int(schedule)))

    def refinement_info(self):
        """(corrections applied, worst |b-Ax|/(|A||x|+|b|) over the batch) of the last mixed solve."""
        it = ct.c_int(0)
        rr = ct.c_double(0.0)
        self._check(self.L.bcr_batch_refinement_info(self.b, ct.byref(it), ct.byref(rr)))
        return it.value, rr.value

    def prepare(self, autotune: bool = False):
        self._check(self.L.bcr_batch_prepare(self.b, 1 if autotune else 0))

    def autotune(self):
        """Time every applicable kernel family and chunk on the loaded systems; keep the fastest."""
        self._check(self.L.bcr_batch_autotune(self.b))

    def classes(self):
        """[(n, systems, family, pairs per CTA)] of every kernel group."""
        out = []
        for c in range(self.L.bcr_batch_classes(self.b)):
            v = [ct.c_int() for _ in range(4)]
            self._check(self.L.bcr_batch_class_info(self.b, c, *[ct.byref(x) for x in v]))
            out.append(tuple(x.value for x in v))
        return out

    def upload(self):
        self._check(self.L.bcr_batch_upload(self.b))

    def factorize(self) -> bool:
        return self._check(self.L.bcr_batch_factorize(self.b), numerical_ok=True)

    def status(self) -> np.ndarray:
        codes = np.zeros(len(self), dtype=np.int32)
        self._check(self.L.bcr_batch_status(self.b, codes.ctypes.data_as(_ip)))
        return codes

    @staticmethod
    def _ptrs(xs):
        for x in xs:
            assert x.dtype == np.float64 and x.flags.c_contiguous
        return (_dp * len(xs))(*[x.ctypes.data_as(_dp) for x in xs])

    def solve(self, xs) -> bool:
        """In place on one float64 vector (length >= max(nrows, ncols)) per system."""
        return self._check(self.L.bcr_batch_solve(self.b, self._ptrs(xs)), numerical_ok=True)

    def factorize_solve(self, xs) -> bool:
        return self._check(self.L.bcr_batch_factorize_solve(self.b, self._ptrs(xs)), numerical_ok=True)

    def set_rhs(self, bs):
        self._check(self.L.bcr_batch_set_rhs(self.b, self._ptrs(bs)))

    def get_x(self, xs):
        self._check(self.L.bcr_batch_get_x(self.b, self._ptrs(xs)))

    def device_x(self, i: int) -> int:
        return self.L.bcr_batch_device_x(self.b, i) or 0

    def graph_capture(self):
        self._check(self.L.bcr_batch_graph_capture(self.b), numerical_ok=False)

    def graph_launch(self):
        self._check(self.L.bcr_batch_graph_launch(self.b))

    def check_status(self) -> bool:
        return self._check(self.L.bcr_batch_check_status(self.b), numerical_ok=True)

    def stream(self) -> int:
        return self.L.bcr_batch_stream(self.b) or 0

    def synchronize(self):
        self._check(self.L.bcr_batch_synchronize(self.b))
