"""Seeded synthetic BABD systems for the BorderedCR benchmarks and tests.

The arrays use the reference storage layout of ``alglin::BorderedCR``
(src/Alglin/BABD_BorderedCR.hxx:972-998): every block is column-major, so a
block of ``r`` rows and ``c`` columns is held as a C-ordered ``(c, r)`` array
(``blk[j, i]`` is element ``(i, j)``).

    D, E : (nblock,   n,  n)      B  : (nblock, nx, n)
    C    : (nblock+1, n,  nr)     Cq : (qx, nr)        F : (nx, nr)
    H    : (Nc, n+qr)  with H = [H0 | HN | Hq | Hp],  Nc = 2n+qx+nx

Workloads (``N(m, v)`` has mean m and variance v):

* trapezoid collocation of x' = J_k x on a uniform mesh, h = 1/nblock:
  J_k iid N(0, kappa/n), D_k = -I - (h/2) J_k, E_k = I - (h/2) J_k;
* B_k, C_k (k = 0..nblock) N(0, 0.1); F = I + N(0, 0.1);
* H0 = [I_{n/2} 0; 0 0] + N(0, 0.01), HN = [0 0; 0 I_{n/2}] + N(0, 0.01)
  (the qr extra rows are pure N(0, 0.01) noise); Hq N(0, 1); Hp N(0, 0.01);
  Cq N(0, 0.1); right-hand sides N(0, 1).
"""
from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass
class BABD:
    nblock: int
    n: int
    qr: int
    qx: int
    nr: int
    nx: int
    D: np.ndarray
    E: np.ndarray
    B: np.ndarray
    C: np.ndarray
    Cq: np.ndarray
    F: np.ndarray
    H: np.ndarray

    @property
    def nrows(self) -> int:
        return self.n * (self.nblock + 1) + self.qr + self.nr

    @property
    def ncols(self) -> int:
        return self.n * (self.nblock + 1) + self.qx + self.nx

    @property
    def Nr(self) -> int:
        return 2 * self.n + self.qr + self.nr

    @property
    def Nc(self) -> int:
        return 2 * self.n + self.qx + self.nx

    def dims(self):
        return (self.nblock, self.n, self.qr, self.qx, self.nr, self.nx)

    def copy(self) -> "BABD":
        return dataclasses.replace(
            self, **{k: getattr(self, k).copy() for k in ("D", "E", "B", "C", "Cq", "F", "H")})

    def norm_inf(self) -> float:
        """||A||_inf (largest absolute row sum) from the blocks."""
        rows = np.abs(self.D).sum(axis=1) + np.abs(self.E).sum(axis=1) + np.abs(self.B).sum(axis=1)
        m = float(rows.max()) if rows.size else 0.0
        if self.H.size:
            m = max(m, float(np.abs(self.H).sum(axis=0).max()))
        if self.nr:
            c = np.abs(self.C).sum(axis=(0, 1)) + np.abs(self.Cq).sum(axis=0) + np.abs(self.F).sum(axis=0)
            m = max(m, float(c.max()))
        return m

    def to_dense(self) -> np.ndarray:
        """Dense matrix (row-major numpy) for small cross-checks."""
        nb, n, qr, qx, nr, nx = self.dims()
        A = np.zeros((self.nrows, self.ncols))
        cb = (nb + 1) * n + qx
        for k in range(nb):
            A[k * n:(k + 1) * n, k * n:(k + 1) * n] = self.D[k].T
            A[k * n:(k + 1) * n, (k + 1) * n:(k + 2) * n] = self.E[k].T
            A[k * n:(k + 1) * n, cb:cb + nx] = self.B[k].T
        Hm = self.H.T  # (n+qr) x Nc
        r0 = nb * n
        A[r0:r0 + n + qr, 0:n] = Hm[:, 0:n]
        A[r0:r0 + n + qr, nb * n:(nb + 1) * n] = Hm[:, n:2 * n]
        A[r0:r0 + n + qr, (nb + 1) * n:(nb + 1) * n + qx + nx] = Hm[:, 2 * n:]
        rc = r0 + n + qr
        for k in range(nb + 1):
            A[rc:rc + nr, k * n:(k + 1) * n] = self.C[k].T
        A[rc:rc + nr, (nb + 1) * n:(nb + 1) * n + qx] = self.Cq.T
        A[rc:rc + nr, cb:cb + nx] = self.F.T
        return A


def _zeros(nblock, n, qr, qx, nr, nx) -> BABD:
    Nc = 2 * n + qx + nx
    return BABD(nblock, n, qr, qx, nr, nx,
                D=np.zeros((nblock, n, n)), E=np.zeros((nblock, n, n)),
                B=np.zeros((nblock, nx, n)), C=np.zeros((nblock + 1, n, nr)),
                Cq=np.zeros((qx, nr)), F=np.zeros((nx, nr)), H=np.zeros((Nc, n + qr)))


def collocation(nblock: int, n: int, qr: int = 0, qx: int = 0, nr: int = 0, nx: int = 0,
                kappa: float = 1.0, seed: int = 0) -> BABD:
    """Trapezoid-collocation BABD system (see module docstring)."""
    rng = np.random.default_rng(seed)
    s = _zeros(nblock, n, qr, qx, nr, nx)
    h = 1.0 / nblock
    J = rng.standard_normal((nblock, n, n)) * np.sqrt(kappa / n)
    eye = np.eye(n)
    # column-major storage: the stored (j, i) entry is element (i, j); D = -I - h/2 J
    Jt = np.ascontiguousarray(J.transpose(0, 2, 1))
    s.D[:] = -eye - 0.5 * h * Jt
    s.E[:] = eye - 0.5 * h * Jt
    s.B[:] = rng.standard_normal(s.B.shape) * np.sqrt(0.1)
    s.C[:] = rng.standard_normal(s.C.shape) * np.sqrt(0.1)
    s.F[:] = rng.standard_normal(s.F.shape) * np.sqrt(0.1)
    for i in range(min(nr, nx)):
        s.F[i, i] += 1.0
    s.Cq[:] = rng.standard_normal(s.Cq.shape) * np.sqrt(0.1)
    m = n + qr
    Hm = np.zeros((m, s.Nc))
    Hm[:, 0:2 * n] = rng.standard_normal((m, 2 * n)) * np.sqrt(0.01)
    half = n // 2
    for i in range(half):
        Hm[i, i] += 1.0                      # H0 = [I_{n/2} 0; 0 0]
    for i in range(half, n):
        Hm[i, n + i] += 1.0                  # HN = [0 0; 0 I_{n/2}]
    Hm[:, 2 * n:2 * n + qx] = rng.standard_normal((m, qx))
    Hm[:, 2 * n + qx:] = rng.standard_normal((m, nx)) * np.sqrt(0.01)
    s.H[:] = Hm.T
    return s


def dominant(nblock: int, n: int, qr: int, qx: int, nr: int, nx: int, seed: int = 2) -> BABD:
    """Diagonally dominant random system in the style of the reference's
    test7/test16 generator (src_tests/test7-BorderedCR.cc:49-100): U(-1,0)
    entries plus 1.01*n on the diagonals of D, H(:, n:) and F, borders
    U(-0.1, 0.1), C_nblock = 1."""
    rng = np.random.default_rng(seed)
    s = _zeros(nblock, n, qr, qx, nr, nx)
    diag = 1.01 * n
    Hm = rng.uniform(-1, 0, (n + qr, s.Nc))
    for i in range(n + qr):
        if i + n < s.Nc:
            Hm[i, i + n] += diag
    s.H[:] = Hm.T
    s.D[:] = rng.uniform(-1, 0, s.D.shape)
    s.E[:] = rng.uniform(-1, 0, s.E.shape)
    idx = np.arange(n)
    s.D[:, idx, idx] += diag
    s.B[:] = rng.uniform(-0.1, 0.1, s.B.shape)
    s.C[:nblock] = rng.uniform(-0.1, 0.1, (nblock, n, nr))
    s.C[nblock] = 1.0
    s.F[:] = rng.uniform(-0.1, 0.1, s.F.shape)
    for i in range(min(nr, nx)):
        s.F[i, i] += diag
    s.Cq[:] = rng.uniform(-0.1, 0.1, s.Cq.shape)
    return s


def stable_small(nblock: int = 6, n: int = 2, qr: int = 1, qx: int = 2, nr: int = 3,
                 nx: int = 2) -> BABD:
    """Deterministic well-conditioned system with the closed-form entries of the
    reference coverage test (src_tests/test18-BorderedCR-coverage.cc:163-230)."""
    s = _zeros(nblock, n, qr, qx, nr, nx)
    m = n + qr
    for k in range(nblock):
        s.D[k, 0, 0] = 5.0 + 0.2 * k
        s.D[k, 0, 1] = 0.15      # D(k,1,0)
        s.D[k, 1, 0] = -0.08     # D(k,0,1)
        s.D[k, 1, 1] = 4.7 + 0.2 * k
        s.E[k, 0, 0] = -0.35
        s.E[k, 0, 1] = 0.04
        s.E[k, 1, 0] = 0.06
        s.E[k, 1, 1] = -0.28
        for j in range(nx):
            for i in range(n):
                s.B[k, j, i] = 0.04 * (1 + k + i + 2 * j)
        for j in range(n):
            for i in range(nr):
                s.C[k, j, i] = 0.03 * (1 + 2 * k + i + j)
    for j in range(n):
        for i in range(nr):
            s.C[nblock, j, i] = 0.05 * (1 + i + j)
    for j in range(qx):
        for i in range(nr):
            s.Cq[j, i] = 0.07 * (1 + i + 2 * j)
    for j in range(nx):
        for i in range(nr):
            s.F[j, i] = 0.02 * (1 + i + j)
    s.F[0, 0] += 3.2
    s.F[1, 1] += 2.8
    Hm = np.zeros((m, s.Nc))
    for j in range(n):
        for i in range(m):
            Hm[i, j] = 0.02 * (1 + i + j)
            Hm[i, n + j] = 0.03 * (1 + i + j)
    Hm[0, n + 0] += 5.1
    Hm[1, n + 1] += 4.9
    Hm[2, n + 0] += 0.2
    Hm[2, n + 1] -= 0.25
    for j in range(qx):
        for i in range(m):
            Hm[i, 2 * n + j] = 0.04 * (1 + i + j)
    for j in range(nx):
        for i in range(m):
            Hm[i, 2 * n + qx + j] = 0.05 * (1 + i + j)
    s.H[:] = Hm.T
    return s


# workloads named in the benchmark plan (sizes of the reference's headline path)
CONFIGS = {
    "A": dict(nblock=1000, n=8, qr=0, qx=0, nr=2, nx=2),
    "B": dict(nblock=100000, n=16, qr=2, qx=2, nr=4, nx=4),
    "C": dict(nblock=65536, n=32, qr=0, qx=0, nr=8, nx=8),
    "E": dict(nblock=8192, n=128, qr=4, qx=4, nr=16, nx=16),
}


def rhs(s: BABD, nrhs: int = 1, seed: int = 1) -> np.ndarray:
    """N(0,1) right-hand sides, column-major (nrhs, max(nrows, ncols))."""
    rng = np.random.default_rng(seed)
    L = max(s.nrows, s.ncols)
    b = np.zeros((nrhs, L))
    b[:, :s.nrows] = rng.standard_normal((nrhs, s.nrows))
    return b


def batch_dims(nsys: int, nblock_lo: int = 64, nblock_hi: int = 4096, ns=(4, 8, 16, 32),
               borders=(0, 2, 4), seed: int = 0):
    """Sizes of the uneven batch workload: nblock ~ U{lo..hi}, n drawn from ns,
    nr = nx drawn from borders, qr = qx = 0; system s is then generated by
    collocation(..., seed=s)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(nsys):
        nb = int(rng.integers(nblock_lo, nblock_hi + 1))
        n = int(rng.choice(ns))
        b = int(rng.choice(borders))
        out.append((nb, n, 0, 0, b, b))
    return out


def collocation_torch(torch, nblock, n, qr=0, qx=0, nr=0, nx=0, kappa=1.0, seed=0, device="cuda"):
    """The collocation generator's distributions drawn on the device with torch
    (its own random stream, so the values differ from collocation()); returns
    contiguous float64 tensors D, E, B, C, Cq, F, H in the reference layout."""
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    f64 = torch.float64
    h = 1.0 / nblock
    J = torch.randn((nblock, n, n), generator=g, device=device, dtype=f64) * (kappa / n) ** 0.5
    eye = torch.eye(n, device=device, dtype=f64)
    D = (-eye - 0.5 * h * J).contiguous()
    E = (eye - 0.5 * h * J).contiguous()
    B = torch.randn((nblock, nx, n), generator=g, device=device, dtype=f64) * 0.1 ** 0.5
    C = torch.randn((nblock + 1, n, nr), generator=g, device=device, dtype=f64) * 0.1 ** 0.5
    F = torch.randn((nx, nr), generator=g, device=device, dtype=f64) * 0.1 ** 0.5
    for i in range(min(nr, nx)):
        F[i, i] += 1.0
    Cq = torch.randn((qx, nr), generator=g, device=device, dtype=f64) * 0.1 ** 0.5
    m, Nc = n + qr, 2 * n + qx + nx
    Hm = torch.zeros((m, Nc), device=device, dtype=f64)
    Hm[:, 0:2 * n] = torch.randn((m, 2 * n), generator=g, device=device, dtype=f64) * 0.1
    half = n // 2
    idx = torch.arange(half, device=device)
    Hm[idx, idx] += 1.0
    idx2 = torch.arange(half, n, device=device)
    Hm[idx2, n + idx2] += 1.0
    Hm[:, 2 * n:2 * n + qx] = torch.randn((m, qx), generator=g, device=device, dtype=f64)
    Hm[:, 2 * n + qx:] = torch.randn((m, nx), generator=g, device=device, dtype=f64) * 0.1
    H = Hm.t().contiguous()
    return D, E, B, C, Cq, F, H
