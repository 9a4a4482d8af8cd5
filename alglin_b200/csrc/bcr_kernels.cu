// BorderedCR device kernels, FP64 path (sm_100a).
//
// One cyclic-reduction (CR) level is one launch of k_factor_level: every pair
// (jp = j-k, j) of the level is independent, and one warp eliminates one pair.
// The warp stages the pair's row blocks in shared memory as one
// (2n + nr) x (3n + nx) work matrix
//
//                x_j      x_jp     x_jpp    xb
//   TOP    [  E_jp  |  D_jp  |   0    | B_jp ]   row block jp
//   BOTTOM [  D_j   |   0    |  E_j   | B_j  ]   row block j
//   border [  C_j   |   0    |   0    |  0   ]   nr border rows
//
// and eliminates x_j from it: partial-pivot LU or Householder QR on the 2n x n
// panel (buildT, BABD_BorderedCR.cc:845-898), applied to the trailing columns
// (applyT, cc:917-982) and, through the U rows, to the border rows (the C/F
// Schur updates of factorize_block, cc:1107-1154).  After elimination
//   rows 0..n-1   hold the U-row  [U | D'_j | E'_j | B'_j ]  (back-substitution)
//   rows n..2n-1  hold the reduced row [0 | D'_jp | E'_jp | B'_jp]
//   border rows   hold [C_j U^-1 | dC_jp | dC_jpp | dF]
// dC_jp is added to C_jp by the owning warp (no other pair of the level writes
// C_jp); dC_jpp goes to a per-block scratch slot and is added to C_jpp by
// k_border_fix after the level, because C_jpp is also C_jp of pair j+2k.
// The F updates dF go to a per-block slot and are summed in a fixed order.
#include <cstdio>

#include "bcr_device.h"

namespace bcr {

static constexpr int WARPS_PANEL = 4;
static constexpr size_t SMEM_MAX = 227 * 1024;

template <typename T>
struct FactorArgs {
  Dims d;
  const double *D0, *E0, *B0, *C0;  // loaded matrix, read at the first level
  T *D, *E, *B, *C;                  // working blocks
  T* Tm;
  int* P;
  T *Rbuf, *Fbuf;
  StatusWords* st;
  int k, first, ldw;
};

__host__ __device__ inline int odd_ld(int r) { return r | 1; }

size_t panel_smem_per_warp(const Dims& d, int elem_bytes) {
  const int R = 2 * d.n + d.nr, NC = 3 * d.n + d.nx;
  size_t b = (size_t)odd_ld(R) * NC * elem_bytes + (size_t)d.n * (elem_bytes + sizeof(int));
  return b;
}

// ---------------------------------------------------------------------------
// warp-level elimination of x_j from the staged work matrix
// ---------------------------------------------------------------------------
template <typename T>
__device__ int warp_eliminate_lu(T* W, int ldw, int n, int R, int NC, int* ipiv, int lane) {
  const int n2 = 2 * n;
  for (int i = 0; i < n; ++i) {
    T* ci = W + (size_t)i * ldw;
    T best = T(-1);
    int bi = i;  // stays in range even when every candidate is NaN
    for (int r = i + lane; r < n2; r += 32) {
      T v = dev_abs(ci[r]);
      if (v > best) { best = v; bi = r; }
    }
    warp_argmax(best, bi);
    if (lane == 0) ipiv[i] = bi;
    const T pv = ci[bi];
    if (pv == T(0)) return i + 1;  // LAPACK getrf INFO
    if (bi != i)
      for (int c = lane; c < NC; c += 32) {
        T* col = W + (size_t)c * ldw;
        T t = col[i]; col[i] = col[bi]; col[bi] = t;
      }
    __syncwarp();
    const T rinv = T(1) / pv;
    for (int r = i + 1 + lane; r < R; r += 32) ci[r] *= rinv;
    __syncwarp();
    for (int c = i + 1 + lane; c < NC; c += 32) {
      T* col = W + (size_t)c * ldw;
      const T u = col[i];
      if (u != T(0))
        for (int r = i + 1; r < R; ++r) col[r] -= ci[r] * u;
    }
    __syncwarp();
  }
  return 0;
}

// Householder QR (optionally with column pivoting) of the panel; the border
// rows are eliminated with the finished R rows.  Returns i+1 if R(i,i) == 0.
template <typename T, bool PIVOT>
__device__ int warp_eliminate_qr(T* W, int ldw, int n, int R, int NC, int* ipiv, T* tau, int lane) {
  const int n2 = 2 * n;
  for (int i = 0; i < n; ++i) {
    if (PIVOT) {
      // largest remaining column 2-norm over the panel rows i..2n-1
      T best = T(-1);
      int bc = i;
      for (int c = i + lane; c < n; c += 32) {
        const T* col = W + (size_t)c * ldw;
        T s = T(0);
        for (int r = i; r < n2; ++r) s += col[r] * col[r];
        if (s > best) { best = s; bc = c; }
      }
      warp_argmax(best, bc);
      if (lane == 0) ipiv[i] = bc;
      if (bc != i)
        for (int r = lane; r < R; r += 32) {
          T t = W[(size_t)i * ldw + r];
          W[(size_t)i * ldw + r] = W[(size_t)bc * ldw + r];
          W[(size_t)bc * ldw + r] = t;
        }
      __syncwarp();
    } else if (lane == 0) {
      ipiv[i] = i;
    }
    T* v = W + (size_t)i * ldw;
    const T alpha = v[i];
    T s = T(0);
    for (int r = i + 1 + lane; r < n2; r += 32) s += v[r] * v[r];
    s = warp_sum(s);
    T t = T(0), beta = alpha;
    if (s != T(0)) {
      T nrm = sqrt(alpha * alpha + s);
      beta = alpha >= T(0) ? -nrm : nrm;
      t = (beta - alpha) / beta;
      const T sc = T(1) / (alpha - beta);
      for (int r = i + 1 + lane; r < n2; r += 32) v[r] *= sc;
    }
    __syncwarp();
    if (lane == 0) { v[i] = beta; tau[i] = t; }
    __syncwarp();
    if (beta == T(0)) return i + 1;
    if (t != T(0))
      for (int c = i + 1 + lane; c < NC; c += 32) {
        T* col = W + (size_t)c * ldw;
        T w = col[i];
        for (int r = i + 1; r < n2; ++r) w += v[r] * col[r];
        w *= t;
        col[i] -= w;
        for (int r = i + 1; r < n2; ++r) col[r] -= w * v[r];
      }
    __syncwarp();
    if (R > n2) {
      const T rb = T(1) / beta;
      for (int r = n2 + lane; r < R; r += 32) v[r] *= rb;
      __syncwarp();
      for (int c = i + 1 + lane; c < NC; c += 32) {
        T* col = W + (size_t)c * ldw;
        const T u = col[i];
        if (u != T(0))
          for (int r = n2; r < R; ++r) col[r] -= v[r] * u;
      }
      __syncwarp();
    }
  }
  return 0;
}

template <typename T, int SEL>
__global__ void __launch_bounds__(WARPS_PANEL * 32) k_factor_level(FactorArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const Dims d = a.d;
  const int n = d.n, nr = d.nr, nx = d.nx, nb = d.nblock;
  const int n2 = 2 * n, R = n2 + nr, NC = 3 * n + nx, ldw = a.ldw;
  const size_t nn = (size_t)n * n, nnx = (size_t)n * nx, nrn = (size_t)nr * n, nrnx = (size_t)nr * nx;
  const size_t wsz = (size_t)ldw * NC;
  T* W = reinterpret_cast<T*>(smem_raw) + warp * wsz;
  T* tau = reinterpret_cast<T*>(smem_raw) + wpb * wsz + warp * n;
  int* ipiv = reinterpret_cast<int*>(reinterpret_cast<T*>(smem_raw) + wpb * wsz + wpb * n) + warp * n;
  const int k = a.k;
  const long np = pairs_at_level(nb, k);
  const bool first = a.first != 0;

  for (long q = (long)blockIdx.x * wpb + warp; q < np; q += (long)gridDim.x * wpb) {
    const int j = k + (int)(2L * k * q), jp = j - k, jpp = min(j + k, nb);
    // ---------------------------------------------------------------- load
    {
      const size_t oj = (size_t)j * nn, ojp = (size_t)jp * nn;
      for (int idx = lane; idx < (int)nn; idx += 32) {
        const int i = idx % n, c = idx / n;
        T ejp, djp, dj, ej;
        if (first) {
          ejp = T(a.E0[ojp + idx]); djp = T(a.D0[ojp + idx]);
          dj = T(a.D0[oj + idx]);   ej = T(a.E0[oj + idx]);
        } else {
          ejp = a.E[ojp + idx]; djp = a.D[ojp + idx];
          dj = a.D[oj + idx];   ej = a.E[oj + idx];
        }
        W[(size_t)c * ldw + i] = ejp;
        W[(size_t)(n + c) * ldw + i] = djp;
        W[(size_t)(n2 + c) * ldw + i] = T(0);
        W[(size_t)c * ldw + n + i] = dj;
        W[(size_t)(n + c) * ldw + n + i] = T(0);
        W[(size_t)(n2 + c) * ldw + n + i] = ej;
      }
      for (int idx = lane; idx < (int)nnx; idx += 32) {
        const int i = idx % n, c = idx / n;
        const size_t o1 = (size_t)jp * nnx + idx, o2 = (size_t)j * nnx + idx;
        W[(size_t)(3 * n + c) * ldw + i] = first ? T(a.B0[o1]) : a.B[o1];
        W[(size_t)(3 * n + c) * ldw + n + i] = first ? T(a.B0[o2]) : a.B[o2];
      }
      for (int idx = lane; idx < (int)nrn; idx += 32) {
        const int r = idx % nr, c = idx / nr;
        const size_t o = (size_t)j * nrn + idx;
        W[(size_t)c * ldw + n2 + r] = first ? T(a.C0[o]) : a.C[o];
        W[(size_t)(n + c) * ldw + n2 + r] = T(0);
        W[(size_t)(n2 + c) * ldw + n2 + r] = T(0);
      }
      for (int idx = lane; idx < (int)nrnx; idx += 32) {
        const int r = idx % nr, c = idx / nr;
        W[(size_t)(3 * n + c) * ldw + n2 + r] = T(0);
      }
    }
    __syncwarp();
    // ----------------------------------------------------------- eliminate
    int info;
    if (SEL == SEL_LU) info = warp_eliminate_lu<T>(W, ldw, n, R, NC, ipiv, lane);
    else if (SEL == SEL_QR) info = warp_eliminate_qr<T, false>(W, ldw, n, R, NC, ipiv, tau, lane);
    else info = warp_eliminate_qr<T, true>(W, ldw, n, R, NC, ipiv, tau, lane);
    __syncwarp();
    if (info != 0) {
      if (lane == 0) report(a.st, DEV_ZERO_PIVOT, j, info, k);
      continue;
    }
    // ---------------------------------------------------------------- store
    {
      T* Tj = a.Tm + (size_t)j * szT(d);
      for (int idx = lane; idx < (int)(2 * nn); idx += 32) {
        const int r = idx % n2, c = idx / n2;
        Tj[idx] = W[(size_t)c * ldw + r];
      }
      if (SEL != SEL_LU)
        for (int i = lane; i < n; i += 32) Tj[2 * nn + i] = tau[i];
      for (int i = lane; i < n; i += 32) a.P[(size_t)j * n + i] = ipiv[i];
      const size_t oj = (size_t)j * nn, ojp = (size_t)jp * nn;
      for (int idx = lane; idx < (int)nn; idx += 32) {
        const int i = idx % n, c = idx / n;
        a.D[oj + idx] = W[(size_t)(n + c) * ldw + i];
        a.E[oj + idx] = W[(size_t)(n2 + c) * ldw + i];
        a.D[ojp + idx] = W[(size_t)(n + c) * ldw + n + i];
        a.E[ojp + idx] = W[(size_t)(n2 + c) * ldw + n + i];
      }
      for (int idx = lane; idx < (int)nnx; idx += 32) {
        const int i = idx % n, c = idx / n;
        a.B[(size_t)j * nnx + idx] = W[(size_t)(3 * n + c) * ldw + i];
        a.B[(size_t)jp * nnx + idx] = W[(size_t)(3 * n + c) * ldw + n + i];
      }
      for (int idx = lane; idx < (int)nrn; idx += 32) {
        const int r = idx % nr, c = idx / nr;
        const size_t oc = (size_t)jp * nrn + idx;
        a.C[(size_t)j * nrn + idx] = W[(size_t)c * ldw + n2 + r];
        const T cjp = first ? T(a.C0[oc]) : a.C[oc];
        a.C[oc] = cjp + W[(size_t)(n + c) * ldw + n2 + r];
        a.Rbuf[(size_t)j * nrn + idx] = W[(size_t)(n2 + c) * ldw + n2 + r];
      }
      for (int idx = lane; idx < (int)nrnx; idx += 32) {
        const int r = idx % nr, c = idx / nr;
        a.Fbuf[(size_t)j * nrnx + idx] = W[(size_t)(3 * n + c) * ldw + n2 + r];
      }
    }
    __syncwarp();
  }
}

// C_jpp += dC_jpp for every pair of the level (one writer per target block)
template <typename T>
__global__ void k_border_fix(Dims d, T* C, const T* Rbuf, int k) {
  const long np = pairs_at_level(d.nblock, k);
  const size_t nrn = (size_t)d.nr * d.n;
  const size_t total = (size_t)np * nrn;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const long q = (long)(e / nrn);
    const int idx = (int)(e % nrn);
    const int j = k + (int)(2L * k * q), jpp = min(j + k, d.nblock);
    C[(size_t)jpp * nrn + idx] += Rbuf[(size_t)j * nrn + idx];
  }
}

// ---------------------------------------------------------------------------
// deterministic sums over blocks 1..nblock-1 of per-block m-vectors
//   stage 1: CTA g sums a fixed chunk of blocks in order
//   stage 2: one CTA sums the chunk partials in order and adds to out
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_reduce_stage1(const T* buf, long first, long count, int m, long chunk, T* part) {
  const long b0 = first + (long)blockIdx.x * chunk;
  const long b1 = min(first + count, b0 + chunk);
  for (int e = threadIdx.x; e < m; e += blockDim.x) {
    T s = T(0);
    for (long b = b0; b < b1; ++b) s += buf[(size_t)b * m + e];
    part[(size_t)blockIdx.x * m + e] = s;
  }
}

// out[e] (stride ld per column of height h) = base[e] + sum of partials
template <typename T>
__global__ void k_reduce_stage2(const T* part, int nparts, int m, int h, const T* base, int ldb,
                                T* out, int ldo) {
  for (int e = threadIdx.x; e < m; e += blockDim.x) {
    T s = T(0);
    for (int g = 0; g < nparts; ++g) s += part[(size_t)g * m + e];
    const int r = e % h, c = e / h;
    out[(size_t)c * ldo + r] = (base ? base[(size_t)c * ldb + r] : T(0)) + s;
  }
}

// ---------------------------------------------------------------------------
// solve sweeps (forward, cc:1615-1795; backward, cc:1805-2075)
// ---------------------------------------------------------------------------
template <typename T>
struct SweepArgs {
  Dims d;
  const T *D, *E, *B, *C, *Tm;
  const int* P;
  T* x;
  int ldx, nrhs;
  T* XB;
  int k, ldw, sel;
};

template <typename T>
__global__ void __launch_bounds__(WARPS_PANEL * 32) k_forward_level(SweepArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const Dims d = a.d;
  const int n = d.n, nr = d.nr, n2 = 2 * n, nrhs = a.nrhs, ldw = a.ldw, k = a.k;
  T* W = reinterpret_cast<T*>(smem_raw) + (size_t)warp * ldw * nrhs;
  const long np = pairs_at_level(d.nblock, k);
  for (long q = (long)blockIdx.x * wpb + warp; q < np; q += (long)gridDim.x * wpb) {
    const int j = k + (int)(2L * k * q), jp = j - k;
    const T* Tj = a.Tm + (size_t)j * szT(d);
    for (int idx = lane; idx < n * nrhs; idx += 32) {
      const int i = idx % n, c = idx / n;
      W[(size_t)c * ldw + i] = a.x[(size_t)c * a.ldx + (size_t)jp * n + i];
      W[(size_t)c * ldw + n + i] = a.x[(size_t)c * a.ldx + (size_t)j * n + i];
    }
    __syncwarp();
    if (a.sel == SEL_LU) {
      const int* Pj = a.P + (size_t)j * n;
      for (int i = 0; i < n; ++i) {
        const int p = Pj[i];
        if (p != i)
          for (int c = lane; c < nrhs; c += 32) {
            T t = W[(size_t)c * ldw + i];
            W[(size_t)c * ldw + i] = W[(size_t)c * ldw + p];
            W[(size_t)c * ldw + p] = t;
          }
        __syncwarp();
      }
      for (int i = 0; i < n; ++i) {
        for (int r = i + 1 + lane; r < n2; r += 32) {
          const T l = Tj[(size_t)i * n2 + r];
          for (int c = 0; c < nrhs; ++c) W[(size_t)c * ldw + r] -= l * W[(size_t)c * ldw + i];
        }
        __syncwarp();
      }
    } else {
      for (int i = 0; i < n; ++i) {
        const T t = Tj[2 * (size_t)n * n + i];
        const T* v = Tj + (size_t)i * n2;
        for (int c = 0; c < nrhs; ++c) {
          T* w = W + (size_t)c * ldw;
          T s = T(0);
          for (int r = i + 1 + lane; r < n2; r += 32) s += v[r] * w[r];
          s = warp_sum(s);
          s = (s + w[i]) * t;
          __syncwarp();
          if (lane == 0) w[i] -= s;
          for (int r = i + 1 + lane; r < n2; r += 32) w[r] -= s * v[r];
          __syncwarp();
        }
      }
    }
    __syncwarp();
    for (int idx = lane; idx < n * nrhs; idx += 32) {
      const int i = idx % n, c = idx / n;
      a.x[(size_t)c * a.ldx + (size_t)jp * n + i] = W[(size_t)c * ldw + n + i];
      a.x[(size_t)c * a.ldx + (size_t)j * n + i] = W[(size_t)c * ldw + i];
    }
    if (nr > 0) {
      const T* Cj = a.C + (size_t)j * nr * n;
      for (int idx = lane; idx < nr * nrhs; idx += 32) {
        const int r = idx % nr, c = idx / nr;
        T s = T(0);
        for (int i = 0; i < n; ++i) s += Cj[(size_t)i * nr + r] * W[(size_t)c * ldw + i];
        a.XB[(size_t)j * nr * nrhs + idx] = -s;
      }
    }
    __syncwarp();
  }
}

template <typename T>
__global__ void __launch_bounds__(WARPS_PANEL * 32) k_backward_level(SweepArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const Dims d = a.d;
  const int n = d.n, nx = d.nx, n2 = 2 * n, nrhs = a.nrhs, k = a.k, nb = d.nblock;
  T* Y = reinterpret_cast<T*>(smem_raw) + (size_t)warp * a.ldw;
  const long np = pairs_at_level(nb, k);
  const size_t xb_off = (size_t)(nb + 1) * n + d.qx;
  for (long q = (long)blockIdx.x * wpb + warp; q < np; q += (long)gridDim.x * wpb) {
    const int j = k + (int)(2L * k * q), jp = j - k, jpp = min(j + k, nb);
    const T* Dj = a.D + (size_t)j * n * n;
    const T* Ej = a.E + (size_t)j * n * n;
    const T* Bj = a.B + (size_t)j * n * nx;
    const T* Tj = a.Tm + (size_t)j * szT(d);
    for (int c = 0; c < nrhs; ++c) {
      T* xc = a.x + (size_t)c * a.ldx;
      for (int i = lane; i < n; i += 32) {
        T s = xc[(size_t)j * n + i];
        for (int m = 0; m < n; ++m) s -= Dj[(size_t)m * n + i] * xc[(size_t)jp * n + m];
        for (int m = 0; m < n; ++m) s -= Ej[(size_t)m * n + i] * xc[(size_t)jpp * n + m];
        for (int m = 0; m < nx; ++m) s -= Bj[(size_t)m * n + i] * xc[xb_off + m];
        Y[i] = s;
      }
      __syncwarp();
      for (int i = n - 1; i >= 0; --i) {
        const T xi = Y[i] / Tj[(size_t)i * n2 + i];
        __syncwarp();
        if (lane == 0) Y[i] = xi;
        for (int r = lane; r < i; r += 32) Y[r] -= Tj[(size_t)i * n2 + r] * xi;
        __syncwarp();
      }
      if (a.sel == SEL_QRP && lane == 0) {
        const int* Pj = a.P + (size_t)j * n;
        for (int i = n - 1; i >= 0; --i) {
          const int p = Pj[i];
          if (p != i) { T t = Y[i]; Y[i] = Y[p]; Y[p] = t; }
        }
      }
      __syncwarp();
      for (int i = lane; i < n; i += 32) xc[(size_t)j * n + i] = Y[i];
      __syncwarp();
    }
  }
}

// ---------------------------------------------------------------------------
// last block (load_and_factorize_last, cc:1281-1374; solve_last, cc:1385-1479)
// one CTA; the Nr x Nc matrix lives in global memory (L2 resident)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_last_assemble(Dims d, const T* D, const T* E, const T* B, const T* C,
                                const double* H, const double* Cq, const T* Ffin, T* Hl) {
  const int n = d.n, Nr = d.Nr, Nc = d.Nc, qx = d.qx, nx = d.nx, nr = d.nr, m = n + d.qr;
  const int total = Nr * Nc;
  const T* CN = C + (size_t)d.nblock * nr * n;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    const int r = e % Nr, c = e / Nr;
    T v = T(0);
    if (r < n) {
      if (c < n) v = D[(size_t)c * n + r];
      else if (c < 2 * n) v = E[(size_t)(c - n) * n + r];
      else if (c >= 2 * n + qx) v = B[(size_t)(c - 2 * n - qx) * n + r];
    } else if (r < n + m) {
      v = T(H[(size_t)c * m + (r - n)]);
    } else {
      const int rr = r - n - m;
      if (c < n) v = C[(size_t)c * nr + rr];
      else if (c < 2 * n) v = CN[(size_t)(c - n) * nr + rr];
      else if (c < 2 * n + qx) v = T(Cq[(size_t)(c - 2 * n) * nr + rr]);
      else v = Ffin[(size_t)(c - 2 * n - qx) * nr + rr];
    }
    Hl[e] = v;
  }
}

template <typename T>
__device__ void block_argmax(T& v, int& idx, T* sv, int* si) {
  warp_argmax(v, idx);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) { sv[w] = v; si[w] = idx; }
  __syncthreads();
  if (w == 0) {
    v = lane < nw ? sv[lane] : T(-1);
    idx = lane < nw ? si[lane] : 0x7fffffff;
    warp_argmax(v, idx);
    if (lane == 0) { sv[0] = v; si[0] = idx; }
  }
  __syncthreads();
  v = sv[0];
  idx = si[0];
}

template <typename T>
__device__ T block_sum(T v, T* sv) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) sv[w] = v;
  __syncthreads();
  if (w == 0) {
    v = lane < nw ? sv[lane] : T(0);
    v = warp_sum(v);
    if (lane == 0) sv[0] = v;
  }
  __syncthreads();
  return sv[0];
}

// kind: LAST_LU or LAST_QR (others are rejected on the host)
template <typename T>
__global__ void k_last_factor(Dims d, T* A, int* piv, T* tau, int kind, StatusWords* st) {
  __shared__ T sv[32];
  __shared__ int si[32];
  const int M = d.Nr, N = d.Nc, tid = threadIdx.x, bs = blockDim.x;
  if (kind == LAST_LU) {
    if (M != N) { if (tid == 0) report(st, DEV_BAD_SHAPE, -1, 0, -1); return; }
    for (int i = 0; i < N; ++i) {
      T best = T(-1);
      int bi = i;  // stays in range even when every candidate is NaN
      for (int r = i + tid; r < N; r += bs) {
        T v = dev_abs(A[(size_t)i * N + r]);
        if (v > best) { best = v; bi = r; }
      }
      block_argmax(best, bi, sv, si);
      if (tid == 0) piv[i] = bi;
      const T pv = A[(size_t)i * N + bi];
      if (pv == T(0)) { if (tid == 0) report(st, DEV_LAST_SINGULAR, -1, i + 1, -1); return; }
      if (bi != i)
        for (int c = tid; c < N; c += bs) {
          T t = A[(size_t)c * N + i]; A[(size_t)c * N + i] = A[(size_t)c * N + bi]; A[(size_t)c * N + bi] = t;
        }
      __syncthreads();
      const T rinv = T(1) / pv;
      for (int r = i + 1 + tid; r < N; r += bs) A[(size_t)i * N + r] *= rinv;
      __syncthreads();
      const int L = N - i - 1;
      for (int e = tid; e < L * L; e += bs) {
        const int r = i + 1 + e % L, c = i + 1 + e / L;
        A[(size_t)c * N + r] -= A[(size_t)i * N + r] * A[(size_t)c * N + i];
      }
      __syncthreads();
    }
  } else {  // Householder QR, M >= N
    if (M < N) { if (tid == 0) report(st, DEV_BAD_SHAPE, -1, 0, -1); return; }
    for (int i = 0; i < N; ++i) {
      T* v = A + (size_t)i * M;
      const T alpha = v[i];
      T s = T(0);
      for (int r = i + 1 + tid; r < M; r += bs) s += v[r] * v[r];
      s = block_sum(s, sv);
      T t = T(0), beta = alpha;
      if (s != T(0)) {
        const T nrm = sqrt(alpha * alpha + s);
        beta = alpha >= T(0) ? -nrm : nrm;
        t = (beta - alpha) / beta;
        const T sc = T(1) / (alpha - beta);
        for (int r = i + 1 + tid; r < M; r += bs) v[r] *= sc;
      }
      __syncthreads();
      if (tid == 0) { v[i] = beta; tau[i] = t; }
      __syncthreads();
      if (beta == T(0)) { if (tid == 0) report(st, DEV_LAST_SINGULAR, -1, i + 1, -1); return; }
      if (t != T(0))
        for (int c = i + 1 + tid; c < N; c += bs) {
          T* col = A + (size_t)c * M;
          T w = col[i];
          for (int r = i + 1; r < M; ++r) w += v[r] * col[r];
          w *= t;
          col[i] -= w;
          for (int r = i + 1; r < M; ++r) col[r] -= w * v[r];
        }
      __syncthreads();
    }
  }
}

template <typename T>
__global__ void k_last_solve(Dims d, const T* A, const int* piv, const T* tau, int kind, T* x,
                             int ldx, int nrhs) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* b = reinterpret_cast<T*>(smem_raw);
  __shared__ T sv[32];
  const int n = d.n, M = d.Nr, N = d.Nc, tid = threadIdx.x, bs = blockDim.x;
  const size_t off = (size_t)d.nblock * n;
  for (int c = 0; c < nrhs; ++c) {
    T* xc = x + (size_t)c * ldx;
    for (int r = tid; r < M; r += bs) b[r] = r < n ? xc[r] : xc[off + (r - n)];
    __syncthreads();
    if (kind == LAST_LU) {
      if (tid == 0)
        for (int i = 0; i < N; ++i) {
          const int p = piv[i];
          if (p != i) { T t = b[i]; b[i] = b[p]; b[p] = t; }
        }
      __syncthreads();
      for (int i = 0; i < N; ++i) {
        const T bi = b[i];
        for (int r = i + 1 + tid; r < N; r += bs) b[r] -= A[(size_t)i * N + r] * bi;
        __syncthreads();
      }
    } else {
      for (int i = 0; i < N; ++i) {
        const T* v = A + (size_t)i * M;
        T s = T(0);
        for (int r = i + 1 + tid; r < M; r += bs) s += v[r] * b[r];
        s = block_sum(s, sv);
        s = (s + b[i]) * tau[i];
        __syncthreads();
        if (tid == 0) b[i] -= s;
        for (int r = i + 1 + tid; r < M; r += bs) b[r] -= s * v[r];
        __syncthreads();
      }
    }
    const int lda = kind == LAST_LU ? N : M;
    for (int i = N - 1; i >= 0; --i) {
      const T xi = b[i] / A[(size_t)i * lda + i];
      __syncthreads();
      if (tid == 0) b[i] = xi;
      for (int r = tid; r < i; r += bs) b[r] -= A[(size_t)i * lda + r] * xi;
      __syncthreads();
    }
    for (int r = tid; r < N; r += bs) {
      if (r < n) xc[r] = b[r];
      else xc[off + (r - n)] = b[r];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Mv with the loaded matrix (add_Mv, cc:2118-2166): res = alpha*A*x + beta*res
// ---------------------------------------------------------------------------
__global__ void k_mv_rows(Dims d, const double* D, const double* E, const double* B, double alpha,
                          const double* x, double beta, double* res) {
  const int n = d.n, nx = d.nx;
  const size_t rows = (size_t)d.nblock * n;
  const size_t xb_off = (size_t)(d.nblock + 1) * n + d.qx;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < rows;
       e += (size_t)gridDim.x * blockDim.x) {
    const size_t k = e / n;
    const int i = (int)(e % n);
    const double* Dk = D + k * n * n;
    const double* Ek = E + k * n * n;
    const double* Bk = B + k * n * nx;
    double s = 0;
    for (int c = 0; c < n; ++c) s += Dk[(size_t)c * n + i] * x[k * n + c];
    for (int c = 0; c < n; ++c) s += Ek[(size_t)c * n + i] * x[(k + 1) * n + c];
    for (int c = 0; c < nx; ++c) s += Bk[(size_t)c * n + i] * x[xb_off + c];
    res[e] = (beta == 0.0 ? 0.0 : beta * res[e]) + alpha * s;
  }
}

__global__ void k_mv_cpart(Dims d, const double* C, const double* x, double* part) {
  const int n = d.n, nr = d.nr;
  const size_t total = (size_t)(d.nblock + 1) * nr;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const size_t k = e / nr;
    const int r = (int)(e % nr);
    const double* Ck = C + k * nr * n;
    double s = 0;
    for (int c = 0; c < n; ++c) s += Ck[(size_t)c * nr + r] * x[k * n + c];
    part[e] = s;
  }
}

// H rows and the nr border rows (Csum = sum_k C_k x_k precomputed)
__global__ void k_mv_tail(Dims d, const double* H, const double* Cq, const double* F,
                          const double* Csum, double alpha, const double* x, double beta,
                          double* res) {
  const int n = d.n, m = n + d.qr, nr = d.nr, qx = d.qx, nx = d.nx, Nc = d.Nc;
  const size_t r0 = (size_t)d.nblock * n;
  const size_t xN = (size_t)d.nblock * n, xq = (size_t)(d.nblock + 1) * n, xb = xq + qx;
  for (int r = threadIdx.x; r < m + nr; r += blockDim.x) {
    double s = 0;
    if (r < m) {
      for (int c = 0; c < Nc; ++c) {
        size_t xi = c < n ? (size_t)c : (c < 2 * n ? xN + (c - n) : xq + (c - 2 * n));
        s += H[(size_t)c * m + r] * x[xi];
      }
    } else {
      const int rr = r - m;
      s = Csum[rr];
      for (int c = 0; c < qx; ++c) s += Cq[(size_t)c * nr + rr] * x[xq + c];
      for (int c = 0; c < nx; ++c) s += F[(size_t)c * nr + rr] * x[xb + c];
    }
    const size_t o = r0 + r;
    res[o] = (beta == 0.0 ? 0.0 : beta * res[o]) + alpha * s;
  }
}

// ---------------------------------------------------------------------------
// host orchestration
// ---------------------------------------------------------------------------
static int grid_for(long work_items, int per_cta, int cap) {
  long g = (work_items + per_cta - 1) / per_cta;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}

static void check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "alglin_b200: launch of %s failed: %s\n", what, cudaGetErrorString(e));
  }
}

static void reduce_blocks(DevState& s, const double* buf, long first, long count, int m, int h,
                          const double* base, int ldb, double* out, int ldo, cudaStream_t st) {
  if (m <= 0) return;
  const long chunk = 64;
  int nparts = count > 0 ? (int)((count + chunk - 1) / chunk) : 0;
  if (nparts > 0) {
    k_reduce_stage1<double><<<nparts, 128, 0, st>>>(buf, first, count, m, chunk, s.part);
    check_launch("k_reduce_stage1");
  }
  k_reduce_stage2<double><<<1, 256, 0, st>>>(s.part, nparts, m, h, base, ldb, out, ldo);
  check_launch("k_reduce_stage2");
}

void launch_factorize(DevState& s, cudaStream_t st) {
  const Dims d = s.d;
  const int n = d.n, nb = d.nblock;
  const size_t nn = (size_t)n * n, nnx = (size_t)n * d.nx, nrn = (size_t)d.nr * n;
  cudaMemsetAsync(s.st, 0, sizeof(StatusWords), st);
  // blocks not touched by the first level: the unpaired tail and C_nblock
  if (nb % 2 == 1) {
    const size_t t = (size_t)(nb - 1);
    cudaMemcpyAsync(s.D + t * nn, s.D0 + t * nn, nn * 8, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(s.E + t * nn, s.E0 + t * nn, nn * 8, cudaMemcpyDeviceToDevice, st);
    if (nnx) cudaMemcpyAsync(s.B + t * nnx, s.B0 + t * nnx, nnx * 8, cudaMemcpyDeviceToDevice, st);
    if (nrn) cudaMemcpyAsync(s.C + t * nrn, s.C0 + t * nrn, nrn * 8, cudaMemcpyDeviceToDevice, st);
  }
  if (nrn)
    cudaMemcpyAsync(s.C + (size_t)nb * nrn, s.C0 + (size_t)nb * nrn, nrn * 8,
                    cudaMemcpyDeviceToDevice, st);
  FactorArgs<double> a;
  a.d = d;
  a.D0 = s.D0; a.E0 = s.E0; a.B0 = s.B0; a.C0 = s.C0;
  a.D = s.D; a.E = s.E; a.B = s.B; a.C = s.C;
  a.Tm = s.T; a.P = s.P; a.Rbuf = s.Rbuf; a.Fbuf = s.Fbuf; a.st = s.st;
  a.ldw = odd_ld(2 * n + d.nr);
  const size_t per_warp = panel_smem_per_warp(d, 8);
  int wpb = (int)(SMEM_MAX / per_warp);
  if (wpb > WARPS_PANEL) wpb = WARPS_PANEL;
  if (wpb < 1) wpb = 1;  // callers reject sizes whose single warp does not fit
  const size_t smem = per_warp * wpb;
  if (smem > 48 * 1024) {
    if (s.sel == SEL_LU)
      cudaFuncSetAttribute(k_factor_level<double, SEL_LU>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_MAX);
    else if (s.sel == SEL_QR)
      cudaFuncSetAttribute(k_factor_level<double, SEL_QR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_MAX);
    else
      cudaFuncSetAttribute(k_factor_level<double, SEL_QRP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_MAX);
  }
  for (int k = 1; k < nb; k *= 2) {
    a.k = k;
    a.first = (k == 1);
    const long np = pairs_at_level(nb, k);
    const int grid = grid_for(np, wpb, 148 * 16);
    if (s.sel == SEL_LU) k_factor_level<double, SEL_LU><<<grid, wpb * 32, smem, st>>>(a);
    else if (s.sel == SEL_QR) k_factor_level<double, SEL_QR><<<grid, wpb * 32, smem, st>>>(a);
    else k_factor_level<double, SEL_QRP><<<grid, wpb * 32, smem, st>>>(a);
    check_launch("k_factor_level");
    if (nrn) {
      const long tot = np * (long)nrn;
      k_border_fix<double><<<grid_for(tot, 256, 148 * 8), 256, 0, st>>>(d, s.C, s.Rbuf, k);
      check_launch("k_border_fix");
    }
  }
  const int nrnx = d.nr * d.nx;
  if (nrnx > 0)
    reduce_blocks(s, s.Fbuf, 1, nb - 1, nrnx, d.nr, s.F0, d.nr, s.Ffin, d.nr, st);
  k_last_assemble<double><<<grid_for((long)d.Nr * d.Nc, 256, 64), 256, 0, st>>>(
      d, s.D, s.E, s.B, s.C, s.H, s.Cq, s.Ffin, s.Hl);
  check_launch("k_last_assemble");
  k_last_factor<double><<<1, 512, 0, st>>>(d, s.Hl, s.piv_l, s.tau_l, s.sel_last, s.st);
  check_launch("k_last_factor");
}

static void solve_chunk(DevState& s, double* x, int ldx, int nrhs, cudaStream_t st);

// right-hand sides are independent: sweep them in chunks of at most 16 columns
void launch_solve(DevState& s, double* x, int ldx, int nrhs, cudaStream_t st) {
  for (int c0 = 0; c0 < nrhs; c0 += 16)
    solve_chunk(s, x + (size_t)c0 * ldx, ldx, nrhs - c0 < 16 ? nrhs - c0 : 16, st);
}

static void solve_chunk(DevState& s, double* x, int ldx, int nrhs, cudaStream_t st) {
  const Dims d = s.d;
  const int n = d.n, nb = d.nblock;
  SweepArgs<double> a;
  a.d = d;
  a.D = s.D; a.E = s.E; a.B = s.B; a.C = s.C; a.Tm = s.T; a.P = s.P;
  a.x = x; a.ldx = ldx; a.nrhs = nrhs; a.XB = s.XB; a.sel = s.sel;
  a.ldw = odd_ld(2 * n);
  const size_t smem_f = (size_t)a.ldw * nrhs * 8 * WARPS_PANEL;
  if (smem_f > 48 * 1024)
    cudaFuncSetAttribute(k_forward_level<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
  int K = 1;
  for (; K < nb; K *= 2) {
    a.k = K;
    const long np = pairs_at_level(nb, K);
    k_forward_level<double><<<grid_for(np, WARPS_PANEL, 148 * 16), WARPS_PANEL * 32, smem_f, st>>>(a);
    check_launch("k_forward_level");
  }
  if (d.nr > 0) {
    double* xb = x + (size_t)(nb + 1) * n + d.qr;
    reduce_blocks(s, s.XB, 1, nb - 1, d.nr * nrhs, d.nr, xb, ldx, xb, ldx, st);
  }
  const size_t smem_l = (size_t)(d.Nr > d.Nc ? d.Nr : d.Nc) * 8;
  k_last_solve<double><<<1, 256, smem_l, st>>>(d, s.Hl, s.piv_l, s.tau_l, s.sel_last, x, ldx, nrhs);
  check_launch("k_last_solve");
  a.ldw = n;
  const size_t smem_b = (size_t)n * 8 * WARPS_PANEL;
  for (int k = K; (k /= 2) > 0;) {
    a.k = k;
    const long np = pairs_at_level(nb, k);
    k_backward_level<double><<<grid_for(np, WARPS_PANEL, 148 * 16), WARPS_PANEL * 32, smem_b, st>>>(a);
    check_launch("k_backward_level");
  }
}

void launch_mv(DevState& s, double alpha, const double* x, double beta, double* res,
               cudaStream_t st) {
  const Dims d = s.d;
  const long rows = (long)d.nblock * d.n;
  if (rows > 0) {
    k_mv_rows<<<grid_for(rows, 256, 148 * 8), 256, 0, st>>>(d, s.D0, s.E0, s.B0, alpha, x, beta, res);
    check_launch("k_mv_rows");
  }
  const int nr = d.nr;
  double* Csum = s.Ffin;  // reuse the small nr x nx buffer only if large enough
  if (nr > 0) {
    const long tot = (long)(d.nblock + 1) * nr;
    k_mv_cpart<<<grid_for(tot, 256, 148 * 8), 256, 0, st>>>(d, s.C0, x, s.mv_part);
    check_launch("k_mv_cpart");
    Csum = s.mv_part + (size_t)(d.nblock + 1) * nr;
    reduce_blocks(s, s.mv_part, 0, d.nblock + 1, nr, nr, nullptr, nr, Csum, nr, st);
  }
  k_mv_tail<<<1, 256, 0, st>>>(d, s.H, s.Cq, s.F0, Csum, alpha, x, beta, res);
  check_launch("k_mv_tail");
}

}  // namespace bcr
