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
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <type_traits>

#include "bcr_device.h"

namespace bcr {

static constexpr int WARPS_PANEL = 4;
static constexpr size_t SMEM_MAX = 227 * 1024;
static constexpr int CTA_KERNEL_MIN_N = 24;  // n above this: one CTA per pair
static constexpr long COMPACT_GRID = 148 * 8;  // CTAs of a sweep over a compacted batch map

template <typename T>
struct FactorArgs {
  Dims d;
  const double *D0, *E0, *B0, *C0;  // loaded matrix, read at the first level
  T *D, *E, *B, *C;                  // working blocks
  T* Tm;
  unsigned char* P;
  T* Rbuf;
  double* Fbuf;  // the F Schur updates are accumulated in FP64 in every precision
  const double* F0;  // loaded F (read by the tree schedule's root)
  StatusWords* st;
  int k, first, ldw;
  // right-hand sides eliminated together with the factorization (forward
  // sweep fused into the pair kernel); nrf == 0 when not fused
  double* x;
  int ldx, nrf;
  double* XB;
  // pair range of a single-system launch, [qb, qe) of the level (qe == 0: all)
  long qb, qe;
};

// element of a block: the loaded FP64 matrix at the first level, the working
// copy (type T) afterwards
template <typename T>
__device__ __forceinline__ T ldsrc(bool first, const double* orig, const T* work, size_t i) {
  return first ? T(orig[i]) : work[i];
}

// the same where another CTA of the same launch may have written the element
// (persistent batch launches): served by L2, never by a stale L1 line
template <bool COH, typename T>
__device__ __forceinline__ T ldsrc_c(bool first, const double* orig, const T* work, size_t i) {
  if constexpr (COH) return first ? T(__ldcg(orig + i)) : __ldcg(work + i);
  else return ldsrc(first, orig, work, i);
}
template <bool COH, typename T>
__device__ __forceinline__ T ldro(const T* p) {
  if constexpr (COH) return __ldcg(p);
  else return __ldg(p);
}

// Pair range of one worker (warp or CTA).  Single system: a grid-stride loop
// over the level's pairs.  Batch: map entry e (by default the CTA's index)
// holds pairs [q0, q1) of system cmap[e].sys, whose arguments come from the
// table; the level is the batch's.
__device__ __forceinline__ void take_level(FactorArgs<float>& a, const FactorArgs<float>& a0) { a.k = a0.k; a.first = a0.first; }
__device__ __forceinline__ void take_level(FactorArgs<double>& a, const FactorArgs<double>& a0) { a.k = a0.k; a.first = a0.first; }

// a batch system whose refinement has converged skips the sweeps (the
// SweepArgs overload below; found at instantiation)
template <typename A>
__device__ __forceinline__ bool system_active(const A&) { return true; }

// the pair range a single-system factorization launch is limited to (sweeps: all)
template <typename T>
__device__ __forceinline__ void launch_pair_range(const FactorArgs<T>& a, long& qb, long& qe) { qb = a.qb; qe = a.qe; }
template <typename A>
__device__ __forceinline__ void launch_pair_range(const A&, long&, long&) {}

template <bool BATCH, typename A>
__device__ __forceinline__ void pair_range(const A& a0, const A* tab, const BatchCta* cmap, int workers, int worker,
                                           A& a, long& q0, long& q1, long& qs, long entry = -1) {
  if constexpr (BATCH) {
    const BatchCta c = cmap[entry < 0 ? (long)blockIdx.x : entry];
    a = tab[c.sys];
    take_level(a, a0);
    q0 = c.q0 + worker;
    q1 = system_active(a) ? c.q1 : q0;
    qs = workers;
  } else {
    q0 = (long)blockIdx.x * workers + worker;
    q1 = pairs_at_level(a0.d.nblock, a0.k);
    qs = (long)gridDim.x * workers;
    long qb = 0, qe = 0;
    launch_pair_range(a0, qb, qe);
    if (qe > 0) { q0 += qb; q1 = qe; }
  }
}

// Map entries of one CTA of a batched sweep: entry b alone (one CTA per
// entry), or, when ecnt is given (the compacted maps of the refinement
// passes, whose length the device wrote), entries b, b + grid, ... below
// *ecnt.  Single systems: the body once.
template <bool BATCH, typename F>
__device__ __forceinline__ void for_entries(const long* ecnt, F&& body) {
  if constexpr (BATCH) {
    const long cnt = ecnt ? *ecnt : (long)gridDim.x;
    for (long e = blockIdx.x; e < cnt; e += gridDim.x) body(e);
  } else {
    body(-1L);
  }
}

// the same through the read-only path; every load of a pair kernel's load
// phase is independent of the shared-memory stores that follow it
template <typename T>
__device__ __forceinline__ T ldg_src(bool first, const double* orig, const T* work, size_t i) {
  if constexpr (sizeof(T) == 8)
    return __ldg(first ? orig + i : reinterpret_cast<const double*>(work) + i);
  else
    return first ? T(__ldg(orig + i)) : __ldg(work + i);
}

template <typename T>
__device__ __forceinline__ void load2(const T* p, T& a, T& b) {
  if constexpr (sizeof(T) == 8) {
    const double2 v = *reinterpret_cast<const double2*>(p);
    a = v.x; b = v.y;
  } else {
    const float2 v = *reinterpret_cast<const float2*>(p);
    a = v.x; b = v.y;
  }
}

template <typename T>
__device__ __forceinline__ void store2(T* p, T a, T b) {
  if constexpr (sizeof(T) == 8) *reinterpret_cast<double2*>(p) = make_double2(a, b);
  else *reinterpret_cast<float2*>(p) = make_float2(a, b);
}

__host__ __device__ inline int odd_ld(int r) { return r | 1; }

// pairs of large blocks go to one CTA each (work matrix in a global slab)
bool use_cta_kernel(const Dims& d) {
  return d.n > CTA_KERNEL_MIN_N || panel_smem_per_warp(d, 8) > SMEM_MAX;
}

size_t cta_slab_elems(const Dims& d) { return (size_t)(2 * d.n + d.nr) * (3 * d.n + d.nx); }

size_t panel_smem_per_warp(const Dims& d, int elem_bytes) {
  const int R = 2 * d.n + d.nr, NC = 3 * d.n + d.nx;
  size_t b = (size_t)odd_ld(R) * NC * elem_bytes + (size_t)d.n * (elem_bytes + sizeof(int));
  return b;
}

template <typename T> __device__ void block_argmax(T& v, int& idx, T* sv, int* si);
template <typename T> __device__ T block_sum(T v, T* sv);

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
    __syncwarp();  // every lane holds the pivot before column i is swapped
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

template <typename T, int SEL, bool BATCH = false>
__global__ void __launch_bounds__(WARPS_PANEL * 32) k_factor_level(FactorArgs<T> a0, const FactorArgs<T>* tab,
                                                               const BatchCta* cmap) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  FactorArgs<T> ab;  // this CTA's system (batch only)
  long q0, q1, qs;
  pair_range<BATCH>(a0, tab, cmap, wpb, warp, ab, q0, q1, qs);
  const FactorArgs<T>& a = BATCH ? ab : a0;
  const Dims d = a.d;
  const int n = d.n, nr = d.nr, nx = d.nx, nb = d.nblock;
  const int n2 = 2 * n, R = n2 + nr, NC = 3 * n + nx, ldw = a.ldw;
  const size_t nn = (size_t)n * n, nnx = (size_t)n * nx, nrn = (size_t)nr * n, nrnx = (size_t)nr * nx;
  const size_t wsz = (size_t)ldw * NC;
  T* W = reinterpret_cast<T*>(smem_raw) + warp * wsz;
  T* tau = reinterpret_cast<T*>(smem_raw) + wpb * wsz + warp * n;
  int* ipiv = reinterpret_cast<int*>(reinterpret_cast<T*>(smem_raw) + wpb * wsz + wpb * n) + warp * n;
  const int k = a.k;
  const bool first = a.first != 0;

  for (long q = q0; q < q1; q += qs) {
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
      __syncwarp();
      // row map (getrf row order) and column map (QRP) from the swap sequence,
      // built in the tau scratch (already stored)
      unsigned char* Pj = a.P + (size_t)j * szP(d);
      unsigned char* mp = reinterpret_cast<unsigned char*>(tau);
      if (lane == 0) {
        if (SEL == SEL_LU) {
          for (int r = 0; r < n2; ++r) mp[r] = (unsigned char)r;
          for (int i = 0; i < n; ++i) { unsigned char t = mp[i]; mp[i] = mp[ipiv[i]]; mp[ipiv[i]] = t; }
        } else {
          for (int r = 0; r < n2; ++r) mp[r] = (unsigned char)r;
          for (int i = 0; i < n; ++i) mp[n2 + i] = (unsigned char)i;
          if (SEL == SEL_QRP)
            for (int i = 0; i < n; ++i) { unsigned char t = mp[n2 + i]; mp[n2 + i] = mp[n2 + ipiv[i]]; mp[n2 + ipiv[i]] = t; }
        }
      }
      __syncwarp();
      for (int i = lane; i < (SEL == SEL_LU ? n2 : 3 * n); i += 32) Pj[i] = mp[i];
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

// ---------------------------------------------------------------------------
// register-resident LU pair elimination for n <= N <= 16 (lane = panel row)
//
// Lane l < 2n holds row l of the work matrix [panel | x_jp | x_jpp | xb] in
// registers.  Row interchanges are not performed physically: every lane keeps
// the LAPACK row position of its row (mypos), and the swap of positions i and
// p at step i (getrf's ipiv) is replayed on those positions, so the final
// positions reproduce the row order of getrf exactly.  The pivot row of each
// step is broadcast through shared memory; the nr border rows are spread over
// the lanes by column (lane c holds column c, and c+32) and are eliminated with
// the same pivot rows, which yields C_j U^-1 and the C/F Schur updates.
// ---------------------------------------------------------------------------
// pairs [q0, q1) step qs of one system and level, one per warp
template <typename T, int N, int NXM, int NRM, bool COH>
__device__ __forceinline__ void rows_body(const FactorArgs<T>& a, long q0, long q1, long qs) {
  constexpr int NC = 3 * N + NXM;
  constexpr int NCP = (NC + 1) & ~1;
  constexpr int SLOTS = (NC + 31) / 32;
  constexpr unsigned FULL = 0xffffffffu;
  __shared__ __align__(16) T ubuf[4][NCP];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const Dims d = a.d;
  const int n = d.n, nr = d.nr, nx = d.nx, n2 = 2 * n;
  const size_t nn = (size_t)n * n, nnx = (size_t)n * nx, nrn = (size_t)nr * n, nrnx = (size_t)nr * nx;
  T* ub = ubuf[warp];
  const int k = a.k;
  const bool first = a.first != 0;
  const bool act = lane < n2, top = lane < n;
  const int ri = top ? lane : lane - n;

  for (long q = q0; q < q1; q += qs) {
    const int j = k + (int)(2L * k * q), jp = j - k;
    T row[NC];
    {
      // panel: E_jp (TOP) / D_j (BOTTOM); x_jp column: D_jp / 0; x_jpp: 0 / E_j
      const size_t op = top ? (size_t)jp * nn : (size_t)j * nn;
      const size_t ob = (size_t)(top ? jp : j) * nnx;
#pragma unroll
      for (int c = 0; c < N; ++c) {
        T pv = T(0), xv = T(0);
        if (act && c < n) {
          const size_t o = op + (size_t)c * n + ri;
          pv = top ? ldsrc_c<COH>(first, a.E0, a.E, o) : ldsrc_c<COH>(first, a.D0, a.D, o);
          xv = top ? ldsrc_c<COH>(first, a.D0, a.D, o) : ldsrc_c<COH>(first, a.E0, a.E, o);
        }
        row[c] = pv;
        row[N + c] = top ? xv : T(0);
        row[2 * N + c] = top ? T(0) : xv;
      }
#pragma unroll
      for (int c = 0; c < NXM; ++c)
        row[3 * N + c] = (act && c < nx) ? ldsrc_c<COH>(first, a.B0, a.B, ob + (size_t)c * n + ri) : T(0);
    }
    T cr[NRM][SLOTS];
#pragma unroll
    for (int r = 0; r < NRM; ++r)
#pragma unroll
      for (int sl = 0; sl < SLOTS; ++sl) cr[r][sl] = T(0);
    if (lane < n) {
      const size_t oc = (size_t)j * nrn + (size_t)lane * nr;
#pragma unroll
      for (int r = 0; r < NRM; ++r)
        if (r < nr) cr[r][0] = ldsrc_c<COH>(first, a.C0, a.C, oc + r);
    }

    int mypos = lane, mykey = 0, info = 0;
    bool done = !act;
#pragma unroll
    for (int i = 0; i < N; ++i) {
      if (i < n) {
        T v = done ? T(-1) : dev_abs(row[i]);
        if (v != v) v = T(-0.5);  // NaN never wins against a number
        int key = done ? 0x7fffffff : mypos;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          const T ov = __shfl_xor_sync(FULL, v, o);
          const int ok = __shfl_xor_sync(FULL, key, o);
          if (ov > v || (ov == v && ok < key)) { v = ov; key = ok; }
        }
        const unsigned m = __ballot_sync(FULL, !done && mypos == key);
        const int p = __ffs(m) - 1;
        if (lane == i) mykey = key;
        if (!done && mypos == i && lane != p) mypos = key;
        if (lane == p) {
          mypos = i;
#pragma unroll
          for (int c = (i & ~1); c < NCP; c += 2)
            store2(&ub[c], row[c], c + 1 < NC ? row[c + 1] : T(0));
        }
        __syncwarp();
        const T piv = ub[i];
        if (piv == T(0) && info == 0) info = i + 1;
        const T rinv = piv != T(0) ? T(1) / piv : T(0);
        if (!done && lane != p) {
          const T l = row[i] * rinv;
          row[i] = l;
#pragma unroll
          for (int c = i + 1; c < NC; ++c) row[c] = fma(-l, ub[c], row[c]);
        }
        if (lane == p) done = true;
#pragma unroll
        for (int r = 0; r < NRM; ++r) {
          if (r < nr) {
            const T mr = __shfl_sync(FULL, cr[r][0], i) * rinv;
            if (lane == i) cr[r][0] = mr;
            else if (lane > i && lane < NC) cr[r][0] = fma(-mr, ub[lane], cr[r][0]);
#pragma unroll
            for (int sl = 1; sl < SLOTS; ++sl)
              if (lane + 32 * sl < NC) cr[r][sl] = fma(-mr, ub[lane + 32 * sl], cr[r][sl]);
          }
        }
        __syncwarp();
      }
    }
    if (info != 0) {
      if (lane == 0) report(a.st, DEV_ZERO_PIVOT, j, info, k);
      continue;
    }
    // ---------------------------------------------------------------- store
    if (act) {
      T* Tj = a.Tm + (size_t)j * szT(d);
      const bool urow = mypos < n;
      const int rr = urow ? mypos : mypos - n;
      const size_t blk = urow ? (size_t)j : (size_t)jp;
      T* Dd = a.D + blk * nn + rr;
      T* Ed = a.E + blk * nn + rr;
      T* Bd = a.B + blk * nnx + rr;
#pragma unroll
      for (int c = 0; c < N; ++c)
        if (c < n) {
          Tj[(size_t)mypos + (size_t)c * n2] = row[c];
          Dd[(size_t)c * n] = row[N + c];
          Ed[(size_t)c * n] = row[2 * N + c];
        }
#pragma unroll
      for (int c = 0; c < NXM; ++c)
        if (c < nx) Bd[(size_t)c * n] = row[3 * N + c];
    }
    if (act) a.P[(size_t)j * szP(d) + mypos] = (unsigned char)lane;
#pragma unroll
    for (int sl = 0; sl < SLOTS; ++sl) {
      const int col = lane + 32 * sl;
      if (col >= NC) continue;
#pragma unroll
      for (int r = 0; r < NRM; ++r) {
        if (r >= nr) continue;
        const T v = cr[r][sl];
        if (col < N) {
          if (col < n) a.C[(size_t)j * nrn + (size_t)col * nr + r] = v;
        } else if (col < 2 * N) {
          const int c = col - N;
          if (c < n) {
            const size_t o = (size_t)jp * nrn + (size_t)c * nr + r;
            a.C[o] = ldsrc_c<COH>(first, a.C0, a.C, o) + v;
          }
        } else if (col < 3 * N) {
          const int c = col - 2 * N;
          if (c < n) a.Rbuf[(size_t)j * nrn + (size_t)c * nr + r] = v;
        } else {
          const int c = col - 3 * N;
          if (c < nx) a.Fbuf[(size_t)j * nrnx + (size_t)c * nr + r] = v;
        }
      }
    }
  }
}

template <typename T, int N, int NXM, int NRM, bool BATCH = false>
__global__ void __launch_bounds__(128) k_factor_lu_rows(FactorArgs<T> a0, const FactorArgs<T>* tab,
                                                         const BatchCta* cmap) {
  const int warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  FactorArgs<T> ab;  // this CTA's system (batch only)
  long q0, q1, qs;
  pair_range<BATCH>(a0, tab, cmap, wpb, warp, ab, q0, q1, qs);
  rows_body<T, N, NXM, NRM, false>(BATCH ? ab : a0, q0, q1, qs);
}

// ---------------------------------------------------------------------------
// Tensor-core LU pair elimination for n == N (N = 8 or 16), nr <= 8, nx <= 8.
//
//   phase 1 (SIMT, lane = panel row): partial-pivot LU of the 2N x N panel
//     [E_jp; D_j] in registers, with getrf's row order replayed on positions
//     (mypos) and the pivot chosen by exact integer reductions on the bits of
//     |a| (largest |a|, then smallest position: the idamax rule).  The nr
//     border rows ride along as a second register row of lanes 0..nr-1 and
//     come out as C_j U^-1.
//   phase 2 (SIMT): the elimination operator on the trailing columns,
//       G = [ L^-1 ; -M L^-1 ; -(C_j U^-1) L^-1 ]      ((2N+8) x N)
//     by a right triangular solve X L = [I; -M; -C'] per lane.
//   phase 3 (FP64 tensor cores, mma.sync m8n8k4): one GEMM
//       [U-row | reduced row | border update] = G (PW)_top + [0; (PW)_bot; 0]
//     over the 2N + nx trailing columns [x_jp | x_jpp | xb].
// The results are staged in shared memory and written with coalesced stores.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

template <int N, typename T = double>
struct TcShape {
  static constexpr int MT = 2 * N + 8;             // GEMM rows: U-row, reduced row, border (padded)
  static constexpr int NTILES = (2 * N + 8 + 7) / 8;  // trailing columns 2N + nx, nx <= 8
  static constexpr int NTP = NTILES * 8;
  // trailing rows, compact: a TOP row keeps [D_jp | B_jp | x_jp], a BOTTOM row
  // [E_j | B_j | x_j]; the structurally zero half of each row is not stored
  static constexpr int LDW = NTP - N + 1;
  static constexpr int PC = (NTILES + 1) / 2;      // column tiles per product pass
  static constexpr int LDG = N + 4;                 // operator rows (16B aligned, conflict-free A loads)
  static constexpr int KSTEPS = N / 4;
  static constexpr int MTILES = MT / 8;
  static constexpr int WS = 2 * N * LDW;            // doubles: the 2N panel rows' trailing part
  static constexpr int GS = MT * LDG;
  static constexpr size_t BYTES = (size_t)(WS + GS + N + 2) * sizeof(T) + 2 * N * sizeof(int);
};

// element (row, col) of the trailing part from the compact rows
template <int N, typename T>
__device__ __forceinline__ T tc_w(const T* Wt, int row, int col) {
  constexpr int LDW = TcShape<N>::LDW;
  const bool top = row < N;
  if (col < N) return top ? Wt[row * LDW + col] : T(0);
  if (col < 2 * N) return top ? T(0) : Wt[row * LDW + col - N];
  return Wt[row * LDW + col - N];
}

size_t tc_smem_per_warp(int n) {
  return n == 16 ? TcShape<16>::BYTES : n == 8 ? TcShape<8>::BYTES : 0;
}
template <typename T>
static size_t tc_smem_per_warp_t(int n) {
  return n == 16 ? TcShape<16, T>::BYTES : n == 8 ? TcShape<8, T>::BYTES : 0;
}

__host__ __device__ inline int lowbit(int v) { return v & -v; }
__host__ __device__ inline void tree_children(int j, int nb, int& c1, int& c2);

// Per-pair extras of the tree-scheduled factorization (k_factor_tree_tc):
// gather = the C_jpp contributions of earlier levels are added to C_j at load
// (Rbuf[j - K'] for K' = 1, 2, ..., gather; 0 in the level-by-level launches,
// where k_border_fix adds them after each level); c1, c2 = the nodes whose F
// and xb partial sums are added to this pair's own (0: none).
struct TcTree {
  int gather, c1, c2;
};

// Coherent load of an element that another warp of the same launch may have
// written (tree schedule): bypasses L1, served by L2.
__device__ __forceinline__ double ldw(const double* p) { return __ldcg(p); }

// Eliminates x_j from the pair (jp = j - k, j); see the comment above.
// Returns false (after reporting) when the panel has an exactly-zero pivot; the
// outputs of that pair are then not written.
//
// The nr <= NRM border rows are spread over the whole warp: lane = r * LPR +
// cg holds columns cg*CPL .. cg*CPL + CPL - 1 of border row r (LPR = 32 / NRM
// lanes per row), so their eliminations (C_j U^-1, then -C' L^-1) run in the
// same instructions as everyone else instead of on nr lanes alone.
template <int N, int NRM, typename T = double>
__device__ __forceinline__ bool tc_pair(const FactorArgs<T>& a, int j, int k, bool first, T* Wt, int lane,
                                        const TcTree& tr) {
  using S = TcShape<N, T>;
  constexpr unsigned FULL = 0xffffffffu;
  T* Gs = Wt + S::WS;
  T* bc = Gs + S::GS;                             // pivot row + its reciprocal
  int* rowof = reinterpret_cast<int*>(bc + N + 2);
  const Dims d = a.d;
  const int nr = d.nr, nx = d.nx;
  constexpr int n = N, n2 = 2 * N;
  constexpr size_t nn = (size_t)N * N;
  const size_t nnx = (size_t)n * nx, nrn = (size_t)nr * n, nrnx = (size_t)nr * nx;
  const int nrf = a.nrf;             // fused right-hand sides
  const int NT = n2 + nx + nrf;      // live trailing columns
  const bool act = lane < n2, top = lane < n;
  const int ri = top ? lane : lane - n;
  const int g = lane >> 2, t = lane & 3;
  const int jp = j - k;
  // block elements: the loaded FP64 matrix at the first level, the working
  // copy (type T) after it; always through L2 (see ldw)
  using SrcT = typename std::conditional<sizeof(T) == 8, double, T>::type;
  const SrcT* srcD = first ? (const SrcT*)a.D0 : (const SrcT*)a.D;
  const SrcT* srcE = first ? (const SrcT*)a.E0 : (const SrcT*)a.E;
  const SrcT* srcB = first ? (const SrcT*)a.B0 : (const SrcT*)a.B;
  const SrcT* srcC = first ? (const SrcT*)a.C0 : (const SrcT*)a.C;
  auto lds = [&](const SrcT* base, const double* orig, size_t i) -> T {
    if constexpr (sizeof(T) == 8) return ldw(base + i);
    else return first ? T(ldw(orig + i)) : __ldcg(base + i);
  };
  // ------------------------------------------------------------ load
  constexpr int LPR = 32 / NRM, CPL = N / LPR;   // border layout (see above)
  const int br = lane / LPR, bc0 = (lane % LPR) * CPL;
  const bool blive = br < nr;
  T rowA[N], cb[CPL];
  double cs1[2] = {0.0, 0.0}, cs2[2] = {0.0, 0.0};  // children's F / xb sums (tree)
  {
    const size_t po = top ? (size_t)jp * nn : (size_t)j * nn;
    const SrcT* Pm = (top ? srcE : srcD) + po;
    const double* Po = (top ? a.E0 : a.D0) + po;
#pragma unroll
    for (int c = 0; c < N; ++c) rowA[c] = act ? lds(Pm, Po, (size_t)c * n + ri) : T(0);
#pragma unroll
    for (int q = 0; q < CPL; ++q)
      cb[q] = blive ? lds(srcC, a.C0, (size_t)j * nrn + (size_t)(bc0 + q) * nr + br) : T(0);
    // C_jpp contributions of the pairs (j - 2K', j - K') of earlier levels,
    // K' = 1, 2, ..., gather: loaded eight levels at a time so that their
    // latencies overlap, then added in level order
    for (int e0 = 0; e0 < 31 && (1 << e0) <= tr.gather; e0 += 8) {
      T v[8][CPL];
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const int kk = e0 + e < 31 ? 1 << (e0 + e) : 0;
        const bool on = blive && kk != 0 && kk <= tr.gather;
#pragma unroll
        for (int q = 0; q < CPL; ++q)
          v[e][q] = on ? T(__ldcg(a.Rbuf + (size_t)(j - kk) * nrn + (size_t)(bc0 + q) * nr + br)) : T(0);
      }
#pragma unroll
      for (int e = 0; e < 8; ++e)
#pragma unroll
        for (int q = 0; q < CPL; ++q) cb[q] += v[e][q];
    }
    // the children's F / xb partial sums of the two border-tile elements this
    // lane holds in the product (row 2N + g, columns 2N + 2t + {0, 1})
    if ((tr.c1 | tr.c2) && g < nr) {
#pragma unroll
      for (int hh = 0; hh < 2; ++hh) {
        const int cl = 2 * t + hh;
        const double* base = nullptr;
        size_t stride = 0, e = 0;
        if (cl < nx) { base = a.Fbuf; stride = nrnx; e = (size_t)cl * nr + g; }
        else if (cl < nx + nrf) { base = a.XB; stride = (size_t)nr * nrf; e = (size_t)(cl - nx) * nr + g; }
        if (base) {
          if (tr.c1) cs1[hh] = ldw(base + (size_t)tr.c1 * stride + e);
          if (tr.c2) cs2[hh] = ldw(base + (size_t)tr.c2 * stride + e);
        }
      }
    }
    // trailing columns in the original row order: TOP [D_jp 0 B_jp], BOTTOM [0 E_j B_j]
    // compile-time trip counts: every load of the pair is issued before the
    // first one is consumed, so a lone pair pays one memory latency
    const SrcT* Djp = srcD + (size_t)jp * nn;
    const SrcT* Ej = srcE + (size_t)j * nn;
    const double* Djp0 = a.D0 + (size_t)jp * nn;
    const double* Ej0 = a.E0 + (size_t)j * nn;
#pragma unroll
    for (int it = 0; it < (int)(nn / 32); ++it) {
      const int idx = lane + 32 * it;
      const int r = idx % n, c = idx / n;
      Wt[r * S::LDW + c] = lds(Djp, Djp0, idx);
      Wt[(n + r) * S::LDW + c] = lds(Ej, Ej0, idx);
    }
    const SrcT* Bjp = srcB + (size_t)jp * nnx;
    const SrcT* Bj = srcB + (size_t)j * nnx;
    const double* Bjp0 = a.B0 + (size_t)jp * nnx;
    const double* Bj0 = a.B0 + (size_t)j * nnx;
#pragma unroll
    for (int it = 0; it < (8 * N + 31) / 32; ++it) {
      const int idx = lane + 32 * it;
      if (idx < (int)nnx) {
        const int r = idx % n, c = idx / n;
        Wt[r * S::LDW + n + c] = lds(Bjp, Bjp0, idx);
        Wt[(n + r) * S::LDW + n + c] = lds(Bj, Bj0, idx);
      }
    }
    // fused right-hand sides: TOP rows hold x_jp, BOTTOM rows x_j
    for (int idx = lane; idx < n2 * nrf; idx += 32) {
      const int r = idx % n2, c = idx / n2;
      const double* xc = a.x + (size_t)c * a.ldx;
      Wt[r * S::LDW + n + nx + c] = T(r < n ? ldw(xc + (size_t)jp * n + r) : ldw(xc + (size_t)j * n + r - n));
    }
    // zero the padding columns of the live rows (they feed padding outputs only,
    // but keep them finite)
    for (int idx = lane; idx < n2 * (S::NTP - NT); idx += 32) {
      const int r = idx % n2, c = NT + idx / n2;
      Wt[r * S::LDW + c - n] = T(0);
    }
  }
  // --------------------------------------------------- phase 1: panel LU
  int mypos = lane, info = 0;
  bool done = !act;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    // every lane forms the reciprocal of its own candidate while the pivot is
    // searched; the pivot lane publishes its value with the pivot row
    // pivot: max |a| over rows not yet used, ties to the smaller position
    // (FP64: upper word of |a|, then the lower word; FP32: the whole word)
    T rc;
    unsigned hi, lob;
    if constexpr (sizeof(T) == 8) {
      rc = __drcp_rn(rowA[i]);
      const double av = fabs(rowA[i]);
      const unsigned long long bits = (unsigned long long)__double_as_longlong(av);
      hi = (unsigned)(bits >> 32) + 1u;
      if (done) hi = 0u;
      else if (av != av) hi = 1u;  // NaN loses against every number
      lob = (unsigned)bits;
    } else {
      rc = __frcp_rn(rowA[i]);
      const float av = fabsf(rowA[i]);
      hi = __float_as_uint(av) + 1u;
      if (done) hi = 0u;
      else if (av != av) hi = 1u;
      lob = 0u;
    }
    const unsigned hmax = __reduce_max_sync(FULL, hi);
    unsigned m = __ballot_sync(FULL, hi == hmax && !done);
    unsigned pmin;
    if (__popc(m) == 1) {  // unique maximum in the upper word: the usual case
      pmin = (unsigned)__shfl_sync(FULL, mypos, __ffs(m) - 1);
    } else {               // exact tie handling: lower word, then smallest position
      const unsigned lo = (hi == hmax) ? lob : 0u;
      const unsigned lmax = __reduce_max_sync(FULL, lo);
      const bool cand = (hi == hmax) && (lo == lmax) && !done;
      pmin = __reduce_min_sync(FULL, cand ? (unsigned)mypos : 0xffffffffu);
      m = __ballot_sync(FULL, cand && (unsigned)mypos == pmin);
    }
    const int p = __ffs(m) - 1;
    if (!done && mypos == i && lane != p) mypos = (int)pmin;
    if (lane == p) {
      mypos = i;
#pragma unroll
      for (int c = (i & ~1); c < N; c += 2) store2(&bc[c], rowA[c], rowA[c + 1]);
      bc[N] = rc;
    }
    __syncwarp();
    const T piv = bc[i];
    if (piv == T(0) && info == 0) info = i + 1;
    const T rinv = piv != T(0) ? bc[N] : T(0);
    T u[N];
#pragma unroll
    for (int c = (i + 1) & ~1; c < N; c += 2) load2(&bc[c], u[c], u[c + 1]);
    if (!done && lane != p) {
      const T l = rowA[i] * rinv;
      rowA[i] = l;
#pragma unroll
      for (int c = i + 1; c < N; ++c) rowA[c] = fma(-l, u[c], rowA[c]);
    }
    {  // border rows: multiplier from the lane holding column i of the row
      const T ci = __shfl_sync(FULL, cb[i % CPL], (lane & ~(LPR - 1)) | (i / CPL));
      const T l = ci * rinv;
#pragma unroll
      for (int q = 0; q < CPL; ++q) {
        const int c = bc0 + q;
        if (c == i) cb[q] = l;
        else if (c > i) cb[q] = fma(-l, bc[c], cb[q]);
      }
    }
    if (lane == p) done = true;
    __syncwarp();
  }
  if (info != 0) {
    if (lane == 0) report(a.st, DEV_ZERO_PIVOT, j, info, k);
    return false;
  }
  // panel factors T_j (L\U and M in getrf row order), pivots, C_j U^-1
  {
    T* Tj = a.Tm + (size_t)j * szT(d);
    if (act) {
#pragma unroll
      for (int c = 0; c < N; ++c) Tj[(size_t)mypos + (size_t)c * n2] = rowA[c];
      rowof[mypos] = lane;
    }
    if (act) a.P[(size_t)j * szP(d) + mypos] = (unsigned char)lane;
    if (blive) {
#pragma unroll
      for (int q = 0; q < CPL; ++q) a.C[(size_t)j * nrn + (size_t)(bc0 + q) * nr + br] = cb[q];
    }
    // rows of L (row m contiguous) for the triangular solve
    if (act && mypos < n) {
#pragma unroll
      for (int c = 0; c < N; c += 2) store2(&Gs[mypos * S::LDG + c], rowA[c], rowA[c + 1]);
    }
  }
  __syncwarp();
  // ------------------------------------ phase 2: operator G (X L = R)
  // R rows: identity for U-row positions, -M for reduced positions, -C' for border rows
  {
    T x[N];
#pragma unroll
    for (int c = 0; c < N; ++c) x[c] = (mypos < n) ? (c == mypos ? T(1) : T(0)) : -rowA[c];
#pragma unroll
    for (int q = 0; q < CPL; ++q) cb[q] = -cb[q];
    // right-looking: once x[mm] is final, update every x[c], c < mm (the
    // updates of one step are independent, so the dependent chain is N long)
#pragma unroll
    for (int mm = N - 1; mm > 0; --mm) {
      const T xm = x[mm];
      const T cm = __shfl_sync(FULL, cb[mm % CPL], (lane & ~(LPR - 1)) | (mm / CPL));
      const T* Lrow = Gs + mm * S::LDG;  // L(mm, 0..mm-1)
#pragma unroll
      for (int c = 0; c < mm; c += 2) {
        T l0, l1;
        load2(&Lrow[c], l0, l1);
        x[c] = fma(-xm, l0, x[c]);
        if (c + 1 < mm) x[c + 1] = fma(-xm, l1, x[c + 1]);
      }
#pragma unroll
      for (int q = 0; q < CPL; ++q)
        if (bc0 + q < mm) cb[q] = fma(-cm, Lrow[bc0 + q], cb[q]);
    }
    __syncwarp();
    if (act) {
#pragma unroll
      for (int c = 0; c < N; c += 2) store2(&Gs[mypos * S::LDG + c], x[c], x[c + 1]);
    }
    // border rows of G (zero for rows >= nr, and rows NRM..7 of the tile)
#pragma unroll
    for (int q = 0; q < CPL; ++q) {
      Gs[(n2 + br) * S::LDG + bc0 + q] = blive ? cb[q] : T(0);
      if constexpr (NRM < 8) Gs[(n2 + NRM + br) * S::LDG + bc0 + q] = T(0);
    }
  }
  __syncwarp();
  // ----------------------------------------- phase 3: the product
  // FP64 tensor cores (DMMA 8x8x4) for double, the FP32 pipe for float, with
  // the same accumulator layout; two passes over the column tiles keep the
  // accumulators within budget
#pragma unroll
  for (int pass = 0; pass < 2; ++pass) {
    constexpr int PC = S::PC;
    T acc[S::MTILES][PC][2];
#pragma unroll
    for (int mt = 0; mt < S::MTILES; ++mt)
#pragma unroll
      for (int ni = 0; ni < PC; ++ni) {
        const int nt = pass * PC + ni;
        const int row = mt * 8 + g;
        T c0 = T(0), c1 = T(0);
        if (nt < S::NTILES && row >= n && row < n2) {  // (PW)_bot
          const int orow = rowof[row];
          c0 = tc_w<N>(Wt, orow, nt * 8 + 2 * t);
          c1 = tc_w<N>(Wt, orow, nt * 8 + 2 * t + 1);
        }
        acc[mt][ni][0] = c0;
        acc[mt][ni][1] = c1;
      }
    if constexpr (sizeof(T) == 8) {
#pragma unroll
      for (int ks = 0; ks < S::KSTEPS; ++ks) {
        double bfr[PC];
        const int orow = rowof[ks * 4 + t];
#pragma unroll
        for (int ni = 0; ni < PC; ++ni) {
          const int nt = pass * PC + ni;
          bfr[ni] = nt < S::NTILES ? tc_w<N>(Wt, orow, nt * 8 + g) : 0.0;
        }
#pragma unroll
        for (int mt = 0; mt < S::MTILES; ++mt) {
          const double afr = Gs[(mt * 8 + g) * S::LDG + ks * 4 + t];
#pragma unroll
          for (int ni = 0; ni < PC; ++ni)
            if (pass * PC + ni < S::NTILES) dmma_8x8x4(acc[mt][ni][0], acc[mt][ni][1], afr, bfr[ni]);
        }
      }
    } else {
      // element (8mt+g, 8nt+2t+h) += sum over kk of G(8mt+g, kk) (PW)_top(kk, 8nt+2t+h)
#pragma unroll 4
      for (int kk = 0; kk < N; ++kk) {
        const int orow = rowof[kk];
        T bv[PC][2];
#pragma unroll
        for (int ni = 0; ni < PC; ++ni) {
          const int nt = pass * PC + ni;
          bv[ni][0] = nt < S::NTILES ? tc_w<N>(Wt, orow, nt * 8 + 2 * t) : T(0);
          bv[ni][1] = nt < S::NTILES ? tc_w<N>(Wt, orow, nt * 8 + 2 * t + 1) : T(0);
        }
#pragma unroll
        for (int mt = 0; mt < S::MTILES; ++mt) {
          const T av = Gs[(mt * 8 + g) * S::LDG + kk];
#pragma unroll
          for (int ni = 0; ni < PC; ++ni) {
            acc[mt][ni][0] = fma(av, bv[ni][0], acc[mt][ni][0]);
            acc[mt][ni][1] = fma(av, bv[ni][1], acc[mt][ni][1]);
          }
        }
      }
    }
    // ------------------------------------------------------------ store
    // accumulator element (row 8mt+g, column 8nt+2t+h) straight to its block:
    // rows [0,N) U-row, [N,2N) reduced row, [2N, 2N+nr) border updates;
    // columns [0,N) x_jp, [N,2N) x_jpp, [2N, 2N+nx) xb
    {
#pragma unroll
      for (int mt = 0; mt < S::MTILES; ++mt) {
        const int row = mt * 8 + g;
#pragma unroll
        for (int ni = 0; ni < PC; ++ni)
#pragma unroll
          for (int hh = 0; hh < 2; ++hh) {
            const int nt = pass * PC + ni;
            if (nt >= S::NTILES) continue;
            const int col = nt * 8 + 2 * t + hh;
            const T v = acc[mt][ni][hh];
            if (mt * 8 < n2) {  // panel rows (compile-time per mt)
              const bool ur = row < n;
              const int rr = ur ? row : row - n;
              const size_t blk = ur ? (size_t)j : (size_t)jp;
              if (col < n) a.D[blk * nn + (size_t)col * n + rr] = v;
              else if (col < n2) a.E[blk * nn + (size_t)(col - n) * n + rr] = v;
              else if (col < n2 + nx) a.B[blk * nnx + (size_t)(col - n2) * n + rr] = v;
              else if (col < NT) a.x[(size_t)(col - n2 - nx) * a.ldx + blk * n + rr] = (double)v;
            } else {
              const int rr = row - n2;
              if (rr < nr) {
                if (col < n) {
                  const size_t o = (size_t)jp * nrn + (size_t)col * nr + rr;
                  a.C[o] = lds(srcC, a.C0, o) + v;
                } else if (col < n2) {
                  a.Rbuf[(size_t)j * nrn + (size_t)(col - n) * nr + rr] = v;
                } else if (col < n2 + nx) {
                  // own F update plus the partial sums of the child nodes (tree)
                  const size_t e = (size_t)(col - n2) * nr + rr;
                  a.Fbuf[(size_t)j * nrnx + e] = (double)v + cs1[hh] + cs2[hh];
                } else if (col < NT) {
                  const size_t e = (size_t)(col - n2 - nx) * nr + rr, nrr = (size_t)nr * nrf;
                  a.XB[(size_t)j * nrr + e] = (double)v + cs1[hh] + cs2[hh];
                }
              }
            }
          }
      }
    }
  }  // pass
  __syncwarp();
  return true;
}

// BOOK: the border bookkeeping of the tree schedule (see k_factor_tree_tc)
// in level-by-level launches: every pair gathers the C_j updates of the lower
// levels and adds its children's F / xb partial sums, so no border fix-up or
// reduction launch is needed between or after the levels (k_tree_root
// finishes C_nblock, F and xb after the last level).
// resident CTAs of 4 warps the register budget is sized for: FP32 pairs take
// half the shared memory and fewer registers, so more of them fit on an SM
template <typename T>
constexpr int tc_min_blocks() { return sizeof(T) == 8 ? 4 : 6; }

template <int N, bool BATCH = false, bool BOOK = false, int NRM = 8, typename T = double>
__global__ void __launch_bounds__(128, tc_min_blocks<T>())
    k_factor_lu_tc(FactorArgs<T> a0, const FactorArgs<T>* tab, const BatchCta* cmap) {
  using S = TcShape<N, T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  FactorArgs<T> ab;  // this CTA's system (batch only)
  long q0, q1, qs;
  pair_range<BATCH>(a0, tab, cmap, wpb, warp, ab, q0, q1, qs);
  const FactorArgs<T>& a = BATCH ? ab : a0;
  T* Wt = reinterpret_cast<T*>(smem_raw + (size_t)warp * S::BYTES);
  TcTree tr{0, 0, 0};
  for (long q = q0; q < q1; q += qs) {
    const int j = a.k + (int)(2L * a.k * q);
    if constexpr (BOOK) {
      tr.gather = a.k / 2;
      tree_children(j, a.d.nblock, tr.c1, tr.c2);
    }
    tc_pair<N, NRM, T>(a, j, a.k, a.first != 0, Wt, lane, tr);
  }
}

// ---------------------------------------------------------------------------
// The whole cyclic reduction of one system in one launch (tree schedule).
//
// Node j >= 1 is the pair (j - K, j) of level K = lowbit(j).  Its TOP row
// jp = j - K is final once the pair (jp, jp + K/2) -- node j - K/2 -- is done
// (K >= 2); its BOTTOM row j once the last pair of row j's own chain, node
// j + k'' (k'' the largest power of two below K with j + k'' < nblock), is
// done.  So each node waits for at most two children, and each node has one
// parent: the next pair of row jp's chain (node jp + 2K, when jp is a multiple
// of 4K and jp + 2K < nblock), otherwise the pair that eliminates row jp
// (node jp); node jp = 0 is the root.  Warps take the level-1 nodes (the
// leaves) from a counter; a warp that finishes a node adds one to its
// parent's arrival counter, and the warp that brings the count to the
// parent's number of children carries on with the parent.  No warp ever
// waits for another: the schedule needs no grid barrier and cannot stall.
//
// The border bookkeeping of the level-by-level schedule moves into the tree:
// the C_jpp updates a pair leaves in Rbuf[j] are gathered by the node that
// eliminates that block (or, for C_nblock, by the root), and the F and xb
// updates are summed up the tree (each node adds its children's partial sums
// to its own, in a fixed order), so results are bit-reproducible run to run.
// ---------------------------------------------------------------------------
// parent node of node j, 0 for the root
__host__ __device__ inline int tree_parent(int j, int nb) {
  const int K = lowbit(j), jp = j - K;
  if ((jp & (4 * K - 1)) == 0 && jp + 2 * K < nb) return jp + 2 * K;
  return jp;
}
// children of node j (0: none): the TOP child, then the BOTTOM child
__host__ __device__ inline void tree_children(int j, int nb, int& c1, int& c2) {
  const int K = lowbit(j);
  c1 = K >= 2 ? j - K / 2 : 0;
  c2 = 0;
  if (K >= 2 && j + 1 < nb) {
    int kk = K / 2;
    while (j + kk >= nb) kk >>= 1;
    c2 = j + kk;
  }
}

struct TreeArgs {
  int* cnt;         // [nblock] arrival counters (zero at launch)
  int* leaf;        // next level-1 node to take (zero at launch)
  double* Ffin;     // out: F0 + all F updates (nr x nx, FP64)
  double* xb;       // fused solve: rows of xb in x (+= sum of the xb updates), or null
};

// Work of the root: C_nblock with the C_jpp updates of the pairs whose jpp is
// nblock (one per level at most, in level order), F = F0 + sum of every F
// update, xb += sum of every xb update.
template <int N>
__device__ void tree_root(const FactorArgs<double>& a, const TreeArgs& ta, int root, int lane) {
  const Dims d = a.d;
  const int nb = d.nblock, nr = d.nr, nx = d.nx;
  const size_t nrn = (size_t)nr * N, nrnx = (size_t)nr * nx;
  // the contributing pair of each level (0: none), found before any load so
  // that every load is in flight at once
  int src[31];
#pragma unroll
  for (int lev = 0; lev < 31; ++lev) {
    const int K = 1 << lev;
    const long np = K < nb ? pairs_at_level(nb, K) : 0;
    const int jl = np > 0 ? (int)(K * (2 * np - 1)) : 0;
    src[lev] = (np > 0 && jl + K >= nb) ? jl : 0;
  }
  for (size_t e = lane; e < nrn; e += 32) {
    double v[31];
#pragma unroll
    for (int lev = 0; lev < 31; ++lev) v[lev] = src[lev] ? ldw(a.Rbuf + (size_t)src[lev] * nrn + e) : 0.0;
    double s = ldw(a.C + (size_t)nb * nrn + e);
#pragma unroll
    for (int lev = 0; lev < 31; ++lev) s += v[lev];
    a.C[(size_t)nb * nrn + e] = s;
  }
  for (size_t e = lane; e < nrnx; e += 32) {
    const int r = (int)(e % nr), c = (int)(e / nr);
    ta.Ffin[e] = a.F0[(size_t)c * nr + r] + ldw(a.Fbuf + (size_t)root * nrnx + e);
  }
  if (ta.xb) {
    for (int e = lane; e < nr * a.nrf; e += 32) {
      const int r = e % nr, c = e / nr;
      ta.xb[(size_t)c * a.ldx + r] += ldw(a.XB + (size_t)root * nr * a.nrf + e);
    }
  }
}

// The top levels of the cyclic reduction (at most TOP_WARPS pairs each) in one
// launch of one CTA: each level's pairs go one per warp, then the CTA applies
// the level's C_jpp updates (k_border_fix's work) before the next level; one
// launch replaces two per level, whose fixed cost dominates there.
constexpr int TOP_WARPS = 16;

template <int N, int NRM>
__global__ void __launch_bounds__(TOP_WARPS * 32, 1) k_factor_top_tc(FactorArgs<double> a, int k_first) {
  using S = TcShape<N>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double* Wt = reinterpret_cast<double*>(smem_raw + (size_t)warp * S::BYTES);
  const TcTree none{0, 0, 0};
  const int nb = a.d.nblock;
  const size_t nrn = (size_t)a.d.nr * N;
  for (int k = k_first; k < nb; k *= 2) {
    const long np = pairs_at_level(nb, k);
    for (long q = warp; q < np; q += TOP_WARPS)
      tc_pair<N, NRM>(a, k + (int)(2L * k * q), k, k == 1, Wt, lane, none);
    __syncthreads();
    for (size_t e = threadIdx.x; e < (size_t)np * nrn; e += blockDim.x) {
      const long q = (long)(e / nrn);
      const size_t idx = e % nrn;
      const int j = k + (int)(2L * k * q), jpp = min(j + k, nb);
      a.C[(size_t)jpp * nrn + idx] += ldw(a.Rbuf + (size_t)j * nrn + idx);
    }
    __syncthreads();
  }
}

// the root work after level-by-level launches with the tree bookkeeping
template <int N>
__global__ void __launch_bounds__(32) k_tree_root(FactorArgs<double> a, TreeArgs ta, int root) {
  tree_root<N>(a, ta, root, threadIdx.x);
}

template <int N, int NRM>
__global__ void __launch_bounds__(128, 4) k_factor_tree_tc(FactorArgs<double> a, TreeArgs ta) {
  using S = TcShape<N>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double* Wt = reinterpret_cast<double*>(smem_raw + (size_t)warp * S::BYTES);
  const int nb = a.d.nblock;
  const long leaves = pairs_at_level(nb, 1);
  for (;;) {
    int q = 0;
    if (lane == 0) q = atomicAdd(ta.leaf, 1);
    q = __shfl_sync(0xffffffffu, q, 0);
    if (q >= leaves) break;
    int j = 2 * q + 1;
    for (;;) {
      const int K = lowbit(j);
      TcTree tr;
      tr.gather = K / 2;
      tree_children(j, nb, tr.c1, tr.c2);
      tc_pair<N, NRM>(a, j, K, K == 1, Wt, lane, tr);
      const int par = tree_parent(j, nb);
      if (par == 0) {  // the root: every pair is done
        __threadfence();
        tree_root<N>(a, ta, j, lane);
        break;
      }
      // publish this node's results, then count the arrival at the parent
      __threadfence();
      int old = 0;
      if (lane == 0) old = atomicAdd(ta.cnt + par, 1);
      old = __shfl_sync(0xffffffffu, old, 0);
      int c1, c2;
      tree_children(par, nb, c1, c2);
      const int expected = (c1 != 0) + (c2 != 0);
      if (old + 1 < expected) break;  // the other child's warp will carry on
      __threadfence();                // acquire: the children's results are visible
      j = par;
    }
  }
}

// ---------------------------------------------------------------------------
// LU pair kernel for n = 16 and n = 32 in either precision.  One CTA per
// pair: 2n panel threads (one panel row each, in registers) plus one warp
// whose first nr lanes hold the border rows C_j.  Three phases as in the
// tensor-core kernel: register panel LU with the getrf pivot rule (the pivot
// search spans the panel warps: each publishes its best candidate row and its
// reciprocal, one barrier per column, double-buffered by column parity); the
// operator G = [L^-1; -M L^-1; -C' L^-1]; one product G * (P W)_top, on the
// FP64 tensor cores (DMMA 8x8x4) for double, as a 3xTF32 split on the tensor
// cores for float at n = 32, on the FP32 pipe for float at n = 16.
// ---------------------------------------------------------------------------
template <typename T> __device__ __forceinline__ T rcp_rn(T x);
template <> __device__ __forceinline__ double rcp_rn<double>(double x) { return __drcp_rn(x); }
template <> __device__ __forceinline__ float rcp_rn<float>(float x) { return __frcp_rn(x); }

// total order of pivot candidates: (hi, lo) of |a|, NaN below every number,
// finished rows below everything
__device__ __forceinline__ void pivot_key(double av, bool done, unsigned& hi, unsigned& lo) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(av);
  hi = done ? 0u : (av != av ? 1u : (unsigned)(b >> 32) + 1u);
  lo = (done || av != av) ? 0u : (unsigned)b;
}
__device__ __forceinline__ void pivot_key(float av, bool done, unsigned& hi, unsigned& lo) {
  hi = done ? 0u : (av != av ? 1u : (unsigned)__float_as_uint(av) + 1u);
  lo = 0u;
}

template <typename T, int N>
struct GrpShape {
  static constexpr int TPP = 2 * N;        // panel threads, one per panel row
  static constexpr int NTH = TPP + 32;     // + the border warp
  static constexpr int NWP = TPP / 32;     // warps in the pivot search
  static constexpr int NWA = NTH / 32;
  static constexpr int MT = 2 * N + 8;     // product rows: U-row, reduced row, border (nr <= 8)
  static constexpr int NTC = 2 * N + 8;    // trailing columns: x_jp, x_jpp, xb (nx <= 8)
  // trailing rows, compact: a TOP row keeps [D_jp | B_jp], a BOTTOM row
  // [E_j | B_j]; the structurally zero half of each row is not stored
  static constexpr int LDW = N + 8 + 1;
  static constexpr int LDG = N + 4;        // G rows (16-byte aligned rows, conflict-free fragments)
  static constexpr int LDS = N + 2;
  // FP64 product: DMMA tiles, warp w owns row tiles [w*RTW, (w+1)*RTW)
  static constexpr int MTILES = MT / 8, NTILES = NTC / 8;
  static constexpr int RTW = (MTILES + NWA - 1) / NWA;
  static constexpr int PC = NTILES % 3 == 0 ? 3 : NTILES;  // column tiles per pass
  // FP32 product: TR x TC thread grid, RPT x CPT elements per thread
  static constexpr int TR = 8, TC = NTH / TR;
  static constexpr int RPT = MT / TR, CPT = NTC / TC;
  static constexpr size_t BYTES =
      (size_t)(2 * N * LDW + MT * LDG + 2 * NWP * LDS) * sizeof(T) + (size_t)(2 * NWP * 4 + 2 * N) * sizeof(int);
  static_assert(MT % TR == 0 && NTC % TC == 0 && NTILES % PC == 0, "product tiling");
};

// element (row, col) of the trailing part of the work matrix from the compact
// rows: columns [0,N) x_jp (TOP rows only), [N,2N) x_jpp (BOTTOM rows only),
// [2N, 2N+8) xb
template <typename T, int N>
__device__ __forceinline__ T w_at(const T* Wt, int row, int col) {
  constexpr int LDW = GrpShape<T, N>::LDW;
  const bool top = row < N;
  if (col < N) return top ? Wt[row * LDW + col] : T(0);
  if (col < 2 * N) return top ? T(0) : Wt[row * LDW + col - N];
  return Wt[row * LDW + col - N];
}

// G * (P W)_top + [0; (P W)_bot; 0] -> the U-row of block j, the reduced row of
// block jp and the border updates (C_jp, the C_jpp buffer, the F buffer)
template <typename T, int N>
struct GrpProduct;

template <int N>
struct GrpProduct<double, N> {
  using S = GrpShape<double, N>;
  template <typename Out>
  __device__ static void run(const double* Wt, const double* Gs, const int* rowof, int t, Out out) {
    const int w = t >> 5, lane = t & 31, g = lane >> 2, q = lane & 3;
    const int mt0 = w * S::RTW;
#pragma unroll
    for (int pass = 0; pass < S::NTILES / S::PC; ++pass) {
      double acc[S::RTW][S::PC][2];
#pragma unroll
      for (int mi = 0; mi < S::RTW; ++mi)
#pragma unroll
        for (int ni = 0; ni < S::PC; ++ni) {
          const int row = (mt0 + mi) * 8 + g, col = (pass * S::PC + ni) * 8 + 2 * q;
          double c0 = 0.0, c1 = 0.0;
          if (mt0 + mi < S::MTILES && row >= N && row < 2 * N) {
            const int orow = rowof[row];
            c0 = w_at<double, N>(Wt, orow, col);
            c1 = w_at<double, N>(Wt, orow, col + 1);
          }
          acc[mi][ni][0] = c0;
          acc[mi][ni][1] = c1;
        }
#pragma unroll
      for (int ks = 0; ks < N / 4; ++ks) {
        double bfr[S::PC];
        const int orow = rowof[ks * 4 + q];
#pragma unroll
        for (int ni = 0; ni < S::PC; ++ni) bfr[ni] = w_at<double, N>(Wt, orow, (pass * S::PC + ni) * 8 + g);
#pragma unroll
        for (int mi = 0; mi < S::RTW; ++mi) {
          if (mt0 + mi < S::MTILES) {
            const double afr = Gs[((mt0 + mi) * 8 + g) * S::LDG + ks * 4 + q];
#pragma unroll
            for (int ni = 0; ni < S::PC; ++ni) dmma_8x8x4(acc[mi][ni][0], acc[mi][ni][1], afr, bfr[ni]);
          }
        }
      }
#pragma unroll
      for (int mi = 0; mi < S::RTW; ++mi)
        if (mt0 + mi < S::MTILES)
#pragma unroll
          for (int ni = 0; ni < S::PC; ++ni)
#pragma unroll
            for (int hh = 0; hh < 2; ++hh)
              out((mt0 + mi) * 8 + g, (pass * S::PC + ni) * 8 + 2 * q + hh, acc[mi][ni][hh]);
    }
  }
};

template <int N>
struct GrpProduct<float, N> {
  using S = GrpShape<float, N>;
  template <typename Out>
  __device__ static void run(const float* Wt, const float* Gs, const int* rowof, int t, Out out) {
    const int tr = t % S::TR, tc = t / S::TR;
    float acc[S::RPT][S::CPT];
#pragma unroll
    for (int ii = 0; ii < S::RPT; ++ii) {
      const int row = tr + S::TR * ii;
#pragma unroll
      for (int jj = 0; jj < S::CPT; ++jj)
        acc[ii][jj] = (row >= N && row < 2 * N) ? w_at<float, N>(Wt, rowof[row], tc + S::TC * jj) : 0.0f;
    }
#pragma unroll 4
    for (int kk = 0; kk < N; ++kk) {
      const int orow = rowof[kk];
      float bv[S::CPT], av[S::RPT];
#pragma unroll
      for (int jj = 0; jj < S::CPT; ++jj) bv[jj] = w_at<float, N>(Wt, orow, tc + S::TC * jj);
#pragma unroll
      for (int ii = 0; ii < S::RPT; ++ii) av[ii] = Gs[(tr + S::TR * ii) * S::LDG + kk];
#pragma unroll
      for (int ii = 0; ii < S::RPT; ++ii)
#pragma unroll
        for (int jj = 0; jj < S::CPT; ++jj) acc[ii][jj] = fmaf(av[ii], bv[jj], acc[ii][jj]);
    }
#pragma unroll
    for (int ii = 0; ii < S::RPT; ++ii)
#pragma unroll
      for (int jj = 0; jj < S::CPT; ++jj) out(tr + S::TR * ii, tc + S::TC * jj, acc[ii][jj]);
  }
};

// FP32 n=32: the product on the tensor cores as a 3xTF32 split
// (mma.sync m16n8k8: a*b ~ a_small*b_big + a_big*b_small + a_big*b_big with
// a_big = tf32(a), a_small = tf32(a - a_big), FP32 accumulators), close to
// FP32 accuracy at a tenth of the FMA product's instructions.  Warp w owns
// column tiles [3w, 3w+3) of all five 16-row tiles (rows >= 72 are padding).
__device__ __forceinline__ unsigned to_tf32(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ void split_tf32(float x, unsigned& big, unsigned& small) {
  big = to_tf32(x);
  small = to_tf32(x - __uint_as_float(big));
}
__device__ __forceinline__ void mma_tf32(float (&c)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

template <>
struct GrpProduct<float, 32> {
  static constexpr int N = 32;
  using S = GrpShape<float, N>;
  static constexpr int M16 = (S::MT + 15) / 16, NPW = S::NTILES / S::NWA;
  static_assert(S::NTILES % S::NWA == 0, "column tiles per warp");
  template <typename Out>
  __device__ static void run(const float* Wt, const float* Gs, const int* rowof, int t, Out out) {
    const int w = t >> 5, lane = t & 31, g = lane >> 2, q = lane & 3;
    float acc[M16][NPW][4];
    // [0; (P W)_bot; 0]: accumulator element c0..c3 = (row r, col c), (r, c+1),
    // (r+8, c), (r+8, c+1) with r = 16 mi + g, c = 8 nt + 2q
#pragma unroll
    for (int mi = 0; mi < M16; ++mi)
#pragma unroll
      for (int ni = 0; ni < NPW; ++ni) {
        const int col = (w * NPW + ni) * 8 + 2 * q;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int row = mi * 16 + g + 8 * h;
          const bool bot = row >= N && row < 2 * N;
          const int orow = bot ? rowof[row] : 0;
          acc[mi][ni][2 * h] = bot ? w_at<float, N>(Wt, orow, col) : 0.0f;
          acc[mi][ni][2 * h + 1] = bot ? w_at<float, N>(Wt, orow, col + 1) : 0.0f;
        }
      }
#pragma unroll
    for (int ks = 0; ks < N / 8; ++ks) {
      // B fragment of (P W)_top: (k = 8 ks + q, col = 8 nt + g) and k + 4
      const int o0 = rowof[ks * 8 + q], o1 = rowof[ks * 8 + q + 4];
      unsigned bb[NPW][2], bs[NPW][2];
#pragma unroll
      for (int ni = 0; ni < NPW; ++ni) {
        const int col = (w * NPW + ni) * 8 + g;
        split_tf32(w_at<float, N>(Wt, o0, col), bb[ni][0], bs[ni][0]);
        split_tf32(w_at<float, N>(Wt, o1, col), bb[ni][1], bs[ni][1]);
      }
#pragma unroll
      for (int mi = 0; mi < M16; ++mi) {
        // A fragment of G: (r, k), (r + 8, k), (r, k + 4), (r + 8, k + 4)
        const int r0 = mi * 16 + g, r1 = r0 + 8, kk = ks * 8 + q;
        const float av[4] = {r0 < S::MT ? Gs[r0 * S::LDG + kk] : 0.0f, r1 < S::MT ? Gs[r1 * S::LDG + kk] : 0.0f,
                             r0 < S::MT ? Gs[r0 * S::LDG + kk + 4] : 0.0f,
                             r1 < S::MT ? Gs[r1 * S::LDG + kk + 4] : 0.0f};
        unsigned ab[4], as[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) split_tf32(av[e], ab[e], as[e]);
#pragma unroll
        for (int ni = 0; ni < NPW; ++ni) {
          mma_tf32(acc[mi][ni], as, bb[ni][0], bb[ni][1]);
          mma_tf32(acc[mi][ni], ab, bs[ni][0], bs[ni][1]);
          mma_tf32(acc[mi][ni], ab, bb[ni][0], bb[ni][1]);
        }
      }
    }
#pragma unroll
    for (int mi = 0; mi < M16; ++mi)
#pragma unroll
      for (int ni = 0; ni < NPW; ++ni)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int row = mi * 16 + g + 8 * h, col = (w * NPW + ni) * 8 + 2 * q;
          if (row < S::MT) {
            out(row, col, acc[mi][ni][2 * h]);
            out(row, col + 1, acc[mi][ni][2 * h + 1]);
          }
        }
  }
};

// CTAs per SM the register budget is sized for (FP64 n=32 is shared-memory
// bound at 5, FP32 n=32 register bound at 6)
template <typename T, int N>
constexpr int grp_min_blocks() { return N == 32 ? (sizeof(T) == 8 ? 5 : 6) : 4; }

// pairs [q0, q1) step qs of one system and level, one per CTA
template <typename T, int N, bool COH>
__device__ __forceinline__ void grp_body(const FactorArgs<T>& a, long q0, long q1, long qs) {
  using S = GrpShape<T, N>;
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* Wt = reinterpret_cast<T*>(smem_raw);          // [2N][LDW] trailing columns, original rows
  T* Gs = Wt + 2 * N * S::LDW;                     // [MT][LDG] L rows, then G
  T* slot = Gs + S::MT * S::LDG;                   // [2][NWP][LDS] candidate pivot row + reciprocal
  int* hdr = reinterpret_cast<int*>(slot + 2 * S::NWP * S::LDS);  // [2][NWP][4] hi, lo, position, thread
  int* rowof = hdr + 2 * S::NWP * 4;               // position -> original row
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const Dims d = a.d;
  const int nr = d.nr, nx = d.nx;
  constexpr int n = N, n2 = 2 * N;
  constexpr size_t nn = (size_t)N * N;
  const size_t nnx = (size_t)n * nx, nrn = (size_t)nr * n, nrnx = (size_t)nr * nx;
  const int k = a.k;
  const bool first = a.first != 0;
  const bool panel = t < n2;                 // panel row t
  const bool brow = !panel && t - n2 < nr;   // border row t - 2N
  const bool top = t < n;
  const int ri = top ? t : t - n;

  for (long qq = q0; qq < q1; qq += qs) {
    const int j = k + (int)(2L * k * qq), jp = j - k;
    __syncthreads();  // the previous pair's readers of Wt/Gs are done
    // ------------------------------------------------------------ load
    // every global load of the pair is issued before the first shared store
    constexpr int IT = (int)((nn + S::NTH - 1) / S::NTH), IB = (8 * N + S::NTH - 1) / S::NTH;
    T row[N], vd[IT], ve[IT], vbt[IB], vbb[IB];
    // the source (loaded FP64 matrix at the first level, working copy after)
    // is chosen once per pair, so every load below is a plain batched load
    auto load = [&](const auto* D, const auto* E, const auto* Bm, const auto* C) {
      if (panel) {
        const size_t base = top ? (size_t)jp * nn : (size_t)j * nn;
        const auto* P = top ? E : D;
#pragma unroll
        for (int c = 0; c < N; ++c) row[c] = T(ldro<COH>(P + base + (size_t)c * n + ri));
      } else {
#pragma unroll
        for (int c = 0; c < N; ++c)
          row[c] = brow ? T(ldro<COH>(C + (size_t)j * nrn + (size_t)c * nr + (t - n2))) : T(0);
      }
#pragma unroll
      for (int it = 0; it < IT; ++it) {
        const int idx = t + S::NTH * it;
        const bool in = idx < (int)nn;
        vd[it] = in ? T(ldro<COH>(D + (size_t)jp * nn + idx)) : T(0);
        ve[it] = in ? T(ldro<COH>(E + (size_t)j * nn + idx)) : T(0);
      }
#pragma unroll
      for (int it = 0; it < IB; ++it) {
        const int idx = t + S::NTH * it;
        const bool in = idx < nx * n;
        vbt[it] = in ? T(ldro<COH>(Bm + (size_t)jp * nnx + idx)) : T(0);
        vbb[it] = in ? T(ldro<COH>(Bm + (size_t)j * nnx + idx)) : T(0);
      }
    };
    if (first) load(a.D0, a.E0, a.B0, a.C0);
    else load(a.D, a.E, a.B, a.C);

    // trailing columns, compact: TOP rows [D_jp B_jp], BOTTOM rows [E_j B_j]
#pragma unroll
    for (int it = 0; it < IT; ++it) {
      const int idx = t + S::NTH * it;
      if (idx < (int)nn) {
        const int r = idx % n, c = idx / n;
        Wt[r * S::LDW + c] = vd[it];
        Wt[(n + r) * S::LDW + c] = ve[it];
      }
    }
#pragma unroll
    for (int it = 0; it < IB; ++it) {
      const int idx = t + S::NTH * it;
      if (idx < 8 * n) {
        const int r = idx % n, c = idx / n;
        Wt[r * S::LDW + n + c] = vbt[it];
        Wt[(n + r) * S::LDW + n + c] = vbb[it];
      }
    }
    // --------------------------------------------------- phase 1: panel LU
    int mypos = t, info = 0;
    bool done = !panel;  // border and idle lanes never pivot
#pragma unroll
    for (int i = 0; i < N; ++i) {
      const int par = i & 1;
      if (w < S::NWP) {
        // every lane forms the reciprocal of its own candidate while the pivot
        // is searched; the winner publishes it with its row
        const T rc = rcp_rn(row[i]);
        unsigned hi, lo;
        pivot_key(dev_abs(row[i]), done, hi, lo);
        const unsigned hmax = __reduce_max_sync(FULL, hi);
        const unsigned m = __ballot_sync(FULL, hi == hmax && !done);
        int wl = -1;  // this warp's best candidate lane
        if (m != 0u) {
          if (__popc(m) == 1) {
            wl = __ffs(m) - 1;
          } else {
            const bool c1 = hi == hmax && !done;
            const unsigned lmax = __reduce_max_sync(FULL, c1 ? lo : 0u);
            const bool cand = c1 && lo == lmax;
            const unsigned pm = __reduce_min_sync(FULL, cand ? (unsigned)mypos : 0xffffffffu);
            wl = __ffs(__ballot_sync(FULL, cand && (unsigned)mypos == pm)) - 1;
          }
        }
        int4* h = reinterpret_cast<int4*>(hdr) + par * S::NWP + w;
        T* sl = slot + (par * S::NWP + w) * S::LDS;
        if (lane == wl) {
          *h = make_int4((int)hi, (int)lo, mypos, t);
#pragma unroll
          for (int c = (i & ~1); c < N; c += 2) store2(sl + c, row[c], row[c + 1]);
          sl[N] = rc;
        } else if (wl < 0 && lane == 0) {
          *h = make_int4(0, 0, 0x7fffffff, 0);  // no candidate left in this warp
        }
      }
      __syncthreads();
      int wb = 0;
      int4 hw = reinterpret_cast<const int4*>(hdr)[par * S::NWP];
      if (S::NWP == 2) {
        const int4 h1 = reinterpret_cast<const int4*>(hdr)[par * S::NWP + 1];
        const unsigned hi0 = (unsigned)hw.x, hi1 = (unsigned)h1.x;
        const unsigned lo0 = (unsigned)hw.y, lo1 = (unsigned)h1.y;
        if (hi1 > hi0 || (hi1 == hi0 && (lo1 > lo0 || (lo1 == lo0 && h1.z < hw.z)))) {
          wb = 1;
          hw = h1;
        }
      }
      const int pmin = hw.z, p = hw.w;
      const T* u = slot + (par * S::NWP + wb) * S::LDS;
      const T piv = u[i];
      if (piv == T(0) && info == 0) info = i + 1;
      const T rinv = piv != T(0) ? u[N] : T(0);
      if (panel) {
        if (!done && mypos == i && t != p) mypos = pmin;
        if (t == p) mypos = i;
      }
      if ((panel && !done && t != p) || brow) {
        const T l = row[i] * rinv;
        row[i] = l;
#pragma unroll
        for (int c = (i + 1) & ~1; c < N; c += 2) {
          T u0, u1;
          load2(u + c, u0, u1);
          if (c > i) row[c] = fma(-l, u0, row[c]);
          row[c + 1] = fma(-l, u1, row[c + 1]);
        }
      }
      if (t == p) done = true;
    }
    if (info != 0) {
      if (t == 0) report(a.st, DEV_ZERO_PIVOT, j, info, k);
      continue;
    }
    // panel factors T_j (L\U and M in getrf row order), row map, C_j U^-1, L rows
    if (panel) {
      T* Tj = a.Tm + (size_t)j * szT(d);
#pragma unroll
      for (int c = 0; c < N; ++c) Tj[(size_t)mypos + (size_t)c * n2] = row[c];
      rowof[mypos] = t;
      a.P[(size_t)j * szP(d) + mypos] = (unsigned char)t;
      if (mypos < n) {
#pragma unroll
        for (int c = 0; c < N; ++c) Gs[mypos * S::LDG + c] = row[c];
      }
    } else if (brow) {
      T* Cj = a.C + (size_t)j * nrn + (t - n2);
#pragma unroll
      for (int c = 0; c < N; ++c) Cj[(size_t)c * nr] = row[c];
    }
    __syncthreads();
    // ------------------------------------ phase 2: operator G (X L = R)
    // R rows: identity for U-row positions, -M for reduced positions, -C' for border rows
    {
      T x[N];
      const bool unit = panel && mypos < n;
#pragma unroll
      for (int c = 0; c < N; ++c) x[c] = unit ? (c == mypos ? T(1) : T(0)) : -row[c];
      // right-looking: once x[mm] is final, update every x[c], c < mm
#pragma unroll
      for (int mm = N - 1; mm > 0; --mm) {
        const T xm = x[mm];
        const T* Lrow = Gs + mm * S::LDG;
#pragma unroll
        for (int c = 0; c < mm; c += 2) {
          const T l0 = Lrow[c], l1 = Lrow[c + 1];
          x[c] = fma(-xm, l0, x[c]);
          if (c + 1 < mm) x[c + 1] = fma(-xm, l1, x[c + 1]);
        }
      }
      __syncthreads();
      const int grow = panel ? mypos : n2 + (t - n2);
      if (panel || t - n2 < 8) {
#pragma unroll
        for (int c = 0; c < N; ++c) Gs[grow * S::LDG + c] = (panel || brow) ? x[c] : T(0);
      }
    }
    __syncthreads();
    // ------------------------------------------ phase 3: G * (P W)_top
    GrpProduct<T, N>::run(Wt, Gs, rowof, t, [&](int prow, int col, T v) {
      if (prow < n2) {
        const bool ur = prow < n;
        const int rr = ur ? prow : prow - n;
        const size_t blk = ur ? (size_t)j : (size_t)jp;
        if (col < n) a.D[blk * nn + (size_t)col * n + rr] = v;
        else if (col < n2) a.E[blk * nn + (size_t)(col - n) * n + rr] = v;
        else if (col < n2 + nx) a.B[blk * nnx + (size_t)(col - n2) * n + rr] = v;
      } else {
        const int rr = prow - n2;
        if (rr < nr) {
          if (col < n) {
            const size_t o = (size_t)jp * nrn + (size_t)col * nr + rr;
            a.C[o] = ldsrc_c<COH>(first, a.C0, a.C, o) + v;
          } else if (col < n2) {
            a.Rbuf[(size_t)j * nrn + (size_t)(col - n) * nr + rr] = v;
          } else if (col < n2 + nx) {
            a.Fbuf[(size_t)j * nrnx + (size_t)(col - n2) * nr + rr] = (double)v;
          }
        }
      }
    });
  }
}

template <typename T, int N, bool BATCH = false>
__global__ void __launch_bounds__(2 * N + 32, grp_min_blocks<T, N>())
    k_factor_lu_grp(FactorArgs<T> a0, const FactorArgs<T>* tab, const BatchCta* cmap) {
  FactorArgs<T> ab;  // this CTA's system (batch only)
  long q0, q1, qs;
  pair_range<BATCH>(a0, tab, cmap, 1, 0, ab, q0, q1, qs);
  grp_body<T, N, false>(BATCH ? ab : a0, q0, q1, qs);
}

// ---------------------------------------------------------------------------
// Large blocks, LU: blocked right-looking elimination of the pair's work
// matrix (one CTA per pair, the matrix in the CTA's global slab, L2
// resident).  The panel columns go in blocks of BLK_W: a block is factored in
// shared memory with the getrf pivot rule (border rows eliminated, never
// pivots), its row interchanges are applied to every other column, the
// BLK_W rows of the trailing columns are solved with the block's unit lower
// triangle, and the rows below are updated with one product of depth BLK_W
// -- FP64 tensor cores (DMMA 8x8x4) for double, FMA tiles for float.  The
// result equals the unblocked elimination (getrf on the panel followed by
// the trailing updates) up to rounding order.
// ---------------------------------------------------------------------------
constexpr int BLK_W = 32;
constexpr int BLK_ROWS_MAX = 512;  // 2n + nr of the blocked kernel
constexpr int LAST_BLOCKED_MIN = 64;  // last blocks of this order and above: blocked LU

// W[c*R + rowp[r]] -= sum_m L[m*LD + r] * W[c*R + rowp[k0 + m]] for positions r in
// [r0, R), c in [c0, NC), m < w; L: the factored block in shared memory (column m,
// position r); rowp: position -> row of W
template <typename T>
__device__ void blk_update(T* W, int R, int NC, const T* Lsm, int LD, int k0, int w, int r0, int c0,
                           const int* rowp) {
  const int tid = threadIdx.x, bs = blockDim.x;
  const int rows = R - r0, cols = NC - c0;
  if (rows <= 0 || cols <= 0) return;
  if constexpr (sizeof(T) == 8) {
    // 16 x 16 output per warp iteration (2 x 2 DMMA tiles)
    const int lane = tid & 31, warp = tid >> 5, nw = bs >> 5;
    const int g = lane >> 2, q = lane & 3;
    const int tr = (rows + 15) / 16, tc = (cols + 15) / 16;
    constexpr int KS = BLK_W / 4;
    for (int t = warp; t < tr * tc; t += nw) {
      const int rb = r0 + (t % tr) * 16, cb = c0 + (t / tr) * 16;
      // every global load of the tile (B fragments, C) is in flight at once
      double bf[KS][2], cv[2][2][2];
#pragma unroll
      for (int ks = 0; ks < KS; ++ks) {
        const int m = ks * 4 + q;
#pragma unroll
        for (int v = 0; v < 2; ++v) {
          const int c = cb + v * 8 + g;
          bf[ks][v] = (m < w && c < NC) ? W[(size_t)c * R + rowp[k0 + m]] : 0.0;
        }
      }
#pragma unroll
      for (int u = 0; u < 2; ++u)
#pragma unroll
        for (int v = 0; v < 2; ++v)
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int r = rb + u * 8 + g, c = cb + v * 8 + 2 * q + h;
            cv[u][v][h] = (r < R && c < NC) ? W[(size_t)c * R + rowp[r]] : 0.0;
          }
      double acc[2][2][2] = {};
#pragma unroll
      for (int ks = 0; ks < KS; ++ks) {
        const int m = ks * 4 + q;
        double af[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const int r = rb + u * 8 + g;
          af[u] = (m < w && r < R) ? Lsm[(size_t)m * LD + r] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 2; ++u)
#pragma unroll
          for (int v = 0; v < 2; ++v) dmma_8x8x4(acc[u][v][0], acc[u][v][1], af[u], bf[ks][v]);
      }
#pragma unroll
      for (int u = 0; u < 2; ++u)
#pragma unroll
        for (int v = 0; v < 2; ++v)
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int r = rb + u * 8 + g, c = cb + v * 8 + 2 * q + h;
            if (r < R && c < NC) W[(size_t)c * R + rowp[r]] = cv[u][v][h] - acc[u][v][h];
          }
    }
  } else {
    // 4 x 4 output per thread
    const int tr = (rows + 3) / 4, tc = (cols + 3) / 4;
    for (int t = tid; t < tr * tc; t += bs) {
      const int rb = r0 + (t % tr) * 4, cb = c0 + (t / tr) * 4;
      T acc[4][4] = {};
#pragma unroll 4
      for (int m = 0; m < w; ++m) {
        T av[4], bv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          av[u] = rb + u < R ? Lsm[(size_t)m * LD + rb + u] : T(0);
          bv[u] = cb + u < NC ? W[(size_t)(cb + u) * R + rowp[k0 + m]] : T(0);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int v = 0; v < 4; ++v) acc[u][v] = fma(av[u], bv[v], acc[u][v]);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v)
          if (rb + u < R && cb + v < NC) W[(size_t)(cb + v) * R + rowp[rb + u]] -= acc[u][v];
    }
  }
}

// Blocked right-looking LU of the first npiv columns of the R x NC column-major
// matrix W (ld R) by one CTA: the getrf pivot rule among positions [i, ncand)
// (rows at positions >= ncand are eliminated but never pivots), the
// interchanges kept in the position -> row map s_perm (rows of W never move;
// s_perm holds the identity on entry), each block of BLK_W columns factored in
// shared memory Pb (BLK_W x R), the block's rows of the columns right of it
// solved with its unit lower triangle, the rows below updated with one product
// of depth BLK_W.  Returns the LAPACK info: 0, or the first zero pivot + 1.
template <typename T>
__device__ int blk_eliminate(T* W, int R, int NC, int npiv, int ncand, T* Pb, int* s_perm, T* sv, int* si) {
  const int tid = threadIdx.x, bs = blockDim.x;
  int info = 0;
  for (int kb = 0; kb < npiv && info == 0; kb += BLK_W) {
    const int w = npiv - kb < BLK_W ? npiv - kb : BLK_W;
    // stage the block's columns (all rows) in shared memory
    for (int e = tid; e < w * R; e += bs) {
      const int r = e % R, c = e / R;
      Pb[(size_t)c * R + r] = W[(size_t)(kb + c) * R + s_perm[r]];
    }
    __syncthreads();
    for (int i = 0; i < w; ++i) {
      const int gi = kb + i;
      T* ci = Pb + (size_t)i * R;
      T best = T(-1);
      int bi = gi;  // stays in range even when every candidate is NaN
      for (int r = gi + tid; r < ncand; r += bs) {
        const T v = dev_abs(ci[r]);
        if (v > best) { best = v; bi = r; }
      }
      block_argmax(best, bi, sv, si);
      const T pv = ci[bi];
      __syncthreads();  // every thread holds the pivot before the rows are swapped
      if (pv == T(0)) { info = gi + 1; break; }
      if (bi != gi && tid < w) {
        T* col = Pb + (size_t)tid * R;
        const T t = col[gi]; col[gi] = col[bi]; col[bi] = t;
      }
      if (bi != gi && tid == w) { const int t = s_perm[gi]; s_perm[gi] = s_perm[bi]; s_perm[bi] = t; }
      __syncthreads();
      // one thread per row below the pivot: its multiplier, then its update
      const T rinv = T(1) / pv;
      for (int r = gi + 1 + tid; r < R; r += bs) {
        const T l = ci[r] * rinv;
        ci[r] = l;
        for (int c = i + 1; c < w; ++c) Pb[(size_t)c * R + r] -= l * Pb[(size_t)c * R + gi];
      }
      __syncthreads();
    }
    if (info != 0) break;
    // the factored block back to the slab (by position)
    for (int e = tid; e < w * R; e += bs) {
      const int r = e % R, c = e / R;
      W[(size_t)(kb + c) * R + s_perm[r]] = Pb[(size_t)c * R + r];
    }
    __syncthreads();
    // rows [kb, kb+w) of the columns right of the block: unit lower solve
    for (int c = kb + w + tid; c < NC; c += bs) {
      T* col = W + (size_t)c * R;
      T y[BLK_W];
#pragma unroll
      for (int r = 0; r < BLK_W; ++r) y[r] = r < w ? col[s_perm[kb + r]] : T(0);
#pragma unroll
      for (int m = 0; m < BLK_W; ++m) {
#pragma unroll
        for (int r = m + 1; r < BLK_W; ++r)
          if (r < w) y[r] = fma(-Pb[(size_t)m * R + kb + r], y[m], y[r]);
      }
#pragma unroll
      for (int r = 0; r < BLK_W; ++r)
        if (r < w) col[s_perm[kb + r]] = y[r];
    }
    __syncthreads();
    // rows below the block: one product of depth w
    blk_update<T>(W, R, NC, Pb, R, kb, w, kb + w, kb + w, s_perm);
    __syncthreads();
  }
  return info;
}

template <typename T>
__global__ void __launch_bounds__(256, 2) k_factor_lu_blocked(FactorArgs<T> a, T* slab, size_t slab_elems) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ T sv[32];
  __shared__ int si[32];
  __shared__ int s_perm[BLK_ROWS_MAX];  // position -> row of the slab (rows never move)
  const int tid = threadIdx.x, bs = blockDim.x;
  const Dims d = a.d;
  const int n = d.n, nr = d.nr, nx = d.nx, nb = d.nblock;
  const int n2 = 2 * n, R = n2 + nr, NC = 3 * n + nx;
  const size_t nn = (size_t)n * n, nnx = (size_t)n * nx, nrn = (size_t)nr * n, nrnx = (size_t)nr * nx;
  T* Pb = reinterpret_cast<T*>(smem_raw);  // [BLK_W][R] the current panel block, column-major
  T* W = slab + (size_t)blockIdx.x * slab_elems;
  const int k = a.k;
  const long np = pairs_at_level(nb, k);
  const bool first = a.first != 0;
  for (long q = blockIdx.x; q < np; q += gridDim.x) {
    const int j = k + (int)(2L * k * q), jp = j - k;
    const size_t oj = (size_t)j * nn, ojp = (size_t)jp * nn;
    // ------------------------------------------------------------ load
    // groups of UL elements per thread: the group's loads are issued before its stores
    constexpr int UL = 4;
    for (int base = 0; base < (int)nn; base += bs * UL) {
      T ejp[UL], djp[UL], dj[UL], ej[UL];
#pragma unroll
      for (int u = 0; u < UL; ++u) {
        const int idx = base + tid + u * bs;
        const bool in = idx < (int)nn;
        ejp[u] = in ? ldg_src(first, a.E0, a.E, ojp + idx) : T(0);
        djp[u] = in ? ldg_src(first, a.D0, a.D, ojp + idx) : T(0);
        dj[u] = in ? ldg_src(first, a.D0, a.D, oj + idx) : T(0);
        ej[u] = in ? ldg_src(first, a.E0, a.E, oj + idx) : T(0);
      }
#pragma unroll
      for (int u = 0; u < UL; ++u) {
        const int idx = base + tid + u * bs;
        if (idx < (int)nn) {
          const int i = idx % n, c = idx / n;
          W[(size_t)c * R + i] = ejp[u];
          W[(size_t)(n + c) * R + i] = djp[u];
          W[(size_t)(n2 + c) * R + i] = T(0);
          W[(size_t)c * R + n + i] = dj[u];
          W[(size_t)(n + c) * R + n + i] = T(0);
          W[(size_t)(n2 + c) * R + n + i] = ej[u];
        }
      }
    }
    for (int idx = tid; idx < (int)nnx; idx += bs) {
      const int i = idx % n, c = idx / n;
      W[(size_t)(3 * n + c) * R + i] = ldsrc(first, a.B0, a.B, (size_t)jp * nnx + idx);
      W[(size_t)(3 * n + c) * R + n + i] = ldsrc(first, a.B0, a.B, (size_t)j * nnx + idx);
    }
    for (int idx = tid; idx < (int)nrn; idx += bs) {
      const int r = idx % nr, c = idx / nr;
      W[(size_t)c * R + n2 + r] = ldsrc(first, a.C0, a.C, (size_t)j * nrn + idx);
      W[(size_t)(n + c) * R + n2 + r] = T(0);
      W[(size_t)(n2 + c) * R + n2 + r] = T(0);
    }
    for (int idx = tid; idx < (int)nrnx; idx += bs) {
      const int r = idx % nr, c = idx / nr;
      W[(size_t)(3 * n + c) * R + n2 + r] = T(0);
    }
    for (int r = tid; r < R; r += bs) s_perm[r] = r;
    __syncthreads();
    // ------------------------------------------------- blocked elimination
    const int info = blk_eliminate<T>(W, R, NC, n, n2, Pb, s_perm, sv, si);
    if (info != 0) {
      if (tid == 0) report(a.st, DEV_ZERO_PIVOT, j, info, k);
      __syncthreads();
      continue;
    }
    // ---------------------------------------------------------------- store
    T* Tj = a.Tm + (size_t)j * szT(d);
    for (int base = 0; base < (int)(2 * nn); base += bs * UL) {
      T v[UL];
#pragma unroll
      for (int u = 0; u < UL; ++u) {
        const int idx = base + tid + u * bs;
        v[u] = idx < (int)(2 * nn) ? W[(size_t)(idx / n2) * R + s_perm[idx % n2]] : T(0);
      }
#pragma unroll
      for (int u = 0; u < UL; ++u) {
        const int idx = base + tid + u * bs;
        if (idx < (int)(2 * nn)) Tj[idx] = v[u];
      }
    }
    unsigned char* Pj = a.P + (size_t)j * szP(d);
    // row map (getrf order): the original row at each position
    for (int r = tid; r < n2; r += bs) Pj[r] = (unsigned char)s_perm[r];
    for (int i = tid; i < n; i += bs) Pj[n2 + i] = (unsigned char)i;
    for (int base = 0; base < (int)nn; base += bs * UL) {
      T v0[UL], v1[UL], v2[UL], v3[UL];
#pragma unroll
      for (int u = 0; u < UL; ++u) {
        const int idx = base + tid + u * bs;
        const int i = idx % n, c = idx / n;
        const bool in = idx < (int)nn;
        const int pu = in ? s_perm[i] : 0, pr = in ? s_perm[n + i] : 0;
        v0[u] = in ? W[(size_t)(n + c) * R + pu] : T(0);
        v1[u] = in ? W[(size_t)(n2 + c) * R + pu] : T(0);
        v2[u] = in ? W[(size_t)(n + c) * R + pr] : T(0);
        v3[u] = in ? W[(size_t)(n2 + c) * R + pr] : T(0);
      }
#pragma unroll
      for (int u = 0; u < UL; ++u) {
        const int idx = base + tid + u * bs;
        if (idx < (int)nn) {
          a.D[oj + idx] = v0[u];
          a.E[oj + idx] = v1[u];
          a.D[ojp + idx] = v2[u];
          a.E[ojp + idx] = v3[u];
        }
      }
    }
    for (int idx = tid; idx < (int)nnx; idx += bs) {
      const int i = idx % n, c = idx / n;
      a.B[(size_t)j * nnx + idx] = W[(size_t)(3 * n + c) * R + s_perm[i]];
      a.B[(size_t)jp * nnx + idx] = W[(size_t)(3 * n + c) * R + s_perm[n + i]];
    }
    for (int idx = tid; idx < (int)nrn; idx += bs) {
      const int r = idx % nr, c = idx / nr;
      const size_t oc = (size_t)jp * nrn + idx;
      a.C[(size_t)j * nrn + idx] = W[(size_t)c * R + n2 + r];
      const T cjp = first ? T(a.C0[oc]) : a.C[oc];
      a.C[oc] = cjp + W[(size_t)(n + c) * R + n2 + r];
      a.Rbuf[(size_t)j * nrn + idx] = W[(size_t)(n2 + c) * R + n2 + r];
    }
    for (int idx = tid; idx < (int)nrnx; idx += bs) {
      const int r = idx % nr, c = idx / nr;
      a.Fbuf[(size_t)j * nrnx + idx] = W[(size_t)(3 * n + c) * R + n2 + r];
    }
    __syncthreads();
  }
}

#include "bcr_umma.cuh"

// ---------------------------------------------------------------------------
// Large blocks: one CTA eliminates one pair; the (2n+nr) x (3n+nx) work
// matrix lives in a global scratch slab of the CTA (column-major, ld = R),
// which stays in L2 while the CTA works on it.  Same elimination as the warp
// kernels (getrf pivot rule, dlarfg reflectors, border rows eliminated by the
// U rows), parallelised over the CTA's threads with block barriers.
// ---------------------------------------------------------------------------
template <typename T, int SEL>
__global__ void __launch_bounds__(256) k_factor_cta(FactorArgs<T> a, T* slab, size_t slab_elems) {
  __shared__ T sv[32];
  __shared__ int si[32];
  __shared__ T s_tau[256];
  __shared__ int s_piv[256];
  const int tid = threadIdx.x, bs = blockDim.x;
  const Dims d = a.d;
  const int n = d.n, nr = d.nr, nx = d.nx, nb = d.nblock;
  const int n2 = 2 * n, R = n2 + nr, NC = 3 * n + nx;
  const size_t nn = (size_t)n * n, nnx = (size_t)n * nx, nrn = (size_t)nr * n, nrnx = (size_t)nr * nx;
  T* W = slab + (size_t)blockIdx.x * slab_elems;
  const int k = a.k;
  const long np = pairs_at_level(nb, k);
  const bool first = a.first != 0;
  for (long q = blockIdx.x; q < np; q += gridDim.x) {
    const int j = k + (int)(2L * k * q), jp = j - k;
    const size_t oj = (size_t)j * nn, ojp = (size_t)jp * nn;
    // ------------------------------------------------------------ load
    for (int idx = tid; idx < (int)nn; idx += bs) {
      const int i = idx % n, c = idx / n;
      T ejp, djp, dj, ej;
      if (first) {
        ejp = T(a.E0[ojp + idx]); djp = T(a.D0[ojp + idx]); dj = T(a.D0[oj + idx]); ej = T(a.E0[oj + idx]);
      } else {
        ejp = a.E[ojp + idx]; djp = a.D[ojp + idx]; dj = a.D[oj + idx]; ej = a.E[oj + idx];
      }
      W[(size_t)c * R + i] = ejp;
      W[(size_t)(n + c) * R + i] = djp;
      W[(size_t)(n2 + c) * R + i] = T(0);
      W[(size_t)c * R + n + i] = dj;
      W[(size_t)(n + c) * R + n + i] = T(0);
      W[(size_t)(n2 + c) * R + n + i] = ej;
    }
    for (int idx = tid; idx < (int)nnx; idx += bs) {
      const int i = idx % n, c = idx / n;
      const size_t o1 = (size_t)jp * nnx + idx, o2 = (size_t)j * nnx + idx;
      W[(size_t)(3 * n + c) * R + i] = first ? T(a.B0[o1]) : a.B[o1];
      W[(size_t)(3 * n + c) * R + n + i] = first ? T(a.B0[o2]) : a.B[o2];
    }
    for (int idx = tid; idx < (int)nrn; idx += bs) {
      const int r = idx % nr, c = idx / nr;
      const size_t o = (size_t)j * nrn + idx;
      W[(size_t)c * R + n2 + r] = first ? T(a.C0[o]) : a.C[o];
      W[(size_t)(n + c) * R + n2 + r] = T(0);
      W[(size_t)(n2 + c) * R + n2 + r] = T(0);
    }
    for (int idx = tid; idx < (int)nrnx; idx += bs) {
      const int r = idx % nr, c = idx / nr;
      W[(size_t)(3 * n + c) * R + n2 + r] = T(0);
    }
    __syncthreads();
    // ----------------------------------------------------------- eliminate
    int info = 0;
    for (int i = 0; i < n && info == 0; ++i) {
      T* ci = W + (size_t)i * R;
      if (SEL == SEL_QRP) {
        // column with the largest remaining 2-norm over the panel rows
        T best = T(-1);
        int bc = i;
        for (int c = i + tid; c < n; c += bs) {
          const T* col = W + (size_t)c * R;
          T s2 = T(0);
          for (int r = i; r < n2; ++r) s2 += col[r] * col[r];
          if (s2 > best) { best = s2; bc = c; }
        }
        block_argmax(best, bc, sv, si);
        if (tid == 0) s_piv[i] = bc;
        if (bc != i)
          for (int r = tid; r < R; r += bs) {
            T t = ci[r]; ci[r] = W[(size_t)bc * R + r]; W[(size_t)bc * R + r] = t;
          }
        __syncthreads();
      }
      if (SEL == SEL_LU) {
        T best = T(-1);
        int bi = i;
        for (int r = i + tid; r < n2; r += bs) {
          T v = dev_abs(ci[r]);
          if (v > best) { best = v; bi = r; }
        }
        block_argmax(best, bi, sv, si);
        if (tid == 0) s_piv[i] = bi;
        const T pv = ci[bi];
        __syncthreads();  // every thread holds the pivot before column i is swapped
        if (pv == T(0)) { info = i + 1; break; }
        if (bi != i)
          for (int c = tid; c < NC; c += bs) {
            T* col = W + (size_t)c * R;
            T t = col[i]; col[i] = col[bi]; col[bi] = t;
          }
        __syncthreads();
        const T rinv = T(1) / pv;
        for (int r = i + 1 + tid; r < R; r += bs) ci[r] *= rinv;
        __syncthreads();
      } else {
        const T alpha = ci[i];
        T s2 = T(0);
        for (int r = i + 1 + tid; r < n2; r += bs) s2 += ci[r] * ci[r];
        s2 = block_sum(s2, sv);
        T tt = T(0), beta = alpha;
        if (s2 != T(0)) {
          const T nrm = sqrt(alpha * alpha + s2);
          beta = alpha >= T(0) ? -nrm : nrm;
          tt = (beta - alpha) / beta;
          const T sc = T(1) / (alpha - beta);
          for (int r = i + 1 + tid; r < n2; r += bs) ci[r] *= sc;
        }
        __syncthreads();
        if (tid == 0) { ci[i] = beta; s_tau[i] = tt; if (SEL == SEL_QR) s_piv[i] = i; }
        __syncthreads();
        if (beta == T(0)) { info = i + 1; break; }
        if (tt != T(0))
          for (int c = i + 1 + tid; c < NC; c += bs) {
            T* col = W + (size_t)c * R;
            T w = col[i];
            for (int r = i + 1; r < n2; ++r) w += ci[r] * col[r];
            w *= tt;
            col[i] -= w;
            for (int r = i + 1; r < n2; ++r) col[r] -= w * ci[r];
          }
        __syncthreads();
        if (R > n2) {
          const T rb = T(1) / beta;
          for (int r = n2 + tid; r < R; r += bs) ci[r] *= rb;
          __syncthreads();
        }
      }
      // rank-1 update of the rows below i (LU) or of the border rows (QR/QRP)
      const int r0 = SEL == SEL_LU ? i + 1 : n2;
      const int rows = R - r0, cols = NC - i - 1;
      if (rows > 0 && cols > 0) {
        const long tot = (long)rows * cols;
        for (long e = tid; e < tot; e += bs) {
          const int r = r0 + (int)(e % rows), c = i + 1 + (int)(e / rows);
          T* col = W + (size_t)c * R;
          col[r] -= ci[r] * col[i];
        }
      }
      __syncthreads();
    }
    if (info != 0) {
      if (tid == 0) report(a.st, DEV_ZERO_PIVOT, j, info, k);
      __syncthreads();
      continue;
    }
    // ---------------------------------------------------------------- store
    T* Tj = a.Tm + (size_t)j * szT(d);
    for (int idx = tid; idx < (int)(2 * nn); idx += bs) {
      const int r = idx % n2, c = idx / n2;
      Tj[idx] = W[(size_t)c * R + r];
    }
    if (SEL != SEL_LU)
      for (int i = tid; i < n; i += bs) Tj[2 * nn + i] = s_tau[i];
    unsigned char* Pj = a.P + (size_t)j * szP(d);
    if (tid == 0) {
      // row map (getrf order) or QRP column map from the swap sequence
      unsigned char mp[768];
      for (int r = 0; r < n2; ++r) mp[r] = (unsigned char)r;
      for (int i = 0; i < n; ++i) mp[n2 + i] = (unsigned char)i;
      if (SEL == SEL_LU)
        for (int i = 0; i < n; ++i) { unsigned char t = mp[i]; mp[i] = mp[s_piv[i]]; mp[s_piv[i]] = t; }
      if (SEL == SEL_QRP)
        for (int i = 0; i < n; ++i) { unsigned char t = mp[n2 + i]; mp[n2 + i] = mp[n2 + s_piv[i]]; mp[n2 + s_piv[i]] = t; }
      for (int r = 0; r < 3 * n; ++r) Pj[r] = mp[r];
    }
    for (int idx = tid; idx < (int)nn; idx += bs) {
      const int i = idx % n, c = idx / n;
      a.D[oj + idx] = W[(size_t)(n + c) * R + i];
      a.E[oj + idx] = W[(size_t)(n2 + c) * R + i];
      a.D[ojp + idx] = W[(size_t)(n + c) * R + n + i];
      a.E[ojp + idx] = W[(size_t)(n2 + c) * R + n + i];
    }
    for (int idx = tid; idx < (int)nnx; idx += bs) {
      const int i = idx % n, c = idx / n;
      a.B[(size_t)j * nnx + idx] = W[(size_t)(3 * n + c) * R + i];
      a.B[(size_t)jp * nnx + idx] = W[(size_t)(3 * n + c) * R + n + i];
    }
    for (int idx = tid; idx < (int)nrn; idx += bs) {
      const int r = idx % nr, c = idx / nr;
      const size_t oc = (size_t)jp * nrn + idx;
      a.C[(size_t)j * nrn + idx] = W[(size_t)c * R + n2 + r];
      const T cjp = first ? T(a.C0[oc]) : a.C[oc];
      a.C[oc] = cjp + W[(size_t)(n + c) * R + n2 + r];
      a.Rbuf[(size_t)j * nrn + idx] = W[(size_t)(n2 + c) * R + n2 + r];
    }
    for (int idx = tid; idx < (int)nrnx; idx += bs) {
      const int r = idx % nr, c = idx / nr;
      a.Fbuf[(size_t)j * nrnx + idx] = W[(size_t)(3 * n + c) * R + n2 + r];
    }
    __syncthreads();
  }
}

// copy of loaded FP64 blocks into the working precision
template <typename T>
__global__ void k_convert_blocks(const double* src, T* dst, size_t count) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < count; e += (size_t)gridDim.x * blockDim.x)
    dst[e] = T(src[e]);
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
// deterministic sums of per-block m-vectors (m <= 256) over blocks
// [first, first+count): CTA g reduces a fixed chunk of blocks with a fixed
// thread-to-block map and a fixed shared-memory tree, so the result does not
// depend on timing.  With out == nullptr the CTA writes its partial to
// part[g]; otherwise (one CTA) it writes out = base + sum (column height h).
// ---------------------------------------------------------------------------
template <typename T>
__device__ void reduce_tree_body(const T* buf, int stride, long first, long count, int m, long chunk,
                                 T* part, const T* base, int h, int ldb, T* out, int ldo, int blk) {
  __shared__ T red[256];
  const int tid = threadIdx.x;
  const int S = 256 / m;  // items reduced in parallel per element
  const int e = tid % m, g = tid / m;
  const long b0 = first + (long)blk * chunk;
  const long b1 = min(first + count, b0 + chunk);
  T a0 = T(0), a1 = T(0);
  if (g < S) {
    long b = b0 + g;
    for (; b + S < b1; b += 2 * S) {
      a0 += buf[(size_t)b * stride + e];
      a1 += buf[(size_t)(b + S) * stride + e];
    }
    if (b < b1) a0 += buf[(size_t)b * stride + e];
  }
  red[tid] = a0 + a1;
  __syncthreads();
  for (int w = 1; w < S; w *= 2) {
    if (g < S && g % (2 * w) == 0 && g + w < S) red[tid] += red[tid + w * m];
    __syncthreads();
  }
  if (g == 0) {
    const T s = red[e];
    if (out) {
      const int r = e % h, c = e / h;
      out[(size_t)c * ldo + r] = (base ? base[(size_t)c * ldb + r] : T(0)) + s;
    } else {
      part[(size_t)blk * m + e] = s;
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_reduce_tree(const T* buf, int stride, long first, long count,
                                                     int m, long chunk, T* part, const T* base, int h,
                                                     int ldb, T* out, int ldo) {
  reduce_tree_body(buf, stride, first, count, m, chunk, part, base, h, ldb, out, ldo, (int)blockIdx.x);
}

// ---------------------------------------------------------------------------
// solve sweeps (forward, cc:1615-1795; backward, cc:1805-2075)
// ---------------------------------------------------------------------------
// factors of type T (FP64, or FP32 for the mixed path); vectors always FP64
template <typename T>
struct SweepArgs {
  Dims d;
  const T *D, *E, *B, *C, *Tm;
  const unsigned char* P;
  double* x;
  int ldx, nrhs;
  double* XB;
  int k, ldw, sel;
  const int* done;  // batch, mixed path: nonzero once this system's refinement converged
};

template <typename T>
__device__ __forceinline__ bool system_active(const SweepArgs<T>& a) { return !(a.done && *a.done); }

__device__ __forceinline__ void take_level(SweepArgs<float>& a, const SweepArgs<float>& a0) { a.k = a0.k; }
__device__ __forceinline__ void take_level(SweepArgs<double>& a, const SweepArgs<double>& a0) { a.k = a0.k; }

template <typename T, bool BATCH = false>
__global__ void __launch_bounds__(WARPS_PANEL * 32) k_forward_level(SweepArgs<T> a0, const SweepArgs<T>* tab,
                                                                const BatchCta* cmap, const long* ecnt) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  for_entries<BATCH>(ecnt, [&](long entry) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    SweepArgs<T> ab;  // this CTA's system (batch only)
    long q0, q1, qs;
    pair_range<BATCH>(a0, tab, cmap, wpb, warp, ab, q0, q1, qs, entry);
    const SweepArgs<T>& a = BATCH ? ab : a0;
    const Dims d = a.d;
    const int n = d.n, nr = d.nr, n2 = 2 * n, nrhs = a.nrhs, ldw = a.ldw, k = a.k;
    double* W = reinterpret_cast<double*>(smem_raw) + (size_t)warp * ldw * nrhs;
    for (long q = q0; q < q1; q += qs) {
      const int j = k + (int)(2L * k * q), jp = j - k;
      const T* Tj = a.Tm + (size_t)j * szT(d);
      const unsigned char* Pj = a.P + (size_t)j * szP(d);
      for (int idx = lane; idx < n2 * nrhs; idx += 32) {
        const int pos = idx % n2, c = idx / n2;
        const int r = a.sel == SEL_LU ? Pj[pos] : pos;  // original row at this position
        const size_t o = (size_t)c * a.ldx + (r < n ? (size_t)jp * n + r : (size_t)j * n + (r - n));
        W[(size_t)c * ldw + pos] = a.x[o];
      }
      __syncwarp();
      if (a.sel == SEL_LU) {
        for (int i = 0; i < n; ++i) {
          for (int r = i + 1 + lane; r < n2; r += 32) {
            const double l = Tj[(size_t)i * n2 + r];
            for (int c = 0; c < nrhs; ++c) W[(size_t)c * ldw + r] -= l * W[(size_t)c * ldw + i];
          }
          __syncwarp();
        }
      } else {
        for (int i = 0; i < n; ++i) {
          const double t = Tj[2 * (size_t)n * n + i];
          const T* v = Tj + (size_t)i * n2;
          for (int c = 0; c < nrhs; ++c) {
            double* w = W + (size_t)c * ldw;
            double s = 0.0;
            for (int r = i + 1 + lane; r < n2; r += 32) s += double(v[r]) * w[r];
            s = warp_sum(s);
            s = (s + w[i]) * t;
            __syncwarp();
            if (lane == 0) w[i] -= s;
            for (int r = i + 1 + lane; r < n2; r += 32) w[r] -= s * double(v[r]);
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
          double s = 0.0;
          for (int i = 0; i < n; ++i) s += double(Cj[(size_t)i * nr + r]) * W[(size_t)c * ldw + i];
          a.XB[(size_t)j * nr * nrhs + idx] = -s;
        }
      }
      __syncwarp();
    }
  });
}

template <typename T, bool BATCH = false>
__global__ void __launch_bounds__(WARPS_PANEL * 32) k_backward_level(SweepArgs<T> a0, const SweepArgs<T>* tab,
                                                                 const BatchCta* cmap, const long* ecnt) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  for_entries<BATCH>(ecnt, [&](long entry) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    SweepArgs<T> ab;  // this CTA's system (batch only)
    long q0, q1, qs;
    pair_range<BATCH>(a0, tab, cmap, wpb, warp, ab, q0, q1, qs, entry);
    const SweepArgs<T>& a = BATCH ? ab : a0;
    const Dims d = a.d;
    const int n = d.n, nx = d.nx, n2 = 2 * n, nrhs = a.nrhs, k = a.k, nb = d.nblock;
    double* Y = reinterpret_cast<double*>(smem_raw) + (size_t)warp * a.ldw;
    const size_t xb_off = (size_t)(nb + 1) * n + d.qx;
    for (long q = q0; q < q1; q += qs) {
      const int j = k + (int)(2L * k * q), jp = j - k, jpp = min(j + k, nb);
      const T* Dj = a.D + (size_t)j * n * n;
      const T* Ej = a.E + (size_t)j * n * n;
      const T* Bj = a.B + (size_t)j * n * nx;
      const T* Tj = a.Tm + (size_t)j * szT(d);
      for (int c = 0; c < nrhs; ++c) {
        double* xc = a.x + (size_t)c * a.ldx;
        for (int i = lane; i < n; i += 32) {
          double s = xc[(size_t)j * n + i];
          for (int m = 0; m < n; ++m) s -= Dj[(size_t)m * n + i] * xc[(size_t)jp * n + m];
          for (int m = 0; m < n; ++m) s -= Ej[(size_t)m * n + i] * xc[(size_t)jpp * n + m];
          for (int m = 0; m < nx; ++m) s -= Bj[(size_t)m * n + i] * xc[xb_off + m];
          Y[i] = s;
        }
        __syncwarp();
        for (int i = n - 1; i >= 0; --i) {
          const double xi = Y[i] / double(Tj[(size_t)i * n2 + i]);
          __syncwarp();
          if (lane == 0) Y[i] = xi;
          for (int r = lane; r < i; r += 32) Y[r] -= Tj[(size_t)i * n2 + r] * xi;
          __syncwarp();
        }
        const unsigned char* cmap = a.P + (size_t)j * szP(d) + 2 * n;
        for (int i = lane; i < n; i += 32) xc[(size_t)j * n + (a.sel == SEL_QRP ? cmap[i] : i)] = Y[i];
        __syncwarp();
      }
    }
  });
}

// ---------------------------------------------------------------------------
// register-resident sweeps for n <= N <= 16: one warp per pair.
//
// forward (forward, cc:1615-1719): lane = position r < 2n of the stacked
//   [x_jp; x_j]; the row map gathers the original row with one shuffle, the
//   unit-lower L and M are applied by n broadcast steps (LU) or the n
//   Householder reflectors by warp reductions (QR/QRP); xb partial -C'_j x_j.
// backward (backward, cc:1805-2075): lanes 0..15 form D'_j x_jp, lanes
//   16..31 E'_j x_jpp for row i = lane & 15; the halves are combined, the B'_j
//   xb term added and U solved by n broadcast steps (QRP: column-map scatter).
// All loads of a pair are issued before the first use.
// ---------------------------------------------------------------------------
template <typename TF, int N, int NRM, bool LU, bool BATCH = false>
__global__ void __launch_bounds__(256, 2) k_forward_rows(SweepArgs<TF> a0, const SweepArgs<TF>* tab,
                                                         const BatchCta* cmap, const long* ecnt) {
  for_entries<BATCH>(ecnt, [&](long entry) {
    constexpr unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    SweepArgs<TF> ab;  // this CTA's system (batch only)
    long q0, q1, qs;
    pair_range<BATCH>(a0, tab, cmap, wpb, warp, ab, q0, q1, qs, entry);
    const SweepArgs<TF>& a = BATCH ? ab : a0;
    const Dims d = a.d;
    const int n = d.n, nr = d.nr, n2 = 2 * n, nrhs = a.nrhs, k = a.k;
    const bool act = lane < n2;
    constexpr bool lu = LU;
    for (long q = q0; q < q1; q += qs) {
      const int j = k + (int)(2L * k * q), jp = j - k;
      const TF* Tj = a.Tm + (size_t)j * szT(d);
      double t[N];
  #pragma unroll
      for (int c = 0; c < N; ++c) t[c] = (act && c < n) ? double(Tj[(size_t)c * n2 + lane]) : 0.0;
      double tau[LU ? 1 : N];
  #pragma unroll
      for (int c = 0; c < (LU ? 1 : N); ++c) tau[c] = (!lu && c < n) ? Tj[2 * (size_t)n * n + c] : 0.0;
      const int src = (act && lu) ? (int)a.P[(size_t)j * szP(d) + lane] : lane;
      double cp[NRM];
      const TF* Cj = a.C + (size_t)j * nr * n;
  #pragma unroll
      for (int r = 0; r < NRM; ++r) cp[r] = (lane < n && r < nr) ? Cj[(size_t)lane * nr + r] : 0.0;
      for (int col = 0; col < nrhs; ++col) {
        double* xc = a.x + (size_t)col * a.ldx;
        const double orig = act ? (lane < n ? xc[(size_t)jp * n + lane] : xc[(size_t)j * n + lane - n]) : 0.0;
        double w = __shfl_sync(FULL, orig, src);
        if (lu) {
  #pragma unroll
          for (int i = 0; i < N; ++i) {
            if (i < n) {
              const double wi = __shfl_sync(FULL, w, i);
              if (lane > i && act) w = fma(-t[i], wi, w);
            }
          }
        } else {
  #pragma unroll
          for (int i = 0; i < N; ++i) {
            if (i < n) {
              const double v = (lane > i && act) ? t[i] : (lane == i ? 1.0 : 0.0);
              double sdot = warp_sum(v * w);
              w = fma(-tau[LU ? 0 : i] * sdot, v, w);
            }
          }
        }
        if (act) {
          if (lane < n) xc[(size_t)j * n + lane] = w;
          else xc[(size_t)jp * n + lane - n] = w;
        }
        const double wt = lane < n ? w : 0.0;
  #pragma unroll
        for (int r = 0; r < NRM; ++r) {
          if (r < nr) {
            const double sr = warp_sum(cp[r] * wt);
            if (lane == 0) a.XB[(size_t)j * nr * nrhs + (size_t)col * nr + r] = -sr;
          }
        }
      }
    }
  });
}

template <typename TF, int N, int NXM, bool BATCH = false>
__global__ void __launch_bounds__(256, 2) k_backward_rows(SweepArgs<TF> a0, const SweepArgs<TF>* tab,
                                                          const BatchCta* cmap, const long* ecnt) {
  for_entries<BATCH>(ecnt, [&](long entry) {
    constexpr unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    SweepArgs<TF> ab;  // this CTA's system (batch only)
    long q0, q1, qs;
    pair_range<BATCH>(a0, tab, cmap, wpb, warp, ab, q0, q1, qs, entry);
    const SweepArgs<TF>& a = BATCH ? ab : a0;
    const Dims d = a.d;
    const int n = d.n, nx = d.nx, nb = d.nblock, n2 = 2 * n, nrhs = a.nrhs, k = a.k;
    const int i = lane & 15;
    const bool hi = lane >= 16, rowok = i < n;
    const bool qrp = a.sel == SEL_QRP;
    const size_t xb_off = (size_t)(nb + 1) * n + d.qx;
    for (long q = q0; q < q1; q += qs) {
      const int j = k + (int)(2L * k * q), jp = j - k, jpp = min(j + k, nb);
      const TF* Mt = (hi ? a.E : a.D) + (size_t)j * n * n;
      const TF* Tj = a.Tm + (size_t)j * szT(d);
      const TF* Bj = a.B + (size_t)j * n * nx;
      double m[N], u[N], bb[NXM];
  #pragma unroll
      for (int c = 0; c < N; ++c) m[c] = (rowok && c < n) ? Mt[(size_t)c * n + i] : 0.0;
  #pragma unroll
      for (int c = 0; c < N; ++c) u[c] = (!hi && rowok && c < n) ? Tj[(size_t)c * n2 + i] : 0.0;
  #pragma unroll
      for (int c = 0; c < NXM; ++c) bb[c] = (!hi && rowok && c < nx) ? Bj[(size_t)c * n + i] : 0.0;
      // 1 / U(i,i): pick the diagonal element first, then one division per lane
      double ud = 1.0;
  #pragma unroll
      for (int c = 0; c < N; ++c)
        if (c == i) ud = u[c];
      const double rdi = (!hi && rowok) ? 1.0 / ud : 0.0;
      const int dst = (qrp && !hi && rowok) ? (int)a.P[(size_t)j * szP(d) + n2 + i] : i;
      for (int col = 0; col < nrhs; ++col) {
        double* xc = a.x + (size_t)col * a.ldx;
        const double xv = rowok ? (hi ? xc[(size_t)jpp * n + i] : xc[(size_t)jp * n + i]) : 0.0;
        const double xj = (!hi && rowok) ? xc[(size_t)j * n + i] : 0.0;
        double xbv[NXM];
  #pragma unroll
        for (int c = 0; c < NXM; ++c) xbv[c] = c < nx ? xc[xb_off + c] : 0.0;
        double s = 0.0;
  #pragma unroll
        for (int c = 0; c < N; ++c) {
          if (c < n) {
            const double xcv = __shfl_sync(FULL, xv, (lane & 16) | c);
            s = fma(m[c], xcv, s);
          }
        }
        s += __shfl_xor_sync(FULL, s, 16);
  #pragma unroll
        for (int c = 0; c < NXM; ++c) s = fma(bb[c], xbv[c], s);
        double y = xj - s;
  #pragma unroll
        for (int ii = N - 1; ii >= 0; --ii) {
          if (ii < n) {
            const double xi = __shfl_sync(FULL, y * rdi, ii);
            if (i == ii) y = xi;
            else if (i < ii) y = fma(-u[ii], xi, y);
          }
        }
        if (!hi && rowok) xc[(size_t)j * n + dst] = y;
      }
    }
  });
}

// ---------------------------------------------------------------------------
// Backward sweep for n = 8 or 16 (FP64 or FP32 factors; single systems and
// batch classes, see PipeItems): the same pair arithmetic as k_backward_rows (lane i < n: U-row i with D'_j, U and B'_j;
// lane 16 + i: E'_j row i), with the factors of the warp's NEXT pair copied
// into shared memory by cp.async (16-byte chunks, straight from the blocks'
// column-major layout, which is also the conflict-free layout for lane = row)
// while the current pair is computed, so every warp keeps a pair's worth of
// loads in flight.  Two buffers per warp.
// ---------------------------------------------------------------------------
template <int N, int NXM, typename T = double>
struct BwdBuf {
  static constexpr int DE = N * N, BB = N * NXM, U = N * N;
  static constexpr int WORDS = 2 * DE + BB + U;  // D', E', B', U (rows 0..N-1 of T)
  static constexpr size_t BYTES = (size_t)2 * WORDS * sizeof(T);  // two buffers
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int K>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(K) : "memory"); }

// the factors of pair q (level stride k) into one buffer (every lane issues
// its share), in 16-byte chunks of V elements; for n = 8, 16 every block (D',
// E', B', the U columns of T) starts and ends on a 16-byte boundary in FP64
// and FP32
template <int N, int NXM, typename T>
__device__ __forceinline__ void bwd_stage(const SweepArgs<T>& a, int k, long q, T* buf, int lane) {
  using Bf = BwdBuf<N, NXM, T>;
  constexpr int V = 16 / (int)sizeof(T);
  const Dims d = a.d;
  const int n = d.n, nx = d.nx;
  const int j = k + (int)(2L * k * q);
  const T* Dj = a.D + (size_t)j * n * n;
  const T* Ej = a.E + (size_t)j * n * n;
  const T* Bj = a.B + (size_t)j * n * nx;
  const T* Tj = a.Tm + (size_t)j * szT(d);
  // D', E': n*n elements each
  for (int c = lane; c < n * n / V; c += 32) {
    cp_async16(buf + V * c, Dj + V * c);
    cp_async16(buf + Bf::DE + V * c, Ej + V * c);
  }
  for (int c = lane; c < n * nx / V; c += 32) cp_async16(buf + 2 * Bf::DE + V * c, Bj + V * c);
  // U: column col of T holds rows 0..n-1 of U at Tj + col * 2n
  for (int c = lane; c < n * n / V; c += 32) {
    const int col = (V * c) / n, r = (V * c) % n;
    cp_async16(buf + 2 * Bf::DE + Bf::BB + col * n + r, Tj + (size_t)col * 2 * n + r);
  }
}

// Work items of a warp in the pipelined sweeps.  Single system: pair q =
// item, items first, first + step, ... below the level's pair count.  Batch:
// item = entry of the level's sweep map (the full map: nent entries; or the
// compacted map of the systems still refining: *ecnt entries), the warp's
// pair is entry.q0 + warp, and the system's arguments come from the table.
template <bool BATCH, typename T>
struct PipeItems {
  SweepArgs<T> a0;
  const SweepArgs<T>* tab;
  const BatchCta* map;
  long cnt, first, step;
  int warp;
  __device__ PipeItems(const SweepArgs<T>& a, const SweepArgs<T>* t, const BatchCta* m, const long* ecnt,
                       long nent, int wpb, int w)
      : a0(a), tab(t), map(m), warp(w) {
    if constexpr (BATCH) {
      cnt = ecnt ? *ecnt : nent;
      first = blockIdx.x;
      step = gridDim.x;
    } else {
      cnt = pairs_at_level(a.d.nblock, a.k);
      first = (long)blockIdx.x * wpb + w;
      step = (long)gridDim.x * wpb;
    }
  }
  // the warp's pair of item it (false: none for this warp)
  __device__ bool pair(long it, int& sys, long& q) const {
    if constexpr (BATCH) {
      const BatchCta c = map[it];
      sys = c.sys;
      q = c.q0 + warp;
      if (q >= c.q1) return false;
      const int* dn = tab[sys].done;
      return !(dn && *dn);
    } else {
      sys = 0;
      q = it;
      return true;
    }
  }
  __device__ const SweepArgs<T>& args(int sys) const {
    if constexpr (BATCH) return tab[sys];
    else return a0;
  }
};

template <int N, int NXM, typename T = double, bool BATCH = false>
__global__ void __launch_bounds__(256, 2) k_backward_pipe(SweepArgs<T> a0, const SweepArgs<T>* tab,
                                                          const BatchCta* map, const long* ecnt, long nent) {
  using Bf = BwdBuf<N, NXM, T>;
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  T* bufs = reinterpret_cast<T*>(smem_raw) + (size_t)warp * 2 * Bf::WORDS;
  const PipeItems<BATCH, T> items(a0, tab, map, ecnt, nent, wpb, warp);
  const int k = a0.k;
  const int i = lane & 15;
  long it = items.first;
  int sys = 0;
  long q = 0;
  bool have = it < items.cnt && items.pair(it, sys, q);
  if (have) bwd_stage<N, NXM, T>(items.args(sys), k, q, bufs, lane);
  cp_async_commit();
  int cur = 0;
  for (; it < items.cnt; it += items.step) {
    int sysn = 0;
    long qn = 0;
    const bool haven = it + items.step < items.cnt && items.pair(it + items.step, sysn, qn);
    if (haven) bwd_stage<N, NXM, T>(items.args(sysn), k, qn, bufs + (cur ^ 1) * Bf::WORDS, lane);
    cp_async_commit();
    if (have) {
      const SweepArgs<T>& a = items.args(sys);
      const Dims d = a.d;
      const int n = d.n, nx = d.nx, nb = d.nblock, nrhs = a.nrhs;
      const bool hi = lane >= 16, rowok = i < n;
      const bool qrp = a.sel == SEL_QRP;
      const size_t xb_off = (size_t)(nb + 1) * n + d.qx;
      const int j = k + (int)(2L * k * q), jp = j - k, jpp = min(j + k, nb);
      // the right-hand side values, loaded while the factors arrive
      double xv0 = 0.0, xj0 = 0.0;
      if (nrhs >= 1) {
        xv0 = rowok ? (hi ? a.x[(size_t)jpp * n + i] : a.x[(size_t)jp * n + i]) : 0.0;
        xj0 = (!hi && rowok) ? a.x[(size_t)j * n + i] : 0.0;
      }
      const int dst = (qrp && !hi && rowok) ? (int)a.P[(size_t)j * szP(d) + 2 * n + i] : i;
      cp_async_wait<1>();  // this pair's factors (the next pair's may still be in flight)
      __syncwarp();
      const T* buf = bufs + cur * Bf::WORDS;
      double m[N], u[N], bb[NXM];
#pragma unroll
      for (int c = 0; c < N; ++c) m[c] = (rowok && c < n) ? buf[(hi ? Bf::DE : 0) + c * n + i] : 0.0;
#pragma unroll
      for (int c = 0; c < N; ++c) u[c] = (!hi && rowok && c < n) ? buf[2 * Bf::DE + Bf::BB + c * n + i] : 0.0;
#pragma unroll
      for (int c = 0; c < NXM; ++c) bb[c] = (!hi && rowok && c < nx) ? buf[2 * Bf::DE + c * n + i] : 0.0;
      double ud = 1.0;
#pragma unroll
      for (int c = 0; c < N; ++c)
        if (c == i) ud = u[c];
      const double rdi = (!hi && rowok) ? 1.0 / ud : 0.0;
      for (int col = 0; col < nrhs; ++col) {
        double* xc = a.x + (size_t)col * a.ldx;
        const double xv = col == 0 ? xv0 : (rowok ? (hi ? xc[(size_t)jpp * n + i] : xc[(size_t)jp * n + i]) : 0.0);
        const double xj = col == 0 ? xj0 : ((!hi && rowok) ? xc[(size_t)j * n + i] : 0.0);
        double xbv[NXM];
#pragma unroll
        for (int c = 0; c < NXM; ++c) xbv[c] = c < nx ? xc[xb_off + c] : 0.0;
        double sacc = 0.0;
#pragma unroll
        for (int c = 0; c < N; ++c) {
          if (c < n) {
            const double xcv = __shfl_sync(FULL, xv, (lane & 16) | c);
            sacc = fma(m[c], xcv, sacc);
          }
        }
        sacc += __shfl_xor_sync(FULL, sacc, 16);
#pragma unroll
        for (int c = 0; c < NXM; ++c) sacc = fma(bb[c], xbv[c], sacc);
        double y = xj - sacc;
#pragma unroll
        for (int ii = N - 1; ii >= 0; --ii) {
          if (ii < n) {
            const double xi = __shfl_sync(FULL, y * rdi, ii);
            if (i == ii) y = xi;
            else if (i < ii) y = fma(-u[ii], xi, y);
          }
        }
        if (!hi && rowok) xc[(size_t)j * n + dst] = y;
      }
    }
    __syncwarp();  // every lane is done with this buffer before it is refilled
    cur ^= 1;
    have = haven;
    sys = sysn;
    q = qn;
  }
  cp_async_wait<0>();
}

// The top levels of the backward sweep (at most 16 pairs each) in one launch
// of one CTA of 16 warps, levels in order with a barrier between them; the
// pair arithmetic is k_backward_rows'.
template <int N, int NXM, typename T = double>
__global__ void __launch_bounds__(512, 1) k_backward_top(SweepArgs<T> a, int k_top, int k_min) {
  constexpr unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const Dims d = a.d;
  const int n = d.n, nx = d.nx, nb = d.nblock, nrhs = a.nrhs;
  const int i = lane & 15;
  const bool hi = lane >= 16, rowok = i < n;
  const bool qrp = a.sel == SEL_QRP;
  const size_t xb_off = (size_t)(nb + 1) * n + d.qx;
  for (int k = k_top; k >= k_min && k > 0; k /= 2) {
    const long np = pairs_at_level(nb, k);
    for (long q = warp; q < np; q += 16) {
      const int j = k + (int)(2L * k * q), jp = j - k, jpp = min(j + k, nb);
      const T* Mt = (hi ? a.E : a.D) + (size_t)j * n * n;
      const T* Tj = a.Tm + (size_t)j * szT(d);
      const T* Bj = a.B + (size_t)j * n * nx;
      double m[N], u[N], bb[NXM];
#pragma unroll
      for (int c = 0; c < N; ++c) m[c] = (rowok && c < n) ? Mt[(size_t)c * n + i] : 0.0;
#pragma unroll
      for (int c = 0; c < N; ++c) u[c] = (!hi && rowok && c < n) ? Tj[(size_t)c * 2 * n + i] : 0.0;
#pragma unroll
      for (int c = 0; c < NXM; ++c) bb[c] = (!hi && rowok && c < nx) ? Bj[(size_t)c * n + i] : 0.0;
      double ud = 1.0;
#pragma unroll
      for (int c = 0; c < N; ++c)
        if (c == i) ud = u[c];
      const double rdi = (!hi && rowok) ? 1.0 / ud : 0.0;
      const int dst = (qrp && !hi && rowok) ? (int)a.P[(size_t)j * szP(d) + 2 * n + i] : i;
      for (int col = 0; col < nrhs; ++col) {
        double* xc = a.x + (size_t)col * a.ldx;
        const double xv = rowok ? (hi ? __ldcg(xc + (size_t)jpp * n + i) : __ldcg(xc + (size_t)jp * n + i)) : 0.0;
        const double xj = (!hi && rowok) ? xc[(size_t)j * n + i] : 0.0;
        double xbv[NXM];
#pragma unroll
        for (int c = 0; c < NXM; ++c) xbv[c] = c < nx ? __ldcg(xc + xb_off + c) : 0.0;
        double sacc = 0.0;
#pragma unroll
        for (int c = 0; c < N; ++c) {
          if (c < n) {
            const double xcv = __shfl_sync(FULL, xv, (lane & 16) | c);
            sacc = fma(m[c], xcv, sacc);
          }
        }
        sacc += __shfl_xor_sync(FULL, sacc, 16);
#pragma unroll
        for (int c = 0; c < NXM; ++c) sacc = fma(bb[c], xbv[c], sacc);
        double y = xj - sacc;
#pragma unroll
        for (int ii = N - 1; ii >= 0; --ii) {
          if (ii < n) {
            const double xi = __shfl_sync(FULL, y * rdi, ii);
            if (i == ii) y = xi;
            else if (i < ii) y = fma(-u[ii], xi, y);
          }
        }
        if (!hi && rowok) xc[(size_t)j * n + dst] = y;
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Forward sweep for LU factors, n = 8 or 16 (FP64 or FP32; single systems and
// batch classes, see PipeItems): the pair arithmetic of k_forward_rows (lane = position r < 2n of the stacked
// [x_jp; x_j], row map gathered by one shuffle, n broadcast steps of L and M,
// xb partial -C'_j x_j), with the factors of the warp's NEXT pair (the 2n x n
// L\U and M block of T, and C_j) copied into shared memory by cp.async while
// the current pair is computed, and the next pair's row-map entry read into a
// register one pair ahead.  Two buffers per warp.
// ---------------------------------------------------------------------------
template <int N, int NRM, typename T = double>
struct FwdBuf {
  static constexpr int TT = 2 * N * N, CC = N * NRM;
  static constexpr int WORDS = TT + CC;                        // T_j (2n x n), C_j (n x nr)
  static constexpr size_t BYTES = (size_t)2 * WORDS * sizeof(T);  // two buffers
};

// the factors of pair q (level stride k) into one buffer, in 16-byte chunks
// of V elements (for n = 8, 16 both blocks are multiples of 16 bytes in FP64
// and FP32)
template <int N, int NRM, typename T>
__device__ __forceinline__ void fwd_stage(const SweepArgs<T>& a, int k, long q, T* buf, int lane) {
  using Bf = FwdBuf<N, NRM, T>;
  constexpr int V = 16 / (int)sizeof(T);
  const Dims d = a.d;
  const int n = d.n, nr = d.nr;
  const int j = k + (int)(2L * k * q);
  const T* Tj = a.Tm + (size_t)j * szT(d);
  const T* Cj = a.C + (size_t)j * nr * n;
  for (int c = lane; c < 2 * n * n / V; c += 32) cp_async16(buf + V * c, Tj + V * c);
  for (int c = lane; c < n * nr / V; c += 32) cp_async16(buf + Bf::TT + V * c, Cj + V * c);
}

template <int N, int NRM, typename T = double, bool BATCH = false>
__global__ void __launch_bounds__(256, 2) k_forward_pipe(SweepArgs<T> a0, const SweepArgs<T>* tab,
                                                         const BatchCta* map, const long* ecnt, long nent) {
  using Bf = FwdBuf<N, NRM, T>;
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  T* bufs = reinterpret_cast<T*>(smem_raw) + (size_t)warp * 2 * Bf::WORDS;
  const PipeItems<BATCH, T> items(a0, tab, map, ecnt, nent, wpb, warp);
  const int k = a0.k;
  // the row-map entry of a pair (read a pair ahead, into a register)
  auto row_src = [&](const SweepArgs<T>& a, long q) -> int {
    const int j = k + (int)(2L * k * q);
    return lane < 2 * a.d.n ? (int)a.P[(size_t)j * szP(a.d) + lane] : lane;
  };
  long it = items.first;
  int sys = 0, src_next = lane;
  long q = 0;
  bool have = it < items.cnt && items.pair(it, sys, q);
  if (have) {
    fwd_stage<N, NRM, T>(items.args(sys), k, q, bufs, lane);
    src_next = row_src(items.args(sys), q);
  }
  cp_async_commit();
  int cur = 0;
  for (; it < items.cnt; it += items.step) {
    const int src = src_next;
    int sysn = 0;
    long qn = 0;
    const bool haven = it + items.step < items.cnt && items.pair(it + items.step, sysn, qn);
    if (haven) {
      fwd_stage<N, NRM, T>(items.args(sysn), k, qn, bufs + (cur ^ 1) * Bf::WORDS, lane);
      src_next = row_src(items.args(sysn), qn);
    }
    cp_async_commit();
    if (have) {
      const SweepArgs<T>& a = items.args(sys);
      const Dims d = a.d;
      const int n = d.n, nr = d.nr, n2 = 2 * n, nrhs = a.nrhs;
      const bool act = lane < n2;
      const int j = k + (int)(2L * k * q), jp = j - k;
      // the first right-hand side's values, loaded while the factors arrive
      const double orig0 = act ? (lane < n ? a.x[(size_t)jp * n + lane] : a.x[(size_t)j * n + lane - n]) : 0.0;
      cp_async_wait<1>();  // this pair's factors (the next pair's may still be in flight)
      __syncwarp();
      const T* buf = bufs + cur * Bf::WORDS;
      double t[N], cp[NRM];
#pragma unroll
      for (int c = 0; c < N; ++c) t[c] = (act && c < n) ? double(buf[c * n2 + lane]) : 0.0;
#pragma unroll
      for (int r = 0; r < NRM; ++r) cp[r] = (lane < n && r < nr) ? double(buf[Bf::TT + lane * nr + r]) : 0.0;
      for (int col = 0; col < nrhs; ++col) {
        double* xc = a.x + (size_t)col * a.ldx;
        const double orig =
            col == 0 ? orig0 : (act ? (lane < n ? xc[(size_t)jp * n + lane] : xc[(size_t)j * n + lane - n]) : 0.0);
        double w = __shfl_sync(FULL, orig, src);
#pragma unroll
        for (int i = 0; i < N; ++i) {
          if (i < n) {
            const double wi = __shfl_sync(FULL, w, i);
            if (lane > i && act) w = fma(-t[i], wi, w);
          }
        }
        if (act) {
          if (lane < n) xc[(size_t)j * n + lane] = w;
          else xc[(size_t)jp * n + lane - n] = w;
        }
        const double wt = lane < n ? w : 0.0;
#pragma unroll
        for (int r = 0; r < NRM; ++r) {
          if (r < nr) {
            const double sr = warp_sum(cp[r] * wt);
            if (lane == 0) a.XB[(size_t)j * nr * nrhs + (size_t)col * nr + r] = -sr;
          }
        }
      }
    }
    __syncwarp();  // every lane is done with this buffer before it is refilled
    cur ^= 1;
    have = haven;
    sys = sysn;
    q = qn;
  }
  cp_async_wait<0>();
}

// ---------------------------------------------------------------------------
// sweeps for n = 32: one warp per pair, lane i holds panel positions i and
// 32 + i (forward) or U-row i (backward); x values are exchanged by shuffles
// and every factor element is read once, coalesced
// ---------------------------------------------------------------------------
template <typename TF, int NRM, bool BATCH = false>
__global__ void __launch_bounds__(256, 2) k_forward_rows32(SweepArgs<TF> a0, const SweepArgs<TF>* tab,
                                                           const BatchCta* cmap, const long* ecnt) {
  for_entries<BATCH>(ecnt, [&](long entry) {
    constexpr unsigned FULL = 0xffffffffu;
    constexpr int n = 32, n2 = 64;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    SweepArgs<TF> ab;  // this CTA's system (batch only)
    long q0, q1, qs;
    pair_range<BATCH>(a0, tab, cmap, wpb, warp, ab, q0, q1, qs, entry);
    const SweepArgs<TF>& a = BATCH ? ab : a0;
    const Dims d = a.d;
    const int nr = d.nr, nrhs = a.nrhs, k = a.k;
    for (long q = q0; q < q1; q += qs) {
      const int j = k + (int)(2L * k * q), jp = j - k;
      const TF* Tj = a.Tm + (size_t)j * szT(d);
      const unsigned char* Pj = a.P + (size_t)j * szP(d);
      const int s0 = Pj[lane], s1 = Pj[n + lane];  // original rows at positions lane, 32 + lane
      double cp[NRM];
      const TF* Cj = a.C + (size_t)j * nr * n;
  #pragma unroll
      for (int r = 0; r < NRM; ++r) cp[r] = r < nr ? double(Cj[(size_t)lane * nr + r]) : 0.0;
      for (int col = 0; col < nrhs; ++col) {
        double* xc = a.x + (size_t)col * a.ldx;
        const double ot = xc[(size_t)jp * n + lane], ob = xc[(size_t)j * n + lane];
        const double a0t = __shfl_sync(FULL, ot, s0 & 31), a0b = __shfl_sync(FULL, ob, s0 & 31);
        const double a1t = __shfl_sync(FULL, ot, s1 & 31), a1b = __shfl_sync(FULL, ob, s1 & 31);
        double w0 = s0 < n ? a0t : a0b, w1 = s1 < n ? a1t : a1b;
  #pragma unroll
        for (int i = 0; i < n; ++i) {
          const double wi = __shfl_sync(FULL, w0, i);
          const double t0 = double(Tj[(size_t)i * n2 + lane]), t1 = double(Tj[(size_t)i * n2 + n + lane]);
          if (lane > i) w0 = fma(-t0, wi, w0);
          w1 = fma(-t1, wi, w1);
        }
        xc[(size_t)j * n + lane] = w0;
        xc[(size_t)jp * n + lane] = w1;
  #pragma unroll
        for (int r = 0; r < NRM; ++r) {
          if (r < nr) {
            const double sr = warp_sum(cp[r] * w0);
            if (lane == 0) a.XB[(size_t)j * nr * nrhs + (size_t)col * nr + r] = -sr;
          }
        }
      }
    }
  });
}

template <typename TF, int NXM, bool BATCH = false>
__global__ void __launch_bounds__(256, 2) k_backward_rows32(SweepArgs<TF> a0, const SweepArgs<TF>* tab,
                                                            const BatchCta* cmap, const long* ecnt) {
  for_entries<BATCH>(ecnt, [&](long entry) {
    constexpr unsigned FULL = 0xffffffffu;
    constexpr int n = 32, n2 = 64;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    SweepArgs<TF> ab;  // this CTA's system (batch only)
    long q0, q1, qs;
    pair_range<BATCH>(a0, tab, cmap, wpb, warp, ab, q0, q1, qs, entry);
    const SweepArgs<TF>& a = BATCH ? ab : a0;
    const Dims d = a.d;
    const int nx = d.nx, nb = d.nblock, nrhs = a.nrhs, k = a.k;
    const bool qrp = a.sel == SEL_QRP;
    const size_t xb_off = (size_t)(nb + 1) * n + d.qx;
    constexpr size_t nn = (size_t)n * n;
    for (long q = q0; q < q1; q += qs) {
      const int j = k + (int)(2L * k * q), jp = j - k, jpp = min(j + k, nb);
      const TF* Dj = a.D + (size_t)j * nn;
      const TF* Ej = a.E + (size_t)j * nn;
      const TF* Bj = a.B + (size_t)j * n * nx;
      const TF* Tj = a.Tm + (size_t)j * szT(d);
      const double rdi = 1.0 / double(Tj[(size_t)lane * n2 + lane]);
      const int dst = qrp ? (int)a.P[(size_t)j * szP(d) + n2 + lane] : lane;
      for (int col = 0; col < nrhs; ++col) {
        double* xc = a.x + (size_t)col * a.ldx;
        const double xjp = xc[(size_t)jp * n + lane], xjpp = xc[(size_t)jpp * n + lane];
        const double xj = xc[(size_t)j * n + lane];
        double s0 = 0.0, s1 = 0.0;
  #pragma unroll
        for (int c = 0; c < n; ++c) {
          s0 = fma(double(Dj[(size_t)c * n + lane]), __shfl_sync(FULL, xjp, c), s0);
          s1 = fma(double(Ej[(size_t)c * n + lane]), __shfl_sync(FULL, xjpp, c), s1);
        }
  #pragma unroll
        for (int c = 0; c < NXM; ++c)
          if (c < nx) s0 = fma(double(Bj[(size_t)c * n + lane]), xc[xb_off + c], s0);
        double y = xj - (s0 + s1);
  #pragma unroll
        for (int ii = n - 1; ii >= 0; --ii) {
          const double xi = __shfl_sync(FULL, y * rdi, ii);
          if (lane == ii) y = xi;
          else if (lane < ii) y = fma(-double(Tj[(size_t)ii * n2 + lane]), xi, y);
        }
        xc[(size_t)j * n + dst] = y;
      }
    }
  });
}

// ---------------------------------------------------------------------------
// sweeps for large blocks (n > 32, n <= 128): one CTA per pair, the 2n
// values of the pair in shared memory, the triangular solves blocked by 32
// rows (one warp solves a diagonal block with shuffles, the CTA applies it to
// the rows that follow)
// ---------------------------------------------------------------------------
constexpr int SWP_MAXN = 128;

template <typename TF, bool BATCH = false>
__global__ void __launch_bounds__(256) k_forward_cta(SweepArgs<TF> a0, const SweepArgs<TF>* tab,
                                                     const BatchCta* cmap) {
  constexpr unsigned FULL = 0xffffffffu;
  __shared__ double w[2 * SWP_MAXN];
  __shared__ double tb[32][33];  // diagonal 32 x 32 block of the triangle
  const int tid = threadIdx.x, bs = blockDim.x, lane = tid & 31, warp = tid >> 5;
  SweepArgs<TF> ab;
  long q0, q1, qs;
  pair_range<BATCH>(a0, tab, cmap, 1, 0, ab, q0, q1, qs);
  const SweepArgs<TF>& a = BATCH ? ab : a0;
  const Dims d = a.d;
  const int n = d.n, n2 = 2 * n, nr = d.nr, nrhs = a.nrhs, k = a.k;
  for (long q = q0; q < q1; q += qs) {
    const int j = k + (int)(2L * k * q), jp = j - k;
    const TF* Tj = a.Tm + (size_t)j * szT(d);
    const unsigned char* Pj = a.P + (size_t)j * szP(d);
    const TF* Cj = a.C + (size_t)j * nr * n;
    for (int col = 0; col < nrhs; ++col) {
      double* xc = a.x + (size_t)col * a.ldx;
      __syncthreads();  // w of the previous column / pair is no longer read
      for (int pos = tid; pos < n2; pos += bs) {
        const int r = Pj[pos];  // original row at this position
        w[pos] = r < n ? xc[(size_t)jp * n + r] : xc[(size_t)j * n + (r - n)];
      }
      __syncthreads();
      // unit lower L on positions [0, n), then the rows below: w -= T(:, c) w[c]
      for (int cb = 0; cb < n; cb += 32) {
        const int cw = n - cb < 32 ? n - cb : 32;
        // the diagonal block of L through shared memory (one coalesced load)
        for (int e = tid; e < cw * 32; e += bs) {
          const int c = e >> 5, r = e & 31;
          tb[c][r] = r < cw ? double(Tj[(size_t)(cb + c) * n2 + cb + r]) : 0.0;
        }
        __syncthreads();
        if (warp == 0) {
          double v = lane < cw ? w[cb + lane] : 0.0;
          for (int c = 0; c < cw; ++c) {
            const double vc = __shfl_sync(FULL, v, c);
            if (lane > c && lane < cw) v = fma(-tb[c][lane], vc, v);
          }
          if (lane < cw) w[cb + lane] = v;
        }
        __syncthreads();
        for (int r = cb + cw + tid; r < n2; r += bs) {
          double s = w[r];
          for (int c0 = 0; c0 < cw; c0 += 8) {  // 8 loads in flight
            double tv[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) tv[u] = c0 + u < cw ? double(Tj[(size_t)(cb + c0 + u) * n2 + r]) : 0.0;
#pragma unroll
            for (int u = 0; u < 8; ++u)
              if (c0 + u < cw) s = fma(-tv[u], w[cb + c0 + u], s);
          }
          w[r] = s;
        }
        __syncthreads();
      }
      for (int pos = tid; pos < n2; pos += bs) {
        if (pos < n) xc[(size_t)j * n + pos] = w[pos];
        else xc[(size_t)jp * n + pos - n] = w[pos];
      }
      // xb contribution of this pair: -C'_j w[0, n)
      for (int r = warp; r < nr; r += bs >> 5) {
        double sr = 0.0;
        for (int c = lane; c < n; c += 32) sr = fma(double(Cj[(size_t)c * nr + r]), w[c], sr);
        sr = warp_sum(sr);
        if (lane == 0) a.XB[(size_t)j * nr * nrhs + (size_t)col * nr + r] = -sr;
      }
    }
  }
}

template <typename TF, bool BATCH = false>
__global__ void __launch_bounds__(256) k_backward_cta(SweepArgs<TF> a0, const SweepArgs<TF>* tab,
                                                      const BatchCta* cmap) {
  constexpr unsigned FULL = 0xffffffffu;
  __shared__ double xa[SWP_MAXN], xz[SWP_MAXN], y[SWP_MAXN];
  __shared__ double part[256];
  __shared__ double tb[32][33];  // diagonal 32 x 32 block of the triangle
  const int tid = threadIdx.x, bs = blockDim.x, lane = tid & 31, warp = tid >> 5;
  SweepArgs<TF> ab;
  long q0, q1, qs;
  pair_range<BATCH>(a0, tab, cmap, 1, 0, ab, q0, q1, qs);
  const SweepArgs<TF>& a = BATCH ? ab : a0;
  const Dims d = a.d;
  const int n = d.n, n2 = 2 * n, nx = d.nx, nb = d.nblock, nrhs = a.nrhs, k = a.k;
  const bool qrp = a.sel == SEL_QRP;
  const size_t xb_off = (size_t)(nb + 1) * n + d.qx;
  const size_t nn = (size_t)n * n;
  const int G = bs / n;  // threads per row in the product (n <= 128: G >= 2)
  for (long q = q0; q < q1; q += qs) {
    const int j = k + (int)(2L * k * q), jp = j - k, jpp = min(j + k, nb);
    const TF* Dj = a.D + (size_t)j * nn;
    const TF* Ej = a.E + (size_t)j * nn;
    const TF* Bj = a.B + (size_t)j * n * nx;
    const TF* Tj = a.Tm + (size_t)j * szT(d);
    for (int col = 0; col < nrhs; ++col) {
      double* xc = a.x + (size_t)col * a.ldx;
      __syncthreads();
      for (int i = tid; i < n; i += bs) {
        xa[i] = xc[(size_t)jp * n + i];
        xz[i] = xc[(size_t)jpp * n + i];
      }
      __syncthreads();
      // y = x_j - D'_j x_jp - E'_j x_jpp - B'_j xb, G threads per row, fixed order
      {
        const int i = tid % n, g = tid / n;
        double s = 0.0;
        if (g < G) {
          for (int c0 = g; c0 < n; c0 += 4 * G) {  // 8 loads in flight
            double dv[4], ev[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
              const int c = c0 + u * G;
              dv[u] = c < n ? double(Dj[(size_t)c * n + i]) : 0.0;
              ev[u] = c < n ? double(Ej[(size_t)c * n + i]) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
              const int c = c0 + u * G;
              if (c < n) {
                s = fma(dv[u], xa[c], s);
                s = fma(ev[u], xz[c], s);
              }
            }
          }
          for (int c = g; c < nx; c += G) s = fma(double(Bj[(size_t)c * n + i]), xc[xb_off + c], s);
        }
        part[tid] = s;
        __syncthreads();
        for (int i2 = tid; i2 < n; i2 += bs) {
          double t = 0.0;
          for (int g2 = 0; g2 < G; ++g2) t += part[g2 * n + i2];
          y[i2] = xc[(size_t)j * n + i2] - t;
        }
        __syncthreads();
      }
      // U y = rhs, from the last block of 32 rows up
      for (int rb = ((n - 1) / 32) * 32; rb >= 0; rb -= 32) {
        const int rw = n - rb < 32 ? n - rb : 32;
        // the diagonal block of U through shared memory (one coalesced load)
        for (int e = tid; e < rw * 32; e += bs) {
          const int c = e >> 5, r = e & 31;
          tb[c][r] = r < rw ? double(Tj[(size_t)(rb + c) * n2 + rb + r]) : 0.0;
        }
        __syncthreads();
        if (warp == 0) {
          double v = lane < rw ? y[rb + lane] : 0.0;
          const double rdi = lane < rw ? 1.0 / tb[lane][lane] : 0.0;
          for (int ii = rw - 1; ii >= 0; --ii) {
            const double xi = __shfl_sync(FULL, v * rdi, ii);
            if (lane == ii) v = xi;
            else if (lane < ii) v = fma(-tb[ii][lane], xi, v);
          }
          if (lane < rw) y[rb + lane] = v;
        }
        __syncthreads();
        for (int r = tid; r < rb; r += bs) {
          double s = y[r];
          for (int c0 = 0; c0 < rw; c0 += 8) {  // 8 loads in flight
            double tv[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) tv[u] = c0 + u < rw ? double(Tj[(size_t)(rb + c0 + u) * n2 + r]) : 0.0;
#pragma unroll
            for (int u = 0; u < 8; ++u)
              if (c0 + u < rw) s = fma(-tv[u], y[rb + c0 + u], s);
          }
          y[r] = s;
        }
        __syncthreads();
      }
      for (int i = tid; i < n; i += bs) {
        const int dst = qrp ? (int)a.P[(size_t)j * szP(d) + n2 + i] : i;
        xc[(size_t)j * n + dst] = y[i];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// last block (load_and_factorize_last, cc:1281-1374; solve_last, cc:1385-1479)
// one CTA; the Nr x Nc matrix lives in global memory (L2 resident)
// ---------------------------------------------------------------------------
template <typename T>
__device__ void last_assemble_range(Dims d, const T* D, const T* E, const T* B, const T* C,
                                    const double* H, const double* Cq, const double* Ffin, double* Hl,
                                    int e0, int es) {
  const int n = d.n, Nr = d.Nr, Nc = d.Nc, qx = d.qx, nr = d.nr, m = n + d.qr;
  const int total = Nr * Nc;
  const T* CN = C + (size_t)d.nblock * nr * n;
  for (int e = e0; e < total; e += es) {
    const int r = e % Nr, c = e / Nr;
    double v = 0.0;
    if (r < n) {
      if (c < n) v = D[(size_t)c * n + r];
      else if (c < 2 * n) v = E[(size_t)(c - n) * n + r];
      else if (c >= 2 * n + qx) v = B[(size_t)(c - 2 * n - qx) * n + r];
    } else if (r < n + m) {
      v = H[(size_t)c * m + (r - n)];
    } else {
      const int rr = r - n - m;
      if (c < n) v = C[(size_t)c * nr + rr];
      else if (c < 2 * n) v = CN[(size_t)(c - n) * nr + rr];
      else if (c < 2 * n + qx) v = Cq[(size_t)(c - 2 * n) * nr + rr];
      else v = Ffin[(size_t)(c - 2 * n - qx) * nr + rr];
    }
    Hl[e] = v;
  }
}

template <typename T>
__global__ void k_last_assemble(Dims d, const T* D, const T* E, const T* B, const T* C,
                                const double* H, const double* Cq, const double* Ffin, double* Hl) {
  last_assemble_range(d, D, E, B, C, H, Cq, Ffin, Hl, blockIdx.x * blockDim.x + threadIdx.x,
                      gridDim.x * blockDim.x);
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

// buffers of the last block (one CTA works on them)
struct LastBufs {
  double* A;    // Nr x Nc (ld Nr): the assembled block, then its factors
  double* A2;   // copy for the fallback solver (null when there is none)
  int* piv;     // row pivots [0, L), column pivots [L, 2L), L = max(Nr, Nc)
  double* tau;  // Householder scalars
  double* U;    // SVD: W = U*S, max(Nr,Nc) x min(Nr,Nc)
  double* V;    // SVD: min x min
  double* S;    // SVD: singular values
};

__device__ inline int last_kind_of(int sel_last, int M, int N) {
  switch (sel_last) {
    case LAST_LU: return FACT_LU;
    case LAST_LUPQ: return FACT_LUPQ;
    case LAST_QR: return FACT_QR;
    case LAST_QRP: return FACT_QRP;
    default: return M >= N ? FACT_SVD : FACT_SVD_T;  // SVD, LSS, LSY, PINV
  }
}

// Minimum-norm least-squares factorization of the SVD family (the solvers
// SVD, LSS, LSY and PINV of the reference's LapackWrapper): one-sided Jacobi
// on W = A (or A^T when Nr < Nc), rotations of a pair of columns p < q by the
// angle that makes them orthogonal, skipped when |g| <= 1e-15 sqrt(a b); the
// pairs of a sweep follow the round-robin (circle) schedule, so the Np/2 pairs
// of a round are independent and run one per warp; at most 80 sweeps, ending
// at the first sweep without a rotation.  On return W = U*S is split into
// unit columns U and S.
__device__ void last_svd(Dims d, const double* A, LastBufs b, StatusWords* st) {
  __shared__ int rotated;
  const int M = d.Nr, N = d.Nc, tid = threadIdx.x, bs = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nw = bs >> 5;
  const bool tr = M < N;
  const int Mp = tr ? N : M, Np = tr ? M : N;
  double* W = b.U;
  double* V = b.V;
  for (int e = tid; e < Mp * Np; e += bs) {
    const int i = e % Mp, j = e / Mp;
    W[(size_t)j * Mp + i] = tr ? A[(size_t)i * M + j] : A[(size_t)j * M + i];
  }
  for (int e = tid; e < Np * Np; e += bs) V[e] = (e % Np == e / Np) ? 1.0 : 0.0;
  __syncthreads();
  const int P = Np + (Np & 1);
  for (int sweep = 0; sweep < 80; ++sweep) {
    if (tid == 0) rotated = 0;
    __syncthreads();
    for (int r = 0; r < P - 1; ++r) {
      for (int k = warp; k < P / 2; k += nw) {
        int p0, q0;
        if (k == 0) { p0 = P - 1; q0 = r; }
        else { p0 = (r + k) % (P - 1); q0 = (r - k + P - 1) % (P - 1); }
        const int p = min(p0, q0), q = max(p0, q0);
        if (q >= Np) continue;
        double* wp = W + (size_t)p * Mp;
        double* wq = W + (size_t)q * Mp;
        double a = 0.0, bb = 0.0, g = 0.0;
        for (int i = lane; i < Mp; i += 32) {
          const double x = wp[i], y = wq[i];
          a = fma(x, x, a);
          bb = fma(y, y, bb);
          g = fma(x, y, g);
        }
        a = warp_sum(a);
        bb = warp_sum(bb);
        g = warp_sum(g);
        if (fabs(g) <= 1e-15 * sqrt(a * bb) || g == 0.0) continue;
        const double zeta = (bb - a) / (2.0 * g);
        const double t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        const double c = 1.0 / sqrt(1.0 + t * t), s = c * t;
        for (int i = lane; i < Mp; i += 32) {
          const double x = wp[i], y = wq[i];
          wp[i] = c * x - s * y;
          wq[i] = s * x + c * y;
        }
        double* vp = V + (size_t)p * Np;
        double* vq = V + (size_t)q * Np;
        for (int i = lane; i < Np; i += 32) {
          const double x = vp[i], y = vq[i];
          vp[i] = c * x - s * y;
          vq[i] = s * x + c * y;
        }
        if (lane == 0) rotated = 1;
      }
      __syncthreads();
    }
    const int any = rotated;
    __syncthreads();
    if (!any) break;
  }
  for (int j = warp; j < Np; j += nw) {
    double* wj = W + (size_t)j * Mp;
    double s2 = 0.0;
    for (int i = lane; i < Mp; i += 32) s2 = fma(wj[i], wj[i], s2);
    const double sj = sqrt(warp_sum(s2));
    if (lane == 0) b.S[j] = sj;
    if (sj > 0.0)
      for (int i = lane; i < Mp; i += 32) wj[i] /= sj;
  }
  if (tid == 0) st->kind = tr ? FACT_SVD_T : FACT_SVD;
  __syncthreads();
}

// load_and_factorize_last (cc:1281-1374) with the reference's last-block
// solvers: LU (getrf), LUPQ (complete pivoting), QR (geqrf), QRP (geqp3: the
// column of largest remaining 2-norm first), and the SVD family
// Last blocks of order <= LAST_SMALL (configs with n <= 16 and small borders):
// the LU runs out of shared memory (the general loop below works in global
// memory, a round trip per column) and the LU solves run on one warp with the
// values in registers.  Same pivot rule (largest |a|, first row on ties, NaN
// never chosen), same operation order.
constexpr int LAST_SMALL = 64;

template <typename T>
__device__ void last_lu_small(Dims d, LastBufs b, StatusWords* st) {
  __shared__ T As[LAST_SMALL * (LAST_SMALL + 1)];
  __shared__ T s_pv;
  __shared__ int s_p;
  const int N = d.Nc, ld = N + 1, tid = threadIdx.x, bs = blockDim.x;
  T* A = b.A;
  for (int c = tid / 32; c < N; c += bs / 32)  // one column per warp: coalesced, all loads in flight
    for (int r = tid & 31; r < N; r += 32) As[c * ld + r] = A[(size_t)c * N + r];
  __syncthreads();
  for (int i = 0; i < N; ++i) {
    if (tid < 32) {  // pivot of column i: largest |a| over rows >= i, first row on ties, NaN never
      T best = T(-2);
      int bi = 0x7fffffff;
      for (int r = i + tid; r < N; r += 32) {
        T v = dev_abs(As[i * ld + r]);
        if (!(v == v)) v = T(-1);
        if (v > best) { best = v; bi = r; }
      }
      // upper words of |a| first (one reduction); the exact argmax only on a tie
      const unsigned key = best < T(0) ? 0u : (unsigned)((unsigned long long)__double_as_longlong((double)best) >> 32) + 1u;
      const unsigned kmax = __reduce_max_sync(0xffffffffu, key);
      const unsigned m = __ballot_sync(0xffffffffu, key == kmax);
      if (__popc(m) == 1 && kmax > 0) {
        bi = __shfl_sync(0xffffffffu, bi, __ffs(m) - 1);
      } else {
        warp_argmax(best, bi);
      }
      if (tid == 0) { s_p = bi; s_pv = As[i * ld + bi]; }
    }
    __syncthreads();
    const int p = s_p;
    const T pv = s_pv;
    if (pv == T(0)) {
      if (tid == 0) report(st, DEV_LAST_SINGULAR, -1, i + 1, -1);
      return;
    }
    if (tid == 0) b.piv[i] = p;
    if (p != i)
      for (int c = tid; c < N; c += bs) {
        const T t = As[c * ld + i]; As[c * ld + i] = As[c * ld + p]; As[c * ld + p] = t;
      }
    __syncthreads();
    const T rinv = T(1) / pv;
    for (int r = i + 1 + tid; r < N; r += bs) As[i * ld + r] *= rinv;
    __syncthreads();
    {  // trailing update: thread -> row (tid % 64), columns every bs/64
      const int r = i + 1 + (tid & 63), cs = bs >> 6;
      if (r < N) {
        const T m = As[i * ld + r];
        for (int c = i + 1 + (tid >> 6); c < N; c += cs)
          As[c * ld + r] = fma(-m, As[c * ld + i], As[c * ld + r]);
      }
    }
    __syncthreads();
  }
  for (int c = tid / 32; c < N; c += bs / 32)
    for (int r = tid & 31; r < N; r += 32) A[(size_t)c * N + r] = As[c * ld + r];
  if (tid == 0) st->kind = FACT_LU;
}

template <typename T>
__device__ void last_factor_body(Dims d, LastBufs b, int sel_last, StatusWords* st) {
  __shared__ T sv[32];
  __shared__ int si[32];
  const int M = d.Nr, N = d.Nc, tid = threadIdx.x, bs = blockDim.x;
  const int kind = last_kind_of(sel_last, M, N);
  T* A = b.A;
  int* piv = b.piv;
  T* tau = b.tau;
  if (kind == FACT_SVD || kind == FACT_SVD_T) {
    last_svd(d, A, b, st);
    return;
  }
  if (kind == FACT_LU && M == N && N <= LAST_SMALL) {
    last_lu_small<T>(d, b, st);
    return;
  }
  if (kind == FACT_LU) {
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
      __syncthreads();  // every thread holds the pivot before column i is swapped
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
  } else if (kind == FACT_LUPQ) {
    if (M != N) { if (tid == 0) report(st, DEV_BAD_SHAPE, -1, 0, -1); return; }
    const int L = M > N ? M : N;
    for (int i = 0; i < N; ++i) {
      // largest |a| of the trailing block, first in column-major order on ties
      const int w = N - i;
      T best = T(-1);
      int bidx = i * N + i;
      for (int e = tid; e < w * w; e += bs) {
        const int r = i + e % w, c = i + e / w;
        const T v = dev_abs(A[(size_t)c * N + r]);
        const int idx = c * N + r;
        if (v > best || (v == best && idx < bidx)) { best = v; bidx = idx; }
      }
      block_argmax(best, bidx, sv, si);
      const int pr = bidx % N, pc = bidx / N;
      if (tid == 0) { piv[i] = pr; piv[L + i] = pc; }
      __syncthreads();
      if (best == T(0)) { if (tid == 0) report(st, DEV_LAST_SINGULAR, -1, i + 1, -1); return; }
      if (pr != i)
        for (int c = tid; c < N; c += bs) {
          T t = A[(size_t)c * N + i]; A[(size_t)c * N + i] = A[(size_t)c * N + pr]; A[(size_t)c * N + pr] = t;
        }
      __syncthreads();
      if (pc != i)
        for (int r = tid; r < N; r += bs) {
          T t = A[(size_t)i * N + r]; A[(size_t)i * N + r] = A[(size_t)pc * N + r]; A[(size_t)pc * N + r] = t;
        }
      __syncthreads();
      const T pv = A[(size_t)i * N + i];
      __syncthreads();
      for (int r = i + 1 + tid; r < N; r += bs) A[(size_t)i * N + r] /= pv;
      __syncthreads();
      const int Lr = N - i - 1;
      for (int e = tid; e < Lr * Lr; e += bs) {
        const int r = i + 1 + e % Lr, c = i + 1 + e / Lr;
        A[(size_t)c * N + r] -= A[(size_t)i * N + r] * A[(size_t)c * N + i];
      }
      __syncthreads();
    }
  } else {  // Householder QR (QRP: largest remaining column first), M >= N
    if (M < N) { if (tid == 0) report(st, DEV_BAD_SHAPE, -1, 0, -1); return; }
    const int L = M > N ? M : N;
    if (kind == FACT_QRP)
      for (int c = tid; c < N; c += bs) piv[L + c] = c;
    __syncthreads();
    for (int i = 0; i < N; ++i) {
      if (kind == FACT_QRP) {
        T best = T(-1);
        int bc = i;
        for (int c = i + tid; c < N; c += bs) {
          const T* col = A + (size_t)c * M;
          T s2 = T(0);
          for (int r = i; r < M; ++r) s2 += col[r] * col[r];
          if (s2 > best) { best = s2; bc = c; }
        }
        block_argmax(best, bc, sv, si);
        if (bc != i) {
          for (int r = tid; r < M; r += bs) {
            T t = A[(size_t)i * M + r]; A[(size_t)i * M + r] = A[(size_t)bc * M + r]; A[(size_t)bc * M + r] = t;
          }
          if (tid == 0) { const int t = piv[L + i]; piv[L + i] = piv[L + bc]; piv[L + bc] = t; }
        }
        __syncthreads();
      }
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
  if (tid == 0) st->kind = kind;
}

// the select_last2 fallback (cc:1347-1369): when the chosen solver failed on
// the last block, factor the saved copy with the SVD family instead
__device__ void last_fallback_body(Dims d, LastBufs b, StatusWords* st) {
  const int code = st->code;
  __syncthreads();
  if (code != DEV_LAST_SINGULAR && code != DEV_BAD_SHAPE) return;
  if (threadIdx.x == 0) *st = StatusWords{0, 0, 0, 0, 0};
  __syncthreads();
  last_svd(d, b.A2, b, st);
}

template <typename T>
__device__ void last_solve_body(Dims d, LastBufs lb, const StatusWords* st, T* x, int ldx, int nrhs) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = d.n, M = d.Nr, N = d.Nc, tid = threadIdx.x, bs = blockDim.x;
  const int L = M > N ? M : N;
  T* b = reinterpret_cast<T*>(smem_raw);
  T* tmp = b + L;
  __shared__ T sv[32];
  // a diagonal 32 x 32 block of the blocked LU's factors, or the whole L\U of a
  // small last block (order <= LAST_SMALL, ld order + 1)
  __shared__ T big[LAST_SMALL * (LAST_SMALL + 1)];
  T (*lt)[33] = reinterpret_cast<T (*)[33]>(big);
  const int kind = st->kind;
  const bool small_lu = kind == FACT_LU && M == N && N <= LAST_SMALL;
  if (small_lu) {
    for (int e = tid; e < N * N; e += bs) big[(e / N) * (N + 1) + e % N] = lb.A[e];
    __syncthreads();
  }
  const T* A = lb.A;
  const int* piv = lb.piv;
  const T* tau = lb.tau;
  const size_t off = (size_t)d.nblock * n;
  T tol = T(0);
  if (kind == FACT_SVD || kind == FACT_SVD_T) {
    const int Np = kind == FACT_SVD ? N : M;
    T smax = T(0);
    for (int j = tid; j < Np; j += bs) smax = fmax(smax, lb.S[j]);
    for (int o = 16; o > 0; o >>= 1) smax = fmax(smax, __shfl_xor_sync(0xffffffffu, smax, o));
    if ((tid & 31) == 0) sv[tid >> 5] = smax;
    __syncthreads();
    if (tid == 0) {
      T m = T(0);
      for (int w = 0; w < (bs >> 5); ++w) m = fmax(m, sv[w]);
      sv[0] = m;
    }
    __syncthreads();
    tol = sv[0] * T(1e-12);
    __syncthreads();
  }
  for (int c = 0; c < nrhs; ++c) {
    T* xc = x + (size_t)c * ldx;
    for (int r = tid; r < M; r += bs) b[r] = r < n ? xc[r] : xc[off + (r - n)];
    __syncthreads();
    if (kind == FACT_SVD || kind == FACT_SVD_T) {
      // x = V S^+ U^T b (Nr >= Nc) or x = U S^+ V^T b (Nr < Nc)
      const bool trn = kind == FACT_SVD_T;
      const int Mp = trn ? N : M, Np = trn ? M : N;
      const int lane = tid & 31, warp = tid >> 5, nw = bs >> 5;
      for (int j = warp; j < Np; j += nw) {
        const T sj = lb.S[j];
        T s = T(0);
        if (sj > tol) {
          const T* col = trn ? lb.V + (size_t)j * Np : lb.U + (size_t)j * Mp;
          const int len = trn ? Np : Mp;
          for (int i = lane; i < len; i += 32) s = fma(col[i], b[i], s);
          s = warp_sum(s) / sj;
        }
        if (lane == 0) tmp[j] = s;
      }
      __syncthreads();
      const int nout = trn ? Mp : Np;
      for (int i = tid; i < nout; i += bs) {
        T s = T(0);
        for (int j = 0; j < Np; ++j)
          s = fma(trn ? lb.U[(size_t)j * Mp + i] : lb.V[(size_t)j * Np + i], tmp[j], s);
        b[i] = s;
      }
      __syncthreads();
    } else if (small_lu) {
      // row interchanges, unit-lower and upper solves on one warp, the values in
      // registers (lane = rows lane and lane + 32) and L\U in shared memory
      if (tid < 32) {
        const int lane = tid, r0 = lane, r1 = lane + 32, ld = N + 1;
        if (lane == 0)
          for (int i = 0; i < N; ++i) {
            const int p = piv[i];
            if (p != i) { T t = b[i]; b[i] = b[p]; b[p] = t; }
          }
        __syncwarp();
        T x0 = r0 < N ? b[r0] : T(0), x1 = r1 < N ? b[r1] : T(0);
        for (int i = 0; i < N; ++i) {
          const T bi = __shfl_sync(0xffffffffu, i < 32 ? x0 : x1, i & 31);
          if (r0 > i && r0 < N) x0 = fma(-big[i * ld + r0], bi, x0);
          if (r1 > i && r1 < N) x1 = fma(-big[i * ld + r1], bi, x1);
        }
        for (int i = N - 1; i >= 0; --i) {
          const T xi = __shfl_sync(0xffffffffu, i < 32 ? x0 : x1, i & 31) / big[i * ld + i];
          if (r0 == i) x0 = xi;
          else if (r0 < i) x0 = fma(-big[i * ld + r0], xi, x0);
          if (r1 == i) x1 = xi;
          else if (r1 < i) x1 = fma(-big[i * ld + r1], xi, x1);
        }
        if (r0 < N) b[r0] = x0;
        if (r1 < N) b[r1] = x1;
      }
      __syncthreads();
    } else {
      if (kind == FACT_LU || kind == FACT_LUPQ) {
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
      } else if (kind == FACT_LU_ROWS) {
        for (int r = tid; r < N; r += bs) tmp[r] = b[piv[r]];
        __syncthreads();
        for (int r = tid; r < N; r += bs) b[r] = tmp[r];
        __syncthreads();
        // unit lower L by blocks of 32 rows: the diagonal block staged in shared
        // memory and solved by one warp, the rows below updated with 8 loads in
        // flight (same operation order as one column at a time)
        const int lane = tid & 31, warp = tid >> 5;
        for (int kb = 0; kb < N; kb += 32) {
          const int w = N - kb < 32 ? N - kb : 32;
          for (int e = tid; e < 32 * 32; e += bs) {
            const int c = e >> 5, r = e & 31;
            lt[c][r] = (c < w && r < w) ? A[(size_t)(kb + c) * N + piv[kb + r]] : T(0);
          }
          __syncthreads();
          if (warp == 0) {
            T v = lane < w ? b[kb + lane] : T(0);
            for (int c = 0; c < w; ++c) {
              const T vc = __shfl_sync(0xffffffffu, v, c);
              if (lane > c && lane < w) v = fma(-lt[c][lane], vc, v);
            }
            if (lane < w) b[kb + lane] = v;
          }
          __syncthreads();
          for (int r = kb + w + tid; r < N; r += bs) {
            const int pr = piv[r];
            T sr = b[r];
            for (int c0 = 0; c0 < w; c0 += 8) {
              T av[8];
#pragma unroll
              for (int u = 0; u < 8; ++u) av[u] = c0 + u < w ? A[(size_t)(kb + c0 + u) * N + pr] : T(0);
#pragma unroll
              for (int u = 0; u < 8; ++u)
                if (c0 + u < w) sr = fma(-av[u], b[kb + c0 + u], sr);
            }
            b[r] = sr;
          }
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
      const int lda = (kind == FACT_LU || kind == FACT_LUPQ) ? N : M;
      if (kind == FACT_LU_ROWS) {
        // U by blocks of 32 rows from the bottom (row of position r: piv[r]), the
        // same operation order as one column at a time
        const int lane = tid & 31, warp = tid >> 5;
        for (int rb = ((N - 1) / 32) * 32; rb >= 0; rb -= 32) {
          const int w = N - rb < 32 ? N - rb : 32;
          for (int e = tid; e < 32 * 32; e += bs) {
            const int c = e >> 5, r = e & 31;
            lt[c][r] = (c < w && r < w) ? A[(size_t)(rb + c) * N + piv[rb + r]] : T(0);
          }
          __syncthreads();
          if (warp == 0) {
            T v = lane < w ? b[rb + lane] : T(0);
            const T dl = lane < w ? lt[lane][lane] : T(1);
            for (int ii = w - 1; ii >= 0; --ii) {
              const T xi = __shfl_sync(0xffffffffu, v / dl, ii);
              if (lane == ii) v = xi;
              else if (lane < ii) v = fma(-lt[ii][lane], xi, v);
            }
            if (lane < w) b[rb + lane] = v;
          }
          __syncthreads();
          for (int r = tid; r < rb; r += bs) {
            const int pr = piv[r];
            T sr = b[r];
            for (int c1 = w; c1 > 0; c1 -= 8) {  // columns rb + w - 1 down to rb
              T av[8];
#pragma unroll
              for (int u = 0; u < 8; ++u) av[u] = c1 - 1 - u >= 0 ? A[(size_t)(rb + c1 - 1 - u) * N + pr] : T(0);
#pragma unroll
              for (int u = 0; u < 8; ++u)
                if (c1 - 1 - u >= 0) sr = fma(-av[u], b[rb + c1 - 1 - u], sr);
            }
            b[r] = sr;
          }
          __syncthreads();
        }
      } else {
        for (int i = N - 1; i >= 0; --i) {
          const T xi = b[i] / A[(size_t)i * lda + i];
          __syncthreads();
          if (tid == 0) b[i] = xi;
          for (int r = tid; r < i; r += bs) b[r] -= A[(size_t)i * lda + r] * xi;
          __syncthreads();
        }
      }
      if (kind == FACT_LUPQ) {
        if (tid == 0)
          for (int i = N - 1; i >= 0; --i) {
            const int q = piv[L + i];
            if (q != i) { T t = b[i]; b[i] = b[q]; b[q] = t; }
          }
        __syncthreads();
      } else if (kind == FACT_QRP) {
        for (int i = tid; i < N; i += bs) tmp[piv[L + i]] = b[i];
        __syncthreads();
        for (int i = tid; i < N; i += bs) b[i] = tmp[i];
        __syncthreads();
      }
    }
    for (int r = tid; r < N; r += bs) {
      if (r < n) xc[r] = b[r];
      else xc[off + (r - n)] = b[r];
    }
    __syncthreads();
  }
}

template <typename T>
__global__ void k_last_factor(Dims d, LastBufs b, int sel_last, StatusWords* st) {
  last_factor_body<T>(d, b, sel_last, st);
}

// load_and_factorize_last with LU for larger blocks (cc:1319-1346, getrf): the
// blocked elimination of the pair kernels on the whole block, FP64 tensor-core
// products, rows left in place (kind FACT_LU_ROWS, piv[pos] = row)
__global__ void __launch_bounds__(256, 1) k_last_lu_blocked(Dims d, LastBufs b, StatusWords* st) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double sv[32];
  __shared__ int si[32];
  __shared__ int s_perm[BLK_ROWS_MAX];
  const int N = d.Nc, tid = threadIdx.x;
  if (d.Nr != N || N > BLK_ROWS_MAX) {
    if (tid == 0) report(st, DEV_BAD_SHAPE, -1, 0, -1);
    return;
  }
  for (int r = tid; r < N; r += blockDim.x) s_perm[r] = r;
  __syncthreads();
  double* Pb = reinterpret_cast<double*>(smem_raw);
  const int info = blk_eliminate<double>(b.A, N, N, N, N, Pb, s_perm, sv, si);
  if (info != 0) {
    if (tid == 0) report(st, DEV_LAST_SINGULAR, -1, info, -1);
    return;
  }
  for (int r = tid; r < N; r += blockDim.x) b.piv[r] = s_perm[r];
  if (tid == 0) st->kind = FACT_LU_ROWS;
}

__global__ void k_last_fallback(Dims d, LastBufs b, StatusWords* st) { last_fallback_body(d, b, st); }

// LU of a last block of order <= LAST_SMALL on its own (one CTA)
__global__ void __launch_bounds__(256) k_last_lu_small(Dims d, LastBufs b, StatusWords* st) {
  last_lu_small<double>(d, b, st);
}

template <typename T>
__global__ void k_last_solve(Dims d, LastBufs b, const StatusWords* st, T* x, int ldx, int nrhs) {
  last_solve_body<T>(d, b, st, x, ldx, nrhs);
}

static LastBufs last_bufs(const DevState& s) {
  LastBufs b;
  b.A = s.Hl; b.A2 = s.Al; b.piv = s.piv_l; b.tau = s.tau_l; b.U = s.Ul; b.V = s.Vl; b.S = s.Sl;
  return b;
}

// ---------------------------------------------------------------------------
// Mv with the loaded matrix (add_Mv, cc:2118-2166): res = alpha*A*x + beta*res
// ---------------------------------------------------------------------------
// ABS: |A| * 1 (row sums of absolute values, for ||A||_inf); x is not read.
// Otherwise, with rowsum non-null, the same pass also writes |A| * 1 there.
template <bool ABS>
__global__ void k_mv_rows(Dims d, const double* D, const double* E, const double* B, double alpha,
                          const double* x, double beta, double* res, double* rowsum = nullptr) {
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
    if constexpr (ABS) {
      for (int c = 0; c < n; ++c) s += fabs(Dk[(size_t)c * n + i]) + fabs(Ek[(size_t)c * n + i]);
      for (int c = 0; c < nx; ++c) s += fabs(Bk[(size_t)c * n + i]);
      res[e] = s;
    } else if (rowsum) {
      double sa = 0;
      for (int c = 0; c < n; ++c) {
        const double a = Dk[(size_t)c * n + i];
        s += a * x[k * n + c];
        sa += fabs(a);
      }
      for (int c = 0; c < n; ++c) {
        const double a = Ek[(size_t)c * n + i];
        s += a * x[(k + 1) * n + c];
        sa += fabs(a);
      }
      for (int c = 0; c < nx; ++c) {
        const double a = Bk[(size_t)c * n + i];
        s += a * x[xb_off + c];
        sa += fabs(a);
      }
      res[e] = (beta == 0.0 ? 0.0 : beta * res[e]) + alpha * s;
      rowsum[e] = sa;
    } else {
      for (int c = 0; c < n; ++c) s += Dk[(size_t)c * n + i] * x[k * n + c];
      for (int c = 0; c < n; ++c) s += Ek[(size_t)c * n + i] * x[(k + 1) * n + c];
      for (int c = 0; c < nx; ++c) s += Bk[(size_t)c * n + i] * x[xb_off + c];
      res[e] = (beta == 0.0 ? 0.0 : beta * res[e]) + alpha * s;
    }
  }
}

template <bool ABS>
__global__ void k_mv_cpart(Dims d, const double* C, const double* x, double* part) {
  const int n = d.n, nr = d.nr;
  const size_t total = (size_t)(d.nblock + 1) * nr;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const size_t k = e / nr;
    const int r = (int)(e % nr);
    const double* Ck = C + k * nr * n;
    double s = 0;
    for (int c = 0; c < n; ++c) s += ABS ? fabs(Ck[(size_t)c * nr + r]) : Ck[(size_t)c * nr + r] * x[k * n + c];
    part[e] = s;
  }
}

// H rows and the nr border rows (Csum = sum_k C_k x_k precomputed)
template <bool ABS>
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
        s += ABS ? fabs(H[(size_t)c * m + r]) : H[(size_t)c * m + r] * x[xi];
      }
    } else {
      const int rr = r - m;
      s = Csum[rr];
      for (int c = 0; c < qx; ++c) s += ABS ? fabs(Cq[(size_t)c * nr + rr]) : Cq[(size_t)c * nr + rr] * x[xq + c];
      for (int c = 0; c < nx; ++c) s += ABS ? fabs(F[(size_t)c * nr + rr]) : F[(size_t)c * nr + rr] * x[xb + c];
    }
    const size_t o = r0 + r;
    res[o] = ABS ? s : (beta == 0.0 ? 0.0 : beta * res[o]) + alpha * s;
  }
}

// ---------------------------------------------------------------------------
// host orchestration
// ---------------------------------------------------------------------------
// Raise a kernel's dynamic shared-memory limit once per process and kernel;
// later calls (for instance inside a CUDA graph capture) only launch.
template <typename K>
static void smem_limit_once(K* kernel, size_t bytes) {
  if (bytes <= 48 * 1024) return;
  static const void* keys[64];
  static size_t done[64];
  static int used = 0;
  const void* key = reinterpret_cast<const void*>(kernel);
  int slot = 0;
  while (slot < used && keys[slot] != key) ++slot;
  if (slot < used && done[slot] >= bytes) return;
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (slot == used && used < 64) { keys[used] = key; ++used; }
  if (slot < 64) done[slot] = bytes;
}

// CTAs of `kernel` resident on one SM (cached per kernel)
template <typename K>
static int resident_ctas(K* kernel, int threads, size_t smem) {
  static const void* keys[64];
  static int value[64];
  static int used = 0;
  const void* key = reinterpret_cast<const void*>(kernel);
  for (int i = 0; i < used; ++i)
    if (keys[i] == key) return value[i];
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, threads, smem) != cudaSuccess || nb < 1) nb = 1;
  if (used < 64) { keys[used] = key; value[used] = nb; ++used; }
  return nb;
}

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

// sums of per-block m-vectors, m = h x cols (column-major, height h <= 256);
// column groups of at most 256 elements are reduced one after the other
static void reduce_blocks(DevState& s, const double* buf, long first, long count, int m, int h,
                          const double* base, int ldb, double* out, int ldo, cudaStream_t st) {
  if (m <= 0 || h <= 0) return;
  const int cols = m / h, cw = h <= 256 ? 256 / h : 1;
  const long chunk = 1024;
  const int nparts = count > 0 ? (int)((count + chunk - 1) / chunk) : 0;
  for (int c0 = 0; c0 < cols; c0 += cw) {
    const int cn = cols - c0 < cw ? cols - c0 : cw, mm = cn * h;
    const double* bb = buf + (size_t)c0 * h;
    const double* ba = base ? base + (size_t)c0 * ldb : nullptr;
    double* oo = out + (size_t)c0 * ldo;
    if (nparts > 1) {
      k_reduce_tree<double><<<nparts, 256, 0, st>>>(bb, m, first, count, mm, chunk, s.part, nullptr, h,
                                                    0, nullptr, 0);
      check_launch("k_reduce_tree");
      k_reduce_tree<double><<<1, 256, 0, st>>>(s.part, mm, 0, nparts, mm, nparts, nullptr, ba, h, ldb,
                                               oo, ldo);
    } else {
      k_reduce_tree<double><<<1, 256, 0, st>>>(bb, m, first, count, mm, chunk, nullptr, ba, h, ldb, oo,
                                               ldo);
    }
    check_launch("k_reduce_tree");
  }
}

// ---------------------------------------------------------------------------
// working arrays of one precision
// ---------------------------------------------------------------------------
template <typename T>
struct WorkSet {
  T *D, *E, *B, *C, *Tm, *Rbuf;
  T* slab;
};

static WorkSet<double> work_set(DevState& s, double*) {
  return {s.D, s.E, s.B, s.C, s.T, s.Rbuf, reinterpret_cast<double*>(s.slab)};
}
static WorkSet<float> work_set(DevState& s, float*) {
  return {s.Df, s.Ef, s.Bf, s.Cf, s.Tf, s.Rbuff, reinterpret_cast<float*>(s.slab)};
}

// ---------------------------------------------------------------------------
// pair-kernel choice for the factorization
// ---------------------------------------------------------------------------
template <typename T>
struct FactorPlan {
  void (*cta)(FactorArgs<T>, T*, size_t) = nullptr;  // CTA per pair (large n)
  void (*blk)(FactorArgs<T>, T*, size_t) = nullptr;  // CTA per pair, blocked LU (large n)
  size_t blk_smem = 0;
  void (*umma)(FactorArgs<T>, T*, size_t) = nullptr;  // CTA per pair, tcgen05 products (FP32, large n)
  size_t umma_smem = 0;
  void (*tc)(FactorArgs<T>, const FactorArgs<T>*, const BatchCta*) = nullptr;               // tensor-core LU (FP64, n = 8, 16)
  size_t tc_smem = 0;
  void (*tree)(FactorArgs<double>, TreeArgs) = nullptr;  // tc pairs, whole reduction in one launch
  int tree_ctas = 0;
  // tc pairs level by level with the tree's border bookkeeping (single systems)
  void (*tcb)(FactorArgs<double>, const FactorArgs<double>*, const BatchCta*) = nullptr;
  void (*top)(FactorArgs<double>, int) = nullptr;  // the top levels in one CTA (single systems)
  void (*root)(FactorArgs<double>, TreeArgs, int) = nullptr;
  void (*grp)(FactorArgs<T>, const FactorArgs<T>*, const BatchCta*) = nullptr;              // CTA of 2n threads per pair (n = 16, 32)
  size_t grp_smem = 0;
  int grp_threads = 0, grp_ctas = 0;
  void (*rows)(FactorArgs<T>, const FactorArgs<T>*, const BatchCta*) = nullptr;             // register LU (n <= 16)
  void (*smem_k)(FactorArgs<T>, const FactorArgs<T>*, const BatchCta*) = nullptr;           // shared-memory kernel
  size_t smem = 0;
  int wpb = 1;
  int tc_cols = 0;                                   // trailing-column capacity of tc
};

template <typename T>
static FactorPlan<T> plan_factor(const DevState& s) {
  const Dims d = s.d;
  const int n = d.n;
  FactorPlan<T> p;
  const size_t per_warp = panel_smem_per_warp(d, (int)sizeof(T));
  p.wpb = (int)(SMEM_MAX / per_warp);
  if (p.wpb > WARPS_PANEL) p.wpb = WARPS_PANEL;
  if (p.wpb < 1) p.wpb = 1;
  p.smem = per_warp * p.wpb;
  p.smem_k = s.sel == SEL_LU ? k_factor_level<T, SEL_LU>
           : s.sel == SEL_QR ? k_factor_level<T, SEL_QR> : k_factor_level<T, SEL_QRP>;
  if (p.smem <= SMEM_MAX) smem_limit_once(p.smem_k, p.smem);
  if constexpr (sizeof(T) == 8) {
    if (s.sel == SEL_LU && d.nr <= 8 && d.nx <= 8 && (n == 16 || n == 8) && s.use_tc &&
        (s.pair_kernel == PAIR_AUTO || s.pair_kernel == PAIR_TC || s.pair_kernel == PAIR_TREE ||
         s.pair_kernel == PAIR_TC_GATHER)) {
      p.tc_smem = tc_smem_per_warp(n) * 4;
      // border rows spread over the warp: 8 lanes per row when nr <= 4, else 4
      const bool r4 = d.nr <= 4;
      if (n == 16) p.tc = r4 ? k_factor_lu_tc<16, false, false, 4> : k_factor_lu_tc<16, false, false, 8>;
      else p.tc = r4 ? k_factor_lu_tc<8, false, false, 4> : k_factor_lu_tc<8, false, false, 8>;
      smem_limit_once(p.tc, p.tc_smem);
      p.tc_cols = n == 16 ? TcShape<16>::NTP : TcShape<8>::NTP;
      if (s.tree_cnt) {  // single systems (batches keep their own level loop)
        if (n == 16) p.top = r4 ? k_factor_top_tc<16, 4> : k_factor_top_tc<16, 8>;
        else p.top = r4 ? k_factor_top_tc<8, 4> : k_factor_top_tc<8, 8>;
        smem_limit_once(p.top, tc_smem_per_warp(n) * TOP_WARPS);
      }
      if (s.pair_kernel == PAIR_TC_GATHER && s.tree_cnt && d.nblock >= 2) {
        if (n == 16) p.tcb = r4 ? k_factor_lu_tc<16, false, true, 4> : k_factor_lu_tc<16, false, true, 8>;
        else p.tcb = r4 ? k_factor_lu_tc<8, false, true, 4> : k_factor_lu_tc<8, false, true, 8>;
        p.root = n == 16 ? k_tree_root<16> : k_tree_root<8>;
        smem_limit_once(p.tcb, p.tc_smem);
      }
      // the tree schedule (single systems with at least one pair), on request:
      // its top levels run one pair per warp along a serial chain, which costs
      // more than the level-by-level launches save at the sizes measured
      if (s.pair_kernel == PAIR_TREE && s.tree_cnt && d.nblock >= 2) {
        if (n == 16) p.tree = r4 ? k_factor_tree_tc<16, 4> : k_factor_tree_tc<16, 8>;
        else p.tree = r4 ? k_factor_tree_tc<8, 4> : k_factor_tree_tc<8, 8>;
        smem_limit_once(p.tree, p.tc_smem);
        p.tree_ctas = 148 * resident_ctas(p.tree, 128, p.tc_smem);
      }
    }
  } else {
    // FP32 factors (mixed path): the same warp-per-pair kernel with FP32
    // products, level by level, no fused right-hand sides
    if (s.sel == SEL_LU && d.nr <= 8 && d.nx <= 8 && (n == 16 || n == 8) && s.use_tc &&
        (s.pair_kernel == PAIR_AUTO || s.pair_kernel == PAIR_TC)) {
      p.tc_smem = tc_smem_per_warp_t<T>(n) * 4;
      const bool r4 = d.nr <= 4;
      if (n == 16) p.tc = r4 ? k_factor_lu_tc<16, false, false, 4, T> : k_factor_lu_tc<16, false, false, 8, T>;
      else p.tc = r4 ? k_factor_lu_tc<8, false, false, 4, T> : k_factor_lu_tc<8, false, false, 8, T>;
      smem_limit_once(p.tc, p.tc_smem);
      p.tc_cols = n == 16 ? TcShape<16, T>::NTP : TcShape<8, T>::NTP;
    }
  }
  const bool grp_ok = s.sel == SEL_LU && d.nr <= 8 && d.nx <= 8 &&
                      (n == 32 || (n == 16 && (sizeof(T) == 4 || s.pair_kernel == PAIR_GRP)));
  if (!p.tc && grp_ok && (s.pair_kernel == PAIR_AUTO || s.pair_kernel == PAIR_GRP)) {
    if (n == 32) {
      p.grp = k_factor_lu_grp<T, 32>;
      p.grp_smem = GrpShape<T, 32>::BYTES;
    } else {
      p.grp = k_factor_lu_grp<T, 16>;
      p.grp_smem = GrpShape<T, 16>::BYTES;
    }
    p.grp_threads = 2 * n + 32;
    smem_limit_once(p.grp, p.grp_smem);
    p.grp_ctas = 148 * resident_ctas(p.grp, p.grp_threads, p.grp_smem);
  }
  if (!p.tc && !p.grp && s.sel == SEL_LU && d.nr <= 4 && d.nx <= 4 && s.pair_kernel != PAIR_CTA &&
      s.pair_kernel != PAIR_SMEM) {
    if (n <= 4) p.rows = k_factor_lu_rows<T, 4, 4, 4>;
    else if (n <= 8) p.rows = k_factor_lu_rows<T, 8, 4, 4>;
    else if (n <= 16) p.rows = k_factor_lu_rows<T, 16, 4, 4>;
  }
  const bool smem_fits = per_warp <= SMEM_MAX;
  if (!p.tc && !p.grp && !p.rows &&
      (use_cta_kernel(d) || s.pair_kernel == PAIR_CTA || !smem_fits) &&
      (s.pair_kernel != PAIR_SMEM || !smem_fits)) {
    p.cta = s.sel == SEL_LU ? k_factor_cta<T, SEL_LU>
          : s.sel == SEL_QR ? k_factor_cta<T, SEL_QR> : k_factor_cta<T, SEL_QRP>;
    const size_t bsm = (size_t)BLK_W * (2 * n + d.nr) * sizeof(T);
    if (s.sel == SEL_LU && n <= 128 && 2 * n + d.nr <= BLK_ROWS_MAX && bsm <= SMEM_MAX) {
      p.blk = k_factor_lu_blocked<T>;
      p.blk_smem = bsm;
      smem_limit_once(p.blk, bsm);
    }
    if constexpr (sizeof(T) == 4) {
      if (s.sel == SEL_LU && umma_fits(d) && (s.pair_kernel == PAIR_AUTO || s.pair_kernel == PAIR_UMMA)) {
        p.umma = k_factor_lu_umma;
        p.umma_smem = umma_layout(d).bytes;
        smem_limit_once(p.umma, p.umma_smem);
      }
    }
  }
  return p;
}

// number of right-hand sides the factorization can carry (0: none)
template <typename T>
static int fusable_rhs(const DevState& s, const FactorPlan<T>& p, int nrhs) {
  if (!p.tc || nrhs < 1 || nrhs > 16) return 0;
  return 2 * s.d.n + s.d.nx + nrhs <= p.tc_cols ? nrhs : 0;
}

// every CR level: pair eliminations and the C_jpp border fix-up.  Returns true
// when the tree schedule ran, which also leaves F (s.Ffin), C_nblock and, for
// fused right-hand sides, xb complete.
template <typename T>
static bool factor_levels(DevState& s, const FactorPlan<T>& p, const WorkSet<T>& w, double* x, int ldx,
                          int nrf, cudaStream_t st) {
  const Dims d = s.d;
  const int n = d.n, nb = d.nblock;
  const size_t nn = (size_t)n * n, nnx = (size_t)n * d.nx, nrn = (size_t)d.nr * n;
  cudaMemsetAsync(s.st, 0, sizeof(StatusWords), st);
  // blocks not touched by the first level: the unpaired tail and C_nblock
  if (nb % 2 == 1) {
    const size_t t = (size_t)(nb - 1);
    k_convert_blocks<T><<<1, 256, 0, st>>>(s.D0 + t * nn, w.D + t * nn, nn);
    k_convert_blocks<T><<<1, 256, 0, st>>>(s.E0 + t * nn, w.E + t * nn, nn);
    if (nnx) k_convert_blocks<T><<<1, 256, 0, st>>>(s.B0 + t * nnx, w.B + t * nnx, nnx);
    if (nrn) k_convert_blocks<T><<<1, 256, 0, st>>>(s.C0 + t * nrn, w.C + t * nrn, nrn);
  }
  if (nrn) k_convert_blocks<T><<<1, 256, 0, st>>>(s.C0 + (size_t)nb * nrn, w.C + (size_t)nb * nrn, nrn);
  FactorArgs<T> a;
  a.d = d;
  a.D0 = s.D0; a.E0 = s.E0; a.B0 = s.B0; a.C0 = s.C0;
  a.D = w.D; a.E = w.E; a.B = w.B; a.C = w.C;
  a.Tm = w.Tm; a.P = s.P; a.Rbuf = w.Rbuf; a.Fbuf = s.Fbuf; a.st = s.st;
  a.ldw = odd_ld(2 * n + d.nr);
  a.x = x; a.ldx = ldx; a.nrf = nrf; a.XB = s.XB;
  a.qb = a.qe = 0;
  if constexpr (sizeof(T) == 8) {
    if (p.tree || p.tcb) {
      a.F0 = s.F0;
      TreeArgs ta;
      ta.cnt = s.tree_cnt;
      ta.leaf = s.tree_cnt + nb;
      ta.Ffin = s.Ffin;
      ta.xb = (nrf > 0 && d.nr > 0) ? x + (size_t)(nb + 1) * n + d.qr : nullptr;
      if (p.tree) {
        cudaMemsetAsync(s.tree_cnt, 0, (size_t)(nb + 1) * sizeof(int), st);
        const long leaves = pairs_at_level(nb, 1);
        p.tree<<<grid_for(leaves, 4, p.tree_ctas), 128, p.tc_smem, st>>>(a, ta);
        check_launch("k_factor_tree_tc");
        return true;
      }
      int root = 1;
      for (int k = 1; k < nb; k *= 2) {
        a.k = k;
        a.first = (k == 1);
        root = k;  // the pair (0, k) of the top level
        // level 1 has no gathers and no children: the plain instantiation
        (k == 1 ? p.tc : p.tcb)<<<grid_for(pairs_at_level(nb, k), 4, 148 * 16), 128, p.tc_smem, st>>>(
            a, nullptr, nullptr);
        check_launch("k_factor_lu_tc");
      }
      p.root<<<1, 32, 0, st>>>(a, ta, root);
      check_launch("k_tree_root");
      return true;
    }
  }
  for (int k = 1; k < nb; k *= 2) {
    a.k = k;
    a.first = (k == 1);
    const long np = pairs_at_level(nb, k);
    if constexpr (sizeof(T) == 8) {
      if (p.tc && p.top && np <= TOP_WARPS) {  // this level and every one above it
        p.top<<<1, TOP_WARPS * 32, tc_smem_per_warp(n) * TOP_WARPS, st>>>(a, k);
        check_launch("k_factor_top_tc");
        break;
      }
    }
    if (p.umma) p.umma<<<grid_for(np, 1, 148), UM_NT, p.umma_smem, st>>>(a, w.slab, s.slab_elems);
    else if (p.blk) p.blk<<<grid_for(np, 1, s.slab_ctas), 256, p.blk_smem, st>>>(a, w.slab, s.slab_elems);
    else if (p.cta) p.cta<<<grid_for(np, 1, s.slab_ctas), 256, 0, st>>>(a, w.slab, s.slab_elems);
    else if (p.grp) p.grp<<<grid_for(np, 1, p.grp_ctas), p.grp_threads, p.grp_smem, st>>>(a, nullptr, nullptr);
    else if (p.tc) p.tc<<<grid_for(np, 4, 148 * 16), 128, p.tc_smem, st>>>(a, nullptr, nullptr);
    else if (p.rows) p.rows<<<grid_for(np, 4, 148 * 16), 128, 0, st>>>(a, nullptr, nullptr);
    else p.smem_k<<<grid_for(np, p.wpb, 148 * 16), p.wpb * 32, p.smem, st>>>(a, nullptr, nullptr);
    check_launch("k_factor_level");
    if (nrn) {
      const long tot = np * (long)nrn;
      k_border_fix<T><<<grid_for(tot, 256, 148 * 8), 256, 0, st>>>(d, w.C, w.Rbuf, k);
      check_launch("k_border_fix");
    }
  }
  return false;
}

// F = F0 + sum of the Schur updates (FP64); assemble and factor the last block (FP64)
template <typename T>
static void factor_last(DevState& s, const WorkSet<T>& w, cudaStream_t st, bool f_done = false) {
  const Dims d = s.d;
  const int nrnx = d.nr * d.nx;
  if (nrnx > 0 && !f_done)
    reduce_blocks(s, s.Fbuf, 1, d.nblock - 1, nrnx, d.nr, s.F0, d.nr, s.Ffin, d.nr, st);
  k_last_assemble<T><<<grid_for((long)d.Nr * d.Nc, 256, 64), 256, 0, st>>>(
      d, w.D, w.E, w.B, w.C, s.H, s.Cq, s.Ffin, s.Hl);
  check_launch("k_last_assemble");
  if (s.sel_last2) {  // a copy of the assembled block for the fallback solver
    cudaMemcpyAsync(s.Al, s.Hl, (size_t)d.Nr * d.Nc * 8, cudaMemcpyDeviceToDevice, st);
  }
  const LastBufs lb = last_bufs(s);
  if (s.sel_last == LAST_LU && d.Nr == d.Nc && d.Nc >= LAST_BLOCKED_MIN && d.Nc <= BLK_ROWS_MAX) {
    const size_t sm = (size_t)BLK_W * d.Nc * sizeof(double);
    smem_limit_once(k_last_lu_blocked, sm);
    k_last_lu_blocked<<<1, 256, sm, st>>>(d, lb, s.st);
    check_launch("k_last_lu_blocked");
  } else if (s.sel_last == LAST_LU && d.Nr == d.Nc && d.Nc <= LAST_SMALL) {
    k_last_lu_small<<<1, 256, 0, st>>>(d, lb, s.st);
    check_launch("k_last_lu_small");
  } else {
    k_last_factor<double><<<1, 512, 0, st>>>(d, lb, s.sel_last, s.st);
    check_launch("k_last_factor");
  }
  if (s.sel_last2) {
    k_last_fallback<<<1, 512, 0, st>>>(d, lb, s.st);
    check_launch("k_last_fallback");
  }
}

template <typename T>
static void factorize_t(DevState& s, cudaStream_t st) {
  T* tag = nullptr;
  const WorkSet<T> w = work_set(s, tag);
  const FactorPlan<T> p = plan_factor<T>(s);
  const bool tree = factor_levels(s, p, w, nullptr, 0, 0, st);
  factor_last(s, w, st, tree);
}

void launch_factorize(DevState& s, cudaStream_t st) {
  if (s.mixed) factorize_t<float>(s, st);
  else factorize_t<double>(s, st);
}

// sweep kernels for one chunk of right-hand sides
template <typename T>
struct SweepPlan {
  void (*fwd)(SweepArgs<T>, const SweepArgs<T>*, const BatchCta*, const long*) = nullptr;
  void (*bwd)(SweepArgs<T>, const SweepArgs<T>*, const BatchCta*, const long*) = nullptr;
  // n = 8, 16 single systems: pipelined forward (LU) and backward levels,
  // the backward top in one CTA
  void (*fwd_pipe)(SweepArgs<T>, const SweepArgs<T>*, const BatchCta*, const long*, long) = nullptr;
  size_t fwd_pipe_smem = 0;
  void (*bwd_pipe)(SweepArgs<T>, const SweepArgs<T>*, const BatchCta*, const long*, long) = nullptr;
  size_t bwd_pipe_smem = 0;
  void (*bwd_top)(SweepArgs<T>, int, int) = nullptr;
  void (*fwd_cta)(SweepArgs<T>, const SweepArgs<T>*, const BatchCta*) = nullptr;  // CTA per pair (large n)
  void (*bwd_cta)(SweepArgs<T>, const SweepArgs<T>*, const BatchCta*) = nullptr;
};

template <typename T>
static SweepPlan<T> plan_sweeps(const DevState& s) {
  const Dims d = s.d;
  const int n = d.n;
  SweepPlan<T> p;
  if (d.nr <= 8 && d.nx <= 8 && n <= 16) {
    const bool lu = s.sel == SEL_LU, r4 = d.nr <= 4, x4 = d.nx <= 4;
#define BCR_FWD(NN) (r4 ? (lu ? k_forward_rows<T, NN, 4, true> : k_forward_rows<T, NN, 4, false>) \
                        : (lu ? k_forward_rows<T, NN, 8, true> : k_forward_rows<T, NN, 8, false>))
#define BCR_BWD(NN) (x4 ? k_backward_rows<T, NN, 4> : k_backward_rows<T, NN, 8>)
    if (n <= 4) { p.fwd = BCR_FWD(4); p.bwd = BCR_BWD(4); }
    else if (n <= 8) { p.fwd = BCR_FWD(8); p.bwd = BCR_BWD(8); }
    else { p.fwd = BCR_FWD(16); p.bwd = BCR_BWD(16); }
#undef BCR_FWD
#undef BCR_BWD
  }
  if ((n == 16 || n == 8) && s.sel == SEL_LU && d.nr <= 8) {  // both precisions
    const bool r4 = d.nr <= 4;
    if (n == 16) {
      p.fwd_pipe = r4 ? k_forward_pipe<16, 4, T> : k_forward_pipe<16, 8, T>;
      p.fwd_pipe_smem = 8 * (r4 ? FwdBuf<16, 4, T>::BYTES : FwdBuf<16, 8, T>::BYTES);
    } else {
      p.fwd_pipe = r4 ? k_forward_pipe<8, 4, T> : k_forward_pipe<8, 8, T>;
      p.fwd_pipe_smem = 8 * (r4 ? FwdBuf<8, 4, T>::BYTES : FwdBuf<8, 8, T>::BYTES);
    }
    smem_limit_once(p.fwd_pipe, p.fwd_pipe_smem);
  }
  if ((n == 16 || n == 8) && d.nx <= 8) {  // both precisions
    const bool x4 = d.nx <= 4;
    if (n == 16) {
      p.bwd_pipe = x4 ? k_backward_pipe<16, 4, T> : k_backward_pipe<16, 8, T>;
      p.bwd_pipe_smem = 8 * (x4 ? BwdBuf<16, 4, T>::BYTES : BwdBuf<16, 8, T>::BYTES);
      p.bwd_top = x4 ? k_backward_top<16, 4, T> : k_backward_top<16, 8, T>;
    } else {
      p.bwd_pipe = x4 ? k_backward_pipe<8, 4, T> : k_backward_pipe<8, 8, T>;
      p.bwd_pipe_smem = 8 * (x4 ? BwdBuf<8, 4, T>::BYTES : BwdBuf<8, 8, T>::BYTES);
      p.bwd_top = x4 ? k_backward_top<8, 4, T> : k_backward_top<8, 8, T>;
    }
    smem_limit_once(p.bwd_pipe, p.bwd_pipe_smem);
  }
  if (n == 32) {
    if (s.sel == SEL_LU && d.nr <= 8) p.fwd = d.nr <= 4 ? k_forward_rows32<T, 4> : k_forward_rows32<T, 8>;
    if (d.nx <= 8) p.bwd = d.nx <= 4 ? k_backward_rows32<T, 4> : k_backward_rows32<T, 8>;
  } else if (n > 16 && n <= SWP_MAXN) {
    if (s.sel == SEL_LU) p.fwd_cta = k_forward_cta<T>;
    p.bwd_cta = k_backward_cta<T>;
  }
  return p;
}

template <typename T>
static SweepArgs<T> sweep_args(DevState& s, const WorkSet<T>& w, double* x, int ldx, int nrhs) {
  SweepArgs<T> a;
  a.d = s.d;
  a.D = w.D; a.E = w.E; a.B = w.B; a.C = w.C; a.Tm = w.Tm; a.P = s.P;
  a.x = x; a.ldx = ldx; a.nrhs = nrhs; a.XB = s.XB; a.sel = s.sel;
  a.done = nullptr;
  return a;
}

static int top_level(int nb) {
  int K = 1;
  while (K < nb) K *= 2;
  return K;
}

// xb += sum of the per-block -C'_j x_j contributions
static void reduce_xb(DevState& s, double* x, int ldx, int nrhs, cudaStream_t st) {
  const Dims d = s.d;
  if (d.nr > 0) {
    double* xb = x + (size_t)(d.nblock + 1) * d.n + d.qr;
    reduce_blocks(s, s.XB, 1, d.nblock - 1, d.nr * nrhs, d.nr, xb, ldx, xb, ldx, st);
  }
}

template <typename T>
static void forward_levels(DevState& s, const SweepPlan<T>& p, const WorkSet<T>& w, double* x, int ldx,
                           int nrhs, cudaStream_t st) {
  const Dims d = s.d;
  SweepArgs<T> a = sweep_args(s, w, x, ldx, nrhs);
  a.ldw = odd_ld(2 * d.n);
  const size_t smem_f = (size_t)a.ldw * nrhs * 8 * WARPS_PANEL;
  smem_limit_once(k_forward_level<T>, smem_f);
  for (int K = 1; K < d.nblock; K *= 2) {
    a.k = K;
    const long np = pairs_at_level(d.nblock, K);
    if (p.fwd_pipe)
      p.fwd_pipe<<<grid_for(np, 8, 148 * 2), 256, p.fwd_pipe_smem, st>>>(a, nullptr, nullptr, nullptr, 0);
    else if (p.fwd_cta) p.fwd_cta<<<grid_for(np, 1, 148 * 8), 256, 0, st>>>(a, nullptr, nullptr);
    else if (p.fwd) p.fwd<<<grid_for(np, 8, 148 * 32), 256, 0, st>>>(a, nullptr, nullptr, nullptr);
    else k_forward_level<T><<<grid_for(np, WARPS_PANEL, 148 * 16), WARPS_PANEL * 32, smem_f, st>>>(a, nullptr, nullptr, nullptr);
    check_launch("k_forward_level");
  }
  reduce_xb(s, x, ldx, nrhs, st);
}

template <typename T>
static void last_and_backward(DevState& s, const SweepPlan<T>& p, const WorkSet<T>& w, double* x, int ldx,
                              int nrhs, cudaStream_t st) {
  const Dims d = s.d;
  const size_t smem_l = 2 * (size_t)(d.Nr > d.Nc ? d.Nr : d.Nc) * 8;
  k_last_solve<double><<<1, 256, smem_l, st>>>(d, last_bufs(s), s.st, x, ldx, nrhs);
  check_launch("k_last_solve");
  SweepArgs<T> a = sweep_args(s, w, x, ldx, nrhs);
  a.ldw = d.n;
  const size_t smem_b = (size_t)d.n * 8 * WARPS_PANEL;
  if (p.bwd_pipe) {
    // the levels with at most 16 pairs (the top) in one CTA, then one
    // pipelined launch per level below
    int k = top_level(d.nblock) / 2, k_split = 0;
    for (int kk = k; kk > 0; kk /= 2)
      if (pairs_at_level(d.nblock, kk) > 16) { k_split = kk; break; }
    if (k > k_split) {
      p.bwd_top<<<1, 512, 0, st>>>(a, k, k_split * 2 > 0 ? k_split * 2 : 1);
      check_launch("k_backward_top");
    }
    for (int kk = k_split; kk > 0; kk /= 2) {
      a.k = kk;
      const long np = pairs_at_level(d.nblock, kk);
      p.bwd_pipe<<<grid_for(np, 8, 148 * 2), 256, p.bwd_pipe_smem, st>>>(a, nullptr, nullptr, nullptr, 0);
      check_launch("k_backward_pipe");
    }
    return;
  }
  for (int k = top_level(d.nblock); (k /= 2) > 0;) {
    a.k = k;
    const long np = pairs_at_level(d.nblock, k);
    if (p.bwd_cta) p.bwd_cta<<<grid_for(np, 1, 148 * 8), 256, 0, st>>>(a, nullptr, nullptr);
    else if (p.bwd) p.bwd<<<grid_for(np, 8, 148 * 32), 256, 0, st>>>(a, nullptr, nullptr, nullptr);
    else k_backward_level<T><<<grid_for(np, WARPS_PANEL, 148 * 16), WARPS_PANEL * 32, smem_b, st>>>(a, nullptr, nullptr, nullptr);
    check_launch("k_backward_level");
  }
}

// right-hand sides are independent: sweep them in chunks of at most 16 columns
template <typename T>
static void solve_t(DevState& s, double* x, int ldx, int nrhs, cudaStream_t st) {
  T* tag = nullptr;
  const WorkSet<T> w = work_set(s, tag);
  const SweepPlan<T> p = plan_sweeps<T>(s);
  for (int c0 = 0; c0 < nrhs; c0 += 16) {
    const int nc = nrhs - c0 < 16 ? nrhs - c0 : 16;
    double* xc = x + (size_t)c0 * ldx;
    forward_levels(s, p, w, xc, ldx, nc, st);
    last_and_backward(s, p, w, xc, ldx, nc, st);
  }
}

void launch_solve(DevState& s, double* x, int ldx, int nrhs, cudaStream_t st) {
  if (s.mixed) solve_t<float>(s, x, ldx, nrhs, st);
  else solve_t<double>(s, x, ldx, nrhs, st);
}

// factorize and solve in one pass: when the pair kernel can carry the right-
// hand sides, their forward elimination rides in the factorization's GEMM and
// the separate forward sweep disappears
template <typename T>
static void factorize_solve_t(DevState& s, double* x, int ldx, int nrhs, cudaStream_t st) {
  T* tag = nullptr;
  const WorkSet<T> w = work_set(s, tag);
  const FactorPlan<T> fp = plan_factor<T>(s);
  const int nrf = fusable_rhs(s, fp, nrhs);
  if (nrf == 0) {
    launch_factorize(s, st);
    launch_solve(s, x, ldx, nrhs, st);
    return;
  }
  const bool tree = factor_levels(s, fp, w, x, ldx, nrf, st);
  if (!tree) reduce_xb(s, x, ldx, nrf, st);
  factor_last(s, w, st, tree);
  last_and_backward(s, plan_sweeps<T>(s), w, x, ldx, nrf, st);
}

void launch_factorize_solve(DevState& s, double* x, int ldx, int nrhs, cudaStream_t st) {
  // FP32 factors (mixed path): the right-hand sides are eliminated in FP32,
  // which is the accuracy of the solve with those factors anyway; the caller
  // refines the result
  if (s.mixed) factorize_solve_t<float>(s, x, ldx, nrhs, st);
  else factorize_solve_t<double>(s, x, ldx, nrhs, st);
}

// Factorize + solve with the matrix uploaded from host memory in chunks of
// 2^m consecutive blocks on the copy stream cst, each chunk's own CR levels
// (the pairs lying inside it) launched on st as soon as it has arrived: the
// tc pair kernels with the tree's border bookkeeping write nothing outside a
// chunk but their own Rbuf/Fbuf/XB slots, so chunks need no fix-up and the
// upload overlaps the factorization.  The levels spanning chunks, the root,
// the last block and the backward sweep follow.  Returns false (nothing
// enqueued) when the shape does not take this path.
bool launch_upload_factorize_solve(DevState& s, const HostMatrix& hm, double* x, int ldx, int nrhs,
                                   cudaStream_t st, cudaStream_t cst, cudaEvent_t* ev, int nev) {
  if (s.mixed || !s.tree_cnt) return false;
  const Dims d = s.d;
  const int n = d.n, nb = d.nblock;
  if (nb < 2048 || nev < 2) return false;
  PairKernel saved = (PairKernel)s.pair_kernel;
  if (saved != PAIR_AUTO && saved != PAIR_TC_GATHER) return false;
  s.pair_kernel = PAIR_TC_GATHER;
  const FactorPlan<double> p = plan_factor<double>(s);
  s.pair_kernel = saved;
  if (!p.tc || !p.tcb || !p.root) return false;
  const int nrf = fusable_rhs(s, p, nrhs);
  if (nrf != nrhs) return false;
  // chunks: a power of two of blocks, at most nev of them
  int chunk = 1024;
  while ((long)chunk * nev < nb) chunk *= 2;
  const int nchunks = (nb + chunk - 1) / chunk;
  double* tag = nullptr;
  const WorkSet<double> w = work_set(s, tag);
  const size_t nn = (size_t)n * n, nnx = (size_t)n * d.nx, nrn = (size_t)d.nr * n;
  // the small arrays first, then the chunks
  auto up = [&](double* dst, const double* src, size_t cnt) {
    if (cnt) cudaMemcpyAsync(dst, src, cnt * 8, cudaMemcpyHostToDevice, cst);
  };
  up(s.Cq, hm.Cq, (size_t)d.nr * d.qx);
  up(s.F0, hm.F, (size_t)d.nr * d.nx);
  up(s.H, hm.H, (size_t)(n + d.qr) * d.Nc);
  FactorArgs<double> a;
  a.d = d;
  a.D0 = s.D0; a.E0 = s.E0; a.B0 = s.B0; a.C0 = s.C0;
  a.D = w.D; a.E = w.E; a.B = w.B; a.C = w.C;
  a.Tm = w.Tm; a.P = s.P; a.Rbuf = w.Rbuf; a.Fbuf = s.Fbuf; a.st = s.st;
  a.ldw = odd_ld(2 * n + d.nr);
  a.x = x; a.ldx = ldx; a.nrf = nrf; a.XB = s.XB;
  a.F0 = s.F0;
  cudaMemsetAsync(s.st, 0, sizeof(StatusWords), st);
  for (int c = 0; c < nchunks; ++c) {
    const long b0 = (long)c * chunk, b1 = std::min<long>(b0 + chunk, nb);
    up(s.D0 + b0 * nn, hm.D + b0 * nn, (size_t)(b1 - b0) * nn);
    up(s.E0 + b0 * nn, hm.E + b0 * nn, (size_t)(b1 - b0) * nn);
    up(s.B0 + b0 * nnx, hm.B + b0 * nnx, (size_t)(b1 - b0) * nnx);
    const long c1 = c == nchunks - 1 ? nb + 1 : b1;  // the last chunk also brings C_nblock
    up(s.C0 + b0 * nrn, hm.C + b0 * nrn, (size_t)(c1 - b0) * nrn);
    cudaEventRecord(ev[c % nev], cst);
    cudaStreamWaitEvent(st, ev[c % nev], 0);
    if (c == nchunks - 1) {  // blocks no pair of the first level touches: the odd tail and C_nblock
      if (nb % 2 == 1) {
        const size_t t = (size_t)(nb - 1);
        k_convert_blocks<double><<<1, 256, 0, st>>>(s.D0 + t * nn, w.D + t * nn, nn);
        k_convert_blocks<double><<<1, 256, 0, st>>>(s.E0 + t * nn, w.E + t * nn, nn);
        if (nnx) k_convert_blocks<double><<<1, 256, 0, st>>>(s.B0 + t * nnx, w.B + t * nnx, nnx);
        if (nrn) k_convert_blocks<double><<<1, 256, 0, st>>>(s.C0 + t * nrn, w.C + t * nrn, nrn);
      }
      if (nrn) k_convert_blocks<double><<<1, 256, 0, st>>>(s.C0 + (size_t)nb * nrn, w.C + (size_t)nb * nrn, nrn);
    }
    // the levels whose pairs lie inside [b0, b1): j = k (2q + 1) with b0 < j < b1
    for (int k = 1; k < chunk; k *= 2) {
      const long qb = b0 / (2L * k), np = pairs_at_level(nb, k);
      const long qe = std::min<long>(np, (b1 + k - 1) / (2L * k));  // j < b1
      if (qe <= qb) continue;
      a.k = k;
      a.first = k == 1;
      a.qb = qb;
      a.qe = qe;
      (k == 1 ? p.tc : p.tcb)<<<grid_for(qe - qb, 4, 148 * 16), 128, p.tc_smem, st>>>(a, nullptr, nullptr);
      check_launch("k_factor_lu_tc (chunk)");
    }
  }
  a.qb = a.qe = 0;
  TreeArgs ta;
  ta.cnt = s.tree_cnt;
  ta.leaf = s.tree_cnt + nb;
  ta.Ffin = s.Ffin;
  ta.xb = (nrf > 0 && d.nr > 0) ? x + (size_t)(nb + 1) * n + d.qr : nullptr;
  int root = 1;
  for (int k = 1; k < nb; k *= 2) {
    root = k;
    if (k < chunk) continue;
    a.k = k;
    a.first = 0;
    p.tcb<<<grid_for(pairs_at_level(nb, k), 4, 148 * 16), 128, p.tc_smem, st>>>(a, nullptr, nullptr);
    check_launch("k_factor_lu_tc");
  }
  p.root<<<1, 32, 0, st>>>(a, ta, root);
  check_launch("k_tree_root");
  factor_last(s, w, st, true);
  last_and_backward(s, plan_sweeps<double>(s), w, x, ldx, nrf, st);
  return true;
}

bool factorize_solve_fuses(const DevState& s, int nrhs) {
  if (s.mixed) return false;
  return fusable_rhs(s, plan_factor<double>(s), nrhs) == nrhs;
}

// rowsum (value pass only): the block rows' |A| * 1 from the same reads;
// skip_rows (ABS pass only): the block rows are already done
template <bool ABS>
static void mv_t(DevState& s, double alpha, const double* x, double beta, double* res, cudaStream_t st,
                 double* rowsum = nullptr, bool skip_rows = false) {
  const Dims d = s.d;
  const long rows = (long)d.nblock * d.n;
  if (rows > 0 && !skip_rows) {
    k_mv_rows<ABS><<<grid_for(rows, 256, 148 * 8), 256, 0, st>>>(d, s.D0, s.E0, s.B0, alpha, x, beta, res,
                                                                  rowsum);
    check_launch("k_mv_rows");
  }
  const int nr = d.nr;
  double* Csum = s.Ffin;  // unused when nr == 0
  if (nr > 0) {
    const long tot = (long)(d.nblock + 1) * nr;
    k_mv_cpart<ABS><<<grid_for(tot, 256, 148 * 8), 256, 0, st>>>(d, s.C0, x, s.mv_part);
    check_launch("k_mv_cpart");
    Csum = s.mv_part + (size_t)(d.nblock + 1) * nr;
    reduce_blocks(s, s.mv_part, 0, d.nblock + 1, nr, nr, nullptr, nr, Csum, nr, st);
  }
  k_mv_tail<ABS><<<1, 256, 0, st>>>(d, s.H, s.Cq, s.F0, Csum, alpha, x, beta, res);
  check_launch("k_mv_tail");
}

void launch_mv(DevState& s, double alpha, const double* x, double beta, double* res, cudaStream_t st) {
  mv_t<false>(s, alpha, x, beta, res, st);
}

// out[slot] = max |v_i| over i < len (exact, order independent)
__global__ void k_absmax(const double* v, long len, unsigned long long* out) {
  double m = 0.0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (long)gridDim.x * blockDim.x)
    m = fmax(m, fabs(v[i]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

__global__ void k_axpy(double* y, const double* x, long len) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (long)gridDim.x * blockDim.x)
    y[i] += x[i];
}

// r = b - A x and the three inf-norms |r|, |x|, |b| into out[0..2]; with rowsum
// (an nrows-long scratch) non-null, also ||A||_inf into *normA, the block rows'
// |A| sums taken from the residual's own reads of the matrix
void launch_residual(DevState& s, const double* b, const double* x, double* r, unsigned long long* out,
                     cudaStream_t st, double* rowsum, unsigned long long* normA) {
  const Dims d = s.d;
  const long nrows = (long)d.n * (d.nblock + 1) + d.qr + d.nr;
  const long ncols = (long)d.n * (d.nblock + 1) + d.qx + d.nx;
  cudaMemcpyAsync(r, b, (size_t)nrows * 8, cudaMemcpyDeviceToDevice, st);
  mv_t<false>(s, -1.0, x, 1.0, r, st, rowsum);
  if (rowsum) {
    mv_t<true>(s, 1.0, nullptr, 0.0, rowsum, st, nullptr, true);  // border and last rows
    cudaMemsetAsync(normA, 0, sizeof(unsigned long long), st);
    k_absmax<<<grid_for(nrows, 256, 148 * 2), 256, 0, st>>>(rowsum, nrows, normA);
  }
  cudaMemsetAsync(out, 0, 3 * sizeof(unsigned long long), st);
  k_absmax<<<grid_for(nrows, 256, 148 * 2), 256, 0, st>>>(r, nrows, out);
  k_absmax<<<grid_for(ncols, 256, 148 * 2), 256, 0, st>>>(x, ncols, out + 1);
  k_absmax<<<grid_for(nrows, 256, 148 * 2), 256, 0, st>>>(b, nrows, out + 2);
  check_launch("k_absmax");
}

void launch_axpy(double* y, const double* x, long len, cudaStream_t st) {
  k_axpy<<<grid_for(len, 256, 148 * 4), 256, 0, st>>>(y, x, len);
  check_launch("k_axpy");
}

// ---------------------------------------------------------------------------
// batches of independent systems (FP64, internal LU)
// ---------------------------------------------------------------------------
struct LastDesc {
  Dims d;
  const double *D0, *E0, *B0, *C0, *H, *Cq, *F0, *Fbuf, *XB;
  void *Dw, *Ew, *Bw, *Cw;  // working blocks: FP64, or FP32 on the mixed path
  double *Ffin, *Hl, *tau, *x;
  int* piv;
  int kind, ldx;
  StatusWords* st;
  LastBufs lb;
  const int* done;  // mixed path: the system's refinement converged (skip its solve)
};

// status reset and the blocks the first level does not touch (odd tail, C_N)
template <typename T>
__global__ void __launch_bounds__(256) kb_begin(const LastDesc* t) {
  const LastDesc& L = t[blockIdx.x];
  const Dims d = L.d;
  const int nb = d.nblock;
  const size_t nn = (size_t)d.n * d.n, nnx = (size_t)d.n * d.nx, nrn = (size_t)d.nr * d.n;
  T* D = static_cast<T*>(L.Dw);
  T* E = static_cast<T*>(L.Ew);
  T* B = static_cast<T*>(L.Bw);
  T* C = static_cast<T*>(L.Cw);
  if (threadIdx.x == 0) *L.st = StatusWords{0, 0, 0, 0, 0};
  if (nb % 2 == 1) {
    const size_t b = (size_t)(nb - 1);
    for (size_t e = threadIdx.x; e < nn; e += blockDim.x) {
      D[b * nn + e] = T(L.D0[b * nn + e]);
      E[b * nn + e] = T(L.E0[b * nn + e]);
    }
    for (size_t e = threadIdx.x; e < nnx; e += blockDim.x) B[b * nnx + e] = T(L.B0[b * nnx + e]);
    for (size_t e = threadIdx.x; e < nrn; e += blockDim.x) C[b * nrn + e] = T(L.C0[b * nrn + e]);
  }
  for (size_t e = threadIdx.x; e < nrn; e += blockDim.x) C[(size_t)nb * nrn + e] = T(L.C0[(size_t)nb * nrn + e]);
}

// C_jpp += dC_jpp for the pairs of each chunk (one writer per target block)
template <typename T>
__global__ void __launch_bounds__(128) kb_border_fix(const FactorArgs<T>* tab, const BatchCta* cmap, int k) {
  const BatchCta c = cmap[blockIdx.x];
  const FactorArgs<T>& a = tab[c.sys];
  const Dims d = a.d;
  const size_t nrn = (size_t)d.nr * d.n;
  for (long q = c.q0; q < c.q1; ++q) {
    const int j = k + (int)(2L * k * q), jpp = min(j + k, d.nblock);
    for (size_t e = threadIdx.x; e < nrn; e += blockDim.x) a.C[(size_t)jpp * nrn + e] += a.Rbuf[(size_t)j * nrn + e];
  }
}

// ---------------------------------------------------------------------------
// Persistent batch factorization: one launch per class works through the
// (system, level, pair range) items of every level, in level order, with a
// per-system level schedule.  A CTA takes the next item from a counter and
// waits (bounded) until that system's previous level is complete; systems
// advance independently, so a deep system does not hold up shallow ones and
// no level ever waits for the whole batch.  The worker that finishes the last
// item of a (system, level) applies that level's C_jpp updates (the work of
// kb_border_fix) and then publishes the level.  Items are taken in level order,
// so every item an item waits for was taken earlier by a running CTA: the
// waits always end.  A wait that exceeds its limit (about a second) reports
// DEV_TIMEOUT for the system and skips the item's pairs.
// ---------------------------------------------------------------------------
struct BatchQueue {
  int* next;         // next item (zero at launch)
  int* done_pairs;   // per system: pairs finished, cumulative over levels
  int* level_done;   // per system: levels published (border fix-up included)
  long items;
};

// pairs of levels 0..L of a system of nb blocks
__device__ __forceinline__ long pairs_through_level(int nb, int L) {
  long s = 0;
  for (int l = 0; l <= L; ++l) s += pairs_at_level(nb, 1 << l);
  return s;
}

// CTA-wide: the next item; false when the queue is empty
template <typename T>
__device__ bool queue_next(const BatchQueue& qu, const BatchCta* items, const FactorArgs<T>* tab,
                           FactorArgs<T>& a, BatchCta& c, bool& ok) {
  __shared__ long s_it;
  __shared__ int s_ok;
  __syncthreads();  // the previous item's readers of s_it / s_ok are done
  if (threadIdx.x == 0) {
    const long it = atomicAdd(qu.next, 1);
    int good = 1;
    if (it < qu.items) {
      const BatchCta ci = items[it];
      if (ci.pad > 0) {
        const volatile int* flag = qu.level_done + ci.sys;
        unsigned spins = 0;
        while (*flag < ci.pad) {
          if (++spins > (1u << 23)) { good = 0; break; }
          __nanosleep(100);
        }
        __threadfence();
      }
    }
    s_it = it;
    s_ok = good;
  }
  __syncthreads();
  const long it = s_it;
  if (it >= qu.items) return false;
  __threadfence();  // acquire: the system's previous level is visible to every thread
  c = items[it];
  ok = s_ok != 0;
  a = tab[c.sys];
  a.k = 1 << c.pad;
  a.first = c.pad == 0;
  if (!ok && threadIdx.x == 0) report(a.st, DEV_TIMEOUT, -1, 0, a.k);
  return true;
}

// CTA-wide: count the item's pairs; the CTA completing the (system, level)
// applies the level's C_jpp updates and publishes the level
// the C_jpp updates of every pair of (system, level): C_jpp += Rbuf[j], four
// elements per thread and round with their loads in flight together
template <typename T>
__device__ void level_fixup(const FactorArgs<T>& a, const BatchCta& c, int tid, int nthr) {
  const Dims d = a.d;
  const int k = 1 << c.pad;
  const size_t nrn = (size_t)d.nr * d.n;
  const long np = pairs_at_level(d.nblock, k);
  const size_t tot = (size_t)np * nrn;
  for (size_t e0 = tid; e0 < tot; e0 += 4 * (size_t)nthr) {
    size_t oc[4];
    T cv[4], rv[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const size_t e = e0 + u * (size_t)nthr;
      oc[u] = 0;
      cv[u] = rv[u] = T(0);
      if (e < tot) {
        const long q = (long)(e / nrn);
        const size_t idx = e % nrn;
        const int j = k + (int)(2L * k * q), jpp = min(j + k, d.nblock);
        oc[u] = (size_t)jpp * nrn + idx;
        cv[u] = __ldcg(a.C + oc[u]);
        rv[u] = __ldcg(a.Rbuf + (size_t)j * nrn + idx);
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (e0 + u * (size_t)nthr < tot) a.C[oc[u]] = cv[u] + rv[u];
  }
}

// CTA-wide: count the item's pairs; the CTA completing the (system, level)
// applies the level's C_jpp updates and publishes the level
template <typename T>
__device__ void queue_done(const BatchQueue& qu, const FactorArgs<T>& a, const BatchCta& c) {
  __shared__ int s_last;
  __threadfence();  // release: this thread's results of the item
  __syncthreads();  // every pair of the item is finished
  if (threadIdx.x == 0) {
    __threadfence();
    const long cnt = c.q1 - c.q0;
    const int old = atomicAdd(qu.done_pairs + c.sys, (int)cnt);
    s_last = (long)old + cnt == pairs_through_level(a.d.nblock, c.pad);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  level_fixup<T>(a, c, threadIdx.x, blockDim.x);
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicExch(qu.level_done + c.sys, c.pad + 1);
  }
}

// The same per warp, for the warp-per-pair families: each warp takes, waits
// for and publishes its own items, so no warp ever waits at a CTA barrier for
// another warp's item.
template <typename T>
__device__ bool queue_next_warp(const BatchQueue& qu, const BatchCta* items, const FactorArgs<T>* tab,
                                FactorArgs<T>& a, BatchCta& c, bool& ok) {
  const int lane = threadIdx.x & 31;
  long it = 0;
  int good = 1;
  if (lane == 0) {
    it = atomicAdd(qu.next, 1);
    if (it < qu.items) {
      const BatchCta ci = items[it];
      if (ci.pad > 0) {
        const volatile int* flag = qu.level_done + ci.sys;
        unsigned spins = 0;
        while (*flag < ci.pad) {
          if (++spins > (1u << 23)) { good = 0; break; }
          __nanosleep(100);
        }
        __threadfence();
      }
    }
  }
  it = __shfl_sync(0xffffffffu, it, 0);
  good = __shfl_sync(0xffffffffu, good, 0);
  if (it >= qu.items) return false;
  __threadfence();
  c = items[it];
  ok = good != 0;
  a = tab[c.sys];
  a.k = 1 << c.pad;
  a.first = c.pad == 0;
  if (!ok && lane == 0) report(a.st, DEV_TIMEOUT, -1, 0, a.k);
  return true;
}

template <typename T>
__device__ void queue_done_warp(const BatchQueue& qu, const FactorArgs<T>& a, const BatchCta& c) {
  const int lane = threadIdx.x & 31;
  __threadfence();
  __syncwarp();
  int last = 0;
  if (lane == 0) {
    const long cnt = c.q1 - c.q0;
    const int old = atomicAdd(qu.done_pairs + c.sys, (int)cnt);
    last = (long)old + cnt == pairs_through_level(a.d.nblock, c.pad);
  }
  last = __shfl_sync(0xffffffffu, last, 0);
  if (!last) return;
  __threadfence();
  level_fixup<T>(a, c, lane, 32);
  __threadfence();
  __syncwarp();
  if (lane == 0) atomicExch(qu.level_done + c.sys, c.pad + 1);
}

template <typename T, int N, int NXM, int NRM>
__global__ void __launch_bounds__(128) kp_factor_rows(const FactorArgs<T>* tab, const BatchCta* items, BatchQueue qu) {
  FactorArgs<T> a;
  BatchCta c;
  bool ok;
  while (queue_next_warp(qu, items, tab, a, c, ok)) {
    if (ok) rows_body<T, N, NXM, NRM, true>(a, c.q0, c.q1, 1);
    queue_done_warp(qu, a, c);
  }
}

template <typename T, int N>
__global__ void __launch_bounds__(2 * N + 32, grp_min_blocks<T, N>())
    kp_factor_grp(const FactorArgs<T>* tab, const BatchCta* items, BatchQueue qu) {
  FactorArgs<T> a;
  BatchCta c;
  bool ok;
  while (queue_next(qu, items, tab, a, c, ok)) {
    if (ok) grp_body<T, N, true>(a, c.q0, c.q1, 1);
    queue_done(qu, a, c);
  }
}

template <int N, typename T = double>
__global__ void __launch_bounds__(128, tc_min_blocks<T>())
    kp_factor_tc(const FactorArgs<T>* tab, const BatchCta* items, BatchQueue qu) {
  using S = TcShape<N, T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T* Wt = reinterpret_cast<T*>(smem_raw + (size_t)warp * S::BYTES);
  FactorArgs<T> a;
  BatchCta c;
  bool ok;
  while (queue_next_warp(qu, items, tab, a, c, ok)) {
    const TcTree tr{0, 0, 0};
    if (ok)
      for (long q = c.q0; q < c.q1; ++q)
        tc_pair<N, 8, T>(a, a.k + (int)(2L * a.k * q), a.k, a.first != 0, Wt, lane, tr);
    queue_done_warp(qu, a, c);
  }
}

// F = F0 + sum of the Schur updates, one CTA per system (fixed order)
__global__ void __launch_bounds__(256) kb_reduce_F(const LastDesc* t) {
  const LastDesc& L = t[blockIdx.x];
  const Dims d = L.d;
  const int m = d.nr * d.nx;
  if (m == 0) return;
  const long cnt = d.nblock - 1;
  reduce_tree_body(L.Fbuf, m, 1, cnt, m, cnt > 0 ? cnt : 1, (double*)nullptr, L.F0, d.nr, d.nr, L.Ffin, d.nr, 0);
}

template <typename T>
__global__ void __launch_bounds__(256) kb_last_assemble(const LastDesc* t) {
  const LastDesc& L = t[blockIdx.x];
  last_assemble_range(L.d, static_cast<const T*>(L.Dw), static_cast<const T*>(L.Ew), static_cast<const T*>(L.Bw),
                      static_cast<const T*>(L.Cw), L.H, L.Cq, L.Ffin, L.Hl, (int)threadIdx.x, (int)blockDim.x);
}

__global__ void __launch_bounds__(512) kb_last_factor(const LastDesc* t) {
  const LastDesc& L = t[blockIdx.x];
  if (L.st->code != 0) return;  // a pair of this system already failed
  __syncthreads();
  last_factor_body<double>(L.d, L.lb, L.kind, L.st);
}

// xb += sum of the per-block -C'_j x_j contributions, one CTA per system
__global__ void __launch_bounds__(256) kb_reduce_xb(const LastDesc* t, int nrhs) {
  const LastDesc& L = t[blockIdx.x];
  const Dims d = L.d;
  if (d.nr == 0 || (L.done && *L.done)) return;
  const int m = d.nr * nrhs;
  const long cnt = d.nblock - 1;
  double* xb = L.x + (size_t)(d.nblock + 1) * d.n + d.qr;
  reduce_tree_body(L.XB, m, 1, cnt, m, cnt > 0 ? cnt : 1, (double*)nullptr, (const double*)xb, d.nr, L.ldx, xb,
                   L.ldx, 0);
}

__global__ void __launch_bounds__(256) kb_last_solve(const LastDesc* t, int nrhs) {
  const LastDesc& L = t[blockIdx.x];
  if (L.done && *L.done) return;
  last_solve_body<double>(L.d, L.lb, L.st, L.x, L.ldx, nrhs);
}

// ---------------------------------------------------------------------------
// FP64 residual of the mixed batch path, one CTA per system:
// r = b - A xs with the loaded matrix (add_Mv, cc:2118-2166), written into the
// system's right-hand-side slot, and |r|, |xs|, |b| (and |A|_inf when asked)
// into nrm[1..3] (nrm[0]); the worst |r|/(|A||x|+|b|) of the batch goes to
// *worst (bits of a non-negative double, so an integer max orders them)
// ---------------------------------------------------------------------------
struct ResDesc {
  Dims d;
  const double *D0, *E0, *B0, *C0, *Cq, *F0, *H;
  double* xs;          // the refined solution
  const double* b;
  double *r, *nrm;     // nrm: |A|, |r|, |x|, |b|, |r|/(|A||x|+|b|)
  int* done;
};

__device__ double block_max(double v, double* sv) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) sv[w] = v;
  __syncthreads();
  if (w == 0) {
    v = lane < nw ? sv[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (lane == 0) sv[0] = v;
  }
  __syncthreads();
  return sv[0];
}

// a batch map with its launch shape: one CTA per entry, or a fixed grid over
// a compacted map whose length (ecnt) the device wrote
struct SweepMap {
  const BatchCta* map;
  const long* ecnt;
  unsigned grid;
};

// r = b - (D_k x_k + E_k x_{k+1} + B_k xb) on block rows [k0, k1) of one
// system, written into the rhs slot; the largest |r| and (with_A) the largest
// row sum of |A| over this thread's rows
__device__ __forceinline__ void res_block_rows(const ResDesc& R, long k0, long k1, int with_A, double& mr,
                                               double& ma) {
  const Dims d = R.d;
  const int n = d.n, nx = d.nx;
  const size_t nn = (size_t)n * n, nnx = (size_t)n * nx;
  const size_t xb = (size_t)(d.nblock + 1) * n + d.qx;
  const double* xs = R.xs;
  for (long e = k0 * n + threadIdx.x; e < k1 * n; e += blockDim.x) {
    const size_t k = (size_t)(e / n);
    const int i = (int)(e % n);
    const double* Dk = R.D0 + k * nn;
    const double* Ek = R.E0 + k * nn;
    const double* Bk = R.B0 + k * nnx;
    double s = 0.0, sa = 0.0;
    for (int c = 0; c < n; ++c) {
      s = fma(Dk[(size_t)c * n + i], xs[k * n + c], s);
      s = fma(Ek[(size_t)c * n + i], xs[(k + 1) * n + c], s);
      if (with_A) sa += fabs(Dk[(size_t)c * n + i]) + fabs(Ek[(size_t)c * n + i]);
    }
    for (int c = 0; c < nx; ++c) {
      s = fma(Bk[(size_t)c * n + i], xs[xb + c], s);
      if (with_A) sa += fabs(Bk[(size_t)c * n + i]);
    }
    const double r = R.b[e] - s;
    R.r[e] = r;
    mr = fmax(mr, fabs(r));
    ma = fmax(ma, sa);
  }
}

// non-negative doubles order like their bit patterns
__device__ __forceinline__ void atomic_max_nonneg(double* p, double v) {
  atomicMax(reinterpret_cast<unsigned long long*>(p), (unsigned long long)__double_as_longlong(v));
}

// Block rows covered by the level-1 pairs [q0, q1) of each map entry
// (rows 2 q0 .. 2 q1 - 1), spread over many CTAs: the full sweep map on the
// first residual of a solve, the compacted map of the systems just corrected
// afterwards (ecnt: its length).  The largest |r| and |A| row sum of each
// entry go to nrm[5], nrm[6] of its system.
__global__ void __launch_bounds__(128) kb_residual_rows(const ResDesc* t, const BatchCta* map, const long* ecnt,
                                                        int with_A) {
  __shared__ double sv[32];
  const long cnt = ecnt ? *ecnt : (long)gridDim.x;
  for (long e = blockIdx.x; e < cnt; e += gridDim.x) {
    const BatchCta c = map[e];
    const ResDesc& R = t[c.sys];
    if (*R.done) continue;  // uniform over the CTA
    double mr = 0.0, ma = 0.0;
    res_block_rows(R, 2 * c.q0, 2 * c.q1, with_A, mr, ma);
    mr = block_max(mr, sv);
    ma = block_max(ma, sv);
    if (threadIdx.x == 0) {
      atomic_max_nonneg(R.nrm + 5, mr);
      if (with_A) atomic_max_nonneg(R.nrm + 6, ma);
    }
  }
}

// The rest of the residual, one CTA per system still refining: block rows
// from 2 * (level-1 pairs) on (the odd tail; every row when nblock = 1), the
// boundary rows (H), the border rows (a CTA-wide sum over every block
// column), |x| and |b|; then the norms with kb_residual_rows' maxima,
// |r|/(|A||x|+|b|), the converged flag and the batch-worst figure (bits of a
// non-negative double, so an integer max orders them).  Bit for bit the
// residual of add_Mv (cc:2118-2166) on the loaded FP64 matrix.
__global__ void __launch_bounds__(256, 2) kb_residual(const ResDesc* t, int with_A, double tol,
                                                   unsigned long long* worst) {
  __shared__ double sv[32];
  const ResDesc& R = t[blockIdx.x];
  if (*R.done) {  // converged earlier: its last figure still counts for the batch
    if (threadIdx.x == 0) atomicMax(worst, (unsigned long long)__double_as_longlong(R.nrm[4]));
    return;
  }
  const Dims d = R.d;
  const int n = d.n, nb = d.nblock, nr = d.nr, nx = d.nx, qx = d.qx, m = n + d.qr, Nc = d.Nc;
  const int tid = threadIdx.x, bs = blockDim.x;
  const size_t nrn = (size_t)nr * n;
  const size_t xN = (size_t)nb * n, xq = (size_t)(nb + 1) * n, xb = xq + qx;
  const double* xs = R.xs;
  double mr = 0.0, ma = 0.0;
  res_block_rows(R, 2 * pairs_at_level(nb, 1), nb, with_A, mr, ma);
  // boundary rows (H)
  for (int row = tid; row < m; row += bs) {
    double s = 0.0, sa = 0.0;
    for (int c = 0; c < Nc; ++c) {
      const size_t xi = c < n ? (size_t)c : (c < 2 * n ? xN + (c - n) : xq + (c - 2 * n));
      const double h = R.H[(size_t)c * m + row];
      s = fma(h, xs[xi], s);
      sa += fabs(h);
    }
    const size_t o = xN + row;
    const double r = R.b[o] - s;
    R.r[o] = r;
    mr = fmax(mr, fabs(r));
    ma = fmax(ma, with_A ? sa : 0.0);
  }
  // border rows, four at a time: one walk over every block column
  // accumulates four rows, each row's terms in the same order as a walk of
  // its own; then one CTA reduction per row.  A thread's columns e = tid,
  // tid + bs, ... are loaded RES_U at a time before any is added, so a lone
  // long system (the late refinement passes) pays one load latency per RES_U
  // columns; the additions keep the column order.
  constexpr int RES_U = 4;
  const long tot = (long)(nb + 1) * n;
  const long dk = bs / n;
  const int dc = bs % n;
  for (int r0 = 0; r0 < nr; r0 += 4) {
    double s4[4] = {0.0, 0.0, 0.0, 0.0}, a4[4] = {0.0, 0.0, 0.0, 0.0};
    size_t k = (size_t)(tid / n);  // block and column of element e
    int c = tid % n;
    for (long e0 = tid; e0 < tot; e0 += (long)RES_U * bs) {
      double xv[RES_U], cv[RES_U][4];
#pragma unroll
      for (int u = 0; u < RES_U; ++u) {
        const bool on = e0 + (long)u * bs < tot;
        const double* cp = R.C0 + k * nrn + (size_t)c * nr + r0;
        xv[u] = on ? xs[k * n + c] : 0.0;
#pragma unroll
        for (int i = 0; i < 4; ++i) cv[u][i] = (on && r0 + i < nr) ? cp[i] : 0.0;
        k += dk;
        c += dc;
        if (c >= n) { c -= n; ++k; }
      }
#pragma unroll
      for (int u = 0; u < RES_U; ++u) {
        if (e0 + (long)u * bs >= tot) break;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          if (r0 + i < nr) {
            s4[i] = fma(cv[u][i], xv[u], s4[i]);
            a4[i] += fabs(cv[u][i]);
          }
        }
      }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int rr = r0 + i;
      if (rr >= nr) break;
      double s = s4[i], sa = a4[i];
      for (int c = tid; c < qx; c += bs) { s = fma(R.Cq[(size_t)c * nr + rr], xs[xq + c], s); sa += fabs(R.Cq[(size_t)c * nr + rr]); }
      for (int c = tid; c < nx; c += bs) { s = fma(R.F0[(size_t)c * nr + rr], xs[xb + c], s); sa += fabs(R.F0[(size_t)c * nr + rr]); }
      s = block_sum(s, sv);
      sa = block_sum(sa, sv);
      if (tid == 0) {
        const size_t o = xN + m + rr;
        const double r = R.b[o] - s;
        R.r[o] = r;
        mr = fmax(mr, fabs(r));
        ma = fmax(ma, with_A ? sa : 0.0);
      }
    }
  }
  const long nrows = (long)n * (nb + 1) + d.qr + nr;
  const long ncols = (long)n * (nb + 1) + qx + nx;
  // |x| and |b|: maxima are exact in any order, so eight loads per round
  double mx = 0.0, mb = 0.0;
  for (long e0 = tid; e0 < ncols; e0 += 8L * bs) {
    double v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) v[u] = e0 + (long)u * bs < ncols ? fabs(xs[e0 + (long)u * bs]) : 0.0;
#pragma unroll
    for (int u = 0; u < 8; ++u) mx = fmax(mx, v[u]);
  }
  for (long e0 = tid; e0 < nrows; e0 += 8L * bs) {
    double v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) v[u] = e0 + (long)u * bs < nrows ? fabs(R.b[e0 + (long)u * bs]) : 0.0;
#pragma unroll
    for (int u = 0; u < 8; ++u) mb = fmax(mb, v[u]);
  }
  mr = block_max(mr, sv);
  mx = block_max(mx, sv);
  mb = block_max(mb, sv);
  if (with_A) ma = block_max(ma, sv);
  if (tid == 0) {
    mr = fmax(mr, R.nrm[5]);  // the block rows of kb_residual_rows
    if (with_A) R.nrm[0] = fmax(ma, R.nrm[6]);
    R.nrm[5] = 0.0;           // ready for the next residual
    R.nrm[6] = 0.0;
    R.nrm[1] = mr;
    R.nrm[2] = mx;
    R.nrm[3] = mb;
    const double den = R.nrm[0] * mx + mb;
    double rel = den > 0.0 ? mr / den : (mr > 0.0 ? INFINITY : 0.0);
    if (rel != rel) rel = INFINITY;
    R.nrm[4] = rel;
    if (rel <= tol) *R.done = 1;
    atomicMax(worst, (unsigned long long)__double_as_longlong(rel));
  }
}

// x_sol += d for the systems still refining (d was solved in place of r):
// the x blocks of each map entry's level-1 pairs (2 q0 .. 2 q1 - 1) ...
__global__ void __launch_bounds__(128) kb_correct_rows(const ResDesc* t, const BatchCta* map, const long* ecnt) {
  const long cnt = ecnt ? *ecnt : (long)gridDim.x;
  for (long e = blockIdx.x; e < cnt; e += gridDim.x) {
    const BatchCta c = map[e];
    const ResDesc& R = t[c.sys];
    if (*R.done) continue;
    const long n = R.d.n;
    for (long i = 2 * c.q0 * n + threadIdx.x; i < 2 * c.q1 * n; i += blockDim.x) R.xs[i] += R.r[i];
  }
}

// ... and the rest of x, one CTA per system
__global__ void __launch_bounds__(256) kb_correct(const ResDesc* t) {
  const ResDesc& R = t[blockIdx.x];
  if (*R.done) return;
  const Dims d = R.d;
  const long ncols = (long)d.n * (d.nblock + 1) + d.qx + d.nx;
  for (long i = 2 * pairs_at_level(d.nblock, 1) * d.n + threadIdx.x; i < ncols; i += blockDim.x)
    R.xs[i] += R.r[i];
}

// the level-1 entries of the sweep map: all of them, or the compacted ones
static SweepMap level1_map(const BatchClass& c, bool compact) {
  if (!compact) return {c.smap, nullptr, (unsigned)c.scnt[0]};
  return {c.cmap, c.ccnt, (unsigned)std::min<long>(c.scnt[0], COMPACT_GRID)};
}

void batch_residual(BatchClass& c, int with_A, double tol, unsigned long long* worst, cudaStream_t st,
                    bool compact) {
  if (c.nsys == 0) return;
  compact = compact && c.cmap != nullptr;
  if (c.levels > 0 && c.scnt[0] > 0) {
    const SweepMap m = level1_map(c, compact);
    kb_residual_rows<<<m.grid, 128, 0, st>>>(static_cast<const ResDesc*>(c.rd), m.map, m.ecnt, with_A);
    check_launch("kb_residual_rows");
  }
  kb_residual<<<c.nsys, 256, 0, st>>>(static_cast<const ResDesc*>(c.rd), with_A, tol, worst);
  check_launch("kb_residual");
}

void batch_correct(BatchClass& c, cudaStream_t st) {
  if (c.nsys == 0) return;
  const bool compact = c.cmap != nullptr;
  if (c.levels > 0 && c.scnt[0] > 0) {
    const SweepMap m = level1_map(c, compact);
    kb_correct_rows<<<m.grid, 128, 0, st>>>(static_cast<const ResDesc*>(c.rd), m.map, m.ecnt);
    check_launch("kb_correct_rows");
  }
  kb_correct<<<c.nsys, 256, 0, st>>>(static_cast<const ResDesc*>(c.rd));
  check_launch("kb_correct");
}

bool batch_family_ok(int fam, const Dims& d, bool mixed) {
  if (d.nr > 8 || d.nx > 8) return false;
  switch (fam) {
    case PAIR_TC: return d.n == 8 || d.n == 16;
    case PAIR_GRP: return d.n == 16 || d.n == 32;
    case PAIR_ROWS: return d.n <= 16 && d.nr <= 4 && d.nx <= 4;
    default: return false;
  }
}

static void build_map(const std::vector<DevState>& sys, int levels, int chunk, std::vector<BatchCta>& map,
                      std::vector<long>& off, std::vector<long>& cnt) {
  off.assign(levels, 0);
  cnt.assign(levels, 0);
  // within a level the deepest systems come first: their chains of levels are
  // the longest, so the persistent launch starts them first
  std::vector<size_t> order(sys.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](size_t x, size_t y) { return sys[x].d.nblock > sys[y].d.nblock; });
  for (int L = 0; L < levels; ++L) {
    const int k = 1 << L;
    off[L] = (long)map.size();
    for (size_t i : order) {
      const long np = pairs_at_level(sys[i].d.nblock, k);
      for (long q0 = 0; q0 < np; q0 += chunk) {
        BatchCta c;
        c.sys = (int)i;
        c.pad = L;  // the level (the persistent launch reads it)
        c.q0 = q0;
        c.q1 = q0 + chunk < np ? q0 + chunk : np;
        map.push_back(c);
      }
    }
    cnt[L] = (long)map.size() - off[L];
  }
}

template <typename X>
static int upload_table(void*& dst, const std::vector<X>& v) {
  if (cudaMalloc(&dst, std::max<size_t>(v.size(), 1) * sizeof(X)) != cudaSuccess) return 1;
  if (!v.empty() && cudaMemcpy(dst, v.data(), v.size() * sizeof(X), cudaMemcpyHostToDevice) != cudaSuccess) return 1;
  return 0;
}

void batch_free(BatchClass& c) {
  if (c.qbuf) cudaFree(c.qbuf);
  c.qbuf = nullptr;
  for (void** p : {&c.fa, &c.sf, &c.sb, &c.ld, &c.rd})
    if (*p) { cudaFree(*p); *p = nullptr; }
  if (c.fmap) { cudaFree(c.fmap); c.fmap = nullptr; }
  if (c.smap) { cudaFree(c.smap); c.smap = nullptr; }
  if (c.cmap) { cudaFree(c.cmap); c.cmap = nullptr; }
  if (c.ccnt) { cudaFree(c.ccnt); c.ccnt = nullptr; }
  c.foff.clear(); c.fcnt.clear(); c.soff.clear(); c.scnt.clear();
}

template <typename T>
static int batch_build_t(BatchClass& c, const std::vector<DevState>& sys, int nrhs) {
  c.nsys = (int)sys.size();
  c.nrhs = nrhs;
  c.levels = 0;
  c.nrm = c.nxm = 0;
  size_t lmax = 0;
  std::vector<FactorArgs<T>> fa(sys.size());
  std::vector<SweepArgs<T>> sf(sys.size()), sb(sys.size());
  std::vector<LastDesc> ld(sys.size());
  std::vector<ResDesc> rd(sys.size());
  T* tag = nullptr;
  for (size_t i = 0; i < sys.size(); ++i) {
    DevState s = sys[i];
    const Dims d = s.d;
    const WorkSet<T> w = work_set(s, tag);
    c.n = d.n;
    c.nrm = std::max(c.nrm, d.nr);
    c.nxm = std::max(c.nxm, d.nx);
    int K = 1, lev = 0;
    while (K < d.nblock) { K *= 2; ++lev; }
    c.levels = std::max(c.levels, lev);
    lmax = std::max<size_t>(lmax, (size_t)std::max(d.Nr, d.Nc));
    FactorArgs<T> a{};
    a.d = d;
    a.D0 = s.D0; a.E0 = s.E0; a.B0 = s.B0; a.C0 = s.C0;
    a.D = w.D; a.E = w.E; a.B = w.B; a.C = w.C; a.Tm = w.Tm; a.P = s.P;
    a.Rbuf = w.Rbuf; a.Fbuf = s.Fbuf; a.st = s.st;
    a.ldw = odd_ld(2 * d.n + d.nr);
    a.x = nullptr; a.ldx = 0; a.nrf = 0; a.XB = s.XB;
    fa[i] = a;
    SweepArgs<T> sw{};
    sw.d = d;
    sw.D = w.D; sw.E = w.E; sw.B = w.B; sw.C = w.C; sw.Tm = w.Tm; sw.P = s.P;
    sw.x = s.bx; sw.ldx = s.bldx; sw.nrhs = nrhs; sw.XB = s.XB; sw.sel = SEL_LU;
    sw.done = s.bdone;
    sw.ldw = odd_ld(2 * d.n);
    sf[i] = sw;
    sw.ldw = d.n;
    sb[i] = sw;
    LastDesc l{};
    l.d = d;
    l.D0 = s.D0; l.E0 = s.E0; l.B0 = s.B0; l.C0 = s.C0; l.H = s.H; l.Cq = s.Cq; l.F0 = s.F0;
    l.Fbuf = s.Fbuf; l.XB = s.XB;
    l.Dw = w.D; l.Ew = w.E; l.Bw = w.B; l.Cw = w.C;
    l.Ffin = s.Ffin; l.Hl = s.Hl; l.tau = s.tau_l; l.x = s.bx;
    l.piv = s.piv_l; l.kind = s.sel_last; l.ldx = s.bldx; l.st = s.st;
    l.lb = last_bufs(s);
    l.done = s.bdone;
    ld[i] = l;
    ResDesc r{};
    r.d = d;
    r.D0 = s.D0; r.E0 = s.E0; r.B0 = s.B0; r.C0 = s.C0; r.Cq = s.Cq; r.F0 = s.F0; r.H = s.H;
    r.xs = s.bsol; r.b = s.bb; r.r = s.bx; r.nrm = s.bnrm; r.done = s.bdone;
    rd[i] = r;
  }
  c.last_smem = 2 * lmax * 8;
  std::vector<BatchCta> fmap, smap;
  build_map(sys, c.levels, c.chunk, fmap, c.foff, c.fcnt);
  build_map(sys, c.levels, 8, smap, c.soff, c.scnt);
  int bad = upload_table(c.fa, fa) | upload_table(c.sf, sf) | upload_table(c.sb, sb) | upload_table(c.ld, ld) |
            upload_table(c.rd, rd);
  void* m1 = nullptr;
  void* m2 = nullptr;
  bad |= upload_table(m1, fmap) | upload_table(m2, smap);
  c.fmap = static_cast<BatchCta*>(m1);
  c.smap = static_cast<BatchCta*>(m2);
  c.items = (long)fmap.size();
  if (cudaMalloc(&c.qbuf, (1 + 2 * (size_t)c.nsys) * sizeof(int)) != cudaSuccess) bad = 1;
  if (c.mixed && c.levels > 0) {  // compacted maps of the refinement passes
    if (cudaMalloc(&c.cmap, std::max<size_t>(smap.size(), 1) * sizeof(BatchCta)) != cudaSuccess) bad = 1;
    if (cudaMalloc(&c.ccnt, (size_t)c.levels * sizeof(long)) != cudaSuccess) bad = 1;
  }
  return bad;
}

int batch_build(BatchClass& c, const std::vector<DevState>& sys, int nrhs) {
  batch_free(c);
  return c.mixed ? batch_build_t<float>(c, sys, nrhs) : batch_build_t<double>(c, sys, nrhs);
}

// one batched launch of the class's pair kernel at level `L`
template <typename T>
static void batch_pairs(BatchClass& c, int L, cudaStream_t st) {
  const long cnt = c.fcnt[L];
  if (cnt == 0) return;
  FactorArgs<T> a0{};
  a0.k = 1 << L;
  a0.first = L == 0;
  const FactorArgs<T>* tab = static_cast<const FactorArgs<T>*>(c.fa);
  const BatchCta* map = c.fmap + c.foff[L];
  const unsigned g = (unsigned)cnt;
  if (c.fam == PAIR_TC) {
    const size_t sm = tc_smem_per_warp_t<T>(c.n) * 4;
    if (c.n == 16) {
      smem_limit_once(k_factor_lu_tc<16, true, false, 8, T>, sm);
      k_factor_lu_tc<16, true, false, 8, T><<<g, 128, sm, st>>>(a0, tab, map);
    } else {
      smem_limit_once(k_factor_lu_tc<8, true, false, 8, T>, sm);
      k_factor_lu_tc<8, true, false, 8, T><<<g, 128, sm, st>>>(a0, tab, map);
    }
    check_launch("batched pair kernel");
  }
  if (c.fam == PAIR_GRP) {
    if (c.n == 32) {
      smem_limit_once(k_factor_lu_grp<T, 32, true>, GrpShape<T, 32>::BYTES);
      k_factor_lu_grp<T, 32, true><<<g, 96, GrpShape<T, 32>::BYTES, st>>>(a0, tab, map);
    } else {
      smem_limit_once(k_factor_lu_grp<T, 16, true>, GrpShape<T, 16>::BYTES);
      k_factor_lu_grp<T, 16, true><<<g, 64, GrpShape<T, 16>::BYTES, st>>>(a0, tab, map);
    }
  } else if (c.fam == PAIR_ROWS) {
    if (c.n <= 4) k_factor_lu_rows<T, 4, 4, 4, true><<<g, 128, 0, st>>>(a0, tab, map);
    else if (c.n <= 8) k_factor_lu_rows<T, 8, 4, 4, true><<<g, 128, 0, st>>>(a0, tab, map);
    else k_factor_lu_rows<T, 16, 4, 4, true><<<g, 128, 0, st>>>(a0, tab, map);
  }
  check_launch("batched pair kernel");
  if (c.nrm > 0) {
    kb_border_fix<T><<<g, 128, 0, st>>>(tab, map, 1 << L);
    check_launch("kb_border_fix");
  }
}

// every level of every system of the class in one persistent launch
template <typename T>
static void batch_pairs_persistent(BatchClass& c, cudaStream_t st) {
  if (c.items == 0) return;
  cudaMemsetAsync(c.qbuf, 0, (1 + 2 * (size_t)c.nsys) * sizeof(int), st);
  BatchQueue qu{c.qbuf, c.qbuf + 1, c.qbuf + 1 + c.nsys, c.items};
  const FactorArgs<T>* tab = static_cast<const FactorArgs<T>*>(c.fa);
  auto grid = [&](auto* kern, int threads, size_t smem) {
    return grid_for(c.items, 1, 148 * resident_ctas(kern, threads, smem));
  };
  if (c.fam == PAIR_TC) {
    const size_t sm = tc_smem_per_warp_t<T>(c.n) * 4;
    if (c.n == 16) {
      smem_limit_once(kp_factor_tc<16, T>, sm);
      kp_factor_tc<16, T><<<grid(kp_factor_tc<16, T>, 128, sm), 128, sm, st>>>(tab, c.fmap, qu);
    } else {
      smem_limit_once(kp_factor_tc<8, T>, sm);
      kp_factor_tc<8, T><<<grid(kp_factor_tc<8, T>, 128, sm), 128, sm, st>>>(tab, c.fmap, qu);
    }
    check_launch("kp_factor_tc");
    return;
  }
  if (c.fam == PAIR_GRP) {
    if (c.n == 32) {
      auto* kern = kp_factor_grp<T, 32>;
      smem_limit_once(kern, GrpShape<T, 32>::BYTES);
      kern<<<grid(kern, 96, GrpShape<T, 32>::BYTES), 96, GrpShape<T, 32>::BYTES, st>>>(tab, c.fmap, qu);
    } else {
      auto* kern = kp_factor_grp<T, 16>;
      smem_limit_once(kern, GrpShape<T, 16>::BYTES);
      kern<<<grid(kern, 64, GrpShape<T, 16>::BYTES), 64, GrpShape<T, 16>::BYTES, st>>>(tab, c.fmap, qu);
    }
  } else if (c.fam == PAIR_ROWS) {
    auto* kern = c.n <= 4 ? kp_factor_rows<T, 4, 4, 4> : c.n <= 8 ? kp_factor_rows<T, 8, 4, 4>
                                                                   : kp_factor_rows<T, 16, 4, 4>;
    kern<<<grid(kern, 128, 0), 128, 0, st>>>(tab, c.fmap, qu);
  }
  check_launch("persistent batched pair kernel");
}

template <typename T>
static void batch_factorize_t(BatchClass& c, cudaStream_t st) {
  const LastDesc* ld = static_cast<const LastDesc*>(c.ld);
  kb_begin<T><<<c.nsys, 256, 0, st>>>(ld);
  check_launch("kb_begin");
  if (c.persist) {
    batch_pairs_persistent<T>(c, st);
  } else {
    for (int L = 0; L < c.levels; ++L) batch_pairs<T>(c, L, st);
  }
  kb_reduce_F<<<c.nsys, 256, 0, st>>>(ld);
  kb_last_assemble<T><<<c.nsys, 256, 0, st>>>(ld);
  kb_last_factor<<<c.nsys, 512, 0, st>>>(ld);
  check_launch("batched last block");
}

void batch_factorize(BatchClass& c, cudaStream_t st) {
  if (c.nsys == 0) return;
  if (c.mixed) batch_factorize_t<float>(c, st);
  else batch_factorize_t<double>(c, st);
}

// the sweep map of level L: the full map (one CTA per entry), or on the
// refinement passes the compacted map of the systems still refining, walked by
// a fixed grid (the launch is captured before the length is known)
static SweepMap sweep_map(const BatchClass& c, int L, bool compact) {
  if (!compact) return {c.smap + c.soff[L], nullptr, (unsigned)c.scnt[L]};
  return {c.cmap + c.soff[L], c.ccnt + L, (unsigned)std::min<long>(c.scnt[L], COMPACT_GRID)};
}

template <typename T, int N>
static void batch_sweeps_rows(BatchClass& c, cudaStream_t st, bool forward, int L, const SweepMap& m) {
  const bool r4 = c.nrm <= 4, x4 = c.nxm <= 4;
  SweepArgs<T> a0{};
  a0.k = 1 << L;
  if constexpr (N == 8 || N == 16) {
    if (c.n == N) {  // pipelined: a fixed grid walks the level's map entries
      const long nent = c.scnt[L];
      const unsigned g = (unsigned)std::min<long>(nent, 148 * 2);
      if (forward) {
        const SweepArgs<T>* tab = static_cast<const SweepArgs<T>*>(c.sf);
        auto* kern = r4 ? k_forward_pipe<N, 4, T, true> : k_forward_pipe<N, 8, T, true>;
        const size_t sm = 8 * (r4 ? FwdBuf<N, 4, T>::BYTES : FwdBuf<N, 8, T>::BYTES);
        smem_limit_once(kern, sm);
        kern<<<g, 256, sm, st>>>(a0, tab, m.map, m.ecnt, nent);
      } else {
        const SweepArgs<T>* tab = static_cast<const SweepArgs<T>*>(c.sb);
        auto* kern = x4 ? k_backward_pipe<N, 4, T, true> : k_backward_pipe<N, 8, T, true>;
        const size_t sm = 8 * (x4 ? BwdBuf<N, 4, T>::BYTES : BwdBuf<N, 8, T>::BYTES);
        smem_limit_once(kern, sm);
        kern<<<g, 256, sm, st>>>(a0, tab, m.map, m.ecnt, nent);
      }
      return;
    }
  }
  if (forward) {
    const SweepArgs<T>* tab = static_cast<const SweepArgs<T>*>(c.sf);
    if (r4) k_forward_rows<T, N, 4, true, true><<<m.grid, 256, 0, st>>>(a0, tab, m.map, m.ecnt);
    else k_forward_rows<T, N, 8, true, true><<<m.grid, 256, 0, st>>>(a0, tab, m.map, m.ecnt);
  } else {
    const SweepArgs<T>* tab = static_cast<const SweepArgs<T>*>(c.sb);
    if (x4) k_backward_rows<T, N, 4, true><<<m.grid, 256, 0, st>>>(a0, tab, m.map, m.ecnt);
    else k_backward_rows<T, N, 8, true><<<m.grid, 256, 0, st>>>(a0, tab, m.map, m.ecnt);
  }
}

template <typename T>
static void batch_sweep_level(BatchClass& c, cudaStream_t st, bool forward, int L, bool compact) {
  if (c.scnt[L] == 0) return;
  const SweepMap m = sweep_map(c, L, compact);
  if (c.n <= 4) batch_sweeps_rows<T, 4>(c, st, forward, L, m);
  else if (c.n <= 8) batch_sweeps_rows<T, 8>(c, st, forward, L, m);
  else if (c.n <= 16) batch_sweeps_rows<T, 16>(c, st, forward, L, m);
  else if (c.n == 32) {
    SweepArgs<T> a0{};
    a0.k = 1 << L;
    if (forward) {
      const SweepArgs<T>* tab = static_cast<const SweepArgs<T>*>(c.sf);
      if (c.nrm <= 4) k_forward_rows32<T, 4, true><<<m.grid, 256, 0, st>>>(a0, tab, m.map, m.ecnt);
      else k_forward_rows32<T, 8, true><<<m.grid, 256, 0, st>>>(a0, tab, m.map, m.ecnt);
    } else {
      const SweepArgs<T>* tab = static_cast<const SweepArgs<T>*>(c.sb);
      if (c.nxm <= 4) k_backward_rows32<T, 4, true><<<m.grid, 256, 0, st>>>(a0, tab, m.map, m.ecnt);
      else k_backward_rows32<T, 8, true><<<m.grid, 256, 0, st>>>(a0, tab, m.map, m.ecnt);
    }
  } else {
    SweepArgs<T> a0{};
    a0.k = 1 << L;
    if (forward) {
      const size_t sm = (size_t)odd_ld(2 * c.n) * c.nrhs * 8 * WARPS_PANEL;
      smem_limit_once(k_forward_level<T, true>, sm);
      k_forward_level<T, true><<<m.grid, WARPS_PANEL * 32, sm, st>>>(a0, static_cast<const SweepArgs<T>*>(c.sf),
                                                                     m.map, m.ecnt);
    } else {
      const size_t sm = (size_t)c.n * 8 * WARPS_PANEL;
      k_backward_level<T, true><<<m.grid, WARPS_PANEL * 32, sm, st>>>(a0, static_cast<const SweepArgs<T>*>(c.sb),
                                                                      m.map, m.ecnt);
    }
  }
  check_launch(forward ? "batched forward sweep" : "batched backward sweep");
}

template <typename T>
static void batch_solve_t(BatchClass& c, cudaStream_t st, bool compact) {
  const LastDesc* ld = static_cast<const LastDesc*>(c.ld);
  for (int L = 0; L < c.levels; ++L) batch_sweep_level<T>(c, st, true, L, compact);
  kb_reduce_xb<<<c.nsys, 256, 0, st>>>(ld, c.nrhs);
  kb_last_solve<<<c.nsys, 256, c.last_smem, st>>>(ld, c.nrhs);
  for (int L = c.levels - 1; L >= 0; --L) batch_sweep_level<T>(c, st, false, L, compact);
  check_launch("batched solve");
}

void batch_solve(BatchClass& c, cudaStream_t st, bool compact) {
  if (c.nsys == 0) return;
  compact = compact && c.cmap != nullptr;
  if (c.mixed) batch_solve_t<float>(c, st, compact);
  else batch_solve_t<double>(c, st, compact);
}

// Compacted sweep maps of the systems still refining: entry e of the full map
// is kept when its system has not converged, at a free position of its level
// (one atomic per warp and level; the pairs of a level are independent, so
// the order within a level does not change any result)
struct LevelOffsets {
  long off[32];
};

__global__ void __launch_bounds__(256) kb_compact_map(const LastDesc* ld, const BatchCta* smap, long nent,
                                                      LevelOffsets lo, BatchCta* cmap, long* ccnt) {
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  BatchCta c{};
  bool keep = false;
  if (e < nent) {
    c = smap[e];
    const int* dn = ld[c.sys].done;
    keep = !(dn && *dn);
  }
  const unsigned act = __ballot_sync(0xffffffffu, keep);
  if (!keep) return;
  const int L = c.pad;  // the entry's level
  const unsigned grp = __match_any_sync(act, L);
  const int leader = __ffs(grp) - 1;
  unsigned long long base = 0;
  if (lane == leader) base = atomicAdd(reinterpret_cast<unsigned long long*>(ccnt + L), (unsigned long long)__popc(grp));
  base = __shfl_sync(grp, base, leader);
  const long pos = (long)base + __popc(grp & ((1u << lane) - 1u));
  cmap[lo.off[L] + pos] = c;
}

void batch_compact(BatchClass& c, cudaStream_t st) {
  if (c.nsys == 0 || !c.cmap || c.levels == 0) return;
  const long nent = c.soff[c.levels - 1] + c.scnt[c.levels - 1];
  LevelOffsets lo{};
  for (int L = 0; L < c.levels; ++L) lo.off[L] = c.soff[L];
  cudaMemsetAsync(c.ccnt, 0, sizeof(long) * c.levels, st);
  if (nent > 0)
    kb_compact_map<<<(unsigned)((nent + 255) / 256), 256, 0, st>>>(static_cast<const LastDesc*>(c.ld), c.smap, nent,
                                                                    lo, c.cmap, c.ccnt);
  check_launch("kb_compact_map");
}

}  // namespace bcr
