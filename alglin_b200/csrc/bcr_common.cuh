// Shared definitions for the BorderedCR device code (sm_100a).
//
// Device storage keeps the block layout of alglin::BorderedCR
// (src/Alglin/BABD_BorderedCR.hxx:972-998, BABD_BorderedCR.cc:102-124):
//   D,E   [nblock][n*n]        column-major n x n
//   B     [nblock][n*nx]       column-major n x nx
//   C     [nblock+1][nr*n]     column-major nr x n
//   T     [nblock][2n*n + n]   panel factors (2n x n, ld 2n) + tau
//   P     [nblock][3n] (uint8)  row map: position -> original panel row (2n
//                               entries, getrf's final row order), then the
//                               column map of QRP (n entries, y index -> x index)
// Each array lives in its own device allocation; a cyclic-reduction level
// touches whole blocks, so every block read or written is one contiguous run.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace bcr {

enum Internal : int { SEL_LU = 0, SEL_QR = 1, SEL_QRP = 2 };
enum LastKind : int { LAST_LU = 0, LAST_LUPQ = 1, LAST_QR = 2, LAST_QRP = 3,
                      LAST_SVD = 4, LAST_LSS = 5, LAST_LSY = 6, LAST_PINV = 7 };

// pair-kernel choice of the factorization (PAIR_AUTO picks by shape)
enum PairKernel : int { PAIR_AUTO = 0, PAIR_TC = 1, PAIR_GRP = 2, PAIR_ROWS = 3, PAIR_CTA = 4, PAIR_SMEM = 5,
                        PAIR_UMMA = 6, PAIR_TREE = 7, PAIR_TC_GATHER = 8 };

// error codes written by kernels into the device status word
enum DevStatus : int {
  DEV_OK = 0,
  DEV_ZERO_PIVOT = 1,      // panel LU hit an exactly-zero pivot
  DEV_LAST_SINGULAR = 2,   // last block factorization failed
  DEV_BAD_SHAPE = 3,       // last block shape unsupported by the selected solver
  DEV_TIMEOUT = 4,         // a bounded wait on the tensor-core pipeline expired
};

struct Dims {
  int nblock, n, qr, qx, nr, nx;
  int Nr, Nc;
};

__host__ __device__ inline size_t szT(const Dims& d) { return 2 * (size_t)d.n * d.n + d.n; }
__host__ __device__ inline size_t szP(const Dims& d) { return 3 * (size_t)d.n; }

// number of pairs (j-k, j) eliminated at the level with stride k
__host__ __device__ inline long pairs_at_level(int nblock, int k) {
  return nblock > k ? (long)(nblock - k - 1) / (2L * k) + 1 : 0;
}

// one CTA of a batched launch: pairs [q0, q1) of system `sys` at the level
struct BatchCta {
  int sys, pad;
  long q0, q1;
};

// factorization of the last block actually in use (written by the device)
// FACT_LU_ROWS: getrf factors with the rows left in place, piv[pos] = the row
// holding position pos of L\U (the blocked last-block LU)
enum LastFact : int { FACT_LU = 0, FACT_LUPQ = 1, FACT_QR = 2, FACT_QRP = 3, FACT_SVD = 4, FACT_SVD_T = 5,
                      FACT_LU_ROWS = 6 };

// status layout: [0] code, [1] block index, [2] LAPACK-style info, [3] level,
// [4] LastFact of the last block
struct StatusWords { int code, block, info, level, kind; };

__device__ inline void report(StatusWords* st, int code, int block, int info, int level) {
  if (atomicCAS(&st->code, 0, code) == 0) {
    st->block = block;
    st->info = info;
    st->level = level;
  }
}

template <typename T> __device__ __forceinline__ T dev_abs(T x) { return x < T(0) ? -x : x; }

template <typename T>
__device__ __forceinline__ T shfl_xor(T v, int m) { return __shfl_xor_sync(0xffffffffu, v, m); }

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += shfl_xor(v, o);
  return v;
}

// warp argmax of (value, index); ties go to the smaller index (idamax rule)
template <typename T>
__device__ __forceinline__ void warp_argmax(T& v, int& idx) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    T ov = shfl_xor(v, o);
    int oi = shfl_xor(idx, o);
    if (ov > v || (ov == v && oi < idx)) { v = ov; idx = oi; }
  }
}

}  // namespace bcr
