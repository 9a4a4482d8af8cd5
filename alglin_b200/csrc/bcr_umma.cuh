// ---------------------------------------------------------------------------
// Large blocks, FP32 working precision, LU: one CTA per pair with the trailing
// products on the 5th-generation tensor cores (tcgen05.mma, kind::tf32, FP32
// accumulators in tensor memory) as 3xTF32 split products.
//
// The pair is eliminated in three steps (the same algebra as buildT/applyT,
// BABD_BorderedCR.cc:845-982, with the border rows of factorize_block,
// cc:1107-1154):
//
//   1. panel LU: the (2n + nr) x n panel [E_jp; D_j; C_j] is factored in
//      shared memory with the getrf pivot rule (largest |a| among the 2n
//      candidate rows, first position on ties), in column blocks of UM_BW.
//      Every thread owns one row of the block in registers.  Per pivot step
//      each warp with candidate rows posts its best row and a shared 64-bit
//      atomicMax of (|a|, first position, warp) picks the winner; one barrier
//      over those warps per step (border-only warps apply the block's
//      eliminations afterwards); the block's U rows are solved with its unit lower
//      triangle and the rows below get one product of depth UM_BW.  Row
//      interchanges are a position map, no row moves.
//   2. Z = L11^-1 (the inverse of the unit lower triangle of the n pivot rows),
//      by 32 x 32 diagonal inverses and block forward substitution.
//   3. with Xt the n pivot rows and Xb the other n rows of the trailing
//      columns X = [D_jp 0 B_jp; 0 E_j B_j] (2n + nx columns):
//        U12 = Z Xt                 (tensor cores: the U-row D'_j E'_j B'_j)
//        Xb' = Xb - L21 U12         (tensor cores: the reduced row)
//        border = -Lc U12           (CUDA cores: dC_jp, dC_jpp, dF)
//      Operands are split as a = hi + lo with hi the TF32 part of a and lo
//      the FP32 remainder; each product is hi*hi + lo*hi + hi*lo accumulated
//      in FP32 (the products' error is about that of FP32 arithmetic).
//
// Shared memory operands use the K-major layout without swizzle: 8-row x
// 16-byte core matrices, 8-row groups 128 bytes apart (SBO), 4-element K
// groups LBO bytes apart.  The K loop of each product is staged 16 deep in two
// buffers; tcgen05.commit arrives on the buffer's mbarrier when the MMAs that
// read it are done.  Every wait on an mbarrier is bounded (about a second):
// on expiry the kernel reports DEV_TIMEOUT, frees its tensor memory and ends.
// ---------------------------------------------------------------------------
#include "bcr_umma_layout.cuh"

// ---- sm_100a primitives ----------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// completion of the phase with the given parity; false after about a second
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity))
    if (clock64() - t0 > (2LL << 30)) return false;
  return true;
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// smem matrix descriptor, K-major, no swizzle
__device__ __forceinline__ uint64_t umma_sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
         (1ull << 46);
}
// instruction descriptor: D f32, A and B tf32, both K-major, M x N
__host__ __device__ constexpr uint32_t umma_idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ void umma_tf32(uint32_t dt, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(dt),
      "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
// 16 consecutive FP32 columns of this thread's tensor-memory lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ float tf32_hi(float v) { return __uint_as_float(__float_as_uint(v) & 0xFFFFE000u); }

// A operand element (row i of 128, K index k): byte offset in one of hi / lo
__device__ __forceinline__ uint32_t umma_a_off(int i, int k) {
  return (uint32_t)((k >> 2) * 2048 + (i >> 3) * 128 + (i & 7) * 16 + (k & 3) * 4);
}
// B stage element (N index c, K index m within the 16-deep stage)
__device__ __forceinline__ uint32_t umma_b_off(int c, int m, int lbo) {
  return (uint32_t)((m >> 2) * lbo + (c >> 3) * 128 + (c & 7) * 16 + (m & 3) * 4);
}

// cnt elements read by ld(e) and written by st(e, v), the reads of a thread
// issued in groups of 16 before their writes (a CTA per SM keeps few loads in
// flight otherwise)
template <typename Ld, typename St>
__device__ __forceinline__ void um_batched(int cnt, Ld ld, St st) {
  constexpr int U = 16;
  for (int base = threadIdx.x; base < cnt; base += U * UM_NT) {
    float v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int e = base + u * UM_NT;
      v[u] = e < cnt ? ld(e) : 0.0f;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int e = base + u * UM_NT;
      if (e < cnt) st(e, v[u]);
    }
  }
}

// One product D[128 x Npad] = A[128 x Kpad] * B[Kpad x Npad] with the B operand
// staged 16 K-rows at a time by all threads from src(c, m) (m the K index).
// A (hi, lo) must be in shared memory and fenced.  Returns false on a timeout.
template <typename Src, typename Obs>
__device__ bool umma_product(const UmmaLayout& L, unsigned char* sm, uint64_t* bars, uint32_t (&par)[2],
                             uint32_t tmem, Src src, Obs obs) {
  const int tid = threadIdx.x;
  const int S = L.Kpad / 16;
  const uint32_t sA = smem_u32(sm);
  const int cnt = 16 * L.Npad;  // <= UM_PF * UM_NT
  // the next stage's elements are loaded one stage ahead, into registers
  float pv[UM_PF];
  auto load_stage = [&](int s) {
#pragma unroll
    for (int u = 0; u < UM_PF; ++u) {
      const int e = tid + u * UM_NT;
      pv[u] = e < cnt ? src(e >> 4, 16 * s + (e & 15)) : 0.0f;
    }
  };
  load_stage(0);
  bool ok = true;
  for (int s = 0; s < S; ++s) {
    const int b = s & 1;
    if (s >= 2) {  // the MMAs of stage s-2 read this buffer
      ok = mbar_wait_bounded(&bars[b], par[b]);
      par[b] ^= 1u;
    }
    if (ok) {
      unsigned char* bh = sm + L.offB + (unsigned)b * 2u * L.szBhalf;
      unsigned char* bl = bh + L.szBhalf;
#pragma unroll
      for (int u = 0; u < UM_PF; ++u) {
        const int e = tid + u * UM_NT;
        if (e < cnt) {
          const float h = tf32_hi(pv[u]);
          const uint32_t o = umma_b_off(e >> 4, e & 15, L.LBO_B);
          *reinterpret_cast<float*>(bh + o) = h;
          *reinterpret_cast<float*>(bl + o) = pv[u] - h;
        }
      }
    }
    fence_async_smem();
    if (__syncthreads_or(!ok)) return false;
    if (s + 1 < S) load_stage(s + 1);
    if (tid == 0) {
      tc_fence_after();
      const uint32_t sB = smem_u32(sm + L.offB + (unsigned)b * 2u * L.szBhalf);
#pragma unroll
      for (int ks = 0; ks < 2; ++ks) {
        const int kg = 16 * s + 8 * ks;
        const uint32_t ao = (uint32_t)(kg >> 2) * 2048u;
        const uint64_t ah = umma_sdesc(sA + ao, 2048, 128);
        const uint64_t al = umma_sdesc(sA + L.szAhalf + ao, 2048, 128);
        const uint32_t bo = (uint32_t)(2 * ks) * (uint32_t)L.LBO_B;
        for (int ch = 0; ch < 2; ++ch) {
          const int nw = ch ? L.N1 : L.N0;
          if (nw == 0) continue;
          const int c0 = ch ? L.N0 : 0;
          const uint32_t co = (uint32_t)(c0 >> 3) * 128u;
          const uint64_t bdh = umma_sdesc(sB + bo + co, (uint32_t)L.LBO_B, 128);
          const uint64_t bdl = umma_sdesc(sB + L.szBhalf + bo + co, (uint32_t)L.LBO_B, 128);
          const uint32_t id = umma_idesc_tf32(128, nw);
          const uint32_t dt = tmem + (uint32_t)c0;
          umma_tf32(dt, ah, bdh, id, (s > 0 || ks > 0) ? 1u : 0u);
          umma_tf32(dt, al, bdh, id, 1u);
          umma_tf32(dt, ah, bdl, id, 1u);
        }
      }
      umma_commit(&bars[b]);
    }
    // CUDA-core work on the staged rows while the tensor cores run
    obs(s, sm + L.offB + (unsigned)b * 2u * L.szBhalf);
  }
  // the last (up to) two commits: every commit is waited exactly once
  for (int s = S - 2 < 0 ? 0 : S - 2; s < S; ++s) {
    const int b = s & 1;
    if (ok) ok = mbar_wait_bounded(&bars[b], par[b]);
    par[b] ^= 1u;
  }
  tc_fence_after();
  return !__syncthreads_or(!ok);
}

// A operand (hi, lo) from a(i, k), i < 128, k < Kpad
template <typename Src>
__device__ void umma_stage_a(const UmmaLayout& L, unsigned char* sm, Src a) {
  um_batched(128 * L.Kpad, [&](int e) { return a((e >> 2) & 127, 4 * (e >> 9) + (e & 3)); },
             [&](int e, float v) {
               const float h = tf32_hi(v);
               const uint32_t o = umma_a_off((e >> 2) & 127, 4 * (e >> 9) + (e & 3));
               *reinterpret_cast<float*>(sm + o) = h;
               *reinterpret_cast<float*>(sm + L.szAhalf + o) = v - h;
             });
  fence_async_smem();
}

// one row of cnt elements, element c at src[c * stride], into dst[0, round_up(cnt, 16))
// (16-byte aligned; zero past cnt), the 16 loads of a group issued together
template <typename S>
__device__ __forceinline__ void um_load_row(const S* src, int stride, int cnt, float* dst) {
  for (int c0 = 0; c0 < cnt; c0 += 16) {
    float v[16];
#pragma unroll
    for (int u = 0; u < 16; ++u) v[u] = c0 + u < cnt ? float(src[(size_t)(c0 + u) * stride]) : 0.0f;
#pragma unroll
    for (int u = 0; u < 4; ++u)
      *reinterpret_cast<float4*>(dst + c0 + 4 * u) = make_float4(v[4 * u], v[4 * u + 1], v[4 * u + 2], v[4 * u + 3]);
  }
}
// cnt elements src[c * stride] (zeros when src is null) to dst[c * dstride]
template <typename S>
__device__ __forceinline__ void um_copy_col(const S* src, int stride, int cnt, float* dst, int dstride) {
  for (int c0 = 0; c0 < cnt; c0 += 16) {
    float v[16];
#pragma unroll
    for (int u = 0; u < 16; ++u) v[u] = (src && c0 + u < cnt) ? float(src[(size_t)(c0 + u) * stride]) : 0.0f;
#pragma unroll
    for (int u = 0; u < 16; ++u)
      if (c0 + u < cnt) dst[(size_t)(c0 + u) * dstride] = v[u];
  }
}

__global__ void __launch_bounds__(UM_NT, 1) k_factor_lu_umma(FactorArgs<float> a, float* slab, size_t slab_elems) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int s_perm[2 * UM_NMAX + UM_NRMAX];  // position -> row
  __shared__ int s_pivrow[UM_NMAX];               // pivot step -> row
  __shared__ __align__(8) uint64_t s_bar[2];
  __shared__ uint32_t s_taddr;
  __shared__ int s_info;
  __shared__ unsigned long long s_best[UM_BW];  // per pivot step: key | first position | warp
  __shared__ int s_pivw[UM_BW];                 // per pivot step: the winning warp
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const Dims d = a.d;
  const int n = d.n, nr = d.nr, nb = d.nblock, n2 = 2 * n;
  const UmmaLayout L = umma_layout(d);
  const int R = L.R, LDP = L.LDP, NP = L.NP, Nc = L.Nc;
  const int nwc = (n2 + 31) / 32;  // warps that own pivot candidates
  const size_t nn = (size_t)n * n, nnx = (size_t)n * d.nx, nrn = (size_t)nr * n, nrnx = (size_t)nr * d.nx;
  float* P = reinterpret_cast<float*>(smem_raw);
  float* Zf = reinterpret_cast<float*>(smem_raw + L.offZ);
  float* Lc = reinterpret_cast<float*>(smem_raw + L.offLc);  // [m][UM_NRMAX], zero past nr
  float* slot = Zf;  // during the LU: [step][warp][UM_BW values, winner row]
  float* Xs = slab + (size_t)blockIdx.x * slab_elems;  // [col][position], 2n x Nc

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_taddr)),
                 "r"(UM_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(&s_bar[0], 1);
    mbar_init(&s_bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_taddr;
  uint32_t par[2] = {0u, 0u};

  const int k = a.k;
  const long np = pairs_at_level(nb, k);
  const bool first = a.first != 0;
  for (long q = blockIdx.x; q < np; q += gridDim.x) {
    const int j = k + (int)(2L * k * q), jp = j - k;
    const size_t oj = (size_t)j * nn, ojp = (size_t)jp * nn;
    float* const Dj = a.D + oj;
    float* const Ej = a.E + oj;
    float* const Bj = a.B + (size_t)j * nnx;
    // column c of the pair's U-row [D'_j E'_j B'_j] (n rows)
    auto ucol = [&](int c) -> float* { return c < n ? Dj + (size_t)c * n : c < n2 ? Ej + (size_t)(c - n) * n : Bj + (size_t)(c - n2) * n; };
    // ------------------------------------------------------------ panel load
    if (tid == 0) s_info = 0;
    if (tid < UM_BW) s_best[tid] = 0ull;
    // row t of [E_jp; D_j; C_j] by thread t
    if (tid < R) {
      float* dst = P + tid * LDP;
      if (tid < n) {
        if (first) um_load_row(a.E0 + ojp + tid, n, n, dst); else um_load_row(a.E + ojp + tid, n, n, dst);
      } else if (tid < n2) {
        if (first) um_load_row(a.D0 + oj + (tid - n), n, n, dst); else um_load_row(Dj + (tid - n), n, n, dst);
      } else {
        const size_t o = (size_t)j * nrn + (tid - n2);
        if (first) um_load_row(a.C0 + o, nr, n, dst); else um_load_row(a.C + o, nr, n, dst);
      }
    }
    __syncthreads();
    // --------------------------------------------------------------- panel LU
    int pos = tid, done = 0, info = 0;
    float rv[UM_BW];
    for (int kb = 0; kb < n && info == 0; kb += UM_BW) {
      const int w = n - kb < UM_BW ? n - kb : UM_BW;
      if (tid < R) {
        const float4* src = reinterpret_cast<const float4*>(P + tid * LDP + kb);
#pragma unroll
        for (int q4 = 0; q4 < UM_BW / 4; ++q4) {
          const float4 t = src[q4];
          rv[4 * q4] = t.x; rv[4 * q4 + 1] = t.y; rv[4 * q4 + 2] = t.z; rv[4 * q4 + 3] = t.w;
        }
      }
      // pivot steps: only the warps with candidate rows take part (named barrier 1)
      if (warp < nwc) {
#pragma unroll
        for (int i = 0; i < UM_BW; ++i) {
          if (i < w && info == 0) {
            const int gi = kb + i;
            {
              // the warp's candidate: largest |a|, then first position
              const bool cand = tid < n2 && !done;
              const uint32_t key = (cand && rv[i] == rv[i]) ? __float_as_uint(fabsf(rv[i])) : 0u;
              const uint32_t kmax = __reduce_max_sync(0xFFFFFFFFu, key);
              uint32_t bal = __ballot_sync(0xFFFFFFFFu, cand && key == kmax);
              if (__popc(bal) > 1) {  // tie: the first position among them
                const uint32_t pmin = __reduce_min_sync(0xFFFFFFFFu, (cand && key == kmax) ? (uint32_t)pos : 0xFFFFu);
                bal = __ballot_sync(0xFFFFFFFFu, cand && key == kmax && (uint32_t)pos == pmin);
              }
              if (bal != 0u && lane == __ffs(bal) - 1) {
                float* sl = slot + (i * UM_NW + warp) * (UM_BW + 4);
#pragma unroll
                for (int q4 = 0; q4 < UM_BW / 4; ++q4)
                  reinterpret_cast<float4*>(sl)[q4] = make_float4(rv[4 * q4], rv[4 * q4 + 1], rv[4 * q4 + 2], rv[4 * q4 + 3]);
                reinterpret_cast<int*>(sl)[UM_BW] = tid;
                atomicMax(&s_best[i], ((unsigned long long)kmax << 32) |
                                          ((unsigned long long)(0xFFFFu - (uint32_t)pos) << 16) | (unsigned)warp);
              }
            }
            asm volatile("bar.sync 1, %0;" ::"r"(nwc * 32) : "memory");
            const unsigned long long bst = *reinterpret_cast<volatile unsigned long long*>(&s_best[i]);
            const int bw = (int)(bst & 0xFFFFu);
            const float* win = slot + (i * UM_NW + bw) * (UM_BW + 4);
            const int wt = reinterpret_cast<const int*>(win)[UM_BW];
            const float pv = win[i];
            if (bst == 0ull || pv == 0.0f) {
              info = gi + 1;
            } else {
              if (tid == 0) { s_pivrow[gi] = wt; s_pivw[i] = bw; }
              if (pos == gi) pos = (int)(0xFFFFu - (uint32_t)((bst >> 16) & 0xFFFFu));
              if (tid == wt) { pos = gi; done = 1; }
              if (tid < R && !done) {
                float rinv;
                asm("rcp.approx.f32 %0, %1;" : "=f"(rinv) : "f"(pv));
                const float l = rv[i] * rinv;
                rv[i] = l;
#pragma unroll
                for (int q4 = (i + 1) / 4; q4 < UM_BW / 4; ++q4) {
                  const float4 u4 = *reinterpret_cast<const float4*>(win + 4 * q4);
                  if (4 * q4 > i) rv[4 * q4] = fmaf(-l, u4.x, rv[4 * q4]);
                  if (4 * q4 + 1 > i) rv[4 * q4 + 1] = fmaf(-l, u4.y, rv[4 * q4 + 1]);
                  if (4 * q4 + 2 > i) rv[4 * q4 + 2] = fmaf(-l, u4.z, rv[4 * q4 + 2]);
                  if (4 * q4 + 3 > i) rv[4 * q4 + 3] = fmaf(-l, u4.w, rv[4 * q4 + 3]);
                }
              }
            }
          }
        }
        if (tid == 0) s_info = info;
      }
      __syncthreads();
      info = s_info;
      // border rows of warps without candidates: the block's eliminations in order
      if (warp >= nwc && tid < R && info == 0) {
#pragma unroll
        for (int i = 0; i < UM_BW; ++i) {
          if (i < w) {
            const float* win = slot + (i * UM_NW + s_pivw[i]) * (UM_BW + 4);
            float rinv;
            asm("rcp.approx.f32 %0, %1;" : "=f"(rinv) : "f"(win[i]));
            const float l = rv[i] * rinv;
            rv[i] = l;
#pragma unroll
            for (int q4 = (i + 1) / 4; q4 < UM_BW / 4; ++q4) {
              const float4 u4 = *reinterpret_cast<const float4*>(win + 4 * q4);
              if (4 * q4 > i) rv[4 * q4] = fmaf(-l, u4.x, rv[4 * q4]);
              if (4 * q4 + 1 > i) rv[4 * q4 + 1] = fmaf(-l, u4.y, rv[4 * q4 + 1]);
              if (4 * q4 + 2 > i) rv[4 * q4 + 2] = fmaf(-l, u4.z, rv[4 * q4 + 2]);
              if (4 * q4 + 3 > i) rv[4 * q4 + 3] = fmaf(-l, u4.w, rv[4 * q4 + 3]);
            }
          }
        }
      }
      if (tid < R) {
        float4* dst = reinterpret_cast<float4*>(P + tid * LDP + kb);
#pragma unroll
        for (int q4 = 0; q4 < UM_BW / 4; ++q4)
          dst[q4] = make_float4(rv[4 * q4], rv[4 * q4 + 1], rv[4 * q4 + 2], rv[4 * q4 + 3]);
      }
      if (tid < UM_BW) s_best[tid] = 0ull;  // read by every candidate warp before the barrier above
      __syncthreads();
      if (kb + UM_BW < n) {  // w == UM_BW here
        int ro[UM_BW];
#pragma unroll
        for (int m = 0; m < UM_BW; ++m) ro[m] = s_pivrow[kb + m] * LDP;
        // the block's U rows in the panel columns right of it: unit lower solve
        for (int c = kb + UM_BW + tid; c < n; c += UM_NT) {
          float y[UM_BW];
#pragma unroll
          for (int r = 0; r < UM_BW; ++r) y[r] = P[ro[r] + c];
#pragma unroll
          for (int m = 0; m < UM_BW; ++m)
#pragma unroll
            for (int r = m + 1; r < UM_BW; ++r) y[r] = fmaf(-P[ro[r] + kb + m], y[m], y[r]);
#pragma unroll
          for (int r = 0; r < UM_BW; ++r) P[ro[r] + c] = y[r];
        }
        __syncthreads();
        // the rows that are not pivots yet: one product of depth UM_BW
        if (tid < R && !done) {
          float* row = P + tid * LDP;
          for (int c = kb + UM_BW; c < n; c += 4) {
            float4 acc = *reinterpret_cast<float4*>(row + c);
#pragma unroll
            for (int m = 0; m < UM_BW; ++m) {
              const float4 u = *reinterpret_cast<const float4*>(P + ro[m] + c);
              acc.x = fmaf(-rv[m], u.x, acc.x);
              acc.y = fmaf(-rv[m], u.y, acc.y);
              acc.z = fmaf(-rv[m], u.z, acc.z);
              acc.w = fmaf(-rv[m], u.w, acc.w);
            }
            *reinterpret_cast<float4*>(row + c) = acc;
          }
        }
        __syncthreads();
      }
    }
    if (info != 0) {
      if (tid == 0) report(a.st, DEV_ZERO_PIVOT, j, info, k);
      __syncthreads();
      continue;
    }
    if (tid < R) s_perm[pos] = tid;
    __syncthreads();
    // ------------------------------------- factors out; X staged by position
    float* Tj = a.Tm + (size_t)j * szT(d);
    if (tid < n2) {  // T in getrf order, column-major 2n x n: one position per thread
      const float* prow = P + s_perm[tid] * LDP;
      for (int c0 = 0; c0 < n; c0 += 4) {
        const float4 v = *reinterpret_cast<const float4*>(prow + c0);
        Tj[(size_t)c0 * n2 + tid] = v.x;
        if (c0 + 1 < n) Tj[(size_t)(c0 + 1) * n2 + tid] = v.y;
        if (c0 + 2 < n) Tj[(size_t)(c0 + 2) * n2 + tid] = v.z;
        if (c0 + 3 < n) Tj[(size_t)(c0 + 3) * n2 + tid] = v.w;
      }
      a.P[(size_t)j * szP(d) + tid] = (unsigned char)s_perm[tid];
      if (tid < n) a.P[(size_t)j * szP(d) + n2 + tid] = (unsigned char)tid;
      // X = [D_jp 0 B_jp; 0 E_j B_j], row tid, to Xs[col * 2n + pos]
      float* xd = Xs + pos;
      const int r = tid % n;
      if (tid < n) {
        if (first) um_copy_col(a.D0 + ojp + r, n, n, xd, n2); else um_copy_col(a.D + ojp + r, n, n, xd, n2);
        um_copy_col((const float*)nullptr, n, n, xd + (size_t)n * n2, n2);
      } else {
        um_copy_col((const float*)nullptr, n, n, xd, n2);
        // E'_j is written here later: plain loads
        if (first) um_copy_col(a.E0 + oj + r, n, n, xd + (size_t)n * n2, n2); else um_copy_col(Ej + r, n, n, xd + (size_t)n * n2, n2);
      }
      const size_t ob = (size_t)(tid < n ? jp : j) * nnx + r;
      if (first) um_copy_col(a.B0 + ob, n, d.nx, xd + (size_t)n2 * n2, n2);
      else um_copy_col(a.B + ob, n, d.nx, xd + (size_t)n2 * n2, n2);
    }
    for (int e = tid; e < n * UM_NRMAX; e += UM_NT) {  // border multipliers C_j U^-1
      const int r = e & (UM_NRMAX - 1), c = e / UM_NRMAX;
      const float v = r < nr ? P[(n2 + r) * LDP + c] : 0.0f;
      Lc[e] = v;
      if (r < nr) a.C[(size_t)j * nrn + r + (size_t)c * nr] = v;
    }
    // ---------------------------------------------------- Z = L11^-1 (FP32)
    // on the last four warps (named barrier 2), while warps 0..7 copy X above
    if (warp >= UM_NW - 4) {
      const int zt = tid - (UM_NT - 128);  // 0..127
      if (zt < NP) {  // zero above the diagonal blocks
        for (int c = 32 * (zt / 32 + 1); c < NP; c += 4)
          *reinterpret_cast<float4*>(Zf + zt * LDP + c) = make_float4(0.f, 0.f, 0.f, 0.f);
      }
      if (zt < NP) {  // diagonal 32 x 32 inverses, one column per lane
        const int a32 = (zt >> 5) * 32, c = lane;
        float z[32];
#pragma unroll
        for (int r = 0; r < 32; ++r) {
          const int gr = a32 + r;
          float v = 0.0f;
          if (gr < n) {
            v = (r == c) ? 1.0f : 0.0f;
            const float* Lr = P + s_perm[gr] * LDP + a32;
#pragma unroll
            for (int m = 0; m < r; ++m) v = fmaf(-Lr[m], z[m], v);
          }
          z[r] = v;
        }
#pragma unroll
        for (int r = 0; r < 32; ++r) Zf[(a32 + r) * LDP + a32 + c] = z[r];
      }
      asm volatile("bar.sync 2, 128;" ::: "memory");
      for (int r0 = 32; r0 < NP; r0 += 32) {
        // Zf[r0:r0+32, 0:r0] = L[r0:r0+32, 0:r0] * Z[0:r0, 0:r0]  (2 rows x 4 columns per thread)
        for (int t = zt; t < 16 * (r0 / 4); t += 128) {
          const int rr = 2 * (t & 15), cc = 4 * (t >> 4);
          const int g0 = r0 + rr, g1 = g0 + 1;
          const float* L0 = g0 < n ? P + s_perm[g0] * LDP : nullptr;
          const float* L1 = g1 < n ? P + s_perm[g1] * LDP : nullptr;
          float4 s0 = make_float4(0.f, 0.f, 0.f, 0.f), s1 = s0;
          for (int m = cc; m < r0; ++m) {  // Z[m][cc..cc+3] = 0 for m < cc
            const float4 zv = *reinterpret_cast<const float4*>(Zf + m * LDP + cc);
            const float l0 = L0 ? L0[m] : 0.0f, l1 = L1 ? L1[m] : 0.0f;
            s0.x = fmaf(l0, zv.x, s0.x); s0.y = fmaf(l0, zv.y, s0.y);
            s0.z = fmaf(l0, zv.z, s0.z); s0.w = fmaf(l0, zv.w, s0.w);
            s1.x = fmaf(l1, zv.x, s1.x); s1.y = fmaf(l1, zv.y, s1.y);
            s1.z = fmaf(l1, zv.z, s1.z); s1.w = fmaf(l1, zv.w, s1.w);
          }
          *reinterpret_cast<float4*>(Zf + g0 * LDP + cc) = s0;
          *reinterpret_cast<float4*>(Zf + g1 * LDP + cc) = s1;
        }
        asm volatile("bar.sync 2, 128;" ::: "memory");
        // Zf[r0:r0+32, 0:r0] = -Z_bb * (that), in place, one column per thread
        for (int c = zt; c < r0; c += 128) {
          float y[32];
#pragma unroll
          for (int r = 0; r < 32; ++r) y[r] = Zf[(r0 + r) * LDP + c];
#pragma unroll
          for (int r = 31; r >= 0; --r) {
            const float* Zr = Zf + (r0 + r) * LDP + r0;
            float s = 0.0f;
#pragma unroll
            for (int m = 0; m <= r; ++m) s = fmaf(Zr[m], y[m], s);
            y[r] = -s;
          }
#pragma unroll
          for (int r = 0; r < 32; ++r) Zf[(r0 + r) * LDP + c] = y[r];
        }
        asm volatile("bar.sync 2, 128;" ::: "memory");
      }
    }
    __syncthreads();
    // ------------------------------------------------ U12 = Z Xt (tensor cores)
    umma_stage_a(L, smem_raw, [&](int i, int kk) {
      return (i < n && kk < n) ? Zf[i * LDP + kk] : 0.0f;
    });
    __syncthreads();
    bool ok = umma_product(L, smem_raw, s_bar, par, tmem, [&](int c, int m) {
      return (m < n && c < Nc) ? Xs[(size_t)c * n2 + m] : 0.0f;
    }, [](int, const unsigned char*) {});
    if (!ok) {
      if (tid == 0) report(a.st, DEV_TIMEOUT, j, 0, k);
      break;
    }
    // U-row out: D'_j, E'_j, B'_j
    {
      const int qd = warp & 3, grp = warp >> 2, m = 32 * qd + lane;
      for (int pc = grp; pc < L.Npad / 16; pc += UM_NW / 4) {
        float v[16];
        tmem_ld16(tmem + ((uint32_t)(32 * qd) << 16) + (uint32_t)(16 * pc), v);
        if (m < n) {
          if ((n & 15) == 0 && 16 * pc + 16 <= Nc) {  // the piece lies in one of D'_j, E'_j, B'_j
            float* col = ucol(16 * pc) + m;
#pragma unroll
            for (int jj = 0; jj < 16; ++jj) col[(size_t)jj * n] = v[jj];
          } else {
#pragma unroll
            for (int jj = 0; jj < 16; ++jj) {
              const int c = 16 * pc + jj;
              if (c < Nc) ucol(c)[m] = v[jj];
            }
          }
        }
      }
    }
    tc_fence_before();
    __syncthreads();
    // ------------------------------------------- Xb - L21 U12 (tensor cores)
    umma_stage_a(L, smem_raw, [&](int i, int kk) {
      return (i < n && kk < n) ? Tj[(size_t)kk * n2 + n + i] : 0.0f;
    });
    __syncthreads();
    // the border rows' -Lc U12 on the CUDA cores from the staged U12 rows, one
    // trailing column per thread
    float bacc[UM_NRMAX];
#pragma unroll
    for (int r = 0; r < UM_NRMAX; ++r) bacc[r] = 0.0f;
    ok = umma_product(L, smem_raw, s_bar, par, tmem, [&](int c, int m) {
      return (m < n && c < Nc) ? ucol(c)[m] : 0.0f;
    }, [&](int s, const unsigned char* bh) {
      if (nr == 0 || tid >= Nc) return;
#pragma unroll
      for (int g = 0; g < 4; ++g) {
        const uint32_t o = umma_b_off(tid, 4 * g, L.LBO_B);
        const float4 h4 = *reinterpret_cast<const float4*>(bh + o);
        const float4 l4 = *reinterpret_cast<const float4*>(bh + L.szBhalf + o);
        const float u[4] = {h4.x + l4.x, h4.y + l4.y, h4.z + l4.z, h4.w + l4.w};
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          const int m = 16 * s + 4 * g + t;
          if (m < n) {
            const float4* l4p = reinterpret_cast<const float4*>(Lc + m * UM_NRMAX);
#pragma unroll
            for (int r4 = 0; r4 < UM_NRMAX / 4; ++r4) {
              const float4 lc = l4p[r4];
              bacc[4 * r4] = fmaf(lc.x, u[t], bacc[4 * r4]);
              bacc[4 * r4 + 1] = fmaf(lc.y, u[t], bacc[4 * r4 + 1]);
              bacc[4 * r4 + 2] = fmaf(lc.z, u[t], bacc[4 * r4 + 2]);
              bacc[4 * r4 + 3] = fmaf(lc.w, u[t], bacc[4 * r4 + 3]);
            }
          }
        }
      }
    });
    if (!ok) {
      if (tid == 0) report(a.st, DEV_TIMEOUT, j, 1, k);
      break;
    }
    if (nr > 0 && tid < Nc) {
      const int c = tid;
#pragma unroll
      for (int r = 0; r < UM_NRMAX; ++r) {
        if (r < nr) {
          if (c < n) {
            const size_t oc = (size_t)jp * nrn + r + (size_t)c * nr;
            const float cjp = first ? float(a.C0[oc]) : a.C[oc];
            a.C[oc] = cjp - bacc[r];
          } else if (c < n2) {
            a.Rbuf[(size_t)j * nrn + r + (size_t)(c - n) * nr] = -bacc[r];
          } else {
            a.Fbuf[(size_t)j * nrnx + r + (size_t)(c - n2) * nr] = -(double)bacc[r];
          }
        }
      }
    }
    // reduced row out: D'_jp, E'_jp, B'_jp
    {
      float* const Djp = a.D + ojp;
      float* const Ejp = a.E + ojp;
      float* const Bjp = a.B + (size_t)jp * nnx;
      const int qd = warp & 3, grp = warp >> 2, i = 32 * qd + lane;
      for (int pc = grp; pc < L.Npad / 16; pc += UM_NW / 4) {
        float v[16];
        float xb[16];
#pragma unroll
        for (int jj = 0; jj < 16; ++jj) {
          const int c = 16 * pc + jj;
          xb[jj] = (i < n && c < Nc) ? Xs[(size_t)c * n2 + n + i] : 0.0f;
        }
        tmem_ld16(tmem + ((uint32_t)(32 * qd) << 16) + (uint32_t)(16 * pc), v);
        if (i < n) {
#pragma unroll
          for (int jj = 0; jj < 16; ++jj) {
            const int c = 16 * pc + jj;
            if (c >= Nc) continue;
            const float y = xb[jj] - v[jj];
            float* col = c < n ? Djp + (size_t)c * n : c < n2 ? Ejp + (size_t)(c - n) * n : Bjp + (size_t)(c - n2) * n;
            col[i] = y;
          }
        }
      }
    }
    tc_fence_before();
    __syncthreads();
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(UM_TMEM_COLS) : "memory");
}

