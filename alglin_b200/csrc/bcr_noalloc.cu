// Allocation-free matrix-vector product res = alpha*A*x + beta*res for a
// bordered BABD matrix held entirely in caller-owned device memory.
//
// Why it exists: some callers of this library cannot allocate device memory at
// the point where they need the product -- code that runs on a fixed memory
// budget handed out up front (for example a solver embedded in a larger
// application that owns every device allocation through its own pool, or a
// real-time Newton loop that must not call into the CUDA allocator), and code
// that must not synchronise the device, which cudaMalloc and cudaFree may do.
// Those callers keep the matrix blocks, x and res in their own buffers and
// call bcr_mv_noalloc; the library then allocates nothing.
//
// The only scratch the product needs -- the partial sums of the nr border rows,
// one set per CTA of the border reduction -- lives in the file-scope device
// array g_noalloc_scratch below: at most NOALLOC_MAX_PARTS x NOALLOC_MAX_NR
// doubles (512 KiB), held by every GPU that loads the library until the
// process exits.  Each call writes every scratch slot it later reads, so
// nothing has to start at zero; all calls share the array, so calls that
// overlap on the GPU (for example on two streams at once) race on it.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "alglin_b200.h"
#include "bcr_common.cuh"

namespace {

constexpr int NOALLOC_MAX_PARTS = 1024;  // CTAs of the border-row reduction
constexpr int NOALLOC_MAX_NR = 64;       // border rows supported
constexpr int NOALLOC_THREADS = 256;

static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_MAX_PARTS * NOALLOC_MAX_NR];

constexpr int MAX_DEVICES = 64;
std::mutex g_setup_mutex;
double* g_scratch_ptr[MAX_DEVICES] = {};
// the context each cached address belongs to: after a device reset the module
// is loaded again in a new context and the array may move
unsigned long long g_scratch_ctx[MAX_DEVICES] = {};

// driver entry points for the current context's unique id (taken through the
// runtime, so the library needs no link to libcuda)
using PfnCtxGetCurrent = CUresult (*)(CUcontext*);
using PfnCtxGetId = CUresult (*)(CUcontext, unsigned long long*);

// unique id of the calling thread's current context, 0 when unknown
unsigned long long current_ctx_id() {
  static PfnCtxGetCurrent get_current = nullptr;
  static PfnCtxGetId get_id = nullptr;
  static bool looked_up = false;
  if (!looked_up) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<PfnCtxGetCurrent>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<PfnCtxGetId>(f);
    looked_up = true;
  }
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (get_current && get_id && get_current(&ctx) == CUDA_SUCCESS && ctx && get_id(ctx, &id) == CUDA_SUCCESS)
    return id;
  return 0;
}

void set_err(char* buf, int len, const char* msg) {
  if (buf && len > 0) snprintf(buf, (size_t)len, "%s", msg);
}

// block rows: res_i = beta*res_i + alpha*(D_k x_k + E_k x_{k+1} + B_k xb)_i
__global__ void k_noalloc_rows(bcr::Dims d, const double* D, const double* E, const double* B,
                               double alpha, const double* x, double beta, double* res) {
  const int n = d.n, nx = d.nx;
  const size_t rows = (size_t)d.nblock * n;
  const size_t xb = (size_t)(d.nblock + 1) * n + d.qx;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < rows; e += (size_t)gridDim.x * blockDim.x) {
    const size_t k = e / n;
    const int i = (int)(e % n);
    double s = 0.0;
    for (int c = 0; c < n; ++c) s += D[k * n * n + (size_t)c * n + i] * x[k * n + c];
    for (int c = 0; c < n; ++c) s += E[k * n * n + (size_t)c * n + i] * x[(k + 1) * n + c];
    for (int c = 0; c < nx; ++c) s += B[k * n * nx + (size_t)c * n + i] * x[xb + c];
    res[e] = (beta == 0.0 ? 0.0 : beta * res[e]) + alpha * s;
  }
}

// border rows, stage 1: CTA g sums C_k x_k over its fixed chunk of blocks into
// scratch[g*nr + r] (fixed thread-to-block map and shared-memory tree)
__global__ void __launch_bounds__(NOALLOC_THREADS)
k_noalloc_border_parts(bcr::Dims d, const double* C, const double* x, long chunk, double* scratch) {
  __shared__ double red[NOALLOC_THREADS];
  const int n = d.n, nr = d.nr, tid = threadIdx.x;
  const int S = NOALLOC_THREADS / nr, r = tid % nr, g = tid / nr;
  const long b0 = (long)blockIdx.x * chunk;
  const long b1 = min((long)d.nblock + 1, b0 + chunk);
  double acc = 0.0;
  if (g < S)
    for (long k = b0 + g; k < b1; k += S) {
      const double* Ck = C + (size_t)k * nr * n;
      for (int c = 0; c < n; ++c) acc += Ck[(size_t)c * nr + r] * x[(size_t)k * n + c];
    }
  red[tid] = acc;
  __syncthreads();
  for (int w = 1; w < S; w *= 2) {
    if (g < S && g % (2 * w) == 0 && g + w < S) red[tid] += red[tid + w * nr];
    __syncthreads();
  }
  if (g == 0) scratch[(size_t)blockIdx.x * nr + r] = red[r];
}

// H rows and border rows, stage 2 (one CTA): the partials are summed in order
__global__ void k_noalloc_tail(bcr::Dims d, const double* H, const double* Cq, const double* F,
                               const double* scratch, int parts, double alpha, const double* x,
                               double beta, double* res) {
  const int n = d.n, m = n + d.qr, nr = d.nr, qx = d.qx, nx = d.nx, Nc = d.Nc;
  const size_t r0 = (size_t)d.nblock * n;
  const size_t xN = (size_t)d.nblock * n, xq = (size_t)(d.nblock + 1) * n, xb = xq + qx;
  for (int row = threadIdx.x; row < m + nr; row += blockDim.x) {
    double s = 0.0;
    if (row < m) {
      for (int c = 0; c < Nc; ++c) {
        const size_t xi = c < n ? (size_t)c : (c < 2 * n ? xN + (c - n) : xq + (c - 2 * n));
        s += H[(size_t)c * m + row] * x[xi];
      }
    } else {
      const int rr = row - m;
      for (int g = 0; g < parts; ++g) s += scratch[(size_t)g * nr + rr];
      for (int c = 0; c < qx; ++c) s += Cq[(size_t)c * nr + rr] * x[xq + c];
      for (int c = 0; c < nx; ++c) s += F[(size_t)c * nr + rr] * x[xb + c];
    }
    const size_t o = r0 + row;
    res[o] = (beta == 0.0 ? 0.0 : beta * res[o]) + alpha * s;
  }
}

}  // namespace

extern "C" int bcr_mv_noalloc(int nblock, int n, int qr, int qx, int nr, int nx, const double* D,
                              const double* E, const double* B, const double* C, const double* Cq,
                              const double* F, const double* H, double alpha, const double* x,
                              double beta, double* res, void* stream, char* errbuf, int errlen) {
  if (nblock < 1 || n < 1 || qr < 0 || qx < 0 || nr < 0 || nx < 0) {
    set_err(errbuf, errlen, "bcr_mv_noalloc: bad sizes (nblock, n >= 1; qr, qx, nr, nx >= 0)");
    return BCR_BAD_ARGUMENT;
  }
  if (nr > NOALLOC_MAX_NR) {
    char msg[160];
    snprintf(msg, sizeof msg, "bcr_mv_noalloc: nr = %d border rows exceeds the maximum of %d "
             "supported by the fixed scratch array", nr, NOALLOC_MAX_NR);
    set_err(errbuf, errlen, msg);
    return BCR_BAD_ARGUMENT;
  }
  if (!D || !E || !H || !x || !res || (nx > 0 && !B) || (nr > 0 && !C) || (nr > 0 && qx > 0 && !Cq) ||
      (nr > 0 && nx > 0 && !F)) {
    set_err(errbuf, errlen, "bcr_mv_noalloc: a required device pointer is NULL");
    return BCR_BAD_ARGUMENT;
  }
  // An error left pending by earlier work on this thread belongs to its owner:
  // report it without clearing it, and launch nothing.
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess) {
    char msg[200];
    snprintf(msg, sizeof msg, "bcr_mv_noalloc: a CUDA error was already pending before the call: %s",
             cudaGetErrorString(e));
    set_err(errbuf, errlen, msg);
    return BCR_CUDA_ERROR;
  }
  // Set-up, once per device (and again if the device's context was reset),
  // with that device current: the address of the scratch array on this device
  // (the array's host-side name is not a device address).  The first call on
  // each device does this look-up, so it should come before any stream capture.
  int dev = 0;
  e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) {
    set_err(errbuf, errlen, "bcr_mv_noalloc: no usable CUDA device");
    return BCR_CUDA_ERROR;
  }
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    const unsigned long long ctx = current_ctx_id();
    if (!g_scratch_ptr[dev] || ctx == 0 || ctx != g_scratch_ctx[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p) {
        set_err(errbuf, errlen, cudaGetErrorString(e));
        return BCR_CUDA_ERROR;
      }
      g_scratch_ptr[dev] = static_cast<double*>(p);
      g_scratch_ctx[dev] = current_ctx_id();
    }
    scratch = g_scratch_ptr[dev];
  }
  bcr::Dims d{};
  d.nblock = nblock; d.n = n; d.qr = qr; d.qx = qx; d.nr = nr; d.nx = nx;
  d.Nr = 2 * n + nr + qr;
  d.Nc = 2 * n + nx + qx;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const long rows = (long)nblock * n;
  long g = (rows + NOALLOC_THREADS - 1) / NOALLOC_THREADS;
  if (g > 148 * 8) g = 148 * 8;
  k_noalloc_rows<<<(int)g, NOALLOC_THREADS, 0, st>>>(d, D, E, B, alpha, x, beta, res);
  int parts = 0;
  if (nr > 0) {
    const long blocks = (long)nblock + 1;
    const long chunk = (blocks + NOALLOC_MAX_PARTS - 1) / NOALLOC_MAX_PARTS;
    parts = (int)((blocks + chunk - 1) / chunk);  // <= NOALLOC_MAX_PARTS
    k_noalloc_border_parts<<<parts, NOALLOC_THREADS, 0, st>>>(d, C, x, chunk, scratch);
  }
  k_noalloc_tail<<<1, NOALLOC_THREADS, 0, st>>>(d, H, Cq, F, scratch, parts, alpha, x, beta, res);
  e = cudaGetLastError();  // nothing was pending at entry: an error here is this call's
  if (e != cudaSuccess) {
    set_err(errbuf, errlen, cudaGetErrorString(e));
    return BCR_CUDA_ERROR;
  }
  return BCR_OK;
}
