// C ABI of the B200 BorderedCR solver (declarations and reference citations in
// include/alglin_b200.h).  The handle owns a host copy of the loaded matrix in
// the reference layout and the device buffers of the factorization; every
// numerical step runs on the GPU through bcr_kernels.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "alglin_b200.h"
#include "bcr_device.h"

using bcr::Dims;

namespace {

std::string fmt(const char* f, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, f);
  vsnprintf(buf, sizeof buf, f, ap);
  va_end(ap);
  return buf;
}

const char* kInternalName[] = {"CyclicReduction+LU", "CyclicReduction+QR", "CyclicReduction+QRP"};
const char* kLastName[] = {"LastBlock LU", "LastBlock LUPQ", "LastBlock QR", "LastBlock QRP",
                           "LastBlock SVD", "LastBlock LSS", "LastBlock LSY", "LastBlock PINV"};
const char* kLast2Name[] = {"LastBlock NONE", "LastBlock SVD", "LastBlock LSS", "LastBlock LSY",
                            "LastBlock PINV"};

template <typename T>
void dfree(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

template <typename T>
cudaError_t dalloc(T*& p, size_t count) {
  dfree(p);
  return cudaMalloc(reinterpret_cast<void**>(&p), std::max<size_t>(count, 1) * sizeof(T));
}

void gecopy(int m, int n, const double* A, int lda, double* B, int ldb) {
  for (int j = 0; j < n; ++j) std::memcpy(B + (size_t)j * ldb, A + (size_t)j * lda, sizeof(double) * m);
}

void geadd(int m, int n, const double* A, int lda, double* B, int ldb) {
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < m; ++i) B[(size_t)j * ldb + i] += A[(size_t)j * lda + i];
}

}  // namespace

struct bcr_handle_s {
  // construction / partition (kept for info(), hxx:373-423, cc:139-158)
  int nthreads = 0;
  int max_parallel_block = 1;
  int used_parallel_block = 1;
  // sizes
  Dims d{};
  bool allocated = false;
  // selections and flags
  int sel = 0, sel_last = 0, sel_last2 = 0;
  bool fthread = true, sthread = true, debug = false;
  int precision = BCR_PRECISION_FP64;
  int use_tc = 1;  // FP64 tensor-core pair kernel where it applies
  // iterative refinement of the mixed path (FP32 factors, FP64 residuals)
  double ir_tol = 1e-12;
  int ir_max = 10;
  int ir_iters = 0;          // corrections applied by the last solve
  double ir_relres = 0.0;    // max over columns of |b-Ax|/(|A||x|+|b|) after it
  int ir_nrhs = 0;
  bool ir_pending = false;   // the norms of the last solve are still on the device
  std::string err = "no error";
  std::string info_buf;
  // host copy of the loaded matrix (reference layout)
  std::vector<double> hD, hE, hB, hC, hCq, hF, hH;
  // device
  bool dev_ready = false, dirty = true, factorized = false, pending_status = false;
  bcr::DevState s{};
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  // chunked uploads of factorize_solve from host buffers: a copy stream and
  // the events that order its chunks (created on first use)
  static constexpr int NCHUNK_EV = 8;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t chunk_ev[NCHUNK_EV] = {};
  double* dX = nullptr;
  size_t dX_cap = 0;
  double* dY = nullptr;
  size_t dY_cap = 0;
  double* dB = nullptr;      // copy of the right-hand sides (refinement)
  size_t dB_cap = 0;
  double* dR = nullptr;      // residuals / corrections (refinement)
  size_t dR_cap = 0;
  double* dNorm = nullptr;   // [0] |A|_inf, then |r|,|x|,|b| per column (as u64 bits)
  size_t dNorm_cap = 0;
  double* dRow = nullptr;    // row sums of |A|
  size_t dRow_cap = 0;
  bool mixed_ready = false;
  std::vector<void*> pinned;
  cudaGraphExec_t graphs[4] = {nullptr, nullptr, nullptr, nullptr};

  void drop_graphs() {
    for (auto& g : graphs)
      if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  }

  int fail(int code, const std::string& m) {
    err = m;
    return code;
  }
  int L() const { return std::max(nrows(), ncols()); }
  int nrows() const { return d.n * (d.nblock + 1) + d.qr + d.nr; }
  int ncols() const { return d.n * (d.nblock + 1) + d.qx + d.nx; }

  void partition() {
    // cc:139-158: each chunk keeps at least two block rows
    int NBLK = std::max(1, max_parallel_block);
    int used = NBLK, red = 2 * NBLK;
    while (red > d.nblock) { red -= 2; --used; }
    used_parallel_block = used <= 1 ? 1 : used;
  }
  int thread_count() const { return nthreads > 0 ? nthreads : 1; }

  void release_device() {
    if (!dev_ready) return;
    cudaDeviceSynchronize();
    drop_graphs();
    for (void* p : pinned) cudaHostUnregister(p);
    pinned.clear();
    bcr::DevState& z = s;
    dfree(z.D0); dfree(z.E0); dfree(z.B0); dfree(z.C0); dfree(z.Cq); dfree(z.F0); dfree(z.H);
    dfree(z.D); dfree(z.E); dfree(z.B); dfree(z.C); dfree(z.T); dfree(z.P);
    dfree(z.Rbuf); dfree(z.Fbuf); dfree(z.XB); dfree(z.part); dfree(z.Ffin); dfree(z.Hl);
    dfree(z.tau_l); dfree(z.piv_l); dfree(z.st); dfree(z.mv_part); dfree(z.slab); dfree(z.tree_cnt);
    dfree(z.Ul); dfree(z.Vl); dfree(z.Sl); dfree(z.Al);
    dfree(z.Df); dfree(z.Ef); dfree(z.Bf); dfree(z.Cf); dfree(z.Tf); dfree(z.Rbuff);
    dfree(dX); dfree(dY); dfree(dB); dfree(dR); dfree(dNorm); dfree(dRow);
    dX_cap = dY_cap = dB_cap = dR_cap = dNorm_cap = dRow_cap = 0;
    mixed_ready = false;
    ir_pending = false;
    if (own_stream && stream) cudaStreamDestroy(stream);
    if (own_stream) stream = nullptr;
    own_stream = false;
    if (copy_stream) cudaStreamDestroy(copy_stream);
    copy_stream = nullptr;
    for (auto& e : chunk_ev) {
      if (e) cudaEventDestroy(e);
      e = nullptr;
    }
    dev_ready = false;
    dirty = true;
    factorized = false;
  }

  int cuda_fail(cudaError_t e, const char* where) {
    return fail(BCR_CUDA_ERROR, fmt("alglin_b200: CUDA error in %s: %s\n", where, cudaGetErrorString(e)));
  }

  int ensure_device() {
    if (dev_ready) return BCR_OK;
    if (!allocated) return fail(BCR_BAD_ARGUMENT, "BorderedCR: allocate() must be called first\n");
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
      return fail(BCR_CUDA_ERROR, "alglin_b200: no CUDA device is available (the solver has no CPU path)\n");
    if (d.n > 128)
      return fail(BCR_BAD_ARGUMENT,
                  fmt("alglin_b200: block size n=%d exceeds the supported maximum of 128\n", d.n));
    if (!stream) {
      e = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
      if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreate");
      own_stream = true;
    }
    const size_t nb = d.nblock, n = d.n, nr = d.nr, nx = d.nx, qx = d.qx, qr = d.qr;
    const size_t Lmax = std::max(d.Nr, d.Nc);
    bcr::DevState& z = s;
    z.d = d;
    cudaError_t r = cudaSuccess;
    auto A = [&](cudaError_t x) { if (r == cudaSuccess) r = x; };
    A(dalloc(z.D0, nb * n * n)); A(dalloc(z.E0, nb * n * n)); A(dalloc(z.B0, nb * n * nx));
    A(dalloc(z.C0, (nb + 1) * nr * n)); A(dalloc(z.Cq, nr * qx)); A(dalloc(z.F0, nr * nx));
    A(dalloc(z.H, (n + qr) * d.Nc));
    A(dalloc(z.D, nb * n * n)); A(dalloc(z.E, nb * n * n)); A(dalloc(z.B, nb * n * nx));
    A(dalloc(z.C, (nb + 1) * nr * n)); A(dalloc(z.T, nb * (2 * n * n + n))); A(dalloc(z.P, nb * 3 * n));
    A(dalloc(z.Rbuf, nb * nr * n)); A(dalloc(z.Fbuf, nb * nr * nx));
    z.xb_cap = 16;
    A(dalloc(z.XB, nb * nr * 16));
    const size_t parts = (nb + 1 + 1023) / 1024 + 1;
    z.part_cap = (int)(parts * 256);
    A(dalloc(z.part, (size_t)z.part_cap));
    A(dalloc(z.Ffin, std::max<size_t>(nr * nx, 1)));
    A(dalloc(z.Hl, (size_t)d.Nr * d.Nc)); A(dalloc(z.tau_l, Lmax)); A(dalloc(z.piv_l, 2 * Lmax));
    A(dalloc(z.Ul, Lmax * Lmax)); A(dalloc(z.Vl, Lmax * Lmax)); A(dalloc(z.Sl, Lmax));
    A(dalloc(z.Al, (size_t)d.Nr * d.Nc));
    A(dalloc(z.st, 1)); A(dalloc(z.mv_part, (nb + 2) * nr));
    A(dalloc(z.tree_cnt, nb + 1));
    z.slab_elems = bcr::cta_slab_elems(d);
    z.slab_ctas = 148 * 2;  // the CTA-per-pair kernel may be chosen for any n
    if (z.slab_ctas) {
      double* slab = nullptr;
      A(dalloc(slab, z.slab_elems * z.slab_ctas));
      z.slab = slab;
    }
    if (r != cudaSuccess) {
      dev_ready = true;
      release_device();
      return cuda_fail(r, "device allocation");
    }
    // pin the host copy so the per-factorize upload runs at full PCIe rate
    for (std::vector<double>* v : {&hD, &hE, &hB, &hC, &hCq, &hF, &hH})
      if (!v->empty() && cudaHostRegister(v->data(), v->size() * 8, cudaHostRegisterDefault) == cudaSuccess)
        pinned.push_back(v->data());
    cudaGetLastError();
    dev_ready = true;
    dirty = true;
    return BCR_OK;
  }

  int upload() {
    int rc = ensure_device();
    if (rc) return rc;
    bcr::DevState& z = s;
    auto up = [&](double* dst, const std::vector<double>& v) {
      if (!v.empty()) cudaMemcpyAsync(dst, v.data(), v.size() * 8, cudaMemcpyHostToDevice, stream);
    };
    up(z.D0, hD); up(z.E0, hE); up(z.B0, hB); up(z.C0, hC); up(z.Cq, hCq); up(z.F0, hF); up(z.H, hH);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "upload");
    dirty = false;
    return BCR_OK;
  }

  int ensure_buffer(double*& p, size_t& cap, size_t count) {
    if (cap >= count) return BCR_OK;
    cudaStreamSynchronize(stream);
    cudaError_t e = dalloc(p, count);
    if (e != cudaSuccess) { cap = 0; return cuda_fail(e, "scratch allocation"); }
    cap = count;
    return BCR_OK;
  }

  int read_status(bcr::StatusWords& st) {
    cudaError_t e = cudaMemcpyAsync(&st, s.st, sizeof st, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_fail(e, "factorize");
    return BCR_OK;
  }

  // FP32 working arrays of the mixed path, allocated on first use
  int ensure_mixed() {
    if (mixed_ready) return BCR_OK;
    if (nrows() != ncols())
      return fail(BCR_BAD_ARGUMENT,
                  fmt("alglin_b200: the mixed-precision path needs a square system (rows %d, cols %d)\n",
                      nrows(), ncols()));
    const size_t nb = d.nblock, n = d.n, nr = d.nr, nx = d.nx;
    bcr::DevState& z = s;
    cudaStreamSynchronize(stream);
    cudaError_t r = cudaSuccess;
    auto A = [&](cudaError_t x) { if (r == cudaSuccess) r = x; };
    A(dalloc(z.Df, nb * n * n)); A(dalloc(z.Ef, nb * n * n)); A(dalloc(z.Bf, nb * n * nx));
    A(dalloc(z.Cf, (nb + 1) * nr * n)); A(dalloc(z.Tf, nb * (2 * n * n + n)));
    A(dalloc(z.Rbuff, nb * nr * n));
    A(dalloc(dRow, (size_t)std::max(nrows(), 1)));
    dRow_cap = (size_t)std::max(nrows(), 1);
    if (r != cudaSuccess) {
      dfree(z.Df); dfree(z.Ef); dfree(z.Bf); dfree(z.Cf); dfree(z.Tf); dfree(z.Rbuff); dfree(dRow);
      dRow_cap = 0;
      return cuda_fail(r, "mixed-precision allocation");
    }
    mixed_ready = true;
    return BCR_OK;
  }

  // selection state copied into the device state before any launch
  int prepare_launch() {
    s.sel = sel;
    s.sel_last = sel_last;
    s.sel_last2 = sel_last2;
    s.use_tc = use_tc;
    s.mixed = precision == BCR_PRECISION_MIXED ? 1 : 0;
    if (s.mixed) {
      int rc = ensure_mixed();
      if (rc) return rc;
      if (dNorm_cap < 4) {
        rc = ensure_buffer(dNorm, dNorm_cap, 4);
        if (rc) return rc;
      }
    }
    return BCR_OK;
  }

  // the factorization kernels (the mixed path measures |A|_inf in the first
  // residual of each solve)
  void enqueue_factorize() { bcr::launch_factorize(s, stream); }

  int factorize_launch() {
    factorized = false;
    int rc = prepare_launch();
    if (rc) return rc;
    enqueue_factorize();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "factorize launch");
    pending_status = true;
    factorized = true;  // provisional until the status word is read
    return BCR_OK;
  }

  int factorize_solve_launch(int nrhs, double* dx, int ld) {
    factorized = false;
    if (nrhs < 0 || ld < L()) return fail(BCR_BAD_ARGUMENT, fmt("BorderedCR::solve: bad ldRhs = %d\n", ld));
    int rc = prepare_launch();
    if (rc) return rc;
    if (s.mixed) {
      // adaptive refinement needs the factorization's status first
      if (nrhs > 0 && (rc = save_rhs(nrhs, dx, ld))) return rc;
      if (nrhs > 0) bcr::launch_factorize_solve(s, dx, ld, nrhs, stream);  // x0 with the factors
      else enqueue_factorize();
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) return cuda_fail(e, "factorize launch");
      pending_status = true;
      factorized = true;
      if ((rc = factorize_status())) return rc;
      return nrhs > 0 ? solve_mixed(nrhs, dx, ld, -1, true) : BCR_OK;
    }
    if (nrhs == 0) bcr::launch_factorize(s, stream);
    else bcr::launch_factorize_solve(s, dx, ld, nrhs, stream);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "factorize_solve launch");
    pending_status = true;
    factorized = true;
    return BCR_OK;
  }

  int factorize_status() {
    if (!pending_status) return factorized ? BCR_OK : fail(BCR_NUMERICAL, err);
    pending_status = false;
    bcr::StatusWords st{};
    int rc = read_status(st);
    if (rc) { factorized = false; return rc; }
    factorized = false;
    if (st.code == bcr::DEV_ZERO_PIVOT) {
      const int n = d.n;
      if (sel == bcr::SEL_LU)
        return fail(BCR_NUMERICAL, fmt("BorderedCR::buildT [LU] getrf(M=%d,N=%d,A,LDA=%d,iperm)::INFO = %d\n",
                                       2 * n, n, 2 * n, st.info));
      return fail(BCR_NUMERICAL, fmt("BorderedCR::buildT [%s] singular R factor at block %d (column %d)\n",
                                     sel == bcr::SEL_QR ? "QR" : "QRP", st.block, st.info));
    }
    if (st.code == bcr::DEV_LAST_SINGULAR || st.code == bcr::DEV_BAD_SHAPE)
      return fail(BCR_NUMERICAL, "BorderedCR<t_Value>::load_and_factorize_last failed\n");
    if (st.code == bcr::DEV_TIMEOUT)
      return fail(BCR_DEVICE_TIMEOUT, fmt("BorderedCR: tensor-core pipeline wait expired at block %d, level %d\n",
                                      st.block, st.level));
    factorized = true;
    return BCR_OK;
  }

  int factorize_device() {
    int rc = factorize_launch();
    if (rc) return rc;
    return factorize_status();
  }

  // |b-Ax|/(|A||x|+|b|), max over the columns of the last mixed solve
  int read_refinement() {
    if (!ir_pending) return BCR_OK;
    ir_pending = false;
    std::vector<unsigned long long> w(1 + 3 * (size_t)ir_nrhs);
    cudaError_t e = cudaMemcpyAsync(w.data(), dNorm, w.size() * 8, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_fail(e, "refinement norms");
    auto as_d = [](unsigned long long u) { double v; std::memcpy(&v, &u, 8); return v; };
    const double nA = as_d(w[0]);
    double worst = 0.0;
    for (int c = 0; c < ir_nrhs; ++c) {
      const double nr_ = as_d(w[1 + 3 * c]), nx_ = as_d(w[2 + 3 * c]), nb_ = as_d(w[3 + 3 * c]);
      const double den = nA * nx_ + nb_;
      double rr = den > 0 ? nr_ / den : (nr_ > 0 ? INFINITY : 0.0);
      if (!(rr <= worst)) worst = rr;  // NaN wins
    }
    ir_relres = worst;
    return BCR_OK;
  }

  // mixed path: the right-hand sides b kept in dB while x0 = A^-1 b is formed
  // in place
  int save_rhs(int nrhs, double* dx, int ld) {
    const size_t Lx = (size_t)L(), nrw = (size_t)nrows();
    int rc = ensure_buffer(dB, dB_cap, Lx * nrhs);
    if (rc) return rc;
    cudaMemcpy2DAsync(dB, Lx * 8, dx, (size_t)ld * 8, nrw * 8, nrhs, cudaMemcpyDeviceToDevice, stream);
    return BCR_OK;
  }
  // mixed factorize + solve on the device: b saved, x0 from the factorization
  // (which carries the first forward elimination where the pair kernel can),
  // then the refinement for exactly `fixed` steps (graph capture)
  int factorize_solve_mixed(int nrhs, double* dx, int ld, int fixed) {
    int rc = save_rhs(nrhs, dx, ld);
    if (rc) return rc;
    bcr::launch_factorize_solve(s, dx, ld, nrhs, stream);
    return solve_mixed(nrhs, dx, ld, fixed, true);
  }
  // mixed path: x = A^-1 b with FP32 factors (unless x0_done: x holds it and
  // dB holds b), then corrections d = A^-1 r from FP64 residuals r = b - Ax
  // until |r|/(|A||x|+|b|) <= ir_tol (adaptive: the host reads the norms after
  // every residual) or for exactly `fixed` steps (graph capture: no host
  // synchronisation)
  int solve_mixed(int nrhs, double* dx, int ld, int fixed, bool x0_done = false) {
    const size_t Lx = (size_t)L(), ncl = (size_t)ncols();
    int rc;
    if (!x0_done && (rc = save_rhs(nrhs, dx, ld))) return rc;
    if ((rc = ensure_buffer(dR, dR_cap, Lx * nrhs))) return rc;
    if ((rc = ensure_buffer(dNorm, dNorm_cap, 1 + 3 * (size_t)nrhs))) return rc;
    auto* norms = reinterpret_cast<unsigned long long*>(dNorm);
    if (!x0_done) bcr::launch_solve(s, dx, ld, nrhs, stream);
    ir_nrhs = nrhs;
    int it = 0;
    for (;;) {
      for (int c = 0; c < nrhs; ++c) {
        const bool with_A = it == 0 && c == 0;  // |A|_inf into norms[0] from this pass
        bcr::launch_residual(s, dB + c * Lx, dx + (size_t)c * ld, dR + c * Lx, norms + 1 + 3 * c, stream,
                             with_A ? dRow : nullptr, with_A ? norms : nullptr);
      }
      if (fixed < 0) {
        ir_pending = true;
        if ((rc = read_refinement())) return rc;
        if (ir_relres <= ir_tol || it >= ir_max) break;
      } else if (it >= fixed) {
        ir_pending = true;
        break;
      }
      bcr::launch_solve(s, dR, (int)Lx, nrhs, stream);
      for (int c = 0; c < nrhs; ++c) bcr::launch_axpy(dx + (size_t)c * ld, dR + c * Lx, (long)ncl, stream);
      ++it;
    }
    ir_iters = it;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "refinement launch");
    return BCR_OK;
  }

  int solve_device(int nrhs, double* dx, int ld, int fixed = -1) {
    if (!factorized) return fail(BCR_NUMERICAL, "BorderedCR::solve: the matrix is not factorized\n");
    if (nrhs < 0 || ld < L()) return fail(BCR_BAD_ARGUMENT, fmt("BorderedCR::solve: bad ldRhs = %d\n", ld));
    if (nrhs == 0) return BCR_OK;
    if (s.mixed) {
      if (pending_status) {
        int rc = factorize_status();
        if (rc) return rc;
      }
      return solve_mixed(nrhs, dx, ld, fixed);
    }
    bcr::launch_solve(s, dx, ld, nrhs, stream);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "solve launch");
    return BCR_OK;
  }

  int solve_host(int nrhs, double* x, int ld) {
    if (pending_status) {
      int rc = factorize_status();
      if (rc) return rc;
    }
    if (!factorized) return fail(BCR_NUMERICAL, "BorderedCR::solve: the matrix is not factorized\n");
    if (nrhs < 0 || ld < L()) return fail(BCR_BAD_ARGUMENT, fmt("BorderedCR::solve: bad ldRhs = %d\n", ld));
    if (nrhs == 0) return BCR_OK;
    const size_t Lx = (size_t)L();
    int rc = ensure_buffer(dX, dX_cap, Lx * nrhs);
    if (rc) return rc;
    cudaMemcpy2DAsync(dX, Lx * 8, x, (size_t)ld * 8, Lx * 8, nrhs, cudaMemcpyHostToDevice, stream);
    rc = solve_device(nrhs, dX, (int)Lx);
    if (rc) return rc;
    cudaMemcpy2DAsync(x, (size_t)ld * 8, dX, Lx * 8, Lx * 8, nrhs, cudaMemcpyDeviceToHost, stream);
    cudaError_t e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_fail(e, "solve");
    return BCR_OK;
  }

  // --------------------------------------------------------------- check ---
  int check_matrix() {
    // cc:2538-2659
    const int n = d.n, nb = d.nblock;
    auto scan = [&](const std::vector<double>& v, int NR, int NC, int nblk, const char* name,
                    bool blocked) -> int {
      const size_t SB = (size_t)NR * NC;
      for (size_t i = 0; i < SB * nblk; ++i)
        if (!std::isfinite(v[i])) {
          const size_t b = i / SB, w = i - b * SB;
          if (blocked)
            return fail(BCR_BAD_ARGUMENT,
                        fmt("BorderedCR::check_matrix, found %g at block %zu position (%zu,%zu) of %dx%d matrix %s\n",
                            v[i], b, w % NR, w / NR, NR, NC, name));
          return fail(BCR_BAD_ARGUMENT,
                      fmt("BorderedCR::check_matrix, found %g at position (%zu,%zu) of %dx%d matrix %s\n",
                          v[i], w % NR, w / NR, NR, NC, name));
        }
      return BCR_OK;
    };
    int rc;
    if ((rc = scan(hH, n + d.qr, d.Nc, 1, "H0Hqp", false))) return rc;
    if ((rc = scan(hB, n, d.nx, nb, "B", true))) return rc;
    if ((rc = scan(hC, d.nr, n, nb + 1, "C", true))) return rc;
    if ((rc = scan(hCq, d.nr, d.qx, 1, "Cq", false))) return rc;
    if ((rc = scan(hD, n, n, nb, "D", true))) return rc;
    if ((rc = scan(hE, n, n, nb, "E", true))) return rc;
    if ((rc = scan(hF, d.nr, d.nx, 1, "F", false))) return rc;
    return BCR_OK;
  }
};

#define H_CHECK(h)                                    \
  do {                                                \
    if (!(h)) return BCR_BAD_ARGUMENT;                \
  } while (0)
#define H_ALLOC(h)                                                                   \
  do {                                                                               \
    H_CHECK(h);                                                                      \
    if (!(h)->allocated) return (h)->fail(BCR_BAD_ARGUMENT, "BorderedCR: allocate() must be called first\n"); \
  } while (0)
#define NBL_CHECK(h, nbl, hi, what)                                                            \
  do {                                                                                         \
    if ((nbl) < 0 || (nbl) > (hi))                                                             \
      return (h)->fail(BCR_BAD_ARGUMENT, fmt("BorderedCR::%s( %d, ...) block index out of range\n", what, nbl)); \
  } while (0)
#define LD_CHECK(h, ld, rows, what)                                                                    \
  do {                                                                                                 \
    if ((ld) < (rows))                                                                                 \
      return (h)->fail(BCR_BAD_ARGUMENT, fmt("BorderedCR::%s, bad leading dimension %d < %d\n", what, ld, rows)); \
  } while (0)

extern "C" {

int bcr_create(bcr_handle* out, int num_threads, int num_parallel_block) {
  if (!out) return BCR_BAD_ARGUMENT;
  auto* h = new bcr_handle_s;
  h->nthreads = num_threads > 0 ? num_threads : 0;
  if (h->nthreads > 0)
    h->max_parallel_block = num_parallel_block == 0 ? h->nthreads : std::min(h->nthreads, num_parallel_block);
  else
    h->max_parallel_block = 1;
  *out = h;
  return BCR_OK;
}

int bcr_destroy(bcr_handle h) {
  if (!h) return BCR_OK;
  h->release_device();
  delete h;
  return BCR_OK;
}

int bcr_allocate(bcr_handle h, int nblock, int n, int qr, int qx, int nr, int nx) {
  H_CHECK(h);
  if (nblock < 1 || n < 1 || qr < 0 || qx < 0 || nr < 0 || nx < 0)
    return h->fail(BCR_BAD_ARGUMENT, fmt("BorderedCR::allocate( nblock=%d, n=%d, qr=%d, qx=%d, nr=%d, nx=%d ) bad sizes\n",
                                         nblock, n, qr, qx, nr, nx));
  if (h->allocated && h->d.nblock == nblock && h->d.n == n && h->d.qr == qr && h->d.qx == qx &&
      h->d.nr == nr && h->d.nx == nx) {
    h->partition();
    return BCR_OK;  // cc:55-61
  }
  h->release_device();
  Dims d{};  // (release_device also drops captured graphs)
  d.nblock = nblock; d.n = n; d.qr = qr; d.qx = qx; d.nr = nr; d.nx = nx;
  d.Nr = 2 * n + nr + qr;
  d.Nc = 2 * n + nx + qx;
  h->d = d;
  const size_t nb = nblock;
  h->hD.assign(nb * n * n, 0.0);
  h->hE.assign(nb * n * n, 0.0);
  h->hB.assign(nb * n * nx, 0.0);
  h->hC.assign((nb + 1) * nr * n, 0.0);
  h->hCq.assign((size_t)nr * qx, 0.0);
  h->hF.assign((size_t)nr * nx, 0.0);
  h->hH.assign((size_t)(n + qr) * d.Nc, 0.0);
  h->allocated = true;
  h->dirty = true;
  h->factorized = false;
  h->partition();
  return BCR_OK;
}

int bcr_dup(bcr_handle dst, bcr_handle src) {
  H_CHECK(dst);
  H_ALLOC(src);
  dst->max_parallel_block = src->max_parallel_block;
  int rc = bcr_allocate(dst, src->d.nblock, src->d.n, src->d.qr, src->d.qx, src->d.nr, src->d.nx);
  if (rc) return rc;
  dst->hD = src->hD; dst->hE = src->hE; dst->hB = src->hB; dst->hC = src->hC;
  dst->hCq = src->hCq; dst->hF = src->hF; dst->hH = src->hH;
  if (dst->dev_ready) dst->release_device();  // host vectors were replaced: re-pin lazily
  dst->nthreads = 0;  // cc:197: the copy runs on the inline pool
  dst->dirty = true;
  dst->factorized = false;
  return BCR_OK;
}

int bcr_nrows(bcr_handle h) { return h ? h->nrows() : 0; }
int bcr_ncols(bcr_handle h) { return h ? h->ncols() : 0; }
int bcr_number_of_blocks(bcr_handle h) { return h ? h->d.nblock : 0; }
int bcr_block_size(bcr_handle h) { return h ? h->d.n : 0; }
int bcr_dim_qr(bcr_handle h) { return h ? h->d.qr : 0; }
int bcr_dim_qx(bcr_handle h) { return h ? h->d.qx : 0; }
int bcr_dim_nr(bcr_handle h) { return h ? h->d.nr : 0; }
int bcr_dim_nx(bcr_handle h) { return h ? h->d.nx : 0; }
int bcr_Nr(bcr_handle h) { return h ? h->d.Nr : 0; }
int bcr_Nc(bcr_handle h) { return h ? h->d.Nc : 0; }

#define ZERO_FN(name, vec)                                 \
  int name(bcr_handle h) {                                 \
    H_ALLOC(h);                                            \
    std::fill(h->vec.begin(), h->vec.end(), 0.0);          \
    h->dirty = true;                                       \
    return BCR_OK;                                         \
  }
ZERO_FN(bcr_zero_B, hB)
ZERO_FN(bcr_zero_C, hC)
ZERO_FN(bcr_zero_Cq, hCq)
ZERO_FN(bcr_zero_D, hD)
ZERO_FN(bcr_zero_E, hE)
ZERO_FN(bcr_zero_F, hF)
ZERO_FN(bcr_zero_H, hH)
#undef ZERO_FN

int bcr_fill_zero(bcr_handle h) {
  H_ALLOC(h);
  bcr_zero_B(h); bcr_zero_C(h); bcr_zero_Cq(h); bcr_zero_D(h); bcr_zero_E(h); bcr_zero_F(h); bcr_zero_H(h);
  return BCR_OK;
}

int bcr_load_B(bcr_handle h, int nbl, const double* B, int ldB) {
  H_ALLOC(h);
  NBL_CHECK(h, nbl, h->d.nblock - 1, "load_B");
  LD_CHECK(h, ldB, h->d.n, "load_B");
  const int n = h->d.n, nx = h->d.nx;
  gecopy(n, nx, B, ldB, h->hB.data() + (size_t)nbl * n * nx, n);
  h->dirty = true;
  return BCR_OK;
}

int bcr_add_to_B(bcr_handle h, int nbl, const double* B, int ldB) {
  H_ALLOC(h);
  NBL_CHECK(h, nbl, h->d.nblock - 1, "add_to_B");
  LD_CHECK(h, ldB, h->d.n, "add_to_B");
  const int n = h->d.n, nx = h->d.nx;
  geadd(n, nx, B, ldB, h->hB.data() + (size_t)nbl * n * nx, n);
  h->dirty = true;
  return BCR_OK;
}

int bcr_load_C(bcr_handle h, int nbl, const double* C, int ldC) {
  H_ALLOC(h);
  NBL_CHECK(h, nbl, h->d.nblock, "load_C");
  LD_CHECK(h, ldC, h->d.nr, "load_C");
  const int n = h->d.n, nr = h->d.nr;
  gecopy(nr, n, C, ldC, h->hC.data() + (size_t)nbl * nr * n, nr);
  h->dirty = true;
  return BCR_OK;
}

int bcr_add_to_C(bcr_handle h, int nbl, const double* C, int ldC) {
  H_ALLOC(h);
  NBL_CHECK(h, nbl, h->d.nblock, "add_to_C");
  if (ldC < h->d.nr) return h->fail(BCR_BAD_ARGUMENT, fmt("BorderedCR::add_to_C( %d, C, ldC = %d ) bad ldC\n", nbl, ldC));
  const int n = h->d.n, nr = h->d.nr;
  geadd(nr, n, C, ldC, h->hC.data() + (size_t)nbl * nr * n, nr);
  h->dirty = true;
  return BCR_OK;
}

int bcr_add_to_C2(bcr_handle h, int nbl, const double* C, int ldC) {
  H_ALLOC(h);
  NBL_CHECK(h, nbl, h->d.nblock - 1, "add_to_C2");
  if (ldC < h->d.nr) return h->fail(BCR_BAD_ARGUMENT, fmt("BorderedCR::add_to_C2( %d, C, ldC = %d ) bad ldC\n", nbl, ldC));
  const int n = h->d.n, nr = h->d.nr;
  geadd(nr, 2 * n, C, ldC, h->hC.data() + (size_t)nbl * nr * n, nr);
  h->dirty = true;
  return BCR_OK;
}

int bcr_add_to_C2F(bcr_handle h, int nbl, const double* C2F, int ldC) {
  H_ALLOC(h);
  NBL_CHECK(h, nbl, h->d.nblock - 1, "add_to_C2F");
  if (ldC < h->d.nr) return h->fail(BCR_BAD_ARGUMENT, fmt("BorderedCR::add_to_C2F( %d, C2F, ldC = %d ) bad ldC\n", nbl, ldC));
  const int n = h->d.n, nr = h->d.nr, nx = h->d.nx;
  geadd(nr, 2 * n, C2F, ldC, h->hC.data() + (size_t)nbl * nr * n, nr);
  geadd(nr, nx, C2F + (size_t)ldC * 2 * n, ldC, h->hF.data(), nr);
  h->dirty = true;
  return BCR_OK;
}

int bcr_load_D(bcr_handle h, int nbl, const double* D, int ldD) {
  H_ALLOC(h);
  NBL_CHECK(h, nbl, h->d.nblock - 1, "load_D");
  LD_CHECK(h, ldD, h->d.n, "load_D");
  const int n = h->d.n;
  gecopy(n, n, D, ldD, h->hD.data() + (size_t)nbl * n * n, n);
  h->dirty = true;
  return BCR_OK;
}

int bcr_load_E(bcr_handle h, int nbl, const double* E, int ldE) {
  H_ALLOC(h);
  NBL_CHECK(h, nbl, h->d.nblock - 1, "load_E");
  LD_CHECK(h, ldE, h->d.n, "load_E");
  const int n = h->d.n;
  gecopy(n, n, E, ldE, h->hE.data() + (size_t)nbl * n * n, n);
  h->dirty = true;
  return BCR_OK;
}

int bcr_load_DE(bcr_handle h, int nbl, const double* DE, int ldDE) {
  H_ALLOC(h);
  NBL_CHECK(h, nbl, h->d.nblock - 1, "load_DE");
  LD_CHECK(h, ldDE, h->d.n, "load_DE");
  const int n = h->d.n;
  gecopy(n, n, DE, ldDE, h->hD.data() + (size_t)nbl * n * n, n);
  gecopy(n, n, DE + (size_t)n * ldDE, ldDE, h->hE.data() + (size_t)nbl * n * n, n);
  h->dirty = true;
  return BCR_OK;
}

int bcr_load_DEB(bcr_handle h, int nbl, const double* DEB, int ldDEB) {
  H_ALLOC(h);
  NBL_CHECK(h, nbl, h->d.nblock - 1, "load_DEB");
  LD_CHECK(h, ldDEB, h->d.n, "load_DEB");
  const int n = h->d.n, nx = h->d.nx;
  gecopy(n, n, DEB, ldDEB, h->hD.data() + (size_t)nbl * n * n, n);
  gecopy(n, n, DEB + (size_t)n * ldDEB, ldDEB, h->hE.data() + (size_t)nbl * n * n, n);
  gecopy(n, nx, DEB + (size_t)2 * n * ldDEB, ldDEB, h->hB.data() + (size_t)nbl * n * nx, n);
  h->dirty = true;
  return BCR_OK;
}

int bcr_load_F(bcr_handle h, const double* F, int ldF) {
  H_ALLOC(h);
  LD_CHECK(h, ldF, h->d.nr, "load_F");
  gecopy(h->d.nr, h->d.nx, F, ldF, h->hF.data(), h->d.nr);
  h->dirty = true;
  return BCR_OK;
}

int bcr_add_to_F(bcr_handle h, const double* F, int ldF) {
  H_ALLOC(h);
  LD_CHECK(h, ldF, h->d.nr, "add_to_F");
  geadd(h->d.nr, h->d.nx, F, ldF, h->hF.data(), h->d.nr);
  h->dirty = true;
  return BCR_OK;
}

int bcr_load_Cq(bcr_handle h, const double* Cq, int ldC) {
  H_ALLOC(h);
  LD_CHECK(h, ldC, h->d.nr, "load_Cq");
  gecopy(h->d.nr, h->d.qx, Cq, ldC, h->hCq.data(), h->d.nr);
  h->dirty = true;
  return BCR_OK;
}

int bcr_load_CqF(bcr_handle h, const double* CqF, int ldCF) {
  H_ALLOC(h);
  LD_CHECK(h, ldCF, h->d.nr, "load_CqF");
  const int nr = h->d.nr, qx = h->d.qx, nx = h->d.nx;
  gecopy(nr, qx, CqF, ldCF, h->hCq.data(), nr);
  gecopy(nr, nx, CqF + (size_t)qx * ldCF, ldCF, h->hF.data(), nr);
  h->dirty = true;
  return BCR_OK;
}

int bcr_load_bottom(bcr_handle h, const double* H0, int ld0, const double* HN, int ldN,
                    const double* Hq, int ldQ, const double* Hp, int ldP) {
  H_ALLOC(h);
  const int n = h->d.n, m = n + h->d.qr;
  LD_CHECK(h, ld0, m, "load_bottom");
  LD_CHECK(h, ldN, m, "load_bottom");
  if (h->d.qx) LD_CHECK(h, ldQ, m, "load_bottom");
  if (h->d.nx) LD_CHECK(h, ldP, m, "load_bottom");
  double* H = h->hH.data();
  gecopy(m, n, H0, ld0, H, m); H += (size_t)m * n;
  gecopy(m, n, HN, ldN, H, m); H += (size_t)m * n;
  gecopy(m, h->d.qx, Hq, ldQ, H, m); H += (size_t)m * h->d.qx;
  gecopy(m, h->d.nx, Hp, ldP, H, m);
  h->dirty = true;
  return BCR_OK;
}

int bcr_load_bottom_H(bcr_handle h, const double* Hm, int ldH) {
  H_ALLOC(h);
  const int m = h->d.n + h->d.qr;
  LD_CHECK(h, ldH, m, "load_bottom");
  gecopy(m, h->d.Nc, Hm, ldH, h->hH.data(), m);
  h->dirty = true;
  return BCR_OK;
}

int bcr_load_bottom2(bcr_handle h, const double* C0, int ld0, const double* CN, int ldN,
                     const double* Cq, int ldCq, const double* F, int ldF) {
  H_ALLOC(h);
  const int n = h->d.n, nr = h->d.nr;
  if (nr == 0) return BCR_OK;
  LD_CHECK(h, ld0, nr, "load_bottom2");
  LD_CHECK(h, ldN, nr, "load_bottom2");
  gecopy(nr, n, C0, ld0, h->hC.data(), nr);
  gecopy(nr, n, CN, ldN, h->hC.data() + (size_t)h->d.nblock * nr * n, nr);
  if (h->d.qx) { LD_CHECK(h, ldCq, nr, "load_bottom2"); gecopy(nr, h->d.qx, Cq, ldCq, h->hCq.data(), nr); }
  if (h->d.nx) { LD_CHECK(h, ldF, nr, "load_bottom2"); gecopy(nr, h->d.nx, F, ldF, h->hF.data(), nr); }
  h->dirty = true;
  return BCR_OK;
}

int bcr_load_bottom2_H(bcr_handle h, const double* P, int ld) {
  H_ALLOC(h);
  const int n = h->d.n, nr = h->d.nr;
  if (nr == 0) return BCR_OK;
  LD_CHECK(h, ld, nr, "load_bottom2");
  gecopy(nr, n, P, ld, h->hC.data(), nr); P += (size_t)ld * n;
  gecopy(nr, n, P, ld, h->hC.data() + (size_t)h->d.nblock * nr * n, nr); P += (size_t)ld * n;
  gecopy(nr, h->d.qx, P, ld, h->hCq.data(), nr); P += (size_t)ld * h->d.qx;
  gecopy(nr, h->d.nx, P, ld, h->hF.data(), nr);
  h->dirty = true;
  return BCR_OK;
}

double* bcr_block_data(bcr_handle h, char which, int nbl) {
  if (!h || !h->allocated) return nullptr;
  const Dims& d = h->d;
  h->dirty = true;  // the caller may write through the pointer
  switch (which) {
    case 'B': return nbl >= 0 && nbl < d.nblock ? h->hB.data() + (size_t)nbl * d.n * d.nx : nullptr;
    case 'C': return nbl >= 0 && nbl <= d.nblock ? h->hC.data() + (size_t)nbl * d.nr * d.n : nullptr;
    case 'D': return nbl >= 0 && nbl < d.nblock ? h->hD.data() + (size_t)nbl * d.n * d.n : nullptr;
    case 'E': return nbl >= 0 && nbl < d.nblock ? h->hE.data() + (size_t)nbl * d.n * d.n : nullptr;
    case 'F': return h->hF.data();
    case 'Q': return h->hCq.data();
    case 'H': return h->hH.data();
    default: return nullptr;
  }
}

int bcr_select(bcr_handle h, const char* c) {
  H_CHECK(h);
  std::string s = c ? c : "";
  if (s == "LU") h->sel = 0;
  else if (s == "QR") h->sel = 1;
  else if (s == "QRP") h->sel = 2;
  else
    return h->fail(BCR_BAD_ARGUMENT, fmt("BorderedCR::select( choice='%s' )\nunknown/unsupported factorization type ('LU','QR','QRP')", s.c_str()));
  h->factorized = false;
  return BCR_OK;
}

int bcr_select_last(bcr_handle h, const char* c) {
  H_CHECK(h);
  std::string s = c ? c : "";
  static const char* names[] = {"LU", "LUPQ", "QR", "QRP", "SVD", "LSS", "LSY", "PINV"};
  for (int i = 0; i < 8; ++i)
    if (s == names[i]) { h->sel_last = i; h->factorized = false; return BCR_OK; }
  return h->fail(BCR_BAD_ARGUMENT, fmt("BorderedCR::select_last( choice='%s' )\nunknown/unsupported factorization type ('LU','LUPQ','QR','QRP','SVD','LSS','LSY','PINV')", s.c_str()));
}

int bcr_select_last2(bcr_handle h, const char* c) {
  H_CHECK(h);
  std::string s = c ? c : "";
  static const char* names[] = {"NONE", "SVD", "LSS", "LSY", "PINV"};
  for (int i = 0; i < 5; ++i)
    if (s == names[i]) { h->sel_last2 = i; h->factorized = false; return BCR_OK; }
  return h->fail(BCR_BAD_ARGUMENT, fmt("BorderedCR::select_last2( choice='%s' )\nunknown/unsupported factorization type ('NONE','SVD','LSS','LSY','PINV')", s.c_str()));
}

int bcr_selected(bcr_handle h, int* internal, int* last, int* last2) {
  H_CHECK(h);
  if (internal) *internal = h->sel;
  if (last) *last = h->sel_last;
  if (last2) *last2 = h->sel_last2;
  return BCR_OK;
}

int bcr_set_factorize_use_thread(bcr_handle h, int yes) { H_CHECK(h); h->fthread = yes != 0; return BCR_OK; }
int bcr_set_solve_use_thread(bcr_handle h, int yes) { H_CHECK(h); h->sthread = yes != 0; return BCR_OK; }
int bcr_factorize_use_thread(bcr_handle h) { return h && h->fthread ? 1 : 0; }
int bcr_solve_use_thread(bcr_handle h) { return h && h->sthread ? 1 : 0; }

int bcr_set_num_parallel_block(bcr_handle h, int npb) {
  H_CHECK(h);
  h->max_parallel_block = std::max(1, std::min(h->thread_count(), npb));  // hxx:407-423
  h->partition();
  return BCR_OK;
}

int bcr_set_precision(bcr_handle h, int p) {
  H_CHECK(h);
  if (p != BCR_PRECISION_FP64 && p != BCR_PRECISION_MIXED)
    return h->fail(BCR_BAD_ARGUMENT, fmt("BorderedCR::set_precision( %d ) unknown precision\n", p));
  h->precision = p;
  h->factorized = false;
  return BCR_OK;
}

const char* bcr_info(bcr_handle h, const char* indent) {
  if (!h) return "";
  const char* in = indent ? indent : "";
  h->info_buf = fmt(
      "%srows   = %d\n%scols   = %d\n%snblock = %d\n%sn      = %d\n%sqr     = %d\n%sqx     = %d\n"
      "%snr     = %d\n%snx     = %d\n%streads = %d/nblk:%d/factorize:%s/solve:%s\n"
      "%sintern = %s\n%slast   = %s\n%slast2  = %s\n",
      in, h->nrows(), in, h->ncols(), in, h->d.nblock, in, h->d.n, in, h->d.qr, in, h->d.qx, in,
      h->d.nr, in, h->d.nx, in, h->thread_count(), h->used_parallel_block, h->fthread ? "true" : "false",
      h->sthread ? "true" : "false", in, kInternalName[h->sel], in, kLastName[h->sel_last], in,
      kLast2Name[h->sel_last2]);
  return h->info_buf.c_str();
}

const char* bcr_last_error(bcr_handle h) { return h ? h->err.c_str() : "invalid handle"; }

int bcr_set_debug(bcr_handle h, int yes) { H_CHECK(h); h->debug = yes != 0; return BCR_OK; }

int bcr_check_matrix(bcr_handle h) {
  H_ALLOC(h);
  return h->check_matrix();
}

int bcr_factorize(bcr_handle h) {
  H_ALLOC(h);
  if (h->debug) {
    int rc = h->check_matrix();
    if (rc) return rc;
  }
  int rc = h->upload();
  if (rc) return rc;
  return h->factorize_device();
}

int bcr_solve(bcr_handle h, double* x) {
  H_ALLOC(h);
  return h->solve_host(1, x, h->L());
}

int bcr_solve_n(bcr_handle h, int nrhs, double* rhs, int ldRhs) {
  H_ALLOC(h);
  return h->solve_host(nrhs, rhs, ldRhs);
}

int bcr_t_solve(bcr_handle h, double*) {
  H_CHECK(h);
  return h->fail(BCR_BAD_ARGUMENT, "BorderedCR::t_solve() not defined\n");
}

int bcr_t_solve_n(bcr_handle h, int, double*, int) {
  H_CHECK(h);
  return h->fail(BCR_BAD_ARGUMENT, "BorderedCR::t_solve() not defined\n");
}

static int mv_host(bcr_handle h, double alpha, const double* x, double beta, double* res) {
  int rc = h->ensure_device();
  if (rc) return rc;
  if (h->dirty && (rc = h->upload())) return rc;
  const size_t nc = h->ncols(), nrw = h->nrows();
  if ((rc = h->ensure_buffer(h->dX, h->dX_cap, std::max(nc, (size_t)1)))) return rc;
  if ((rc = h->ensure_buffer(h->dY, h->dY_cap, std::max(nrw, (size_t)1)))) return rc;
  cudaMemcpyAsync(h->dX, x, nc * 8, cudaMemcpyHostToDevice, h->stream);
  if (beta != 0.0) cudaMemcpyAsync(h->dY, res, nrw * 8, cudaMemcpyHostToDevice, h->stream);
  bcr::launch_mv(h->s, alpha, h->dX, beta, h->dY, h->stream);
  cudaMemcpyAsync(res, h->dY, nrw * 8, cudaMemcpyDeviceToHost, h->stream);
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, "Mv");
  return BCR_OK;
}

int bcr_mv(bcr_handle h, const double* x, double* res) {
  H_ALLOC(h);
  return mv_host(h, 1.0, x, 0.0, res);
}

int bcr_add_mv(bcr_handle h, double alpha, const double* x, double* res) {
  H_ALLOC(h);
  return mv_host(h, alpha, x, 1.0, res);
}

// ----------------------------------------------------------------- sparse ---
int bcr_sparse_nnz(bcr_handle h) {
  if (!h) return 0;
  const Dims& d = h->d;
  return d.n * d.nblock * (2 * d.n + d.nx + d.nr) + d.nr * (d.n + d.qx + d.nx) + (d.n + d.qr) * (2 * d.n + d.qx + d.nx);
}

int bcr_sparse_pattern(bcr_handle h, int* I, int* J, int offs) {
  H_ALLOC(h);
  const Dims& d = h->d;
  const int n = d.n, nb = d.nblock, nr = d.nr, nx = d.nx, qr = d.qr, qx = d.qx;
  int k = 0;
  for (int nbl = 0; nbl < nb; ++nbl) {
    for (int ij = 0; ij < n * n; ++ij) { I[k] = nbl * n + offs + ij % n; J[k] = nbl * n + offs + ij / n; ++k; }
    for (int ij = 0; ij < n * n; ++ij) { I[k] = nbl * n + offs + ij % n; J[k] = (nbl + 1) * n + offs + ij / n; ++k; }
    for (int ij = 0; ij < n * nx; ++ij) { I[k] = nbl * n + offs + ij % n; J[k] = (nb + 1) * n + qx + offs + ij / n; ++k; }
  }
  const int nqr = n + qr;
  for (int ij = 0; ij < nqr * d.Nc; ++ij) {
    int i = ij % nqr, j = ij / nqr;
    I[k] = nb * n + i + offs;
    if (j >= n) j += nb * n - n;
    J[k] = j + offs;
    ++k;
  }
  for (int nbl = 0; nbl <= nb; ++nbl)
    for (int ij = 0; ij < nr * n; ++ij) { I[k] = (nb + 1) * n + qr + offs + ij % nr; J[k] = nbl * n + offs + ij / nr; ++k; }
  for (int ij = 0; ij < nr * qx; ++ij) { I[k] = (nb + 1) * n + qr + offs + ij % nr; J[k] = (nb + 1) * n + offs + ij / nr; ++k; }
  for (int ij = 0; ij < nr * nx; ++ij) { I[k] = (nb + 1) * n + qr + offs + ij % nr; J[k] = (nb + 1) * n + qx + offs + ij / nr; ++k; }
  if (k != bcr_sparse_nnz(h))
    return h->fail(BCR_BAD_ARGUMENT, fmt("BorderedCR::sparse_pattern( I, J, offs ), inserted %d values, expected %d\n", k, bcr_sparse_nnz(h)));
  return BCR_OK;
}

int bcr_sparse_values(bcr_handle h, double* V) {
  H_ALLOC(h);
  const Dims& d = h->d;
  const size_t n = d.n, nx = d.nx, nr = d.nr;
  size_t k = 0;
  for (int nbl = 0; nbl < d.nblock; ++nbl) {
    std::memcpy(V + k, h->hD.data() + nbl * n * n, n * n * 8); k += n * n;
    std::memcpy(V + k, h->hE.data() + nbl * n * n, n * n * 8); k += n * n;
    std::memcpy(V + k, h->hB.data() + nbl * n * nx, n * nx * 8); k += n * nx;
  }
  std::memcpy(V + k, h->hH.data(), h->hH.size() * 8); k += h->hH.size();
  std::memcpy(V + k, h->hC.data(), h->hC.size() * 8); k += h->hC.size();
  std::memcpy(V + k, h->hCq.data(), h->hCq.size() * 8); k += h->hCq.size();
  std::memcpy(V + k, h->hF.data(), nr * nx * 8); k += nr * nx;
  return BCR_OK;
}

int bcr_sparse_load(bcr_handle h, const double* V, const int* I, int r_offs, const int* J, int c_offs,
                    int nnz, int do_error) {
  H_ALLOC(h);
  // cc:2419-2482
  const Dims& d = h->d;
  const int n = d.n, nb = d.nblock;
  const int rH = n * nb, rC = rH + n + d.qr, nrow = rC + d.nr;
  const int cCq = rH + n, cF = cCq + d.qx, ncol = cF + d.nx;
  bcr_fill_zero(h);
  int status = BCR_OK;
  for (int kk = 0; kk < nnz; ++kk) {
    const int i = I[kk] - r_offs, j = J[kk] - c_offs;
    const double v = V[kk];
    const int ib = i / n, jb = j / n;
    bool ok = true;
    if (i < 0 || j < 0) ok = false;
    else if (i < rH) {
      if (j < cCq) {
        if (ib == jb) h->hD[(size_t)ib * n * n + (i % n) + (size_t)(j % n) * n] = v;
        else if (ib + 1 == jb) h->hE[(size_t)ib * n * n + (i % n) + (size_t)(j % n) * n] = v;
        else ok = false;
      } else if (j < cF) ok = false;
      else if (j < ncol) h->hB[(size_t)ib * n * d.nx + (i % n) + (size_t)(j - cF) * n] = v;
      else ok = false;
    } else if (i < rC) {
      const int m = n + d.qr;
      if (j < n) h->hH[(i - rH) + (size_t)j * m] = v;
      else if (j < rH) ok = false;
      else if (j < ncol) h->hH[(i - rH) + (size_t)(j - rH + n) * m] = v;
      else ok = false;
    } else if (i < nrow) {
      if (j < cCq) h->hC[(size_t)jb * d.nr * n + (i - rC) + (size_t)(j % n) * d.nr] = v;
      else if (j < cF) h->hCq[(i - rC) + (size_t)(j - cCq) * d.nr] = v;
      else if (j < ncol) h->hF[(i - rC) + (size_t)(j - cF) * d.nr] = v;
      else ok = false;
    } else ok = false;
    if (!ok) {
      h->err = fmt("in BorderedCR<t_Value>::sparse_load, indices (i,j) = ( %d, %d) out of pattern!\n", I[kk], J[kk]);
      if (do_error) return BCR_BAD_ARGUMENT;
      status = BCR_OK;
    }
  }
  h->dirty = true;
  return status;
}

// ------------------------------------------------------- device-resident ---
int bcr_set_stream(bcr_handle h, void* stream) {
  H_CHECK(h);
  if (h->own_stream && h->stream) {
    cudaStreamSynchronize(h->stream);
    cudaStreamDestroy(h->stream);
  }
  h->own_stream = false;
  h->stream = static_cast<cudaStream_t>(stream);
  return BCR_OK;
}

int bcr_upload(bcr_handle h) {
  H_ALLOC(h);
  int rc = h->upload();
  if (rc) return rc;
  cudaError_t e = cudaStreamSynchronize(h->stream);
  return e == cudaSuccess ? BCR_OK : h->cuda_fail(e, "upload");
}

int bcr_factorize_device(bcr_handle h) {
  H_ALLOC(h);
  int rc = h->ensure_device();
  if (rc) return rc;
  if (h->dirty && (rc = h->upload())) return rc;
  return h->factorize_device();
}

int bcr_factorize_async(bcr_handle h) {
  H_ALLOC(h);
  int rc = h->ensure_device();
  if (rc) return rc;
  if (h->dirty && (rc = h->upload())) return rc;
  return h->factorize_launch();
}

int bcr_factorize_status(bcr_handle h) {
  H_ALLOC(h);
  return h->factorize_status();
}

int bcr_factorize_solve(bcr_handle h, int nrhs, double* rhs, int ldRhs) {
  H_ALLOC(h);
  if (h->debug) {
    int rc = h->check_matrix();
    if (rc) return rc;
  }
  if (nrhs < 0 || ldRhs < h->L()) return h->fail(BCR_BAD_ARGUMENT, fmt("BorderedCR::solve: bad ldRhs = %d\n", ldRhs));
  int rc = h->ensure_device();
  if (rc) return rc;
  const size_t Lx = (size_t)h->L();
  // the FP64 n = 8/16 path overlaps the upload of the matrix with the
  // factorization of the chunks already on the device
  if (nrhs > 0 && h->precision == BCR_PRECISION_FP64) {
    if ((rc = h->ensure_buffer(h->dX, h->dX_cap, Lx * nrhs))) return rc;
    if ((rc = h->prepare_launch())) return rc;
    if (!h->copy_stream) {
      if (cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking) != cudaSuccess) h->copy_stream = nullptr;
      for (auto& e : h->chunk_ev)
        if (h->copy_stream && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) e = nullptr;
    }
    bool evs = h->copy_stream != nullptr;
    for (auto e : h->chunk_ev) evs = evs && e;
    if (evs) {
      cudaMemcpy2DAsync(h->dX, Lx * 8, rhs, (size_t)ldRhs * 8, Lx * 8, nrhs, cudaMemcpyHostToDevice, h->stream);
      // the copy stream starts after the previous use of the matrix arrays
      cudaEventRecord(h->chunk_ev[0], h->stream);
      cudaStreamWaitEvent(h->copy_stream, h->chunk_ev[0], 0);
      const bcr::HostMatrix hm{h->hD.data(), h->hE.data(), h->hB.data(), h->hC.data(), h->hCq.data(),
                               h->hF.data(), h->hH.data()};
      h->factorized = false;
      if (bcr::launch_upload_factorize_solve(h->s, hm, h->dX, (int)Lx, nrhs, h->stream, h->copy_stream,
                                             h->chunk_ev, bcr_handle_s::NCHUNK_EV)) {
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return h->cuda_fail(e, "factorize_solve launch");
        h->dirty = false;
        h->pending_status = true;
        h->factorized = true;
        cudaMemcpy2DAsync(rhs, (size_t)ldRhs * 8, h->dX, Lx * 8, Lx * 8, nrhs, cudaMemcpyDeviceToHost, h->stream);
        return h->factorize_status();
      }
    }
  }
  rc = h->upload();
  if (rc) return rc;
  if (nrhs > 0) {
    if ((rc = h->ensure_buffer(h->dX, h->dX_cap, Lx * nrhs))) return rc;
    cudaMemcpy2DAsync(h->dX, Lx * 8, rhs, (size_t)ldRhs * 8, Lx * 8, nrhs, cudaMemcpyHostToDevice, h->stream);
  }
  if ((rc = h->factorize_solve_launch(nrhs, h->dX, (int)Lx))) return rc;
  if (nrhs > 0)
    cudaMemcpy2DAsync(rhs, (size_t)ldRhs * 8, h->dX, Lx * 8, Lx * 8, nrhs, cudaMemcpyDeviceToHost, h->stream);
  return h->factorize_status();
}

int bcr_factorize_solve_device(bcr_handle h, int nrhs, double* d_x, int ld) {
  H_ALLOC(h);
  int rc = h->ensure_device();
  if (rc) return rc;
  if (h->dirty && (rc = h->upload())) return rc;
  return h->factorize_solve_launch(nrhs, d_x, ld);
}

int bcr_solve_device(bcr_handle h, int nrhs, double* d_x, int ld) {
  H_ALLOC(h);
  return h->solve_device(nrhs, d_x, ld);
}

int bcr_mv_device(bcr_handle h, double alpha, const double* d_x, double beta, double* d_res) {
  H_ALLOC(h);
  int rc = h->ensure_device();
  if (rc) return rc;
  if (h->dirty && (rc = h->upload())) return rc;
  bcr::launch_mv(h->s, alpha, d_x, beta, d_res, h->stream);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? BCR_OK : h->cuda_fail(e, "Mv launch");
}

void* bcr_get_stream(bcr_handle h) {
  if (!h || !h->allocated) return nullptr;
  if (h->ensure_device()) return nullptr;
  return h->stream;
}

int bcr_graph_capture(bcr_handle h, int what, int nrhs, double* d_x, int ld, const double* d_rhs) {
  H_ALLOC(h);
  if (what < BCR_GRAPH_FACTORIZE || what > BCR_GRAPH_STEP)
    return h->fail(BCR_BAD_ARGUMENT, fmt("bcr_graph_capture: unknown graph kind %d\n", what));
  int rc = h->ensure_device();
  if (rc) return rc;
  if (h->dirty && (rc = h->upload())) return rc;
  if ((what & BCR_GRAPH_SOLVE) && (nrhs < 1 || ld < h->L() || !d_x))
    return h->fail(BCR_BAD_ARGUMENT, "bcr_graph_capture: bad right-hand-side buffer\n");
  // one eager run first: it validates the selection and sets kernel attributes
  // (a mixed step runs exactly what the graph will, so that the graph replays
  // the number of corrections this run needed)
  if (what == BCR_GRAPH_STEP && h->s.mixed) {
    if (d_rhs) cudaMemcpyAsync(d_x, d_rhs, (size_t)ld * nrhs * 8, cudaMemcpyDeviceToDevice, h->stream);
    if ((rc = h->factorize_solve_launch(nrhs, d_x, ld))) return rc;
  } else {
    if (what & BCR_GRAPH_FACTORIZE) {
      if ((rc = h->factorize_device())) return rc;
    } else if (!h->factorized) {
      return h->fail(BCR_NUMERICAL, "bcr_graph_capture: factorize before capturing a solve\n");
    }
    if (what & BCR_GRAPH_SOLVE) {
      if (d_rhs) cudaMemcpyAsync(d_x, d_rhs, (size_t)ld * nrhs * 8, cudaMemcpyDeviceToDevice, h->stream);
      if ((rc = h->solve_device(nrhs, d_x, ld))) return rc;
    }
  }
  // the mixed path's graph replays the refinement steps the eager run needed
  const int ir_steps = h->ir_iters;
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, "graph warm-up");
  if (h->graphs[what]) { cudaGraphExecDestroy(h->graphs[what]); h->graphs[what] = nullptr; }
  e = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeRelaxed);
  if (e != cudaSuccess) return h->cuda_fail(e, "cudaStreamBeginCapture");
  const bool mixed = h->s.mixed != 0;
  if (what == BCR_GRAPH_STEP) {
    if (d_rhs) cudaMemcpyAsync(d_x, d_rhs, (size_t)ld * nrhs * 8, cudaMemcpyDeviceToDevice, h->stream);
    if (mixed) {
      rc = h->factorize_solve_mixed(nrhs, d_x, ld, ir_steps);
    } else {
      bcr::launch_factorize_solve(h->s, d_x, ld, nrhs, h->stream);
    }
  } else if (what == BCR_GRAPH_FACTORIZE) {
    h->enqueue_factorize();
  } else {
    if (d_rhs) cudaMemcpyAsync(d_x, d_rhs, (size_t)ld * nrhs * 8, cudaMemcpyDeviceToDevice, h->stream);
    if (mixed) rc = h->solve_mixed(nrhs, d_x, ld, ir_steps);
    else bcr::launch_solve(h->s, d_x, ld, nrhs, h->stream);
  }
  h->ir_pending = false;
  cudaGraph_t graph = nullptr;
  e = cudaStreamEndCapture(h->stream, &graph);
  if (e != cudaSuccess) { cudaGetLastError(); return h->cuda_fail(e, "cudaStreamEndCapture"); }
  if (rc) { cudaGraphDestroy(graph); return rc; }
  e = cudaGraphInstantiate(&h->graphs[what], graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) { h->graphs[what] = nullptr; return h->cuda_fail(e, "cudaGraphInstantiate"); }
  return BCR_OK;
}

int bcr_graph_launch(bcr_handle h, int what) {
  H_ALLOC(h);
  if (what < BCR_GRAPH_FACTORIZE || what > BCR_GRAPH_STEP || !h->graphs[what])
    return h->fail(BCR_BAD_ARGUMENT, "bcr_graph_launch: graph not captured\n");
  cudaError_t e = cudaGraphLaunch(h->graphs[what], h->stream);
  if (e != cudaSuccess) return h->cuda_fail(e, "cudaGraphLaunch");
  if (what & BCR_GRAPH_FACTORIZE) { h->pending_status = true; h->factorized = true; }
  if ((what & BCR_GRAPH_SOLVE) && h->s.mixed) h->ir_pending = true;
  return BCR_OK;
}

int bcr_set_pair_kernel(bcr_handle h, int choice) {
  H_CHECK(h);
  if (choice < BCR_PAIR_AUTO || choice > BCR_PAIR_TC_GATHER)
    return h->fail(BCR_BAD_ARGUMENT, fmt("bcr_set_pair_kernel: unknown choice %d\n", choice));
  h->s.pair_kernel = choice;
  h->drop_graphs();
  h->factorized = false;
  return BCR_OK;
}

int bcr_set_refinement(bcr_handle h, double tol, int max_iter) {
  H_CHECK(h);
  if (!(tol >= 0.0) || max_iter < 0)
    return h->fail(BCR_BAD_ARGUMENT, fmt("bcr_set_refinement: bad tolerance %g or iteration limit %d\n", tol, max_iter));
  h->ir_tol = tol;
  h->ir_max = max_iter;
  return BCR_OK;
}

int bcr_refinement_info(bcr_handle h, int* iters, double* relres) {
  H_CHECK(h);
  int rc = h->read_refinement();
  if (rc) return rc;
  if (iters) *iters = h->s.mixed ? h->ir_iters : 0;
  if (relres) *relres = h->s.mixed ? h->ir_relres : 0.0;
  return BCR_OK;
}

int bcr_synchronize(bcr_handle h) {
  H_CHECK(h);
  if (!h->stream) return BCR_OK;
  cudaError_t e = cudaStreamSynchronize(h->stream);
  return e == cudaSuccess ? BCR_OK : h->cuda_fail(e, "synchronize");
}

}  // extern "C"

// ===================================================================== batch
// Many independent BorderedCR systems solved together.  The handles are host
// containers (their loaders fill the host mirrors); the batch packs every
// system into one device arena for the loaded matrices and one for the
// working arrays, groups the systems by pair-kernel instance, and runs each
// level of every system of a group in one launch.
namespace {

// per-system norm slots of the mixed batch (see kb_residual): |A|, |r|, |x|,
// |b|, the relative residual, two block-row maxima, one spare
constexpr int NRM_SLOTS = 8;

struct BatchTune {
  int n, nrm, nxm, mixed, persist, fam, chunk;  // shape, precision, schedule -> choice
};
std::vector<BatchTune> g_batch_tuning;  // in-process autotuner cache

int default_family(const Dims& d, bool mixed) {
  if ((d.n == 8 || d.n == 16) && bcr::batch_family_ok(bcr::PAIR_TC, d, mixed)) return bcr::PAIR_TC;
  if ((d.n == 32 || (mixed && d.n == 16)) && bcr::batch_family_ok(bcr::PAIR_GRP, d, mixed)) return bcr::PAIR_GRP;
  if (bcr::batch_family_ok(bcr::PAIR_ROWS, d, mixed)) return bcr::PAIR_ROWS;
  return -1;
}

struct Bump {
  size_t top = 0;
  size_t take(size_t bytes) {
    const size_t o = top;
    top += (bytes + 255) & ~size_t(255);
    return o;
  }
};

}  // namespace

struct bcr_batch_s {
  std::vector<bcr_handle> hs;      // null for a system that lives only on the device
  std::vector<Dims> dims;          // per system
  std::vector<int> last_sel;       // per system: last-block solver
  std::vector<size_t> in_len;      // per system: bytes of its loaded matrix in d_in
  std::vector<bcr::DevState> sys;
  std::vector<bcr::BatchClass> cls;
  std::vector<std::vector<int>> members;
  std::vector<int> cls_of;
  unsigned char* d_in = nullptr;   // loaded matrices of every system
  unsigned char* d_work = nullptr; // working arrays, factors, last blocks
  double* h_in = nullptr;          // pinned staging of d_in
  size_t in_bytes = 0, work_bytes = 0;
  std::vector<size_t> in_off;      // per system: byte offset of its D0 in d_in
  double* d_x = nullptr;           // right-hand sides / solutions, packed
  double* d_b = nullptr;           // copy of the right-hand sides (graph replay)
  double* h_x = nullptr;           // pinned staging of d_x
  std::vector<size_t> x_off;       // per system: element offset in d_x
  size_t x_elems = 0;
  bcr::StatusWords* d_st = nullptr;
  std::vector<bcr::StatusWords> h_st;
  // mixed path: FP32 working arrays, refined solutions, per-system norms
  int schedule = BCR_BATCH_LEVELS;  // factorization: one launch per level, or one persistent launch
  int precision = BCR_PRECISION_FP64;
  double ir_tol = 1e-12;
  // corrections after the first sweep compacted maps of the systems still
  // refining, so each extra pass costs about one solve of those systems
  int ir_max = 30;
  int ir_iters = 0;
  double ir_worst = 0.0;
  bool ir_pending = false;
  double* d_sol = nullptr;             // refined solutions, same packing as d_x
  double* d_nrm = nullptr;             // NRM_SLOTS per system: |A|, |r|, |x|, |b|, relative residual, block-row maxima
  int* d_done = nullptr;               // per system: refinement converged
  unsigned long long* d_worst = nullptr;
  cudaStream_t stream = nullptr;
  // one stream per class: a phase of the step (factorize, solve, a
  // refinement pass) forks from `stream` into the classes and joins back, so
  // the classes' launches overlap (they share no device memory but the
  // batch-worst word, which they update atomically)
  std::vector<cudaStream_t> cls_stream;
  std::vector<cudaEvent_t> cls_done;
  cudaEvent_t fork_ev = nullptr;
  cudaGraphExec_t graph = nullptr;
  bool prepared = false, factorized = false;
  std::string err = "no error";

  int fail(int code, const std::string& m) {
    err = m;
    return code;
  }
  int cuda_fail(cudaError_t e, const char* where) {
    return fail(BCR_CUDA_ERROR, fmt("alglin_b200 batch: CUDA error in %s: %s\n", where, cudaGetErrorString(e)));
  }

  void release() {
    if (stream) cudaStreamSynchronize(stream);
    if (graph) { cudaGraphExecDestroy(graph); graph = nullptr; }
    for (cudaStream_t q : cls_stream) cudaStreamDestroy(q);
    for (cudaEvent_t ev : cls_done) cudaEventDestroy(ev);
    if (fork_ev) cudaEventDestroy(fork_ev);
    cls_stream.clear();
    cls_done.clear();
    fork_ev = nullptr;
    for (auto& c : cls) bcr::batch_free(c);
    cls.clear();
    members.clear();
    if (d_in) cudaFree(d_in);
    if (d_work) cudaFree(d_work);
    if (d_x) cudaFree(d_x);
    if (d_b) cudaFree(d_b);
    if (d_st) cudaFree(d_st);
    if (d_sol) cudaFree(d_sol);
    if (d_nrm) cudaFree(d_nrm);
    if (d_worst) cudaFree(d_worst);
    if (d_done) cudaFree(d_done);
    d_done = nullptr;
    d_sol = d_nrm = nullptr;
    d_worst = nullptr;
    ir_pending = false;
    if (h_in) cudaFreeHost(h_in);
    if (h_x) cudaFreeHost(h_x);
    d_in = d_work = nullptr;
    d_x = d_b = h_in = h_x = nullptr;
    d_st = nullptr;
    prepared = factorized = false;
  }

  int L(size_t i) const { return std::max(dims[i].n * (dims[i].nblock + 1) + dims[i].qr + dims[i].nr,
                                          dims[i].n * (dims[i].nblock + 1) + dims[i].qx + dims[i].nx); }

  // pack every handle's host mirrors into the pinned staging buffer
  void pack_inputs() {
    for (size_t i = 0; i < hs.size(); ++i) {
      bcr_handle h = hs[i];
      if (!h) continue;
      unsigned char* base = reinterpret_cast<unsigned char*>(h_in);
      const bcr::DevState& s = sys[i];
      auto put = [&](const double* dev, const std::vector<double>& v) {
        if (!v.empty())
          std::memcpy(base + (reinterpret_cast<const unsigned char*>(dev) - d_in), v.data(), v.size() * 8);
      };
      put(s.D0, h->hD); put(s.E0, h->hE); put(s.B0, h->hB); put(s.C0, h->hC);
      put(s.Cq, h->hCq); put(s.F0, h->hF); put(s.H, h->hH);
    }
  }

  // one copy per run of consecutive handle systems (device-only systems keep
  // what the caller wrote into their part of the arena)
  int upload_inputs() {
    if (!h_in) return BCR_OK;
    pack_inputs();
    cudaError_t e = cudaSuccess;
    for (size_t i = 0; i < hs.size() && e == cudaSuccess;) {
      if (!hs[i]) { ++i; continue; }
      size_t j = i;
      while (j + 1 < hs.size() && hs[j + 1]) ++j;
      const size_t b0 = in_off[i], b1 = in_off[j] + in_len[j];
      e = cudaMemcpyAsync(d_in + b0, reinterpret_cast<unsigned char*>(h_in) + b0, b1 - b0,
                          cudaMemcpyHostToDevice, stream);
      i = j + 1;
    }
    return e == cudaSuccess ? BCR_OK : cuda_fail(e, "matrix upload");
  }

  int prepare(int autotune);
  int tune_class(size_t c);
  // fn(class, its stream) for every class: forked from `stream` and joined
  // back into it (all on `stream` when there is one class or no class streams)
  template <typename F>
  void per_class(F&& fn) {
    if (cls.size() < 2 || cls_stream.size() != cls.size()) {
      for (auto& c : cls) fn(c, stream);
      return;
    }
    cudaEventRecord(fork_ev, stream);
    for (size_t c = 0; c < cls.size(); ++c) {
      cudaStreamWaitEvent(cls_stream[c], fork_ev, 0);
      fn(cls[c], cls_stream[c]);
      cudaEventRecord(cls_done[c], cls_stream[c]);
    }
    for (size_t c = 0; c < cls.size(); ++c) cudaStreamWaitEvent(stream, cls_done[c], 0);
  }
  int make_class_streams() {
    for (size_t c = 0; c < cls.size() && cls.size() > 1; ++c) {
      cudaStream_t q = nullptr;
      cudaEvent_t ev = nullptr;
      if (cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking) != cudaSuccess) return 1;
      cls_stream.push_back(q);
      if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return 1;
      cls_done.push_back(ev);
    }
    if (cls.size() > 1 && cudaEventCreateWithFlags(&fork_ev, cudaEventDisableTiming) != cudaSuccess) return 1;
    return 0;
  }
  void enqueue_factorize() {
    per_class([](bcr::BatchClass& c, cudaStream_t q) { bcr::batch_factorize(c, q); });
  }
  void enqueue_solve() {
    per_class([](bcr::BatchClass& c, cudaStream_t q) { bcr::batch_solve(c, q); });
  }
  bool mixed() const { return precision == BCR_PRECISION_MIXED; }
  // the worst relative residual of the last mixed solve
  int read_worst() {
    if (!ir_pending) return BCR_OK;
    ir_pending = false;
    unsigned long long w = 0;
    cudaError_t e = cudaMemcpyAsync(&w, d_worst, 8, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_fail(e, "batch refinement norms");
    std::memcpy(&ir_worst, &w, 8);
    return BCR_OK;
  }
  // mixed path: x = A^-1 b with the FP32 factors into the solution region,
  // then corrections from FP64 residuals (each solved in place in the rhs
  // region) until the worst system is under ir_tol (adaptive: the host reads
  // the batch-worst norm after each residual) or for exactly `fixed` steps;
  // the refined solutions end in the rhs region
  int solve_mixed(int fixed, bool with_A) {
    cudaMemsetAsync(d_done, 0, hs.size() * sizeof(int), stream);  // every system solves x0
    cudaMemsetAsync(d_nrm, 0, hs.size() * NRM_SLOTS * sizeof(double), stream);
    enqueue_solve();
    cudaMemcpyAsync(d_sol, d_x, x_elems * 8, cudaMemcpyDeviceToDevice, stream);
    int it = 0;
    for (;;) {
      cudaMemsetAsync(d_worst, 0, 8, stream);
      // after the first, the residual covers the systems just corrected
      const int wa = with_A && it == 0 ? 1 : 0;
      per_class([&](bcr::BatchClass& c, cudaStream_t q) { bcr::batch_residual(c, wa, ir_tol, d_worst, q, it > 0); });
      ir_pending = true;
      if (fixed < 0) {
        int rc = read_worst();
        if (rc) return rc;
        if (ir_worst <= ir_tol || it >= ir_max) break;
      } else if (it >= fixed) {
        break;
      }
      // the correction solve covers only the systems still refining
      per_class([](bcr::BatchClass& c, cudaStream_t q) {
        bcr::batch_compact(c, q);
        bcr::batch_solve(c, q, true);
        bcr::batch_correct(c, q);
      });
      ++it;
    }
    cudaMemcpyAsync(d_x, d_sol, x_elems * 8, cudaMemcpyDeviceToDevice, stream);
    ir_iters = it;
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? BCR_OK : cuda_fail(e, "batch refinement");
  }
  // the solve step after a factorization, on the rhs region (b kept in d_b)
  int solve_step(int fixed) {
    if (!mixed()) {
      enqueue_solve();
      cudaError_t e = cudaGetLastError();
      return e == cudaSuccess ? BCR_OK : cuda_fail(e, "batch solve");
    }
    return solve_mixed(fixed, true);
  }
  int read_status() {
    cudaError_t e = cudaMemcpyAsync(h_st.data(), d_st, h_st.size() * sizeof(bcr::StatusWords),
                                    cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_fail(e, "batch status");
    for (size_t i = 0; i < h_st.size(); ++i)
      if (h_st[i].code != 0) {
        factorized = false;
        return fail(BCR_NUMERICAL,
                    fmt("batch system %zu: factorization failed (code %d, block %d, info %d)\n", i,
                        h_st[i].code, h_st[i].block, h_st[i].info));
      }
    factorized = true;
    return BCR_OK;
  }
};

int bcr_batch_s::prepare(int autotune) {
  release();
  if (hs.empty()) return fail(BCR_BAD_ARGUMENT, "bcr_batch_prepare: the batch is empty\n");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(BCR_CUDA_ERROR, "alglin_b200: no CUDA device is available (the solver has no CPU path)\n");
  if (!stream) {
    cudaError_t e = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreate");
  }
  const size_t ns = hs.size();
  sys.assign(ns, bcr::DevState{});
  dims.resize(ns);
  last_sel.resize(ns);
  in_off.assign(ns, 0);
  x_off.assign(ns, 0);
  cls_of.assign(ns, -1);
  // ---------------------------------------------------------- validation
  std::vector<int> fam(ns);
  bool any_handle = false;
  for (size_t i = 0; i < ns; ++i) {
    bcr_handle h = hs[i];
    if (h) {
      any_handle = true;
      if (!h->allocated) return fail(BCR_BAD_ARGUMENT, fmt("batch system %zu: allocate() was not called\n", i));
      if (h->sel != bcr::SEL_LU)
        return fail(BCR_BAD_ARGUMENT, fmt("batch system %zu: batches support the internal LU selection only\n", i));
      if (h->precision != BCR_PRECISION_FP64)
        return fail(BCR_BAD_ARGUMENT, fmt("batch system %zu: batches run in FP64\n", i));
      dims[i] = h->d;
      last_sel[i] = h->sel_last;
    }
    if (mixed() && dims[i].Nr != dims[i].Nc)
      return fail(BCR_BAD_ARGUMENT, fmt("batch system %zu: the mixed-precision path needs a square system\n", i));
    fam[i] = default_family(dims[i], mixed());
    if (fam[i] < 0)
      return fail(BCR_BAD_ARGUMENT,
                  fmt("batch system %zu: block size n=%d with nr=%d, nx=%d has no batched pair kernel\n", i,
                      dims[i].n, dims[i].nr, dims[i].nx));
  }
  // ------------------------------------------------------------ layout
  Bump in, work;
  struct Off { size_t D0, E0, B0, C0, Cq, F0, H, D, E, B, C, T, P, Rbuf, Fbuf, XB, Ffin, Hl, tau, piv, U, V, S; };
  std::vector<Off> off(ns);
  in_len.assign(ns, 0);
  for (size_t i = 0; i < ns; ++i) {
    const Dims& d = dims[i];
    const size_t nb = d.nblock, n = d.n, nr = d.nr, nx = d.nx, qx = d.qx, qr = d.qr;
    const size_t Lb = std::max(d.Nr, d.Nc);
    Off& o = off[i];
    o.D0 = in.take(nb * n * n * 8); o.E0 = in.take(nb * n * n * 8); o.B0 = in.take(nb * n * nx * 8);
    o.C0 = in.take((nb + 1) * nr * n * 8); o.Cq = in.take(nr * qx * 8); o.F0 = in.take(nr * nx * 8);
    o.H = in.take((n + qr) * d.Nc * 8);
    in_len[i] = in.top - o.D0;
    const size_t ws = mixed() ? 4 : 8;  // bytes of a working element
    o.D = work.take(nb * n * n * ws); o.E = work.take(nb * n * n * ws); o.B = work.take(nb * n * nx * ws);
    o.C = work.take((nb + 1) * nr * n * ws); o.T = work.take(nb * (2 * n * n + n) * ws);
    o.P = work.take(nb * 3 * n); o.Rbuf = work.take(nb * nr * n * ws); o.Fbuf = work.take(nb * nr * nx * 8);
    o.XB = work.take(nb * nr * 8); o.Ffin = work.take(std::max<size_t>(nr * nx, 1) * 8);
    o.Hl = work.take((size_t)d.Nr * d.Nc * 8); o.tau = work.take(Lb * 8); o.piv = work.take(2 * Lb * 4);
    const bool svd = last_sel[i] >= bcr::LAST_SVD;  // the SVD family needs U, V, S
    o.U = svd ? work.take(Lb * Lb * 8) : 0;
    o.V = svd ? work.take(Lb * Lb * 8) : 0;
    o.S = svd ? work.take(Lb * 8) : 0;
    x_off[i] = x_elems;
    x_elems += ((size_t)L(i) + 31) & ~size_t(31);
  }
  in_bytes = std::max<size_t>(in.top, 256);
  work_bytes = std::max<size_t>(work.top, 256);
  cudaError_t e = cudaMalloc(&d_in, in_bytes);
  if (e == cudaSuccess) e = cudaMalloc(&d_work, work_bytes);
  if (e == cudaSuccess) e = cudaMalloc(&d_x, std::max<size_t>(x_elems, 1) * 8);
  if (e == cudaSuccess) e = cudaMalloc(&d_b, std::max<size_t>(x_elems, 1) * 8);
  if (e == cudaSuccess) e = cudaMalloc(&d_st, ns * sizeof(bcr::StatusWords));
  if (e == cudaSuccess && mixed()) e = cudaMalloc(&d_sol, std::max<size_t>(x_elems, 1) * 8);
  if (e == cudaSuccess && mixed()) e = cudaMalloc(&d_nrm, ns * NRM_SLOTS * sizeof(double));
  if (e == cudaSuccess && mixed()) e = cudaMalloc(&d_done, ns * sizeof(int));
  if (e == cudaSuccess && mixed()) e = cudaMalloc(&d_worst, 8);
  if (e == cudaSuccess && any_handle) e = cudaMallocHost(&h_in, in_bytes);
  if (e == cudaSuccess) e = cudaMallocHost(&h_x, std::max<size_t>(x_elems, 1) * 8);
  if (e != cudaSuccess) {
    cudaGetLastError();
    release();
    return cuda_fail(e, "batch allocation");
  }
  if (h_in) std::memset(h_in, 0, in_bytes);
  cudaMemsetAsync(d_in, 0, in_bytes, stream);
  cudaMemsetAsync(d_x, 0, std::max<size_t>(x_elems, 1) * 8, stream);  // the padding between systems stays zero
  cudaMemsetAsync(d_b, 0, std::max<size_t>(x_elems, 1) * 8, stream);
  std::memset(h_x, 0, std::max<size_t>(x_elems, 1) * 8);
  h_st.assign(ns, bcr::StatusWords{});
  for (size_t i = 0; i < ns; ++i) {
    const Off& o = off[i];
    bcr::DevState& s = sys[i];
    auto I = [&](size_t b) { return reinterpret_cast<double*>(d_in + b); };
    auto W = [&](size_t b) { return reinterpret_cast<double*>(d_work + b); };
    s.d = dims[i];
    s.sel = bcr::SEL_LU;
    s.sel_last = last_sel[i];
    s.D0 = I(o.D0); s.E0 = I(o.E0); s.B0 = I(o.B0); s.C0 = I(o.C0); s.Cq = I(o.Cq); s.F0 = I(o.F0); s.H = I(o.H);
    s.mixed = mixed() ? 1 : 0;
    if (mixed()) {
      auto F = [&](size_t b) { return reinterpret_cast<float*>(d_work + b); };
      s.Df = F(o.D); s.Ef = F(o.E); s.Bf = F(o.B); s.Cf = F(o.C); s.Tf = F(o.T); s.Rbuff = F(o.Rbuf);
      s.bsol = d_sol + x_off[i];
      s.bb = d_b + x_off[i];
      s.bnrm = d_nrm + NRM_SLOTS * i;
      s.bdone = d_done + i;
    } else {
      s.D = W(o.D); s.E = W(o.E); s.B = W(o.B); s.C = W(o.C); s.T = W(o.T);
      s.Rbuf = W(o.Rbuf);
    }
    s.P = d_work + o.P;
    s.Rbuf = mixed() ? nullptr : W(o.Rbuf); s.Fbuf = W(o.Fbuf); s.XB = W(o.XB); s.xb_cap = 1;
    s.Ffin = W(o.Ffin); s.Hl = W(o.Hl); s.tau_l = W(o.tau); s.piv_l = reinterpret_cast<int*>(d_work + o.piv);
    const bool svd = last_sel[i] >= bcr::LAST_SVD;
    s.Ul = svd ? W(o.U) : nullptr; s.Vl = svd ? W(o.V) : nullptr; s.Sl = svd ? W(o.S) : nullptr;
    s.Al = nullptr; s.sel_last2 = 0;
    s.st = d_st + i;
    s.bx = d_x + x_off[i];
    s.bldx = L(i);
    in_off[i] = o.D0;
  }
  cudaMemsetAsync(d_work, 0, work_bytes, stream);
  int rc = upload_inputs();
  if (rc) return rc;
  // ----------------------------------------------------------- classes
  std::vector<std::pair<long, int>> keys;  // (n * 8 + family) -> class
  for (size_t i = 0; i < ns; ++i) {
    const long key = (long)dims[i].n * 8 + fam[i];
    int c = -1;
    for (auto& kv : keys)
      if (kv.first == key) c = kv.second;
    if (c < 0) {
      c = (int)members.size();
      keys.push_back({key, c});
      members.emplace_back();
    }
    members[c].push_back((int)i);
    cls_of[i] = c;
  }
  cls.assign(members.size(), bcr::BatchClass{});
  for (size_t c = 0; c < members.size(); ++c) {
    cls[c].fam = fam[members[c][0]];
    std::vector<bcr::DevState> v;
    for (int i : members[c]) v.push_back(sys[i]);
    // a tuned choice for this shape, if one is cached
    const Dims& d0 = dims[members[c][0]];
    int nrm = 0, nxm = 0;
    for (int i : members[c]) { nrm = std::max(nrm, dims[i].nr); nxm = std::max(nxm, dims[i].nx); }
    cls[c].mixed = mixed() ? 1 : 0;
    cls[c].persist = schedule == BCR_BATCH_PERSISTENT ? 1 : 0;
    for (const auto& t : g_batch_tuning)
      if (t.n == d0.n && t.nrm == nrm && t.nxm == nxm && t.mixed == cls[c].mixed && t.persist == cls[c].persist) {
        cls[c].fam = t.fam;
        cls[c].chunk = t.chunk;
      }
    if (bcr::batch_build(cls[c], v, 1)) {
      release();
      return fail(BCR_CUDA_ERROR, "alglin_b200 batch: table upload failed\n");
    }
  }
  if (make_class_streams()) {
    release();
    return fail(BCR_CUDA_ERROR, "alglin_b200 batch: stream creation failed\n");
  }
  e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return cuda_fail(e, "batch prepare");
  prepared = true;
  if (autotune)
    for (size_t c = 0; c < cls.size(); ++c)
      if ((rc = tune_class(c))) return rc;
  return BCR_OK;
}

// time every applicable (family, chunk) on this class's own systems and keep
// the fastest; the choice is cached for later batches of the same shape
int bcr_batch_s::tune_class(size_t ci) {
  bcr::BatchClass& c = cls[ci];
  std::vector<bcr::DevState> v;
  int nrm = 0, nxm = 0;
  for (int i : members[ci]) {
    v.push_back(sys[i]);
    nrm = std::max(nrm, sys[i].d.nr);
    nxm = std::max(nxm, sys[i].d.nx);
  }
  Dims dm = sys[members[ci][0]].d;
  dm.nr = nrm;
  dm.nx = nxm;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  int bf = c.fam, bc = c.chunk;
  for (int f : {bcr::PAIR_TC, bcr::PAIR_GRP, bcr::PAIR_ROWS}) {
    if (!bcr::batch_family_ok(f, dm, c.mixed != 0)) continue;
    for (int ch : {2, 4, 8, 16}) {
      c.fam = f;
      c.chunk = ch;
      if (bcr::batch_build(c, v, 1)) return fail(BCR_CUDA_ERROR, "alglin_b200 batch: table upload failed\n");
      bcr::batch_factorize(c, stream);  // warm-up (also sets kernel attributes)
      cudaEventRecord(e0, stream);
      for (int r = 0; r < 3; ++r) bcr::batch_factorize(c, stream);
      cudaEventRecord(e1, stream);
      cudaError_t e = cudaEventSynchronize(e1);
      if (e != cudaSuccess) return cuda_fail(e, "batch autotune");
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (ms < best) { best = ms; bf = f; bc = ch; }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c.fam = bf;
  c.chunk = bc;
  if (bcr::batch_build(c, v, 1)) return fail(BCR_CUDA_ERROR, "alglin_b200 batch: table upload failed\n");
  bool found = false;
  for (auto& t : g_batch_tuning)
    if (t.n == dm.n && t.nrm == nrm && t.nxm == nxm && t.mixed == c.mixed && t.persist == c.persist) {
      t.fam = bf;
      t.chunk = bc;
      found = true;
    }
  if (!found) g_batch_tuning.push_back({dm.n, nrm, nxm, c.mixed, c.persist, bf, bc});
  return BCR_OK;
}

#define B_CHECK(b)                                 \
  do {                                             \
    if (!(b)) return BCR_BAD_ARGUMENT;             \
  } while (0)
#define B_READY(b)                                                                            \
  do {                                                                                        \
    B_CHECK(b);                                                                               \
    if (!(b)->prepared) return (b)->fail(BCR_BAD_ARGUMENT, "bcr_batch: prepare() must be called first\n"); \
  } while (0)

extern "C" {

int bcr_batch_create(bcr_batch* out) {
  if (!out) return BCR_BAD_ARGUMENT;
  *out = new bcr_batch_s;
  return BCR_OK;
}

int bcr_batch_destroy(bcr_batch b) {
  if (!b) return BCR_OK;
  b->release();
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return BCR_OK;
}

int bcr_batch_add(bcr_batch b, bcr_handle h) {
  B_CHECK(b);
  if (!h) return b->fail(BCR_BAD_ARGUMENT, "bcr_batch_add: null handle\n");
  b->release();
  b->hs.push_back(h);
  b->dims.push_back(h->d);
  b->last_sel.push_back(h->sel_last);
  return BCR_OK;
}

int bcr_batch_add_device(bcr_batch b, int nblock, int n, int qr, int qx, int nr, int nx, const char* last) {
  B_CHECK(b);
  if (nblock < 1 || n < 1 || qr < 0 || qx < 0 || nr < 0 || nx < 0)
    return b->fail(BCR_BAD_ARGUMENT, fmt("bcr_batch_add_device( nblock=%d, n=%d, qr=%d, qx=%d, nr=%d, nx=%d ) bad sizes\n",
                                         nblock, n, qr, qx, nr, nx));
  const std::string ls = last ? last : "LU";
  static const char* names[] = {"LU", "LUPQ", "QR", "QRP", "SVD", "LSS", "LSY", "PINV"};
  int sl = -1;
  for (int k = 0; k < 8; ++k)
    if (ls == names[k]) sl = k;
  if (sl < 0)
    return b->fail(BCR_BAD_ARGUMENT, fmt("bcr_batch_add_device: unknown last block solver '%s'\n", ls.c_str()));
  b->release();
  Dims d{};
  d.nblock = nblock; d.n = n; d.qr = qr; d.qx = qx; d.nr = nr; d.nx = nx;
  d.Nr = 2 * n + qr + nr;
  d.Nc = 2 * n + qx + nx;
  b->hs.push_back(nullptr);
  b->dims.push_back(d);
  b->last_sel.push_back(sl);
  return BCR_OK;
}

int bcr_batch_matrix(bcr_batch b, int i, double** D, double** E, double** B, double** C, double** Cq,
                     double** F, double** H) {
  B_READY(b);
  if (i < 0 || i >= (int)b->hs.size()) return b->fail(BCR_BAD_ARGUMENT, "bcr_batch_matrix: bad system index\n");
  const bcr::DevState& s = b->sys[i];
  if (D) *D = s.D0;
  if (E) *E = s.E0;
  if (B) *B = s.B0;
  if (C) *C = s.C0;
  if (Cq) *Cq = s.Cq;
  if (F) *F = s.F0;
  if (H) *H = s.H;
  return BCR_OK;
}

int bcr_batch_load_device(bcr_batch b, int i, const double* D, const double* E, const double* B, const double* C,
                          const double* Cq, const double* F, const double* H) {
  B_READY(b);
  if (i < 0 || i >= (int)b->hs.size()) return b->fail(BCR_BAD_ARGUMENT, "bcr_batch_load_device: bad system index\n");
  const Dims& d = b->dims[i];
  const bcr::DevState& s = b->sys[i];
  const size_t nb = d.nblock, n = d.n;
  const struct { double* dst; const double* src; size_t count; } cp[] = {
      {s.D0, D, nb * n * n}, {s.E0, E, nb * n * n}, {s.B0, B, nb * n * d.nx},
      {s.C0, C, (nb + 1) * d.nr * n}, {s.Cq, Cq, (size_t)d.nr * d.qx}, {s.F0, F, (size_t)d.nr * d.nx},
      {s.H, H, (size_t)(n + d.qr) * d.Nc}};
  for (const auto& c : cp)
    if (c.src && c.count) {
      cudaError_t e = cudaMemcpyAsync(c.dst, c.src, c.count * 8, cudaMemcpyDeviceToDevice, b->stream);
      if (e != cudaSuccess) return b->cuda_fail(e, "bcr_batch_load_device");
    }
  // the sources may be released or reused as soon as this returns
  cudaError_t e = cudaStreamSynchronize(b->stream);
  return e == cudaSuccess ? BCR_OK : b->cuda_fail(e, "bcr_batch_load_device");
}

double* bcr_batch_device_b(bcr_batch b, int i) {
  if (!b || !b->prepared || i < 0 || i >= (int)b->hs.size()) return nullptr;
  return b->d_b + b->x_off[i];
}

int bcr_batch_system_size(bcr_batch b, int i, int* nrows, int* ncols) {
  B_CHECK(b);
  if (i < 0 || i >= (int)b->dims.size()) return b->fail(BCR_BAD_ARGUMENT, "bcr_batch_system_size: bad index\n");
  const Dims& d = b->dims[i];
  if (nrows) *nrows = d.n * (d.nblock + 1) + d.qr + d.nr;
  if (ncols) *ncols = d.n * (d.nblock + 1) + d.qx + d.nx;
  return BCR_OK;
}

int bcr_batch_size(bcr_batch b) { return b ? (int)b->hs.size() : 0; }

int bcr_batch_prepare(bcr_batch b, int autotune) {
  B_CHECK(b);
  return b->prepare(autotune);
}

int bcr_batch_autotune(bcr_batch b) {
  B_READY(b);
  if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
  for (size_t c = 0; c < b->cls.size(); ++c) {
    int rc = b->tune_class(c);
    if (rc) return rc;
  }
  return BCR_OK;
}

int bcr_batch_classes(bcr_batch b) { return b && b->prepared ? (int)b->cls.size() : 0; }

int bcr_batch_class_info(bcr_batch b, int c, int* n, int* nsys, int* family, int* chunk) {
  B_READY(b);
  if (c < 0 || c >= (int)b->cls.size()) return b->fail(BCR_BAD_ARGUMENT, "bcr_batch_class_info: bad class\n");
  if (n) *n = b->cls[c].n;
  if (nsys) *nsys = b->cls[c].nsys;
  if (family) *family = b->cls[c].fam;
  if (chunk) *chunk = b->cls[c].chunk;
  return BCR_OK;
}

int bcr_batch_upload(bcr_batch b) {
  B_READY(b);
  int rc = b->upload_inputs();
  if (rc) return rc;
  cudaError_t e = cudaStreamSynchronize(b->stream);
  return e == cudaSuccess ? BCR_OK : b->cuda_fail(e, "batch upload");
}

int bcr_batch_factorize(bcr_batch b) {
  B_READY(b);
  b->enqueue_factorize();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return b->cuda_fail(e, "batch factorize");
  return b->read_status();
}

int bcr_batch_status(bcr_batch b, int* codes) {
  B_READY(b);
  for (size_t i = 0; i < b->h_st.size(); ++i) codes[i] = b->h_st[i].code;
  return BCR_OK;
}

static int batch_rhs_in(bcr_batch b, double* const* x) {
  for (size_t i = 0; i < b->hs.size(); ++i)
    std::memcpy(b->h_x + b->x_off[i], x[i], (size_t)b->L(i) * 8);
  cudaError_t e = cudaMemcpyAsync(b->d_x, b->h_x, b->x_elems * 8, cudaMemcpyHostToDevice, b->stream);
  return e == cudaSuccess ? BCR_OK : b->cuda_fail(e, "batch rhs upload");
}

static int batch_rhs_out(bcr_batch b, double* const* x) {
  cudaError_t e = cudaMemcpyAsync(b->h_x, b->d_x, b->x_elems * 8, cudaMemcpyDeviceToHost, b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return b->cuda_fail(e, "batch solution download");
  for (size_t i = 0; i < b->hs.size(); ++i)
    std::memcpy(x[i], b->h_x + b->x_off[i], (size_t)b->L(i) * 8);
  return BCR_OK;
}

int bcr_batch_solve(bcr_batch b, double* const* x) {
  B_READY(b);
  if (!x) return b->fail(BCR_BAD_ARGUMENT, "bcr_batch_solve: null vector list\n");
  if (!b->factorized) return b->fail(BCR_NUMERICAL, "bcr_batch_solve: the batch is not factorized\n");
  int rc = batch_rhs_in(b, x);
  if (rc) return rc;
  if (b->mixed()) cudaMemcpyAsync(b->d_b, b->d_x, b->x_elems * 8, cudaMemcpyDeviceToDevice, b->stream);
  if ((rc = b->solve_step(-1))) return rc;
  return batch_rhs_out(b, x);
}

int bcr_batch_factorize_solve(bcr_batch b, double* const* x) {
  B_READY(b);
  if (!x) return b->fail(BCR_BAD_ARGUMENT, "bcr_batch_factorize_solve: null vector list\n");
  int rc = b->upload_inputs();
  if (rc) return rc;
  if ((rc = batch_rhs_in(b, x))) return rc;
  if (b->mixed()) cudaMemcpyAsync(b->d_b, b->d_x, b->x_elems * 8, cudaMemcpyDeviceToDevice, b->stream);
  b->enqueue_factorize();
  if (b->mixed()) {  // the refinement needs the factorization's status first
    if ((rc = b->read_status())) return rc;
    if ((rc = b->solve_step(-1))) return rc;
  } else {
    b->enqueue_solve();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return b->cuda_fail(e, "batch factorize_solve");
    if ((rc = b->read_status())) return rc;
  }
  return batch_rhs_out(b, x);
}

double* bcr_batch_device_x(bcr_batch b, int i) {
  if (!b || !b->prepared || i < 0 || i >= (int)b->hs.size()) return nullptr;
  return b->d_x + b->x_off[i];
}

int bcr_batch_set_rhs(bcr_batch b, const double* const* rhs) {
  B_READY(b);
  for (size_t i = 0; i < b->hs.size(); ++i)
    std::memcpy(b->h_x + b->x_off[i], rhs[i], (size_t)b->L(i) * 8);
  cudaError_t e = cudaMemcpyAsync(b->d_b, b->h_x, b->x_elems * 8, cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(b->d_x, b->d_b, b->x_elems * 8, cudaMemcpyDeviceToDevice, b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  return e == cudaSuccess ? BCR_OK : b->cuda_fail(e, "batch rhs");
}

int bcr_batch_get_x(bcr_batch b, double* const* x) {
  B_READY(b);
  return batch_rhs_out(b, x);
}

int bcr_batch_graph_capture(bcr_batch b) {
  B_READY(b);
  // eager run first: kernel attributes, status check
  cudaMemcpyAsync(b->d_x, b->d_b, b->x_elems * 8, cudaMemcpyDeviceToDevice, b->stream);
  b->enqueue_factorize();
  int rc = b->read_status();
  if (rc) return rc;
  if ((rc = b->solve_step(-1))) return rc;
  rc = b->read_status();
  if (rc) return rc;
  // the mixed graph replays the refinement steps the eager run needed
  const int steps = b->ir_iters;
  if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
  cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeRelaxed);
  if (e != cudaSuccess) return b->cuda_fail(e, "cudaStreamBeginCapture");
  cudaMemcpyAsync(b->d_x, b->d_b, b->x_elems * 8, cudaMemcpyDeviceToDevice, b->stream);
  b->enqueue_factorize();
  rc = b->solve_step(steps);
  b->ir_pending = false;
  cudaGraph_t g = nullptr;
  e = cudaStreamEndCapture(b->stream, &g);
  if (e != cudaSuccess) { cudaGetLastError(); return b->cuda_fail(e, "cudaStreamEndCapture"); }
  if (rc) { cudaGraphDestroy(g); return rc; }
  e = cudaGraphInstantiate(&b->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) { b->graph = nullptr; return b->cuda_fail(e, "cudaGraphInstantiate"); }
  return BCR_OK;
}

int bcr_batch_graph_launch(bcr_batch b) {
  B_READY(b);
  if (!b->graph) return b->fail(BCR_BAD_ARGUMENT, "bcr_batch_graph_launch: no graph captured\n");
  cudaError_t e = cudaGraphLaunch(b->graph, b->stream);
  if (e != cudaSuccess) return b->cuda_fail(e, "cudaGraphLaunch");
  if (b->mixed()) b->ir_pending = true;
  return BCR_OK;
}

int bcr_batch_set_precision(bcr_batch b, int precision) {
  B_CHECK(b);
  if (precision != BCR_PRECISION_FP64 && precision != BCR_PRECISION_MIXED)
    return b->fail(BCR_BAD_ARGUMENT, fmt("bcr_batch_set_precision: unknown precision %d\n", precision));
  b->release();
  b->precision = precision;
  return BCR_OK;
}

int bcr_batch_set_schedule(bcr_batch b, int schedule) {
  B_CHECK(b);
  if (schedule != BCR_BATCH_PERSISTENT && schedule != BCR_BATCH_LEVELS)
    return b->fail(BCR_BAD_ARGUMENT, fmt("bcr_batch_set_schedule: unknown schedule %d\n", schedule));
  b->release();
  b->schedule = schedule;
  return BCR_OK;
}

int bcr_batch_set_refinement(bcr_batch b, double tol, int max_iter) {
  B_CHECK(b);
  if (!(tol >= 0.0) || max_iter < 0)
    return b->fail(BCR_BAD_ARGUMENT, fmt("bcr_batch_set_refinement: bad tolerance %g or iteration limit %d\n", tol, max_iter));
  b->ir_tol = tol;
  b->ir_max = max_iter;
  return BCR_OK;
}

int bcr_batch_refinement_info(bcr_batch b, int* iters, double* worst) {
  B_CHECK(b);
  int rc = b->read_worst();
  if (rc) return rc;
  if (iters) *iters = b->mixed() ? b->ir_iters : 0;
  if (worst) *worst = b->mixed() ? b->ir_worst : 0.0;
  return BCR_OK;
}

int bcr_batch_check_status(bcr_batch b) {
  B_READY(b);
  return b->read_status();
}

void* bcr_batch_stream(bcr_batch b) { return b ? b->stream : nullptr; }

int bcr_batch_synchronize(bcr_batch b) {
  B_CHECK(b);
  if (!b->stream) return BCR_OK;
  cudaError_t e = cudaStreamSynchronize(b->stream);
  return e == cudaSuccess ? BCR_OK : b->cuda_fail(e, "batch synchronize");
}

const char* bcr_batch_last_error(bcr_batch b) { return b ? b->err.c_str() : "invalid batch"; }

}  // extern "C"
