// Host-side launchers for the BorderedCR device kernels (internal interface
// between the C-ABI layer and the CUDA translation units).
#pragma once
#include <vector>
#include <cuda_runtime.h>

#include "bcr_common.cuh"

namespace bcr {

// device buffers of one factorization, FP64 path
struct DevState {
  Dims d;
  int sel;        // Internal
  int sel_last;   // LastKind actually used (after fallback)
  int use_tc;     // allow the FP64 tensor-core pair kernel
  int pair_kernel;  // PairKernel: AUTO, or a forced pair-kernel family
  double* bx;       // batch: right-hand side / solution of this system
  int bldx;         // batch: its leading dimension
  double* bsol;     // batch, mixed path: the refined solution
  const double* bb; // batch, mixed path: the right-hand side
  double* bnrm;     // batch, mixed path: |A|, |r|, |x|, |b|, relative residual, then two block-row maxima
  int* bdone;       // batch, mixed path: refinement converged (null otherwise)
  // loaded matrix (reference layout), never modified on the device
  double *D0, *E0, *B0, *C0, *Cq, *F0, *H;
  // working blocks / factors
  double *D, *E, *B, *C, *T;
  unsigned char* P;   // row / column maps, szP bytes per block
  // scratch: border contributions per eliminated block
  double *Rbuf, *Fbuf, *XB;
  int xb_cap;           // nrhs capacity of XB
  double *part;         // reduction partials
  int part_cap;         // doubles
  double *Ffin;         // F + sum of Schur updates (nr x nx)
  double *Hl;           // last block Nr x Nc
  double *tau_l;        // last block Householder scalars
  int* piv_l;           // last block pivots: rows, then columns (2 * max(Nr, Nc))
  double *Ul, *Vl, *Sl; // last block SVD: W = U*S (max(Nr,Nc) x min), V, S
  double* Al;           // copy of the assembled last block for the fallback solver
  int sel_last2;        // fallback solver (0: none, else the SVD family)
  StatusWords* st;      // device status
  double* mv_part;      // Mv border partials ((nblock+1) x nr)
  int* tree_cnt;        // tree schedule: arrival counter per node + leaf counter (nblock+1);
                        // null where the tree schedule is not used (batches)
  // mixed precision: FP32 working blocks and factors (the loaded matrix, F,
  // the last block, the vectors and the residual stay FP64)
  int mixed;
  float *Df, *Ef, *Bf, *Cf, *Tf, *Rbuff;
  void* slab;           // CTA-per-pair work matrices (large n)
  size_t slab_elems;    // doubles per CTA
  int slab_ctas;        // CTAs that own a slab
};

// large blocks: one CTA per pair with the work matrix in a global slab
bool use_cta_kernel(const Dims& d);
size_t cta_slab_elems(const Dims& d);

// factorization of every cyclic-reduction level plus the last block
void launch_factorize(DevState& s, cudaStream_t st);
// x: device, column-major (ldx x nrhs); in place, reference semantics
void launch_solve(DevState& s, double* x, int ldx, int nrhs, cudaStream_t st);
// factorize, then solve x in place (ldx x nrhs); the forward elimination of
// the right-hand sides is fused into the factorization when the pair kernel
// can carry them
void launch_factorize_solve(DevState& s, double* x, int ldx, int nrhs, cudaStream_t st);
bool factorize_solve_fuses(const DevState& s, int nrhs);
// host copies of the loaded matrix (reference layout, pinned for full-rate copies)
struct HostMatrix {
  const double *D, *E, *B, *C, *Cq, *F, *H;
};
// factorize + solve with the matrix uploaded from hm in chunks on the copy
// stream cst (events ev[0..nev) order the chunks), overlapped with the
// factorization of the chunks already on the device; false (nothing enqueued)
// when the shape does not take this path (FP64 n = 8/16 LU with fused
// right-hand sides, at least 2048 blocks)
bool launch_upload_factorize_solve(DevState& s, const HostMatrix& hm, double* x, int ldx, int nrhs,
                                   cudaStream_t st, cudaStream_t cst, cudaEvent_t* ev, int nev);
// res = alpha * A * x + beta * res with the loaded (unfactored) matrix
void launch_mv(DevState& s, double alpha, const double* x, double beta, double* res,
               cudaStream_t st);

// iterative-refinement helpers (FP64): r = b - A x with the norms |r|, |x|, |b|
// (as non-negative doubles stored in unsigned 64-bit words) and, when rowsum is
// given, ||A||_inf from the same pass over the matrix; y += x
void launch_residual(DevState& s, const double* b, const double* x, double* r, unsigned long long* out,
                     cudaStream_t st, double* rowsum = nullptr, unsigned long long* normA = nullptr);
void launch_axpy(double* y, const double* x, long len, cudaStream_t st);

// smem bytes needed by one warp of the panel kernel; 0 if it does not fit
size_t panel_smem_per_warp(const Dims& d, int elem_bytes);

// ---------------------------------------------------------------------------
// batches of independent systems.  Systems that run the same pair-kernel
// instance form a class; every launch of a class covers all its systems
// through a CTA -> (system, pair range) map.
// ---------------------------------------------------------------------------
struct BatchClass {
  int nsys = 0;
  int fam = PAIR_AUTO;   // PAIR_TC, PAIR_GRP or PAIR_ROWS
  int mixed = 0;         // FP32 working blocks (refined by the caller)
  int chunk = 8;         // pairs per CTA of the factorization launches
  int n = 0, nrm = 0, nxm = 0, levels = 0, nrhs = 1;
  size_t last_smem = 0;
  void* fa = nullptr;    // device FactorArgs<double>[nsys]
  void* sf = nullptr;    // device SweepArgs<double>[nsys], forward layout
  void* sb = nullptr;    // device SweepArgs<double>[nsys], backward layout
  void* ld = nullptr;    // device last-block descriptors [nsys]
  void* rd = nullptr;    // device residual descriptors [nsys] (mixed path)
  BatchCta* fmap = nullptr;  // device: factorization chunks of every level (level order)
  BatchCta* smap = nullptr;  // device: sweep chunks of every level
  BatchCta* cmap = nullptr;  // device, mixed path: smap entries of the systems still refining
  long* ccnt = nullptr;      // device, mixed path: cmap entries per level
  int persist = 1;           // factorization: one persistent launch with a per-system level schedule
  long items = 0;            // factorization chunks in fmap
  int* qbuf = nullptr;       // device: item counter, per-system pair counters, published levels
  std::vector<long> foff, fcnt, soff, scnt;
};

// the pair-kernel families a batch class may use for systems of shape d (LU)
bool batch_family_ok(int fam, const Dims& d, bool mixed);
// tables and maps of one class; sys[i] holds the device pointers of system i
// (x, ldx: its right-hand side; st: its status word)
int batch_build(BatchClass& c, const std::vector<DevState>& sys, int nrhs);
void batch_free(BatchClass& c);
void batch_factorize(BatchClass& c, cudaStream_t st);
// compact: the sweeps walk the compacted maps of the last batch_compact
void batch_solve(BatchClass& c, cudaStream_t st, bool compact = false);
// mixed path: the sweep-map entries of the systems not yet converged, per
// level, for the next correction solve
void batch_compact(BatchClass& c, cudaStream_t st);
// mixed path: r = b - A x_sol into the rhs slots, per-system norms and
// converged flags (relative residual <= tol), batch-worst relative residual
// (|A| is measured when with_A)
// (compact: the block rows of the systems in the compacted maps only, i.e. the
// systems corrected since the last residual)
void batch_residual(BatchClass& c, int with_A, double tol, unsigned long long* worst, cudaStream_t st,
                    bool compact = false);
// x_sol += d for the systems that have not converged
void batch_correct(BatchClass& c, cudaStream_t st);

}  // namespace bcr
