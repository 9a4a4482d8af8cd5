/*
 * alglin_b200 -- C ABI of the B200 BorderedCR solver for bordered
 * block-almost-bidiagonal (BABD) linear systems.
 *
 * Each entry point replaces one member of the reference C++ class
 * alglin::BorderedCR<double> (ebertolazzi/alglin, src/Alglin/BABD_BorderedCR.hxx,
 * src/BABD_BorderedCR.cc); the citation beside each declaration names it.
 * The reference's historic C interface header (Alglin/BABD_C_interface.h,
 * included by src_tests/test8-Cinterface.c:20 and test9-Cinterface.c:20) is
 * absent from the reference tree, so this ABI follows the C++ method names.
 *
 * Conventions
 *   - plain pointers and sizes only; matrices are column-major with a leading
 *     dimension, exactly as the reference loaders take them;
 *   - every call returns an int status:
 *       BCR_OK (0), BCR_NUMERICAL (1: factorize/solve returned false in the
 *       reference), BCR_BAD_ARGUMENT (2: the reference throws
 *       Utils::Runtime_Error), BCR_CUDA_ERROR (3), BCR_DEVICE_TIMEOUT (4);
 *     bcr_last_error() returns the message of the last failure, in the
 *     reference's wording where the reference has one;
 *   - the handle keeps a host copy of the loaded matrix; factorize() copies it
 *     to the GPU once and leaves it untouched (the reference overwrites it),
 *     so bcr_mv() after bcr_factorize() still multiplies by the loaded matrix;
 *   - all compute runs on the current CUDA device; there is no CPU fallback:
 *     without a usable GPU the compute calls return BCR_CUDA_ERROR.
 */
#ifndef ALGLIN_B200_H
#define ALGLIN_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define BCR_OK 0
#define BCR_NUMERICAL 1
#define BCR_BAD_ARGUMENT 2
#define BCR_CUDA_ERROR 3
#define BCR_DEVICE_TIMEOUT 4

/* working precision of the device factorization (extension: set_precision) */
#define BCR_PRECISION_FP64 0
#define BCR_PRECISION_MIXED 1

typedef struct bcr_handle_s *bcr_handle;

/* --- life cycle ----------------------------------------------------------- */
/* BorderedCR(Utils::ThreadPoolBase* TP, integer npb)  hxx:373-384.
 * num_threads stands for TP->thread_count() (0: no pool); it only feeds info() */
int bcr_create(bcr_handle *h, int num_threads, int num_parallel_block);
int bcr_destroy(bcr_handle h);                                    /* ~BorderedCR hxx:386 */
int bcr_allocate(bcr_handle h, int nblock, int n, int qr, int qx,
                 int nr, int nx);                                 /* allocate cc:42-170 */
int bcr_dup(bcr_handle dst, bcr_handle src);                      /* dup cc:181-198 */

/* --- sizes (hxx:617-650) -------------------------------------------------- */
int bcr_nrows(bcr_handle h);
int bcr_ncols(bcr_handle h);
int bcr_number_of_blocks(bcr_handle h);
int bcr_block_size(bcr_handle h);
int bcr_dim_qr(bcr_handle h);
int bcr_dim_qx(bcr_handle h);
int bcr_dim_nr(bcr_handle h);
int bcr_dim_nx(bcr_handle h);
int bcr_Nr(bcr_handle h);
int bcr_Nc(bcr_handle h);

/* --- zeroing (hxx:658-682, cc:237-279) ------------------------------------ */
int bcr_zero_B(bcr_handle h);
int bcr_zero_C(bcr_handle h);
int bcr_zero_Cq(bcr_handle h);
int bcr_zero_D(bcr_handle h);
int bcr_zero_E(bcr_handle h);
int bcr_zero_F(bcr_handle h);
int bcr_zero_H(bcr_handle h);
int bcr_fill_zero(bcr_handle h);

/* --- loaders (cc:289-793) --------------------------------------------------- */
int bcr_load_B(bcr_handle h, int nbl, const double *B, int ldB);      /* cc:453 */
int bcr_add_to_B(bcr_handle h, int nbl, const double *B, int ldB);    /* cc:479 */
int bcr_load_C(bcr_handle h, int nbl, const double *C, int ldC);      /* cc:507 */
int bcr_add_to_C(bcr_handle h, int nbl, const double *C, int ldC);    /* cc:534 */
int bcr_add_to_C2(bcr_handle h, int nbl, const double *C, int ldC);   /* cc:567 */
int bcr_add_to_C2F(bcr_handle h, int nbl, const double *C2F, int ldC);/* cc:765 */
int bcr_load_D(bcr_handle h, int nbl, const double *D, int ldD);      /* cc:598 */
int bcr_load_E(bcr_handle h, int nbl, const double *E, int ldE);      /* cc:625 */
int bcr_load_DE(bcr_handle h, int nbl, const double *DE, int ldDE);   /* cc:654 */
int bcr_load_DEB(bcr_handle h, int nbl, const double *DEB, int ldDEB);/* cc:666 */
int bcr_load_F(bcr_handle h, const double *F, int ldF);               /* cc:681 */
int bcr_add_to_F(bcr_handle h, const double *F, int ldF);             /* cc:705 */
int bcr_load_Cq(bcr_handle h, const double *Cq, int ldC);             /* cc:729 */
int bcr_load_CqF(bcr_handle h, const double *CqF, int ldCF);          /* cc:753 */
int bcr_load_bottom(bcr_handle h, const double *H0, int ld0, const double *HN, int ldN,
                    const double *Hq, int ldQ, const double *Hp, int ldP);  /* cc:291 */
int bcr_load_bottom_H(bcr_handle h, const double *H, int ldH);        /* cc:358 */
int bcr_load_bottom2(bcr_handle h, const double *C0, int ld0, const double *CN, int ldN,
                     const double *Cq, int ldCq, const double *F, int ldF); /* cc:382 */
/* [C0 | CN | Cq | F] as one nr x Nc matrix: load_bottom2(MatW)  cc:430-447 */
int bcr_load_bottom2_H(bcr_handle h, const double *CCqF, int ld);

/* host copy of a block for element access (accessors hxx:972-998):
 * which = 'B','C','D','E' (block nbl), 'F', 'Q' (Cq), 'H' (nbl ignored);
 * column-major with the reference leading dimensions; NULL if out of range */
double *bcr_block_data(bcr_handle h, char which, int nbl);

/* --- algorithm selection (hxx:459-540) ------------------------------------ */
int bcr_select(bcr_handle h, const char *choice);        /* "LU" "QR" "QRP" */
int bcr_select_last(bcr_handle h, const char *choice);   /* "LU" "LUPQ" "QR" "QRP" "SVD" "LSS" "LSY" "PINV" */
int bcr_select_last2(bcr_handle h, const char *choice);  /* "NONE" "SVD" "LSS" "LSY" "PINV" */
int bcr_selected(bcr_handle h, int *internal, int *last, int *last2);
int bcr_set_factorize_use_thread(bcr_handle h, int yes); /* hxx:391 (kept for info()) */
int bcr_set_solve_use_thread(bcr_handle h, int yes);     /* hxx:393 */
int bcr_factorize_use_thread(bcr_handle h);              /* hxx:396 */
int bcr_solve_use_thread(bcr_handle h);                  /* hxx:398 */
int bcr_set_num_parallel_block(bcr_handle h, int npb);   /* hxx:407-423 */
int bcr_set_precision(bcr_handle h, int precision);      /* extension: FP64 / mixed */
/* Pair-kernel family of the factorization (extension, no reference
   counterpart; for tuning and tests).  AUTO picks by block size, selection and
   precision; a forced family that does not apply to the shape falls back to
   the next one that does (TC -> GRP -> ROWS -> CTA -> SMEM).  UMMA is the
   FP32 (mixed-precision) large-block LU kernel with tcgen05 tensor-core
   products (33 <= n <= 128, nr <= 16, nx <= 16); under AUTO it is the choice
   for those shapes, and CTA selects the CUDA-core blocked kernel instead. */
#define BCR_PAIR_AUTO 0
#define BCR_PAIR_TC 1
#define BCR_PAIR_GRP 2
#define BCR_PAIR_ROWS 3
#define BCR_PAIR_CTA 4
#define BCR_PAIR_SMEM 5
#define BCR_PAIR_UMMA 6
#define BCR_PAIR_TREE 7
#define BCR_PAIR_TC_GATHER 8
int bcr_set_pair_kernel(bcr_handle h, int choice);

/* Iterative refinement of the mixed path (extension, no reference counterpart):
   corrections d = A^-1 r from FP64 residuals r = b - A x stop once
   |r|_inf / (|A|_inf |x|_inf + |b|_inf) <= tol (default 1e-12) or after
   max_iter corrections (default 10).  The mixed path needs a square system. */
int bcr_set_refinement(bcr_handle h, double tol, int max_iter);
/* corrections applied by the last mixed solve and its final relative residual
   (max over right-hand sides); 0 and 0.0 on the FP64 path */
int bcr_refinement_info(bcr_handle h, int* iters, double* relres);
/* info(indent) cc:208-235; the returned string lives until the next call */
const char *bcr_info(bcr_handle h, const char *indent);
const char *bcr_last_error(bcr_handle h);                /* hxx:445 */
int bcr_set_debug(bcr_handle h, int yes);                /* hxx:1172 */
int bcr_check_matrix(bcr_handle h);                      /* cc:2538-2659 */

/* --- factorize / solve (hxx:1029-1038) ------------------------------------- */
int bcr_factorize(bcr_handle h);                         /* factorize cc:803-839 */
/* x: length >= max(nrows, ncols); in place: rhs in, solution out (cc:1489) */
int bcr_solve(bcr_handle h, double *x);
/* rhs: ldRhs x nrhs, ldRhs >= max(nrows, ncols)  (cc:1546-1605) */
int bcr_solve_n(bcr_handle h, int nrhs, double *rhs, int ldRhs);
/* factorize() followed by solve(nrhs, rhs, ldRhs) in one pass (the Newton-step
 * use of factorize + solve, BABD.hxx:271-313): the forward elimination of the
 * right-hand sides rides in the factorization kernels where they fit; the
 * factors are kept for later solve() calls */
int bcr_factorize_solve(bcr_handle h, int nrhs, double *rhs, int ldRhs);
int bcr_t_solve(bcr_handle h, double *x);                /* cc:2089: not defined */
int bcr_t_solve_n(bcr_handle h, int nrhs, double *rhs, int ldRhs); /* cc:2096 */

/* --- products (cc:2111-2166) ---------------------------------------------- */
int bcr_mv(bcr_handle h, const double *x, double *res);
int bcr_add_mv(bcr_handle h, double alpha, const double *x, double *res);

/* --- sparse export / import (hxx:1079-1115, cc:2342-2482) ------------------ */
int bcr_sparse_nnz(bcr_handle h);
int bcr_sparse_pattern(bcr_handle h, int *I, int *J, int offs);
int bcr_sparse_values(bcr_handle h, double *V);
int bcr_sparse_load(bcr_handle h, const double *V, const int *I, int r_offs,
                    const int *J, int c_offs, int nnz, int do_error);

/* --- device-resident variants (extension for callers whose data is on the GPU) */
/* stream: a cudaStream_t (NULL = the handle's own stream) */
int bcr_set_stream(bcr_handle h, void *stream);
int bcr_upload(bcr_handle h);          /* host copy of the matrix -> device */
int bcr_factorize_device(bcr_handle h);/* factorize the device-resident matrix */
/* enqueue the factorization on the handle's stream and return at once (no
 * host synchronisation, so it can be captured in a CUDA graph); the outcome is
 * read by bcr_factorize_status(), which synchronises the stream */
int bcr_factorize_async(bcr_handle h);
int bcr_factorize_status(bcr_handle h);
/* d_x: device pointer, ld x nrhs column-major; stream-ordered, asynchronous */
int bcr_solve_device(bcr_handle h, int nrhs, double *d_x, int ld);
/* bcr_factorize_solve on device memory, asynchronous like bcr_factorize_async */
int bcr_factorize_solve_device(bcr_handle h, int nrhs, double *d_x, int ld);
int bcr_mv_device(bcr_handle h, double alpha, const double *d_x, double beta, double *d_res);
int bcr_synchronize(bcr_handle h);
/* the cudaStream_t the handle enqueues on (its own non-blocking stream unless
 * bcr_set_stream chose another); NULL without a device */
void *bcr_get_stream(bcr_handle h);

/* CUDA graphs of the device-resident path: capture once, replay many times.
 * what = BCR_GRAPH_FACTORIZE, BCR_GRAPH_SOLVE or BCR_GRAPH_STEP (both).  The
 * solve part works in place on d_x (ld x nrhs); when d_rhs is not NULL it
 * first copies d_rhs into d_x.  The factorization status of a replay is read
 * with bcr_factorize_status(). */
#define BCR_GRAPH_FACTORIZE 1
#define BCR_GRAPH_SOLVE 2
#define BCR_GRAPH_STEP 3
int bcr_graph_capture(bcr_handle h, int what, int nrhs, double *d_x, int ld, const double *d_rhs);
int bcr_graph_launch(bcr_handle h, int what);

/* --- allocation-free product ------------------------------------------------
 * No counterpart in the reference.  res = alpha*A*x + beta*res for a matrix whose blocks
 * (reference layout, see bcr_block_data), x and res are all caller-owned
 * DEVICE memory; for callers that cannot allocate device memory where they
 * need the product (a fixed memory budget owned by the host application, or a
 * loop that must not call into the CUDA allocator).  The library allocates
 * nothing: its only scratch is a fixed 512 KiB array in device memory, so nr
 * is limited to 64 border rows (larger nr is rejected with BCR_BAD_ARGUMENT).
 * The first call on each device looks the array up (cudaGetSymbolAddress),
 * and looks it up again after the device's context was reset; make that
 * first call before any stream capture.  All calls share the array: calls
 * that overlap on the GPU race.  A CUDA error already pending on the calling
 * thread is reported (BCR_CUDA_ERROR) and left pending for its owner, and
 * nothing is launched.  Enqueued on `stream` (a cudaStream_t, NULL for the
 * legacy stream); errbuf (may be NULL) receives the reason of a failure. */
int bcr_mv_noalloc(int nblock, int n, int qr, int qx, int nr, int nx,
                   const double *D, const double *E, const double *B, const double *C,
                   const double *Cq, const double *F, const double *H,
                   double alpha, const double *x, double beta, double *res,
                   void *stream, char *errbuf, int errlen);

/* --- batches of independent systems -----------------------------------------
 * No counterpart in the reference (each BorderedCR object there is factored
 * on its own thread pool).  Many systems -- each a bcr_handle filled through
 * the usual loaders, internal LU, FP64 -- are factored
 * and solved together: prepare() packs every system into one device arena,
 * groups the systems by pair-kernel instance (by block size n) and runs each
 * cyclic-reduction level of all systems of a group in one launch.  Systems
 * may differ in nblock, n (4..16 with nr, nx <= 4; 8, 16, 32 with nr, nx <= 8),
 * borders and last-block solver (select_last2 fallbacks are not applied).
 * The handles must stay alive while the batch uses them: their
 * host copies are read at prepare() and upload(). */
typedef struct bcr_batch_s *bcr_batch;
int bcr_batch_create(bcr_batch *out);
int bcr_batch_destroy(bcr_batch b);
int bcr_batch_add(bcr_batch b, bcr_handle h);
/* a system that lives only on the device (no handle, no host copy): after
   prepare(), bcr_batch_matrix() gives the device addresses of its blocks in
   the reference layout (see bcr_block_data) for the caller to fill; last is
   the last-block solver ("LU", "LUPQ", "QR", "QRP", "SVD", "LSS", "LSY",
   "PINV") */
int bcr_batch_add_device(bcr_batch b, int nblock, int n, int qr, int qx, int nr, int nx, const char *last);
int bcr_batch_matrix(bcr_batch b, int i, double **D, double **E, double **B, double **C, double **Cq,
                     double **F, double **H);
int bcr_batch_system_size(bcr_batch b, int i, int *nrows, int *ncols);
/* copy system i's blocks from caller device buffers (reference layout,
   contiguous; NULL skips a block).  The sources must be complete when the
   call is made (synchronize the stream that wrote them); the call returns
   when the copies are done, so the sources may then be reused. */
int bcr_batch_load_device(bcr_batch b, int i, const double *D, const double *E, const double *B,
                          const double *C, const double *Cq, const double *F, const double *H);
int bcr_batch_size(bcr_batch b);
/* autotune != 0: time every applicable pair-kernel family and pairs-per-CTA
   chunk on each group's own systems and keep the fastest (cached per shape) */
int bcr_batch_prepare(bcr_batch b, int autotune);
int bcr_batch_autotune(bcr_batch b);  /* the same tuning later, e.g. after bcr_batch_load_device */
int bcr_batch_classes(bcr_batch b);
int bcr_batch_class_info(bcr_batch b, int cls, int *n, int *nsys, int *family, int *chunk);
int bcr_batch_upload(bcr_batch b);                       /* re-read the handles' matrices */
int bcr_batch_factorize(bcr_batch b);                    /* BCR_NUMERICAL if any system failed */
int bcr_batch_status(bcr_batch b, int *codes);           /* per system: 0 ok, else device code */
int bcr_batch_solve(bcr_batch b, double *const *x);      /* x[i]: host vector of system i, in place */
int bcr_batch_factorize_solve(bcr_batch b, double *const *x);  /* upload + factorize + solve */
/* device-resident use: rhs copies kept on the device, a graph of the whole
   factorize + solve step, solutions in device vectors */
int bcr_batch_set_rhs(bcr_batch b, const double *const *rhs);
double *bcr_batch_device_x(bcr_batch b, int i);
double *bcr_batch_device_b(bcr_batch b, int i);  /* device copy of the rhs the graph starts from */
int bcr_batch_get_x(bcr_batch b, double *const *x);
int bcr_batch_graph_capture(bcr_batch b);
int bcr_batch_graph_launch(bcr_batch b);
int bcr_batch_check_status(bcr_batch b);
void *bcr_batch_stream(bcr_batch b);
int bcr_batch_synchronize(bcr_batch b);
const char *bcr_batch_last_error(bcr_batch b);
/* mixed precision for the whole batch (set before prepare): FP32 working
   blocks, FP64 F, last block and vectors, FP64 refinement of every system until
   the worst |b-Ax|/(|A||x|+|b|) of the batch is <= tol or after max_iter
   corrections (defaults 1e-12 and 30); a system that has converged drops out
   of the later corrections; the systems must be square */
int bcr_batch_set_precision(bcr_batch b, int precision);
int bcr_batch_set_refinement(bcr_batch b, double tol, int max_iter);
/* Schedule of the batched factorization (set before prepare; extension, no
   reference counterpart).  LEVELS (the default): one launch per level for all
   systems of a class.  PERSISTENT: one launch per class works through every
   (system, level, pair range) item in level order with a per-system level
   schedule -- a worker waits (bounded, about a second, then
   BCR_DEVICE_TIMEOUT for that system) only for its own system's previous
   level, and the worker completing a level applies its border updates; the
   results are bit-identical to LEVELS. */
#define BCR_BATCH_PERSISTENT 0
#define BCR_BATCH_LEVELS 1
int bcr_batch_set_schedule(bcr_batch b, int schedule);
int bcr_batch_refinement_info(bcr_batch b, int *iters, double *worst);

#ifdef __cplusplus
}
#endif
#endif
