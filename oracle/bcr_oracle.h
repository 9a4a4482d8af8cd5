/*
 * CPU oracle for the bordered cyclic-reduction (BorderedCR) BABD solver.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the algorithm in
 * ebertolazzi/alglin src/BABD_BorderedCR.cc, used by the tests, by the smoke
 * check and by the CPU-baseline leg of the benchmark as the checker.  The
 * product (alglin_b200/) never links, loads or calls it.
 *
 * Storage follows the reference layout exactly (column-major blocks):
 *   D[nblock][n*n], E[nblock][n*n], B[nblock][n*nx], C[nblock+1][nr*n],
 *   Cq[nr*qx], F[nr*nx], H[(n+qr) * (2n+qx+nx)]  (H = [H0 | HN | Hq | Hp]).
 * (BABD_BorderedCR.hxx:972-998 accessors; BABD_BorderedCR.cc:102-124 arena.)
 */
#ifndef BCR_ORACLE_H
#define BCR_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_bcr orc_bcr;

/* internal (cyclic-reduction) block choice: 0 LU, 1 QR, 2 QRP            */
/* last block choice: 0 LU 1 LUPQ 2 QR 3 QRP 4 SVD 5 LSS 6 LSY 7 PINV     */
/* fallback choice:   0 NONE 1 SVD 2 LSS 3 LSY 4 PINV                       */

orc_bcr *orc_create(int nblock, int n, int qr, int qx, int nr, int nx);
void     orc_destroy(orc_bcr *h);
/* copy the whole matrix in (reference layout, see above) */
void     orc_load(orc_bcr *h, const double *D, const double *E, const double *B,
                  const double *C, const double *Cq, const double *F,
                  const double *H);
void     orc_select(orc_bcr *h, int internal, int last, int last2);
/* number of chunks used for the reference's chunked schedule (>=1) */
void     orc_set_num_parallel_block(orc_bcr *h, int npb);
int      orc_used_parallel_block(const orc_bcr *h);
/* returns 1 on success, 0 on failure (message in orc_last_error) */
int      orc_factorize(orc_bcr *h);
int      orc_solve(const orc_bcr *h, int nrhs, double *x, int ldx);
/* res = alpha*A*x + beta*res using the ORIGINAL (loaded) matrix */
void     orc_add_mv(const orc_bcr *h, double alpha, const double *x,
                    double beta, double *res);
const char *orc_last_error(const orc_bcr *h);
int      orc_nrows(const orc_bcr *h);
int      orc_ncols(const orc_bcr *h);

#ifdef __cplusplus
}
#endif
#endif
