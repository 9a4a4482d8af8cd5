/*
 * CPU oracle for BorderedCR -- TEST INFRASTRUCTURE ONLY (see bcr_oracle.h).
 *
 * A plain-C restatement of ebertolazzi/alglin src/BABD_BorderedCR.cc.  Each
 * function names the reference lines it follows.  The small dense kernels that
 * the reference takes from its (un-vendored) LapackWrapper submodule -- getrf,
 * geqrf, geqp3, ormqr, trsm, gemm and the last-block solver classes -- are
 * restated here from the published LAPACK algorithms (unblocked):
 *   getrf : right-looking LU with partial pivoting, first max |a| wins (idamax)
 *   geqrf : Householder QR, reflector convention of dlarfg (v(1)=1,
 *           beta = -sign(alpha)*||x||, tau = (beta-alpha)/beta)
 *   geqp3 : Householder QR with column pivoting on the largest remaining
 *           column 2-norm (norms recomputed exactly each step)
 *   SVD-family last-block solvers: one-sided Jacobi SVD (Hestenes) and the
 *           minimum-norm least-squares solution x = V S^+ U^T b.
 */
#include "bcr_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define IDX(i, j, ld) ((size_t)(i) + (size_t)(j) * (size_t)(ld))

enum { SEL_LU = 0, SEL_QR = 1, SEL_QRP = 2 };
enum { LAST_LU = 0, LAST_LUPQ, LAST_QR, LAST_QRP, LAST_SVD, LAST_LSS, LAST_LSY, LAST_PINV };
enum { L2_NONE = 0, L2_SVD, L2_LSS, L2_LSY, L2_PINV };

/* ------------------------------------------------------------------------ */
/* last-block dense solver state                                            */
/* ------------------------------------------------------------------------ */
typedef struct {
  int kind; /* 0 LU, 1 LUPQ, 2 QR, 3 QRP, 4 PINV-family */
  int m, n;
  double *A;   /* m x n factors */
  int *p, *q;  /* row / column permutations */
  double *tau;
  double *U, *S, *V; /* SVD: U m x n, S n, V n x n (thin) */
  int transposed;    /* SVD taken of A^T when m < n */
} dense_fact;

struct orc_bcr {
  int nblock, n, qr, qx, nr, nx, Nr, Nc;
  int sel, sel_last, sel_last2;
  int npb_req, npb, reduced_nblk;
  int *iBlock, *kBlock;
  /* loaded matrix (kept untouched for Mv) */
  double *D0, *E0, *B0, *C0, *Cq, *F0, *H;
  /* working copies overwritten by factorize */
  double *D, *E, *B, *C, *F; /* F holds npb partial blocks */
  double *T;
  int *P;
  dense_fact last;
  int use2;
  int factorized;
  char err[512];
};

static void *xcalloc(size_t n, size_t s) {
  void *p = calloc(n ? n : 1, s ? s : 1);
  if (!p) { fprintf(stderr, "bcr_oracle: out of memory\n"); abort(); }
  return p;
}

static void gecopy(int m, int n, const double *A, int lda, double *B, int ldb) {
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < m; ++i) B[IDX(i, j, ldb)] = A[IDX(i, j, lda)];
}

/* C(m x n) += alpha * A(m x k) * B(k x n) */
static void gemm_acc(int m, int n, int k, double alpha, const double *A, int lda,
                     const double *B, int ldb, double *C, int ldc) {
  for (int j = 0; j < n; ++j)
    for (int l = 0; l < k; ++l) {
      double b = alpha * B[IDX(l, j, ldb)];
      if (b == 0.0) continue;
      for (int i = 0; i < m; ++i) C[IDX(i, j, ldc)] += A[IDX(i, l, lda)] * b;
    }
}

/* ------------------------------------------------------------------------ */
/* panel factorizations (buildT, BABD_BorderedCR.cc:845-898)                */
/* ------------------------------------------------------------------------ */

/* LU with partial pivoting of an m x n matrix (m >= n), 0-based ipiv.
 * Returns 0 or i+1 of the first exactly-zero pivot (LAPACK getrf INFO). */
static int lu_partial(int m, int n, double *A, int lda, int *ipiv) {
  int info = 0;
  for (int i = 0; i < n; ++i) {
    int p = i;
    double best = fabs(A[IDX(i, i, lda)]);
    for (int r = i + 1; r < m; ++r) {
      double v = fabs(A[IDX(r, i, lda)]);
      if (v > best) { best = v; p = r; }
    }
    ipiv[i] = p;
    if (A[IDX(p, i, lda)] == 0.0) { if (!info) info = i + 1; continue; }
    if (p != i)
      for (int c = 0; c < n; ++c) {
        double t = A[IDX(i, c, lda)];
        A[IDX(i, c, lda)] = A[IDX(p, c, lda)];
        A[IDX(p, c, lda)] = t;
      }
    double piv = A[IDX(i, i, lda)];
    for (int r = i + 1; r < m; ++r) A[IDX(r, i, lda)] /= piv;
    for (int c = i + 1; c < n; ++c) {
      double u = A[IDX(i, c, lda)];
      if (u == 0.0) continue;
      for (int r = i + 1; r < m; ++r) A[IDX(r, c, lda)] -= A[IDX(r, i, lda)] * u;
    }
  }
  return info;
}

/* dlarfg-style Householder of column i of A rows i..m-1; returns tau */
static double householder(int m, int i, double *A, int lda) {
  double alpha = A[IDX(i, i, lda)];
  double xn2 = 0;
  for (int r = i + 1; r < m; ++r) xn2 += A[IDX(r, i, lda)] * A[IDX(r, i, lda)];
  if (xn2 == 0.0) return 0.0;
  double nrm = sqrt(alpha * alpha + xn2);
  double beta = alpha >= 0 ? -nrm : nrm;
  double tau = (beta - alpha) / beta;
  double scal = 1.0 / (alpha - beta);
  for (int r = i + 1; r < m; ++r) A[IDX(r, i, lda)] *= scal;
  A[IDX(i, i, lda)] = beta;
  return tau;
}

/* apply H = I - tau v v^T (v = [1; A(i+1:m-1, i)]) to columns c0..c1-1 of W */
static void apply_reflector(int m, int i, const double *A, int lda, double tau,
                            double *W, int ldw, int ncol) {
  if (tau == 0.0) return;
  for (int c = 0; c < ncol; ++c) {
    double w = W[IDX(i, c, ldw)];
    for (int r = i + 1; r < m; ++r) w += A[IDX(r, i, lda)] * W[IDX(r, c, ldw)];
    w *= tau;
    W[IDX(i, c, ldw)] -= w;
    for (int r = i + 1; r < m; ++r) W[IDX(r, c, ldw)] -= w * A[IDX(r, i, lda)];
  }
}

/* Householder QR of m x n (geqrf) */
static void qr_house(int m, int n, double *A, int lda, double *tau) {
  int kmax = m < n ? m : n;
  for (int i = 0; i < kmax; ++i) {
    tau[i] = householder(m, i, A, lda);
    if (i + 1 < n) apply_reflector(m, i, A, lda, tau[i], A + IDX(0, i + 1, lda), lda, n - i - 1);
  }
}

/* Householder QR with column pivoting (geqp3): jpvt 1-based like LAPACK */
static void qrp_house(int m, int n, double *A, int lda, int *jpvt, double *tau) {
  for (int j = 0; j < n; ++j) jpvt[j] = j + 1;
  int kmax = m < n ? m : n;
  for (int i = 0; i < kmax; ++i) {
    int p = i;
    double best = -1;
    for (int c = i; c < n; ++c) {
      double s = 0;
      for (int r = i; r < m; ++r) s += A[IDX(r, c, lda)] * A[IDX(r, c, lda)];
      if (s > best) { best = s; p = c; }
    }
    if (p != i) {
      for (int r = 0; r < m; ++r) {
        double t = A[IDX(r, i, lda)];
        A[IDX(r, i, lda)] = A[IDX(r, p, lda)];
        A[IDX(r, p, lda)] = t;
      }
      int t = jpvt[i]; jpvt[i] = jpvt[p]; jpvt[p] = t;
    }
    tau[i] = householder(m, i, A, lda);
    if (i + 1 < n) apply_reflector(m, i, A, lda, tau[i], A + IDX(0, i + 1, lda), lda, n - i - 1);
  }
}

/* BorderedCR::permutation_to_exchange (BABD_BorderedCR.hxx:266-275) */
static void permutation_to_exchange(int nn, int *P, int *S) {
  for (int i = 0; i < nn; ++i) {
    int j = i;
    while (j < nn) { if (P[j] == i + 1) break; ++j; }
    if (j >= nn) j = i;
    int t = P[j]; P[j] = P[i]; P[i] = t;
    S[i] = j;
  }
}

/* buildT (BABD_BorderedCR.cc:845-898); T is 2n x n (ld 2n) + tau[n] */
static int buildT(orc_bcr *h, double *T, int *iperm) {
  int n = h->n, n2 = 2 * n;
  switch (h->sel) {
    case SEL_LU: {
      int info = lu_partial(n2, n, T, n2, iperm);
      if (info) {
        snprintf(h->err, sizeof h->err,
                 "BorderedCR::buildT [LU] getrf(M=%d,N=%d,A,LDA=%d,iperm)::INFO = %d\n",
                 n2, n, n2, info);
        return 0;
      }
      break;
    }
    case SEL_QR: qr_house(n2, n, T, n2, T + 2 * n * n); break;
    case SEL_QRP: {
      int *P = (int *)xcalloc((size_t)n, sizeof(int));
      qrp_house(n2, n, T, n2, P, T + 2 * n * n);
      permutation_to_exchange(n, P, iperm);
      free(P);
      break;
    }
  }
  return 1;
}

/* applyT (BABD_BorderedCR.cc:917-1044): W=[TOP;BOTTOM] -> TOP<-W_bot, BOTTOM<-W_top */
static void applyT(const orc_bcr *h, const double *T, const int *iperm, double *TOP,
                   int ldTOP, double *BOTTOM, int ldBOT, int ncol) {
  int n = h->n, n2 = 2 * n;
  if (ncol <= 0) return;
  double *W = (double *)xcalloc((size_t)n2 * ncol, sizeof(double));
  gecopy(n, ncol, TOP, ldTOP, W, n2);
  gecopy(n, ncol, BOTTOM, ldBOT, W + n, n2);
  if (h->sel == SEL_LU) {
    for (int i = 0; i < n; ++i) {
      int p = iperm[i];
      if (p != i)
        for (int c = 0; c < ncol; ++c) {
          double t = W[IDX(i, c, n2)];
          W[IDX(i, c, n2)] = W[IDX(p, c, n2)];
          W[IDX(p, c, n2)] = t;
        }
    }
    /* trsm LEFT LOWER NO UNIT: W_top = L^{-1} W_top */
    for (int c = 0; c < ncol; ++c)
      for (int i = 0; i < n; ++i) {
        double wi = W[IDX(i, c, n2)];
        if (wi == 0.0) continue;
        for (int r = i + 1; r < n; ++r) W[IDX(r, c, n2)] -= T[IDX(r, i, n2)] * wi;
      }
    /* gemm: W_bot -= M * W_top */
    gemm_acc(n, ncol, n, -1.0, T + n, n2, W, n2, W + n, n2);
  } else {
    const double *tau = T + 2 * n * n;
    for (int i = 0; i < n; ++i) apply_reflector(n2, i, T, n2, tau[i], W, n2, ncol);
  }
  gecopy(n, ncol, W + n, n2, TOP, ldTOP);
  gecopy(n, ncol, W, n2, BOTTOM, ldBOT);
  free(W);
}

/* C(nr x n) <- C * U^{-1}, U upper non-unit = top n x n of T (trsm RIGHT UPPER) */
static void trsm_right_upper(int nr, int n, const double *T, int ldt, double *C, int ldc) {
  for (int i = 0; i < n; ++i) {
    double d = T[IDX(i, i, ldt)];
    for (int r = 0; r < nr; ++r) {
      double s = C[IDX(r, i, ldc)];
      for (int m = 0; m < i; ++m) s -= C[IDX(r, m, ldc)] * T[IDX(m, i, ldt)];
      C[IDX(r, i, ldc)] = s / d;
    }
  }
}

/* x(n x nrhs) <- U^{-1} x  (trsv / trsm LEFT UPPER NON_UNIT) */
static void trsm_left_upper(int n, int nrhs, const double *T, int ldt, double *x, int ldx) {
  for (int c = 0; c < nrhs; ++c)
    for (int i = n - 1; i >= 0; --i) {
      double s = x[IDX(i, c, ldx)];
      for (int m = i + 1; m < n; ++m) s -= T[IDX(i, m, ldt)] * x[IDX(m, c, ldx)];
      x[IDX(i, c, ldx)] = s / T[IDX(i, i, ldt)];
    }
}

static void zero_blk(double *A, size_t cnt) { memset(A, 0, cnt * sizeof(double)); }

/* one CR elimination step on the pair (jp, j) with border target jpp
 * (inner body of factorize_block, BABD_BorderedCR.cc:1088-1155) */
static int eliminate_pair(orc_bcr *h, int jp, int j, int jpp, double *Fwork) {
  int n = h->n, nn = n * n, n2 = 2 * n, nr = h->nr, nx = h->nx;
  double *T = h->T + (size_t)j * (2 * nn + n);
  int *P = h->P + (size_t)j * n;
  double *Djp = h->D + (size_t)jp * nn, *Dj = h->D + (size_t)j * nn;
  double *Ejp = h->E + (size_t)jp * nn, *Ej = h->E + (size_t)j * nn;
  gecopy(n, n, Ejp, n, T, n2);
  gecopy(n, n, Dj, n, T + n, n2);
  if (!buildT(h, T, P)) return 0;
  zero_blk(Dj, (size_t)nn);
  zero_blk(Ejp, (size_t)nn);
  applyT(h, T, P, Djp, n, Dj, n, n);
  applyT(h, T, P, Ejp, n, Ej, n, n);
  if (nx > 0) applyT(h, T, P, h->B + (size_t)jp * n * nx, n, h->B + (size_t)j * n * nx, n, nx);
  double *Cj = h->C + (size_t)j * nr * n;
  if (nr > 0) {
    double *Cjp = h->C + (size_t)jp * nr * n;
    if (h->sel == SEL_QRP) {
      int i = n;
      do {
        --i;
        if (P[i] > i)
          for (int r = 0; r < nr; ++r) {
            double t = Cj[IDX(r, i, nr)];
            Cj[IDX(r, i, nr)] = Cj[IDX(r, P[i], nr)];
            Cj[IDX(r, P[i], nr)] = t;
          }
      } while (i > 0);
    }
    trsm_right_upper(nr, n, T, n2, Cj, nr);
    gemm_acc(nr, n, n, -1.0, Cj, nr, Dj, n, Cjp, nr);
    double *Cpp = h->C + (size_t)jpp * nr * n;
    gemm_acc(nr, n, n, -1.0, Cj, nr, Ej, n, Cpp, nr);
  }
  if (nr > 0 && nx > 0)
    gemm_acc(nr, nx, n, -1.0, Cj, nr, h->B + (size_t)j * n * nx, n, Fwork, nr);
  return 1;
}

/* factorize_block (BABD_BorderedCR.cc:1055-1171) */
static int factorize_block(orc_bcr *h, int t) {
  int iblock = h->iBlock[2 * t], eblock = h->iBlock[2 * t + 1];
  int nblk = eblock - iblock;
  double *Fwork = h->F + (size_t)t * h->nr * h->nx;
  int k = 1;
  while (k < nblk) {
    for (int j = iblock + k; j < eblock; j += 2 * k) {
      int jpp = j + k < eblock ? j + k : eblock;
      if (!eliminate_pair(h, j - k, j, jpp, Fwork)) return 0;
    }
    k *= 2;
  }
  h->kBlock[t] = k;
  return 1;
}

/* factorize_reduced (BABD_BorderedCR.cc:1175-1266) */
static int factorize_reduced(orc_bcr *h) {
  int k = 1, R = h->reduced_nblk;
  while (k < R) {
    for (int jj = k; jj < R; jj += 2 * k) {
      int j = h->iBlock[jj], jp = h->iBlock[jj - k];
      int jpp = h->iBlock[jj + k < R ? jj + k : R];
      if (!eliminate_pair(h, jp, j, jpp, h->F)) return 0;
    }
    k *= 2;
  }
  return 1;
}

/* ------------------------------------------------------------------------ */
/* last block solvers (LapackWrapper LU/LUPQ/QR/QRP/SVD/LSS/LSY/PINV)       */
/* ------------------------------------------------------------------------ */
static void dense_free(dense_fact *f) {
  free(f->A); free(f->p); free(f->q); free(f->tau);
  free(f->U); free(f->S); free(f->V);
  memset(f, 0, sizeof *f);
}

/* one-sided Jacobi SVD of W (m x n, m >= n): on return W = U*S (columns),
 * V (n x n) accumulates the rotations */
static void jacobi_svd(int m, int n, double *W, double *V) {
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) V[IDX(i, j, n)] = (i == j);
  for (int sweep = 0; sweep < 80; ++sweep) {
    int rotated = 0;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        double a = 0, b = 0, g = 0;
        for (int i = 0; i < m; ++i) {
          double wp = W[IDX(i, p, m)], wq = W[IDX(i, q, m)];
          a += wp * wp; b += wq * wq; g += wp * wq;
        }
        if (fabs(g) <= 1e-15 * sqrt(a * b) || g == 0.0) continue;
        rotated = 1;
        double zeta = (b - a) / (2 * g);
        double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1 + zeta * zeta));
        double c = 1 / sqrt(1 + t * t), s = c * t;
        for (int i = 0; i < m; ++i) {
          double wp = W[IDX(i, p, m)], wq = W[IDX(i, q, m)];
          W[IDX(i, p, m)] = c * wp - s * wq;
          W[IDX(i, q, m)] = s * wp + c * wq;
        }
        for (int i = 0; i < n; ++i) {
          double vp = V[IDX(i, p, n)], vq = V[IDX(i, q, n)];
          V[IDX(i, p, n)] = c * vp - s * vq;
          V[IDX(i, q, n)] = s * vp + c * vq;
        }
      }
    if (!rotated) break;
  }
}

static int dense_factorize(dense_fact *f, int kind, int m, int n, const double *A, int lda) {
  dense_free(f);
  f->kind = kind; f->m = m; f->n = n;
  f->A = (double *)xcalloc((size_t)m * n, sizeof(double));
  gecopy(m, n, A, lda, f->A, m);
  int mn = m < n ? m : n;
  switch (kind) {
    case 0: { /* LU */
      if (m != n) return 0;
      f->p = (int *)xcalloc((size_t)n, sizeof(int));
      return lu_partial(n, n, f->A, n, f->p) == 0;
    }
    case 1: { /* LUPQ: complete pivoting */
      if (m != n) return 0;
      f->p = (int *)xcalloc((size_t)n, sizeof(int));
      f->q = (int *)xcalloc((size_t)n, sizeof(int));
      double *a = f->A;
      for (int i = 0; i < n; ++i) {
        int pr = i, pc = i;
        double best = -1;
        for (int c = i; c < n; ++c)
          for (int r = i; r < n; ++r) {
            double v = fabs(a[IDX(r, c, n)]);
            if (v > best) { best = v; pr = r; pc = c; }
          }
        f->p[i] = pr; f->q[i] = pc;
        if (best == 0.0) return 0;
        for (int c = 0; c < n; ++c) { double t = a[IDX(i, c, n)]; a[IDX(i, c, n)] = a[IDX(pr, c, n)]; a[IDX(pr, c, n)] = t; }
        for (int r = 0; r < n; ++r) { double t = a[IDX(r, i, n)]; a[IDX(r, i, n)] = a[IDX(r, pc, n)]; a[IDX(r, pc, n)] = t; }
        double piv = a[IDX(i, i, n)];
        for (int r = i + 1; r < n; ++r) a[IDX(r, i, n)] /= piv;
        for (int c = i + 1; c < n; ++c) {
          double u = a[IDX(i, c, n)];
          for (int r = i + 1; r < n; ++r) a[IDX(r, c, n)] -= a[IDX(r, i, n)] * u;
        }
      }
      return 1;
    }
    case 2: /* QR */
    case 3: { /* QRP */
      if (m < n) return 0;
      f->tau = (double *)xcalloc((size_t)mn, sizeof(double));
      if (kind == 2) qr_house(m, n, f->A, m, f->tau);
      else {
        f->q = (int *)xcalloc((size_t)n, sizeof(int));
        qrp_house(m, n, f->A, m, f->q, f->tau);
      }
      for (int i = 0; i < n; ++i) if (f->A[IDX(i, i, m)] == 0.0) return 0;
      return 1;
    }
    default: { /* SVD / LSS / LSY / PINV: minimum-norm least squares */
      int M = m, N = n;
      f->transposed = (m < n);
      double *W;
      if (f->transposed) {
        M = n; N = m;
        W = (double *)xcalloc((size_t)M * N, sizeof(double));
        for (int i = 0; i < m; ++i)
          for (int j = 0; j < n; ++j) W[IDX(j, i, M)] = f->A[IDX(i, j, m)];
      } else {
        W = (double *)xcalloc((size_t)M * N, sizeof(double));
        memcpy(W, f->A, sizeof(double) * (size_t)M * N);
      }
      f->V = (double *)xcalloc((size_t)N * N, sizeof(double));
      f->S = (double *)xcalloc((size_t)N, sizeof(double));
      jacobi_svd(M, N, W, f->V);
      for (int j = 0; j < N; ++j) {
        double s = 0;
        for (int i = 0; i < M; ++i) s += W[IDX(i, j, M)] * W[IDX(i, j, M)];
        s = sqrt(s);
        f->S[j] = s;
        if (s > 0) for (int i = 0; i < M; ++i) W[IDX(i, j, M)] /= s;
      }
      f->U = W;
      return 1;
    }
  }
}

/* solve in place; x has length max(m, n) per column (stride ldx) */
static int dense_solve(const dense_fact *f, int nrhs, double *x, int ldx) {
  int m = f->m, n = f->n;
  double *tmp = (double *)xcalloc((size_t)(m > n ? m : n), sizeof(double));
  for (int c = 0; c < nrhs; ++c) {
    double *b = x + (size_t)c * ldx;
    switch (f->kind) {
      case 0:
      case 1: {
        for (int i = 0; i < n; ++i) { int p = f->p[i]; double t = b[i]; b[i] = b[p]; b[p] = t; }
        for (int i = 0; i < n; ++i)
          for (int r = i + 1; r < n; ++r) b[r] -= f->A[IDX(r, i, n)] * b[i];
        trsm_left_upper(n, 1, f->A, n, b, n);
        if (f->kind == 1)
          for (int i = n - 1; i >= 0; --i) { int q = f->q[i]; double t = b[i]; b[i] = b[q]; b[q] = t; }
        break;
      }
      case 2:
      case 3: {
        for (int i = 0; i < n; ++i) apply_reflector(m, i, f->A, m, f->tau[i], b, m, 1);
        trsm_left_upper(n, 1, f->A, m, b, m);
        if (f->kind == 3) {
          for (int i = 0; i < n; ++i) tmp[f->q[i] - 1] = b[i];
          for (int i = 0; i < n; ++i) b[i] = tmp[i];
        }
        break;
      }
      default: {
        int M = f->transposed ? n : m, N = f->transposed ? m : n;
        /* A = U S V^T (not transposed) or A^T = U S V^T (transposed) */
        double smax = 0;
        for (int j = 0; j < N; ++j) if (f->S[j] > smax) smax = f->S[j];
        double tol = smax * 1e-12;
        if (!f->transposed) {
          /* x = V S^+ U^T b, b length m, x length n */
          for (int j = 0; j < N; ++j) {
            double s = 0;
            if (f->S[j] > tol) {
              for (int i = 0; i < M; ++i) s += f->U[IDX(i, j, M)] * b[i];
              s /= f->S[j];
            }
            tmp[j] = s;
          }
          for (int i = 0; i < n; ++i) {
            double s = 0;
            for (int j = 0; j < N; ++j) s += f->V[IDX(i, j, N)] * tmp[j];
            b[i] = s;
          }
        } else {
          /* A = V S U^T, x = U S^+ V^T b, b length m (=N), x length n (=M) */
          for (int j = 0; j < N; ++j) {
            double s = 0;
            if (f->S[j] > tol) {
              for (int i = 0; i < N; ++i) s += f->V[IDX(i, j, N)] * b[i];
              s /= f->S[j];
            }
            tmp[j] = s;
          }
          for (int i = 0; i < M; ++i) {
            double s = 0;
            for (int j = 0; j < N; ++j) s += f->U[IDX(i, j, M)] * tmp[j];
            b[i] = s;
          }
        }
        break;
      }
    }
  }
  free(tmp);
  return 1;
}

static int last_kind(int sel_last) {
  switch (sel_last) {
    case LAST_LU: return 0;
    case LAST_LUPQ: return 1;
    case LAST_QR: return 2;
    case LAST_QRP: return 3;
    default: return 4;
  }
}

/* load_and_factorize_last (BABD_BorderedCR.cc:1281-1374) */
static int load_and_factorize_last(orc_bcr *h) {
  int n = h->n, Nr = h->Nr, Nc = h->Nc, nr = h->nr, qx = h->qx, nx = h->nx, qr = h->qr;
  double *Hm = (double *)xcalloc((size_t)Nr * Nc, sizeof(double));
  double *W0 = Hm, *WN = W0 + (size_t)n * Nr, *Wq = WN + (size_t)n * Nr, *Wp = Wq + (size_t)qx * Nr;
  gecopy(n, n, h->D, n, W0, Nr);
  gecopy(n, n, h->E, n, WN, Nr);
  gecopy(n, nx, h->B, n, Wp, Nr);
  gecopy(n + qr, Nc, h->H, n + qr, Hm + n, Nr);
  int offs = 2 * n + qr;
  gecopy(nr, n, h->C, nr, W0 + offs, Nr);
  gecopy(nr, n, h->C + (size_t)h->nblock * nr * n, nr, WN + offs, Nr);
  gecopy(nr, qx, h->Cq, nr, Wq + offs, Nr);
  gecopy(nr, nx, h->F, nr, Wp + offs, Nr);
  int ok = dense_factorize(&h->last, last_kind(h->sel_last), Nr, Nc, Hm, Nr);
  h->use2 = 0;
  if (!ok && h->sel_last2 != L2_NONE) {
    h->use2 = 1;
    ok = dense_factorize(&h->last, 4, Nr, Nc, Hm, Nr);
  }
  if (!ok) snprintf(h->err, sizeof h->err, "BorderedCR<t_Value>::load_and_factorize_last failed\n");
  free(Hm);
  return ok;
}

/* ------------------------------------------------------------------------ */
/* public API                                                               */
/* ------------------------------------------------------------------------ */
static void partition(orc_bcr *h) {
  /* allocate(): chunk partition, BABD_BorderedCR.cc:139-158 */
  int NBLK = h->npb_req < 1 ? 1 : h->npb_req;
  free(h->iBlock); free(h->kBlock); free(h->F);
  h->iBlock = (int *)xcalloc((size_t)2 * NBLK, sizeof(int));
  h->kBlock = (int *)xcalloc((size_t)NBLK, sizeof(int));
  h->F = (double *)xcalloc((size_t)NBLK * h->nr * h->nx, sizeof(double));
  int used = NBLK, red = 2 * NBLK;
  while (red > h->nblock) { red -= 2; --used; }
  if (used <= 1) {
    used = 1;
    h->iBlock[0] = 0;
    h->iBlock[1] = h->nblock;
  } else {
    h->iBlock[0] = 0;
    h->iBlock[1] = h->nblock / used;
    for (int nt = 1; nt < used; ++nt) {
      h->iBlock[2 * nt] = h->iBlock[2 * nt - 1] + 1;
      h->iBlock[2 * nt + 1] = (int)(((long long)(nt + 1) * h->nblock) / used);
    }
    --red;
  }
  h->npb = used;
  h->reduced_nblk = red;
}

orc_bcr *orc_create(int nblock, int n, int qr, int qx, int nr, int nx) {
  orc_bcr *h = (orc_bcr *)xcalloc(1, sizeof *h);
  h->nblock = nblock; h->n = n; h->qr = qr; h->qx = qx; h->nr = nr; h->nx = nx;
  h->Nr = 2 * n + nr + qr;
  h->Nc = 2 * n + nx + qx;
  size_t nb = (size_t)nblock;
  h->D0 = (double *)xcalloc(nb * n * n, sizeof(double));
  h->E0 = (double *)xcalloc(nb * n * n, sizeof(double));
  h->B0 = (double *)xcalloc(nb * n * nx, sizeof(double));
  h->C0 = (double *)xcalloc((nb + 1) * nr * n, sizeof(double));
  h->Cq = (double *)xcalloc((size_t)nr * qx, sizeof(double));
  h->F0 = (double *)xcalloc((size_t)nr * nx, sizeof(double));
  h->H = (double *)xcalloc((size_t)(n + qr) * h->Nc, sizeof(double));
  h->D = (double *)xcalloc(nb * n * n, sizeof(double));
  h->E = (double *)xcalloc(nb * n * n, sizeof(double));
  h->B = (double *)xcalloc(nb * n * nx, sizeof(double));
  h->C = (double *)xcalloc((nb + 1) * nr * n, sizeof(double));
  h->T = (double *)xcalloc(nb * (2 * n * n + n), sizeof(double));
  h->P = (int *)xcalloc(nb * n, sizeof(int));
  h->npb_req = 1;
  partition(h);
  strcpy(h->err, "no error");
  return h;
}

void orc_destroy(orc_bcr *h) {
  if (!h) return;
  free(h->D0); free(h->E0); free(h->B0); free(h->C0); free(h->Cq); free(h->F0); free(h->H);
  free(h->D); free(h->E); free(h->B); free(h->C); free(h->F); free(h->T); free(h->P);
  free(h->iBlock); free(h->kBlock);
  dense_free(&h->last);
  free(h);
}

void orc_load(orc_bcr *h, const double *D, const double *E, const double *B, const double *C,
              const double *Cq, const double *F, const double *H) {
  size_t nb = (size_t)h->nblock, n = (size_t)h->n;
  memcpy(h->D0, D, sizeof(double) * nb * n * n);
  memcpy(h->E0, E, sizeof(double) * nb * n * n);
  if (h->nx) memcpy(h->B0, B, sizeof(double) * nb * n * h->nx);
  if (h->nr) memcpy(h->C0, C, sizeof(double) * (nb + 1) * h->nr * n);
  if (h->nr && h->qx) memcpy(h->Cq, Cq, sizeof(double) * h->nr * h->qx);
  if (h->nr && h->nx) memcpy(h->F0, F, sizeof(double) * h->nr * h->nx);
  memcpy(h->H, H, sizeof(double) * (n + h->qr) * h->Nc);
  h->factorized = 0;
}

void orc_select(orc_bcr *h, int internal, int last, int last2) {
  h->sel = internal; h->sel_last = last; h->sel_last2 = last2;
}

void orc_set_num_parallel_block(orc_bcr *h, int npb) {
  h->npb_req = npb < 1 ? 1 : npb;
  partition(h);
}

int orc_used_parallel_block(const orc_bcr *h) { return h->npb; }

/* factorize (BABD_BorderedCR.cc:803-839), thread fan-out run sequentially */
int orc_factorize(orc_bcr *h) {
  size_t nb = (size_t)h->nblock, n = (size_t)h->n;
  memcpy(h->D, h->D0, sizeof(double) * nb * n * n);
  memcpy(h->E, h->E0, sizeof(double) * nb * n * n);
  memcpy(h->B, h->B0, sizeof(double) * nb * n * h->nx);
  memcpy(h->C, h->C0, sizeof(double) * (nb + 1) * h->nr * n);
  size_t nrnx = (size_t)h->nr * h->nx;
  memset(h->F, 0, sizeof(double) * nrnx * h->npb);
  if (nrnx) memcpy(h->F, h->F0, sizeof(double) * nrnx);
  h->factorized = 0;
  int ok = 1;
  for (int t = 0; t < h->npb && ok; ++t) ok = factorize_block(h, t);
  if (ok && h->npb > 1) {
    for (int t = 1; t < h->npb; ++t)
      for (size_t i = 0; i < nrnx; ++i) h->F[i] += h->F[t * nrnx + i];
    ok = factorize_reduced(h);
  }
  if (ok) ok = load_and_factorize_last(h);
  h->factorized = ok;
  return ok;
}

/* forward (BABD_BorderedCR.cc:1615-1719) on chunk t; accumulates -C_j x_j in work */
static void forward_chunk(const orc_bcr *h, int t, int nrhs, double *x, int ldx, double *work) {
  int n = h->n, nr = h->nr;
  int iblock = h->iBlock[2 * t], eblock = h->iBlock[2 * t + 1], nblk = eblock - iblock;
  size_t Ts = 2 * (size_t)n * n + n;
  int k = 1;
  while (k < nblk) {
    for (int j = iblock + k; j < eblock; j += 2 * k) {
      double *xj = x + (size_t)j * n, *xjp = x + (size_t)(j - k) * n;
      applyT(h, h->T + (size_t)j * Ts, h->P + (size_t)j * n, xjp, ldx, xj, ldx, nrhs);
      if (nr > 0) gemm_acc(nr, nrhs, n, -1.0, h->C + (size_t)j * nr * n, nr, xj, ldx, work, nr);
    }
    k *= 2;
  }
}

/* backward (BABD_BorderedCR.cc:1805-1949) on chunk t */
static void backward_step(const orc_bcr *h, int j, int jp, int jpp, int nrhs, double *x, int ldx) {
  int n = h->n, nx = h->nx;
  size_t Ts = 2 * (size_t)n * n + n;
  double *xn = x + (size_t)(h->nblock + 1) * n + h->qx;
  double *xj = x + (size_t)j * n;
  gemm_acc(n, nrhs, n, -1.0, h->D + (size_t)j * n * n, n, x + (size_t)jp * n, ldx, xj, ldx);
  gemm_acc(n, nrhs, n, -1.0, h->E + (size_t)j * n * n, n, x + (size_t)jpp * n, ldx, xj, ldx);
  if (nx > 0) gemm_acc(n, nrhs, nx, -1.0, h->B + (size_t)j * n * nx, n, xn, ldx, xj, ldx);
  trsm_left_upper(n, nrhs, h->T + (size_t)j * Ts, 2 * n, xj, ldx);
  if (h->sel == SEL_QRP) {
    const int *P = h->P + (size_t)j * n;
    for (int c = 0; c < nrhs; ++c)
      for (int i = 0; i < n; ++i)
        if (P[i] > i) {
          double t = xj[IDX(i, c, ldx)];
          xj[IDX(i, c, ldx)] = xj[IDX(P[i], c, ldx)];
          xj[IDX(P[i], c, ldx)] = t;
        }
  }
}

int orc_solve(const orc_bcr *h, int nrhs, double *x, int ldx) {
  if (!h->factorized) return 0;
  int n = h->n, nr = h->nr, nb = h->nblock;
  double *xb = x + (size_t)(nb + 1) * n + h->qr;
  double *work = (double *)xcalloc((size_t)nr * nrhs + 1, sizeof(double));
  /* forward: chunks, xb partial sums, reduced (cc:1499-1523, 1564-1586) */
  for (int t = 0; t < h->npb; ++t) {
    memset(work, 0, sizeof(double) * (size_t)nr * nrhs);
    forward_chunk(h, t, nrhs, x, ldx, work);
    for (int c = 0; c < nrhs; ++c)
      for (int r = 0; r < nr; ++r) xb[IDX(r, c, ldx)] += work[IDX(r, c, nr)];
  }
  free(work);
  if (h->npb > 1) {
    /* forward_reduced (cc:1723-1795) */
    int k = 1, R = h->reduced_nblk;
    size_t Ts = 2 * (size_t)n * n + n;
    while (k < R) {
      for (int jj = k; jj < R; jj += 2 * k) {
        int j = h->iBlock[jj], jp = h->iBlock[jj - k];
        double *xj = x + (size_t)j * n;
        applyT(h, h->T + (size_t)j * Ts, h->P + (size_t)j * n, x + (size_t)jp * n, ldx, xj, ldx, nrhs);
        if (nr > 0) gemm_acc(nr, nrhs, n, -1.0, h->C + (size_t)j * nr * n, nr, xj, ldx, xb, ldx);
      }
      k *= 2;
    }
  }
  /* solve_last (cc:1385-1479): swap first block into slot nblock-1 */
  double *X = x + (size_t)(nb - 1) * n;
  for (int c = 0; c < nrhs; ++c)
    for (int i = 0; i < n; ++i) {
      double t = X[IDX(i, c, ldx)];
      X[IDX(i, c, ldx)] = x[IDX(i, c, ldx)];
      x[IDX(i, c, ldx)] = t;
    }
  dense_solve(&h->last, nrhs, X, ldx);
  for (int c = 0; c < nrhs; ++c)
    for (int i = 0; i < n; ++i) {
      double t = X[IDX(i, c, ldx)];
      X[IDX(i, c, ldx)] = x[IDX(i, c, ldx)];
      x[IDX(i, c, ldx)] = t;
    }
  /* backward: reduced (cc:1953-2075) then chunks */
  if (h->npb > 1) {
    int k = 1, R = h->reduced_nblk;
    while (k < R) k *= 2;
    while ((k /= 2) > 0)
      for (int jj = k; jj < R; jj += 2 * k)
        backward_step(h, h->iBlock[jj], h->iBlock[jj - k], h->iBlock[jj + k < R ? jj + k : R], nrhs, x, ldx);
  }
  for (int t = 0; t < h->npb; ++t) {
    int iblock = h->iBlock[2 * t], eblock = h->iBlock[2 * t + 1];
    int k = h->kBlock[t];
    while ((k /= 2) > 0)
      for (int j = iblock + k; j < eblock; j += 2 * k)
        backward_step(h, j, j - k, j + k < eblock ? j + k : eblock, nrhs, x, ldx);
  }
  return 1;
}

/* add_Mv (BABD_BorderedCR.cc:2111-2166) on the loaded matrix */
void orc_add_mv(const orc_bcr *h, double alpha, const double *x, double beta, double *res) {
  int n = h->n, nb = h->nblock, nr = h->nr, nx = h->nx, qx = h->qx, qr = h->qr;
  int NR = orc_nrows(h);
  for (int i = 0; i < NR; ++i) res[i] = beta == 0.0 ? 0.0 : beta * res[i];
  const double *xe = x + (size_t)nb * n, *xq = xe + n, *xb = xq + qx;
  double *yy = res;
  for (int i = 0; i < nb; ++i) {
    gemm_acc(n, 1, n, alpha, h->D0 + (size_t)i * n * n, n, x + (size_t)i * n, n, yy, n);
    gemm_acc(n, 1, n, alpha, h->E0 + (size_t)i * n * n, n, x + (size_t)(i + 1) * n, n, yy, n);
    gemm_acc(n, 1, nx, alpha, h->B0 + (size_t)i * n * nx, n, xb, nx, yy, n);
    yy += n;
  }
  int m = n + qr;
  const double *H = h->H;
  gemm_acc(m, 1, n, alpha, H, m, x, n, yy, m); H += (size_t)m * n;
  gemm_acc(m, 1, n, alpha, H, m, xe, n, yy, m); H += (size_t)m * n;
  gemm_acc(m, 1, qx, alpha, H, m, xq, qx, yy, m); H += (size_t)m * qx;
  gemm_acc(m, 1, nx, alpha, H, m, xb, nx, yy, m);
  if (nr > 0) {
    yy += m;
    gemm_acc(nr, 1, nx, alpha, h->F0, nr, xb, nx, yy, nr);
    for (int i = 0; i <= nb; ++i)
      gemm_acc(nr, 1, n, alpha, h->C0 + (size_t)i * nr * n, nr, x + (size_t)i * n, n, yy, nr);
    gemm_acc(nr, 1, qx, alpha, h->Cq, nr, x + (size_t)(nb + 1) * n, qx, yy, nr);
  }
}

const char *orc_last_error(const orc_bcr *h) { return h->err; }
int orc_nrows(const orc_bcr *h) { return h->n * (h->nblock + 1) + h->qr + h->nr; }
int orc_ncols(const orc_bcr *h) { return h->n * (h->nblock + 1) + h->qx + h->nx; }
