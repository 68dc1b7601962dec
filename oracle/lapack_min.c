/*
 * Minimal complex LAPACK stand-ins for the reference CPU build.
 *
 * TEST INFRASTRUCTURE ONLY: this file is linked into the reference oracle
 * under oracle/_ref/ (the reference's own C code, built unmodified); nothing
 * in the shipped library uses it.
 *
 * The reference links three LAPACK routines and no BLAS symbols:
 *   zgetrf_  LU factorisation      (4d_Q16/susy/determinant.c:25,72)
 *   zgetri_  inverse from the LU   (4d_Q16/susy/determinant.c:75)
 *   zheev_   Hermitian eigensolver (4d_Q16/susy/unit.c:25,69,
 *                                   4d_Q16/susy/scalar_eig.c:68)
 * The image has no system LAPACK, so these are written here from the
 * textbook algorithms for the NCOL <= 4 matrices the reference passes:
 * partial-pivot Doolittle LU with LAPACK's |re|+|im| pivot measure and
 * reciprocal column scaling, column-by-column forward/back substitution for
 * the inverse, and cyclic complex Jacobi rotations for the eigenproblem
 * (eigenvalues ascending, eigenvectors in the columns).  Fortran calling
 * convention: column-major, 1-based pivots, arguments by pointer.
 */
#include <math.h>
#include <string.h>

typedef struct { double re, im; } zc;

static inline zc zmul(zc a, zc b) {
  zc c = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
  return c;
}
static inline zc zsub(zc a, zc b) { zc c = {a.re - b.re, a.im - b.im}; return c; }
static inline zc zrecip(zc a) {
  double d = a.re * a.re + a.im * a.im;
  zc c = {a.re / d, -a.im / d};
  return c;
}
static inline double zabs1(zc a) { return fabs(a.re) + fabs(a.im); }

#define AT(A, lda, r, c) ((A)[(size_t)(c) * (lda) + (r)])

void zgetrf_(int *m, int *n, double *a, int *lda, int *ipiv, int *info) {
  int M = *m, N = *n, L = *lda, j, i, k, p, kmax = M < N ? M : N;
  zc *A = (zc *)a;
  *info = 0;
  for (j = 0; j < kmax; j++) {
    p = j;
    for (i = j + 1; i < M; i++)
      if (zabs1(AT(A, L, i, j)) > zabs1(AT(A, L, p, j)))
        p = i;
    ipiv[j] = p + 1;
    if (AT(A, L, p, j).re == 0.0 && AT(A, L, p, j).im == 0.0) {
      if (*info == 0)
        *info = j + 1;
      continue;
    }
    if (p != j) {
      for (k = 0; k < N; k++) {
        zc t = AT(A, L, j, k);
        AT(A, L, j, k) = AT(A, L, p, k);
        AT(A, L, p, k) = t;
      }
    }
    zc r = zrecip(AT(A, L, j, j));
    for (i = j + 1; i < M; i++)
      AT(A, L, i, j) = zmul(AT(A, L, i, j), r);
    for (k = j + 1; k < N; k++)
      for (i = j + 1; i < M; i++)
        AT(A, L, i, k) = zsub(AT(A, L, i, k), zmul(AT(A, L, i, j), AT(A, L, j, k)));
  }
}

void zgetri_(int *n, double *a, int *lda, int *ipiv, double *work, int *lwork,
             int *info) {
  int N = *n, L = *lda, i, j, k;
  zc *A = (zc *)a, X[16 * 16], col[16];
  (void)work;
  (void)lwork;
  *info = 0;
  if (N > 16) {
    *info = -1;
    return;
  }
  for (j = 0; j < N; j++) {
    /* Solve A x = e_j with P A = L U: apply the row interchanges to e_j */
    for (i = 0; i < N; i++) {
      col[i].re = (i == j) ? 1.0 : 0.0;
      col[i].im = 0.0;
    }
    for (i = 0; i < N; i++) {
      int p = ipiv[i] - 1;
      if (p != i) {
        zc t = col[i];
        col[i] = col[p];
        col[p] = t;
      }
    }
    for (i = 0; i < N; i++)            /* unit lower triangle */
      for (k = 0; k < i; k++)
        col[i] = zsub(col[i], zmul(AT(A, L, i, k), col[k]));
    for (i = N - 1; i >= 0; i--) {     /* upper triangle */
      for (k = i + 1; k < N; k++)
        col[i] = zsub(col[i], zmul(AT(A, L, i, k), col[k]));
      col[i] = zmul(col[i], zrecip(AT(A, L, i, i)));
    }
    for (i = 0; i < N; i++)
      X[j * N + i] = col[i];
  }
  for (j = 0; j < N; j++)
    for (i = 0; i < N; i++)
      AT(A, L, i, j) = X[j * N + i];
}

void zheev_(char *jobz, char *uplo, int *n, double *a, int *lda, double *w,
            double *work, int *lwork, double *rwork, int *info) {
  int N = *n, L = *lda, i, j, p, q, sweep;
  int wantv = (*jobz == 'V' || *jobz == 'v');
  int upper = (*uplo == 'U' || *uplo == 'u');
  zc *A = (zc *)a, H[16][16], V[16][16];
  (void)work;
  (void)lwork;
  (void)rwork;
  *info = 0;
  if (N > 16) {
    *info = -1;
    return;
  }
  /* Rebuild the full Hermitian matrix from the referenced triangle */
  for (i = 0; i < N; i++) {
    for (j = 0; j < N; j++) {
      int use_ij = upper ? (i <= j) : (i >= j);
      zc v = use_ij ? AT(A, L, i, j) : AT(A, L, j, i);
      if (!use_ij)
        v.im = -v.im;
      H[i][j] = v;
      V[i][j].re = (i == j) ? 1.0 : 0.0;
      V[i][j].im = 0.0;
    }
    H[i][i].im = 0.0;
  }

  for (sweep = 0; sweep < 100; sweep++) {
    double off = 0.0, diag = 0.0;
    for (i = 0; i < N; i++) {
      diag += H[i][i].re * H[i][i].re;
      for (j = i + 1; j < N; j++)
        off += H[i][j].re * H[i][j].re + H[i][j].im * H[i][j].im;
    }
    if (off <= 1e-32 * diag || off == 0.0)
      break;
    for (p = 0; p < N; p++) {
      for (q = p + 1; q < N; q++) {
        double r = hypot(H[p][q].re, H[p][q].im);
        if (r == 0.0)
          continue;
        /* Phase that makes H[p][q] real: D = diag(1, e^{-i phi}) on q */
        zc ph = {H[p][q].re / r, H[p][q].im / r};     /* e^{i phi} */
        double theta = (H[q][q].re - H[p][p].re) / (2.0 * r);
        double t = (theta >= 0.0 ? 1.0 : -1.0)
                   / (fabs(theta) + sqrt(theta * theta + 1.0));
        double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
        /* U = D R with R = [[c, s], [-s, c]] in the (p, q) plane:
         *   U_pp = c, U_pq = s, U_qp = -s conj(ph), U_qq = c conj(ph)   */
        zc upp = {c, 0.0}, upq = {s, 0.0};
        zc uqp = {-s * ph.re, s * ph.im}, uqq = {c * ph.re, -c * ph.im};
        /* H <- H U (columns p, q) */
        for (i = 0; i < N; i++) {
          zc hip = H[i][p], hiq = H[i][q];
          zc np = {hip.re * upp.re + hiq.re * uqp.re - hiq.im * uqp.im,
                   hip.im * upp.re + hiq.re * uqp.im + hiq.im * uqp.re};
          zc nq = {hip.re * upq.re + hiq.re * uqq.re - hiq.im * uqq.im,
                   hip.im * upq.re + hiq.re * uqq.im + hiq.im * uqq.re};
          H[i][p] = np;
          H[i][q] = nq;
          zc vip = V[i][p], viq = V[i][q];
          zc wp = {vip.re * upp.re + viq.re * uqp.re - viq.im * uqp.im,
                   vip.im * upp.re + viq.re * uqp.im + viq.im * uqp.re};
          zc wq = {vip.re * upq.re + viq.re * uqq.re - viq.im * uqq.im,
                   vip.im * upq.re + viq.re * uqq.im + viq.im * uqq.re};
          V[i][p] = wp;
          V[i][q] = wq;
        }
        /* H <- U^dag H (rows p, q) */
        for (j = 0; j < N; j++) {
          zc hpj = H[p][j], hqj = H[q][j];
          /* row p: conj(U_pp) H_pj + conj(U_qp) H_qj */
          zc np = {upp.re * hpj.re + uqp.re * hqj.re + uqp.im * hqj.im,
                   upp.re * hpj.im + uqp.re * hqj.im - uqp.im * hqj.re};
          zc nq = {upq.re * hpj.re + uqq.re * hqj.re + uqq.im * hqj.im,
                   upq.re * hpj.im + uqq.re * hqj.im - uqq.im * hqj.re};
          H[p][j] = np;
          H[q][j] = nq;
        }
        H[p][q].re = H[p][q].im = 0.0;
        H[q][p].re = H[q][p].im = 0.0;
        H[p][p].im = H[q][q].im = 0.0;
      }
    }
  }

  /* Sort eigenvalues ascending, carrying eigenvector columns */
  int order[16];
  for (i = 0; i < N; i++)
    order[i] = i;
  for (i = 0; i < N; i++)
    for (j = i + 1; j < N; j++)
      if (H[order[j]][order[j]].re < H[order[i]][order[i]].re) {
        int t = order[i];
        order[i] = order[j];
        order[j] = t;
      }
  for (i = 0; i < N; i++)
    w[i] = H[order[i]][order[i]].re;
  if (wantv)
    for (j = 0; j < N; j++)
      for (i = 0; i < N; i++)
        AT(A, L, i, j) = V[i][order[j]];
}
