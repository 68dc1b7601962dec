// Small dense linear algebra on NCOL x NCOL complex matrices in registers
// (NCOL <= 4, FP64), used by the derived fields and the measurements.
//   det_inv    determinant and inverse: Gauss-Jordan elimination with
//              partial pivoting on |re| + |im| (LAPACK's pivot measure), in
//              place of the reference's zgetrf/zgetri (determinant.c:10-85)
//   herm_eig   eigenvalues (ascending) and optionally eigenvectors of a
//              Hermitian matrix by the cyclic Jacobi method (a complex
//              rotation per off-diagonal pair, Golub & Van Loan section 8.5
//              extended to Hermitian matrices by a diagonal phase), in place
//              of the reference's zheev (scalar_eig.c:68, unit.c:24,64)
#pragma once
#include "common.cuh"

namespace susy {

template <int N>
SUSY_D void det_inv(const Mat<N, double>& A, Cx<double>& det, Mat<N, double>& inv) {
  Mat<N, double> a = A;
  inv.zero();
#pragma unroll
  for (int i = 0; i < N; i++) inv.e[i][i] = Cx<double>(1, 0);
  det = Cx<double>(1, 0);
#pragma unroll
  for (int k = 0; k < N; k++) {
    int p = k;
    double best = fabs(a.e[k][k].re) + fabs(a.e[k][k].im);
#pragma unroll
    for (int i = k + 1; i < N; i++) {
      double v = fabs(a.e[i][k].re) + fabs(a.e[i][k].im);
      if (v > best) { best = v; p = i; }
    }
    if (p != k) {
      det = Cx<double>(-det.re, -det.im);
#pragma unroll
      for (int j = 0; j < N; j++) {
        // swap rows k and p (register arrays indexed through a select)
#pragma unroll
        for (int i = k + 1; i < N; i++)
          if (i == p) {
            Cx<double> t = a.e[k][j]; a.e[k][j] = a.e[i][j]; a.e[i][j] = t;
            t = inv.e[k][j]; inv.e[k][j] = inv.e[i][j]; inv.e[i][j] = t;
          }
      }
    }
    Cx<double> piv = a.e[k][k];
    det = det * piv;
    double d2 = piv.re * piv.re + piv.im * piv.im;
    Cx<double> r(piv.re / d2, -piv.im / d2);
#pragma unroll
    for (int j = 0; j < N; j++) {
      a.e[k][j] = a.e[k][j] * r;
      inv.e[k][j] = inv.e[k][j] * r;
    }
#pragma unroll
    for (int i = 0; i < N; i++) {
      if (i == k) continue;
      Cx<double> f = a.e[i][k];
#pragma unroll
      for (int j = 0; j < N; j++) {
        a.e[i][j] = a.e[i][j] - f * a.e[k][j];
        inv.e[i][j] = inv.e[i][j] - f * inv.e[k][j];
      }
    }
  }
}

// Hermitian A = V diag(w) V^dag, w ascending.  Each rotation zeroes
// A[p][q] = g e^{i phi}: with tau = (A_qq - A_pp) / 2g, t = sign(tau) /
// (|tau| + sqrt(1 + tau^2)), c = 1 / sqrt(1 + t^2), s = t c, the unitary Q
// acting on columns p, q as [[c, s], [-s e^{-i phi}, c e^{-i phi}]] gives
// Q^dag A Q with a zero (p, q) entry.  Sweeps stop once the off-diagonal
// weight is below 1e-30 of the diagonal (quadratic convergence: a handful
// of sweeps at NCOL <= 4).
template <int N>
SUSY_D void herm_eig(Mat<N, double> A, double (&w)[N], Mat<N, double>* V) {
  if (V) {
    V->zero();
#pragma unroll
    for (int i = 0; i < N; i++) V->e[i][i] = Cx<double>(1, 0);
  }
#pragma unroll 1
  for (int sweep = 0; sweep < 16; sweep++) {
    double off = 0.0, dg = 0.0;
#pragma unroll
    for (int p = 0; p < N; p++) {
      dg += A.e[p][p].re * A.e[p][p].re;
#pragma unroll
      for (int q = p + 1; q < N; q++) off += A.e[p][q].re * A.e[p][q].re + A.e[p][q].im * A.e[p][q].im;
    }
    if (!(off > 1e-30 * dg)) break;
#pragma unroll
    for (int p = 0; p < N; p++)
#pragma unroll
      for (int q = p + 1; q < N; q++) {
        const Cx<double> apq = A.e[p][q];
        const double g = sqrt(apq.re * apq.re + apq.im * apq.im);
        if (g == 0.0) continue;
        const Cx<double> e(apq.re / g, apq.im / g);     // e^{i phi}
        const Cx<double> ec(e.re, -e.im);               // e^{-i phi}
        const double tau = (A.e[q][q].re - A.e[p][p].re) / (2.0 * g);
        const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
        const double c = 1.0 / sqrt(1.0 + t * t), s = t * c;
        // columns: A Q
#pragma unroll
        for (int k = 0; k < N; k++) {
          const Cx<double> akp = A.e[k][p], akq = ec * A.e[k][q];
          A.e[k][p] = Cx<double>(c * akp.re - s * akq.re, c * akp.im - s * akq.im);
          A.e[k][q] = Cx<double>(s * akp.re + c * akq.re, s * akp.im + c * akq.im);
        }
        // rows: Q^dag (A Q)
#pragma unroll
        for (int k = 0; k < N; k++) {
          const Cx<double> apk = A.e[p][k], aqk = e * A.e[q][k];
          A.e[p][k] = Cx<double>(c * apk.re - s * aqk.re, c * apk.im - s * aqk.im);
          A.e[q][k] = Cx<double>(s * apk.re + c * aqk.re, s * apk.im + c * aqk.im);
        }
        A.e[p][q] = A.e[q][p] = Cx<double>(0, 0);
        A.e[p][p].im = A.e[q][q].im = 0.0;
        if (V) {
#pragma unroll
          for (int k = 0; k < N; k++) {
            const Cx<double> vkp = V->e[k][p], vkq = ec * V->e[k][q];
            V->e[k][p] = Cx<double>(c * vkp.re - s * vkq.re, c * vkp.im - s * vkq.im);
            V->e[k][q] = Cx<double>(s * vkp.re + c * vkq.re, s * vkp.im + c * vkq.im);
          }
        }
      }
  }
#pragma unroll
  for (int i = 0; i < N; i++) w[i] = A.e[i][i].re;
  // ascending order (with the eigenvectors): exchange sort over fixed indices
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = i + 1; j < N; j++)
      if (w[j] < w[i]) {
        const double tw = w[i];
        w[i] = w[j];
        w[j] = tw;
        if (V) {
#pragma unroll
          for (int k = 0; k < N; k++) {
            const Cx<double> tv = V->e[k][i];
            V->e[k][i] = V->e[k][j];
            V->e[k][j] = tv;
          }
        }
      }
}

}  // namespace susy
