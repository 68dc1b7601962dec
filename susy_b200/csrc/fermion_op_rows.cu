// Row-split variant of the fermion operator (same terms as fermion_op.cu,
// 4d_Q16/susy/utilities.c:141-865): one thread computes ONE ROW of one
// output matrix of one site.  Row i of a product needs row i (or column i)
// of the left factor and the whole right factor, so each thread keeps an
// N-vector accumulator and at most N + N^2 operand values live: about a
// quarter of the registers of the matrix-per-thread kernel, so many more
// warps are resident to hide L2 latency.  The N row-threads of a site sit
// in different warps of the same block and share the right factors through
// L1.  Block = 32 sites x N rows x G site groups; lanes run over
// consecutive sites so every load is a coalesced 32-site transaction.
#include "common.cuh"
#include "fop.cuh"
#include "kernels.h"

namespace susy {

template <int N, typename R>
struct Row {
  Cx<R> e[N];
};

// Row i of X, or of X^dag if ADJ
template <int N, typename R, bool ADJ>
SUSY_D Row<N, R> ldrow(const typename CT<R>::T* f, int k, int s, int S, int i) {
  Row<N, R> r;
  const typename CT<R>::T* p = f + (size_t)(k * N * N) * S + s;
#pragma unroll
  for (int j = 0; j < N; j++)
    r.e[j] = ADJ ? conj(ldc<R>(p + (size_t)(j * N + i) * S)) : ldc<R>(p + (size_t)(i * N + j) * S);
  return r;
}

// Column i of X (X not adjointed): c[k] = X[k][i]
template <int N, typename R>
SUSY_D Row<N, R> ldcol(const typename CT<R>::T* f, int k, int s, int S, int i) {
  Row<N, R> r;
  const typename CT<R>::T* p = f + (size_t)(k * N * N) * S + s;
#pragma unroll
  for (int j = 0; j < N; j++) r.e[j] = ldc<R>(p + (size_t)(j * N + i) * S);
  return r;
}

// acc[j] += s * (row of A*B)[j]:  M = 0: a = row i of A, product A B
//                                 M = 1: a = row i of A, product A B^dag
//                                 M = 2: a = column i of A, product A^dag B
template <int M, int N, typename R>
SUSY_D void macr(Row<N, R>& acc, R s, const Row<N, R>& a, const Mat<N, R>& B) {
#pragma unroll
  for (int j = 0; j < N; j++) {
    R re = 0, im = 0;
#pragma unroll
    for (int k = 0; k < N; k++) {
      const Cx<R> x = (M == 2) ? conj(a.e[k]) : a.e[k];
      const Cx<R> y = (M == 1) ? conj(B.e[j][k]) : B.e[k][j];
      re += x.re * y.re - x.im * y.im;
      im += x.re * y.im + x.im * y.re;
    }
    acc.e[j].re += s * re;
    acc.e[j].im += s * im;
  }
}

template <int N, typename R, int SIGN, int A, int B, int C, int P, int Q>
SUSY_D void ptop_rows(Row<N, R>& acc, const FopArgs<R>& a, const Site& c, int i) {
  const bool ADJ = SIGN < 0;
  const Geo& g = a.g;
  const int S = g.S;
  const Row<N, R> Ucm = ldcol<N, R>(a.U, C, nbr(g, c, -ex(C), -ey(C), -ez(C), -et(C)), S, i);
  {
    constexpr int dx = ex(A) + ex(B), dy = ey(A) + ey(B), dz = ez(A) + ez(B), dt = et(A) + et(B);
    const R t = (R)(0.5 * eps5(A, B, C, P, Q));
    Row<N, R> chi = ldrow<N, R, ADJ>(a.src, 6 + pidx(P, Q),
                                     nbr(g, c, dx + ex(C), dy + ey(C), dz + ez(C), dt + et(C)), S, i);
    Mat<N, R> Uc = ldm<N, R>(a.U, C, nbr(g, c, dx, dy, dz, dt), S);
    macr<1>(acc, t * bcf<R>(g, c, dt + et(C)), chi, Uc);
    Mat<N, R> chi2 = ldm<N, R, ADJ>(a.src, 6 + pidx(P, Q), nbr(g, c, dx, dy, dz, dt), S);
    macr<2>(acc, -t * bcf<R>(g, c, dt), Ucm, chi2);
  }
  {
    constexpr int dx = -ex(P) - ex(Q), dy = -ey(P) - ey(Q), dz = -ez(P) - ez(Q), dt = -et(P) - et(Q);
    const R t = (R)(0.5 * eps5(P, Q, C, A, B));
    Row<N, R> chi = ldrow<N, R, ADJ>(a.src, 6 + pidx(P, Q), nbr(g, c, dx, dy, dz, dt), S, i);
    Mat<N, R> Uc = ldm<N, R>(a.U, C, nbr(g, c, dx - ex(C), dy - ey(C), dz - ez(C), dt - et(C)), S);
    macr<1>(acc, t * bcf<R>(g, c, dt), chi, Uc);
    Mat<N, R> chi2 = ldm<N, R, ADJ>(a.src, 6 + pidx(P, Q),
                                    nbr(g, c, dx - ex(C), dy - ey(C), dz - ez(C), dt - et(C)), S);
    macr<2>(acc, -t * bcf<R>(g, c, dt - et(C)), Ucm, chi2);
  }
}

template <int N, typename R, int SIGN, int A, int B>
SUSY_D Row<N, R> plaq_rows(const FopArgs<R>& a, const Site& c, int i) {
  const bool ADJ = SIGN < 0;
  const Geo& g = a.g;
  const int S = g.S, s = c.s;
  const int pA = nbr(g, c, ex(A), ey(A), ez(A), et(A));
  const int pB = nbr(g, c, ex(B), ey(B), ez(B), et(B));
  Row<N, R> acc;
#pragma unroll
  for (int j = 0; j < N; j++) acc.e[j] = Cx<R>(0, 0);
  {
    Row<N, R> r = ldrow<N, R, false>(a.U, A, s, S, i);
    Mat<N, R> m = ldm<N, R, ADJ>(a.src, 1 + B, pA, S);
    macr<0>(acc, bcf<R>(g, c, et(A)), r, m);
    r = ldrow<N, R, ADJ>(a.src, 1 + B, s, S, i);
    m = ldm<N, R>(a.U, A, pB, S);
    macr<0>(acc, (R)-1, r, m);
    r = ldrow<N, R, false>(a.U, B, s, S, i);
    m = ldm<N, R, ADJ>(a.src, 1 + A, pB, S);
    macr<0>(acc, -bcf<R>(g, c, et(B)), r, m);
    r = ldrow<N, R, ADJ>(a.src, 1 + A, s, S, i);
    m = ldm<N, R>(a.U, B, pA, S);
    macr<0>(acc, (R)1, r, m);
  }
  typedef Compl<A, B> K;
  ptop_rows<N, R, SIGN, A, B, K::K0, K::K1, K::K2>(acc, a, c, i);
  ptop_rows<N, R, SIGN, A, B, K::K1, K::K0, K::K2>(acc, a, c, i);
  ptop_rows<N, R, SIGN, A, B, K::K2, K::K0, K::K1>(acc, a, c, i);
  return acc;
}

template <int N, typename R, int SIGN, int B>
SUSY_D Row<N, R> link_rows(const FopArgs<R>& a, const Site& c, int i) {
  const bool ADJ = SIGN < 0;
  const Geo& g = a.g;
  const int S = g.S, s = c.s;
  Row<N, R> acc;
#pragma unroll
  for (int j = 0; j < N; j++) acc.e[j] = Cx<R>(0, 0);
  const int pB = nbr(g, c, ex(B), ey(B), ez(B), et(B));
#pragma unroll
  for (int e = 0; e < NUMLINK; e++) {
    if (e == B) continue;
    const R sg = e < B ? (R)1 : (R)-1;
    const int mA = nbr(g, c, -ex(e), -ey(e), -ez(e), -et(e));
    Row<N, R> r = ldrow<N, R, false>(a.U, e, pB, S, i);
    Mat<N, R> m = ldm<N, R, ADJ>(a.src, 6 + pidx(e, B), s, S);
    macr<0>(acc, sg, r, m);
    r = ldrow<N, R, ADJ>(a.src, 6 + pidx(e, B), mA, S, i);
    m = ldm<N, R>(a.U, e, mA, S);
    macr<0>(acc, -sg * bcf<R>(g, c, -et(e)), r, m);
  }
  {
    Mat<N, R> u = ldm<N, R>(a.U, B, s, S);
    Row<N, R> eta = ldrow<N, R, ADJ>(a.src, 0, pB, S, i);
    macr<1>(acc, (R)0.5 * bcf<R>(g, c, et(B)), eta, u);
    Row<N, R> uc = ldcol<N, R>(a.U, B, s, S, i);
    Mat<N, R> etm = ldm<N, R, ADJ>(a.src, 0, s, S);
    macr<2>(acc, (R)-0.5, uc, etm);
  }
  if (a.doG) {
    Cx<R> tsum(0, 0);
    const Cx<R> tr0 = ldtr<N, R, ADJ>(a.src, 0, s, S);
#pragma unroll
    for (int e = 0; e < NUMLINK; e++) {
      if (e == B) continue;
      const int mE = nbr(g, c, -ex(e), -ey(e), -ez(e), -et(e));
      tsum = tsum + tr0 * ldc<R>(a.pd + (size_t)(e * 5 + B) * S + s);
      const Cx<R> trm = ldtr<N, R, ADJ>(a.src, 0, mE, S);
      tsum = tsum + bcf<R>(g, c, -et(e)) * (trm * ldc<R>(a.pd + (size_t)(B * 5 + e) * S + mE));
    }
    const Cx<R> cf = ((R)(-0.5) * a.G) * tsum;
    Row<N, R> ui = ldrow<N, R, false>(a.Uinv, B, s, S, i);
#pragma unroll
    for (int j = 0; j < N; j++) acc.e[j] = acc.e[j] + cf * ui.e[j];
  }
  return acc;
}

template <int N, typename R, int SIGN>
SUSY_D Row<N, R> site_rows(const FopArgs<R>& a, const Site& c, int i) {
  const bool ADJ = SIGN < 0;
  const Geo& g = a.g;
  const int S = g.S, s = c.s;
  Row<N, R> acc;
#pragma unroll
  for (int j = 0; j < N; j++) acc.e[j] = Cx<R>(0, 0);
#pragma unroll
  for (int e = 0; e < NUMLINK; e++) {
    const int mE = nbr(g, c, -ex(e), -ey(e), -ez(e), -et(e));
    Row<N, R> r = ldrow<N, R, ADJ>(a.src, 1 + e, s, S, i);
    Mat<N, R> m = ldm<N, R>(a.U, e, s, S);
    macr<1>(acc, (R)0.5, r, m);
    r = ldcol<N, R>(a.U, e, mE, S, i);
    m = ldm<N, R, ADJ>(a.src, 1 + e, mE, S);
    macr<2>(acc, (R)-0.5 * bcf<R>(g, c, -et(e)), r, m);
  }
  if (a.doG) {
    Cx<R> T0[NUMLINK];
#pragma unroll
    for (int e = 0; e < NUMLINK; e++)
      T0[e] = trace_nn(ldm<N, R>(a.Uinv, e, s, S), ldm<N, R, ADJ>(a.src, 1 + e, s, S));
    Cx<R> tsum(0, 0);
#pragma unroll
    for (int b = 0; b < NUMLINK; b++) {
      const int pb = nbr(g, c, ex(b), ey(b), ez(b), et(b));
      const R bcb = bcf<R>(g, c, et(b));
#pragma unroll
      for (int e = 0; e < NUMLINK; e++) {
        if (e == b) continue;
        const Cx<R> Tp = trace_nn(ldm<N, R>(a.Uinv, e, pb, S), ldm<N, R, ADJ>(a.src, 1 + e, pb, S));
        tsum = tsum + ldc<R>(a.pd + (size_t)(e * 5 + b) * S + s) * (T0[b] + bcb * Tp);
      }
    }
    acc.e[i] = acc.e[i] + ((R)0.5 * a.G) * tsum;
  }
  return acc;
}

template <int N> struct RowShape {
  static constexpr int G = (N == 4) ? 1 : 2;   // site groups per block
  static constexpr int SB = 32 * G;             // sites per block
  static constexpr int NT = 32 * N * G;         // threads per block
};

template <int N, typename R, int SIGN>
__global__ void __launch_bounds__(RowShape<N>::NT)
fermion_op_rows_kernel(FopArgs<R> a) {
  if (a.skip && *a.skip) return;
  typedef RowShape<N> SH;
  const int comp = blockIdx.x / a.nsb;   // component-major block order
  const int lane = threadIdx.x & 31;
  const int i = (threadIdx.x >> 5) % N;
  const int grp = threadIdx.x / (32 * N);
  const int s = (blockIdx.x % a.nsb) * SH::SB + grp * 32 + lane;
  double part = 0.0;
  if (s < a.g.V) {
    const Site c = site_of(a.g, s);
    Row<N, R> r;
    switch (comp) {
      case 0: r = site_rows<N, R, SIGN>(a, c, i); break;
      case 1: r = link_rows<N, R, SIGN, 0>(a, c, i); break;
      case 2: r = link_rows<N, R, SIGN, 1>(a, c, i); break;
      case 3: r = link_rows<N, R, SIGN, 2>(a, c, i); break;
      case 4: r = link_rows<N, R, SIGN, 3>(a, c, i); break;
      case 5: r = link_rows<N, R, SIGN, 4>(a, c, i); break;
      case 6: r = plaq_rows<N, R, SIGN, 0, 1>(a, c, i); break;
      case 7: r = plaq_rows<N, R, SIGN, 0, 2>(a, c, i); break;
      case 8: r = plaq_rows<N, R, SIGN, 0, 3>(a, c, i); break;
      case 9: r = plaq_rows<N, R, SIGN, 0, 4>(a, c, i); break;
      case 10: r = plaq_rows<N, R, SIGN, 1, 2>(a, c, i); break;
      case 11: r = plaq_rows<N, R, SIGN, 1, 3>(a, c, i); break;
      case 12: r = plaq_rows<N, R, SIGN, 1, 4>(a, c, i); break;
      case 13: r = plaq_rows<N, R, SIGN, 2, 3>(a, c, i); break;
      case 14: r = plaq_rows<N, R, SIGN, 2, 4>(a, c, i); break;
      default: r = plaq_rows<N, R, SIGN, 3, 4>(a, c, i); break;
    }
    const typename CT<R>::T* addp = a.add;
    typename CT<R>::T* dstp = a.dst + (size_t)(comp * N * N) * a.g.S + s;
#pragma unroll
    for (int j = 0; j < N; j++) {
      // sign +1: element (i, j) = acc[j];  sign -1: element (j, i) = -conj(acc[j])
      const int off = SIGN > 0 ? (i * N + j) : (j * N + i);
      Cx<R> v = SIGN > 0 ? r.e[j] : Cx<R>(-r.e[j].re, r.e[j].im);
      if (addp) {
        const Cx<R> x = ldc<R>(addp + (size_t)(comp * N * N + off) * a.g.S + s);
        v = v + a.addc * x;
        part += (double)x.re * v.re + (double)x.im * v.im;
      }
      stc<R>(dstp + (size_t)off * a.g.S, v);
    }
  }
  if (a.dot) {
    part = block_sum<RowShape<N>::NT>(part);
    if (threadIdx.x == 0) a.dot[blockIdx.x] = part;
  }
}

template <int N, typename R>
static int launch_rows(FopArgs<R> a, int sign, cudaStream_t st) {
  typedef RowShape<N> SH;
  a.nsb = (a.g.V + SH::SB - 1) / SH::SB;
  const int nblk = a.nsb * NTF;
  if (sign > 0)
    count_launch(), fermion_op_rows_kernel<N, R, 1><<<nblk, SH::NT, 0, st>>>(a);
  else
    count_launch(), fermion_op_rows_kernel<N, R, -1><<<nblk, SH::NT, 0, st>>>(a);
  return nblk;
}

template <typename R>
int fermion_op_rows(const FopArgs<R>& a, int N, int sign, cudaStream_t st) {
  switch (N) {
    case 2: return launch_rows<2, R>(a, sign, st);
    case 3: return launch_rows<3, R>(a, sign, st);
    default: return launch_rows<4, R>(a, sign, st);
  }
}

template int fermion_op_rows<double>(const FopArgs<double>&, int, int, cudaStream_t);
template int fermion_op_rows<float>(const FopArgs<float>&, int, int, cudaStream_t);

}  // namespace susy
