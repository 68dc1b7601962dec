// Twisted fermion operator D (sign +1) and D^dag (sign -1) on a
// Twist_Fermion field, fused over all terms of the reference's fermion_op
// (4d_Q16/susy/utilities.c:765-865):
//   Dplus        link -> plaq   (utilities.c:137-221)
//   Dminus       plaq -> link   (utilities.c:228-321)
//   DbplusStoL   site -> link   (utilities.c:517-545)
//   detStoL      site -> link   (utilities.c:551-628, G != 0)
//   DbminusLtoS  link -> site   (utilities.c:634-682)
//   detLtoS      link -> site   (utilities.c:688-756, G != 0)
//   DbminusPtoP, DbplusPtoP plaq -> plaq (utilities.c:327-510)
// sign -1 applies D to the adjoint of every input matrix and stores the
// negated adjoint, exactly as fermion_op(..., MINUS) does.
//
// Decomposition: one thread computes one of the 16 output matrices of one
// site; block b handles output component b % 16 for sites
// (b / 16) * 128 ... + 127, so the 16 components of a site range run
// back to back and neighbour re-reads are served from L2.  All neighbour
// offsets are compile-time constants; no index tables are read.
//
// Optional epilogue (used by DSq inside the CG): out += addc * add and a
// per-block partial of Re<add, out> in FP64.
#include "common.cuh"
#include "fop.cuh"
#include "kernels.h"

namespace susy {

template <int N, typename R, int SIGN, int A, int B, int C, int P, int Q>
SUSY_D void ptop_terms(Mat<N, R>& acc, const FopArgs<R>& a, const Site& c) {
  const bool ADJ = SIGN < 0;
  const Geo& g = a.g;
  const int S = g.S;
  // Ubar_c(x - c), shared by both term families
  Mat<N, R> Ucm = ldm<N, R>(a.U, C, nbr(g, c, -ex(C), -ey(C), -ez(C), -et(C)), S);
  // DbplusPtoP with output (a,b) = (A,B) and (d,e) = (P,Q):
  //   0.5 eps(A,B,C,P,Q) [bc3 chi_PQ(x+A+B+C) Ubar_C(x+A+B) - bc2 Ubar_C(x-C) chi_PQ(x+A+B)]
  {
    constexpr int dx = ex(A) + ex(B), dy = ey(A) + ey(B), dz = ez(A) + ez(B), dt = et(A) + et(B);
    const R t = (R)(0.5 * eps5(A, B, C, P, Q));
    Mat<N, R> chi = ldm<N, R, ADJ>(a.src, 6 + pidx(P, Q),
                                   nbr(g, c, dx + ex(C), dy + ey(C), dz + ez(C), dt + et(C)), S);
    Mat<N, R> Uc = ldm<N, R>(a.U, C, nbr(g, c, dx, dy, dz, dt), S);
    mac<1>(acc, t * bcf<R>(g, c, dt + et(C)), chi, Uc);
    Mat<N, R> chi2 = ldm<N, R, ADJ>(a.src, 6 + pidx(P, Q), nbr(g, c, dx, dy, dz, dt), S);
    mac<2>(acc, -t * bcf<R>(g, c, dt), Ucm, chi2);
  }
  // DbminusPtoP with output (d,e) = (A,B) and (a,b) = (P,Q):
  //   0.5 eps(P,Q,C,A,B) [bc2 chi_PQ(x-P-Q) Ubar_C(x-P-Q-C) - bc3 Ubar_C(x-C) chi_PQ(x-P-Q-C)]
  {
    constexpr int dx = -ex(P) - ex(Q), dy = -ey(P) - ey(Q), dz = -ez(P) - ez(Q), dt = -et(P) - et(Q);
    const R t = (R)(0.5 * eps5(P, Q, C, A, B));
    Mat<N, R> chi = ldm<N, R, ADJ>(a.src, 6 + pidx(P, Q), nbr(g, c, dx, dy, dz, dt), S);
    Mat<N, R> Uc = ldm<N, R>(a.U, C, nbr(g, c, dx - ex(C), dy - ey(C), dz - ez(C), dt - et(C)), S);
    mac<1>(acc, t * bcf<R>(g, c, dt), chi, Uc);
    Mat<N, R> chi2 = ldm<N, R, ADJ>(a.src, 6 + pidx(P, Q),
                                    nbr(g, c, dx - ex(C), dy - ey(C), dz - ez(C), dt - et(C)), S);
    mac<2>(acc, -t * bcf<R>(g, c, dt - et(C)), Ucm, chi2);
  }
}

// Output chi'_AB (A < B)
template <int N, typename R, int SIGN, int A, int B>
SUSY_D Mat<N, R> plaq_out(const FopArgs<R>& a, const Site& c) {
  const bool ADJ = SIGN < 0;
  const Geo& g = a.g;
  const int S = g.S, s = c.s;
  const int pA = nbr(g, c, ex(A), ey(A), ez(A), et(A));
  const int pB = nbr(g, c, ex(B), ey(B), ez(B), et(B));
  Mat<N, R> acc;
  acc.zero();
  // Dplus: bc[A] U_A psi_B(x+A) - psi_B U_A(x+B) - bc[B] U_B psi_A(x+B) + psi_A U_B(x+A)
  {
    Mat<N, R> m1 = ldm<N, R>(a.U, A, s, S);
    Mat<N, R> m2 = ldm<N, R, ADJ>(a.src, 1 + B, pA, S);
    mac<0>(acc, bcf<R>(g, c, et(A)), m1, m2);
    m1 = ldm<N, R, ADJ>(a.src, 1 + B, s, S);
    m2 = ldm<N, R>(a.U, A, pB, S);
    mac<0>(acc, (R)-1, m1, m2);
    m1 = ldm<N, R>(a.U, B, s, S);
    m2 = ldm<N, R, ADJ>(a.src, 1 + A, pB, S);
    mac<0>(acc, -bcf<R>(g, c, et(B)), m1, m2);
    m1 = ldm<N, R, ADJ>(a.src, 1 + A, s, S);
    m2 = ldm<N, R>(a.U, B, pA, S);
    mac<0>(acc, (R)1, m1, m2);
  }
  typedef Compl<A, B> K;
  ptop_terms<N, R, SIGN, A, B, K::K0, K::K1, K::K2>(acc, a, c);
  ptop_terms<N, R, SIGN, A, B, K::K1, K::K0, K::K2>(acc, a, c);
  ptop_terms<N, R, SIGN, A, B, K::K2, K::K0, K::K1>(acc, a, c);
  return acc;
}

// Output psi'_B
template <int N, typename R, int SIGN, int B>
SUSY_D Mat<N, R> link_out(const FopArgs<R>& a, const Site& c) {
  const bool ADJ = SIGN < 0;
  const Geo& g = a.g;
  const int S = g.S, s = c.s;
  Mat<N, R> acc;
  acc.zero();
  // Dminus: sum_{a != B} U_a(x+B) chi_aB(x) - bc[-a] chi_aB(x-a) U_a(x-a)
  const int pB = nbr(g, c, ex(B), ey(B), ez(B), et(B));
#pragma unroll
  for (int e = 0; e < NUMLINK; e++) {
    if (e == B) continue;
    const R sg = e < B ? (R)1 : (R)-1;
    const int mA = nbr(g, c, -ex(e), -ey(e), -ez(e), -et(e));
    Mat<N, R> m1 = ldm<N, R>(a.U, e, pB, S);
    Mat<N, R> m2 = ldm<N, R, ADJ>(a.src, 6 + pidx(e, B), s, S);
    mac<0>(acc, sg, m1, m2);
    m1 = ldm<N, R, ADJ>(a.src, 6 + pidx(e, B), mA, S);
    m2 = ldm<N, R>(a.U, e, mA, S);
    mac<0>(acc, -sg * bcf<R>(g, c, -et(e)), m1, m2);
  }
  // DbplusStoL: 1/2 [bc[B] eta(x+B) Ubar_B - Ubar_B eta]
  {
    Mat<N, R> u = ldm<N, R>(a.U, B, s, S);
    Mat<N, R> eta = ldm<N, R, ADJ>(a.src, 0, pB, S);
    mac<1>(acc, (R)0.5 * bcf<R>(g, c, et(B)), eta, u);
    eta = ldm<N, R, ADJ>(a.src, 0, s, S);
    mac<2>(acc, (R)-0.5, u, eta);
  }
  // detStoL: -1/2 C2 G U_B^{-1} sum_e [Tr eta pd[e][B](x) + bc[-e] Tr eta pd[B][e](x-e)]
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
    const R localG = (R)(-0.5) * a.G;
    Mat<N, R> ui = ldm<N, R>(a.Uinv, B, s, S);
    axpy(acc, localG * tsum, ui);
  }
  return acc;
}

// Output eta'
template <int N, typename R, int SIGN>
SUSY_D Mat<N, R> site_out(const FopArgs<R>& a, const Site& c) {
  const bool ADJ = SIGN < 0;
  const Geo& g = a.g;
  const int S = g.S, s = c.s;
  Mat<N, R> acc;
  acc.zero();
  // DbminusLtoS: 1/2 sum_a [psi_a Ubar_a - bc[-a] Ubar_a(x-a) psi_a(x-a)]
#pragma unroll
  for (int e = 0; e < NUMLINK; e++) {
    const int mE = nbr(g, c, -ex(e), -ey(e), -ez(e), -et(e));
    Mat<N, R> m1 = ldm<N, R, ADJ>(a.src, 1 + e, s, S);
    Mat<N, R> m2 = ldm<N, R>(a.U, e, s, S);
    mac<1>(acc, (R)0.5, m1, m2);
    m1 = ldm<N, R>(a.U, e, mE, S);
    m2 = ldm<N, R, ADJ>(a.src, 1 + e, mE, S);
    mac<2>(acc, (R)-0.5 * bcf<R>(g, c, -et(e)), m1, m2);
  }
  // detLtoS: eta' -= Lambda_U(1) * sum_{a!=b} i G' pd[a][b] (T_b(x) + bc[b] T_a(x+b)),
  // T_a = Tr[U_a^{-1} psi_a], G' = C2 G sqrt(N) / 2, Lambda_U(1) = i I / sqrt(N)
  if (a.doG) {
    Cx<R> T0[NUMLINK];
#pragma unroll
    for (int e = 0; e < NUMLINK; e++) {
      Mat<N, R> ui = ldm<N, R>(a.Uinv, e, s, S);
      Mat<N, R> ps = ldm<N, R, ADJ>(a.src, 1 + e, s, S);
      T0[e] = trace_nn(ui, ps);
    }
    Cx<R> tsum(0, 0);
#pragma unroll
    for (int b = 0; b < NUMLINK; b++) {
      const int pb = nbr(g, c, ex(b), ey(b), ez(b), et(b));
      const R bcb = bcf<R>(g, c, et(b));
#pragma unroll
      for (int e = 0; e < NUMLINK; e++) {
        if (e == b) continue;
        Mat<N, R> ui = ldm<N, R>(a.Uinv, e, pb, S);
        Mat<N, R> ps = ldm<N, R, ADJ>(a.src, 1 + e, pb, S);
        Cx<R> Tp = trace_nn(ui, ps);
        tsum = tsum + ldc<R>(a.pd + (size_t)(e * 5 + b) * S + s) * (T0[b] + bcb * Tp);
      }
    }
    // -(i/sqrt N) * (i G') * tsum = (G'/sqrt N) tsum = (C2 G / 2) tsum
    const Cx<R> d = ((R)0.5 * a.G) * tsum;
#pragma unroll
    for (int i = 0; i < N; i++) acc.e[i][i] = acc.e[i][i] + d;
  }
  return acc;
}

template <int N, typename R, int SIGN, int MINB>
__global__ void __launch_bounds__(FOP_THREADS, MINB)
fermion_op_kernel(FopArgs<R> a) {
  if (a.skip && *a.skip) return;
  const int comp = a.comp_major ? blockIdx.x / a.nsb : blockIdx.x % NTF;
  const int sb = a.comp_major ? blockIdx.x % a.nsb : blockIdx.x / NTF;
  const int s = sb * FOP_THREADS + threadIdx.x;
  const bool live = s < a.g.V;
  double part = 0.0;
  if (live) {
    Site c = site_of(a.g, s);
    Mat<N, R> m;
    switch (comp) {
      case 0: m = site_out<N, R, SIGN>(a, c); break;
      case 1: m = link_out<N, R, SIGN, 0>(a, c); break;
      case 2: m = link_out<N, R, SIGN, 1>(a, c); break;
      case 3: m = link_out<N, R, SIGN, 2>(a, c); break;
      case 4: m = link_out<N, R, SIGN, 3>(a, c); break;
      case 5: m = link_out<N, R, SIGN, 4>(a, c); break;
      case 6: m = plaq_out<N, R, SIGN, 0, 1>(a, c); break;
      case 7: m = plaq_out<N, R, SIGN, 0, 2>(a, c); break;
      case 8: m = plaq_out<N, R, SIGN, 0, 3>(a, c); break;
      case 9: m = plaq_out<N, R, SIGN, 0, 4>(a, c); break;
      case 10: m = plaq_out<N, R, SIGN, 1, 2>(a, c); break;
      case 11: m = plaq_out<N, R, SIGN, 1, 3>(a, c); break;
      case 12: m = plaq_out<N, R, SIGN, 1, 4>(a, c); break;
      case 13: m = plaq_out<N, R, SIGN, 2, 3>(a, c); break;
      case 14: m = plaq_out<N, R, SIGN, 2, 4>(a, c); break;
      default: m = plaq_out<N, R, SIGN, 3, 4>(a, c); break;
    }
    if (SIGN < 0) {
      Mat<N, R> t = m;
#pragma unroll
      for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = 0; j < N; j++) m.e[i][j] = Cx<R>(-t.e[j][i].re, t.e[j][i].im);
    }
    if (a.add) {
      Mat<N, R> x = ldm<N, R>(a.add, comp, s, a.g.S);
      axpy(m, Cx<R>(a.addc, 0), x);
      if (a.dot) part = rdot(x, m);
    }
    stm<N, R>(a.dst, comp, s, a.g.S, m);
  }
  if (a.dot) {
    part = block_sum<FOP_THREADS>(part);
    if (threadIdx.x == 0) a.dot[blockIdx.x] = part;
  }
}

template <int N, typename R, int MINB>
static int launch_fop(FopArgs<R> a, int sign, cudaStream_t st) {
  a.nsb = (a.g.V + FOP_THREADS - 1) / FOP_THREADS;
  const int nblk = a.nsb * NTF;
  if (sign > 0)
    count_launch(), fermion_op_kernel<N, R, 1, MINB><<<nblk, FOP_THREADS, 0, st>>>(a);
  else
    count_launch(), fermion_op_kernel<N, R, -1, MINB><<<nblk, FOP_THREADS, 0, st>>>(a);
  return nblk;
}

// Upper bound on the dot partials any variant writes
int fop_partials(const Geo& g) { return ((g.V + 31) / 32) * NTF; }

// Launch one application; returns the number of dot partials written.
template <typename R>
int fermion_op(const Geo& g, int N, const void* U, const void* Uinv, const void* pd,
                const void* src, void* dst, int sign, double G, const void* add,
                double addc, double* dot, const int* skip, int variant, const int* nbrtab,
                cudaStream_t st, double eta_scale, void* trace) {
  typedef typename CT<R>::T T;
  FopArgs<R> a;
  a.g = g;
  a.U = (const T*)U;
  a.Uinv = (const T*)Uinv;
  a.pd = (const T*)pd;
  a.src = (const T*)src;
  a.dst = (T*)dst;
  a.G = (R)G;
  a.doG = G > 1e-8;
  a.add = (const T*)add;
  a.addc = (R)addc;
  a.dot = dot;
  a.skip = skip;
  a.nbrtab = nbrtab;
  a.eta_scale = (R)eta_scale;
  a.trace = (T*)trace;
  if (variant == FOP_SITE_MAJOR_TR && !trace) variant = FOP_SITE_MAJOR_FRONT;
  if (variant == FOP_ROWS) return fermion_op_rows<R>(a, N, sign, st);
  if (variant >= FOP_COMPACT) return fermion_op_compact<R>(a, N, sign, variant, st);
  a.comp_major = variant == FOP_MAT_CM;
  switch (N) {
    case 2: return launch_fop<2, R, 1>(a, sign, st);
    case 3: return launch_fop<3, R, 1>(a, sign, st);
    default: return launch_fop<4, R, 1>(a, sign, st);
  }
}

template int fermion_op<double>(const Geo&, int, const void*, const void*, const void*,
                                 const void*, void*, int, double, const void*, double,
                                 double*, const int*, int, const int*, cudaStream_t, double,
                                 void*);
template int fermion_op<float>(const Geo&, int, const void*, const void*, const void*,
                                const void*, void*, int, double, const void*, double,
                                double*, const int*, int, const int*, cudaStream_t, double,
                                void*);

}  // namespace susy
