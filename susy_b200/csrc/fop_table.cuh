// The fermion operator as a table of NCOL x NCOL products (host builder) and
// the device pieces every table-driven operator kernel shares: temporal BC
// masks, the determinant terms and the epilogue.
//
// Every product of 4d_Q16/susy/utilities.c:141-865 is one row: output
// component, operand pattern, coefficient, the net time displacement that
// selects its BC factor (setup_offset.c:67-145), and for each factor the
// field component and the neighbour displacement (an index into the
// displacement list).
//
// On the A4* basis e_0 + e_1 + e_2 + e_3 + e_4 = 0 (e_4 = (-1,-1,-1,-1),
// setup_offset.c:155-162).  For an output chi_AB and C, P, Q the other three
// link indices, A + B + C = -(P + Q) and A + B = -(P + Q + C).  Then the
// terms DbminusPtoP (utilities.c:420-510) adds to chi_AB,
//   chi_PQ(x-P-Q) Ubar_C(x-P-Q-C)  and  Ubar_C(x-C) chi_PQ(x-P-Q-C),
// are the very products DbplusPtoP (utilities.c:327-414) adds,
//   chi_PQ(x+A+B+C) Ubar_C(x+A+B)  and  Ubar_C(x-C) chi_PQ(x+A+B),
// with the same BC factors and equal coefficients (eps(P,Q,C,A,B) =
// eps(A,B,C,P,Q): the two permutations differ by two transpositions).  The
// builder therefore merges rows with identical operands, summing their
// coefficients: 220 products per site become 160, every output component
// has exactly 10.  The merged operator equals the reference's up to the
// order of floating-point additions.
#pragma once
#include <initializer_list>
#include <vector>
#include "common.cuh"
#include "fop.cuh"

namespace susy {

// Operand patterns: every product is one of
//   P_UF: U * F     P_FU: F * U     P_FUD: F * U^dag     P_UDF: U^dag * F
// (F = the source Twist_Fermion, itself adjointed when sign = -1)
enum { P_UF = 0, P_FU = 1, P_FUD = 2, P_UDF = 3, NPAT = 4 };

struct FTerm {
  int8_t kl, dl, kr, dr;   // components and displacement indices of the factors
  int8_t bcdt;
  int8_t sl, sr;           // slots of dl, dr in the output's displacement list
  int8_t pad;
  float coef;
};

constexpr int MAX_TERMS = 224;
constexpr int MAX_DISP = 64;

struct TermBuilder {
  std::vector<FTerm> terms[NTF][NPAT];
  std::vector<char4> disp;

  int d(int dx, int dy, int dz, int dt) {
    for (size_t i = 0; i < disp.size(); i++)
      if (disp[i].x == dx && disp[i].y == dy && disp[i].z == dz && disp[i].w == dt) return (int)i;
    disp.push_back(make_char4(dx, dy, dz, dt));
    return (int)disp.size() - 1;
  }
  // displacement of a signed sum of link offsets
  int dl(std::initializer_list<int> plus, std::initializer_list<int> minus = {}) {
    int x = 0, y = 0, z = 0, t = 0;
    for (int a : plus) { x += ex(a); y += ey(a); z += ez(a); t += et(a); }
    for (int a : minus) { x -= ex(a); y -= ey(a); z -= ez(a); t -= et(a); }
    return d(x, y, z, t);
  }
  static int tdt(std::initializer_list<int> plus, std::initializer_list<int> minus = {}) {
    int t = 0;
    for (int a : plus) t += et(a);
    for (int a : minus) t -= et(a);
    return t;
  }
  // A row; a row with the same pattern, BC displacement and operands as an
  // earlier one of the same output is merged into it
  void add(int comp, int pat, double coef, int bcdt, int kl, int dlv, int kr, int drv) {
    for (FTerm& o : terms[comp][pat])
      if (o.kl == kl && o.dl == dlv && o.kr == kr && o.dr == drv && o.bcdt == bcdt) {
        o.coef = (float)(o.coef + coef);
        return;
      }
    FTerm T;
    T.kl = kl; T.dl = dlv; T.kr = kr; T.dr = drv;
    T.bcdt = bcdt; T.sl = T.sr = T.pad = 0;
    T.coef = (float)coef;
    terms[comp][pat].push_back(T);
  }

  void build() {
    // component 0: eta'  (DbminusLtoS, utilities.c:634-682)
    for (int e = 0; e < 5; e++) {
      add(0, P_FUD, 0.5, 0, 1 + e, dl({}), e, dl({}));
      add(0, P_UDF, -0.5, tdt({}, {e}), e, dl({}, {e}), 1 + e, dl({}, {e}));
    }
    // components 1..5: psi'_B  (Dminus 228-321, DbplusStoL 517-545)
    for (int B = 0; B < 5; B++) {
      for (int e = 0; e < 5; e++) {
        if (e == B) continue;
        const double sg = e < B ? 1.0 : -1.0;
        add(1 + B, P_UF, sg, 0, e, dl({B}), 6 + pidx(e, B), dl({}));
        add(1 + B, P_FU, -sg, tdt({}, {e}), 6 + pidx(e, B), dl({}, {e}), e, dl({}, {e}));
      }
      add(1 + B, P_FUD, 0.5, tdt({B}), 0, dl({B}), B, dl({}));
      add(1 + B, P_UDF, -0.5, 0, B, dl({}), 0, dl({}));
    }
    // components 6..15: chi'_AB  (Dplus 137-221, DbplusPtoP 327-414,
    // DbminusPtoP 420-510; the last two merge, see the file comment)
    for (int A = 0; A < 5; A++)
      for (int B = A + 1; B < 5; B++) {
        const int q = 6 + pidx(A, B);
        add(q, P_UF, 1.0, tdt({A}), A, dl({}), 1 + B, dl({A}));
        add(q, P_FU, -1.0, 0, 1 + B, dl({}), A, dl({B}));
        add(q, P_UF, -1.0, tdt({B}), B, dl({}), 1 + A, dl({B}));
        add(q, P_FU, 1.0, 0, 1 + A, dl({}), B, dl({A}));
        int K[3], k = 0;
        for (int v = 0; v < 5; v++)
          if (v != A && v != B) K[k++] = v;
        for (int ci = 0; ci < 3; ci++) {
          const int C = K[ci];
          const int P = ci == 0 ? K[1] : K[0];
          const int Q = ci == 2 ? K[1] : K[2];
          const int pq = 6 + pidx(P, Q);
          const double t1 = 0.5 * eps5(A, B, C, P, Q), t2 = 0.5 * eps5(P, Q, C, A, B);
          add(q, P_FUD, t1, tdt({A, B, C}), pq, dl({A, B, C}), C, dl({A, B}));
          add(q, P_UDF, -t1, tdt({A, B}), C, dl({}, {C}), pq, dl({A, B}));
          add(q, P_FUD, t2, tdt({}, {P, Q}), pq, dl({}, {P, Q}), C, dl({}, {P, Q, C}));
          add(q, P_UDF, -t2, tdt({}, {P, Q, C}), C, dl({}, {C}), pq, dl({}, {P, Q, C}));
        }
      }
  }
};

// The builder's result, made once per process (thread-safe static init)
const TermBuilder& fop_terms();

// ---------------------------------------------------------------------------
// Device
// Temporal BC factors of a thread's site for net displacements -3..3:
// bit (dt + 3) set when t + dt leaves [0, nt - 1]
SUSY_D unsigned bc_mask(const Geo& g, const Site& c) {
  unsigned m = 0;
#pragma unroll
  for (int dt = -3; dt <= 3; dt++) {
    const int t = c.t + dt;
    if (t < 0 || t > g.nt - 1) m |= 1u << (dt + 3);
  }
  return m;
}

template <typename R>
SUSY_D R bc_of(unsigned mask, int dt, R pbc) {
  return ((mask >> (dt + 3)) & 1u) ? pbc : (R)1;
}

// Tr(A op(B)) for A = component ka of fa at site sa and B = component kb of
// fb at site sb (op(B) = B^dag when ADJB), one element pair at a time: the
// determinant terms run while the accumulator is live, and holding whole
// matrices here made the register-capped kernels spill
template <int N, typename R, bool ADJB>
SUSY_D Cx<R> trace_ld(const typename CT<R>::T* fa, int ka, int sa, const typename CT<R>::T* fb,
                      int kb, int sb, int S) {
  const typename CT<R>::T* pa = fa + (size_t)(ka * N * N) * S + sa;
  const typename CT<R>::T* pb = fb + (size_t)(kb * N * N) * S + sb;
  Cx<R> t(0, 0);
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int k = 0; k < N; k++) {
      const Cx<R> x = ldc<R>(pa + (size_t)(i * N + k) * S);
      const Cx<R> y = ADJB ? conj(ldc<R>(pb + (size_t)(i * N + k) * S))
                           : ldc<R>(pb + (size_t)(k * N + i) * S);
      t = t + x * y;
    }
  return t;
}

// detStoL for output link B (utilities.c:551-628)
template <int N, typename R, int SIGN>
SUSY_D void det_stol_rt(Mat<N, R>& acc, const FopArgs<R>& a, const Site& c, int B) {
  const bool ADJ = SIGN < 0;
  const Geo& g = a.g;
  const int S = g.S, s = c.s;
  Cx<R> tsum(0, 0);
  const Cx<R> tr0 = ldtr<N, R, ADJ>(a.src, 0, s, S);
#pragma unroll 1
  for (int e = 0; e < NUMLINK; e++) {
    if (e == B) continue;
    const int mE = nbr(g, c, -ex(e), -ey(e), -ez(e), -et(e));
    tsum = tsum + tr0 * ldc<R>(a.pd + (size_t)(e * 5 + B) * S + s);
    const Cx<R> trm = ldtr<N, R, ADJ>(a.src, 0, mE, S);
    tsum = tsum + bcf<R>(g, c, -et(e)) * (trm * ldc<R>(a.pd + (size_t)(B * 5 + e) * S + mE));
  }
  // every term carries Tr eta, doubled with the reference's RESCALE
  const Cx<R> f = ((R)(-0.5) * a.G * a.eta_scale) * tsum;
  const typename CT<R>::T* pu = a.Uinv + (size_t)(B * N * N) * S + s;
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) acc.e[i][j] = acc.e[i][j] + f * ldc<R>(pu + (size_t)(i * N + j) * S);
}

// detLtoS for the site output (utilities.c:688-756)
template <int N, typename R, int SIGN>
SUSY_D void det_ltos_rt(Mat<N, R>& acc, const FopArgs<R>& a, const Site& c) {
  const bool ADJ = SIGN < 0;
  const Geo& g = a.g;
  const int S = g.S, s = c.s;
  Cx<R> T0[NUMLINK];
#pragma unroll
  for (int e = 0; e < NUMLINK; e++) T0[e] = trace_ld<N, R, ADJ>(a.Uinv, e, s, a.src, 1 + e, s, S);
  Cx<R> tsum(0, 0);
#pragma unroll 1
  for (int b = 0; b < NUMLINK; b++) {
    const int pb = nbr(g, c, ex(b), ey(b), ez(b), et(b));
    const R bcb = bcf<R>(g, c, et(b));
    Cx<R> T0b = T0[0];
#pragma unroll
    for (int e = 1; e < NUMLINK; e++)
      if (e == b) T0b = T0[e];
#pragma unroll 1
    for (int e = 0; e < NUMLINK; e++) {
      if (e == b) continue;
      const Cx<R> Tp = trace_ld<N, R, ADJ>(a.Uinv, e, pb, a.src, 1 + e, pb, S);
      tsum = tsum + ldc<R>(a.pd + (size_t)(e * 5 + b) * S + s) * (T0b + bcb * Tp);
    }
  }
  const Cx<R> d = ((R)0.5 * a.G) * tsum;
#pragma unroll
  for (int i = 0; i < N; i++) acc.e[i][i] = acc.e[i][i] + d;
}

// Every site's five detLtoS traces Tr(U_e^-1(x) src_{1+e}(x)) (the source
// adjointed for D^dag), tr[e * S + x], summed as trace_ld sums them: the
// pre-pass of FOP_SITE_MAJOR_TR.  One thread per (site, e), e = blockIdx.y:
// one thread per site looping over e left too few loads in flight (the
// pre-pass took ~25 us in FP64 at 12^3x24 U(3), for 63 MB; now 11.5 us).
// Measured there (ncu, FP64): the operator kernel after it takes 147-154 us
// against 167-176 us recomputing the traces, moves 2.01 against 2.30 GB
// from L2 and 319 against 372 MB of DRAM (the site component's blocks no
// longer gather 470 complex numbers each); pre-pass included, D^dag D runs
// at 0.169 / 0.098 ms per launch (FP64 / FP32) against 0.170 / 0.099
// without it, and 0.171 / 0.101 with the trace pre-pass but the plain
// site-major block order.
template <int N, typename R, bool ADJ>
__global__ void k_det_traces(FopArgs<R> a) {
  if (a.skip && *a.skip) return;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int e = blockIdx.y;
  if (s >= a.g.V) return;
  const int S = a.g.S;
  stc<R>(a.trace + (size_t)e * S + s, trace_ld<N, R, ADJ>(a.Uinv, e, s, a.src, 1 + e, s, S));
}

// detLtoS from the pre-pass's traces: the sums of det_ltos_rt in the same
// order, 25 trace loads in place of 25 traces of two matrices each
template <int N, typename R, int SIGN>
SUSY_D void det_ltos_tr(Mat<N, R>& acc, const FopArgs<R>& a, const Site& c) {
  const Geo& g = a.g;
  const int S = g.S, s = c.s;
  Cx<R> tsum(0, 0);
#pragma unroll 1
  for (int b = 0; b < NUMLINK; b++) {
    const int pb = nbr(g, c, ex(b), ey(b), ez(b), et(b));
    const R bcb = bcf<R>(g, c, et(b));
    const Cx<R> T0b = ldc<R>(a.trace + (size_t)b * S + s);
#pragma unroll 1
    for (int e = 0; e < NUMLINK; e++) {
      if (e == b) continue;
      const Cx<R> Tp = ldc<R>(a.trace + (size_t)e * S + pb);
      tsum = tsum + ldc<R>(a.pd + (size_t)(e * 5 + b) * S + s) * (T0b + bcb * Tp);
    }
  }
  const Cx<R> d = ((R)0.5 * a.G) * tsum;
#pragma unroll
  for (int i = 0; i < N; i++) acc.e[i][i] = acc.e[i][i] + d;
}

// The reference's RESCALE doubles the site component of the output
// (utilities.c:841-844)
template <int N, typename R>
SUSY_D void eta_rescale(Mat<N, R>& acc, R sc) {
  if (sc == (R)1) return;
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) acc.e[i][j] = sc * acc.e[i][j];
}

// Shared epilogue: determinant terms, adjoint for D^dag, axpy and dot
// (TR: detLtoS from the traces of k_det_traces)
template <int N, typename R, int SIGN, bool TR = false>
SUSY_D double fop_finish(Mat<N, R>& acc, const FopArgs<R>& a, const Site& c, int comp) {
  if (a.doG) {
    if (comp == 0) {
      if (TR)
        det_ltos_tr<N, R, SIGN>(acc, a, c);
      else
        det_ltos_rt<N, R, SIGN>(acc, a, c);
    } else if (comp <= NUMLINK) {
      det_stol_rt<N, R, SIGN>(acc, a, c, comp - 1);
    }
  }
  if (comp == 0) eta_rescale(acc, a.eta_scale);
  if (SIGN < 0) {
    Mat<N, R> t = acc;
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
      for (int j = 0; j < N; j++) acc.e[i][j] = Cx<R>(-t.e[j][i].re, t.e[j][i].im);
  }
  double part = 0.0;
  if (a.add) {
    Mat<N, R> x = ldm<N, R>(a.add, comp, c.s, a.g.S);
    axpy(acc, Cx<R>(a.addc, 0), x);
    if (a.dot) part = rdot(x, acc);
  }
  stm<N, R>(a.dst, comp, c.s, a.g.S, acc);
  return part;
}

}  // namespace susy
