// Forces, momentum and link updates, and action densities.
//
//   fermion force of one pole     assemble_fermion_force  update_h.c:666-916
//     S/L terms                                            update_h.c:705-746
//     V/P terms                                            update_h.c:753-894
//     determinant terms  detF                              update_h.c:469-651
//     Q-closed terms     F1Q, F2Q                          update_h.c:266-462
//   pole sum and momentum update  fermion_force            update_h.c:928-978
//   gauge force                   gauge_force              update_h.c:15-261
//   determinant force             det_force                det_force.c:6-78
//   link update                   update_u                 update_o.c:20-35
//   action densities              action.c:106-286
// One thread computes the force on one link (site x, direction M): every
// neighbour product the reference builds by gathers is formed in registers
// from the SoA fields, with compile-time offsets.
#include "common.cuh"
#include "kernels.h"

namespace susy {

constexpr int FT = 128;

struct FfArgs {
  Geo g;
  const double2 *U, *Uinv, *pd;
  const double2 *sol, *psol;  // psol = D sol (not yet scaled by amp)
  double2* force;             // accumulates amp * f_U^dag
  double amp, G;
  int doG;
};

// T_b(y) = Tr[U_b(y)^{-1} psi_b(y)], psi read from fld component 1+b
template <int N, bool ADJ>
SUSY_D Cx<double> Ttr(const FfArgs& a, const double2* fld, int b, int y) {
  Mat<N, double> ui = ldm<N, double>(a.Uinv, b, y, a.g.S);
  Mat<N, double> ps = ldm<N, double, ADJ>(fld, 1 + b, y, a.g.S);
  return trace_nn(ui, ps);
}

// detF(eta, psi, sign) contribution to f_U[M] (update_h.c:477-651);
// ADJ_ETA/ADJ_PSI select whether eta / psi are read adjointed from psol.
template <int N, int M, bool ETA_PSOL>
SUSY_D void detF_term(Mat<N, double>& f, const FfArgs& a, const Site& c) {
  const Geo& g = a.g;
  const int S = g.S, s = c.s;
  // sign +1: eta = psol site (adjointed), psi = sol links, localG = -G/2
  // sign -1: eta = sol site, psi = psol links (adjointed), localG = +G/2
  const double2* etaf = ETA_PSOL ? a.psol : a.sol;
  const double2* psif = ETA_PSOL ? a.sol : a.psol;
  constexpr bool AE = ETA_PSOL, AP = !ETA_PSOL;
  const double localG = (ETA_PSOL ? -0.5 : 0.5) * a.G;
  const Cx<double> te0 = ldtr<N, double, AE>(etaf, 0, s, S);
  const Cx<double> TM0 = Ttr<N, AP>(a, psif, M, s);
  const int pM = nbr(g, c, ex(M), ey(M), ez(M), et(M));
  Cx<double> plaq(0, 0), adjt(0, 0), inv(0, 0);
#pragma unroll
  for (int b = 0; b < NUMLINK; b++) {
    if (b == M) continue;
    const int mb = nbr(g, c, -ex(b), -ey(b), -ez(b), -et(b));
    const int pb = nbr(g, c, ex(b), ey(b), ez(b), et(b));
    const int mbpM = nbr(g, c, ex(M) - ex(b), ey(M) - ey(b), ez(M) - ez(b), et(M) - et(b));
    const double bcM = bcf<double>(g, c, et(M));
    const double bcb = bcf<double>(g, c, et(b));
    const double bcmb = bcf<double>(g, c, -et(b));
    // bc[M] evaluated at site x - b
    Site cm = c;
    cm.t = wrap(c.t - et(b), g.nt);
    const double bcM_mb = bcf<double>(g, cm, et(M));
    const Cx<double> te_mb = ldtr<N, double, AE>(etaf, 0, mb, S);
    const Cx<double> DbM = te0 * ldc<double>(a.pd + (size_t)(b * 5 + M) * S + s);
    const Cx<double> DMb = te0 * ldc<double>(a.pd + (size_t)(M * 5 + b) * S + s);
    const Cx<double> DMb_mb = te_mb * ldc<double>(a.pd + (size_t)(M * 5 + b) * S + mb);
    const Cx<double> DbM_mb = te_mb * ldc<double>(a.pd + (size_t)(b * 5 + M) * S + mb);
    const Cx<double> Tb0 = Ttr<N, AP>(a, psif, b, s);
    const Cx<double> Tb_pM = Ttr<N, AP>(a, psif, b, pM);
    const Cx<double> Tb_mb = Ttr<N, AP>(a, psif, b, mb);
    const Cx<double> TM_pb = Ttr<N, AP>(a, psif, M, pb);
    const Cx<double> TM_mb = Ttr<N, AP>(a, psif, M, mb);
    const Cx<double> Tb_mbpM = Ttr<N, AP>(a, psif, b, mbpM);
    plaq = plaq + DbM * (TM0 + bcM * Tb_pM);
    plaq = plaq + DMb_mb * (Tb_mb + bcmb * TM0);
    adjt = adjt + DMb * (Tb0 + bcb * TM_pb);
    adjt = adjt + DbM_mb * (TM_mb + bcM_mb * Tb_mbpM);
    inv = inv + DbM + bcmb * DMb_mb;
  }
  Mat<N, double> ui = ldm<N, double>(a.Uinv, M, s, S);
  Mat<N, double> ps = ldm<N, double, AP>(psif, 1 + M, s, S);
  Mat<N, double> upu = mul(mul(ui, ps), ui);
  axpy(f, localG * plaq, ui);
  axpy(f, conj(localG * adjt), ui);
  axpy(f, Cx<double>(-localG * inv.re, -localG * inv.im), upu);
}

// Q-closed pieces with c = M for one split of the complement into (A,B), (D,E)
template <int N, int M, int A, int B, int D, int E>
SUSY_D void fq_terms(Mat<N, double>& f, const FfArgs& a, const Site& c) {
  const Geo& g = a.g;
  const int S = g.S;
  constexpr int abx = ex(A) + ex(B), aby = ey(A) + ey(B), abz = ez(A) + ez(B), abt = et(A) + et(B);
  const int pM = nbr(g, c, ex(M), ey(M), ez(M), et(M));
  const int pabM = nbr(g, c, abx + ex(M), aby + ey(M), abz + ez(M), abt + et(M));
  const int mab = nbr(g, c, -abx, -aby, -abz, -abt);
  const double bcM = bcf<double>(g, c, et(M));
  const double bc3 = bcf<double>(g, c, abt + et(M));
  const double bc2m = bcf<double>(g, c, -abt);
  Mat<N, double> tm;
  tm.zero();
  // F1Q: chi'_DE(x+A+B+M) (p bc3 bc[M] chi_AB(x+M)) + (-p bc2 bc[M] chi_AB(x-A-B)) chi'_DE(x+M)
  {
    const double p = (double)eps5(D, E, M, A, B);
    Mat<N, double> l0 = ldm<N, double, true>(a.psol, 6 + pidx(D, E), pabM, S);
    Mat<N, double> l1 = ldm<N, double>(a.sol, 6 + pidx(A, B), pM, S);
    mac<0>(tm, p * bc3 * bcM, l0, l1);
    Mat<N, double> l3 = ldm<N, double>(a.sol, 6 + pidx(A, B), mab, S);
    Mat<N, double> l2 = ldm<N, double, true>(a.psol, 6 + pidx(D, E), pM, S);
    mac<0>(tm, -p * bc2m * bcM, l3, l2);
  }
  // F2Q: chi'_AB(x-A-B) (p bc2 bc[M] chi_DE(x+M)) + (-p bc3 bc[M] chi_DE(x+A+B+M)) chi'_AB(x+M)
  {
    const double p = (double)eps5(A, B, M, D, E);
    Mat<N, double> l0 = ldm<N, double, true>(a.psol, 6 + pidx(A, B), mab, S);
    Mat<N, double> l1 = ldm<N, double>(a.sol, 6 + pidx(D, E), pM, S);
    mac<0>(tm, p * bc2m * bcM, l0, l1);
    Mat<N, double> l3 = ldm<N, double>(a.sol, 6 + pidx(D, E), pabM, S);
    Mat<N, double> l2 = ldm<N, double, true>(a.psol, 6 + pidx(A, B), pM, S);
    mac<0>(tm, -p * bc3 * bcM, l3, l2);
  }
  // f_U[M] += -1/2 tm^dag
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) {
      f.e[i][j].re -= 0.5 * tm.e[j][i].re;
      f.e[i][j].im += 0.5 * tm.e[j][i].im;
    }
}

template <int M>
struct Compl4 {
  static constexpr int k(int n) {
    int c = 0;
    for (int v = 0; v < 5; v++) {
      if (v == M) continue;
      if (c == n) return v;
      c++;
    }
    return -1;
  }
  static constexpr int K0 = k(0), K1 = k(1), K2 = k(2), K3 = k(3);
};

template <int N, int M>
SUSY_D Mat<N, double> fforce_out(const FfArgs& a, const Site& c) {
  const Geo& g = a.g;
  const int S = g.S, s = c.s;
  const int pM = nbr(g, c, ex(M), ey(M), ez(M), et(M));
  const double bcM = bcf<double>(g, c, et(M));
  Mat<N, double> f;
  // S/L terms: up = psi_M bc eta'(x+M) - eta' psi_M - psi'_M bc eta(x+M) + eta psi'_M
  {
    Mat<N, double> up;
    up.zero();
    Mat<N, double> psM = ldm<N, double>(a.sol, 1 + M, s, S);
    Mat<N, double> etp = ldm<N, double, true>(a.psol, 0, pM, S);
    mac<0>(up, bcM, psM, etp);
    etp = ldm<N, double, true>(a.psol, 0, s, S);
    mac<0>(up, -1.0, etp, psM);
    Mat<N, double> ppM = ldm<N, double, true>(a.psol, 1 + M, s, S);
    Mat<N, double> et_ = ldm<N, double>(a.sol, 0, pM, S);
    mac<0>(up, -bcM, ppM, et_);
    et_ = ldm<N, double>(a.sol, 0, s, S);
    mac<0>(up, 1.0, et_, ppM);
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
      for (int j = 0; j < N; j++) f.e[i][j] = Cx<double>(0.5 * up.e[j][i].re, -0.5 * up.e[j][i].im);
  }
  // V/P terms
#pragma unroll
  for (int nu = 0; nu < NUMLINK; nu++) {
    if (nu == M) continue;
    const double sg = M < nu ? 1.0 : -1.0;
    const int q = 6 + pidx(M, nu);
    const int mn = nbr(g, c, -ex(nu), -ey(nu), -ez(nu), -et(nu));
    // -bc[M] psi_nu(x+M) chi'_{M nu}(x) + chi'_{M nu}(x-nu) psi_nu(x-nu)
    Mat<N, double> P = ldm<N, double, true>(a.psol, q, s, S);
    Mat<N, double> ps = ldm<N, double>(a.sol, 1 + nu, pM, S);
    mac<0>(f, -bcM * sg, ps, P);
    P = ldm<N, double, true>(a.psol, q, mn, S);
    ps = ldm<N, double>(a.sol, 1 + nu, mn, S);
    mac<0>(f, sg, P, ps);
    // psi'_nu(x+M) bc[M] chi_{M nu}(x) - chi_{M nu}(x-nu) psi'_nu(x-nu)
    Mat<N, double> C = ldm<N, double>(a.sol, q, s, S);
    Mat<N, double> pp = ldm<N, double, true>(a.psol, 1 + nu, pM, S);
    mac<0>(f, bcM * sg, pp, C);
    C = ldm<N, double>(a.sol, q, mn, S);
    pp = ldm<N, double, true>(a.psol, 1 + nu, mn, S);
    mac<0>(f, -sg, C, pp);
  }
  if (a.doG) {
    detF_term<N, M, true>(f, a, c);
    detF_term<N, M, false>(f, a, c);
  }
  typedef Compl4<M> K;
  fq_terms<N, M, K::K0, K::K1, K::K2, K::K3>(f, a, c);
  fq_terms<N, M, K::K2, K::K3, K::K0, K::K1>(f, a, c);
  fq_terms<N, M, K::K0, K::K2, K::K1, K::K3>(f, a, c);
  fq_terms<N, M, K::K1, K::K3, K::K0, K::K2>(f, a, c);
  fq_terms<N, M, K::K0, K::K3, K::K1, K::K2>(f, a, c);
  fq_terms<N, M, K::K1, K::K2, K::K0, K::K3>(f, a, c);
  return f;
}

template <int N>
__global__ void __launch_bounds__(FT) k_fermion_force(FfArgs a) {
  const int M = blockIdx.x % NUMLINK;
  const int s = (blockIdx.x / NUMLINK) * FT + threadIdx.x;
  if (s >= a.g.V) return;
  const Site c = site_of(a.g, s);
  Mat<N, double> f;
  switch (M) {
    case 0: f = fforce_out<N, 0>(a, c); break;
    case 1: f = fforce_out<N, 1>(a, c); break;
    case 2: f = fforce_out<N, 2>(a, c); break;
    case 3: f = fforce_out<N, 3>(a, c); break;
    default: f = fforce_out<N, 4>(a, c); break;
  }
  // fullforce[M] += amp f_U^dag  (update_h.c:943-958)
  Mat<N, double> acc = ldm<N, double>(a.force, M, s, a.g.S);
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) {
      acc.e[i][j].re += a.amp * f.e[j][i].re;
      acc.e[i][j].im -= a.amp * f.e[j][i].im;
    }
  stm<N, double>(a.force, M, s, a.g.S, acc);
}

// mom -= eps force; partials of |force|^2   (update_h.c:965-971)
__global__ void __launch_bounds__(256) k_mom_sub(long n, const double2* force, double2* mom,
                                                 double eps, double* part) {
  const long i = (long)blockIdx.x * 256 + threadIdx.x;
  double acc = 0.0;
  if (i < n) {
    const double2 f = force[i];
    double2 m = mom[i];
    m.x -= eps * f.x;
    m.y -= eps * f.y;
    mom[i] = m;
    acc = f.x * f.x + f.y * f.y;
  }
  acc = block_sum<256>(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

// y += s x over n complex
__global__ void k_axpy(long n, double s, const double2* x, double2* y) {
  const long i = (long)blockIdx.x * 256 + threadIdx.x;
  if (i >= n) return;
  double2 v = y[i];
  const double2 u = x[i];
  v.x += s * u.x;
  v.y += s * u.y;
  y[i] = v;
}

// ---------------------------------------------------------------------------
struct GfArgs {
  Geo g;
  const double2 *U, *Uinv, *pd, *zw, *D, *F;
  double2* mom;
  double G, bmass, kappa, kappa_u1, eps;
  int doG, N, det_only;
  double* part;  // [2][nblocks]: |f_U|^2 and |f_det|^2 partials
  int nblk;
};

template <int N, int M>
SUSY_D void gforce_site(const GfArgs& a, const Site& c, double& n1, double& n2) {
  const Geo& g = a.g;
  const int S = g.S, s = c.s;
  const int pM = nbr(g, c, ex(M), ey(M), ez(M), et(M));
  Mat<N, double> u = ldm<N, double>(a.U, M, s, S);
  Mat<N, double> ui = ldm<N, double>(a.Uinv, M, s, S);
  Mat<N, double> m = ldm<N, double>(a.mom, M, s, S);
  if (!a.det_only) {
  Mat<N, double> f;
  f.zero();
  // Ubar_M DmuUmu - DmuUmu(x+M) Ubar_M
  mac<2>(f, 1.0, u, ldm<N, double>(a.D, 0, s, S));
  mac<1>(f, -1.0, ldm<N, double>(a.D, 0, pM, S), u);
  if (a.doG) {
    // G U_M^{-1} sum_nu [Tr D(x) pd[nu][M](x) + Tr D(x-nu) pd[M][nu](x-nu)]
    const Cx<double> t0 = ldtr<N, double>(a.D, 0, s, S);
    Cx<double> sum(0, 0);
#pragma unroll
    for (int nu = 0; nu < NUMLINK; nu++) {
      if (nu == M) continue;
      const int mn = nbr(g, c, -ex(nu), -ey(nu), -ez(nu), -et(nu));
      sum = sum + t0 * ldc<double>(a.pd + (size_t)(nu * 5 + M) * S + s);
      sum = sum + ldtr<N, double>(a.D, 0, mn, S) * ldc<double>(a.pd + (size_t)(M * 5 + nu) * S + mn);
    }
    axpy(f, a.G * sum, ui);
  }
  // 2 sum_nu [U_nu(x+M) F_{M nu}^dag - (F_{M nu}^dag U_nu)(x - nu)]
#pragma unroll
  for (int nu = 0; nu < NUMLINK; nu++) {
    if (nu == M) continue;
    const double sg = M < nu ? 2.0 : -2.0;
    const int mn = nbr(g, c, -ex(nu), -ey(nu), -ez(nu), -et(nu));
    const int q = pidx(M, nu);
    mac<1>(f, sg, ldm<N, double>(a.U, nu, pM, S), ldm<N, double>(a.F, q, s, S));
    mac<2>(f, -sg, ldm<N, double>(a.F, q, mn, S), ldm<N, double>(a.U, nu, mn, S));
  }
  if (a.bmass > 1e-8) {
    const double dmu = 2.0 * a.bmass * a.bmass / N;
    double tr = 0.0;
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
      for (int j = 0; j < N; j++) tr += u.e[i][j].re * u.e[i][j].re + u.e[i][j].im * u.e[i][j].im;
    tr = dmu * (tr / N - 1.0);
    Mat<N, double> ud = adjm(u);
    axpy(f, Cx<double>(tr, 0.0), ud);
  }
  // mom -= kappa eps f^dag
  const double ke = a.kappa * a.eps;
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) {
      m.e[i][j].re -= ke * f.e[j][i].re;
      m.e[i][j].im += ke * f.e[j][i].im;
      n1 += f.e[i][j].re * f.e[i][j].re + f.e[i][j].im * f.e[i][j].im;
    }
  }
  if (a.kappa_u1 > 1e-8) {
    // det_force: kappa_u1 sum_b [ZW[b][M](x) + ZW[M][b](x-b)] U_M^{-1}
    Cx<double> t(0, 0);
#pragma unroll
    for (int b = 0; b < NUMLINK; b++) {
      if (b == M) continue;
      const int mb = nbr(g, c, -ex(b), -ey(b), -ez(b), -et(b));
      t = t + ldc<double>(a.zw + (size_t)(b * 5 + M) * S + s);
      t = t + ldc<double>(a.zw + (size_t)(M * 5 + b) * S + mb);
    }
    t = a.kappa_u1 * t;
    Mat<N, double> f2;
    f2.zero();
    axpy(f2, t, ui);
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
      for (int j = 0; j < N; j++) {
        m.e[i][j].re -= a.eps * f2.e[j][i].re;
        m.e[i][j].im += a.eps * f2.e[j][i].im;
        n2 += f2.e[i][j].re * f2.e[i][j].re + f2.e[i][j].im * f2.e[i][j].im;
      }
  }
  stm<N, double>(a.mom, M, s, S, m);
}

template <int N>
__global__ void __launch_bounds__(FT) k_gauge_force(GfArgs a) {
  const int M = blockIdx.x % NUMLINK;
  const int s = (blockIdx.x / NUMLINK) * FT + threadIdx.x;
  double n1 = 0.0, n2 = 0.0;
  if (s < a.g.V) {
    const Site c = site_of(a.g, s);
    switch (M) {
      case 0: gforce_site<N, 0>(a, c, n1, n2); break;
      case 1: gforce_site<N, 1>(a, c, n1, n2); break;
      case 2: gforce_site<N, 2>(a, c, n1, n2); break;
      case 3: gforce_site<N, 3>(a, c, n1, n2); break;
      default: gforce_site<N, 4>(a, c, n1, n2); break;
    }
  }
  n1 = block_sum<FT>(n1);
  __syncthreads();
  n2 = block_sum<FT>(n2);
  if (threadIdx.x == 0) {
    a.part[blockIdx.x] = n1;
    a.part[a.nblk + blockIdx.x] = n2;
  }
}

// ---------------------------------------------------------------------------
// Action densities per site: gauge, bmass, det, mom partials (action.c:106-286)
template <int N>
__global__ void __launch_bounds__(FT) k_action(Geo g, const double2* U, const double2* D,
                                              const double2* F, const double2* pd,
                                              const double2* mom, double* part, int nblk) {
  const int s = blockIdx.x * FT + threadIdx.x;
  double ga = 0.0, ba = 0.0, da = 0.0, ma = 0.0;
  if (s < g.V) {
    Mat<N, double> d = ldm<N, double>(D, 0, s, g.S);
    Mat<N, double> t;
    t.zero();
    mac<0>(t, 0.5, d, d);
#pragma unroll 1
    for (int p = 0; p < NPLAQ; p++) {
      Mat<N, double> f = ldm<N, double>(F, p, s, g.S);
      mac<2>(t, 2.0, f, f);
    }
    ga = trace(t).re;
#pragma unroll
    for (int a = 0; a < NUMLINK; a++) {
      Mat<N, double> u = ldm<N, double>(U, a, s, g.S);
      double tr = rdot(u, u) / N - 1.0;
      ba += tr * tr;
      Mat<N, double> m = ldm<N, double>(mom, a, s, g.S);
      ma += rdot(m, m);
#pragma unroll
      for (int b = a + 1; b < NUMLINK; b++) {
        Cx<double> p = ldc<double>(pd + (size_t)(a * 5 + b) * g.S + s);
        da += (p.re - 1.0) * (p.re - 1.0) + p.im * p.im;
      }
    }
  }
  double v[4] = {ga, ba, da, ma};
#pragma unroll
  for (int k = 0; k < 4; k++) {
    double r = block_sum<FT>(v[k]);
    __syncthreads();
    if (threadIdx.x == 0) part[k * nblk + blockIdx.x] = r;
  }
}

// Fermion action partials: ampdeg |src|^2 + sum_j amp_j Re<src, sol_j>
__global__ void __launch_bounds__(256) k_fermion_action(long n, const double2* src, int nsol,
                                                        const double2* const* sol,
                                                        const double* amp, double ampdeg,
                                                        double* part) {
  const long i = (long)blockIdx.x * 256 + threadIdx.x;
  double acc = 0.0;
  if (i < n) {
    const double2 x = src[i];
    acc = ampdeg * (x.x * x.x + x.y * x.y);
    for (int j = 0; j < nsol; j++) {
      const double2 y = sol[j][i];
      acc += amp[j] * (x.x * y.x + x.y * y.y);
    }
  }
  acc = block_sum<256>(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

// ---------------------------------------------------------------------------
static inline int nbk(long n, int t) { return (int)((n + t - 1) / t); }

int force_blocks(const Geo& g) { return nbk(g.V, FT) * NUMLINK; }
int site_blocks(const Geo& g) { return nbk(g.V, FT); }

void fermion_force_pole(const Geo& g, int N, const void* U, const void* Uinv, const void* pd,
                        const void* sol, const void* psol, void* force, double amp, double G,
                        cudaStream_t st) {
  FfArgs a;
  a.g = g;
  a.U = (const double2*)U;
  a.Uinv = (const double2*)Uinv;
  a.pd = (const double2*)pd;
  a.sol = (const double2*)sol;
  a.psol = (const double2*)psol;
  a.force = (double2*)force;
  a.amp = amp;
  a.G = G;
  a.doG = G > 1e-8;
  const int nb = force_blocks(g);
  switch (N) {
    case 2: count_launch(), k_fermion_force<2><<<nb, FT, 0, st>>>(a); break;
    case 3: count_launch(), k_fermion_force<3><<<nb, FT, 0, st>>>(a); break;
    case 4: count_launch(), k_fermion_force<4><<<nb, FT, 0, st>>>(a); break;
  }
}

int mom_sub(long n, const void* force, void* mom, double eps, double* part, cudaStream_t st) {
  const int nb = nbk(n, 256);
  count_launch(), k_mom_sub<<<nb, 256, 0, st>>>(n, (const double2*)force, (double2*)mom, eps, part);
  return nb;
}

void axpy_field(long n, double s, const void* x, void* y, cudaStream_t st) {
  count_launch(), k_axpy<<<nbk(n, 256), 256, 0, st>>>(n, s, (const double2*)x, (double2*)y);
}

int gauge_force(const Geo& g, int N, const void* U, const void* Uinv, const void* pd,
                const void* zw, const void* D, const void* F, void* mom, double G, double bmass,
                double kappa, double kappa_u1, double eps, int det_only, double* part,
                cudaStream_t st) {
  GfArgs a;
  a.g = g;
  a.U = (const double2*)U;
  a.Uinv = (const double2*)Uinv;
  a.pd = (const double2*)pd;
  a.zw = (const double2*)zw;
  a.D = (const double2*)D;
  a.F = (const double2*)F;
  a.mom = (double2*)mom;
  a.G = G;
  a.bmass = bmass;
  a.kappa = kappa;
  a.kappa_u1 = kappa_u1;
  a.eps = eps;
  a.doG = G > 1e-8;
  a.N = N;
  a.det_only = det_only;
  a.part = part;
  a.nblk = force_blocks(g);
  switch (N) {
    case 2: count_launch(), k_gauge_force<2><<<a.nblk, FT, 0, st>>>(a); break;
    case 3: count_launch(), k_gauge_force<3><<<a.nblk, FT, 0, st>>>(a); break;
    case 4: count_launch(), k_gauge_force<4><<<a.nblk, FT, 0, st>>>(a); break;
  }
  return a.nblk;
}

int action_partials(const Geo& g, int N, const void* U, const void* D, const void* F,
                    const void* pd, const void* mom, double* part, cudaStream_t st) {
  const int nb = site_blocks(g);
  switch (N) {
    case 2: count_launch(), k_action<2><<<nb, FT, 0, st>>>(g, (const double2*)U, (const double2*)D, (const double2*)F, (const double2*)pd, (const double2*)mom, part, nb); break;
    case 3: count_launch(), k_action<3><<<nb, FT, 0, st>>>(g, (const double2*)U, (const double2*)D, (const double2*)F, (const double2*)pd, (const double2*)mom, part, nb); break;
    case 4: count_launch(), k_action<4><<<nb, FT, 0, st>>>(g, (const double2*)U, (const double2*)D, (const double2*)F, (const double2*)pd, (const double2*)mom, part, nb); break;
  }
  return nb;
}

int fermion_action_partials(long n, const void* src, int nsol, const void* const* sol_dev_array,
                            const double* amp_dev, double ampdeg, double* part, cudaStream_t st) {
  const int nb = nbk(n, 256);
  count_launch(), k_fermion_action<<<nb, 256, 0, st>>>(n, (const double2*)src, nsol,
                                        (const double2* const*)sol_dev_array, amp_dev, ampdeg,
                                        part);
  return nb;
}

}  // namespace susy
