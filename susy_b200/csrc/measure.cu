// Per-trajectory measurements of the reference's control.c:85-138 on the
// device fields of a lattice handle (susy_b200_measure, susy_b200_plaquette):
//   FLINK, FLINK_DET         link_trace       link_trace.c:9-56
//   GMES, LINES, LINES_POLAR ploop            ploop.c:8-126
//   GMES (ss, st plaquette)  plaquette        plaq.c:7-53
//   BACTION                  gauge_action     action.c:106-142 (NODET)
//   DET                      measure_det      determinant.c:92-120
//   WIDTHS                   widths           widths.c:8-71
//   UUBAR_EIG, POLAR_EIG     scalar_eig       scalar_eig.c:15-115
// One site kernel accumulates every per-site sum (block partials, summed on
// the host in FP64 in a fixed order) and the per-block extremes of the
// scalar eigenvalues; one line kernel per direction multiplies the links
// along each line through the lattice (thread per line start).  The
// reference's zheev calls become the Jacobi eigen-solver of linalg.cuh:
// POLAR_EIG is the spectrum of log P, P = sqrt(U Ubar), i.e. half the
// logarithm of the spectrum of U Ubar, so one eigen-solve per link serves
// both scalar_eig calls.
#include <cmath>
#include <vector>
#include "lattice.h"
#include "linalg.cuh"

namespace susy {

constexpr int MT = 128;
// per-site sums: 0-4 linktr[dir], 5-9 link_det[dir], 10 linktr^2, 11 det^2,
// 12 ss, 13 st, 14 plaq, 15 plaq^2, 16 det re, 17 det re^2, 18 det im,
// 19 det im^2, 20-21 sum plaqdet, 22-23 sum of squared parts, 24 |pd-1|^2,
// 25 gauge action density, then uubar ave/sq and polar ave/sq [NCOL] each
constexpr int MS_BASE = 26;
constexpr int ms_count(int N) { return MS_BASE + 4 * N; }

template <int N>
__global__ void __launch_bounds__(MT) k_meas_site(Geo g, const double2* U, const double2* pd,
                                                  const double2* D, const double2* F,
                                                  double* sums, double* ext, int nblk) {
  const int s = blockIdx.x * MT + threadIdx.x;
  const bool live = s < g.V;
  double v[ms_count(N)];
#pragma unroll
  for (int k = 0; k < ms_count(N); k++) v[k] = 0.0;
  double emin[2 * N], emax[2 * N];
#pragma unroll
  for (int k = 0; k < 2 * N; k++) {
    emin[k] = 1e300;
    emax[k] = -1e300;
  }
  if (live) {
    const Site c = site_of(g, s);
#pragma unroll 1
    for (int a = 0; a < NUMLINK; a++) {
      const Mat<N, double> u = ldm<N, double>(U, a, s, g.S);
      Mat<N, double> m;
      m.zero();
      mac<1>(m, 1.0, u, u);                                   // U Ubar
      const double tr = trace(m).re;
      double w[N];
      herm_eig<N>(m, w, nullptr);
      Mat<N, double> t = m, ti;
#pragma unroll
      for (int i = 0; i < N; i++) t.e[i][i].re -= tr / N;
      Cx<double> dt;
      det_inv<N>(t, dt, ti);
#pragma unroll
      for (int k = 0; k < NUMLINK; k++)
        if (k == a) {
          v[k] += tr / N;
          v[5 + k] += dt.re;
        }
      v[10] += tr * tr / (N * N);
      v[11] += dt.re * dt.re;
#pragma unroll
      for (int j = 0; j < N; j++) {
        const double eu = w[j] - tr / N, ep = 0.5 * log(w[j]);
        v[MS_BASE + j] += eu;
        v[MS_BASE + N + j] += eu * eu;
        v[MS_BASE + 2 * N + j] += ep;
        v[MS_BASE + 3 * N + j] += ep * ep;
        emin[j] = fmin(emin[j], eu);
        emax[j] = fmax(emax[j], eu);
        emin[N + j] = fmin(emin[N + j], ep);
        emax[N + j] = fmax(emax[N + j], ep);
      }
    }
    // plaquettes and widths
#pragma unroll 1
    for (int a = 0; a < NUMLINK; a++) {
#pragma unroll 1
      for (int b = 0; b < NUMLINK; b++) {
        if (a == b) continue;
        const int xa = nbr(g, c, ex(a), ey(a), ez(a), et(a));
        const int xb = nbr(g, c, ex(b), ey(b), ez(b), et(b));
        const Mat<N, double> ua = ldm<N, double>(U, a, s, g.S);
        const Mat<N, double> ub = ldm<N, double>(U, b, s, g.S);
        const Mat<N, double> ubxa = ldm<N, double>(U, b, xa, g.S);
        const Mat<N, double> uaxb = ldm<N, double>(U, a, xb, g.S);
        const Mat<N, double> w1 = mul(ua, ubxa);             // U_a(x) U_b(x+a)
        if (b < a) {
          // plaq.c: Re Tr[U_a(x+b)^dag U_b(x)^dag U_a(x) U_b(x+a)]
          Mat<N, double> t;
          t.zero();
          mac<2>(t, 1.0, ub, w1);
          const double p = rdot(uaxb, t);
          if (a == 3 || b == 3)
            v[13] += p;
          else
            v[12] += p;
          // measure_det over the same pairs
          const Cx<double> q = ldc<double>(pd + (size_t)(a * 5 + b) * g.S + s);
          v[20] += q.re;
          v[21] += q.im;
          v[22] += q.re * q.re;
          v[23] += q.im * q.im;
          v[24] += (q.re - 1.0) * (q.re - 1.0) + q.im * q.im;
        } else {
          // widths.c: P_ab = U_b(x) U_a(x+b) [U_a(x) U_b(x+a)]^dag, a < b
          Mat<N, double> t, P;
          t.zero();
          mac<1>(t, 1.0, uaxb, w1);
          P = mul(ub, t);
          const double pr = trace(P).re;
          Mat<N, double> pi;
          Cx<double> dp;
          det_inv<N>(P, dp, pi);
          v[14] += pr;
          v[15] += pr * pr;
          v[16] += dp.re;
          v[17] += dp.re * dp.re;
          v[18] += dp.im;
          v[19] += dp.im * dp.im;
        }
      }
    }
    // gauge action density: Re Tr[D^2 / 2 + 2 sum F^dag F]
    {
      const Mat<N, double> d = ldm<N, double>(D, 0, s, g.S);
      Mat<N, double> t;
      t.zero();
      mac<0>(t, 0.5, d, d);
#pragma unroll 1
      for (int p = 0; p < NPLAQ; p++) {
        const Mat<N, double> f = ldm<N, double>(F, p, s, g.S);
        mac<2>(t, 2.0, f, f);
      }
      v[25] += trace(t).re;
    }
  }
#pragma unroll 1
  for (int k = 0; k < ms_count(N); k++) {
    const double r = block_sum<MT>(v[k]);
    __syncthreads();
    if (threadIdx.x == 0) sums[(size_t)k * nblk + blockIdx.x] = r;
  }
  __shared__ double red[MT];
#pragma unroll 1
  for (int k = 0; k < 2 * N; k++) {
    for (int side = 0; side < 2; side++) {
      red[threadIdx.x] = side == 0 ? emin[k] : -emax[k];
      __syncthreads();
      for (int o = MT / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] = fmin(red[threadIdx.x], red[threadIdx.x + o]);
        __syncthreads();
      }
      if (threadIdx.x == 0) ext[(size_t)(2 * k + side) * nblk + blockIdx.x] = red[0];
      __syncthreads();
    }
  }
}

// Unitary part of the polar decomposition U = P u (unit.c:52-98):
// u = V diag(w^-1/2) V^dag U with U Ubar = V diag(w) V^dag
template <int N>
SUSY_D Mat<N, double> polar_u(const Mat<N, double>& u) {
  Mat<N, double> m, V;
  m.zero();
  mac<1>(m, 1.0, u, u);
  double w[N];
  herm_eig<N>(m, w, &V);
  Mat<N, double> vs = V;
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) {
      const double f = 1.0 / sqrt(w[j]);
      vs.e[i][j] = Cx<double>(vs.e[i][j].re * f, vs.e[i][j].im * f);
    }
  Mat<N, double> pinv;
  pinv.zero();
  mac<1>(pinv, 1.0, vs, V);       // V diag(w^-1/2) V^dag
  return mul(pinv, u);
}

// Line products along direction d from every site with coordinate 0 along
// it (t for the fifth link): partial sums of Re, Im and |Tr|
template <int N>
__global__ void __launch_bounds__(MT) k_ploop(Geo g, const double2* U, int d, int project,
                                              double* part, int nblk) {
  const int axis = d < 4 ? d : 3;
  const int len = axis == 0 ? g.nx : axis == 1 ? g.ny : axis == 2 ? g.nz : g.nt;
  const int nstart = g.V / len;
  const int i = blockIdx.x * MT + threadIdx.x;
  double re = 0.0, im = 0.0, md = 0.0;
  if (i < nstart) {
    // the i-th site (lexicographic) of the hyperplane with coordinate 0
    int x, y, z, t;
    int r = i;
    if (axis == 0) { x = 0; y = r % g.ny; r /= g.ny; z = r % g.nz; t = r / g.nz; }
    else if (axis == 1) { x = r % g.nx; r /= g.nx; y = 0; z = r % g.nz; t = r / g.nz; }
    else if (axis == 2) { x = r % g.nx; r /= g.nx; y = r % g.ny; z = 0; t = r / g.ny; }
    else { x = r % g.nx; r /= g.nx; y = r % g.ny; z = r / g.ny; t = 0; }
    Site c;
    c.x = x; c.y = y; c.z = z; c.t = t;
    c.s = x + g.nx * (y + g.ny * (z + g.nz * t));
    Mat<N, double> prod = ldm<N, double>(U, d, c.s, g.S);
    if (project) prod = polar_u<N>(prod);
#pragma unroll 1
    for (int k = 1; k < len; k++) {
      const int ns = nbr(g, c, ex(d), ey(d), ez(d), et(d));
      c = site_of(g, ns);
      Mat<N, double> l = ldm<N, double>(U, d, ns, g.S);
      if (project) l = polar_u<N>(l);
      prod = mul(prod, l);
    }
    const Cx<double> tr = trace(prod);
    re = tr.re;
    im = tr.im;
    md = sqrt(tr.re * tr.re + tr.im * tr.im);
  }
  const double v[3] = {re, im, md};
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const double r = block_sum<MT>(v[k]);
    __syncthreads();
    if (threadIdx.x == 0) part[(size_t)k * nblk + blockIdx.x] = r;
  }
}

template <int N>
static void launch_site(susy_b200_lattice* h, double* sums, double* ext, int nb) {
  count_launch(), k_meas_site<N><<<nb, MT, 0, h->stream>>>(
      h->g, (const double2*)h->U, (const double2*)h->pd, (const double2*)h->D,
      (const double2*)h->F, sums, ext, nb);
}

template <int N>
static void launch_ploop(susy_b200_lattice* h, int d, int project, double* part, int nb) {
  count_launch(), k_ploop<N><<<nb, MT, 0, h->stream>>>(h->g, (const double2*)h->U, d, project,
                                                        part, nb);
}

static double* meas_buffer(susy_b200_lattice* h, size_t n) {
  if (h->meas_n < n) {
    if (h->meas) cudaFree(h->meas);
    h->meas = (double*)dalloc(h, n * sizeof(double));
    h->meas_n = h->meas ? n : 0;
  }
  return h->meas;
}

static double sum_range(const std::vector<double>& v, size_t off, int n) {
  double s = 0.0;
  for (int i = 0; i < n; i++) s += v[off + i];
  return s;
}

int measure(susy_b200_lattice* h, susy_b200_meas* m) {
  const int N = h->N;
  const Geo& g = h->g;
  const int nb = (g.V + MT - 1) / MT;
  const int K = ms_count(N);
  // site partials, extremes, then 11 line kernels (3 partials each)
  const size_t n_site = (size_t)K * nb, n_ext = (size_t)4 * N * nb;
  const size_t n_line = (size_t)3 * nb;
  double* buf = meas_buffer(h, n_site + n_ext + 11 * n_line);
  if (!buf) return set_err(h, SUSY_B200_ENOMEM);
  double* sums = buf;
  double* ext = buf + n_site;
  double* lines = ext + n_ext;
  switch (N) {
    case 2: launch_site<2>(h, sums, ext, nb); break;
    case 3: launch_site<3>(h, sums, ext, nb); break;
    default: launch_site<4>(h, sums, ext, nb); break;
  }
  // line kernels: (dir, NODET) for dir 0..4, then (dir, YESDET)
  for (int q = 0; q < 10; q++) {
    const int d = q % 5, pr = q / 5;
    switch (N) {
      case 2: launch_ploop<2>(h, d, pr, lines + q * n_line, nb); break;
      case 3: launch_ploop<3>(h, d, pr, lines + q * n_line, nb); break;
      default: launch_ploop<4>(h, d, pr, lines + q * n_line, nb); break;
    }
  }
  std::vector<double> hv(n_site + n_ext + 10 * n_line);
  cudaMemcpyAsync(hv.data(), buf, hv.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
  if (!ck(h, cudaStreamSynchronize(h->stream))) return SUSY_B200_ECUDA;
  const double V = g.V;
  auto S = [&](int k) { return sum_range(hv, (size_t)k * nb, nb); };
  // link_trace
  double ave = 0.0, dave = 0.0;
  for (int a = 0; a < NUMLINK; a++) {
    m->linktr[a] = S(a) / V;
    m->link_det[a] = S(5 + a) / V;
    ave += m->linktr[a];
    dave += m->link_det[a];
  }
  ave /= NUMLINK;
  dave /= NUMLINK;
  m->linktr_ave = ave;
  m->linktr_width = sqrt(S(10) / (V * NUMLINK) - ave * ave);
  m->det_ave = dave;
  m->det_width = sqrt(S(11) / (V * NUMLINK) - dave * dave);
  // plaquette, gauge action
  m->ss_plaq = S(12) / (6.0 * V);
  m->st_plaq = S(13) / (4.0 * V);
  m->gauge_action = h->prm.kappa * S(25);
  // measure_det
  const double nd = 1.0 / (V * NPLAQ);
  m->det_tot_re = S(20) * nd;
  m->det_tot_im = S(21) * nd;
  m->det_sq_re = S(22) * nd;
  m->det_sq_im = S(23) * nd;
  m->det_wsq = S(24) * nd;
  // widths
  const double nw = 0.1 / V;
  const double pl = S(14) * nw, pl2 = S(15) * nw, dr = S(16) * nw, dr2 = S(17) * nw;
  const double di = S(18) * nw, di2 = S(19) * nw;
  m->width_plaq = sqrt(pl2 - pl * pl);
  m->width_det_re = sqrt(dr2 - dr * dr);
  m->width_det_im = sqrt(di2 - di * di);
  // scalar eigenvalues
  const double ne = 1.0 / (NUMLINK * V);
  for (int j = 0; j < 4; j++) {
    m->uubar_ave[j] = m->uubar_width[j] = m->uubar_min[j] = m->uubar_max[j] = 0.0;
    m->polar_ave[j] = m->polar_width[j] = m->polar_min[j] = m->polar_max[j] = 0.0;
  }
  for (int j = 0; j < N; j++) {
    const double ua = S(MS_BASE + j) * ne, us = S(MS_BASE + N + j) * ne;
    const double pa = S(MS_BASE + 2 * N + j) * ne, ps = S(MS_BASE + 3 * N + j) * ne;
    m->uubar_ave[j] = ua;
    m->uubar_width[j] = sqrt(us - ua * ua);
    m->polar_ave[j] = pa;
    m->polar_width[j] = sqrt(ps - pa * pa);
    double mn[2] = {1e300, 1e300}, mx[2] = {1e300, 1e300};
    for (int side = 0; side < 2; side++)
      for (int b = 0; b < nb; b++) {
        const double uv = hv[n_site + (size_t)(2 * j + side) * nb + b];
        const double pv = hv[n_site + (size_t)(2 * (N + j) + side) * nb + b];
        if (side == 0) {
          mn[0] = fmin(mn[0], uv);
          mn[1] = fmin(mn[1], pv);
        } else {
          mx[0] = fmin(mx[0], uv);
          mx[1] = fmin(mx[1], pv);
        }
      }
    m->uubar_min[j] = mn[0];
    m->uubar_max[j] = -mx[0];
    m->polar_min[j] = mn[1];
    m->polar_max[j] = -mx[1];
  }
  // lines
  const size_t l0 = n_site + n_ext;
  for (int q = 0; q < 10; q++) {
    const int d = q % 5;
    const int axis = d < 4 ? d : 3;
    const int len = axis == 0 ? g.nx : axis == 1 ? g.ny : axis == 2 ? g.nz : g.nt;
    const double norm = (double)len / V;
    const double re = sum_range(hv, l0 + q * n_line, nb) * norm;
    const double im = sum_range(hv, l0 + q * n_line + nb, nb) * norm;
    const double md = sum_range(hv, l0 + q * n_line + 2 * nb, nb) * norm;
    if (q < 5) {
      m->lines_re[d] = re;
      m->lines_im[d] = im;
      if (d == 3) {
        m->ploop_re = re;
        m->ploop_im = im;
        m->ploop_mod = md;
      }
    } else {
      m->lines_polar_re[d] = re;
      m->lines_polar_im[d] = im;
    }
  }
  return SUSY_B200_OK;
}

}  // namespace susy
