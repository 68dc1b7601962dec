// Per-site random numbers on the device.
//
// The reference gives every site its own generator (SITERAND,
// susy/defines.h:6): a 24-bit feedback shift register XOR a 32-bit linear
// congruential generator (generic/ranstuff.c:22-63), seeded from the
// global lexicographic site index (generic/make_lattice.c:48).  Gaussians
// are Marsaglia polar pairs with density exp(-x^2) (libraries/gaussrand.c:
// 12-32); every site draws an even number of them per call, so the pairing
// stays inside a site and all sites can run in parallel.  The integer
// stream is bit-identical to the reference; the Gaussians differ only where
// the device log() and the host libm log() round differently.
//
// State layout: prn[k * S + s], k = 0..6 shift register, 7 multiplier,
// 8 addend, 9 congruential state (all uint32).
#include "common.cuh"
#include "kernels.h"

namespace susy {

struct Prn {
  uint32_t r[7], mult, add, ic;
};

SUSY_D Prn load_prn(const uint32_t* st, int s, int S) {
  Prn p;
#pragma unroll
  for (int k = 0; k < 7; k++) p.r[k] = st[(size_t)k * S + s];
  p.mult = st[(size_t)7 * S + s];
  p.add = st[(size_t)8 * S + s];
  p.ic = st[(size_t)9 * S + s];
  return p;
}

SUSY_D void store_prn(uint32_t* st, int s, int S, const Prn& p) {
#pragma unroll
  for (int k = 0; k < 7; k++) st[(size_t)k * S + s] = p.r[k];
  st[(size_t)9 * S + s] = p.ic;
}

SUSY_D double myrand(Prn& p) {
  const uint32_t t = (((p.r[5] >> 7) | (p.r[6] << 17)) ^ ((p.r[4] >> 1) | (p.r[5] << 23))) & 0xffffffu;
  p.r[6] = p.r[5];
  p.r[5] = p.r[4];
  p.r[4] = p.r[3];
  p.r[3] = p.r[2];
  p.r[2] = p.r[1];
  p.r[1] = p.r[0];
  p.r[0] = t;
  p.ic = p.ic * p.mult + p.add;
  return (double)(t ^ ((p.ic >> 8) & 0xffffffu)) * (1.0 / 16777216.0);
}

// One pair of gaussian_rand_no calls: returns (v2 fac, v1 fac) as the
// reference hands them out.  The rejection loop is bounded; *bad is set if
// the bound is ever hit (probability ~ 0.27^256).
SUSY_D void gauss_pair(Prn& p, double& g1, double& g2, int* bad) {
  double v1 = 0.0, v2 = 0.0, r = 2.0;
  for (int k = 0; k < 256; k++) {
    v1 = 2.0 * myrand(p) - 1.0;
    v2 = 2.0 * myrand(p) - 1.0;
    r = v1 * v1 + v2 * v2;
    if (r < 1.0) break;
  }
  if (r >= 1.0) {
    *bad = 1;
    r = 0.5;
  }
  const double fac = sqrt(-log(r) / r);
  g1 = v2 * fac;
  g2 = v1 * fac;
}

// initialize_prn(prn, seed, index) with index = lexicographic site index
__global__ void k_init_prn(Geo g, int seed, uint32_t* st) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.V) return;
  const uint32_t m = 69607u + 8u * (uint32_t)s;
  uint32_t sd = (uint32_t)seed;
#pragma unroll
  for (int k = 0; k < 7; k++) {
    sd = m * sd + 12345u;
    st[(size_t)k * g.S + s] = (sd >> 8) & 0xffffffu;
  }
  sd = m * sd + 12345u;
  st[(size_t)7 * g.S + s] = 100005u + 8u * (uint32_t)s;
  st[(size_t)8 * g.S + s] = 12345u;
  st[(size_t)9 * g.S + s] = sd;
}

// Fill K matrices per site with sum_j (g + i g') Lambda_j, in the reference
// draw order: ranmom (grsource.c:49-63) loops links outer, generators inner;
// the pseudofermion (grsource.c:213-245) loops generators outer, components
// inner.  gen holds Lambda_j as [dimf][N][N] complex.
template <int N>
__global__ void k_gauss_fill(Geo g, uint32_t* st, const double2* gen, int K, int gen_outer,
                             double2* out, int* bad) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= g.V) return;
  constexpr int DIMF = N * N;
  Prn p = load_prn(st, s, g.S);
  Mat<N, double> acc[1];
  if (!gen_outer) {
    for (int k = 0; k < K; k++) {
      acc[0].zero();
      for (int j = 0; j < DIMF; j++) {
        double gr, gi;
        gauss_pair(p, gr, gi, bad);
        const Cx<double> z(gr, gi);
#pragma unroll
        for (int a = 0; a < N; a++)
#pragma unroll
          for (int b = 0; b < N; b++) {
            const double2 l = gen[(j * N + a) * N + b];
            acc[0].e[a][b] = acc[0].e[a][b] + z * Cx<double>(l.x, l.y);
          }
      }
      stm<N, double>(out, k, s, g.S, acc[0]);
    }
  } else {
    for (int k = 0; k < K; k++) {
      acc[0].zero();
      stm<N, double>(out, k, s, g.S, acc[0]);
    }
    for (int j = 0; j < DIMF; j++) {
      for (int k = 0; k < K; k++) {
        double gr, gi;
        gauss_pair(p, gr, gi, bad);
        const Cx<double> z(gr, gi);
        Mat<N, double> m = ldm<N, double>(out, k, s, g.S);
#pragma unroll
        for (int a = 0; a < N; a++)
#pragma unroll
          for (int b = 0; b < N; b++) {
            const double2 l = gen[(j * N + a) * N + b];
            m.e[a][b] = m.e[a][b] + z * Cx<double>(l.x, l.y);
          }
        stm<N, double>(out, k, s, g.S, m);
      }
    }
  }
  store_prn(st, s, g.S, p);
}

void init_prn(const Geo& g, int seed, void* st, cudaStream_t s) {
  count_launch(), k_init_prn<<<(g.V + 127) / 128, 128, 0, s>>>(g, seed, (uint32_t*)st);
}

void gauss_fill(const Geo& g, int N, void* st, const void* gen, int K, int gen_outer, void* out,
                int* bad, cudaStream_t s) {
  const int nb = (g.V + 127) / 128;
  switch (N) {
    case 2: count_launch(), k_gauss_fill<2><<<nb, 128, 0, s>>>(g, (uint32_t*)st, (const double2*)gen, K, gen_outer, (double2*)out, bad); break;
    case 3: count_launch(), k_gauss_fill<3><<<nb, 128, 0, s>>>(g, (uint32_t*)st, (const double2*)gen, K, gen_outer, (double2*)out, bad); break;
    case 4: count_launch(), k_gauss_fill<4><<<nb, 128, 0, s>>>(g, (uint32_t*)st, (const double2*)gen, K, gen_outer, (double2*)out, bad); break;
  }
}

}  // namespace susy
