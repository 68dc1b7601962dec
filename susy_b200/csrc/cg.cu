// Multi-shift conjugate gradient on (D^dag D + fmass^2 + shift_j), the
// reference's congrad_multi (4d_Q16/susy/congrad_multi.c:26-221): zero
// initial guess, Jegerlehner recurrences for the shifted systems, shift j
// frozen once zeta_j^2 |r|^2 <= errormin |src|^2, stop when |r|^2 of the
// base system reaches errormin |src|^2 or MaxCG iterations.
//
// Everything stays on the device.  The scalar recurrences run in FP64 in
// one-block kernels that read the FP64 block partials of the two inner
// products, so an iteration needs no host round trip; the host only polls
// the state every few iterations.  Per iteration:
//   fermion_op(+1)              tmp = D p0
//   fermion_op(-1, epilogue)    mp = D^dag tmp + (fmass^2 + shift_0) p0,
//                               partials of Re<p0, mp>
//   k_ms_scalars1               beta_0 = -|r|^2 / <p0, mp>, zeta/beta_j
//   k_ms_update_a               psi_j -= beta_j p_j; r += beta_0 mp;
//                               partials of |r|^2
//   k_ms_scalars2               alpha_j, freeze test, scroll
//   k_ms_update_b               p_j = zeta_j r + alpha_j p_j
// Vectors are FP64 (VT = double2) for the reference-faithful solver or FP32
// (float2) for the low-precision pass of the mixed solver.
#include "common.cuh"
#include "kernels.h"

namespace susy {

constexpr int UT = 256;
constexpr int ST = 256;

__global__ void k_ms_init(MsState* st, const double* partials, int np, int maxcg,
                          double errormin, int record) {
  __shared__ double sh[ST];
  double v = 0.0;
  for (int i = threadIdx.x; i < np; i += ST) v += partials[i];
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int o = ST / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double sn = sh[0];
    st->source_norm = sn;
    st->rsq = sn;
    st->rsqstop = errormin * sn;
    st->rsqfreeze = errormin * sn;
    st->iter = 0;
    st->maxcg = maxcg;
    for (int j = 0; j < st->nshift; j++) {
      st->zeta_im1[j] = 1.0;
      st->zeta_i[j] = 1.0;
      st->zeta_ip1[j] = 1.0;
      st->alpha[j] = 0.0;
      st->beta_im1[j] = 1.0;
      st->beta_i[j] = 0.0;
      st->converged[j] = 0;
      st->active_p[j] = 1;
      st->pz[j] = 1.0;
      st->pa[j] = 0.0;
      st->pact[j] = 1;
    }
    st->skip = (st->rsq <= st->rsqstop || maxcg <= 0) ? 1 : 0;
    st->skip_b = 1;
    st->record = record;
    st->done_r = 0;
    st->blk_len = 0;
    st->blk_start = 0;
    for (int j = 0; j < MS_MAXS; j++) st->live[j] = j < st->nshift;
  }
}

SUSY_D double block_reduce_all(double v, double* sh) {
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int o = ST / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  return sh[0];
}

// The scalar recurrences after the operator, run by one block of ST threads
SUSY_D void scalars1_block(MsState* st, const double* partials, int np, double* sh) {
  if (st->skip) {
    if (threadIdx.x == 0) st->skip_b = 1;
    return;
  }
  double v = 0.0;
  for (int i = threadIdx.x; i < np; i += ST) v += partials[i];
  const double cd = block_reduce_all(v, sh);
  if (threadIdx.x != 0) return;
  st->skip_b = 0;
  st->cd = cd;
  st->iter += 1;
  const double b0 = -st->rsq / cd;
  st->beta_i[0] = b0;
  st->zeta_ip1[0] = 1.0;
  const double s0 = st->shift[0];
  for (int j = 1; j < st->nshift; j++) {
    if (st->converged[j]) continue;
    double z = st->zeta_i[j] * st->zeta_im1[j] * st->beta_im1[0];
    const double c1 = b0 * st->alpha[0] * (st->zeta_im1[j] - st->zeta_i[j]);
    const double c2 = st->zeta_im1[j] * st->beta_im1[0] * (1.0 - (st->shift[j] - s0) * b0);
    z /= c1 + c2;
    st->zeta_ip1[j] = z;
    st->beta_i[j] = b0 * z / st->zeta_i[j];
  }
}

__global__ void k_ms_scalars1(MsState* st, const double* partials, int np) {
  __shared__ double sh[ST];
  scalars1_block(st, partials, np, sh);
}

// The scalar recurrences after the residual update, run by one block of ST
// threads: its own kernel, or the last block of the fused residual update
// (partials read from L2: other blocks wrote them)
SUSY_D void scalars2_block(MsState* st, const double* partials, int np, double* sh) {
  double v = 0.0;
  for (int i = threadIdx.x; i < np; i += ST) v += __ldcg(partials + i);
  const double rsqnew = block_reduce_all(v, sh);
  if (threadIdx.x != 0) return;
  const double a0 = rsqnew / st->rsq;
  st->alpha[0] = a0;
  st->active_p[0] = 1;
  for (int j = 1; j < st->nshift; j++) {
    st->active_p[j] = !st->converged[j];
    if (st->converged[j]) continue;
    st->alpha[j] = a0 * st->zeta_ip1[j] * st->beta_i[j] / (st->zeta_i[j] * st->beta_i[0]);
  }
  if (st->record && st->blk_len < MS_BLK) {
    // this iteration's coefficients, before this iteration's freeze test:
    // a shift frozen in an earlier iteration took no step in this one
    const int t = st->blk_len++;
    for (int j = 0; j < st->nshift; j++) {
      const bool live = j == 0 || !st->converged[j];
      st->hb[t][j] = live ? st->beta_i[j] : 0.0;
      st->hz[t][j] = j == 0 ? 1.0 : st->zeta_ip1[j];
      st->ha[t][j] = st->alpha[j];
    }
  }
  for (int j = 0; j < st->nshift; j++) {
    st->pz[j] = st->zeta_ip1[j];
    st->pa[j] = st->alpha[j];
    st->pact[j] = st->active_p[j];
  }
  st->rsq = rsqnew;
  for (int j = 1; j < st->nshift; j++) {
    if (st->converged[j]) continue;
    // converged[j] = the iteration at which shift j froze (>= 1; 0 = live)
    if (rsqnew * st->zeta_ip1[j] * st->zeta_ip1[j] <= st->rsqfreeze) st->converged[j] = st->iter;
  }
  for (int j = 0; j < st->nshift; j++) {
    if (st->converged[j]) continue;
    st->beta_im1[j] = st->beta_i[j];
    st->zeta_im1[j] = st->zeta_i[j];
    st->zeta_i[j] = st->zeta_ip1[j];
  }
  st->skip = (rsqnew <= st->rsqstop || st->iter >= st->maxcg) ? 1 : 0;
}

__global__ void k_ms_scalars2(MsState* st, const double* partials, int np) {
  __shared__ double sh[ST];
  if (st->skip) return;
  scalars2_block(st, partials, np, sh);
}

// psi_j -= beta_j p_j (j = 0 and every live shift), r += beta_0 mp, |r|^2
// VT: type of p, r, mp; XT: type of the solutions psi
template <typename VT, typename XT>
__global__ void __launch_bounds__(UT) k_ms_update_a(MsState* st, MsVecs v, long n, double* part) {
  __shared__ double sb[MS_MAXS];
  __shared__ int sc[MS_MAXS];
  if (st->skip) return;
  const int ns = st->nshift;
  if (threadIdx.x < ns) {
    sb[threadIdx.x] = st->beta_i[threadIdx.x];
    sc[threadIdx.x] = threadIdx.x == 0 ? 0 : st->converged[threadIdx.x];
  }
  __syncthreads();
  const long i = (long)blockIdx.x * UT + threadIdx.x;
  double acc = 0.0;
  if (i < n) {
    const VT* mp = (const VT*)v.mp;
    VT* r = (VT*)v.r;
#pragma unroll 1
    for (int j = 0; j < ns; j++) {
      if (sc[j]) continue;
      const VT pj = ((const VT*)v.p[j])[i];
      XT* pp = (XT*)v.psi[j] + i;
      XT x = *pp;
      x.x -= sb[j] * pj.x;
      x.y -= sb[j] * pj.y;
      *pp = x;
    }
    VT rr = r[i];
    const VT m = mp[i];
    rr.x += sb[0] * m.x;
    rr.y += sb[0] * m.y;
    r[i] = rr;
    acc = (double)rr.x * rr.x + (double)rr.y * rr.y;
  }
  acc = block_sum<UT>(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

// p_j = zeta_ip1_j r + alpha_j p_j for the shifts that were live
template <typename VT>
__global__ void __launch_bounds__(UT) k_ms_update_b(MsState* st, MsVecs v, long n) {
  __shared__ double sz[MS_MAXS], sa[MS_MAXS];
  __shared__ int sc[MS_MAXS];
  if (st->skip_b) return;
  const int ns = st->nshift;
  if (threadIdx.x < ns) {
    sz[threadIdx.x] = st->zeta_ip1[threadIdx.x];
    sa[threadIdx.x] = st->alpha[threadIdx.x];
    sc[threadIdx.x] = st->active_p[threadIdx.x];
  }
  __syncthreads();
  const long i = (long)blockIdx.x * UT + threadIdx.x;
  if (i >= n) return;
  const VT r = ((const VT*)v.r)[i];
#pragma unroll 1
  for (int j = 0; j < ns; j++) {
    if (!sc[j]) continue;
    VT* pp = (VT*)v.p[j] + i;
    VT p = *pp;
    p.x = sz[j] * r.x + sa[j] * p.x;
    p.y = sz[j] * r.y + sa[j] * p.y;
    *pp = p;
  }
}

// One pass per iteration over every live shift (congrad_multi.c:109-150 with
// the p_j update of the previous iteration folded in):
//   p_j = pz_j r + pa_j p_j  (deferred from the previous iteration, j >= 1)
//   psi_j -= beta_j p_j      (j = 0 uses p0, updated by k_ms_update_p0)
//   r += beta_0 mp;  partials of |r|^2
// Each live shift costs 4 field streams (read p, psi; write p, psi); the
// arithmetic per element is the same as the two-pass form.
// blk: the block's index among the field's ceil(n / UT) blocks
template <typename VT, typename XT>
SUSY_D void update_fused_block(MsState* st, const MsVecs& v, long n, double* part, int blk) {
  __shared__ double sb[MS_MAXS], sz[MS_MAXS], sa[MS_MAXS];
  __shared__ int sc[MS_MAXS], sp[MS_MAXS];
  if (st->skip) return;
  const int ns = st->nshift;
  if (threadIdx.x < ns) {
    const int j = threadIdx.x;
    sb[j] = st->beta_i[j];
    sc[j] = j == 0 ? 0 : st->converged[j];
    sz[j] = st->pz[j];
    sa[j] = st->pa[j];
    sp[j] = j == 0 ? 0 : st->pact[j];
  }
  __syncthreads();
  const long i = (long)blk * UT + threadIdx.x;
  double acc = 0.0;
  if (i < n) {
    VT rr = ((VT*)v.r)[i];
#pragma unroll 1
    for (int j = 0; j < ns; j++) {
      if (sc[j]) continue;
      VT* pq = (VT*)v.p[j] + i;
      VT pj = *pq;
      if (sp[j]) {
        pj.x = sz[j] * rr.x + sa[j] * pj.x;
        pj.y = sz[j] * rr.y + sa[j] * pj.y;
        *pq = pj;
      }
      XT* pp = (XT*)v.psi[j] + i;
      XT x = *pp;
      x.x -= sb[j] * pj.x;
      x.y -= sb[j] * pj.y;
      *pp = x;
    }
    const VT m = ((const VT*)v.mp)[i];
    rr.x += sb[0] * m.x;
    rr.y += sb[0] * m.y;
    ((VT*)v.r)[i] = rr;
    acc = (double)rr.x * rr.x + (double)rr.y * rr.y;
  }
  acc = block_sum<UT>(acc);
  if (threadIdx.x == 0) part[blk] = acc;
}

template <typename VT, typename XT>
__global__ void __launch_bounds__(UT) k_ms_update_fused(MsState* st, MsVecs v, long n,
                                                        double* part) {
  update_fused_block<VT, XT>(st, v, n, part, blockIdx.x);
}

// p0 = r + alpha_0 p0 (zeta_0 = 1), ahead of the next D^dag D p0
template <typename VT>
SUSY_D void update_p0_block(MsState* st, const MsVecs& v, long n, int blk) {
  if (st->skip_b) return;
  const long i = (long)blk * UT + threadIdx.x;
  if (i >= n) return;
  const double a0 = st->alpha[0];
  const VT r = ((const VT*)v.r)[i];
  VT* pp = (VT*)v.p[0] + i;
  VT p = *pp;
  p.x = r.x + a0 * p.x;
  p.y = r.y + a0 * p.y;
  *pp = p;
}

template <typename VT>
__global__ void __launch_bounds__(UT) k_ms_update_p0(MsState* st, MsVecs v, long n) {
  update_p0_block<VT>(st, v, n, blockIdx.x);
}

// |x|^2 partials over n complex entries
template <typename VT>
__global__ void __launch_bounds__(UT) k_norm2(const VT* x, long n, double* part) {
  const long i = (long)blockIdx.x * UT + threadIdx.x;
  double acc = 0.0;
  if (i < n) {
    const VT a = x[i];
    acc = (double)a.x * a.x + (double)a.y * a.y;
  }
  acc = block_sum<UT>(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

int vec_blocks(long n) { return (int)((n + UT - 1) / UT); }

void ms_init(MsState* st, const void* src, int prec, long n, double* part, int maxcg,
             double errormin, cudaStream_t s, int record) {
  const int nb = vec_blocks(n);
  if (prec == 64)
    count_launch(), k_norm2<double2><<<nb, UT, 0, s>>>((const double2*)src, n, part);
  else
    count_launch(), k_norm2<float2><<<nb, UT, 0, s>>>((const float2*)src, n, part);
  count_launch(), k_ms_init<<<1, ST, 0, s>>>(st, part, nb, maxcg, errormin, record);
}

void ms_scalars1(MsState* st, const double* part, int np, cudaStream_t s) {
  count_launch(), k_ms_scalars1<<<1, ST, 0, s>>>(st, part, np);
}

void ms_scalars2(MsState* st, const double* part, int np, cudaStream_t s) {
  count_launch(), k_ms_scalars2<<<1, ST, 0, s>>>(st, part, np);
}

void ms_update_a(MsState* st, const MsVecs& v, int prec, int prec_x, long n, double* part,
                 cudaStream_t s) {
  if (prec == 64)
    count_launch(), k_ms_update_a<double2, double2><<<vec_blocks(n), UT, 0, s>>>(st, v, n, part);
  else if (prec_x == 64)
    count_launch(), k_ms_update_a<float2, double2><<<vec_blocks(n), UT, 0, s>>>(st, v, n, part);
  else
    count_launch(), k_ms_update_a<float2, float2><<<vec_blocks(n), UT, 0, s>>>(st, v, n, part);
}

// r64 = b - ax, r32 = (float) r64, partials of |r64|^2
__global__ void __launch_bounds__(UT) k_residual(long n, const double2* b, const double2* ax,
                                                 double2* r64, float2* r32, double* part) {
  const long i = (long)blockIdx.x * UT + threadIdx.x;
  double acc = 0.0;
  if (i < n) {
    const double2 u = b[i], w = ax[i];
    const double2 r = make_double2(u.x - w.x, u.y - w.y);
    if (r64) r64[i] = r;
    if (r32) r32[i] = make_float2((float)r.x, (float)r.y);
    acc = r.x * r.x + r.y * r.y;
  }
  acc = block_sum<UT>(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

// x64 += e32
__global__ void k_add_low(long n, const float2* e, double2* x) {
  const long i = (long)blockIdx.x * UT + threadIdx.x;
  if (i >= n) return;
  double2 v = x[i];
  const float2 d = e[i];
  v.x += d.x;
  v.y += d.y;
  x[i] = v;
}

__global__ void k_scale(long n, double s, double2* x) {
  const long i = (long)blockIdx.x * UT + threadIdx.x;
  if (i >= n) return;
  double2 v = x[i];
  v.x *= s;
  v.y *= s;
  x[i] = v;
}

int residual_partials(long n, const void* b, const void* ax, void* r64, void* r32, double* part,
                      cudaStream_t s) {
  count_launch(), k_residual<<<vec_blocks(n), UT, 0, s>>>(n, (const double2*)b, (const double2*)ax,
                                          (double2*)r64, (float2*)r32, part);
  return vec_blocks(n);
}

void add_low(long n, const void* e32, void* x64, cudaStream_t s) {
  count_launch(), k_add_low<<<vec_blocks(n), UT, 0, s>>>(n, (const float2*)e32, (double2*)x64);
}

void scale_field(long n, double sc, void* x, cudaStream_t s) {
  count_launch(), k_scale<<<vec_blocks(n), UT, 0, s>>>(n, sc, (double2*)x);
}

void ms_update_b(MsState* st, const MsVecs& v, int prec, long n, cudaStream_t s) {
  if (prec == 64)
    count_launch(), k_ms_update_b<double2><<<vec_blocks(n), UT, 0, s>>>(st, v, n);
  else
    count_launch(), k_ms_update_b<float2><<<vec_blocks(n), UT, 0, s>>>(st, v, n);
}

void ms_update_fused(MsState* st, const MsVecs& v, int prec, int prec_x, long n, double* part,
                     cudaStream_t s) {
  if (prec == 64)
    count_launch(), k_ms_update_fused<double2, double2><<<vec_blocks(n), UT, 0, s>>>(st, v, n, part);
  else if (prec_x == 64)
    count_launch(), k_ms_update_fused<float2, double2><<<vec_blocks(n), UT, 0, s>>>(st, v, n, part);
  else
    count_launch(), k_ms_update_fused<float2, float2><<<vec_blocks(n), UT, 0, s>>>(st, v, n, part);
}

void ms_update_p0(MsState* st, const MsVecs& v, int prec, long n, cudaStream_t s) {
  if (prec == 64)
    count_launch(), k_ms_update_p0<double2><<<vec_blocks(n), UT, 0, s>>>(st, v, n);
  else
    count_launch(), k_ms_update_p0<float2><<<vec_blocks(n), UT, 0, s>>>(st, v, n);
}

// ---------------------------------------------------------------------------
// Blocked update of the solutions and shifted search vectors.
//
// The per-iteration pass of the reference's recurrences reads and writes
// psi_j and p_j of every live shift every iteration (4 field streams per
// shift).  Over a block of L iterations starting at iteration k, with
// R_s = r(k + s) the residuals the base recurrence produces,
//   p_j(k + t) = c_t p_j(k) + sum_{s <= t} d_{t,s} R_s
//   (c_0 = 1, c_{t+1} = a_t c_t, d_{t+1,s} = a_t d_{t,s}, d_{t+1,t+1} = z_t)
//   psi_j(k + L) = psi_j(k) - sum_t b_t p_j(k + t)
// with b_t, z_t, a_t shift j's beta, zeta(i+1), alpha of iteration k + t.
// So one pass per block reads R_1..R_L once (shared by all shifts) and
// psi_j, p_j once per shift: 4 streams per shift per L iterations instead
// of per iteration.  The residual itself lives in a ring of L + 1 fields
// so no copy is made.  Same arithmetic, summed in a different order.

// r(i) = r(i-1) + beta_0 mp and partials of |r(i)|^2; i = iteration count
// after this iteration's scalars1.  MT: type of mp (FP64, or FP32 when the
// operator ran in FP32).  The block that finishes last (a counter in the
// solver state, taken after each block's partial is written and fenced)
// sums the partials and runs the scalar recurrences, which saves a
// dependent single-block launch per iteration; it resets the counter for
// the next launch.  Every block reads skip before the last one can change
// it.
// RT: type of the ring (FP64, or FP32 with f32 vectors)
template <typename VT> SUSY_D double2 ld2(const VT* p, long i) {
  const VT v = p[i];
  return make_double2(v.x, v.y);
}
template <typename VT> SUSY_D void st2(VT* p, long i, double2 v);
template <> SUSY_D void st2<double2>(double2* p, long i, double2 v) { p[i] = v; }
template <> SUSY_D void st2<float2>(float2* p, long i, double2 v) {
  p[i] = make_float2((float)v.x, (float)v.y);
}
// v as a VT holds it
template <typename VT> SUSY_D double2 rnd2(double2 v);
template <> SUSY_D double2 rnd2<double2>(double2 v) { return v; }
template <> SUSY_D double2 rnd2<float2>(double2 v) {
  return make_double2((double)(float)v.x, (double)(float)v.y);
}

template <typename MT, typename RT>
__global__ void __launch_bounds__(UT) k_msb_update_r(MsState* st, MsBlockVecs v, long n,
                                                     double* part) {
  static_assert(UT == ST, "the last block runs the ST-thread scalar step");
  __shared__ double sh[ST];
  __shared__ int last;
  if (st->skip) return;
  const int it = st->iter;
  const double b0 = st->beta_i[0];
  const RT* rin = (const RT*)v.ring[(it - 1) % (MS_BLK + 1)];
  RT* rout = (RT*)v.ring[it % (MS_BLK + 1)];
  const MT* mp = (const MT*)(sizeof(MT) == 16 ? v.mp : v.mp32);
  double acc = 0.0;
  // grid-stride: few blocks, so the scalar kernel sums few partials
  for (long i = (long)blockIdx.x * UT + threadIdx.x; i < n; i += (long)gridDim.x * UT) {
    double2 r = ld2(rin, i);
    const MT m = mp[i];
    r.x += b0 * m.x;
    r.y += b0 * m.y;
    st2(rout, i, r);
    const double2 rr = rnd2<RT>(r);   // |r|^2 of the residual as stored
    acc += rr.x * rr.x + rr.y * rr.y;
  }
  acc = block_sum<UT>(acc);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = acc;
    __threadfence();
    last = atomicAdd(&st->done_r, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  if (threadIdx.x == 0) st->done_r = 0;
  scalars2_block(st, part, gridDim.x, sh);
}

// p0 = r(i) + alpha_0 p0 (and its FP32 copy for an FP32 operator)
template <typename RT>
__global__ void __launch_bounds__(UT) k_msb_update_p0(MsState* st, MsBlockVecs v, long n) {
  if (st->skip_b) return;
  const long i = (long)blockIdx.x * UT + threadIdx.x;
  if (i >= n) return;
  const double a0 = st->alpha[0];
  const double2 r = ld2((const RT*)v.ring[st->iter % (MS_BLK + 1)], i);
  double2 p = ld2((const RT*)v.p0, i);
  p.x = r.x + a0 * p.x;
  p.y = r.y + a0 * p.y;
  st2((RT*)v.p0, i, p);
  if (v.p0_32) ((float2*)v.p0_32)[i] = make_float2((float)p.x, (float)p.y);
}

// Residual replacement at a block boundary (k = st->iter): r(k) becomes the
// true residual rt, and the search vectors built from the old r(k) get the
// same correction d = rt - r(k) so that p0 = r(k) + alpha p0_prev and
// P_j = zeta_j r(k) + alpha_j P_j,prev keep holding (zeta_0 = 1)
template <typename RT>
__global__ void __launch_bounds__(UT) k_msb_replace(MsState* st, MsBlockVecs v, long n,
                                                    const double2* rt) {
  __shared__ double z[MS_MAXS];
  __shared__ int lv[MS_MAXS];
  const int ns = st->nshift;
  if (threadIdx.x < ns) {
    const int j = threadIdx.x;
    lv[j] = st->live[j];
    z[j] = j == 0 ? 1.0 : st->zeta_i[j];
  }
  __syncthreads();
  const long i = (long)blockIdx.x * UT + threadIdx.x;
  if (i >= n) return;
  RT* r = (RT*)v.ring[st->iter % (MS_BLK + 1)];
  const double2 t = rt[i];
  const double2 r0 = ld2(r, i);
  const double2 d = make_double2(t.x - r0.x, t.y - r0.y);
  st2(r, i, t);
  double2 p = ld2((const RT*)v.p0, i);
  p.x += d.x;
  p.y += d.y;
  st2((RT*)v.p0, i, p);
  if (v.p0_32) ((float2*)v.p0_32)[i] = make_float2((float)p.x, (float)p.y);
#pragma unroll 1
  for (int j = 0; j < ns; j++) {
    if (!lv[j]) continue;
    double2* pj = (double2*)v.P[j] + i;
    double2 q = *pj;
    q.x += z[j] * d.x;
    q.y += z[j] * d.y;
    *pj = q;
  }
}

// Stop the base system at errormin_base |src|^2 (shifts keep freezing at
// rsqfreeze)
__global__ void k_ms_set_stop(MsState* st, double errormin_base) {
  st->rsqstop = errormin_base * st->source_norm;
  st->skip = (st->rsq <= st->rsqstop || st->maxcg <= 0) ? 1 : 0;
}

void ms_set_stop(MsState* st, double errormin_base, cudaStream_t s) {
  count_launch(), k_ms_set_stop<<<1, 1, 0, s>>>(st, errormin_base);
}

__global__ void k_msb_set_rsq(MsState* st, double rsq) {
  st->rsq = rsq;
  st->skip = (rsq <= st->rsqstop || st->iter >= st->maxcg) ? 1 : 0;
}

// The block pass: every live shift's psi_j and P_j advanced over the
// recorded iterations.  Each CTA first derives the combination
// coefficients of every live shift in shared memory.
template <typename RT>
__global__ void __launch_bounds__(UT) k_msb_block(MsState* st, MsBlockVecs v, long n) {
  __shared__ double cx0[MS_MAXS], cp0[MS_MAXS];
  __shared__ double cxr[MS_MAXS][MS_BLK], cpr[MS_MAXS][MS_BLK];
  __shared__ int lv[MS_MAXS];
  const int L = st->blk_len;
  if (L == 0) return;
  const int ns = st->nshift;
  const int k = st->blk_start;
  if (threadIdx.x < ns) {
    const int j = threadIdx.x;
    lv[j] = st->live[j];
    // c_t and d_{t,s} for t = 0..L, s = 1..t (d indexed s-1)
    double c = 1.0, d[MS_BLK];
    double x0 = 0.0, xr[MS_BLK];
#pragma unroll
    for (int q = 0; q < MS_BLK; q++) d[q] = xr[q] = 0.0;
    for (int t = 0; t < L; t++) {
      const double b = st->hb[t][j], z = st->hz[t][j], a = st->ha[t][j];
      // psi -= b_t p(k + t)
      x0 += b * c;
#pragma unroll
      for (int q = 0; q < MS_BLK; q++)
        if (q < t) xr[q] += b * d[q];
      // p(k + t + 1) = z_t R_{t+1} + a_t p(k + t)
      c *= a;
#pragma unroll
      for (int q = 0; q < MS_BLK; q++) {
        if (q < t) d[q] *= a;
        if (q == t) d[q] = z;
      }
    }
    cx0[j] = x0;
    cp0[j] = c;
#pragma unroll
    for (int q = 0; q < MS_BLK; q++) {
      cxr[j][q] = xr[q];
      cpr[j][q] = d[q];
    }
  }
  __syncthreads();
  const long i = (long)blockIdx.x * UT + threadIdx.x;
  if (i >= n) return;
  double2 R[MS_BLK];
#pragma unroll
  for (int q = 0; q < MS_BLK; q++)
    R[q] = q < L ? ld2((const RT*)v.ring[(k + 1 + q) % (MS_BLK + 1)], i) : make_double2(0, 0);
#pragma unroll 1
  for (int j = 0; j < ns; j++) {
    if (!lv[j]) continue;
    double2* xp = (double2*)v.x[j] + i;
    double2* pp = (double2*)v.P[j] + i;
    const double2 p = *pp;
    double2 x = *xp;
    double2 pn;
    x.x -= cx0[j] * p.x;
    x.y -= cx0[j] * p.y;
    pn.x = cp0[j] * p.x;
    pn.y = cp0[j] * p.y;
#pragma unroll
    for (int q = 0; q < MS_BLK; q++) {
      x.x -= cxr[j][q] * R[q].x;
      x.y -= cxr[j][q] * R[q].y;
      pn.x += cpr[j][q] * R[q].x;
      pn.y += cpr[j][q] * R[q].y;
    }
    *xp = x;
    *pp = pn;
  }
}

// Close the block: shifts frozen by now take no part in later blocks
__global__ void k_msb_block_reset(MsState* st) {
  const int j = threadIdx.x;
  if (j < MS_MAXS) st->live[j] = j < st->nshift && (j == 0 || !st->converged[j]);
  __syncthreads();
  if (j == 0) {
    st->blk_start = st->iter;
    st->blk_len = 0;
  }
}

// Returns the number of partials written (at most 8 blocks per SM of a
// 148-SM B200)
void msb_update_r(MsState* st, const MsBlockVecs& v, long n, double* part, bool mp32,
                  cudaStream_t s) {
  const int nb = vec_blocks(n) < 1184 ? vec_blocks(n) : 1184;
  if (v.f32)
    count_launch(), k_msb_update_r<float2, float2><<<nb, UT, 0, s>>>(st, v, n, part);
  else if (mp32)
    count_launch(), k_msb_update_r<float2, double2><<<nb, UT, 0, s>>>(st, v, n, part);
  else
    count_launch(), k_msb_update_r<double2, double2><<<nb, UT, 0, s>>>(st, v, n, part);
}

// Residual replacement: r(k) <- rt with the matching search-vector
// correction, and the iterated |r|^2 becomes the true one (the stop flag
// follows it)
void msb_replace(MsState* st, const MsBlockVecs& v, long n, const void* rt, double rsq,
                 cudaStream_t s) {
  if (v.f32)
    count_launch(), k_msb_replace<float2><<<vec_blocks(n), UT, 0, s>>>(st, v, n, (const double2*)rt);
  else
    count_launch(), k_msb_replace<double2><<<vec_blocks(n), UT, 0, s>>>(st, v, n, (const double2*)rt);
  count_launch(), k_msb_set_rsq<<<1, 1, 0, s>>>(st, rsq);
}

void msb_update_p0(MsState* st, const MsBlockVecs& v, long n, cudaStream_t s) {
  if (v.f32)
    count_launch(), k_msb_update_p0<float2><<<vec_blocks(n), UT, 0, s>>>(st, v, n);
  else
    count_launch(), k_msb_update_p0<double2><<<vec_blocks(n), UT, 0, s>>>(st, v, n);
}

void msb_block(MsState* st, const MsBlockVecs& v, long n, cudaStream_t s) {
  if (v.f32)
    count_launch(), k_msb_block<float2><<<vec_blocks(n), UT, 0, s>>>(st, v, n);
  else
    count_launch(), k_msb_block<double2><<<vec_blocks(n), UT, 0, s>>>(st, v, n);
  count_launch(), k_msb_block_reset<<<1, MS_MAXS, 0, s>>>(st);
}

// Re <a, b> partials over n FP64 complex entries
__global__ void __launch_bounds__(UT) k_rdot(long n, const double2* a, const double2* b,
                                             double* part) {
  const long i = (long)blockIdx.x * UT + threadIdx.x;
  double acc = 0.0;
  if (i < n) {
    const double2 u = a[i], v = b[i];
    acc = u.x * v.x + u.y * v.y;
  }
  acc = block_sum<UT>(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

int rdot_partials(long n, const void* a, const void* b, double* part, cudaStream_t s) {
  count_launch(), k_rdot<<<vec_blocks(n), UT, 0, s>>>(n, (const double2*)a, (const double2*)b, part);
  return vec_blocks(n);
}

void copy_field(long n, const void* a, void* b, cudaStream_t s) {
  cudaMemcpyAsync(b, a, (size_t)n * sizeof(double2), cudaMemcpyDeviceToDevice, s);
}

void norm2_partials(const void* x, int prec, long n, double* part, cudaStream_t s) {
  if (prec == 64)
    count_launch(), k_norm2<double2><<<vec_blocks(n), UT, 0, s>>>((const double2*)x, n, part);
  else
    count_launch(), k_norm2<float2><<<vec_blocks(n), UT, 0, s>>>((const float2*)x, n, part);
}

}  // namespace susy

// ---------------------------------------------------------------------------
// Batched FP64 multi-shift solve: the per-iteration kernels above for every
// lattice of a batch in one launch each.  The recurrence kernels run one
// block per lattice; the vector kernels walk a table of vector blocks in
// which lattice i owns blocks [vblk0, vblk0 + vblocks).  Each lattice's
// state, stop flag and partials are its own, so every lattice follows the
// solo recurrences and stops at its own iteration.
namespace susy {

// Largest i < nl with L[i].vblk0 <= b
SUSY_D int vblock_lattice(const MsLat* L, int nl, int b) {
  int lo = 0, hi = nl - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (L[mid].vblk0 <= b)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

__global__ void k_msbat_scalars1(const MsLat* L) {
  __shared__ double sh[ST];
  const MsLat& l = L[blockIdx.x];
  scalars1_block(l.st, l.part0, l.np0, sh);
}

__global__ void k_msbat_scalars2(const MsLat* L) {
  __shared__ double sh[ST];
  const MsLat& l = L[blockIdx.x];
  if (l.st->skip) return;
  scalars2_block(l.st, l.part1, l.vblocks, sh);
}

__global__ void __launch_bounds__(UT) k_msbat_update_fused(const MsLat* L, int nl) {
  const MsLat& l = L[vblock_lattice(L, nl, blockIdx.x)];
  update_fused_block<double2, double2>(l.st, l.v, l.n, l.part1, blockIdx.x - l.vblk0);
}

__global__ void __launch_bounds__(UT) k_msbat_update_p0(const MsLat* L, int nl) {
  const MsLat& l = L[vblock_lattice(L, nl, blockIdx.x)];
  update_p0_block<double2>(l.st, l.v, l.n, blockIdx.x - l.vblk0);
}

__global__ void k_msbat_skips(const MsLat* L, int nl, int* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nl) out[i] = L[i].st->skip;
}

void ms_batch_scalars1(const MsLat* L, int nl, cudaStream_t s) {
  count_launch(), k_msbat_scalars1<<<nl, ST, 0, s>>>(L);
}
void ms_batch_update_fused(const MsLat* L, int nl, int vtot, cudaStream_t s) {
  count_launch(), k_msbat_update_fused<<<vtot, UT, 0, s>>>(L, nl);
}
void ms_batch_scalars2(const MsLat* L, int nl, cudaStream_t s) {
  count_launch(), k_msbat_scalars2<<<nl, ST, 0, s>>>(L);
}
void ms_batch_update_p0(const MsLat* L, int nl, int vtot, cudaStream_t s) {
  count_launch(), k_msbat_update_p0<<<vtot, UT, 0, s>>>(L, nl);
}
void ms_batch_skips(const MsLat* L, int nl, int* out, cudaStream_t s) {
  count_launch(), k_msbat_skips<<<(nl + 63) / 64, 64, 0, s>>>(L, nl, out);
}

}  // namespace susy
