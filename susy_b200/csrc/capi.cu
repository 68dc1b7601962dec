// C ABI (include/susy_b200.h): lattice handle, host <-> device transfers,
// fermion operator, DSq and the multi-shift CG driver.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <vector>
#include <atomic>
#include <climits>
#include "../../include/susy_b200.h"
#include "kernels.h"
#include "lattice.h"
#include "hmc.h"

using namespace susy;

namespace susy {

static std::atomic<long long> g_launches(0);
// Per host thread as well, so that a thread capturing a CUDA graph can
// count its own launches while other threads launch (update_batch)
static thread_local long long t_launches = 0;
void count_launch() {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  t_launches++;
}
void count_launches(long long n) {
  g_launches.fetch_add(n, std::memory_order_relaxed);
  t_launches += n;
}
long long thread_launch_count() { return t_launches; }

static size_t mat_c(const susy_b200_lattice* h) { return (size_t)h->N * h->N; }

bool make_geo(long nx, long ny, long nz, long nt, int ncol, int pbc, Geo* g) {
  if (ncol < 2 || ncol > 4 || (pbc != 1 && pbc != -1)) return false;
  const long ext[4] = {nx, ny, nz, nt};
  for (long e : ext)
    if (e < 2 || (e & 1) || e > INT_MAX) return false;
  // Each factor is below 2^31, so the products are checked step by step
  // against the bound before they can leave the 64-bit range.
  const long lim = INT_MAX / (NTF * (long)ncol * ncol);
  long V = 1;
  for (long e : ext) {
    if (V > lim / e) return false;
    V *= e;
  }
  const long S = (V + 31) / 32 * 32;
  if ((long)NTF * ncol * ncol * S > INT_MAX) return false;
  g->nx = (int)nx;
  g->ny = (int)ny;
  g->nz = (int)nz;
  g->nt = (int)nt;
  g->V = (int)V;
  g->S = (int)S;
  g->pbc = pbc;
  return true;
}

bool ck(susy_b200_lattice* h, cudaError_t e) {
  if (e == cudaSuccess) return true;
  if (h && h->err == 0) h->err = SUSY_B200_ECUDA;
  if (h) h->cuda_err = (int)e;
  return false;
}

int set_err(susy_b200_lattice* h, int code) {
  if (h && h->err == 0) h->err = code;
  return code;
}

void* dalloc(susy_b200_lattice* h, size_t bytes) {
  void* p = nullptr;
  if (cudaMalloc(&p, bytes) != cudaSuccess) {
    cudaGetLastError();
    set_err(h, SUSY_B200_ENOMEM);
    return nullptr;
  }
  cudaMemsetAsync(p, 0, bytes, h->stream);
  return p;
}

size_t field_bytes(const susy_b200_lattice* h, int K, int prec) {
  return (size_t)K * mat_c(h) * h->g.S * (prec == 64 ? sizeof(double2) : sizeof(float2));
}

// Host link-type array (strided) -> device SoA FP64 field of K matrices
int upload_links(susy_b200_lattice* h, void* dev, const double* host, size_t stride, int K) {
  const size_t row = (size_t)K * mat_c(h) * 2 * sizeof(double);
  if (stride == 0) stride = row;
  if (!ck(h, cudaMemcpy2DAsync(h->stage, row, host, stride, row, h->g.V,
                               cudaMemcpyHostToDevice, h->stream)))
    return SUSY_B200_ECUDA;
  aos_to_soa(h->g, K, h->N, h->stage, dev, 64, h->stream);
  return ck(h, cudaGetLastError()) ? SUSY_B200_OK : SUSY_B200_ECUDA;
}

int download_links(susy_b200_lattice* h, const void* dev, double* host, size_t stride, int K) {
  const size_t row = (size_t)K * mat_c(h) * 2 * sizeof(double);
  if (stride == 0) stride = row;
  soa_to_aos(h->g, K, h->N, dev, h->stage, 64, h->stream);
  if (!ck(h, cudaMemcpy2DAsync(host, stride, h->stage, row, row, h->g.V,
                               cudaMemcpyDeviceToHost, h->stream)))
    return SUSY_B200_ECUDA;
  return ck(h, cudaStreamSynchronize(h->stream)) ? SUSY_B200_OK : SUSY_B200_ECUDA;
}

int refresh_derived(susy_b200_lattice* h) {
  compute_uinv(h->g, h->N, h->U, h->det, h->Uinv, h->stream);
  compute_plaqdet(h->g, h->det, h->pd, h->zw, h->stream);
  compute_dmuumu(h->g, h->N, h->U, h->pd, h->G, h->D, h->stream);
  compute_fmunu(h->g, h->N, h->U, h->F, h->stream);
  refresh_low(h);
  return ck(h, cudaGetLastError()) ? SUSY_B200_OK : SUSY_B200_ECUDA;
}

// FP32 copies of the operator's inputs
void refresh_low(susy_b200_lattice* h) {
  const long nm = 5L * mat_c(h) * h->g.S;
  convert_field(nm, h->U, 64, h->U32, 32, h->stream);
  convert_field(nm, h->Uinv, 64, h->Uinv32, 32, h->stream);
  convert_field(25L * h->g.S, h->pd, 64, h->pd32, 32, h->stream);
}

// With the RESCALE option only the table-driven kernels (variants from
// FOP_COMPACT on) apply the factor; a variant below them is replaced by
// FOP_SITE_MAJOR_OCC.
static int launch_variant(susy_b200_lattice* h, const void* src, void* dst, int sign, int prec,
                          const void* add, double addc, double* dot, const int* skip, int v) {
  const double es = h->rescale ? 2.0 : 1.0;
  if (h->rescale && v < FOP_COMPACT) v = FOP_SITE_MAJOR_OCC;
  if (prec == 64)
    return fermion_op<double>(h->g, h->N, h->U, h->Uinv, h->pd, src, dst, sign, h->G, add, addc,
                              dot, skip, v, h->nbrtab, h->stream, es, h->trace[0]);
  return fermion_op<float>(h->g, h->N, h->U32, h->Uinv32, h->pd32, src, dst, sign, h->G, add,
                           addc, dot, skip, v, h->nbrtab, h->stream, es, h->trace[1]);
}

// Project-written autotuner: time one D^dag D with every kernel variant on
// this lattice and keep the fastest for this precision.  Runs on the first
// operator call of each precision (before any stream capture).
static_assert(FOP_NVARIANTS == SUSY_B200_FOP_NVARIANTS, "variant count");

int autotune_fop(susy_b200_lattice* h, int prec) {
  const int pi = prec == 64 ? 0 : 1;
  void* a = scratch_tf(h, 6, prec);
  void* b = scratch_tf(h, 7, prec);
  if (!a || !b) return SUSY_B200_ENOMEM;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  int bestv = h->rescale ? FOP_SITE_MAJOR_OCC : FOP_MAT;
  for (int v = h->rescale ? FOP_COMPACT : 0; v < FOP_NVARIANTS; v++) {
    launch_variant(h, a, b, 1, prec, nullptr, 0.0, nullptr, nullptr, v);
    cudaEventRecord(e0, h->stream);
    for (int r = 0; r < 3; r++) {
      launch_variant(h, a, b, 1, prec, nullptr, 0.0, nullptr, nullptr, v);
      launch_variant(h, b, a, -1, prec, nullptr, 0.0, nullptr, nullptr, v);
    }
    cudaEventRecord(e1, h->stream);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    h->fop_ms[pi][v] = ms / 3.f;
    if (ms < best) {
      best = ms;
      bestv = v;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  h->fop_variant[pi] = bestv;
  return ck(h, cudaGetLastError()) ? SUSY_B200_OK : SUSY_B200_ECUDA;
}

int dev_fop(susy_b200_lattice* h, const void* src, void* dst, int sign, int prec,
            const void* add, double addc, double* dot, const int* skip) {
  const int pi = prec == 64 ? 0 : 1;
  if (h->fop_variant[pi] < 0) autotune_fop(h, prec);
  return launch_variant(h, src, dst, sign, prec, add, addc, dot, skip, h->fop_variant[pi]);
}

void* scratch_tf(susy_b200_lattice* h, int which, int prec) {
  void** slot = prec == 64 ? &h->tf64[which] : &h->tf32[which];
  if (!*slot) *slot = dalloc(h, field_bytes(h, NTF, prec));
  return *slot;
}

double* partials(susy_b200_lattice* h, int which) {
  if (!h->part[which]) {
    const long n = (long)NTF * mat_c(h) * h->g.S;
    size_t np = std::max((size_t)fop_partials(h->g), (size_t)vec_blocks(n)) + 64;
    h->part[which] = (double*)dalloc(h, np * sizeof(double));
  }
  return h->part[which];
}

long tf_complex(const susy_b200_lattice* h) { return (long)NTF * mat_c(h) * h->g.S; }

// Stream and event of the host congrad_multi's early solution copies
cudaStream_t copy_stream(susy_b200_lattice* h) {
  if (!h->copy) {
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    if (cudaEventCreateWithFlags(&h->copy_ev, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      h->copy_ev = nullptr;
      cudaStreamDestroy(st);
      return nullptr;
    }
    h->copy = st;
  }
  return h->copy;
}

// The handle's second solver context, made on first use: its own stream,
// multi-shift state and scratch fields (allocated as its solves need them);
// the links, their derived fields in both precisions and the neighbour
// table are the handle's, which the solvers only read.  The settings the
// solvers read are copied from the handle at every call.
susy_b200_lattice* solver_shadow(susy_b200_lattice* h) {
  if (!h->shadow) {
    susy_b200_lattice* c = new susy_b200_lattice();
    c->prm = h->prm;
    c->g = h->g;
    c->N = h->N;
    c->shares_fields = true;
    if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      delete c;
      return nullptr;
    }
    c->stream = c->own_stream;
    c->ms = (MsState*)dalloc(c, sizeof(MsState));
    c->trace[0] = dalloc(c, 5 * c->g.S * sizeof(double2));
    c->trace[1] = dalloc(c, 5 * c->g.S * sizeof(float2));
    if (!c->ms || !c->trace[0] || !c->trace[1]) {
      susy_b200_destroy(c);
      return nullptr;
    }
    h->shadow = c;
  }
  susy_b200_lattice* c = h->shadow;
  c->U = h->U;
  c->Uinv = h->Uinv;
  c->pd = h->pd;
  c->U32 = h->U32;
  c->Uinv32 = h->Uinv32;
  c->pd32 = h->pd32;
  c->nbrtab = h->nbrtab;
  c->prm = h->prm;
  c->G = h->G;
  c->ms_blocked = h->ms_blocked;
  c->use_graphs = h->use_graphs;
  c->mix_switch = h->mix_switch;
  c->mix_reliable = h->mix_reliable;
  c->mix_interval = h->mix_interval;
  c->mix_correct32 = h->mix_correct32;
  c->mix_vec32 = h->mix_vec32;
  c->rescale = h->rescale;
  for (int pi = 0; pi < 2; pi++) {
    c->fop_variant[pi] = h->fop_variant[pi];
    for (int v = 0; v < SUSY_B200_FOP_NVARIANTS; v++) c->fop_ms[pi][v] = h->fop_ms[pi][v];
  }
  c->err = 0;
  return c;
}

}  // namespace susy

// ===========================================================================
extern "C" {

susy_b200_lattice* susy_b200_create(const susy_b200_params* p) {
  Geo geo;
  if (!p || !make_geo(p->nx, p->ny, p->nz, p->nt, p->ncol, p->pbc, &geo)) return nullptr;
  if (cudaSetDevice(p->device) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  susy_b200_lattice* h = new susy_b200_lattice();
  h->prm = *p;
  h->N = p->ncol;
  h->G = p->G;
  h->g = geo;
  if (cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    delete h;
    return nullptr;
  }
  h->stream = h->own_stream;
  if (upload_fop_terms(p->device, h->stream) != 0) {
    cudaGetLastError();
    cudaStreamDestroy(h->own_stream);
    delete h;
    return nullptr;
  }
  const size_t m5 = field_bytes(h, 5, 64);
  h->U = dalloc(h, m5);
  h->mom = dalloc(h, m5);
  h->Uinv = dalloc(h, m5);
  h->force = dalloc(h, m5);
  h->det = dalloc(h, 5 * h->g.S * sizeof(double2));
  h->pd = dalloc(h, 25 * h->g.S * sizeof(double2));
  h->zw = dalloc(h, 25 * h->g.S * sizeof(double2));
  h->D = dalloc(h, field_bytes(h, 1, 64));
  h->F = dalloc(h, field_bytes(h, 10, 64));
  h->U32 = dalloc(h, field_bytes(h, 5, 32));
  h->Uinv32 = dalloc(h, field_bytes(h, 5, 32));
  h->pd32 = dalloc(h, 25 * h->g.S * sizeof(float2));
  h->stage = dalloc(h, (size_t)h->g.V * NTF * mat_c(h) * 2 * sizeof(double));
  h->ms = (MsState*)dalloc(h, sizeof(MsState));
  h->nbrtab = (int*)dalloc(h, (size_t)fop_ndisp() * h->g.S * sizeof(int));
  h->trace[0] = dalloc(h, 5 * h->g.S * sizeof(double2));
  h->trace[1] = dalloc(h, 5 * h->g.S * sizeof(float2));
  if (h->nbrtab) build_nbr_table(h->g, h->nbrtab, h->stream);
  if (h->err) {
    susy_b200_destroy(h);
    return nullptr;
  }
  node_prn_init(h->node_prn, p->iseed, h->g.V);
  // Unit links until the caller sets some (coldlat, io_helpers.c:95)
  std::vector<double> unit((size_t)h->g.V * 5 * mat_c(h) * 2, 0.0);
  for (int s = 0; s < h->g.V; s++)
    for (int a = 0; a < 5; a++)
      for (int i = 0; i < h->N; i++)
        unit[(((size_t)s * 5 + a) * mat_c(h) + i * h->N + i) * 2] = 1.0;
  susy_b200_set_links(h, unit.data(), 0);
  cudaStreamSynchronize(h->stream);
  if (h->err) {
    susy_b200_destroy(h);
    return nullptr;
  }
  return h;
}

void susy_b200_destroy(susy_b200_lattice* h) {
  if (!h) return;
  cudaStreamSynchronize(h->stream);
  if (h->shadow) susy_b200_destroy(h->shadow);
  if (h->shares_fields)  // a solver context: these belong to its handle
    h->U = h->Uinv = h->pd = h->U32 = h->Uinv32 = h->pd32 = nullptr, h->nbrtab = nullptr;
  void* ptrs[] = {h->U, h->mom, h->Uinv, h->force, h->det, h->pd, h->zw, h->D, h->F,
                  h->U32, h->Uinv32, h->pd32, h->stage, h->ms, h->bigpart, h->gen, h->prn,
                  h->rng_bad, h->ptrbuf, h->nbrtab, h->meas, h->trace[0], h->trace[1]};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (int i = 0; i < SUSY_NSCRATCH; i++) {
    if (h->tf64[i]) cudaFree(h->tf64[i]);
    if (h->tf32[i]) cudaFree(h->tf32[i]);
  }
  for (int i = 0; i < SUSY_NPART; i++)
    if (h->part[i]) cudaFree(h->part[i]);
  for (std::vector<void*>* v : {&h->extra, &h->sols, &h->pvec64, &h->pvec32, &h->ring, &h->vec32, &h->gsrc,
                                &h->gr_psim, &h->traj_psim, &h->extra5, &h->refine})
    for (void* p : *v)
      if (p) cudaFree(p);
  if (h->poll) cudaFreeHost(h->poll);
  if (h->copy) cudaStreamSynchronize(h->copy), cudaStreamDestroy(h->copy);
  if (h->copy_ev) cudaEventDestroy(h->copy_ev);
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
  delete h;
}

long long susy_b200_launch_count(void) { return g_launches.load(); }

int susy_b200_measure(susy_b200_lattice* h, susy_b200_meas* m) {
  if (!h || !m) return SUSY_B200_EINVAL;
  return measure(h, m);
}

int susy_b200_plaquette(susy_b200_lattice* h, double* ss_plaq, double* st_plaq) {
  if (!h || !ss_plaq || !st_plaq) return SUSY_B200_EINVAL;
  susy_b200_meas m;
  const int rc = measure(h, &m);
  if (rc) return rc;
  *ss_plaq = m.ss_plaq;
  *st_plaq = m.st_plaq;
  return SUSY_B200_OK;
}

int susy_b200_mixed_params(susy_b200_lattice* h, double fp32_below, double reliable_factor) {
  if (!h || !(fp32_below > 0.0 && fp32_below <= 1.0) ||
      !(reliable_factor > 0.0 && reliable_factor < 1.0))
    return SUSY_B200_EINVAL;
  h->mix_switch = fp32_below;
  h->mix_reliable = reliable_factor;
  return SUSY_B200_OK;
}

int susy_b200_mixed_reliable_interval(susy_b200_lattice* h, int iters) {
  if (!h || iters < 0) return SUSY_B200_EINVAL;
  h->mix_interval = iters;
  return SUSY_B200_OK;
}

int susy_b200_mixed_correction(susy_b200_lattice* h, int fp32) {
  if (!h || (fp32 != 0 && fp32 != 1)) return SUSY_B200_EINVAL;
  h->mix_correct32 = fp32;
  return SUSY_B200_OK;
}

int susy_b200_set_rescale(susy_b200_lattice* h, int on) {
  if (!h || on > 1) return SUSY_B200_EINVAL;
  const int prev = h->rescale;
  if (on >= 0) {
    h->rescale = on;
    if (h->shadow) h->shadow->rescale = on;
  }
  return prev;
}

int susy_b200_mixed_vectors(susy_b200_lattice* h, int fp32) {
  if (!h || fp32 > 1) return SUSY_B200_EINVAL;
  const int prev = h->mix_vec32;
  if (fp32 >= 0) {
    h->mix_vec32 = fp32;
    if (h->shadow) h->shadow->mix_vec32 = fp32;
  }
  return prev;
}

int susy_b200_dev_congrad_multi_learned(susy_b200_lattice* h, susy_b200_net* net,
                                        const void* src, void* const* psim, int norder,
                                        const double* shift, int MaxCG, double errormin,
                                        int nrefine, double loose, double* size_r, int* iters,
                                        int* refine_iters) {
  if (!h || !src || !psim || !shift || norder < 1 || norder > MS_MAXS || nrefine < 0 ||
      !(loose > 0.0))
    return set_err(h, SUSY_B200_EINVAL);
  return multishift_learned(h, net, src, psim, norder, shift, MaxCG, errormin, nrefine,
                            loose < errormin ? errormin : loose, size_r, iters, refine_iters);
}

int susy_b200_set_solver(susy_b200_lattice* h, int solver) {
  if (!h || (solver != SUSY_B200_SOLVER_FP64 && solver != SUSY_B200_SOLVER_MIXED))
    return SUSY_B200_EINVAL;
  const int prev = h->host_solver;
  h->host_solver = solver;
  return prev;
}

int susy_b200_use_graphs(susy_b200_lattice* h, int on) {
  if (!h) return SUSY_B200_EINVAL;
  const int prev = h->use_graphs;
  if (on >= 0) h->use_graphs = on ? 1 : 0;
  return prev;
}

int susy_b200_pf_streams(susy_b200_lattice* h, int on) {
  if (!h) return SUSY_B200_EINVAL;
  const int prev = h->pf_streams;
  if (on >= 0) h->pf_streams = on ? 1 : 0;
  return prev;
}

int susy_b200_cg_blocked(susy_b200_lattice* h, int on) {
  if (!h) return SUSY_B200_EINVAL;
  const int prev = h->ms_blocked;
  if (on >= 0) h->ms_blocked = on ? 1 : 0;
  return prev;
}

int susy_b200_cg_freeze_iterations(susy_b200_lattice* h, int* iters, int norder) {
  if (!h || !iters || norder < 1 || norder > MS_MAXS) return SUSY_B200_EINVAL;
  std::vector<int> c(norder, 0), n(1, 0);
  if (!ck(h, cudaMemcpyAsync(c.data(), h->ms->converged, norder * sizeof(int),
                             cudaMemcpyDeviceToHost, h->stream)) ||
      !ck(h, cudaMemcpyAsync(n.data(), &h->ms->iter, sizeof(int), cudaMemcpyDeviceToHost,
                             h->stream)) ||
      !ck(h, cudaStreamSynchronize(h->stream)))
    return SUSY_B200_ECUDA;
  for (int j = 0; j < norder; j++) iters[j] = j == 0 || c[j] == 0 ? n[0] : c[j];
  return SUSY_B200_OK;
}

int susy_b200_last_error(const susy_b200_lattice* h) { return h ? h->err : SUSY_B200_EINVAL; }

const char* susy_b200_error_string(int code) {
  switch (code) {
    case SUSY_B200_OK: return "ok";
    case SUSY_B200_EINVAL: return "invalid argument";
    case SUSY_B200_ECUDA: return "CUDA runtime error";
    case SUSY_B200_ENOMEM: return "device allocation failed";
    case SUSY_B200_ENOCONV: return "solver did not converge";
    case SUSY_B200_ENAN: return "non-finite value";
    case SUSY_B200_ESCRATCH: return "field exceeds the 16 MiB scratch of susy_b200_DSq_noalloc";
    default: return "unknown error";
  }
}

int susy_b200_set_stream(susy_b200_lattice* h, void* s) {
  if (!h) return SUSY_B200_EINVAL;
  h->stream = s ? (cudaStream_t)s : h->own_stream;
  return SUSY_B200_OK;
}

void* susy_b200_get_stream(const susy_b200_lattice* h) { return h ? (void*)h->stream : nullptr; }

int susy_b200_sync(susy_b200_lattice* h) {
  if (!h) return SUSY_B200_EINVAL;
  return ck(h, cudaStreamSynchronize(h->stream)) ? SUSY_B200_OK : SUSY_B200_ECUDA;
}

int susy_b200_volume(const susy_b200_lattice* h) { return h ? h->g.V : 0; }

int susy_b200_set_links(susy_b200_lattice* h, const double* links, size_t stride) {
  if (!h || !links) return set_err(h, SUSY_B200_EINVAL);
  int r = upload_links(h, h->U, links, stride, 5);
  if (r) return r;
  return refresh_derived(h);
}

int susy_b200_get_links(susy_b200_lattice* h, double* links, size_t stride) {
  if (!h || !links) return set_err(h, SUSY_B200_EINVAL);
  return download_links(h, h->U, links, stride, 5);
}

int susy_b200_set_mom(susy_b200_lattice* h, const double* mom, size_t stride) {
  if (!h || !mom) return set_err(h, SUSY_B200_EINVAL);
  return upload_links(h, h->mom, mom, stride, 5);
}

int susy_b200_get_mom(susy_b200_lattice* h, double* mom, size_t stride) {
  if (!h || !mom) return set_err(h, SUSY_B200_EINVAL);
  return download_links(h, h->mom, mom, stride, 5);
}

int susy_b200_compute_plaqdet(susy_b200_lattice* h) {
  if (!h) return SUSY_B200_EINVAL;
  compute_uinv(h->g, h->N, h->U, h->det, h->Uinv, h->stream);
  compute_plaqdet(h->g, h->det, h->pd, h->zw, h->stream);
  refresh_low(h);
  return ck(h, cudaGetLastError()) ? SUSY_B200_OK : SUSY_B200_ECUDA;
}

int susy_b200_compute_Uinv(susy_b200_lattice* h) {
  if (!h) return SUSY_B200_EINVAL;
  compute_uinv(h->g, h->N, h->U, h->det, h->Uinv, h->stream);
  refresh_low(h);
  return ck(h, cudaGetLastError()) ? SUSY_B200_OK : SUSY_B200_ECUDA;
}

int susy_b200_compute_DmuUmu(susy_b200_lattice* h) {
  if (!h) return SUSY_B200_EINVAL;
  compute_dmuumu(h->g, h->N, h->U, h->pd, h->G, h->D, h->stream);
  return ck(h, cudaGetLastError()) ? SUSY_B200_OK : SUSY_B200_ECUDA;
}

int susy_b200_compute_Fmunu(susy_b200_lattice* h) {
  if (!h) return SUSY_B200_EINVAL;
  compute_fmunu(h->g, h->N, h->U, h->F, h->stream);
  return ck(h, cudaGetLastError()) ? SUSY_B200_OK : SUSY_B200_ECUDA;
}

int susy_b200_get_derived(susy_b200_lattice* h, double* plaqdet, double* DmuUmu, double* Fmunu,
                          double* Uinv) {
  if (!h) return SUSY_B200_EINVAL;
  int r = 0;
  if (plaqdet) {
    // pd is 25 complex per site: a "field" of 25 1x1 matrices
    Geo g = h->g;
    std::vector<double> tmp((size_t)g.V * 25 * 2);
    // reuse the generic converter with N = 1, K = 25
    soa_to_aos(g, 25, 1, h->pd, h->stage, 64, h->stream);
    if (!ck(h, cudaMemcpyAsync(plaqdet, h->stage, tmp.size() * sizeof(double),
                               cudaMemcpyDeviceToHost, h->stream)))
      return SUSY_B200_ECUDA;
  }
  if (DmuUmu && (r = download_links(h, h->D, DmuUmu, 0, 1))) return r;
  if (Fmunu && (r = download_links(h, h->F, Fmunu, 0, 10))) return r;
  if (Uinv && (r = download_links(h, h->Uinv, Uinv, 0, 5))) return r;
  return ck(h, cudaStreamSynchronize(h->stream)) ? SUSY_B200_OK : SUSY_B200_ECUDA;
}

// ---- device-resident Twist_Fermion fields ---------------------------------
size_t susy_b200_tf_bytes(const susy_b200_lattice* h, int prec) {
  return h ? field_bytes(h, NTF, prec) : 0;
}

void* susy_b200_tf_alloc(susy_b200_lattice* h, int prec) {
  if (!h || (prec != 64 && prec != 32)) return nullptr;
  return dalloc(h, field_bytes(h, NTF, prec));
}

void susy_b200_tf_free(susy_b200_lattice* h, void* dev) {
  if (h && dev) {
    cudaStreamSynchronize(h->stream);
    cudaFree(dev);
  }
}

int susy_b200_tf_upload(susy_b200_lattice* h, void* dev, int prec, const double* host) {
  if (!h || !dev || !host) return set_err(h, SUSY_B200_EINVAL);
  const size_t bytes = (size_t)h->g.V * NTF * mat_c(h) * 2 * sizeof(double);
  if (!ck(h, cudaMemcpyAsync(h->stage, host, bytes, cudaMemcpyHostToDevice, h->stream)))
    return SUSY_B200_ECUDA;
  aos_to_soa(h->g, NTF, h->N, h->stage, dev, prec, h->stream);
  return ck(h, cudaGetLastError()) ? SUSY_B200_OK : SUSY_B200_ECUDA;
}

int susy_b200_tf_download(susy_b200_lattice* h, const void* dev, int prec, double* host) {
  if (!h || !dev || !host) return set_err(h, SUSY_B200_EINVAL);
  const size_t bytes = (size_t)h->g.V * NTF * mat_c(h) * 2 * sizeof(double);
  soa_to_aos(h->g, NTF, h->N, dev, h->stage, prec, h->stream);
  if (!ck(h, cudaMemcpyAsync(host, h->stage, bytes, cudaMemcpyDeviceToHost, h->stream)))
    return SUSY_B200_ECUDA;
  return ck(h, cudaStreamSynchronize(h->stream)) ? SUSY_B200_OK : SUSY_B200_ECUDA;
}

int susy_b200_tf_convert(susy_b200_lattice* h, const void* src, int ps, void* dst, int pd) {
  if (!h || !src || !dst) return set_err(h, SUSY_B200_EINVAL);
  convert_field(tf_complex(h), src, ps, dst, pd, h->stream);
  return ck(h, cudaGetLastError()) ? SUSY_B200_OK : SUSY_B200_ECUDA;
}

int susy_b200_dev_fermion_op(susy_b200_lattice* h, const void* src, void* dst, int sign,
                             int prec) {
  if (!h || !src || !dst) return set_err(h, SUSY_B200_EINVAL);
  if (sign != 1 && sign != -1) return set_err(h, SUSY_B200_EINVAL);
  if (prec != 64 && prec != 32) return set_err(h, SUSY_B200_EINVAL);
  dev_fop(h, src, dst, sign, prec, nullptr, 0.0, nullptr, nullptr);
  return ck(h, cudaGetLastError()) ? SUSY_B200_OK : SUSY_B200_ECUDA;
}

int susy_b200_autotune(susy_b200_lattice* h) {
  if (!h) return SUSY_B200_EINVAL;
  int r = autotune_fop(h, 64);
  return r ? r : autotune_fop(h, 32);
}

int susy_b200_fop_variant(susy_b200_lattice* h, int prec, int set_to, float* ms_per_variant) {
  if (!h || (prec != 64 && prec != 32) || set_to >= FOP_NVARIANTS) return SUSY_B200_EINVAL;
  const int pi = prec == 64 ? 0 : 1;
  if (set_to >= 0) h->fop_variant[pi] = set_to;
  if (ms_per_variant)
    for (int v = 0; v < FOP_NVARIANTS; v++) ms_per_variant[v] = h->fop_ms[pi][v];
  return h->fop_variant[pi];
}

int susy_b200_dev_DSq(susy_b200_lattice* h, const void* src, void* dst, int prec) {
  if (!h || !src || !dst) return set_err(h, SUSY_B200_EINVAL);
  if (prec != 64 && prec != 32) return set_err(h, SUSY_B200_EINVAL);
  void* tmp = scratch_tf(h, 0, prec);
  if (!tmp) return SUSY_B200_ENOMEM;
  const double fm2 = h->prm.fmass > 1e-8 ? h->prm.fmass * h->prm.fmass : 0.0;
  dev_fop(h, src, tmp, 1, prec, nullptr, 0.0, nullptr, nullptr);
  dev_fop(h, tmp, dst, -1, prec, fm2 != 0.0 ? src : nullptr, fm2, nullptr, nullptr);
  return ck(h, cudaGetLastError()) ? SUSY_B200_OK : SUSY_B200_ECUDA;
}

int susy_b200_fermion_op(susy_b200_lattice* h, const double* src, double* dest, int sign) {
  if (!h || !src || !dest) return set_err(h, SUSY_B200_EINVAL);
  if (sign != 1 && sign != -1) return set_err(h, SUSY_B200_EINVAL);
  void* a = scratch_tf(h, 1, 64);
  void* b = scratch_tf(h, 2, 64);
  if (!a || !b) return SUSY_B200_ENOMEM;
  int r = susy_b200_tf_upload(h, a, 64, src);
  if (r) return r;
  if ((r = susy_b200_dev_fermion_op(h, a, b, sign, 64))) return r;
  return susy_b200_tf_download(h, b, 64, dest);
}

int susy_b200_DSq(susy_b200_lattice* h, const double* src, double* dest) {
  if (!h || !src || !dest) return set_err(h, SUSY_B200_EINVAL);
  void* a = scratch_tf(h, 1, 64);
  void* b = scratch_tf(h, 2, 64);
  if (!a || !b) return SUSY_B200_ENOMEM;
  int r = susy_b200_tf_upload(h, a, 64, src);
  if (r) return r;
  if ((r = susy_b200_dev_DSq(h, a, b, 64))) return r;
  return susy_b200_tf_download(h, b, 64, dest);
}

int susy_b200_dev_congrad_multi(susy_b200_lattice* h, const void* src, void* const* psim,
                                int norder, const double* shift, int MaxCG, double errormin,
                                double* size_r, int* iters) {
  if (!h || !src || !psim || !shift || norder < 1 || norder > MS_MAXS)
    return set_err(h, SUSY_B200_EINVAL);
  return multishift_fp64(h, src, psim, norder, shift, MaxCG, errormin, size_r, iters);
}

int susy_b200_dev_congrad_multi_mixed(susy_b200_lattice* h, const void* src, void* const* psim,
                                      int norder, const double* shift, int MaxCG,
                                      double errormin, double* size_r, int* iters) {
  if (!h || !src || !psim || !shift || norder < 1 || norder > MS_MAXS)
    return set_err(h, SUSY_B200_EINVAL);
  return multishift_mixed(h, src, psim, norder, shift, MaxCG, errormin, size_r, iters);
}

int susy_b200_congrad_multi(susy_b200_lattice* h, const double* src, double* const* psim,
                            int norder, const double* shift, int MaxCG, double errormin,
                            double* size_r) {
  if (!h || !src || !psim || !shift || norder < 1 || norder > MS_MAXS)
    return set_err(h, SUSY_B200_EINVAL);
  void* s = scratch_tf(h, 1, 64);
  if (!s) return SUSY_B200_ENOMEM;
  int r = susy_b200_tf_upload(h, s, 64, src);
  if (r) return r;
  std::vector<void*> ps(norder);
  for (int j = 0; j < norder; j++) {
    ps[j] = sol_field(h, j);
    if (!ps[j]) return SUSY_B200_ENOMEM;
  }
  // When every psim[j] is page-locked host memory, a shift's solution goes
  // back (layout change into the staging buffer, then the copy) on a second
  // stream as soon as the shift has frozen, while the solve continues; the
  // rest, and any the mixed solver corrected afterwards, follow the solve.
  // Pageable buffers would make the copies block the host, so they wait.
  bool early = copy_stream(h) != nullptr;
  for (int j = 0; j < norder && early; j++) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, psim[j]) != cudaSuccess || a.type != cudaMemoryTypeHost) {
      cudaGetLastError();
      early = false;
    }
  }
  const size_t bytes = (size_t)h->g.V * NTF * mat_c(h) * 2 * sizeof(double);
  std::vector<char> sent(norder, 0), redo(norder, 0);
  FrozenHook hook = [&](int j) {
    cudaEventRecord(h->copy_ev, h->stream);
    cudaStreamWaitEvent(h->copy, h->copy_ev, 0);
    soa_to_aos(h->g, NTF, h->N, ps[j], h->stage, 64, h->copy);
    cudaMemcpyAsync(psim[j], h->stage, bytes, cudaMemcpyDeviceToHost, h->copy);
    sent[j] = 1;
  };
  int it = 0;
  double sr = 0.0;
  r = h->host_solver == SUSY_B200_SOLVER_MIXED
          ? multishift_mixed(h, s, ps.data(), norder, shift, MaxCG, errormin, &sr, &it,
                             early ? &hook : nullptr, redo.data())
          : multishift_fp64(h, s, ps.data(), norder, shift, MaxCG, errormin, &sr, &it,
                            early ? &hook : nullptr);
  // the early copies finish before the staging buffer is used again
  if (early && !ck(h, cudaStreamSynchronize(h->copy))) return SUSY_B200_ECUDA;
  if (r) return r;
  for (int j = 0; j < norder; j++)
    if (!sent[j] || redo[j])
      if ((r = susy_b200_tf_download(h, ps[j], 64, psim[j]))) return r;
  if (size_r) *size_r = sr;
  return it;
}

}  // extern "C"
