// lcs_api.cu -- the extern "C" entry points of include/lcs_b200.h.
// Each call validates its arguments, forwards to the handle's engine, and
// turns every failure into a status code plus a message (no exceptions or
// aborts cross the ABI).
#include <vector>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>

#include <cuda_runtime.h>

#include "lcs_base.h"

namespace lcs {
EngineBase* make_engine_f64(const lcs_config& c, std::string* err, int* rc);
int64_t footprint_f64(const lcs_config& c);
EngineBase* make_engine_f32(const lcs_config& c, std::string* err, int* rc);
int64_t footprint_f32(const lcs_config& c);
}  // namespace lcs

struct lcs_handle {
  lcs::EngineBase* e;
};

static thread_local char g_err[512];

static int set_global_error(int code, const char* msg) {
  snprintf(g_err, sizeof g_err, "%s", msg);
  return code;
}

namespace lcs {
// Error text of the handle-less entry points, read by lcs_last_error(NULL).
void set_global_error_message(const char* msg) { snprintf(g_err, sizeof g_err, "%s", msg); }
}  // namespace lcs

// Config checks shared by lcs_create and lcs_footprint (the reference's
// constructors throw ArgumentError for the same cases).
static int validate(const lcs_config* c, std::string* why) {
  if (!c) { *why = "null config"; return LCS_EINVAL; }
  if (c->abi_version != LCS_ABI_VERSION) { *why = "abi_version mismatch"; return LCS_EINVAL; }
  if (c->mode != LCS_MODE_FLOW && c->mode != LCS_MODE_FLOW_PARTICLE) { *why = "bad mode"; return LCS_EINVAL; }
  for (int a = 0; a < 3; a++)
    if (c->dims[a] < 4 || c->dims[a] % 2) { *why = "grid dims must be even and >= 4 (periodic red-black sweeps)"; return LCS_EINVAL; }
  if (c->halo_size < 3) { *why = "halo_size must be >= 3 (4th-order stencils, time-blocked HSMAC)"; return LCS_EINVAL; }
  if (c->coloring == LCS_COLORING_NO) {
    *why = "coloring 'no' updates shared faces concurrently on a GPU (nondeterministic in the reference too); use red-black-fast";
    return LCS_EINVAL;
  }
  if (c->coloring < 0 || c->coloring > LCS_COLORING_RED_BLACK_BLOCK) { *why = "bad coloring"; return LCS_EINVAL; }
  if (c->coloring == LCS_COLORING_RED_BLACK_BLOCK && c->coloring_block < 1) { *why = "red-black-block size must be >= 1"; return LCS_EINVAL; }
  if (!(c->omega > 0.0 && c->omega < 2.0)) { *why = "HSMAC omega must be in (0, 2)"; return LCS_EINVAL; }
  if (c->itrmax < 0 || c->itrmin < 0) { *why = "HSMAC itrmin/itrmax must be >= 0"; return LCS_EINVAL; }
  if (!(c->cfl > 0) || !(c->dtmax > 0)) { *why = "cfl and dtmax must be positive"; return LCS_EINVAL; }
  if (!(c->U0 > 0) || !(c->L0 > 0) || !(c->NU > 0)) { *why = "flow params must be positive"; return LCS_EINVAL; }
  if (c->forcing < LCS_FORCING_NO || c->forcing > LCS_FORCING_RC_ENERGY) { *why = "bad forcing kind"; return LCS_EINVAL; }
  if (c->forcing == LCS_FORCING_RC_ENERGY) {
    if (c->kmin < 1) { *why = "kmin must be at least 1"; return LCS_EINVAL; }
    if (c->kmax < c->kmin) { *why = "kmax must be at least kmin"; return LCS_EINVAL; }
    if (c->kmax > 4) { *why = "rc-energy supports kmax <= 4"; return LCS_EINVAL; }
    // fftindex into the coarse rfft stays in bounds only for kmax <= coarse_size/2 (FourierTools.jl:9)
    if (2 * c->kmax > c->coarse_size || c->dims[0] % c->coarse_size || c->dims[1] % c->coarse_size ||
        c->dims[2] % c->coarse_size) {
      *why = "rc-energy coarse_size must divide the grid dims and be >= 2*kmax";
      return LCS_EINVAL;
    }
  }
  if (c->n_species < 0 || c->n_species > LCS_MAX_SPECIES) { *why = "n_species out of range"; return LCS_EINVAL; }
  for (int s = 0; s < c->n_species; s++) {
    // Particles.timestep reduces `maximum` over the species' diameters, which
    // throws for an empty species in the reference (src/particles/timestep.jl:22)
    if (c->mode == LCS_MODE_FLOW_PARTICLE && c->species[s].nvalid < 1) {
      *why = "every particle species needs at least one particle";
      return LCS_EINVAL;
    }
    if (c->species[s].drag != LCS_DRAG_LINEAR && c->species[s].drag != LCS_DRAG_NONLINEAR) { *why = "bad drag kind"; return LCS_EINVAL; }
    if (!(c->species[s].density_ratio > 0)) { *why = "density_ratio must be positive"; return LCS_EINVAL; }
  }
  if (c->precision != LCS_PRECISION_FP64 && c->precision != LCS_PRECISION_FP32_MIXED) { *why = "bad precision"; return LCS_EINVAL; }
  return LCS_OK;
}

// FP64 FMA throughput: every thread runs 8 independent chains of fused
// multiply-adds (values stay bounded); the sums are stored so nothing is
// dropped.  2 flops per FMA.
__global__ void __launch_bounds__(512) k_fp64_peak(double* out, int iters, double a, double b) {
  double x[8];
#pragma unroll
  for (int q = 0; q < 8; q++) x[q] = 1e-3 * (threadIdx.x + q);
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int q = 0; q < 8; q++) x[q] = __fma_rn(x[q], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int q = 0; q < 8; q++) s += x[q];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

extern "C" {

int lcs_measure_fp64_peak(int32_t device, double* tflops) {
  if (!tflops) return set_global_error(LCS_EINVAL, "null output");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return set_global_error(LCS_EINVAL, "no such CUDA device");
  }
  cudaSetDevice(device);
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const int blocks = sms * 4, threads = 512, iters = 4096;
  double* out = nullptr;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaMalloc(&out, (size_t)blocks * threads * sizeof(double));
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  float best = 1e30f;
  for (int rep = 0; rep < 6 && e == cudaSuccess; rep++) {  // the first launch warms up
    cudaEventRecord(e0, st);
    k_fp64_peak<<<blocks, threads, 0, st>>>(out, iters, 0.9999999, 1e-7);
    cudaEventRecord(e1, st);
    e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaGetLastError();
    float ms = 0.f;
    if (e == cudaSuccess && rep > 0 && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess) best = ms < best ? ms : best;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (st) cudaStreamDestroy(st);
  cudaFree(out);
  if (e != cudaSuccess) return set_global_error(LCS_ECUDA, cudaGetErrorString(e));
  *tflops = 2.0 * 8.0 * iters * (double)blocks * threads / (best * 1e-3) / 1e12;
  return LCS_OK;
}

int lcs_footprint(const lcs_config* cfg, int64_t* bytes) {
  std::string why;
  int rc = validate(cfg, &why);
  if (rc) return set_global_error(rc, why.c_str());
  if (!bytes) return set_global_error(LCS_EINVAL, "null output");
  *bytes = cfg->precision == LCS_PRECISION_FP32_MIXED ? lcs::footprint_f32(*cfg) : lcs::footprint_f64(*cfg);
  return LCS_OK;
}

int lcs_create(const lcs_config* cfg, lcs_handle** out) {
  if (!out) return set_global_error(LCS_EINVAL, "null output handle");
  *out = nullptr;
  std::string why;
  int rc = validate(cfg, &why);
  if (rc) return set_global_error(rc, why.c_str());
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return set_global_error(LCS_ECUDA, "no CUDA device available for the B200 backend");
  }
  if (cfg->device < 0 || cfg->device >= ndev) return set_global_error(LCS_EINVAL, "device ordinal out of range");
  lcs::EngineBase* eng = cfg->precision == LCS_PRECISION_FP32_MIXED ? lcs::make_engine_f32(*cfg, &why, &rc)
                                                                     : lcs::make_engine_f64(*cfg, &why, &rc);
  if (!eng) return set_global_error(rc, why.c_str());
  lcs_handle* h = new (std::nothrow) lcs_handle;
  if (!h) {
    delete eng;
    return set_global_error(LCS_ENOMEM, "host allocation failed");
  }
  h->e = eng;
  *out = h;
  return LCS_OK;
}

void lcs_destroy(lcs_handle* h) {
  if (!h) return;
  delete h->e;
  delete h;
}

const char* lcs_last_error(const lcs_handle* h) { return h ? h->e->err.c_str() : g_err; }

int lcs_get_config(const lcs_handle* h, lcs_config* out) {
  if (!h || !out) return set_global_error(LCS_EINVAL, "null argument");
  *out = h->e->config();
  return LCS_OK;
}

#define H(h) \
  if (!(h)) return set_global_error(LCS_EINVAL, "null handle");

int lcs_upload_flow(lcs_handle* h, const double* U, const double* V, const double* W, const double* P) { H(h); return h->e->upload_flow(U, V, W, P); }
int lcs_download_flow(lcs_handle* h, double* U, double* V, double* W, double* P) { H(h); return h->e->download_flow(U, V, W, P); }
int lcs_field_set(lcs_handle* h, int32_t f, const double* d, int32_t haloed) { H(h); return h->e->field_set(f, d, haloed); }
int lcs_field_get(lcs_handle* h, int32_t f, double* d, int32_t haloed) { H(h); return h->e->field_get(f, d, haloed); }
int lcs_upload_particles(lcs_handle* h, int32_t s, int64_t n, const int64_t* ids, const double* diam, const double* x,
                         const double* y, const double* z, const double* u, const double* v, const double* w) {
  H(h);
  return h->e->upload_particles(s, n, ids, diam, x, y, z, u, v, w);
}
int lcs_download_particles(lcs_handle* h, int32_t s, int64_t* ids, double* diam, double* x, double* y, double* z,
                           double* u, double* v, double* w) {
  H(h);
  return h->e->download_particles(s, ids, diam, x, y, z, u, v, w);
}
int lcs_prop_set(lcs_handle* h, int32_t s, int32_t p, const double* d) { H(h); return h->e->prop_set(s, p, d); }
int lcs_prop_get(lcs_handle* h, int32_t s, int32_t p, double* d) { H(h); return h->e->prop_get(s, p, d); }
int lcs_set_state(lcs_handle* h, int64_t step, double t) { H(h); return h->e->set_state(step, t); }
int lcs_get_state(lcs_handle* h, int64_t* step, double* t) { H(h); return h->e->get_state(step, t); }
int lcs_timestep(lcs_handle* h, double* dt) { H(h); if (!dt) return LCS_EINVAL; return h->e->timestep(dt); }
int lcs_evolve(lcs_handle* h, double dt, lcs_log* log) { H(h); return h->e->evolve(dt, log); }
int lcs_step(lcs_handle* h, int32_t n, lcs_log* logs) { H(h); return h->e->step(n, logs); }
int lcs_step_timed(lcs_handle* h, int32_t n, lcs_log* logs, double* ms) { H(h); return h->e->step_timed(n, logs, ms); }
int lcs_step_begin(lcs_handle* h, int32_t n) { H(h); return h->e->step_begin(n); }
int lcs_step_poll(lcs_handle* h, int32_t* done) {
  H(h);
  int d = 0;
  const int rc = h->e->step_poll(&d);
  if (done) *done = d;
  return rc;
}
int lcs_step_finish(lcs_handle* h, lcs_log* logs) { H(h); return h->e->step_finish(logs); }
int lcs_flow_stat(lcs_handle* h, lcs_flow_stats* out) { H(h); return h->e->flow_stat(out); }
int lcs_set_particle_sort(lcs_handle* h, int32_t interval, int32_t ratio) {
  H(h);
  return h->e->set_particle_sort(interval, ratio);
}
int lcs_particles_makeindex(lcs_handle* h, int32_t s, int32_t stage, int32_t ratio) {
  H(h);
  return h->e->particles_makeindex(s, stage, ratio);
}
int lcs_particles_cellindex(lcs_handle* h, int32_t s, int64_t* hashes, int64_t* starts, int64_t* stops) {
  H(h);
  return h->e->particles_cellindex(s, hashes, starts, stops);
}
int lcs_particles_stat(lcs_handle* h, int32_t s, const lcs_particle_stat_config* pc, double tau_eta,
                       lcs_particle_stats* out) {
  H(h);
  return h->e->particles_stat(s, pc, tau_eta, out);
}
struct lcs_group {
  lcs::GroupBase* g;
};
int lcs_group_create(lcs_handle* const* members, int32_t m, lcs_group** out) {
  if (!out) return set_global_error(LCS_EINVAL, "null output");
  *out = nullptr;
  if (!members || m < 2) return set_global_error(LCS_EINVAL, "a group needs at least two handles");
  std::vector<lcs::EngineBase*> es;
  for (int32_t q = 0; q < m; q++) {
    if (!members[q]) return set_global_error(LCS_EINVAL, "null group member");
    es.push_back(members[q]->e);
  }
  lcs::GroupBase* g = nullptr;
  const int rc = es[0]->group_create(es.data(), m, &g);
  if (rc != LCS_OK) return set_global_error(rc, es[0]->err.c_str());
  *out = new lcs_group{g};
  return LCS_OK;
}
int lcs_group_step_begin(lcs_group* gr, int32_t nsteps) {
  if (!gr) return set_global_error(LCS_EINVAL, "null group");
  const int rc = gr->g->step_begin(nsteps);
  if (rc != LCS_OK) return set_global_error(rc, gr->g->err.c_str());
  return LCS_OK;
}
void lcs_group_destroy(lcs_group* gr) {
  if (!gr) return;
  delete gr->g;
  delete gr;
}
int lcs_flow_divergence(lcs_handle* h, double* rms, double* maxabs) {
  H(h);
  return h->e->flow_divergence(rms, maxabs);
}
int lcs_debug_unreachable_waits(lcs_handle* h, int32_t kind) {
  H(h);
  return h->e->debug_waits(kind);
}
int lcs_upload_flow_coarse(lcs_handle* h, const double* U, const double* V, const double* W, const double* P) {
  H(h);
  return h->e->upload_flow_coarse(U, V, W, P);
}
int lcs_particles_density(lcs_handle* h, int32_t s, int32_t ratio, double* densities) {
  H(h);
  return h->e->particles_density(s, ratio, densities);
}
int lcs_set_tuning(lcs_handle* h, int32_t rw_rows, int32_t zchunk, double share) {
  H(h);
  return h->e->set_tuning(rw_rows, zchunk, share);
}
int lcs_device_bytes(lcs_handle* h, int64_t* bytes) {
  H(h);
  if (!bytes) return LCS_EINVAL;
  *bytes = h->e->device_bytes();
  return LCS_OK;
}
int lcs_transfer_stats(lcs_handle* h, int64_t* a, int64_t* b) { H(h); return h->e->transfer_stats(a, b); }
int lcs_synchalo(lcs_handle* h, int32_t mask, int32_t r, int32_t full) { H(h); return h->e->synchalo(mask, r, full); }
int lcs_flow_rhs(lcs_handle* h, int32_t stage) { H(h); return h->e->rhs(stage); }
int lcs_flow_update(lcs_handle* h, int32_t stage, double dtrk) { H(h); return h->e->update(stage, dtrk); }
int lcs_flow_rhs_update(lcs_handle* h, int32_t stage, double dtrk) { H(h); return h->e->rhs_update(stage, dtrk); }
int lcs_flow_couple(lcs_handle* h, int32_t stage, double dtrk, lcs_couple_log* log) { H(h); return h->e->couple(stage, dtrk, log); }
int lcs_flow_forcing(lcs_handle* h, double dtrk, double* p, double* e10) { H(h); return h->e->forcing(dtrk, p, e10); }
int lcs_flow_timestep(lcs_handle* h, double* dt) { H(h); return h->e->flow_timestep(dt); }
int lcs_particles_timestep(lcs_handle* h, double* dt) { H(h); return h->e->particles_timestep(dt); }
int lcs_particles_boundary(lcs_handle* h, int32_t s, int32_t stage) { H(h); return h->e->particles_boundary(s, stage); }
int lcs_particles_motion(lcs_handle* h, int32_t s, int32_t stage) { H(h); return h->e->particles_motion(s, stage); }
int lcs_particles_update(lcs_handle* h, int32_t s, int32_t stage, double dtrk) { H(h); return h->e->particles_update(s, stage, dtrk); }
int lcs_init_particle_velocity(lcs_handle* h, int32_t s) { H(h); return h->e->init_particle_velocity(s); }
int lcs_profile_enable(lcs_handle* h, int32_t on) { H(h); return h->e->profile_enable(on); }
int lcs_profile_reset(lcs_handle* h) { H(h); return h->e->profile_reset(); }
int lcs_profile_count(lcs_handle* h, int32_t* n) { H(h); if (!n) return LCS_EINVAL; int v = 0; int rc = h->e->profile_count(&v); *n = v; return rc; }
int lcs_profile_entry(lcs_handle* h, int32_t i, char* name, int32_t cap, double* ms, int64_t* n) { H(h); return h->e->profile_entry(i, name, cap, ms, n); }
int lcs_launch_count(lcs_handle* h, int64_t* n) { H(h); if (!n) return LCS_EINVAL; return h->e->launch_count(n); }
int lcs_synchronize(lcs_handle* h) { H(h); return h->e->synchronize(); }

}  // extern "C"
