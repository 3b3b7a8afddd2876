// lcs_base.h -- the precision-independent engine interface behind the C ABI.
#pragma once

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/lcs_b200.h"

namespace lcs {

// A batch group (lcs_group_*): handles of one shape and launch shapes whose
// steps run as one CUDA graph with group-wide HSMAC launches.
struct GroupBase {
  std::string err;
  virtual ~GroupBase() {}
  virtual int step_begin(int nsteps) = 0;
  int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    err = buf;
    return code;
  }
};

struct EngineBase {
  std::string err;
  virtual ~EngineBase() {}
  virtual int upload_flow(const double* U, const double* V, const double* W, const double* P) = 0;
  virtual int download_flow(double* U, double* V, double* W, double* P) = 0;
  virtual int field_set(int f, const double* d, int haloed) = 0;
  virtual int field_get(int f, double* d, int haloed) = 0;
  virtual int upload_particles(int s, int64_t n, const int64_t* ids, const double* diam, const double* x,
                               const double* y, const double* z, const double* u, const double* v,
                               const double* w) = 0;
  virtual int download_particles(int s, int64_t* ids, double* diam, double* x, double* y, double* z, double* u,
                                 double* v, double* w) = 0;
  virtual int prop_set(int s, int prop, const double* d) = 0;
  virtual int prop_get(int s, int prop, double* d) = 0;
  virtual int set_state(int64_t step, double t) = 0;
  virtual int get_state(int64_t* step, double* t) = 0;
  virtual int timestep(double* dt) = 0;
  virtual int evolve(double dt, lcs_log* log) = 0;
  virtual int step(int nsteps, lcs_log* logs) = 0;
  virtual int step_timed(int nsteps, lcs_log* logs, double* ms) = 0;
  // asynchronous steps: enqueue, query without blocking, collect
  virtual int step_begin(int nsteps) = 0;
  virtual int step_poll(int* done) = 0;
  virtual int step_finish(lcs_log* logs) = 0;
  virtual int64_t device_bytes() const = 0;
  virtual int set_tuning(int rw_rows, int zchunk, double share) = 0;
  virtual int flow_stat(lcs_flow_stats* out) = 0;
  virtual int particles_makeindex(int s, int stage, int grid_ratio) = 0;
  virtual int set_particle_sort(int interval, int grid_ratio) = 0;
  virtual int particles_cellindex(int s, int64_t* hashes, int64_t* starts, int64_t* stops) = 0;
  virtual int particles_stat(int s, const lcs_particle_stat_config* pc, double tau_eta, lcs_particle_stats* out) = 0;
  virtual int particles_density(int s, int grid_ratio, double* densities) = 0;
  virtual int upload_flow_coarse(const double* U, const double* V, const double* W, const double* P) = 0;
  virtual int transfer_stats(int64_t* h2d, int64_t* d2h) = 0;
  virtual int synchalo(int mask, int r, int full) = 0;
  virtual int rhs(int stage) = 0;
  virtual int update(int stage, double dtrk) = 0;
  virtual int rhs_update(int stage, double dtrk) = 0;
  virtual int couple(int stage, double dtrk, lcs_couple_log* log) = 0;
  virtual int forcing(double dtrk, double* p, double* e10) = 0;
  virtual int flow_timestep(double* dt) = 0;
  virtual int particles_timestep(double* dt) = 0;
  virtual int particles_boundary(int s, int stage) = 0;
  virtual int particles_motion(int s, int stage) = 0;
  virtual int particles_update(int s, int stage, double dtrk) = 0;
  virtual int init_particle_velocity(int s) = 0;
  virtual int profile_enable(int on) = 0;
  virtual int profile_reset() = 0;
  virtual int profile_count(int* n) = 0;
  virtual int profile_entry(int i, char* name, int cap, double* ms, int64_t* launches) = 0;
  virtual int launch_count(int64_t* n) = 0;
  virtual int synchronize() = 0;
  virtual int group_create(EngineBase* const* members, int m, GroupBase** out) = 0;
  virtual const lcs_config& config() const = 0;
  virtual int flow_divergence(double* rms, double* maxabs) = 0;
  virtual int debug_waits(int kind) = 0;
  int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    err = buf;
    return code;
  }
};

#define LCS_CUDA(call)                                                                         \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess) return fail(LCS_ECUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

#define LCS_TRY(expr)        \
  do {                       \
    int rc_ = (expr);        \
    if (rc_ != LCS_OK) return rc_; \
  } while (0)

}  // namespace lcs
