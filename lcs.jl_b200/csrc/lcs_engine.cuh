// lcs_engine.cuh -- host orchestration of one time-step handle.
//
// Engine<T> owns a single device allocation (the pool) carved into the
// haloed fields, scratch and particle arrays, one CUDA stream, and the
// device context.  It replays `LCS.evolve!` (src/evolve.jl:63-146) stage by
// stage, and `lcs_step` captures whole steps into CUDA graphs whose HSMAC
// loops are device-side WHILE nodes, so a step needs no host round trip.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <memory>
#include <vector>

#include "../../include/lcs_b200.h"
#include <cudaTypedefs.h>

#include <cstdlib>

#include "lcs_base.h"
#include "lcs_kernels.cuh"
#include "lcs_tma.cuh"
#include "lcs_hsmac_rw.cuh"
#include "lcs_makeindex.cuh"
#include "lcs_pstat.cuh"

// bin edges of logrange(a, b, len) in extended precision (lcs_hostmath.cpp)
extern "C" void lcs_logrange(double a, double b, int len, double* out);

namespace lcs {

// Bytes of the device pool for a config (every allocation the handle makes).
template <typename T>
struct Plan {
  Grid g;
  size_t off_vel[3][3], off_P, off_dU[3], off_stage, off_partials, off_ctx, off_logs, off_rcf, off_sp[LCS_MAX_SPECIES];
  size_t bytes;
  int64_t stage_elems, partials_cap, logs_cap;
  int64_t rcf_coarse, rcf_hat, rcf_Ac, rcf_tw, rcf_en0, rcf_ph;
};

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

template <typename T>
Plan<T> make_plan(const lcs_config& c) {
  Plan<T> p;
  p.g = make_grid<T>(c.dims, c.halo_size);
  size_t o = 0;
  auto take = [&](size_t bytes) {
    size_t at = o;
    o = align_up(o + bytes, 256);
    return at;
  };
  const size_t fb = (size_t)p.g.elems * sizeof(T);
  for (int s = 0; s < 3; s++)
    for (int q = 0; q < 3; q++) p.off_vel[s][q] = take(fb);
  p.off_P = take(fb);
  const int64_t ni = (int64_t)c.dims[0] * c.dims[1] * c.dims[2];
  for (int q = 0; q < 3; q++) p.off_dU[q] = take((size_t)ni * sizeof(T));
  const int64_t hs = (int64_t)(c.dims[0] + 2 * c.halo_size) * (c.dims[1] + 2 * c.halo_size) *
                     (c.dims[2] + 2 * c.halo_size);
  int64_t pmax = 0;
  for (int s = 0; s < c.n_species; s++) pmax = std::max<int64_t>(pmax, c.species[s].nvalid);
  p.stage_elems = std::max<int64_t>(hs, pmax);
  p.off_stage = take((size_t)p.stage_elems * sizeof(double));
  p.partials_cap = 1 << 20;
  p.off_partials = take((size_t)p.partials_cap * sizeof(double));
  p.off_ctx = take(sizeof(Ctx));
  p.logs_cap = 4096;
  p.off_logs = take((size_t)p.logs_cap * sizeof(StepLog));
  // rc-energy buffers
  const int cs = c.forcing == LCS_FORCING_RC_ENERGY ? c.coarse_size : 1;
  const int km = c.forcing == LCS_FORCING_RC_ENERGY ? c.kmax : 1;
  const int nm = (km + 1) * (2 * km + 1) * (2 * km + 1);
  p.rcf_coarse = 3 * (int64_t)cs * cs * cs;
  p.rcf_hat = 2 * 3 * (int64_t)nm;
  p.rcf_Ac = p.rcf_hat;
  p.rcf_tw = 2 * (int64_t)cs;
  p.rcf_en0 = 16;
  p.rcf_ph = 2 * (int64_t)(c.dims[0] + c.dims[1] + c.dims[2] + 3);
  p.off_rcf = take((size_t)(p.rcf_coarse + p.rcf_hat + p.rcf_Ac + p.rcf_tw + p.rcf_en0 + p.rcf_ph) * sizeof(double));
  for (int s = 0; s < c.n_species; s++) p.off_sp[s] = take((size_t)c.species[s].nvalid * (16 * sizeof(double) + 8));
  p.bytes = o;
  return p;
}

inline void sincospi_host(double x, double* s, double* c) {
  // sin(pi x), cos(pi x) with exact reduction of x (Julia's cispi)
  double r = std::fmod(x, 2.0);
  if (r < 0) r += 2.0;
  int neg_s = 0, neg_c = 0;
  if (r >= 1.0) { r -= 1.0; neg_s = 1; neg_c = 1; }
  if (r > 0.5) { r = 1.0 - r; neg_c = !neg_c; }
  double ss, cc;
  const double pi = 3.14159265358979323846;
  if (r == 0.0) { ss = 0.0; cc = 1.0; }
  else if (r == 0.5) { ss = 1.0; cc = 0.0; }
  else if (r <= 0.25) { ss = std::sin(pi * r); cc = std::cos(pi * r); }
  else { double t = 0.5 - r; ss = std::cos(pi * t); cc = std::sin(pi * t); }
  *s = neg_s ? -ss : ss;
  *c = neg_c ? -cc : cc;
}

inline int host_kcount(int k0) {
  int c = 0;
  for (int kz = -k0; kz <= k0; kz++)
    for (int ky = -k0; ky <= k0; ky++)
      for (int kx = -k0; kx <= k0; kx++) {
        int r2 = kx * kx + ky * ky + kz * kz;
        if ((k0 - 0.5) * (k0 - 0.5) <= r2 && r2 < (k0 + 0.5) * (k0 + 0.5)) c++;
      }
  return c;
}

// kset(k0) in the reference's generation order (FourierTools.jl:59-80)
inline void host_kset(int k0, std::vector<std::array<int, 3>>& out) {
  std::vector<std::array<int, 3>> K;
  for (int kz = -k0; kz <= k0; kz++)
    for (int ky = -k0; ky <= k0; ky++)
      for (int kx = 0; kx <= k0; kx++) {
        int r2 = kx * kx + ky * ky + kz * kz;
        if (!((k0 - 0.5) * (k0 - 0.5) <= r2 && r2 < (k0 + 0.5) * (k0 + 0.5))) continue;
        int sgn = 1;
        const int k[3] = {kx, ky, kz};
        for (int a = 0; a < 3; a++) {
          if (k[a] > 0) { sgn = 1; break; }
          if (k[a] < 0) { sgn = -1; break; }
        }
        std::array<int, 3> cc = {sgn * kx, sgn * ky, sgn * kz};
        bool seen = false;
        for (auto& e : K) seen |= (e == cc);
        if (!seen) K.push_back(cc);
      }
  out.insert(out.end(), K.begin(), K.end());
}

template <typename T>
class Engine : public EngineBase {
 public:
  lcs_config cfg;
  Plan<T> plan;
  Grid g;
  cudaStream_t stream = nullptr;
  char* pool = nullptr;
  Ctx* dctx = nullptr;
  StepLog* dlogs = nullptr;
  T* P = nullptr;
  T* dU[3] = {nullptr, nullptr, nullptr};
  void* vel0[3][3];
  double* stage = nullptr;
  double* partials = nullptr;
  double *rcf_coarse = nullptr, *rcf_hat = nullptr, *rcf_Ac = nullptr, *rcf_tw = nullptr, *rcf_en0 = nullptr;
  double2 *ph[3] = {nullptr, nullptr, nullptr};
  RcfModes modes;
  SpeciesDev sp[LCS_MAX_SPECIES];
  // cell index of a species (makeindex!), allocated on its first use
  struct CellIndex {
    CellGeom cg{};
    int ratio = 0;
    int64_t H = 0;
    int64_t* hashes = nullptr;
    int64_t* starts = nullptr;  // and stops = starts + H
    int64_t* S = nullptr;       // run ends S[0..H] and their max-scan M = S + H + 1
    uint32_t* kv = nullptr;     // keys in/out, values in/out: 4 x n
    void* temp = nullptr;       // CUB scratch of the sort and the scan
    size_t temp_bytes = 0;
    bool built = false;
  } ci[LCS_MAX_SPECIES];
  // A second property block per species (17 x n x 8 bytes, allocated on the
  // first index): the permutation writes the spare block and the two swap.
  uint64_t* sp_alloc[LCS_MAX_SPECIES] = {};  // owned (cudaMalloc)
  uint64_t* sp_spare[LCS_MAX_SPECIES] = {};  // the block not in use (sp_alloc or the one in the pool)
  // Batch group (EngineGroup): while the leader captures the group's HSMAC
  // loop, grp lists the members and the HSMAC launches cover all of them.
  const std::vector<Engine<T>*>* grp = nullptr;
  int tuning_gen = 0;            // bumped by set_tuning (a group's graph is rebuilt)
  GroupPtrs<T> grp_ptrs{};       // per member Ctx, P, partials (set by the group)
  int face_group_per_sm = 0;     // co-resident blocks per SM of k_hsmac_faces_group
  // scratch of the particle statistics (grown on demand)
  char* pbuf = nullptr;
  size_t pbuf_bytes = 0;
  bool uploaded_flow = false;
  int64_t launches = 0;
  // profiling
  bool prof = false;
  struct Rec { std::string label; cudaEvent_t a, b; };
  std::vector<Rec> recs;
  std::vector<cudaEvent_t> event_pool;
  struct Tot { std::string label; double ms; int64_t n; };
  std::vector<Tot> totals;
  // host-pinned mirrors
  Ctx* hctx = nullptr;
  StepLog* hlogs = nullptr;  // staging of the step-log ring for asynchronous steps
  cudaEvent_t async_ev = nullptr;
  int async_pending = 0;      // steps enqueued by step_begin and not yet collected
  long long host_step = 0;    // the device's step counter as last read (valid when host_step_known)
  bool host_step_known = false;
  // graphs
  cudaGraphExec_t step_exec = nullptr, evolve_exec = nullptr;
  cudaGraph_t step_graph = nullptr, evolve_graph = nullptr;
  int64_t graph_launches_per_step = 0, graph_launches_per_evolve = 0;

  HsmacCoef hc;
  RhsCoef rc;
  DtCoef dc;
  PartCoef pc;

  ~Engine() override {
    if (step_exec) cudaGraphExecDestroy(step_exec);
    if (step_graph) cudaGraphDestroy(step_graph);
    if (evolve_exec) cudaGraphExecDestroy(evolve_exec);
    if (evolve_graph) cudaGraphDestroy(evolve_graph);
    for (auto& r : recs) { event_pool.push_back(r.a); event_pool.push_back(r.b); }
    for (auto e : event_pool) cudaEventDestroy(e);
    if (hctx) cudaFreeHost(hctx);
    if (hlogs) cudaFreeHost(hlogs);
    for (auto& c : ci) free_index(c);
    for (auto* a : sp_alloc) cudaFree(a);
    cudaFree(pbuf);
    if (async_ev) cudaEventDestroy(async_ev);
    if (pool) cudaFree(pool);
    if (stream) cudaStreamDestroy(stream);
  }

  int init(const lcs_config& c) {
    cfg = c;
    plan = make_plan<T>(c);
    g = plan.g;
    LCS_CUDA(cudaSetDevice(c.device));
    LCS_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    cudaError_t e = cudaMalloc(&pool, plan.bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      pool = nullptr;
      return fail(LCS_ENOMEM, "cudaMalloc of %zu bytes failed: %s", plan.bytes, cudaGetErrorString(e));
    }
    LCS_CUDA(cudaMallocHost(&hctx, sizeof(Ctx)));
    LCS_CUDA(cudaMallocHost(&hlogs, (size_t)plan.logs_cap * sizeof(StepLog)));
    LCS_CUDA(cudaEventCreateWithFlags(&async_ev, cudaEventDisableTiming));
    for (int s = 0; s < 3; s++)
      for (int q = 0; q < 3; q++) vel0[s][q] = pool + plan.off_vel[s][q];
    P = (T*)(pool + plan.off_P);
    for (int q = 0; q < 3; q++) dU[q] = (T*)(pool + plan.off_dU[q]);
    stage = (double*)(pool + plan.off_stage);
    partials = (double*)(pool + plan.off_partials);
    dctx = (Ctx*)(pool + plan.off_ctx);
    dlogs = (StepLog*)(pool + plan.off_logs);
    double* r = (double*)(pool + plan.off_rcf);
    rcf_coarse = r; r += plan.rcf_coarse;
    rcf_hat = r; r += plan.rcf_hat;
    rcf_Ac = r; r += plan.rcf_Ac;
    rcf_tw = r; r += plan.rcf_tw;
    rcf_en0 = r; r += plan.rcf_en0;
    ph[0] = (double2*)r;
    ph[1] = ph[0] + (c.dims[0] + 1);
    ph[2] = ph[1] + (c.dims[1] + 1);
    // zero every field (halos included) so no stale bits are ever read
    LCS_CUDA(cudaMemsetAsync(pool, 0, plan.off_stage, stream));
    Ctx h0;
    memset(&h0, 0, sizeof h0);
    for (int s = 0; s < 3; s++)
      for (int q = 0; q < 3; q++) {
        h0.vel[s][q] = vel0[s][q];
        h0.vphys[s][q] = 3 * s + q;
      }
    h0.dt_particles = c.dtmax;
    static_assert(sizeof(h0.sp_base) / sizeof(h0.sp_base[0]) == LCS_MAX_SPECIES, "one block per species");
    for (int s = 0; s < c.n_species; s++) h0.sp_base[s] = (double*)(pool + plan.off_sp[s]);
    h0.cur.p = NAN;
    h0.cur.e10 = NAN;
    *hctx = h0;
    LCS_CUDA(cudaMemcpyAsync(dctx, hctx, sizeof(Ctx), cudaMemcpyHostToDevice, stream));
    for (int s = 0; s < c.n_species; s++) {
      char* b = pool + plan.off_sp[s];
      sp[s].n = c.species[s].nvalid;
      for (int q = 0; q < 16; q++) sp[s].p[q] = (double*)b + (size_t)q * sp[s].n;
      sp[s].gravity = c.species[s].gravity;
      sp[s].density_ratio = c.species[s].density_ratio;
      sp[s].drag = c.species[s].drag;
      LCS_CUDA(cudaMemsetAsync(b, 0, (size_t)sp[s].n * (16 * sizeof(double) + 8), stream));
    }
    // coefficients
    const double dx = kDomainLength / c.dims[0], dy = kDomainLength / c.dims[1], dz = kDomainLength / c.dims[2];
    const double Re = c.U0 * c.L0 / c.NU;
    rc.dxi = 1.0 / dx; rc.dyi = 1.0 / dy; rc.dzi = 1.0 / dz; rc.Rei = 1.0 / Re;
    hc.dxi = rc.dxi; hc.dyi = rc.dyi; hc.dzi = rc.dzi;
    hc.dl = 1.0 / (2.0 * (hc.dxi * hc.dxi + hc.dyi * hc.dyi + hc.dzi * hc.dzi));
    hc.omega = c.omega;
    hc.dxmin = std::fmin(dx, std::fmin(dy, dz));
    hc.epsp = c.epsp;
    hc.count = (double)((int64_t)(c.dims[0] + 1) * (c.dims[1] + 1) * (c.dims[2] + 1));
    hc.itrmin = c.itrmin;
    hc.itrmax = c.itrmax;
    hc.coloring = c.coloring;
    dc.cfl = c.cfl; dc.dtmax = c.dtmax; dc.dx = dx; dc.dy = dy; dc.dz = dz; dc.Re = Re;
    dc.with_particles = c.mode == LCS_MODE_FLOW_PARTICLE && c.n_species > 0;
    pc.dx = dx; pc.dy = dy; pc.dz = dz; pc.Re = Re;
    if (c.forcing == LCS_FORCING_RC_ENERGY) LCS_TRY(init_rcf());
    // the TMA-fed row-warp sweep serves red-black-fast (the production
    // colouring); LCS_B200_FUSED_SWEEP=plain selects the plain-load sweep
    const char* sweep = std::getenv("LCS_B200_FUSED_SWEEP");
    const std::string sw = sweep ? std::string(sweep) : std::string("rw");
    use_rw = c.coloring == LCS_COLORING_RED_BLACK_FAST && sw != "plain";
    // the row-warp sweep addresses a field with 32-bit offsets
    if (use_rw && (uint64_t)g.pz * (uint64_t)(g.n[2] + 2 * g.h) >= (1ull << 32))
      return fail(LCS_EINVAL, "a field of 2^32 or more elements");
    if (use_rw) LCS_TRY(init_tma());
    LCS_TRY(init_faces());
    LCS_CUDA(cudaStreamSynchronize(stream));
    return LCS_OK;
  }

  // ---------------------------------------------------------- tensor maps
  // LCS_B200_ZCHUNK forces the z chunk of the row-warp sweep
  int zchunk_force = 0;
  int init_tma() {
    if (const char* z = std::getenv("LCS_B200_ZCHUNK")) zchunk_force = std::atoi(z);
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    LCS_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
    if (!fn || q != cudaDriverEntryPointSuccess) return fail(LCS_ECUDA, "cuTensorMapEncodeTiled is unavailable");
    auto encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    LCS_CUDA(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, cfg.device));
    encode_fn = encode;
    if (use_rw) {
      // row-warp sweep tile rows: FP64 13 (one CTA of 16 warps per SM, a row
      // per warp); FP32 29 (16 warps of two rows each: 1019-1034 against
      // 1127-1136 us a sweep at 512^3, 177-184 against 201-207 at 256^3);
      // LCS_B200_RW=13 | 8 | 5 | 29 (FP32 only) chooses another
      rw_variant = std::is_same<T, float>::value ? 3 : 0;
      if (const char* v = std::getenv("LCS_B200_RW")) {
        const std::string t(v);
        rw_variant = t == "8" ? 1 : t == "5" ? 2 : (t == "29" && std::is_same<T, float>::value) ? 3 : 0;
      }
      LCS_TRY(init_rw_maps());
    }
    return LCS_OK;
  }
  // The row-warp sweep of the current rw_variant: kernel, shared memory,
  // occupancy and its tensor maps (box 64 x rows+4 and 64 x rows).
  int init_rw_maps() {
    switch (rw_variant) {
      case 1: RTY = 8; rw_smem = RwLayout<T, 8, 3>::total; rw_fn = (const void*)k_hsmac_rw<T, 8, 3>;
              rw_threads = RwLayout<T, 8, 3>::NT; break;
      case 2: RTY = 5; rw_smem = RwLayout<T, 5, 3>::total; rw_fn = (const void*)k_hsmac_rw<T, 5, 3>;
              rw_threads = RwLayout<T, 5, 3>::NT; break;
      case 3:
        if constexpr (std::is_same<T, float>::value) {
          RTY = 29; rw_smem = RwLayout<T, 29, 3, 2>::total; rw_fn = (const void*)k_hsmac_rw<T, 29, 3, 2>;
          rw_threads = RwLayout<T, 29, 3, 2>::NT;
          break;
        }
        return fail(LCS_EINVAL, "29-row sweep tiles are FP32 only");
      default: RTY = 13; rw_smem = RwLayout<T, 13, kRwRing<T>>::total; rw_fn = (const void*)k_hsmac_rw<T, 13, kRwRing<T>>;
               rw_threads = RwLayout<T, 13, kRwRing<T>>::NT; break;
    }
    const CUtensorMapDataType dtype =
        std::is_same<T, double>::value ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    const cuuint64_t dims[3] = {(cuuint64_t)g.px, (cuuint64_t)(g.n[1] + 2 * g.h), (cuuint64_t)(g.n[2] + 2 * g.h)};
    const cuuint64_t strides[2] = {(cuuint64_t)g.px * sizeof(T), (cuuint64_t)g.pz * sizeof(T)};
    const cuuint32_t estr[3] = {1, 1, 1};
    const cuuint32_t rbox[3] = {(cuuint32_t)RW_W, (cuuint32_t)RTY + 4, 1};
    for (int b = 0; b < kVelMaps; b++) {
      CUresult rr = encode_fn(&tmaps_rw.vel[b], dtype, 3, vel0[b / 3][b % 3], dims, strides, rbox, estr,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      if (rr != CUDA_SUCCESS) return fail(LCS_ECUDA, "cuTensorMapEncodeTiled (row-warp velocity %d) failed: %d", b,
                                          (int)rr);
    }
    const cuuint32_t rpbox[3] = {(cuuint32_t)RW_W, (cuuint32_t)RTY, 1};
    CUresult rp = encode_fn(&tmaps_rw.P, dtype, 3, (void*)P, dims, strides, rpbox, estr,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (rp != CUDA_SUCCESS) return fail(LCS_ECUDA, "cuTensorMapEncodeTiled (row-warp P) failed: %d", (int)rp);
    LCS_CUDA(cudaFuncSetAttribute(rw_fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rw_smem));
    const void* rw_group_fn = rw_variant == 1   ? (const void*)k_hsmac_rw_group<T, 8, 3>
                              : rw_variant == 2 ? (const void*)k_hsmac_rw_group<T, 5, 3>
                                                : (const void*)k_hsmac_rw_group<T, 13, kRwRing<T>>;
    if constexpr (std::is_same<T, float>::value) {
      if (rw_variant == 3) rw_group_fn = (const void*)k_hsmac_rw_group<T, 29, 3, 2>;
    }
    LCS_CUDA(cudaFuncSetAttribute(rw_group_fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rw_smem));
    LCS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&rw_ctas_per_sm, rw_fn, rw_threads, rw_smem));
    if (rw_ctas_per_sm < 1) return fail(LCS_ECUDA, "the row-warp sweep does not fit on an SM");
    return LCS_OK;
  }
  PFN_cuTensorMapEncodeTiled_v12000 encode_fn = nullptr;
  int num_sms = 148;
  bool use_rw = false;
  TensorMaps tmaps_rw;
  int rw_variant = 0, RTY = 13, rw_threads = 512, rw_ctas_per_sm = 1;
  size_t rw_smem = 0;
  const void* rw_fn = nullptr;

  // blocks of the cooperative face-phase kernel (0: twelve in-place launches)
  int face_grid = 0;
  int init_faces() {
    int coop = 0, per_sm = 0;
    LCS_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, cfg.device));
    LCS_CUDA(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, cfg.device));
    LCS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_hsmac_faces<T>, 256, 0));
    const char* f = std::getenv("LCS_B200_FACES");
    const bool sequential = f && std::string(f) == "phases";
    face_grid = (coop && per_sm > 0 && !sequential) ? std::min(per_sm, 2) * num_sms : 0;
    LCS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&face_group_per_sm, k_hsmac_faces_group<T>, 256, 0));
    return LCS_OK;
  }

  int init_rcf() {
    const int cs = cfg.coarse_size;
    std::vector<double> tw(2 * cs);
    for (int x = 0; x < cs; x++) sincospi_host(-2.0 * x / cs, &tw[2 * x + 1], &tw[2 * x]);
    LCS_TRY(copy(rcf_tw, tw.data(), tw.size() * sizeof(double), cudaMemcpyHostToDevice));
    std::vector<double> en0(16, 0.0);
    for (int k0 = cfg.kmin; k0 <= cfg.kmax; k0++) {  // enespe0 (rcf.jl:187-191)
      const double c1 = host_kcount(1), ck = host_kcount(k0);
      const double a = k0 + 0.5, b = k0 - 0.5;
      en0[k0 - cfg.kmin] = cfg.energy * std::pow((double)k0, -5.0 / 3.0) * (1.5 * 1.5 * 1.5 - 0.5 * 0.5 * 0.5) /
                           (a * a * a - b * b * b) * ck / c1;
    }
    LCS_TRY(copy(rcf_en0, en0.data(), 16 * sizeof(double), cudaMemcpyHostToDevice));
    const double phi = (double)(cfg.dims[0] / cs) / 2.0;  // phase_shift (flows/config.jl:149)
    for (int a = 0; a < 3; a++) {
      std::vector<double> t(2 * (cfg.dims[a] + 1), 0.0);
      for (int i = 1; i <= cfg.dims[a]; i++) sincospi_host(2.0 * (i - phi) * (1.0 / cfg.dims[a]), &t[2 * i + 1], &t[2 * i]);
      LCS_TRY(copy(ph[a], t.data(), t.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    std::vector<std::array<int, 3>> ks;
    memset(&modes, 0, sizeof modes);
    modes.nshell = cfg.kmax - cfg.kmin + 1;
    for (int K = cfg.kmin; K <= cfg.kmax; K++) {
      modes.kofs[K - cfg.kmin] = (int)ks.size();
      host_kset(K, ks);
    }
    modes.kofs[modes.nshell] = (int)ks.size();
    if (ks.size() > 256) return fail(LCS_EINVAL, "rc-energy kset too large (%zu modes)", ks.size());
    modes.n = (int)ks.size();
    for (size_t q = 0; q < ks.size(); q++)
      for (int a = 0; a < 3; a++) modes.k[q][a] = (signed char)ks[q][a];
    return LCS_OK;
  }

  // ---------------------------------------------------------------- launch
  cudaEvent_t get_event() {
    if (!event_pool.empty()) {
      cudaEvent_t e = event_pool.back();
      event_pool.pop_back();
      return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
  }
  bool capturing = false;
  template <typename K, typename... A>
  int launch(const char* label, K kernel, dim3 grid, dim3 block, size_t smem, A... args) {
    cudaEvent_t a = nullptr, b = nullptr;
    if (prof && !capturing) {
      a = get_event();
      b = get_event();
      cudaEventRecord(a, stream);
    }
    kernel<<<grid, block, smem, stream>>>(args...);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(LCS_ECUDA, "launch %s: %s", label, cudaGetErrorString(e));
    if (a) {
      cudaEventRecord(b, stream);
      recs.push_back({label, a, b});
    }
    launches++;
    return LCS_OK;
  }
  // launch whose blocks are all co-resident (they meet at grid barriers)
  template <typename... P, typename... A>
  int launch_coop(const char* label, void (*kernel)(P...), dim3 grid, dim3 block, A... args) {
    cudaEvent_t a = nullptr, b = nullptr;
    if (prof && !capturing) {
      a = get_event();
      b = get_event();
      cudaEventRecord(a, stream);
    }
    cudaLaunchConfig_t lc = {};
    lc.gridDim = grid;
    lc.blockDim = block;
    lc.dynamicSmemBytes = 0;
    lc.stream = stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    lc.attrs = at;
    lc.numAttrs = 1;
    cudaError_t e = cudaLaunchKernelEx(&lc, kernel, args...);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return fail(LCS_ECUDA, "launch %s: %s", label, cudaGetErrorString(e));
    if (a) {
      cudaEventRecord(b, stream);
      recs.push_back({label, a, b});
    }
    launches++;
    return LCS_OK;
  }
  int collect_profile() {
    if (recs.empty()) return LCS_OK;
    LCS_CUDA(cudaStreamSynchronize(stream));
    for (auto& r : recs) {
      float ms = 0;
      cudaEventElapsedTime(&ms, r.a, r.b);
      bool found = false;
      for (auto& t : totals)
        if (t.label == r.label) { t.ms += ms; t.n++; found = true; break; }
      if (!found) totals.push_back({r.label, (double)ms, 1});
      event_pool.push_back(r.a);
      event_pool.push_back(r.b);
    }
    recs.clear();
    return LCS_OK;
  }

  static unsigned int blocks_for(int64_t n, int bs, int64_t cap = 148 * 16) {
    int64_t b = (n + bs - 1) / bs;
    return (unsigned int)std::max<int64_t>(1, std::min<int64_t>(b, cap));
  }

  // host<->device copies, counted for lcs_transfer_stats
  int64_t h2d_bytes = 0, d2h_bytes = 0;
  int copy(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind) {
    if (bytes == 0) return LCS_OK;
    LCS_CUDA(cudaMemcpyAsync(dst, src, bytes, kind, stream));
    if (kind == cudaMemcpyHostToDevice) h2d_bytes += (int64_t)bytes;
    if (kind == cudaMemcpyDeviceToHost) d2h_bytes += (int64_t)bytes;
    return LCS_OK;
  }

  // ------------------------------------------------------------ primitives
  int fill(int set, bool withP, int r, int full) {
    FillArgs fa;
    memset(&fa, 0, sizeof fa);
    fa.nf = 0;
    if (set >= 0)
      for (int q = 0; q < 3; q++) { fa.set[fa.nf] = set; fa.comp[fa.nf] = q; fa.ptr[fa.nf] = nullptr; fa.nf++; }
    if (withP) { fa.set[fa.nf] = -1; fa.comp[fa.nf] = 0; fa.ptr[fa.nf] = P; fa.nf++; }  // a group fill: each member's P
    const int64_t total = fill_count(g, r, full);
    if (total >= INT32_MAX) return fail(LCS_EINVAL, "halo too large for 32-bit fill indices");
    if (grp)
      return launch("synchalo", k_fill_halo_group<T>, dim3(blocks_for(total, 256, 148 * 32), (unsigned)grp->size()),
                    dim3(256), 0, grp_ptrs, g, fa, r, full, total);
    return launch("synchalo", k_fill_halo<T>, dim3(blocks_for(total, 256, 148 * 32)), dim3(256), 0, (const Ctx*)dctx, g, fa, r,
                  full, total);
  }

  int set_stage_dt(int stage) { return launch("stage_dt", k_set_stage_dt, dim3(1), dim3(1), 0, dctx, stage); }
  int set_scalar(double* dst, double v) { return launch("set_scalar", k_set_scalar, dim3(1), dim3(1), 0, dst, v); }

  int rhs_kernel(int in_set, int out_set, int mode, int use_stage_dt, double dt) {
    dim3 grid((g.n[0] + 127) / 128, g.n[1], g.n[2]);
    return launch(mode ? "rhs_update" : "rhs", k_rhs<T>, grid, dim3(128), 0, (const Ctx*)dctx, g, (const T*)P, in_set,
                  out_set, (int)kSetUs, mode, dU[0], dU[1], dU[2], rc, use_stage_dt, dt);
  }

  // ----------------------------------------------------------------- HSMAC
  static Box bbox(const Box& a, const Box& b) {
    Box r;
    for (int q = 0; q < 3; q++) { r.lo[q] = std::min(a.lo[q], b.lo[q]); r.hi[q] = std::max(a.hi[q], b.hi[q]); }
    return r;
  }
  static constexpr int TX = 32, TY = 8;
  // Launch geometry of a fused sweep whose outputs cover `out`.
  struct FusedGeom { Box gb; unsigned int gx, gy, gz; int zchunk; };
  FusedGeom fused_geom(Box out) const {
    FusedGeom f;
    f.gb = bbox(out, cube(g, 1, 0));
    const int nzc = f.gb.len(2);
    f.gx = (f.gb.len(0) + TX - 1) / TX;
    f.gy = (f.gb.len(1) + TY - 1) / TY;
    // enough CTAs to fill the 148 SMs several times over: chunk z
    int zchunk = nzc;
    const int64_t cols = (int64_t)f.gx * f.gy;
    while (cols * ((nzc + zchunk - 1) / zchunk) < 148 * 8 && zchunk > 16) zchunk = (zchunk + 1) / 2;
    f.zchunk = zchunk;
    f.gz = (nzc + zchunk - 1) / zchunk;
    return f;
  }
  int fused(int set, Box D, Box out, int fill_r, double* part, int finalize, int group_end, int* nblocks = nullptr) {
    if (grp && !use_rw) return fail(LCS_EINVAL, "group sweeps need the row-warp sweep");
    if (use_rw) return fused_rw(set, D, out, fill_r, part, finalize, group_end, nblocks);
    const FusedGeom f = fused_geom(out);
    const int64_t nb = (int64_t)f.gx * f.gy * f.gz;
    if (nb > plan.partials_cap / 2) return fail(LCS_EINVAL, "grid too large for the partials buffer");
    if (nblocks) *nblocks = (int)nb;
    return launch("hsmac_fused", k_hsmac_fused<T, TX, TY>, dim3(f.gx, f.gy, f.gz), dim3(TX * TY), 0, dctx, g, set, P, D,
                  out, f.gb, fill_r, f.zchunk, hc, part, finalize, group_end, 1);
  }
  // TMA-fed sweep: the periodic fill first (in place, like synchalo!), then
  // one pass over tiles whose first column is odd (16-byte TMA rule)
  // z chunk of a TMA-fed sweep: minimise (waves of resident CTAs) x (planes
  // per chunk + the 4 warm-up/drain planes a chunk costs)
  // Share of the GPU this handle's launches are sized for: 1 alone; a batch
  // member or served run gets its part, so that concurrent runs do not each
  // split their work to fill every SM.
  double sm_share = 1.0;
  int share_slots(int slots) const { return std::max(1, (int)std::lround(slots * sm_share)); }
  // Schedule of a row-warp sweep: chunks of zc planes per tile column, chunk
  // major, in full waves of the resident CTAs; the chunks of a last, partial
  // wave are split into q sub-ranges so that it fills the GPU too.  zc
  // minimises the cost in plane-steps: full waves x (zc + 4 warm-up/drain
  // planes) + the last wave's (sub-range + 4), with chunks of at most
  // kMaxChunk planes: CTAs that stream whole columns at once move through z in
  // step and read the same few planes together, which measured far slower
  // (512^3 FP32, 29-row tiles: 1484 us a sweep with 514-plane chunks, 1019-1034
  // with 48-96).
  static constexpr int kMaxChunk = 96;
  RwSched rw_schedule(int ncols, int nzc, int slots) const {
    slots = share_slots(slots);
    RwSched best{ncols, nzc, ncols, 1, ncols};
    double best_cost = 1e300;
    for (int nc = std::max(1, (nzc + kMaxChunk - 1) / kMaxChunk); nc <= std::max(std::min(nzc, 64), 1); nc++) {
      const int zc = zchunk_force > 0 ? std::min(zchunk_force, nzc) : (nzc + nc - 1) / nc;
      const int nch = (nzc + zc - 1) / zc;
      const int items = ncols * nch;
      const int waves = items / slots, rem = items - waves * slots;
      int q = rem > 0 ? std::max(1, slots / rem) : 1;
      q = std::max(1, std::min(q, zc / 2));  // sub-ranges of 2 planes at least
      const double cost = waves * (zc + 4.0) + (rem > 0 ? std::ceil((double)zc / q) + 4.0 : 0.0);
      if (cost < best_cost - 1e-9) {
        best_cost = cost;
        best = RwSched{ncols, zc, waves * slots, q, waves * slots + rem * q};
      }
      if (zchunk_force > 0) break;
    }
    return best;
  }
  // row-warp sweep: tiles of RW_TX x RTY whose first column is odd
  int fused_rw(int set, Box D, Box out, int fill_r, double* part, int finalize, int group_end, int* nblocks) {
    if (fill_r > 0) LCS_TRY(fill(set, false, fill_r, 1));
    const Box gb = bbox(out, cube(g, 1, 0));
    // first tile column: the largest x0 <= gb.lo[0] with x0-2 on a 16-byte
    // boundary (x0 odd in FP64, x0 = 3 mod 4 in FP32); tiles step by RW_TX = 60
    const int am = 16 / (int)sizeof(T), ar = am - 1;
    int xo = gb.lo[0];
    while (((xo % am) + am) % am != ar % am) xo--;
    const int gx = (gb.hi[0] - xo + 1 + RW_TX - 1) / RW_TX, gy = (gb.len(1) + RTY - 1) / RTY;
    const int nzc = gb.len(2), ncols = gx * gy;
    const RwSched sc = rw_schedule(ncols, nzc, num_sms * rw_ctas_per_sm);
    const int nitems = sc.nitems;
    if (nitems > plan.partials_cap / 2) return fail(LCS_EINVAL, "grid too large for the partials buffer");
    if (nblocks) *nblocks = nitems;
    if (grp) return fused_rw_group(set, D, out, gb, xo, gx, gy, sc, finalize, group_end);
    const dim3 grid(nitems), block(rw_threads);
    if constexpr (std::is_same<T, float>::value) {
      if (rw_variant == 3)
        return launch("hsmac_rw", k_hsmac_rw<T, 29, 3, 2>, grid, block, rw_smem, dctx, g, set, tmaps_rw, P, D, out, gb,
                      xo, gx, gy, sc, hc, part, finalize, group_end);
    }
    switch (rw_variant) {
      case 1: return launch("hsmac_rw", k_hsmac_rw<T, 8, 3>, grid, block, rw_smem, dctx, g, set, tmaps_rw, P, D,
                            out, gb, xo, gx, gy, sc, hc, part, finalize, group_end);
      case 2: return launch("hsmac_rw", k_hsmac_rw<T, 5, 3>, grid, block, rw_smem, dctx, g, set, tmaps_rw, P, D,
                            out, gb, xo, gx, gy, sc, hc, part, finalize, group_end);
      default: return launch("hsmac_rw", k_hsmac_rw<T, 13, kRwRing<T>>, grid, block, rw_smem, dctx, g, set, tmaps_rw, P,
                             D, out, gb, xo, gx, gy, sc, hc, part, finalize, group_end);
    }
  }
  // the same sweep for every member of the group, kGroupMax members a launch
  int fused_rw_group(int set, Box D, Box out, Box gb, int xo, int gx, int gy, RwSched sc, int finalize, int group_end) {
    const int M = (int)grp->size();
    for (int m0 = 0; m0 < M; m0 += kGroupMax) {
      const int mc = std::min(kGroupMax, M - m0);
      GroupRwArgs<T> ga;
      memset(&ga, 0, sizeof ga);
      for (int q = 0; q < mc; q++) {
        Engine<T>* e = (*grp)[m0 + q];
        ga.tm[q] = e->tmaps_rw;
        ga.ctx[q] = e->dctx;
        ga.P[q] = e->P;
        ga.partials[q] = e->partials;
      }
      const dim3 grid(sc.nitems, mc), block(rw_threads);
      int rc2;
      if constexpr (std::is_same<T, float>::value)
        if (rw_variant == 3) {
          LCS_TRY(launch("hsmac_rw", k_hsmac_rw_group<T, 29, 3, 2>, grid, block, rw_smem, ga, g, set, D, out, gb, xo,
                         gx, gy, sc, hc, finalize, group_end));
          continue;
        }
      switch (rw_variant) {
        case 1: rc2 = launch("hsmac_rw", k_hsmac_rw_group<T, 8, 3>, grid, block, rw_smem, ga, g, set, D, out, gb, xo,
                             gx, gy, sc, hc, finalize, group_end); break;
        case 2: rc2 = launch("hsmac_rw", k_hsmac_rw_group<T, 5, 3>, grid, block, rw_smem, ga, g, set, D, out, gb, xo,
                             gx, gy, sc, hc, finalize, group_end); break;
        default: rc2 = launch("hsmac_rw", k_hsmac_rw_group<T, 13, kRwRing<T>>, grid, block, rw_smem, ga, g, set, D, out, gb,
                              xo, gx, gy, sc, hc, finalize, group_end);
      }
      LCS_TRY(rc2);
    }
    return LCS_OK;
  }
  // in-place colour phases over a box (both colours), partial sums appended
  int phases(int set, Box b, double* part, int* used) {
    if (grp) return fail(LCS_EINVAL, "group sweeps need the cooperative face kernel");
    if (b.lo[0] > b.hi[0] || b.lo[1] > b.hi[1] || b.lo[2] > b.hi[2]) return LCS_OK;
    if (cfg.coloring == LCS_COLORING_RED_BLACK_BLOCK) {
      const int bs = cfg.coloring_block;
      const int64_t nb = (int64_t)((b.len(0) + bs - 1) / bs) * ((b.len(1) + bs - 1) / bs) * ((b.len(2) + bs - 1) / bs);
      const unsigned int gbk = blocks_for(nb, 128, 4096);
      for (int color = 0; color <= 1; color++) {
        LCS_TRY(launch("hsmac_block", k_hsmac_block<T>, dim3(gbk), dim3(128), 0, dctx, g, set, P, b, color, bs, hc,
                       part + *used));
        *used += gbk;
      }
      return LCS_OK;
    }
    const int64_t total = (int64_t)((b.len(0) + 1) / 2) * b.len(1) * b.len(2);
    const unsigned int gbk = blocks_for(total, 256, 4096);
    for (int color = 0; color <= 1; color++) {
      LCS_TRY(launch("hsmac_phase", k_hsmac_phase<T>, dim3(gbk), dim3(256), 0, dctx, g, set, P, b, color, hc,
                     part + *used));
      *used += gbk;
    }
    return LCS_OK;
  }
  static void faces_of(Box d, Box c, Box out[6]) {  // Topologies.faces (halo.jl:349-366)
    for (int f = 0; f < 6; f++) out[f] = d;
    out[0].hi[2] = c.lo[2] - 1;
    out[1].lo[2] = c.hi[2] + 1;
    out[2].hi[1] = c.lo[1] - 1; out[2].lo[2] = c.lo[2]; out[2].hi[2] = c.hi[2];
    out[3].lo[1] = c.hi[1] + 1; out[3].lo[2] = c.lo[2]; out[3].hi[2] = c.hi[2];
    out[4].hi[0] = c.lo[0] - 1; out[4].lo[1] = c.lo[1]; out[4].hi[1] = c.hi[1]; out[4].lo[2] = c.lo[2]; out[4].hi[2] = c.hi[2];
    out[5].lo[0] = c.hi[0] + 1; out[5].lo[1] = c.lo[1]; out[5].hi[1] = c.hi[1]; out[5].lo[2] = c.lo[2]; out[5].hi[2] = c.hi[2];
  }
  int finalize_sweep(int n, int group_end) {
    if (grp) return fail(LCS_EINVAL, "group sweeps finalize inside the sweep kernels");
    return launch("hsmac_finalize", k_hsmac_finalize, dim3(1), dim3(256), 0, dctx, (const double*)partials, n, hc,
                  group_end);
  }
  // one sweep of the phased kind: [fill +] core, then the 6 faces of dom
  int sweep_overlap(int set, Box dom, int fill_r, int group_end) {
    const Box core = cube(g, 2, 0);
    int used = 0;
    if (cfg.coloring == LCS_COLORING_RED_BLACK_BLOCK) {
      LCS_TRY(fill(set, false, fill_r, 1));
      LCS_TRY(phases(set, core, partials, &used));
    } else {
      // the fused core sweep writes every position the face phases read
      Box out = dom;
      for (int q = 0; q < 3; q++) { out.lo[q] -= 1; out.hi[q] = std::min(out.hi[q], g.n[q] + g.h); }
      for (int q = 0; q < 3; q++) out.lo[q] = std::max(out.lo[q], 1 - g.h);
      LCS_TRY(fused(set, core, out, fill_r, partials, 0, 0, &used));
    }
    Box f[6];
    faces_of(dom, core, f);
    const bool core_nonempty = core.len(0) > 0 && core.len(1) > 0 && core.len(2) > 0;
    int64_t slab_cells = 0;  // the face kernel indexes a pair of slabs with 32-bit integers
    for (int q = 0; q < 6; q++)
      slab_cells = std::max<int64_t>(slab_cells, (int64_t)((f[q].len(0) + 1) / 2) * f[q].len(1) * f[q].len(2));
    // blocks: enough for one round of the largest phase (4 cells per thread),
    // at most the co-resident grid and the handle's share of it
    const int fblocks = (int)std::max<int64_t>(
        1, std::min<int64_t>({(int64_t)face_grid, (int64_t)share_slots(face_grid), (2 * slab_cells + 1023) / 1024}));
    if (face_grid > 0 && core_nonempty && cfg.coloring != LCS_COLORING_RED_BLACK_BLOCK &&
        used + fblocks <= plan.partials_cap && 2 * slab_cells < INT32_MAX) {
      FaceSet fs;
      for (int q = 0; q < 6; q++) fs.f[q] = f[q];
      if (grp) {  // members in co-resident chunks; each member's blocks meet at its own barrier
        const int M = (int)grp->size();
        const int per = std::max(1, std::min(kGroupPtrMax, face_group_per_sm * num_sms / fblocks));
        if (face_group_per_sm * num_sms < fblocks) return fail(LCS_EINVAL, "face grid too large for a group");
        for (int m0 = 0; m0 < M; m0 += per) {
          const int mc = std::min(per, M - m0);
          GroupPtrs<T> gp;
          memset(&gp, 0, sizeof gp);
          for (int q = 0; q < mc; q++) {
            gp.ctx[q] = grp_ptrs.ctx[m0 + q];
            gp.P[q] = grp_ptrs.P[m0 + q];
            gp.partials[q] = grp_ptrs.partials[m0 + q];
          }
          LCS_TRY(launch_coop("hsmac_faces", k_hsmac_faces_group<T>, dim3(fblocks, mc), dim3(256), gp, g, set, fs,
                              hc, used, group_end));
        }
        return LCS_OK;
      }
      return launch_coop("hsmac_faces", k_hsmac_faces<T>, dim3(fblocks), dim3(256), dctx, g, set, P, fs, hc,
                         partials, used, group_end);
    }
    for (int q = 0; q < 6; q++) LCS_TRY(phases(set, f[q], partials, &used));
    return finalize_sweep(used, group_end);
  }
  // one plain sweep over the box D; `out` = positions the next consumer reads
  int sweep_plain(int set, Box D, Box out, int fill_r, int group_end) {
    if (cfg.coloring == LCS_COLORING_RED_BLACK_BLOCK) {
      if (fill_r > 0) LCS_TRY(fill(set, false, fill_r, 1));
      int used = 0;
      LCS_TRY(phases(set, D, partials, &used));
      return finalize_sweep(used, group_end);
    }
    return fused(set, D, out, fill_r, partials, 1, group_end);
  }
  // One iteration of the reference's `while itr < itrmax` loop.
  int couple_group(int set) {
    const int n0 = g.n[0], h = g.h;
    (void)n0;
    const Box full = cube(g, 1 - h, h);
    if (cfg.time_blocking) {  // _couple_time_blocking! (hsmac.jl:131-201)
      const Box d1 = cube(g, -1, 3), d2 = cube(g, 0, 2), d3 = cube(g, 1, 1);
      const Box o1 = cube(g, -1, 2), o2 = cube(g, 0, 1), o3 = cube(g, 1, 0);
      if (cfg.overlap) {
        LCS_TRY(sweep_overlap(set, d1, h, 0));
      } else {
        LCS_TRY(sweep_plain(set, d1, o1, h, 0));
      }
      (void)full;
      LCS_TRY(sweep_plain(set, d2, o2, 0, 0));
      LCS_TRY(sweep_plain(set, d3, o3, 0, 1));
    } else {  // _couple_naive! (hsmac.jl:77-129)
      const Box d = cube(g, 1, 1);
      if (cfg.overlap) {
        LCS_TRY(sweep_overlap(set, d, 1, 1));
      } else {
        LCS_TRY(sweep_plain(set, d, cube(g, 1, 0), 1, 1));
      }
    }
    return LCS_OK;
  }
  int sweeps_per_group() const { return cfg.time_blocking ? 3 : 1; }
  // iterations of a couple's loop: at most ceil(itrmax / sweeps per group),
  // plus a margin (the device loop and the host loop use the same bound)
  int max_loop_groups() const { return cfg.itrmax / sweeps_per_group() + 2; }

  int read_ctx() {
    LCS_TRY(copy(hctx, dctx, sizeof(Ctx), cudaMemcpyDeviceToHost));
    LCS_CUDA(cudaStreamSynchronize(stream));
    host_step = hctx->step;
    host_step_known = true;
    return LCS_OK;
  }

  // Host-driven couple loop: groups are enqueued while no exit is possible
  // (itr < itrmin), then the loop state is read back after each group.
  int couple_direct(int stage) {
    const int set = stage == 1 ? kSetUs2 : kSetUs;  // Us_couple (couple.jl:1-2)
    LCS_TRY(launch("couple_reset", k_couple_reset, dim3(1), dim3(1), 0, dctx, cfg.itrmax));
    int itr = 0;
    const int spg = sweeps_per_group();
    // the device advances itr by one per sweep until it exits; the group
    // count is bounded so the host loop ends even if that ever failed
    const int max_groups = max_loop_groups();
    for (int grp = 0; itr < cfg.itrmax; grp++) {
      if (grp >= max_groups) return fail(LCS_ETIMEDOUT, "HSMAC loop did not advance");
      LCS_TRY(couple_group(set));
      const int last_itr_in_group = itr + spg - 1;
      if (last_itr_in_group >= cfg.itrmin) {
        LCS_TRY(read_ctx());
        if (hctx->wait_error) return fail(LCS_ETIMEDOUT, "a bounded device wait (TMA tile load or grid barrier) ran out");
        if (hctx->nonfinite) return fail(LCS_ENONFINITE, "HSMAC residual is not finite");
        if (hctx->cs.done) break;
        itr = hctx->cs.itr;
      } else {
        itr += spg;
      }
    }
    return launch("couple_log", k_couple_log, dim3(1), dim3(1), 0, dctx, stage);
  }

  // ---------------------------------------------------------------- stages
  int forcing_stage() {
    const int64_t ni = (int64_t)g.n[0] * g.n[1] * g.n[2];
    const unsigned int nb = blocks_for(ni, 256, 148 * 8);
    if (cfg.forcing == LCS_FORCING_LINEAR_POWER) {
      LCS_TRY(fill(kSetUs, false, g.h, 1));
      LCS_TRY(launch("lf_sums", k_lf_sums<T>, dim3(nb), dim3(256), 0, (const Ctx*)dctx, g, partials));
      LCS_TRY(launch("lf_coef", k_lf_coef, dim3(1), dim3(256), 0, dctx, (const double*)partials, (int)nb, (double)ni,
                     cfg.power));
      LCS_TRY(launch("lf_apply", k_lf_apply<T>, dim3(nb), dim3(256), 0, dctx, g, partials));
      return launch("power_mean", k_power_finalize, dim3(1), dim3(256), 0, dctx, (const double*)partials, (int)nb,
                    (double)ni, (double)NAN);
    }
    if (cfg.forcing == LCS_FORCING_RC_ENERGY) {
      const int cs = cfg.coarse_size, km = cfg.kmax;
      const int nm = (km + 1) * (2 * km + 1) * (2 * km + 1);
      LCS_TRY(launch("rcf_boxmean", k_rcf_boxmean<T>, dim3((3 * cs * cs * cs + 127) / 128), dim3(128), 0,
                     (const Ctx*)dctx, g, cs, rcf_coarse));
      LCS_TRY(launch("rcf_dft", k_rcf_dft, dim3(3 * nm), dim3(256), 0, (const double*)rcf_coarse, cs, km,
                     (const double*)rcf_tw, rcf_hat));
      const double norm = (double)(2 * (cs / 2 + 1) - 2) * cs * cs;
      LCS_TRY(launch("rcf_spectrum", k_rcf_spectrum, dim3(1), dim3(32), 0, (const double*)rcf_hat, cfg.kmin, km, norm,
                     (const double*)rcf_en0, rcf_Ac));
      LCS_TRY(launch("rcf_apply", k_rcf_apply<T>, dim3(nb), dim3(256), 0, dctx, g, (const double*)rcf_Ac,
                     (const double2*)ph[0], (const double2*)ph[1], (const double2*)ph[2], modes, km, partials));
      return launch("power_mean", k_power_finalize, dim3(1), dim3(256), 0, dctx, (const double*)partials, (int)nb,
                    (double)ni, cfg.energy);
    }
    return LCS_OK;
  }

  int particles_stage(int stage, int modes_mask, int use_stage_dt, double dt, int only = -1) {
    if (cfg.mode != LCS_MODE_FLOW_PARTICLE) return LCS_OK;
    for (int s = 0; s < cfg.n_species; s++) {
      if (only >= 0 && s != only) continue;
      if (sp[s].n == 0) continue;
      LCS_TRY(launch("particles", k_particles<T>, dim3((unsigned)((sp[s].n + 255) / 256)), dim3(256), 0,
                     (const Ctx*)dctx, g, s, sp[s], pc, stage, modes_mask, use_stage_dt, dt));
    }
    return LCS_OK;
  }

  int timestep_kernels(int flow_only, double* dout) {
    LCS_TRY(fill(kSetUs, false, g.h, 0));  // FaceHalo(grid) (flows/timestep.jl:33)
    const int64_t ni = (int64_t)g.n[0] * g.n[1] * g.n[2];
    const unsigned int nb = blocks_for(ni, 256, 148 * 8);
    LCS_TRY(launch("cfl_max", k_cfl_max<T>, dim3(nb), dim3(256), 0, (const Ctx*)dctx, g, partials));
    return launch("cfl_finalize", k_cfl_finalize, dim3(1), dim3(256), 0, dctx, (const double*)partials, (int)nb, dc,
                  flow_only, dout);
  }

  // evolve! body with state.dt already in ctx->dt
  int evolve_kernels(bool direct_couple) {
    LCS_TRY(launch("step_begin", k_step_begin, dim3(1), dim3(1), 0, dctx));
    for (int stage = 1; stage <= 2; stage++) {
      const int set = stage == 1 ? kSetUs : kSetUs2;
      LCS_TRY(set_stage_dt(stage));
      LCS_TRY(fill(set, true, g.h, 1));                 // synchalo!(FullHalo(grid), (Us.., P))
      LCS_TRY(particles_stage(stage, 7, 1, 0.0));       // boundary!, motion!, update!
      LCS_TRY(rhs_kernel(set, stage == 1 ? kSetUs2 : kSetUs, 1, 1, 0.0));  // rhs! + update!
      if (stage == 2) LCS_TRY(forcing_stage());
      if (direct_couple) LCS_TRY(couple_direct(stage));
      else LCS_TRY(couple_graph_nodes(stage));
    }
    return LCS_OK;
  }

  // ------------------------------------------------------------ graph mode
  // Appends a device-side loop for one couple to the stream being captured:
  // reset; WHILE(cont) { group }; log.
  int couple_graph_nodes(int stage) {
    const int set = stage == 1 ? kSetUs2 : kSetUs;
    LCS_TRY(launch("couple_reset", k_couple_reset, dim3(1), dim3(1), 0, dctx, cfg.itrmax));
    cudaStreamCaptureStatus st;
    cudaGraph_t graph;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    LCS_CUDA(cudaStreamGetCaptureInfo(stream, &st, nullptr, &graph, &deps, &ndeps));
    if (st != cudaStreamCaptureStatusActive) return fail(LCS_ESTATE, "couple_graph_nodes outside a capture");
    cudaGraphConditionalHandle handle;
    LCS_CUDA(cudaGraphConditionalHandleCreate(&handle, graph, cfg.itrmax > 0 ? 1u : 0u, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    LCS_CUDA(cudaGraphAddNode(&node, graph, deps, ndeps, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    // capture the loop body on a side stream into the body graph
    cudaStream_t main = stream;
    cudaStream_t side;
    LCS_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
    LCS_CUDA(cudaStreamBeginCaptureToGraph(side, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    stream = side;
    int rc2 = couple_group(set);
    if (rc2 == LCS_OK)
      rc2 = launch("couple_continue", k_couple_continue, dim3(1), dim3(1), 0, dctx, handle, max_loop_groups());
    stream = main;
    cudaGraph_t body_out;
    cudaError_t e = cudaStreamEndCapture(side, &body_out);
    cudaStreamDestroy(side);
    if (rc2 != LCS_OK) return rc2;
    if (e != cudaSuccess) return fail(LCS_ECUDA, "capture of the couple loop: %s", cudaGetErrorString(e));
    LCS_CUDA(cudaStreamUpdateCaptureDependencies(stream, &node, 1, cudaStreamSetCaptureDependencies));
    return launch("couple_log", k_couple_log, dim3(1), dim3(1), 0, dctx, stage);
  }

  // Captures one step (with_timestep) or one evolve! into an executable graph.
  int build_graph(bool with_timestep, cudaGraph_t* gout, cudaGraphExec_t* xout, int64_t* per_launch) {
    if (*xout) return LCS_OK;
    LCS_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeRelaxed));
    capturing = true;
    const int64_t l0 = launches;
    int rc2 = with_timestep ? timestep_kernels(0, nullptr) : LCS_OK;
    if (rc2 == LCS_OK) rc2 = evolve_kernels(false);
    if (rc2 == LCS_OK)
      rc2 = launch("step_end", k_step_end, dim3(1), dim3(1), 0, dctx, with_timestep ? dlogs : (StepLog*)nullptr,
                   (int)plan.logs_cap);
    capturing = false;
    cudaGraph_t gr = nullptr;
    cudaError_t e = cudaStreamEndCapture(stream, &gr);
    if (rc2 != LCS_OK) {
      if (gr) cudaGraphDestroy(gr);
      return rc2;
    }
    if (e != cudaSuccess) return fail(LCS_ECUDA, "graph capture: %s", cudaGetErrorString(e));
    *per_launch = launches - l0;
    launches = l0;
    *gout = gr;
    LCS_CUDA(cudaGraphInstantiate(xout, gr, 0));
    return LCS_OK;
  }
  int build_step_graph() { return build_graph(true, &step_graph, &step_exec, &graph_launches_per_step); }
  int build_evolve_graph() { return build_graph(false, &evolve_graph, &evolve_exec, &graph_launches_per_evolve); }

  // ------------------------------------------------------------ interface
  int check_flow() { return uploaded_flow ? LCS_OK : fail(LCS_ESTATE, "flow fields were never uploaded"); }
  int check_stage(int stage) { return (stage == 1 || stage == 2) ? LCS_OK : fail(LCS_EINVAL, "stage must be 1 or 2"); }
  int check_species(int s) {
    return (s >= 0 && s < cfg.n_species) ? LCS_OK : fail(LCS_EINVAL, "bad species index %d", s);
  }

  int upload_field(int set, int comp, T* direct, const double* host, int haloed) {
    const int w = haloed ? g.h : 0;
    const int64_t n = (int64_t)(g.n[0] + 2 * w) * (g.n[1] + 2 * w) * (g.n[2] + 2 * w);
    LCS_TRY(copy(stage, host, (size_t)n * sizeof(double), cudaMemcpyHostToDevice));
    return launch("scatter", k_scatter<T>, dim3(blocks_for(n, 256)), dim3(256), 0, (const Ctx*)dctx, g, set, comp,
                  direct, (const double*)stage, haloed);
  }
  int download_field(int set, int comp, const T* direct, double* host, int haloed) {
    const int w = haloed ? g.h : 0;
    const int64_t n = (int64_t)(g.n[0] + 2 * w) * (g.n[1] + 2 * w) * (g.n[2] + 2 * w);
    LCS_TRY(launch("gather", k_gather<T>, dim3(blocks_for(n, 256)), dim3(256), 0, (const Ctx*)dctx, g, set, comp,
                   direct, stage, haloed));
    LCS_TRY(copy(host, stage, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost));
    LCS_CUDA(cudaStreamSynchronize(stream));
    return LCS_OK;
  }

  int upload_flow(const double* U, const double* V, const double* W, const double* Pp) override {
    if (!U || !V || !W || !Pp) return fail(LCS_EINVAL, "null field");
    LCS_TRY(upload_field(kSetUs, 0, nullptr, U, 0));
    LCS_TRY(upload_field(kSetUs, 1, nullptr, V, 0));
    LCS_TRY(upload_field(kSetUs, 2, nullptr, W, 0));
    LCS_TRY(upload_field(-1, 0, P, Pp, 0));
    LCS_CUDA(cudaStreamSynchronize(stream));
    uploaded_flow = true;
    return LCS_OK;
  }
  // `load_coarse_flow_fields!` (src/LCSIO/upsample.jl:1-45) after the read:
  // coarse (n/2)^3 interiors of U, V, W, P, upsampled 2x into the fields
  int upload_flow_coarse(const double* U, const double* V, const double* W, const double* Pp) override {
    if (!U || !V || !W || !Pp) return fail(LCS_EINVAL, "null field");
    if (g.n[0] % 2 || g.n[1] % 2 || g.n[2] % 2) return fail(LCS_EINVAL, "upsampling needs even dims");
    if (async_pending) return fail(LCS_ESTATE, "asynchronous steps are in flight on this handle");
    const int64_t nc = (int64_t)(g.n[0] / 2) * (g.n[1] / 2) * (g.n[2] / 2);
    const double* src[4] = {U, V, W, Pp};
    for (int q = 0; q < 4; q++) {
      LCS_TRY(copy(stage, src[q], (size_t)nc * sizeof(double), cudaMemcpyHostToDevice));
      LCS_TRY(launch("upsample2x", k_upsample2x<T>, dim3(blocks_for(nc, 256)), dim3(256), 0, (const Ctx*)dctx, g,
                     q < 3 ? kSetUs : -1, q < 3 ? q : 0, q < 3 ? (T*)nullptr : P, (const double*)stage));
    }
    LCS_CUDA(cudaStreamSynchronize(stream));
    uploaded_flow = true;
    return LCS_OK;
  }
  int download_flow(double* U, double* V, double* W, double* Pp) override {
    if (U) LCS_TRY(download_field(kSetUs, 0, nullptr, U, 0));
    if (V) LCS_TRY(download_field(kSetUs, 1, nullptr, V, 0));
    if (W) LCS_TRY(download_field(kSetUs, 2, nullptr, W, 0));
    if (Pp) LCS_TRY(download_field(-1, 0, P, Pp, 0));
    return LCS_OK;
  }
  int field_loc(int f, int* set, int* comp, T** direct) {
    *direct = nullptr;
    if (f >= LCS_FIELD_U && f <= LCS_FIELD_W2) { *set = f <= LCS_FIELD_W ? kSetUs : kSetUs2; *comp = f % 3; return LCS_OK; }
    if (f == LCS_FIELD_P) { *set = -1; *comp = 0; *direct = P; return LCS_OK; }
    if (f >= LCS_FIELD_DUDT && f <= LCS_FIELD_DWDT) { *set = -2; *comp = f - LCS_FIELD_DUDT; *direct = dU[*comp]; return LCS_OK; }
    return fail(LCS_EINVAL, "bad field %d", f);
  }
  int field_set(int f, const double* d, int haloed) override {
    if (!d) return fail(LCS_EINVAL, "null data");
    int set, comp;
    T* direct;
    LCS_TRY(field_loc(f, &set, &comp, &direct));
    if (set == -2) {
      const int64_t n = (int64_t)g.n[0] * g.n[1] * g.n[2];
      LCS_TRY(copy(stage, d, (size_t)n * sizeof(double), cudaMemcpyHostToDevice));
      LCS_TRY(launch("convert", k_convert_in<T>, dim3(blocks_for(n, 256)), dim3(256), 0, direct, (const double*)stage, n));
    } else {
      LCS_TRY(upload_field(set, comp, direct, d, haloed));
    }
    LCS_CUDA(cudaStreamSynchronize(stream));
    if (f <= LCS_FIELD_P) uploaded_flow = true;
    return LCS_OK;
  }
  int field_get(int f, double* d, int haloed) override {
    if (!d) return fail(LCS_EINVAL, "null data");
    int set, comp;
    T* direct;
    LCS_TRY(field_loc(f, &set, &comp, &direct));
    if (set == -2) {
      const int64_t n = (int64_t)g.n[0] * g.n[1] * g.n[2];
      LCS_TRY(launch("convert", k_convert_out<T>, dim3(blocks_for(n, 256)), dim3(256), 0, stage, (const T*)direct, n));
      LCS_TRY(copy(d, stage, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost));
      LCS_CUDA(cudaStreamSynchronize(stream));
      return LCS_OK;
    }
    return download_field(set, comp, direct, d, haloed);
  }

  int refresh_particle_dt() {
    // Particles.timestep: min over species of min(0.5 taup(max diam), dtmax)
    double m = INFINITY;
    for (int s = 0; s < cfg.n_species; s++) {
      double dmax = 0.0;
      if (sp[s].n > 0) {
        const unsigned int nb = blocks_for(sp[s].n, 256, 148 * 4);
        LCS_TRY(launch("max_diam", k_max_partial, dim3(nb), dim3(256), 0, (const double*)sp[s].p[LCS_PROP_DIAM], sp[s].n,
                       partials));
        LCS_TRY(launch("max_diam", k_max_reduce, dim3(1), dim3(256), 0, (const double*)partials, (int64_t)nb, stage));
        LCS_TRY(copy(&hctx->scal[7], stage, sizeof(double), cudaMemcpyDeviceToHost));
        LCS_CUDA(cudaStreamSynchronize(stream));
        dmax = hctx->scal[7];
      }
      const double Re = cfg.U0 * cfg.L0 / cfg.NU;
      const double taup = 1.0 / 18.0 * cfg.species[s].density_ratio * Re * (dmax * dmax);
      m = jl_min(m, jl_min(0.5 * taup, cfg.dtmax));
    }
    if (cfg.n_species == 0) m = cfg.dtmax;
    return set_scalar(&dctx->dt_particles, m);
  }

  int upload_particles(int s, int64_t n, const int64_t* ids, const double* diam, const double* x, const double* y,
                       const double* z, const double* u, const double* v, const double* w) override {
    LCS_TRY(check_species(s));
    if (n != sp[s].n) return fail(LCS_EINVAL, "species %d holds %lld particles, got %lld", s, (long long)sp[s].n, (long long)n);
    const double* src[7] = {diam, x, y, z, u, v, w};
    const int dst[7] = {LCS_PROP_DIAM, LCS_PROP_X, LCS_PROP_Y, LCS_PROP_Z, LCS_PROP_U, LCS_PROP_V, LCS_PROP_W};
    for (int q = 0; q < 7; q++)
      if (src[q]) LCS_TRY(copy(sp[s].p[dst[q]], src[q], (size_t)n * sizeof(double), cudaMemcpyHostToDevice));
    if (ids) LCS_TRY(copy((int64_t*)(sp[s].p[0] + 16 * n), ids, (size_t)n * 8, cudaMemcpyHostToDevice));
    LCS_TRY(refresh_particle_dt());
    LCS_CUDA(cudaStreamSynchronize(stream));
    return LCS_OK;
  }
  int download_particles(int s, int64_t* ids, double* diam, double* x, double* y, double* z, double* u, double* v,
                         double* w) override {
    LCS_TRY(check_species(s));
    double* dst[7] = {diam, x, y, z, u, v, w};
    const int src[7] = {LCS_PROP_DIAM, LCS_PROP_X, LCS_PROP_Y, LCS_PROP_Z, LCS_PROP_U, LCS_PROP_V, LCS_PROP_W};
    for (int q = 0; q < 7; q++)
      if (dst[q]) LCS_TRY(copy(dst[q], sp[s].p[src[q]], (size_t)sp[s].n * sizeof(double), cudaMemcpyDeviceToHost));
    if (ids) LCS_TRY(copy(ids, (int64_t*)(sp[s].p[0] + 16 * sp[s].n), (size_t)sp[s].n * 8, cudaMemcpyDeviceToHost));
    LCS_CUDA(cudaStreamSynchronize(stream));
    return LCS_OK;
  }
  int prop_set(int s, int prop, const double* d) override {
    LCS_TRY(check_species(s));
    if (prop < 0 || prop >= LCS_NPROP || !d) return fail(LCS_EINVAL, "bad property");
    LCS_TRY(copy(sp[s].p[prop], d, (size_t)sp[s].n * sizeof(double), cudaMemcpyHostToDevice));
    if (prop == LCS_PROP_DIAM) LCS_TRY(refresh_particle_dt());
    LCS_CUDA(cudaStreamSynchronize(stream));
    return LCS_OK;
  }
  int prop_get(int s, int prop, double* d) override {
    LCS_TRY(check_species(s));
    if (prop < 0 || prop >= LCS_NPROP || !d) return fail(LCS_EINVAL, "bad property");
    LCS_TRY(copy(d, sp[s].p[prop], (size_t)sp[s].n * sizeof(double), cudaMemcpyDeviceToHost));
    LCS_CUDA(cudaStreamSynchronize(stream));
    return LCS_OK;
  }
  int set_state(int64_t step, double t) override {
    if (async_pending) return fail(LCS_ESTATE, "asynchronous steps are in flight on this handle");
    LCS_TRY(set_scalar(&dctx->t, t));
    LCS_TRY(copy(&dctx->step, &step, sizeof(long long), cudaMemcpyHostToDevice));
    LCS_CUDA(cudaStreamSynchronize(stream));
    host_step = step;
    host_step_known = true;
    return LCS_OK;
  }
  int get_state(int64_t* step, double* t) override {
    LCS_TRY(read_ctx());
    if (step) *step = hctx->step;
    if (t) *t = hctx->t;
    return LCS_OK;
  }

  int timestep(double* dt) override {
    LCS_TRY(check_flow());
    LCS_TRY(timestep_kernels(0, nullptr));
    LCS_TRY(collect_profile());
    LCS_TRY(read_ctx());
    if (hctx->nonfinite) return fail(LCS_ENONFINITE, "dt is not finite/positive");
    if (dt) *dt = hctx->dt;
    return LCS_OK;
  }
  void fill_log(const StepLog& s, lcs_log* log) {
    log->couple1.itr = s.itr1; log->couple1.sweeps = s.sweeps1; log->couple1.div = s.div1;
    log->couple2.itr = s.itr2; log->couple2.sweeps = s.sweeps2; log->couple2.div = s.div2;
    log->forcing_p = s.p; log->forcing_e10 = s.e10; log->dt = s.dt; log->t = s.t; log->step = s.step;
  }
  int evolve(double dt, lcs_log* log) override {
    LCS_TRY(check_flow());
    if (async_pending) return fail(LCS_ESTATE, "asynchronous steps are in flight on this handle");
    host_step_known = false;  // the step counter advances on the device
    if (!(dt > 0) || !std::isfinite(dt)) return fail(LCS_EINVAL, "dt must be finite and positive");
    LCS_TRY(set_scalar(&dctx->dt, dt));
    if (cfg.use_graphs && !prof) {
      LCS_TRY(build_evolve_graph());
      LCS_CUDA(cudaGraphLaunch(evolve_exec, stream));
      launches += graph_launches_per_evolve;
    } else {
      LCS_TRY(evolve_kernels(true));
      LCS_TRY(launch("step_end", k_step_end, dim3(1), dim3(1), 0, dctx, (StepLog*)nullptr, 1));
    }
    LCS_TRY(collect_profile());
    LCS_TRY(read_ctx());
    if (hctx->wait_error) return fail(LCS_ETIMEDOUT, "a bounded device wait (TMA tile load or grid barrier) ran out");
    if (hctx->nonfinite) return fail(LCS_ENONFINITE, "non-finite residual or dt");
    if (log) fill_log(hctx->cur, log);
    return LCS_OK;
  }
  int step(int nsteps, lcs_log* logs) override { return step_impl(nsteps, logs, nullptr); }
  int step_timed(int nsteps, lcs_log* logs, double* ms) override { return step_impl(nsteps, logs, ms); }
  int transfer_stats(int64_t* h2d, int64_t* d2h) override {
    if (h2d) *h2d = h2d_bytes;
    if (d2h) *d2h = d2h_bytes;
    return LCS_OK;
  }
  int64_t device_bytes() const override { return (int64_t)plan.bytes; }

  // Launch shapes chosen from outside (the batch's autotuner, the server):
  // rw_rows = tile rows of the row-warp sweep (13, 8 or 5; 0 keeps it),
  // zchunk = planes per z chunk of the TMA sweeps (0: the cost model),
  // share = part of the GPU the launches are sized for (0 < share <= 1).
  // The step graphs are captured again with the new shapes.
  int set_tuning(int rw_rows, int zchunk, double share) override {
    if (async_pending) return fail(LCS_ESTATE, "asynchronous steps are in flight on this handle");
    if (rw_rows != 0 && rw_rows != 13 && rw_rows != 8 && rw_rows != 5 && rw_rows != 29)
      return fail(LCS_EINVAL, "rw_rows must be 0, 13, 8, 5 or 29 (FP32)");
    if (rw_rows == 29 && !std::is_same<T, float>::value) return fail(LCS_EINVAL, "29-row sweep tiles are FP32 only");
    if (zchunk < 0) return fail(LCS_EINVAL, "zchunk < 0");
    if (!(share > 0.0 && share <= 1.0)) return fail(LCS_EINVAL, "share must be in (0, 1]");
    LCS_CUDA(cudaStreamSynchronize(stream));
    if (rw_rows != 0 && use_rw) {
      rw_variant = rw_rows == 8 ? 1 : rw_rows == 5 ? 2 : rw_rows == 29 ? 3 : 0;
      LCS_TRY(init_rw_maps());
    }
    zchunk_force = zchunk;
    sm_share = share;
    tuning_gen++;
    drop_graphs();
    return LCS_OK;
  }
  void drop_graphs() {
    if (step_exec) cudaGraphExecDestroy(step_exec);
    if (step_graph) cudaGraphDestroy(step_graph);
    if (evolve_exec) cudaGraphExecDestroy(evolve_exec);
    if (evolve_graph) cudaGraphDestroy(evolve_graph);
    step_exec = nullptr;
    step_graph = nullptr;
    evolve_exec = nullptr;
    evolve_graph = nullptr;
  }

  // Asynchronous steps (the batch and the server drive many handles at once):
  // step_begin enqueues nsteps graph replays of the step, then copies of the
  // context and of those steps' log entries into pinned memory, and an event;
  // step_poll tests the event; step_finish waits for it and returns the logs.
  int step_begin(int nsteps) override {
    LCS_TRY(check_flow());
    if (async_pending) return fail(LCS_ESTATE, "steps are already in flight on this handle");
    if (nsteps < 1 || nsteps > plan.logs_cap) return fail(LCS_EINVAL, "nsteps must be in 1..%lld", (long long)plan.logs_cap);
    if (prof) return fail(LCS_ESTATE, "asynchronous steps do not run with profiling on");
    if (!host_step_known) LCS_TRY(read_ctx());
    LCS_TRY(build_step_graph());
    for (int q = 0; q < nsteps; q++) {
      LCS_CUDA(cudaGraphLaunch(step_exec, stream));
      launches += graph_launches_per_step;
      LCS_TRY(sort_after(host_step + q + 1));
    }
    return async_tail(nsteps);
  }
  // After nsteps enqueued steps: the context and the steps' logs back into
  // pinned memory, and the event step_poll/step_finish wait for.
  int async_tail(int nsteps) {
    LCS_TRY(copy(hctx, dctx, sizeof(Ctx), cudaMemcpyDeviceToHost));
    const int64_t cap = plan.logs_cap, i0 = host_step % cap;  // ring index of step host_step + 1
    const int64_t n1 = std::min<int64_t>(nsteps, cap - i0);
    LCS_TRY(copy(hlogs + i0, dlogs + i0, (size_t)n1 * sizeof(StepLog), cudaMemcpyDeviceToHost));
    if (n1 < nsteps) LCS_TRY(copy(hlogs, dlogs, (size_t)(nsteps - n1) * sizeof(StepLog), cudaMemcpyDeviceToHost));
    LCS_CUDA(cudaEventRecord(async_ev, stream));
    async_pending = nsteps;
    return LCS_OK;
  }
  // checks of a handle before steps are enqueued for it (alone or in a group)
  int async_ready(int nsteps) {
    LCS_TRY(check_flow());
    if (async_pending) return fail(LCS_ESTATE, "steps are already in flight on this handle");
    if (nsteps < 1 || nsteps > plan.logs_cap) return fail(LCS_EINVAL, "nsteps must be in 1..%lld", (long long)plan.logs_cap);
    if (prof) return fail(LCS_ESTATE, "asynchronous steps do not run with profiling on");
    if (!host_step_known) LCS_TRY(read_ctx());
    return LCS_OK;
  }
  int group_create(EngineBase* const* members, int m, GroupBase** out) override;
  const lcs_config& config() const override { return cfg; }
  int step_poll(int* done) override {
    if (!done) return fail(LCS_EINVAL, "null output");
    if (!async_pending) return fail(LCS_ESTATE, "no steps in flight on this handle");
    const cudaError_t q = cudaEventQuery(async_ev);
    if (q == cudaErrorNotReady) {
      *done = 0;
      return LCS_OK;
    }
    LCS_CUDA(q);
    *done = 1;
    return LCS_OK;
  }
  int step_finish(lcs_log* logs) override {
    if (!async_pending) return fail(LCS_ESTATE, "no steps in flight on this handle");
    const int n = async_pending;
    async_pending = 0;
    LCS_CUDA(cudaEventSynchronize(async_ev));
    if (hctx->wait_error) return fail(LCS_ETIMEDOUT, "a bounded device wait (TMA tile load or grid barrier) ran out");
    if (hctx->nonfinite) return fail(LCS_ENONFINITE, "non-finite residual or dt near step %lld", (long long)hctx->step);
    if (hctx->step != host_step + n) return fail(LCS_ECUDA, "step counter %lld, expected %lld", (long long)hctx->step,
                                                 (long long)(host_step + n));
    if (logs)
      for (int q = 0; q < n; q++) fill_log(hlogs[(host_step + q) % plan.logs_cap], &logs[q]);
    host_step += n;
    return LCS_OK;
  }

  int step_impl(int nsteps, lcs_log* logs, double* ms) {
    LCS_TRY(check_flow());
    if (async_pending) return fail(LCS_ESTATE, "asynchronous steps are in flight on this handle");
    if (nsteps < 0) return fail(LCS_EINVAL, "nsteps < 0");
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (ms) {
      LCS_CUDA(cudaEventCreate(&e0));
      LCS_CUDA(cudaEventCreate(&e1));
    }
    int rc2 = step_body(nsteps, logs, e0, e1);
    if (ms && rc2 == LCS_OK) {
      float f = 0.f;
      cudaEventElapsedTime(&f, e0, e1);
      *ms = f;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    return rc2;
  }
  // Records e0 before the first step and e1 after the last one (if given).
  int step_body(int nsteps, lcs_log* logs, cudaEvent_t e0, cudaEvent_t e1) {
    const bool graphs = cfg.use_graphs && !prof;
    if (graphs) LCS_TRY(build_step_graph());
    if (sort_interval > 0 && !host_step_known) LCS_TRY(read_ctx());
    if (e0) LCS_CUDA(cudaEventRecord(e0, stream));
    if (!graphs) {
      for (int q = 0; q < nsteps; q++) {
        LCS_TRY(timestep_kernels(0, nullptr));
        LCS_TRY(evolve_kernels(true));
        LCS_TRY(launch("step_end", k_step_end, dim3(1), dim3(1), 0, dctx, (StepLog*)nullptr, 1));
        if (e1 && q == nsteps - 1) LCS_CUDA(cudaEventRecord(e1, stream));
        LCS_TRY(collect_profile());
        LCS_TRY(read_ctx());
        if (hctx->wait_error) return fail(LCS_ETIMEDOUT, "a bounded device wait (TMA tile load or grid barrier) ran out");
        if (hctx->nonfinite) return fail(LCS_ENONFINITE, "non-finite residual or dt at step %lld", (long long)hctx->step);
        if (logs) fill_log(hctx->cur, &logs[q]);
        LCS_TRY(sort_after(hctx->step));
      }
      if (e1 && nsteps == 0) LCS_CUDA(cudaEventRecord(e1, stream));
      return LCS_OK;
    }
    int done = 0;
    if (nsteps == 0 && e1) LCS_CUDA(cudaEventRecord(e1, stream));
    while (done < nsteps) {
      const int chunk = std::min<int>(nsteps - done, (int)plan.logs_cap);
      for (int q = 0; q < chunk; q++) {
        LCS_CUDA(cudaGraphLaunch(step_exec, stream));
        launches += graph_launches_per_step;
        LCS_TRY(sort_after(host_step + q + 1));  // host_step: the counter before this chunk
      }
      if (e1 && done + chunk == nsteps) LCS_CUDA(cudaEventRecord(e1, stream));
      LCS_TRY(read_ctx());
      if (hctx->wait_error) return fail(LCS_ETIMEDOUT, "a bounded device wait (TMA tile load or grid barrier) ran out");
      if (hctx->nonfinite) return fail(LCS_ENONFINITE, "non-finite residual or dt near step %lld", (long long)hctx->step);
      if (logs) {
        std::vector<StepLog> hl(chunk);
        for (int q = 0; q < chunk; q++) {
          const long long st = hctx->step - chunk + q + 1;
          LCS_TRY(copy(&hl[q], dlogs + (st - 1) % plan.logs_cap, sizeof(StepLog), cudaMemcpyDeviceToHost));
        }
        LCS_CUDA(cudaStreamSynchronize(stream));
        for (int q = 0; q < chunk; q++) fill_log(hl[q], &logs[done + q]);
      }
      done += chunk;
    }
    return LCS_OK;
  }

  int synchalo(int mask, int r, int full) override {
    if (r < 0 || r > g.h) return fail(LCS_EINVAL, "halo width out of range");
    const bool us = mask & 7, us2 = (mask >> 3) & 7, withP = (mask >> LCS_FIELD_P) & 1;
    if (us) LCS_TRY(fill(kSetUs, false, r, full));
    if (us2) LCS_TRY(fill(kSetUs2, false, r, full));
    if (withP) LCS_TRY(fill(-1, true, r, full));
    LCS_CUDA(cudaStreamSynchronize(stream));
    return LCS_OK;
  }
  int rhs(int stage) override {
    LCS_TRY(check_stage(stage));
    LCS_TRY(rhs_kernel(stage == 1 ? kSetUs : kSetUs2, 0, 0, 0, 0.0));
    LCS_TRY(collect_profile());
    LCS_CUDA(cudaStreamSynchronize(stream));
    return LCS_OK;
  }
  int update(int stage, double dtrk) override {
    LCS_TRY(check_stage(stage));
    dim3 grid((g.n[0] + 127) / 128, g.n[1], g.n[2]);
    LCS_TRY(launch("update", k_update<T>, grid, dim3(128), 0, (const Ctx*)dctx, g, stage == 1 ? (int)kSetUs2 : (int)kSetUs,
                   (int)kSetUs, (const T*)dU[0], (const T*)dU[1], (const T*)dU[2], dtrk));
    LCS_CUDA(cudaStreamSynchronize(stream));
    return LCS_OK;
  }
  int rhs_update(int stage, double dtrk) override {
    LCS_TRY(check_stage(stage));
    LCS_TRY(rhs_kernel(stage == 1 ? kSetUs : kSetUs2, stage == 1 ? kSetUs2 : kSetUs, 1, 0, dtrk));
    LCS_TRY(collect_profile());
    LCS_CUDA(cudaStreamSynchronize(stream));
    return LCS_OK;
  }
  int couple(int stage, double dtrk, lcs_couple_log* log) override {
    LCS_TRY(check_stage(stage));
    LCS_TRY(set_scalar(&dctx->scal[0], dtrk));
    LCS_TRY(couple_direct(stage));
    LCS_TRY(collect_profile());
    LCS_TRY(read_ctx());
    if (hctx->nonfinite) return fail(LCS_ENONFINITE, "HSMAC residual is not finite");
    if (log) {
      log->itr = hctx->cs.itr;
      log->sweeps = hctx->cs.sweeps;
      log->div = hctx->cs.div;
    }
    return LCS_OK;
  }
  int forcing(double dtrk, double* p, double* e10) override {
    LCS_TRY(set_scalar(&dctx->scal[0], dtrk));
    LCS_TRY(launch("step_begin", k_step_begin, dim3(1), dim3(1), 0, dctx));
    LCS_TRY(forcing_stage());
    LCS_TRY(collect_profile());
    LCS_TRY(read_ctx());
    if (p) *p = hctx->cur.p;
    if (e10) *e10 = hctx->cur.e10;
    return LCS_OK;
  }
  int flow_timestep(double* dt) override {
    LCS_TRY(timestep_kernels(1, stage));
    LCS_TRY(copy(&hctx->scal[7], stage, sizeof(double), cudaMemcpyDeviceToHost));
    LCS_CUDA(cudaStreamSynchronize(stream));
    if (dt) *dt = hctx->scal[7];
    return LCS_OK;
  }
  int flow_stat(lcs_flow_stats* out) override {
    LCS_TRY(check_flow());
    if (async_pending) return fail(LCS_ESTATE, "asynchronous steps are in flight on this handle");
    if (!out) return fail(LCS_EINVAL, "null output");
    const int64_t total = (int64_t)g.n[0] * g.n[1] * g.n[2];
    const unsigned int nb = blocks_for(total, 256, 148 * 8);
    LCS_TRY(launch("flow_stat", k_flow_stat<T>, dim3(nb), dim3(256), 0, (const Ctx*)dctx, g, hc.dxi, hc.dyi, hc.dzi,
                   partials));
    LCS_TRY(launch("flow_stat_final", k_flow_stat_final, dim3(1), dim3(256), 0, (const double*)partials, (int)nb,
                   stage));
    double v[kStatVals];
    LCS_TRY(copy(v, stage, sizeof v, cudaMemcpyDeviceToHost));
    LCS_TRY(collect_profile());
    LCS_CUDA(cudaStreamSynchronize(stream));
    const double N = (double)total;
    lcs_flow_stats& o = *out;
    o.u_mean = v[5] / N; o.v_mean = v[6] / N; o.w_mean = v[7] / N;
    o.u_max = v[8]; o.v_max = v[9]; o.w_max = v[10];
    o.u_min = v[11]; o.v_min = v[12]; o.w_min = v[13];
    const double u2 = v[0] / N, s2 = v[1] / N, d2 = v[2] / N, d3 = v[3] / N, d4 = v[4] / N;
    const double Re = cfg.U0 * cfg.L0 / cfg.NU;  // Flows.Re(params)
    // stat.jl:135-151
    o.urms = std::sqrt(u2 / 3.0);
    o.k = 0.5 * (u2 - o.u_mean * o.u_mean - o.v_mean * o.v_mean - o.w_mean * o.w_mean);
    o.epsilon = s2 / Re;
    o.tau_eta = std::sqrt(1.0 / o.epsilon / Re);
    o.l_mu = std::sqrt(15.0 * o.urms * o.urms / o.epsilon / Re);
    o.l_eta = std::pow(1.0 / o.epsilon / (Re * Re * Re), 0.25);
    o.Re_lambda = o.l_mu * o.urms * Re;
    o.k_eta = (std::min(g.n[0], std::min(g.n[1], g.n[2])) / 2.0) * o.l_eta;
    o.skewness = -d3 / std::pow(d2, 1.5);
    o.flatness = d4 / (d2 * d2);
    o.L = 0.0;
    o.C_epsilon = 0.0;
    return LCS_OK;
  }
  // test hook: makes the bounded device waits of one kind unreachable
  // (Ctx::debug_wait), so that the next launch that waits runs its limit out
  int debug_waits(int kind) override {
    if (kind < 0 || kind > 2) return fail(LCS_EINVAL, "debug wait kind must be 0, 1 or 2");
    if (async_pending) return fail(LCS_ESTATE, "asynchronous steps are in flight on this handle");
    LCS_TRY(launch("set_debug_wait", k_set_debug_wait, dim3(1), dim3(1), 0, dctx, kind));
    LCS_CUDA(cudaStreamSynchronize(stream));
    return LCS_OK;
  }
  // divergence of the current velocity (diagnostic): RMS and max over n^3
  int flow_divergence(double* rms, double* maxabs) override {
    LCS_TRY(check_flow());
    if (async_pending) return fail(LCS_ESTATE, "asynchronous steps are in flight on this handle");
    const int64_t total = (int64_t)g.n[0] * g.n[1] * g.n[2];
    const unsigned int nb = blocks_for(total, 256, 148 * 8);
    LCS_TRY(launch("div_stat", k_div_stat<T>, dim3(nb), dim3(256), 0, (const Ctx*)dctx, g, hc.dxi, hc.dyi, hc.dzi,
                   partials));
    LCS_TRY(launch("div_stat_final", k_div_stat_final, dim3(1), dim3(256), 0, (const double*)partials, (int)nb, stage));
    double v[2];
    LCS_TRY(copy(v, stage, sizeof v, cudaMemcpyDeviceToHost));
    LCS_TRY(collect_profile());
    LCS_CUDA(cudaStreamSynchronize(stream));
    if (rms) *rms = std::sqrt(v[0] / (double)total);
    if (maxabs) *maxabs = v[1];
    return LCS_OK;
  }
  static void free_index(CellIndex& c) {
    cudaFree(c.hashes);
    cudaFree(c.starts);
    cudaFree(c.S);
    cudaFree(c.kv);
    cudaFree(c.temp);
    c = CellIndex{};
  }
  // a device-timed span of library calls under a label (when profiling)
  template <typename F>
  int timed(const char* label, F&& f) {
    cudaEvent_t a = nullptr, b = nullptr;
    if (prof && !capturing) {
      a = get_event();
      b = get_event();
      cudaEventRecord(a, stream);
    }
    cudaError_t e = f();
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return fail(LCS_ECUDA, "%s: %s", label, cudaGetErrorString(e));
    if (a) {
      cudaEventRecord(b, stream);
      recs.push_back({label, a, b});
    }
    return LCS_OK;
  }
  // `Particles.makeindex!` (src/particles/makeindex.jl:29-67) on species s
  // with the positions of `stage`; the species' device order becomes the
  // sorted one.
  int particles_makeindex(int s, int stage_, int ratio) override {
    LCS_TRY(check_species(s));
    LCS_TRY(check_stage(stage_));
    if (async_pending) return fail(LCS_ESTATE, "asynchronous steps are in flight on this handle");
    LCS_TRY(index_alloc(s, ratio));
    LCS_TRY(makeindex_enqueue(s, stage_));
    LCS_TRY(collect_profile());
    LCS_CUDA(cudaStreamSynchronize(stream));
    return LCS_OK;
  }
  // Cell geometry and buffers of species s's index for this grid_ratio
  // (allocated when the ratio changes: the stream is synchronised first).
  int index_alloc(int s, int ratio) {
    if (ratio < 1 || g.n[0] % ratio || g.n[1] % ratio || g.n[2] % ratio)
      return fail(LCS_EINVAL, "grid_ratio must be positive and divide the grid dims");
    CellIndex& c = ci[s];
    const int64_t n = sp[s].n;
    CellGeom cg;
    int64_t H = 1;
    for (int a = 0; a < 3; a++) {
      cg.nc[a] = g.n[a] / ratio;
      cg.dxc[a] = (kDomainLength / g.n[a]) * ratio;  // LCS.spacings(grid) .* grid_ratio
      H *= cg.nc[a] + 2;
    }
    if (H >= (int64_t)INT32_MAX || n > (int64_t)INT32_MAX) return fail(LCS_EINVAL, "cell index too large");  // 32-bit sort and scan sizes
    if (c.ratio != ratio) {  // (re)allocate for this cell size
      LCS_CUDA(cudaStreamSynchronize(stream));
      free_index(c);
      const size_t nn = (size_t)std::max<int64_t>(n, 1);
      LCS_CUDA(cudaMalloc(&c.hashes, nn * sizeof(int64_t)));
      LCS_CUDA(cudaMalloc(&c.starts, (size_t)2 * H * sizeof(int64_t)));
      LCS_CUDA(cudaMalloc(&c.S, (size_t)2 * (H + 1) * sizeof(int64_t)));
      LCS_CUDA(cudaMalloc(&c.kv, 4 * nn * sizeof(uint32_t)));
      if (!sp_alloc[s]) {
        LCS_CUDA(cudaMalloc(&sp_alloc[s], (size_t)kSortedProps * nn * sizeof(uint64_t)));
        sp_spare[s] = sp_alloc[s];
      }
      size_t sort_bytes = 0, scan_bytes = 0;
      LCS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, c.kv, c.kv + n, c.kv + 2 * n, c.kv + 3 * n,
                                               (int)n, 0, 32, stream));
      LCS_CUDA(cub::DeviceScan::InclusiveScan(nullptr, scan_bytes, c.S, c.S + H + 1, MaxI64(), (int)(H + 1),
                                              stream));
      c.temp_bytes = std::max<size_t>(std::max(sort_bytes, scan_bytes), 1);
      LCS_CUDA(cudaMalloc(&c.temp, c.temp_bytes));
      c.ratio = ratio;
    }
    c.cg = cg;
    c.H = H;
    return LCS_OK;
  }
  // The index of species s on the stream (after index_alloc): hashes of the
  // positions of stage_, the stable sort, the permutation of every property,
  // starts and stops.  Nothing waits for the stream.
  int makeindex_enqueue(int s, int stage_) {
    CellIndex& c = ci[s];
    const int64_t n = sp[s].n, H = c.H;
    const CellGeom cg = c.cg;
    cudaEvent_t span = nullptr;  // the whole index, device-timed when profiling
    if (prof && !capturing) {
      span = get_event();
      cudaEventRecord(span, stream);
    }
    int end_bit = 1;
    while (end_bit < 32 && ((int64_t)1 << end_bit) <= H) end_bit++;
    const int pos = stage_ == 1 ? LCS_PROP_X : LCS_PROP_X2;
    const unsigned int nb = blocks_for(n, 256, 148 * 16);
    uint32_t *kin = c.kv, *kout = c.kv + n, *vin = c.kv + 2 * n, *vout = c.kv + 3 * n;
    LCS_TRY(launch("cell_hash", k_cell_hash, dim3(nb), dim3(256), 0, (const double*)sp[s].p[pos],
                   (const double*)sp[s].p[pos + 1], (const double*)sp[s].p[pos + 2], n, cg, kin, vin));
    // a stable LSD radix sort of (hash, index): equal hashes keep their order
    LCS_TRY(timed("radix_sort", [&] {
      size_t tb = c.temp_bytes;
      return cub::DeviceRadixSort::SortPairs(c.temp, tb, kin, kout, vin, vout, (int)n, 0, end_bit, stream);
    }));
    // every property (16 FP64 ones and the ids, back to back from p[0]) in
    // the sorted order into the spare block, which becomes the species' block
    uint64_t* block = (uint64_t*)sp[s].p[0];
    LCS_TRY(launch("permute", k_permute_props, dim3(nb), dim3(256), 0, (const uint64_t*)block, (const uint32_t*)vout,
                   n, sp_spare[s]));
    for (int q = 0; q < 16; q++) sp[s].p[q] = (double*)sp_spare[s] + (size_t)q * n;
    sp_spare[s] = block;
    LCS_TRY(launch("species_base", k_set_species_base, dim3(1), dim3(1), 0, dctx, s, sp[s].p[0]));
    LCS_CUDA(cudaMemsetAsync(c.S, 0, (size_t)(H + 1) * sizeof(int64_t), stream));
    LCS_TRY(launch("hash_runs", k_hash_runs, dim3(nb), dim3(256), 0, (const uint32_t*)kout, n, H, c.hashes, c.S));
    LCS_TRY(timed("run_scan", [&] {
      size_t tb = c.temp_bytes;
      return cub::DeviceScan::InclusiveScan(c.temp, tb, c.S, c.S + H + 1, MaxI64(), (int)(H + 1), stream);
    }));
    LCS_TRY(launch("starts_stops", k_starts_stops, dim3(blocks_for(H, 256, 148 * 16)), dim3(256), 0,
                   (const int64_t*)(c.S + H + 1), H, c.starts, c.starts + H));
    if (span) {
      cudaEvent_t b = get_event();
      cudaEventRecord(b, stream);
      recs.push_back({"makeindex", span, b});
    }
    c.built = true;
    return LCS_OK;
  }

  // Particle sort (no reference counterpart): every sort_interval-th step of
  // lcs_step / lcs_step_begin is followed by makeindex! of every species on
  // its positions, so that the fluid gathers of the next steps read
  // neighbouring cells together.  Each particle's arithmetic does not depend
  // on its place in the arrays, so only the order changes (ids follow).
  int sort_interval = 0, sort_ratio = 0;
  int set_particle_sort(int interval, int ratio) override {
    if (async_pending) return fail(LCS_ESTATE, "asynchronous steps are in flight on this handle");
    if (interval < 0) return fail(LCS_EINVAL, "interval < 0");
    if (interval > 0) {
      if (cfg.mode != LCS_MODE_FLOW_PARTICLE || cfg.n_species < 1)
        return fail(LCS_EINVAL, "the particle sort needs the flow-particle mode");
      for (int s = 0; s < cfg.n_species; s++) LCS_TRY(index_alloc(s, ratio));  // buffers before any step
    }
    sort_interval = interval;
    sort_ratio = ratio;
    return LCS_OK;
  }
  // after the step that brought the step counter to `step`
  int sort_after(int64_t step) {
    if (sort_interval <= 0 || step % sort_interval != 0) return LCS_OK;
    for (int s = 0; s < cfg.n_species; s++) {
      LCS_TRY(index_alloc(s, sort_ratio));  // a no-op unless a stat changed the ratio
      LCS_TRY(makeindex_enqueue(s, 1));
    }
    return LCS_OK;
  }
  int particles_cellindex(int s, int64_t* hashes, int64_t* starts, int64_t* stops) override {
    LCS_TRY(check_species(s));
    if (!ci[s].built) return fail(LCS_ESTATE, "no cell index built for species %d", s);
    const CellIndex& c = ci[s];
    if (hashes) LCS_TRY(copy(hashes, c.hashes, (size_t)sp[s].n * 8, cudaMemcpyDeviceToHost));
    if (starts) LCS_TRY(copy(starts, c.starts, (size_t)c.H * 8, cudaMemcpyDeviceToHost));
    if (stops) LCS_TRY(copy(stops, c.starts + c.H, (size_t)c.H * 8, cudaMemcpyDeviceToHost));
    LCS_CUDA(cudaStreamSynchronize(stream));
    return LCS_OK;
  }
  int ensure_pbuf(size_t bytes) {
    if (bytes <= pbuf_bytes) return LCS_OK;
    LCS_CUDA(cudaStreamSynchronize(stream));
    cudaFree(pbuf);
    pbuf = nullptr;
    pbuf_bytes = 0;
    LCS_CUDA(cudaMalloc(&pbuf, bytes));
    pbuf_bytes = bytes;
    return LCS_OK;
  }
  // `Particles.stat` (src/particles/stat.jl:113-151)
  int particles_stat(int s, const lcs_particle_stat_config* pc, double tau_eta, lcs_particle_stats* out) override {
    LCS_TRY(check_species(s));
    if (!pc || !out) return fail(LCS_EINVAL, "null config or output");
    if (async_pending) return fail(LCS_ESTATE, "asynchronous steps are in flight on this handle");
    const int nbins = pc->bin_size, ns = pc->nsamples;
    if (nbins < 1 || nbins > LCS_RDF_MAX_BINS) return fail(LCS_EINVAL, "bin_size must be 1..%d", LCS_RDF_MAX_BINS);
    if (ns < 2 || ns > LCS_SPECTRUM_MAX_SAMPLES) return fail(LCS_EINVAL, "nsamples must be 2..%d", LCS_SPECTRUM_MAX_SAMPLES);
    if (pc->search_cell_size < 0 || pc->search_cell_size > 64) return fail(LCS_EINVAL, "search_cell_size must be 0..64");
    if (!(pc->min_radius > 0.0)) return fail(LCS_EINVAL, "min_radius must be positive");
    const int64_t n = sp[s].n;
    const double* P[7] = {sp[s].p[LCS_PROP_X], sp[s].p[LCS_PROP_Y], sp[s].p[LCS_PROP_Z], sp[s].p[LCS_PROP_U],
                          sp[s].p[LCS_PROP_V], sp[s].p[LCS_PROP_W], sp[s].p[LCS_PROP_DIAM]};
    // Summary of xss, uss, diams (stat.jl:131-139)
    const unsigned int nbs = blocks_for(n, 256, 148 * 4);
    LCS_TRY(launch("psummary", k_psummary, dim3(nbs), dim3(256), 0, P[0], P[1], P[2], P[3], P[4], P[5], P[6], n,
                   partials));
    LCS_TRY(launch("psummary_final", k_psummary_final, dim3(1), dim3(256), 0, (const double*)partials, (int)nbs, stage));
    double v[kPSumVals];
    LCS_TRY(copy(v, stage, sizeof v, cudaMemcpyDeviceToHost));
    LCS_CUDA(cudaStreamSynchronize(stream));
    lcs_summary* S[7] = {&out->x, &out->y, &out->z, &out->u, &out->v, &out->w, &out->diam};
    for (int q = 0; q < 7; q++) {
      S[q]->mean = v[3 * q] / (double)n;
      S[q]->max = v[3 * q + 1];
      S[q]->min = v[3 * q + 2];
    }
    const double Re = cfg.U0 * cfg.L0 / cfg.NU;
    const double dm = out->diam.mean;
    out->taup = 1.0 / 18.0 * cfg.species[s].density_ratio * Re * (dm * dm);  // config.jl:41
    out->St = out->taup / tau_eta;
    LCS_TRY(particles_makeindex(s, 1, pc->grid_ratio));
    const CellIndex& c = ci[s];
    // rdf_assume_ci (rdf.jl:1-103)
    const double hmin = std::min(kDomainLength / g.n[0], std::min(kDomainLength / g.n[1], kDomainLength / g.n[2]));
    const double rmax = pc->search_cell_size * hmin;
    out->nbins = nbins;
    lcs_logrange(pc->min_radius, rmax, nbins + 1, out->edges);
    const size_t need = (size_t)(nbins + 1) * 16;  // edges, then the counters
    const int nshells = spectrum_shells(pc->max_wavenumber);
    const int npairs = nshells * ns;
    const unsigned int nbx = 148 * 2;
    const size_t spec_bytes = (size_t)npairs * 3 * 8 + (size_t)nbx * npairs * 2 * 8 + (size_t)npairs * 2 * 8;
    LCS_TRY(ensure_pbuf(need + spec_bytes + 64));
    double* d_edges = (double*)pbuf;
    unsigned long long* d_counts = (unsigned long long*)(pbuf + (size_t)(nbins + 1) * 8);
    LCS_TRY(copy(d_edges, out->edges, (size_t)(nbins + 1) * 8, cudaMemcpyHostToDevice));
    LCS_CUDA(cudaMemsetAsync(d_counts, 0, (size_t)(nbins + 1) * 8, stream));
    const size_t rdf_smem = (size_t)(nbins + 1) * 16;
    LCS_TRY(launch("rdf", k_rdf, dim3(blocks_for(n, 256, 148 * 8)), dim3(256), rdf_smem, (const double*)sp[s].p[0],
                   (const double*)sp[s].p[1], (const double*)sp[s].p[2], (const int64_t*)(sp[s].p[0] + 16 * n),
                   (const int64_t*)c.hashes, (const int64_t*)c.starts, (const int64_t*)(c.starts + c.H), n, c.cg,
                   pc->search_cell_size, (const double*)d_edges, nbins, dm, pc->contact_tolerance, d_counts));
    std::vector<unsigned long long> counts(nbins + 1);
    LCS_TRY(copy(counts.data(), d_counts, (size_t)(nbins + 1) * 8, cudaMemcpyDeviceToHost));
    // the spectrum (spectrum.jl:11-78)
    std::vector<double> kvec((size_t)npairs * 3 + 1), sums((size_t)npairs * 2 + 1);
    out->nshells = nshells;
    spectrum_directions(nshells, ns, kvec.data(), out->wavenumbers);
    if (npairs > 0) {
      double* d_k = (double*)(pbuf + need);
      double* d_part = d_k + (size_t)npairs * 3;
      double* d_sums = d_part + (size_t)nbx * npairs * 2;
      LCS_TRY(copy(d_k, kvec.data(), (size_t)npairs * 3 * 8, cudaMemcpyHostToDevice));
      const unsigned int nby = (unsigned)((npairs + 256 * kSpecPairs - 1) / (256 * kSpecPairs));
      LCS_TRY(launch("spectrum", k_spectrum, dim3(nbx, nby), dim3(256), 0, (const double*)sp[s].p[0],
                     (const double*)sp[s].p[1], (const double*)sp[s].p[2], n, (const double*)d_k, npairs, d_part));
      LCS_TRY(launch("spectrum_final", k_spectrum_final, dim3((unsigned)((2 * npairs + 255) / 256)), dim3(256), 0,
                     (const double*)d_part, (int)nbx, npairs, d_sums));
      LCS_TRY(copy(sums.data(), d_sums, (size_t)npairs * 2 * 8, cudaMemcpyDeviceToHost));
    }
    LCS_TRY(collect_profile());
    LCS_CUDA(cudaStreamSynchronize(stream));
    // host finish: rdf.jl:80-100, spectrum.jl:63-75, in the reference's order
    const double L = kDomainLength;
    const double vol = L * L * L;
    const double rho0 = (double)(n * (n - 1) / 2) / vol;
    for (int k = 0; k < nbins; k++) {
      const double e0 = out->edges[k], e1 = out->edges[k + 1];
      const double vol_shell = (4.0 / 3.0) * M_PI * (e1 * e1 * e1 - e0 * e0 * e0);
      out->npairs[k] = (int64_t)counts[k];
      out->gr[k] = ((double)counts[k] / vol_shell) / rho0;
    }
    out->npairs_contact = (int64_t)counts[nbins];
    const double vol_contact = (4.0 / 3.0) * M_PI * (dm * dm * dm) * 6.0 * pc->contact_tolerance;
    out->gr_contact = ((double)counts[nbins] / vol_contact) / rho0;
    const double N2 = (double)(n * n);
    for (int b = 0; b < nshells; b++) {
      double phi = 0.0;
      for (int i = 0; i < ns; i++) {
        const double cc = sums[2 * (b * ns + i)], ss = sums[2 * (b * ns + i) + 1];
        phi += (cc * cc + ss * ss) / N2 - 1.0 / (double)n;
      }
      const double kk = out->wavenumbers[b];
      out->Enp[b] = phi / ns * 4.0 * M_PI * (kk * kk);
    }
    return LCS_OK;
  }
  static int spectrum_shells(int max_wavenumber) {
    int c = 0;
    while (c < LCS_SPECTRUM_MAX_SHELLS && kWavenumbers[c] <= max_wavenumber) c++;
    return c;  // Utils.searchsortedlast(WAVENUMBERS, max_wavenumber)
  }
  // k = kk .* _fibonacci_direction(i, nsamples) (spectrum.jl:3-9, 37-38)
  static void spectrum_directions(int nshells, int ns, double* kvec, double* wavenumbers) {
    const double phi = M_PI * (3.0 - std::sqrt(5.0));
    for (int b = 0; b < nshells; b++) {
      const double kk = kWavenumbers[b];
      wavenumbers[b] = kk;
      for (int i = 0; i < ns; i++) {
        const double y = 1.0 - ((double)i / (double)(ns - 1)) * 2.0;
        const double radius = std::sqrt(1.0 - y * y);
        const double theta = phi * i;
        double* k = kvec + 3 * ((size_t)b * ns + i);
        k[0] = kk * (std::cos(theta) * radius);
        k[1] = kk * y;
        k[2] = kk * (std::sin(theta) * radius);
      }
    }
  }
  static constexpr int kWavenumbers[LCS_SPECTRUM_MAX_SHELLS] = {1,  2,  3,   4,   6,   8,   12,  16,  24, 32,
                                                                48, 64, 96, 128, 192, 256, 384, 512, 768};
  // `Particles.density` (src/particles/stat.jl:176-215)
  int particles_density(int s, int ratio, double* densities) override {
    LCS_TRY(check_species(s));
    if (!densities) return fail(LCS_EINVAL, "null output");
    LCS_TRY(particles_makeindex(s, 1, ratio));
    const CellIndex& c = ci[s];
    const int64_t n = sp[s].n;
    const double h = std::min(kDomainLength / g.n[0], std::min(kDomainLength / g.n[1], kDomainLength / g.n[2]));
    const double factor = 1.0 / (M_PI * (h * h * h));
    LCS_TRY(ensure_pbuf((size_t)n * 8));
    LCS_TRY(launch("density", k_density, dim3(blocks_for(n, 256, 148 * 8)), dim3(256), 0, (const double*)sp[s].p[0],
                   (const double*)sp[s].p[1], (const double*)sp[s].p[2], (const int64_t*)c.hashes,
                   (const int64_t*)c.starts, (const int64_t*)(c.starts + c.H), n, c.cg, h, factor, (double*)pbuf));
    LCS_TRY(copy(densities, pbuf, (size_t)n * 8, cudaMemcpyDeviceToHost));
    LCS_TRY(collect_profile());
    LCS_CUDA(cudaStreamSynchronize(stream));
    return LCS_OK;
  }
  int particles_timestep(double* dt) override {
    LCS_TRY(read_ctx());
    if (dt) *dt = (cfg.mode == LCS_MODE_FLOW_PARTICLE && cfg.n_species > 0) ? hctx->dt_particles : cfg.dtmax;
    return LCS_OK;
  }
  int particles_boundary(int s, int stage) override {
    LCS_TRY(check_species(s));
    LCS_TRY(check_stage(stage));
    LCS_TRY(particles_stage(stage, 1, 0, 0.0, s));
    LCS_CUDA(cudaStreamSynchronize(stream));
    return LCS_OK;
  }
  int particles_motion(int s, int stage) override {
    LCS_TRY(check_species(s));
    LCS_TRY(check_stage(stage));
    LCS_TRY(particles_stage(stage, 2, 0, 0.0, s));
    LCS_CUDA(cudaStreamSynchronize(stream));
    return LCS_OK;
  }
  int particles_update(int s, int stage, double dtrk) override {
    LCS_TRY(check_species(s));
    LCS_TRY(check_stage(stage));
    LCS_TRY(particles_stage(stage, 4, 0, dtrk, s));
    LCS_CUDA(cudaStreamSynchronize(stream));
    return LCS_OK;
  }
  int init_particle_velocity(int s) override {
    LCS_TRY(check_species(s));
    LCS_TRY(fill(kSetUs, false, g.h, 1));
    if (sp[s].n > 0)
      LCS_TRY(launch("particles_init_velocity", k_particles_init_velocity<T>, dim3((unsigned)((sp[s].n + 255) / 256)),
                     dim3(256), 0, (const Ctx*)dctx, g, s, sp[s], pc));
    LCS_CUDA(cudaStreamSynchronize(stream));
    return LCS_OK;
  }

  int profile_enable(int on) override {
    prof = on != 0;
    return LCS_OK;
  }
  int profile_reset() override {
    LCS_TRY(collect_profile());
    totals.clear();
    launches = 0;
    return LCS_OK;
  }
  int profile_count(int* n) override {
    LCS_TRY(collect_profile());
    *n = (int)totals.size();
    return LCS_OK;
  }
  int profile_entry(int i, char* name, int cap, double* ms, int64_t* n) override {
    if (i < 0 || i >= (int)totals.size()) return fail(LCS_EINVAL, "profile index out of range");
    if (name && cap > 0) {
      strncpy(name, totals[i].label.c_str(), cap - 1);
      name[cap - 1] = 0;
    }
    if (ms) *ms = totals[i].ms;
    if (n) *n = totals[i].n;
    return LCS_OK;
  }
  int launch_count(int64_t* n) override {
    *n = launches;
    return LCS_OK;
  }
  int synchronize() override {
    LCS_CUDA(cudaStreamSynchronize(stream));
    return LCS_OK;
  }
};

// ---------------------------------------------------------------- batch group
// Handles of one shape (dims, halo, HSMAC settings, precision) and one set of
// launch shapes (tile rows, z chunk, GPU share) step as one CUDA graph on the
// first member's stream.  Each member's own kernels (time step, halo fill,
// particles, rhs/update, forcing, logs) are captured member after member;
// the HSMAC loop of each couple is one conditional WHILE node for the whole
// group whose body launches every sweep kernel once for all members
// (blockIdx.y = member): a member's blocks do exactly what its own launch
// does, so each member computes what it computes alone with the same launch
// shapes, and a member whose loop has ended returns at once.
template <typename T>
struct EngineGroup : GroupBase {
  std::vector<Engine<T>*> mem;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<int64_t> per_step;
  std::vector<int> gens;
  cudaEvent_t ready = nullptr;
  GroupMember<T>* gm = nullptr;  // the members' arguments of the group-wide launches (device)
  ~EngineGroup() override {
    if (mem.size()) cudaStreamSynchronize(mem[0]->stream);
    drop();
    if (ready) cudaEventDestroy(ready);
    if (gm) cudaFree(gm);
  }
  // The members' arguments for the group-wide launches, uploaded once.
  int member_args() {
    const int M = (int)mem.size();
    if (!gm) LCS_CUDA(cudaMalloc(&gm, (size_t)M * sizeof(GroupMember<T>)));
    std::vector<GroupMember<T>> h(M);
    memset(h.data(), 0, h.size() * sizeof(GroupMember<T>));
    for (int q = 0; q < M; q++) {
      Engine<T>* m = mem[q];
      GroupMember<T>& a = h[q];
      a.ctx = m->dctx;
      a.P = m->P;
      a.partials = m->partials;
      for (int c = 0; c < 3; c++) a.dU[c] = m->dU[c];
      a.logs = m->dlogs;
      a.logs_cap = (int)m->plan.logs_cap;
      a.itrmax = m->cfg.itrmax;
      a.nspecies = m->cfg.mode == LCS_MODE_FLOW_PARTICLE ? m->cfg.n_species : 0;
      a.rc = m->rc;
      a.dc = m->dc;
      a.pc = m->pc;
      a.power = m->cfg.power;
      for (int sp = 0; sp < a.nspecies; sp++) a.sp[sp] = m->sp[sp];
    }
    LCS_CUDA(cudaMemcpy(gm, h.data(), h.size() * sizeof(GroupMember<T>), cudaMemcpyHostToDevice));
    return LCS_OK;
  }
  // one-thread work of every member (k_member_op_group: 0 step_begin,
  // 1 set_stage_dt, 2 couple_reset, 3 couple_log, 4 step_end)
  int member_op(int what, int stage, const char* label) {
    const int M = (int)mem.size();
    return mem[0]->launch(label, k_member_op_group<T>, dim3((M + 63) / 64), dim3(64), 0, (const GroupMember<T>*)gm, M,
                          what, stage);
  }
  void drop() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  }
  int member_fail(Engine<T>* m, int rc) { return fail(rc, "%s", m->err.c_str()); }
#define LCS_GTRY(m, expr)                              \
  do {                                                 \
    int rc_ = (expr);                                  \
    if (rc_ != LCS_OK) return member_fail((m), rc_);   \
  } while (0)

  int couple_nodes(int stage) {
    Engine<T>* L = mem[0];
    const int set = stage == 1 ? kSetUs2 : kSetUs;
    LCS_GTRY(L, member_op(2, stage, "couple_reset"));
    cudaStream_t s = L->stream;
    cudaStreamCaptureStatus st;
    cudaGraph_t gr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    LCS_CUDA(cudaStreamGetCaptureInfo(s, &st, nullptr, &gr, &deps, &ndeps));
    if (st != cudaStreamCaptureStatusActive) return fail(LCS_ESTATE, "group couple outside a capture");
    cudaGraphConditionalHandle handle;
    LCS_CUDA(cudaGraphConditionalHandleCreate(&handle, gr, L->cfg.itrmax > 0 ? 1u : 0u, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    LCS_CUDA(cudaGraphAddNode(&node, gr, deps, ndeps, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    cudaStream_t side;
    LCS_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
    cudaError_t eb = cudaStreamBeginCaptureToGraph(side, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
    int rc2 = eb == cudaSuccess ? LCS_OK : fail(LCS_ECUDA, "capture of the group loop: %s", cudaGetErrorString(eb));
    if (rc2 == LCS_OK) {
      L->stream = side;
      L->grp = &mem;
      rc2 = L->couple_group(set);
      if (rc2 == LCS_OK)
        rc2 = L->launch("couple_continue", k_group_continue<T>, dim3(1), dim3(1), 0, L->grp_ptrs, (int)mem.size(),
                        handle, L->max_loop_groups());
      L->grp = nullptr;
      L->stream = s;
      if (rc2 != LCS_OK) rc2 = member_fail(L, rc2);
      cudaGraph_t body_out;
      cudaError_t e = cudaStreamEndCapture(side, &body_out);
      if (rc2 == LCS_OK && e != cudaSuccess) rc2 = fail(LCS_ECUDA, "capture of the group loop: %s", cudaGetErrorString(e));
    }
    cudaStreamDestroy(side);
    if (rc2 != LCS_OK) return rc2;
    LCS_CUDA(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    LCS_GTRY(L, member_op(3, stage, "couple_log"));
    return LCS_OK;
  }
  // One step of every member: each per-member kernel of Engine::timestep_kernels
  // and evolve_kernels as one group-wide launch (members' blocks side by side),
  // the couples as the group's WHILE loops.  The rc-energy forcing keeps one
  // launch sequence per member.
  int capture_step() {
    Engine<T>* L = mem[0];
    const int M = (int)mem.size();
    const Grid& g = L->g;
    const int64_t ni = (int64_t)g.n[0] * g.n[1] * g.n[2];
    const unsigned int nb = Engine<T>::blocks_for(ni, 256, 148 * 8);
    L->grp = &mem;
    // timestep!: FaceHalo fill, the CFL maxima and dt (flows/timestep.jl, timestep.jl)
    int rc2 = L->fill(kSetUs, false, g.h, 0);
    if (rc2 == LCS_OK)
      rc2 = L->launch("cfl_max", k_cfl_max_group<T>, dim3(nb, M), dim3(256), 0, (const GroupMember<T>*)gm, g);
    if (rc2 == LCS_OK)
      rc2 = L->launch("cfl_finalize", k_cfl_finalize_group<T>, dim3(M), dim3(256), 0, (const GroupMember<T>*)gm, (int)nb);
    L->grp = nullptr;
    LCS_GTRY(L, rc2);
    LCS_GTRY(L, member_op(0, 0, "step_begin"));
    bool lf = true, any_forcing = false;
    int nspec = 0;
    int64_t np_max = 0;
    for (auto* m : mem) {
      lf = lf && m->cfg.forcing == LCS_FORCING_LINEAR_POWER;
      any_forcing = any_forcing || m->cfg.forcing != LCS_FORCING_NO;
      if (m->cfg.mode == LCS_MODE_FLOW_PARTICLE) {
        nspec = std::max(nspec, (int)m->cfg.n_species);
        for (int q = 0; q < m->cfg.n_species; q++) np_max = std::max<int64_t>(np_max, m->sp[q].n);
      }
    }
    for (int stage = 1; stage <= 2; stage++) {
      const int set = stage == 1 ? kSetUs : kSetUs2;
      LCS_GTRY(L, member_op(1, stage, "stage_dt"));
      L->grp = &mem;
      rc2 = L->fill(set, true, g.h, 1);  // synchalo!(FullHalo(grid), (Us.., P))
      L->grp = nullptr;
      LCS_GTRY(L, rc2);
      for (int q = 0; q < nspec && np_max > 0; q++)  // boundary!, motion!, update! of species q of every member
        LCS_GTRY(L, L->launch("particles", k_particles_group<T>, dim3((unsigned)((np_max + 255) / 256), M), dim3(256), 0,
                              (const GroupMember<T>*)gm, g, q, stage, 7));
      LCS_GTRY(L, L->launch("rhs_update", k_rhs_group<T>, dim3((g.n[0] + 127) / 128, g.n[1], g.n[2] * M), dim3(128), 0,
                            (const GroupMember<T>*)gm, g, set, stage == 1 ? kSetUs2 : kSetUs, (int)kSetUs, 1, 1));
      if (stage == 2 && any_forcing) {
        if (lf) {  // forcing!(::ConstantPowerLF) of every member (lf.jl:27-106)
          L->grp = &mem;
          rc2 = L->fill(kSetUs, false, g.h, 1);
          L->grp = nullptr;
          LCS_GTRY(L, rc2);
          LCS_GTRY(L, L->launch("lf_sums", k_lf_sums_group<T>, dim3(nb, M), dim3(256), 0, (const GroupMember<T>*)gm, g));
          LCS_GTRY(L, L->launch("lf_coef", k_lf_coef_group<T>, dim3(M), dim3(256), 0, (const GroupMember<T>*)gm, (int)nb,
                                (double)ni));
          LCS_GTRY(L, L->launch("lf_apply", k_lf_apply_group<T>, dim3(nb, M), dim3(256), 0, (const GroupMember<T>*)gm, g));
          LCS_GTRY(L, L->launch("power_mean", k_power_finalize_group<T>, dim3(M), dim3(256), 0, (const GroupMember<T>*)gm,
                                (int)nb, (double)ni));
        } else {
          for (auto* m : mem) LCS_GTRY(m, m->forcing_stage());
        }
      }
      LCS_TRY(couple_nodes(stage));
    }
    LCS_GTRY(L, member_op(4, 0, "step_end"));
    return LCS_OK;
  }
#undef LCS_GTRY
  int build() {
    Engine<T>* L = mem[0];
    cudaStream_t s = L->stream;
    LCS_TRY(member_args());
    std::vector<cudaStream_t> saved(mem.size());
    LCS_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
    for (size_t q = 0; q < mem.size(); q++) {
      saved[q] = mem[q]->stream;
      mem[q]->stream = s;
      mem[q]->capturing = true;
      per_step[q] = mem[q]->launches;
    }
    int rc2 = capture_step();
    for (size_t q = 0; q < mem.size(); q++) {
      mem[q]->stream = saved[q];
      mem[q]->capturing = false;
      per_step[q] = mem[q]->launches - per_step[q];
      mem[q]->launches -= per_step[q];
    }
    cudaGraph_t gr = nullptr;
    cudaError_t e = cudaStreamEndCapture(s, &gr);
    if (rc2 != LCS_OK) {
      if (gr) cudaGraphDestroy(gr);
      return rc2;
    }
    if (e != cudaSuccess) return fail(LCS_ECUDA, "group graph capture: %s", cudaGetErrorString(e));
    graph = gr;
    LCS_CUDA(cudaGraphInstantiate(&exec, gr, 0));
    for (size_t q = 0; q < mem.size(); q++) gens[q] = mem[q]->tuning_gen;
    return LCS_OK;
  }
  int step_begin(int nsteps) override {
    for (auto* m : mem)
      if (int rc2 = m->async_ready(nsteps)) return member_fail(m, rc2);
    for (auto* m : mem)  // a member retuned alone since the group was made: its tiles no longer match
      if (m->rw_variant != mem[0]->rw_variant || m->zchunk_force != mem[0]->zchunk_force ||
          m->sm_share != mem[0]->sm_share)
        return fail(LCS_EINVAL, "group members differ in launch shapes");
    for (size_t q = 0; q < mem.size(); q++)
      if (gens[q] != mem[q]->tuning_gen) drop();
    if (!exec) LCS_TRY(build());
    Engine<T>* L = mem[0];
    cudaStream_t s = L->stream;
    for (size_t q = 1; q < mem.size(); q++) {  // the members' own earlier work first
      LCS_CUDA(cudaEventRecord(ready, mem[q]->stream));
      LCS_CUDA(cudaStreamWaitEvent(s, ready, 0));
    }
    for (int q = 0; q < nsteps; q++) {
      LCS_CUDA(cudaGraphLaunch(exec, s));
      for (auto* m : mem) {  // a member's particle sort, on the group's stream after the step
        if (m->sort_interval <= 0) continue;
        cudaStream_t own = m->stream;
        m->stream = s;
        const int rc2 = m->sort_after(m->host_step + q + 1);
        m->stream = own;
        if (rc2 != LCS_OK) return member_fail(m, rc2);
      }
    }
    for (size_t q = 0; q < mem.size(); q++) {
      Engine<T>* m = mem[q];
      m->launches += per_step[q] * nsteps;
      cudaStream_t own = m->stream;
      m->stream = s;
      const int rc2 = m->async_tail(nsteps);
      m->stream = own;
      if (rc2 != LCS_OK) return member_fail(m, rc2);
    }
    return LCS_OK;
  }
};

template <typename T>
int Engine<T>::group_create(EngineBase* const* members, int m, GroupBase** out) {
  *out = nullptr;
  if (m < 2 || m > kGroupPtrMax) return fail(LCS_EINVAL, "a group has 2..%d members", kGroupPtrMax);
  std::unique_ptr<EngineGroup<T>> gp(new EngineGroup<T>);
  for (int q = 0; q < m; q++) {
    Engine<T>* e = dynamic_cast<Engine<T>*>(members[q]);
    if (!e) return fail(LCS_EINVAL, "group member %d has another precision", q);
    for (auto* o : gp->mem)
      if (o == e) return fail(LCS_EINVAL, "group member %d appears twice", q);
    gp->mem.push_back(e);
  }
  Engine<T>* L = gp->mem[0];
  if (L != this) return fail(LCS_EINVAL, "the first member creates the group");
  for (auto* e : gp->mem) {
    const lcs_config &a = L->cfg, &b = e->cfg;
    const bool same = a.dims[0] == b.dims[0] && a.dims[1] == b.dims[1] && a.dims[2] == b.dims[2] &&
                      a.halo_size == b.halo_size && a.device == b.device && a.time_blocking == b.time_blocking &&
                      a.overlap == b.overlap && a.coloring == b.coloring && a.coloring_block == b.coloring_block &&
                      a.omega == b.omega && a.epsp == b.epsp && a.itrmin == b.itrmin && a.itrmax == b.itrmax;
    if (!same) return fail(LCS_EINVAL, "group members differ in shape or HSMAC settings");
    if (!e->use_rw) return fail(LCS_EINVAL, "group members need the row-warp sweep");
    if (e->rw_variant != L->rw_variant || e->zchunk_force != L->zchunk_force || e->sm_share != L->sm_share)
      return fail(LCS_EINVAL, "group members differ in launch shapes");
    if (e->async_pending) return fail(LCS_ESTATE, "asynchronous steps are in flight on a member");
    if (e->face_grid <= 0) return fail(LCS_EINVAL, "group members need the cooperative face kernel");
  }
  memset(&L->grp_ptrs, 0, sizeof L->grp_ptrs);
  for (int q = 0; q < m; q++) {
    L->grp_ptrs.ctx[q] = gp->mem[q]->dctx;
    L->grp_ptrs.P[q] = gp->mem[q]->P;
    L->grp_ptrs.partials[q] = gp->mem[q]->partials;
  }
  gp->per_step.assign(m, 0);
  gp->gens.assign(m, -1);
  LCS_CUDA(cudaEventCreateWithFlags(&gp->ready, cudaEventDisableTiming));
  *out = gp.release();
  return LCS_OK;
}

}  // namespace lcs
