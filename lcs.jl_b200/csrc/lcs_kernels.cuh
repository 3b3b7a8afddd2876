// lcs_kernels.cuh -- the CUDA kernels of the B200 time-step backend.
//
// Every kernel restates one step of the reference in the reference's own
// evaluation order; FP64 builds use --fmad=false so each element-wise result
// is bit-identical to the CPU restatement (Julia does not contract a*b+c).
// Reductions are deterministic (fixed per-block order, partials summed in
// index order by one block), so reruns are bit-reproducible.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "lcs_common.cuh"

namespace lcs {
// Kernels have internal linkage: each precision's translation unit carries
// its own copy.
namespace {

// --------------------------------------------------------------------------
// deterministic block reductions
// --------------------------------------------------------------------------
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* sh /* NT/32 */) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x / 32, l = threadIdx.x % 32;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0) {
    s = sh[0];
    for (int q = 1; q < NT / 32; q++) s += sh[q];
  }
  return s;  // valid in thread 0
}

template <int NT>
__device__ __forceinline__ double block_max(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v = jl_max(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int w = threadIdx.x / 32, l = threadIdx.x % 32;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0) {
    s = sh[0];
    for (int q = 1; q < NT / 32; q++) s = jl_max(s, sh[q]);
  }
  return s;
}

// Sum partials[0..n) in a fixed order with the whole block; result in thread 0.
template <int NT>
__device__ __forceinline__ double sum_partials(const double* partials, int n, double* sh) {
  double v = 0.0;
  for (int q = threadIdx.x; q < n; q += NT) v += __ldcg(&partials[q]);
  return block_sum<NT>(v, sh);
}

// Last-block-done: returns true in every thread of the block that finishes last.
__device__ __forceinline__ bool last_block(unsigned int* ticket, unsigned int nblocks, int* flag_sh) {
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int t = atomicAdd(ticket, 1u);
    *flag_sh = (t == nblocks - 1);
  }
  __syncthreads();
  return *flag_sh != 0;
}

// --------------------------------------------------------------------------
// periodic halo fill, single process (lib/topologies/src/halo.jl:138-159):
// every halo cell within r of the interior (all 26 directions, or the 6 face
// directions) receives the interior cell it wraps onto.
// --------------------------------------------------------------------------
struct FillArgs {
  int nf;           // number of fields
  int set[4];       // velocity set per field, or -1 when ptr[] is used
  int comp[4];
  void* ptr[4];     // direct pointer (P) when set < 0
};

template <typename T>
__device__ __forceinline__ void fill_halo_body(const Ctx* __restrict__ ctx, const Grid& g, const FillArgs& fa, int r,
                                               int full, int64_t total, T* Pm = nullptr) {
  const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
  const int wx = full ? nx + 2 * r : nx, wy = full ? ny + 2 * r : ny;
  const int bx = full ? 1 - r : 1, by = full ? 1 - r : 1;
  const int segA = 2 * r * wx * wy;  // z slabs
  const int segB = 2 * r * nz * wx;  // y slabs, k interior
  const int r2 = 2 * r;
  T* f[4];
#pragma unroll
  for (int q = 0; q < 4; q++)
    f[q] = q < fa.nf ? (T*)(fa.set[q] >= 0 ? ctx->vel[fa.set[q]][fa.comp[q]] : (Pm ? Pm : (T*)fa.ptr[q])) : nullptr;
  // total < 2^31 (checked on the host): 32-bit index arithmetic
  const int tot = (int)total;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += gridDim.x * blockDim.x) {
    int i, j, k;
    if (t < segA) {
      int u = t;
      i = bx + u % wx; u /= wx;
      j = by + u % wy; u /= wy;
      k = u < r ? 1 - r + u : nz + 1 + (u - r);
    } else if (t < segA + segB) {
      int u = t - segA;
      i = bx + u % wx; u /= wx;
      const int jj = u % r2; u /= r2;
      k = 1 + u;
      j = jj < r ? 1 - r + jj : ny + 1 + (jj - r);
    } else {
      int u = t - segA - segB;
      const int ii = u % r2; u /= r2;
      j = 1 + u % ny; u /= ny;
      k = 1 + u;
      i = ii < r ? 1 - r + ii : nx + 1 + (ii - r);
    }
    const int64_t dst = g.at(i, j, k), src = g.at(wrap1(i, nx), wrap1(j, ny), wrap1(k, nz));
    // every source is an interior cell and every destination a halo cell:
    // all loads go out before the stores
    T v[4];
#pragma unroll
    for (int q = 0; q < 4; q++)
      if (q < fa.nf) v[q] = f[q][src];
#pragma unroll
    for (int q = 0; q < 4; q++)
      if (q < fa.nf) f[q][dst] = v[q];
  }
}
template <typename T>
__global__ void __launch_bounds__(256) k_fill_halo(const Ctx* __restrict__ ctx, Grid g, FillArgs fa, int r, int full,
                                                   int64_t total) {
  fill_halo_body<T>(ctx, g, fa, r, full, total);
}

inline int64_t fill_count(const Grid& g, int r, int full) {
  const int64_t nx = g.n[0], ny = g.n[1], nz = g.n[2];
  const int64_t wx = full ? nx + 2 * r : nx, wy = full ? ny + 2 * r : ny;
  return 2 * r * wx * wy + 2 * r * nz * wx + 2 * r * ny * nz;
}

// --------------------------------------------------------------------------
// rhs (src/flows/rhs.jl:44-252) and update (src/flows/update.jl:37-51)
//
// One thread per interior cell and component.  The six flux arrays of the
// reference (J = c * a at -1:n+1) are recomputed where the flux divergence
// needs them, with the same operands and operation order as the stored ones.
// mode 0: write dUdt (rhs! only); mode 1: U = U0 + dUdt*dt (rhs! + update!).
// --------------------------------------------------------------------------
struct RhsCoef {
  double dxi, dyi, dzi, Rei;
};

template <typename T, int C>
__device__ __forceinline__ T rhs_component(const T* __restrict__ U, const T* __restrict__ V, const T* __restrict__ W,
                                           const T* __restrict__ P, int64_t c, int64_t sx, int64_t sy, int64_t sz,
                                           T dxi, T dyi, T dzi, T Rei) {
  const T* A = C == 0 ? U : C == 1 ? V : W;
  const int64_t sc = C == 0 ? sx : C == 1 ? sy : sz;
  const T dci = C == 0 ? dxi : C == 1 ? dyi : dzi;
  // velocities interpolated along the component axis (uc, vc, wc at a J point)
  auto uc = [&](int64_t q) { return interp_o4_at_half<T>(U[q - sc], U[q], U[q + sc], U[q + 2 * sc]); };
  auto vc = [&](int64_t q) { return interp_o4_at_half<T>(V[q - sc], V[q], V[q + sc], V[q + 2 * sc]); };
  auto wc = [&](int64_t q) { return interp_o4_at_half<T>(W[q - sc], W[q], W[q + sc], W[q + 2 * sc]); };
  auto a1 = [&](int64_t q, int64_t s) { return interp_o2_at_half<T>(A[q], A[q + s]); };
  auto a3 = [&](int64_t q, int64_t s) { return interp_o2_at_half<T>(A[q - s], A[q + 2 * s]); };
  const T diff = (dxi * dxi * diff2_o4_at_node<T>(A[c - 2 * sx], A[c - sx], A[c], A[c + sx], A[c + 2 * sx]) +
                  dyi * dyi * diff2_o4_at_node<T>(A[c - 2 * sy], A[c - sy], A[c], A[c + sy], A[c + 2 * sy]) +
                  dzi * dzi * diff2_o4_at_node<T>(A[c - 2 * sz], A[c - sz], A[c], A[c + sz], A[c + 2 * sz])) *
                 Rei;
  const T pres = dci * diff1_o2_at_half<T>(P[c], P[c + sc]);
  const T d0 = diff - pres;
  // Jx1 at i-1, i; Jx3 at i-2, i+1 (and the same along y, z)
  const T jx1a = uc(c - sx) * a1(c - sx, sx), jx1b = uc(c) * a1(c, sx);
  const T jx3a = uc(c - 2 * sx) * a3(c - 2 * sx, sx), jx3b = uc(c + sx) * a3(c + sx, sx);
  const T jy1a = vc(c - sy) * a1(c - sy, sy), jy1b = vc(c) * a1(c, sy);
  const T jy3a = vc(c - 2 * sy) * a3(c - 2 * sy, sy), jy3b = vc(c + sy) * a3(c + sy, sy);
  const T jz1a = wc(c - sz) * a1(c - sz, sz), jz1b = wc(c) * a1(c, sz);
  const T jz3a = wc(c - 2 * sz) * a3(c - 2 * sz, sz), jz3b = wc(c + sz) * a3(c + sz, sz);
  const T advect = dxi * sum_flux_o4<T>(jx1a, jx1b, jx3a, jx3b) + dyi * sum_flux_o4<T>(jy1a, jy1b, jy3a, jy3b) +
                   dzi * sum_flux_o4<T>(jz1a, jz1b, jz3a, jz3b);
  return d0 - advect;
}

// in_set: velocity set read by rhs; out_set: set written (mode 1); u0_set: U0
template <typename T>
__device__ __forceinline__ void rhs_body(const Ctx* __restrict__ ctx, const Grid& g, const T* __restrict__ P,
                                         int in_set, int out_set, int u0_set, int mode, T* __restrict__ dU,
                                         T* __restrict__ dV, T* __restrict__ dW, const RhsCoef& cf, int use_stage_dt,
                                         double dt_arg, int kz) {
  const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y;
  const int k = 1 + kz;
  if (i > nx || j > ny || k > nz) return;
  const T* U = (const T*)ctx->vel[in_set][0];
  const T* V = (const T*)ctx->vel[in_set][1];
  const T* W = (const T*)ctx->vel[in_set][2];
  const int64_t c = g.at(i, j, k), sx = 1, sy = g.px, sz = g.pz;
  const T dxi = (T)cf.dxi, dyi = (T)cf.dyi, dzi = (T)cf.dzi, Rei = (T)cf.Rei;
  const T ru = rhs_component<T, 0>(U, V, W, P, c, sx, sy, sz, dxi, dyi, dzi, Rei);
  const T rv = rhs_component<T, 1>(U, V, W, P, c, sx, sy, sz, dxi, dyi, dzi, Rei);
  const T rw = rhs_component<T, 2>(U, V, W, P, c, sx, sy, sz, dxi, dyi, dzi, Rei);
  if (mode == 0) {
    const int64_t o = ((int64_t)(k - 1) * ny + (j - 1)) * nx + (i - 1);
    dU[o] = ru;
    dV[o] = rv;
    dW[o] = rw;
  } else {
    const T dt = (T)(use_stage_dt ? ctx->scal[0] : dt_arg);
    T* Uo = (T*)ctx->vel[out_set][0];
    T* Vo = (T*)ctx->vel[out_set][1];
    T* Wo = (T*)ctx->vel[out_set][2];
    const T* U0 = (const T*)ctx->vel[u0_set][0];
    const T* V0 = (const T*)ctx->vel[u0_set][1];
    const T* W0 = (const T*)ctx->vel[u0_set][2];
    const T du = ru * dt, dv = rv * dt, dw = rw * dt;
    const T u = U0[c], v = V0[c], w = W0[c];
    Uo[c] = u + du;
    Vo[c] = v + dv;
    Wo[c] = w + dw;
  }
}
template <typename T>
__global__ void __launch_bounds__(256) k_rhs(const Ctx* __restrict__ ctx, Grid g, const T* __restrict__ P, int in_set,
                                             int out_set, int u0_set, int mode, T* __restrict__ dU,
                                             T* __restrict__ dV, T* __restrict__ dW, RhsCoef cf, int use_stage_dt,
                                             double dt_arg) {
  rhs_body<T>(ctx, g, P, in_set, out_set, u0_set, mode, dU, dV, dW, cf, use_stage_dt, dt_arg, (int)blockIdx.z);
}

// update! alone (the reference's separate kernel), reading dUdts.
template <typename T>
__global__ void k_update(const Ctx* __restrict__ ctx, Grid g, int out_set, int u0_set, const T* __restrict__ dU,
                         const T* __restrict__ dV, const T* __restrict__ dW, double dt_arg) {
  const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x, j = 1 + blockIdx.y, k = 1 + blockIdx.z;
  if (i > nx || j > ny || k > nz) return;
  const int64_t c = g.at(i, j, k), o = ((int64_t)(k - 1) * ny + (j - 1)) * nx + (i - 1);
  const T dt = (T)dt_arg;
  const T du = dU[o] * dt, dv = dV[o] * dt, dw = dW[o] * dt;
  const T u = ((const T*)ctx->vel[u0_set][0])[c], v = ((const T*)ctx->vel[u0_set][1])[c],
          w = ((const T*)ctx->vel[u0_set][2])[c];
  ((T*)ctx->vel[out_set][0])[c] = u + du;
  ((T*)ctx->vel[out_set][1])[c] = v + dv;
  ((T*)ctx->vel[out_set][2])[c] = w + dw;
}

// --------------------------------------------------------------------------
// HSMAC (src/flows/couples/hsmac.jl)
// --------------------------------------------------------------------------
struct HsmacCoef {
  double dxi, dyi, dzi, dl, omega, dxmin, epsp, count;  // count = (n+1)^3
  int itrmin, itrmax;
  int coloring;  // enum lcs_coloring
};

// Colour of a cell in the swept box, or -1 when the colouring never visits
// it: RedBlackFast visits every cell with (i+j+k) mod 2 == colour
// (lib/parallel/src/foraxes.jl:93-107); RedBlack tests `sum(i) % 2 == colour`
// with Julia's signed remainder, so cells with a negative odd index sum are
// never updated (foraxes.jl:82-88).
__device__ __forceinline__ int cell_color(int coloring, int i, int j, int k) {
  const int s = i + j + k;
  if (coloring == 1 /* RED_BLACK */) {
    const int r = s % 2;
    return r < 0 ? -1 : r;
  }
  return s & 1;
}

// One HSMAC cell update (hsmac.jl:1-35), in place; returns div.
template <typename T>
__device__ __forceinline__ T hsmac_cellwise(T* __restrict__ U, T* __restrict__ V, T* __restrict__ W,
                                           T* __restrict__ P, int64_t c, int64_t sy, int64_t sz, T dxi, T dyi,
                                           T dzi, T dl, T omega, T dti) {
  const T dudx = dxi * diff1_o2_at_half<T>(U[c - 1], U[c]);
  const T dvdy = dyi * diff1_o2_at_half<T>(V[c - sy], V[c]);
  const T dwdz = dzi * diff1_o2_at_half<T>(W[c - sz], W[c]);
  const T div = dudx + dvdy + dwdz;
  const T dp = -omega * div * dl;
  P[c] = P[c] + dp * dti;
  U[c - 1] = U[c - 1] - dp * dxi;
  U[c] = U[c] + dp * dxi;
  V[c - sy] = V[c - sy] - dp * dyi;
  V[c] = V[c] + dp * dyi;
  W[c - sz] = W[c - sz] - dp * dzi;
  W[c] = W[c] + dp * dzi;
  return div;
}

// In-place colour phase over a box: the reference's foraxes kernel for one
// colour.  Used for the thin face slabs of the overlap variant and for the
// RedBlack colouring on boxes with negative indices.  div^2 of cells inside
// R = [1,n+1]^3 is summed into partials[blockIdx.x].
template <typename T>
__global__ void __launch_bounds__(256) k_hsmac_phase(Ctx* __restrict__ ctx, Grid g, int set, T* __restrict__ P, Box b,
                                                     int color, HsmacCoef cf, double* __restrict__ partials) {
  __shared__ double sh[8];
  if (ctx->cs.done) return;
  T* U = (T*)ctx->vel[set][0];
  T* V = (T*)ctx->vel[set][1];
  T* W = (T*)ctx->vel[set][2];
  const T dxi = (T)cf.dxi, dyi = (T)cf.dyi, dzi = (T)cf.dzi, dl = (T)cf.dl, om = (T)cf.omega;
  const T dti = (T)(1.0 / ctx->scal[0]);
  const int lx = b.len(0), ly = b.len(1), lz = b.len(2);
  const int hx = (lx + 1) / 2;  // half range along x (RedBlackFast layout)
  const int64_t total = (int64_t)hx * ly * lz;
  const int R = g.n[0] + 1;
  double acc = 0.0;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t u = t;
    const int m = (int)(u % hx); u /= hx;
    const int j = b.lo[1] + (int)(u % ly); u /= ly;
    const int k = b.lo[2] + (int)u;
    // i with (i + j + k) of colour parity (foraxes.jl:100-104)
    const int a = b.lo[0];
    const int i = a + 2 * m + ((j + k - a + color) & 1);
    if (i > b.hi[0]) continue;
    if (cell_color(cf.coloring, i, j, k) != color) continue;
    const T div = hsmac_cellwise<T>(U, V, W, P, g.at(i, j, k), g.px, g.pz, dxi, dyi, dzi, dl, om, dti);
    if (i >= 1 && i <= R && j >= 1 && j <= g.n[1] + 1 && k >= 1 && k <= g.n[2] + 1) acc += (double)div * (double)div;
  }
  const double s = block_sum<256>(acc, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

// RedBlackBlock(size) (foraxes.jl:114-136): one thread per block of size^3
// cells of the given colour, cells visited sequentially, x fastest.
template <typename T>
__global__ void __launch_bounds__(128) k_hsmac_block(Ctx* __restrict__ ctx, Grid g, int set, T* __restrict__ P, Box b,
                                                     int color, int bs, HsmacCoef cf, double* __restrict__ partials) {
  __shared__ double sh[4];
  if (ctx->cs.done) return;
  T* U = (T*)ctx->vel[set][0];
  T* V = (T*)ctx->vel[set][1];
  T* W = (T*)ctx->vel[set][2];
  const T dxi = (T)cf.dxi, dyi = (T)cf.dyi, dzi = (T)cf.dzi, dl = (T)cf.dl, om = (T)cf.omega;
  const T dti = (T)(1.0 / ctx->scal[0]);
  const int nbx = (b.len(0) + bs - 1) / bs, nby = (b.len(1) + bs - 1) / bs, nbz = (b.len(2) + bs - 1) / bs;
  const int64_t total = (int64_t)nbx * nby * nbz;
  double acc = 0.0;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t u = t;
    const int bi = 1 + (int)(u % nbx); u /= nbx;
    const int bj = 1 + (int)(u % nby); u /= nby;
    const int bk = 1 + (int)u;
    if ((bi + bj + bk) % 2 != color) continue;
    for (int lk = 1; lk <= bs; lk++)
      for (int lj = 1; lj <= bs; lj++)
        for (int li = 1; li <= bs; li++) {
          const int i = b.lo[0] + bs * (bi - 1) + li - 1;
          const int j = b.lo[1] + bs * (bj - 1) + lj - 1;
          const int k = b.lo[2] + bs * (bk - 1) + lk - 1;
          if (i > b.hi[0] || j > b.hi[1] || k > b.hi[2]) continue;
          const T div = hsmac_cellwise<T>(U, V, W, P, g.at(i, j, k), g.px, g.pz, dxi, dyi, dzi, dl, om, dti);
          if (i >= 1 && i <= g.n[0] + 1 && j >= 1 && j <= g.n[1] + 1 && k >= 1 && k <= g.n[2] + 1)
            acc += (double)div * (double)div;
        }
  }
  const double s = block_sum<128>(acc, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

// The exit test after a sweep (hsmac.jl:120-123, 177-180) on the summed
// div^2 of R = [1,n+1]^3: div = sqrt(mean); exit when div*dxmin < epsp and
// itr >= itrmin; otherwise itr += 1.  `group_end` marks the last sweep of a
// `while itr < itrmax` iteration, where the loop condition is re-evaluated.
__device__ __forceinline__ void hsmac_check(Ctx* ctx, const HsmacCoef& cf, double sum, int group_end) {
  CoupleState& cs = ctx->cs;
  const double div = sqrt(sum / cf.count);
  cs.sum = sum;
  cs.div = div;
  cs.sweeps += 1;
  if (!isfinite(div)) ctx->nonfinite = 1;
  if (div * cf.dxmin < cf.epsp && cf.itrmin <= cs.itr) {
    cs.done = 1;
  } else {
    cs.itr += 1;
  }
  cs.cont = (!cs.done && cs.itr < cf.itrmax && isfinite(div)) ? 1 : 0;
  if (!isfinite(div)) cs.done = 1;  // stop sweeping; the host reports ENONFINITE
  (void)group_end;
}

// Sum the partials of one sweep and run the exit test (1 block).
__global__ void __launch_bounds__(256) k_hsmac_finalize(Ctx* ctx, const double* __restrict__ partials, int n,
                                                        HsmacCoef cf, int group_end) {
  __shared__ double sh[8];
  if (ctx->cs.done) return;
  const double s = sum_partials<256>(partials, n, sh);
  if (threadIdx.x == 0) hsmac_check(ctx, cf, s, group_end);
}

// --------------------------------------------------------------------------
// grid-wide barrier of a cooperative launch (all blocks co-resident), with a
// bounded wait: false when the generation did not advance within the limit.
// --------------------------------------------------------------------------
__device__ __forceinline__ unsigned int ld_acquire_gpu(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
constexpr long long kGridBarrierCycles = 200000000;  // ~0.1 s at 2 GHz
constexpr int kGridBarrierPolls = 1 << 24;

// Barrier number b (1, 2, ...) of a launch waits until the arrival counter
// reaches b x nblocks: one fire-and-forget add per block, no reset between
// barriers.  The block that finishes last resets the counter to 0 for the
// next launch (every block has then left its last barrier).
__device__ __forceinline__ bool grid_barrier(Ctx* ctx, unsigned int target, int* flag_sh) {
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    if (ctx->debug_wait == 1) target += 1;  // test hook: an arrival that never comes
    __threadfence();  // the block's writes (ordered by the __syncthreads) before the arrival
    atomicAdd(&ctx->gbar_count, 1u);
    const long long t0 = clock64();
    for (int it = 0; ld_acquire_gpu(&ctx->gbar_count) < target; it++) {
      if (it > kGridBarrierPolls || clock64() - t0 > kGridBarrierCycles) {
        ok = 0;
        break;
      }
    }
    __threadfence();
    *flag_sh = ok;
  }
  __syncthreads();
  return *flag_sh != 0;
}

// The six face slabs of an overlap sweep (Topologies.faces, halo.jl:349-366),
// in the reference's order: z-low, z-high, y-low, y-high, x-low, x-high.
struct FaceSet {
  Box f[6];
};

// Cell with flat index t among the cells of colour `color` of a face slab (the
// k_hsmac_phase mapping): false when the index maps to no such cell.
__device__ __forceinline__ bool face_locate(const Grid& g, const Box& b, int t, int color, int coloring, int64_t* c,
                                            bool* in_r) {
  const int lx = b.len(0), ly = b.len(1);
  const int hx = (lx + 1) / 2;
  int u = t;
  const int m = u % hx; u /= hx;
  const int j = b.lo[1] + u % ly; u /= ly;
  const int k = b.lo[2] + u;
  const int a = b.lo[0];
  const int i = a + 2 * m + ((j + k - a + color) & 1);
  if (i > b.hi[0]) return false;
  if (cell_color(coloring, i, j, k) != color) return false;
  *c = g.at(i, j, k);
  *in_r = i >= 1 && i <= g.n[0] + 1 && j >= 1 && j <= g.n[1] + 1 && k >= 1 && k <= g.n[2] + 1;
  return true;
}

// All face phases of one overlap sweep in one cooperative launch.  The
// reference runs, after the core, colour 0 then colour 1 of each face in
// turn (hsmac.jl:146-160).  Opposite faces never share a cell, a face value
// or a P value (they are separated by the non-empty core), so each pair runs
// as one phase: 3 pairs x 2 colours = 6 phases with a grid barrier between
// them, the same in-place result as the twelve sequential launches.  Then
// the block partials join the core sweep's partials[0, part0), and the last
// block runs the exit test (k_hsmac_finalize's work).
// Block `bid` of `nb` of one handle's face phases (k_hsmac_faces: the launch's
// grid; k_hsmac_faces_group: one handle per blockIdx.y, each handle's blocks
// meeting at the handle's own grid barrier).
template <typename T>
__device__ __forceinline__ void hsmac_faces_body(Ctx* __restrict__ ctx, const Grid& g, int set, T* __restrict__ P,
                                                 const FaceSet& fs, const HsmacCoef& cf,
                                                 double* __restrict__ partials, int part0, int group_end,
                                                 const unsigned int bid, const unsigned int nb) {
  __shared__ double sh[8];
  __shared__ int flag;
  if (ctx->cs.done) return;  // written before this launch: the same in every block
  T* U = (T*)ctx->vel[set][0];
  T* V = (T*)ctx->vel[set][1];
  T* W = (T*)ctx->vel[set][2];
  const T dxi = (T)cf.dxi, dyi = (T)cf.dyi, dzi = (T)cf.dzi, dl = (T)cf.dl, om = (T)cf.omega;
  const T dti = (T)(1.0 / ctx->scal[0]);
  const int stride = (int)nb * blockDim.x;
  double acc = 0.0;
  bool ok = true;
  for (int p = 0; p < 6; p++) {
    const int color = p & 1;
    const Box& ba = fs.f[p & ~1];
    const Box& bb = fs.f[(p & ~1) + 1];
    auto ncell = [](const Box& b) -> int {  // a face slab holds < 2^31 cells (checked on the host)
      if (b.lo[0] > b.hi[0] || b.lo[1] > b.hi[1] || b.lo[2] > b.hi[2]) return 0;
      return ((b.len(0) + 1) / 2) * b.len(1) * b.len(2);
    };
    const int na = ncell(ba), nt = na + ncell(bb);
    // Cells of one colour share no face, so the KB cells a thread takes per
    // round are independent: all their loads are issued before any store.
    // Loads bypass L1 (__ldcg): after a grid barrier a block reads cells that
    // other blocks have just written.
    constexpr int KB = 4;
    for (int t0 = (int)bid * blockDim.x + threadIdx.x; t0 < nt; t0 += KB * stride) {
      int64_t c[KB];
      bool v[KB], inr[KB];
      T u0[KB], u1[KB], v0[KB], v1[KB], w0[KB], w1[KB], p0[KB];
#pragma unroll
      for (int q = 0; q < KB; q++) {
        const int t = t0 + q * stride;
        c[q] = 0;
        inr[q] = false;
        v[q] = t < nt && (t < na ? face_locate(g, ba, t, color, cf.coloring, &c[q], &inr[q])
                                 : face_locate(g, bb, t - na, color, cf.coloring, &c[q], &inr[q]));
        if (v[q]) {
          const int64_t cc = c[q], sy = g.px, sz = g.pz;
          u0[q] = __ldcg(U + cc - 1); u1[q] = __ldcg(U + cc);
          v0[q] = __ldcg(V + cc - sy); v1[q] = __ldcg(V + cc);
          w0[q] = __ldcg(W + cc - sz); w1[q] = __ldcg(W + cc);
          p0[q] = __ldcg(P + cc);
        }
      }
#pragma unroll
      for (int q = 0; q < KB; q++) {
        if (!v[q]) continue;
        const int64_t cc = c[q], sy = g.px, sz = g.pz;
        // hsmac.jl:1-35, the reference's operation order
        const T dudx = dxi * diff1_o2_at_half<T>(u0[q], u1[q]);
        const T dvdy = dyi * diff1_o2_at_half<T>(v0[q], v1[q]);
        const T dwdz = dzi * diff1_o2_at_half<T>(w0[q], w1[q]);
        const T div = dudx + dvdy + dwdz;
        const T dp = -om * div * dl;
        P[cc] = p0[q] + dp * dti;
        U[cc - 1] = u0[q] - dp * dxi;
        U[cc] = u1[q] + dp * dxi;
        V[cc - sy] = v0[q] - dp * dyi;
        V[cc] = v1[q] + dp * dyi;
        W[cc - sz] = w0[q] - dp * dzi;
        W[cc] = w1[q] + dp * dzi;
        if (inr[q]) acc += (double)div * (double)div;
      }
    }
    if (p < 5 && !grid_barrier(ctx, (unsigned int)(p + 1) * nb, &flag)) {
      if (threadIdx.x == 0) ctx->wait_error = 1;
      ok = false;
      break;
    }
  }
  const double s = block_sum<256>(acc, sh);
  if (threadIdx.x == 0) partials[part0 + bid] = s;
  if (last_block(&ctx->ticket, nb, &flag)) {
    const double tot = sum_partials<256>(partials, part0 + (int)nb, sh);
    if (threadIdx.x == 0) {
      ctx->ticket = 0;
      ctx->gbar_count = 0;  // every block has left its last barrier
      if (ok && !ctx->wait_error) {
        hsmac_check(ctx, cf, tot, group_end);
      } else {
        ctx->wait_error = 1;
        ctx->cs.done = 1;
        ctx->cs.cont = 0;
      }
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_hsmac_faces(Ctx* __restrict__ ctx, Grid g, int set, T* __restrict__ P,
                                                     FaceSet fs, HsmacCoef cf, double* __restrict__ partials,
                                                     int part0, int group_end) {
  hsmac_faces_body<T>(ctx, g, set, P, fs, cf, partials, part0, group_end, blockIdx.x, gridDim.x);
}

// Per-handle pointers of a batch group (one handle per blockIdx.y).
constexpr int kGroupPtrMax = 64;
template <typename T>
struct GroupPtrs {
  Ctx* ctx[kGroupPtrMax];
  T* P[kGroupPtrMax];
  double* partials[kGroupPtrMax];
};
template <typename T>
__global__ void __launch_bounds__(256) k_hsmac_faces_group(const __grid_constant__ GroupPtrs<T> ga, Grid g, int set,
                                                           FaceSet fs, HsmacCoef cf, int part0, int group_end) {
  const int m = blockIdx.y;
  hsmac_faces_body<T>(ga.ctx[m], g, set, ga.P[m], fs, cf, ga.partials[m], part0, group_end, blockIdx.x, gridDim.x);
}
template <typename T>
__global__ void __launch_bounds__(256) k_fill_halo_group(const __grid_constant__ GroupPtrs<T> ga, Grid g, FillArgs fa,
                                                         int r, int full, int64_t total) {
  fill_halo_body<T>(ga.ctx[blockIdx.y], g, fa, r, full, total, ga.P[blockIdx.y]);  // P: the member's own
}

// Fused red-black sweep over the box D with the velocities ping-ponged:
// reads set `set` (through an optional periodic halo fill of radius fill_r,
// the synchalo! that precedes the sweep), writes the swept velocities into
// the spare set over the box `out`, and updates P in place.  Both colour
// phases of the reference's two foraxes launches are done in one pass:
//   phase 0: dp0(c) = -omega * div(old faces) * dl for colour-0 cells
//   phase 1: dp1(c) from faces after phase 0, i.e. old face + the colour-0
//            neighbour's delta, exactly the value the in-place sweep reads
// and each face is written as (old + delta_colour0) + delta_colour1, the
// in-place order.  So the result is bit-identical to the two in-place phases.
//
// CTA: a TX x TY column of the x-y plane, streaming along z through a chunk
// of planes; shared memory keeps 3 planes of U,V,W tiles (2-cell halo) and
// 3 planes of dp (1-cell halo).  Pipeline at plane s: load s, dp0 at s,
// dp1 at s-1, write outputs at s-2.
template <int TX, int TY, typename T>
struct FusedSmem {
  T u[3][TY + 4][TX + 4];
  T v[3][TY + 4][TX + 4];
  T w[3][TY + 4][TX + 4];
  T dp[3][TY + 3][TX + 3];
  double red[(TX * TY) / 32];
  int last;
};

__device__ __forceinline__ int ring3(int s) { return ((s % 3) + 3) % 3; }

template <typename T, int TX, int TY>
__global__ void __launch_bounds__(TX * TY) k_hsmac_fused(Ctx* __restrict__ ctx, Grid g, int set, T* __restrict__ P,
                                                         Box D, Box out, Box gb, int fill_r, int zchunk,
                                                         HsmacCoef cf, double* __restrict__ partials, int finalize,
                                                         int group_end, int swap) {
  __shared__ FusedSmem<TX, TY, T> sm;
  const bool skip = ctx->cs.done != 0;
  const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
  const int x0 = gb.lo[0] + blockIdx.x * TX, y0 = gb.lo[1] + blockIdx.y * TY;
  const int kb = gb.lo[2] + blockIdx.z * zchunk;
  const int ke = min(gb.hi[2], kb + zchunk - 1);
  const int nx = g.n[0], ny = g.n[1], nz = g.n[2], h = g.h;
  double racc = 0.0;
  if (!skip) {
    const T* Ui = (const T*)ctx->vel[set][0];
    const T* Vi = (const T*)ctx->vel[set][1];
    const T* Wi = (const T*)ctx->vel[set][2];
    T* Uo = (T*)ctx->vel[kSetSpare][0];
    T* Vo = (T*)ctx->vel[kSetSpare][1];
    T* Wo = (T*)ctx->vel[kSetSpare][2];
    const T dxi = (T)cf.dxi, dyi = (T)cf.dyi, dzi = (T)cf.dzi, dl = (T)cf.dl, om = (T)cf.omega;
    const T dti = (T)(1.0 / ctx->scal[0]);
    const int coloring = cf.coloring;
    // residual ownership: this tile's x/y/z ranges inside gb, extended by one
    // past gb's upper end so that R = [1,n+1] is covered exactly once
    const int ox_hi = (x0 + TX - 1 >= gb.hi[0]) ? gb.hi[0] + 1 : x0 + TX - 1;
    const int oy_hi = (y0 + TY - 1 >= gb.hi[1]) ? gb.hi[1] + 1 : y0 + TY - 1;
    const int oz_hi = (ke >= gb.hi[2]) ? gb.hi[2] + 1 : ke;
    auto owned = [&](int i, int j, int k) {
      return i >= x0 && i <= ox_hi && j >= y0 && j <= oy_hi && k >= kb && k <= oz_hi && i >= 1 && i <= nx + 1 &&
             j >= 1 && j <= ny + 1 && k >= 1 && k <= nz + 1;
    };
    auto color_of = [&](int i, int j, int k) { return D.contains(i, j, k) ? cell_color(coloring, i, j, k) : -1; };
    // source index of a storage position after the (optional) periodic fill
    auto src_at = [&](int i, int j, int k) -> int64_t {
      if (fill_r > 0 && i >= 1 - fill_r && i <= nx + fill_r && j >= 1 - fill_r && j <= ny + fill_r &&
          k >= 1 - fill_r && k <= nz + fill_r)
        return g.at(wrap1(i, nx), wrap1(j, ny), wrap1(k, nz));
      return g.at(i, j, k);
    };
    for (int s = kb - 2; s <= ke + 2; s++) {
      const int ps = ring3(s);
      // 1. load plane s of U,V,W over [x0-2, x0+TX+1] x [y0-2, y0+TY+1]
      const bool plane_ok = s >= 1 - h && s <= nz + h;
      for (int q = threadIdx.x; q < (TX + 4) * (TY + 4); q += TX * TY) {
        const int sx = q % (TX + 4), sy = q / (TX + 4);
        const int i = x0 - 2 + sx, j = y0 - 2 + sy;
        T a = T(0), b = T(0), c = T(0);
        if (plane_ok && i >= 1 - h && i <= nx + h && j >= 1 - h && j <= ny + h) {
          const int64_t src = src_at(i, j, s);
          a = Ui[src];
          b = Vi[src];
          c = Wi[src];
        }
        sm.u[ps][sy][sx] = a;
        sm.v[ps][sy][sx] = b;
        sm.w[ps][sy][sx] = c;
      }
      __syncthreads();
      // 2. dp0 at plane s over cells [x0-1, x0+TX+1] x [y0-1, y0+TY+1]
      if (s >= kb - 1) {
        const int pm = ring3(s - 1);
        for (int q = threadIdx.x; q < (TX + 3) * (TY + 3); q += TX * TY) {
          const int dx = q % (TX + 3), dy = q / (TX + 3);
          const int i = x0 - 1 + dx, j = y0 - 1 + dy;
          T dp = T(0);
          if (color_of(i, j, s) == 0) {
            const int sx = dx + 1, sy = dy + 1;
            const T dudx = dxi * diff1_o2_at_half<T>(sm.u[ps][sy][sx - 1], sm.u[ps][sy][sx]);
            const T dvdy = dyi * diff1_o2_at_half<T>(sm.v[ps][sy - 1][sx], sm.v[ps][sy][sx]);
            const T dwdz = dzi * diff1_o2_at_half<T>(sm.w[pm][sy][sx], sm.w[ps][sy][sx]);
            const T div = dudx + dvdy + dwdz;
            dp = -om * div * dl;
            if (owned(i, j, s)) racc += (double)div * (double)div;
          }
          sm.dp[ps][dy][dx] = dp;
        }
      }
      __syncthreads();
      // 3. dp1 at plane q = s-1 over cells [x0, x0+TX] x [y0, y0+TY]
      if (s - 1 >= kb) {
        const int qz = s - 1;
        const int pq = ring3(qz), pb = ring3(qz - 1), pa = ring3(qz + 1);
        for (int q = threadIdx.x; q < (TX + 1) * (TY + 1); q += TX * TY) {
          const int ex = q % (TX + 1), ey = q / (TX + 1);
          const int i = x0 + ex, j = y0 + ey;
          if (color_of(i, j, qz) != 1) continue;
          const int dx = ex + 1, dy = ey + 1, sx = ex + 2, sy = ey + 2;
          T ul = sm.u[pq][sy][sx - 1], ur = sm.u[pq][sy][sx];
          T vl = sm.v[pq][sy - 1][sx], vr = sm.v[pq][sy][sx];
          T wl = sm.w[pb][sy][sx], wr = sm.w[pq][sy][sx];
          if (color_of(i - 1, j, qz) == 0) ul = ul + sm.dp[pq][dy][dx - 1] * dxi;
          if (color_of(i + 1, j, qz) == 0) ur = ur - sm.dp[pq][dy][dx + 1] * dxi;
          if (color_of(i, j - 1, qz) == 0) vl = vl + sm.dp[pq][dy - 1][dx] * dyi;
          if (color_of(i, j + 1, qz) == 0) vr = vr - sm.dp[pq][dy + 1][dx] * dyi;
          if (color_of(i, j, qz - 1) == 0) wl = wl + sm.dp[pb][dy][dx] * dzi;
          if (color_of(i, j, qz + 1) == 0) wr = wr - sm.dp[pa][dy][dx] * dzi;
          const T dudx = dxi * diff1_o2_at_half<T>(ul, ur);
          const T dvdy = dyi * diff1_o2_at_half<T>(vl, vr);
          const T dwdz = dzi * diff1_o2_at_half<T>(wl, wr);
          const T div = dudx + dvdy + dwdz;
          sm.dp[pq][dy][dx] = -om * div * dl;
          if (owned(i, j, qz)) racc += (double)div * (double)div;
        }
      }
      __syncthreads();
      // 4. outputs at plane k = s-2
      const int k = s - 2;
      if (k >= kb && k <= ke) {
        const int i = x0 + tx, j = y0 + ty;
        const int pk = ring3(k), pk1 = ring3(k + 1);
        const int dx = tx + 1, dy = ty + 1, sx = tx + 2, sy = ty + 2;
        const int c0 = color_of(i, j, k);
        const T dpc = sm.dp[pk][dy][dx];
        if (c0 >= 0 && i >= gb.lo[0] && i <= gb.hi[0] && j >= gb.lo[1] && j <= gb.hi[1]) {
          const int64_t pc = g.at(i, j, k);
          P[pc] = P[pc] + dpc * dti;
        }
        if (out.contains(i, j, k)) {
          const int64_t o = g.at(i, j, k);
          // U face between cells i and i+1
          {
            const int cb = color_of(i + 1, j, k);
            const T db = sm.dp[pk][dy][dx + 1];
            T val = sm.u[pk][sy][sx];
            if (c0 == 0) val = val + dpc * dxi;
            if (cb == 0) val = val - db * dxi;
            if (c0 == 1) val = val + dpc * dxi;
            if (cb == 1) val = val - db * dxi;
            Uo[o] = val;
          }
          {
            const int cb = color_of(i, j + 1, k);
            const T db = sm.dp[pk][dy + 1][dx];
            T val = sm.v[pk][sy][sx];
            if (c0 == 0) val = val + dpc * dyi;
            if (cb == 0) val = val - db * dyi;
            if (c0 == 1) val = val + dpc * dyi;
            if (cb == 1) val = val - db * dyi;
            Vo[o] = val;
          }
          {
            const int cb = color_of(i, j, k + 1);
            const T db = sm.dp[pk1][dy][dx];
            T val = sm.w[pk][sy][sx];
            if (c0 == 0) val = val + dpc * dzi;
            if (cb == 0) val = val - db * dzi;
            if (c0 == 1) val = val + dpc * dzi;
            if (cb == 1) val = val - db * dzi;
            Wo[o] = val;
          }
        }
      }
      // the next iteration overwrites ring slot (s+1)%3 == (s-2)%3 only after
      // its own barrier, which every thread reaches after step 4
      __syncthreads();
    }
  }
  // residual partial of this CTA, then the last CTA finalizes the sweep
  const double bs = block_sum<TX * TY>(racc, sm.red);
  const unsigned int nb = gridDim.x * gridDim.y * gridDim.z;
  const unsigned int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  if (threadIdx.x == 0) partials[bid] = bs;
  if (last_block(&ctx->ticket, nb, &sm.last)) {
    if (skip) {
      if (threadIdx.x == 0) ctx->ticket = 0;
      return;
    }
    if (finalize) {
      const double s = sum_partials<TX * TY>(partials, (int)nb, sm.red);
      if (threadIdx.x == 0) hsmac_check(ctx, cf, s, group_end);
    }
    if (threadIdx.x == 0) {
      ctx->ticket = 0;
      if (swap)
        for (int c = 0; c < 3; c++) {
          void* tmp = ctx->vel[set][c];
          ctx->vel[set][c] = ctx->vel[kSetSpare][c];
          ctx->vel[kSetSpare][c] = tmp;
          const int tp = ctx->vphys[set][c];
          ctx->vphys[set][c] = ctx->vphys[kSetSpare][c];
          ctx->vphys[kSetSpare][c] = tp;
        }
    }
  }
}

// Reset the couple state before a couple! call.
__device__ __forceinline__ void couple_reset_body(Ctx* ctx, int itrmax) {
  ctx->cs.itr = 0;
  ctx->cs.sweeps = 0;
  ctx->cs.done = 0;
  ctx->cs.div = 0.0;
  ctx->cs.sum = 0.0;
  ctx->cs.cont = itrmax > 0 ? 1 : 0;
  ctx->cs.groups = 0;
  ctx->ticket = 0;
}
__global__ void k_couple_reset(Ctx* ctx, int itrmax) { couple_reset_body(ctx, itrmax); }

// Record the couple result into the step log (stage 1 or 2).
__device__ __forceinline__ void couple_log_body(Ctx* ctx, int stage) {
  if (stage == 1) {
    ctx->cur.itr1 = ctx->cs.itr;
    ctx->cur.sweeps1 = ctx->cs.sweeps;
    ctx->cur.div1 = ctx->cs.div;
  } else {
    ctx->cur.itr2 = ctx->cs.itr;
    ctx->cur.sweeps2 = ctx->cs.sweeps;
    ctx->cur.div2 = ctx->cs.div;
  }
}
__global__ void k_couple_log(Ctx* ctx, int stage) { couple_log_body(ctx, stage); }

// WHILE-node condition of the device-resident couple loop.
// The loop goes on while the exit test says so, no sweep has stopped the
// couple (a failed bounded wait, a non-finite residual) and fewer than
// max_groups iterations have run (the reference's loop runs at most
// ceil(itrmax / sweeps per group) of them; the bound holds the loop even if a
// kernel failed before its exit test).
__device__ __forceinline__ bool couple_goes_on(Ctx* ctx, int max_groups) {
  const int gdone = ++ctx->cs.groups;
  return ctx->cs.cont && !ctx->cs.done && !ctx->wait_error && !ctx->nonfinite && gdone < max_groups;
}
__global__ void k_couple_continue(Ctx* ctx, cudaGraphConditionalHandle handle, int max_groups) {
  cudaGraphSetConditional(handle, couple_goes_on(ctx, max_groups) ? 1u : 0u);
}
// the group's loop goes on while any member's does (done members' blocks
// return at once in every group launch)
template <typename T>
__global__ void k_group_continue(const __grid_constant__ GroupPtrs<T> ga, int m, cudaGraphConditionalHandle handle,
                                 int max_groups) {
  unsigned int c = 0;
  for (int q = 0; q < m; q++) c |= couple_goes_on(ga.ctx[q], max_groups) ? 1u : 0u;
  cudaGraphSetConditional(handle, c);
}

// --------------------------------------------------------------------------
// time step (src/flows/timestep.jl:18-65; src/timestep.jl:14-27)
// --------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void cfl_max_body(const Ctx* __restrict__ ctx, const Grid& g, double* __restrict__ partials) {
  __shared__ double sh[8];
  const T* U = (const T*)ctx->vel[kSetUs][0];
  const T* V = (const T*)ctx->vel[kSetUs][1];
  const T* W = (const T*)ctx->vel[kSetUs][2];
  const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
  const int64_t total = (int64_t)nx * ny * nz;
  double mu = 0.0, mv = 0.0, mw = 0.0;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int i = 1 + (int)(t % nx);
    const int j = 1 + (int)((t / nx) % ny);
    const int k = 1 + (int)(t / ((int64_t)nx * ny));
    const int64_t c = g.at(i, j, k);
    const T uc = interp_o4_at_half<T>(U[c - 2], U[c - 1], U[c], U[c + 1]);
    const T vc = interp_o4_at_half<T>(V[c - 2 * g.px], V[c - g.px], V[c], V[c + g.px]);
    const T wc = interp_o4_at_half<T>(W[c - 2 * g.pz], W[c - g.pz], W[c], W[c + g.pz]);
    mu = jl_max(mu, fabs((double)uc));
    mv = jl_max(mv, fabs((double)vc));
    mw = jl_max(mw, fabs((double)wc));
  }
  const double a = block_max<256>(mu, sh);
  const double b = block_max<256>(mv, sh);
  const double c = block_max<256>(mw, sh);
  if (threadIdx.x == 0) {
    partials[3 * blockIdx.x + 0] = a;
    partials[3 * blockIdx.x + 1] = b;
    partials[3 * blockIdx.x + 2] = c;
  }
}
template <typename T>
__global__ void __launch_bounds__(256) k_cfl_max(const Ctx* __restrict__ ctx, Grid g, double* __restrict__ partials) {
  cfl_max_body<T>(ctx, g, partials);
}

// --------------------------------------------------------------------------
// flow statistics (src/flows/stat.jl:66-138): per interior cell the squared
// speed u2, the strain-rate invariant s2 = 2 S_ij S_ij and du/dx^2,3,4 with
// the fourth-order half-point derivatives of src/diff.jl, read with periodic
// wrapping (the reference fills a FullHalo first); block sums in FP64 plus
// the mean, max and min of U, V, W.  14 values per block:
// sum u2, s2, d2, d3, d4, sum U, V, W, max U, V, W, min U, V, W.
// --------------------------------------------------------------------------
constexpr int kStatVals = 14;

template <typename T>
__device__ __forceinline__ double d1o4(const T* A, int64_t c0, int64_t c1, int64_t c2, int64_t c3) {
  return (1.0 / 24.0) * ((double)A[c0] - 27.0 * (double)A[c1] + 27.0 * (double)A[c2] - (double)A[c3]);
}

template <typename T>
__global__ void __launch_bounds__(256) k_flow_stat(const Ctx* __restrict__ ctx, Grid g, double dxi, double dyi,
                                                   double dzi, double* __restrict__ partials) {
  __shared__ double sh[8];
  const T* U = (const T*)ctx->vel[kSetUs][0];
  const T* V = (const T*)ctx->vel[kSetUs][1];
  const T* W = (const T*)ctx->vel[kSetUs][2];
  const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
  const int64_t total = (int64_t)nx * ny * nz;
  double acc[kStatVals];
  for (int q = 0; q < 8; q++) acc[q] = 0.0;
  for (int q = 8; q < 11; q++) acc[q] = -INFINITY;
  for (int q = 11; q < 14; q++) acc[q] = INFINITY;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int i = 1 + (int)(t % nx);
    const int j = 1 + (int)((t / nx) % ny);
    const int k = 1 + (int)(t / ((int64_t)nx * ny));
    auto at = [&](int a, int b, int c) { return g.at(wrap1(a, nx), wrap1(b, ny), wrap1(c, nz)); };
    const int64_t c = g.at(i, j, k);
    const double u = (double)U[c], v = (double)V[c], w = (double)W[c];
    const double u2 = u * u + v * v + w * w;
    // stat.jl:90-103
    const double dudx = dxi * d1o4(U, at(i - 2, j, k), at(i - 1, j, k), c, at(i + 1, j, k));
    const double dvdy = dyi * d1o4(V, at(i, j - 2, k), at(i, j - 1, k), c, at(i, j + 1, k));
    const double dwdz = dzi * d1o4(W, at(i, j, k - 2), at(i, j, k - 1), c, at(i, j, k + 1));
    const double dudy = dyi * d1o4(U, at(i, j - 2, k), at(i, j - 1, k), c, at(i, j + 1, k));
    const double dvdx = dxi * d1o4(V, at(i - 1, j - 1, k), at(i, j - 1, k), at(i + 1, j - 1, k), at(i + 2, j - 1, k));
    const double dvdz = dzi * d1o4(V, at(i, j - 1, k - 1), at(i, j - 1, k), at(i, j - 1, k + 1), at(i, j - 1, k + 2));
    const double dwdy = dyi * d1o4(W, at(i, j - 2, k), at(i, j - 1, k), c, at(i, j + 1, k));
    const double dwdx = dxi * d1o4(W, at(i - 1, j, k - 1), at(i, j, k - 1), at(i + 1, j, k - 1), at(i + 2, j, k - 1));
    const double dudz = dzi * d1o4(U, at(i, j, k - 2), at(i, j, k - 1), c, at(i, j, k + 1));
    const double s11 = 0.5 * (dudx + dudx), s22 = 0.5 * (dvdy + dvdy), s33 = 0.5 * (dwdz + dwdz);
    const double s12 = 0.5 * (dudy + dvdx), s13 = 0.5 * (dudz + dwdx), s23 = 0.5 * (dvdz + dwdy);
    const double s2 = 2.0 * (s11 * s11 + s22 * s22 + s33 * s33 + 2.0 * (s12 * s12 + s13 * s13 + s23 * s23));
    const double d2 = dudx * dudx;
    acc[0] += u2;
    acc[1] += s2;
    acc[2] += d2;
    acc[3] += d2 * dudx;
    acc[4] += d2 * d2;
    acc[5] += u;
    acc[6] += v;
    acc[7] += w;
    acc[8] = jl_max(acc[8], u);
    acc[9] = jl_max(acc[9], v);
    acc[10] = jl_max(acc[10], w);
    acc[11] = jl_min(acc[11], u);
    acc[12] = jl_min(acc[12], v);
    acc[13] = jl_min(acc[13], w);
  }
  for (int q = 0; q < kStatVals; q++) {
    double r;
    if (q < 8) {
      r = block_sum<256>(acc[q], sh);
    } else if (q < 11) {
      r = block_max<256>(acc[q], sh);
    } else {
      r = -block_max<256>(-acc[q], sh);
    }
    if (threadIdx.x == 0) partials[kStatVals * blockIdx.x + q] = r;
  }
}

// Combine the block values in a fixed order (1 block); result in out[0..13].
// Divergence of the velocity over the interior cells, in the HSMAC form
// (hsmac.jl: dxi (U[i] - U[i-1]) + dyi (V[j] - V[j-1]) + dzi (W[k] - W[k-1]),
// periodic reads): per block the sum of div^2 and the max |div|.
template <typename T>
__global__ void __launch_bounds__(256) k_div_stat(const Ctx* __restrict__ ctx, Grid g, double dxi, double dyi,
                                                  double dzi, double* __restrict__ partials) {
  __shared__ double sh[8];
  const T* U = (const T*)ctx->vel[kSetUs][0];
  const T* V = (const T*)ctx->vel[kSetUs][1];
  const T* W = (const T*)ctx->vel[kSetUs][2];
  const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
  const int64_t total = (int64_t)nx * ny * nz;
  double s2 = 0.0, mx = 0.0;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int i = 1 + (int)(t % nx), j = 1 + (int)((t / nx) % ny), k = 1 + (int)(t / ((int64_t)nx * ny));
    const int64_t c = g.at(i, j, k);
    const double dudx = dxi * (-(double)U[g.at(wrap1(i - 1, nx), j, k)] + (double)U[c]);
    const double dvdy = dyi * (-(double)V[g.at(i, wrap1(j - 1, ny), k)] + (double)V[c]);
    const double dwdz = dzi * (-(double)W[g.at(i, j, wrap1(k - 1, nz))] + (double)W[c]);
    const double div = dudx + dvdy + dwdz;
    s2 += div * div;
    mx = jl_max(mx, fabs(div));
  }
  const double bs = block_sum<256>(s2, sh);
  const double bm = block_max<256>(mx, sh);
  if (threadIdx.x == 0) {
    partials[2 * blockIdx.x] = bs;
    partials[2 * blockIdx.x + 1] = bm;
  }
}
__global__ void __launch_bounds__(256) k_div_stat_final(const double* __restrict__ partials, int nb,
                                                        double* __restrict__ out) {
  __shared__ double sh[8];
  double s = 0.0, m = 0.0;
  for (int b = threadIdx.x; b < nb; b += 256) {
    s += partials[2 * b];
    m = jl_max(m, partials[2 * b + 1]);
  }
  const double bs = block_sum<256>(s, sh);
  const double bm = block_max<256>(m, sh);
  if (threadIdx.x == 0) {
    out[0] = bs;
    out[1] = bm;
  }
}

__global__ void __launch_bounds__(256) k_flow_stat_final(const double* __restrict__ partials, int nb,
                                                         double* __restrict__ out) {
  __shared__ double sh[8];
  for (int q = 0; q < kStatVals; q++) {
    double v = q < 8 ? 0.0 : (q < 11 ? -INFINITY : INFINITY);
    for (int b = threadIdx.x; b < nb; b += 256) {
      const double x = partials[kStatVals * b + q];
      v = q < 8 ? v + x : (q < 11 ? jl_max(v, x) : jl_min(v, x));
    }
    const double r = q < 8 ? block_sum<256>(v, sh) : (q < 11 ? block_max<256>(v, sh) : -block_max<256>(-v, sh));
    if (threadIdx.x == 0) out[q] = r;
  }
}

struct DtCoef {
  double cfl, dtmax, dx, dy, dz, Re;
  int with_particles;
};

// dt = min(dtmax, cfl dx/umax, cfl dy/vmax, cfl dz/wmax, 0.5 (dx/2)^2 / (1/Re))
// [, particle dt]; writes ctx->dt (and *out).
__device__ __forceinline__ void cfl_finalize_body(Ctx* ctx, const double* __restrict__ partials, int nb,
                                                  const DtCoef& c, int flow_only, double* out) {
  __shared__ double sh[8];
  double m[3];
  for (int a = 0; a < 3; a++) {
    double v = 0.0;
    for (int q = threadIdx.x; q < nb; q += 256) v = jl_max(v, partials[3 * q + a]);
    m[a] = block_max<256>(v, sh);
  }
  if (threadIdx.x == 0) {
    const double umax = m[0] + 1e-10, vmax = m[1] + 1e-10, wmax = m[2] + 1e-10;
    double d = c.dtmax;
    d = jl_min(d, c.cfl * c.dx / umax);
    d = jl_min(d, c.cfl * c.dy / vmax);
    d = jl_min(d, c.cfl * c.dz / wmax);
    d = jl_min(d, 0.5 * ((c.dx / 2.0) * (c.dx / 2.0)) / (1.0 / c.Re));
    if (!flow_only && c.with_particles) d = jl_min(d, ctx->dt_particles);
    if (!(d > 0.0) || !isfinite(d)) ctx->nonfinite = 1;
    if (!flow_only) {
      ctx->dt = d;
      ctx->cur.dt = d;
    }
    if (out) *out = d;
  }
}
__global__ void __launch_bounds__(256) k_cfl_finalize(Ctx* ctx, const double* __restrict__ partials, int nb, DtCoef c,
                                                      int flow_only, double* out) {
  cfl_finalize_body(ctx, partials, nb, c, flow_only, out);
}

// --------------------------------------------------------------------------
// forcing: linear-power (src/flows/forcings/lf.jl:27-106)
// pass 1: sums of |u_cc|^2, U, V, W over the interior; pass 2: apply.
// --------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void lf_sums_body(const Ctx* __restrict__ ctx, const Grid& g, double* __restrict__ partials) {
  __shared__ double sh[8];
  const T* U = (const T*)ctx->vel[kSetUs][0];
  const T* V = (const T*)ctx->vel[kSetUs][1];
  const T* W = (const T*)ctx->vel[kSetUs][2];
  const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
  const int64_t total = (int64_t)nx * ny * nz;
  double s2 = 0.0, su = 0.0, sv = 0.0, sw = 0.0;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int i = 1 + (int)(t % nx);
    const int j = 1 + (int)((t / nx) % ny);
    const int k = 1 + (int)(t / ((int64_t)nx * ny));
    const int64_t c = g.at(i, j, k);
    const T u = interp_o2_at_half<T>(U[c - 1], U[c]);
    const T v = interp_o2_at_half<T>(V[c - g.px], V[c]);
    const T w = interp_o2_at_half<T>(W[c - g.pz], W[c]);
    const T u2 = u * u + v * v + w * w;
    s2 += (double)u2;
    su += (double)U[c];
    sv += (double)V[c];
    sw += (double)W[c];
  }
  const double a = block_sum<256>(s2, sh), b = block_sum<256>(su, sh), c = block_sum<256>(sv, sh),
               d = block_sum<256>(sw, sh);
  if (threadIdx.x == 0) {
    partials[4 * blockIdx.x + 0] = a;
    partials[4 * blockIdx.x + 1] = b;
    partials[4 * blockIdx.x + 2] = c;
    partials[4 * blockIdx.x + 3] = d;
  }
}
template <typename T>
__global__ void __launch_bounds__(256) k_lf_sums(const Ctx* __restrict__ ctx, Grid g, double* __restrict__ partials) {
  lf_sums_body<T>(ctx, g, partials);
}

// scal[1..4] = means (u2, u, v, w); scal[5] = A = p0 / (2e)
__device__ __forceinline__ void lf_coef_body(Ctx* ctx, const double* __restrict__ partials, int nb, double count,
                                             double p0) {
  __shared__ double sh[8];
  double m[4];
  for (int a = 0; a < 4; a++) {
    double v = 0.0;
    for (int q = threadIdx.x; q < nb; q += 256) v += partials[4 * q + a];
    m[a] = block_sum<256>(v, sh);
  }
  if (threadIdx.x == 0) {
    const double u2 = m[0] / count, u = m[1] / count, v = m[2] / count, w = m[3] / count;
    const double e = 0.5 * (u2 - u * u - v * v - w * w);
    ctx->scal[1] = u;
    ctx->scal[2] = v;
    ctx->scal[3] = w;
    ctx->scal[4] = u2;
    ctx->scal[5] = p0 / (2.0 * e);
  }
}
__global__ void __launch_bounds__(256) k_lf_coef(Ctx* ctx, const double* __restrict__ partials, int nb, double count,
                                                 double p0) {
  lf_coef_body(ctx, partials, nb, count, p0);
}

template <typename T>
__device__ __forceinline__ void lf_apply_body(Ctx* __restrict__ ctx, const Grid& g, double* __restrict__ partials) {
  __shared__ double sh[8];
  T* U = (T*)ctx->vel[kSetUs][0];
  T* V = (T*)ctx->vel[kSetUs][1];
  T* W = (T*)ctx->vel[kSetUs][2];
  const T A = (T)ctx->scal[5], um = (T)ctx->scal[1], vm = (T)ctx->scal[2], wm = (T)ctx->scal[3];
  const T dt = (T)ctx->scal[0];
  const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
  const int64_t total = (int64_t)nx * ny * nz;
  double sp = 0.0;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int i = 1 + (int)(t % nx);
    const int j = 1 + (int)((t / nx) % ny);
    const int k = 1 + (int)(t / ((int64_t)nx * ny));
    const int64_t c = g.at(i, j, k);
    const T usrc = A * (U[c] - um), vsrc = A * (V[c] - vm), wsrc = A * (W[c] - wm);
    const T u = U[c], v = V[c], w = W[c];
    const T p = u * usrc + v * vsrc + w * wsrc;
    U[c] = u + usrc * dt;
    V[c] = v + vsrc * dt;
    W[c] = w + wsrc * dt;
    sp += (double)p;
  }
  const double s = block_sum<256>(sp, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}
template <typename T>
__global__ void __launch_bounds__(256) k_lf_apply(Ctx* __restrict__ ctx, Grid g, double* __restrict__ partials) {
  lf_apply_body<T>(ctx, g, partials);
}

// mean of the per-cell power -> ctx->scal[6], and the step log
__device__ __forceinline__ void power_finalize_body(Ctx* ctx, const double* __restrict__ partials, int nb,
                                                    double count, double e10) {
  __shared__ double sh[8];
  const double s = sum_partials<256>(partials, nb, sh);
  if (threadIdx.x == 0) {
    ctx->scal[6] = s / count;
    ctx->cur.p = s / count;
    ctx->cur.e10 = e10;
  }
}
__global__ void __launch_bounds__(256) k_power_finalize(Ctx* ctx, const double* __restrict__ partials, int nb,
                                                        double count, double e10) {
  power_finalize_body(ctx, partials, nb, count, e10);
}

// --------------------------------------------------------------------------
// forcing: rc-energy (src/flows/forcings/rcf.jl:21-191, lib/fouriertools)
// --------------------------------------------------------------------------
// boxmean_l! as the plain loop of ext/AMDGPUExt.jl:25-40 (dk, dj, di order):
// one thread per coarse cell and component.
template <typename T>
__global__ void __launch_bounds__(128) k_rcf_boxmean(const Ctx* __restrict__ ctx, Grid g, int cs,
                                                     double* __restrict__ coarse) {
  const int ncs = cs * cs * cs;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * ncs) return;
  const int a = t / ncs, q = t % ncs;
  const int ic = 1 + q % cs, jc = 1 + (q / cs) % cs, kc = 1 + q / (cs * cs);
  const int fx = g.n[0] / cs, fy = g.n[1] / cs, fz = g.n[2] / cs;
  const T* A = (const T*)ctx->vel[kSetUs][a];
  T s = T(0);
  for (int dk = 1; dk <= fz; dk++)
    for (int dj = 1; dj <= fy; dj++) {
      const T* row = A + g.at((ic - 1) * fx + 1, (jc - 1) * fy + dj, (kc - 1) * fz + dk);
      for (int di = 0; di < fx; di++) s += row[di];
    }
  const T w = T(1.0 / (double)(fx * fy * fz));
  coarse[t] = (double)(s * w);
}

// Direct DFT of the coarse fields at the modes kx in 0..kmax, ky,kz in
// -kmax..kmax (FFTW rfft in the reference): one block per (component, mode).
__global__ void __launch_bounds__(256) k_rcf_dft(const double* __restrict__ coarse, int cs, int kmax,
                                                 const double* __restrict__ tw /* re,im of exp(-2 pi i x/cs) */,
                                                 double* __restrict__ hat /* [a][mode] re,im */) {
  __shared__ double sh[8];
  const int KX = kmax + 1, KY = 2 * kmax + 1;
  const int nm = KX * KY * KY;
  const int a = blockIdx.x / nm, m = blockIdx.x % nm;
  const int kx = m % KX, ky = (m / KX) % KY - kmax, kz = m / (KX * KY) - kmax;
  const int ncs = cs * cs * cs;
  double sre = 0.0, sim = 0.0;
  for (int q = threadIdx.x; q < ncs; q += 256) {
    const int x = q % cs, y = (q / cs) % cs, z = q / (cs * cs);
    const int ph = (((kx * x + ky * y + kz * z) % cs) + cs) % cs;
    const double v = coarse[(size_t)a * ncs + q];
    sre += v * tw[2 * ph];
    sim += v * tw[2 * ph + 1];
  }
  const double r = block_sum<256>(sre, sh);
  const double i = block_sum<256>(sim, sh);
  if (threadIdx.x == 0) {
    hat[2 * ((size_t)a * nm + m)] = r;
    hat[2 * ((size_t)a * nm + m) + 1] = i;
  }
}

// Shell energies, rescale and crop (rcf.jl:49-70): one thread.
// en0[k0-kmin] is enespe0(k0, e10) computed on the host.
__global__ void k_rcf_spectrum(const double* __restrict__ hat, int kmin, int kmax, double norm,
                               const double* __restrict__ en0, double* __restrict__ Ac /* [a][mode] re,im */) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int KX = kmax + 1, KY = 2 * kmax + 1;
  const int nm = KX * KY * KY;
  double r_of_shell[8];
  for (int k0 = kmin; k0 <= kmax; k0++) {
    const double lo = (k0 - 0.5) * (k0 - 0.5), hi = (k0 + 0.5) * (k0 + 0.5);
    double e = 0.0;
    for (int kz = -k0; kz <= k0; kz++)
      for (int ky = -k0; ky <= k0; ky++)
        for (int kx = 0; kx <= k0; kx++) {
          const int r2 = kx * kx + ky * ky + kz * kz;
          if (lo <= r2 && r2 < hi) {
            const double wgt = kx == 0 ? 1.0 : 2.0;
            double acc = 0.0;
            for (int a = 0; a < 3; a++) {
              const size_t id = (size_t)a * nm + ((kz + kmax) * KY + (ky + kmax)) * KX + kx;
              const double zr = hat[2 * id] / norm, zi = hat[2 * id + 1] / norm;
              const double ab = zr * zr + zi * zi;
              acc = a == 0 ? ab : acc + ab;
            }
            e += wgt * acc;
          }
        }
    const double en = e / 2.0;
    r_of_shell[k0 - kmin] = sqrt(en0[k0 - kmin] / jl_max(en, 1e-8)) - 1.0;
  }
  for (int a = 0; a < 3; a++)
    for (int kz = -kmax; kz <= kmax; kz++)
      for (int ky = -kmax; ky <= kmax; ky++)
        for (int kx = 0; kx <= kmax; kx++) {
          const size_t id = (size_t)a * nm + ((kz + kmax) * KY + (ky + kmax)) * KX + kx;
          double zr = hat[2 * id], zi = hat[2 * id + 1];
          const int r2 = kx * kx + ky * ky + kz * kz;
          for (int k0 = kmin; k0 <= kmax; k0++) {
            const double lo = (k0 - 0.5) * (k0 - 0.5), hi = (k0 + 0.5) * (k0 + 0.5);
            if (lo <= r2 && r2 < hi) {
              zr *= r_of_shell[k0 - kmin];
              zi *= r_of_shell[k0 - kmin];
            }
          }
          Ac[2 * id] = zr / norm;
          Ac[2 * id + 1] = zi / norm;
        }
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {  // Julia *(::Complex, ::Complex)
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Per-cell sparse inverse DFT (FourierTools.sirdft, kset order) and update
// U += usrc; Power = (u.usrc) * dti (rcf.jl:74-96).
// modes: (kx,ky,kz) triples of kset(kmin..kmax), shells delimited by kofs.
struct RcfModes {
  int n;
  int nshell;
  int kofs[9];
  signed char k[256][3];  // kset(1..4): 9 + 31 + 49 + 105 vectors
};

template <typename T>
__global__ void __launch_bounds__(256) k_rcf_apply(Ctx* __restrict__ ctx, Grid g, const double* __restrict__ Ac,
                                                   const double2* __restrict__ phx, const double2* __restrict__ phy,
                                                   const double2* __restrict__ phz, RcfModes md, int kmax,
                                                   double* __restrict__ partials) {
  __shared__ double sh[8];
  __shared__ double2 sA[3][256];
  __shared__ signed char sk[256][3];
  const int KX = kmax + 1, KY = 2 * kmax + 1, nm = KX * KY * KY;
  for (int q = threadIdx.x; q < md.n; q += blockDim.x) {
    const int kx = md.k[q][0], ky = md.k[q][1], kz = md.k[q][2];
    const int id = ((kz + kmax) * KY + (ky + kmax)) * KX + kx;
    for (int a = 0; a < 3; a++) sA[a][q] = make_double2(Ac[2 * ((size_t)a * nm + id)], Ac[2 * ((size_t)a * nm + id) + 1]);
    sk[q][0] = md.k[q][0];
    sk[q][1] = md.k[q][1];
    sk[q][2] = md.k[q][2];
  }
  __syncthreads();
  T* U = (T*)ctx->vel[kSetUs][0];
  T* V = (T*)ctx->vel[kSetUs][1];
  T* W = (T*)ctx->vel[kSetUs][2];
  const double dti = 1.0 / ctx->scal[0];
  const int nx = g.n[0], ny = g.n[1], nz = g.n[2];
  const int64_t total = (int64_t)nx * ny * nz;
  double sp = 0.0;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int i = 1 + (int)(t % nx);
    const int j = 1 + (int)((t / nx) % ny);
    const int k = 1 + (int)(t / ((int64_t)nx * ny));
    const double2 ei = phx[i], ej = phy[j], ek = phz[k];
    double src[3];
    for (int a = 0; a < 3; a++) src[a] = 0.0;
    for (int sh_i = 0; sh_i < md.nshell; sh_i++) {
      double acc[3] = {0.0, 0.0, 0.0};
      for (int q = md.kofs[sh_i]; q < md.kofs[sh_i + 1]; q++) {
        const int kx = sk[q][0], ky = sk[q][1], kz = sk[q][2];
        // powi: right-nested products, conj for negative powers; the Int 1
        // factors of the reference are exact and skipped
        double2 prod = make_double2(1.0, 0.0);
        bool have = false;
        const int e3[3] = {kx, ky, kz};
        const double2 b3[3] = {ei, ej, ek};
        for (int d = 0; d < 3; d++) {
          const int n = e3[d];
          if (n == 0) continue;
          const int m = n < 0 ? -n : n;
          double2 p = b3[d];
          for (int r = 2; r <= m; r++) p = cmul(b3[d], p);
          if (n < 0) p.y = -p.y;
          prod = have ? cmul(prod, p) : p;
          have = true;
        }
        for (int a = 0; a < 3; a++) {
          const double2 A = sA[a][q];
          acc[a] += 2.0 * (A.x * prod.x - A.y * prod.y);
        }
      }
      for (int a = 0; a < 3; a++) src[a] += acc[a];
    }
    const int64_t c = g.at(i, j, k);
    const double u = (double)U[c], v = (double)V[c], w = (double)W[c];
    const double p = (u * src[0] + v * src[1] + w * src[2]) * dti;
    U[c] = (T)((double)U[c] + src[0]);
    V[c] = (T)((double)V[c] + src[1]);
    W[c] = (T)((double)W[c] + src[2]);
    sp += p;
  }
  const double s = block_sum<256>(sp, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

// --------------------------------------------------------------------------
// particles (src/particles/{boundary,interp,motion,update}.jl)
// --------------------------------------------------------------------------
struct Mapping {
  int i, j, k;
  double r1, r2, r3;
};
__device__ __forceinline__ Mapping xmapping(double x, double y, double z, double dx, double dy, double dz) {
  Mapping m;
  m.i = (int)floor(x / dx);
  m.j = (int)floor(y / dy + 0.5);
  m.k = (int)floor(z / dz + 0.5);
  m.r1 = x / dx - m.i;
  m.r2 = y / dy - m.j + 0.5;
  m.r3 = z / dz - m.k + 0.5;
  return m;
}
__device__ __forceinline__ Mapping ymapping(double x, double y, double z, double dx, double dy, double dz) {
  Mapping m;
  m.j = (int)floor(y / dy);
  m.k = (int)floor(z / dz + 0.5);
  m.i = (int)floor(x / dx + 0.5);
  m.r2 = y / dy - m.j;
  m.r3 = z / dz - m.k + 0.5;
  m.r1 = x / dx - m.i + 0.5;
  return m;
}
__device__ __forceinline__ Mapping zmapping(double x, double y, double z, double dx, double dy, double dz) {
  Mapping m;
  m.k = (int)floor(z / dz);
  m.i = (int)floor(x / dx + 0.5);
  m.j = (int)floor(y / dy + 0.5);
  m.r3 = z / dz - m.k;
  m.r2 = y / dy - m.j + 0.5;
  m.r1 = x / dx - m.i + 0.5;
  return m;
}

// Trilinear interpolation (interp.jl:62-90).  Indices outside the halo
// (a position far outside [0, 2pi)) are clamped to keep the read in bounds.
template <typename T>
__device__ __forceinline__ double interp(const T* __restrict__ U, const Grid& g, Mapping m) {
  const int lo = 1 - g.h;
  int i = min(max(m.i, lo), g.n[0] + g.h - 1), j = min(max(m.j, lo), g.n[1] + g.h - 1),
      k = min(max(m.k, lo), g.n[2] + g.h - 1);
  const int64_t c = g.at(i, j, k), sy = g.px, sz = g.pz;
  const double c0 = (double)U[c], c1 = (double)U[c + 1], c2 = (double)U[c + 1 + sy], c3 = (double)U[c + sy],
               c4 = (double)U[c + sz], c5 = (double)U[c + 1 + sz], c6 = (double)U[c + 1 + sy + sz],
               c7 = (double)U[c + sy + sz];
  const double r1 = m.r1, r2 = m.r2, r3 = m.r3;
  return (1 - r1) * (1 - r2) * (1 - r3) * c0 + r1 * (1 - r2) * (1 - r3) * c1 + r1 * r2 * (1 - r3) * c2 +
         (1 - r1) * r2 * (1 - r3) * c3 + (1 - r1) * (1 - r2) * r3 * c4 + r1 * (1 - r2) * r3 * c5 +
         r1 * r2 * r3 * c6 + (1 - r1) * r2 * r3 * c7;
}

struct SpeciesDev {
  double* p[16];  // enum lcs_prop order
  int64_t n;
  double gravity, density_ratio;
  int drag;
};

struct PartCoef {
  double dx, dy, dz, Re;
};

// modes: bit0 boundary!, bit1 motion!, bit2 update!.  With motion and update
// together dudt stays in registers.  `use_stage_dt` reads dtrk from the
// device context (graph replays), else dt_arg.
// The property arrays of species s are read from the device context (the
// species' block moves when a cell index reorders it), so graphs captured
// before the move stay valid.
__device__ __forceinline__ void species_arrays(const Ctx* __restrict__ ctx, int s, SpeciesDev& sp) {
  double* b = ctx->sp_base[s];
#pragma unroll
  for (int q = 0; q < 16; q++) sp.p[q] = b + q * sp.n;
}

template <typename T>
__device__ __forceinline__ void particles_body(const Ctx* __restrict__ ctx, const Grid& g, int s, SpeciesDev sp,
                                               const PartCoef& pc, int stage, int modes, int use_stage_dt,
                                               double dt_arg) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= sp.n) return;
  species_arrays(ctx, s, sp);
  const double L = kDomainLength;
  // stage 1: xss / xss2 partner; stage 2: xss2 / xss partner (boundary.jl:22-26)
  double* X[3] = {sp.p[stage == 1 ? 0 : 3], sp.p[stage == 1 ? 1 : 4], sp.p[stage == 1 ? 2 : 5]};
  double* Xp[3] = {sp.p[stage == 1 ? 3 : 0], sp.p[stage == 1 ? 4 : 1], sp.p[stage == 1 ? 5 : 2]};
  double xs[3];
  for (int a = 0; a < 3; a++) xs[a] = X[a][p];
  if (modes & 1) {
    for (int a = 0; a < 3; a++) {
      const double x = xs[a], x2 = Xp[a][p];
      if (x < 0.0) {
        xs[a] = x + L;
        X[a][p] = x + L;
        Xp[a][p] = x2 + L;
      }
      if (x >= 0.0 + L) {
        xs[a] = x - L;
        X[a][p] = x - L;
        Xp[a][p] = x2 - L;
      }
    }
  }
  double dudt[3];
  if (modes & 2) {
    const int vset = stage == 1 ? kSetUs : kSetUs2;
    const T* U = (const T*)ctx->vel[vset][0];
    const T* V = (const T*)ctx->vel[vset][1];
    const T* W = (const T*)ctx->vel[vset][2];
    const double* Us = sp.p[stage == 1 ? 6 : 9];
    const double* Vs = sp.p[stage == 1 ? 7 : 10];
    const double* Ws = sp.p[stage == 1 ? 8 : 11];
    const double xp = xs[0] - 0.0, yp = xs[1] - 0.0, zp = xs[2] - 0.0;
    const double up = Us[p], vp = Vs[p], wp = Ws[p];
    const double diam = sp.p[15][p];
    const double uf = interp<T>(U, g, xmapping(xp, yp, zp, pc.dx, pc.dy, pc.dz));
    const double vf = interp<T>(V, g, ymapping(xp, yp, zp, pc.dx, pc.dy, pc.dz));
    const double wf = interp<T>(W, g, zmapping(xp, yp, zp, pc.dx, pc.dy, pc.dz));
    double f = 1.0;
    if (sp.drag == 1) {
      const double a = uf - up, b = vf - vp, c = wf - wp;
      const double vrel = sqrt(a * a + b * b + c * c);
      const double Rep = diam * vrel * pc.Re;
      f = 1.0 + 0.15 * pow(Rep, 0.687);
    }
    const double taup = 1.0 / 18.0 * sp.density_ratio * pc.Re * (diam * diam);
    const double taui = 1.0 / taup;
    dudt[0] = f * (uf - up) * taui - sp.gravity;
    dudt[1] = f * (vf - vp) * taui;
    dudt[2] = f * (wf - wp) * taui;
    if (!(modes & 4)) {
      sp.p[12][p] = dudt[0];
      sp.p[13][p] = dudt[1];
      sp.p[14][p] = dudt[2];
    }
  } else if (modes & 4) {
    dudt[0] = sp.p[12][p];
    dudt[1] = sp.p[13][p];
    dudt[2] = sp.p[14][p];
  }
  if (modes & 4) {
    const double dt = use_stage_dt ? ctx->scal[0] : dt_arg;
    // stage 1: xss2 = xss + dt uss, uss2 = uss + dt dudt; stage 2: in place
    // from the stage-start xss, uss (update.jl:1-11, 48-62)
    for (int a = 0; a < 3; a++) {
      const double x0 = (stage == 1 || !(modes & 1)) ? sp.p[a][p] : (stage == 1 ? xs[a] : Xp[a][p]);
      const double u0 = sp.p[6 + a][p];
      sp.p[(stage == 1 ? 3 : 0) + a][p] = x0 + dt * u0;
      sp.p[(stage == 1 ? 9 : 6) + a][p] = u0 + dt * dudt[a];
    }
  }
}
template <typename T>
__global__ void __launch_bounds__(256) k_particles(const Ctx* __restrict__ ctx, Grid g, int s, SpeciesDev sp,
                                                   PartCoef pc, int stage, int modes, int use_stage_dt, double dt_arg) {
  particles_body<T>(ctx, g, s, sp, pc, stage, modes, use_stage_dt, dt_arg);
}

// New init kind: particle velocity = trilinear interpolation of Us.
template <typename T>
__global__ void k_particles_init_velocity(const Ctx* __restrict__ ctx, Grid g, int s, SpeciesDev sp, PartCoef pc) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= sp.n) return;
  species_arrays(ctx, s, sp);
  const double x = sp.p[0][p], y = sp.p[1][p], z = sp.p[2][p];
  sp.p[6][p] = interp<T>((const T*)ctx->vel[kSetUs][0], g, xmapping(x, y, z, pc.dx, pc.dy, pc.dz));
  sp.p[7][p] = interp<T>((const T*)ctx->vel[kSetUs][1], g, ymapping(x, y, z, pc.dx, pc.dy, pc.dz));
  sp.p[8][p] = interp<T>((const T*)ctx->vel[kSetUs][2], g, zmapping(x, y, z, pc.dx, pc.dy, pc.dz));
}

// max(0, a[0..n)) (maximum(diams) of particles/timestep.jl) in two passes:
// block maxima over a grid-stride range, then the maximum of the blocks'.
__global__ void __launch_bounds__(256) k_max_partial(const double* __restrict__ a, int64_t n,
                                                      double* __restrict__ partials) {
  __shared__ double sh[8];
  double v = 0.0;
  for (int64_t q = (int64_t)blockIdx.x * 256 + threadIdx.x; q < n; q += (int64_t)gridDim.x * 256) v = jl_max(v, a[q]);
  const double m = block_max<256>(v, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = m;
}
__global__ void __launch_bounds__(256) k_max_reduce(const double* __restrict__ a, int64_t n, double* __restrict__ out) {
  __shared__ double sh[8];
  double v = 0.0;
  for (int64_t q = threadIdx.x; q < n; q += 256) v = jl_max(v, a[q]);
  const double m = block_max<256>(v, sh);
  if (threadIdx.x == 0) *out = m;
}

// --------------------------------------------------------------------------
// transfers between the host layout (FP64, interior or haloed) and the
// device fields
// --------------------------------------------------------------------------
template <typename T>
__global__ void k_scatter(const Ctx* __restrict__ ctx, Grid g, int set, int comp, T* __restrict__ direct,
                          const double* __restrict__ src, int haloed) {
  T* f = direct ? direct : (T*)ctx->vel[set][comp];
  const int w = haloed ? g.h : 0;
  const int lx = g.n[0] + 2 * w, ly = g.n[1] + 2 * w, lz = g.n[2] + 2 * w;
  const int64_t total = (int64_t)lx * ly * lz;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int i = 1 - w + (int)(t % lx), j = 1 - w + (int)((t / lx) % ly), k = 1 - w + (int)(t / ((int64_t)lx * ly));
    f[g.at(i, j, k)] = (T)src[t];
  }
}

// trilinear_upsample2x! (src/LCSIO/upsample.jl:47-91): every coarse cell
// (i, j, k) of the (n/2)^3 interior writes the 8 fine cells (2i-1..2i, ...),
// the coarse neighbours at i+1 read through the periodic halo (the reference's
// FullHalo(1) synchalo!).  Sums left to right as written there, in FP64,
// rounded once to T.
template <typename T>
__global__ void __launch_bounds__(256) k_upsample2x(const Ctx* __restrict__ ctx, Grid g, int set, int comp,
                                                    T* __restrict__ direct, const double* __restrict__ c) {
  T* f = direct ? direct : (T*)ctx->vel[set][comp];
  const int nx = g.n[0] / 2, ny = g.n[1] / 2, nz = g.n[2] / 2;
  const int64_t total = (int64_t)nx * ny * nz;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(t % nx), j = (int)((t / nx) % ny), k = (int)(t / ((int64_t)nx * ny));  // 0-based
    const int i1 = i + 1 < nx ? i + 1 : 0, j1 = j + 1 < ny ? j + 1 : 0, k1 = k + 1 < nz ? k + 1 : 0;
    auto C = [&](int a, int b, int d) { return c[a + (int64_t)nx * (b + (int64_t)ny * d)]; };
    const double c000 = C(i, j, k), c100 = C(i1, j, k), c010 = C(i, j1, k), c001 = C(i, j, k1);
    const double c110 = C(i1, j1, k), c101 = C(i1, j, k1), c011 = C(i, j1, k1), c111 = C(i1, j1, k1);
    const int ii = 2 * i + 1, jj = 2 * j + 1, kk = 2 * k + 1;  // 1-based fine index 2i-1
    f[g.at(ii, jj, kk)] = (T)c000;
    f[g.at(ii + 1, jj, kk)] = (T)(0.5 * __dadd_rn(c000, c100));
    f[g.at(ii, jj + 1, kk)] = (T)(0.5 * __dadd_rn(c000, c010));
    f[g.at(ii, jj, kk + 1)] = (T)(0.5 * __dadd_rn(c000, c001));
    f[g.at(ii + 1, jj + 1, kk)] = (T)(0.25 * __dadd_rn(__dadd_rn(__dadd_rn(c000, c100), c010), c110));
    f[g.at(ii + 1, jj, kk + 1)] = (T)(0.25 * __dadd_rn(__dadd_rn(__dadd_rn(c000, c100), c001), c101));
    f[g.at(ii, jj + 1, kk + 1)] = (T)(0.25 * __dadd_rn(__dadd_rn(__dadd_rn(c000, c010), c001), c011));
    double s8 = __dadd_rn(__dadd_rn(__dadd_rn(c000, c100), c010), c001);
    s8 = __dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(s8, c110), c101), c011), c111);
    f[g.at(ii + 1, jj + 1, kk + 1)] = (T)(0.125 * s8);
  }
}

template <typename T>
__global__ void k_gather(const Ctx* __restrict__ ctx, Grid g, int set, int comp, const T* __restrict__ direct,
                         double* __restrict__ dst, int haloed) {
  const T* f = direct ? direct : (const T*)ctx->vel[set][comp];
  const int w = haloed ? g.h : 0;
  const int lx = g.n[0] + 2 * w, ly = g.n[1] + 2 * w, lz = g.n[2] + 2 * w;
  const int64_t total = (int64_t)lx * ly * lz;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int i = 1 - w + (int)(t % lx), j = 1 - w + (int)((t / lx) % ly), k = 1 - w + (int)(t / ((int64_t)lx * ly));
    dst[t] = (double)f[g.at(i, j, k)];
  }
}

template <typename T>
__global__ void k_convert_in(T* __restrict__ dst, const double* __restrict__ src, int64_t n) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
    dst[t] = (T)src[t];
}
template <typename T>
__global__ void k_convert_out(double* __restrict__ dst, const T* __restrict__ src, int64_t n) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
    dst[t] = (double)src[t];
}

// --------------------------------------------------------------------------
// step bookkeeping (src/evolve.jl:10-13, src/state.jl:37-38)
// --------------------------------------------------------------------------
__device__ __forceinline__ void stage_dt_body(Ctx* ctx, int stage) {
  ctx->scal[0] = stage == 1 ? 0.5 * ctx->dt : ctx->dt;  // dtrk (src/state.jl:37-38)
}
__global__ void k_set_stage_dt(Ctx* ctx, int stage) { stage_dt_body(ctx, stage); }
__global__ void k_set_scalar(double* dst, double v) { *dst = v; }
__global__ void k_set_debug_wait(Ctx* ctx, int kind) { ctx->debug_wait = kind; }
__global__ void k_set_species_base(Ctx* ctx, int s, double* base) { ctx->sp_base[s] = base; }
__device__ __forceinline__ void step_begin_body(Ctx* ctx) {
  ctx->cur.p = __longlong_as_double(0x7ff8000000000000LL);
  ctx->cur.e10 = __longlong_as_double(0x7ff8000000000000LL);
}
__global__ void k_step_begin(Ctx* ctx) { step_begin_body(ctx); }
__device__ __forceinline__ void step_end_body(Ctx* ctx, StepLog* logs, int cap) {
  ctx->step += 1;
  ctx->t += ctx->dt;
  ctx->cur.t = ctx->t;
  ctx->cur.step = ctx->step;
  ctx->cur.dt = ctx->dt;
  if (logs) logs[(ctx->step - 1) % cap] = ctx->cur;
}
__global__ void k_step_end(Ctx* ctx, StepLog* logs, int cap) { step_end_body(ctx, logs, cap); }

// --------------------------------------------------------------------------
// Batch groups: the per-member kernels of a step as group-wide launches, one
// launch for all members.  Members share dims and halo; each member's own
// arguments (context, P, partials, coefficients, particle arrays) come from a
// device array indexed by blockIdx.y (blockIdx.z / nz for the rhs, blockIdx.x
// for the one-block kernels), and blockIdx.x and gridDim.x keep the meaning
// they have in the member's own launch.  So each member computes exactly what
// its own kernels compute, and its reductions group their partial sums in the
// same order.
// --------------------------------------------------------------------------
template <typename T>
struct GroupMember {
  Ctx* ctx;
  T* P;
  double* partials;
  T* dU[3];
  StepLog* logs;
  int logs_cap;
  int itrmax;
  int nspecies;  // 0 in FlowMode
  int pad_;
  RhsCoef rc;
  DtCoef dc;
  PartCoef pc;
  double power;  // linear-power P0
  SpeciesDev sp[LCS_MAX_SPECIES];
};
template <typename T>
__global__ void __launch_bounds__(256) k_cfl_max_group(const GroupMember<T>* __restrict__ gm, Grid g) {
  const GroupMember<T>& m = gm[blockIdx.y];
  cfl_max_body<T>(m.ctx, g, m.partials);
}
template <typename T>
__global__ void __launch_bounds__(256) k_cfl_finalize_group(const GroupMember<T>* __restrict__ gm, int nb) {
  const GroupMember<T>& m = gm[blockIdx.x];
  cfl_finalize_body(m.ctx, m.partials, nb, m.dc, 0, nullptr);
}
template <typename T>
__global__ void __launch_bounds__(256) k_rhs_group(const GroupMember<T>* __restrict__ gm, Grid g, int in_set,
                                                   int out_set, int u0_set, int mode, int use_stage_dt) {
  const int nz = g.n[2];
  const GroupMember<T>& m = gm[blockIdx.z / nz];
  rhs_body<T>(m.ctx, g, m.P, in_set, out_set, u0_set, mode, m.dU[0], m.dU[1], m.dU[2], m.rc, use_stage_dt, 0.0,
              (int)(blockIdx.z % nz));
}
template <typename T>
__global__ void __launch_bounds__(256) k_particles_group(const GroupMember<T>* __restrict__ gm, Grid g, int s,
                                                         int stage, int modes) {
  const GroupMember<T>& m = gm[blockIdx.y];
  if (s >= m.nspecies) return;
  particles_body<T>(m.ctx, g, s, m.sp[s], m.pc, stage, modes, 1, 0.0);
}
template <typename T>
__global__ void __launch_bounds__(256) k_lf_sums_group(const GroupMember<T>* __restrict__ gm, Grid g) {
  const GroupMember<T>& m = gm[blockIdx.y];
  lf_sums_body<T>(m.ctx, g, m.partials);
}
template <typename T>
__global__ void __launch_bounds__(256) k_lf_coef_group(const GroupMember<T>* __restrict__ gm, int nb, double count) {
  const GroupMember<T>& m = gm[blockIdx.x];
  lf_coef_body(m.ctx, m.partials, nb, count, m.power);
}
template <typename T>
__global__ void __launch_bounds__(256) k_lf_apply_group(const GroupMember<T>* __restrict__ gm, Grid g) {
  const GroupMember<T>& m = gm[blockIdx.y];
  lf_apply_body<T>(m.ctx, g, m.partials);
}
template <typename T>
__global__ void __launch_bounds__(256) k_power_finalize_group(const GroupMember<T>* __restrict__ gm, int nb,
                                                              double count) {
  const GroupMember<T>& m = gm[blockIdx.x];
  power_finalize_body(m.ctx, m.partials, nb, count, (double)NAN);
}
// the one-thread kernels of a step, one thread per member: what 0 step_begin,
// 1 set_stage_dt(stage), 2 couple_reset, 3 couple_log(stage), 4 step_end
template <typename T>
__global__ void k_member_op_group(const GroupMember<T>* __restrict__ gm, int M, int what, int stage) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= M) return;
  const GroupMember<T>& m = gm[q];
  Ctx* ctx = m.ctx;
  switch (what) {
    case 0: step_begin_body(ctx); break;
    case 1: stage_dt_body(ctx, stage); break;
    case 2: couple_reset_body(ctx, m.itrmax); break;
    case 3: couple_log_body(ctx, stage); break;
    default: step_end_body(ctx, m.logs, m.logs_cap);
  }
}

}  // namespace
}  // namespace lcs
