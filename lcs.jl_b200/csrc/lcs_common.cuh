// lcs_common.cuh -- device data layout, the per-handle device context and the
// staggered-grid stencil primitives of the B200 time-step backend.
//
// Layout in HBM.  Every haloed field (U,V,W,U2,V2,W2,P and three spare
// velocity buffers) is one (n+2h)^3 box, x fastest, with logical index
// i in 1-h..n+h (the reference's `@offsetviews`, lib/offsets/src/Offsets.jl).
// Rows are padded so that logical i = 1 starts on a 128-byte boundary and
// every row starts on one; a warp reading 32 consecutive x cells of a row
// then touches whole 32-byte sectors only.
#pragma once

#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

namespace lcs {

// 2*pi as Julia's `2pi` rounds it (src/LCS.jl:17).
constexpr double kDomainLength = 2.0 * 3.14159265358979323846;

struct Grid {
  int n[3];         // interior cells per axis
  int h;            // halo width
  int64_t px;       // row pitch (elements)
  int64_t pz;       // plane pitch (elements) = px * (ny + 2h)
  int64_t off0;     // element offset of logical (0,0,0)
  int64_t elems;    // elements per haloed field
  __host__ __device__ __forceinline__ int64_t at(int i, int j, int k) const {
    return off0 + (int64_t)i + (int64_t)j * px + (int64_t)k * pz;
  }
};

// Column of logical i = 1 and the row-pitch granule: one 128-byte line.
template <typename T> constexpr int kAlignElems = 128 / (int)sizeof(T);

template <typename T>
inline Grid make_grid(const int dims[3], int h) {
  Grid g;
  for (int a = 0; a < 3; a++) g.n[a] = dims[a];
  g.h = h;
  const int A = kAlignElems<T>;
  const int64_t need = (int64_t)A + dims[0] + h;  // columns A-h .. A+n+h-1 hold i = 1-h .. n+h
  g.px = (need + A - 1) / A * A;
  g.pz = g.px * (dims[1] + 2 * h);
  // logical (i,j,k) -> (k+h-1)*pz + (j+h-1)*px + (i-1+A)
  g.off0 = (int64_t)(h - 1) * g.pz + (int64_t)(h - 1) * g.px + (A - 1);
  g.elems = g.pz * (dims[2] + 2 * h);
  return g;
}

struct Box {
  int lo[3], hi[3];  // inclusive logical bounds
  __host__ __device__ __forceinline__ bool contains(int i, int j, int k) const {
    return i >= lo[0] && i <= hi[0] && j >= lo[1] && j <= hi[1] && k >= lo[2] && k <= hi[2];
  }
  __host__ __device__ __forceinline__ int len(int a) const { return hi[a] - lo[a] + 1; }
};

inline Box cube(const Grid& g, int lo, int hiplus) {
  Box b;
  for (int a = 0; a < 3; a++) { b.lo[a] = lo; b.hi[a] = g.n[a] + hiplus; }
  return b;
}

// Velocity sets addressed through the device context so that the HSMAC
// ping-pong can swap buffers on the device (inside a CUDA graph whose sweep
// count is data dependent).
enum : int { kSetUs = 0, kSetUs2 = 1, kSetSpare = 2 };

struct CoupleState {
  int itr;      // reference `itr`
  int sweeps;   // sweeps executed
  int done;     // exit criterion met
  int cont;     // WHILE-loop condition value (itr < itrmax && !done)
  int groups;   // iterations of the graph's WHILE loop so far (bounds it)
  double div;   // last residual
  double sum;   // last sum of div^2
};

struct StepLog {
  int itr1, sweeps1, itr2, sweeps2;
  double div1, div2, p, e10, dt, t;
  long long step;
};

// Device-resident context.  Kernels read field pointers and the time step
// from here, so the same launches serve direct calls and graph replays.
struct Ctx {
  void* vel[3][3];      // [set][component] haloed velocity buffers
  int vphys[3][3];      // [set][component] index 0..8 of the physical buffer (tensor map)
  double dt;            // state.dt
  double t;             // state.t
  long long step;       // state.step
  double dt_particles;  // Particles.timestep (constant while diameters are)
  double scal[8];       // scratch scalars of the current stage (means, amplitudes)
  CoupleState cs;       // HSMAC loop state of the current couple
  StepLog cur;          // log of the step in progress
  unsigned int ticket;  // last-block-done counter
  int nonfinite;        // sticky: a NaN/Inf dt or residual was seen
  int wait_error;       // sticky: a bounded device wait (TMA copy, grid barrier) ran out
  unsigned int gbar_count;  // arrivals at the grid-wide barriers of a cooperative launch (0 between launches)
  double* sp_base[16];  // property block of each species: 16 FP64 properties, then the ids
  // test hook (lcs_debug_unreachable_waits): 1 makes the grid barriers of the
  // cooperative face kernel wait for one arrival more than there are blocks,
  // 2 makes the sweep's TMA plane barriers expect 16 bytes more than its
  // copies deliver; either wait then runs out at its bound.  0 in production.
  int debug_wait;
};

// ---- stencil primitives (src/diff.jl:1-39), same evaluation order --------
template <typename T> __device__ __forceinline__ T interp_o2_at_half(T a, T b) { return T(0.5) * (a + b); }
template <typename T> __device__ __forceinline__ T interp_o4_at_half(T a, T b, T c, T d) {
  return T(1.0 / 16.0) * (-a + T(9) * b + T(9) * c - d);
}
template <typename T> __device__ __forceinline__ T diff1_o2_at_half(T a, T b) { return -a + b; }
template <typename T> __device__ __forceinline__ T diff2_o4_at_node(T a, T b, T c, T d, T e) {
  return T(1.0 / 12.0) * (-a + T(16) * b - T(30) * c + T(16) * d - e);
}
template <typename T> __device__ __forceinline__ T sum_flux_o4(T j1a, T j1b, T j3a, T j3b) {
  return T(9.0 / 8.0) * (-j1a + j1b) - T((1.0 / 8.0) * (1.0 / 3.0)) * (-j3a + j3b);
}

// Julia's max and min of two floats (Base.max, Base.min): a NaN operand gives
// NaN, and max(-0.0, 0.0) = 0.0, min(-0.0, 0.0) = -0.0.  C's fmax/fmin drop a
// NaN instead, which would hide a non-finite field from maximum(abs, U) and
// the time step built on it (src/flows/timestep.jl:48-64).
__host__ __device__ __forceinline__ double jl_max(double a, double b) {
  if (a != a) return a;
  if (b != b) return b;
  return (a > b || (a == b && !signbit(a))) ? a : b;
}
__host__ __device__ __forceinline__ double jl_min(double a, double b) {
  if (a != a) return a;
  if (b != b) return b;
  return (a < b || (a == b && signbit(a))) ? a : b;
}

// mod1 onto 1..n
__host__ __device__ __forceinline__ int wrap1(int i, int n) {
  int r = (i - 1) % n;
  return (r < 0 ? r + n : r) + 1;
}

}  // namespace lcs
