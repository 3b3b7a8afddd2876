// lcs_makeindex.cuh -- `Particles.makeindex!` (src/particles/makeindex.jl:29-67):
// the cell-based spatial index of a particle species.
//
//  - cell index ci = unsafe_floor(Int32, (x - x0) / dxc) + 1 per axis, with
//    x0 = 0 and dxc = (2pi/n) * grid_ratio (particles/config.jl:60), the
//    division and floor in FP64 as in the reference (makeindex.jl:50);
//  - hash = the column-major linear index of ci over the cell axes 0:nc+1,
//    1-based (Utils.Hasher, src/utils/hasher.jl:15-38);
//  - a stable sort of the particles by hash (AcceleratedKernels sortperm!,
//    src/utils/sort.jl:3-5; here a stable LSD radix sort of (hash, index)
//    pairs), after which every property is permuted (makeindex.jl:56-58);
//  - starts[x] / stops[x] for every hash x: the first index whose hash is >= x
//    and the last index whose hash is <= x, 1-based, the results of the binary
//    searches of src/utils/fast.jl:8-40 (makeindex.jl:60-66), here from a
//    max-scan of the run ends of the sorted hashes (k_starts_stops).
// Positions must lie in the periodic box (as after boundary!): a position
// outside the cell axes 0:nc+1 gets a hash outside 1:(nc+2)^3, as in the
// reference, and it is only sorted, never used as an address.
#pragma once

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "lcs_common.cuh"

namespace lcs {
namespace {

struct CellGeom {
  int nc[3];     // cells per axis = n / grid_ratio
  double dxc[3]; // cell spacing
};

__global__ void __launch_bounds__(256) k_cell_hash(const double* __restrict__ X, const double* __restrict__ Y,
                                                   const double* __restrict__ Z, int64_t n, CellGeom cg,
                                                   uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double x[3] = {X[i], Y[i], Z[i]};
    int64_t h = 1, stride = 1;
    for (int a = 0; a < 3; a++) {
      const int ci = (int)floor((x[a] - 0.0) / cg.dxc[a]) + 1;  // unsafe_floor(Int32, .) + 1
      h += (int64_t)ci * stride;                                 // offset from the axis start 0
      stride *= cg.nc[a] + 2;
    }
    keys[i] = (uint32_t)h;
    vals[i] = (uint32_t)i;
  }
}

// tmp[q * n + i] = A[q * n + perm[i]] for the 17 8-byte properties of a
// species, held back to back (16 FP64 properties, then the Int64 ids): one
// read of perm and 17 independent loads in flight per particle.
constexpr int kSortedProps = 17;
__global__ void __launch_bounds__(256) k_permute_props(const uint64_t* __restrict__ A,
                                                       const uint32_t* __restrict__ perm, int64_t n,
                                                       uint64_t* __restrict__ tmp) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = perm[i];
    uint64_t v[kSortedProps];
#pragma unroll
    for (int q = 0; q < kSortedProps; q++) v[q] = __ldg(A + q * n + j);
#pragma unroll
    for (int q = 0; q < kSortedProps; q++) tmp[q * n + i] = v[q];
  }
}

// hashes[i] = keys[i] (Int64); at the end of every run of equal hashes x in
// 0..H, S[x] = its 1-based last index = #(hashes <= x).  Hashes above H write
// nothing (they lie outside the cell axes).
__global__ void __launch_bounds__(256) k_hash_runs(const uint32_t* __restrict__ keys, int64_t n, int64_t H,
                                                   int64_t* __restrict__ hashes, int64_t* __restrict__ S) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t k = keys[i];
    hashes[i] = (int64_t)k;
    if ((i == n - 1 || keys[i + 1] != k) && (int64_t)k <= H) S[k] = i + 1;
  }
}

struct MaxI64 {
  __device__ __forceinline__ int64_t operator()(int64_t a, int64_t b) const { return a > b ? a : b; }
};

// From M = the inclusive max-scan of S (M[x] = #(hashes <= x)), the binary
// searches of src/utils/fast.jl:8-40 over the sorted hashes:
//   searchsortedfirst(hashes, x) = #(hashes < x) + 1 = M[x-1] + 1,
//   searchsortedlast(hashes, x)  = #(hashes <= x)    = M[x],
// for every hash x = 1..H, exactly (the hashes are integers).
__global__ void __launch_bounds__(256) k_starts_stops(const int64_t* __restrict__ M, int64_t H,
                                                      int64_t* __restrict__ starts, int64_t* __restrict__ stops) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < H; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t a = M[t], b = M[t + 1];
    starts[t] = a + 1;
    stops[t] = b;
  }
}

}  // namespace
}  // namespace lcs
