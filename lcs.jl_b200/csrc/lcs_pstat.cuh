// lcs_pstat.cuh -- particle statistics over the cell index:
//  - the Summary reductions of `Particles.stat` (src/particles/stat.jl:127-139,
//    src/stat.jl:20-22): sum, max and min of x, y, z, u, v, w and diams;
//  - `rdf_assume_ci` (src/particles/rdf.jl:1-103): pairs per logarithmic
//    distance bin and contact pairs, searched over the cells within
//    search_cell_size of each particle's cell (no periodic images: neighbour
//    cells outside the axes 0:nc+1 are skipped, as in the reference);
//  - `spectrum` (src/particles/spectrum.jl:11-78): sums of cos and sin of k.x
//    over the particles for every shell wavenumber and Fibonacci direction;
//  - `density` (src/particles/stat.jl:176-215): the cubic-spline SPH sum over
//    the 27 neighbouring cells.
// Distances and the SPH sum use explicit round-to-nearest intrinsics, so no
// multiply-add is contracted in either precision form: the results are those
// of the reference's expression order (Utils.norm = sqrt((dx^2 + dy^2) + dz^2),
// src/utils/fast.jl:43-47).  Pair counts are integers (exact in any order);
// the spectrum sums are FP64 in a fixed order (the reference adds them with
// atomics, in no fixed order).
#pragma once

#include "lcs_common.cuh"
#include "lcs_makeindex.cuh"

namespace lcs {
namespace {

constexpr int kPSumVals = 21;  // 7 arrays x (sum, max, min)

// per block: sum, max, min of the 7 arrays (x, y, z, u, v, w, diam)
__global__ void __launch_bounds__(256) k_psummary(const double* X, const double* Y, const double* Z, const double* U,
                                                  const double* V, const double* W, const double* D, int64_t n,
                                                  double* __restrict__ partials) {
  __shared__ double sh[8];
  const double* A[7] = {X, Y, Z, U, V, W, D};
  for (int q = 0; q < 7; q++) {
    double s = 0.0, mx = -INFINITY, mn = INFINITY;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
      const double a = A[q][i];
      s += a;
      mx = jl_max(mx, a);
      mn = jl_min(mn, a);
    }
    const double bs = block_sum<256>(s, sh);
    const double bmx = block_max<256>(mx, sh);
    const double bmn = -block_max<256>(-mn, sh);
    if (threadIdx.x == 0) {
      partials[kPSumVals * blockIdx.x + 3 * q] = bs;
      partials[kPSumVals * blockIdx.x + 3 * q + 1] = bmx;
      partials[kPSumVals * blockIdx.x + 3 * q + 2] = bmn;
    }
  }
}

__global__ void __launch_bounds__(256) k_psummary_final(const double* __restrict__ partials, int nb,
                                                        double* __restrict__ out) {
  __shared__ double sh[8];
  for (int q = 0; q < kPSumVals; q++) {
    const int kind = q % 3;  // 0 sum, 1 max, 2 min
    double v = kind == 0 ? 0.0 : (kind == 1 ? -INFINITY : INFINITY);
    for (int b = threadIdx.x; b < nb; b += 256) {
      const double x = partials[kPSumVals * b + q];
      v = kind == 0 ? v + x : (kind == 1 ? jl_max(v, x) : jl_min(v, x));
    }
    const double r = kind == 0 ? block_sum<256>(v, sh) : (kind == 1 ? block_max<256>(v, sh) : -block_max<256>(-v, sh));
    if (threadIdx.x == 0) out[q] = r;
  }
}

// cell coordinates (0-based offsets from the axis start 0) of a 1-based hash
// over the axes 0:nc+1 (Utils.decode, src/utils/hasher.jl:40-59)
__device__ __forceinline__ void cell_of(int64_t hash, const CellGeom& cg, int ci[3]) {
  int64_t lin = hash - 1;
  for (int a = 0; a < 3; a++) {
    const int64_t m = cg.nc[a] + 2;
    ci[a] = (int)(lin % m);
    lin /= m;
  }
}

__device__ __forceinline__ double dist3(double x1, double y1, double z1, double x2, double y2, double z2) {
  const double a = __dsub_rn(x1, x2), b = __dsub_rn(y1, y2), c = __dsub_rn(z1, z2);
  return sqrt(__dadd_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)), __dmul_rn(c, c)));
}

// Pairs (id1 < id2) per bin k (edges[k] < d <= edges[k+1], the bin of
// searchsortedfirst(edges, d) - 1) and contact pairs |d / diam - 1| < tol.
// Dynamic shared memory: nbins + 1 counters, then nbins + 1 edges.
__global__ void __launch_bounds__(256) k_rdf(const double* __restrict__ X, const double* __restrict__ Y,
                                             const double* __restrict__ Z, const int64_t* __restrict__ ids,
                                             const int64_t* __restrict__ hashes, const int64_t* __restrict__ starts,
                                             const int64_t* __restrict__ stops, int64_t n, CellGeom cg, int ncell,
                                             const double* __restrict__ edges_g, int nbins, double diam, double tol,
                                             unsigned long long* __restrict__ counts) {
  extern __shared__ unsigned long long rdf_sh[];
  unsigned long long* hist = rdf_sh;                   // [0, nbins): bins, [nbins]: contact
  double* edges = (double*)(rdf_sh + nbins + 1);       // nbins + 1
  for (int k = threadIdx.x; k <= nbins; k += blockDim.x) {
    hist[k] = 0ull;
    edges[k] = edges_g[k];
  }
  __syncthreads();
  const int64_t W = cg.nc[0] + 2, WH = W * (cg.nc[1] + 2);
  for (int64_t i1 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i1 < n; i1 += (int64_t)gridDim.x * blockDim.x) {
    int c1[3];
    cell_of(hashes[i1], cg, c1);
    if (c1[0] < 1 || c1[0] > cg.nc[0] || c1[1] < 1 || c1[1] > cg.nc[1] || c1[2] < 1 || c1[2] > cg.nc[2]) continue;
    const double x1 = X[i1], y1 = Y[i1], z1 = Z[i1];
    const int64_t id1 = ids[i1];
    for (int di = -ncell; di <= ncell; di++) {
      const int a = c1[0] + di;
      if (a < 0 || a > cg.nc[0] + 1) continue;
      for (int dj = -ncell; dj <= ncell; dj++) {
        const int b = c1[1] + dj;
        if (b < 0 || b > cg.nc[1] + 1) continue;
        for (int dk = -ncell; dk <= ncell; dk++) {
          const int c = c1[2] + dk;
          if (c < 0 || c > cg.nc[2] + 1) continue;
          const int64_t h2 = 1 + a + b * W + c * WH;
          const int64_t lo = starts[h2 - 1], hi = stops[h2 - 1];  // 1-based, inclusive
          for (int64_t i2 = lo; i2 <= hi; i2++) {
            if (!(id1 < ids[i2 - 1])) continue;
            const double d = dist3(x1, y1, z1, X[i2 - 1], Y[i2 - 1], Z[i2 - 1]);
            // searchsortedfirst(edges, d): first 1-based index with edges >= d
            int lo_e = 0, len = nbins + 1;
            while (len > 0) {
              const int half = len >> 1;
              if (edges[lo_e + half] < d) {
                lo_e += half + 1;
                len -= half + 1;
              } else {
                len = half;
              }
            }
            const int k = lo_e;  // = searchsortedfirst - 1 (1-based bin), 0-based: k - 1
            if (k >= 1 && k <= nbins) atomicAdd(&hist[k - 1], 1ull);
            if (fabs(__dsub_rn(d / diam, 1.0)) < tol) atomicAdd(&hist[nbins], 1ull);
          }
        }
      }
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k <= nbins; k += blockDim.x)
    if (hist[k]) atomicAdd(&counts[k], hist[k]);
}

// Spectrum sums: block (bx, by) adds cos and sin of k.x over its particle
// chunk for the pairs [by * 256 * kSpecPairs, ...) (thread t: pairs t + 256 j),
// particles staged in shared memory; partials[(bx * npairs + pair) * 2 + {0,1}].
constexpr int kSpecPairs = 4;
constexpr int kSpecTile = 512;
__global__ void __launch_bounds__(256) k_spectrum(const double* __restrict__ X, const double* __restrict__ Y,
                                                  const double* __restrict__ Z, int64_t n,
                                                  const double* __restrict__ kvec, int npairs,
                                                  double* __restrict__ partials) {
  __shared__ double px[kSpecTile], py[kSpecTile], pz[kSpecTile];
  const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
  const int64_t p0 = (int64_t)blockIdx.x * chunk, p1 = p0 + chunk < n ? p0 + chunk : n;
  double kx[kSpecPairs], ky[kSpecPairs], kz[kSpecPairs], ac[kSpecPairs], as[kSpecPairs];
  int pr[kSpecPairs];
#pragma unroll
  for (int j = 0; j < kSpecPairs; j++) {
    pr[j] = blockIdx.y * 256 * kSpecPairs + threadIdx.x + 256 * j;
    const int q = pr[j] < npairs ? pr[j] : 0;
    kx[j] = kvec[3 * q];
    ky[j] = kvec[3 * q + 1];
    kz[j] = kvec[3 * q + 2];
    ac[j] = 0.0;
    as[j] = 0.0;
  }
  for (int64_t t0 = p0; t0 < p1; t0 += kSpecTile) {
    const int m = (int)(p1 - t0 < kSpecTile ? p1 - t0 : kSpecTile);
    __syncthreads();
    for (int i = threadIdx.x; i < m; i += 256) {
      px[i] = X[t0 + i];
      py[i] = Y[t0 + i];
      pz[i] = Z[t0 + i];
    }
    __syncthreads();
    for (int i = 0; i < m; i++) {
      const double x = px[i], y = py[i], z = pz[i];
#pragma unroll
      for (int j = 0; j < kSpecPairs; j++) {
        // sum(k .* x) = (kx x + ky y) + kz z
        const double kd = __dadd_rn(__dadd_rn(__dmul_rn(kx[j], x), __dmul_rn(ky[j], y)), __dmul_rn(kz[j], z));
        double s, c;
        sincos(kd, &s, &c);
        ac[j] += c;
        as[j] += s;
      }
    }
  }
#pragma unroll
  for (int j = 0; j < kSpecPairs; j++)
    if (pr[j] < npairs) {
      partials[((int64_t)blockIdx.x * npairs + pr[j]) * 2] = ac[j];
      partials[((int64_t)blockIdx.x * npairs + pr[j]) * 2 + 1] = as[j];
    }
}

__global__ void __launch_bounds__(256) k_spectrum_final(const double* __restrict__ partials, int nb, int npairs,
                                                        double* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2 * npairs) return;
  double s = 0.0;
  for (int b = 0; b < nb; b++) s += partials[(int64_t)b * 2 * npairs + t];
  out[t] = s;
}

// cubic_spline_kernel (stat.jl:217-227) with factor = 1 / (pi h^3) given
__device__ __forceinline__ double cubic_spline(double r, double h, double factor) {
  const double q = r / h;
  if (q < 1.0) {
    const double q2 = __dmul_rn(q, q), q3 = __dmul_rn(q2, q);
    return __dmul_rn(factor, __dadd_rn(__dsub_rn(1.0, __dmul_rn(1.5, q2)), __dmul_rn(0.75, q3)));
  }
  if (q < 2.0) {
    const double t = __dsub_rn(2.0, q);
    return __dmul_rn(__dmul_rn(factor, 0.25), __dmul_rn(__dmul_rn(t, t), t));
  }
  return 0.0;
}

__global__ void __launch_bounds__(256) k_density(const double* __restrict__ X, const double* __restrict__ Y,
                                                 const double* __restrict__ Z, const int64_t* __restrict__ hashes,
                                                 const int64_t* __restrict__ starts, const int64_t* __restrict__ stops,
                                                 int64_t n, CellGeom cg, double h, double factor,
                                                 double* __restrict__ rho_out) {
  const int64_t W = cg.nc[0] + 2, WH = W * (cg.nc[1] + 2);
  for (int64_t i1 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i1 < n; i1 += (int64_t)gridDim.x * blockDim.x) {
    int c1[3];
    cell_of(hashes[i1], cg, c1);
    double rho = 0.0;
    if (c1[0] >= 1 && c1[0] <= cg.nc[0] && c1[1] >= 1 && c1[1] <= cg.nc[1] && c1[2] >= 1 && c1[2] <= cg.nc[2]) {
      const double x1 = X[i1], y1 = Y[i1], z1 = Z[i1];
      const double h2x = __dmul_rn(2.0, h);
      for (int di = -1; di <= 1; di++)
        for (int dj = -1; dj <= 1; dj++)
          for (int dk = -1; dk <= 1; dk++) {
            const int64_t hash2 = 1 + (c1[0] + di) + (c1[1] + dj) * W + (c1[2] + dk) * WH;
            const int64_t lo = starts[hash2 - 1], hi = stops[hash2 - 1];
            for (int64_t i2 = lo; i2 <= hi; i2++) {
              const double d = dist3(x1, y1, z1, X[i2 - 1], Y[i2 - 1], Z[i2 - 1]);
              if (d < h2x) rho = __dadd_rn(rho, cubic_spline(d, h, factor));
            }
          }
    }
    rho_out[i1] = rho;
  }
}

}  // namespace
}  // namespace lcs
