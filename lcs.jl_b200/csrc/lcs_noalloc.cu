// lcs_noalloc.cu -- the CFL time step on caller-owned device arrays, with no
// device allocation.
//
// Some callers cannot call cudaMalloc: a process whose device memory is owned
// by another allocator (a Julia CUDA.jl pool, a serving process with a fixed
// per-request budget) must not have a library grab memory behind its back,
// and code recording a CUDA stream capture cannot allocate at all.  This entry
// point lets them run `Flows.timestep` (src/flows/timestep.jl:18-65) on U, V,
// W arrays they already hold.  Its only scratch is the file-scope array below:
// one partial maximum per z-plane and component, so grids of at most
// LCS_NOALLOC_MAX_PLANES planes along z.  Every GPU that loads the library
// holds that array until the process exits.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>

#include "../../include/lcs_b200.h"

namespace lcs {
void set_global_error_message(const char* msg);  // lcs_api.cu: lcs_last_error(NULL)
}

namespace {

constexpr int kMaxPlanes = LCS_NOALLOC_MAX_PLANES;
constexpr double kTwoPi = 2.0 * 3.14159265358979323846;

// Per-plane partial maxima of |U|, |V|, |W| interpolated to the cell centre:
// [component][plane].  Shared by every call on a device.
static __device__ __align__(256) double g_cfl_scratch[3 * kMaxPlanes];

int fail(int code, const char* msg) {
  lcs::set_global_error_message(msg);
  return code;
}

struct Layout {
  int n[3], h;
  long long sx, sy;  // elements per row, per plane of the haloed (n+2h)^3 box
};

__device__ __forceinline__ int wrap1(int i, int n) {
  int r = (i - 1) % n;
  return (r < 0 ? r + n : r) + 1;
}
__device__ __forceinline__ long long at(const Layout& L, int i, int j, int k) {
  return ((long long)(k + L.h - 1) * L.sy) + (long long)(j + L.h - 1) * L.sx + (i + L.h - 1);
}
__device__ __forceinline__ double o4(double a, double b, double c, double d) {
  return (1.0 / 16.0) * (-a + 9.0 * b + 9.0 * c - d);
}
// Julia's max/min of floats: a NaN operand gives NaN (fmax/fmin would drop
// it), so a non-finite U, V or W gives a NaN dt as maximum(abs, U) does.
__device__ __forceinline__ double jl_max(double a, double b) {
  if (a != a) return a;
  if (b != b) return b;
  return (a > b || (a == b && !signbit(a))) ? a : b;
}
__device__ __forceinline__ double jl_min(double a, double b) {
  if (a != a) return a;
  if (b != b) return b;
  return (a < b || (a == b && signbit(a))) ? a : b;
}

// One block per z-plane: the plane's maxima of |uc|, |vc|, |wc|, the o4
// cell-centre interpolations of flows/timestep.jl:35-45.  The interior is
// read with periodic wrapping, which is what the FaceHalo fill of the
// reference places in the halo, so the caller's halo cells are not read.
__global__ void __launch_bounds__(256) k_cfl_planes(const double* __restrict__ U, const double* __restrict__ V,
                                                    const double* __restrict__ W, Layout L, double* scratch) {
  __shared__ double sh[3][8];
  const int k = 1 + blockIdx.x;
  const int nx = L.n[0], ny = L.n[1], nz = L.n[2];
  double mu = 0.0, mv = 0.0, mw = 0.0;
  for (int t = threadIdx.x; t < nx * ny; t += blockDim.x) {
    const int i = 1 + t % nx, j = 1 + t / nx;
    const double uc = o4(U[at(L, wrap1(i - 2, nx), j, k)], U[at(L, wrap1(i - 1, nx), j, k)], U[at(L, i, j, k)],
                         U[at(L, wrap1(i + 1, nx), j, k)]);
    const double vc = o4(V[at(L, i, wrap1(j - 2, ny), k)], V[at(L, i, wrap1(j - 1, ny), k)], V[at(L, i, j, k)],
                         V[at(L, i, wrap1(j + 1, ny), k)]);
    const double wc = o4(W[at(L, i, j, wrap1(k - 2, nz))], W[at(L, i, j, wrap1(k - 1, nz))], W[at(L, i, j, k)],
                         W[at(L, i, j, wrap1(k + 1, nz))]);
    mu = jl_max(mu, fabs(uc));
    mv = jl_max(mv, fabs(vc));
    mw = jl_max(mw, fabs(wc));
  }
  double m[3] = {mu, mv, mw};
  for (int c = 0; c < 3; c++) {
    double v = m[c];
    for (int o = 16; o > 0; o >>= 1) v = jl_max(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (threadIdx.x % 32 == 0) sh[c][threadIdx.x / 32] = v;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double v = sh[threadIdx.x][0];
    for (int w = 1; w < 8; w++) v = jl_max(v, sh[threadIdx.x][w]);
    scratch[threadIdx.x * kMaxPlanes + blockIdx.x] = v;  // every slot of this call is rewritten
  }
}

struct DtArgs {
  double cfl, dtmax, dx, dy, dz, Re;
};

// Maxima over the planes, then the candidates of flows/timestep.jl:53-64.
__global__ void __launch_bounds__(256) k_cfl_final(const double* scratch, int nz, DtArgs a, double* dt_out) {
  __shared__ double sh[3][8];
  for (int c = 0; c < 3; c++) {
    double v = 0.0;
    for (int k = threadIdx.x; k < nz; k += blockDim.x) v = jl_max(v, scratch[c * kMaxPlanes + k]);
    for (int o = 16; o > 0; o >>= 1) v = jl_max(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (threadIdx.x % 32 == 0) sh[c][threadIdx.x / 32] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double m[3];
    for (int c = 0; c < 3; c++) {
      m[c] = sh[c][0];
      for (int w = 1; w < 8; w++) m[c] = jl_max(m[c], sh[c][w]);
      m[c] = m[c] + 1e-10;
    }
    double d = a.dtmax;
    d = jl_min(d, a.cfl * a.dx / m[0]);
    d = jl_min(d, a.cfl * a.dy / m[1]);
    d = jl_min(d, a.cfl * a.dz / m[2]);
    d = jl_min(d, 0.5 * ((a.dx / 2.0) * (a.dx / 2.0)) / (1.0 / a.Re));
    *dt_out = d;
  }
}

// Device address of the scratch array in the current device's context.  Host
// code only sees a host-side stand-in for the symbol, so the address is looked
// up with cudaGetSymbolAddress (which allocates nothing) on every call: a
// context that the caller reset or destroyed and created again (CUDA.jl's
// device_reset!, cudaDeviceReset) loads the module again at another address,
// and an address kept from before would point into freed memory.  The first
// call on a device loads the module, so it should come before any stream
// capture.
int scratch_for_current_device(double** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) {
    cudaGetLastError();
    return fail(LCS_ECUDA, "lcs_flow_timestep_noalloc: no current CUDA device");
  }
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_cfl_scratch);
  if (e != cudaSuccess || p == nullptr) {
    cudaGetLastError();
    return fail(LCS_ECUDA, "lcs_flow_timestep_noalloc: cudaGetSymbolAddress of the scratch array failed");
  }
  *out = (double*)p;
  return LCS_OK;
}

}  // namespace

extern "C" {

LCS_API int lcs_flow_timestep_noalloc(const double* U, const double* V, const double* W, const int32_t dims[3],
                                      int32_t halo_size, double cfl, double dtmax, double Re, double* dt_out,
                                      void* stream) {
  if (!U || !V || !W || !dims || !dt_out) return fail(LCS_EINVAL, "lcs_flow_timestep_noalloc: null argument");
  for (int a = 0; a < 3; a++)
    if (dims[a] < 4) return fail(LCS_EINVAL, "lcs_flow_timestep_noalloc: grid dims must be >= 4");
  if (halo_size < 0) return fail(LCS_EINVAL, "lcs_flow_timestep_noalloc: negative halo_size");
  if (dims[2] > kMaxPlanes) {
    char msg[200];
    snprintf(msg, sizeof msg,
             "lcs_flow_timestep_noalloc: dims[2] = %d exceeds the %d z-planes its static scratch holds",
             (int)dims[2], kMaxPlanes);
    return fail(LCS_EINVAL, msg);
  }
  if (!(cfl > 0) || !(dtmax > 0) || !(Re > 0)) return fail(LCS_EINVAL, "lcs_flow_timestep_noalloc: cfl, dtmax, Re must be positive");
  double* scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc) return rc;
  Layout L;
  for (int a = 0; a < 3; a++) L.n[a] = dims[a];
  L.h = halo_size;
  L.sx = dims[0] + 2LL * halo_size;
  L.sy = L.sx * (dims[1] + 2LL * halo_size);
  cudaStream_t s = (cudaStream_t)stream;
  k_cfl_planes<<<dims[2], 256, 0, s>>>(U, V, W, L, scratch);
  DtArgs a;
  a.cfl = cfl;
  a.dtmax = dtmax;
  a.dx = kTwoPi / dims[0];
  a.dy = kTwoPi / dims[1];
  a.dz = kTwoPi / dims[2];
  a.Re = Re;
  k_cfl_final<<<1, 256, 0, s>>>(scratch, dims[2], a, dt_out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    char msg[200];
    snprintf(msg, sizeof msg, "lcs_flow_timestep_noalloc: launch failed: %s", cudaGetErrorString(e));
    return fail(LCS_ECUDA, msg);
  }
  return LCS_OK;
}

}  // extern "C"
