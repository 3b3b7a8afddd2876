// lcs_hsmac_tma.cuh -- the fused red-black HSMAC sweep fed by TMA.
//
// Same computation as k_hsmac_fused (both colour phases of the reference's
// `foraxes(...; coloring=RedBlackFast())` sweep over a box D, hsmac.jl:1-35,
// ping-ponged so that one pass replaces the two in-place launches), arranged
// for throughput on sm_100a:
//  - plane tiles of U, V, W (2-cell halo) and P are brought into a shared
//    memory ring by cp.async.bulk.tensor loads completing on mbarriers,
//    two planes ahead of the plane being computed; no per-thread loads;
//  - every thread owns an x-pair of cells, one of each colour, so both colour
//    phases keep all lanes busy (no red-black divergence);
//  - writes are 16-byte stores of a pair; P is updated in place.
// Waits on the mbarriers are bounded; a wait that runs out sets ctx->wait_error
// and the kernel stops computing (the host reports LCS_ETIMEDOUT).
#pragma once

#include <cuda.h>

#include <type_traits>

#include "lcs_common.cuh"

namespace lcs {
namespace {

constexpr int kVelMaps = 9;

// Kernel parameter (__grid_constant__): tensor maps of the 9 physical
// velocity buffers (box TX+4 x TY+4 x 1) and of P (box TX x TY x 1).
struct TensorMaps {
  CUtensorMap vel[kVelMaps];
  CUtensorMap P;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// 3-D tiled TMA load into shared memory, completion counted on `bar`.  No
// multicast: every CTA loads its own tiles from this GPU's memory.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// Bounded wait: true when the phase completed, false after 2^22 polls or
// about 0.25 s (5e8 SM cycles), whichever comes first.  A try_wait may itself
// suspend the thread for a while, so the poll count alone does not bound the
// time.  The clock is read only once the first poll has failed.
constexpr long long kMbarWaitCycles = 500000000;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  for (int it = 0; it < (1 << 22); it++) {
    if (mbar_try_wait(bar, parity)) return true;
    if (clock64() - t0 > kMbarWaitCycles) break;
  }
  return false;
}

template <int TX, int TY, int NS>
struct TmaLayout {
  static constexpr int VW = TX + 4, VH = TY + 4;  // velocity tile with a 2-cell halo
  static constexpr int VEL_TILE = VW * VH;        // doubles per field per plane
  static constexpr int P_TILE = TX * TY;
  static constexpr int DW = TX + 3, DH = TY + 3;  // dp of cells x0-1 .. x0+TX+1
  static constexpr size_t vel_bytes = (size_t)NS * 3 * VEL_TILE * 8;
  static constexpr size_t p_bytes = (size_t)NS * P_TILE * 8;
  // the dp ring sits between the velocity and P rings: the mask-free path of
  // full tiles reads (and discards) neighbours up to a row beyond it
  static constexpr size_t dp_bytes = ((size_t)3 * DW * DH * 8 + 127) / 128 * 128;
  static constexpr size_t bar_bytes = 8 * NS;
  static constexpr size_t red_bytes = 8 * 32;
  static constexpr size_t total = vel_bytes + p_bytes + dp_bytes + bar_bytes + red_bytes + 16;
  static_assert((VEL_TILE * 8) % 128 == 0, "TMA destinations must stay 128-byte aligned");
  static_assert((P_TILE * 8) % 128 == 0, "TMA destinations must stay 128-byte aligned");
};

// Threads of a CTA: one per phase-X item (an x-pair of the dp region, whose
// rows are y0-1 .. y0+TY+1), rounded up to whole warps; the first
// (TX/2)*TY of them also own an output pair in phase Y.
template <int TX, int TY>
struct TmaThreads {
  static constexpr int NITEM = (TX / 2 + 2) * (TY + 3);
  static constexpr int NT = (NITEM + 31) / 32 * 32;
  static constexpr int MINB = NT <= 512 ? 2 : 1;  // resident CTAs the register budget is sized for
};

// Adds the contributions of the two cells sharing a face in the order of the
// in-place sweep: the colour-0 cell's first, then the colour-1 cell's.
// `sa` is +1 for the face's lower cell (its own face, `+= dp*dci`) and the
// upper cell subtracts (`-= dp*dci`); a cell outside D contributes nothing.
__device__ __forceinline__ double face_update(double val, bool lower_first, bool ma, double da, bool mb, double db,
                                              double dci) {
  // lower cell a (adds), upper cell b (subtracts)
  const double ta = da * dci, tb = db * dci;
  if (lower_first) {
    val = ma ? val + ta : val;
    val = mb ? val - tb : val;
  } else {
    val = mb ? val - tb : val;
    val = ma ? val + ta : val;
  }
  return val;
}

// x0 (a tile's first output column) is odd, so that the 16-byte rule of the
// tiled TMA holds for the velocity box (starting at x0-2) and for the P box
// (starting at x0), and the output pairs (x0+2p, x0+2p+1) are 16-byte aligned.
//
// Work items are (z chunk, tile column), chunk major, x fastest: CTA b takes
// items b, b+G, b+2G, ... so that the CTAs resident at any moment work on
// neighbouring columns of the same planes and share their tile halos in L2.
//
// Per plane s (one iteration):
//   phase X: for every pair of the dp region, the colour-0 cell at plane s and
//            the colour-1 cell at plane s-1 are the same (i, j); one thread
//            computes dp0 there at s and then dp1 there at s-1, whose only
//            dependency on plane s is that dp0 (held in a register);
//   phase Y: faces U, V and P at plane s-1, faces W at plane s-2 (which need
//            dp at s-2 and s-1, both complete after phase X).
template <int TX, int TY, int NS>
__global__ void __launch_bounds__(TmaThreads<TX, TY>::NT, TmaThreads<TX, TY>::MINB) k_hsmac_tma(Ctx* __restrict__ ctx, Grid g, int set,
                                                            const __grid_constant__ TensorMaps tm,
                                                            double* __restrict__ P, Box D, Box out, Box gb,
                                                            int x_origin, int gx, int gy, int zc, int nitems,
                                                            HsmacCoef cf,
                                                            double* __restrict__ partials, int finalize,
                                                            int group_end) {
  using L = TmaLayout<TX, TY, NS>;
  constexpr int NT = TmaThreads<TX, TY>::NT;
  constexpr int NP = (TX / 2) * TY;  // output pairs (phase Y)
  constexpr int PW = TX / 2 + 2;                  // pairs per row of the dp region (x0-1 .. x0+TX+2)
  constexpr int NITEM = PW * (TY + 3);            // rows y0-1 .. y0+TY+1
  constexpr int NROUND = (NITEM + NT - 1) / NT;
  constexpr int VW = L::VW, DW = L::DW, VT = L::VEL_TILE, DP = L::DW * L::DH;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  double* svel = (double*)smem_raw;                                 // [NS][3][VH][VW]
  double* sdp = (double*)(smem_raw + L::vel_bytes);                 // [3][DH][DW]
  double* sP = (double*)(smem_raw + L::vel_bytes + L::dp_bytes);    // [NS][TY][TX]
  uint64_t* bars = (uint64_t*)(smem_raw + L::vel_bytes + L::p_bytes + L::dp_bytes);
  double* red = (double*)(smem_raw + L::vel_bytes + L::p_bytes + L::dp_bytes + L::bar_bytes);
  int* last_flag = (int*)(red + 32);

  const int tid = threadIdx.x;
  const bool skip = ctx->cs.done != 0;
  const int nx = g.n[0], ny = g.n[1], nz = g.n[2], h = g.h;
  double racc = 0.0;

  if (!skip) {
    const int m0 = ctx->vphys[set][0], m1 = ctx->vphys[set][1], m2 = ctx->vphys[set][2];
    double* Uo = (double*)ctx->vel[kSetSpare][0];
    double* Vo = (double*)ctx->vel[kSetSpare][1];
    double* Wo = (double*)ctx->vel[kSetSpare][2];
    const double dxi = cf.dxi, dyi = cf.dyi, dzi = cf.dzi, dl = cf.dl, om = cf.omega;
    const double dti = 1.0 / ctx->scal[0];
    const int A = kAlignElems<double>;
    const uint32_t vel_tx = 3u * VT * 8u;
    if (tid == 0) {
      for (int q = 0; q < NS; q++) mbar_init(&bars[q], 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const int ncols = gx * gy;
    int loads = 0;  // TMA plane loads issued by this CTA: slot = index % NS, parity = (index / NS) & 1
    int issued = 0;  // thread 0: loads issued so far (index of the next one)
    bool ok = true;
    for (int item = blockIdx.x; item < nitems && ok; item += gridDim.x) {
      const int col = item % ncols;
      const int kb = gb.lo[2] + (item / ncols) * zc;
      const int ke = min(gb.hi[2], kb + zc - 1);
      const int x0 = x_origin + (col % gx) * TX;
      const int y0 = gb.lo[1] + (col / gx) * TY;
      const int cx_vel = x0 - 2 - 1 + A, cy_vel = y0 - 2 + h - 1;
      const int cx_p = x0 - 1 + A, cy_p = y0 + h - 1;
      const int nplanes = ke - kb + 5;  // planes kb-2 .. ke+2
      const int load0 = loads;
      auto issue = [&](int l) {  // plane s = kb-2+l
        const int s = kb - 2 + l, li = load0 + l, slot = li % NS;
        issued = li + 1;
        const bool withP = s >= kb && s <= ke;
        mbar_arrive_expect_tx(&bars[slot], vel_tx + (withP ? (uint32_t)L::P_TILE * 8u : 0u));
        double* base = svel + slot * 3 * VT;
        const int cz = s + h - 1;
        tma_load_3d(base, &tm.vel[m0], &bars[slot], cx_vel, cy_vel, cz);
        tma_load_3d(base + VT, &tm.vel[m1], &bars[slot], cx_vel, cy_vel, cz);
        tma_load_3d(base + 2 * VT, &tm.vel[m2], &bars[slot], cx_vel, cy_vel, cz);
        if (withP) tma_load_3d(sP + slot * L::P_TILE, &tm.P, &bars[slot], cx_p, cy_p, cz);
      };
      if (tid == 0)
        for (int l = 0; l < NS - 2 && l < nplanes; l++) issue(l);
      loads += nplanes;

      // ---- per-thread geometry of this column ------------------------------
      const int ox_hi = (x0 + TX - 1 >= gb.hi[0]) ? gb.hi[0] + 1 : x0 + TX - 1;
      const int ox_lo = max(x0, gb.lo[0]);
      const int oy_hi = (y0 + TY - 1 >= gb.hi[1]) ? gb.hi[1] + 1 : y0 + TY - 1;
      const int oz_hi = (ke >= gb.hi[2]) ? gb.hi[2] + 1 : ke;
      auto inDx = [&](int i) { return i >= D.lo[0] && i <= D.hi[0]; };
      auto inDy = [&](int j) { return j >= D.lo[1] && j <= D.hi[1]; };
      auto ownx = [&](int i) { return i >= ox_lo && i <= ox_hi && i >= 1 && i <= nx + 1; };
      auto owny = [&](int j) { return j >= y0 && j <= oy_hi && j >= 1 && j <= ny + 1; };
      int it_xj[NROUND], it_vrow[NROUND], it_drow[NROUND], it_dx[NROUND];
      unsigned it_bits[NROUND];  // see below
      bool it_valid[NROUND];
#pragma unroll
      for (int rd = 0; rd < NROUND; rd++) {
        const int q = tid + rd * NT;
        it_valid[rd] = q < NITEM;
        const int pp = q % PW, r = q / PW;
        const int xb = x0 - 1 + 2 * pp, j = y0 - 1 + r;
        it_xj[rd] = xb + j;
        it_vrow[rd] = (r + 1) * VW;
        it_drow[rd] = r * DW;
        it_dx[rd] = 2 * pp;
        // bits 0..3: x in D of cells xb-1..xb+2; 4..6: y in D of j-1..j+1;
        // 7, 8: cell xb, xb+1 inside [x0, x0+TX]; 9: j inside [y0, y0+TY];
        // 10, 11: x owned; 12: y owned; 13, 14: cell inside the dp tile
        unsigned b = 0;
        for (int o = -1; o <= 2; o++) b |= (inDx(xb + o) ? 1u : 0u) << (o + 1);
        for (int o = -1; o <= 1; o++) b |= (inDy(j + o) ? 1u : 0u) << (5 + o);
        for (int o = 0; o <= 1; o++) b |= ((xb + o >= x0 && xb + o <= x0 + TX) ? 1u : 0u) << (7 + o);
        b |= ((j >= y0 && j <= y0 + TY) ? 1u : 0u) << 9;
        for (int o = 0; o <= 1; o++) b |= (ownx(xb + o) ? 1u : 0u) << (10 + o);
        b |= (owny(j) ? 1u : 0u) << 12;
        for (int o = 0; o <= 1; o++) b |= ((2 * pp + o <= TX + 2) ? 1u : 0u) << (13 + o);
        it_bits[rd] = b;
      }
      // output pair of phase Y (threads tid < NP): cells (x0+2op, x0+2op+1) in row y0+orow
      const bool ythread = tid < NP;
      const int op = tid % (TX / 2), orow = tid / (TX / 2);
      const int oi = x0 + 2 * op, oj = y0 + orow;
      // bits 0..2: x in D of oi..oi+2; 3, 4: y in D of oj, oj+1; 5, 6: x in out;
      // 7: y in out; 8, 9: x interior; 10: y interior
      unsigned ob = 0;
      for (int o = 0; o <= 2; o++) ob |= (inDx(oi + o) ? 1u : 0u) << o;
      ob |= (inDy(oj) ? 1u : 0u) << 3;
      ob |= (inDy(oj + 1) ? 1u : 0u) << 4;
      for (int o = 0; o <= 1; o++) ob |= ((oi + o >= out.lo[0] && oi + o <= out.hi[0]) ? 1u : 0u) << (5 + o);
      ob |= ((oj >= out.lo[1] && oj <= out.hi[1]) ? 1u : 0u) << 7;
      for (int o = 0; o <= 1; o++) ob |= ((oi + o >= 1 && oi + o <= nx) ? 1u : 0u) << (8 + o);
      ob |= ((oj >= 1 && oj <= ny) ? 1u : 0u) << 10;
      const int o_vofs = (orow + 2) * VW + 2 * op + 2;  // velocity tile offset of cell oi
      const int o_dofs = (orow + 1) * DW + 2 * op + 1;  // dp offset of cell oi
      const int o_pofs = orow * TX + 2 * op;
      const int64_t o_g0 = g.at(oi, oj, 0);
      const int oij = oi + oj;

      // A tile whose neighbourhood lies inside D (x, y), whose outputs lie inside
      // `out` and whose cells are interior (x, y) needs no per-cell masks.
      const bool full = x0 - 3 >= D.lo[0] && x0 + TX + 3 <= D.hi[0] && y0 - 2 >= D.lo[1] &&
                        y0 + TY + 2 <= D.hi[1] && x0 >= out.lo[0] && x0 + TX - 1 <= out.hi[0] &&
                        y0 >= out.lo[1] && y0 + TY - 1 <= out.hi[1] && x0 >= 1 && x0 + TX - 1 <= nx && y0 >= 1 &&
                        y0 + TY - 1 <= ny;
      auto sweep_planes = [&](auto full_tag) {
      constexpr bool FULL = decltype(full_tag)::value;
      for (int l = 0; l < nplanes; l++) {
        const int s = kb - 2 + l;
        const int li = load0 + l;
        const int slot = li % NS;
        if (!mbar_wait_bounded(&bars[slot], (uint32_t)((li / NS) & 1))) {
          ctx->wait_error = 1;
          ok = false;
        }
        if (__syncthreads_or(!ok)) {
          ok = false;
          break;
        }
        const int slm = (li + NS - 1) % NS, slb = (li + NS - 2) % NS;  // planes s-1, s-2
        const double* Us = svel + slot * 3 * VT;
        const double* Vs = Us + VT;
        const double* Ws = Us + 2 * VT;
        const double* Um = svel + slm * 3 * VT;
        const double* Vm = Um + VT;
        const double* Wm = Um + 2 * VT;
        const double* Wb = svel + slb * 3 * VT + 2 * VT;
        double* d_s = sdp + ring3(s) * DP;
        double* d_m = sdp + ring3(s - 1) * DP;
        const double* d_b = sdp + ring3(s - 2) * DP;
        const bool do0 = s >= kb - 1, do1 = s - 1 >= kb;
        const bool z_s = s >= D.lo[2] && s <= D.hi[2];
        const bool z_m = s - 1 >= D.lo[2] && s - 1 <= D.hi[2];
        const bool z_b = s - 2 >= D.lo[2] && s - 2 <= D.hi[2];
        const bool own_s = s >= kb && s <= oz_hi && s >= 1 && s <= nz + 1;
        const bool own_m = s - 1 >= kb && s - 1 <= oz_hi && s - 1 >= 1 && s - 1 <= nz + 1;
        // ---- phase X
#pragma unroll
        for (int rd = 0; rd < NROUND; rd++) {
          if (!it_valid[rd]) continue;
          const unsigned b = it_bits[rd];
          const int o = (it_xj[rd] + s) & 1;  // colour-0 cell at s = colour-1 cell at s-1
          const int dx = it_dx[rd] + o;
          const int sx = it_vrow[rd] + dx + 1;
          const int dofs = it_drow[rd] + dx;
          const bool mxy = FULL || (((b >> (o + 1)) & 1u) && ((b >> 5) & 1u));
          const bool inside = (b >> (13 + o)) & 1u;
          const bool own = ((b >> (10 + o)) & 1u) && ((b >> 12) & 1u);
          double dp0 = 0.0;
          // (FULL: the cell beyond the dp region is computed and not stored)
          const bool m0 = do0 && z_s && (FULL || (inside && mxy));
          if (m0) {
            const double dudx = dxi * (-Us[sx - 1] + Us[sx]);
            const double dvdy = dyi * (-Vs[sx - VW] + Vs[sx]);
            const double dwdz = dzi * (-Wm[sx] + Ws[sx]);
            const double div = dudx + dvdy + dwdz;
            dp0 = -om * div * dl;
            if (own_s && own) racc += div * div;
          }
          if (do0 && inside) d_s[dofs] = dp0;
          // dp1 at (same i, j, plane s-1)
          const bool in1 = ((b >> (7 + o)) & 1u) && ((b >> 9) & 1u);  // inside the dp1 region
          if (do1 && z_m && (FULL || (mxy && in1))) {
            double ul = Um[sx - 1], ur = Um[sx];
            double vl = Vm[sx - VW], vr = Vm[sx];
            double wl = Wb[sx], wr = Wm[sx];
            const double cl = d_m[dofs - 1] * dxi, cr = d_m[dofs + 1] * dxi;
            const double cd = d_m[dofs - DW] * dyi, cu = d_m[dofs + DW] * dyi;
            const double cb = d_b[dofs] * dzi, ct = dp0 * dzi;
            ul = (FULL || ((b >> o) & 1u)) ? ul + cl : ul;
            ur = (FULL || ((b >> (o + 2)) & 1u)) ? ur - cr : ur;
            vl = (FULL || ((b >> 4) & 1u)) ? vl + cd : vl;
            vr = (FULL || ((b >> 6) & 1u)) ? vr - cu : vr;
            wl = z_b ? wl + cb : wl;
            wr = m0 ? wr - ct : wr;
            const double dudx = dxi * (-ul + ur);
            const double dvdy = dyi * (-vl + vr);
            const double dwdz = dzi * (-wl + wr);
            const double div = dudx + dvdy + dwdz;
            if (!FULL || in1) d_m[dofs] = -om * div * dl;
            if (own_m && own) racc += div * div;
          }
        }
        __syncthreads();
        // ---- phase Y: U, V, P at k1 = s-1; W at k2 = s-2
        const int k1 = s - 1, k2 = s - 2;
        const bool lower_first1 = ((oij + k1) & 1) == 0;  // cell oi is colour 0 at k1
        if (ythread && k1 >= kb && k1 <= ke) {
          const double dA = d_m[o_dofs], dB = d_m[o_dofs + 1], dC = d_m[o_dofs + 2];
          const bool mA = z_m && (FULL || (((ob >> 0) & 1u) && ((ob >> 3) & 1u)));
          const bool mB = z_m && (FULL || (((ob >> 1) & 1u) && ((ob >> 3) & 1u)));
          const bool mC = z_m && (FULL || (((ob >> 2) & 1u) && ((ob >> 3) & 1u)));
          const bool yup = z_m && (FULL || ((ob >> 4) & 1u));
          // cell oi (colour c0) and oi+1 (colour 1-c0)
          const double u0 = face_update(Um[o_vofs], lower_first1, mA, dA, mB, dB, dxi);
          const double u1 = face_update(Um[o_vofs + 1], !lower_first1, mB, dB, mC, dC, dxi);
          const double v0 = face_update(Vm[o_vofs], lower_first1, mA, dA, yup && (FULL || ((ob >> 0) & 1u)),
                                        d_m[o_dofs + DW], dyi);
          const double v1 = face_update(Vm[o_vofs + 1], !lower_first1, mB, dB, yup && (FULL || ((ob >> 1) & 1u)),
                                        d_m[o_dofs + 1 + DW], dyi);
          const double p0o = sP[slm * L::P_TILE + o_pofs], p1o = sP[slm * L::P_TILE + o_pofs + 1];
          const double p0 = mA ? p0o + dA * dti : p0o;
          const double p1 = mB ? p1o + dB * dti : p1o;
          const bool oy = (FULL || ((ob >> 7) & 1u)) && k1 >= out.lo[2] && k1 <= out.hi[2];
          const bool oa = oy && (FULL || ((ob >> 5) & 1u)), obb = oy && (FULL || ((ob >> 6) & 1u));
          const int64_t o = o_g0 + (int64_t)k1 * g.pz;
          if (oa && obb) {
            *(double2*)(Uo + o) = make_double2(u0, u1);
            *(double2*)(Vo + o) = make_double2(v0, v1);
          } else {
            if (oa) { Uo[o] = u0; Vo[o] = v0; }
            if (obb) { Uo[o + 1] = u1; Vo[o + 1] = v1; }
          }
          // P in place on the interior only (P halos are refilled before any read)
          const bool pj = k1 >= 1 && k1 <= nz && (FULL || ((ob >> 10) & 1u));
          const bool pa = pj && (FULL || ((ob >> 8) & 1u)), pb = pj && (FULL || ((ob >> 9) & 1u));
          if (pa && pb) {
            *(double2*)(P + o) = make_double2(p0, p1);
          } else {
            if (pa) P[o] = p0;
            if (pb) P[o + 1] = p1;
          }
        }
        if (ythread && k2 >= kb && k2 <= ke) {
          // W face between planes k2 and k1 = k2+1; cell oi at k2 has colour 1-c0(k1)
          const bool mxA = FULL || (((ob >> 0) & 1u) && ((ob >> 3) & 1u));
          const bool mxB = FULL || (((ob >> 1) & 1u) && ((ob >> 3) & 1u));
          const double w0 = face_update(Wb[o_vofs], !lower_first1, z_b && mxA, d_b[o_dofs], z_m && mxA,
                                        d_m[o_dofs], dzi);
          const double w1 = face_update(Wb[o_vofs + 1], lower_first1, z_b && mxB, d_b[o_dofs + 1], z_m && mxB,
                                        d_m[o_dofs + 1], dzi);
          const bool oy = (FULL || ((ob >> 7) & 1u)) && k2 >= out.lo[2] && k2 <= out.hi[2];
          const bool oa = oy && (FULL || ((ob >> 5) & 1u)), obb = oy && (FULL || ((ob >> 6) & 1u));
          const int64_t o = o_g0 + (int64_t)k2 * g.pz;
          if (oa && obb) {
            *(double2*)(Wo + o) = make_double2(w0, w1);
          } else {
            if (oa) Wo[o] = w0;
            if (obb) Wo[o + 1] = w1;
          }
        }
        __syncthreads();
        if (tid == 0 && l + NS - 2 < nplanes) issue(l + NS - 2);
      }
      };
      if (full) {
        sweep_planes(std::true_type{});
      } else {
        sweep_planes(std::false_type{});
      }
    }
    if (!ok) {
      // let the copies already issued land before the CTA's shared memory goes away
      if (tid == 0)
        for (int li = max(0, issued - NS); li < issued; li++) mbar_wait_bounded(&bars[li % NS], (uint32_t)((li / NS) & 1));
      __syncthreads();
    }
  }
  // residual partial of this CTA; the last CTA finalizes the sweep and swaps
  const double bs = block_sum<NT>(racc, red);
  const unsigned int nb = gridDim.x;
  const unsigned int bid = blockIdx.x;
  if (tid == 0) partials[bid] = bs;
  if (last_block(&ctx->ticket, nb, last_flag)) {
    if (skip || ctx->wait_error) {
      if (tid == 0) {
        ctx->ticket = 0;
        if (ctx->wait_error) {  // stop the couple: no more sweeps, and the graph's loop ends
          ctx->cs.done = 1;
          ctx->cs.cont = 0;
        }
      }
      return;
    }
    if (finalize) {
      double v = 0.0;
      for (int q = tid; q < (int)nb; q += NT) v += __ldcg(&partials[q]);
      const double s2 = block_sum<NT>(v, red);
      if (tid == 0) hsmac_check(ctx, cf, s2, group_end);
    }
    if (tid == 0) {
      ctx->ticket = 0;
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

}  // namespace
}  // namespace lcs
