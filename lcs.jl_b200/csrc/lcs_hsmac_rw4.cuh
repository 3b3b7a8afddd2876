// lcs_hsmac_rw4.cuh -- the row-warp fused red-black HSMAC sweep for FP32
// fields with four cells per lane.
//
// The computation is k_hsmac_rw's (both colour phases of the reference's
// `foraxes(...; coloring=RedBlackFast())` sweep over a box D, hsmac.jl:1-35,
// ping-ponged into one pass, bit-identical to the two in-place launches) with
// the lane owning the x-quad (x0-4+4l .. x0-1+4l) instead of a pair:
//  - a tile is RW4_TX = 120 output columns (lanes 1..30) of TY rows; lane 0
//    and lane 31 hold the halo columns x0-4 .. x0-1 and x0+120 .. x0+123;
//  - x0 - 4 sits on a 16-byte boundary, so every quad is one float4 in HBM
//    and in shared memory (TMA boxes 128 columns wide);
//  - at a plane s the colour-0 cells of a quad are its even or its odd
//    elements (a compile-time choice per plane parity), so a lane computes
//    dp0 of two cells at s and dp1 of the same two cells at s-1 in phase X, and
//    the faces of all four cells in phase Y;
//  - everything else (TMA ring of 3 planes on mbarriers, the dp ring, z state
//    in registers indexed by plane parity, one CTA barrier per plane, mask-free
//    code for interior tiles and planes, the work schedule and the residual)
//    is k_hsmac_rw's.
// The FP32 state of a quad takes the registers the FP64 state of a pair takes,
// so a CTA sweeps twice the cells per plane at the same occupancy.
#pragma once

#include "lcs_hsmac_rw.cuh"

namespace lcs {
namespace {

constexpr int RW4_TX = 120;  // output columns of a tile: lanes 1..30
constexpr int RW4_W = 128;   // columns of every shared-memory row: x0-4 .. x0+123

template <int TY, int NS>
struct Rw4Layout {
  static constexpr int VH = TY + 4;  // velocity rows y0-2 .. y0+TY+1
  static constexpr int DH = TY + 3;  // dp rows y0-1 .. y0+TY+1
  static constexpr int NW = TY + 3;  // warps
  static constexpr int NT = NW * 32;
  static constexpr int MINB = NT <= 256 ? 2 : 1;
  static constexpr int VT = RW4_W * VH;
  static constexpr int DP = RW4_W * DH;
  static constexpr int PT = RW4_W * TY;
  static constexpr size_t vel_bytes = (size_t)NS * 3 * VT * sizeof(float);
  static constexpr size_t p_bytes = (size_t)NS * PT * sizeof(float);
  static constexpr size_t dp_bytes = (size_t)NS * DP * sizeof(float);
  static constexpr size_t bar_bytes = 8 * NS;
  static constexpr size_t red_bytes = 8 * 32;
  static constexpr size_t total = vel_bytes + p_bytes + dp_bytes + bar_bytes + red_bytes + 16;
  static_assert(NS == 3, "the dp ring shares the slot index of the TMA ring (3 planes)");
  static_assert((VT * sizeof(float)) % 128 == 0 && (PT * sizeof(float)) % 128 == 0,
                "TMA destinations must stay 128-byte aligned");
  static_assert(NW <= 32, "one reduction slot per warp");
};

struct Quad {
  float e[4];
};
__device__ __forceinline__ Quad ldq(const float* p) {
  const float4 v = *reinterpret_cast<const float4*>(p);
  return Quad{{v.x, v.y, v.z, v.w}};
}
__device__ __forceinline__ void stq(float* p, const float (&v)[4]) {
  *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}

// Per-lane (x) and per-warp (y) membership bits of one tile, for the quad
// elements e = 0..3 (x = x0-4+4l+e); dX covers x-1 .. x+4 (index e+1).
struct Rw4Bits {
  bool dX[6];
  bool own[4], d1x[4], outx[4], intx[4];
  bool dym, dy, dyp;
  bool owny, d1y, outy, inty;
  bool yrow;
};

template <int TY, int NS>
__device__ __forceinline__ void hsmac_rw4_body(Ctx* __restrict__ ctx, const Grid& g, int set, const TensorMaps& tm,
                                               float* __restrict__ P, const Box& D, const Box& out, const Box& gb,
                                               int x_origin, int gx, int gy, const RwSched& sc, const HsmacCoef& cf,
                                               double* __restrict__ partials, int finalize, int group_end,
                                               const unsigned int bid, const unsigned int nb) {
  using L = Rw4Layout<TY, NS>;
  constexpr int NT = L::NT, VT = L::VT, DP = L::DP, PT = L::PT, W = RW4_W;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float* svel = (float*)smem_raw;                               // [NS][3][VH][W]
  float* sP = (float*)(smem_raw + L::vel_bytes);                // [NS][TY][W]
  float* sdp = (float*)(smem_raw + L::vel_bytes + L::p_bytes);  // [NS][DH][W]
  uint64_t* bars = (uint64_t*)(smem_raw + L::vel_bytes + L::p_bytes + L::dp_bytes);
  double* red = (double*)(smem_raw + L::vel_bytes + L::p_bytes + L::dp_bytes + L::bar_bytes);
  int* last_flag = (int*)(red + 32);

  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const bool skip = ctx->cs.done != 0;
  const int nx = g.n[0], ny = g.n[1], nz = g.n[2], h = g.h;
  double racc = 0.0;

  if (!skip) {
    const int m0i = ctx->vphys[set][0], m1i = ctx->vphys[set][1], m2i = ctx->vphys[set][2];
    float* Uo = (float*)ctx->vel[kSetSpare][0];
    float* Vo = (float*)ctx->vel[kSetSpare][1];
    float* Wo = (float*)ctx->vel[kSetSpare][2];
    const float dxi = (float)cf.dxi, dyi = (float)cf.dyi, dzi = (float)cf.dzi, dl = (float)cf.dl,
                om = (float)cf.omega;
    const float dti = (float)(1.0 / ctx->scal[0]);
    const int A = kAlignElems<float>;
    const uint32_t plane_tx = (3u * VT + PT) * (uint32_t)sizeof(float);
    if (tid == 0) {
      for (int q = 0; q < NS; q++) mbar_init(&bars[q], 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    int loads = 0;
    int issued = 0;  // thread 0: loads issued so far (index of the next one)
    bool ok = true;
    for (int item = (int)bid; item < sc.nitems && ok; item += (int)nb) {
      int col, kb, ke;
      rw_item(sc, gb.lo[2], gb.hi[2], item, &col, &kb, &ke);
      if (kb > ke) continue;
      const int x0 = x_origin + (col % gx) * RW4_TX;
      const int y0 = gb.lo[1] + (col / gx) * TY;
      const int cx = x0 - 4 - 1 + A, cy = y0 - 2 + h - 1;
      const int nplanes = ke - kb + 5;
      const int load0 = loads;
      auto issue = [&](int l) {
        const int li = load0 + l, slot = li % NS;
        issued = li + 1;
        mbar_arrive_expect_tx(&bars[slot], plane_tx);
        float* base = svel + slot * 3 * VT;
        const int cz = kb - 2 + l + h - 1;
        tma_load_3d(base, &tm.vel[m0i], &bars[slot], cx, cy, cz);
        tma_load_3d(base + VT, &tm.vel[m1i], &bars[slot], cx, cy, cz);
        tma_load_3d(base + 2 * VT, &tm.vel[m2i], &bars[slot], cx, cy, cz);
        tma_load_3d(sP + slot * PT, &tm.P, &bars[slot], cx, cy + 2, cz);
      };
      if (tid == 0)
        for (int l = 0; l < NS && l < nplanes; l++) issue(l);
      loads += nplanes;

      const int xb = x0 - 4 + 4 * lane, j = y0 - 1 + w;
      const int ox_lo = max(x0, gb.lo[0]);
      const int ox_hi = (x0 + RW4_TX - 1 >= gb.hi[0]) ? gb.hi[0] + 1 : x0 + RW4_TX - 1;
      const int oy_hi = (y0 + TY - 1 >= gb.hi[1]) ? gb.hi[1] + 1 : y0 + TY - 1;
      const int oz_hi = (ke >= gb.hi[2]) ? gb.hi[2] + 1 : ke;
      Rw4Bits bt;
#pragma unroll
      for (int e = -1; e <= 4; e++) bt.dX[e + 1] = xb + e >= D.lo[0] && xb + e <= D.hi[0];
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const int x = xb + e;
        bt.own[e] = x >= ox_lo && x <= ox_hi && x >= 1 && x <= nx + 1;
        bt.d1x[e] = x >= x0 && x <= x0 + RW4_TX;
        bt.outx[e] = x >= x0 && x <= x0 + RW4_TX - 1 && x >= out.lo[0] && x <= out.hi[0];
        bt.intx[e] = x >= x0 && x <= x0 + RW4_TX - 1 && x >= 1 && x <= nx;
      }
      auto inDy = [&](int y) { return y >= D.lo[1] && y <= D.hi[1]; };
      bt.dym = inDy(j - 1); bt.dy = inDy(j); bt.dyp = inDy(j + 1);
      bt.owny = j >= y0 && j <= oy_hi && j >= 1 && j <= ny + 1;
      bt.d1y = j >= y0 && j <= y0 + TY;
      bt.yrow = w >= 1 && w <= TY;
      bt.outy = bt.yrow && j >= out.lo[1] && j <= out.hi[1];
      bt.inty = bt.yrow && j >= 1 && j <= ny;
      // no x or y masks: every cell that feeds an output lies inside D, the
      // outputs are interior and inside `out`, and this is not the last column
      const bool full = x0 - 1 >= D.lo[0] && x0 + RW4_TX + 1 <= D.hi[0] && y0 - 1 >= D.lo[1] &&
                        y0 + TY + 1 <= D.hi[1] && x0 >= max(1, out.lo[0]) &&
                        x0 + RW4_TX - 1 <= min(nx, out.hi[0]) && y0 >= max(1, out.lo[1]) &&
                        y0 + TY - 1 <= min(ny, out.hi[1]) && x0 + RW4_TX - 1 < gb.hi[0];
      const int s_lo = max(max(kb + 2, D.lo[2] + 2), max(out.lo[2] + 2, 2));
      const int s_hi = min(min(min(ke + 1, D.hi[2]), min(oz_hi, nz + 1)), out.hi[2] + 1);
      const int64_t grow = g.at(xb, j, 0);
      const int vofs = (w + 1) * W + 4 * lane;
      const int dofs = w * W + 4 * lane;
      const int pofs = (w - 1) * W + 4 * lane;
      const bool lane_out = lane >= 1 && lane <= 30;

      // z state by plane parity: U, V (row j), V (row j-1), W, P of the plane;
      // D0 = dp0 of the plane's two colour-0 cells (elements p, p+2); DM = the
      // final dp of the quad at s-1 computed at plane s; wb = W at s-2.
      Quad Us[2], Vs[2], Vb[2], Ws[2], Ps[2], DM[2], wb;
      float D0[2][2];
#pragma unroll
      for (int q = 0; q < 2; q++) {
#pragma unroll
        for (int e = 0; e < 4; e++) {
          Us[q].e[e] = Vs[q].e[e] = Vb[q].e[e] = Ws[q].e[e] = Ps[q].e[e] = DM[q].e[e] = 0.f;
        }
        D0[q][0] = D0[q][1] = 0.f;
      }
#pragma unroll
      for (int e = 0; e < 4; e++) wb.e[e] = 0.f;
      int sl = load0 % NS;
      uint32_t par = (uint32_t)((load0 / NS) & 1);

      // One plane: FULL (no x/y masks), ZF (no z masks), R (the colour-0 cells
      // at s are the odd elements), Q (parity index of plane s).
      auto plane = [&](int l, auto full_tag, auto zf_tag, auto r_tag, auto q_tag) -> bool {
        constexpr bool FULL = decltype(full_tag)::value, ZF = decltype(zf_tag)::value;
        constexpr bool R = decltype(r_tag)::value;
        constexpr int Q = decltype(q_tag)::value, QM = 1 - Q;
        constexpr int p = R ? 1 : 0;  // colour-0 elements at s: p, p+2; at s-1: 1-p, 3-p
        const int s = kb - 2 + l;
        if (!mbar_wait_bounded(&bars[sl], par)) {
          ctx->wait_error = 1;
          ok = false;
        }
        const bool do0 = ZF || s >= kb - 1, do1 = ZF || s - 1 >= kb;
        const bool z_s = ZF || (s >= D.lo[2] && s <= D.hi[2]);
        const bool z_m = ZF || (s - 1 >= D.lo[2] && s - 1 <= D.hi[2]);
        const bool z_b = ZF || (s - 2 >= D.lo[2] && s - 2 <= D.hi[2]);
        const bool own_s = ZF || (s >= kb && s <= oz_hi && s >= 1 && s <= nz + 1);
        const bool own_m = ZF || (s - 1 >= kb && s - 1 <= oz_hi && s - 1 >= 1 && s - 1 <= nz + 1);
        const int k1 = s - 1, k2 = s - 2;
        const bool y1 = bt.yrow && (ZF || (k1 >= kb && k1 <= ke));
        const bool y2 = bt.yrow && (ZF || (k2 >= kb && k2 <= ke));
        const int slm = sl == 0 ? NS - 1 : sl - 1;
        const float* Vt = svel + sl * 3 * VT;
        Us[Q] = ldq(Vt + vofs);
        Vs[Q] = ldq(Vt + VT + vofs);
        Vb[Q] = ldq(Vt + VT + vofs - W);
        Ws[Q] = ldq(Vt + 2 * VT + vofs);
        if (bt.yrow) Ps[Q] = ldq(sP + sl * PT + pofs);
        const Quad us = Us[Q], vs = Vs[Q], vbs = Vb[Q], ws = Ws[Q];
        const Quad um = Us[QM], vm = Vs[QM], vbm = Vb[QM], wm = Ws[QM];
        const Quad dpb = DM[QM];  // final dp at s-2
        float* dps = sdp + sl * DP + dofs;
        float* dpm = sdp + slm * DP + dofs;

        // ---- phase X: dp0 at (e, s) and dp1 at (e, s-1) for e = p, p+2
        float d0[2] = {0.f, 0.f}, d1[2] = {0.f, 0.f};
        {
          // U of x-1 for element 0, at s and s-1 (the lane below), when p = 0
          float upA = 0.f, upM = 0.f;
          if constexpr (!R) {
            upA = shfl_up1(us.e[3]);
            upM = shfl_up1(um.e[3]);
          }
          // dp0 at s-1 of the neighbours e-1 and e+1 (colour 0 at s-1):
          // D0[QM][0] is element 1-p, D0[QM][1] is element 3-p
          const float n_lo = R ? shfl_down1(D0[QM][0]) : shfl_up1(D0[QM][1]);  // across the quad edge
#pragma unroll
          for (int c = 0; c < 2; c++) {
            const int e = p + 2 * c;
            // neighbour e-1 is D0[QM][(e-2+p)/2], e+1 is D0[QM][(e+p)/2] inside the quad
            const int il = (e - 2 + p) / 2 < 0 ? 0 : (e - 2 + p) / 2;
            const int ir = (e + p) / 2 > 1 ? 1 : (e + p) / 2;
            const float dleft = (e == 0) ? n_lo : D0[QM][il];
            const float dright = (e == 3) ? n_lo : D0[QM][ir];
            const float uA = us.e[e], uAm = (e == 0) ? upA : us.e[e == 0 ? 0 : e - 1];
            const float vA = vs.e[e], vbA = vbs.e[e];
            const float wA = ws.e[e], wmA = wm.e[e];
            const bool inA = FULL || (bt.dy && bt.dX[e + 1]);
            const bool m0 = do0 && z_s && inA;
            const bool ownA = bt.owny && (FULL ? lane_out : bt.own[e]);
            if (m0) {
              const float dudx = dxi * (-uAm + uA);
              const float dvdy = dyi * (-vbA + vA);
              const float dwdz = dzi * (-wmA + wA);
              const float div = dudx + dvdy + dwdz;
              d0[c] = -om * div * dl;
              if (own_s && ownA) racc += (double)div * (double)div;
            }
            if (do0) dps[e] = d0[c];
            const bool m1 = do1 && z_m && bt.d1y && inA;
            if (m1) {
              const float dyl = dpm[e - W], dyu = dpm[e + W];  // dp0 of rows j-1, j+1 at s-1
              float ul = (e == 0) ? upM : um.e[e == 0 ? 0 : e - 1], ur = um.e[e];
              float vl = vbm.e[e], vr = vm.e[e];
              float wl = wb.e[e], wr = wm.e[e];
              const float cl = dleft * dxi, cr = dright * dxi;
              const float cd = dyl * dyi, cu = dyu * dyi;
              const float cb = dpb.e[e] * dzi, ct = d0[c] * dzi;
              ul = (FULL || bt.dX[e]) ? ul + cl : ul;
              ur = (FULL || bt.dX[e + 2]) ? ur - cr : ur;
              vl = (FULL || bt.dym) ? vl + cd : vl;
              vr = (FULL || bt.dyp) ? vr - cu : vr;
              wl = z_b ? wl + cb : wl;
              wr = m0 ? wr - ct : wr;
              const float dudx = dxi * (-ul + ur);
              const float dvdy = dyi * (-vl + vr);
              const float dwdz = dzi * (-wl + wr);
              const float div = dudx + dvdy + dwdz;
              d1[c] = -om * div * dl;
              if (own_m && ownA) racc += (double)div * (double)div;
            }
            if (do1 && bt.d1y && (FULL || bt.d1x[e])) dpm[e] = d1[c];
          }
        }
        Quad dm;  // final dp at s-1: dp0 there on elements 1-p, 3-p; dp1 on p, p+2
        dm.e[1 - p] = D0[QM][0];
        dm.e[3 - p] = D0[QM][1];
        dm.e[p] = d1[0];
        dm.e[p + 2] = d1[1];
        D0[Q][0] = d0[0];
        D0[Q][1] = d0[1];
        DM[Q] = dm;
        if (__syncthreads_or(!ok)) return false;
        if (tid == 0 && l + NS < nplanes) issue(l + NS);

        // ---- phase Y: U, V, P at s-1 and W at s-2 of the quad
        const float dN = shfl_down1(dm.e[0]);  // dp(x+4, s-1)
        const Quad pv = Ps[QM];
        const int64_t o1 = grow + (int64_t)k1 * g.pz;
        if (y1) {
          const Quad dup = ldq(dpm + W);  // final dp of row j+1 at s-1
          bool mx[5], up[4];
#pragma unroll
          for (int e = 0; e < 5; e++) mx[e] = z_m && (FULL || (bt.dy && bt.dX[e + 1]));
#pragma unroll
          for (int e = 0; e < 4; e++) up[e] = z_m && (FULL || (bt.dyp && bt.dX[e + 1]));
          float u[4], v[4], pp[4];
#pragma unroll
          for (int e = 0; e < 4; e++) {
            const bool lower_first = (e & 1) == 1 - p;  // the cell is colour 0 at s-1
            const float dnext = e == 3 ? dN : dm.e[e == 3 ? 3 : e + 1];
            u[e] = face_update_t<float>(um.e[e], lower_first, mx[e], dm.e[e], mx[e + 1], dnext, dxi);
            v[e] = face_update_t<float>(vm.e[e], lower_first, mx[e], dm.e[e], up[e], dup.e[e], dyi);
            pp[e] = mx[e] ? pv.e[e] + dm.e[e] * dti : pv.e[e];
          }
          if (FULL) {
            if (lane_out) {
              stq(Uo + o1, u);
              stq(Vo + o1, v);
              stq(P + o1, pp);
            }
          } else {
            const bool oy = bt.outy && k1 >= out.lo[2] && k1 <= out.hi[2];
            const bool pj = bt.inty && k1 >= 1 && k1 <= nz;
            bool oall = oy, pall = pj;
#pragma unroll
            for (int e = 0; e < 4; e++) {
              oall = oall && bt.outx[e];
              pall = pall && bt.intx[e];
            }
            if (oall) {
              stq(Uo + o1, u);
              stq(Vo + o1, v);
            } else {
#pragma unroll
              for (int e = 0; e < 4; e++)
                if (oy && bt.outx[e]) {
                  Uo[o1 + e] = u[e];
                  Vo[o1 + e] = v[e];
                }
            }
            if (pall) {
              stq(P + o1, pp);
            } else {
#pragma unroll
              for (int e = 0; e < 4; e++)
                if (pj && bt.intx[e]) P[o1 + e] = pp[e];
            }
          }
        }
        if (y2) {
          float ww[4];
#pragma unroll
          for (int e = 0; e < 4; e++) {
            const bool mxe = FULL || (bt.dy && bt.dX[e + 1]);
            const bool lower_first = (e & 1) == p;  // the cell is colour 0 at s-2
            ww[e] = face_update_t<float>(wb.e[e], lower_first, z_b && mxe, dpb.e[e], z_m && mxe, dm.e[e], dzi);
          }
          const int64_t o2 = o1 - g.pz;
          if (FULL) {
            if (lane_out) stq(Wo + o2, ww);
          } else {
            const bool oy = bt.outy && k2 >= out.lo[2] && k2 <= out.hi[2];
            bool oall = oy;
#pragma unroll
            for (int e = 0; e < 4; e++) oall = oall && bt.outx[e];
            if (oall) {
              stq(Wo + o2, ww);
            } else {
#pragma unroll
              for (int e = 0; e < 4; e++)
                if (oy && bt.outx[e]) Wo[o2 + e] = ww[e];
            }
          }
        }
        wb = wm;
        if (++sl == NS) {
          sl = 0;
          par ^= 1u;
        }
        return true;
      };

      using T_ = std::true_type;
      using F_ = std::false_type;
      using Q0 = std::integral_constant<int, 0>;
      using Q1 = std::integral_constant<int, 1>;
      auto run = [&](auto full_tag) {
        int l = 0;
        while (l < nplanes) {
          const int s = kb - 2 + l;
          // xb has the parity of x0 - 4 + 4l, i.e. of x0 (odd): the colour-0
          // cells at s are the odd elements when (xb + 1 + j + s) is even
          const bool ar = ((j + s) & 1) == 0;
          bool good;
          if ((l & 1) == 0 && s >= s_lo && s + 1 <= s_hi) {
            if (ar) {
              good = plane(l, full_tag, T_{}, T_{}, Q0{}) && plane(l + 1, full_tag, T_{}, F_{}, Q1{});
            } else {
              good = plane(l, full_tag, T_{}, F_{}, Q0{}) && plane(l + 1, full_tag, T_{}, T_{}, Q1{});
            }
            l += 2;
          } else {
            if (l & 1) {
              good = ar ? plane(l, F_{}, F_{}, T_{}, Q1{}) : plane(l, F_{}, F_{}, F_{}, Q1{});
            } else {
              good = ar ? plane(l, F_{}, F_{}, T_{}, Q0{}) : plane(l, F_{}, F_{}, F_{}, Q0{});
            }
            l += 1;
          }
          if (!good) {
            ok = false;
            break;
          }
        }
      };
      if (full) {
        run(T_{});
      } else {
        run(F_{});
      }
    }
    if (!ok) {
      if (tid == 0)
        for (int li = max(0, issued - NS); li < issued; li++) mbar_wait_bounded(&bars[li % NS], (uint32_t)((li / NS) & 1));
      __syncthreads();
    }
  }
  const double bs = block_sum<NT>(racc, red);
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

template <int TY, int NS>
__global__ void __launch_bounds__(Rw4Layout<TY, NS>::NT, Rw4Layout<TY, NS>::MINB)
    k_hsmac_rw4(Ctx* __restrict__ ctx, Grid g, int set, const __grid_constant__ TensorMaps tm, float* __restrict__ P,
                Box D, Box out, Box gb, int x_origin, int gx, int gy, RwSched sc, HsmacCoef cf,
                double* __restrict__ partials, int finalize, int group_end) {
  hsmac_rw4_body<TY, NS>(ctx, g, set, tm, P, D, out, gb, x_origin, gx, gy, sc, cf, partials, finalize, group_end,
                         blockIdx.x, gridDim.x);
}

template <int TY, int NS>
__global__ void __launch_bounds__(Rw4Layout<TY, NS>::NT, Rw4Layout<TY, NS>::MINB)
    k_hsmac_rw4_group(const __grid_constant__ GroupRwArgs<float> ga, Grid g, int set, Box D, Box out, Box gb,
                      int x_origin, int gx, int gy, RwSched sc, HsmacCoef cf, int finalize, int group_end) {
  const int m = blockIdx.y;
  hsmac_rw4_body<TY, NS>(ga.ctx[m], g, set, ga.tm[m], ga.P[m], D, out, gb, x_origin, gx, gy, sc, cf, ga.partials[m],
                         finalize, group_end, blockIdx.x, gridDim.x);
}

}  // namespace
}  // namespace lcs
