// lcs_hsmac_rw.cuh -- the fused red-black HSMAC sweep, one warp per tile row.
//
// Same computation as k_hsmac_fused (both colour phases of
// the reference's `foraxes(...; coloring=RedBlackFast())` sweep over a box D,
// hsmac.jl:1-35, ping-ponged so that one pass replaces the two in-place
// launches, bit-identical to them), arranged so that almost everything stays
// in registers:
//  - a CTA owns a tile of RW_TX x TY output cells of the x-y plane and streams
//    along z through a chunk of planes; the TY+3 rows (the rows of the tile,
//    one below and two above) go to the warps RW at a time: warp w owns rows
//    y0-1+RW*w .. y0-2+RW*(w+1) (one row per warp for the FP64 13-row tiles,
//    two for the FP32 29-row tiles);
//  - lane l owns the x-pair (x0-2+2l, x0-1+2l), aligned to the pair's size in
//    HBM and in shared memory, so every shared-memory access is a vector of a
//    pair (or one element of it);
//  - in a row the colour-0 cell of every pair is on the same side at a given
//    plane, so the colour logic is a compile-time branch per plane parity;
//  - U, V, W, P of the previous plane and the pair's dp values stay in
//    registers (indexed by plane parity, so nothing is moved between planes);
//    x neighbours come from the adjacent lane (shuffles), y neighbours from
//    shared memory (U, V, W and P planes loaded by TMA into a ring of 3 slots,
//    and a ring of 3 dp planes);
//  - planes away from the ends of a z chunk, and tiles away from the edges of
//    D, run code without membership masks;
//  - one __syncthreads per plane.
//
// Per plane s, in every warp (row j):
//   phase X: dp0 of the colour-0 cell A at plane s, then dp1 of the same
//            (i, j) at plane s-1, where A is colour 1; dp1 needs dp0 at s-1 of
//            the x neighbours (registers of this and the adjacent lane), of
//            the y neighbours (rows j-1, j+1 in shared memory) and dp0 at s
//            (just computed) and s-2 (registers);
//   barrier;
//   phase Y: the faces U, V and P of plane s-1 and the faces W of plane s-2 of
//            the pair, from old values in registers and dp of the pair (this
//            lane), of x+1 (next lane) and of row j+1 (shared memory).
// Waits on the mbarriers are bounded; a wait that runs out sets
// ctx->wait_error and the kernel stops computing (the host reports
// LCS_ETIMEDOUT).
#pragma once

#include <type_traits>

#include "lcs_tma.cuh"

namespace lcs {
namespace {

constexpr int RW_TX = 60;  // output columns of a tile: pairs of lanes 1..30
// TMA ring depth of the 13-row sweep (planes in flight = depth - 1), per
// element size: FP32 planes carry half the bytes, so the FP32 sweep keeps four
// planes in flight to have as many bytes outstanding (1136 against 1227 us a
// sweep at 512^3); a deeper FP64 ring measured slower (1792 against 1714 us)
#ifndef LCS_RW_RING64
#define LCS_RW_RING64 3
#endif
#ifndef LCS_RW_RING32
#define LCS_RW_RING32 5
#endif
template <typename T> constexpr int kRwRing = sizeof(T) == 8 ? LCS_RW_RING64 : LCS_RW_RING32;
constexpr int RW_W = 64;   // columns of every shared-memory row: x0-2 .. x0+61

// Pair vector of the field type (a lane's two cells).
template <typename T> struct Pair2;
template <> struct Pair2<double> { using type = double2; };
template <> struct Pair2<float> { using type = float2; };
template <typename T> using pair_t = typename Pair2<T>::type;
template <typename T> __device__ __forceinline__ pair_t<T> mk2(T a, T b) { return pair_t<T>{a, b}; }

template <typename T, int TY, int NS, int RW = 1>
struct RwLayout {
  static constexpr int VH = TY + 4;  // velocity rows y0-2 .. y0+TY+1
  static constexpr int DH = TY + 3;  // dp rows y0-1 .. y0+TY+1
  static constexpr int NW = (TY + 3) / RW;  // warps: RW consecutive rows each
  static_assert((TY + 3) % RW == 0, "the rows of a tile split evenly over the warps");
  static constexpr int NT = NW * 32;
  // resident CTAs the register budget is sized for (FP32 state fits two
  // CTAs of up to 11 warps without spilling; FP64 state only 8 warps)
  static constexpr int MINB = (NT <= 256 || (sizeof(T) == 4 && NT <= 352)) ? 2 : 1;
  static constexpr int VT = RW_W * VH;  // elements of one field's plane tile
  static constexpr int DP = RW_W * DH;  // elements of one dp plane
  static constexpr int PT = RW_W * TY;  // elements of one P plane tile (rows y0 .. y0+TY-1)
  static constexpr int ND = 3;  // dp planes s-2, s-1, s (a ring of its own)
  static constexpr size_t vel_bytes = (size_t)NS * 3 * VT * sizeof(T);
  static constexpr size_t p_bytes = (size_t)NS * PT * sizeof(T);
  static constexpr size_t dp_bytes = (size_t)ND * DP * sizeof(T);
  static constexpr size_t bar_bytes = 8 * NS;
  static constexpr size_t red_bytes = 8 * 32;
  static constexpr size_t total = vel_bytes + p_bytes + dp_bytes + bar_bytes + red_bytes + 16;
  static_assert(NS >= 3, "TMA ring: the plane being read and at least two in flight");
  static_assert((VT * sizeof(T)) % 128 == 0 && (PT * sizeof(T)) % 128 == 0, "TMA destinations must stay 128-byte aligned");
  static_assert((DP * sizeof(T)) % 16 == 0, "dp rows must stay 16-byte aligned");
  static_assert(NW <= 32, "one reduction slot per warp");
};

template <typename T> __device__ __forceinline__ pair_t<T> lds2(const T* p) {
  return *reinterpret_cast<const pair_t<T>*>(p);
}
template <typename T> __device__ __forceinline__ void st2(T* p, T a, T b) {
  *reinterpret_cast<pair_t<T>*>(p) = mk2<T>(a, b);
}
template <typename T> __device__ __forceinline__ T shfl_up1(T v) { return __shfl_up_sync(0xffffffffu, v, 1); }
template <typename T> __device__ __forceinline__ T shfl_down1(T v) { return __shfl_down_sync(0xffffffffu, v, 1); }

// The velocity update of one face for either field type: the contributions
// of the two cells sharing the face in the order of the in-place sweep.
template <typename T>
__device__ __forceinline__ T face_update_t(T val, bool lower_first, bool ma, T da, bool mb, T db, T dci) {
  const T ta = da * dci, tb = db * dci;
  if (lower_first) {
    val = ma ? val + ta : val;
    val = mb ? val - tb : val;
  } else {
    val = mb ? val - tb : val;
    val = ma ? val + ta : val;
  }
  return val;
}

// Work items of a sweep: (tile column, z range), chunk major.  The first
// `full` items are whole chunks of `zc` planes; every later chunk is split into
// q sub-ranges, so that the last wave of CTAs is as full as the first.
struct RwSched {
  int ncols, zc, full, q, nitems;
};

// The item's column and planes kb..ke (an empty range when kb > ke).
__device__ __forceinline__ void rw_item(const RwSched& sc, int lo, int hi, int item, int* col, int* kb, int* ke) {
  int i = item, sub = 0;
  if (item >= sc.full) {
    i = sc.full + (item - sc.full) / sc.q;
    sub = (item - sc.full) % sc.q;
  }
  *col = i % sc.ncols;
  const int kb0 = lo + (i / sc.ncols) * sc.zc, ke0 = min(hi, kb0 + sc.zc - 1);
  if (item < sc.full) {
    *kb = kb0;
    *ke = ke0;
    return;
  }
  const int len = (ke0 - kb0 + sc.q) / sc.q;  // ceil((ke0 - kb0 + 1) / q)
  *kb = kb0 + sub * len;
  *ke = min(ke0, *kb + len - 1);
}

// Per-lane (x) and per-warp (y) membership bits of one tile.
struct RwBits {
  // x, this lane's pair (L = x0-2+2l, R = L+1)
  bool dLm, dL, dR, dRp;  // L-1, L, R, R+1 inside D
  bool ownL, ownR;        // residual ownership
  bool d1L, d1R;          // inside the dp1 region [x0, x0+RW_TX]
  bool outL, outR;        // output column of this tile and inside `out`
  bool intL, intR;        // interior column (P is stored on the interior only)
};
// y membership bits of one row j of a warp.
struct RwRowBits {
  bool dym, dy, dyp;      // j-1, j, j+1 inside D
  bool owny, d1y, outy, inty;
  bool yrow;              // the row has outputs (rows y0 .. y0+TY-1)
};


// x0 (a tile's first output column) puts x0-2 on a 16-byte boundary (x0 odd
// in FP64, x0 = 3 mod 4 in FP32): the TMA boxes start there and every pair
// (x0-2+2l, x0-1+2l) is aligned to its own size.  Work items are
// (z chunk, tile column), chunk major.
// The sweep of one handle as block `bid` of `nb` (k_hsmac_rw: the launch's
// own grid; k_hsmac_rw_group: one handle per blockIdx.y).
template <typename T, int TY, int NS, int RW>
__device__ __forceinline__ void hsmac_rw_body(Ctx* __restrict__ ctx, const Grid& g, int set, const TensorMaps& tm,
                                              T* __restrict__ P, const Box& D, const Box& out, const Box& gb,
                                              int x_origin, int gx, int gy, const RwSched& sc, const HsmacCoef& cf,
                                              double* __restrict__ partials, int finalize, int group_end,
                                              const unsigned int bid, const unsigned int nb) {
  using L = RwLayout<T, TY, NS, RW>;
  using T2 = pair_t<T>;
  constexpr int NT = L::NT, VT = L::VT, DP = L::DP, W = RW_W;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  constexpr int PT = L::PT;
  T* svel = (T*)smem_raw;                               // [NS][3][VH][W]
  T* sP = (T*)(smem_raw + L::vel_bytes);                // [NS][TY][W]
  T* sdp = (T*)(smem_raw + L::vel_bytes + L::p_bytes);  // [ND][DH][W]
  uint64_t* bars = (uint64_t*)(smem_raw + L::vel_bytes + L::p_bytes + L::dp_bytes);
  double* red = (double*)(smem_raw + L::vel_bytes + L::p_bytes + L::dp_bytes + L::bar_bytes);
  int* last_flag = (int*)(red + 32);

  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const bool skip = ctx->cs.done != 0;
  const int nx = g.n[0], ny = g.n[1], nz = g.n[2], h = g.h;
  double racc = 0.0;

  if (!skip) {
    const int m0i = ctx->vphys[set][0], m1i = ctx->vphys[set][1], m2i = ctx->vphys[set][2];
    T* Uo = (T*)ctx->vel[kSetSpare][0];
    T* Vo = (T*)ctx->vel[kSetSpare][1];
    T* Wo = (T*)ctx->vel[kSetSpare][2];
    const T dxi = (T)cf.dxi, dyi = (T)cf.dyi, dzi = (T)cf.dzi, dl = (T)cf.dl, om = (T)cf.omega;
    const T dti = (T)(1.0 / ctx->scal[0]);
    const int A = kAlignElems<T>;
    // bytes of one plane's four copies (16 more under the test hook that
    // makes the plane barriers unreachable)
    const uint32_t plane_tx = (3u * VT + PT) * (uint32_t)sizeof(T) + (ctx->debug_wait == 2 ? 16u : 0u);
    if (tid == 0) {
      for (int q = 0; q < NS; q++) mbar_init(&bars[q], 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    int loads = 0;  // plane loads issued by this CTA: slot = index % NS, parity = (index / NS) & 1
    int issued = 0;  // thread 0: loads issued so far (index of the next one)
    bool ok = true;
    for (int item = (int)bid; item < sc.nitems && ok; item += (int)nb) {
      int col, kb, ke;
      rw_item(sc, gb.lo[2], gb.hi[2], item, &col, &kb, &ke);
      if (kb > ke) continue;  // an empty sub-range (uniform in the CTA)
      const int x0 = x_origin + (col % gx) * RW_TX;
      const int y0 = gb.lo[1] + (col / gx) * TY;
      const int cx = x0 - 2 - 1 + A, cy = y0 - 2 + h - 1;
      const int nplanes = ke - kb + 5;  // planes kb-2 .. ke+2
      const int load0 = loads;
      auto issue = [&](int l) {  // plane s = kb-2+l into slot (load0+l) % NS
        const int li = load0 + l, slot = li % NS;
        issued = li + 1;
        mbar_arrive_expect_tx(&bars[slot], plane_tx);
        T* base = svel + slot * 3 * VT;
        const int cz = kb - 2 + l + h - 1;
        tma_load_3d(base, &tm.vel[m0i], &bars[slot], cx, cy, cz);
        tma_load_3d(base + VT, &tm.vel[m1i], &bars[slot], cx, cy, cz);
        tma_load_3d(base + 2 * VT, &tm.vel[m2i], &bars[slot], cx, cy, cz);
        tma_load_3d(sP + slot * PT, &tm.P, &bars[slot], cx, cy + 2, cz);  // rows y0 .. y0+TY-1
      };
      if (tid == 0)
        for (int l = 0; l < NS && l < nplanes; l++) issue(l);
      loads += nplanes;

      // ---- membership bits of this lane's pair and this warp's row ----------
      const int xL = x0 - 2 + 2 * lane, xR = xL + 1;
      const int j0 = y0 - 1 + w * RW;  // the warp's first row; its rows are j0 .. j0+RW-1
      const int ox_lo = max(x0, gb.lo[0]);
      const int ox_hi = (x0 + RW_TX - 1 >= gb.hi[0]) ? gb.hi[0] + 1 : x0 + RW_TX - 1;
      const int oy_hi = (y0 + TY - 1 >= gb.hi[1]) ? gb.hi[1] + 1 : y0 + TY - 1;
      const int oz_hi = (ke >= gb.hi[2]) ? gb.hi[2] + 1 : ke;
      auto inDx = [&](int i) { return i >= D.lo[0] && i <= D.hi[0]; };
      auto inDy = [&](int y) { return y >= D.lo[1] && y <= D.hi[1]; };
      auto ownx = [&](int i) { return i >= ox_lo && i <= ox_hi && i >= 1 && i <= nx + 1; };
      auto outx = [&](int i) { return i >= x0 && i <= x0 + RW_TX - 1 && i >= out.lo[0] && i <= out.hi[0]; };
      auto intx = [&](int i) { return i >= x0 && i <= x0 + RW_TX - 1 && i >= 1 && i <= nx; };
      RwBits bt;
      bt.dLm = inDx(xL - 1); bt.dL = inDx(xL); bt.dR = inDx(xR); bt.dRp = inDx(xR + 1);
      bt.ownL = ownx(xL); bt.ownR = ownx(xR);
      bt.d1L = xL >= x0 && xL <= x0 + RW_TX; bt.d1R = xR >= x0 && xR <= x0 + RW_TX;
      bt.outL = outx(xL); bt.outR = outx(xR);
      bt.intL = intx(xL); bt.intR = intx(xR);
      RwRowBits rb[RW];
#pragma unroll
      for (int r = 0; r < RW; r++) {
        const int j = j0 + r, rho = w * RW + r;
        rb[r].dym = inDy(j - 1); rb[r].dy = inDy(j); rb[r].dyp = inDy(j + 1);
        rb[r].owny = j >= y0 && j <= oy_hi && j >= 1 && j <= ny + 1;
        rb[r].d1y = j >= y0 && j <= y0 + TY;
        rb[r].yrow = rho >= 1 && rho <= TY;
        rb[r].outy = rb[r].yrow && j >= out.lo[1] && j <= out.hi[1];
        rb[r].inty = rb[r].yrow && j >= 1 && j <= ny;
      }
      // Tiles whose every cell that matters lies inside D (x and y), whose
      // outputs are interior and inside `out`, and which are not the last
      // column (whose residual ownership reaches one cell further) need no x or
      // y masks: their output and owned pairs are those of lanes 1..30.
      const bool full = x0 - 1 >= D.lo[0] && x0 + RW_W - 3 <= D.hi[0] && y0 - 1 >= D.lo[1] &&
                        y0 + TY + 1 <= D.hi[1] && x0 >= max(1, out.lo[0]) &&
                        x0 + RW_TX - 1 <= min(nx, out.hi[0]) && y0 >= max(1, out.lo[1]) &&
                        y0 + TY - 1 <= min(ny, out.hi[1]) && x0 + RW_TX - 1 < gb.hi[0];
      // Planes s_lo .. s_hi need no z masks: every z condition below holds there.
      const int s_lo = max(max(kb + 2, D.lo[2] + 2), max(out.lo[2] + 2, 2));
      const int s_hi = min(min(min(ke + 1, D.hi[2]), min(oz_hi, nz + 1)), out.hi[2] + 1);
      // HBM offsets in 32 bits (a field holds < 2^32 elements: 13 fields of
      // 2^32 FP32 values would need 223 GB); a lane whose offset is negative
      // stores nothing, so its wrapped value is never used
      const uint32_t pz32 = (uint32_t)g.pz;
      uint32_t grow[RW];
      int vofs[RW], dofs[RW], pofs[RW];
#pragma unroll
      for (int r = 0; r < RW; r++) {
        const int rho = w * RW + r;
        grow[r] = (uint32_t)g.at(xL, j0 + r, 0);
        vofs[r] = (rho + 1) * W + 2 * lane;  // row j0+r's pair in a velocity plane tile
        dofs[r] = rho * W + 2 * lane;        // its pair in a dp plane
        pofs[r] = (rho - 1) * W + 2 * lane;  // its pair in a P plane tile (rows y0 ..)
      }
      const bool lane_out = lane >= 1 && lane <= 30;  // output pairs of a full tile

      // Registers carried along z, indexed by plane parity q (q of plane s holds
      // plane s): U, V (row j), V (row j-1), W and P of the plane; D0[q] = dp0 of
      // the colour-0 cell of the pair at that plane; DM[q] = the final dp pair
      // at s-1 computed at plane s; wb = W at s-2.
      // (one set per row of the warp)
      const T2 zero2 = mk2<T>(T(0), T(0));
      T2 Us2[RW][2], Vs2[RW][2], Vb2[RW][2], Ws2[RW][2], Ps2[RW][2], DM[RW][2];
      T D0[RW][2];
      T2 wb[RW];
#pragma unroll
      for (int r = 0; r < RW; r++) {
        for (int q = 0; q < 2; q++) {
          Us2[r][q] = Vs2[r][q] = Vb2[r][q] = Ws2[r][q] = Ps2[r][q] = DM[r][q] = zero2;
          D0[r][q] = T(0);
        }
        wb[r] = zero2;
      }
      int sl = load0 % NS;  // TMA ring slot of plane s (velocity and P)
      uint32_t par = (uint32_t)((load0 / NS) & 1);
      int sd = 0;           // dp ring slot of plane s

      // One plane: FULL (no x/y masks), ZF (no z masks), R (the colour-0 cell
      // of the pair at s is the right one in the warp's first row; it flips
      // from row to row), Q (parity index of plane s).
      auto plane = [&](int l, auto full_tag, auto zf_tag, auto r_tag, auto q_tag) -> bool {
        constexpr bool FULL = decltype(full_tag)::value, ZF = decltype(zf_tag)::value;
        constexpr bool R0 = decltype(r_tag)::value;
        constexpr int Q = decltype(q_tag)::value, QM = 1 - Q;
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
        const bool zk1 = ZF || (k1 >= kb && k1 <= ke);  // U, V, P of plane s-1 are outputs
        const bool zk2 = ZF || (k2 >= kb && k2 <= ke);  // W of plane s-2
        const int sdm = sd == 0 ? L::ND - 1 : sd - 1;  // dp slot of plane s-1
        const T* Vt = svel + sl * 3 * VT;
        T2 dm[RW];
#pragma unroll
        for (int r = 0; r < RW; r++) {
          Us2[r][Q] = lds2(Vt + vofs[r]);
          Vs2[r][Q] = lds2(Vt + VT + vofs[r]);
          // the V row below row j0+r: that of row j0+r-1 of this warp, or shared memory
          Vb2[r][Q] = r > 0 ? Vs2[r > 0 ? r - 1 : 0][Q] : lds2(Vt + VT + vofs[r] - W);
          Ws2[r][Q] = lds2(Vt + 2 * VT + vofs[r]);
          if (rb[r].yrow) Ps2[r][Q] = lds2(sP + sl * PT + pofs[r]);
        }

        // ---- phase X: dp0 at (A, s), dp1 at (A, s-1), row by row
#pragma unroll
        for (int r = 0; r < RW; r++) {
          const bool R = R0 ^ ((r & 1) != 0);
          const RwRowBits& by = rb[r];
          const T2 us = Us2[r][Q], vs = Vs2[r][Q], vbs = Vb2[r][Q], ws = Ws2[r][Q];
          const T2 um = Us2[r][QM], vm = Vs2[r][QM], vbm = Vb2[r][QM], wm = Ws2[r][QM];
          const T d0p = D0[r][QM];   // dp0 at s-1 of the pair's colour-0 cell there
          const T2 dpb = DM[r][QM];  // final dp pair at s-2
          T* dps = sdp + sd * DP + dofs[r];   // this row's pair, plane s
          T* dpm = sdp + sdm * DP + dofs[r];  // this row's pair, plane s-1
          T d0 = T(0), d1 = T(0);
          // U[xL-1] at s and s-1 from the lane below (read on the left side only)
          T upA = T(0), upM = T(0);
          if (!R) {
            upA = shfl_up1(us.y);
            upM = shfl_up1(um.y);
          }
          // dp0 at s-1 of the x neighbour held by the adjacent lane (A+1 for R, A-1 for L)
          const T d0x = R ? shfl_down1(d0p) : shfl_up1(d0p);
          const T uA = R ? us.y : us.x, uAm = R ? us.x : upA;
          const T vA = R ? vs.y : vs.x, vbA = R ? vbs.y : vbs.x;
          const T wA = R ? ws.y : ws.x, wmA = R ? wm.y : wm.x;
          const bool inA = FULL || (by.dy && (R ? bt.dR : bt.dL));
          const bool m0 = do0 && z_s && inA;
          const bool ownA = by.owny && (FULL ? lane_out : (R ? bt.ownR : bt.ownL));
          if (m0) {
            const T dudx = dxi * (-uAm + uA);
            const T dvdy = dyi * (-vbA + vA);
            const T dwdz = dzi * (-wmA + wA);
            const T div = dudx + dvdy + dwdz;
            d0 = -om * div * dl;
            if (own_s && ownA) racc += (double)div * (double)div;
          }
          if (do0) dps[R ? 1 : 0] = d0;
          const bool m1 = do1 && z_m && by.d1y && inA;
          if (m1) {
            const T dyl = dpm[(R ? 1 : 0) - W], dyu = dpm[(R ? 1 : 0) + W];  // dp0 of rows j-1, j+1
            T ul = R ? um.x : upM, ur = R ? um.y : um.x;
            T vl = R ? vbm.y : vbm.x, vr = R ? vm.y : vm.x;
            T wl = R ? wb[r].y : wb[r].x, wr = R ? wm.y : wm.x;
            const T cl = (R ? d0p : d0x) * dxi, cr = (R ? d0x : d0p) * dxi;
            const T cd = dyl * dyi, cu = dyu * dyi;
            const T cb = (R ? dpb.y : dpb.x) * dzi, ct = d0 * dzi;
            ul = (FULL || (R ? bt.dL : bt.dLm)) ? ul + cl : ul;
            ur = (FULL || (R ? bt.dRp : bt.dR)) ? ur - cr : ur;
            vl = (FULL || by.dym) ? vl + cd : vl;
            vr = (FULL || by.dyp) ? vr - cu : vr;
            wl = z_b ? wl + cb : wl;
            wr = m0 ? wr - ct : wr;
            const T dudx = dxi * (-ul + ur);
            const T dvdy = dyi * (-vl + vr);
            const T dwdz = dzi * (-wl + wr);
            const T div = dudx + dvdy + dwdz;
            d1 = -om * div * dl;
            if (own_m && ownA) racc += (double)div * (double)div;
          }
          if (do1 && by.d1y && (FULL || (R ? bt.d1R : bt.d1L))) dpm[R ? 1 : 0] = d1;
          D0[r][Q] = d0;
          dm[r] = R ? mk2<T>(d0p, d1) : mk2<T>(d1, d0p);  // final dp at s-1
          DM[r][Q] = dm[r];
        }
        if (__syncthreads_or(!ok)) return false;
        if (tid == 0 && l + NS < nplanes) issue(l + NS);  // every warp is past its reads of this slot

        // ---- phase Y: U, V, P at s-1 and W at s-2 of the pair, row by row
#pragma unroll
        for (int r = 0; r < RW; r++) {
          const bool R = R0 ^ ((r & 1) != 0);
          const RwRowBits& by = rb[r];
          const T2 um = Us2[r][QM], vm = Vs2[r][QM], wm = Ws2[r][QM];
          const T2 dpb = DM[r][QM];
          const T* dpm = sdp + sdm * DP + dofs[r];
          const T dN = shfl_down1(dm[r].x);  // dp(xR+1, s-1)
          const T2 pv = Ps2[r][QM];          // P at s-1
          const uint32_t o1 = grow[r] + (uint32_t)k1 * pz32;
          if (by.yrow && zk1) {
            const T2 dup = lds2(dpm + W);  // final dp of row j+1 at s-1
            const bool mL = z_m && (FULL || (by.dy && bt.dL)), mR = z_m && (FULL || (by.dy && bt.dR));
            const bool mRp = z_m && (FULL || (by.dy && bt.dRp));
            const bool upL = z_m && (FULL || (by.dyp && bt.dL)), upR = z_m && (FULL || (by.dyp && bt.dR));
            // the left cell is colour 0 at s-1 exactly when R
            const T u0 = face_update_t<T>(um.x, R, mL, dm[r].x, mR, dm[r].y, dxi);
            const T u1 = face_update_t<T>(um.y, !R, mR, dm[r].y, mRp, dN, dxi);
            const T v0 = face_update_t<T>(vm.x, R, mL, dm[r].x, upL, dup.x, dyi);
            const T v1 = face_update_t<T>(vm.y, !R, mR, dm[r].y, upR, dup.y, dyi);
            const T p0 = mL ? pv.x + dm[r].x * dti : pv.x;
            const T p1 = mR ? pv.y + dm[r].y * dti : pv.y;
            if (FULL) {
              if (lane_out) {
                st2<T>(Uo + o1, u0, u1);
                st2<T>(Vo + o1, v0, v1);
                st2<T>(P + o1, p0, p1);  // interior: 1 <= k1 <= nz in ZF
              }
            } else {
              const bool oy = by.outy && k1 >= out.lo[2] && k1 <= out.hi[2];
              const bool oL = oy && bt.outL, oR = oy && bt.outR;
              if (oL && oR) {
                st2<T>(Uo + o1, u0, u1);
                st2<T>(Vo + o1, v0, v1);
              } else {
                if (oL) { Uo[o1] = u0; Vo[o1] = v0; }
                if (oR) { Uo[o1 + 1] = u1; Vo[o1 + 1] = v1; }
              }
              // P in place on the interior only (P halos are refilled before any read)
              const bool pj = by.inty && k1 >= 1 && k1 <= nz;
              const bool pL = pj && bt.intL, pR = pj && bt.intR;
              if (pL && pR) {
                st2<T>(P + o1, p0, p1);
              } else {
                if (pL) P[o1] = p0;
                if (pR) P[o1 + 1] = p1;
              }
            }
          }
          if (by.yrow && zk2) {
            // W faces between planes s-2 and s-1; the left cell is colour 0 at s-2 exactly when !R
            const bool mxL = FULL || (by.dy && bt.dL), mxR = FULL || (by.dy && bt.dR);
            const T w0 = face_update_t<T>(wb[r].x, !R, z_b && mxL, dpb.x, z_m && mxL, dm[r].x, dzi);
            const T w1 = face_update_t<T>(wb[r].y, R, z_b && mxR, dpb.y, z_m && mxR, dm[r].y, dzi);
            const uint32_t o2 = o1 - pz32;
            if (FULL) {
              if (lane_out) st2<T>(Wo + o2, w0, w1);
            } else {
              const bool oy = by.outy && k2 >= out.lo[2] && k2 <= out.hi[2];
              const bool oL = oy && bt.outL, oR = oy && bt.outR;
              if (oL && oR) {
                st2<T>(Wo + o2, w0, w1);
              } else {
                if (oL) Wo[o2] = w0;
                if (oR) Wo[o2 + 1] = w1;
              }
            }
          }
          wb[r] = wm;
        }
        if (++sl == NS) {
          sl = 0;
          par ^= 1u;
        }
        if (++sd == L::ND) sd = 0;
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
          const bool ar = ((j0 + s) & 1) == 0;  // the colour-0 cell at s is the right one (first row)
          bool good;
          if ((l & 1) == 0 && s >= s_lo && s + 1 <= s_hi) {
            // two planes without z masks (the colour-0 side flips between them)
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
      // let the copies already issued land before the CTA's shared memory goes
      // away: a slot is refilled only after its previous phase was consumed, so
      // each slot has at most one phase outstanding, that of its latest load
      if (tid == 0)
        for (int li = max(0, issued - NS); li < issued; li++) mbar_wait_bounded(&bars[li % NS], (uint32_t)((li / NS) & 1));
      __syncthreads();
    }
  }
  // residual partial of this CTA; the last CTA finalizes the sweep and swaps
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

template <typename T, int TY, int NS, int RW = 1>
__global__ void __launch_bounds__(RwLayout<T, TY, NS, RW>::NT, RwLayout<T, TY, NS, RW>::MINB)
    k_hsmac_rw(Ctx* __restrict__ ctx, Grid g, int set, const __grid_constant__ TensorMaps tm,
               T* __restrict__ P, Box D, Box out, Box gb, int x_origin, int gx, int gy, RwSched sc,
               HsmacCoef cf, double* __restrict__ partials, int finalize, int group_end) {
  hsmac_rw_body<T, TY, NS, RW>(ctx, g, set, tm, P, D, out, gb, x_origin, gx, gy, sc, cf, partials, finalize,
                               group_end, blockIdx.x, gridDim.x);
}

// Handles of the same shape and launch shapes swept in one launch (a batch
// group): blockIdx.y picks the handle; each handle's blocks do exactly what
// its own k_hsmac_rw launch does, so its fields and residual are those of the
// handle alone.  The tensor maps travel as kernel parameters (__grid_constant__)
// like the single-handle launch.
constexpr int kGroupMax = 24;
template <typename T>
struct GroupRwArgs {
  TensorMaps tm[kGroupMax];
  Ctx* ctx[kGroupMax];
  T* P[kGroupMax];
  double* partials[kGroupMax];
};
template <typename T, int TY, int NS, int RW = 1>
__global__ void __launch_bounds__(RwLayout<T, TY, NS, RW>::NT, RwLayout<T, TY, NS, RW>::MINB)
    k_hsmac_rw_group(const __grid_constant__ GroupRwArgs<T> ga, Grid g, int set, Box D, Box out, Box gb,
                     int x_origin, int gx, int gy, RwSched sc, HsmacCoef cf, int finalize, int group_end) {
  const int m = blockIdx.y;
  hsmac_rw_body<T, TY, NS, RW>(ga.ctx[m], g, set, ga.tm[m], ga.P[m], D, out, gb, x_origin, gx, gy, sc, cf,
                               ga.partials[m], finalize, group_end, blockIdx.x, gridDim.x);
}
}  // namespace
}  // namespace lcs
