// hllc_step.cu -- the well-balanced HLLC finite-volume step (SSP-RK2, Heun).
//
// Each Heun stage is one launch; the reference launches ~11 kernels per stage
// (solver/core/hllc.py:1152-1269 _eval_L) plus the RK, friction and source
// kernels (:1272-1373):
//   _primitives (:262) -> _flux_x/_flux_y (:285/:357, _hllc :191, MUSCL-minmod :158,
//   _dryfactor :174, Audusse hydrostatic reconstruction) -> _apply_boundaries
//   (:993; walls :442-521, fixed_stage ghosts :537-628) -> _mass_beta (:700) ->
//   _limit_fx/_limit_fy (:739/:758) -> _bank_* (:638-677) -> _accumulate (:776) ->
//   _rk_stage1 (:850)                      [stage 1]
//   _rk_stage2 (:881) -> _friction (:912) -> rain / rain field / infiltration
//   (:1350-1373) -> _reduce_wavespeed (:948) for the next dt   [stage 2]
//
// Tiling. A CTA owns a TX x TY tile of cells. The limited mass flux of a tile face
// needs the beta of both neighbouring cells, and a beta needs the four faces of
// its cell, each of which reads a 4-cell MUSCL stencil: a halo of 3 cells of
// (h, u, v, z) is staged in shared memory with edge-clamped indices (exactly the
// reference's _cget transmissive ghosts). Mass fluxes are computed for the tile's
// faces plus a 1-cell ring (for beta), the momentum components only for the tile's
// own faces. Stage 1 writes U1 = (h1, hu1, hv1) to workspace buffers; stage 2
// reads U1 with the halo and U^n on the tile and writes U^{n+1} to the other
// buffer of the caller's double-buffered (h, hu, hv).
#include <cuda.h>  // CUtensorMap and its encoder's signature (reached through the runtime)

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cstring>
#include <mutex>
#include <type_traits>
#include <unordered_map>

#include "rb_common.cuh"
#include "rb_kernels.h"

namespace rb {
RB_ARITH_BEGIN

// hllc.py:158-165 _minmod
#if defined(RB_FAST_MATH)
// Fast arithmetic: minmod is the median of a, b and 0 (four min / max operations, no
// compares). It differs from the reference's form only where a * b underflows to 0
// for two same-signed slopes below 1e-19, and in the sign of a zero.
__device__ __forceinline__ float minmod(float a, float b) { return fmaxf(fminf(a, b), fminf(fmaxf(a, b), 0.0f)); }
#else
__device__ __forceinline__ float minmod(float a, float b) {
  if (a * b <= 0.0f) return 0.0f;
  if (fabsf(a) < fabsf(b)) return a;
  return b;
}
#endif

// hllc.py:174-188 _dryfactor
__device__ __forceinline__ float dryfactor(float h0, float hm, float hp) {
  return (h0 <= kHDry || hm <= kHDry || hp <= kHDry) ? 0.0f : 1.0f;
}

// hllc.py:191-256 _hllc: (mass, normal momentum, transverse momentum) flux.
__device__ __forceinline__ void hllc_flux(float hl, float ul, float vtl, float hr, float ur, float vtr, float& f0,
                                          float& f1, float& f2) {
  const float g = kG;
  const float cl = sqrtf(g * rmax(hl, 0.0f));
  const float cr = sqrtf(g * rmax(hr, 0.0f));
  const bool dry_l = hl <= kHDry, dry_r = hr <= kHDry;
  if (dry_l && dry_r) {
    f0 = 0.0f;
    f1 = 0.0f;
    f2 = 0.0f;
    return;
  }
  float sl, sr;
  if (dry_l) {
    sl = ur - 2.0f * cr;
    sr = ur + cr;
  } else if (dry_r) {
    sl = ul - cl;
    sr = ul + 2.0f * cl;
  } else {
    const float hs = 0.5f * (cl + cr) + 0.25f * (ul - ur);
#if defined(RB_FAST_MATH)
    const float c_star = fabsf(hs);  // sqrt(g * max(hs * hs / g, 0)) = |hs|
#else
    const float h_star = rmax(div_g(hs * hs), 0.0f);  // hs * hs / g
    const float c_star = sqrtf(g * h_star);
#endif
    const float u_star = 0.5f * (ul + ur) + cl - cr;
    sl = rmin(ul - cl, u_star - c_star);
    sr = rmax(ur + cr, u_star + c_star);
  }
  const float fh_l = hl * ul;
  const float fmn_l = hl * ul * ul + 0.5f * g * hl * hl;
  const float fh_r = hr * ur;
  const float fmn_r = hr * ur * ur + 0.5f * g * hr * hr;
  float fh, fmn;
#if defined(RB_FAST_MATH)
  {
    // Fast arithmetic: the three cases in one formula. With the wave speeds clamped
    // to sl <= 0 <= sr, the HLL flux is the left flux when sl >= 0 and the right one
    // when sr <= 0 (to rounding); sl < sr whenever one side is wet.
    const float a = fminf(sl, 0.0f), b = fmaxf(sr, 0.0f);
    const float inv = 1.0f / fmaxf(b - a, 1.0e-30f);
    fh = (b * fh_l - a * fh_r + a * b * (hr - hl)) * inv;
    fmn = (b * fmn_l - a * fmn_r + a * b * (hr * ur - hl * ul)) * inv;
  }
#else
  if (sl >= 0.0f) {
    fh = fh_l;
    fmn = fmn_l;
  } else if (sr <= 0.0f) {
    fh = fh_r;
    fmn = fmn_r;
  } else {
    const float inv = 1.0f / (sr - sl);
    fh = (sr * fh_l - sl * fh_r + sl * sr * (hr - hl)) * inv;
    fmn = (sr * fmn_l - sl * fmn_r + sl * sr * (hr * ur - hl * ul)) * inv;
  }
#endif
  // The contact speed s_star is read only through s_star >= 0 (hllc.py:231-238), so
  // its sign is decided without the division (quotient_nonneg).
  const float den_s = hr * (ur - sr) - hl * (ul - sl);
#if defined(RB_FAST_MATH)
  // fast arithmetic: the sign of the quotient from the sign of the product
  const bool star_nonneg =
      fabsf(den_s) > 1.0e-12f ? (sl * hr * (ur - sr) - sr * hl * (ul - sl)) * den_s >= 0.0f : ul + ur >= 0.0f;
#else
  const bool star_nonneg = fabsf(den_s) > 1.0e-12f
                               ? quotient_nonneg(sl * hr * (ur - sr) - sr * hl * (ul - sl), den_s)
                               : 0.5f * (ul + ur) >= 0.0f;
#endif
  const float vt = star_nonneg ? vtl : vtr;
  f0 = fh;
  f1 = fmn;
  f2 = fh * vt;
}

// hllc.py:262-282 _primitives: u = hu / h and v = hv / h on a wet cell, 0 on a dry
// one. Still water (hu = hv = 0) is common, and its quotients are the zero momenta
// themselves, so such cells branch around both divisions (a zero dividend would take
// the division's slow path); a cell with one zero momentum divides 1 in its place.
#if defined(RB_FAST_MATH)
// Fast arithmetic: one approximate reciprocal per wet cell.
__device__ __forceinline__ void primitives(float h, float hu, float hv, float& u, float& v) {
  const bool wet = h > kHDry;
  const float r = 1.0f / (wet ? h : 1.0f);
  u = wet ? hu * r : 0.0f;
  v = wet ? hv * r : 0.0f;
}
#else
__device__ __forceinline__ void primitives(float h, float hu, float hv, float& u, float& v) {
  const bool wet = h > kHDry;
  u = wet ? hu : 0.0f;
  v = wet ? hv : 0.0f;
  if (wet && !(hu == 0.0f && hv == 0.0f)) {
    const float qu = div_in_branch(opaque(hu == 0.0f ? 1.0f : hu), h);
    const float qv = div_in_branch(opaque(hv == 0.0f ? 1.0f : hv), h);
    if (hu != 0.0f) u = qu;
    if (hv != 0.0f) v = qv;
  }
}
#endif

// A cell of the stencil, in the face's frame: depth, normal and transverse
// velocity, bed.
struct Cell {
  float h, un, ut, z;
};

// A staged cell (h, u, v, z) in the frame of an x-face (normal u) or a y-face
// (normal v).
__device__ __forceinline__ Cell cell_x(const float4& q) { return Cell{q.x, q.y, q.z, q.w}; }
__device__ __forceinline__ Cell cell_y(const float4& q) { return Cell{q.x, q.z, q.y, q.w}; }

// MUSCL-minmod reconstruction of one cell to its two faces along the normal
// (hllc.py:325-342): the east ("E", +1/2) and west ("W", -1/2) values of the water
// surface, bed, normal and transverse velocity, first order at a dry-adjacent cell;
// and sz = dryfactor * minmod of the bed, the slope of the cell's centred bed
// source (hllc.py:805-813, the same operands).
struct Rec {
  float eE, zE, nE, tE, eW, zW, nW, tW, sz;
};

__device__ __forceinline__ Rec recon(const Cell& m, const Cell& c, const Cell& p) {
  const float em = m.h + m.z, ec = c.h + c.z, ep = p.h + p.z;
  const float dry = dryfactor(c.h, m.h, p.h);
  const float hw = 0.5f * dry;
  const float me = minmod(ec - em, ep - ec);
  const float mz = minmod(c.z - m.z, p.z - c.z);
  const float mn = minmod(c.un - m.un, p.un - c.un);
  const float mt = minmod(c.ut - m.ut, p.ut - c.ut);
  Rec r;
  r.eE = ec + hw * me;
  r.eW = ec - hw * me;
  r.zE = c.z + hw * mz;
  r.zW = c.z - hw * mz;
  r.nE = c.un + hw * mn;
  r.nW = c.un - hw * mn;
  r.tE = c.ut + hw * mt;
  r.tW = c.ut - hw * mt;
  r.sz = dry * mz;
  return r;
}

// Any face of the face loop, between a left cell's east values and a right cell's
// west values. An interior face (kind open: an inner face, or an open edge with its
// transmissive clamped stencil) is the Audusse hydrostatic reconstruction and HLLC
// (hllc.py:344-354) with the left and right bed-slope corrections of the normal
// momentum flux. A closed or fixed_stage edge face is a ghost-state Riemann problem
// on the edge cell e (hllc.py:439-628): a reflective wall mirrors e's normal
// velocity (:442-521), a prescribed surface puts the ghost depth max(stage - z_e, 0)
// on the outside (:537-628), and only the inward normal-momentum slot is read.
// `low` is the edge at index 0 (west / north). Both kinds feed one HLLC solve, so
// the solver is inlined once per loop rather than once per edge case; the operands
// and every rounding are those of separate calls. h_l and h_r, the left cell's
// reconstructed depth at its east face and the right cell's at its west face, are
// also the depths of those cells' centred bed source (hllc.py:805-813).
// The face's operands: the left cell's east values (eta, z, normal and transverse
// velocity) and the right cell's west values.
struct FaceSides {
  float eL, zL, nL, tL, eR, zR, nR, tR;
};

__device__ __forceinline__ FaceSides sides(const Rec& L, const Rec& R) {
  return FaceSides{L.eE, L.zE, L.nE, L.tE, R.eW, R.zW, R.nW, R.tW};
}

__device__ __forceinline__ void any_face_flux(const FaceSides& F, int kind, bool low, const Cell& e, float stage,
                                              float& fh, float& fl, float& fr, float& ft, float& h_l_out,
                                              float& h_r_out) {
  const float g = kG;
  const float h_l = rmax(F.eL - F.zL, 0.0f);
  const float h_r = rmax(F.eR - F.zR, 0.0f);
  const float z_star = rmax(F.zL, F.zR);
  const float hl_star = rmax(F.eL - z_star, 0.0f);
  const float hr_star = rmax(F.eR - z_star, 0.0f);
  h_l_out = h_l;
  h_r_out = h_r;
  float hl = hl_star, ul = F.nL, vl = F.tL, hr = hr_star, ur = F.nR, vr = F.tR;
  const bool edge = kind != RB_BC_OPEN;
  if (edge) {
    const bool closed = kind == RB_BC_CLOSED;
    const float h_g = rmax(stage - e.z, 0.0f);
    hl = (!closed && low) ? h_g : e.h;
    hr = (!closed && !low) ? h_g : e.h;
    ul = (closed && low) ? -e.un : e.un;
    ur = (closed && !low) ? -e.un : e.un;
    vl = e.ut;
    vr = e.ut;
  }
  float f0, f1, f2;
  hllc_flux(hl, ul, vl, hr, ur, vr, f0, f1, f2);
  fh = f0;
  ft = f2;
  if (!edge) {
    fl = f1 + 0.5f * g * (h_l * h_l - hl_star * hl_star);
    fr = f1 + 0.5f * g * (h_r * h_r - hr_star * hr_star);
  } else {
    fl = low ? 0.0f : f1;
    fr = low ? f1 : 0.0f;
  }
}

__device__ __forceinline__ void any_face_flux(const Rec& L, const Rec& R, int kind, bool low, const Cell& e,
                                              float stage, float& fh, float& fl, float& fr, float& ft,
                                              float& h_l_out, float& h_r_out) {
  any_face_flux(sides(L, R), kind, low, e, stage, fh, fl, fr, ft, h_l_out, h_r_out);
}

template <int TX, int TY>
struct HllcSmem {
  static constexpr int H = 3;                     // halo
  static constexpr int RW = TX + 2 * H, RH = TY + 2 * H;
  static constexpr int XW = TX + 3, XH = TY + 2;  // x-face mass flux: cols x0-1..x0+TX+1, rows y0-1..y0+TY
  static constexpr int YW = TX + 2, YH = TY + 3;  // y-face mass flux: cols x0-1..x0+TX,   rows y0-1..y0+TY+1
  static constexpr int BW = TX + 2, BH = TY + 2;  // beta on the tile + ring
  // the staged cells (h, u, v, z) as one 16-byte word each: a face reads its four
  // stencil cells with four vector loads
  float4 c[RH][RW];
  float fxh[XH][XW], fyh[YH][YW];
  float fxl[TY][TX + 1], fxr[TY][TX + 1], fxt[TY][TX + 1];  // tile x-faces
  float fyl[TY + 1][TX], fyr[TY + 1][TX], fyt[TY + 1][TX];  // tile y-faces
  float beta[BH][BW];
  // per tile cell, from the face phase: the reconstructed depths at the cell's east
  // (hp) and west (hm) faces and the bed slope sz, along x and along y
  float hpx[TY][TX], hmx[TY][TX], szx[TY][TX], hpy[TY][TX], hmy[TY][TX], szy[TY][TX];
  double red[32];  // one slot per warp of a block of up to 1024 threads
  float redf[32];
};

// LP = 2 stages interior tiles with tensor-memory-accelerator copies: one 2-D box per
// field (h, hu, hv, z) of TY + 6 rows by TX + 8 columns starting at column x0 - 4 (a
// multiple of 4, so the copy starts on a 16-byte boundary) and row y0 - 3, each into
// its own 128-byte aligned landing area, completed on one shared-memory barrier.
template <int TX, int TY>
struct HllcSmemTma : HllcSmem<TX, TY> {
  static constexpr int LW = TX + 8, LH = TY + 6;
  static constexpr int LAND = (LW * LH + 31) / 32 * 32;  // floats per field, a multiple of 128 bytes
  alignas(128) float land[4][LAND];
  unsigned long long bar;
  int iter;  // LP 3: how many tiles this persistent CTA has finished
};

template <int TX, int TY, int FU, int LP>
struct HllcSmemOf {
  using type = HllcSmem<TX, TY>;
};
template <int TX, int TY>
struct HllcSmemOf<TX, TY, 1, 2> {
  using type = HllcSmemTma<TX, TY>;
};
template <int TX, int TY>
struct HllcSmemOf<TX, TY, 1, 3> {
  using type = HllcSmemTma<TX, TY>;
};

__device__ __forceinline__ unsigned smem_addr(const void* ptr) {
  return static_cast<unsigned>(__cvta_generic_to_shared(ptr));
}

// One 2-D tile copy global -> this CTA's shared memory, completing on `bar`. Every
// copy reads this GPU's own memory into the issuing CTA alone.
__device__ __forceinline__ void tma_load_tile(void* dst, const TileMap* map, int x, int y, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_addr(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(smem_addr(bar))
      : "memory");
}

// Wait for phase `parity` of `bar` for at most `max_cycles` SM clocks; false if it gave up.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity, long long max_cycles) {
  const long long t0 = clock64();
  for (;;) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > max_cycles) return false;
  }
}

// A copy that has not landed after ~1 s at the B200's clock is treated as lost.
constexpr long long kTmaWaitCycles = 2000000000LL;


// A tile whose four halo boxes (columns x0-4 .. x0+TX+3, rows y0-3 .. y0+TY+2) lie
// inside the domain.
template <int TX, int TY>
__device__ __forceinline__ bool tma_interior(int x0, int y0, int ny, int nx) {
  return x0 >= 4 && x0 + TX + 4 <= nx && y0 >= 3 && y0 + TY + 3 <= ny;
}

// Thread 0: the four halo boxes of the tile at (x0, y0) into the landing areas, one
// transaction on the barrier.
template <int TX, int TY>
__device__ __forceinline__ void tma_issue_halo(float (*land)[HllcSmemTma<TX, TY>::LAND], unsigned long long* bar,
                                               const HllcMaps* maps, int stage, int cur, int x0, int y0) {
  using ST = HllcSmemTma<TX, TY>;
  constexpr unsigned kBytes = 4u * ST::LW * ST::LH * sizeof(float);
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(kBytes) : "memory");
  tma_load_tile(&land[0][0], stage == 1 ? &maps->h[cur] : &maps->h1, x0 - 4, y0 - 3, bar);
  tma_load_tile(&land[1][0], stage == 1 ? &maps->hu[cur] : &maps->hu1, x0 - 4, y0 - 3, bar);
  tma_load_tile(&land[2][0], stage == 1 ? &maps->hv[cur] : &maps->hv1, x0 - 4, y0 - 3, bar);
  tma_load_tile(&land[3][0], &maps->z, x0 - 4, y0 - 3, bar);
}

// The tile at (x0, y0) is staged from the landing areas (their copies can be issued).
template <int TX, int TY, class SMEM>
__device__ __forceinline__ bool tma_ready(SMEM& S, int x0, int y0, int ny, int nx) {
  return (smem_addr(&S.land[0][0]) & 127u) == 0 && tma_interior<TX, TY>(x0, y0, ny, nx);
}

// Thread 0 of a persistent CTA at tile (bx, by): start the next phase of the barrier
// for the CTA's next tile (gridDim.x tiles on, row-major), if it has one.
template <int TX, int TY, class SMEM>
__device__ __forceinline__ void tma_issue_for(SMEM& S, const HllcMaps* maps, int stage, int cur, int t, int ny,
                                              int nx) {
  const int tiles_x = (nx + TX - 1) / TX;
  if (t >= tiles_x * ((ny + TY - 1) / TY)) return;
  const int x0 = (t % tiles_x) * TX, y0 = (t / tiles_x) * TY;
  if (tma_ready<TX, TY>(S, x0, y0, ny, nx))
    tma_issue_halo<TX, TY>(S.land, &S.bar, maps, stage, cur, x0, y0);
  else
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(&S.bar)) : "memory");
}

template <int TX, int TY, class SMEM>
__device__ __forceinline__ void tma_prefetch_next(SMEM& S, const HllcMaps* maps, int stage, int cur, int bx, int by,
                                                  int ny, int nx) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // the reads above come before the copies
  tma_issue_for<TX, TY>(S, maps, stage, cur, by * ((nx + TX - 1) / TX) + bx + (int)gridDim.x, ny, nx);
}

// A tile whose whole staged region (the tile and a 3-cell halo) lies inside the
// domain: every bounds check and edge case of the tile is known to be false there.
template <int TX, int TY>
__device__ __forceinline__ bool hllc_deep_interior(int x0, int y0, int ny, int nx) {
  return x0 >= 3 && y0 >= 3 && x0 + TX + 3 <= nx && y0 + TY + 3 <= ny;
}

// One Heun stage of tile (bx, by) of domain p; ledger slot `slot`. Called by every
// thread of the block; returns uniformly (false only when a tensor copy never landed:
// the block stops). FU selects the face phase: 1, each face reconstructs its
// four-cell stencil; 2 or 3, FU faces per work item in a rolling window that
// reconstructs each cell once. LP 1 issues a thread's halo loads before its
// divisions; LP 2 stages tiles whose halo lies inside the domain with tensor-memory
// copies from the tensor maps in `maps` (edge tiles take the LP 1 path); LP 3 does
// the same for a persistent block whose next tile's copies complete barrier phase
// `phase`. IN is the instantiation for a tile hllc_deep_interior admits, without the
// bounds checks and edge cases. SRC says whether stage 2 has per-cell sources (the
// compensated rain's h_comp, a rain field, infiltration): 0 no, 1 yes, 2 read from
// the pointers at run time; uniform rain is in every instantiation. Every choice
// computes the same bits.
template <int TX, int TY, int NT, int STAGE, int FU = 1, int LP = 1, bool IN = false, int SRC = 2,
          class SMEM = HllcSmem<TX, TY>>
__device__ __forceinline__ bool hllc_tile(const HllcParams& p, int bx, int by, size_t slot, SMEM& S,
                                          const HllcMaps* maps = nullptr, unsigned phase = 0) {
  static_assert(NT / 32 <= 32, "reduction scratch sized for <= 32 warps");
  static_assert(HllcSmem<TX, TY>::H == 3, "hllc_deep_interior assumes a 3-cell halo");
  using SM = HllcSmem<TX, TY>;
  constexpr int H = SM::H, RW = SM::RW, RH = SM::RH, XW = SM::XW, XH = SM::XH, YW = SM::YW, YH = SM::YH;
  constexpr int BW = SM::BW, BH = SM::BH;
  auto& s_c = S.c;
  auto& s_fxh = S.fxh;
  auto& s_fyh = S.fyh;
  auto& s_fxl = S.fxl;
  auto& s_fxr = S.fxr;
  auto& s_fxt = S.fxt;
  auto& s_fyl = S.fyl;
  auto& s_fyr = S.fyr;
  auto& s_fyt = S.fyt;
  auto& s_beta = S.beta;
  double* s_red = S.red;
  float* s_redf = S.redf;

  const int ny = p.ny, nx = p.nx;
  const int x0 = bx * TX, y0 = by * TY;
  int cur = p.cur, rain_mode = p.rain_mode;
  float dt = p.dt32, rain32 = p.rain32, scale32 = p.scale32;
  float stage_w = p.stage[RB_EDGE_WEST], stage_e = p.stage[RB_EDGE_EAST];
  float stage_n = p.stage[RB_EDGE_NORTH], stage_s = p.stage[RB_EDGE_SOUTH];
  double wt = p.wt;
  if (p.clk != nullptr) {  // device-resident clock: this step's dt and forcing
    const DevClock* c = p.clk;
    if (!c->active) return true;
    cur = c->cur;
    dt = c->dt32;
    wt = c->wt;
    rain32 = c->rain32;
    scale32 = c->scale32;
    rain_mode = (p.h_comp != nullptr && p.rain_field == nullptr) ? 1 : (rain32 != 0.0f ? 2 : 0);
    stage_w = c->stage32[RB_EDGE_WEST];
    stage_e = c->stage32[RB_EDGE_EAST];
    stage_n = c->stage32[RB_EDGE_NORTH];
    stage_s = c->stage32[RB_EDGE_SOUTH];
  }
  // Stage input U_s (U^n for stage 1, U1 for stage 2) and U^n.
  const float* __restrict__ h_s = STAGE == 1 ? p.hb[cur] : p.h1;
  const float* __restrict__ hu_s = STAGE == 1 ? p.hub[cur] : p.hu1;
  const float* __restrict__ hv_s = STAGE == 1 ? p.hvb[cur] : p.hv1;
  const float* __restrict__ h_n = p.hb[cur];
  const float* __restrict__ hu_n = p.hub[cur];
  const float* __restrict__ hv_n = p.hvb[cur];
  const float dx = p.dx32;

  // 1. stage the clamped halo and the primitives (hllc.py:262-282).
  bool staged = false;
  if constexpr (LP == 2) {
    using ST = HllcSmemTma<TX, TY>;
    constexpr int LW = ST::LW, LAND = ST::LAND;
    constexpr unsigned kBytes = 4u * LW * ST::LH * sizeof(float);
    const bool interior = x0 >= 4 && x0 + TX + 4 <= nx && y0 >= 3 && y0 + TY + 3 <= ny &&
                          (smem_addr(&S.land[0][0]) & 127u) == 0;
    if (interior) {
      if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&S.bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(&S.bar)), "r"(kBytes)
                     : "memory");
        const TileMap* mh = STAGE == 1 ? &maps->h[cur] : &maps->h1;
        const TileMap* mu = STAGE == 1 ? &maps->hu[cur] : &maps->hu1;
        const TileMap* mv = STAGE == 1 ? &maps->hv[cur] : &maps->hv1;
        tma_load_tile(&S.land[0][0], mh, x0 - 4, y0 - H, &S.bar);
        tma_load_tile(&S.land[1][0], mu, x0 - 4, y0 - H, &S.bar);
        tma_load_tile(&S.land[2][0], mv, x0 - 4, y0 - H, &S.bar);
        tma_load_tile(&S.land[3][0], &maps->z, x0 - 4, y0 - H, &S.bar);
      }
      // every thread waits for the copies, each for a bounded time; the block agrees
      // on the outcome, so a copy that never lands flags an error and the whole block
      // returns (after waiting, bounded again, for the copies it started)
      const bool ok = mbar_wait_bounded(&S.bar, 0, kTmaWaitCycles);
      if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) flag_error(p.err, RB_DEVERR_TIMEOUT);
        mbar_wait_bounded(&S.bar, 0, kTmaWaitCycles);
        return false;
      }
      // every thread is past its wait: the barrier object is retired before its memory
      // is anything else again
      if (threadIdx.x == 0) asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(&S.bar)) : "memory");
      for (int k = threadIdx.x; k < RH * RW; k += NT) {
        const int r = k / RW, c = k - r * RW;
        const int l = r * LW + c + 1;  // the box starts one column left of the staged region
        const float hh = S.land[0][l];
        float u, v;
        primitives(hh, S.land[1][l], S.land[2][l], u, v);
        s_c[r][c] = make_float4(hh, u, v, S.land[3][l]);
      }
      static_assert(RH * LW <= LAND, "landing area too small");
      staged = true;
    }
  }
  if constexpr (LP == 3) {
    using ST = HllcSmemTma<TX, TY>;
    constexpr int LW = ST::LW;
    if (tma_ready<TX, TY>(S, x0, y0, ny, nx)) {
      const bool ok = mbar_wait_bounded(&S.bar, phase, kTmaWaitCycles);
      if (__syncthreads_or(!ok)) {  // block-uniform: flag, wait once more (bounded), stop
        if (threadIdx.x == 0) flag_error(p.err, RB_DEVERR_TIMEOUT);
        mbar_wait_bounded(&S.bar, phase, kTmaWaitCycles);
        return false;
      }
      for (int k = threadIdx.x; k < RH * RW; k += NT) {
        const int r = k / RW, c = k - r * RW;
        const int l = r * LW + c + 1;  // the box starts one column left of the staged region
        const float hh = S.land[0][l];
        float u, v;
        primitives(hh, S.land[1][l], S.land[2][l], u, v);
        s_c[r][c] = make_float4(hh, u, v, S.land[3][l]);
      }
      staged = true;
    }
  }
  if (staged) {
  } else if constexpr (LP == 0) {
    for (int k = threadIdx.x; k < RH * RW; k += NT) {
      const int r = k / RW, c = k - r * RW;
      const int gi = IN ? y0 - H + r : min(max(y0 - H + r, 0), ny - 1);
      const int gj = IN ? x0 - H + c : min(max(x0 - H + c, 0), nx - 1);
      const size_t id = (size_t)gi * nx + gj;
      const float hh = h_s[id];
      float u, v;
      primitives(hh, hu_s[id], hv_s[id], u, v);
      s_c[r][c] = make_float4(hh, u, v, p.z[id]);
    }
  } else {
    // All of a thread's loads are issued before any of its divisions, so the
    // global-memory latency of the whole halo overlaps.
    constexpr int NL = (RH * RW + NT - 1) / NT;
    float lh[NL], lhu[NL], lhv[NL], lz[NL];
#pragma unroll
    for (int i = 0; i < NL; i++) {
      const int k = threadIdx.x + i * NT;
      if (k < RH * RW) {
        const int r = k / RW, c = k - r * RW;
        const int gi = IN ? y0 - H + r : min(max(y0 - H + r, 0), ny - 1);
        const int gj = IN ? x0 - H + c : min(max(x0 - H + c, 0), nx - 1);
        const size_t id = (size_t)gi * nx + gj;
        lh[i] = h_s[id];
        lhu[i] = hu_s[id];
        lhv[i] = hv_s[id];
        lz[i] = p.z[id];
      }
    }
#pragma unroll
    for (int i = 0; i < NL; i++) {
      const int k = threadIdx.x + i * NT;
      if (k < RH * RW) {
        const int r = k / RW, c = k - r * RW;
        const float hh = lh[i];
        float u, v;
        primitives(hh, lhu[i], lhv[i], u, v);
        s_c[r][c] = make_float4(hh, u, v, lz[i]);
      }
    }
  }
  __syncthreads();

  // 2. face fluxes (hllc.py:285-424) with boundary corrections (:993-1109); an edge
  // face (gj == 0 / nx, gi == 0 / ny) of a closed or fixed_stage edge is the
  // ghost-state problem of any_face_flux.
  // The face phase also keeps, for each tile cell, the reconstructed depths of its
  // east / west (south / north) faces and its bed slope: x-face (a, b) has its left
  // cell at tile (a - 1, b - 2) and its right cell at (a - 1, b - 1); y-face (a, b)
  // its upper cell at (a - 2, b - 1) and its lower cell at (a - 1, b - 1).
  auto keep_x = [&](int a, int b, float h_l, float h_r, float sz_l) {
    if (a >= 1 && a <= TY) {
      if (b >= 2 && b <= TX + 1) {
        S.hpx[a - 1][b - 2] = h_l;
        S.szx[a - 1][b - 2] = sz_l;
      }
      if (b >= 1 && b <= TX) S.hmx[a - 1][b - 1] = h_r;
    }
  };
  auto keep_y = [&](int a, int b, float h_l, float h_r, float sz_l) {
    if (b >= 1 && b <= TX) {
      if (a >= 2 && a <= TY + 1) {
        S.hpy[a - 2][b - 1] = h_l;
        S.szy[a - 2][b - 1] = sz_l;
      }
      if (a >= 1 && a <= TY) S.hmy[a - 1][b - 1] = h_r;
    }
  };
  if constexpr (FU == 1) {
    // One face per work item: four cells along the normal. x- and y-faces share
    // one loop, so the last pass over the block is partly filled once, not twice.
    // A tile whose faces (and the ring's) are all inner faces of the domain runs an
    // instantiation without bounds checks and with the boundary kind fixed at
    // "open", so the edge-ghost code compiles away; the others run the general one.
    constexpr int NXF = XH * XW, NF = XH * XW + YH * YW;
    auto face_loop = [&](auto inner_tag) {
      constexpr bool INNER = decltype(inner_tag)::value;
      for (int k = threadIdx.x; k < NF; k += NT) {
        float fh, fl, fr, ft;
        if (k < NXF) {
          const int a = k / XW, b = k - a * XW;
          const int gi = y0 - 1 + a, gj = x0 - 1 + b;
          if (!INNER && (gi < 0 || gi >= ny || gj < 0 || gj > nx)) continue;
          const int r = a + 2;  // cell row; stencil columns b .. b+3 (cells gj-2 .. gj+1)
          const int kind =
              INNER ? RB_BC_OPEN : (gj == 0 ? p.bc[RB_EDGE_WEST] : (gj == nx ? p.bc[RB_EDGE_EAST] : RB_BC_OPEN));
          const Cell c0 = cell_x(s_c[r][b]);
          const Cell c1 = cell_x(s_c[r][b + 1]);
          const Cell c2 = cell_x(s_c[r][b + 2]);
          const Cell c3 = cell_x(s_c[r][b + 3]);
          // at an edge the clamped stencil is in the staged region; the edge cell is
          // column 0 (c2) or nx-1 (c1)
          const Rec L = recon(c0, c1, c2);
          float h_l, h_r;
          any_face_flux(L, recon(c1, c2, c3), kind, gj == 0, gj == 0 ? c2 : c1, gj == 0 ? stage_w : stage_e, fh,
                        fl, fr, ft, h_l, h_r);
          keep_x(a, b, h_l, h_r, L.sz);
          s_fxh[a][b] = fh;
          if (a >= 1 && a <= TY && b >= 1 && b <= TX + 1) {
            s_fxl[a - 1][b - 1] = fl;
            s_fxr[a - 1][b - 1] = fr;
            s_fxt[a - 1][b - 1] = ft;
          }
        } else {  // y-faces: normal velocity v, transverse u (hllc.py:357-424)
          const int ky = k - NXF;
          const int a = ky / YW, b = ky - a * YW;
          const int gi = y0 - 1 + a, gj = x0 - 1 + b;
          if (!INNER && (gj < 0 || gj >= nx || gi < 0 || gi > ny)) continue;
          const int c = b + 2;  // cell column; stencil rows a .. a+3 (cells gi-2 .. gi+1)
          const int kind =
              INNER ? RB_BC_OPEN : (gi == 0 ? p.bc[RB_EDGE_NORTH] : (gi == ny ? p.bc[RB_EDGE_SOUTH] : RB_BC_OPEN));
          const Cell c0 = cell_y(s_c[a][c]);
          const Cell c1 = cell_y(s_c[a + 1][c]);
          const Cell c2 = cell_y(s_c[a + 2][c]);
          const Cell c3 = cell_y(s_c[a + 3][c]);
          // the edge cell: row 0 (c2) or ny-1 (c1)
          const Rec L = recon(c0, c1, c2);
          float h_l, h_r;
          any_face_flux(L, recon(c1, c2, c3), kind, gi == 0, gi == 0 ? c2 : c1, gi == 0 ? stage_n : stage_s, fh,
                        fl, fr, ft, h_l, h_r);
          keep_y(a, b, h_l, h_r, L.sz);
          s_fyh[a][b] = fh;
          if (a >= 1 && a <= TY + 1 && b >= 1 && b <= TX) {
            s_fyl[a - 1][b - 1] = fl;
            s_fyr[a - 1][b - 1] = fr;
            s_fyt[a - 1][b - 1] = ft;
          }
        }
      }
    };
    // x-faces span columns x0-1 .. x0+TX+1 and rows y0-1 .. y0+TY, y-faces columns
    // x0-1 .. x0+TX and rows y0-1 .. y0+TY+1: all inner faces when these hold
    if constexpr (IN) {
      face_loop(std::true_type{});
    } else {
      const bool inner = x0 >= 2 && y0 >= 2 && x0 + TX + 2 <= nx && y0 + TY + 2 <= ny;
      if (inner)
        face_loop(std::true_type{});
      else
        face_loop(std::false_type{});
    }
  } else {
    // FU consecutive faces per work item along the normal, each cell reconstructed
    // once in a rolling window: the reference's face-local eta_l / eta_r are the
    // left cell's east and the right cell's west values.
    constexpr int GX = (XW + FU - 1) / FU, GY = (YH + FU - 1) / FU;
    for (int k = threadIdx.x; k < XH * GX; k += NT) {
      const int a = k / GX, g = k - a * GX;
      const int gi = y0 - 1 + a;
      if (gi < 0 || gi >= ny) continue;
      const int r = a + 2;
      const int b0 = g * FU;
      Cell c0 = cell_x(s_c[r][b0 + 1]);
      Cell cp = cell_x(s_c[r][b0 + 2]);
      Rec left = recon(cell_x(s_c[r][b0]), c0, cp);
#pragma unroll
      for (int f = 0; f < FU; f++) {
        const int b = b0 + f;
        const int bb = b < XW ? b : XW - 1;  // a unit past the row end recomputes the last face, unstored
        const Cell cn = cell_x(s_c[r][bb + 3]);
        const Rec right = recon(c0, cp, cn);
        const int gj = x0 - 1 + b;
        if (b < XW && gj >= 0 && gj <= nx) {
          float fh, fl, fr, ft;
          const int kind = gj == 0 ? p.bc[RB_EDGE_WEST] : (gj == nx ? p.bc[RB_EDGE_EAST] : RB_BC_OPEN);
          // edge cell: column 0 (cp) or nx-1 (c0)
          float h_l, h_r;
          any_face_flux(left, right, kind, gj == 0, gj == 0 ? cp : c0, gj == 0 ? stage_w : stage_e, fh, fl, fr, ft,
                        h_l, h_r);
          keep_x(a, b, h_l, h_r, left.sz);
          s_fxh[a][b] = fh;
          if (a >= 1 && a <= TY && b >= 1 && b <= TX + 1) {
            s_fxl[a - 1][b - 1] = fl;
            s_fxr[a - 1][b - 1] = fr;
            s_fxt[a - 1][b - 1] = ft;
          }
        }
        left = right;
        c0 = cp;
        cp = cn;
      }
    }
    for (int k = threadIdx.x; k < GY * YW; k += NT) {
      const int g = k / YW, b = k - g * YW;
      const int gj = x0 - 1 + b;
      if (gj < 0 || gj >= nx) continue;
      const int c = b + 2;
      const int a0 = g * FU;
      Cell c0 = cell_y(s_c[a0 + 1][c]);
      Cell cp = cell_y(s_c[a0 + 2][c]);
      Rec left = recon(cell_y(s_c[a0][c]), c0, cp);
#pragma unroll
      for (int f = 0; f < FU; f++) {
        const int a = a0 + f;
        const int aa = a < YH ? a : YH - 1;
        const Cell cn = cell_y(s_c[aa + 3][c]);
        const Rec right = recon(c0, cp, cn);
        const int gi = y0 - 1 + a;
        if (a < YH && gi >= 0 && gi <= ny) {
          float fh, fl, fr, ft;
          const int kind = gi == 0 ? p.bc[RB_EDGE_NORTH] : (gi == ny ? p.bc[RB_EDGE_SOUTH] : RB_BC_OPEN);
          // edge cell: row 0 (cp) or ny-1 (c0)
          float h_l, h_r;
          any_face_flux(left, right, kind, gi == 0, gi == 0 ? cp : c0, gi == 0 ? stage_n : stage_s, fh, fl, fr, ft,
                        h_l, h_r);
          keep_y(a, b, h_l, h_r, left.sz);
          s_fyh[a][b] = fh;
          if (a >= 1 && a <= TY + 1 && b >= 1 && b <= TX) {
            s_fyl[a - 1][b - 1] = fl;
            s_fyr[a - 1][b - 1] = fr;
            s_fyt[a - 1][b - 1] = ft;
          }
        }
        left = right;
        c0 = cp;
        cp = cn;
      }
    }
  }
  __syncthreads();
  if constexpr (LP == 3) {
    // every thread has long read the landing areas: thread 0 refills them with the
    // CTA's next tile's halo while this tile's update is computed
    if (threadIdx.x == 0) tma_prefetch_next<TX, TY>(S, maps, STAGE, cur, bx, by, ny, nx);
  }

  // 3. mass-only donor beta on the tile + ring (hllc.py:700-736).
  const float dtdx = dt / dx;
  for (int k = threadIdx.x; k < BH * BW; k += NT) {
    const int a = k / BW, b = k - a * BW;
    const int gi = y0 - 1 + a, gj = x0 - 1 + b;
    float beta = 1.0f;
    if (IN || (gi >= 0 && gi < ny && gj >= 0 && gj < nx)) {
      float q_out = 0.0f;
      const float fl = s_fxh[a][b];
      if (fl < 0.0f) q_out = q_out - fl;
      const float fr = s_fxh[a][b + 1];
      if (fr > 0.0f) q_out = q_out + fr;
      const float ft = s_fyh[a][b];
      if (ft < 0.0f) q_out = q_out - ft;
      const float fb = s_fyh[a + 1][b];
      if (fb > 0.0f) q_out = q_out + fb;
      const float out_depth = dtdx * q_out;
      const bool out = out_depth > 0.0f;
      const float ratio = div_if(out, s_c[a + 2][b + 2].x, out_depth);
      if (out) beta = rclamp(ratio, 0.0f, 1.0f);
    }
    s_beta[a][b] = beta;
  }
  __syncthreads();

  double loss = 0.0;

  // 4. divergence + centred bed source (hllc.py:776-847) and the Heun update. Each
  //    cell limits its four mass faces by their donor as it reads them
  //    (hllc.py:739-773): a face shared by two cells is limited by both with the same
  //    operands, so both see the same bits, and no pass over the faces and no barrier
  //    sits between the beta and the update. The cell at a domain edge banks the
  //    limited flux of its edge face if that edge is open or fixed_stage
  //    (hllc.py:638-677).
  const float inv_dx = 1.0f / dx;
  const float g = kG;
  float smax = 0.0f;
  bool bad = false;
  // The global inputs of this thread's cells are loaded first, all of them, so their
  // latency overlaps instead of stalling each cell's update in turn.
  constexpr int NC = (TX * TY + NT - 1) / NT;
  float g_hus[NC], g_hvs[NC], g_hn[NC], g_hun[NC], g_hvn[NC], g_n[NC];
#pragma unroll
  for (int i = 0; i < NC; i++) {
    const int k = threadIdx.x + i * NT;
    const int r = k / TX, c = k - r * TX;
    const int gi = y0 + r, gj = x0 + c;
    if (k < TX * TY && (IN || (gi < ny && gj < nx))) {
      const size_t id = (size_t)gi * nx + gj;
      g_hus[i] = hu_s[id];
      g_hvs[i] = hv_s[id];
      if (STAGE == 2) {
        g_hn[i] = h_n[id];
        g_hun[i] = hu_n[id];
        g_hvn[i] = hv_n[id];
        g_n[i] = p.n[id];
      }
    }
  }
#pragma unroll
  for (int i = 0; i < NC; i++) {
    const int k = threadIdx.x + i * NT;
    const int r = k / TX, c = k - r * TX;
    const int gi = y0 + r, gj = x0 + c;
    if (k >= TX * TY || (!IN && (gi >= ny || gj >= nx))) continue;
    const size_t id = (size_t)gi * nx + gj;
    const int R = r + H, Cc = c + H;  // this cell in the staged region
    // west / east faces: the donor of q > 0 is the cell to the west, of q < 0 the
    // cell to the east, and a face with no donor cell inside the domain stays as is
    float qw = s_fxh[r + 1][c + 1];
    if (qw > 0.0f) {
      if (IN || gj >= 1) qw = qw * s_beta[r + 1][c];
    } else if (qw < 0.0f) {
      qw = qw * s_beta[r + 1][c + 1];
    }
    float qe = s_fxh[r + 1][c + 2];
    if (qe > 0.0f) {
      qe = qe * s_beta[r + 1][c + 1];
    } else if (qe < 0.0f) {
      if (IN || gj + 1 <= nx - 1) qe = qe * s_beta[r + 1][c + 2];
    }
    float qn = s_fyh[r + 1][c + 1];
    if (qn > 0.0f) {
      if (IN || gi >= 1) qn = qn * s_beta[r][c + 1];
    } else if (qn < 0.0f) {
      qn = qn * s_beta[r + 1][c + 1];
    }
    float qs = s_fyh[r + 2][c + 1];
    if (qs > 0.0f) {
      qs = qs * s_beta[r + 1][c + 1];
    } else if (qs < 0.0f) {
      if (IN || gi + 1 <= ny - 1) qs = qs * s_beta[r + 2][c + 1];
    }
    if (!IN && p.ledger != nullptr) {  // an interior tile has no edge face
      if (gj == 0 && p.bc[RB_EDGE_WEST] != RB_BC_CLOSED) loss -= wt * (double)qw;
      if (gj == nx - 1 && p.bc[RB_EDGE_EAST] != RB_BC_CLOSED) loss += wt * (double)qe;
      if (gi == 0 && p.bc[RB_EDGE_NORTH] != RB_BC_CLOSED) loss -= wt * (double)qn;
      if (gi == ny - 1 && p.bc[RB_EDGE_SOUTH] != RB_BC_CLOSED) loss += wt * (double)qs;
    }
    const float dh = -((qe - qw) + (qs - qn)) * inv_dx;
    const float hg = s_c[R][Cc].x;
    // the centred bed source (hllc.py:805-813): the cell's reconstructed depths at
    // its two faces and its bed slope, as the face phase computed them (the
    // reference's hp = max((eta + se/2) - (z + sz/2), 0) is the reconstruction's
    // east depth bit for bit, hm its west depth)
    const float sz_x = S.szx[r][c];
    const float src_x = -g * 0.5f * (S.hpx[r][c] + S.hmx[r][c]) * sz_x;
    const float dhu = (-((s_fxl[r][c + 1] - s_fxr[r][c]) + (s_fyt[r + 1][c] - s_fyt[r][c])) + src_x) * inv_dx;
    const float sz_y = S.szy[r][c];
    const float src_y = -g * 0.5f * (S.hpy[r][c] + S.hmy[r][c]) * sz_y;
    const float dhv = (-((s_fyl[r + 1][c] - s_fyr[r][c]) + (s_fxt[r][c + 1] - s_fxt[r][c])) + src_y) * inv_dx;

    if (STAGE == 1) {  // hllc.py:850-878
      const float hh = rmax(hg + dt * dh, 0.0f);
      float hu1 = 0.0f, hv1 = 0.0f;
      if (hh > kHDry) {
        hu1 = g_hus[i] + dt * dhu;
        hv1 = g_hvs[i] + dt * dhv;
      }
      p.h1[id] = hh;
      p.hu1[id] = hu1;
      p.hv1[id] = hv1;
    } else {  // hllc.py:881-909, then friction :912-939, then sources :1350-1373
      float hh = rmax(0.5f * (g_hn[i] + hg + dt * dh), 0.0f);
      float hu = 0.0f, hv = 0.0f;
      if (hh > kHDry) {
        hu = 0.5f * (g_hun[i] + g_hus[i] + dt * dhu);
        hv = 0.5f * (g_hvn[i] + g_hvs[i] + dt * dhv);
        // friction (hllc.py:912-939): the numerator g dt n^2 |q| is zero, and the
        // denominator exactly 1 so hu and hv stand as they are, whenever n = 0 with a
        // finite |q|^2 or the water is still with a finite g dt n^2; neither the
        // square root nor the power is needed then
        const float m2 = hu * hu + hv * hv;
        const float k = g * dt * g_n[i] * g_n[i];
        if (!((k == 0.0f && m2 <= FLT_MAX) || (m2 == 0.0f && k <= FLT_MAX))) {
          const float f = k * sqrtf(m2);
          if (!(f == 0.0f)) {
            const float denom = 1.0f + f / pow73(hh);
#if defined(RB_FAST_MATH)
            const float rd = 1.0f / denom;
            hu = hu * rd;
            hv = hv * rd;
#else
            hu = div_pos(hu, denom);
            hv = div_pos(hv, denom);
#endif
          }
        }
      }
      if (SRC != 0 && rain_mode == 1) {
        float comp = p.h_comp[id];
        kahan_add(hh, comp, rain32 * dt);
        p.h_comp[id] = comp;
      } else if (rain_mode == 2) {
        hh = hh + rain32 * dt;  // hllc.py:942-945
      }
      if (SRC != 0 && p.rain_field != nullptr) {
        if (p.h_comp != nullptr) {
          float comp = p.h_comp[id];
          kahan_add(hh, comp, p.rain_field[id] * scale32 * dt);
          p.h_comp[id] = comp;
        } else {
          hh = hh + p.rain_field[id] * scale32 * dt;
        }
      }
      if (SRC != 0 && p.infil != nullptr) {  // local_inertial.py:170-194
        const float avail = hh;
        float inf = p.infil[id] * dt;
        if (inf > avail) inf = avail;
        if (inf < 0.0f) inf = 0.0f;
        hh = avail - inf;
        loss += (double)avail - (double)hh;
      }
      p.hb[cur ^ 1][id] = hh;
      p.hub[cur ^ 1][id] = hu;
      p.hvb[cur ^ 1][id] = hv;
      // hllc.py:948-966 _reduce_wavespeed on the new state
      const float cw = sqrtf(g * rmax(hh, 0.0f));
      const bool wet = hh > kHDry;
#if defined(RB_FAST_MATH)
      const float s = wet ? rmax(fabsf(hu), fabsf(hv)) * (1.0f / (wet ? hh : 1.0f)) + cw : cw;
#else
      const float s = wet ? rmax(div_if(wet, fabsf(hu), hh), div_if(wet, fabsf(hv), hh)) + cw : cw;
#endif
      smax = s > smax ? s : smax;
      bad |= !(fabsf(hh) <= FLT_MAX) || !(fabsf(hu) <= FLT_MAX) || !(fabsf(hv) <= FLT_MAX);
    }
  }

  // An interior tile banks nothing but infiltration (it has no edge face), so without
  // infiltration its loss is 0 and its slot, zero from the start, stays exactly 0:
  // the block sum is skipped.
  if (p.ledger != nullptr && (!IN || (STAGE == 2 && SRC != 0 && p.infil != nullptr))) {
    const double s = block_sum<NT>(loss, s_red);
    if (threadIdx.x == 0) ledger_add(p.ledger + 2 * slot, s);
  }
  if (STAGE == 2) {
    if (p.smax_key != nullptr) block_max_to<NT>(smax, p.smax_key, s_redf);
    if (bad) flag_error(p.err, RB_DEVERR_NONFINITE);
  }
  __syncthreads();  // the shared tile is reused by the caller's next tile
  return true;
}

// The single-domain stage kernel. Shared memory is dynamic (a 32 x 32 tile needs
// more than the 48 KB a static array may take); __launch_bounds__ asks for two
// resident blocks of 512 threads or more (four of 256) per SM: at most 64 registers
// a thread for 512, 51 for 640.
template <int TX, int TY, int NT, int STAGE, int FU, int LP, int SRC>
__global__ void __launch_bounds__(NT, NT > 512 ? 2 : 1024 / NT) hllc_stage_kernel(const HllcParams p) {
  extern __shared__ __align__(16) unsigned char hllc_smem_raw[];
  using SMEM = typename HllcSmemOf<TX, TY, FU, LP>::type;
  auto& S = *reinterpret_cast<SMEM*>(hllc_smem_raw);
  pdl_enter();
  const size_t slot = (size_t)blockIdx.y * gridDim.x + blockIdx.x;
  if (hllc_deep_interior<TX, TY>(blockIdx.x * TX, blockIdx.y * TY, p.ny, p.nx))
    hllc_tile<TX, TY, NT, STAGE, FU, LP, true, SRC>(p, blockIdx.x, blockIdx.y, slot, S);
  else
    hllc_tile<TX, TY, NT, STAGE, FU, LP, false, SRC>(p, blockIdx.x, blockIdx.y, slot, S);
}

// The shared-memory opt-in is a per-device function attribute: set once per device
// for an instantiation (setting it twice is harmless if threads race here).
template <int TX, int TY, int NT, int FU, int LP>
static void prepare_hllc() {
  constexpr int smem = (int)sizeof(typename HllcSmemOf<TX, TY, FU, LP>::type);
  static std::atomic<unsigned long long> attr_set{0};
  int dev = 0;
  cudaGetDevice(&dev);
  const unsigned long long bit = 1ull << (dev & 63);
  if (!(attr_set.load() & bit)) {
    cudaFuncSetAttribute(hllc_stage_kernel<TX, TY, NT, 1, FU, LP, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         smem);
    cudaFuncSetAttribute(hllc_stage_kernel<TX, TY, NT, 2, FU, LP, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         smem);
    cudaFuncSetAttribute(hllc_stage_kernel<TX, TY, NT, 2, FU, LP, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         smem);
    attr_set.fetch_or(bit);
  }
}

template <int TX, int TY, int NT, int FU, int LP>
static cudaError_t launch_hllc(const HllcParams& p, int stage, cudaStream_t s) {
  constexpr size_t smem = sizeof(typename HllcSmemOf<TX, TY, FU, LP>::type);
  static_assert(smem <= 227 * 1024, "tile does not fit in shared memory");
  prepare_hllc<TX, TY, NT, FU, LP>();
  const dim3 grid((p.nx + TX - 1) / TX, (p.ny + TY - 1) / TY);
  // stage 1 has no sources; stage 2 carries their code only when one is armed
  if (stage == 1) return launch_chain(hllc_stage_kernel<TX, TY, NT, 1, FU, LP, 0>, grid, dim3(NT), smem, s, p);
  const bool src = p.h_comp != nullptr || p.rain_field != nullptr || p.infil != nullptr;
  return src ? launch_chain(hllc_stage_kernel<TX, TY, NT, 2, FU, LP, 1>, grid, dim3(NT), smem, s, p)
             : launch_chain(hllc_stage_kernel<TX, TY, NT, 2, FU, LP, 0>, grid, dim3(NT), smem, s, p);
}

// The TMA-staged stage kernel: interior tiles copy their halo with tensor-memory
// copies from the tensor maps passed by value (grid constants).
template <int TX, int TY, int NT, int STAGE>
__global__ void __launch_bounds__(NT, NT > 512 ? 2 : 1024 / NT)
    hllc_stage_tma_kernel(const HllcParams p, const __grid_constant__ HllcMaps maps) {
  extern __shared__ __align__(1024) unsigned char hllc_tma_smem_raw[];
  auto& S = *reinterpret_cast<HllcSmemTma<TX, TY>*>(hllc_tma_smem_raw);
  pdl_enter();
  const size_t slot = (size_t)blockIdx.y * gridDim.x + blockIdx.x;
  if (hllc_deep_interior<TX, TY>(blockIdx.x * TX, blockIdx.y * TY, p.ny, p.nx))
    hllc_tile<TX, TY, NT, STAGE, 1, 2, true>(p, blockIdx.x, blockIdx.y, slot, S, &maps);
  else
    hllc_tile<TX, TY, NT, STAGE, 1, 2, false>(p, blockIdx.x, blockIdx.y, slot, S, &maps);
}

// The persistent, prefetching form: a grid of as many CTAs as fit the device at once,
// each taking tiles blockIdx.x, blockIdx.x + gridDim.x, ... (one ledger slot per tile,
// as in the one-tile-per-block grid, so the sums are the same bits). While a CTA
// computes one tile, the halo of its next interior tile is already on its way.
template <int TX, int TY, int NT, int STAGE>
__global__ void __launch_bounds__(NT, NT > 512 ? 2 : 1024 / NT)
    hllc_stage_tma_pipe_kernel(const HllcParams p, const __grid_constant__ HllcMaps maps) {
  extern __shared__ __align__(1024) unsigned char hllc_pipe_smem_raw[];
  auto& S = *reinterpret_cast<HllcSmemTma<TX, TY>*>(hllc_pipe_smem_raw);
  pdl_enter();
  if (p.clk != nullptr && !p.clk->active) return;  // no tile works this step
  const int cur = p.clk != nullptr ? p.clk->cur : p.cur;
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&S.bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    tma_issue_for<TX, TY>(S, &maps, STAGE, cur, blockIdx.x, p.ny, p.nx);
  }
  if (threadIdx.x == 0) S.iter = 0;
  __syncthreads();
  // The tile counter lives in shared memory, so nothing of the loop is held in
  // registers across a tile (the tile itself needs all 48 that two resident blocks of
  // 640 threads leave a thread). The k-th tile of this CTA waits on barrier parity k & 1.
  for (;;) {
    const int k = S.iter;
    const int tiles_x = (p.nx + TX - 1) / TX;
    const int t = blockIdx.x + k * gridDim.x;
    if (t >= tiles_x * ((p.ny + TY - 1) / TY)) return;
    if (!hllc_tile<TX, TY, NT, STAGE, 1, 3>(p, t % tiles_x, t / tiles_x, (size_t)t, S, &maps, k & 1u)) return;
    if (threadIdx.x == 0) S.iter++;  // every thread read it before the tile's last barrier
    __syncthreads();
  }
}

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// The driver's tensor-map encoder, reached through the runtime (the library links no
// driver library); null if the driver does not offer it.
static EncodeTiledFn tensor_map_encoder() {
  static const EncodeTiledFn fn = []() -> EncodeTiledFn {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    return reinterpret_cast<EncodeTiledFn>(f);
  }();
  return fn;
}

// The tensor map of one ny x nx float32 field for boxes of bw columns by bh rows.
// Maps depend only on (address, shape, box), so they are kept in a small cache.
static bool field_map(TileMap& out, const float* base, int ny, int nx, int bw, int bh) {
  static_assert(sizeof(CUtensorMap) == sizeof(TileMap), "a tensor map is 128 bytes");
  if (base == nullptr || (reinterpret_cast<uintptr_t>(base) & 15u) != 0 || nx % 4 != 0 || nx < bw || ny < bh)
    return false;  // the copies need 16-byte aligned rows
  struct Key {
    const float* base;
    int ny, nx, bw, bh;
    bool operator==(const Key& o) const {
      return base == o.base && ny == o.ny && nx == o.nx && bw == o.bw && bh == o.bh;
    }
  };
  struct KeyHash {
    size_t operator()(const Key& k) const {
      return std::hash<const void*>()(k.base) ^ ((size_t)k.ny * 1000003u + (size_t)k.nx * 8191u + k.bw * 131u + k.bh);
    }
  };
  static std::mutex mu;
  static std::unordered_map<Key, TileMap, KeyHash> cache;
  const Key key{base, ny, nx, bw, bh};
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(key);
    if (it != cache.end()) {
      out = it->second;
      return true;
    }
  }
  const EncodeTiledFn enc = tensor_map_encoder();
  if (enc == nullptr) return false;
  CUtensorMap m;
  const cuuint64_t dims[2] = {(cuuint64_t)nx, (cuuint64_t)ny};
  const cuuint64_t strides[1] = {(cuuint64_t)nx * sizeof(float)};
  const cuuint32_t box[2] = {(cuuint32_t)bw, (cuuint32_t)bh};
  const cuuint32_t elem[2] = {1, 1};
  if (enc(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box, elem,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return false;
  std::memcpy(&out, &m, sizeof m);
  std::lock_guard<std::mutex> lock(mu);
  if (cache.size() > 4096) cache.clear();
  cache.emplace(key, out);
  return true;
}

template <int TX, int TY, int NT>
static void prepare_hllc_tma() {
  constexpr int smem = (int)sizeof(HllcSmemTma<TX, TY>);
  static std::atomic<unsigned long long> attr_set{0};
  int dev = 0;
  cudaGetDevice(&dev);
  const unsigned long long bit = 1ull << (dev & 63);
  if (!(attr_set.load() & bit)) {
    cudaFuncSetAttribute(hllc_stage_tma_kernel<TX, TY, NT, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaFuncSetAttribute(hllc_stage_tma_kernel<TX, TY, NT, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    attr_set.fetch_or(bit);
  }
}

// The resident-CTA count of the persistent kernel on the current device (its SMs times
// the blocks one SM holds), found once per device; 0 if the device cannot hold a block.
template <int TX, int TY, int NT>
static int hllc_pipe_grid() {
  static std::atomic<int> per_dev[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  int g = per_dev[dev & 63].load();
  if (g == 0) {
    constexpr int smem = (int)sizeof(HllcSmemTma<TX, TY>);
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaFuncSetAttribute(hllc_stage_tma_pipe_kernel<TX, TY, NT, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             smem) != cudaSuccess ||
        cudaFuncSetAttribute(hllc_stage_tma_pipe_kernel<TX, TY, NT, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, hllc_stage_tma_pipe_kernel<TX, TY, NT, 2>, NT, smem) !=
            cudaSuccess) {
      cudaGetLastError();
      per_sm = 0;
    }
    g = per_sm > 0 && sms > 0 ? per_sm * sms : -1;
    per_dev[dev & 63].store(g);
  }
  return g > 0 ? g : 0;
}

// Launch a TMA-staged kernel when every staged field can be mapped (16-byte aligned
// rows, a grid at least one box large); otherwise the same tile with plain loads.
// PIPE selects the persistent, prefetching kernel.
template <int TX, int TY, int NT, bool PIPE = false>
static cudaError_t launch_hllc_tma(const HllcParams& p, int stage, cudaStream_t s) {
  constexpr size_t smem = sizeof(HllcSmemTma<TX, TY>);
  static_assert(smem <= 113 * 1024, "two blocks of the TMA-staged tile must fit an SM");
  constexpr int BW = TX + 8, BH = TY + 6;
  HllcMaps m;
  bool ok = true;
  for (int b = 0; b < 2 && ok; b++)
    ok = field_map(m.h[b], p.hb[b], p.ny, p.nx, BW, BH) && field_map(m.hu[b], p.hub[b], p.ny, p.nx, BW, BH) &&
         field_map(m.hv[b], p.hvb[b], p.ny, p.nx, BW, BH);
  ok = ok && field_map(m.z, p.z, p.ny, p.nx, BW, BH) && field_map(m.h1, p.h1, p.ny, p.nx, BW, BH) &&
       field_map(m.hu1, p.hu1, p.ny, p.nx, BW, BH) && field_map(m.hv1, p.hv1, p.ny, p.nx, BW, BH);
  if (!ok) return launch_hllc<TX, TY, NT, 1, 1>(p, stage, s);
  const int tiles = ((p.nx + TX - 1) / TX) * ((p.ny + TY - 1) / TY);
  if constexpr (PIPE) {
    const int resident = hllc_pipe_grid<TX, TY, NT>();
    if (resident == 0) return launch_hllc<TX, TY, NT, 1, 1>(p, stage, s);
    const dim3 grid(std::min(resident, tiles));
    return stage == 1 ? launch_chain(hllc_stage_tma_pipe_kernel<TX, TY, NT, 1>, grid, dim3(NT), smem, s, p, m)
                      : launch_chain(hllc_stage_tma_pipe_kernel<TX, TY, NT, 2>, grid, dim3(NT), smem, s, p, m);
  }
  prepare_hllc_tma<TX, TY, NT>();
  const dim3 grid((p.nx + TX - 1) / TX, (p.ny + TY - 1) / TY);
  return stage == 1 ? launch_chain(hllc_stage_tma_kernel<TX, TY, NT, 1>, grid, dim3(NT), smem, s, p, m)
                    : launch_chain(hllc_stage_tma_kernel<TX, TY, NT, 2>, grid, dim3(NT), smem, s, p, m);
}

// Kernel variants of the single-domain stage: tile, block size, faces per work item,
// load batching. All compute the same bits; they differ only in speed. The default
// (6: 32 x 32 tiles, 640 threads, two blocks and 40 warps per SM, 44-48 registers)
// is the fastest measured on B200: 0.316 ms per 2048 x 2048 dam-break step against
// 0.326 for 512 threads, 0.337 for 576, 0.323 for 608, 0.328 for 768 and 0.348 for
// 800 (which spills at its 40-register bound). The 2380 face work items of a tile
// fill 3.7 passes of 640 threads against 4.6 of 512. Staging interior tiles with
// tensor-memory copies measures 0.319 ms (7: one tile a block) and 0.360 ms (8: one
// resident block of 512 threads per slot walking the tiles and prefetching the next
// one's halo, against 0.330 for the same block as a grid of tiles): the copies free no
// issue slots the tile needs, and a static walk leaves SMs idle at the end.
struct HllcKernelVariant {
  int tx, ty, nt, fu, lp;
};
static const HllcKernelVariant kHllcVariants[] = {
    {32, 16, 256, 1, 0}, {32, 16, 256, 1, 1}, {32, 16, 256, 3, 1},
    {32, 16, 256, 2, 1}, {32, 32, 512, 1, 1}, {64, 16, 512, 1, 1}, {32, 32, 640, 1, 1},
    {32, 32, 640, 1, 2}, {32, 32, 512, 1, 3},
};
constexpr int kNumHllcVariants = (int)(sizeof(kHllcVariants) / sizeof(kHllcVariants[0]));
constexpr int kDefaultHllcVariant = 6;
#if !defined(RB_FAST_MATH)
static std::atomic<int> g_hllc_variant{kDefaultHllcVariant};

int hllc_kernel_variant_count() { return kNumHllcVariants; }
#endif

// Set every variant's shared-memory opt-in on the current device, outside any
// stream capture (called by the non-capturable set-up entry points).
void hllc_prepare_device() {
  prepare_hllc<32, 16, 256, 1, 0>();
  prepare_hllc<32, 16, 256, 1, 1>();
  prepare_hllc<32, 16, 256, 3, 1>();
  prepare_hllc<32, 16, 256, 2, 1>();
  prepare_hllc<32, 32, 512, 1, 1>();
  prepare_hllc<64, 16, 512, 1, 1>();
  prepare_hllc<32, 32, 640, 1, 1>();
  prepare_hllc_tma<32, 32, 640>();
  hllc_pipe_grid<32, 32, 512>();
#if !defined(RB_FAST_MATH)
  fast::hllc_prepare_device();
#endif
}
#if !defined(RB_FAST_MATH)
bool hllc_set_kernel_variant(int v) {
  if (v < 0 || v >= kNumHllcVariants) return false;
  g_hllc_variant.store(v);
  return true;
}

int hllc_current_variant() { return g_hllc_variant.load(); }

cudaError_t hllc_stage_launch(const HllcParams& p, int stage, cudaStream_t s) {
  return hllc_stage_launch_variant(p, stage, g_hllc_variant.load(), s);
}

#endif  // !RB_FAST_MATH

cudaError_t hllc_stage_launch_variant(const HllcParams& p, int stage, int variant, cudaStream_t s) {
#if !defined(RB_FAST_MATH)
  if (arith_mode() == RB_ARITH_FAST) return fast::hllc_stage_launch_variant(p, stage, variant, s);
  return hllc_stage_launch_exact(p, stage, variant, s);
}

// This build's stage kernel whatever the arithmetic mode (the exact build: what the
// ensembles, which run exact arithmetic only, launch for their large domains).
cudaError_t hllc_stage_launch_exact(const HllcParams& p, int stage, int variant, cudaStream_t s) {
#endif
  switch (variant) {
    case 1: return launch_hllc<32, 16, 256, 1, 1>(p, stage, s);
    case 2: return launch_hllc<32, 16, 256, 3, 1>(p, stage, s);
    case 3: return launch_hllc<32, 16, 256, 2, 1>(p, stage, s);
    case 5: return launch_hllc<64, 16, 512, 1, 1>(p, stage, s);
    case 0: return launch_hllc<32, 16, 256, 1, 0>(p, stage, s);
    case 4: return launch_hllc<32, 32, 512, 1, 1>(p, stage, s);
    case 7: return launch_hllc_tma<32, 32, 640>(p, stage, s);
    case 8: return launch_hllc_tma<32, 32, 512, true>(p, stage, s);
    default: return launch_hllc<32, 32, 640, 1, 1>(p, stage, s);
  }
}

#if !defined(RB_FAST_MATH)
// Tiles of the current variant (one ledger slot each); never more than the 32 x 8
// tiling the workspace ledger is sized for.
int hllc_tiles(int ny, int nx) { return hllc_tiles_of(g_hllc_variant.load(), ny, nx); }

int hllc_tiles_of(int variant, int ny, int nx) {
  const HllcKernelVariant& v = kHllcVariants[variant >= 0 && variant < kNumHllcVariants ? variant : kDefaultHllcVariant];
  return ((nx + v.tx - 1) / v.tx) * ((ny + v.ty - 1) / v.ty);
}

// Ensemble: one Heun stage over the (domain, local tile) work-list of every HLLC
// domain (stage 2 of any domain starts only after stage 1 of all of them, as the
// single-domain step requires for its own tiles). The work item's domain parameters
// are staged in shared memory: read from there, the dozens of pointers and scalars
// need not stay in registers through the tile.
template <int TX, int TY, int NT, int STAGE>
__device__ __forceinline__ void ens_hllc_items(const HllcParams* __restrict__ P, const int2* __restrict__ map,
                                               long long total, HllcSmem<TX, TY>& S, HllcParams& sp) {
  static_assert(sizeof(HllcParams) % 4 == 0, "parameters copied as 32-bit words");
  constexpr int NW = (int)(sizeof(HllcParams) / 4);
  static_assert(NW <= NT, "one word per thread");
  for (long long t = blockIdx.x; t < total; t += gridDim.x) {
    const int2 m = map[t];
    // every thread is done with the previous item's parameters (a tile of a domain
    // whose clock is inactive returns without a barrier)
    __syncthreads();
    if (threadIdx.x < NW)
      reinterpret_cast<unsigned*>(&sp)[threadIdx.x] = reinterpret_cast<const unsigned*>(P + m.x)[threadIdx.x];
    __syncthreads();
    const int tiles_x = (sp.nx + TX - 1) / TX;
    hllc_tile<TX, TY, NT, STAGE>(sp, m.y % tiles_x, m.y / tiles_x, (size_t)m.y, S);
  }
}

// 32 x 16 and 32 x 8 tiles, 256 threads. Three resident blocks per SM (at most 80
// registers) measured fastest: 0.479 ms per step for 16 domains of 512 x 512 against
// 0.552 with no register bound and 0.517 with four blocks (which spills).
template <int TX, int TY, int NT, int STAGE>
__global__ void __launch_bounds__(NT, 768 / NT) ens_hllc_kernel(const HllcParams* __restrict__ P,
                                                                 const int2* __restrict__ map, long long total) {
  __shared__ HllcSmem<TX, TY> S;
  __shared__ __align__(16) HllcParams sp;
  ens_hllc_items<TX, TY, NT, STAGE>(P, map, total, S, sp);
}

// The 32 x 32 tile of the single-domain default as a plain grid: one block of 640
// threads per (domain, tile) work item, the domain's parameters read from global
// memory (shared memory, more than a static array may take, is dynamic). Measured
// against a persistent form of the same tile (512 threads, parameters staged in
// shared memory, which spilled at its 64-register bound): 11.4 vs 9.4
// Gcell-updates/s on dam breaks of 8 x 512^2, 16 x 256^2 and 2 x 768^2.
constexpr int kEnsWideNT = 640;
constexpr size_t kEnsWideSmem = sizeof(HllcSmem<32, 32>);
template <int STAGE>
__global__ void __launch_bounds__(kEnsWideNT, 2) ens_hllc_wide_kernel(const HllcParams* __restrict__ P,
                                                                     const int2* __restrict__ map) {
  extern __shared__ __align__(16) unsigned char ens_wide_smem[];
  auto& S = *reinterpret_cast<HllcSmem<32, 32>*>(ens_wide_smem);
  const int2 m = map[blockIdx.x];
  const HllcParams& p = P[m.x];
  const int tiles_x = (p.nx + 31) / 32;
  hllc_tile<32, 32, kEnsWideNT, STAGE>(p, m.y % tiles_x, m.y / tiles_x, (size_t)m.y, S);
}

template <int TX, int TY, int NT>
static int ens_hllc_grid() {
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ens_hllc_kernel<TX, TY, NT, 2>, NT, 0);
  return (per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1);
}

// Sets the wide kernel's shared-memory opt-in on the current device (outside any
// stream capture: called while an ensemble is initialised); 0 when the device refuses
// the opt-in or cannot hold one block (its launches are one block per work item).
static int ens_hllc_wide_grid() {
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaFuncSetAttribute(ens_hllc_wide_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kEnsWideSmem) !=
          cudaSuccess ||
      cudaFuncSetAttribute(ens_hllc_wide_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kEnsWideSmem) !=
          cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ens_hllc_wide_kernel<2>, kEnsWideNT, kEnsWideSmem) !=
          cudaSuccess ||
      per_sm < 1) {
    cudaGetLastError();  // the refusal is reported by the caller, not left to a later launch
    return 0;
  }
  return per_sm * (sms > 0 ? sms : 1);
}

// Ensemble HLLC variants: 0 = 32 x 16 tiles, 1 = 32 x 8 (256 threads), 2 = 32 x 32.
void hllc_variant_tile(int variant, int* tx, int* ty) {
  *tx = 32;
  *ty = variant == 1 ? 8 : (variant == 2 ? 32 : 16);
}

int ens_hllc_grid_size(int variant) {
  if (variant == 2) return ens_hllc_wide_grid();
  return variant == 1 ? ens_hllc_grid<32, 8, 256>() : ens_hllc_grid<32, 16, 256>();
}

cudaError_t ens_hllc_launch(int variant, int grid, int stage, const HllcParams* P, const int2* map, long long total,
                            cudaStream_t s) {
  if (total <= 0) return cudaSuccess;
  const int g = (int)(total < grid ? total : grid);
  if (variant == 2) {  // one block per work item
    if (stage == 1)
      ens_hllc_wide_kernel<1><<<(unsigned)total, kEnsWideNT, kEnsWideSmem, s>>>(P, map);
    else
      ens_hllc_wide_kernel<2><<<(unsigned)total, kEnsWideNT, kEnsWideSmem, s>>>(P, map);
  } else if (variant == 1) {
    if (stage == 1)
      ens_hllc_kernel<32, 8, 256, 1><<<g, 256, 0, s>>>(P, map, total);
    else
      ens_hllc_kernel<32, 8, 256, 2><<<g, 256, 0, s>>>(P, map, total);
  } else {
    if (stage == 1)
      ens_hllc_kernel<32, 16, 256, 1><<<g, 256, 0, s>>>(P, map, total);
    else
      ens_hllc_kernel<32, 16, 256, 2><<<g, 256, 0, s>>>(P, map, total);
  }
  return cudaGetLastError();
}
#endif  // !RB_FAST_MATH: the ensembles run the exact arithmetic only

RB_ARITH_END
}  // namespace rb
