// li_step.cu -- the fused local-inertial step (Bates et al. 2010).
//
// One launch performs what the reference launches as ~12 kernels per step
// (solver/core/local_inertial.py:547-727):
//   compute_eta (:61) -> update_qx/update_qy (:72/:102, friction.py:18) ->
//   apply_closed_bc (boundaries.py:237) -> compute_outflow_beta (:197) ->
//   limit_qx/limit_qy (:242/:254) -> accumulate_qs_x/y (sediment.py:218/:247) ->
//   update_h (:132) -> add_uniform_rain_c / add_rain_field_c (sources.py:85/:104)
//   or apply_rain_field (:154) -> apply_infiltration (:170) ->
//   apply_open_outflow (boundaries.py:321).
//
// Tiling. A CTA owns a TX x TY tile of cells. The donor limiter makes a cell's new
// depth depend on the limited fluxes of its four faces, which depend on the beta of
// the neighbouring cells, which depend on *their* four unlimited faces: a halo of 2
// cells of (h, z, n) is staged in shared memory, the unlimited faces of the tile
// and a 1-cell ring are computed there (redundantly with the neighbouring CTAs),
// then beta on the tile plus ring, then the limited faces of the tile, then the
// cell updates. Each output is written by exactly one CTA. Because neighbours read
// the old h, qx, qy while this CTA writes new ones, the step reads buffer [cur]
// and writes buffer [cur ^ 1].
//
// Sub-grid channels (solver/core/channels.py, local_inertial.py:275-500) are a
// second instantiation (CH = true): eta through the storage curve, each face a
// floodplain plus a channel component (both double buffered like qx / qy), both
// scaled by the total flux's donor beta, the two-component bedload capacity, and
// the water column instead of h for the next dt. The unarmed instantiation does
// none of it.
//
// Per-cell HBM traffic (compulsory): read h, z, n, qx, qy, write h, qx, qy (32 B),
// + h_comp read/write (8 B) when compensated rain is armed, + rain field / infil
// reads (4 B each), + d50 and the four transport accumulators (36 B) when
// morphology is armed. Infiltration and open-edge losses go to one float64 ledger
// slot per tile instead of a per-cell float64 field.
#include <atomic>
#include <cfloat>
#include <type_traits>

#include "rb_common.cuh"
#include "rb_kernels.h"

namespace rb {
RB_ARITH_BEGIN

#if defined(RB_FAST_MATH)
constexpr bool kEarlySedLoads = true;
#else
constexpr bool kEarlySedLoads = false;
#endif

// sediment.py:161-207 kinematic_shear / shields_number / mpm_capacity / face_capacity.
__device__ __forceinline__ float face_capacity(float q, float h, float radius, float n, float d50) {
  if (h < kHDry || d50 <= 0.0f || q == 0.0f) return 0.0f;
  const float tau = div_pos(kG * n * n * q * q, h * h * pow13(radius));
  const float theta = div_pos(tau, 1.65f * kG * d50);
  float qs;
  if (theta <= 0.047f) {
    qs = 0.0f;
  } else {
    const float excess = theta - 0.047f;
    qs = 8.0f * pow15(excess) * sqrtf(1.65f * kG * d50 * d50 * d50);
  }
  return q < 0.0f ? -qs : qs;
}

// boundaries.py:244-256 _drain
__device__ __forceinline__ float drain(float h_edge, float q_out, float dxdt) {
  float removed = dxdt * q_out;
  if (removed > h_edge) removed = h_edge;
  if (removed < 0.0f) removed = 0.0f;
  return h_edge - removed;
}

// local_inertial.py:294-320 _channel_flux with channels.py:120-135 and the
// hydraulic-radius Manning denominator of friction.py:35-58: the channel component
// of a face, per unit channel width.
__device__ __forceinline__ float channel_flux(float q_prev, float eta_max, float slope, float w_face, float z_bank,
                                              float z_ch, float n_ch, float dt) {
  if (w_face <= 0.0f) return 0.0f;
  const float h_ch = rmin(eta_max, z_bank) - z_ch;
  if (h_ch < kHDry) return 0.0f;
  const float radius = div_pos(w_face * h_ch, w_face + 2.0f * h_ch);
  const float num = q_prev - kG * h_ch * dt * slope;
  // zero dividends as in manning_divide: a zero friction numerator makes den exactly 1
  const float f = kG * dt * n_ch * n_ch * fabsf(q_prev);
  if (f == 0.0f) return num;
  const float den = 1.0f + f / (h_ch * pow43(radius));
  return div_pos(num, den);
}

// local_inertial.py:323-336 _floodplain_flux: the plain face update above the banks.
__device__ __forceinline__ float floodplain_flux(float q_prev, float eta_max, float slope, float z_bank, float n_fp,
                                                 float dt) {
  const float h_fp = eta_max - z_bank;
  if (h_fp < kHDry) return 0.0f;
  const float num = q_prev - kG * h_fp * dt * slope;
  return manning_divide(num, q_prev, h_fp, n_fp, kG, dt);
}

// sediment.py:276-305 _combined_capacity: bedload per unit cell width of a
// two-component face.
__device__ __forceinline__ float combined_capacity(float q_ch, float q_fp, float eta_max, float z_bank, float z_ch,
                                                   float w_face, float n_fp, float n_ch, float d50, float dx) {
  const float h_fp = eta_max - z_bank;
  const float qs_fp = face_capacity(q_fp, h_fp, h_fp, n_fp, d50);
  float qs_ch = 0.0f;
  if (w_face > 0.0f) {
    const float h_ch = rmin(eta_max, z_bank) - z_ch;
    if (h_ch >= kHDry) qs_ch = face_capacity(q_ch, h_ch, w_face * h_ch / (w_face + 2.0f * h_ch), n_ch, d50);
  }
  const float frac = div_pos(w_face, dx);
  return qs_fp * (1.0f - frac) + qs_ch * frac;
}

template <int TX, int TY>
struct LiGeom {
  static constexpr int RW = TX + 4, RH = TY + 4;  // cells: cols x0-2 .. x0+TX+1, rows y0-2 .. y0+TY+1
  static constexpr int XW = TX + 3, XH = TY + 2;  // x-faces: cols x0-1 .. x0+TX+1, rows y0-1 .. y0+TY
  static constexpr int YW = TX + 2, YH = TY + 3;  // y-faces: cols x0-1 .. x0+TX,   rows y0-1 .. y0+TY+1
  static constexpr int BW = TX + 2, BH = TY + 2;  // beta:    cols x0-1 .. x0+TX,   rows y0-1 .. y0+TY
};

// Channel geometry of the halo and the two face components (sub-grid channels only).
template <int TX, int TY, bool CH>
struct LiChanSmem {};
template <int TX, int TY>
struct LiChanSmem<TX, TY, true> : LiGeom<TX, TY> {
  using G = LiGeom<TX, TY>;
  float w[G::RH][G::RW], d[G::RH][G::RW], cn[G::RH][G::RW];
  float qxc[G::XH][G::XW], qxf[G::XH][G::XW], qyc[G::YH][G::YW], qyf[G::YH][G::YW];
};

template <int TX, int TY, bool CH = false>
struct LiSmem : LiGeom<TX, TY> {
  using G = LiGeom<TX, TY>;
  float h[G::RH][G::RW], z[G::RH][G::RW], n[G::RH][G::RW], eta[G::RH][G::RW];
  float qx[G::XH][G::XW], qy[G::YH][G::YW], beta[G::BH][G::BW];
  double red[16];
  float redf[16];
  LiChanSmem<TX, TY, CH> ch;
};

// A tile whose staged region (the tile and a 2-cell halo) lies inside the domain:
// all its faces are inner faces and no cell of it is on a domain edge.
template <int TX, int TY>
__device__ __forceinline__ bool li_deep_interior(int x0, int y0, int ny, int nx) {
  return x0 >= 2 && y0 >= 2 && x0 + TX + 2 <= nx && y0 + TY + 2 <= ny;
}

// One CTA-wide tile of the step: tile (bx, by) of domain p, ledger slot `slot`.
// Called by every thread of the block; returns uniformly. IN is the instantiation
// for a tile li_deep_interior admits, without bounds checks and edge cases (the
// same bits). SED says whether the bedload integral is armed: 0 no, 1 yes, 2 read
// from p.d50 at run time (an ensemble's domains differ); the single-domain kernel
// is instantiated for 0 and 1, so a run without bedload carries none of its code.
template <int TX, int TY, int NT, bool CH = false, bool IN = false, int SED = 2>
__device__ __forceinline__ void li_tile(const LiParams& p, int bx, int by, size_t slot, LiSmem<TX, TY, CH>& S) {
  static_assert(NT / 32 <= 16, "reduction scratch sized for <= 16 warps");
  const bool has_sed = SED == 2 ? p.d50 != nullptr : SED == 1;
  using SM = LiSmem<TX, TY, CH>;
  constexpr int RW = SM::RW, RH = SM::RH, XW = SM::XW, XH = SM::XH, YW = SM::YW, YH = SM::YH;
  constexpr int BW = SM::BW, BH = SM::BH;
  auto& s_h = S.h;
  auto& s_z = S.z;
  auto& s_n = S.n;
  auto& s_eta = S.eta;
  auto& s_qx = S.qx;
  auto& s_qy = S.qy;
  auto& s_beta = S.beta;
  double* s_red = S.red;
  float* s_redf = S.redf;

  const int ny = p.ny, nx = p.nx;
  const int x0 = bx * TX, y0 = by * TY;
  int cur = p.cur, limit = p.limit;
  float dt = p.dt32, rain_cont = p.rain_cont, rain32 = p.rain32, scale32 = p.scale32, dxdt = p.dxdt;
  if (p.clk != nullptr) {  // device-resident clock: this step's dt and forcing
    const DevClock* c = p.clk;
    if (!c->active) return;
    cur = c->cur;
    limit = c->limit;
    dt = c->dt32;
    rain32 = c->rain32;
    rain_cont = p.h_comp != nullptr ? 0.0f : rain32;
    scale32 = c->scale32;
    dxdt = c->dxdt32;
  }
  const float* __restrict__ h_in = p.hb[cur];
  const float* __restrict__ qx_in = p.qxb[cur];
  const float* __restrict__ qy_in = p.qyb[cur];
  float* __restrict__ h_out = p.hb[cur ^ 1];
  float* __restrict__ qx_out = p.qxb[cur ^ 1];
  float* __restrict__ qy_out = p.qyb[cur ^ 1];
  const float dx = p.dx32;
  const float dtdx = dt / dx;

  // 1. stage h, z, n (halo 2) and eta = h + z (local_inertial.py:61-69), and the
  //    previous discharge of every face the tile updates. Each thread issues all of
  //    its loads before it stores any, so their latency overlaps.
  {
    constexpr int NL = (RH * RW + NT - 1) / NT;
    float lh[NL], lz[NL], ln[NL], lw[NL], ld[NL], lc[NL];
#pragma unroll
    for (int i = 0; i < NL; i++) {
      const int k = threadIdx.x + i * NT;
      const int r = k / RW, c = k - r * RW;
      const int gi = y0 - 2 + r, gj = x0 - 2 + c;
      lh[i] = lz[i] = ln[i] = lw[i] = ld[i] = lc[i] = 0.0f;
      if (k < RH * RW && (IN || (gi >= 0 && gi < ny && gj >= 0 && gj < nx))) {
        const size_t id = (size_t)gi * nx + gj;
        lh[i] = h_in[id];
        lz[i] = p.z[id];
        ln[i] = p.n[id];
        if constexpr (CH) {
          lw[i] = p.cw[id];
          ld[i] = p.cd[id];
          lc[i] = p.cn[id];
        }
      }
    }
#pragma unroll
    for (int i = 0; i < NL; i++) {
      const int k = threadIdx.x + i * NT;
      if (k >= RH * RW) continue;
      const int r = k / RW, c = k - r * RW;
      s_h[r][c] = lh[i];
      s_z[r][c] = lz[i];
      s_n[r][c] = ln[i];
      if constexpr (CH) {  // local_inertial.py:278-291 compute_eta_channels
        S.ch.w[r][c] = lw[i];
        S.ch.d[r][c] = ld[i];
        S.ch.cn[r][c] = lc[i];
        s_eta[r][c] = eta_subgrid(lh[i], lz[i], lw[i], ld[i], dx);
      } else {
        s_eta[r][c] = lh[i] + lz[i];
      }
    }
    // previous face discharges (interior faces only; the rest are never read)
    constexpr int NX_ = (XH * XW + NT - 1) / NT, NY_ = (YH * YW + NT - 1) / NT;
    float fq[NX_], fc[NX_], ff[NX_], gq[NY_], gc[NY_], gf[NY_];
#pragma unroll
    for (int i = 0; i < NX_; i++) {
      const int k = threadIdx.x + i * NT;
      const int a = k / XW, b = k - a * XW;
      const int gi = y0 - 1 + a, gj = x0 - 1 + b;
      fq[i] = fc[i] = ff[i] = 0.0f;
      if (k < XH * XW && (IN || (gi >= 0 && gi < ny && gj >= 1 && gj <= nx - 1))) {
        const size_t fid = (size_t)gi * (nx + 1) + gj;
        if constexpr (CH) {
          fc[i] = p.qxcb[cur][fid];
          ff[i] = p.qxfb[cur][fid];
        } else {
          fq[i] = qx_in[fid];
        }
      }
    }
#pragma unroll
    for (int i = 0; i < NY_; i++) {
      const int k = threadIdx.x + i * NT;
      const int a = k / YW, b = k - a * YW;
      const int gi = y0 - 1 + a, gj = x0 - 1 + b;
      gq[i] = gc[i] = gf[i] = 0.0f;
      if (k < YH * YW && (IN || (gi >= 1 && gi <= ny - 1 && gj >= 0 && gj < nx))) {
        const size_t fid = (size_t)gi * nx + gj;
        if constexpr (CH) {
          gc[i] = p.qycb[cur][fid];
          gf[i] = p.qyfb[cur][fid];
        } else {
          gq[i] = qy_in[fid];
        }
      }
    }
#pragma unroll
    for (int i = 0; i < NX_; i++) {
      const int k = threadIdx.x + i * NT;
      if (k >= XH * XW) continue;
      const int a = k / XW, b = k - a * XW;
      if constexpr (CH) {
        S.ch.qxc[a][b] = fc[i];
        S.ch.qxf[a][b] = ff[i];
      } else {
        s_qx[a][b] = fq[i];
      }
    }
#pragma unroll
    for (int i = 0; i < NY_; i++) {
      const int k = threadIdx.x + i * NT;
      if (k >= YH * YW) continue;
      const int a = k / YW, b = k - a * YW;
      if constexpr (CH) {
        S.ch.qyc[a][b] = gc[i];
        S.ch.qyf[a][b] = gf[i];
      } else {
        s_qy[a][b] = gq[i];
      }
    }
  }
  __syncthreads();

  // 2. unlimited face updates (local_inertial.py:72-129); boundary faces stay 0,
  //    which is the closed boundary (boundaries.py:223-241).
  // x- and y-faces share one loop, so the last pass over the block is partly
  // filled once, not twice.
  constexpr int NXF = XH * XW, NF = XH * XW + YH * YW;
  // A tile whose faces (and the ring's) are all inner faces of the domain runs an
  // instantiation without the bounds checks.
  auto face_loop = [&](auto inner_tag) {
    constexpr bool INNER = decltype(inner_tag)::value;
    for (int kk = threadIdx.x; kk < NF; kk += NT) {
      if (kk < NXF) {
        const int k = kk;
        const int a = k / XW, b = k - a * XW;
        const int gi = y0 - 1 + a, gj = x0 - 1 + b;
        float q = 0.0f;
        if constexpr (!CH) {
          if (INNER || (gi >= 0 && gi < ny && gj >= 1 && gj <= nx - 1)) {
            const float eta_l = s_eta[a + 1][b], eta_r = s_eta[a + 1][b + 1];
            const float h_flow = rmax(eta_l, eta_r) - rmax(s_z[a + 1][b], s_z[a + 1][b + 1]);
            if (!(h_flow < kHDry)) {
              const float qo = s_qx[a][b];  // previous discharge, staged above
              const float n_face = 0.5f * (s_n[a + 1][b] + s_n[a + 1][b + 1]);
              const float slope = div_pos(eta_r - eta_l, dx);
              const float num = qo - kG * h_flow * dt * slope;
              q = manning_divide(num, qo, h_flow, n_face, kG, dt);
            }
          }
        } else {  // local_inertial.py:338-384 update_qx_channels
          float qc = 0.0f, qf = 0.0f;
          if (INNER || (gi >= 0 && gi < ny && gj >= 1 && gj <= nx - 1)) {
            const int r = a + 1, cl = b, cr = b + 1;
            const float eta_l = s_eta[r][cl], eta_r = s_eta[r][cr];
            const float eta_max = rmax(eta_l, eta_r);
            const float slope = div_pos(eta_r - eta_l, dx);
            const float z_bank = rmax(s_z[r][cl], s_z[r][cr]);
            qf = floodplain_flux(S.ch.qxf[a][b], eta_max, slope, z_bank, 0.5f * (s_n[r][cl] + s_n[r][cr]), dt);
            const float w_face = rmin(S.ch.w[r][cl], S.ch.w[r][cr]);
            const float z_ch = rmax(s_z[r][cl] - S.ch.d[r][cl], s_z[r][cr] - S.ch.d[r][cr]);
            qc = channel_flux(S.ch.qxc[a][b], eta_max, slope, w_face, z_bank, z_ch,
                              0.5f * (S.ch.cn[r][cl] + S.ch.cn[r][cr]), dt);
            const float frac = div_pos(w_face, dx);
            q = qf * (1.0f - frac) + qc * frac;
          }
          S.ch.qxc[a][b] = qc;
          S.ch.qxf[a][b] = qf;
        }
        s_qx[a][b] = q;
      } else {
        const int k = kk - NXF;
        const int a = k / YW, b = k - a * YW;
        const int gi = y0 - 1 + a, gj = x0 - 1 + b;
        float q = 0.0f;
        if constexpr (!CH) {
          if (INNER || (gi >= 1 && gi <= ny - 1 && gj >= 0 && gj < nx)) {
            const float eta_t = s_eta[a][b + 1], eta_b = s_eta[a + 1][b + 1];
            const float h_flow = rmax(eta_t, eta_b) - rmax(s_z[a][b + 1], s_z[a + 1][b + 1]);
            if (!(h_flow < kHDry)) {
              const float qo = s_qy[a][b];
              const float n_face = 0.5f * (s_n[a][b + 1] + s_n[a + 1][b + 1]);
              const float slope = div_pos(eta_b - eta_t, dx);
              const float num = qo - kG * h_flow * dt * slope;
              q = manning_divide(num, qo, h_flow, n_face, kG, dt);
            }
          }
        } else {  // local_inertial.py:387-427 update_qy_channels
          float qc = 0.0f, qf = 0.0f;
          if (INNER || (gi >= 1 && gi <= ny - 1 && gj >= 0 && gj < nx)) {
            const int c = b + 1, rt = a, rb = a + 1;
            const float eta_t = s_eta[rt][c], eta_b = s_eta[rb][c];
            const float eta_max = rmax(eta_t, eta_b);
            const float slope = div_pos(eta_b - eta_t, dx);
            const float z_bank = rmax(s_z[rt][c], s_z[rb][c]);
            qf = floodplain_flux(S.ch.qyf[a][b], eta_max, slope, z_bank, 0.5f * (s_n[rt][c] + s_n[rb][c]), dt);
            const float w_face = rmin(S.ch.w[rt][c], S.ch.w[rb][c]);
            const float z_ch = rmax(s_z[rt][c] - S.ch.d[rt][c], s_z[rb][c] - S.ch.d[rb][c]);
            qc = channel_flux(S.ch.qyc[a][b], eta_max, slope, w_face, z_bank, z_ch,
                              0.5f * (S.ch.cn[rt][c] + S.ch.cn[rb][c]), dt);
            const float frac = div_pos(w_face, dx);
            q = qf * (1.0f - frac) + qc * frac;
          }
          S.ch.qyc[a][b] = qc;
          S.ch.qyf[a][b] = qf;
        }
        s_qy[a][b] = q;
      }
    }
  };
  // x-faces span columns x0-1 .. x0+TX+1 and rows y0-1 .. y0+TY, y-faces columns
  // x0-1 .. x0+TX and rows y0-1 .. y0+TY+1: all inner faces when these hold
  if (IN || li_deep_interior<TX, TY>(x0, y0, ny, nx))
    face_loop(std::true_type{});
  else
    face_loop(std::false_type{});
  __syncthreads();

  // 3. donor-cell beta on the tile plus a 1-cell ring (local_inertial.py:197-239).
  if (limit) {
    for (int k = threadIdx.x; k < BH * BW; k += NT) {
      const int a = k / BW, b = k - a * BW;
      float q_out = 0.0f;
      const float ql = s_qx[a][b];
      if (ql < 0.0f) q_out = q_out - ql;
      const float qr = s_qx[a][b + 1];
      if (qr > 0.0f) q_out = q_out + qr;
      const float qt = s_qy[a][b];
      if (qt < 0.0f) q_out = q_out - qt;
      const float qb = s_qy[a + 1][b];
      if (qb > 0.0f) q_out = q_out + qb;
      const float out_depth = dtdx * q_out;
      const bool out = out_depth > 0.0f;
      const float ratio = div_if(out, s_h[a + 1][b + 1], out_depth);
      s_beta[a][b] = out ? rclamp(ratio, 0.0f, 1.0f) : 1.0f;
    }
    __syncthreads();
  }

  // 4. scale each interior face of the tile by its donor's beta (:242-263), write
  //    the tile's faces and integrate bedload on them (sediment.py:218-273). x- and
  //    y-faces in one loop, as in the face update. The limited discharge goes back
  //    to shared memory for the continuity below; the east (south) face of a tile
  //    is limited here but written by the next tile, except at the domain's edge.
  constexpr int NXW = TY * (TX + 1), NW = TY * (TX + 1) + (TY + 1) * TX;
  for (int kk = threadIdx.x; kk < NW; kk += NT) {
    if (kk < NXW) {
      const int k = kk;
      const int a = 1 + k / (TX + 1), b = 1 + (k - (a - 1) * (TX + 1));
      const int gi = y0 - 1 + a, gj = x0 - 1 + b;
      if (!IN && (gi >= ny || gj > nx)) continue;
      float q = s_qx[a][b];
      if (limit && (IN || (gj >= 1 && gj <= nx - 1))) {
        if constexpr (!CH) {
          if (q > 0.0f)
            q = q * s_beta[a][b - 1];
          else if (q < 0.0f)
            q = q * s_beta[a][b];
        } else if (!(q == 0.0f)) {  // local_inertial.py:430-452 limit_qx_channels
          const float bb = q < 0.0f ? s_beta[a][b] : s_beta[a][b - 1];
          q = q * bb;
          S.ch.qxc[a][b] = S.ch.qxc[a][b] * bb;
          S.ch.qxf[a][b] = S.ch.qxf[a][b] * bb;
        }
        s_qx[a][b] = q;
      }
      if (b == TX + 1 && (IN || gj != nx)) continue;
      const size_t fid = (size_t)gi * (nx + 1) + gj;
      // the fast build loads the face's bedload operands before the discharge store
      // (which the compiler may not move them past), so their latency overlaps the
      // capacity arithmetic (-3 % on the 8192^2 reach; the exact build measured
      // +1.7 % with it and loads them at their use)
      const bool sed = !CH && has_sed && (IN || (gj >= 1 && gj <= nx - 1));
      float tot = 0.0f, comp = 0.0f, d50l = 0.0f, d50r = 0.0f;
      if constexpr (kEarlySedLoads) {
        if (sed) {
          const size_t cl = (size_t)gi * nx + gj - 1;
          tot = p.qs_int_x[fid];
          comp = p.qs_comp_x[fid];
          d50l = p.d50[cl];
          d50r = p.d50[cl + 1];
        }
      }
      qx_out[fid] = q;
      if constexpr (CH) {
        p.qxcb[cur ^ 1][fid] = S.ch.qxc[a][b];
        p.qxfb[cur ^ 1][fid] = S.ch.qxf[a][b];
        if (p.d50 != nullptr && gj >= 1 && gj <= nx - 1) {  // sediment.py:308-342
          const int r = a + 1, cl = b, cr = b + 1;
          const size_t ci = (size_t)gi * nx + gj - 1;
          const float qs = combined_capacity(
              S.ch.qxc[a][b], S.ch.qxf[a][b], rmax(s_eta[r][cl], s_eta[r][cr]), rmax(s_z[r][cl], s_z[r][cr]),
              rmax(s_z[r][cl] - S.ch.d[r][cl], s_z[r][cr] - S.ch.d[r][cr]), rmin(S.ch.w[r][cl], S.ch.w[r][cr]),
              0.5f * (s_n[r][cl] + s_n[r][cr]), 0.5f * (S.ch.cn[r][cl] + S.ch.cn[r][cr]),
              0.5f * (p.d50[ci] + p.d50[ci + 1]), dx);
          float tot = p.qs_int_x[fid], comp = p.qs_comp_x[fid];
          kahan_add(tot, comp, qs * dt);
          p.qs_int_x[fid] = tot;
          p.qs_comp_x[fid] = comp;
        }
      } else if (sed) {
        if constexpr (!kEarlySedLoads) {
          const size_t cl = (size_t)gi * nx + gj - 1;
          d50l = p.d50[cl];
          d50r = p.d50[cl + 1];
        }
        const float eta_max = rmax(s_eta[a + 1][b], s_eta[a + 1][b + 1]);
        const float z_bank = rmax(s_z[a + 1][b], s_z[a + 1][b + 1]);
        const float h_face = eta_max - z_bank;
        const float qs = face_capacity(q, h_face, h_face, 0.5f * (s_n[a + 1][b] + s_n[a + 1][b + 1]),
                                       0.5f * (d50l + d50r));
        if constexpr (!kEarlySedLoads) {
          tot = p.qs_int_x[fid];
          comp = p.qs_comp_x[fid];
        }
        kahan_add(tot, comp, qs * dt);
        p.qs_int_x[fid] = tot;
        p.qs_comp_x[fid] = comp;
      }
    } else {
      const int k = kk - NXW;
      const int a = 1 + k / TX, b = 1 + (k - (a - 1) * TX);
      const int gi = y0 - 1 + a, gj = x0 - 1 + b;
      if (!IN && (gj >= nx || gi > ny)) continue;
      float q = s_qy[a][b];
      if (limit && (IN || (gi >= 1 && gi <= ny - 1))) {
        if constexpr (!CH) {
          if (q > 0.0f)
            q = q * s_beta[a - 1][b];
          else if (q < 0.0f)
            q = q * s_beta[a][b];
        } else if (!(q == 0.0f)) {  // local_inertial.py:455-472 limit_qy_channels
          const float bb = q < 0.0f ? s_beta[a][b] : s_beta[a - 1][b];
          q = q * bb;
          S.ch.qyc[a][b] = S.ch.qyc[a][b] * bb;
          S.ch.qyf[a][b] = S.ch.qyf[a][b] * bb;
        }
        s_qy[a][b] = q;
      }
      if (a == TY + 1 && (IN || gi != ny)) continue;
      const size_t fid = (size_t)gi * nx + gj;
      const bool sed = !CH && has_sed && (IN || (gi >= 1 && gi <= ny - 1));
      float tot = 0.0f, comp = 0.0f, d50t = 0.0f, d50b = 0.0f;
      if constexpr (kEarlySedLoads) {
        if (sed) {
          tot = p.qs_int_y[fid];
          comp = p.qs_comp_y[fid];
          d50t = p.d50[fid - nx];
          d50b = p.d50[fid];
        }
      }
      qy_out[fid] = q;
      if constexpr (CH) {
        p.qycb[cur ^ 1][fid] = S.ch.qyc[a][b];
        p.qyfb[cur ^ 1][fid] = S.ch.qyf[a][b];
        if (p.d50 != nullptr && gi >= 1 && gi <= ny - 1) {  // sediment.py:345-377
          const int c = b + 1, rt = a, rb = a + 1;
          const float qs = combined_capacity(
              S.ch.qyc[a][b], S.ch.qyf[a][b], rmax(s_eta[rt][c], s_eta[rb][c]), rmax(s_z[rt][c], s_z[rb][c]),
              rmax(s_z[rt][c] - S.ch.d[rt][c], s_z[rb][c] - S.ch.d[rb][c]), rmin(S.ch.w[rt][c], S.ch.w[rb][c]),
              0.5f * (s_n[rt][c] + s_n[rb][c]), 0.5f * (S.ch.cn[rt][c] + S.ch.cn[rb][c]),
              0.5f * (p.d50[fid - nx] + p.d50[fid]), dx);
          float tot = p.qs_int_y[fid], comp = p.qs_comp_y[fid];
          kahan_add(tot, comp, qs * dt);
          p.qs_int_y[fid] = tot;
          p.qs_comp_y[fid] = comp;
        }
      } else if (sed) {
        if constexpr (!kEarlySedLoads) {
          d50t = p.d50[fid - nx];
          d50b = p.d50[fid];
        }
        const float eta_max = rmax(s_eta[a][b + 1], s_eta[a + 1][b + 1]);
        const float z_bank = rmax(s_z[a][b + 1], s_z[a + 1][b + 1]);
        const float h_face = eta_max - z_bank;
        const float qs = face_capacity(q, h_face, h_face, 0.5f * (s_n[a][b + 1] + s_n[a + 1][b + 1]),
                                       0.5f * (d50t + d50b));
        if constexpr (!kEarlySedLoads) {
          tot = p.qs_int_y[fid];
          comp = p.qs_comp_y[fid];
        }
        kahan_add(tot, comp, qs * dt);
        p.qs_int_y[fid] = tot;
        p.qs_comp_y[fid] = comp;
      }
    }
  }

  __syncthreads();

  // 5. continuity, areal sources, infiltration, open-edge sinks, per tile cell.
  const float rain_dt = rain_cont * dt;
  double loss = 0.0;
  float hmax = 0.0f;
  bool bad = false;
  // The per-cell global inputs of this thread's cells are loaded first, all of them,
  // so their latency overlaps instead of stalling each cell's update in turn.
  constexpr int NC = (TX * TY + NT - 1) / NT;
  float g_comp[NC], g_rain[NC], g_inf[NC];
#pragma unroll
  for (int i = 0; i < NC; i++) {
    const int k = threadIdx.x + i * NT;
    const int r = k / TX, c = k - r * TX;
    const int gi = y0 + r, gj = x0 + c;
    g_comp[i] = g_rain[i] = g_inf[i] = 0.0f;
    if (k < TX * TY && (IN || (gi < ny && gj < nx))) {
      const size_t id = (size_t)gi * nx + gj;
      if (p.h_comp != nullptr) g_comp[i] = p.h_comp[id];
      if (p.rain_field != nullptr) g_rain[i] = p.rain_field[id];
      if (p.infil != nullptr) g_inf[i] = p.infil[id];
    }
  }
#pragma unroll
  for (int i = 0; i < NC; i++) {
    const int k = threadIdx.x + i * NT;
    const int r = k / TX, c = k - r * TX;
    const int gi = y0 + r, gj = x0 + c;
    if (k >= TX * TY || (!IN && (gi >= ny || gj >= nx))) continue;
    const size_t id = (size_t)gi * nx + gj;
    const float qxl = s_qx[r + 1][c + 1], qxr = s_qx[r + 1][c + 2];
    const float qyt = s_qy[r + 1][c + 1], qyb = s_qy[r + 2][c + 1];
    const float net = qxl - qxr + qyt - qyb;
    float h = s_h[r + 2][c + 2] + dtdx * net + rain_dt;  // local_inertial.py:150-151
    if (p.h_comp != nullptr) {
      float comp = g_comp[i];
      if (p.rain_field == nullptr)
        kahan_add(h, comp, rain32 * dt);  // sources.py:85-101
      else
        kahan_add(h, comp, g_rain[i] * scale32 * dt);  // sources.py:104-121
      p.h_comp[id] = comp;
    } else if (p.rain_field != nullptr) {
      h = h + g_rain[i] * scale32 * dt;  // local_inertial.py:154-167
    }
    if (p.infil != nullptr) {  // local_inertial.py:170-194
      const float avail = h;
      float inf = g_inf[i] * dt;
      if (inf > avail) inf = avail;
      if (inf < 0.0f) inf = 0.0f;
      h = avail - inf;
      loss += (double)avail - (double)h;
    }
    // boundaries.py:259-318, launched west, east, north, south (no interior tile
    // has a cell on an edge).
    if (!IN && p.bc[RB_EDGE_WEST] == RB_BC_OPEN && nx > 1 && gj == 0) {
      const float avail = h;
      h = drain(avail, rmax(-qxr, 0.0f), dxdt);
      loss += (double)avail - (double)h;
    }
    if (!IN && p.bc[RB_EDGE_EAST] == RB_BC_OPEN && nx > 1 && gj == nx - 1) {
      const float avail = h;
      h = drain(avail, rmax(qxl, 0.0f), dxdt);
      loss += (double)avail - (double)h;
    }
    if (!IN && p.bc[RB_EDGE_NORTH] == RB_BC_OPEN && ny > 1 && gi == 0) {
      const float avail = h;
      h = drain(avail, rmax(-qyb, 0.0f), dxdt);
      loss += (double)avail - (double)h;
    }
    if (!IN && p.bc[RB_EDGE_SOUTH] == RB_BC_OPEN && ny > 1 && gi == ny - 1) {
      const float avail = h;
      h = drain(avail, rmax(qyt, 0.0f), dxdt);
      loss += (double)avail - (double)h;
    }
    h_out[id] = h;
    if constexpr (CH) {  // local_inertial.py:475-489: the water column sets the next dt
      const float col = column_depth(h, S.ch.w[r + 2][c + 2], S.ch.d[r + 2][c + 2], dx);
      hmax = col > hmax ? col : hmax;
    } else {
      hmax = h > hmax ? h : hmax;
    }
    bad |= !(fabsf(h) <= FLT_MAX);
  }

  // An interior tile banks nothing but infiltration (no cell of it drains through an
  // edge), so without infiltration its loss is 0 and its slot, zero from the start,
  // stays exactly 0: the block sum is skipped.
  if (p.ledger != nullptr && (!IN || p.infil != nullptr)) {
    const double s = block_sum<NT>(loss, s_red);
    if (threadIdx.x == 0) ledger_add(p.ledger + 2 * slot, s);
  }
  if (p.hmax_key != nullptr) block_max_to<NT>(hmax, p.hmax_key, s_redf);
  if (bad) flag_error(p.err, RB_DEVERR_NONFINITE);
  __syncthreads();  // the shared tile is reused by the caller's next tile
}

// The single-domain step kernel. MINB is __launch_bounds__' resident-block hint (it
// caps registers at 65536 / (MINB * NT)).
template <int TX, int TY, int NT, bool CH, int MINB, int SED>
__global__ void __launch_bounds__(NT, MINB) li_step_kernel(const LiParams p) {
  __shared__ LiSmem<TX, TY, CH> S;
  pdl_enter();
  const size_t slot = (size_t)blockIdx.y * gridDim.x + blockIdx.x;
  if (li_deep_interior<TX, TY>(blockIdx.x * TX, blockIdx.y * TY, p.ny, p.nx))
    li_tile<TX, TY, NT, CH, true, SED>(p, blockIdx.x, blockIdx.y, slot, S);
  else
    li_tile<TX, TY, NT, CH, false, SED>(p, blockIdx.x, blockIdx.y, slot, S);
}

// Sub-grid channel states keep the run-time bedload switch (one instantiation).
template <int TX, int TY, int NT, bool CH, int MINB>
static cudaError_t launch_li(const LiParams& p, cudaStream_t s) {
  const dim3 grid((p.nx + TX - 1) / TX, (p.ny + TY - 1) / TY);
  if constexpr (CH) return launch_chain(li_step_kernel<TX, TY, NT, CH, MINB, 2>, grid, dim3(NT), 0, s, p);
  return p.d50 != nullptr ? launch_chain(li_step_kernel<TX, TY, NT, CH, MINB, 1>, grid, dim3(NT), 0, s, p)
                          : launch_chain(li_step_kernel<TX, TY, NT, CH, MINB, 0>, grid, dim3(NT), 0, s, p);
}

// Tile variants of the single-domain step (sub-grid channels always use 32 x 16);
// all compute the same bits. The default is the fastest measured on B200 for the
// 2048^2 and 4096^2 rain-on-grid steps (ms per 2048^2 step: 0.158, 0.142, 0.145,
// 0.208, 0.149 for variants 0..4).
struct LiKernelVariant {
  int tx, ty, nt;
};
static const LiKernelVariant kLiVariants[] = {{32, 16, 256}, {32, 32, 512}, {64, 16, 512}, {32, 8, 256}, {32, 16, 256}};
constexpr int kNumLiVariants = (int)(sizeof(kLiVariants) / sizeof(kLiVariants[0]));
constexpr int kDefaultLiVariant = 1;
#if !defined(RB_FAST_MATH)
static std::atomic<int> g_li_variant{kDefaultLiVariant};

int li_kernel_variant_count() { return kNumLiVariants; }
bool li_set_kernel_variant(int v) {
  if (v < 0 || v >= kNumLiVariants) return false;
  g_li_variant.store(v);
  return true;
}

int li_current_variant() { return g_li_variant.load(); }

cudaError_t li_step_launch(const LiParams& p, cudaStream_t s) {
  if (arith_mode() == RB_ARITH_FAST) return fast::li_step_launch_variant(p, g_li_variant.load(), s);
  return li_step_launch_variant(p, g_li_variant.load(), s);
}
#endif  // !RB_FAST_MATH

cudaError_t li_step_launch_variant(const LiParams& p, int variant, cudaStream_t s) {
  if (p.cw != nullptr) return launch_li<32, 16, 256, true, 1>(p, s);
  switch (variant) {
    case 0: return launch_li<32, 16, 256, false, 1>(p, s);
    case 2: return launch_li<64, 16, 512, false, 3>(p, s);
    case 3: return launch_li<32, 8, 256, false, 1>(p, s);
    case 4: return launch_li<32, 16, 256, false, 5>(p, s);  // at most 48 registers
    default: return launch_li<32, 32, 512, false, 3>(p, s);
  }
}

#if !defined(RB_FAST_MATH)
// Ensemble: a persistent grid walks the (domain, local tile) work-list of every
// local-inertial domain; a tile of a domain whose clock is not active returns at
// its first instruction. Each domain's tiles, ledger slots and clock are its own,
// so a domain's result does not depend on what else is in the batch. Three
// resident 512-thread blocks (six of 256) per SM measured fastest for 16 domains of
// 512 x 512 rain-on-grid (21.6 Gcell-updates/s on 32 x 32 tiles against 21.1 with
// two blocks), despite a few spilled registers.
template <int TX, int TY, int NT>
__global__ void __launch_bounds__(NT, NT >= 512 ? 3 : 6) ens_li_kernel(const LiParams* __restrict__ P,
                                                                   const int2* __restrict__ map, long long total) {
  __shared__ LiSmem<TX, TY> S;
  // The work item's domain parameters are staged in shared memory: read from there,
  // the pointers and scalars need not stay in registers through the tile.
  __shared__ __align__(16) LiParams sp;
  static_assert(sizeof(LiParams) % 4 == 0, "parameters copied as 32-bit words");
  constexpr int NW = (int)(sizeof(LiParams) / 4);
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
    const int bx = m.y % tiles_x, by = m.y / tiles_x;
    if (li_deep_interior<TX, TY>(bx * TX, by * TY, sp.ny, sp.nx))
      li_tile<TX, TY, NT, false, true>(sp, bx, by, (size_t)m.y, S);
    else
      li_tile<TX, TY, NT, false, false>(sp, bx, by, (size_t)m.y, S);
  }
}

// The 32 x 32 tile as a plain grid: one block per (domain, tile) work item, the
// domain's parameters read from global memory, three resident blocks of 512 threads
// per SM as in the single-domain step.
__global__ void __launch_bounds__(512, 3) ens_li_grid_kernel(const LiParams* __restrict__ P,
                                                             const int2* __restrict__ map) {
  __shared__ LiSmem<32, 32> S;
  const int2 m = map[blockIdx.x];
  const LiParams& p = P[m.x];
  const int tiles_x = (p.nx + 31) / 32;
  const int bx = m.y % tiles_x, by = m.y / tiles_x;
  if (li_deep_interior<32, 32>(bx * 32, by * 32, p.ny, p.nx))
    li_tile<32, 32, 512, false, true>(p, bx, by, (size_t)m.y, S);
  else
    li_tile<32, 32, 512, false, false>(p, bx, by, (size_t)m.y, S);
}

template <int TX, int TY, int NT>
static int ens_li_grid() {
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ens_li_kernel<TX, TY, NT>, NT, 0);
  return (per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1);
}

void li_variant_tile(int variant, int* tx, int* ty) {
  static const int T[4][2] = {{32, 16}, {32, 8}, {64, 8}, {32, 32}};
  const int v = variant < 0 || variant > 3 ? 0 : variant;
  *tx = T[v][0];
  *ty = T[v][1];
}

int ens_li_grid_size(int variant) {
  switch (variant) {
    case 1: return ens_li_grid<32, 8, 256>();
    case 2: return ens_li_grid<64, 8, 256>();
    case 3: return ens_li_grid<32, 32, 512>();
    default: return ens_li_grid<32, 16, 256>();
  }
}

cudaError_t ens_li_launch(int variant, int grid, const LiParams* P, const int2* map, long long total, cudaStream_t s) {
  if (total <= 0) return cudaSuccess;
  const int g = (int)(total < grid ? total : grid);
  switch (variant) {
    case 1: ens_li_kernel<32, 8, 256><<<g, 256, 0, s>>>(P, map, total); break;
    case 2: ens_li_kernel<64, 8, 256><<<g, 256, 0, s>>>(P, map, total); break;
    case 3: ens_li_grid_kernel<<<(unsigned)total, 512, 0, s>>>(P, map); break;  // one block per work item
    default: ens_li_kernel<32, 16, 256><<<g, 256, 0, s>>>(P, map, total); break;
  }
  return cudaGetLastError();
}
#endif  // !RB_FAST_MATH: the ensembles run the exact arithmetic only

RB_ARITH_END
}  // namespace rb
