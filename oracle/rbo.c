/*
 * rbo.c -- CPU oracle for the river-basin solver hot path.
 *
 * TEST INFRASTRUCTURE. This file restates, kernel by kernel and in the reference's
 * launch order, the arithmetic of the reference solver path (BoykoNeov/river-basin-sim):
 *   solver/core/local_inertial.py:50-544, friction.py:18-31, sources.py:66-121,
 *   boundaries.py:223-318, hllc.py:158-967, sediment.py:161-441,
 *   solver/processes/inflow.py:74-113, morphology.py:261-276.
 * It is the checker the CUDA path is compared against (by tests/, by
 * __graft_entry__.smoke and by bench.py's CPU-baseline and float64-error legs) and
 * is never linked into the product library.
 *
 * Arithmetic model: one IEEE rounding per operation in the reference's expression
 * order (build with -ffp-contract=off, no fast-math), `wp.max(a,b)` = a > b ? a : b,
 * `wp.min(a,b)` = a < b ? a : b, `wp.clamp(x,lo,hi)` = min(max(lo,x),hi). The four
 * fractional powers go through rbo_pow: mode 0 calls libm powf (how the
 * reference's CPU build evaluates `wp.pow`), mode 1 calls the deterministic
 * functions of include/rb_detmath.h that the CUDA kernels use.
 *
 * Built twice: REAL=float (the parity target) and REAL=double (the error
 * reference: the same kernels in float64), with RBO_SUFFIX naming the exports.
 *
 * Every kernel loops over its launch domain with one writer per output, so the
 * OpenMP row loops cannot change a result.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "rb_detmath.h"

#ifndef REAL
#define REAL float
#endif
#ifndef RBO_SUFFIX
#define RBO_SUFFIX _f32
#endif
#define RBO_CAT2(a, b) a##b
#define RBO_CAT(a, b) RBO_CAT2(a, b)
#define API(name) RBO_CAT(name, RBO_SUFFIX)

typedef REAL R;
#define C(x) ((R)(x))

static const R G = C(9.81);      /* solver/core/grid.py:43 */
static const R H_DRY = C(1.0e-3); /* solver/core/grid.py:48 */

/* Edge order of the boundary arrays: north, south, east, west (state.py:35). */
enum { EDGE_N = 0, EDGE_S = 1, EDGE_E = 2, EDGE_W = 3 };
enum { BC_CLOSED = 0, BC_OPEN = 1, BC_STAGE = 2 };

static int g_pow_mode = 0;
void API(rbo_set_pow_mode)(int mode) { g_pow_mode = mode; }

static inline R rmax(R a, R b) { return a > b ? a : b; }
static inline R rmin(R a, R b) { return a < b ? a : b; }
static inline R rclamp(R x, R lo, R hi) { return rmin(rmax(lo, x), hi); }
static inline R rabs(R x) { return (R)fabs((double)x); }
static inline R r_sqrt(R x) { return (R)(sizeof(R) == 4 ? (double)sqrtf((float)x) : sqrt((double)x)); }

/* which: 0 -> x^(7/3), 1 -> x^(1/3), 2 -> x^1.5, 3 -> x^(4/3), each with the
 * reference's float32 exponent. */
static inline R rbo_pow(R x, int which) {
  if (sizeof(R) == 8) {
    static const double P[4] = {7.0 / 3.0, 1.0 / 3.0, 1.5, 4.0 / 3.0};
    return (R)pow((double)x, P[which]);
  }
  if (g_pow_mode == 1) {
    switch (which) {
      case 0: return rb_pow73f((float)x);
      case 1: return rb_pow13f((float)x);
      case 2: return rb_pow15f((float)x);
      default: return rb_pow43f((float)x);
    }
  }
  static const float PF[4] = {7.0f / 3.0f, 1.0f / 3.0f, 1.5f, 4.0f / 3.0f};
  return powf((float)x, PF[which]);
}

/* The power functions themselves, for the accuracy tests. */
float API(rbo_pow)(float x, int which) { return (float)rbo_pow((R)x, which); }

#define IX(i, j) ((size_t)(i) * (size_t)nx + (size_t)(j))         /* cells (ny, nx)    */
#define FX(i, j) ((size_t)(i) * (size_t)(nx + 1) + (size_t)(j))   /* x-faces (ny, nx+1) */
#define FY(i, j) ((size_t)(i) * (size_t)nx + (size_t)(j))         /* y-faces (ny+1, nx) */

/* ========================================================================= */
/* Local-inertial kernels (solver/core/local_inertial.py)                     */
/* ========================================================================= */

/* friction.py:18-31 manning_denominator */
static inline R manning_denominator(R q_prev, R h_flow, R n, R g, R dt) {
  return C(1.0) + g * dt * n * n * rabs(q_prev) / rbo_pow(h_flow, 0);
}

/* local_inertial.py:61-69 compute_eta */
void API(rbo_compute_eta)(int ny, int nx, const R *h, const R *z, R *eta) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < ny; i++)
    for (int j = 0; j < nx; j++) eta[IX(i, j)] = h[IX(i, j)] + z[IX(i, j)];
}

/* local_inertial.py:72-99 update_qx (interior faces j = 1..nx-1) */
void API(rbo_update_qx)(int ny, int nx, R *qx, const R *eta, const R *z, const R *n, R dx, R dt, R g) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < ny; i++) {
    for (int j = 1; j <= nx - 1; j++) {
      const R eta_l = eta[IX(i, j - 1)], eta_r = eta[IX(i, j)];
      const R h_flow = rmax(eta_l, eta_r) - rmax(z[IX(i, j - 1)], z[IX(i, j)]); /* :50-58 */
      if (h_flow < H_DRY) {
        qx[FX(i, j)] = C(0.0);
        continue;
      }
      const R q = qx[FX(i, j)];
      const R n_face = C(0.5) * (n[IX(i, j - 1)] + n[IX(i, j)]);
      const R slope = (eta_r - eta_l) / dx;
      const R num = q - g * h_flow * dt * slope;
      const R den = manning_denominator(q, h_flow, n_face, g, dt);
      qx[FX(i, j)] = num / den;
    }
  }
}

/* local_inertial.py:102-129 update_qy (interior faces i = 1..ny-1) */
void API(rbo_update_qy)(int ny, int nx, R *qy, const R *eta, const R *z, const R *n, R dx, R dt, R g) {
#pragma omp parallel for schedule(static)
  for (int i = 1; i <= ny - 1; i++) {
    for (int j = 0; j < nx; j++) {
      const R eta_t = eta[IX(i - 1, j)], eta_b = eta[IX(i, j)];
      const R h_flow = rmax(eta_t, eta_b) - rmax(z[IX(i - 1, j)], z[IX(i, j)]);
      if (h_flow < H_DRY) {
        qy[FY(i, j)] = C(0.0);
        continue;
      }
      const R q = qy[FY(i, j)];
      const R n_face = C(0.5) * (n[IX(i - 1, j)] + n[IX(i, j)]);
      const R slope = (eta_b - eta_t) / dx;
      const R num = q - g * h_flow * dt * slope;
      const R den = manning_denominator(q, h_flow, n_face, g, dt);
      qy[FY(i, j)] = num / den;
    }
  }
}

/* boundaries.py:223-241 apply_closed_bc */
void API(rbo_zero_edges)(int ny, int nx, R *qx, R *qy) {
  for (int i = 0; i < ny; i++) {
    qx[FX(i, 0)] = C(0.0);
    qx[FX(i, nx)] = C(0.0);
  }
  for (int j = 0; j < nx; j++) {
    qy[FY(0, j)] = C(0.0);
    qy[FY(ny, j)] = C(0.0);
  }
}

/* local_inertial.py:197-239 compute_outflow_beta */
void API(rbo_outflow_beta)(int ny, int nx, const R *h, const R *qx, const R *qy, R dx, R dt, R *beta) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < ny; i++) {
    for (int j = 0; j < nx; j++) {
      R q_out = C(0.0);
      const R ql = qx[FX(i, j)];
      if (ql < C(0.0)) q_out = q_out - ql;
      const R qr = qx[FX(i, j + 1)];
      if (qr > C(0.0)) q_out = q_out + qr;
      const R qt = qy[FY(i, j)];
      if (qt < C(0.0)) q_out = q_out - qt;
      const R qb = qy[FY(i + 1, j)];
      if (qb > C(0.0)) q_out = q_out + qb;
      const R out_depth = dt / dx * q_out;
      if (out_depth > C(0.0))
        beta[IX(i, j)] = rclamp(h[IX(i, j)] / out_depth, C(0.0), C(1.0));
      else
        beta[IX(i, j)] = C(1.0);
    }
  }
}

/* local_inertial.py:242-263 limit_qx / limit_qy */
void API(rbo_limit_q)(int ny, int nx, R *qx, R *qy, const R *beta) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < ny; i++) {
    for (int j = 1; j <= nx - 1; j++) {
      const R q = qx[FX(i, j)];
      if (q > C(0.0))
        qx[FX(i, j)] = q * beta[IX(i, j - 1)];
      else if (q < C(0.0))
        qx[FX(i, j)] = q * beta[IX(i, j)];
    }
  }
#pragma omp parallel for schedule(static)
  for (int i = 1; i <= ny - 1; i++) {
    for (int j = 0; j < nx; j++) {
      const R q = qy[FY(i, j)];
      if (q > C(0.0))
        qy[FY(i, j)] = q * beta[IX(i - 1, j)];
      else if (q < C(0.0))
        qy[FY(i, j)] = q * beta[IX(i, j)];
    }
  }
}

/* local_inertial.py:132-151 update_h */
void API(rbo_update_h)(int ny, int nx, R *h, const R *qx, const R *qy, R dx, R dt, R rain) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < ny; i++) {
    for (int j = 0; j < nx; j++) {
      const R net = qx[FX(i, j)] - qx[FX(i, j + 1)] + qy[FY(i, j)] - qy[FY(i + 1, j)];
      h[IX(i, j)] = h[IX(i, j)] + dt / dx * net + rain * dt;
    }
  }
}

/* local_inertial.py:154-167 apply_rain_field (uncompensated) */
void API(rbo_rain_field_plain)(int ny, int nx, R *h, const R *rain, R dt, R scale) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < ny; i++)
    for (int j = 0; j < nx; j++) h[IX(i, j)] = h[IX(i, j)] + rain[IX(i, j)] * scale * dt;
}

/* local_inertial.py:170-194 apply_infiltration */
void API(rbo_infiltration)(int ny, int nx, R *h, const R *infil, double *loss_cum, R dt) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < ny; i++) {
    for (int j = 0; j < nx; j++) {
      const R avail = h[IX(i, j)];
      R inf = infil[IX(i, j)] * dt;
      if (inf > avail) inf = avail;
      if (inf < C(0.0)) inf = C(0.0);
      const R h_new = avail - inf;
      h[IX(i, j)] = h_new;
      loss_cum[IX(i, j)] = loss_cum[IX(i, j)] + ((double)avail - (double)h_new);
    }
  }
}

/* local_inertial.py:503-512 reduce_hmax, starting from the zeroed h_max (:527). */
R API(rbo_reduce_hmax)(int ny, int nx, const R *h) {
  R m = C(0.0);
  for (size_t k = 0; k < (size_t)ny * (size_t)nx; k++)
    if (h[k] > m) m = h[k];
  return m;
}

/* ========================================================================= */
/* Compensated areal sources (solver/core/sources.py)                        */
/* ========================================================================= */

/* sources.py:66-82 kahan_add */
static inline void kahan_add(R *total, R *comp, R inc) {
  const R y = inc - *comp;
  const R t = *total + y;
  *comp = (t - *total) - y;
  *total = t;
}

/* sources.py:85-101 add_uniform_rain_c */
void API(rbo_uniform_rain_c)(int ny, int nx, R *h, R *comp, R rate, R dt) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < ny; i++)
    for (int j = 0; j < nx; j++) kahan_add(&h[IX(i, j)], &comp[IX(i, j)], rate * dt);
}

/* sources.py:104-121 add_rain_field_c */
void API(rbo_rain_field_c)(int ny, int nx, R *h, R *comp, const R *rain, R dt, R scale) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < ny; i++)
    for (int j = 0; j < nx; j++) kahan_add(&h[IX(i, j)], &comp[IX(i, j)], rain[IX(i, j)] * scale * dt);
}

/* ========================================================================= */
/* Open-edge sinks (solver/core/boundaries.py:244-358)                        */
/* ========================================================================= */

/* boundaries.py:244-256 _drain */
static inline R drain(R h_edge, R q_out, R dxdt) {
  R removed = dxdt * q_out;
  if (removed > h_edge) removed = h_edge;
  if (removed < C(0.0)) removed = C(0.0);
  return h_edge - removed;
}

/* boundaries.py:321-358 apply_open_outflow; edges launched west, east, north, south. */
void API(rbo_open_outflow)(int ny, int nx, R *h, const R *qx, const R *qy, double *loss_cum, R dxdt,
                           const int32_t *bc) {
  if (bc[EDGE_W] == BC_OPEN && nx > 1)
    for (int i = 0; i < ny; i++) {
      const R avail = h[IX(i, 0)];
      const R h_new = drain(avail, rmax(-qx[FX(i, 1)], C(0.0)), dxdt);
      h[IX(i, 0)] = h_new;
      loss_cum[IX(i, 0)] = loss_cum[IX(i, 0)] + ((double)avail - (double)h_new);
    }
  if (bc[EDGE_E] == BC_OPEN && nx > 1)
    for (int i = 0; i < ny; i++) {
      const R avail = h[IX(i, nx - 1)];
      const R h_new = drain(avail, rmax(qx[FX(i, nx - 1)], C(0.0)), dxdt);
      h[IX(i, nx - 1)] = h_new;
      loss_cum[IX(i, nx - 1)] = loss_cum[IX(i, nx - 1)] + ((double)avail - (double)h_new);
    }
  if (bc[EDGE_N] == BC_OPEN && ny > 1)
    for (int j = 0; j < nx; j++) {
      const R avail = h[IX(0, j)];
      const R h_new = drain(avail, rmax(-qy[FY(1, j)], C(0.0)), dxdt);
      h[IX(0, j)] = h_new;
      loss_cum[IX(0, j)] = loss_cum[IX(0, j)] + ((double)avail - (double)h_new);
    }
  if (bc[EDGE_S] == BC_OPEN && ny > 1)
    for (int j = 0; j < nx; j++) {
      const R avail = h[IX(ny - 1, j)];
      const R h_new = drain(avail, rmax(qy[FY(ny - 1, j)], C(0.0)), dxdt);
      h[IX(ny - 1, j)] = h_new;
      loss_cum[IX(ny - 1, j)] = loss_cum[IX(ny - 1, j)] + ((double)avail - (double)h_new);
    }
}

/* ========================================================================= */
/* Sediment transport and Exner (solver/core/sediment.py)                    */
/* ========================================================================= */

#define SUBMERGED_SG C(1.65)     /* sediment.py:146 */
#define SHIELDS_CRITICAL C(0.047) /* sediment.py:148 */
#define MPM_COEFFICIENT C(8.0)    /* sediment.py:150 */

/* sediment.py:161-207 kinematic_shear, shields_number, mpm_capacity, face_capacity */
static inline R face_capacity(R q, R h, R radius, R n, R d50) {
  if (h < H_DRY || d50 <= C(0.0) || q == C(0.0)) return C(0.0);
  const R tau = G * n * n * q * q / (h * h * rbo_pow(radius, 1));
  const R theta = tau / (SUBMERGED_SG * G * d50);
  R qs;
  if (theta <= SHIELDS_CRITICAL) {
    qs = C(0.0);
  } else {
    const R excess = theta - SHIELDS_CRITICAL;
    qs = MPM_COEFFICIENT * rbo_pow(excess, 2) * r_sqrt(SUBMERGED_SG * G * d50 * d50 * d50);
  }
  if (q < C(0.0)) return -qs;
  return qs;
}

/* sediment.py:218-273 accumulate_qs_x / accumulate_qs_y (interior faces) */
void API(rbo_accumulate_qs)(int ny, int nx, const R *qx, const R *qy, const R *eta, const R *z, const R *n,
                            const R *d50, R dt, R *qs_int_x, R *qs_comp_x, R *qs_int_y, R *qs_comp_y) {
  if (nx > 1) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < ny; i++)
      for (int j = 1; j <= nx - 1; j++) {
        const R eta_max = rmax(eta[IX(i, j - 1)], eta[IX(i, j)]);
        const R z_bank = rmax(z[IX(i, j - 1)], z[IX(i, j)]);
        const R h_face = eta_max - z_bank; /* channels.py:136-138 */
        const R qs = face_capacity(qx[FX(i, j)], h_face, h_face, C(0.5) * (n[IX(i, j - 1)] + n[IX(i, j)]),
                                   C(0.5) * (d50[IX(i, j - 1)] + d50[IX(i, j)]));
        kahan_add(&qs_int_x[FX(i, j)], &qs_comp_x[FX(i, j)], qs * dt);
      }
  }
  if (ny > 1) {
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= ny - 1; i++)
      for (int j = 0; j < nx; j++) {
        const R eta_max = rmax(eta[IX(i - 1, j)], eta[IX(i, j)]);
        const R z_bank = rmax(z[IX(i - 1, j)], z[IX(i, j)]);
        const R h_face = eta_max - z_bank;
        const R qs = face_capacity(qy[FY(i, j)], h_face, h_face, C(0.5) * (n[IX(i - 1, j)] + n[IX(i, j)]),
                                   C(0.5) * (d50[IX(i - 1, j)] + d50[IX(i, j)]));
        kahan_add(&qs_int_y[FY(i, j)], &qs_comp_y[FY(i, j)], qs * dt);
      }
  }
}

/* sediment.py:383-426 exner_update; dx and inv_one_minus_p arrive as float32 kernel args. */
void API(rbo_exner_update)(int ny, int nx, const R *qs_int_x, const R *qs_int_y, const float *dz_lo,
                           const float *dz_hi, float dx, float inv_one_minus_p, double *dz_cum,
                           double *dz_unapplied) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < ny; i++) {
    for (int j = 0; j < nx; j++) {
      const double div_x = (double)qs_int_x[FX(i, j + 1)] - (double)qs_int_x[FX(i, j)];
      const double div_y = (double)qs_int_y[FY(i + 1, j)] - (double)qs_int_y[FY(i, j)];
      const double want = dz_cum[IX(i, j)] - (double)inv_one_minus_p * (div_x + div_y) / (double)dx;
      double nw = want;
      const double lo = (double)dz_lo[IX(i, j)], hi = (double)dz_hi[IX(i, j)];
      if (nw < lo) nw = lo;
      if (nw > hi) nw = hi;
      if (nw != want) dz_unapplied[IX(i, j)] = dz_unapplied[IX(i, j)] + (want - nw);
      dz_cum[IX(i, j)] = nw;
    }
  }
}

/* sediment.py:429-441 rebuild_bed */
void API(rbo_rebuild_bed)(int ny, int nx, const R *z0, const double *dz_cum, R *z) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < ny; i++)
    for (int j = 0; j < nx; j++) z[IX(i, j)] = (R)((double)z0[IX(i, j)] + dz_cum[IX(i, j)]);
}

/* ========================================================================= */
/* Sub-grid channels (solver/core/channels.py, local_inertial.py:275-500,     */
/* friction.py:35-58, sediment.py:276-377)                                    */
/* ========================================================================= */

/* channels.py:58-70 eta_subgrid */
static inline R eta_subgrid(R h, R z, R w, R d, R dx) {
  R eta = h + z;
  if (w > C(0.0) && d > C(0.0)) {
    const R h_bf = w * d / dx;
    if (h <= h_bf)
      eta = z - d + h * dx / w;
    else
      eta = z + (h - h_bf);
  }
  return eta;
}

/* channels.py:73-83 column_depth */
static inline R column_depth(R h, R w, R d, R dx) {
  R col = h;
  if (w > C(0.0) && d > C(0.0)) {
    const R h_bf = w * d / dx;
    if (h <= h_bf)
      col = h * dx / w;
    else
      col = d + (h - h_bf);
  }
  return col;
}

/* local_inertial.py:278-291 compute_eta_channels */
void API(rbo_compute_eta_channels)(int ny, int nx, const R *h, const R *z, const R *w, const R *d, R dx, R *eta) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < ny; i++)
    for (int j = 0; j < nx; j++) eta[IX(i, j)] = eta_subgrid(h[IX(i, j)], z[IX(i, j)], w[IX(i, j)], d[IX(i, j)], dx);
}

/* friction.py:35-58 manning_denominator_radius */
static inline R manning_denominator_radius(R q_prev, R h_flow, R radius, R n, R g, R dt) {
  return C(1.0) + g * dt * n * n * rabs(q_prev) / (h_flow * rbo_pow(radius, 3));
}

/* local_inertial.py:294-320 _channel_flux, with channels.py:120-135 (flow depth, radius) */
static inline R channel_flux(R q_prev, R eta_max, R slope, R w_face, R z_bank, R z_ch, R n_ch, R dt, R g) {
  if (w_face <= C(0.0)) return C(0.0);
  const R h_ch = rmin(eta_max, z_bank) - z_ch;
  if (h_ch < H_DRY) return C(0.0);
  const R radius = w_face * h_ch / (w_face + C(2.0) * h_ch);
  const R num = q_prev - g * h_ch * dt * slope;
  const R den = manning_denominator_radius(q_prev, h_ch, radius, n_ch, g, dt);
  return num / den;
}

/* local_inertial.py:323-336 _floodplain_flux */
static inline R floodplain_flux(R q_prev, R eta_max, R slope, R z_bank, R n_fp, R dt, R g) {
  const R h_fp = eta_max - z_bank;
  if (h_fp < H_DRY) return C(0.0);
  const R num = q_prev - g * h_fp * dt * slope;
  const R den = manning_denominator(q_prev, h_fp, n_fp, g, dt);
  return num / den;
}

/* One two-component face between cell a (left / top) and cell b (right / bottom):
 * local_inertial.py:355-383 (x) and :401-427 (y), channels.py:98-117 (face width, bed). */
static inline void channel_face(R *q, R *q_ch, R *q_fp, R eta_a, R eta_b, R z_a, R z_b, R n_a, R n_b, R w_a, R w_b,
                                R d_a, R d_b, R cn_a, R cn_b, R dx, R dt, R g) {
  const R eta_max = rmax(eta_a, eta_b);
  const R slope = (eta_b - eta_a) / dx;
  const R z_bank = rmax(z_a, z_b);
  const R f_fp = floodplain_flux(*q_fp, eta_max, slope, z_bank, C(0.5) * (n_a + n_b), dt, g);
  const R w_face = rmin(w_a, w_b);
  const R z_ch = rmax(z_a - d_a, z_b - d_b);
  const R f_ch = channel_flux(*q_ch, eta_max, slope, w_face, z_bank, z_ch, C(0.5) * (cn_a + cn_b), dt, g);
  *q_fp = f_fp;
  *q_ch = f_ch;
  const R frac = w_face / dx;
  *q = f_fp * (C(1.0) - frac) + f_ch * frac;
}

/* local_inertial.py:338-427 update_qx_channels / update_qy_channels (interior faces) */
void API(rbo_update_q_channels)(int ny, int nx, R *qx, R *qx_ch, R *qx_fp, R *qy, R *qy_ch, R *qy_fp, const R *eta,
                                const R *z, const R *n, const R *w, const R *d, const R *cn, R dx, R dt, R g) {
  if (nx > 1) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < ny; i++)
      for (int j = 1; j <= nx - 1; j++) {
        const size_t a = IX(i, j - 1), b = IX(i, j), f = FX(i, j);
        channel_face(&qx[f], &qx_ch[f], &qx_fp[f], eta[a], eta[b], z[a], z[b], n[a], n[b], w[a], w[b], d[a], d[b],
                     cn[a], cn[b], dx, dt, g);
      }
  }
  if (ny > 1) {
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= ny - 1; i++)
      for (int j = 0; j < nx; j++) {
        const size_t a = IX(i - 1, j), b = IX(i, j), f = FY(i, j);
        channel_face(&qy[f], &qy_ch[f], &qy_fp[f], eta[a], eta[b], z[a], z[b], n[a], n[b], w[a], w[b], d[a], d[b],
                     cn[a], cn[b], dx, dt, g);
      }
  }
}

/* local_inertial.py:430-472 limit_qx_channels / limit_qy_channels */
void API(rbo_limit_q_channels)(int ny, int nx, R *qx, R *qx_ch, R *qx_fp, R *qy, R *qy_ch, R *qy_fp,
                               const R *beta) {
  if (nx > 1) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < ny; i++)
      for (int j = 1; j <= nx - 1; j++) {
        const size_t f = FX(i, j);
        const R q = qx[f];
        if (q == C(0.0)) continue;
        R b = beta[IX(i, j - 1)];
        if (q < C(0.0)) b = beta[IX(i, j)];
        qx[f] = q * b;
        qx_ch[f] = qx_ch[f] * b;
        qx_fp[f] = qx_fp[f] * b;
      }
  }
  if (ny > 1) {
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= ny - 1; i++)
      for (int j = 0; j < nx; j++) {
        const size_t f = FY(i, j);
        const R q = qy[f];
        if (q == C(0.0)) continue;
        R b = beta[IX(i - 1, j)];
        if (q < C(0.0)) b = beta[IX(i, j)];
        qy[f] = q * b;
        qy_ch[f] = qy_ch[f] * b;
        qy_fp[f] = qy_fp[f] * b;
      }
  }
}

/* local_inertial.py:475-489 reduce_column_max */
R API(rbo_reduce_column_max)(int ny, int nx, const R *h, const R *w, const R *d, R dx) {
  R m = C(0.0);
  for (int i = 0; i < ny; i++)
    for (int j = 0; j < nx; j++) {
      const R c = column_depth(h[IX(i, j)], w[IX(i, j)], d[IX(i, j)], dx);
      if (c > m) m = c;
    }
  return m;
}

/* sediment.py:276-305 _combined_capacity */
static inline R combined_capacity(R q_ch, R q_fp, R eta_max, R z_bank, R z_ch, R w_face, R n_fp, R n_ch, R d50,
                                  R dx) {
  const R h_fp = eta_max - z_bank;
  const R qs_fp = face_capacity(q_fp, h_fp, h_fp, n_fp, d50);
  R qs_ch = C(0.0);
  if (w_face > C(0.0)) {
    const R h_ch = rmin(eta_max, z_bank) - z_ch;
    if (h_ch >= H_DRY) qs_ch = face_capacity(q_ch, h_ch, w_face * h_ch / (w_face + C(2.0) * h_ch), n_ch, d50);
  }
  const R frac = w_face / dx;
  return qs_fp * (C(1.0) - frac) + qs_ch * frac;
}

/* sediment.py:308-377 accumulate_qs_x_channels / accumulate_qs_y_channels */
void API(rbo_accumulate_qs_channels)(int ny, int nx, const R *qx_ch, const R *qx_fp, const R *qy_ch, const R *qy_fp,
                                     const R *eta, const R *z, const R *n, const R *d50, const R *w, const R *d,
                                     const R *cn, R dx, R dt, R *qs_int_x, R *qs_comp_x, R *qs_int_y,
                                     R *qs_comp_y) {
  if (nx > 1) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < ny; i++)
      for (int j = 1; j <= nx - 1; j++) {
        const size_t a = IX(i, j - 1), b = IX(i, j), f = FX(i, j);
        const R qs = combined_capacity(qx_ch[f], qx_fp[f], rmax(eta[a], eta[b]), rmax(z[a], z[b]),
                                       rmax(z[a] - d[a], z[b] - d[b]), rmin(w[a], w[b]), C(0.5) * (n[a] + n[b]),
                                       C(0.5) * (cn[a] + cn[b]), C(0.5) * (d50[a] + d50[b]), dx);
        kahan_add(&qs_int_x[f], &qs_comp_x[f], qs * dt);
      }
  }
  if (ny > 1) {
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= ny - 1; i++)
      for (int j = 0; j < nx; j++) {
        const size_t a = IX(i - 1, j), b = IX(i, j), f = FY(i, j);
        const R qs = combined_capacity(qy_ch[f], qy_fp[f], rmax(eta[a], eta[b]), rmax(z[a], z[b]),
                                       rmax(z[a] - d[a], z[b] - d[b]), rmin(w[a], w[b]), C(0.5) * (n[a] + n[b]),
                                       C(0.5) * (cn[a] + cn[b]), C(0.5) * (d50[a] + d50[b]), dx);
        kahan_add(&qs_int_y[f], &qs_comp_y[f], qs * dt);
      }
  }
}

/* ========================================================================= */
/* Point sources (solver/processes/inflow.py:74-113)                          */
/* ========================================================================= */
void API(rbo_inject_points)(int ny, int nx, R *h, R *comp, int nsrc, const int32_t *rows, const int32_t *cols,
                            const R *add_depth) {
  (void)ny;
  for (int k = 0; k < nsrc; k++) {
    const size_t c = IX(rows[k], cols[k]);
    if (comp)
      kahan_add(&h[c], &comp[k], add_depth[k]);
    else
      h[c] = h[c] + add_depth[k];
  }
}

/* ========================================================================= */
/* Local-inertial step orchestration (local_inertial.py:547-727)             */
/* ========================================================================= */
typedef struct {
  int32_t ny, nx;
  double dx;      /* Grid.dx, a host double */
  R *h, *z, *n;   /* (ny, nx) */
  R *qx, *qy;     /* (ny, nx+1), (ny+1, nx) */
  R *eta, *beta;  /* (ny, nx) scratch */
  R *h_comp;      /* NULL: areal-source compensation unarmed */
  R *rain;        /* NULL: no rain field */
  R *infil;       /* NULL: no infiltration */
  double *loss_cum; /* (ny, nx) float64, NULL when unarmed */
  int32_t bc[4];  /* per edge (north, south, east, west): 0 closed, 1 open, 2 fixed_stage */
  R *d50;         /* NULL: sediment unarmed */
  R *qs_int_x, *qs_comp_x, *qs_int_y, *qs_comp_y;
  R *chan_w, *chan_d, *chan_n; /* (ny, nx); chan_w NULL: sub-grid channels unarmed */
  R *qx_ch, *qx_fp;            /* (ny, nx+1) channel / floodplain components */
  R *qy_ch, *qy_fp;            /* (ny+1, nx) */
} rbo_li_state;

void API(rbo_li_step)(rbo_li_state *s, double dt, double rain, int limit, double rain_scale) {
  const int ny = s->ny, nx = s->nx;
  const R dxf = (R)s->dx, dtf = (R)dt, gf = G;
  const int chan = s->chan_w != NULL;
  if (!chan) {
    API(rbo_compute_eta)(ny, nx, s->h, s->z, s->eta);
    if (nx > 1) API(rbo_update_qx)(ny, nx, s->qx, s->eta, s->z, s->n, dxf, dtf, gf);
    if (ny > 1) API(rbo_update_qy)(ny, nx, s->qy, s->eta, s->z, s->n, dxf, dtf, gf);
  } else {
    API(rbo_compute_eta_channels)(ny, nx, s->h, s->z, s->chan_w, s->chan_d, dxf, s->eta);
    API(rbo_update_q_channels)(ny, nx, s->qx, s->qx_ch, s->qx_fp, s->qy, s->qy_ch, s->qy_fp, s->eta, s->z, s->n,
                               s->chan_w, s->chan_d, s->chan_n, dxf, dtf, gf);
  }
  API(rbo_zero_edges)(ny, nx, s->qx, s->qy);
  if (limit) {
    API(rbo_outflow_beta)(ny, nx, s->h, s->qx, s->qy, dxf, dtf, s->beta);
    if (!chan)
      API(rbo_limit_q)(ny, nx, s->qx, s->qy, s->beta);
    else
      API(rbo_limit_q_channels)(ny, nx, s->qx, s->qx_ch, s->qx_fp, s->qy, s->qy_ch, s->qy_fp, s->beta);
  }
  if (s->d50 && !chan)
    API(rbo_accumulate_qs)(ny, nx, s->qx, s->qy, s->eta, s->z, s->n, s->d50, dtf, s->qs_int_x, s->qs_comp_x,
                           s->qs_int_y, s->qs_comp_y);
  if (s->d50 && chan)
    API(rbo_accumulate_qs_channels)(ny, nx, s->qx_ch, s->qx_fp, s->qy_ch, s->qy_fp, s->eta, s->z, s->n, s->d50,
                                    s->chan_w, s->chan_d, s->chan_n, dxf, dtf, s->qs_int_x, s->qs_comp_x,
                                    s->qs_int_y, s->qs_comp_y);
  const int compensated = s->h_comp != NULL;
  API(rbo_update_h)(ny, nx, s->h, s->qx, s->qy, dxf, dtf, compensated ? C(0.0) : (R)rain);
  if (compensated && s->rain == NULL) API(rbo_uniform_rain_c)(ny, nx, s->h, s->h_comp, (R)rain, dtf);
  if (s->rain != NULL) {
    if (compensated)
      API(rbo_rain_field_c)(ny, nx, s->h, s->h_comp, s->rain, dtf, (R)rain_scale);
    else
      API(rbo_rain_field_plain)(ny, nx, s->h, s->rain, dtf, (R)rain_scale);
  }
  if (s->infil != NULL) API(rbo_infiltration)(ny, nx, s->h, s->infil, s->loss_cum, dtf);
  const int any_open = s->bc[0] == BC_OPEN || s->bc[1] == BC_OPEN || s->bc[2] == BC_OPEN || s->bc[3] == BC_OPEN;
  if (any_open) {
    const R dxdt = (R)(dt / s->dx); /* boundaries.py:329 float(dt)/float(g.dx) */
    API(rbo_open_outflow)(ny, nx, s->h, s->qx, s->qy, s->loss_cum, dxdt, s->bc);
  }
}

/* local_inertial.py:515-544 compute_dt (host float64 arithmetic); with channels
 * armed (w, d non-NULL) the reduction is over the water column (:475-489). */
double API(rbo_li_compute_dt)(int ny, int nx, const R *h, const R *w, const R *d, double dx, double alpha,
                              double dt_max) {
  const double h_max = (double)(w != NULL ? API(rbo_reduce_column_max)(ny, nx, h, w, d, (R)dx)
                                          : API(rbo_reduce_hmax)(ny, nx, h));
  if (h_max <= 1.0e-3) return dt_max;
  const double dt = alpha * dx / sqrt(9.81 * h_max);
  return dt < dt_max ? dt : dt_max;
}

/* ========================================================================= */
/* HLLC kernels (solver/core/hllc.py)                                         */
/* ========================================================================= */

/* hllc.py:158-165 _minmod */
static inline R minmod(R a, R b) {
  if (a * b <= C(0.0)) return C(0.0);
  if (rabs(a) < rabs(b)) return a;
  return b;
}

/* hllc.py:168-171 _cget: edge-clamped read */
static inline R cget(const R *a, int i, int j, int ny, int nx) {
  const int ii = i < 0 ? 0 : (i > ny - 1 ? ny - 1 : i);
  const int jj = j < 0 ? 0 : (j > nx - 1 ? nx - 1 : j);
  return a[IX(ii, jj)];
}

/* hllc.py:174-188 _dryfactor */
static inline R dryfactor(R h0, R hm, R hp, R dry) {
  if (h0 <= dry || hm <= dry || hp <= dry) return C(0.0);
  return C(1.0);
}

/* hllc.py:191-256 _hllc */
static inline void hllc(R hl, R ul, R vtl, R hr, R ur, R vtr, R g, R dry, R *f0, R *f1, R *f2) {
  const R cl = r_sqrt(g * rmax(hl, C(0.0)));
  const R cr = r_sqrt(g * rmax(hr, C(0.0)));
  const int dry_l = hl <= dry, dry_r = hr <= dry;
  if (dry_l && dry_r) {
    *f0 = C(0.0);
    *f1 = C(0.0);
    *f2 = C(0.0);
    return;
  }
  R sl, sr;
  if (dry_l) {
    sl = ur - C(2.0) * cr;
    sr = ur + cr;
  } else if (dry_r) {
    sl = ul - cl;
    sr = ul + C(2.0) * cl;
  } else {
    const R hs = C(0.5) * (cl + cr) + C(0.25) * (ul - ur);
    const R h_star = rmax(hs * hs / g, C(0.0));
    const R c_star = r_sqrt(g * h_star);
    const R u_star = C(0.5) * (ul + ur) + cl - cr;
    sl = rmin(ul - cl, u_star - c_star);
    sr = rmax(ur + cr, u_star + c_star);
  }
  const R fh_l = hl * ul;
  const R fmn_l = hl * ul * ul + C(0.5) * g * hl * hl;
  const R fh_r = hr * ur;
  const R fmn_r = hr * ur * ur + C(0.5) * g * hr * hr;
  R fh, fmn;
  if (sl >= C(0.0)) {
    fh = fh_l;
    fmn = fmn_l;
  } else if (sr <= C(0.0)) {
    fh = fh_r;
    fmn = fmn_r;
  } else {
    const R inv = C(1.0) / (sr - sl);
    fh = (sr * fh_l - sl * fh_r + sl * sr * (hr - hl)) * inv;
    fmn = (sr * fmn_l - sl * fmn_r + sl * sr * (hr * ur - hl * ul)) * inv;
  }
  const R den_s = hr * (ur - sr) - hl * (ul - sl);
  R s_star = C(0.5) * (ul + ur);
  if (rabs(den_s) > C(1.0e-12)) s_star = (sl * hr * (ur - sr) - sr * hl * (ul - sl)) / den_s;
  R vt = vtr;
  if (s_star >= C(0.0)) vt = vtl;
  *f0 = fh;
  *f1 = fmn;
  *f2 = fh * vt;
}

typedef struct {
  int32_t ny, nx;
  double dx;
  R *h, *hu, *hv, *z, *n; /* (ny, nx) */
  R *eta, *beta;          /* (ny, nx) scratch shared with LI */
  R *h_comp, *rain, *infil;
  double *loss_cum;
  int32_t bc[4];          /* north, south, east, west */
  double stage[4];        /* prescribed surface per fixed_stage edge, this step */
  /* _HllcScratch (hllc.py:96-120) */
  R *uvel, *vvel;
  R *fx_h, *fx_mn_l, *fx_mn_r, *fx_mt; /* (ny, nx+1) */
  R *fy_h, *fy_mn_l, *fy_mn_r, *fy_mt; /* (ny+1, nx) */
  R *dh, *dhu, *dhv, *h1, *hu1, *hv1;
} rbo_hllc_state;

/* hllc.py:262-282 _primitives */
static void hllc_primitives(rbo_hllc_state *s, const R *h, const R *hu, const R *hv, R dry) {
  const int ny = s->ny, nx = s->nx;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < ny; i++)
    for (int j = 0; j < nx; j++) {
      const R hh = h[IX(i, j)];
      if (hh > dry) {
        s->uvel[IX(i, j)] = hu[IX(i, j)] / hh;
        s->vvel[IX(i, j)] = hv[IX(i, j)] / hh;
      } else {
        s->uvel[IX(i, j)] = C(0.0);
        s->vvel[IX(i, j)] = C(0.0);
      }
      s->eta[IX(i, j)] = hh + s->z[IX(i, j)];
    }
}

/* hllc.py:285-354 _flux_x over all faces (ny, nx+1) */
static void hllc_flux_x(rbo_hllc_state *s, const R *h, R g, R dry) {
  const int ny = s->ny, nx = s->nx;
  const R *eta = s->eta, *z = s->z, *uv = s->uvel, *vv = s->vvel;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < ny; i++)
    for (int j = 0; j <= nx; j++) {
      const R e0 = cget(eta, i, j - 2, ny, nx), e1 = cget(eta, i, j - 1, ny, nx), e2 = cget(eta, i, j, ny, nx),
              e3 = cget(eta, i, j + 1, ny, nx);
      const R z0 = cget(z, i, j - 2, ny, nx), z1 = cget(z, i, j - 1, ny, nx), z2 = cget(z, i, j, ny, nx),
              z3 = cget(z, i, j + 1, ny, nx);
      const R u0 = cget(uv, i, j - 2, ny, nx), u1 = cget(uv, i, j - 1, ny, nx), u2 = cget(uv, i, j, ny, nx),
              u3 = cget(uv, i, j + 1, ny, nx);
      const R v0 = cget(vv, i, j - 2, ny, nx), v1 = cget(vv, i, j - 1, ny, nx), v2 = cget(vv, i, j, ny, nx),
              v3 = cget(vv, i, j + 1, ny, nx);
      const R h0 = cget(h, i, j - 2, ny, nx), h1 = cget(h, i, j - 1, ny, nx), h2 = cget(h, i, j, ny, nx),
              h3 = cget(h, i, j + 1, ny, nx);
      const R wl = dryfactor(h1, h0, h2, dry);
      const R wr = dryfactor(h2, h1, h3, dry);
      const R eta_l = e1 + C(0.5) * wl * minmod(e1 - e0, e2 - e1);
      const R eta_r = e2 - C(0.5) * wr * minmod(e2 - e1, e3 - e2);
      const R zf_l = z1 + C(0.5) * wl * minmod(z1 - z0, z2 - z1);
      const R zf_r = z2 - C(0.5) * wr * minmod(z2 - z1, z3 - z2);
      const R u_l = u1 + C(0.5) * wl * minmod(u1 - u0, u2 - u1);
      const R u_r = u2 - C(0.5) * wr * minmod(u2 - u1, u3 - u2);
      const R v_l = v1 + C(0.5) * wl * minmod(v1 - v0, v2 - v1);
      const R v_r = v2 - C(0.5) * wr * minmod(v2 - v1, v3 - v2);
      const R h_l = rmax(eta_l - zf_l, C(0.0));
      const R h_r = rmax(eta_r - zf_r, C(0.0));
      const R z_star = rmax(zf_l, zf_r);
      const R hl_star = rmax(eta_l - z_star, C(0.0));
      const R hr_star = rmax(eta_r - z_star, C(0.0));
      R f0, f1, f2;
      hllc(hl_star, u_l, v_l, hr_star, u_r, v_r, g, dry, &f0, &f1, &f2);
      s->fx_h[FX(i, j)] = f0;
      s->fx_mn_l[FX(i, j)] = f1 + C(0.5) * g * (h_l * h_l - hl_star * hl_star);
      s->fx_mn_r[FX(i, j)] = f1 + C(0.5) * g * (h_r * h_r - hr_star * hr_star);
      s->fx_mt[FX(i, j)] = f2;
    }
}

/* hllc.py:357-424 _flux_y over all faces (ny+1, nx) */
static void hllc_flux_y(rbo_hllc_state *s, const R *h, R g, R dry) {
  const int ny = s->ny, nx = s->nx;
  const R *eta = s->eta, *z = s->z, *uv = s->uvel, *vv = s->vvel;
#pragma omp parallel for schedule(static)
  for (int i = 0; i <= ny; i++)
    for (int j = 0; j < nx; j++) {
      const R e0 = cget(eta, i - 2, j, ny, nx), e1 = cget(eta, i - 1, j, ny, nx), e2 = cget(eta, i, j, ny, nx),
              e3 = cget(eta, i + 1, j, ny, nx);
      const R z0 = cget(z, i - 2, j, ny, nx), z1 = cget(z, i - 1, j, ny, nx), z2 = cget(z, i, j, ny, nx),
              z3 = cget(z, i + 1, j, ny, nx);
      const R u0 = cget(uv, i - 2, j, ny, nx), u1 = cget(uv, i - 1, j, ny, nx), u2 = cget(uv, i, j, ny, nx),
              u3 = cget(uv, i + 1, j, ny, nx);
      const R v0 = cget(vv, i - 2, j, ny, nx), v1 = cget(vv, i - 1, j, ny, nx), v2 = cget(vv, i, j, ny, nx),
              v3 = cget(vv, i + 1, j, ny, nx);
      const R h0 = cget(h, i - 2, j, ny, nx), h1 = cget(h, i - 1, j, ny, nx), h2 = cget(h, i, j, ny, nx),
              h3 = cget(h, i + 1, j, ny, nx);
      const R wl = dryfactor(h1, h0, h2, dry);
      const R wr = dryfactor(h2, h1, h3, dry);
      const R eta_l = e1 + C(0.5) * wl * minmod(e1 - e0, e2 - e1);
      const R eta_r = e2 - C(0.5) * wr * minmod(e2 - e1, e3 - e2);
      const R zf_l = z1 + C(0.5) * wl * minmod(z1 - z0, z2 - z1);
      const R zf_r = z2 - C(0.5) * wr * minmod(z2 - z1, z3 - z2);
      const R vn_l = v1 + C(0.5) * wl * minmod(v1 - v0, v2 - v1);
      const R vn_r = v2 - C(0.5) * wr * minmod(v2 - v1, v3 - v2);
      const R ut_l = u1 + C(0.5) * wl * minmod(u1 - u0, u2 - u1);
      const R ut_r = u2 - C(0.5) * wr * minmod(u2 - u1, u3 - u2);
      const R h_l = rmax(eta_l - zf_l, C(0.0));
      const R h_r = rmax(eta_r - zf_r, C(0.0));
      const R z_star = rmax(zf_l, zf_r);
      const R hl_star = rmax(eta_l - z_star, C(0.0));
      const R hr_star = rmax(eta_r - z_star, C(0.0));
      R f0, f1, f2;
      hllc(hl_star, vn_l, ut_l, hr_star, vn_r, ut_r, g, dry, &f0, &f1, &f2);
      s->fy_h[FY(i, j)] = f0;
      s->fy_mn_l[FY(i, j)] = f1 + C(0.5) * g * (h_l * h_l - hl_star * hl_star);
      s->fy_mn_r[FY(i, j)] = f1 + C(0.5) * g * (h_r * h_r - hr_star * hr_star);
      s->fy_mt[FY(i, j)] = f2;
    }
}

/* hllc.py:993-1109 _apply_boundaries: fixed_stage ghosts (:537-628), then walls (:442-521). */
static void hllc_apply_boundaries(rbo_hllc_state *s, const R *h, R g, R dry) {
  const int ny = s->ny, nx = s->nx;
  const R *z = s->z, *uv = s->uvel, *vv = s->vvel;
  R f0, f1, f2;
  if (s->bc[EDGE_W] == BC_STAGE) {
    const R stage = (R)s->stage[EDGE_W];
    for (int i = 0; i < ny; i++) {
      const R h_g = rmax(stage - z[IX(i, 0)], C(0.0));
      hllc(h_g, uv[IX(i, 0)], vv[IX(i, 0)], h[IX(i, 0)], uv[IX(i, 0)], vv[IX(i, 0)], g, dry, &f0, &f1, &f2);
      s->fx_h[FX(i, 0)] = f0;
      s->fx_mn_r[FX(i, 0)] = f1;
      s->fx_mt[FX(i, 0)] = f2;
    }
  }
  if (s->bc[EDGE_E] == BC_STAGE) {
    const R stage = (R)s->stage[EDGE_E];
    for (int i = 0; i < ny; i++) {
      const R u = uv[IX(i, nx - 1)], v = vv[IX(i, nx - 1)];
      const R h_g = rmax(stage - z[IX(i, nx - 1)], C(0.0));
      hllc(h[IX(i, nx - 1)], u, v, h_g, u, v, g, dry, &f0, &f1, &f2);
      s->fx_h[FX(i, nx)] = f0;
      s->fx_mn_l[FX(i, nx)] = f1;
      s->fx_mt[FX(i, nx)] = f2;
    }
  }
  if (s->bc[EDGE_N] == BC_STAGE) {
    const R stage = (R)s->stage[EDGE_N];
    for (int j = 0; j < nx; j++) {
      const R h_g = rmax(stage - z[IX(0, j)], C(0.0));
      hllc(h_g, vv[IX(0, j)], uv[IX(0, j)], h[IX(0, j)], vv[IX(0, j)], uv[IX(0, j)], g, dry, &f0, &f1, &f2);
      s->fy_h[FY(0, j)] = f0;
      s->fy_mn_r[FY(0, j)] = f1;
      s->fy_mt[FY(0, j)] = f2;
    }
  }
  if (s->bc[EDGE_S] == BC_STAGE) {
    const R stage = (R)s->stage[EDGE_S];
    for (int j = 0; j < nx; j++) {
      const R u = uv[IX(ny - 1, j)], v = vv[IX(ny - 1, j)];
      const R h_g = rmax(stage - z[IX(ny - 1, j)], C(0.0));
      hllc(h[IX(ny - 1, j)], v, u, h_g, v, u, g, dry, &f0, &f1, &f2);
      s->fy_h[FY(ny, j)] = f0;
      s->fy_mn_l[FY(ny, j)] = f1;
      s->fy_mt[FY(ny, j)] = f2;
    }
  }
  if (s->bc[EDGE_W] == BC_CLOSED)
    for (int i = 0; i < ny; i++) {
      const R h0 = h[IX(i, 0)];
      hllc(h0, -uv[IX(i, 0)], vv[IX(i, 0)], h0, uv[IX(i, 0)], vv[IX(i, 0)], g, dry, &f0, &f1, &f2);
      s->fx_h[FX(i, 0)] = f0;
      s->fx_mn_r[FX(i, 0)] = f1;
      s->fx_mt[FX(i, 0)] = f2;
    }
  if (s->bc[EDGE_E] == BC_CLOSED)
    for (int i = 0; i < ny; i++) {
      const R h0 = h[IX(i, nx - 1)];
      hllc(h0, uv[IX(i, nx - 1)], vv[IX(i, nx - 1)], h0, -uv[IX(i, nx - 1)], vv[IX(i, nx - 1)], g, dry, &f0, &f1,
           &f2);
      s->fx_h[FX(i, nx)] = f0;
      s->fx_mn_l[FX(i, nx)] = f1;
      s->fx_mt[FX(i, nx)] = f2;
    }
  if (s->bc[EDGE_N] == BC_CLOSED)
    for (int j = 0; j < nx; j++) {
      const R h0 = h[IX(0, j)];
      hllc(h0, -vv[IX(0, j)], uv[IX(0, j)], h0, vv[IX(0, j)], uv[IX(0, j)], g, dry, &f0, &f1, &f2);
      s->fy_h[FY(0, j)] = f0;
      s->fy_mn_r[FY(0, j)] = f1;
      s->fy_mt[FY(0, j)] = f2;
    }
  if (s->bc[EDGE_S] == BC_CLOSED)
    for (int j = 0; j < nx; j++) {
      const R h0 = h[IX(ny - 1, j)];
      hllc(h0, vv[IX(ny - 1, j)], uv[IX(ny - 1, j)], h0, -vv[IX(ny - 1, j)], uv[IX(ny - 1, j)], g, dry, &f0, &f1,
           &f2);
      s->fy_h[FY(ny, j)] = f0;
      s->fy_mn_l[FY(ny, j)] = f1;
      s->fy_mt[FY(ny, j)] = f2;
    }
}

/* hllc.py:700-773 _mass_beta, _limit_fx, _limit_fy */
static void hllc_mass_limit(rbo_hllc_state *s, const R *h, R dx, R dt) {
  const int ny = s->ny, nx = s->nx;
  R *fx_h = s->fx_h, *fy_h = s->fy_h, *beta = s->beta;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < ny; i++)
    for (int j = 0; j < nx; j++) {
      R q_out = C(0.0);
      const R fl = fx_h[FX(i, j)];
      if (fl < C(0.0)) q_out = q_out - fl;
      const R fr = fx_h[FX(i, j + 1)];
      if (fr > C(0.0)) q_out = q_out + fr;
      const R ft = fy_h[FY(i, j)];
      if (ft < C(0.0)) q_out = q_out - ft;
      const R fb = fy_h[FY(i + 1, j)];
      if (fb > C(0.0)) q_out = q_out + fb;
      const R out_depth = dt / dx * q_out;
      if (out_depth > C(0.0))
        beta[IX(i, j)] = rclamp(h[IX(i, j)] / out_depth, C(0.0), C(1.0));
      else
        beta[IX(i, j)] = C(1.0);
    }
#pragma omp parallel for schedule(static)
  for (int i = 0; i < ny; i++)
    for (int j = 0; j <= nx; j++) {
      const R q = fx_h[FX(i, j)];
      if (q > C(0.0)) {
        if (j >= 1) fx_h[FX(i, j)] = q * beta[IX(i, j - 1)];
      } else if (q < C(0.0)) {
        if (j <= nx - 1) fx_h[FX(i, j)] = q * beta[IX(i, j)];
      }
    }
#pragma omp parallel for schedule(static)
  for (int i = 0; i <= ny; i++)
    for (int j = 0; j < nx; j++) {
      const R q = fy_h[FY(i, j)];
      if (q > C(0.0)) {
        if (i >= 1) fy_h[FY(i, j)] = q * beta[IX(i - 1, j)];
      } else if (q < C(0.0)) {
        if (i <= ny - 1) fy_h[FY(i, j)] = q * beta[IX(i, j)];
      }
    }
}

/* hllc.py:776-847 _accumulate */
static void hllc_accumulate(rbo_hllc_state *s, const R *h, R dx, R g, R dry) {
  const int ny = s->ny, nx = s->nx;
  const R *eta = s->eta, *z = s->z;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < ny; i++)
    for (int j = 0; j < nx; j++) {
      const R inv_dx = C(1.0) / dx;
      s->dh[IX(i, j)] = -((s->fx_h[FX(i, j + 1)] - s->fx_h[FX(i, j)]) + (s->fy_h[FY(i + 1, j)] - s->fy_h[FY(i, j)])) *
                        inv_dx;
      const R hg = cget(h, i, j, ny, nx);
      const R wx = dryfactor(hg, cget(h, i, j - 1, ny, nx), cget(h, i, j + 1, ny, nx), dry);
      const R wy = dryfactor(hg, cget(h, i - 1, j, ny, nx), cget(h, i + 1, j, ny, nx), dry);
      const R sz_x = wx * minmod(cget(z, i, j, ny, nx) - cget(z, i, j - 1, ny, nx),
                                 cget(z, i, j + 1, ny, nx) - cget(z, i, j, ny, nx));
      const R se_x = wx * minmod(cget(eta, i, j, ny, nx) - cget(eta, i, j - 1, ny, nx),
                                 cget(eta, i, j + 1, ny, nx) - cget(eta, i, j, ny, nx));
      const R hp_x = rmax((eta[IX(i, j)] + C(0.5) * se_x) - (z[IX(i, j)] + C(0.5) * sz_x), C(0.0));
      const R hm_x = rmax((eta[IX(i, j)] - C(0.5) * se_x) - (z[IX(i, j)] - C(0.5) * sz_x), C(0.0));
      const R src_x = -g * C(0.5) * (hp_x + hm_x) * sz_x;
      s->dhu[IX(i, j)] = (-((s->fx_mn_l[FX(i, j + 1)] - s->fx_mn_r[FX(i, j)]) +
                            (s->fy_mt[FY(i + 1, j)] - s->fy_mt[FY(i, j)])) +
                          src_x) *
                         inv_dx;
      const R sz_y = wy * minmod(cget(z, i, j, ny, nx) - cget(z, i - 1, j, ny, nx),
                                 cget(z, i + 1, j, ny, nx) - cget(z, i, j, ny, nx));
      const R se_y = wy * minmod(cget(eta, i, j, ny, nx) - cget(eta, i - 1, j, ny, nx),
                                 cget(eta, i + 1, j, ny, nx) - cget(eta, i, j, ny, nx));
      const R hp_y = rmax((eta[IX(i, j)] + C(0.5) * se_y) - (z[IX(i, j)] + C(0.5) * sz_y), C(0.0));
      const R hm_y = rmax((eta[IX(i, j)] - C(0.5) * se_y) - (z[IX(i, j)] - C(0.5) * sz_y), C(0.0));
      const R src_y = -g * C(0.5) * (hp_y + hm_y) * sz_y;
      s->dhv[IX(i, j)] = (-((s->fy_mn_l[FY(i + 1, j)] - s->fy_mn_r[FY(i, j)]) +
                            (s->fx_mt[FX(i, j + 1)] - s->fx_mt[FX(i, j)])) +
                          src_y) *
                         inv_dx;
    }
}

/* hllc.py:1152-1269 _eval_L */
static void hllc_eval_L(rbo_hllc_state *s, const R *h, const R *hu, const R *hv, R dt) {
  const R dxf = (R)s->dx, gf = G, dryf = H_DRY;
  hllc_primitives(s, h, hu, hv, dryf);
  hllc_flux_x(s, h, gf, dryf);
  hllc_flux_y(s, h, gf, dryf);
  hllc_apply_boundaries(s, h, gf, dryf);
  hllc_mass_limit(s, h, dxf, dt);
  hllc_accumulate(s, h, dxf, gf, dryf);
}

/* hllc.py:1115-1149 _bank_boundary_flux; edges open or fixed_stage are banked. */
static void hllc_bank(rbo_hllc_state *s, double wt) {
  if (s->loss_cum == NULL) return;
  const int ny = s->ny, nx = s->nx;
  double *loss = s->loss_cum;
#define BANKED(e) (s->bc[e] == BC_OPEN || s->bc[e] == BC_STAGE)
  if (BANKED(EDGE_W))
    for (int i = 0; i < ny; i++) loss[IX(i, 0)] = loss[IX(i, 0)] - wt * (double)s->fx_h[FX(i, 0)];
  if (BANKED(EDGE_E))
    for (int i = 0; i < ny; i++) loss[IX(i, nx - 1)] = loss[IX(i, nx - 1)] + wt * (double)s->fx_h[FX(i, nx)];
  if (BANKED(EDGE_N))
    for (int j = 0; j < nx; j++) loss[IX(0, j)] = loss[IX(0, j)] - wt * (double)s->fy_h[FY(0, j)];
  if (BANKED(EDGE_S))
    for (int j = 0; j < nx; j++) loss[IX(ny - 1, j)] = loss[IX(ny - 1, j)] + wt * (double)s->fy_h[FY(ny, j)];
#undef BANKED
}

/* hllc.py:1272-1373 step */
void API(rbo_hllc_step)(rbo_hllc_state *s, double dt, double rain, double rain_scale) {
  const int ny = s->ny, nx = s->nx;
  const R dtf = (R)dt, gf = G, dryf = H_DRY;
  const double wt = 0.5 * dt / s->dx;
  hllc_eval_L(s, s->h, s->hu, s->hv, dtf);
  hllc_bank(s, wt);
  /* hllc.py:850-878 _rk_stage1 */
#pragma omp parallel for schedule(static)
  for (int i = 0; i < ny; i++)
    for (int j = 0; j < nx; j++) {
      const size_t k = IX(i, j);
      const R hh = rmax(s->h[k] + dtf * s->dh[k], C(0.0));
      s->h1[k] = hh;
      if (hh > dryf) {
        s->hu1[k] = s->hu[k] + dtf * s->dhu[k];
        s->hv1[k] = s->hv[k] + dtf * s->dhv[k];
      } else {
        s->hu1[k] = C(0.0);
        s->hv1[k] = C(0.0);
      }
    }
  hllc_eval_L(s, s->h1, s->hu1, s->hv1, dtf);
  hllc_bank(s, wt);
  /* hllc.py:881-909 _rk_stage2 */
#pragma omp parallel for schedule(static)
  for (int i = 0; i < ny; i++)
    for (int j = 0; j < nx; j++) {
      const size_t k = IX(i, j);
      const R hh = rmax(C(0.5) * (s->h[k] + s->h1[k] + dtf * s->dh[k]), C(0.0));
      s->h[k] = hh;
      if (hh > dryf) {
        s->hu[k] = C(0.5) * (s->hu[k] + s->hu1[k] + dtf * s->dhu[k]);
        s->hv[k] = C(0.5) * (s->hv[k] + s->hv1[k] + dtf * s->dhv[k]);
      } else {
        s->hu[k] = C(0.0);
        s->hv[k] = C(0.0);
      }
    }
  /* hllc.py:912-939 _friction */
#pragma omp parallel for schedule(static)
  for (int i = 0; i < ny; i++)
    for (int j = 0; j < nx; j++) {
      const size_t k = IX(i, j);
      const R hh = s->h[k];
      if (hh <= dryf) {
        s->hu[k] = C(0.0);
        s->hv[k] = C(0.0);
        continue;
      }
      const R mom = r_sqrt(s->hu[k] * s->hu[k] + s->hv[k] * s->hv[k]);
      const R denom = manning_denominator(mom, hh, s->n[k], gf, dtf);
      s->hu[k] = s->hu[k] / denom;
      s->hv[k] = s->hv[k] / denom;
    }
  /* hllc.py:1350-1373 sources and sinks */
  const int compensated = s->h_comp != NULL;
  if (compensated && s->rain == NULL) {
    API(rbo_uniform_rain_c)(ny, nx, s->h, s->h_comp, (R)rain, dtf);
  } else if (rain != 0.0) {
    const R r = (R)rain; /* hllc.py:942-945 _add_uniform_rain */
#pragma omp parallel for schedule(static)
    for (int i = 0; i < ny; i++)
      for (int j = 0; j < nx; j++) s->h[IX(i, j)] = s->h[IX(i, j)] + r * dtf;
  }
  if (s->rain != NULL) {
    if (compensated)
      API(rbo_rain_field_c)(ny, nx, s->h, s->h_comp, s->rain, dtf, (R)rain_scale);
    else
      API(rbo_rain_field_plain)(ny, nx, s->h, s->rain, dtf, (R)rain_scale);
  }
  if (s->infil != NULL) API(rbo_infiltration)(ny, nx, s->h, s->infil, s->loss_cum, dtf);
}

/* hllc.py:948-966 _reduce_wavespeed, from a zeroed accumulator (:980). */
R API(rbo_reduce_wavespeed)(int ny, int nx, const R *h, const R *hu, const R *hv) {
  R m = C(0.0);
  for (size_t k = 0; k < (size_t)ny * (size_t)nx; k++) {
    const R hh = h[k];
    const R c = r_sqrt(G * rmax(hh, C(0.0)));
    R sp = c;
    if (hh > H_DRY) {
      const R au = rabs(hu[k]) / hh;
      const R av = rabs(hv[k]) / hh;
      sp = rmax(au, av) + c;
    }
    if (sp > m) m = sp;
  }
  return m;
}

/* hllc.py:972-990 compute_dt */
double API(rbo_hllc_compute_dt)(int ny, int nx, const R *h, const R *hu, const R *hv, double dx, double alpha,
                                double dt_max) {
  const double smax = (double)API(rbo_reduce_wavespeed)(ny, nx, h, hu, hv);
  if (smax <= 0.0) return dt_max;
  const double dt = alpha * dx / smax;
  return dt < dt_max ? dt : dt_max;
}
