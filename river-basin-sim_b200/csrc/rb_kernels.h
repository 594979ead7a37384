// rb_kernels.h -- kernel parameter blocks and launchers shared by the .cu files.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace rb {

// The device-resident clock (solver/scheduler.py:171-246 + compute_dt + the run
// loop's rain gating and source ledger, run.py:369-388), one per workspace. The
// plan kernel fills the per-step fields below from the state-derived reduction;
// step kernels given a clock read their dt, forcing and buffer index from it.
struct DevClock {
  double t;          // simulated time at the start of the next step
  double t1;         // end of the planned step
  double dt;         // the planned step (float64, as the host scheduler has it)
  double t_target;   // the span ends when t >= t_target - EPS_T
  double alpha, dt_max, dx;
  double rain_rate, rain_until, rain_field_sum, cell_area;
  double n_cells;
  double rain_in[2];    // Kahan (total, compensation) of areal rain volume, m^3
  double inflow_in[2];  // Kahan of point-source volume, m^3
  double wt;            // 0.5 * dt / dx (HLLC banking weight)
  const double* sync;   // ascending sync times (device memory owned by the caller)
  int nsync, sync_pos;
  int scheme;           // 0 local inertial, 1 HLLC
  int rain_is_field;
  int cur;              // buffer holding the current state
  int active;           // the planned step runs
  int pending;          // a planned step awaits commit by the next plan
  int steps;            // committed steps since the clock was set
  int max_steps;        // step budget of the current span
  unsigned int red_key; // state-derived max for the next dt (filled by the step kernel)
  unsigned int err;
  float dt32, dxdt32, rain32, scale32;
  int limit;
  // point sources sampled on the device (solver/processes/inflow.py:167-200)
  int nsrc;
  const int* src_cell;   // row * nx + col
  const int* knot_off;   // nsrc + 1 offsets into knot_t / knot_q
  const double* knot_t;
  const double* knot_q;
  float* src_comp;       // per-source Kahan residue, or null for the plain add
  // fixed_stage curves per edge (boundaries.py:199-220), evaluated at t + dt/2
  int stage_off[5];      // edge e's knots are stage_t/v[stage_off[e] .. stage_off[e+1])
  const double* stage_t;
  const double* stage_v;
  float stage32[4];
};

struct LiParams {
  int ny, nx;
  float dx32, dt32;
  float rain_cont;   // uniform rain fused into continuity (0 when compensated)
  float rain32;      // uniform rain for the compensated add
  float scale32;     // rain-field temporal scale
  float dxdt;        // float32(dt / dx) in float64, the open-edge drain factor
  int limit;
  int bc[4];
  float *hb[2], *qxb[2], *qyb[2];   // double buffers; the step reads [cur], writes [cur ^ 1]
  int cur;
  const float *z, *n;
  const DevClock* clk;               // when set: dt, forcing and cur come from the device clock
  float *h_comp;
  const float *rain_field, *infil;
  const float *d50;
  float *qs_int_x, *qs_comp_x, *qs_int_y, *qs_comp_y;
  const float *cw, *cd, *cn;           // sub-grid channel geometry, or null (unarmed)
  float *qxcb[2], *qxfb[2];            // channel / floodplain x-face components, double buffered
  float *qycb[2], *qyfb[2];
  double *ledger;          // 2 doubles per tile, or null when nothing is banked
  unsigned int *hmax_key;  // fused max(h_new) (water column with channels) for the next dt, or null
  unsigned int *err;
};

struct HllcParams {
  int ny, nx;
  float dx32, dt32;
  float *hb[2], *hub[2], *hvb[2];  // double-buffered U: U^n = [cur], U^{n+1} = [cur ^ 1]
  int cur;
  const float *z, *n;
  float *h1, *hu1, *hv1;           // stage-1 output U1 (workspace)
  const DevClock* clk;
  float *h_comp;
  const float *rain_field, *infil;
  float rain32, scale32;
  int rain_mode;  // 0 none, 1 compensated uniform, 2 plain uniform
  int bc[4];
  float stage[4];
  double wt;  // 0.5 * dt / dx, the Heun weight of one stage's boundary banking
  double *ledger;
  unsigned int *smax_key;
  unsigned int *err;
};

// The tensor maps (CUtensorMap, 128 bytes each, held opaque here) of the fields the
// TMA-staged HLLC stage kernel copies into shared memory: both buffers of h, hu, hv
// (the clock picks one at run time), the bed and the stage-1 state.
struct alignas(64) TileMap {
  unsigned char bytes[128];
};
struct HllcMaps {
  TileMap h[2], hu[2], hv[2], z, h1, hu1, hv1;
};

cudaError_t li_step_launch(const LiParams& p, cudaStream_t s);
cudaError_t li_step_launch_variant(const LiParams& p, int variant, cudaStream_t s);
int li_current_variant();
// Arithmetic of the single-domain step kernels (RB_ARITH_EXACT / RB_ARITH_FAST),
// set with rb_set_arith_mode; the launchers above dispatch on it.
int arith_mode();
cudaError_t clock_plan_launch(DevClock* clk, cudaStream_t s);
cudaError_t clock_commit_launch(DevClock* clk, cudaStream_t s);
cudaError_t clock_target_launch(DevClock* clk, double t_target, int max_steps, cudaStream_t s);
cudaError_t clock_inflow_launch(DevClock* clk, float* const* hb, cudaStream_t s);
cudaError_t clock_plan_many_launch(DevClock* clocks, int n, cudaStream_t s);
cudaError_t clock_commit_many_launch(DevClock* clocks, int n, cudaStream_t s);
cudaError_t clock_target_many_launch(DevClock* clocks, int n, const double* t_target, const int* max_steps,
                                     cudaStream_t s);
cudaError_t hllc_stage_launch(const HllcParams& p, int stage, cudaStream_t s);
void li_variant_tile(int variant, int* tx, int* ty);
void hllc_variant_tile(int variant, int* tx, int* ty);
int ens_li_grid_size(int variant);
int ens_hllc_grid_size(int variant);
cudaError_t ens_li_launch(int variant, int grid, const LiParams* P, const int2* map, long long total, cudaStream_t s);
cudaError_t ens_hllc_launch(int variant, int grid, int stage, const HllcParams* P, const int2* map, long long total,
                            cudaStream_t s);
void set_last_error(const char* msg);  // the message rb_last_error returns on this thread
// Argument checks of the C ABI: RB_OK, or an error code with the message set.
int check_grid(int ny, int nx, double dx, const char* who);
int check_bc(const int32_t* bc, bool allow_stage, const char* who);
int check_dt(double dt, const char* who);
int hllc_tiles(int ny, int nx);
// The HLLC stage-kernel variant in force now; the launch and tile count of one call
// can take it once, so a concurrent rb_hllc_set_kernel_variant cannot split them.
int hllc_current_variant();
int hllc_tiles_of(int variant, int ny, int nx);
cudaError_t hllc_stage_launch_variant(const HllcParams& p, int stage, int variant, cudaStream_t s);
// The exact build's stage kernel regardless of the arithmetic mode.
cudaError_t hllc_stage_launch_exact(const HllcParams& p, int stage, int variant, cudaStream_t s);
int li_kernel_variant_count();
bool li_set_kernel_variant(int v);
int hllc_kernel_variant_count();
bool hllc_set_kernel_variant(int v);
void hllc_prepare_device();

// Workspace layout (byte offsets from the workspace base).
struct WsHeader {
  unsigned int red_key;  // reduction slot (max of non-negative floats)
  unsigned int err;      // device error bits
  unsigned int pad[2];
  double sum;            // f64 reduction result
  double pad2[5];
  DevClock clock;        // the device-resident clock (offset 64)
};
static_assert(sizeof(WsHeader) <= 1024, "workspace header overflows its reserved block");
constexpr size_t WS_HEADER = 1024;
constexpr int WS_SUM_BLOCKS = 1184;  // 8 x 148 SMs: fixed so the f64 sum order is fixed
constexpr size_t WS_PARTIALS = WS_HEADER;                             // WS_SUM_BLOCKS doubles
constexpr size_t WS_LEDGER = WS_PARTIALS + WS_SUM_BLOCKS * sizeof(double);  // 2 doubles / tile

size_t ws_ledger_bytes(int ny, int nx);
size_t ws_li_bytes(int ny, int nx);
size_t ws_hllc_bytes(int ny, int nx);
size_t ws_hllc_u1_offset(int ny, int nx);

cudaError_t reduce_max_h(const float* h, size_t n, unsigned int* key, cudaStream_t s);
// Max of the water column (channels.py:73-83) when w is set, else of h.
cudaError_t reduce_max_column(const float* h, const float* w, const float* d, float dx32, size_t n,
                              unsigned int* key, cudaStream_t s);
cudaError_t reduce_wavespeed(const float* h, const float* hu, const float* hv, size_t n, unsigned int* key,
                             cudaStream_t s);
cudaError_t sum_f64(const float* x, size_t n, double* partials, double* out, cudaStream_t s);
cudaError_t sum_ledger(const double* ledger, size_t nslots, double* partials, double* out, cudaStream_t s);
cudaError_t reservoir_withdraw(float* h, int nx, int r0, int c0, int rows, int cols, float scale, double* taken,
                               cudaStream_t s);
cudaError_t reservoir_deliver(float* h, int nx, int r0, int c0, int rows, int cols, double add_depth,
                              double* ledger_slot, cudaStream_t s);
cudaError_t inject_points(float* h, int ny, int nx, int nsrc, const int32_t* rows, const int32_t* cols,
                          const float* add, float* comp, cudaStream_t s);
cudaError_t exner_apply(int ny, int nx, float dx32, float inv1mp, float* qs_int_x, float* qs_int_y,
                        const float* dz_lo, const float* dz_hi, double* dz_cum, double* dz_unapplied,
                        const float* z0, float* z, cudaStream_t s);

// The same step kernels built with fast arithmetic (csrc/fast/, RB_FAST_MATH).
namespace fast {
cudaError_t li_step_launch_variant(const LiParams& p, int variant, cudaStream_t s);
cudaError_t hllc_stage_launch_variant(const HllcParams& p, int stage, int variant, cudaStream_t s);
void hllc_prepare_device();
}  // namespace fast

}  // namespace rb
