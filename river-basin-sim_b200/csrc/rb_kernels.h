// rb_kernels.h -- kernel parameter blocks and launchers shared by the .cu files.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace rb {

// Tile shapes (cells per CTA) and threads per CTA.
constexpr int LI_TX = 32, LI_TY = 16, LI_NT = 256;
constexpr int HLLC_TX = 32, HLLC_TY = 16, HLLC_NT = 256;

struct LiParams {
  int ny, nx;
  float dx32, dt32;
  float rain_cont;   // uniform rain fused into continuity (0 when compensated)
  float rain32;      // uniform rain for the compensated add
  float scale32;     // rain-field temporal scale
  float dxdt;        // float32(dt / dx) in float64, the open-edge drain factor
  int limit;
  int bc[4];
  const float *h, *z, *n, *qx, *qy;  // buffer [cur]
  float *h_out, *qx_out, *qy_out;    // buffer [cur ^ 1]
  float *h_comp;
  const float *rain_field, *infil;
  const float *d50;
  float *qs_int_x, *qs_comp_x, *qs_int_y, *qs_comp_y;
  double *ledger;          // 2 doubles per tile, or null when nothing is banked
  unsigned int *hmax_key;  // fused max(h_new) for the next dt, or null
  unsigned int *err;
};

struct HllcParams {
  int ny, nx;
  float dx32, dt32;
  const float *h_s, *hu_s, *hv_s;  // the stage's input state (U^n, then U1)
  const float *z, *n;
  float *h1, *hu1, *hv1;           // stage-1 output (workspace)
  const float *h_n, *hu_n, *hv_n;  // U^n for the stage-2 convex combination
  float *h_out, *hu_out, *hv_out;  // U^{n+1}
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

cudaError_t li_step_launch(const LiParams& p, cudaStream_t s);
cudaError_t hllc_stage_launch(const HllcParams& p, int stage, cudaStream_t s);
int li_tiles(int ny, int nx);
int hllc_tiles(int ny, int nx);

// Workspace layout (byte offsets from the workspace base).
struct WsHeader {
  unsigned int red_key;  // reduction slot (max of non-negative floats)
  unsigned int err;      // device error bits
  unsigned int pad[2];
  double sum;            // f64 reduction result
};
constexpr size_t WS_HEADER = 1024;
constexpr int WS_SUM_BLOCKS = 1184;  // 8 x 148 SMs: fixed so the f64 sum order is fixed
constexpr size_t WS_PARTIALS = WS_HEADER;                             // WS_SUM_BLOCKS doubles
constexpr size_t WS_LEDGER = WS_PARTIALS + WS_SUM_BLOCKS * sizeof(double);  // 2 doubles / tile

size_t ws_ledger_bytes(int ny, int nx);
size_t ws_li_bytes(int ny, int nx);
size_t ws_hllc_bytes(int ny, int nx);
size_t ws_hllc_u1_offset(int ny, int nx);

cudaError_t reduce_max_h(const float* h, size_t n, unsigned int* key, cudaStream_t s);
cudaError_t reduce_wavespeed(const float* h, const float* hu, const float* hv, size_t n, unsigned int* key,
                             cudaStream_t s);
cudaError_t sum_f64(const float* x, size_t n, double* partials, double* out, cudaStream_t s);
cudaError_t sum_ledger(const double* ledger, size_t nslots, double* partials, double* out, cudaStream_t s);
cudaError_t inject_points(float* h, int nx, int nsrc, const int32_t* rows, const int32_t* cols,
                          const float* add, float* comp, cudaStream_t s);
cudaError_t exner_apply(int ny, int nx, float dx32, float inv1mp, float* qs_int_x, float* qs_int_y,
                        const float* dz_lo, const float* dz_hi, double* dz_cum, double* dz_unapplied,
                        const float* z0, float* z, cudaStream_t s);

}  // namespace rb
