// capi.cu -- the extern "C" entry points of librbsim.so (declared in include/rbsim.h).
//
// Host-side float64 arithmetic here mirrors the reference's Python exactly where
// the reference computes in float64 (compute_dt, the open-edge drain factor, the
// Heun banking weight), and every float32 kernel argument is rounded from the
// float64 value exactly as Warp rounds a Python float at launch.
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "rb_common.cuh"
#include "rb_kernels.h"

namespace {

thread_local char g_err[512] = {0};
std::atomic<int> g_arith_mode{RB_ARITH_EXACT};

int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
  return code;
}

int cuda_fail(cudaError_t e, const char* where) {
  return fail(RB_ERR_CUDA, "%s: %s (%s)", where, cudaGetErrorString(e), cudaGetErrorName(e));
}

#define RB_CUDA(call, where)                      \
  do {                                            \
    cudaError_t e_ = (call);                      \
    if (e_ != cudaSuccess) return cuda_fail(e_, where); \
  } while (0)

inline size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

rb::WsHeader* header(void* ws) { return static_cast<rb::WsHeader*>(ws); }

bool any_bc(const int32_t* bc, int kind) {
  return bc[0] == kind || bc[1] == kind || bc[2] == kind || bc[3] == kind;
}

}  // namespace

namespace rb {

void set_last_error(const char* msg) { snprintf(g_err, sizeof g_err, "%s", msg); }

int arith_mode() { return g_arith_mode.load(); }

bool pdl_enabled() {
  static const bool on = [] {
    const char* v = std::getenv("RBSIM_PDL");
    return v == nullptr || std::strcmp(v, "0") != 0;
  }();
  return on;
}

// Argument checks shared by every entry point that takes a grid, edge kinds or a
// timestep, so that all of them refuse the same inputs with the same messages.
int check_grid(int ny, int nx, double dx, const char* who) {
  if (ny < 1 || nx < 1) return fail(RB_ERR_ARG, "%s: grid %d x %d must be at least 1 x 1", who, ny, nx);
  if ((long long)ny * (long long)(nx + 1) > (1LL << 40)) return fail(RB_ERR_ARG, "%s: grid too large", who);
  if (!(dx > 0.0) || !std::isfinite(dx)) return fail(RB_ERR_ARG, "%s: dx must be a positive finite number", who);
  return RB_OK;
}

int check_bc(const int32_t* bc, bool allow_stage, const char* who) {
  for (int e = 0; e < 4; e++) {
    if (bc[e] < RB_BC_CLOSED || bc[e] > RB_BC_STAGE || (!allow_stage && bc[e] == RB_BC_STAGE))
      return fail(RB_ERR_ARG, "%s: edge %d has unsupported boundary kind %d", who, e, bc[e]);
  }
  return RB_OK;
}

int check_dt(double dt, const char* who) {
  if (!(dt > 0.0) || !std::isfinite(dt)) return fail(RB_ERR_STEP, "%s: non-positive timestep %.17g", who, dt);
  return RB_OK;
}


size_t ws_ledger_bytes(int ny, int nx) {
  // one slot per tile of the smallest tile any kernel variant uses (32 x 8)
  const size_t t = (size_t)((nx + 31) / 32) * (size_t)((ny + 7) / 8);
  return align256(t * 2 * sizeof(double));
}
size_t ws_li_bytes(int ny, int nx) { return WS_LEDGER + ws_ledger_bytes(ny, nx); }
size_t ws_hllc_u1_offset(int ny, int nx) { return WS_LEDGER + ws_ledger_bytes(ny, nx); }
size_t ws_hllc_bytes(int ny, int nx) {
  return ws_hllc_u1_offset(ny, nx) + 3 * align256((size_t)ny * nx * sizeof(float));
}

}  // namespace rb

using rb::check_bc;
using rb::check_dt;
using rb::check_grid;

extern "C" {

int rb_last_error(char* buf, size_t n) {
  const int len = (int)strlen(g_err);
  if (buf != nullptr && n > 0) {
    strncpy(buf, g_err, n - 1);
    buf[n - 1] = '\0';
  }
  return len;
}

int rb_version(int32_t* major, int32_t* minor, int32_t* sm_arch) {
  if (major) *major = 0;
  if (minor) *minor = 1;
  if (sm_arch) *sm_arch = 100;
  return RB_OK;
}

size_t rb_li_workspace_bytes(int32_t ny, int32_t nx) {
  if (ny < 1 || nx < 1) return 0;
  return rb::ws_li_bytes(ny, nx);
}

size_t rb_hllc_workspace_bytes(int32_t ny, int32_t nx) {
  if (ny < 1 || nx < 1) return 0;
  return rb::ws_hllc_bytes(ny, nx);
}

int rb_workspace_init(void* ws, size_t bytes, void* stream) {
  if (ws == nullptr || bytes < rb::WS_LEDGER) return fail(RB_ERR_ARG, "rb_workspace_init: workspace too small");
  RB_CUDA(cudaMemsetAsync(ws, 0, bytes, (cudaStream_t)stream), "rb_workspace_init");
  rb::hllc_prepare_device();  // kernel attributes, before any stream capture
  return RB_OK;
}

static int li_params(const rb_li_fields* f, void* ws, rb::LiParams& p, const char* who) {
  if (f == nullptr || ws == nullptr) return fail(RB_ERR_ARG, "%s: null argument", who);
  int rc = check_grid(f->ny, f->nx, f->dx, who);
  if (rc) return rc;
  if ((rc = check_bc(f->bc, false, who))) return rc;
  if (!f->h[0] || !f->h[1] || !f->qx[0] || !f->qx[1] || !f->qy[0] || !f->qy[1] || !f->z || !f->n)
    return fail(RB_ERR_ARG, "%s: missing state buffer", who);
  if (f->d50 && (!f->qs_int_x || !f->qs_comp_x || !f->qs_int_y || !f->qs_comp_y))
    return fail(RB_ERR_ARG, "%s: d50 given without the transport accumulators", who);
  if (f->chan_w && (!f->chan_d || !f->chan_n || !f->qx_ch[0] || !f->qx_ch[1] || !f->qx_fp[0] || !f->qx_fp[1] ||
                    !f->qy_ch[0] || !f->qy_ch[1] || !f->qy_fp[0] || !f->qy_fp[1]))
    return fail(RB_ERR_ARG, "%s: chan_w given without the channel depth, roughness or face components", who);
  const bool banks = f->infil != nullptr || any_bc(f->bc, RB_BC_OPEN);
  p = rb::LiParams{};
  p.ny = f->ny;
  p.nx = f->nx;
  p.dx32 = (float)f->dx;
  for (int e = 0; e < 4; e++) p.bc[e] = f->bc[e];
  for (int b = 0; b < 2; b++) {
    p.hb[b] = f->h[b];
    p.qxb[b] = f->qx[b];
    p.qyb[b] = f->qy[b];
  }
  p.z = f->z;
  p.n = f->n;
  p.h_comp = f->h_comp;
  p.rain_field = f->rain_field;
  p.infil = f->infil;
  p.d50 = f->d50;
  p.qs_int_x = f->qs_int_x;
  p.qs_comp_x = f->qs_comp_x;
  p.qs_int_y = f->qs_int_y;
  p.qs_comp_y = f->qs_comp_y;
  if (f->chan_w != nullptr) {
    p.cw = f->chan_w;
    p.cd = f->chan_d;
    p.cn = f->chan_n;
    for (int b = 0; b < 2; b++) {
      p.qxcb[b] = f->qx_ch[b];
      p.qxfb[b] = f->qx_fp[b];
      p.qycb[b] = f->qy_ch[b];
      p.qyfb[b] = f->qy_fp[b];
    }
  }
  p.ledger = banks ? (double*)((char*)ws + rb::WS_LEDGER) : nullptr;
  p.err = &header(ws)->err;
  return RB_OK;
}

int rb_li_step_clocked(const rb_li_fields* f, void* ws, void* stream) {
  rb::LiParams p;
  int rc = li_params(f, ws, p, "rb_li_step_clocked");
  if (rc) return rc;
  p.clk = &header(ws)->clock;
  p.hmax_key = &header(ws)->clock.red_key;
  RB_CUDA(rb::li_step_launch(p, (cudaStream_t)stream), "rb_li_step_clocked launch");
  return RB_OK;
}

int rb_li_step(const rb_li_fields* f, int32_t cur, const rb_step_args* a, void* ws, void* stream) {
  if (f == nullptr || a == nullptr || ws == nullptr) return fail(RB_ERR_ARG, "rb_li_step: null argument");
  int rc = check_grid(f->ny, f->nx, f->dx, "rb_li_step");
  if (rc) return rc;
  if ((rc = check_bc(f->bc, false, "rb_li_step"))) return rc;
  if ((rc = check_dt(a->dt, "rb_li_step"))) return rc;
  if (cur != 0 && cur != 1) return fail(RB_ERR_ARG, "rb_li_step: cur must be 0 or 1");
  rb::LiParams p;
  if ((rc = li_params(f, ws, p, "rb_li_step"))) return rc;
  p.dt32 = (float)a->dt;
  p.rain_cont = f->h_comp != nullptr ? 0.0f : (float)a->rain;  // local_inertial.py:697
  p.rain32 = (float)a->rain;
  p.scale32 = (float)a->rain_scale;
  p.dxdt = (float)(a->dt / f->dx);  // boundaries.py:329
  p.limit = a->limit ? 1 : 0;
  p.cur = cur;
  p.clk = nullptr;
  p.hmax_key = nullptr;
  RB_CUDA(rb::li_step_launch(p, (cudaStream_t)stream), "rb_li_step launch");
  return RB_OK;
}

int rb_li_compute_dt(const rb_li_fields* f, int32_t cur, double alpha, double dt_max, void* ws, void* stream,
                     double* dt_out) {
  if (f == nullptr || ws == nullptr || dt_out == nullptr) return fail(RB_ERR_ARG, "rb_li_compute_dt: null argument");
  int rc = check_grid(f->ny, f->nx, f->dx, "rb_li_compute_dt");
  if (rc) return rc;
  if (cur != 0 && cur != 1) return fail(RB_ERR_ARG, "rb_li_compute_dt: cur must be 0 or 1");
  if (!f->h[cur]) return fail(RB_ERR_ARG, "rb_li_compute_dt: missing depth buffer");
  cudaStream_t s = (cudaStream_t)stream;
  unsigned int* key = &header(ws)->red_key;
  if (f->chan_w && !f->chan_d) return fail(RB_ERR_ARG, "rb_li_compute_dt: chan_w given without chan_d");
  // local_inertial.py:529-539: the water column with channels armed, else h.
  RB_CUDA(rb::reduce_max_column(f->h[cur], f->chan_w, f->chan_d, (float)f->dx, (size_t)f->ny * f->nx, key, s),
          "rb_li_compute_dt reduce");
  unsigned int host_key = 0;
  RB_CUDA(cudaMemcpyAsync(&host_key, key, sizeof host_key, cudaMemcpyDeviceToHost, s), "rb_li_compute_dt copy");
  RB_CUDA(cudaStreamSynchronize(s), "rb_li_compute_dt sync");
  float hmax32;
  memcpy(&hmax32, &host_key, sizeof hmax32);
  // local_inertial.py:540-544, in host float64 as the reference computes it.
  const double h_max = (double)hmax32;
  if (h_max <= 1.0e-3) {
    *dt_out = dt_max;
    return RB_OK;
  }
  const double dt = alpha * f->dx / std::sqrt(9.81 * h_max);
  *dt_out = dt < dt_max ? dt : dt_max;
  return RB_OK;
}

static int hllc_params(const rb_hllc_fields* f, void* ws, rb::HllcParams& p, const char* who) {
  if (f == nullptr || ws == nullptr) return fail(RB_ERR_ARG, "%s: null argument", who);
  int rc = check_grid(f->ny, f->nx, f->dx, who);
  if (rc) return rc;
  if ((rc = check_bc(f->bc, true, who))) return rc;
  if (!f->h[0] || !f->h[1] || !f->hu[0] || !f->hu[1] || !f->hv[0] || !f->hv[1] || !f->z || !f->n)
    return fail(RB_ERR_ARG, "%s: missing state buffer", who);
  const bool banks = f->infil != nullptr || any_bc(f->bc, RB_BC_OPEN) || any_bc(f->bc, RB_BC_STAGE);
  const size_t cells = (size_t)f->ny * f->nx;
  char* u1 = (char*)ws + rb::ws_hllc_u1_offset(f->ny, f->nx);
  const size_t plane = align256(cells * sizeof(float));
  p = rb::HllcParams{};
  p.ny = f->ny;
  p.nx = f->nx;
  p.dx32 = (float)f->dx;
  p.z = f->z;
  p.n = f->n;
  p.h1 = (float*)u1;
  p.hu1 = (float*)(u1 + plane);
  p.hv1 = (float*)(u1 + 2 * plane);
  p.h_comp = f->h_comp;
  p.rain_field = f->rain_field;
  p.infil = f->infil;
  for (int e = 0; e < 4; e++) p.bc[e] = f->bc[e];
  for (int b = 0; b < 2; b++) {
    p.hb[b] = f->h[b];
    p.hub[b] = f->hu[b];
    p.hvb[b] = f->hv[b];
  }
  p.ledger = banks ? (double*)((char*)ws + rb::WS_LEDGER) : nullptr;
  p.err = &header(ws)->err;
  return RB_OK;
}

static int hllc_stage_impl(const rb_hllc_fields* f, int32_t cur, const rb_step_args* a, void* ws, void* stream,
                           int stage_mask) {
  if (a == nullptr) return fail(RB_ERR_ARG, "rb_hllc_step: null argument");
  rb::HllcParams p;
  int rc = hllc_params(f, ws, p, "rb_hllc_step");
  if (rc) return rc;
  if ((rc = check_dt(a->dt, "rb_hllc_step"))) return rc;
  if (cur != 0 && cur != 1) return fail(RB_ERR_ARG, "rb_hllc_step: cur must be 0 or 1");
  p.cur = cur;
  p.dt32 = (float)a->dt;
  p.rain32 = (float)a->rain;
  p.scale32 = (float)a->rain_scale;
  const bool comp = f->h_comp != nullptr;
  p.rain_mode = (comp && f->rain_field == nullptr) ? 1 : (a->rain != 0.0 ? 2 : 0);  // hllc.py:1350-1356
  for (int e = 0; e < 4; e++) p.stage[e] = (float)a->stage[e];
  p.wt = 0.5 * a->dt / f->dx;  // hllc.py:1320
  p.clk = nullptr;
  p.smax_key = nullptr;
  cudaStream_t s = (cudaStream_t)stream;
  if (stage_mask & 1) RB_CUDA(rb::hllc_stage_launch(p, 1, s), "rb_hllc_step stage 1");  // U^n -> U1
  if (stage_mask & 2) RB_CUDA(rb::hllc_stage_launch(p, 2, s), "rb_hllc_step stage 2");  // (U^n, U1) -> U^{n+1}
  return RB_OK;
}

int rb_hllc_step(const rb_hllc_fields* f, int32_t cur, const rb_step_args* a, void* ws, void* stream) {
  return hllc_stage_impl(f, cur, a, ws, stream, 3);
}

int rb_hllc_stage(const rb_hllc_fields* f, int32_t cur, const rb_step_args* a, void* ws, void* stream,
                  int32_t stage) {
  if (stage != 1 && stage != 2) return fail(RB_ERR_ARG, "rb_hllc_stage: stage must be 1 or 2");
  return hllc_stage_impl(f, cur, a, ws, stream, stage);
}

int rb_hllc_compute_dt(const rb_hllc_fields* f, int32_t cur, double alpha, double dt_max, void* ws, void* stream,
                       double* dt_out) {
  if (f == nullptr || ws == nullptr || dt_out == nullptr) return fail(RB_ERR_ARG, "rb_hllc_compute_dt: null argument");
  int rc = check_grid(f->ny, f->nx, f->dx, "rb_hllc_compute_dt");
  if (rc) return rc;
  if (cur != 0 && cur != 1) return fail(RB_ERR_ARG, "rb_hllc_compute_dt: cur must be 0 or 1");
  if (!f->h[cur] || !f->hu[cur] || !f->hv[cur]) return fail(RB_ERR_ARG, "rb_hllc_compute_dt: missing state buffer");
  cudaStream_t s = (cudaStream_t)stream;
  unsigned int* key = &header(ws)->red_key;
  RB_CUDA(rb::reduce_wavespeed(f->h[cur], f->hu[cur], f->hv[cur], (size_t)f->ny * f->nx, key, s),
          "rb_hllc_compute_dt reduce");
  unsigned int host_key = 0;
  RB_CUDA(cudaMemcpyAsync(&host_key, key, sizeof host_key, cudaMemcpyDeviceToHost, s), "rb_hllc_compute_dt copy");
  RB_CUDA(cudaStreamSynchronize(s), "rb_hllc_compute_dt sync");
  float smax32;
  memcpy(&smax32, &host_key, sizeof smax32);
  const double smax = (double)smax32;  // hllc.py:987-990
  if (smax <= 0.0) {
    *dt_out = dt_max;
    return RB_OK;
  }
  const double dt = alpha * f->dx / smax;
  *dt_out = dt < dt_max ? dt : dt_max;
  return RB_OK;
}

// --- device-resident clock ---------------------------------------------------
static int clock_start(int scheme, int ny, int nx, double dx, int32_t cur, const rb_clock_config* cfg, void* ws,
                       cudaStream_t s) {
  if (cfg == nullptr) return fail(RB_ERR_ARG, "clock start: null config");
  if (cur != 0 && cur != 1) return fail(RB_ERR_ARG, "clock start: cur must be 0 or 1");
  if (cfg->nsync < 0 || (cfg->nsync > 0 && cfg->sync == nullptr))
    return fail(RB_ERR_ARG, "clock start: nsync > 0 needs a device sync array");
  if (!(cfg->alpha > 0.0) || !(cfg->dt_max > 0.0)) return fail(RB_ERR_ARG, "clock start: alpha and dt_max must be > 0");
  rb::DevClock c{};
  c.t = cfg->t0;
  c.t1 = cfg->t0;
  c.t_target = cfg->t0;
  c.alpha = cfg->alpha;
  c.dt_max = cfg->dt_max;
  c.dx = dx;
  c.rain_rate = cfg->rain_rate;
  c.rain_until = cfg->rain_until;
  c.rain_field_sum = cfg->rain_field_sum;
  c.cell_area = dx * dx;
  c.n_cells = (double)ny * (double)nx;
  c.sync = cfg->sync;
  c.nsync = cfg->nsync;
  c.sync_pos = 0;
  c.scheme = scheme;
  c.rain_is_field = cfg->rain_is_field ? 1 : 0;
  c.cur = cur;
  c.limit = cfg->limit ? 1 : 0;
  if (cfg->nsrc < 0 || (cfg->nsrc > 0 && (!cfg->src_cell || !cfg->knot_off || !cfg->knot_t || !cfg->knot_q)))
    return fail(RB_ERR_ARG, "clock start: point sources need device cell, offset and knot arrays");
  c.nsrc = cfg->nsrc;
  c.src_cell = cfg->src_cell;
  c.knot_off = cfg->knot_off;
  c.knot_t = cfg->knot_t;
  c.knot_q = cfg->knot_q;
  c.src_comp = cfg->src_comp;
  for (int e = 0; e < 5; e++) {
    c.stage_off[e] = cfg->stage_off[e];
    if (e > 0 && cfg->stage_off[e] < cfg->stage_off[e - 1]) return fail(RB_ERR_ARG, "clock start: stage_off must be ascending");
  }
  if (c.stage_off[4] > c.stage_off[0] && (!cfg->stage_t || !cfg->stage_v))
    return fail(RB_ERR_ARG, "clock start: stage curves need device knot arrays");
  c.stage_t = cfg->stage_t;
  c.stage_v = cfg->stage_v;
  rb::DevClock* dc = &header(ws)->clock;
  RB_CUDA(cudaMemcpyAsync(dc, &c, sizeof c, cudaMemcpyHostToDevice, s), "clock start copy");
  RB_CUDA(cudaStreamSynchronize(s), "clock start sync");  // the source is a stack object
  return RB_OK;
}

int rb_li_clock_start(const rb_li_fields* f, int32_t cur, const rb_clock_config* cfg, void* ws, void* stream) {
  rb::LiParams p;
  int rc = li_params(f, ws, p, "rb_li_clock_start");
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  if ((rc = clock_start(0, f->ny, f->nx, f->dx, cur, cfg, ws, s))) return rc;
  RB_CUDA(rb::reduce_max_column(f->h[cur], f->chan_w, f->chan_d, (float)f->dx, (size_t)f->ny * f->nx,
                                &header(ws)->clock.red_key, s),
          "rb_li_clock_start");
  return RB_OK;
}

int rb_hllc_clock_start(const rb_hllc_fields* f, int32_t cur, const rb_clock_config* cfg, void* ws, void* stream) {
  rb::HllcParams p;
  int rc = hllc_params(f, ws, p, "rb_hllc_clock_start");
  if (rc) return rc;
  if (cfg == nullptr) return fail(RB_ERR_ARG, "rb_hllc_clock_start: null config");  // read just below
  for (int e = 0; e < 4; e++)
    if (f->bc[e] == RB_BC_STAGE && cfg->stage_off[e + 1] <= cfg->stage_off[e])
      return fail(RB_ERR_ARG, "rb_hllc_clock_start: fixed_stage edge %d has no stage curve", e);
  cudaStream_t s = (cudaStream_t)stream;
  rb::hllc_prepare_device();
  if ((rc = clock_start(1, f->ny, f->nx, f->dx, cur, cfg, ws, s))) return rc;
  RB_CUDA(rb::reduce_wavespeed(f->h[cur], f->hu[cur], f->hv[cur], (size_t)f->ny * f->nx, &header(ws)->clock.red_key,
                               s),
          "rb_hllc_clock_start");
  return RB_OK;
}

int rb_li_set_kernel_variant(int32_t variant) {
  if (!rb::li_set_kernel_variant(variant))
    return fail(RB_ERR_ARG, "rb_li_set_kernel_variant: variant %d is not in [0, %d)", variant,
                rb::li_kernel_variant_count());
  return RB_OK;
}

int rb_li_kernel_variants(int32_t* count) {
  if (count == nullptr) return fail(RB_ERR_ARG, "rb_li_kernel_variants: null argument");
  *count = rb::li_kernel_variant_count();
  return RB_OK;
}

int rb_set_arith_mode(int32_t mode) {
  if (mode != RB_ARITH_EXACT && mode != RB_ARITH_FAST)
    return fail(RB_ERR_ARG, "rb_set_arith_mode: mode %d is neither RB_ARITH_EXACT nor RB_ARITH_FAST", mode);
  g_arith_mode.store(mode);
  return RB_OK;
}

int rb_arith_mode(int32_t* mode) {
  if (mode == nullptr) return fail(RB_ERR_ARG, "rb_arith_mode: null argument");
  *mode = g_arith_mode.load();
  return RB_OK;
}

int rb_launch_config(int32_t* li_variant, int32_t* hllc_variant, int32_t* arith_mode) {
  if (li_variant == nullptr || hllc_variant == nullptr || arith_mode == nullptr)
    return fail(RB_ERR_ARG, "rb_launch_config: null argument");
  *li_variant = rb::li_current_variant();
  *hllc_variant = rb::hllc_current_variant();
  *arith_mode = g_arith_mode.load();
  return RB_OK;
}

int rb_hllc_set_kernel_variant(int32_t variant) {
  if (!rb::hllc_set_kernel_variant(variant))
    return fail(RB_ERR_ARG, "rb_hllc_set_kernel_variant: variant %d is not in [0, %d)", variant,
                rb::hllc_kernel_variant_count());
  return RB_OK;
}

int rb_hllc_kernel_variants(int32_t* count) {
  if (count == nullptr) return fail(RB_ERR_ARG, "rb_hllc_kernel_variants: null argument");
  *count = rb::hllc_kernel_variant_count();
  return RB_OK;
}

int rb_li_clock_reseed(const rb_li_fields* f, int32_t cur, void* ws, void* stream) {
  if (f == nullptr || ws == nullptr || !f->h[0] || !f->h[1]) return fail(RB_ERR_ARG, "rb_li_clock_reseed: null argument");
  int rc = check_grid(f->ny, f->nx, f->dx, "rb_li_clock_reseed");
  if (rc) return rc;
  if (cur != 0 && cur != 1) return fail(RB_ERR_ARG, "rb_li_clock_reseed: cur must be 0 or 1");
  if (f->chan_w && !f->chan_d) return fail(RB_ERR_ARG, "rb_li_clock_reseed: chan_w given without chan_d");
  RB_CUDA(rb::reduce_max_column(f->h[cur], f->chan_w, f->chan_d, (float)f->dx, (size_t)f->ny * f->nx,
                                &header(ws)->clock.red_key, (cudaStream_t)stream),
          "rb_li_clock_reseed");
  return RB_OK;
}

int rb_hllc_clock_reseed(const rb_hllc_fields* f, int32_t cur, void* ws, void* stream) {
  if (f == nullptr || ws == nullptr || !f->h[cur & 1] || !f->hu[cur & 1] || !f->hv[cur & 1])
    return fail(RB_ERR_ARG, "rb_hllc_clock_reseed: null argument");
  int rc = check_grid(f->ny, f->nx, f->dx, "rb_hllc_clock_reseed");
  if (rc) return rc;
  if (cur != 0 && cur != 1) return fail(RB_ERR_ARG, "rb_hllc_clock_reseed: cur must be 0 or 1");
  RB_CUDA(rb::reduce_wavespeed(f->h[cur], f->hu[cur], f->hv[cur], (size_t)f->ny * f->nx, &header(ws)->clock.red_key,
                               (cudaStream_t)stream),
          "rb_hllc_clock_reseed");
  return RB_OK;
}

int rb_clock_set_target(void* ws, double t_target, int32_t max_steps, void* stream) {
  if (ws == nullptr || max_steps < 0) return fail(RB_ERR_ARG, "rb_clock_set_target: bad argument");
  RB_CUDA(rb::clock_target_launch(&header(ws)->clock, t_target, max_steps, (cudaStream_t)stream), "rb_clock_set_target");
  return RB_OK;
}

int rb_clock_inflow(const float* h0, const float* h1, void* ws, void* stream) {
  if (ws == nullptr || h0 == nullptr || h1 == nullptr) return fail(RB_ERR_ARG, "rb_clock_inflow: null argument");
  float* hb[2] = {const_cast<float*>(h0), const_cast<float*>(h1)};
  RB_CUDA(rb::clock_inflow_launch(&header(ws)->clock, hb, (cudaStream_t)stream), "rb_clock_inflow");
  return RB_OK;
}

int rb_clock_plan(void* ws, void* stream) {
  if (ws == nullptr) return fail(RB_ERR_ARG, "rb_clock_plan: null workspace");
  RB_CUDA(rb::clock_plan_launch(&header(ws)->clock, (cudaStream_t)stream), "rb_clock_plan");
  return RB_OK;
}

int rb_hllc_stage_clocked(const rb_hllc_fields* f, int32_t stage, void* ws, void* stream) {
  if (stage != 1 && stage != 2) return fail(RB_ERR_ARG, "rb_hllc_stage_clocked: stage must be 1 or 2");
  rb::HllcParams p;
  int rc = hllc_params(f, ws, p, "rb_hllc_stage_clocked");
  if (rc) return rc;
  p.clk = &header(ws)->clock;
  p.smax_key = &header(ws)->clock.red_key;
  RB_CUDA(rb::hllc_stage_launch(p, stage, (cudaStream_t)stream), "rb_hllc_stage_clocked");
  return RB_OK;
}

int rb_li_enqueue_steps(const rb_li_fields* f, int32_t nsteps, int32_t with_sources, void* ws, void* stream) {
  if (nsteps < 0) return fail(RB_ERR_ARG, "rb_li_enqueue_steps: nsteps < 0");
  rb::LiParams p;
  int rc = li_params(f, ws, p, "rb_li_enqueue_steps");
  if (rc) return rc;
  p.clk = &header(ws)->clock;
  p.hmax_key = &header(ws)->clock.red_key;
  cudaStream_t s = (cudaStream_t)stream;
  for (int k = 0; k < nsteps; k++) {
    RB_CUDA(rb::clock_plan_launch(&header(ws)->clock, s), "rb_li_enqueue_steps plan");
    if (with_sources) RB_CUDA(rb::clock_inflow_launch(&header(ws)->clock, p.hb, s), "rb_li_enqueue_steps inflow");
    RB_CUDA(rb::li_step_launch(p, s), "rb_li_enqueue_steps step");
  }
  return RB_OK;
}

int rb_hllc_enqueue_steps(const rb_hllc_fields* f, int32_t nsteps, int32_t with_sources, void* ws, void* stream) {
  if (nsteps < 0) return fail(RB_ERR_ARG, "rb_hllc_enqueue_steps: nsteps < 0");
  rb::HllcParams p;
  int rc = hllc_params(f, ws, p, "rb_hllc_enqueue_steps");
  if (rc) return rc;
  p.clk = &header(ws)->clock;
  p.smax_key = &header(ws)->clock.red_key;
  cudaStream_t s = (cudaStream_t)stream;
  for (int k = 0; k < nsteps; k++) {
    RB_CUDA(rb::clock_plan_launch(&header(ws)->clock, s), "rb_hllc_enqueue_steps plan");
    if (with_sources) RB_CUDA(rb::clock_inflow_launch(&header(ws)->clock, p.hb, s), "rb_hllc_enqueue_steps inflow");
    RB_CUDA(rb::hllc_stage_launch(p, 1, s), "rb_hllc_enqueue_steps stage 1");
    RB_CUDA(rb::hllc_stage_launch(p, 2, s), "rb_hllc_enqueue_steps stage 2");
  }
  return RB_OK;
}

int rb_clock_read(void* ws, void* stream, rb_clock_state* out) {
  if (ws == nullptr || out == nullptr) return fail(RB_ERR_ARG, "rb_clock_read: null argument");
  cudaStream_t s = (cudaStream_t)stream;
  rb::DevClock* dc = &header(ws)->clock;
  RB_CUDA(rb::clock_commit_launch(dc, s), "rb_clock_read commit");
  rb::DevClock c;
  unsigned int err = 0;
  RB_CUDA(cudaMemcpyAsync(&c, dc, sizeof c, cudaMemcpyDeviceToHost, s), "rb_clock_read copy");
  RB_CUDA(cudaMemcpyAsync(&err, &header(ws)->err, sizeof err, cudaMemcpyDeviceToHost, s), "rb_clock_read err");
  RB_CUDA(cudaStreamSynchronize(s), "rb_clock_read sync");
  out->t = c.t;
  out->dt = c.dt;
  out->rain_volume = c.rain_in[0];
  out->inflow_volume = c.inflow_in[0];
  out->cur = c.cur;
  out->steps = c.steps;
  out->err = c.err | err;
  out->reserved = 0;
  return RB_OK;
}

// --- ensembles ----------------------------------------------------------------
static int64_t tiles_of(int ny, int nx, int tx, int ty) {
  return (int64_t)((nx + tx - 1) / tx) * (int64_t)((ny + ty - 1) / ty);
}

// A domain of at least this many 32 x 32 tiles fills the GPU by itself: it is stepped
// by the single-domain kernels, launched for it alone inside the ensemble's step,
// instead of by the persistent (domain, tile) kernel. Measured on B200 (exact build,
// Gcell-updates/s, persistent vs single-domain kernel): LI 2048^2 27.6 vs 35.4, 1024^2
// 27.1 vs 30.0, 512^2 25.5 vs 14.1; HLLC 2048^2 9.9 vs 13.7, 1024^2 9.6 vs 12.1, 512^2
// 9.2 vs 8.0.
constexpr int64_t kEnsSoloTiles = 1024;

// The single-domain launch parameters of an ensemble's large domains, by ensemble
// buffer (kernel parameters are passed by value, so the host keeps them).
struct EnsSolo {
  std::vector<rb::LiParams> li;
  std::vector<rb::HllcParams> hllc;
};
static std::mutex g_ens_solo_mu;
static std::unordered_map<const void*, EnsSolo> g_ens_solo;

int rb_ensemble_layout_make(int32_t ndom, const int32_t* scheme, const int32_t* ny, const int32_t* nx,
                            int32_t li_variant, int32_t hllc_variant, rb_ensemble_layout* out) {
  if (ndom < 1 || !scheme || !ny || !nx || !out) return fail(RB_ERR_ARG, "rb_ensemble_layout_make: bad argument");
  if (li_variant < 0 || li_variant > 3 || hllc_variant < 0 || hllc_variant > 2)
    return fail(RB_ERR_ARG, "rb_ensemble_layout_make: unknown tile variant");
  rb_ensemble_layout L{};
  L.ndom = ndom;
  L.li_variant = li_variant;
  L.hllc_variant = hllc_variant;
  int ltx, lty, htx, hty;
  rb::li_variant_tile(li_variant, &ltx, &lty);
  rb::hllc_variant_tile(hllc_variant, &htx, &hty);
  for (int d = 0; d < ndom; d++) {
    if (ny[d] < 1 || nx[d] < 1) return fail(RB_ERR_ARG, "rb_ensemble_layout_make: domain %d has an empty grid", d);
    if (scheme[d] == 0) {
      L.n_li++;
      L.li_tiles += tiles_of(ny[d], nx[d], ltx, lty);
    } else if (scheme[d] == 1) {
      L.n_hllc++;
      L.hllc_tiles += tiles_of(ny[d], nx[d], htx, hty);
    } else {
      return fail(RB_ERR_ARG, "rb_ensemble_layout_make: domain %d has unknown scheme %d", d, scheme[d]);
    }
  }
  size_t off = 256;
  L.off_clocks = (int64_t)off;
  off += align256((size_t)ndom * sizeof(rb::DevClock));
  L.off_li = (int64_t)off;
  off += align256((size_t)L.n_li * sizeof(rb::LiParams));
  L.off_hllc = (int64_t)off;
  off += align256((size_t)L.n_hllc * sizeof(rb::HllcParams));
  L.off_map_li = (int64_t)off;
  off += align256((size_t)L.li_tiles * sizeof(int2));
  L.off_map_hllc = (int64_t)off;
  off += align256((size_t)L.hllc_tiles * sizeof(int2));
  L.off_targets = (int64_t)off;
  off += align256((size_t)ndom * (sizeof(double) + sizeof(int32_t)));
  L.bytes = (int64_t)off;
  *out = L;
  return RB_OK;
}

int rb_ensemble_init(rb_ensemble_layout* L, void* ens, const int32_t* scheme, const rb_li_fields* li,
                     const rb_hllc_fields* hl, void* const* dom_ws, const rb_clock_config* cfg, const int32_t* cur,
                     void* stream) {
  if (!L || !ens || !scheme || !dom_ws || !cfg || !cur) return fail(RB_ERR_ARG, "rb_ensemble_init: null argument");
  if ((L->n_li > 0 && !li) || (L->n_hllc > 0 && !hl)) return fail(RB_ERR_ARG, "rb_ensemble_init: missing fields");
  // The layout sizes every host vector and device area below: it must be the one
  // rb_ensemble_layout_make made for this scheme array.
  if (L->ndom < 1 || L->n_li < 0 || L->n_hllc < 0 || L->n_li + L->n_hllc != L->ndom || L->li_variant < 0 ||
      L->li_variant > 3 || L->hllc_variant < 0 || L->hllc_variant > 2)
    return fail(RB_ERR_ARG, "rb_ensemble_init: the layout is not one rb_ensemble_layout_make made");
  {
    int32_t n_li = 0, n_hllc = 0;
    for (int d = 0; d < L->ndom; d++) {
      if (scheme[d] != 0 && scheme[d] != 1)
        return fail(RB_ERR_ARG, "rb_ensemble_init: domain %d has unknown scheme %d", d, scheme[d]);
      if (cur[d] != 0 && cur[d] != 1) return fail(RB_ERR_ARG, "rb_ensemble_init: domain %d: cur must be 0 or 1", d);
      (scheme[d] == 0 ? n_li : n_hllc)++;
    }
    if (n_li != L->n_li || n_hllc != L->n_hllc)
      return fail(RB_ERR_ARG, "rb_ensemble_init: the scheme array does not match the layout");
  }
  cudaStream_t s = (cudaStream_t)stream;
  char* base = (char*)ens;
  rb::DevClock* clocks = (rb::DevClock*)(base + L->off_clocks);
  std::vector<rb::DevClock> hc(L->ndom);
  std::vector<rb::LiParams> hli(L->n_li);
  std::vector<rb::HllcParams> hhl(L->n_hllc);
  std::vector<int2> mli, mhl;
  mli.reserve((size_t)L->li_tiles);
  mhl.reserve((size_t)L->hllc_tiles);
  int ltx, lty, htx, hty;
  rb::li_variant_tile(L->li_variant, &ltx, &lty);
  rb::hllc_variant_tile(L->hllc_variant, &htx, &hty);
  EnsSolo solo;
  int ili = 0, ihl = 0;
  for (int d = 0; d < L->ndom; d++) {
    if (!dom_ws[d]) return fail(RB_ERR_ARG, "rb_ensemble_init: domain %d has no workspace", d);
    int rc;
    rb::DevClock c{};
    const rb_clock_config& k = cfg[d];
    int ny, nx;
    double dx;
    if (scheme[d] == 0) {
      const rb_li_fields& f = li[ili];
      if ((rc = li_params(&f, dom_ws[d], hli[ili], "rb_ensemble_init"))) return rc;
      if (f.chan_w != nullptr)
        return fail(RB_ERR_ARG, "rb_ensemble_init: domain %d: sub-grid channels are stepped one domain at a time "
                    "(rb_li_step / rb_li_enqueue_steps)", d);
      hli[ili].clk = &clocks[d];
      hli[ili].hmax_key = &clocks[d].red_key;
      ny = f.ny, nx = f.nx, dx = f.dx;
      if (tiles_of(ny, nx, 32, 32) >= kEnsSoloTiles) {
        solo.li.push_back(hli[ili]);
      } else {
        const int64_t nt = tiles_of(ny, nx, ltx, lty);
        for (int64_t t = 0; t < nt; t++) mli.push_back(make_int2(ili, (int)t));
      }
      ili++;
    } else {
      const rb_hllc_fields& f = hl[ihl];
      if ((rc = hllc_params(&f, dom_ws[d], hhl[ihl], "rb_ensemble_init"))) return rc;
      hhl[ihl].clk = &clocks[d];
      hhl[ihl].smax_key = &clocks[d].red_key;
      ny = f.ny, nx = f.nx, dx = f.dx;
      if (tiles_of(ny, nx, 32, 32) >= kEnsSoloTiles) {
        solo.hllc.push_back(hhl[ihl]);
      } else {
        const int64_t nt = tiles_of(ny, nx, htx, hty);
        for (int64_t t = 0; t < nt; t++) mhl.push_back(make_int2(ihl, (int)t));
      }
      ihl++;
    }
    if (!(k.alpha > 0.0) || !(k.dt_max > 0.0)) return fail(RB_ERR_ARG, "rb_ensemble_init: domain %d alpha/dt_max", d);
    if (k.nsrc != 0 || k.stage_off[4] != k.stage_off[0])
      return fail(RB_ERR_ARG, "rb_ensemble_init: domain %d: ensembles step rain and fields only (no point "
                  "sources or stage curves)", d);
    c.t = c.t1 = c.t_target = k.t0;
    c.alpha = k.alpha;
    c.dt_max = k.dt_max;
    c.dx = dx;
    c.rain_rate = k.rain_rate;
    c.rain_until = k.rain_until;
    c.rain_field_sum = k.rain_field_sum;
    c.cell_area = dx * dx;
    c.n_cells = (double)ny * (double)nx;
    c.sync = k.sync;
    c.nsync = k.nsync;
    c.scheme = scheme[d];
    c.rain_is_field = k.rain_is_field ? 1 : 0;
    c.cur = cur[d];
    c.limit = k.limit ? 1 : 0;
    hc[d] = c;
  }
  if ((int64_t)mli.size() > L->li_tiles || (int64_t)mhl.size() > L->hllc_tiles)
    return fail(RB_ERR_ARG, "rb_ensemble_init: the domains have more tiles than the layout was made for");
  // the persistent kernels walk the small domains' tiles only
  L->li_tiles = (int64_t)mli.size();
  L->hllc_tiles = (int64_t)mhl.size();
  {
    std::lock_guard<std::mutex> lock(g_ens_solo_mu);
    g_ens_solo[ens] = std::move(solo);
  }
  L->li_grid = rb::ens_li_grid_size(L->li_variant);
  L->hllc_grid = rb::ens_hllc_grid_size(L->hllc_variant);
  if (L->n_hllc > 0 && L->hllc_grid < 1)
    return fail(RB_ERR_CUDA, "rb_ensemble_init: the device cannot run HLLC tile variant %d (shared memory)",
                L->hllc_variant);
  RB_CUDA(cudaMemcpyAsync(clocks, hc.data(), hc.size() * sizeof(rb::DevClock), cudaMemcpyHostToDevice, s), "ens clocks");
  if (!hli.empty())
    RB_CUDA(cudaMemcpyAsync(base + L->off_li, hli.data(), hli.size() * sizeof(rb::LiParams), cudaMemcpyHostToDevice, s),
            "ens li");
  if (!hhl.empty())
    RB_CUDA(cudaMemcpyAsync(base + L->off_hllc, hhl.data(), hhl.size() * sizeof(rb::HllcParams),
                            cudaMemcpyHostToDevice, s),
            "ens hllc");
  if (!mli.empty())
    RB_CUDA(cudaMemcpyAsync(base + L->off_map_li, mli.data(), mli.size() * sizeof(int2), cudaMemcpyHostToDevice, s),
            "ens map li");
  if (!mhl.empty())
    RB_CUDA(cudaMemcpyAsync(base + L->off_map_hllc, mhl.data(), mhl.size() * sizeof(int2), cudaMemcpyHostToDevice, s),
            "ens map hllc");
  // seed each domain's compute_dt reduction from its current state
  ili = ihl = 0;
  for (int d = 0; d < L->ndom; d++) {
    if (scheme[d] == 0) {
      const rb_li_fields& f = li[ili++];
      RB_CUDA(rb::reduce_max_h(f.h[cur[d]], (size_t)f.ny * f.nx, &clocks[d].red_key, s), "ens seed");
    } else {
      const rb_hllc_fields& f = hl[ihl++];
      RB_CUDA(rb::reduce_wavespeed(f.h[cur[d]], f.hu[cur[d]], f.hv[cur[d]], (size_t)f.ny * f.nx, &clocks[d].red_key, s),
              "ens seed");
    }
  }
  RB_CUDA(cudaStreamSynchronize(s), "rb_ensemble_init sync");  // host vectors are the copy sources
  return RB_OK;
}

int rb_ensemble_set_targets(const rb_ensemble_layout* L, void* ens, const double* t_target, const int32_t* max_steps,
                            void* stream) {
  if (!L || !ens || !t_target || !max_steps) return fail(RB_ERR_ARG, "rb_ensemble_set_targets: null argument");
  cudaStream_t s = (cudaStream_t)stream;
  char* base = (char*)ens;
  double* dt_t = (double*)(base + L->off_targets);
  int* dm = (int*)(base + L->off_targets + (int64_t)L->ndom * (int64_t)sizeof(double));
  RB_CUDA(cudaMemcpyAsync(dt_t, t_target, (size_t)L->ndom * sizeof(double), cudaMemcpyHostToDevice, s), "targets");
  RB_CUDA(cudaMemcpyAsync(dm, max_steps, (size_t)L->ndom * sizeof(int32_t), cudaMemcpyHostToDevice, s), "targets");
  RB_CUDA(rb::clock_target_many_launch((rb::DevClock*)(base + L->off_clocks), L->ndom, dt_t, dm, s), "targets");
  RB_CUDA(cudaStreamSynchronize(s), "rb_ensemble_set_targets sync");
  return RB_OK;
}

int rb_ensemble_enqueue(const rb_ensemble_layout* L, void* ens, int32_t nsteps, void* stream) {
  if (!L || !ens || nsteps < 0) return fail(RB_ERR_ARG, "rb_ensemble_enqueue: bad argument");
  cudaStream_t s = (cudaStream_t)stream;
  char* base = (char*)ens;
  rb::DevClock* clocks = (rb::DevClock*)(base + L->off_clocks);
  const rb::LiParams* P = (const rb::LiParams*)(base + L->off_li);
  const rb::HllcParams* Q = (const rb::HllcParams*)(base + L->off_hllc);
  const int2* mli = (const int2*)(base + L->off_map_li);
  const int2* mhl = (const int2*)(base + L->off_map_hllc);
  EnsSolo solo;
  {
    std::lock_guard<std::mutex> lock(g_ens_solo_mu);
    auto it = g_ens_solo.find(ens);
    if (it == g_ens_solo.end()) return fail(RB_ERR_ARG, "rb_ensemble_enqueue: the ensemble was not initialised");
    solo = it->second;
  }
  const int li_v = rb::li_current_variant(), hl_v = rb::hllc_current_variant();
  for (int k = 0; k < nsteps; k++) {
    RB_CUDA(rb::clock_plan_many_launch(clocks, L->ndom, s), "ens plan");
    for (const rb::LiParams& p : solo.li) RB_CUDA(rb::li_step_launch_variant(p, li_v, s), "ens li, large domain");
    RB_CUDA(rb::ens_li_launch(L->li_variant, L->li_grid, P, mli, L->li_tiles, s), "ens li");
    for (const rb::HllcParams& p : solo.hllc)
      RB_CUDA(rb::hllc_stage_launch_exact(p, 1, hl_v, s), "ens hllc 1, large domain");
    RB_CUDA(rb::ens_hllc_launch(L->hllc_variant, L->hllc_grid, 1, Q, mhl, L->hllc_tiles, s), "ens hllc 1");
    for (const rb::HllcParams& p : solo.hllc)
      RB_CUDA(rb::hllc_stage_launch_exact(p, 2, hl_v, s), "ens hllc 2, large domain");
    RB_CUDA(rb::ens_hllc_launch(L->hllc_variant, L->hllc_grid, 2, Q, mhl, L->hllc_tiles, s), "ens hllc 2");
  }
  return RB_OK;
}

int rb_ensemble_read(const rb_ensemble_layout* L, void* ens, rb_clock_state* out, void* stream) {
  if (!L || !ens || !out) return fail(RB_ERR_ARG, "rb_ensemble_read: null argument");
  cudaStream_t s = (cudaStream_t)stream;
  rb::DevClock* clocks = (rb::DevClock*)((char*)ens + L->off_clocks);
  RB_CUDA(rb::clock_commit_many_launch(clocks, L->ndom, s), "ens commit");
  std::vector<rb::DevClock> hc(L->ndom);
  RB_CUDA(cudaMemcpyAsync(hc.data(), clocks, hc.size() * sizeof(rb::DevClock), cudaMemcpyDeviceToHost, s), "ens read");
  RB_CUDA(cudaStreamSynchronize(s), "rb_ensemble_read sync");
  for (int d = 0; d < L->ndom; d++) {
    out[d].t = hc[d].t;
    out[d].dt = hc[d].dt;
    out[d].rain_volume = hc[d].rain_in[0];
    out[d].inflow_volume = hc[d].inflow_in[0];
    out[d].cur = hc[d].cur;
    out[d].steps = hc[d].steps;
    out[d].err = hc[d].err;
    out[d].reserved = 0;
  }
  return RB_OK;
}

int rb_inject_points(float* h, int32_t ny, int32_t nx, int32_t nsrc, const int32_t* rows, const int32_t* cols,
                     const float* add_depth, float* comp, void* stream) {
  if (ny < 1 || nx < 1 || nsrc < 0) return fail(RB_ERR_ARG, "rb_inject_points: bad sizes");
  if (nsrc == 0) return RB_OK;
  if (!h || !rows || !cols || !add_depth) return fail(RB_ERR_ARG, "rb_inject_points: null argument");
  RB_CUDA(rb::inject_points(h, ny, nx, nsrc, rows, cols, add_depth, comp, (cudaStream_t)stream), "rb_inject_points");
  return RB_OK;
}

static int check_box(int32_t ny, int32_t nx, int32_t r0, int32_t c0, int32_t r1, int32_t c1, const char* who) {
  if (ny < 1 || nx < 1) return fail(RB_ERR_ARG, "%s: bad grid %d x %d", who, ny, nx);
  if (!(0 <= r0 && r0 <= r1 && r1 < ny && 0 <= c0 && c0 <= c1 && c1 < nx))
    return fail(RB_ERR_ARG, "%s: box (%d, %d, %d, %d) is outside the %d x %d grid", who, r0, c0, r1, c1, ny, nx);
  return RB_OK;
}

int rb_reservoir_withdraw(float* h, int32_t ny, int32_t nx, int32_t r0, int32_t c0, int32_t r1, int32_t c1,
                          float scale, double* taken, void* stream) {
  int rc = check_box(ny, nx, r0, c0, r1, c1, "rb_reservoir_withdraw");
  if (rc) return rc;
  if (!h || !taken) return fail(RB_ERR_ARG, "rb_reservoir_withdraw: null argument");
  if (!(scale >= 0.0f && scale <= 1.0f)) return fail(RB_ERR_ARG, "rb_reservoir_withdraw: scale must be in [0, 1]");
  RB_CUDA(rb::reservoir_withdraw(h, nx, r0, c0, r1 - r0 + 1, c1 - c0 + 1, scale, taken, (cudaStream_t)stream),
          "rb_reservoir_withdraw");
  return RB_OK;
}

int rb_reservoir_deliver(float* h, int32_t ny, int32_t nx, int32_t r0, int32_t c0, int32_t r1, int32_t c1,
                         double add_depth, void* ws, void* stream) {
  int rc = check_box(ny, nx, r0, c0, r1, c1, "rb_reservoir_deliver");
  if (rc) return rc;
  if (!h || !ws) return fail(RB_ERR_ARG, "rb_reservoir_deliver: null argument");
  if (!(add_depth >= 0.0) || !std::isfinite(add_depth))
    return fail(RB_ERR_ARG, "rb_reservoir_deliver: add_depth must be finite and >= 0");
  double* slot0 = (double*)((char*)ws + rb::WS_LEDGER);  // ledger slot 0 of the domain's workspace
  RB_CUDA(rb::reservoir_deliver(h, nx, r0, c0, r1 - r0 + 1, c1 - c0 + 1, add_depth, slot0, (cudaStream_t)stream),
          "rb_reservoir_deliver");
  return RB_OK;
}

int rb_exner_apply(int32_t ny, int32_t nx, double dx, float* qs_int_x, float* qs_int_y, const float* dz_lo,
                   const float* dz_hi, float inv_one_minus_p, double* dz_cum, double* dz_unapplied, const float* z0,
                   float* z, void* stream) {
  int rc = check_grid(ny, nx, dx, "rb_exner_apply");
  if (rc) return rc;
  if (!qs_int_x || !qs_int_y || !dz_lo || !dz_hi || !dz_cum || !dz_unapplied || !z0 || !z)
    return fail(RB_ERR_ARG, "rb_exner_apply: null argument");
  RB_CUDA(rb::exner_apply(ny, nx, (float)dx, inv_one_minus_p, qs_int_x, qs_int_y, dz_lo, dz_hi, dz_cum,
                          dz_unapplied, z0, z, (cudaStream_t)stream),
          "rb_exner_apply");
  return RB_OK;
}

int rb_ledger_loss(void* ws, int32_t ny, int32_t nx, void* stream, double* out) {
  if (ws == nullptr || out == nullptr) return fail(RB_ERR_ARG, "rb_ledger_loss: null argument");
  if (ny < 1 || nx < 1) return fail(RB_ERR_ARG, "rb_ledger_loss: bad grid %d x %d", ny, nx);
  cudaStream_t s = (cudaStream_t)stream;
  const size_t nslots = rb::ws_ledger_bytes(ny, nx) / (2 * sizeof(double));
  const double* ledger = (const double*)((char*)ws + rb::WS_LEDGER);
  double* partials = (double*)((char*)ws + rb::WS_PARTIALS);
  double* res = &header(ws)->sum;
  RB_CUDA(rb::sum_ledger(ledger, nslots, partials, res, s), "rb_ledger_loss");
  RB_CUDA(cudaMemcpyAsync(out, res, sizeof(double), cudaMemcpyDeviceToHost, s), "rb_ledger_loss copy");
  RB_CUDA(cudaStreamSynchronize(s), "rb_ledger_loss sync");
  return RB_OK;
}

int rb_sum_f64(const float* x, int64_t n, void* ws, size_t ws_bytes, void* stream, double* out) {
  if (x == nullptr || ws == nullptr || out == nullptr || n < 0 || ws_bytes < rb::WS_LEDGER)
    return fail(RB_ERR_ARG, "rb_sum_f64: bad argument");
  cudaStream_t s = (cudaStream_t)stream;
  double* partials = (double*)((char*)ws + rb::WS_PARTIALS);
  double* res = &header(ws)->sum;
  RB_CUDA(rb::sum_f64(x, (size_t)n, partials, res, s), "rb_sum_f64");
  RB_CUDA(cudaMemcpyAsync(out, res, sizeof(double), cudaMemcpyDeviceToHost, s), "rb_sum_f64 copy");
  RB_CUDA(cudaStreamSynchronize(s), "rb_sum_f64 sync");
  return RB_OK;
}

int rb_read_device_error(void* ws, void* stream, uint32_t* err_out) {
  if (ws == nullptr || err_out == nullptr) return fail(RB_ERR_ARG, "rb_read_device_error: null argument");
  cudaStream_t s = (cudaStream_t)stream;
  unsigned int host = 0;
  RB_CUDA(cudaMemcpyAsync(&host, &header(ws)->err, sizeof host, cudaMemcpyDeviceToHost, s), "rb_read_device_error");
  RB_CUDA(cudaMemsetAsync(&header(ws)->err, 0, sizeof(unsigned int), s), "rb_read_device_error clear");
  RB_CUDA(cudaStreamSynchronize(s), "rb_read_device_error sync");
  *err_out = host;
  return RB_OK;
}

}  // extern "C"
