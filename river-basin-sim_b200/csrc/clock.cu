// clock.cu -- the device-resident simulated clock.
//
// The reference advances one step per Python iteration (solver/run.py:369-388):
// scheme.compute_dt reads max(h) (or the max wave speed) back to the host, the
// scheduler (solver/scheduler.py:171-246) clamps it with fill_span to the next
// sync point, the run loop gates rain on `t < rain_duration - EPS_T` and banks
// the rain volume in the float64 ledger. Here one single-thread "plan" kernel
// does all of that in float64 on the device, reading the max the previous step
// kernel folded into the clock, so K steps run back to back (and can be captured
// in a CUDA graph) with no host round trip. Same float64 operations in the same
// order as the reference's Python, so the step sequence is bit-identical to the
// host-driven loop.
//
// Termination is bounded by construction: a plan kernel plans a step only while
// t < t_target - EPS_T and fewer than max_steps steps were taken since the span
// was set; otherwise it clears `active` and every later kernel of the graph
// returns at its first instruction. There are no device-side waits.
#include <cmath>

#include "rb_common.cuh"
#include "rb_kernels.h"

namespace rb {

constexpr double kEpsT = 1e-6;  // solver/scheduler.py:45 EPS_T

// scheduler.py:48-72 fill_span
__device__ __forceinline__ double fill_span(double span, double dt_raw) {
  if (!isfinite(span)) return dt_raw;
  if (span <= dt_raw) return span;
  const double n = ceil(span / dt_raw);
  const double dt = span / n;
  if (dt > dt_raw) return span / (n + 1.0);
  return dt;
}

// boundaries.py:199-220 stage_at: piecewise linear, held (not zeroed) outside.
__device__ double stage_at(const double* tk, const double* vk, int n, double t) {
  if (t <= tk[0]) return vk[0];
  if (t >= tk[n - 1]) return vk[n - 1];
  for (int i = 0; i + 1 < n; i++) {
    if (tk[i] <= t && t <= tk[i + 1]) {
      if (tk[i + 1] == tk[i]) return vk[i + 1];
      return vk[i] + (vk[i + 1] - vk[i]) * (t - tk[i]) / (tk[i + 1] - tk[i]);
    }
  }
  return vk[n - 1];
}

// config.py:111-122 Inflow.discharge_at: piecewise linear, zero outside.
__device__ double discharge_at(const double* tk, const double* qk, int n, double t) {
  if (n == 0 || t < tk[0] || t > tk[n - 1]) return 0.0;
  for (int i = 0; i + 1 < n; i++) {
    if (tk[i] <= t && t <= tk[i + 1]) {
      if (tk[i + 1] == tk[i]) return qk[i + 1];
      return qk[i] + (qk[i + 1] - qk[i]) * (t - tk[i]) / (tk[i + 1] - tk[i]);
    }
  }
  return qk[n - 1];
}

__device__ __forceinline__ void kahan64(double* acc, double x) {
  const double y = x - acc[1];
  const double t = acc[0] + y;
  acc[1] = (t - acc[0]) - y;
  acc[0] = t;
}

__device__ __forceinline__ void commit(DevClock* c) {
  if (c->pending) {
    c->t = c->t1;
    c->cur ^= 1;
    c->steps += 1;
    c->pending = 0;
  }
}

// steps + budget, saturated at INT_MAX (a budget of INT_MAX means "no limit").
__device__ __forceinline__ int step_limit(int steps, int budget) {
  const long long m = (long long)steps + (long long)(budget < 0 ? 0 : budget);
  return m > 2147483647LL ? 2147483647 : (int)m;
}

__device__ void clock_plan(DevClock* c) {
  commit(c);
  c->active = 0;
  const double t = c->t;
  if (t >= c->t_target - kEpsT) return;
  if (c->steps >= c->max_steps) return;  // the span's step budget is spent
  // compute_dt: local_inertial.py:540-544 / hllc.py:987-990
  const double m = (double)__uint_as_float(c->red_key);
  double dt_raw;
  if (c->scheme == 0) {
    if (m <= 1.0e-3) {
      dt_raw = c->dt_max;
    } else {
      const double d = c->alpha * c->dx / sqrt(9.81 * m);
      dt_raw = d < c->dt_max ? d : c->dt_max;
    }
  } else {
    if (m <= 0.0) {
      dt_raw = c->dt_max;
    } else {
      const double d = c->alpha * c->dx / m;
      dt_raw = d < c->dt_max ? d : c->dt_max;
    }
  }
  if (!(dt_raw > 0.0)) {  // scheduler.py:221-224
    c->err |= RB_DEVERR_CLOCK;
    return;
  }
  // scheduler.py:165-168 next_sync over the ascending sync list, then :225 fill_span
  int k = c->sync_pos;
  while (k < c->nsync && !(c->sync[k] > t + kEpsT)) k++;
  c->sync_pos = k;
  const double dt = k < c->nsync ? fill_span(c->sync[k] - t, dt_raw) : dt_raw;
  if (!(dt > 0.0)) {
    c->err |= RB_DEVERR_CLOCK;
    return;
  }
  // run.py:378-388: rain while t < rain_duration - EPS_T, banked in the ledger
  const bool raining = t < c->rain_until - kEpsT;
  double rain = 0.0;
  float scale = 0.0f;
  if (c->rain_is_field) {
    scale = raining ? 1.0f : 0.0f;
    if (raining) kahan64(c->rain_in, c->rain_field_sum * dt * c->cell_area);
  } else {
    rain = raining ? c->rain_rate : 0.0;
    if (rain > 0.0) kahan64(c->rain_in, rain * dt * c->cell_area * c->n_cells);
  }
  c->dt = dt;
  c->t1 = t + dt;
  c->dt32 = (float)dt;
  c->dxdt32 = (float)(dt / c->dx);  // boundaries.py:329
  c->wt = 0.5 * dt / c->dx;         // hllc.py:1320
  c->rain32 = (float)rain;
  c->scale32 = scale;
  for (int e = 0; e < 4; e++) {  // hllc.py:1308-1312, once per step at the midpoint
    const int a = c->stage_off[e], b = c->stage_off[e + 1];
    c->stage32[e] = b > a ? (float)stage_at(c->stage_t + a, c->stage_v + a, b - a, t + 0.5 * dt) : 0.0f;
  }
  c->red_key = 0u;  // the step kernel folds max(h) / max wave speed of its output here
  c->active = 1;
  c->pending = 1;
}

__global__ void clock_plan_kernel(DevClock* c) {
  pdl_enter();
  clock_plan(c);
}

// One plan per domain of an ensemble (each domain has its own clock).
__global__ void clock_plan_many_kernel(DevClock* clocks, int n) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d < n) clock_plan(&clocks[d]);
}

__global__ void clock_commit_many_kernel(DevClock* clocks, int n) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d < n) {
    commit(&clocks[d]);
    clocks[d].active = 0;
  }
}

__global__ void clock_target_many_kernel(DevClock* clocks, int n, const double* t_target, const int* max_steps) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d < n) {
    DevClock* c = &clocks[d];
    commit(c);
    c->active = 0;
    c->t_target = t_target[d];
    c->max_steps = step_limit(c->steps, max_steps[d]);
  }
}

cudaError_t clock_plan_many_launch(DevClock* clocks, int n, cudaStream_t s) {
  clock_plan_many_kernel<<<(n + 127) / 128, 128, 0, s>>>(clocks, n);
  return cudaGetLastError();
}

cudaError_t clock_commit_many_launch(DevClock* clocks, int n, cudaStream_t s) {
  clock_commit_many_kernel<<<(n + 127) / 128, 128, 0, s>>>(clocks, n);
  return cudaGetLastError();
}

cudaError_t clock_target_many_launch(DevClock* clocks, int n, const double* t_target, const int* max_steps,
                                     cudaStream_t s) {
  clock_target_many_kernel<<<(n + 127) / 128, 128, 0, s>>>(clocks, n, t_target, max_steps);
  return cudaGetLastError();
}

__global__ void clock_commit_kernel(DevClock* c) {
  commit(c);
  c->active = 0;
}

__global__ void clock_target_kernel(DevClock* c, double t_target, int max_steps) {
  commit(c);
  c->active = 0;
  c->t_target = t_target;
  c->max_steps = step_limit(c->steps, max_steps);
}

// inflow.py:167-200 InflowInjector.apply for the planned step: midpoint discharge,
// float32 depth request Q*dt/A per source, Kahan add into the cell (sources are
// distinct cells), and the float64 sum of the requests banked into the ledger.
constexpr int INFLOW_NT = 256;
__global__ void __launch_bounds__(INFLOW_NT) clock_inflow_kernel(DevClock* c, float* h0, float* h1) {
  if (!c->active) return;
  __shared__ float s_add[INFLOW_NT];
  const double t_mid = c->t + 0.5 * c->dt;
  float* h = c->cur ? h1 : h0;
  double total = 0.0;
  for (int base = 0; base < c->nsrc; base += INFLOW_NT) {
    const int k = base + threadIdx.x;
    float add = 0.0f;
    if (k < c->nsrc) {
      const int a = c->knot_off[k], b = c->knot_off[k + 1];
      const double vol = discharge_at(c->knot_t + a, c->knot_q + a, b - a, t_mid) * c->dt;
      add = (float)(vol / c->cell_area);
      const int cell = c->src_cell[k];
      if (cell < 0 || (double)cell >= c->n_cells) {
        add = 0.0f;  // a source outside the grid adds, and banks, nothing
      } else if (c->src_comp != nullptr) {
        float tot = h[cell], cp = c->src_comp[k];
        kahan_add(tot, cp, add);
        h[cell] = tot;
        c->src_comp[k] = cp;
      } else {
        h[cell] = h[cell] + add;
      }
    }
    s_add[threadIdx.x] = add;
    __syncthreads();
    if (threadIdx.x == 0) {
      const int m = min(INFLOW_NT, c->nsrc - base);
      for (int i = 0; i < m; i++) total += (double)s_add[i];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) kahan64(c->inflow_in, total * c->cell_area);
}

cudaError_t clock_inflow_launch(DevClock* clk, float* const* hb, cudaStream_t s) {
  clock_inflow_kernel<<<1, INFLOW_NT, 0, s>>>(clk, hb[0], hb[1]);
  return cudaGetLastError();
}

cudaError_t clock_plan_launch(DevClock* clk, cudaStream_t s) {
  return launch_chain(clock_plan_kernel, dim3(1), dim3(1), 0, s, clk);
}

cudaError_t clock_commit_launch(DevClock* clk, cudaStream_t s) {
  clock_commit_kernel<<<1, 1, 0, s>>>(clk);
  return cudaGetLastError();
}

cudaError_t clock_target_launch(DevClock* clk, double t_target, int max_steps, cudaStream_t s) {
  clock_target_kernel<<<1, 1, 0, s>>>(clk, t_target, max_steps);
  return cudaGetLastError();
}

}  // namespace rb
