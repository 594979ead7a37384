// rb_common.cuh -- shared device helpers for the river-basin solver kernels.
//
// Arithmetic contract (identical to the CPU oracle): every kernel is compiled with
// --fmad=false and IEEE division/square root, so each operation rounds once in
// the reference's expression order; the fractional powers come from
// include/rb_detmath.h. `rmax/rmin/rclamp` are the scalar builtins of the
// reference's kernel language (a > b ? a : b, a < b ? a : b, min(max(lo,x),hi)),
// which differ from fmaxf/fminf on signed zeros.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "rb_detmath.h"
#include "rbsim.h"

namespace rb {

constexpr float kG = 9.81f;     // solver/core/grid.py:43 GRAVITY
constexpr float kHDry = 1.0e-3f;  // solver/core/grid.py:48 H_DRY

__device__ __forceinline__ float rmax(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float rmin(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float rclamp(float x, float lo, float hi) { return rmin(rmax(lo, x), hi); }

// sources.py:66-82 kahan_add: (total, comp) <- compensated total + inc.
__device__ __forceinline__ void kahan_add(float& total, float& comp, float inc) {
  const float y = inc - comp;
  const float t = total + y;
  comp = (t - total) - y;
  total = t;
}

// Zero operands. The IEEE single-precision division takes its slow path when the
// dividend is zero (about 3x the cost on B200), and still water, dry neighbours and
// frictionless beds make zero dividends common. For a divisor y > 0 (finite or +inf,
// never NaN) the quotient of +-0 is that same +-0, so returning x unchanged is the
// division's exact result. Callers guarantee y > 0.
__device__ __forceinline__ float div_pos(float x, float y) { return x == 0.0f ? x : x / y; }

// The IEEE square root of a zero argument also leaves its fast path (about 1.6x the
// cost); sqrt(+-0) is that same +-0.
__device__ __forceinline__ float sqrt_z(float x) { return x == 0.0f ? x : sqrtf(x); }

// channels.py:58-70 eta_subgrid: the storage curve h -> eta.
__device__ __forceinline__ float eta_subgrid(float h, float z, float w, float d, float dx) {
  float eta = h + z;
  if (w > 0.0f && d > 0.0f) {
    const float h_bf = w * d / dx;
    if (h <= h_bf)
      eta = z - d + div_pos(h * dx, w);
    else
      eta = z + (h - h_bf);
  }
  return eta;
}

// channels.py:73-83 column_depth: the water column that sets the wave speed.
__device__ __forceinline__ float column_depth(float h, float w, float d, float dx) {
  float col = h;
  if (w > 0.0f && d > 0.0f) {
    const float h_bf = w * d / dx;
    if (h <= h_bf)
      col = div_pos(h * dx, w);
    else
      col = d + (h - h_bf);
  }
  return col;
}

// friction.py:18-31 manning_denominator
__device__ __forceinline__ float manning_denominator(float q_prev, float h_flow, float n, float g, float dt) {
  return 1.0f + g * dt * n * n * fabsf(q_prev) / rb_pow73f(h_flow);
}

// num / manning_denominator(q_prev, h_flow, n, g, dt) for h_flow >= H_DRY, with the
// same bits: when the friction numerator g dt n^2 |q_prev| is +0 the denominator is
// exactly 1 (and num / 1 == num), so neither the power nor the divisions are needed.
__device__ __forceinline__ float manning_divide(float num, float q_prev, float h_flow, float n, float g, float dt) {
  const float f = g * dt * n * n * fabsf(q_prev);
  if (f == 0.0f) return num;
  const float den = 1.0f + f / rb_pow73f(h_flow);
  return (num == 0.0f && den > 0.0f) ? num : num / den;
}

// Float key whose unsigned order is the float order for values >= 0.
// Reductions here start from 0 (the reference zeroes its h_max slot before the
// atomic max), so only non-negative values are ever compared.
__device__ __forceinline__ unsigned int max_key(float v) { return __float_as_uint(v > 0.0f ? v : 0.0f); }

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Fixed-order warp sum (a butterfly tree; every lane ends with the same value).
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide max of non-negative values folded into *key with one atomic per block.
template <int NT>
__device__ __forceinline__ void block_max_to(float v, unsigned int* key, float* s_warp) {
  v = warp_max(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) s_warp[w] = v;
  __syncthreads();
  if (w == 0) {
    float x = l < NT / 32 ? s_warp[l] : 0.0f;
    x = warp_max(x);
    if (l == 0) atomicMax(key, max_key(x));
  }
}

// Block-wide f64 sum in a fixed order; the result is valid in thread 0.
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* s_warp) {
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) s_warp[w] = v;
  __syncthreads();
  double x = 0.0;
  if (w == 0) {
    x = l < NT / 32 ? s_warp[l] : 0.0;
    x = warp_sum(x);
  }
  return x;
}

// Kahan-accumulate one tile's per-step f64 contribution into its ledger slot
// (slot[0] = running total, slot[1] = compensation). One writer per slot.
__device__ __forceinline__ void ledger_add(double* slot, double inc) {
  const double y = inc - slot[1];
  const double t = slot[0] + y;
  slot[1] = (t - slot[0]) - y;
  slot[0] = t;
}

__device__ __forceinline__ void flag_error(unsigned int* err, unsigned int bit) {
  if (err) atomicOr(err, bit);
}

}  // namespace rb
