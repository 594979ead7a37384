// rb_common.cuh -- shared device helpers for the river-basin solver kernels.
//
// Two arithmetic contracts, one source:
//  * exact (every translation unit in csrc/): compiled with --fmad=false and IEEE
//    division / square root, so each operation rounds once in the reference's
//    expression order (identical to the CPU oracle); the fractional powers come
//    from include/rb_detmath.h;
//  * fast (csrc/fast/, RB_FAST_MATH defined, everything in namespace rb::fast):
//    contracted multiply-adds, the hardware's approximate division and square root
//    and __powf for the fractional powers -- the arithmetic of a GPU build of the
//    reference, held to the solver tolerance instead of bit equality. Compensated
//    (Kahan) additions stay explicit IEEE adds in both.
// `rmax/rmin/rclamp` are the scalar builtins of the reference's kernel language
// (a > b ? a : b, a < b ? a : b, min(max(lo,x),hi)), which differ from
// fmaxf/fminf on signed zeros.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "rb_detmath.h"
#include "rbsim.h"

// The kernels of a translation unit live in rb (exact) or rb::fast (fast).
#if defined(RB_FAST_MATH)
#define RB_ARITH_BEGIN namespace fast {
#define RB_ARITH_END }
#else
#define RB_ARITH_BEGIN
#define RB_ARITH_END
#endif

namespace rb {

constexpr float kG = 9.81f;     // solver/core/grid.py:43 GRAVITY
constexpr float kHDry = 1.0e-3f;  // solver/core/grid.py:48 H_DRY

RB_ARITH_BEGIN

__device__ __forceinline__ float rmax(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float rmin(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float rclamp(float x, float lo, float hi) { return rmin(rmax(lo, x), hi); }

// sources.py:66-82 kahan_add: (total, comp) <- compensated total + inc. Explicit
// IEEE adds, which no build contracts or reassociates.
__device__ __forceinline__ void kahan_add(float& total, float& comp, float inc) {
  const float y = __fsub_rn(inc, comp);
  const float t = __fadd_rn(total, y);
  comp = __fsub_rn(__fsub_rn(t, total), y);
  total = t;
}

#if defined(RB_FAST_MATH)
// Fast arithmetic: the approximate division has no slow path to steer around, so
// the quotient helpers are plain divisions (an unused lane divides by 1).
__device__ __forceinline__ float opaque(float v) { return v; }
__device__ __forceinline__ float div_pos(float x, float y) { return x / y; }
__device__ __forceinline__ float div_if(bool use, float x, float y) { return use ? x / (use ? y : 1.0f) : 0.0f; }
__device__ __forceinline__ float div_in_branch(float x, float y) { return x / y; }
// x / g
__device__ __forceinline__ float div_g(float x) { return x * (1.0f / kG); }
// n / d >= 0 for |d| > 0, from the signs
__device__ __forceinline__ bool quotient_nonneg(float n, float d) { return n == 0.0f || ((n > 0.0f) == (d > 0.0f)); }
// x ^ float32(p) for x > 0 with the float32 exponents of the reference (7/3, 1/3, 4/3, 1.5)
__device__ __forceinline__ float pow73(float x) { return __powf(x, 2.33333325f); }
__device__ __forceinline__ float pow13(float x) { return __powf(x, 0.333333343f); }
__device__ __forceinline__ float pow43(float x) { return __powf(x, 1.33333337f); }
__device__ __forceinline__ float pow15(float x) { return x * sqrtf(x); }
#else
// Zero operands. The IEEE single-precision division takes its slow path when the
// dividend is zero (about 3x the cost of the fast path on B200) or the divisor is.
// Still water, dry neighbours and frictionless beds make such operands common, and
// a guard in the source does not keep them away: the compiler evaluates a guarded
// division unconditionally and selects the result, so a discarded quotient of a
// dry cell still pays the slow path. The helpers below give the division 1 in place of an
// operand that would send it down the slow path, and select the exact result
// themselves (0 / y = 0 with the dividend's sign for y > 0).
// `opaque` hides the substituted operand from the optimizer, which would otherwise
// fold the two selects back into the original division; the move itself compiles to
// nothing.
__device__ __forceinline__ float opaque(float v) {
  float r;
  asm("mov.b32 %0, %1;" : "=f"(r) : "f"(v));
  return r;
}

// x / y, bit for bit, for any x and y.
__device__ __forceinline__ float div_pos(float x, float y) {
  const bool same = x == 0.0f && y > 0.0f;  // the quotient is x itself
  const float q = opaque(same ? 1.0f : x) / y;
  return same ? x : q;
}

// use ? x / y : 0, where the division of an unused lane divides by 1 (its divisor,
// e.g. the depth of a dry cell, may be 0).
__device__ __forceinline__ float div_if(bool use, float x, float y) {
  const float q = div_pos(x, opaque(use ? y : 1.0f));
  return use ? q : 0.0f;
}

// The IEEE quotient x / y as inline PTX, which the compiler cannot evaluate ahead
// of the branch that guards it: for divisions that a data-dependent branch is meant
// to skip, where an ordinary '/' would be computed for every lane regardless.
__device__ __forceinline__ float div_in_branch(float x, float y) {
  float q;
  asm volatile("div.rn.f32 %0, %1, %2;" : "=f"(q) : "f"(x), "f"(y));
  return q;
}

__device__ __forceinline__ float div_g(float x) { return rb_div_g(x); }  // x / g, bit for bit
__device__ __forceinline__ bool quotient_nonneg(float n, float d) { return rb_quotient_nonneg(n, d) != 0; }
__device__ __forceinline__ float pow73(float x) { return rb_pow73f(x); }
__device__ __forceinline__ float pow13(float x) { return rb_pow13f(x); }
__device__ __forceinline__ float pow43(float x) { return rb_pow43f(x); }
__device__ __forceinline__ float pow15(float x) { return rb_pow15f(x); }
#endif  // RB_FAST_MATH

// channels.py:58-70 eta_subgrid: the storage curve h -> eta.
__device__ __forceinline__ float eta_subgrid(float h, float z, float w, float d, float dx) {
  float eta = h + z;
  if (w > 0.0f && d > 0.0f) {
    const float h_bf = div_pos(w * d, dx);
    if (h <= h_bf)
      eta = z - d + div_pos(h * dx, opaque(w > 0.0f ? w : 1.0f));
    else
      eta = z + (h - h_bf);
  }
  return eta;
}

// channels.py:73-83 column_depth: the water column that sets the wave speed.
__device__ __forceinline__ float column_depth(float h, float w, float d, float dx) {
  float col = h;
  if (w > 0.0f && d > 0.0f) {
    const float h_bf = div_pos(w * d, dx);
    if (h <= h_bf)
      col = div_pos(h * dx, opaque(w > 0.0f ? w : 1.0f));
    else
      col = d + (h - h_bf);
  }
  return col;
}

// friction.py:18-31 manning_denominator
__device__ __forceinline__ float manning_denominator(float q_prev, float h_flow, float n, float g, float dt) {
  return 1.0f + g * dt * n * n * fabsf(q_prev) / pow73(h_flow);
}

// num / manning_denominator(q_prev, h_flow, n, g, dt) for h_flow >= H_DRY, with the
// same bits: when the friction numerator g dt n^2 |q_prev| is +0 the denominator is
// exactly 1 (and num / 1 == num), so neither the power nor the divisions are needed.
__device__ __forceinline__ float manning_divide(float num, float q_prev, float h_flow, float n, float g, float dt) {
  const float f = g * dt * n * n * fabsf(q_prev);
  if (f == 0.0f) return num;
  const float den = 1.0f + f / pow73(h_flow);
  return div_pos(num, den);
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

RB_ARITH_END

// Programmatic dependent launch of the step chain (plan -> stage 1 -> stage 2 ->
// plan ..., or plan -> LI step -> plan ...). Each kernel of the chain first lets the
// next kernel of the stream be scheduled (it launches once every block of this grid
// has begun, so its blocks take the SM slots this grid's last wave frees), then
// waits until the kernel before it has completed with its memory visible, before it
// reads anything. A kernel launched without the attribute does not start early, and
// for it the wait returns at once.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

// Whether the step chain is launched with programmatic stream serialization
// (default on; RBSIM_PDL=0 in the environment turns it off, for comparison).
bool pdl_enabled();

// Launch a kernel of the step chain, with the programmatic-serialization attribute
// when pdl_enabled(). The kernel must begin with pdl_enter().
template <class... Params, class... Args>
cudaError_t launch_chain(void (*kernel)(Params...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                         Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<Args&&>(args)...);
}
}  // namespace rb
