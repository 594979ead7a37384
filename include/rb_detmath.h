/*
 * rb_detmath.h -- deterministic float32 power functions for the river-basin solver path.
 *
 * The reference evaluates four fractional powers in float32 through the platform
 * libm (`wp.pow`), each with a float32 exponent:
 *   - h_flow ^ float32(7/3) in the semi-implicit Manning denominator
 *     (solver/core/friction.py:30, used by local_inertial.py:98,128 and hllc.py:937);
 *   - R ^ float32(1/3) in the Manning bed shear (solver/core/sediment.py:168);
 *   - R ^ float32(4/3) in the sub-grid channel's Manning denominator
 *     (solver/core/friction.py:56-58, used by local_inertial.py:310);
 *   - (theta - theta_c) ^ 1.5 in the Meyer-Peter-Mueller capacity (sediment.py:192).
 * Note the exponents: float32(7/3) = 2.3333332538604736, so the reference computes
 * x^2.33333325..., not x^(7/3) (a difference of up to ~10 ulp for large x).
 *
 * A vendor powf differs between the CPU libm and the CUDA math library by a few
 * ulp, which would turn every GPU-vs-CPU comparison into a tolerance test. These
 * replacements use only IEEE-754 single and double precision +, -, *, /, sqrt and
 * exact bit manipulation, so the same source compiled by gcc (-ffp-contract=off)
 * and by nvcc (--fmad=false) returns bit-identical floats. Each result is the float
 * rounding of a double whose relative error is about 1e-12, i.e. the correctly
 * rounded x^float32(p) for all but a few inputs in a million, which are one ulp
 * away.
 *
 * Method. A positive float is split once, x = m * 2^e with m in [1, 2) (subnormals
 * scaled by 2^24 first); both parts below reuse the split.
 *  Cube root: write e = 3q + r with r in {0, 1, 2} and t = m * 2^r in [1, 8) (exact
 *  in float), so cbrt(x) = cbrt(t) * 2^q. A cubic polynomial in m, least-squares
 *  fitted to m^(-1/3) at 400 Chebyshev nodes on [1, 2] (relative error 2.9e-4),
 *  times float(2^(-r/3)), seeds w ~ t^(-1/3) in float. The division-free Newton
 *  iteration for the inverse cube root, w <- w + w (1 - t w^3) / 3, squares the
 *  error: one step in float (to ~3e-7, the float rounding floor) and one in double
 *  (to ~2e-13). Then cbrt(t) = t w^2 in double, and the 2^q scaling is exact.
 *  Exponent offset: x^(p - delta) = x^p * exp(-delta ln x) with |delta ln x| < 1e-5,
 *  so exp(-u) = 1 - u + u^2/2 to 1e-16. Because |delta| < 1e-7, ln x is needed only
 *  to ~1e-5 absolute for a 1e-12 result: ln x = (e + log2 m) ln 2 in float, with
 *  log2 m a degree-5 polynomial in m - 1 (least squares at the same nodes, absolute
 *  error 1.4e-5).
 *  Checked against the float rounding of a long-double powl on every 97th positive
 *  float up to 1e30 (19.6 million inputs): never more than 1 ulp away, and off the
 *  correctly rounded value for 2.5 in a million (x^(7/3)), 0.8 (x^(1/3)) and 1.8
 *  (x^(4/3)).
 */
#ifndef RB_DETMATH_H
#define RB_DETMATH_H

#include <stdint.h>

#if defined(__CUDACC__)
#define RB_HD __host__ __device__ __forceinline__
#else
#include <math.h>
#include <string.h>
#define RB_HD static inline
#endif

/* p - float32(p) for p = 7/3, 1/3 and 4/3. */
#define RB_DELTA_73 7.947285984855057e-08
#define RB_DELTA_13 (-9.934107481068821e-09)
#define RB_DELTA_43 (-3.9736429850260414e-08)

RB_HD uint64_t rb_bits_of(double d) {
#if defined(__CUDA_ARCH__)
  return (uint64_t)__double_as_longlong(d);
#else
  uint64_t u;
  memcpy(&u, &d, sizeof u);
  return u;
#endif
}

RB_HD double rb_double_of(uint64_t u) {
#if defined(__CUDA_ARCH__)
  return __longlong_as_double((long long)u);
#else
  double d;
  memcpy(&d, &u, sizeof d);
  return d;
#endif
}

RB_HD uint32_t rb_fbits(float f) {
#if defined(__CUDA_ARCH__)
  return __float_as_uint(f);
#else
  uint32_t u;
  memcpy(&u, &f, sizeof u);
  return u;
#endif
}

RB_HD float rb_float_of(uint32_t u) {
#if defined(__CUDA_ARCH__)
  return __uint_as_float(u);
#else
  float f;
  memcpy(&f, &u, sizeof f);
  return f;
#endif
}

/* x = m * 2^e for a positive finite float x: returns m in [1, 2), sets *e. */
RB_HD float rb_split_pos(float x, int* e) {
  uint32_t b = rb_fbits(x);
  int k = 0;
  if (b < 0x00800000u) { /* subnormal: scale into the normal range, exactly */
    x = x * 16777216.0f;
    b = rb_fbits(x);
    k = -24;
  }
  *e = (int)(b >> 23) - 127 + k;
  return rb_float_of((b & 0x007fffffu) | 0x3f800000u);
}

/* cbrt(m * 2^e) as a double, relative error about 2e-13. */
RB_HD double rb_cbrt_split(float m, int e) {
  const int q = e >= 0 ? e / 3 : -((-e + 2) / 3);
  const int r = e - 3 * q;
  const float tf = m * (r == 0 ? 1.0f : (r == 1 ? 2.0f : 4.0f));
  float w = ((-0.0488736666738987f * m + 0.3129411041736603f) * m - 0.8028873205184937f) * m + 1.5385289192199707f;
  w = w * (r == 0 ? 1.0f : (r == 1 ? 0.7937005162239075f : 0.6299605369567871f)); /* 2^(-r/3) */
  w = w + w * ((1.0f - tf * ((w * w) * w)) * 0.333333343f);
  const double t = (double)tf;
  double wd = (double)w;
  wd = wd + wd * ((1.0 - t * ((wd * wd) * wd)) * 0.3333333333333333);
  return (t * (wd * wd)) * rb_double_of((uint64_t)(q + 1023) << 52);
}

/* exp(-delta * ln(m * 2^e)) for the tiny exponent offsets above. */
RB_HD double rb_offset_split(float m, int e, double delta) {
  const float t = m - 1.0f;
  const float log2m = ((((0.04392862692475319f * t - 0.18983244895935059f) * t + 0.4115614891052246f) * t -
                        0.7072534561157227f) * t + 1.4415920972824097f) * t + 1.4390930118679535e-05f;
  const float ln = ((float)e + log2m) * 0.693147182f;
  const double u = delta * (double)ln;
  return (1.0 - u) + 0.5 * (u * u);
}

/* x ^ float32(7/3) as a float; 0 at 0, NaN for negative or NaN input, inf at inf. */
RB_HD float rb_pow73f(float x) {
  if (!(x > 0.0f)) return x == 0.0f ? 0.0f : (x - x) / (x - x);
  if (x > 3.4028234663852886e38f) return x;
  int e;
  const float m = rb_split_pos(x, &e);
  const double d = (double)x;
  return (float)(((d * d) * rb_cbrt_split(m, e)) * rb_offset_split(m, e, RB_DELTA_73));
}

/* x ^ float32(1/3) as a float; same special cases as rb_pow73f. */
RB_HD float rb_pow13f(float x) {
  if (!(x > 0.0f)) return x == 0.0f ? 0.0f : (x - x) / (x - x);
  if (x > 3.4028234663852886e38f) return x;
  int e;
  const float m = rb_split_pos(x, &e);
  return (float)(rb_cbrt_split(m, e) * rb_offset_split(m, e, RB_DELTA_13));
}

/* x ^ float32(4/3) as a float; same special cases as rb_pow73f. */
RB_HD float rb_pow43f(float x) {
  if (!(x > 0.0f)) return x == 0.0f ? 0.0f : (x - x) / (x - x);
  if (x > 3.4028234663852886e38f) return x;
  int e;
  const float m = rb_split_pos(x, &e);
  const double d = (double)x;
  return (float)((d * rb_cbrt_split(m, e)) * rb_offset_split(m, e, RB_DELTA_43));
}

/* x ^ 1.5 as a float for x >= 0 (NaN below 0 or for NaN). */
RB_HD float rb_pow15f(float x) {
  if (!(x >= 0.0f)) return (x - x) / (x - x);
  const double d = (double)x;
  return (float)(d * sqrt(d));
}

/* n / d, the IEEE quotient, on a path the caller takes rarely. On the device it is
 * inline PTX, which the compiler cannot evaluate ahead of the branch that guards it
 * (an ordinary division would be computed on every lane and selected, and would
 * cost its full price, or its slow path for a zero operand, on all of them). */
RB_HD float rb_div_rare(float n, float d) {
#if defined(__CUDA_ARCH__)
  float q;
  asm volatile("div.rn.f32 %0, %1, %2;" : "=f"(q) : "f"(n), "f"(d));
  return q;
#else
  return n / d;
#endif
}

/* (n / d >= 0.0f) for a float quotient, without the division in all but a rare
 * case, for any n and any non-NaN d with |d| > 1e-12 (the only use: the HLLC
 * contact-wave sign, solver/core/hllc.py:231-238, whose quotient is read only
 * through that comparison). IEEE semantics of the quotient: +-0 for n = +-0 or
 * an infinite d, NaN for NaN n or inf/inf, otherwise the sign of n times the sign
 * of d, where a negative quotient that underflows rounds to -0 (which compares
 * >= 0). That last case needs |n / d| <= 2^-150; when |n| > |d| 2^-100 it cannot
 * happen, and otherwise the quotient itself is formed. */
RB_HD int rb_quotient_nonneg(float n, float d) {
  if (!(n == n)) return 0;
  if (n == 0.0f) return 1;
  if (d > 3.4028234663852886e38f || d < -3.4028234663852886e38f) {
    const int n_inf = n > 3.4028234663852886e38f || n < -3.4028234663852886e38f;
    return n_inf ? 0 : 1;
  }
  if ((n > 0.0f) == (d > 0.0f)) return 1;
  const float an = n < 0.0f ? -n : n, ad = d < 0.0f ? -d : d;
  if (an > ad * 0x1p-100f) return 0;
  return rb_div_rare(n, d) >= 0.0f;
}

/* x / 9.81f (the float32 gravity of solver/core/grid.py:43), the IEEE quotient
 * bit for bit, without a division for x >= 2^-99: the method of Brisebarre, Muller
 * and Raina for division by a constant ("Accelerating correctly rounded
 * floating-point division when the divisor is known in advance", IEEE Trans.
 * Computers 53(8), 2004), q = RN(x zh + RN(x zl)) with zh = RN(1/g) and
 * zl = RN(1/g - zh), one multiply and one fused multiply-add. Whether it is
 * correctly rounded depends on the divisor; for this one it was checked against
 * the division for every float from 2^-99 to +inf. Below 2^-99 x zl underflows
 * and the method can miss, and NaN and negative x are not its business: those
 * take the division. The only use is the HLLC star-depth estimate
 * (solver/core/hllc.py:224, hs * hs / g). */
RB_HD float rb_div_g(float x) {
  const float g = 9.81f, zh = 0x1.a1887ap-4f, zl = 0x1.dcb5p-38f;
  if (x >= 0x1p-99f) return fmaf(x, zh, x * zl);
  return rb_div_rare(x, g);
}

#endif /* RB_DETMATH_H */
