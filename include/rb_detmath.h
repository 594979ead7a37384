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
 * replacements use only IEEE-754 double precision +, -, *, /, sqrt and exact bit
 * manipulation, so the same source compiled by gcc (-ffp-contract=off) and by nvcc
 * (--fmad=false) returns bit-identical floats. Each result is the float rounding of
 * a double whose relative error is below 1e-12, i.e. the correctly rounded
 * x^float32(p) for all but roughly one input in a hundred thousand, which are one
 * ulp away.
 *
 * Method.
 *  Cube root: split the widened input d = m * 2^e with m in [1,2), write e = 3q + r
 *  with r in {0,1,2} and t = m * 2^r in [1,8), so cbrt(d) = cbrt(t) * 2^q. A cubic
 *  polynomial in m, least-squares fitted to m^(-1/3) at 200 Chebyshev nodes on
 *  [1,2] (max relative error 2.6e-4), times 2^(-r/3), seeds w ~ t^(-1/3). Two steps
 *  of the division-free Newton iteration for the inverse cube root,
 *  w <- w + w (1 - t w^3) / 3, square the error each time (2.6e-4 -> 1.4e-7 ->
 *  4e-14). Then cbrt(t) = t w^2, and the 2^q scaling is exact.
 *  Exponent offset: x^(p - delta) = x^p * exp(-delta ln x) with |delta ln x| < 1e-5,
 *  so exp(-u) = 1 - u + u^2/2 to 1e-16. Because delta < 1e-7, ln x is needed only
 *  to ~1e-5 absolute for a 1e-12 result: ln x = e ln2 (double) + ln m, with m (the
 *  float mantissa, exact in float) moved into [0.75, 1.5) and ln m = 2 atanh(s),
 *  s = (m-1)/(m+1) in float, |s| <= 1/5, summed to s^9 in float (abs error < 2e-7).
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

/* Cube root of a finite d > 0 that is a widened float (so d is a normal double). */
RB_HD double rb_cbrt_pos(double d) {
  const uint64_t b = rb_bits_of(d);
  const int e = (int)((b >> 52) & 0x7ff) - 1023;
  const double m = rb_double_of((b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);
  const int q = e >= 0 ? e / 3 : -((-e + 2) / 3);
  const int r = e - 3 * q;
  const double t = m * (r == 0 ? 1.0 : (r == 1 ? 2.0 : 4.0));
  /* 2^(-1/3) and 2^(-2/3) */
  const double s = r == 0 ? 1.0 : (r == 1 ? 0.7937005259840998 : 0.6299605249474366);
  double w = ((-0.049690080091556635 * m + 0.31664422097129163) * m - 0.8083339085256394) * m +
             1.5411186775286052;
  w = w * s;
  w = w + w * ((1.0 - t * ((w * w) * w)) * 0.3333333333333333);
  w = w + w * ((1.0 - t * ((w * w) * w)) * 0.3333333333333333);
  const double c = t * (w * w);
  return c * rb_double_of((uint64_t)(q + 1023) << 52);
}

/* Natural log of a finite d > 0 that is a widened float, absolute error < 3e-7:
 * enough for the exponent offsets below, which scale it by |delta| < 1e-7. */
RB_HD double rb_log_pos(double d) {
  const uint64_t b = rb_bits_of(d);
  int e = (int)((b >> 52) & 0x7ff) - 1023;
  float m = (float)rb_double_of((b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL); /* exact */
  if (m >= 1.5f) {
    m = m * 0.5f;
    e = e + 1;
  }
  const float s = (m - 1.0f) / (m + 1.0f);
  const float s2 = s * s;
  const float series = ((((0.111111112f * s2 + 0.142857149f) * s2 + 0.200000003f) * s2 + 0.333333343f) * s2 + 1.0f) * s;
  return (double)e * 0.6931471805599453 + 2.0 * (double)series;
}

/* exp(-delta * ln d) for the tiny exponent offsets above. */
RB_HD double rb_offset_factor(double d, double delta) {
  const double u = delta * rb_log_pos(d);
  return (1.0 - u) + 0.5 * (u * u);
}

/* x ^ float32(7/3) as a float; 0 at 0, NaN for negative or NaN input, inf at inf. */
RB_HD float rb_pow73f(float x) {
  if (!(x > 0.0f)) return x == 0.0f ? 0.0f : (x - x) / (x - x);
  if (x > 3.4028234663852886e38f) return x;
  const double d = (double)x;
  return (float)(((d * d) * rb_cbrt_pos(d)) * rb_offset_factor(d, RB_DELTA_73));
}

/* x ^ float32(1/3) as a float; same special cases as rb_pow73f. */
RB_HD float rb_pow13f(float x) {
  if (!(x > 0.0f)) return x == 0.0f ? 0.0f : (x - x) / (x - x);
  if (x > 3.4028234663852886e38f) return x;
  const double d = (double)x;
  return (float)(rb_cbrt_pos(d) * rb_offset_factor(d, RB_DELTA_13));
}

/* x ^ float32(4/3) as a float; same special cases as rb_pow73f. */
RB_HD float rb_pow43f(float x) {
  if (!(x > 0.0f)) return x == 0.0f ? 0.0f : (x - x) / (x - x);
  if (x > 3.4028234663852886e38f) return x;
  const double d = (double)x;
  return (float)((d * rb_cbrt_pos(d)) * rb_offset_factor(d, RB_DELTA_43));
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
