/* Elementary functions of doubles for the PressureDependMultiYield device update: exp, log, pow and
 * cos, evaluated with IEEE-exact operations only (+, -, *, / and sqrt are correctly rounded; fma is
 * one rounding; integer operations on the bit patterns), so that a host build and a device build of
 * the same calls give the same bits. Compile without contraction (nvcc --fmad=false, gcc
 * -ffp-contract=off): every fused multiply-add here is an explicit fma().
 *
 * Methods (published ones, restated here):
 *   - exp: Cody-Waite reduction x = k ln2/32 + r with ln2/32 in three parts, |r| <= ln2/64, the
 *     Taylor polynomial of e^r - 1 - r to degree 7, and 2^(j/32) from a 32-entry double-double
 *     table (Tang's table-driven method); the scale 2^(k/32 - j/32) by exponent arithmetic.
 *   - log: x = 2^e m with m in [sqrt(1/2), sqrt(2)), log m = 2 atanh(s), s = (m - 1)/(m + 1) formed
 *     in double-double, the odd series of atanh to s^27; e ln 2 with ln 2 in two parts.
 *   - pow: exp(y log x) with log x in double-double and y log x formed with an exact product.
 *   - cos: Cody-Waite reduction x = k pi/2 + r with pi/2 in three parts (|k| < 2^20), then the
 *     Taylor series of cos r (to r^20) or sin r (to r^19) in double, the terms to r^4 (cos) and
 *     r^3 (sin) in double-double.
 * Errors (measured against 60-digit decimal arithmetic, tests/test_fx_math.py): within 0.51 ulp for
 * exp, pow (|x| in [e^-5, e^5], |y| <= 3) and cos (|x| <= 10), 0.45 ulp for log; the host C library's
 * result on 99.6-100 % of arguments and one ulp from it otherwise. The leading terms of the sine and
 * cosine series are carried in double-double. Special values follow C99 Annex F for exp, log and
 * pow; cos is NaN for
 * infinities and NaNs, and for |x| >= 2^20 pi/2 it reduces with the same three parts (accuracy
 * degrades there; the material's angles are below pi).
 * No counterpart in the reference, which calls its host C library (std::pow, std::exp, std::log,
 * std::cos in src/physics/materials/pressure_depend_multi_yield.hpp). */
#ifndef FX_MATH_H
#define FX_MATH_H

#include <math.h>
#include <stdint.h>
#include <string.h>

#include "fx_math_consts.h"

#if defined(__CUDACC__)
#define FXM_FN __host__ __device__ inline
#elif defined(__cplusplus)
#define FXM_FN inline
#else
#define FXM_FN static inline
#endif
#if defined(__GNUC__) && !defined(__cplusplus)
#define FXM_UNUSED __attribute__((unused))
#else
#define FXM_UNUSED
#endif

/* 2^(j/32), j = 0..31: the high parts, then the low parts (constant memory on the device) */
static const double fxm_exp2_host[64] FXM_UNUSED = {FXM_EXP2_HI_INIT, FXM_EXP2_LO_INIT};
#if defined(__CUDACC__)
static __constant__ const double fxm_exp2_dev[64] = {FXM_EXP2_HI_INIT, FXM_EXP2_LO_INIT};
#endif

FXM_FN uint64_t fxm_bits(double x) {
  uint64_t u;
  memcpy(&u, &x, sizeof u);
  return u;
}
FXM_FN double fxm_from(uint64_t u) {
  double x;
  memcpy(&x, &u, sizeof x);
  return x;
}
FXM_FN double fxm_inf(void) { return fxm_from(0x7ff0000000000000ULL); }
FXM_FN double fxm_nan(void) { return fxm_from(0x7ff8000000000000ULL); }
FXM_FN int fxm_isinf(double x) { return (fxm_bits(x) & 0x7fffffffffffffffULL) == 0x7ff0000000000000ULL; }

/* s + e = a + b exactly (Knuth's two-sum) */
FXM_FN void fxm_two_sum(double a, double b, double* s, double* e) {
  const double t = a + b;
  const double bb = t - a;
  *e = (a - (t - bb)) + (b - bb);
  *s = t;
}
/* s + e = a + b exactly, for |a| >= |b| or a = 0 (Dekker's fast two-sum) */
FXM_FN void fxm_fast_two_sum(double a, double b, double* s, double* e) {
  const double t = a + b;
  *e = b - (t - a);
  *s = t;
}

/* 2^(j/32), high and low parts */
FXM_FN double fxm_exp2_hi(int j) {
#if defined(__CUDA_ARCH__)
  return fxm_exp2_dev[j];
#else
  return fxm_exp2_host[j];
#endif
}
FXM_FN double fxm_exp2_lo(int j) {
#if defined(__CUDA_ARCH__)
  return fxm_exp2_dev[32 + j];
#else
  return fxm_exp2_host[32 + j];
#endif
}

/* y 2^n for y in [0.5, 4) and n in [-2023, 2023]: exact unless the result is subnormal (one rounding)
   or overflows (infinity) */
FXM_FN double fxm_scale(double y, int64_t n) {
  if (n > 1000) {
    y *= 0x1p1000;
    n -= 1000;
  } else if (n < -1000) {
    y *= 0x1p-1000;
    n += 1000;
  }
  return y * fxm_from((uint64_t)(n + 1023) << 52);
}

/* e^(xh + xl), xl a correction of at most a few ulps of xh */
FXM_FN double fxm_exp_dd(double xh, double xl) {
  if (xh != xh) return xh + xh;
  if (xh > 710.0) return fxm_inf();
  if (xh < -746.0) return 0.0;
  const double shift = 0x1.8p52;
  const double kd = (xh * FXM_INV_LN2_32 + shift) - shift; /* nearest integer to x 32 / ln 2 */
  const int64_t k = (int64_t)kd;
  const double a = xh - kd * FXM_LN2_32_1; /* exact: kd ln2_1 has at most 53 bits, a is near it */
  double s, e;
  fxm_two_sum(a, -(kd * FXM_LN2_32_2), &s, &e);
  const double rl = (e - kd * FXM_LN2_32_3) + xl;
  /* e^(s + rl) - 1 = s + s^2 (1/2 + s/6 + ... + s^5/7!) + rl (1 + s) */
  const double q =
      (s * s) * (0.5 + s * (FXM_EXP_C3 + s * (FXM_EXP_C4 + s * (FXM_EXP_C5 + s * (FXM_EXP_C6 + s * FXM_EXP_C7)))));
  const double m = fma(rl, s, rl) + q;
  const int j = (int)(k & 31);
  const int64_t n = (k - j) / 32;
  const double th = fxm_exp2_hi(j), tl = fxm_exp2_lo(j);
  /* T (1 + s + m) = th + (th s + th m + tl + tl s) */
  const double tail = fma(th, s, fma(th, m, fma(tl, s, tl)));
  return fxm_scale(th + tail, n);
}

FXM_FN double fxm_exp(double x) { return fxm_exp_dd(x, 0.0); }

/* log x as hi + lo, for finite x > 0 */
FXM_FN void fxm_log_dd(double x, double* hi, double* lo) {
  uint64_t u = fxm_bits(x);
  int64_t e = (int64_t)(u >> 52) - 1023;
  if ((u >> 52) == 0) { /* subnormal */
    u = fxm_bits(x * 0x1p54);
    e = (int64_t)(u >> 52) - 1023 - 54;
  }
  double m = fxm_from((u & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL); /* [1, 2) */
  if (m > FXM_SQRT2) {
    m *= 0.5;
    e += 1;
  }
  const double a = m - 1.0; /* exact */
  double bh, bl;
  fxm_two_sum(m, 1.0, &bh, &bl);
  const double s = a / bh;
  const double sl = (fma(-s, bh, a) - s * bl) / bh; /* s + sl = a / (bh + bl) to double-double */
  const double z = s * s;
  const double tail =
      (s * z) *
      (FXM_LOG_A1 +
       z * (FXM_LOG_A2 +
            z * (FXM_LOG_A3 +
                 z * (FXM_LOG_A4 +
                      z * (FXM_LOG_A5 +
                           z * (FXM_LOG_A6 +
                                z * (FXM_LOG_A7 +
                                     z * (FXM_LOG_A8 +
                                          z * (FXM_LOG_A9 +
                                               z * (FXM_LOG_A10 +
                                                    z * (FXM_LOG_A11 + z * (FXM_LOG_A12 + z * FXM_LOG_A13))))))))))));
  const double ed = (double)e;
  double h, l;
  fxm_two_sum(ed * FXM_LN2_HI, 2.0 * s, &h, &l); /* ed ln2_hi exact */
  l += (ed * FXM_LN2_LO + 2.0 * sl) + tail;
  fxm_fast_two_sum(h, l, hi, lo);
}

FXM_FN double fxm_log(double x) {
  if (x != x) return x + x;
  if (x < 0.0) return fxm_nan();
  if (x == 0.0) return -fxm_inf();
  if (fxm_isinf(x)) return x;
  double hi, lo;
  fxm_log_dd(x, &hi, &lo);
  return hi;
}

/* y is an integer (finite) */
FXM_FN int fxm_is_int(double y) {
  if (fabs(y) >= 0x1p52) return 1;
  return (double)(int64_t)y == y;
}
FXM_FN int fxm_is_odd_int(double y) {
  if (fabs(y) >= 0x1p53 || !fxm_is_int(y)) return 0;
  return (int)((int64_t)y & 1);
}

FXM_FN double fxm_pow(double x, double y) {
  if (y == 0.0 || x == 1.0) return 1.0;
  if (x != x || y != y) return x + y;
  const int odd = fxm_is_odd_int(y);
  const int xneg = (fxm_bits(x) >> 63) != 0;
  if (x == 0.0) {
    const double r = y > 0.0 ? 0.0 : fxm_inf();
    return (xneg && odd) ? -r : r;
  }
  if (fxm_isinf(y)) {
    const double ax = fabs(x);
    if (ax == 1.0) return 1.0;
    return ((ax < 1.0) == (y < 0.0)) ? fxm_inf() : 0.0;
  }
  if (fxm_isinf(x)) {
    const double r = y > 0.0 ? fxm_inf() : 0.0;
    return (xneg && odd) ? -r : r;
  }
  double sign = 1.0;
  if (xneg) {
    if (!fxm_is_int(y)) return fxm_nan();
    if (odd) sign = -1.0;
    x = -x;
  }
  double lh, ll;
  fxm_log_dd(x, &lh, &ll);
  const double ph = y * lh;
  const double pl = fma(y, lh, -ph) + y * ll; /* y (lh + ll) = ph + pl */
  double th, tl;
  fxm_fast_two_sum(ph, pl, &th, &tl);
  return sign * fxm_exp_dd(th, tl);
}

/* cos and sin of s + sl, |s| <= pi/4 */
FXM_FN double fxm_cos_kernel(double s, double sl) {
  const double z = s * s;
  const double zl = fma(s, s, -z) + 2.0 * s * sl; /* (s + sl)^2 = z + zl */
  const double w = 0.5 * z, wl = 0.5 * zl;
  /* z^2/24 in double-double (1/24 = C2 + C2_LO) */
  const double q = z * z;
  const double ql = fma(z, z, -q) + 2.0 * z * zl;
  const double t2 = q * FXM_COS_C2;
  const double t2e = fma(q, FXM_COS_C2, -t2) + (ql * FXM_COS_C2 + q * FXM_COS_C2_LO);
  const double rest =
      (q * z) *
      (FXM_COS_C3 +
       z * (FXM_COS_C4 + z * (FXM_COS_C5 + z * (FXM_COS_C6 + z * (FXM_COS_C7 + z * (FXM_COS_C8 + z * (FXM_COS_C9 + z * FXM_COS_C10)))))));
  /* cos(s + sl) = 1 - (z + zl)/2 + z^2/24 + rest */
  double h, l, h2, l2;
  fxm_two_sum(1.0, -w, &h, &l);
  fxm_fast_two_sum(h, t2, &h2, &l2);
  l2 += (l - wl) + (t2e + rest);
  return h2 + l2;
}
FXM_FN double fxm_sin_kernel(double s, double sl) {
  const double z = s * s;
  const double zl = fma(s, s, -z);
  const double u = s * z;
  const double ue = fma(s, z, -u) + s * zl; /* s^3 = u + ue */
  /* -s^3/6 in double-double (-1/6 = S1 + S1_LO) */
  const double t1 = u * FXM_SIN_S1;
  const double t1e = fma(u, FXM_SIN_S1, -t1) + (ue * FXM_SIN_S1 + u * FXM_SIN_S1_LO);
  const double poly =
      (z * z) *
      (FXM_SIN_S2 +
       z * (FXM_SIN_S3 +
            z * (FXM_SIN_S4 + z * (FXM_SIN_S5 + z * (FXM_SIN_S6 + z * (FXM_SIN_S7 + z * (FXM_SIN_S8 + z * FXM_SIN_S9)))))));
  /* sin(s + sl) = s - s^3/6 + s poly + sl cos s, cos s ~ 1 - z/2 */
  double h, l;
  fxm_fast_two_sum(s, t1, &h, &l);
  l += t1e + fma(s, poly, fma(-0.5 * z, sl, sl));
  return h + l;
}

FXM_FN double fxm_cos(double x) {
  if (x != x || fxm_isinf(x)) return fxm_nan();
  const double ax = fabs(x);
  if (ax < 0x1p-27) return 1.0;
  const double shift = 0x1.8p52;
  const double kd = (ax * FXM_TWO_OVER_PI + shift) - shift; /* nearest integer to x 2 / pi */
  const double a = ax - kd * FXM_PIO2_1;                     /* exact for kd < 2^20 */
  double s, e;
  fxm_two_sum(a, -(kd * FXM_PIO2_2), &s, &e);
  double sl = e - kd * FXM_PIO2_3;
  fxm_fast_two_sum(s, sl, &s, &sl);
  switch ((int)((int64_t)kd & 3)) {
    case 0: return fxm_cos_kernel(s, sl);
    case 1: return -fxm_sin_kernel(s, sl);
    case 2: return -fxm_cos_kernel(s, sl);
    default: return fxm_sin_kernel(s, sl);
  }
}

#endif
