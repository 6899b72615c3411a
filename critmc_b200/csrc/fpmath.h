/*
 * Single-precision elementary functions with a fixed sequence of IEEE-754
 * operations, identical on the host and on the GPU.
 *
 * The O(n) samplers feed their random numbers through exp, log, sin/cos,
 * atan2 and acos.  Library implementations differ between CUDA and the host
 * C library by an ulp or two, and the over-relaxation dynamics amplify such
 * differences exponentially, so a CPU replay could only follow the GPU for a
 * few sweeps.  These functions use only +, -, *, /, sqrt, rint, exponent
 * bit manipulation and explicit fused multiply-adds (CM_FMAF / CM_FMA, one
 * rounding, the same on both sides), so a translation unit compiled without
 * implicit floating-point contraction (nvcc --fmad=false, gcc
 * -ffp-contract=off) gives bit-identical results on both sides.
 *
 * Methods (textbook, e.g. J.-M. Muller, "Elementary Functions"): Cody-Waite
 * argument reduction with a three-part constant, then truncated Taylor
 * series (exp, sin, cos), the atanh series of log((1+s)/(1-s)) and the atan
 * series after a pi/6 shift.  Accuracy is a few ulp (tests/test_fpmath_cpu.py
 * checks it against double-precision libm).
 */
#ifndef CRITMC_FPMATH_H
#define CRITMC_FPMATH_H

#include <math.h>
#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define CM_HD __host__ __device__ __forceinline__
#else
#define CM_HD static inline
#endif

/* Fused multiply-add, rounded once (IEEE fma): the same operation on both
 * sides, so the Horner steps below cost one instruction each on the GPU and
 * the host replay (C99 fmaf/fma, correctly rounded) gives the same bits. */
#if defined(__CUDA_ARCH__)
#define CM_FMAF(a, b, c) __fmaf_rn((a), (b), (c))
#define CM_FMA(a, b, c) __fma_rn((a), (b), (c))
#else
#define CM_FMAF(a, b, c) fmaf((a), (b), (c))
#define CM_FMA(a, b, c) fma((a), (b), (c))
#endif

CM_HD uint32_t cm_f2u(float x) {
#if defined(__CUDA_ARCH__)
  return __float_as_uint(x);
#else
  uint32_t u;
  memcpy(&u, &x, 4);
  return u;
#endif
}

CM_HD float cm_u2f(uint32_t u) {
#if defined(__CUDA_ARCH__)
  return __uint_as_float(u);
#else
  float x;
  memcpy(&x, &u, 4);
  return x;
#endif
}

/* x * 2^k for |k| <= 252, with an exact power-of-two factor per step */
CM_HD float cm_scale2(float x, int k) {
  while (k > 126) {
    x = x * cm_u2f(0x7F000000u); /* 2^127 */
    k -= 127;
  }
  while (k < -126) {
    x = x * cm_u2f(0x00800000u); /* 2^-126 */
    k += 126;
  }
  return x * cm_u2f((uint32_t)(k + 127) << 23);
}

/* e^x */
CM_HD float cm_expf(float x) {
  if (x != x) return x;
  if (x > 88.7228f) return INFINITY;
  if (x < -103.973f) return 0.0f;
  const float k = rintf(x * 1.44269502f); /* round(x / ln 2) */
  /* ln 2 = 0.693115234375 + 3.1933188e-05 + 1.2996507e-08 (first two: 12 bits) */
  float r = CM_FMAF(-k, 0.693115234375f, x);
  r = CM_FMAF(-k, 3.193318843841553e-05f, r);
  r = CM_FMAF(-k, 1.2996506981721723e-08f, r);
  /* e^r, |r| <= 0.347: Taylor series to r^8 */
  float p = 2.48015873e-05f; /* 1/8! */
  p = CM_FMAF(p, r, 1.98412698e-04f);
  p = CM_FMAF(p, r, 1.38888889e-03f);
  p = CM_FMAF(p, r, 8.33333333e-03f);
  p = CM_FMAF(p, r, 4.16666667e-02f);
  p = CM_FMAF(p, r, 1.66666667e-01f);
  p = CM_FMAF(p, r, 0.5f);
  p = CM_FMAF(p, r, 1.0f);
  p = CM_FMAF(p, r, 1.0f);
  return cm_scale2(p, (int)k);
}

/* x * 2^k for |k| <= 2100 (double), with exact power-of-two factors */
CM_HD double cm_scale2d(double x, int k) {
  while (k > 1000) {
    x = x * 0x1p1000;
    k -= 1000;
  }
  while (k < -1000) {
    x = x * 0x1p-1000;
    k += 1000;
  }
  uint64_t b = (uint64_t)(k + 1023) << 52;
  double f;
#if defined(__CUDA_ARCH__)
  f = __longlong_as_double((long long)b);
#else
  memcpy(&f, &b, 8);
#endif
  return x * f;
}

/* e^x in double precision: k = round(x / ln 2), r = x - k ln 2 with ln 2 split
 * into 0x1.62e42fp-1 (25 bits, so k * hi is exact) + 0x1.df473de6af279p-26,
 * then the Taylor series of e^r to r^13 for |r| <= 0.347 (truncation below
 * 1e-17 relative), scaled by 2^k. */
CM_HD double cm_exp(double x) {
  if (x != x) return x;
  if (x > 709.79) return INFINITY;
  if (x < -745.2) return 0.0;
  const double k = rint(x * 1.4426950408889634);
  double r = CM_FMA(-k, 0x1.62e42fp-1, x);
  r = CM_FMA(-k, 0x1.df473de6af279p-26, r);
  double p = 1.0 / 6227020800.0; /* 1/13! */
  p = CM_FMA(p, r, 1.0 / 479001600.0);
  p = CM_FMA(p, r, 1.0 / 39916800.0);
  p = CM_FMA(p, r, 1.0 / 3628800.0);
  p = CM_FMA(p, r, 1.0 / 362880.0);
  p = CM_FMA(p, r, 1.0 / 40320.0);
  p = CM_FMA(p, r, 1.0 / 5040.0);
  p = CM_FMA(p, r, 1.0 / 720.0);
  p = CM_FMA(p, r, 1.0 / 120.0);
  p = CM_FMA(p, r, 1.0 / 24.0);
  p = CM_FMA(p, r, 1.0 / 6.0);
  p = CM_FMA(p, r, 0.5);
  p = CM_FMA(p, r, 1.0);
  p = CM_FMA(p, r, 1.0);
  return cm_scale2d(p, (int)k);
}

/* natural logarithm (double): x = 2^e m with m in [sqrt(1/2), sqrt(2)),
 * log m = 2 atanh(s), s = (m - 1) / (m + 1), |s| <= 0.1716, series to s^23 */
CM_HD double cm_log(double x) {
  if (!(x > 0.0)) return x == 0.0 ? -INFINITY : NAN;
  if (x == INFINITY) return x;
  uint64_t b;
  int adj = 0;
#if defined(__CUDA_ARCH__)
  b = (uint64_t)__double_as_longlong(x);
#else
  memcpy(&b, &x, 8);
#endif
  if (((b >> 52) & 0x7FF) == 0) { /* subnormal */
    x = x * 0x1p54;
    adj = 54;
#if defined(__CUDA_ARCH__)
    b = (uint64_t)__double_as_longlong(x);
#else
    memcpy(&b, &x, 8);
#endif
  }
  int e = (int)((b >> 52) & 0x7FF) - 1023 - adj;
  uint64_t mb = (b & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull;
  double m;
#if defined(__CUDA_ARCH__)
  m = __longlong_as_double((long long)mb);
#else
  memcpy(&m, &mb, 8);
#endif
  if (m > 1.4142135623730951) {
    m = m * 0.5;
    e += 1;
  }
  const double f = m - 1.0;
  const double s = f / (m + 1.0);
  const double z = s * s;
  double p = 1.0 / 23.0;
  p = CM_FMA(p, z, 1.0 / 21.0);
  p = CM_FMA(p, z, 1.0 / 19.0);
  p = CM_FMA(p, z, 1.0 / 17.0);
  p = CM_FMA(p, z, 1.0 / 15.0);
  p = CM_FMA(p, z, 1.0 / 13.0);
  p = CM_FMA(p, z, 1.0 / 11.0);
  p = CM_FMA(p, z, 1.0 / 9.0);
  p = CM_FMA(p, z, 1.0 / 7.0);
  p = CM_FMA(p, z, 1.0 / 5.0);
  p = CM_FMA(p, z, 1.0 / 3.0);
  /* log m = 2 s + 2 s z p, written as f - (f - 2 s) + ... to keep f's bits:
   * 2 s = f - s f, so log m = f - s (f - 2 z p) */
  const double lm = f - s * (f - 2.0 * z * p);
  const double ed = (double)e;
  return ed * 0x1.62e42fp-1 + (ed * 0x1.df473de6af279p-26 + lm);
}

/* natural logarithm, x > 0 */
CM_HD float cm_logf(float x) {
  if (!(x > 0.0f)) return x == 0.0f ? -INFINITY : NAN;
  if (x == INFINITY) return x;
  uint32_t b = cm_f2u(x);
  int e = (int)((b >> 23) & 0xFFu) - 127;
  if (((b >> 23) & 0xFFu) == 0) { /* subnormal */
    x = x * 8388608.0f;        /* 2^23 */
    b = cm_f2u(x);
    e = (int)((b >> 23) & 0xFFu) - 127 - 23;
  }
  float m = cm_u2f((b & 0x007FFFFFu) | 0x3F800000u); /* [1, 2) */
  if (m > 1.41421356f) {
    m = m * 0.5f;
    e += 1;
  }
  /* log m = 2 atanh(s), s = (m - 1)/(m + 1), |s| <= 0.1716 */
  const float s = (m - 1.0f) / (m + 1.0f);
  const float s2 = s * s;
  float p = 0.0769230769f; /* 1/13 */
  p = CM_FMAF(p, s2, 0.0909090909f);
  p = CM_FMAF(p, s2, 0.111111111f);
  p = CM_FMAF(p, s2, 0.142857143f);
  p = CM_FMAF(p, s2, 0.2f);
  p = CM_FMAF(p, s2, 0.333333333f);
  p = CM_FMAF(p, s2, 1.0f);
  const float lm = 2.0f * s * p;
  const float fe = (float)e;
  return CM_FMAF(fe, 0.693115234375f, CM_FMAF(fe, 3.193318843841553e-05f, CM_FMAF(fe, 1.2996506981721723e-08f, lm)));
}

/* sin and cos of x (|x| up to about 1e4) */
CM_HD void cm_sincosf(float x, float* sp, float* cp) {
  const float k = rintf(x * 0.636619747f); /* x / (pi/2) */
  /* pi/2 = 1.5703125 + 4.8375130e-04 + 7.5497901e-08 (first two: 12 bits) */
  float r = CM_FMAF(-k, 1.5703125f, x);
  r = CM_FMAF(-k, 4.837512969970703e-04f, r);
  r = CM_FMAF(-k, 7.549790126404332e-08f, r);
  const float r2 = r * r;
  /* |r| <= pi/4: Taylor series to r^11 (sin) and r^12 (cos) */
  float ps = -2.50521084e-08f;
  ps = CM_FMAF(ps, r2, 2.75573192e-06f);
  ps = CM_FMAF(ps, r2, -1.98412698e-04f);
  ps = CM_FMAF(ps, r2, 8.33333333e-03f);
  ps = CM_FMAF(ps, r2, -1.66666667e-01f);
  const float sn = CM_FMAF(r * r2, ps, r);
  float pc = 2.08767570e-09f;
  pc = CM_FMAF(pc, r2, -2.75573192e-07f);
  pc = CM_FMAF(pc, r2, 2.48015873e-05f);
  pc = CM_FMAF(pc, r2, -1.38888889e-03f);
  pc = CM_FMAF(pc, r2, 4.16666667e-02f);
  pc = CM_FMAF(pc, r2, -0.5f);
  const float cs = CM_FMAF(r2, pc, 1.0f);
  const int q = ((int)k) & 3;
  if (q == 0) {
    *sp = sn;
    *cp = cs;
  } else if (q == 1) {
    *sp = cs;
    *cp = -sn;
  } else if (q == 2) {
    *sp = -sn;
    *cp = -cs;
  } else {
    *sp = -cs;
    *cp = sn;
  }
}

CM_HD float cm_cosf(float x) {
  float s, c;
  cm_sincosf(x, &s, &c);
  return c;
}

CM_HD float cm_sinf(float x) {
  float s, c;
  cm_sincosf(x, &s, &c);
  return s;
}

/* atan(t) for |t| <= 2 - sqrt 3 */
CM_HD float cm_atan_small(float t) {
  const float t2 = t * t;
  float p = 0.0769230769f; /* 1/13 */
  p = CM_FMAF(p, t2, -0.0909090909f);
  p = CM_FMAF(p, t2, 0.111111111f);
  p = CM_FMAF(p, t2, -0.142857143f);
  p = CM_FMAF(p, t2, 0.2f);
  p = CM_FMAF(p, t2, -0.333333333f);
  return CM_FMAF(t * t2, p, t);
}

/* atan2(y, x); returns 0 for x = y = 0 */
CM_HD float cm_atan2f(float y, float x) {
  const float ax = fabsf(x), ay = fabsf(y);
  if (ax == 0.0f && ay == 0.0f) return 0.0f;
  const int swap = ay > ax;
  const float t = swap ? ax / ay : ay / ax; /* [0, 1] */
  float a;
  if (t > 0.267949194f) {
    /* atan t = pi/6 + atan((t sqrt3 - 1)/(t + sqrt3)) */
    const float tt = (t * 1.73205081f - 1.0f) / (t + 1.73205081f);
    a = 0.523598790f + cm_atan_small(tt);
  } else {
    a = cm_atan_small(t);
  }
  if (swap) a = 1.57079637f - a;
  if (x < 0.0f) a = 3.14159274f - a;
  return y < 0.0f ? -a : a;
}

/* acos(x), x in [-1, 1] */
CM_HD float cm_acosf(float x) { return cm_atan2f(sqrtf((1.0f - x) * (1.0f + x)), x); }

#endif /* CRITMC_FPMATH_H */
