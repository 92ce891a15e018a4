/*
 * gx_math.h -- the elementary functions of the FP64 parity build.
 *
 * The FP64 parity variant of the transport kernels (gx_transport_parity.cu)
 * and the oracle's parity build (oracle/, compiled with -DGXO_OWN_MATH) both
 * take log, exp, pow, sin, cos, expm1 and log1p from this one header, written
 * in plain C with IEEE double operations only (+, -, *, /, sqrt, floor and
 * exponent-field access), each sum and product rounded on its own: on the
 * device through __dadd_rn / __dmul_rn, which are never fused into an FMA,
 * on the host with contraction off (-ffp-contract=off).  The same inputs
 * therefore give the same bits on the GPU and on the CPU, which the libraries'
 * own functions (CUDA's and glibc's) do not promise; the step loop then
 * follows the same path on both, track by track.
 *
 * Methods (published, restated here; every constant is derived from the
 * mathematics, not taken from a library):
 *   - Argument reduction after Cody and Waite (W. J. Cody, W. Waite,
 *     "Software Manual for the Elementary Functions", Prentice-Hall 1980):
 *     x = k c + r with c = ln 2 (exp, expm1) or pi/2 (sin, cos) split into
 *     parts of 30 significant bits (so that k times a part is exact for
 *     |k| < 2^23) and a full-precision tail.
 *   - exp(r), expm1(r) on |r| <= ln 2 / 2: the Taylor series of e^r through
 *     r^13, as r + r^2 P(r) (remainder below 1e-17 relative).
 *   - sin r, cos r on |r| <= pi/4: Taylor series through r^17 and r^18.
 *   - log(x) = e ln 2 + log(1 + f), 1 + f = x 2^-e in [sqrt(1/2), sqrt(2)]:
 *     log(1 + f) = 2 atanh(s), s = f / (2 + f), as f - s (f - 2 s^2 T(s^2))
 *     with T(z) = sum z^k / (2k + 3), k = 0..10 (remainder below 1e-18).
 *   - log1p(x): the same kernel with f = x exactly when 1 + x lies in that
 *     interval; otherwise log(u) + (x - (u - 1)) / u for u = 1 + x rounded
 *     (D. Goldberg, ACM Computing Surveys 23 (1991) 5-48, the correction of
 *     a rounded 1 + x).
 *   - pow(x, y) = exp(y log x) with log x carried as a sum of two doubles and
 *     the product y log x formed exactly with Dekker's algorithm (T. J.
 *     Dekker, Numer. Math. 18 (1971) 224-242), so that the error does not grow
 *     with |y log x|.
 * Accuracy (checked against glibc and CUDA in the tests): log, exp, sin, cos
 * within 1 ulp, expm1, log1p, pow within 2 ulp, on the arguments the
 * transport uses (sin, cos: |x| < 1e6; pow: x >= 0).  Not correctly rounded,
 * and not meant to be: they are meant to be the same on both machines.
 */
#ifndef GX_MATH_H
#define GX_MATH_H

#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define GXM_FN static __host__ __device__ __forceinline__
#else
#define GXM_FN static inline
#endif

/* one rounding per operation, never fused */
GXM_FN double gxm_add(double a, double b)
{
#if defined(__CUDA_ARCH__)
  return __dadd_rn(a, b);
#else
  return a + b;
#endif
}
GXM_FN double gxm_sub(double a, double b)
{
#if defined(__CUDA_ARCH__)
  return __dsub_rn(a, b);
#else
  return a - b;
#endif
}
GXM_FN double gxm_mul(double a, double b)
{
#if defined(__CUDA_ARCH__)
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}
GXM_FN uint64_t gxm_bits(double x)
{
#if defined(__CUDA_ARCH__)
  return (uint64_t)__double_as_longlong(x);
#else
  union { double d; uint64_t u; } v;
  v.d = x;
  return v.u;
#endif
}
GXM_FN double gxm_from_bits(uint64_t u)
{
#if defined(__CUDA_ARCH__)
  return __longlong_as_double((long long)u);
#else
  union { double d; uint64_t u; } v;
  v.u = u;
  return v.d;
#endif
}

/* ln 2 = GXM_LN2_HI + GXM_LN2_LO (hi: 30 significant bits) */
#define GXM_LN2_HI 0x1.62e42ffp-1
#define GXM_LN2_LO -0x1.718432a1b0e26p-35
#define GXM_INV_LN2 0x1.71547652b82fep+0
/* pi / 2 = P1 + P2 + P3 (P1, P2: 30 significant bits) */
#define GXM_PIO2_1 0x1.921fb548p+0
#define GXM_PIO2_2 -0x1.de973dc8p-31
#define GXM_PIO2_3 -0x1.9d9cceba3f91fp-62
#define GXM_TWO_OVER_PI 0x1.45f306dc9c883p-1
#define GXM_SQRT2 0x1.6a09e667f3bcdp+0
#define GXM_INF gxm_from_bits(0x7ff0000000000000ull)

/* 1/n! rounded to double */
#define GXM_F2 0x1p-1
#define GXM_F3 0x1.5555555555555p-3
#define GXM_F4 0x1.5555555555555p-5
#define GXM_F5 0x1.1111111111111p-7
#define GXM_F6 0x1.6c16c16c16c17p-10
#define GXM_F7 0x1.a01a01a01a01ap-13
#define GXM_F8 0x1.a01a01a01a01ap-16
#define GXM_F9 0x1.71de3a556c734p-19
#define GXM_F10 0x1.27e4fb7789f5cp-22
#define GXM_F11 0x1.ae64567f544e4p-26
#define GXM_F12 0x1.1eed8eff8d898p-29
#define GXM_F13 0x1.6124613a86d09p-33
#define GXM_F14 0x1.93974a8c07c9dp-37
#define GXM_F15 0x1.ae7f3e733b81fp-41
#define GXM_F16 0x1.ae7f3e733b81fp-45
#define GXM_F17 0x1.952c77030ad4ap-49
#define GXM_F18 0x1.6827863b97d97p-53

/* (e^r - 1 - r) / r^2 = 1/2! + r/3! + ... + r^11/13!, |r| <= ln2/2 */
GXM_FN double gxm_exp_tail(double r)
{
  double p = GXM_F13;
  p = gxm_add(GXM_F12, gxm_mul(r, p));
  p = gxm_add(GXM_F11, gxm_mul(r, p));
  p = gxm_add(GXM_F10, gxm_mul(r, p));
  p = gxm_add(GXM_F9, gxm_mul(r, p));
  p = gxm_add(GXM_F8, gxm_mul(r, p));
  p = gxm_add(GXM_F7, gxm_mul(r, p));
  p = gxm_add(GXM_F6, gxm_mul(r, p));
  p = gxm_add(GXM_F5, gxm_mul(r, p));
  p = gxm_add(GXM_F4, gxm_mul(r, p));
  p = gxm_add(GXM_F3, gxm_mul(r, p));
  p = gxm_add(GXM_F2, gxm_mul(r, p));
  return p;
}

/* e^r - 1 for |r| <= ln2/2 */
GXM_FN double gxm_expm1_small(double r) { return gxm_add(r, gxm_mul(gxm_mul(r, r), gxm_exp_tail(r))); }

/* e 2^k for e in [0.5, 2]: exact unless the result is subnormal */
GXM_FN double gxm_scale2(double e, int k)
{
  if (k > 1023) {
    e = gxm_mul(e, 0x1p1023);
    k -= 1023;
    if (k > 1023) k = 1023;
  } else if (k < -1022) {
    e = gxm_mul(e, 0x1p-1022);
    k += 1022;
    if (k < -1022) k = -1022;
  }
  return gxm_mul(e, gxm_from_bits((uint64_t)(k + 1023) << 52));
}

/* x = k ln2 + r, |r| <= ln2/2 (slightly more at the rounding edge) */
GXM_FN double gxm_reduce_ln2(double x, double *kd)
{
  double k = floor(gxm_add(gxm_mul(x, GXM_INV_LN2), 0.5));
  *kd = k;
  return gxm_sub(gxm_sub(x, gxm_mul(k, GXM_LN2_HI)), gxm_mul(k, GXM_LN2_LO));
}

GXM_FN double gxm_exp(double x)
{
  if (x != x) return x;
  if (x > 709.79) return GXM_INF;
  if (x < -745.2) return 0.0;
  double kd;
  double r = gxm_reduce_ln2(x, &kd);
  double e = gxm_add(1.0, gxm_expm1_small(r));
  return gxm_scale2(e, (int)kd);
}

GXM_FN double gxm_expm1(double x)
{
  if (x != x) return x;
  if (x > 709.79) return GXM_INF;
  if (x < -40.0) return -1.0;
  if (x > -0.34 && x < 0.34) return gxm_expm1_small(x);
  double kd;
  double r = gxm_reduce_ln2(x, &kd);
  int k = (int)kd;
  double em1 = gxm_expm1_small(r);
  if (k > 60) return gxm_scale2(gxm_add(1.0, em1), k);
  double two = gxm_from_bits((uint64_t)(k + 1023) << 52); /* 2^k, -58 <= k <= 60 */
  /* e^x - 1 = 2^k (e^r - 1) + (2^k - 1); both terms exact for these k but the last */
  return gxm_add(gxm_mul(two, em1), gxm_sub(two, 1.0));
}

/* log(1 + f) for f with 1 + f in [sqrt(1/2), sqrt(2)]: f - corr, corr returned */
GXM_FN double gxm_log1p_corr(double f)
{
  double s = f / gxm_add(2.0, f);
  double z = gxm_mul(s, s);
  double t = 0x1.642c8590b2164p-5; /* 1/23 */
  t = gxm_add(0x1.8618618618618p-5 /* 1/21 */, gxm_mul(z, t));
  t = gxm_add(0x1.af286bca1af28p-5 /* 1/19 */, gxm_mul(z, t));
  t = gxm_add(0x1.e1e1e1e1e1e1ep-5 /* 1/17 */, gxm_mul(z, t));
  t = gxm_add(0x1.1111111111111p-4 /* 1/15 */, gxm_mul(z, t));
  t = gxm_add(0x1.3b13b13b13b14p-4 /* 1/13 */, gxm_mul(z, t));
  t = gxm_add(0x1.745d1745d1746p-4 /* 1/11 */, gxm_mul(z, t));
  t = gxm_add(0x1.c71c71c71c71cp-4 /* 1/9 */, gxm_mul(z, t));
  t = gxm_add(0x1.2492492492492p-3 /* 1/7 */, gxm_mul(z, t));
  t = gxm_add(0x1.999999999999ap-3 /* 1/5 */, gxm_mul(z, t));
  t = gxm_add(0x1.5555555555555p-2 /* 1/3 */, gxm_mul(z, t));
  /* 2 atanh(s) = 2s + s (2 z T), 2s = f - s f */
  return gxm_mul(s, gxm_sub(f, gxm_mul(gxm_add(z, z), t)));
}

/* log x = hi + lo (x > 0 finite), hi the rounded value of e ln2_hi + f */
GXM_FN void gxm_log_parts(double x, double *hi, double *lo)
{
  uint64_t u = gxm_bits(x);
  int e = 0;
  if (u < 0x0010000000000000ull) { /* subnormal */
    x = gxm_mul(x, 0x1p54);
    u = gxm_bits(x);
    e = -54;
  }
  e += (int)(u >> 52) - 1023;
  double m = gxm_from_bits((u & 0x000fffffffffffffull) | 0x3ff0000000000000ull); /* [1, 2) */
  if (m > GXM_SQRT2) {
    m = gxm_mul(m, 0.5);
    e += 1;
  }
  double f = gxm_sub(m, 1.0); /* exact */
  double corr = gxm_log1p_corr(f);
  double ed = (double)e;
  double a = gxm_mul(ed, GXM_LN2_HI); /* exact */
  double h = gxm_add(a, f);
  /* the rounding error of h, exactly (|a| >= |f| whenever a != 0) */
  double err = (e != 0) ? gxm_sub(f, gxm_sub(h, a)) : 0.0;
  *hi = h;
  *lo = gxm_add(err, gxm_sub(gxm_mul(ed, GXM_LN2_LO), corr));
}

GXM_FN double gxm_log(double x)
{
  if (x != x) return x;
  if (x <= 0.0) return x == 0.0 ? -GXM_INF : (x - x) / (x - x);
  if (x == GXM_INF) return x;
  double h, l;
  gxm_log_parts(x, &h, &l);
  return gxm_add(h, l);
}

GXM_FN double gxm_log1p(double x)
{
  if (x != x) return x;
  if (x == 0.0) return x;
  if (x <= -1.0) return x == -1.0 ? -GXM_INF : (x - x) / (x - x);
  if (x == GXM_INF) return x;
  if (x > -0.29289321881345248 && x < 0.41421356237309503) return gxm_sub(x, gxm_log1p_corr(x));
  double u = gxm_add(1.0, x);
  double c = (u < 0x1p53) ? gxm_sub(x, gxm_sub(u, 1.0)) / u : 0.0;
  return gxm_add(gxm_log(u), c);
}

/* Dekker: a b = p + e exactly (no overflow assumed) */
GXM_FN void gxm_split(double a, double *h, double *l)
{
  double c = gxm_mul(134217729.0, a); /* 2^27 + 1 */
  *h = gxm_sub(c, gxm_sub(c, a));
  *l = gxm_sub(a, *h);
}
GXM_FN void gxm_two_prod(double a, double b, double *p, double *e)
{
  double ah, al, bh, bl;
  *p = gxm_mul(a, b);
  gxm_split(a, &ah, &al);
  gxm_split(b, &bh, &bl);
  *e = gxm_add(gxm_add(gxm_add(gxm_sub(gxm_mul(ah, bh), *p), gxm_mul(ah, bl)), gxm_mul(al, bh)), gxm_mul(al, bl));
}

/* x^y for x >= 0 (x < 0 gives NaN) */
GXM_FN double gxm_pow(double x, double y)
{
  if (y == 0.0 || x == 1.0) return 1.0;
  if (x != x || y != y) return x + y;
  if (x < 0.0) return (x - x) / (x - x);
  if (x == 0.0) return y > 0.0 ? 0.0 : GXM_INF;
  if (x == GXM_INF) return y > 0.0 ? GXM_INF : 0.0;
  double lh, ll, ph, pe;
  gxm_log_parts(x, &lh, &ll);
  gxm_two_prod(y, lh, &ph, &pe);
  double tl = gxm_add(pe, gxm_mul(y, ll));
  double t = gxm_add(ph, tl);
  double tt = gxm_sub(tl, gxm_sub(t, ph)); /* what t lost of tl */
  double e = gxm_exp(t);
  if (e == 0.0 || e == GXM_INF) return e;
  return gxm_add(e, gxm_mul(e, tt)); /* e^(t + tt) */
}

/* sin and cos of x (|x| < 1e6 for full accuracy) */
GXM_FN void gxm_sincos(double x, double *sn, double *cs)
{
  if (gxm_sub(x, x) != 0.0) { /* inf or NaN */
    *sn = *cs = gxm_sub(x, x);
    return;
  }
  double kd = floor(gxm_add(gxm_mul(x, GXM_TWO_OVER_PI), 0.5));
  /* r + rl = x - k pi/2: a and b exact, r1 and r rounded with their errors
   * e1, e2 recovered exactly (|a| >= |b|, |r1| >= |c|) */
  double a = gxm_sub(x, gxm_mul(kd, GXM_PIO2_1)), b = gxm_mul(kd, GXM_PIO2_2), c3 = gxm_mul(kd, GXM_PIO2_3);
  double r1 = gxm_sub(a, b);
  double e1 = gxm_sub(gxm_sub(a, r1), b);
  double r = gxm_sub(r1, c3);
  double e2 = gxm_sub(gxm_sub(r1, r), c3);
  double rl = gxm_add(e1, e2);
  double q = gxm_sub(kd, gxm_mul(4.0, floor(gxm_mul(kd, 0.25)))); /* k mod 4, exact */
  double w = gxm_mul(r, r);
  /* sin r = r + r w S(w), S = -1/3! + w/5! - ... + w^7/17! */
  double S = GXM_F17;
  S = gxm_sub(gxm_mul(w, S), GXM_F15);
  S = gxm_add(gxm_mul(w, S), GXM_F13);
  S = gxm_sub(gxm_mul(w, S), GXM_F11);
  S = gxm_add(gxm_mul(w, S), GXM_F9);
  S = gxm_sub(gxm_mul(w, S), GXM_F7);
  S = gxm_add(gxm_mul(w, S), GXM_F5);
  S = gxm_sub(gxm_mul(w, S), GXM_F3);
  double s0 = gxm_add(r, gxm_mul(gxm_mul(r, w), S));
  /* cos r = 1 - (w/2 - w^2 C(w)), C = 1/4! - w/6! + ... - w^7/18! */
  double Cp = -GXM_F18;
  Cp = gxm_add(gxm_mul(w, Cp), GXM_F16);
  Cp = gxm_sub(gxm_mul(w, Cp), GXM_F14);
  Cp = gxm_add(gxm_mul(w, Cp), GXM_F12);
  Cp = gxm_sub(gxm_mul(w, Cp), GXM_F10);
  Cp = gxm_add(gxm_mul(w, Cp), GXM_F8);
  Cp = gxm_sub(gxm_mul(w, Cp), GXM_F6);
  Cp = gxm_add(gxm_mul(w, Cp), GXM_F4);
  double c0 = gxm_sub(1.0, gxm_sub(gxm_mul(0.5, w), gxm_mul(gxm_mul(w, w), Cp)));
  /* sin(r + rl) = sin r + rl cos r, cos(r + rl) = cos r - rl sin r */
  double s = gxm_add(s0, gxm_mul(rl, c0)), c = gxm_sub(c0, gxm_mul(rl, s0));
  if (q == 0.0) {
    *sn = s;
    *cs = c;
  } else if (q == 1.0) {
    *sn = c;
    *cs = -s;
  } else if (q == 2.0) {
    *sn = -s;
    *cs = -c;
  } else {
    *sn = -c;
    *cs = s;
  }
}

GXM_FN double gxm_sin(double x)
{
  double s, c;
  gxm_sincos(x, &s, &c);
  return s;
}

GXM_FN double gxm_cos(double x)
{
  double s, c;
  gxm_sincos(x, &s, &c);
  return c;
}

#endif
