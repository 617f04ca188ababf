/* rg_pow.h -- the power function of the library's uncontracted build.
 *
 * The reference evaluates x**y (gfortran: the C library's pow) for the
 * entropy variable p/rho**Gamma (calflx.f90:474, caluu.f90:303), for the
 * floors dmin r**-1.5 and pmin r**-2.5 (correction.f90:897-898) and inside
 * the primitive recovery (recov.f90:1044-1186).  Two math libraries (the
 * host's and CUDA's) round a few of those powers differently in the last
 * bit, and MP5's limiter switches amplify such bits over a thousand steps.
 * This header gives one power function, written only with IEEE-754 basic
 * operations (add, multiply, divide, fused multiply-add), so that the host
 * and the device evaluate it to the same bits: libraishin_gpu_exact.so uses it
 * for every power of the step, and a host program that uses it too (a CPU
 * restatement of the step, or the driver's own checks) reproduces the GPU's
 * arithmetic exactly.
 *
 * Method.  x = 2^e m with m in [sqrt(1/2), sqrt(2)); ln m = 2 atanh(s),
 * s = (m-1)/(m+1), by its Taylor series 2 (s + s^3/3 + s^5/5 + ...)
 * (Abramowitz & Stegun 4.1.27); ln x = e ln 2 + ln m; t = y ln x.  Then
 * exp(t) = 2^k exp(r) with r = t - k ln 2, |r| <= ln(2)/2 (Cody & Waite
 * reduction), exp(r) = exp(r/16)^16, exp(r/16) by its Taylor series.  The
 * leading terms are carried in double-double arithmetic (Dekker 1971; the
 * sum and product of Hida, Li & Bailey, "Algorithms for quad-double precision
 * floating point arithmetic", 2001), the tails in double, so t carries a
 * relative error near 2^-68 and the result is rounded once from about 100
 * bits: within 0.5 + |t| 2^-16 units in the last place, i.e. correctly rounded
 * for all but a small fraction of inputs.
 *
 * Special values follow C99 pow: pow(x, 0) = 1 and pow(1, y) = 1 (NaN
 * included), otherwise NaN in -> NaN out, a negative x with a non-integer y gives NaN, x = 0 or infinite and
 * infinite y give the limits.  Results below 2^-1022 are rounded twice (to
 * 53 bits, then to the subnormal grid); the step never produces them.
 *
 * Header-only C++ (host and CUDA device).  Build host code that includes it
 * without floating-point contraction (-ffp-contract=off); device code uses
 * rounding intrinsics, so it is unaffected by --fmad.
 */
#ifndef RG_POW_H
#define RG_POW_H

#include <stdint.h>
#include <string.h>
#include <math.h>

#if defined(__CUDACC__)
#define RGM_FN __host__ __device__ __forceinline__
#else
#define RGM_FN static inline
#endif

namespace rgm {

RGM_FN double add(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dadd_rn(a, b);
#else
  return a + b;
#endif
}
RGM_FN double sub(double a, double b) { return add(a, -b); }
RGM_FN double mul(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}
RGM_FN double dvd(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __ddiv_rn(a, b);
#else
  return a / b;
#endif
}
RGM_FN double fmad(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
  return __fma_rn(a, b, c);
#else
  return fma(a, b, c);
#endif
}
RGM_FN uint64_t bits(double x) {
#if defined(__CUDA_ARCH__)
  return (uint64_t)__double_as_longlong(x);
#else
  uint64_t u;
  memcpy(&u, &x, sizeof u);
  return u;
#endif
}
RGM_FN double from_bits(uint64_t u) {
#if defined(__CUDA_ARCH__)
  return __longlong_as_double((long long)u);
#else
  double x;
  memcpy(&x, &u, sizeof x);
  return x;
#endif
}

// Double-double value h + l with |l| <= ulp(h)/2.
struct dd {
  double h, l;
};

RGM_FN dd two_sum(double a, double b) {
  const double s = add(a, b);
  const double bb = sub(s, a);
  return dd{s, add(sub(a, sub(s, bb)), sub(b, bb))};
}
RGM_FN dd fast_two_sum(double a, double b) {  // |a| >= |b| or a == 0
  const double s = add(a, b);
  return dd{s, sub(b, sub(s, a))};
}
RGM_FN dd two_prod(double a, double b) {
  const double p = mul(a, b);
  return dd{p, fmad(a, b, -p)};
}
RGM_FN dd dd_add(dd x, dd y) {
  dd s = two_sum(x.h, y.h);
  const dd t = two_sum(x.l, y.l);
  s.l = add(s.l, t.h);
  s = fast_two_sum(s.h, s.l);
  s.l = add(s.l, t.l);
  return fast_two_sum(s.h, s.l);
}
RGM_FN dd dd_add_d(dd x, double b) {
  dd s = two_sum(x.h, b);
  s.l = add(s.l, x.l);
  return fast_two_sum(s.h, s.l);
}
RGM_FN dd dd_mul(dd x, dd y) {
  dd p = two_prod(x.h, y.h);
  p.l = add(p.l, add(mul(x.h, y.l), mul(x.l, y.h)));
  return fast_two_sum(p.h, p.l);
}
RGM_FN dd dd_mul_d(dd x, double b) {
  dd p = two_prod(x.h, b);
  p.l = add(p.l, mul(x.l, b));
  return fast_two_sum(p.h, p.l);
}

// ln 2, 1/3 and 1/5 split into two doubles (hi = the nearest double, lo = the
// nearest double to the remainder).
#define RGM_LN2_H 0x1.62e42fefa39efp-1
#define RGM_LN2_L 0x1.abc9e3b39803fp-56
#define RGM_INV_LN2 0x1.71547652b82fep+0
#define RGM_SQRT2 0x1.6a09e667f3bcdp+0

// ln x as a double-double for a finite x > 0.
RGM_FN dd log_dd(double x) {
  int e = 0;
  uint64_t ix = bits(x);
  if ((ix >> 52) == 0) {  // subnormal: scale into the normal range
    x = mul(x, 0x1p54);
    ix = bits(x);
    e = -54;
  }
  e += (int)(ix >> 52) - 1023;
  double m = from_bits((ix & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);  // [1, 2)
  if (m > RGM_SQRT2) {
    m = mul(m, 0.5);
    e += 1;
  }
  const double f = sub(m, 1.0);  // exact: m lies in [1/2, 2]
  const dd d = two_sum(m, 1.0);
  const double sh = dvd(f, d.h);
  const double rem = sub(fmad(-sh, d.h, f), mul(sh, d.l));
  const dd s = fast_two_sum(sh, dvd(rem, d.h));  // s = (m-1)/(m+1), |s| <= 0.1716
  const dd z = dd_mul(s, s);
  const dd z2 = dd_mul(z, z);
  // T = z/3 + z^2/5 + z^3 (1/7 + z/9 + ... + z^9/25)
  const double zh = z.h;
  double p = 1.0 / 25.0;
  p = add(mul(p, zh), 1.0 / 23.0);
  p = add(mul(p, zh), 1.0 / 21.0);
  p = add(mul(p, zh), 1.0 / 19.0);
  p = add(mul(p, zh), 1.0 / 17.0);
  p = add(mul(p, zh), 1.0 / 15.0);
  p = add(mul(p, zh), 1.0 / 13.0);
  p = add(mul(p, zh), 1.0 / 11.0);
  p = add(mul(p, zh), 1.0 / 9.0);
  p = add(mul(p, zh), 1.0 / 7.0);
  dd T = dd_add(dd_mul(z, dd{0x1.5555555555555p-2, 0x1.5555555555555p-56}),
                dd_mul(z2, dd{0x1.999999999999ap-3, -0x1.999999999999ap-57}));
  T = dd_add_d(T, mul(mul(z2.h, zh), p));
  // ln m = 2 s (1 + T)
  dd L = dd_add(s, dd_mul(s, T));
  L.h = mul(L.h, 2.0);
  L.l = mul(L.l, 2.0);
  const double ed = (double)e;
  dd E = two_prod(ed, RGM_LN2_H);
  E = fast_two_sum(E.h, add(E.l, mul(ed, RGM_LN2_L)));
  return dd_add(E, L);
}

// exp(t) for a double-double t, rounded once to double.
RGM_FN double exp_dd(dd t) {
  if (t.h != t.h) return t.h;
  if (t.h > 710.0) return from_bits(0x7ff0000000000000ULL);
  if (t.h < -746.0) return 0.0;
  const double kd = rint(mul(t.h, RGM_INV_LN2));
  const dd a = two_prod(kd, RGM_LN2_H);
  dd r = dd_add(t, dd{-a.h, -a.l});
  r = dd_add_d(r, -mul(kd, RGM_LN2_L));  // |r| <= ln(2)/2 + tiny
  r.h = mul(r.h, 0.0625);
  r.l = mul(r.l, 0.0625);
  // exp(r) - 1 = r + r^2/2 + r^3 (1/6 + r/24 + ... + r^7/10!)
  const double rh = r.h;
  double p = 1.0 / 3628800.0;
  p = add(mul(p, rh), 1.0 / 362880.0);
  p = add(mul(p, rh), 1.0 / 40320.0);
  p = add(mul(p, rh), 1.0 / 5040.0);
  p = add(mul(p, rh), 1.0 / 720.0);
  p = add(mul(p, rh), 1.0 / 120.0);
  p = add(mul(p, rh), 1.0 / 24.0);
  p = add(mul(p, rh), 1.0 / 6.0);
  const dd r2 = dd_mul(r, r);
  dd em1 = dd_add(r, dd{mul(r2.h, 0.5), mul(r2.l, 0.5)});
  em1 = dd_add_d(em1, mul(mul(r2.h, rh), p));
  // (1 + E)^2 - 1 = 2E + E^2, four times: exp(r) - 1
  for (int n = 0; n < 4; ++n) em1 = dd_add(dd{mul(em1.h, 2.0), mul(em1.l, 2.0)}, dd_mul(em1, em1));
  const double v = dd_add_d(em1, 1.0).h;  // exp(r), rounded to nearest
  const int k = (int)kd;
  if (k >= -1022 && k <= 1023) return mul(v, from_bits((uint64_t)(k + 1023) << 52));
  if (k > 1023) return mul(mul(v, 0x1p1023), from_bits((uint64_t)(k - 1023 + 1023) << 52));
  if (k < -1076) return 0.0;
  return mul(mul(v, from_bits((uint64_t)(k + 54 + 1023) << 52)), 0x1p-54);
}

// x**y with C99 semantics for the special values.
RGM_FN double pow(double x, double y) {
  if (y == 0.0 || x == 1.0) return 1.0;
  if (x != x || y != y) return add(x, y);
  const double ay = fabs(y);
  bool neg = false;
  if (bits(x) >> 63) {  // x < 0 or x = -0
    if (ay < 0x1p53) {
      const double yt = trunc(y);
      if (yt != y) return x == 0.0 ? (y > 0.0 ? 0.0 : from_bits(0x7ff0000000000000ULL))
                                   : from_bits(0x7ff8000000000000ULL);
      neg = (((int64_t)yt) & 1) != 0;
    }
    x = -x;
  }
  const double inf = from_bits(0x7ff0000000000000ULL);
  double r;
  if (ay == inf) {
    if (x == 1.0) return 1.0;
    r = ((x < 1.0) == (y > 0.0)) ? 0.0 : inf;
  } else if (x == 0.0) {
    r = y > 0.0 ? 0.0 : inf;
  } else if (x == inf) {
    r = y > 0.0 ? inf : 0.0;
  } else {
    const dd L = log_dd(x);
    dd t = two_prod(L.h, y);
    t = fast_two_sum(t.h, add(t.l, mul(L.l, y)));
    r = exp_dd(t);
  }
  return neg ? -r : r;
}

}  // namespace rgm

#endif /* RG_POW_H */
