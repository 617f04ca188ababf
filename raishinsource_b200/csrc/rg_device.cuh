// rg_device.cuh -- pointwise GRMHD physics of the RAISHIN update as device
// functions, templated on the arithmetic type T.  With T = double every
// expression keeps the reference Fortran's evaluation order (left to right,
// parenthesised as written), so an uncontracted build reproduces the
// reference arithmetic up to the last bit of the math library; T = float is
// the FP32 half of the mixed-precision path.  Each function states the
// reference routine it follows.
#pragma once
#include <cstdint>

#include "../../include/rg_pow.h"
#include "rg_types.h"

namespace rg {

// A power of the step with a real exponent (the reference's x**y): CUDA's pow
// in the product build; in the uncontracted build (RG_EXACT_ARITH) the
// library's own rg_pow, which a host program evaluates to the same bits, so
// that build repeats a host restatement's arithmetic exactly.
__device__ __forceinline__ double spow(double x, double y) {
#ifdef RG_EXACT_ARITH
  return rgm::pow(x, y);
#else
  return pow(x, y);
#endif
}

// Type-exact math: no silent promotion of float arguments to double.
__device__ __forceinline__ double msqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float msqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double mpow(double x, double y) { return pow(x, y); }
__device__ __forceinline__ float mpow(float x, float y) { return powf(x, y); }
__device__ __forceinline__ double mabs(double x) { return fabs(x); }
__device__ __forceinline__ float mabs(float x) { return fabsf(x); }
__device__ __forceinline__ double sgn1(double x) { return copysign(1.0, x); }
__device__ __forceinline__ float sgn1(float x) { return copysignf(1.0f, x); }
// Division in the arithmetic type: exact IEEE division in FP64 (the
// reference's arithmetic); in the FP32 half of the mixed path the fast
// approximate division (at most 2 ulp), whose error is far below that of the
// FP32 arithmetic around it.
__device__ __forceinline__ double mdiv(double a, double b) { return a / b; }
__device__ __forceinline__ float mdiv(float a, float b) { return __fdividef(a, b); }
template <typename T>
__device__ __forceinline__ T mrcp(T x) { return mdiv(T(1), x); }

template <typename T>
__device__ __forceinline__ T fmax3(T a, T b, T c) {
  T r = a;
  if (b > r) r = b;
  if (c > r) r = c;
  return r;
}
template <typename T>
__device__ __forceinline__ T fmin3(T a, T b, T c) {
  T r = a;
  if (b < r) r = b;
  if (c < r) r = c;
  return r;
}
template <typename T>
__device__ __forceinline__ T dmin2(T a, T b) { return (b < a) ? b : a; }
template <typename T>
__device__ __forceinline__ T dmax2(T a, T b) { return (b > a) ? b : a; }

// Metric at one point.  Every metric of this build (Minkowski 1, Kerr-Schild
// 303, modified Kerr-Schild 403, coord.f90:149-792) couples only (t, r, phi)
// and keeps theta diagonal, so g^{mu 3} and g_{mu 3} vanish for mu != 3 (the
// host checks this at admission).  gcov is symmetric; gcon, an LU inverse
// (coord.f90:1504), is not symmetric to the last bit and keeps its full 3x3
// block.  Sums below run over the nonzero terms in the reference's order.
// The last eight fields are functions of the others that the reference
// recomputes at every use (lapse, shift, cal3met's gcon3a diagonal,
// coord.f90:970-1013, and 1/sqrt(-g)); k_met_derive evaluates them once per
// point with the same expressions, so using them changes no result.
template <typename T>
struct MetT {
  T g00, g01, g02, g11, g12, g22, g33;                 // gcov
  T c00, c01, c02, c10, c11, c12, c20, c21, c22, c33;  // gcon
  T detg;                                              // sqrt(-g)
  T al;                                                // alpha = 1/sqrt(-g^00)
  T ial;                                               // 1/alpha
  T be1, be2;                                          // beta^r, beta^phi = alpha^2 g^0i
  T g3_11, g3_22, g3_33;                               // g^dd + (beta^d/alpha)^2
  T idetg;                                             // 1/sqrt(-g)
};
using Met = MetT<double>;

// Metric cache layout: per (i,k) point q, component c at c*nik + q, in the
// order of the MetT fields (FP64, with FP32 copies for the mixed path's FP32
// kernels).  Components a kernel does
// not use are never loaded (dead loads are removed by the compiler).
template <typename T, typename S, bool LDG = true>
__device__ __forceinline__ void load_met(const S* __restrict__ base, size_t nik, size_t q, MetT<T>& m) {
  // LDG: through the read-only cache (global memory); otherwise plain loads
  // (a shared-memory copy of the cache, component stride nik)
  const S* b = base + q;
  auto ld = [&](int c) -> T {
    if constexpr (LDG) return T(__ldg(b + c * nik));
    else return T(b[c * nik]);
  };
  m.g00 = ld(0); m.g01 = ld(1); m.g02 = ld(2);
  m.g11 = ld(3); m.g12 = ld(4); m.g22 = ld(5);
  m.g33 = ld(6);
  m.c00 = ld(7); m.c01 = ld(8); m.c02 = ld(9);
  m.c10 = ld(10); m.c11 = ld(11); m.c12 = ld(12);
  m.c20 = ld(13); m.c21 = ld(14); m.c22 = ld(15);
  m.c33 = ld(16);
  m.detg = ld(17);
  m.al = ld(18); m.ial = ld(19);
  m.be1 = ld(20); m.be2 = ld(21);
  m.g3_11 = ld(22); m.g3_22 = ld(23); m.g3_33 = ld(24);
  m.idetg = ld(25);
}

// The derived fields of one point from its base fields: calucon's
// alpha1/b1/b2 (physfunc.f90:58-66), calcha4*'s gcon3a(d,d) via cal3met
// (calcha.f90:400-410, coord.f90:990-1005) and recov1a's 1/detg.
__device__ __forceinline__ void met_derive(const double base[kMetBase], double out[kMetComps - kMetBase]) {
  const double alpha1 = 1. / sqrt(-base[7]);
  const double b1 = alpha1 * alpha1 * base[8];
  const double b2 = alpha1 * alpha1 * base[9];
  const double on1 = b1 / alpha1, on2 = b2 / alpha1, on3 = 0.0 / alpha1;
  out[0] = alpha1;
  out[1] = 1. / alpha1;
  out[2] = b1;
  out[3] = b2;
  out[4] = base[11] + (on1 * on1);
  out[5] = base[15] + (on2 * on2);
  out[6] = base[16] + (on3 * on3);
  out[7] = 1. / base[17];
}

// x**gam for the adiabatic indices of the reference's setups: 4/3
// (pram.f90:40) as x*cbrt(x) and 5/3 as x*cbrt(x)^2, otherwise pow.  The
// cube-root forms agree with pow to a few ulp at a fraction of its cost.
// Negative or NaN x keeps pow's result (NaN), as in the reference, where a
// reconstructed negative density makes the entropy variable NaN.
// kind: 1 for gam == 4/3, 2 for gam == 5/3 (bitwise), 0 otherwise.
__device__ __forceinline__ double pow_gam(double x, double gam, int kind) {
  if (kind == 0 || !(x >= 0.0)) return spow(x, gam);
  const double c = cbrt(x);
  return kind == 1 ? x * c : x * c * c;
}
__device__ __forceinline__ float pow_gam(float x, float gam, int kind) {
  if (kind == 0 || !(x >= 0.f)) return powf(x, gam);
  const float c = cbrtf(x);
  return kind == 1 ? x * c : x * c * c;
}
// x**(1-gam) for x > 0: 1/cbrt(x) for 4/3, 1/cbrt(x)^2 for 5/3.
__device__ __forceinline__ double pow_1mgam(double x, double gam, int kind) {
  if (kind == 0 || !(x > 0.0)) return spow(x, 1. - gam);
  const double c = rcbrt(x);
  return kind == 1 ? c : c * c;
}
// x**(gam-1): cbrt(x) for 4/3, cbrt(x)^2 for 5/3.
__device__ __forceinline__ double pow_gam1(double x, double gam, int kind) {
  if (kind == 0 || !(x >= 0.0)) return spow(x, gam - 1.);
  const double c = cbrt(x);
  return kind == 1 ? c : c * c;
}

// sum_{a,b=1..3} g_ab x_a x_b over the nonzero terms in (a,b) order
// (physfunc.f90:16-20, calcha.f90:251-256, correction.f90:806-811).
template <typename T>
__device__ __forceinline__ T qform3(const MetT<T>& m, T x1, T x2, T x3) {
  T s = T(0);
  s = s + m.g11 * x1 * x1;
  s = s + m.g12 * x1 * x2;
  s = s + m.g12 * x2 * x1;  // g_21 = g_12
  s = s + m.g22 * x2 * x2;
  s = s + m.g33 * x3 * x3;
  return s;
}

// g_ab v^b (physfunc.f90:161-195)
template <typename T>
__device__ __forceinline__ void lower_g(const T v[4], T o[4], const MetT<T>& m) {
  o[0] = m.g00 * v[0] + m.g01 * v[1] + m.g02 * v[2];
  o[1] = m.g01 * v[0] + m.g11 * v[1] + m.g12 * v[2];
  o[2] = m.g02 * v[0] + m.g12 * v[1] + m.g22 * v[2];
  o[3] = m.g33 * v[3];
}

// g^ab v_b (physfunc.f90:198-232)
template <typename T>
__device__ __forceinline__ void upper_gc(const T v[4], T o[4], const MetT<T>& m) {
  o[0] = m.c00 * v[0] + m.c01 * v[1] + m.c02 * v[2];
  o[1] = m.c10 * v[0] + m.c11 * v[1] + m.c12 * v[2];
  o[2] = m.c20 * v[0] + m.c21 * v[1] + m.c22 * v[2];
  o[3] = m.c33 * v[3];
}

// physfunc.f90:2-42
template <typename T>
__device__ __forceinline__ T calgfl(const T u1, const T u2, const T u3, const MetT<T>& m) {
  T utsq = qform3(m, u1, u2, u3);
  if (utsq < T(0)) {
    if (mabs(utsq) <= T(1.0e-10)) utsq = mabs(utsq);
    else utsq = T(1.e-10);
  }
  if (mabs(utsq) > T(5.e2)) utsq = T(5.0e2);
  return msqrt(T(1) + utsq);
}

// physfunc.f90:45-78 (alpha1, b1, b2 and 1/alpha1 from the metric cache)
template <typename T>
__device__ __forceinline__ void calucon(T u1, T u2, T u3, T gfl, const MetT<T>& m, T ucon[4]) {
  ucon[0] = gfl * m.ial;
  ucon[1] = u1 - gfl * m.be1 * m.ial;
  ucon[2] = u2 - gfl * m.be2 * m.ial;
  ucon[3] = u3;  // beta^theta = 0
}

// Velocity and magnetic 4-vectors of one primitive state (the common head of
// caluu1/caluu3/calflx3*/caltenr, caluu.f90:40-90).
template <typename T>
struct PST {
  T ucon[4], ucov[4], bbcon[4], bbcov[4];
  T bbsq, roh, gfl, de, pr, b1, b2, b3;
};
using PS = PST<double>;

// The state of q with a given Lorentz factor gfl (pstate below computes it
// with calgfl; the output converter uses its own clamps).
template <typename T>
__device__ __forceinline__ void pstate_gfl(const T q[9], const MetT<T>& m, T gam, T gfl, PST<T>& s) {
  s.de = q[0];
  s.pr = q[4];
  s.b1 = q[6]; s.b2 = q[7]; s.b3 = q[8];
  s.roh = s.de + (gam / (gam - T(1))) * s.pr;
  s.gfl = gfl;
  calucon(q[1], q[2], q[3], s.gfl, m, s.ucon);
  lower_g(s.ucon, s.ucov, m);
  // physfunc.f90:81-100
  s.bbcon[0] = s.b1 * s.ucov[1] + s.b2 * s.ucov[2] + s.b3 * s.ucov[3];
  s.bbcon[1] = (s.b1 + s.bbcon[0] * s.ucon[1]) * mrcp(s.ucon[0]);
  s.bbcon[2] = (s.b2 + s.bbcon[0] * s.ucon[2]) * mrcp(s.ucon[0]);
  s.bbcon[3] = (s.b3 + s.bbcon[0] * s.ucon[3]) * mrcp(s.ucon[0]);
  lower_g(s.bbcon, s.bbcov, m);
  s.bbsq = s.bbcon[0] * s.bbcov[0] + s.bbcon[1] * s.bbcov[1] + s.bbcon[2] * s.bbcov[2] + s.bbcon[3] * s.bbcov[3];
}
template <typename T>
__device__ __forceinline__ void pstate(const T q[9], const MetT<T>& m, T gam, PST<T>& s) {
  pstate_gfl(q, m, gam, calgfl(q[1], q[2], q[3], m), s);
}

// p / rho^Gamma of a state (caluu.f90:303, calflx.f90:474), computed once per state.
template <typename T>
__device__ __forceinline__ T ent_ratio(const PST<T>& s, T gam, int gkind) { return mdiv(s.pr, pow_gam(s.de, gam, gkind)); }

// caluu.f90:92-118: sqrt(-g) (rho u^t, T^t_i, T^t_t + rho u^t, s u^t, B^i).
// delta(0,n) is the literal identity of caldelta (physfunc.f90:122-158).
template <typename T>
__device__ __forceinline__ void p2c(const PST<T>& s, T gam, T detg, T u[9], T sr) {
  const T a = s.roh + s.bbsq, b = s.pr + T(0.5) * s.bbsq;
  u[0] = s.de * s.ucon[0];
#pragma unroll
  for (int m = 1; m <= 3; ++m) u[m] = a * s.ucon[0] * s.ucov[m] + b * T(0) - s.bbcon[0] * s.bbcov[m];
  u[4] = a * s.ucon[0] * s.ucov[0] + b * T(1) - s.bbcon[0] * s.bbcov[0] + s.de * s.ucon[0];
  u[5] = s.de * sr * s.ucon[0];
  u[6] = s.b1; u[7] = s.b2; u[8] = s.b3;
#pragma unroll
  for (int n = 0; n < 9; ++n) u[n] = detg * u[n];
}
template <typename T>
__device__ __forceinline__ void p2c(const PST<T>& s, T gam, int gkind, T detg, T u[9]) {
  p2c(s, gam, detg, u, ent_ratio(s, gam, gkind));
}

// calflx.f90:391-795, direction D (1 = r, 2 = phi, 3 = theta).  The induction
// flux is (u^D/u^0) B^m - (u^m/u^0) B^D with the D component set to 0.
template <int D, typename T>
__device__ __forceinline__ void flux(const PST<T>& s, T gam, T detg, T w[9], T sr) {
  const T a = s.roh + s.bbsq, b = s.pr + T(0.5) * s.bbsq;
  const T ud = s.ucon[D];
  const T bc[4] = {T(0), s.b1, s.b2, s.b3};
  w[0] = s.de * ud;
#pragma unroll
  for (int m = 1; m <= 3; ++m) w[m] = a * ud * s.ucov[m] + b * (D == m ? T(1) : T(0)) - s.bbcon[D] * s.bbcov[m];
  w[4] = a * ud * s.ucov[0] + b * T(0) - s.bbcon[D] * s.bbcov[0] + s.de * ud;
  w[5] = s.de * sr * ud;
#pragma unroll
  for (int m = 1; m <= 3; ++m) {
    if (m == D) w[5 + m] = T(0);
    else w[5 + m] = (ud * mrcp(s.ucon[0])) * bc[m] - (s.ucon[m] * mrcp(s.ucon[0])) * bc[D];
  }
#pragma unroll
  for (int n = 0; n < 9; ++n) w[n] = detg * w[n];
}

// calcha.f90:370-908 (icha = 2, Del Zanna et al. 2007) in direction D, using
// the state already evaluated in PST.  cal3met (coord.f90:970-1013) gives the
// spatial metrics: gcov3a = gcov + 0*0, gcon3a(D,D) = gcon(D,D) + (beta^D/alpha)^2.
template <int D, typename T>
__device__ __forceinline__ void wavespeed(const T q[9], const PST<T>& s, const MetT<T>& m, T gam, T& vfp, T& vfm) {
  const T alpha1 = m.al;
  const T betad = (D == 1) ? m.be1 : (D == 2 ? m.be2 : T(0));
  const T gc3dd = (D == 1) ? m.g3_11 : (D == 2 ? m.g3_22 : m.g3_33);
  const T vcon[4] = {T(0), q[1] * mrcp(s.gfl), q[2] * mrcp(s.gfl), q[3] * mrcp(s.gfl)};
  const T vsq = qform3(m, vcon[1], vcon[2], vcon[3]);
  const T cssq = mdiv(gam * s.pr, s.roh);
  const T vasq = s.bbsq * mrcp(s.roh + s.bbsq);
  const T omsq = vasq + cssq * (T(1) - vasq);
  const T f1 = vcon[D] * (T(1) - omsq);
  const T f2 = T(1) - vsq * omsq;
  const T f3 = omsq * (T(1) - vsq) * ((T(1) - vsq * omsq) * gc3dd - (T(1) - omsq) * vcon[D] * vcon[D]);
  vfp = (f1 + msqrt(f3)) * mrcp(f2);
  vfm = (f1 - msqrt(f3)) * mrcp(f2);
  vfp = alpha1 * vfp - betad;
  vfm = alpha1 * vfm - betad;
  if (mabs(vfp) > T(1)) vfp = T(1);
  if (mabs(vfm) > T(1)) vfm = T(-1);
}

}  // namespace rg

#include "rg_recon.cuh"
