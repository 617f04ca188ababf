// rg_device.cuh -- pointwise GRMHD physics of the RAISHIN update as device
// functions (FP64).  Each function states the reference routine it follows;
// the evaluation order of every expression matches the reference Fortran
// (left-to-right, parenthesised as written) so that a --fmad=false build
// reproduces the reference arithmetic up to the last bit of the math library.
#pragma once
#include <cstdint>

#include "rg_types.h"

namespace rg {

// Metric at one point: covariant and contravariant 4-metric and sqrt(-g).
struct Met {
  double g[4][4];
  double gc[4][4];
  double detg;
};

// Metric cache layout (per (i,k) point, 33 components, structure of arrays):
// component c in [0,16) gcov(c/4, c%4), [16,32) gcon, 32 detg.
__device__ __forceinline__ void load_met(const double* __restrict__ base, size_t nik, size_t q, Met& m) {
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      m.g[a][b] = __ldg(base + (size_t)(4 * a + b) * nik + q);
      m.gc[a][b] = __ldg(base + (size_t)(16 + 4 * a + b) * nik + q);
    }
  m.detg = __ldg(base + (size_t)32 * nik + q);
}

__device__ __forceinline__ double sgn1(double x) { return copysign(1.0, x); }
__device__ __forceinline__ double fmax3(double a, double b, double c) {
  double r = a;
  if (b > r) r = b;
  if (c > r) r = c;
  return r;
}
__device__ __forceinline__ double fmin3(double a, double b, double c) {
  double r = a;
  if (b < r) r = b;
  if (c < r) r = c;
  return r;
}
__device__ __forceinline__ double dmin2(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double dmax2(double a, double b) { return (b > a) ? b : a; }

// physfunc.f90:2-42
__device__ __forceinline__ double calgfl(const double u1, const double u2, const double u3, const Met& m) {
  const double ut[4] = {0.0, u1, u2, u3};
  double utsq = 0.0;
#pragma unroll
  for (int a = 1; a <= 3; ++a)
#pragma unroll
    for (int b = 1; b <= 3; ++b) utsq = utsq + m.g[a][b] * ut[a] * ut[b];
  if (utsq < 0.0) {
    if (fabs(utsq) <= 1.0e-10) utsq = fabs(utsq);
    else utsq = 1.e-10;
  }
  if (fabs(utsq) > 5.e2) utsq = 5.0e2;
  return sqrt(1. + utsq);
}

// physfunc.f90:45-78
__device__ __forceinline__ void calucon(double u1, double u2, double u3, double gfl, const Met& m, double ucon[4]) {
  const double alpha1 = 1. / sqrt(-m.gc[0][0]);
  const double b1 = alpha1 * alpha1 * m.gc[0][1];
  const double b2 = alpha1 * alpha1 * m.gc[0][2];
  const double b3 = alpha1 * alpha1 * m.gc[0][3];
  ucon[0] = gfl * (1. / alpha1);
  ucon[1] = u1 - gfl * b1 * (1. / alpha1);
  ucon[2] = u2 - gfl * b2 * (1. / alpha1);
  ucon[3] = u3 - gfl * b3 * (1. / alpha1);
}

// physfunc.f90:161-195 / 198-232
__device__ __forceinline__ void lower4(const double v[4], double o[4], const double g[4][4]) {
#pragma unroll
  for (int a = 0; a < 4; ++a) o[a] = g[a][0] * v[0] + g[a][1] * v[1] + g[a][2] * v[2] + g[a][3] * v[3];
}

// Velocity and magnetic 4-vectors of one primitive state (the common head of
// caluu1/caluu3/calflx3*/caltenr, caluu.f90:40-90).
struct PS {
  double ucon[4], ucov[4], bbcon[4], bbcov[4];
  double bbsq, roh, gfl, de, pr, b1, b2, b3;
};

__device__ __forceinline__ void pstate(const double q[9], const Met& m, double gam, PS& s) {
  s.de = q[0];
  s.pr = q[4];
  s.b1 = q[6]; s.b2 = q[7]; s.b3 = q[8];
  s.roh = s.de + (gam / (gam - 1.0)) * s.pr;
  s.gfl = calgfl(q[1], q[2], q[3], m);
  calucon(q[1], q[2], q[3], s.gfl, m, s.ucon);
  lower4(s.ucon, s.ucov, m.g);
  // physfunc.f90:81-100
  s.bbcon[0] = s.b1 * s.ucov[1] + s.b2 * s.ucov[2] + s.b3 * s.ucov[3];
  s.bbcon[1] = (s.b1 + s.bbcon[0] * s.ucon[1]) * (1. / s.ucon[0]);
  s.bbcon[2] = (s.b2 + s.bbcon[0] * s.ucon[2]) * (1. / s.ucon[0]);
  s.bbcon[3] = (s.b3 + s.bbcon[0] * s.ucon[3]) * (1. / s.ucon[0]);
  lower4(s.bbcon, s.bbcov, m.g);
  s.bbsq = s.bbcon[0] * s.bbcov[0] + s.bbcon[1] * s.bbcov[1] + s.bbcon[2] * s.bbcov[2] + s.bbcon[3] * s.bbcov[3];
}

// caluu.f90:92-118: sqrt(-g) (rho u^t, T^t_i, T^t_t + rho u^t, s u^t, B^i).
// delta(0,n) is the literal identity of caldelta (physfunc.f90:122-158).
__device__ __forceinline__ void p2c(const PS& s, double gam, double detg, double u[9]) {
  const double a = s.roh + s.bbsq, b = s.pr + 0.5 * s.bbsq;
  u[0] = s.de * s.ucon[0];
#pragma unroll
  for (int m = 1; m <= 3; ++m) u[m] = a * s.ucon[0] * s.ucov[m] + b * 0.0 - s.bbcon[0] * s.bbcov[m];
  u[4] = a * s.ucon[0] * s.ucov[0] + b * 1.0 - s.bbcon[0] * s.bbcov[0] + s.de * s.ucon[0];
  u[5] = s.de * (s.pr / pow(s.de, gam)) * s.ucon[0];
  u[6] = s.b1; u[7] = s.b2; u[8] = s.b3;
#pragma unroll
  for (int n = 0; n < 9; ++n) u[n] = detg * u[n];
}

// calflx.f90:391-795, direction D (1 = r, 2 = phi, 3 = theta).  The induction
// flux is (u^D/u^0) B^m - (u^m/u^0) B^D with the D component set to 0.
template <int D>
__device__ __forceinline__ void flux(const PS& s, double gam, double detg, double w[9]) {
  const double a = s.roh + s.bbsq, b = s.pr + 0.5 * s.bbsq;
  const double ud = s.ucon[D];
  const double bc[4] = {0.0, s.b1, s.b2, s.b3};
  w[0] = s.de * ud;
#pragma unroll
  for (int m = 1; m <= 3; ++m) w[m] = a * ud * s.ucov[m] + b * (D == m ? 1.0 : 0.0) - s.bbcon[D] * s.bbcov[m];
  w[4] = a * ud * s.ucov[0] + b * 0.0 - s.bbcon[D] * s.bbcov[0] + s.de * ud;
  w[5] = s.de * (s.pr / pow(s.de, gam)) * ud;
#pragma unroll
  for (int m = 1; m <= 3; ++m) {
    if (m == D) w[5 + m] = 0.0;
    else w[5 + m] = (ud * (1. / s.ucon[0])) * bc[m] - (s.ucon[m] * (1. / s.ucon[0])) * bc[D];
  }
#pragma unroll
  for (int n = 0; n < 9; ++n) w[n] = detg * w[n];
}

// calcha.f90:370-908 (icha = 2, Del Zanna et al. 2007) in direction D, using
// the state already evaluated in PS.  cal3met (coord.f90:970-1013) gives the
// spatial metrics: gcov3a = gcov + 0*0, gcon3a(D,D) = gcon(D,D) + (beta^D/alpha)^2.
template <int D>
__device__ __forceinline__ void wavespeed(const double q[9], const PS& s, const Met& m, double gam, double& vfp,
                                          double& vfm) {
  const double alpha1 = 1. / sqrt(-m.gc[0][0]);
  const double beta[4] = {0.0, alpha1 * alpha1 * m.gc[0][1], alpha1 * alpha1 * m.gc[0][2],
                          alpha1 * alpha1 * m.gc[0][3]};
  const double oncon_d = beta[D] / alpha1;
  const double gc3dd = m.gc[D][D] + (oncon_d * oncon_d);
  const double vcon[4] = {0.0, q[1] * (1. / s.gfl), q[2] * (1. / s.gfl), q[3] * (1. / s.gfl)};
  double vsq = 0.0;
#pragma unroll
  for (int a = 1; a <= 3; ++a)
#pragma unroll
    for (int b = 1; b <= 3; ++b) vsq = vsq + (m.g[a][b] + (0.0 * 0.0)) * vcon[a] * vcon[b];
  const double cssq = gam * s.pr / s.roh;
  const double vasq = s.bbsq * (1. / (s.roh + s.bbsq));
  const double omsq = vasq + cssq * (1.0 - vasq);
  const double f1 = vcon[D] * (1.0 - omsq);
  const double f2 = 1.0 - vsq * omsq;
  const double f3 = omsq * (1.0 - vsq) * ((1.0 - vsq * omsq) * gc3dd - (1.0 - omsq) * vcon[D] * vcon[D]);
  vfp = (f1 + sqrt(f3)) * (1. / f2);
  vfm = (f1 - sqrt(f3)) * (1. / f2);
  vfp = alpha1 * vfp - beta[D];
  vfm = alpha1 * vfm - beta[D];
  if (fabs(vfp) > 1.0) vfp = 1.0;
  if (fabs(vfm) > 1.0) vfm = -1.0;
}

// rec.f90:2346-2370
__device__ __forceinline__ double dmm(double xx, double yy) {
  return 0.5 * (sgn1(xx) + sgn1(yy)) * dmin2(fabs(xx), fabs(yy));
}
__device__ __forceinline__ double dm4(double ww, double xx, double yy, double zz) {
  double mn = fabs(ww);
  if (fabs(xx) < mn) mn = fabs(xx);
  if (fabs(yy) < mn) mn = fabs(yy);
  if (fabs(zz) < mn) mn = fabs(zz);
  return 0.125 * (sgn1(ww) + sgn1(xx)) * fabs(sgn1(ww) + sgn1(yy)) * (sgn1(ww) + sgn1(zz)) * mn;
}

// rec.f90:2095-2130: MP5 state at the +1/2 face of cell 0 from u(-2..+2).
__device__ __forceinline__ double mp5_left(double um2, double um1, double u0, double up1, double up2) {
  const double tmp1 = 1.0 / 60.0, tmp2 = 4.0 / 3.0, alpha = 4.0, eps1 = 1.0e-10;
  const double ul1 = tmp1 * (2. * um2 - 13. * um1 + 47. * u0 + 27. * up1 - 3. * up2);
  const double ulmp = u0 + dmm(up1 - u0, alpha * (u0 - um1));
  const double t = (ul1 - u0) * (ul1 - ulmp);
  if (t <= eps1) return ul1;
  const double dim1 = um2 - 2. * um1 + u0;
  const double di1 = um1 - 2. * u0 + up1;
  const double dip1 = u0 - 2. * up1 + up2;
  const double dm4iph = dm4(4. * di1 - dip1, 4. * dip1 - di1, di1, dip1);
  const double dm4imh = dm4(4. * di1 - dim1, 4. * dim1 - di1, di1, dim1);
  const double ul = u0 + alpha * (u0 - um1);
  const double av = 0.5 * (u0 + up1);
  const double md = av - 0.5 * dm4iph;
  const double lc = u0 + 0.5 * (u0 - um1) + tmp2 * dm4imh;
  const double m1 = fmin3(u0, up1, md), m2 = fmin3(u0, ul, lc);
  const double m3 = fmax3(u0, up1, md), m4 = fmax3(u0, ul, lc);
  const double umax = dmax2(m1, m2), umin = dmin2(m3, m4);
  return ul1 + dmm(umin - ul1, umax - ul1);
}

// rec.f90:2134-2178: MP5 state at the -1/2 face of cell 0 from u(-2..+2),
// with the reference's sign convention for md/lc (rec.f90:2172-2176).
__device__ __forceinline__ double mp5_right(double um2, double um1, double u0, double up1, double up2) {
  const double tmp1 = 1.0 / 60.0, tmp2 = 4.0 / 3.0, alpha = 4.0, eps1 = 1.0e-10;
  const double ur1 = tmp1 * (2. * up2 - 13. * up1 + 47. * u0 + 27. * um1 - 3. * um2);
  const double urmp = u0 + dmm(um1 - u0, alpha * (u0 - up1));
  const double t = (ur1 - u0) * (ur1 - urmp);
  if (t <= eps1) return ur1;
  const double dim1 = um2 - 2. * um1 + u0;
  const double di1 = um1 - 2. * u0 + up1;
  const double dip1 = u0 - 2. * up1 + up2;
  const double dm4iph = dm4(4. * di1 - dip1, 4. * dip1 - di1, di1, dip1);
  const double dm4imh = dm4(4. * di1 - dim1, 4. * dim1 - di1, di1, dim1);
  const double ul = u0 + alpha * (u0 - up1);
  const double av = 0.5 * (u0 + um1);
  const double md = av + 0.5 * dm4imh;
  const double lc = u0 + 0.5 * (u0 - up1) - tmp2 * dm4iph;
  const double m1 = fmin3(u0, um1, md), m2 = fmin3(u0, ul, lc);
  const double m3 = fmax3(u0, um1, md), m4 = fmax3(u0, ul, lc);
  const double umax = dmax2(m1, m2), umin = dmin2(m3, m4);
  return ur1 + dmm(umin - ur1, umax - ur1);
}

// rec.f90:2373-2643 (WENO5-JS); left state at +1/2 and right state at -1/2
// of cell 0.  (13./12.) is a single-precision literal in the reference.
__device__ __forceinline__ double weno5_state(double a2, double a1, double u0, double b1, double b2) {
  // a2 = u(-2), a1 = u(-1), b1 = u(+1), b2 = u(+2) mirrored by the caller for the right state
  const double cd0 = 1.0 / 10.0, cd1 = 6.0 / 10.0, cd2 = 3.0 / 10.0;
  const double c00 = 2.0 / 6.0, c01 = -7.0 / 6.0, c02 = 11.0 / 6.0;
  const double c10 = -1.0 / 6.0, c11 = 5.0 / 6.0, c12 = 2.0 / 6.0;
  const double c20 = 2.0 / 6.0, c21 = 5.0 / 6.0, c22 = -1.0 / 6.0;
  const double epsi = 1.0e-6, c1312 = (double)(13.0f / 12.0f), c14 = 0.25;
  const double s0 = a2 - 2. * a1 + u0, t0 = a2 - 4. * a1 + 3. * u0;
  const double s1 = a1 - 2. * u0 + b1, t1 = a1 - b1;
  const double s2 = u0 - 2. * b1 + b2, t2 = 3. * u0 - 4. * b1 + b2;
  const double be0 = c1312 * (s0 * s0) + c14 * (t0 * t0) + epsi;
  const double be1 = c1312 * (s1 * s1) + c14 * (t1 * t1) + epsi;
  const double be2 = c1312 * (s2 * s2) + c14 * (t2 * t2) + epsi;
  const double w0 = cd0 / (be0 * be0), w1 = cd1 / (be1 * be1), w2 = cd2 / (be2 * be2);
  const double wt = w0 + w1 + w2;
  const double o0 = w0 / wt, o1 = w1 / wt, o2 = w2 / wt;
  const double q0 = c00 * a2 + c01 * a1 + c02 * u0;
  const double q1 = c10 * a1 + c11 * u0 + c12 * b1;
  const double q2 = c20 * u0 + c21 * b1 + c22 * b2;
  return o0 * q0 + o1 * q1 + o2 * q2;
}

}  // namespace rg
