// rg_device.cuh -- pointwise GRMHD physics of the RAISHIN update as device
// functions (FP64).  Each function states the reference routine it follows;
// the evaluation order of every expression matches the reference Fortran
// (left-to-right, parenthesised as written) so that a --fmad=false build
// reproduces the reference arithmetic up to the last bit of the math library.
#pragma once
#include <cstdint>

#include "rg_types.h"

namespace rg {

// Metric at one point.  Every metric of this build (Minkowski 1, Kerr-Schild
// 303, modified Kerr-Schild 403, coord.f90:149-792) couples only (t, r, phi)
// and keeps theta diagonal, so g^{mu 3} and g_{mu 3} vanish for mu != 3 (the
// host checks this at admission).  gcov is symmetric; gcon, an LU inverse
// (coord.f90:1504), is not symmetric to the last bit and keeps its full 3x3
// block.  Sums below run over the nonzero terms in the reference's order.
struct Met {
  double g00, g01, g02, g11, g12, g22, g33;                 // gcov
  double c00, c01, c02, c10, c11, c12, c20, c21, c22, c33;  // gcon
  double detg;                                              // sqrt(-g)
};
constexpr int kMetComps = 18;

// Metric cache layout: per (i,k) point q, component c at c*nik + q, in the
// order of the Met fields.
__device__ __forceinline__ void load_met(const double* __restrict__ base, size_t nik, size_t q, Met& m) {
  const double* b = base + q;
  m.g00 = __ldg(b + 0 * nik); m.g01 = __ldg(b + 1 * nik); m.g02 = __ldg(b + 2 * nik);
  m.g11 = __ldg(b + 3 * nik); m.g12 = __ldg(b + 4 * nik); m.g22 = __ldg(b + 5 * nik);
  m.g33 = __ldg(b + 6 * nik);
  m.c00 = __ldg(b + 7 * nik); m.c01 = __ldg(b + 8 * nik); m.c02 = __ldg(b + 9 * nik);
  m.c10 = __ldg(b + 10 * nik); m.c11 = __ldg(b + 11 * nik); m.c12 = __ldg(b + 12 * nik);
  m.c20 = __ldg(b + 13 * nik); m.c21 = __ldg(b + 14 * nik); m.c22 = __ldg(b + 15 * nik);
  m.c33 = __ldg(b + 16 * nik);
  m.detg = __ldg(b + 17 * nik);
}

// sum_{a,b=1..3} g_ab x_a x_b over the nonzero terms in (a,b) order
// (physfunc.f90:16-20, calcha.f90:251-256, correction.f90:806-811).
__device__ __forceinline__ double qform3(const Met& m, double x1, double x2, double x3) {
  double s = 0.0;
  s = s + m.g11 * x1 * x1;
  s = s + m.g12 * x1 * x2;
  s = s + m.g12 * x2 * x1;  // g_21 = g_12
  s = s + m.g22 * x2 * x2;
  s = s + m.g33 * x3 * x3;
  return s;
}

// g_ab v^b (physfunc.f90:161-195)
__device__ __forceinline__ void lower_g(const double v[4], double o[4], const Met& m) {
  o[0] = m.g00 * v[0] + m.g01 * v[1] + m.g02 * v[2];
  o[1] = m.g01 * v[0] + m.g11 * v[1] + m.g12 * v[2];
  o[2] = m.g02 * v[0] + m.g12 * v[1] + m.g22 * v[2];
  o[3] = m.g33 * v[3];
}

// g^ab v_b (physfunc.f90:198-232)
__device__ __forceinline__ void upper_gc(const double v[4], double o[4], const Met& m) {
  o[0] = m.c00 * v[0] + m.c01 * v[1] + m.c02 * v[2];
  o[1] = m.c10 * v[0] + m.c11 * v[1] + m.c12 * v[2];
  o[2] = m.c20 * v[0] + m.c21 * v[1] + m.c22 * v[2];
  o[3] = m.c33 * v[3];
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
  double utsq = qform3(m, u1, u2, u3);
  if (utsq < 0.0) {
    if (fabs(utsq) <= 1.0e-10) utsq = fabs(utsq);
    else utsq = 1.e-10;
  }
  if (fabs(utsq) > 5.e2) utsq = 5.0e2;
  return sqrt(1. + utsq);
}

// physfunc.f90:45-78
__device__ __forceinline__ void calucon(double u1, double u2, double u3, double gfl, const Met& m, double ucon[4]) {
  const double alpha1 = 1. / sqrt(-m.c00);
  const double b1 = alpha1 * alpha1 * m.c01;
  const double b2 = alpha1 * alpha1 * m.c02;
  ucon[0] = gfl * (1. / alpha1);
  ucon[1] = u1 - gfl * b1 * (1. / alpha1);
  ucon[2] = u2 - gfl * b2 * (1. / alpha1);
  ucon[3] = u3;  // beta^theta = 0
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
  lower_g(s.ucon, s.ucov, m);
  // physfunc.f90:81-100
  s.bbcon[0] = s.b1 * s.ucov[1] + s.b2 * s.ucov[2] + s.b3 * s.ucov[3];
  s.bbcon[1] = (s.b1 + s.bbcon[0] * s.ucon[1]) * (1. / s.ucon[0]);
  s.bbcon[2] = (s.b2 + s.bbcon[0] * s.ucon[2]) * (1. / s.ucon[0]);
  s.bbcon[3] = (s.b3 + s.bbcon[0] * s.ucon[3]) * (1. / s.ucon[0]);
  lower_g(s.bbcon, s.bbcov, m);
  s.bbsq = s.bbcon[0] * s.bbcov[0] + s.bbcon[1] * s.bbcov[1] + s.bbcon[2] * s.bbcov[2] + s.bbcon[3] * s.bbcov[3];
}

// p / rho^Gamma of a state (caluu.f90:303, calflx.f90:474), computed once per state.
__device__ __forceinline__ double ent_ratio(const PS& s, double gam) { return s.pr / pow(s.de, gam); }

__device__ __forceinline__ void p2c(const PS& s, double gam, double detg, double u[9]) {
  const double a = s.roh + s.bbsq, b = s.pr + 0.5 * s.bbsq;
  u[0] = s.de * s.ucon[0];
#pragma unroll
  for (int m = 1; m <= 3; ++m) u[m] = a * s.ucon[0] * s.ucov[m] + b * 0.0 - s.bbcon[0] * s.bbcov[m];
  u[4] = a * s.ucon[0] * s.ucov[0] + b * 1.0 - s.bbcon[0] * s.bbcov[0] + s.de * s.ucon[0];
  u[5] = s.de * ent_ratio(s, gam) * s.ucon[0];
  u[6] = s.b1; u[7] = s.b2; u[8] = s.b3;
#pragma unroll
  for (int n = 0; n < 9; ++n) u[n] = detg * u[n];
}

// caluu.f90:92-118: sqrt(-g) (rho u^t, T^t_i, T^t_t + rho u^t, s u^t, B^i).
// delta(0,n) is the literal identity of caldelta (physfunc.f90:122-158).
__device__ __forceinline__ void p2c(const PS& s, double gam, double detg, double u[9], double sr) {
  const double a = s.roh + s.bbsq, b = s.pr + 0.5 * s.bbsq;
  u[0] = s.de * s.ucon[0];
#pragma unroll
  for (int m = 1; m <= 3; ++m) u[m] = a * s.ucon[0] * s.ucov[m] + b * 0.0 - s.bbcon[0] * s.bbcov[m];
  u[4] = a * s.ucon[0] * s.ucov[0] + b * 1.0 - s.bbcon[0] * s.bbcov[0] + s.de * s.ucon[0];
  u[5] = s.de * sr * s.ucon[0];
  u[6] = s.b1; u[7] = s.b2; u[8] = s.b3;
#pragma unroll
  for (int n = 0; n < 9; ++n) u[n] = detg * u[n];
}

// calflx.f90:391-795, direction D (1 = r, 2 = phi, 3 = theta).  The induction
// flux is (u^D/u^0) B^m - (u^m/u^0) B^D with the D component set to 0.
template <int D>
__device__ __forceinline__ void flux(const PS& s, double gam, double detg, double w[9], double sr) {
  const double a = s.roh + s.bbsq, b = s.pr + 0.5 * s.bbsq;
  const double ud = s.ucon[D];
  const double bc[4] = {0.0, s.b1, s.b2, s.b3};
  w[0] = s.de * ud;
#pragma unroll
  for (int m = 1; m <= 3; ++m) w[m] = a * ud * s.ucov[m] + b * (D == m ? 1.0 : 0.0) - s.bbcon[D] * s.bbcov[m];
  w[4] = a * ud * s.ucov[0] + b * 0.0 - s.bbcon[D] * s.bbcov[0] + s.de * ud;
  w[5] = s.de * sr * ud;
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
  const double alpha1 = 1. / sqrt(-m.c00);
  const double betad = (D == 1) ? alpha1 * alpha1 * m.c01 : (D == 2 ? alpha1 * alpha1 * m.c02 : 0.0);
  const double oncon_d = betad / alpha1;
  const double gcdd = (D == 1) ? m.c11 : (D == 2 ? m.c22 : m.c33);
  const double gc3dd = gcdd + (oncon_d * oncon_d);
  const double vcon[4] = {0.0, q[1] * (1. / s.gfl), q[2] * (1. / s.gfl), q[3] * (1. / s.gfl)};
  const double vsq = qform3(m, vcon[1], vcon[2], vcon[3]);
  const double cssq = gam * s.pr / s.roh;
  const double vasq = s.bbsq * (1. / (s.roh + s.bbsq));
  const double omsq = vasq + cssq * (1.0 - vasq);
  const double f1 = vcon[D] * (1.0 - omsq);
  const double f2 = 1.0 - vsq * omsq;
  const double f3 = omsq * (1.0 - vsq) * ((1.0 - vsq * omsq) * gc3dd - (1.0 - omsq) * vcon[D] * vcon[D]);
  vfp = (f1 + sqrt(f3)) * (1. / f2);
  vfm = (f1 - sqrt(f3)) * (1. / f2);
  vfp = alpha1 * vfp - betad;
  vfm = alpha1 * vfm - betad;
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

// rec.f90:2095-2178: MP5 face state of cell 0 from u(-2..+2) given in the
// order (a2, a1, u0, b1, b2): the left state at +1/2 takes
// (u-2, u-1, u0, u+1, u+2) and sg = +1; the right state at -1/2 takes the
// mirrored stencil (u+2, u+1, u0, u-1, u-2) and sg = -1, because the
// reference's right state flips the signs of the dm4 terms of md and lc
// (rec.f90:2172-2176).  Negation is exact, so both equal the reference's
// separate formulas bit for bit, and the two lanes of a face run one code path.
__device__ __forceinline__ double mp5_state(double a2, double a1, double u0, double b1, double b2, double sg) {
  const double tmp1 = 1.0 / 60.0, tmp2 = 4.0 / 3.0, alpha = 4.0, eps1 = 1.0e-10;
  const double ul1 = tmp1 * (2. * a2 - 13. * a1 + 47. * u0 + 27. * b1 - 3. * b2);
  const double ulmp = u0 + dmm(b1 - u0, alpha * (u0 - a1));
  const double t = (ul1 - u0) * (ul1 - ulmp);
  if (t <= eps1) return ul1;
  const double dim1 = a2 - 2. * a1 + u0;
  const double di1 = a1 - 2. * u0 + b1;
  const double dip1 = u0 - 2. * b1 + b2;
  const double dm4p = dm4(4. * di1 - dip1, 4. * dip1 - di1, di1, dip1);
  const double dm4m = dm4(4. * di1 - dim1, 4. * dim1 - di1, di1, dim1);
  const double ul = u0 + alpha * (u0 - a1);
  const double av = 0.5 * (u0 + b1);
  const double md = av - (sg * 0.5) * dm4p;
  const double lc = u0 + 0.5 * (u0 - a1) + (sg * tmp2) * dm4m;
  const double m1 = fmin3(u0, b1, md), m2 = fmin3(u0, ul, lc);
  const double m3 = fmax3(u0, b1, md), m4 = fmax3(u0, ul, lc);
  const double umax = dmax2(m1, m2), umin = dmin2(m3, m4);
  return ul1 + dmm(umin - ul1, umax - ul1);
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


// ------------------------------------------------------------------- PPM
// rPPM of Marti & Muller (1996) as restated by rec.f90:1261-2058.  The four
// passes (interp, detect, flaten, monoto) touch only the two face states of
// one cell each, so both states of cell c follow from the cells c-3..c+3:
// L = state at c-1/2 (the reference's uriir(c-1)), R = state at c+1/2
// (uriil(c)).  dx is rec2's shifted dx?b (dummy dx?b(m) = actual dx?b(m-1),
// rec.f90:58), x the cell centres (contact detection).

// interp Eq. (60)-(61) (rec.f90:1346-1418); the theta direction lacks the
// factor 2 of r and phi (rec.f90:1414).
__device__ __forceinline__ double ppm_dma(double um, double u0, double up, double dxm, double dx0, double dxp,
                                          bool kdir) {
  const double t1a = dx0 / (dxm + dx0 + dxp);
  const double t1b = (2.0 * dxm + dx0) / (dxp + dx0);
  const double t1c = (dx0 + 2.0 * dxp) / (dxm + dx0);
  const double sp1 = up - u0, sm1 = u0 - um;
  const double spm1 = sp1 * sm1;
  const double da = t1a * (t1b * sp1 + t1c * sm1);
  if (spm1 <= 0.0) return 0.0;
  const double t1 = (da < 0.0) ? -1.0 : 1.0;
  const double t1d = dmin2(fabs(sm1), fabs(sp1));
  return kdir ? t1 * dmin2(fabs(da), t1d) : t1 * dmin2(fabs(da), 2.0 * t1d);
}

// interp Eq. (51) (rec.f90:1422-1468): interface value at c+1/2.
__device__ __forceinline__ double ppm_face(double u0, double u1, double dma0, double dma1, double dxm, double dx0,
                                           double dx1, double dx2) {
  const double t2 = (dx0 / (dx0 + dx1)) * (u1 - u0);
  const double t3a = 1.0 / (dxm + dx0 + dx1 + dx2);
  const double t3b = (2.0 * dx1 * dx0) / (dx0 + dx1);
  const double t3c = ((dxm + dx0) / (2.0 * dx0 + dx1)) - ((dx2 + dx1) / (2.0 * dx1 + dx0));
  const double t3 = t3a * t3b * t3c * (u1 - u0);
  const double t4 = t3a * dx0 * ((dxm + dx0) / (2.0 * dx0 + dx1));
  const double t5 = t3a * dx1 * ((dx1 + dx2) / (dx0 + 2.0 * dx1));
  return u0 + t2 + t3 - t4 * dma1 + t5 * dma0;
}

// Both face states of the cell at p (primitive v at p[v*N]), stride st along
// the direction D; dx[o], x[o] are the shifted spacing and centre at offset o
// from the cell (o in -4..4).  gam enters the contact test (rec.f90:1623).
template <int D>
__device__ void ppm_cell(const double* __restrict__ p, size_t N, long long st, const double dx[9], const double x[9],
                         double gam, double L[9], double R[9]) {
  auto U = [&](int v, int o) { return p[(size_t)v * N + o * st]; };
  auto DX = [&](int o) { return dx[o + 4]; };
  // detect (rec.f90:1479-1686): contact steepening factor eta on density
  double eta;
  {
    const double eta1 = 5.0, eta2 = 0.05, eps1 = 0.1, ak0 = 1.0;
    auto dda = [&](int o) {
      const double t0a = 1.0 / (DX(o - 1) + DX(o) + DX(o + 1));
      const double t0b = (U(0, o + 1) - U(0, o)) / (DX(o + 1) + DX(o));
      const double t0c = (U(0, o) - U(0, o - 1)) / (DX(o) + DX(o - 1));
      return t0a * (t0b - t0c);
    };
    const double ddp = dda(1), ddm = dda(-1);
    const double rp = U(0, 1), rm = U(0, -1);
    const double t1 = ddp * ddm;
    const double t2 = fabs(rp - rm) - eps1 * dmin2(fabs(rp), fabs(rm));
    double etatil;
    if (t1 >= 0.0 && t2 <= 0.0) {
      etatil = 0.0;
    } else {
      const double t2a = -(ddp - ddm) / (x[5] - x[3]);
      const double a = x[4] - x[3], b = x[5] - x[4];
      const double t2b = (a * a * a + b * b * b) / (rp - rm);
      etatil = t2a * t2b;
    }
    eta = dmax2(0.0, dmin2(eta1 * (etatil - eta2), 1.0));
    const double pp = U(4, 1), pm = U(4, -1);
    const double t3 = fabs(rp - rm) / dmin2(rp, rm);
    const double t4 = fabs(pp - pm) / dmin2(pp, pm);
    if (gam * ak0 * t3 < t4) eta = 0.0;
  }
  // flaten (rec.f90:1689-1884): shock flattening f2a from p and u^D
  double f2a;
  {
    const double eps2 = 1.0, omg2 = 0.52, omg3 = 10.0;
    auto f1a = [&](int o) {
      const double pp1 = U(4, o + 1), pm1 = U(4, o - 1);
      const double t3a = fabs(pp1 - pm1);
      const double t1 = eps2 * dmin2(pp1, pm1) - t3a;
      const double t2 = U(D, o + 1) - U(D, o - 1);
      const double omg1 = (t1 < 0.0 && t2 < 0.0) ? 1.0 : 0.0;
      const double t3b = U(4, o + 2) - U(4, o - 2);
      double t4;
      if (t3b == 0.0) t4 = (t3a == 0.0) ? -omg2 : 1.0 - omg2;
      else t4 = (t3a / t3b) - omg2;
      return dmin2(1.0, omg1 * dmax2(0.0, t4 * omg3));
    };
    const double f1b = (U(4, 1) - U(4, -1) < 0.0) ? f1a(1) : f1a(-1);
    f2a = dmax2(f1a(0), f1b);
  }
#pragma unroll 1
  for (int v = 0; v < 9; ++v) {
    if (v == 5) { L[v] = 0.0; R[v] = 0.0; continue; }  // var 6 faces are never read downstream
    const double um2 = U(v, -2), um1 = U(v, -1), u0 = U(v, 0), up1 = U(v, 1), up2 = U(v, 2);
    const double dm = ppm_dma(um2, um1, u0, DX(-2), DX(-1), DX(0), D == 3);
    const double d0 = ppm_dma(um1, u0, up1, DX(-1), DX(0), DX(1), D == 3);
    const double dp = ppm_dma(u0, up1, up2, DX(0), DX(1), DX(2), D == 3);
    double l = ppm_face(um1, u0, dm, d0, DX(-2), DX(-1), DX(0), DX(1));
    double r = ppm_face(u0, up1, d0, dp, DX(-1), DX(0), DX(1), DX(2));
    if (v == 0) {
      r = r * (1.0 - eta) + (up1 - 0.5 * dp) * eta;
      l = l * (1.0 - eta) + (um1 + 0.5 * dm) * eta;
    }
    r = u0 * f2a + r * (1.0 - f2a);
    l = u0 * f2a + l * (1.0 - f2a);
    // monoto (rec.f90:1887-2056)
    if ((r - u0) * (l - u0) >= 0.0) { r = u0; l = u0; }
    const double t3 = 6.0 * (r - l) * (u0 - 0.5 * (r + l));
    const double t4 = (r - l) * (r - l);
    if (t3 > t4) l = 3.0 * u0 - 2.0 * r;
    if (-t3 > t4) r = 3.0 * u0 - 2.0 * l;
    L[v] = l;
    R[v] = r;
  }
}

}  // namespace rg
