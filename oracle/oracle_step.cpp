// oracle_step.cpp -- one RK3 step of the reference (main.f90:743-1147),
// restated routine by routine for the CPU oracle (test infrastructure only;
// see oracle.hpp).  Loops are parallelised over k with OpenMP where the
// reference loop body is independent per cell; the results do not depend on
// the thread count.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "oracle.hpp"

namespace orc {

namespace {

// Fortran MAX/MIN over several arguments (first argument seeds the result).
inline double fmax3(double a, double b, double c) {
  double r = a;
  if (b > r) r = b;
  if (c > r) r = c;
  return r;
}
inline double fmin3(double a, double b, double c) {
  double r = a;
  if (b < r) r = b;
  if (c < r) r = c;
  return r;
}
inline double sgn(double x) { return std::copysign(1.0, x); }  // sign(1.0d0, x)

// rec.f90:2346-2356
inline double dmm(double xx, double yy) {
  return 0.5 * (sgn(xx) + sgn(yy)) * std::min(std::fabs(xx), std::fabs(yy));
}
// rec.f90:2358-2370
inline double dm4(double ww, double xx, double yy, double zz) {
  double m = std::fabs(ww);
  if (std::fabs(xx) < m) m = std::fabs(xx);
  if (std::fabs(yy) < m) m = std::fabs(yy);
  if (std::fabs(zz) < m) m = std::fabs(zz);
  return 0.125 * (sgn(ww) + sgn(xx)) * std::fabs(sgn(ww) + sgn(yy)) * (sgn(ww) + sgn(zz)) * m;
}

// Common part of caluu1/caluu3/calflx3*/caltenr: the 4-velocity and
// 4-magnetic field of a primitive state (caluu.f90:40-90).
struct PS {
  double ucon[4], ucov[4], bbcon[4], bbcov[4], bbsq, roh, gfl, de, pr, bcon[4];
};
inline void pstate(const double* q, const M4& g, const M4& gc, double gam, PS& s) {
  const double util[4] = {0.0, q[1], q[2], q[3]};
  s.de = q[0];
  s.pr = q[4];
  s.bcon[0] = 0.0; s.bcon[1] = q[6]; s.bcon[2] = q[7]; s.bcon[3] = q[8];
  s.roh = s.de + (gam / (gam - 1.0)) * s.pr;
  calgfl(util, s.gfl, g);
  calucon(util, s.ucon, s.gfl, gc);
  lower(s.ucon, s.ucov, g);
  calbbcon(s.bcon, s.bbcon, s.ucov, s.ucon);
  lower(s.bbcon, s.bbcov, g);
  s.bbsq = calbbsq(s.bbcon, s.bbcov);
}

// caluu.f90:92-118 (delta(0,n) is the literal identity of caldelta)
inline void p2c(const PS& s, double gam, double detg, double* u) {
  const double a = s.roh + s.bbsq, b = s.pr + 0.5 * s.bbsq;
  u[0] = s.de * s.ucon[0];
  for (int m = 1; m <= 3; ++m) u[m] = a * s.ucon[0] * s.ucov[m] + b * 0.0 - s.bbcon[0] * s.bbcov[m];
  u[4] = a * s.ucon[0] * s.ucov[0] + b * 1.0 - s.bbcon[0] * s.bbcov[0] + s.de * s.ucon[0];
  u[5] = s.de * (s.pr / fpow(s.de, gam)) * s.ucon[0];
  u[6] = s.bcon[1]; u[7] = s.bcon[2]; u[8] = s.bcon[3];
  for (int n = 0; n < 9; ++n) u[n] = detg * u[n];
}

// calflx.f90:391-795 for direction d (1 = i, 2 = j, 3 = k)
inline void flux(const PS& s, int d, double gam, double detg, double* w) {
  const double a = s.roh + s.bbsq, b = s.pr + 0.5 * s.bbsq;
  const double ud = s.ucon[d];
  w[0] = s.de * ud;
  for (int m = 1; m <= 3; ++m) w[m] = a * ud * s.ucov[m] + b * (d == m ? 1.0 : 0.0) - s.bbcon[d] * s.bbcov[m];
  w[4] = a * ud * s.ucov[0] + b * 0.0 - s.bbcon[d] * s.bbcov[0] + s.de * ud;
  w[5] = s.de * (s.pr / fpow(s.de, gam)) * ud;
  for (int m = 1; m <= 3; ++m) {
    if (m == d) w[5 + m] = 0.0;
    else w[5 + m] = (ud * (1. / s.ucon[0])) * s.bcon[m] - (s.ucon[m] * (1. / s.ucon[0])) * s.bcon[d];
  }
  for (int n = 0; n < 9; ++n) w[n] = detg * w[n];
}

// calcha.f90:370-549 (icha = 2, Del Zanna et al. 2007) for direction d
inline void calcha4d(const double* q, const M4& g, const M4& gc, double gam, int d, double& vfp,
                     double& vfm) {
  PS s;
  pstate(q, g, gc, gam, s);
  const double alpha1 = 1. / std::sqrt(-gc.a[0][0]);
  const double betad = alpha1 * alpha1 * gc.a[0][d];
  double g3[4][4], gc3[4][4];
  cal3met(g, gc, g3, gc3);
  const double vcon[4] = {0.0, q[1] * (1. / s.gfl), q[2] * (1. / s.gfl), q[3] * (1. / s.gfl)};
  double vsq = 0.0;
  for (int m = 1; m <= 3; ++m)
    for (int n = 1; n <= 3; ++n) vsq = vsq + g3[m][n] * vcon[m] * vcon[n];
  const double cssq = gam * s.pr / s.roh;
  const double vasq = s.bbsq * (1. / (s.roh + s.bbsq));
  const double omsq = vasq + cssq * (1.0 - vasq);
  const double f1 = vcon[d] * (1.0 - omsq);
  const double f2 = 1.0 - vsq * omsq;
  const double f3 = omsq * (1.0 - vsq) * ((1.0 - vsq * omsq) * gc3[d][d] - (1.0 - omsq) * vcon[d] * vcon[d]);
  vfp = (f1 + std::sqrt(f3)) * (1. / f2);
  vfm = (f1 - std::sqrt(f3)) * (1. / f2);
  vfp = alpha1 * vfp - betad;
  vfm = alpha1 * vfm - betad;
  if (std::fabs(vfp) > 1.0) vfp = 1.0;
  if (std::fabs(vfm) > 1.0) vfm = -1.0;
}

}  // namespace

// caluu.f90:2-126 (all cells)
void caluu1(State& s, const std::vector<double>& uri, std::vector<double>& uu) {
  const double gam = s.p.gam;
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= s.kmax; ++k)
    for (int j = 1; j <= s.jmax; ++j)
      for (int i = 1; i <= s.imax; ++i) {
        const size_t q = s.ik(i, k);
        PS ps;
        pstate(&uri[s.a(1, i, j, k)], s.gcov[q], s.gcon[q], gam, ps);
        p2c(ps, gam, s.detg[q], &uu[s.a(1, i, j, k)]);
      }
}

// --------------------------------------------------------------- reconstruction
// rec.f90:2059-2343 (MP5).  The right-state update keeps the reference's sign
// convention (rec.f90:2172-2176): uriirmd = av + 0.5 dm4imh, uriirlc = ... - (4/3) dm4iph.
static void mp5(State& s) {
  const double tmp1 = 1.0 / 60.0, tmp2 = 4.0 / 3.0, alpha = 4.0, eps1 = 1.0e-10;
  const int is1 = 1, ie1 = s.imax, js1 = 1, je1 = s.jmax, ks1 = 1, ke1 = s.kmax;
  std::vector<double>* L[3] = {&s.uriil, &s.urijl, &s.urikl};
  std::vector<double>* R[3] = {&s.uriir, &s.urijr, &s.urikr};
#pragma omp parallel for schedule(static)
  for (int k = ks1 + 2; k <= ke1 - 2; ++k)
    for (int j = js1 + 2; j <= je1 - 2; ++j)
      for (int i = is1 + 2; i <= ie1 - 2; ++i)
        for (int n = 1; n <= NV; ++n)
          for (int d = 0; d < 3; ++d) {
            const int di = (d == 0), dj = (d == 1), dk = (d == 2);
            auto U = [&](int o) { return s.uri[s.a(n, i + o * di, j + o * dj, k + o * dk)]; };
            const double um2 = U(-2), um1 = U(-1), u0 = U(0), up1 = U(1), up2 = U(2);
            // left state at the +1/2 face
            {
              const double ul1 = tmp1 * (2. * um2 - 13. * um1 + 47. * u0 + 27. * up1 - 3. * up2);
              const double ulmp = u0 + dmm(up1 - u0, alpha * (u0 - um1));
              const double t = (ul1 - u0) * (ul1 - ulmp);
              double out;
              if (t <= eps1) {
                out = ul1;
              } else {
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
                const double umax = std::max(m1, m2), umin = std::min(m3, m4);
                out = ul1 + dmm(umin - ul1, umax - ul1);
              }
              (*L[d])[s.a(n, i, j, k)] = out;
            }
            // right state at the -1/2 face (stored at index - 1)
            {
              const double ur1 = tmp1 * (2. * up2 - 13. * up1 + 47. * u0 + 27. * um1 - 3. * um2);
              const double urmp = u0 + dmm(um1 - u0, alpha * (u0 - up1));
              const double t = (ur1 - u0) * (ur1 - urmp);
              double out;
              if (t <= eps1) {
                out = ur1;
              } else {
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
                const double umax = std::max(m1, m2), umin = std::min(m3, m4);
                out = ur1 + dmm(umin - ur1, umax - ur1);
              }
              (*R[d])[s.a(n, i - di, j - dj, k - dk)] = out;
            }
          }
}

// rec.f90:2373-2643 (WENO5-JS; (13./12.) is a single-precision literal)
static void weno5(State& s) {
  const double cd0 = 1.0 / 10.0, cd1 = 6.0 / 10.0, cd2 = 3.0 / 10.0;
  const double c00 = 2.0 / 6.0, c01 = -7.0 / 6.0, c02 = 11.0 / 6.0;
  const double c10 = -1.0 / 6.0, c11 = 5.0 / 6.0, c12 = 2.0 / 6.0;
  const double c20 = 2.0 / 6.0, c21 = 5.0 / 6.0, c22 = -1.0 / 6.0;
  const double epsi = 1.0e-6;
  const double c1312 = sp(13.0f / 12.0f), c14 = 0.25;
  std::vector<double>* L[3] = {&s.uriil, &s.urijl, &s.urikl};
  std::vector<double>* R[3] = {&s.uriir, &s.urijr, &s.urikr};
  auto sq = [](double x) { return x * x; };
#pragma omp parallel for schedule(static)
  for (int k = 3; k <= s.kmax - 2; ++k)
    for (int j = 3; j <= s.jmax - 2; ++j)
      for (int i = 3; i <= s.imax - 2; ++i)
        for (int n = 1; n <= NV; ++n)
          for (int d = 0; d < 3; ++d) {
            const int di = (d == 0), dj = (d == 1), dk = (d == 2);
            auto U = [&](int o) { return s.uri[s.a(n, i + o * di, j + o * dj, k + o * dk)]; };
            const double um2 = U(-2), um1 = U(-1), u0 = U(0), up1 = U(1), up2 = U(2);
            const double bl0 = c1312 * sq(um2 - 2. * um1 + u0) + c14 * sq(um2 - 4. * um1 + 3. * u0) + epsi;
            const double bl1 = c1312 * sq(um1 - 2. * u0 + up1) + c14 * sq(um1 - up1) + epsi;
            const double bl2 = c1312 * sq(u0 - 2. * up1 + up2) + c14 * sq(3. * u0 - 4. * up1 + up2) + epsi;
            const double br0 = c1312 * sq(up2 - 2. * up1 + u0) + c14 * sq(up2 - 4. * up1 + 3. * u0) + epsi;
            const double br1 = c1312 * sq(up1 - 2. * u0 + um1) + c14 * sq(up1 - um1) + epsi;
            const double br2 = c1312 * sq(u0 - 2. * um1 + um2) + c14 * sq(3. * u0 - 4. * um1 + um2) + epsi;
            const double wl0 = cd0 / sq(bl0), wl1 = cd1 / sq(bl1), wl2 = cd2 / sq(bl2);
            const double wlt = wl0 + wl1 + wl2;
            const double wr0 = cd0 / sq(br0), wr1 = cd1 / sq(br1), wr2 = cd2 / sq(br2);
            const double wrt = wr0 + wr1 + wr2;
            const double ol0 = wl0 / wlt, ol1 = wl1 / wlt, ol2 = wl2 / wlt;
            const double or0 = wr0 / wrt, or1 = wr1 / wrt, or2 = wr2 / wrt;
            const double ql0 = c00 * um2 + c01 * um1 + c02 * u0;
            const double ql1 = c10 * um1 + c11 * u0 + c12 * up1;
            const double ql2 = c20 * u0 + c21 * up1 + c22 * up2;
            const double qr0 = c00 * up2 + c01 * up1 + c02 * u0;
            const double qr1 = c10 * up1 + c11 * u0 + c12 * um1;
            const double qr2 = c20 * u0 + c21 * um1 + c22 * um2;
            (*L[d])[s.a(n, i, j, k)] = ol0 * ql0 + ol1 * ql1 + ol2 * ql2;
            (*R[d])[s.a(n, i - di, j - dj, k - dk)] = or0 * qr0 + or1 * qr1 + or2 * qr2;
          }
}

// The second-order limiters on i,j,k = 2..n-1: mclim (irec 1,
// rec.f90:208-367), minlim (2, 568-739), lim03a (11, 4037-4267), mvllim (12,
// 4269-4477) and koren (13, 4480-4697).  Slopes in the MKS coordinates x?b,
// x?ab for metric 403, else in x?, x?a; MAX/MIN take the first argument as
// the seed (Fortran's order).  koren's j sweep takes tmp2i, the sign of the
// same cell's i-direction slope, in its backward state (rec.f90:4628).
static void limiters(State& s, int irec) {
  const double small = 1.0e-12;
  const bool mks = (s.p.metric == 403);
  const std::vector<double>* X[3] = {mks ? &s.x1b : &s.x1, mks ? &s.x2b : &s.x2, mks ? &s.x3b : &s.x3};
  const std::vector<double>* XA[3] = {mks ? &s.x1ab : &s.x1a, mks ? &s.x2ab : &s.x2a, mks ? &s.x3ab : &s.x3a};
  std::vector<double>* L[3] = {&s.uriil, &s.urijl, &s.urikl};
  std::vector<double>* R[3] = {&s.uriir, &s.urijr, &s.urikr};
  auto mx = [](double a, double b) { return (b > a) ? b : a; };  // Fortran MAX(a, b)
  auto mn = [](double a, double b) { return (b < a) ? b : a; };  // Fortran MIN(a, b)
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= s.kmax - 1; ++k)
    for (int j = 2; j <= s.jmax - 1; ++j)
      for (int i = 2; i <= s.imax - 1; ++i)
        for (int n = 1; n <= NV; ++n) {
          double tmp2i = 1.0;
          for (int d = 0; d < 3; ++d) {
            const int di = (d == 0), dj = (d == 1), dk = (d == 2);
            const int m = (d == 0) ? i : (d == 1 ? j : k);
            const std::vector<double>& x = *X[d];
            const std::vector<double>& xa = *XA[d];
            const double xp = x[m + 1], xc = x[m], xm = x[m - 1], xap = xa[m], xam = xa[m - 1];
            const double um = s.uri[s.a(n, i - di, j - dj, k - dk)], u0 = s.uri[s.a(n, i, j, k)],
                         up = s.uri[s.a(n, i + di, j + dj, k + dk)];
            double left, right;
            if (irec == 12) {  // mvllim
              const double ta = xp - xc + small, tb = xc - xm + small;
              const double sp = (up - u0) / ta, sm = (u0 - um) / tb;
              const double spm = sp * sm;
              const double tc = xap - xc + small, td = xc - xam + small;
              const double cf = ta / tc, cb = tb / td;
              double dkm;
              if (spm <= 0.0) {
                dkm = 0.0;
              } else {
                const double t = sm * sm + (cf + cb - 2.0) * sm * sp + sp * sp;
                dkm = (sm * sp * (cf * sm + cb * sp)) / (t + small);
              }
              left = u0 + dkm * tc;
              right = u0 - dkm * td;
            } else if (irec == 11 || irec == 13) {  // lim03a, koren
              const double ta = xp - xc + small, tb = xc - xm + small;
              const double tc = xap - xc + small, td = xc - xam + small;
              const double sp = (up - u0) * (1.0 / ta), sm = (u0 - um) * (1.0 / tb);
              const double cf = ta * (1.0 / tc), cb = tb * (1.0 / td);
              const double tmp = (sp < 0.0) ? -1.0 : 1.0;
              if (d == 0) tmp2i = tmp;
              double dkf, dkb;
              if (irec == 11) {
                const double al = 0.5, be = 2.0, ga = 1.6;
                const double eb = (2.0 * std::fabs(sp) + tmp * sm) * (1.0 / 3.0);
                const double ef = (std::fabs(sp) + tmp * 2.0 * sm) * (1.0 / 3.0);
                dkb = mx(0.0, mn(eb, mx(-al * sm * tmp, fmin3(be * sm * tmp, eb, ga * std::fabs(sp)))));
                dkf = mx(0.0, mn(ef, mx(-al * std::fabs(sp), fmin3(be * std::fabs(sp), ef, ga * tmp * sm))));
              } else {
                const double tb_sign = (d == 1) ? tmp2i : tmp;
                dkf = tmp * mx(0.0, fmin3(std::fabs(cf * sp), tmp * cb * sm, (2.0 * std::fabs(sp) + tmp * sm) * (1.0 / 3.0)));
                dkb = tmp * mx(0.0, fmin3(std::fabs(cf * sp), tmp * cb * sm,
                                          (std::fabs(sp) + 2.0 * tb_sign * sm) * (1.0 / 3.0)));
              }
              left = u0 + dkf * (xap - xc);
              right = u0 - dkb * (xc - xam);
            } else {  // mclim, minlim
              const double sp = (up - u0) * (1. / (xp - xc + small));
              const double sm = (u0 - um) * (1. / (xc - xm + small));
              const double tmp = (sp < 0.0) ? -1.0 : 1.0;
              const double lim = (irec == 1) ? fmin3(2.0 * std::fabs(sp), tmp * 2.0 * sm, tmp * 0.5 * (sp + sm))
                                             : mn(std::fabs(sp), tmp * sm);
              const double dkm = tmp * mx(0.0, lim);
              left = u0 + dkm * (xap - xc);
              right = u0 - dkm * (xc - xam);
            }
            (*L[d])[s.a(n, i, j, k)] = left;
            (*R[d])[s.a(n, i - di, j - dj, k - dk)] = right;
          }
        }
}

// rec.f90:742-1258 (ceno, convex ENO) in its three passes: the minmod state
// on i,j,k = 2..n-1 from the physical cell centres x?, the three quadratic
// candidates and their weighted deviations (alp = 1, 0.7, 1) on 3..n-2, and
// the selection on 3..n-2.  In the theta sweep's negative branch the
// reference compares |dklp| with itself (rec.f90:1211), so the third
// candidate is never taken there.
static void ceno(State& s) {
  const double alp1 = 1.0, alp2 = 0.7, alp3 = 1.0;
  const std::vector<double>* X[3] = {&s.x1, &s.x2, &s.x3};
  std::vector<double>* L[3] = {&s.uriil, &s.urijl, &s.urikl};
  std::vector<double>* R[3] = {&s.uriir, &s.urijr, &s.urikr};
  const size_t nn = s.uri.size();
  std::vector<double> l1[3], r1[3];
  for (int d = 0; d < 3; ++d) { l1[d].assign(nn, 0.0); r1[d].assign(nn, 0.0); }
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= s.kmax - 1; ++k)
    for (int j = 2; j <= s.jmax - 1; ++j)
      for (int i = 2; i <= s.imax - 1; ++i)
        for (int n = 1; n <= NV; ++n)
          for (int d = 0; d < 3; ++d) {
            const int di = (d == 0), dj = (d == 1), dk = (d == 2);
            const int m = (d == 0) ? i : (d == 1 ? j : k);
            const std::vector<double>& x = *X[d];
            const double um = s.uri[s.a(n, i - di, j - dj, k - dk)], u0 = s.uri[s.a(n, i, j, k)],
                         up = s.uri[s.a(n, i + di, j + dj, k + dk)];
            const double sp = (up - u0) / (x[m + 1] - x[m]), sm = (u0 - um) / (x[m] - x[m - 1]);
            double dkm = 0.0;
            if (!(sp * sm <= 0.0)) {
              const double tmp = (sp < 0.0) ? -1.0 : 1.0;
              dkm = tmp * std::min(std::fabs(sp), std::fabs(sm));
            }
            l1[d][s.a(n, i, j, k)] = u0 + dkm * (0.5 * (x[m + 1] - x[m]));
            r1[d][s.a(n, i - di, j - dj, k - dk)] = u0 - dkm * (0.5 * (x[m] - x[m - 1]));
          }
  auto pick = [](double u1, double cm, double c0, double cp, double dm, double d0, double dp, bool quirk) {
    double out = u1;
    if (dp > 0.0 && d0 > 0.0 && dm > 0.0) {
      out = cm;
      if (std::fabs(d0) < std::fabs(dm) && std::fabs(d0) < std::fabs(dp)) out = c0;
      if (std::fabs(dp) < std::fabs(dm) && std::fabs(dp) < std::fabs(d0)) out = cp;
    }
    if (dm < 0.0 && d0 < 0.0 && dp < 0.0) {
      out = cm;
      if (std::fabs(d0) < std::fabs(dm) && std::fabs(d0) < std::fabs(dp)) out = c0;
      if (std::fabs(dp) < std::fabs(dm) && std::fabs(dp) < (quirk ? std::fabs(dp) : std::fabs(d0))) out = cp;
    }
    return out;
  };
#pragma omp parallel for schedule(static)
  for (int k = 3; k <= s.kmax - 2; ++k)
    for (int j = 3; j <= s.jmax - 2; ++j)
      for (int i = 3; i <= s.imax - 2; ++i)
        for (int n = 1; n <= NV; ++n)
          for (int d = 0; d < 3; ++d) {
            const int di = (d == 0), dj = (d == 1), dk = (d == 2);
            const int m = (d == 0) ? i : (d == 1 ? j : k);
            const std::vector<double>& x = *X[d];
            auto U = [&](int o) { return s.uri[s.a(n, i + o * di, j + o * dj, k + o * dk)]; };
            const double d2m = 0.5 * (U(0) - U(-2)), d20 = 0.5 * (U(1) - U(-1)), d2p = 0.5 * (U(2) - U(0));
            const double d3m = U(0) - 2.0 * U(-1) + U(-2), d30 = U(1) - 2.0 * U(0) + U(-1),
                         d3p = U(2) - 2.0 * U(1) + U(0);
            const double t2m = (0.5 * (x[m + 1] + x[m]) - x[m - 1]) / (x[m + 1] - x[m]);
            const double t20 = (0.5 * (x[m + 1] + x[m]) - x[m]) / (x[m + 1] - x[m]);
            const double t2p = (0.5 * (x[m + 1] + x[m]) - x[m + 1]) / (x[m + 1] - x[m]);
            const double t3m = (0.5 * (x[m] + x[m - 1]) - x[m - 1]) / (x[m] - x[m - 1]);
            const double t30 = (0.5 * (x[m] + x[m - 1]) - x[m]) / (x[m] - x[m - 1]);
            const double t3p = (0.5 * (x[m] + x[m - 1]) - x[m + 1]) / (x[m] - x[m - 1]);
            const size_t ol = s.a(n, i, j, k), orr = s.a(n, i - di, j - dj, k - dk);
            const double lm = U(0) + d2m * t2m + 0.5 * d3m * (t2m * t2m);
            const double l0 = U(0) + d20 * t20 + 0.5 * d30 * (t20 * t20);
            const double lp = U(0) + d2p * t2p + 0.5 * d3p * (t2p * t2p);
            const double rm = U(0) + d2m * t3m + 0.5 * d3m * (t3m * t3m);
            const double r0 = U(0) + d20 * t30 + 0.5 * d30 * (t30 * t30);
            const double rp = U(0) + d2p * t3p + 0.5 * d3p * (t3p * t3p);
            const double ul1 = l1[d][ol], ur1 = r1[d][orr];
            (*L[d])[ol] = pick(ul1, lm, l0, lp, alp1 * (lm - ul1), alp2 * (l0 - ul1), alp3 * (lp - ul1), d == 2);
            (*R[d])[orr] = pick(ur1, rm, r0, rp, alp1 * (rm - ur1), alp2 * (r0 - ur1), alp3 * (rp - ur1), false);
          }
}

// rec.f90:145-205 (muscl, beta = 1/3) on i,j,k = 2..n-2: uriil and uriir of
// the face i+1/2 from cells i and i+1.
static void muscl(State& s) {
  const double beta = 1.0 / 3.0;
  std::vector<double>* L[3] = {&s.uriil, &s.urijl, &s.urikl};
  std::vector<double>* R[3] = {&s.uriir, &s.urijr, &s.urikr};
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= s.kmax - 2; ++k)
    for (int j = 2; j <= s.jmax - 2; ++j)
      for (int i = 2; i <= s.imax - 2; ++i)
        for (int n = 1; n <= NV; ++n)
          for (int d = 0; d < 3; ++d) {
            const int di = (d == 0), dj = (d == 1), dk = (d == 2);
            auto U = [&](int o) { return s.uri[s.a(n, i + o * di, j + o * dj, k + o * dk)]; };
            (*L[d])[s.a(n, i, j, k)] = U(0) + 0.25 * ((1.0 + beta) * (U(1) - U(0)) + (1.0 - beta) * (U(0) - U(-1)));
            (*R[d])[s.a(n, i, j, k)] = U(1) - 0.25 * ((1.0 + beta) * (U(1) - U(0)) + (1.0 - beta) * (U(2) - U(1)));
          }
}

// rec.f90:3161-3436 (WENO-Z, Borges et al. 2008) on i,j,k = 3..n-2: WENO5's
// stencils and coefficients with the weights cd (1 + tau/(beta + eps)),
// tau = |beta0 - beta2|; (13./12.) is a single-precision literal, and
// (beta + eps)**p0 with p0 = 1.d0 is the plain sum.
static void weno5z(State& s) {
  const double cd0 = 1.0 / 10.0, cd1 = 6.0 / 10.0, cd2 = 3.0 / 10.0;
  const double c00 = 2.0 / 6.0, c01 = -7.0 / 6.0, c02 = 11.0 / 6.0;
  const double c10 = -1.0 / 6.0, c11 = 5.0 / 6.0, c12 = 2.0 / 6.0;
  const double c20 = 2.0 / 6.0, c21 = 5.0 / 6.0, c22 = -1.0 / 6.0;
  const double epsi = 1.0e-6;
  const double c1312 = sp(13.0f / 12.0f), c14 = 0.25;
  std::vector<double>* L[3] = {&s.uriil, &s.urijl, &s.urikl};
  std::vector<double>* R[3] = {&s.uriir, &s.urijr, &s.urikr};
  auto sq = [](double x) { return x * x; };
  auto state = [&](double b0, double b1, double b2, double q0, double q1, double q2) {
    const double tau = std::fabs(b0 - b2);
    const double w0 = cd0 * (1.0 + (tau / (b0 + epsi)));
    const double w1 = cd1 * (1.0 + (tau / (b1 + epsi)));
    const double w2 = cd2 * (1.0 + (tau / (b2 + epsi)));
    const double wt = w0 + w1 + w2;
    const double o0 = w0 / wt, o1 = w1 / wt, o2 = w2 / wt;
    return o0 * q0 + o1 * q1 + o2 * q2;
  };
#pragma omp parallel for schedule(static)
  for (int k = 3; k <= s.kmax - 2; ++k)
    for (int j = 3; j <= s.jmax - 2; ++j)
      for (int i = 3; i <= s.imax - 2; ++i)
        for (int n = 1; n <= NV; ++n)
          for (int d = 0; d < 3; ++d) {
            const int di = (d == 0), dj = (d == 1), dk = (d == 2);
            auto U = [&](int o) { return s.uri[s.a(n, i + o * di, j + o * dj, k + o * dk)]; };
            const double um2 = U(-2), um1 = U(-1), u0 = U(0), up1 = U(1), up2 = U(2);
            const double bl0 = c1312 * sq(um2 - 2. * um1 + u0) + c14 * sq(um2 - 4. * um1 + 3. * u0);
            const double bl1 = c1312 * sq(um1 - 2. * u0 + up1) + c14 * sq(um1 - up1);
            const double bl2 = c1312 * sq(u0 - 2. * up1 + up2) + c14 * sq(3. * u0 - 4. * up1 + up2);
            const double br0 = c1312 * sq(up2 - 2. * up1 + u0) + c14 * sq(up2 - 4. * up1 + 3. * u0);
            const double br1 = c1312 * sq(up1 - 2. * u0 + um1) + c14 * sq(up1 - um1);
            const double br2 = c1312 * sq(u0 - 2. * um1 + um2) + c14 * sq(3. * u0 - 4. * um1 + um2);
            (*L[d])[s.a(n, i, j, k)] = state(bl0, bl1, bl2, c00 * um2 + c01 * um1 + c02 * u0,
                                             c10 * um1 + c11 * u0 + c12 * up1, c20 * u0 + c21 * up1 + c22 * up2);
            (*R[d])[s.a(n, i - di, j - dj, k - dk)] =
                state(br0, br1, br2, c00 * up2 + c01 * up1 + c02 * u0, c10 * up1 + c11 * u0 + c12 * um1,
                      c20 * u0 + c21 * um1 + c22 * um2);
          }
}

// rec.f90:2645-3158 (mpweno5) on i,j,k = 3..n-2: the WENO5-JS face value
// (beta with +epsi, weights cd/beta**2) limited by MP5's bounds, with MP5's
// right-state sign convention.  The radial right state's beta_1 reads
// uri(n,i-11,j,k) where uri(n,i-1,j,k) is meant (rec.f90:2757); gfortran
// addresses it in the column-major array, which below i = 1 is the element
// (n, imax + i - 11, j - 1, k).
static void mpweno5(State& s) {
  const double cd0 = 1.0 / 10.0, cd1 = 6.0 / 10.0, cd2 = 3.0 / 10.0;
  const double c00 = 2.0 / 6.0, c01 = -7.0 / 6.0, c02 = 11.0 / 6.0;
  const double c10 = -1.0 / 6.0, c11 = 5.0 / 6.0, c12 = 2.0 / 6.0;
  const double c20 = 2.0 / 6.0, c21 = 5.0 / 6.0, c22 = -1.0 / 6.0;
  const double tmp2 = 4.0 / 3.0, alpha = 4.0, eps1 = 1.0e-10, epsi = 1.0e-6;
  const double c1312 = sp(13.0f / 12.0f), c14 = 0.25;
  std::vector<double>* L[3] = {&s.uriil, &s.urijl, &s.urikl};
  std::vector<double>* R[3] = {&s.uriir, &s.urijr, &s.urikr};
  auto sq = [](double x) { return x * x; };
#pragma omp parallel for schedule(static)
  for (int k = 3; k <= s.kmax - 2; ++k)
    for (int j = 3; j <= s.jmax - 2; ++j)
      for (int i = 3; i <= s.imax - 2; ++i)
        for (int n = 1; n <= NV; ++n)
          for (int d = 0; d < 3; ++d) {
            const int di = (d == 0), dj = (d == 1), dk = (d == 2);
            auto U = [&](int o) { return s.uri[s.a(n, i + o * di, j + o * dj, k + o * dk)]; };
            const double um2 = U(-2), um1 = U(-1), u0 = U(0), up1 = U(1), up2 = U(2);
            double typo = um1;
            if (d == 0) typo = (i - 11 >= 1) ? s.uri[s.a(n, i - 11, j, k)] : s.uri[s.a(n, s.imax + i - 11, j - 1, k)];
            const double bl0 = c1312 * sq(um2 - 2. * um1 + u0) + c14 * sq(um2 - 4. * um1 + 3. * u0) + epsi;
            const double bl1 = c1312 * sq(um1 - 2. * u0 + up1) + c14 * sq(um1 - up1) + epsi;
            const double bl2 = c1312 * sq(u0 - 2. * up1 + up2) + c14 * sq(3. * u0 - 4. * up1 + up2) + epsi;
            const double br0 = c1312 * sq(up2 - 2. * up1 + u0) + c14 * sq(up2 - 4. * up1 + 3. * u0) + epsi;
            const double br1 = c1312 * sq(up1 - 2. * u0 + typo) + c14 * sq(up1 - um1) + epsi;
            const double br2 = c1312 * sq(u0 - 2. * um1 + um2) + c14 * sq(3. * u0 - 4. * um1 + um2) + epsi;
            const double wl0 = cd0 / sq(bl0), wl1 = cd1 / sq(bl1), wl2 = cd2 / sq(bl2), wlt = wl0 + wl1 + wl2;
            const double wr0 = cd0 / sq(br0), wr1 = cd1 / sq(br1), wr2 = cd2 / sq(br2), wrt = wr0 + wr1 + wr2;
            const double ul1 = (wl0 / wlt) * (c00 * um2 + c01 * um1 + c02 * u0) +
                               (wl1 / wlt) * (c10 * um1 + c11 * u0 + c12 * up1) +
                               (wl2 / wlt) * (c20 * u0 + c21 * up1 + c22 * up2);
            const double ur1 = (wr0 / wrt) * (c00 * up2 + c01 * up1 + c02 * u0) +
                               (wr1 / wrt) * (c10 * up1 + c11 * u0 + c12 * um1) +
                               (wr2 / wrt) * (c20 * u0 + c21 * um1 + c22 * um2);
            const double dim1 = um2 - 2. * um1 + u0, di1 = um1 - 2. * u0 + up1, dip1 = u0 - 2. * up1 + up2;
            // left state (as mp5)
            {
              const double ulmp = u0 + dmm(up1 - u0, alpha * (u0 - um1));
              double out = ul1;
              if (!((ul1 - u0) * (ul1 - ulmp) <= eps1)) {
                const double dm4iph = dm4(4. * di1 - dip1, 4. * dip1 - di1, di1, dip1);
                const double dm4imh = dm4(4. * di1 - dim1, 4. * dim1 - di1, di1, dim1);
                const double ul = u0 + alpha * (u0 - um1), av = 0.5 * (u0 + up1);
                const double md = av - 0.5 * dm4iph, lc = u0 + 0.5 * (u0 - um1) + tmp2 * dm4imh;
                const double umax = std::max(fmin3(u0, up1, md), fmin3(u0, ul, lc));
                const double umin = std::min(fmax3(u0, up1, md), fmax3(u0, ul, lc));
                out = ul1 + dmm(umin - ul1, umax - ul1);
              }
              (*L[d])[s.a(n, i, j, k)] = out;
            }
            // right state (as mp5: md = av + 0.5 dm4imh, lc = ... - tmp2 dm4iph)
            {
              const double urmp = u0 + dmm(um1 - u0, alpha * (u0 - up1));
              double out = ur1;
              if (!((ur1 - u0) * (ur1 - urmp) <= eps1)) {
                const double dm4iph = dm4(4. * di1 - dip1, 4. * dip1 - di1, di1, dip1);
                const double dm4imh = dm4(4. * di1 - dim1, 4. * dim1 - di1, di1, dim1);
                const double ul = u0 + alpha * (u0 - up1), av = 0.5 * (u0 + um1);
                const double md = av + 0.5 * dm4imh, lc = u0 + 0.5 * (u0 - up1) - tmp2 * dm4iph;
                const double umax = std::max(fmin3(u0, um1, md), fmin3(u0, ul, lc));
                const double umin = std::min(fmax3(u0, um1, md), fmax3(u0, ul, lc));
                out = ur1 + dmm(umin - ur1, umax - ur1);
              }
              (*R[d])[s.a(n, i - di, j - dj, k - dk)] = out;
            }
          }
}

// rec.f90:3439-3793 (mapped WENO5, Henrick et al. 2005) on i,j,k = 3..n-2:
// JS weights cd/(beta + eps)**2 with eps = 1e-40, normalised, mapped by
// w (cd + cd**2 - 3 cd w + w**2) / (cd**2 + w (1 - 2 cd)), normalised again.
static void weno5m(State& s) {
  const double cd[3] = {1.0 / 10.0, 6.0 / 10.0, 3.0 / 10.0};
  const double c00 = 2.0 / 6.0, c01 = -7.0 / 6.0, c02 = 11.0 / 6.0;
  const double c10 = -1.0 / 6.0, c11 = 5.0 / 6.0, c12 = 2.0 / 6.0;
  const double c20 = 2.0 / 6.0, c21 = 5.0 / 6.0, c22 = -1.0 / 6.0;
  const double epsi = 1.0e-40;
  const double c1312 = sp(13.0f / 12.0f), c14 = 0.25;
  std::vector<double>* L[3] = {&s.uriil, &s.urijl, &s.urikl};
  std::vector<double>* R[3] = {&s.uriir, &s.urijr, &s.urikr};
  auto sq = [](double x) { return x * x; };
  auto state = [&](const double be[3], double q0, double q1, double q2) {
    double wa[3], g[3];
    for (int m = 0; m < 3; ++m) wa[m] = cd[m] / sq(be[m] + epsi);
    const double wat = wa[0] + wa[1] + wa[2];
    for (int m = 0; m < 3; ++m) {
      const double w = wa[m] / wat;
      g[m] = w * (cd[m] + sq(cd[m]) - 3. * cd[m] * w + sq(w)) / (sq(cd[m]) + w * (1. - 2. * cd[m]));
    }
    const double gt = g[0] + g[1] + g[2];
    return (g[0] / gt) * q0 + (g[1] / gt) * q1 + (g[2] / gt) * q2;
  };
#pragma omp parallel for schedule(static)
  for (int k = 3; k <= s.kmax - 2; ++k)
    for (int j = 3; j <= s.jmax - 2; ++j)
      for (int i = 3; i <= s.imax - 2; ++i)
        for (int n = 1; n <= NV; ++n)
          for (int d = 0; d < 3; ++d) {
            const int di = (d == 0), dj = (d == 1), dk = (d == 2);
            auto U = [&](int o) { return s.uri[s.a(n, i + o * di, j + o * dj, k + o * dk)]; };
            const double um2 = U(-2), um1 = U(-1), u0 = U(0), up1 = U(1), up2 = U(2);
            const double bl[3] = {c1312 * sq(um2 - 2. * um1 + u0) + c14 * sq(um2 - 4. * um1 + 3. * u0),
                                  c1312 * sq(um1 - 2. * u0 + up1) + c14 * sq(um1 - up1),
                                  c1312 * sq(u0 - 2. * up1 + up2) + c14 * sq(3. * u0 - 4. * up1 + up2)};
            const double br[3] = {c1312 * sq(up2 - 2. * up1 + u0) + c14 * sq(up2 - 4. * up1 + 3. * u0),
                                  c1312 * sq(up1 - 2. * u0 + um1) + c14 * sq(up1 - um1),
                                  c1312 * sq(u0 - 2. * um1 + um2) + c14 * sq(3. * u0 - 4. * um1 + um2)};
            (*L[d])[s.a(n, i, j, k)] = state(bl, c00 * um2 + c01 * um1 + c02 * u0, c10 * um1 + c11 * u0 + c12 * up1,
                                             c20 * u0 + c21 * up1 + c22 * up2);
            (*R[d])[s.a(n, i - di, j - dj, k - dk)] =
                state(br, c00 * up2 + c01 * up1 + c02 * u0, c10 * up1 + c11 * u0 + c12 * um1,
                      c20 * u0 + c21 * um1 + c22 * um2);
          }
}

// rec.f90:1261-2058 (PPM: interp -> detect -> flaten -> monoto).
// rec2 declares dx1b(2:imax-1) while main passes dx1b(1:imax-1) (rec.f90:58,
// main.f90:120), so dummy dx1b(i) is actual dx1b(i-1).  Dummy dx1b(1), read
// at i = is1+1, lies before the actual array (undefined in the reference);
// it is taken as actual dx1b(1) here.
static void ppm(State& s) {
  const int imax = s.imax, jmax = s.jmax, kmax = s.kmax;
  const double gam = s.p.gam;
  auto shifted = [](const std::vector<double>& v) {
    // index m -> actual v[m-1]; m = 1 -> v[1]
    std::vector<double> o(v.size() + 2, 0.0);
    for (size_t m = 2; m < v.size(); ++m) o[m] = v[m - 1];
    o[1] = v[1];
    o[v.size()] = v[v.size() - 1];
    return o;
  };
  const std::vector<double> d1 = shifted(s.dx1b), d2 = shifted(s.dx2b), d3 = shifted(s.dx3b);
  const std::vector<double>* DX[3] = {&d1, &d2, &d3};
  const std::vector<double>* XX[3] = {&s.x1, &s.x2, &s.x3};
  std::vector<double>* L[3] = {&s.uriil, &s.urijl, &s.urikl};
  std::vector<double>* R[3] = {&s.uriir, &s.urijr, &s.urikr};
  const size_t N = s.ncell;
  std::vector<double> dma[3];
  for (auto& v : dma) v.assign(N * NV, 0.0);
  auto idx = [&](int d, int i, int j, int k) { return d == 0 ? i : (d == 1 ? j : k); };

  // interp, Eq. (60)-(61) (rec.f90:1346-1420); note the missing factor 2 in k (rec.f90:1414)
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= kmax - 1; ++k)
    for (int j = 2; j <= jmax - 1; ++j)
      for (int i = 2; i <= imax - 1; ++i)
        for (int n = 1; n <= NV; ++n)
          for (int d = 0; d < 3; ++d) {
            const int di = (d == 0), dj = (d == 1), dk = (d == 2);
            const std::vector<double>& dx = *DX[d];
            const int c = idx(d, i, j, k);
            const double t1a = dx[c] / (dx[c - 1] + dx[c] + dx[c + 1]);
            const double t1b = (2.0 * dx[c - 1] + dx[c]) / (dx[c + 1] + dx[c]);
            const double t1c = (dx[c] + 2.0 * dx[c + 1]) / (dx[c - 1] + dx[c]);
            const double u0 = s.uri[s.a(n, i, j, k)];
            const double sp1 = s.uri[s.a(n, i + di, j + dj, k + dk)] - u0;
            const double sm1 = u0 - s.uri[s.a(n, i - di, j - dj, k - dk)];
            const double spm1 = sp1 * sm1;
            const double da = t1a * (t1b * sp1 + t1c * sm1);
            double out;
            if (spm1 <= 0.0) {
              out = 0.0;
            } else {
              const double t1 = (da < 0.0) ? -1.0 : 1.0;
              const double t1d = std::min(std::fabs(sm1), std::fabs(sp1));
              out = (d == 2) ? t1 * std::min(std::fabs(da), t1d) : t1 * std::min(std::fabs(da), 2.0 * t1d);
            }
            dma[d][s.a(n, i, j, k)] = out;
          }
  // interp, Eq. (51) (rec.f90:1422-1468): one interface value for both states
#pragma omp parallel for schedule(static)
  for (int k = 2; k <= kmax - 2; ++k)
    for (int j = 2; j <= jmax - 2; ++j)
      for (int i = 2; i <= imax - 2; ++i)
        for (int n = 1; n <= NV; ++n)
          for (int d = 0; d < 3; ++d) {
            const int di = (d == 0), dj = (d == 1), dk = (d == 2);
            const std::vector<double>& dx = *DX[d];
            const int c = idx(d, i, j, k);
            const double u0 = s.uri[s.a(n, i, j, k)];
            const double u1 = s.uri[s.a(n, i + di, j + dj, k + dk)];
            const double t2 = (dx[c] / (dx[c] + dx[c + 1])) * (u1 - u0);
            const double t3a = 1.0 / (dx[c - 1] + dx[c] + dx[c + 1] + dx[c + 2]);
            const double t3b = (2.0 * dx[c + 1] * dx[c]) / (dx[c] + dx[c + 1]);
            const double t3c = ((dx[c - 1] + dx[c]) / (2.0 * dx[c] + dx[c + 1])) -
                               ((dx[c + 2] + dx[c + 1]) / (2.0 * dx[c + 1] + dx[c]));
            const double t3 = t3a * t3b * t3c * (u1 - u0);
            const double t4 = t3a * dx[c] * ((dx[c - 1] + dx[c]) / (2.0 * dx[c] + dx[c + 1]));
            const double t5 = t3a * dx[c + 1] * ((dx[c + 1] + dx[c + 2]) / (dx[c] + 2.0 * dx[c + 1]));
            const double v = u0 + t2 + t3 - t4 * dma[d][s.a(n, i + di, j + dj, k + dk)] +
                             t5 * dma[d][s.a(n, i, j, k)];
            (*R[d])[s.a(n, i, j, k)] = v;
            (*L[d])[s.a(n, i, j, k)] = v;
          }

  // detect (rec.f90:1479-1686), contact steepening on density
  {
    const double eta1 = 5.0, eta2 = 0.05, eps1 = 0.1, ak0 = 1.0;
    std::vector<double> dda[3], eta[3];
    for (int d = 0; d < 3; ++d) { dda[d].assign(N, 0.0); eta[d].assign(N, 0.0); }
#pragma omp parallel for schedule(static)
    for (int k = 2; k <= kmax - 1; ++k)
      for (int j = 2; j <= jmax - 1; ++j)
        for (int i = 2; i <= imax - 1; ++i)
          for (int d = 0; d < 3; ++d) {
            const int di = (d == 0), dj = (d == 1), dk = (d == 2);
            const std::vector<double>& dx = *DX[d];
            const int c = idx(d, i, j, k);
            const double t0a = 1.0 / (dx[c - 1] + dx[c] + dx[c + 1]);
            const double t0b = (s.uri[s.a(1, i + di, j + dj, k + dk)] - s.uri[s.a(1, i, j, k)]) / (dx[c + 1] + dx[c]);
            const double t0c = (s.uri[s.a(1, i, j, k)] - s.uri[s.a(1, i - di, j - dj, k - dk)]) / (dx[c] + dx[c - 1]);
            dda[d][s.cell(i, j, k)] = t0a * (t0b - t0c);
          }
#pragma omp parallel for schedule(static)
    for (int k = 3; k <= kmax - 2; ++k)
      for (int j = 3; j <= jmax - 2; ++j)
        for (int i = 3; i <= imax - 2; ++i)
          for (int d = 0; d < 3; ++d) {
            const int di = (d == 0), dj = (d == 1), dk = (d == 2);
            const std::vector<double>& x = *XX[d];
            const int c = idx(d, i, j, k);
            const double rp = s.uri[s.a(1, i + di, j + dj, k + dk)], rm = s.uri[s.a(1, i - di, j - dj, k - dk)];
            const double ddp = dda[d][s.cell(i + di, j + dj, k + dk)], ddm = dda[d][s.cell(i - di, j - dj, k - dk)];
            const double t1 = ddp * ddm;
            const double t2 = std::fabs(rp - rm) - eps1 * std::min(std::fabs(rp), std::fabs(rm));
            double etatil;
            if (t1 >= 0.0 && t2 <= 0.0) {
              etatil = 0.0;
            } else {
              const double t2a = -(ddp - ddm) / (x[c + 1] - x[c - 1]);
              const double a = x[c] - x[c - 1], b = x[c + 1] - x[c];
              const double t2b = (a * a * a + b * b * b) / (rp - rm);
              etatil = t2a * t2b;
            }
            eta[d][s.cell(i, j, k)] = std::max(0.0, std::min(eta1 * (etatil - eta2), 1.0));
          }
#pragma omp parallel for schedule(static)
    for (int k = 3; k <= kmax - 2; ++k)
      for (int j = 3; j <= jmax - 2; ++j)
        for (int i = 3; i <= imax - 2; ++i)
          for (int d = 0; d < 3; ++d) {
            const int di = (d == 0), dj = (d == 1), dk = (d == 2);
            const double rp = s.uri[s.a(1, i + di, j + dj, k + dk)], rm = s.uri[s.a(1, i - di, j - dj, k - dk)];
            const double pp = s.uri[s.a(5, i + di, j + dj, k + dk)], pm = s.uri[s.a(5, i - di, j - dj, k - dk)];
            const double t3 = std::fabs(rp - rm) / std::min(rp, rm);
            const double t4 = std::fabs(pp - pm) / std::min(pp, pm);
            if (gam * ak0 * t3 < t4) eta[d][s.cell(i, j, k)] = 0.0;
          }
#pragma omp parallel for schedule(static)
    for (int k = 3; k <= kmax - 2; ++k)
      for (int j = 3; j <= jmax - 2; ++j)
        for (int i = 3; i <= imax - 2; ++i)
          for (int d = 0; d < 3; ++d) {
            const int di = (d == 0), dj = (d == 1), dk = (d == 2);
            const double e = eta[d][s.cell(i, j, k)];
            double& l = (*L[d])[s.a(1, i, j, k)];
            l = l * (1.0 - e) + (s.uri[s.a(1, i + di, j + dj, k + dk)] - 0.5 * dma[d][s.a(1, i + di, j + dj, k + dk)]) * e;
            double& r = (*R[d])[s.a(1, i - di, j - dj, k - dk)];
            r = r * (1.0 - e) + (s.uri[s.a(1, i - di, j - dj, k - dk)] + 0.5 * dma[d][s.a(1, i - di, j - dj, k - dk)]) * e;
          }
  }

  // flaten (rec.f90:1689-1884); velocity index of direction d is uri(d+1)
  {
    const double eps2 = 1.0, omg2 = 0.52, omg3 = 10.0;
    std::vector<double> f1a[3], f2a[3];
    for (int d = 0; d < 3; ++d) { f1a[d].assign(N, 0.0); f2a[d].assign(N, 0.0); }
#pragma omp parallel for schedule(static)
    for (int k = 3; k <= kmax - 2; ++k)
      for (int j = 3; j <= jmax - 2; ++j)
        for (int i = 3; i <= imax - 2; ++i)
          for (int d = 0; d < 3; ++d) {
            const int di = (d == 0), dj = (d == 1), dk = (d == 2);
            const double pp1 = s.uri[s.a(5, i + di, j + dj, k + dk)], pm1 = s.uri[s.a(5, i - di, j - dj, k - dk)];
            const double t3a = std::fabs(pp1 - pm1);
            const double t1 = eps2 * std::min(pp1, pm1) - t3a;
            const double t2 = s.uri[s.a(d + 2, i + di, j + dj, k + dk)] - s.uri[s.a(d + 2, i - di, j - dj, k - dk)];
            const double omg1 = (t1 < 0.0 && t2 < 0.0) ? 1.0 : 0.0;
            const double t3b = s.uri[s.a(5, i + 2 * di, j + 2 * dj, k + 2 * dk)] - s.uri[s.a(5, i - 2 * di, j - 2 * dj, k - 2 * dk)];
            double t4;
            if (t3b == 0.0) t4 = (t3a == 0.0) ? -omg2 : 1.0 - omg2;
            else t4 = (t3a / t3b) - omg2;
            f1a[d][s.cell(i, j, k)] = std::min(1.0, omg1 * std::max(0.0, t4 * omg3));
          }
#pragma omp parallel for schedule(static)
    for (int k = 4; k <= kmax - 3; ++k)
      for (int j = 4; j <= jmax - 3; ++j)
        for (int i = 4; i <= imax - 3; ++i)
          for (int d = 0; d < 3; ++d) {
            const int di = (d == 0), dj = (d == 1), dk = (d == 2);
            const double f1b = (s.uri[s.a(5, i + di, j + dj, k + dk)] - s.uri[s.a(5, i - di, j - dj, k - dk)] < 0.0)
                                   ? f1a[d][s.cell(i + di, j + dj, k + dk)]
                                   : f1a[d][s.cell(i - di, j - dj, k - dk)];
            f2a[d][s.cell(i, j, k)] = std::max(f1a[d][s.cell(i, j, k)], f1b);
          }
#pragma omp parallel for schedule(static)
    for (int k = 4; k <= kmax - 3; ++k)
      for (int j = 4; j <= jmax - 3; ++j)
        for (int i = 4; i <= imax - 3; ++i)
          for (int n = 1; n <= NV; ++n)
            for (int d = 0; d < 3; ++d) {
              const int di = (d == 0), dj = (d == 1), dk = (d == 2);
              const double f = f2a[d][s.cell(i, j, k)];
              const double u0 = s.uri[s.a(n, i, j, k)];
              double& l = (*L[d])[s.a(n, i, j, k)];
              l = u0 * f + l * (1.0 - f);
              double& r = (*R[d])[s.a(n, i - di, j - dj, k - dk)];
              r = u0 * f + r * (1.0 - f);
            }
  }

  // monoto (rec.f90:1887-2056); the uriil1/uriir1 pass has no effect and is omitted
#pragma omp parallel for schedule(static)
  for (int k = 3; k <= kmax - 2; ++k)
    for (int j = 3; j <= jmax - 2; ++j)
      for (int i = 3; i <= imax - 2; ++i)
        for (int n = 1; n <= NV; ++n)
          for (int d = 0; d < 3; ++d) {
            const int di = (d == 0), dj = (d == 1), dk = (d == 2);
            const double u0 = s.uri[s.a(n, i, j, k)];
            double& l = (*L[d])[s.a(n, i, j, k)];
            double& r = (*R[d])[s.a(n, i - di, j - dj, k - dk)];
            if ((l - u0) * (r - u0) >= 0.0) { l = u0; r = u0; }
          }
#pragma omp parallel for schedule(static)
  for (int k = 3; k <= kmax - 2; ++k)
    for (int j = 3; j <= jmax - 2; ++j)
      for (int i = 3; i <= imax - 2; ++i)
        for (int n = 1; n <= NV; ++n)
          for (int d = 0; d < 3; ++d) {
            const int di = (d == 0), dj = (d == 1), dk = (d == 2);
            const double u0 = s.uri[s.a(n, i, j, k)];
            double& l = (*L[d])[s.a(n, i, j, k)];
            double& r = (*R[d])[s.a(n, i - di, j - dj, k - dk)];
            const double t3 = 6.0 * (l - r) * (u0 - 0.5 * (l + r));
            const double t4 = (l - r) * (l - r);
            if (t3 > t4) r = 3.0 * u0 - 2.0 * l;
            if (-t3 > t4) l = 3.0 * u0 - 2.0 * r;
          }
}

// rec.f90:2-142: reconstruction, then face conserved (caluu3, caluu.f90:236-356)
// and face fluxes (calflx3i/j/k) for both states in all three directions.
// Positivity guard (guard = 1 only; not part of the reference).  MP5's
// monotonicity switch compares against an absolute 1e-10 (rec.f90:2092) and
// WENO5's smoothness indicators carry an absolute epsi = 1e-6 (rec.f90:2400),
// so on 1e-7-scale floor densities both reduce to unlimited high-order
// interpolation and undershoot to rho < 0 next to a torus surface.  The
// reference then evaluates de**gam of a negative number (calflx.f90:474) and
// NaN enters the entropy flux and, through the entropy fallback of recov1a,
// the primitives.  With guard = 1 a face state whose reconstructed rho or p is
// not positive is replaced by its owner cell's primitives (first order).
static void face_guard(State& s) {
  const int nm0 = s.nm0;
  std::vector<double>* L[3] = {&s.uriil, &s.urijl, &s.urikl};
  std::vector<double>* R[3] = {&s.uriir, &s.urijr, &s.urikr};
#pragma omp parallel for schedule(static)
  for (int k = nm0; k <= s.kmax - nm0; ++k)
    for (int j = nm0; j <= s.jmax - nm0; ++j)
      for (int i = nm0; i <= s.imax - nm0; ++i)
        for (int d = 0; d < 3; ++d) {
          const int di = (d == 0), dj = (d == 1), dk = (d == 2);
          double* l = &(*L[d])[s.a(1, i, j, k)];
          if (!(l[0] > 0.0 && l[4] > 0.0)) std::memcpy(l, &s.uri[s.a(1, i, j, k)], NV * sizeof(double));
          double* r = &(*R[d])[s.a(1, i, j, k)];
          if (!(r[0] > 0.0 && r[4] > 0.0))
            std::memcpy(r, &s.uri[s.a(1, i + di, j + dj, k + dk)], NV * sizeof(double));
        }
}

void rec2(State& s) {
  if (s.p.irec == 1 || s.p.irec == 2 || s.p.irec == 11 || s.p.irec == 12 || s.p.irec == 13) limiters(s, s.p.irec);
  else if (s.p.irec == 3) muscl(s);
  else if (s.p.irec == 4) ceno(s);
  else if (s.p.irec == 6) mp5(s);
  else if (s.p.irec == 7) weno5(s);
  else if (s.p.irec == 8) mpweno5(s);
  else if (s.p.irec == 9) weno5z(s);
  else if (s.p.irec == 10) weno5m(s);
  else ppm(s);
  if (s.p.guard & 1) face_guard(s);
  const double gam = s.p.gam;
  const int nm0 = s.nm0;
  struct Dir { std::vector<double>*r, *l, *ur, *ul, *wr, *wl; };
  Dir D[3] = {{&s.uriir, &s.uriil, &s.uuir, &s.uuil, &s.wwir, &s.wwil},
              {&s.urijr, &s.urijl, &s.uujr, &s.uujl, &s.wwjr, &s.wwjl},
              {&s.urikr, &s.urikl, &s.uukr, &s.uukl, &s.wwkr, &s.wwkl}};
#pragma omp parallel for schedule(static)
  for (int k = nm0; k <= s.kmax - nm0; ++k)
    for (int j = nm0; j <= s.jmax - nm0; ++j)
      for (int i = nm0; i <= s.imax - nm0; ++i) {
        const size_t q = s.ik(i, k);
        for (int d = 0; d < 3; ++d) {
          const M4& g = (d == 0) ? s.gcovi[q] : (d == 1 ? s.gcov[q] : s.gcovk[q]);
          const M4& gc = (d == 0) ? s.gconi[q] : (d == 1 ? s.gcon[q] : s.gconk[q]);
          const double dg = (d == 0) ? s.detgi[q] : (d == 1 ? s.detg[q] : s.detgk[q]);
          const size_t o = s.a(1, i, j, k);
          PS ps;
          pstate(&(*D[d].r)[o], g, gc, gam, ps);
          p2c(ps, gam, dg, &(*D[d].ur)[o]);
          flux(ps, d + 1, gam, dg, &(*D[d].wr)[o]);
          pstate(&(*D[d].l)[o], g, gc, gam, ps);
          p2c(ps, gam, dg, &(*D[d].ul)[o]);
          flux(ps, d + 1, gam, dg, &(*D[d].wl)[o]);
        }
      }
}

// calcha.f90:2-126 (with the reference's cmink quirk at calcha.f90:107)
void calcha(State& s) {
  const double gam = s.p.gam;
  const int nm0 = s.nm0;
  const std::vector<double>* R[3] = {&s.uriir, &s.urijr, &s.urikr};
  const std::vector<double>* L[3] = {&s.uriil, &s.urijl, &s.urikl};
  std::vector<double>* CX[3] = {&s.cmaxi, &s.cmaxj, &s.cmaxk};
  std::vector<double>* CN[3] = {&s.cmini, &s.cminj, &s.cmink};
#pragma omp parallel for schedule(static)
  for (int k = nm0; k <= s.kmax - nm0; ++k)
    for (int j = nm0; j <= s.jmax - nm0; ++j)
      for (int i = nm0; i <= s.imax - nm0; ++i) {
        const size_t q = s.ik(i, k);
        for (int d = 0; d < 3; ++d) {
          const M4& g = (d == 0) ? s.gcovi[q] : (d == 1 ? s.gcov[q] : s.gcovk[q]);
          const M4& gc = (d == 0) ? s.gconi[q] : (d == 1 ? s.gcon[q] : s.gconk[q]);
          const size_t o = s.a(1, i, j, k);
          double vpr, vmr, vpl, vml;
          calcha4d(&(*R[d])[o], g, gc, gam, d + 1, vpr, vmr);
          calcha4d(&(*L[d])[o], g, gc, gam, d + 1, vpl, vml);
          const size_t c = s.cell(i, j, k);
          (*CX[d])[c] = fmax3(0.0, vpr, vpl);
          (*CN[d])[c] = (d == 2) ? fmin3(0.0, vpr, vml) : fmin3(0.0, vmr, vml);
        }
      }
}

// hll.f90:47-192 ("HLLE" whose subsonic branch is Rusanov/LLF)
void hlle(State& s) {
  const int nm0 = s.nm0;
  const std::vector<double>* WL[3] = {&s.wwil, &s.wwjl, &s.wwkl};
  const std::vector<double>* WR[3] = {&s.wwir, &s.wwjr, &s.wwkr};
  const std::vector<double>* UL[3] = {&s.uuil, &s.uujl, &s.uukl};
  const std::vector<double>* UR[3] = {&s.uuir, &s.uujr, &s.uukr};
  const std::vector<double>* CX[3] = {&s.cmaxi, &s.cmaxj, &s.cmaxk};
  const std::vector<double>* CN[3] = {&s.cmini, &s.cminj, &s.cmink};
#pragma omp parallel for schedule(static)
  for (int k = nm0; k <= s.kmax - nm0; ++k)
    for (int j = nm0; j <= s.jmax - nm0; ++j)
      for (int i = nm0; i <= s.imax - nm0; ++i)
        for (int n = 1; n <= NV; ++n)
          for (int d = 0; d < 3; ++d) {
            const size_t c = s.cell(i, j, k), o = s.a(n, i, j, k);
            const double cmin = (*CN[d])[c], cmax = (*CX[d])[c];
            double& w = s.ww[s.w(d + 1, n, i, j, k)];
            if (cmin > 0.0) {
              w = (*WL[d])[o];
            } else if (cmin <= 0.0 && cmax > 0.0) {
              const double c1 = std::max(std::fabs(cmax), std::fabs(cmin));
              w = 0.5 * ((*WL[d])[o] + (*WR[d])[o] - c1 * ((*UR[d])[o] - (*UL[d])[o]));
            } else if (cmax <= 0.0) {
              w = (*WR[d])[o];
            }
            if (std::fabs(w) < 1.0e-40) w = 0.0;
          }
}

namespace {
// ct.f90:30-118 (Toth flux-CT)
void fluxct(State& s) {
  const int nm0 = s.nm0, nm1 = s.nm1;
  const size_t N = s.ncell;
  std::vector<double> fyx(N), fzx(N), fxy(N), fzy(N), fxz(N), fyz(N);
#pragma omp parallel for schedule(static)
  for (int k = nm0; k <= s.kmax - nm0; ++k)
    for (int j = nm0; j <= s.jmax - nm0; ++j)
      for (int i = nm0; i <= s.imax - nm0; ++i) {
        const size_t c = s.cell(i, j, k);
        fyx[c] = s.ww[s.w(2, 7, i, j, k)];
        fzx[c] = s.ww[s.w(3, 7, i, j, k)];
        fxy[c] = s.ww[s.w(1, 8, i, j, k)];
        fzy[c] = s.ww[s.w(3, 8, i, j, k)];
        fxz[c] = s.ww[s.w(1, 9, i, j, k)];
        fyz[c] = s.ww[s.w(2, 9, i, j, k)];
      }
  auto C = [&](int i, int j, int k) { return s.cell(i, j, k); };
#pragma omp parallel for schedule(static)
  for (int k = nm1; k <= s.kmax - nm1; ++k)
    for (int j = nm1; j <= s.jmax - nm1; ++j)
      for (int i = nm1; i <= s.imax - nm1; ++i) {
        const double e = 1.0 / 8.0;
        s.ww[s.w(2, 7, i, j, k)] = e * (2.0 * fyx[C(i, j, k)] + fyx[C(i + 1, j, k)] + fyx[C(i - 1, j, k)] -
                                        fxy[C(i, j, k)] - fxy[C(i, j + 1, k)] - fxy[C(i - 1, j, k)] - fxy[C(i - 1, j + 1, k)]);
        s.ww[s.w(3, 7, i, j, k)] = e * (2.0 * fzx[C(i, j, k)] + fzx[C(i + 1, j, k)] + fzx[C(i - 1, j, k)] -
                                        fxz[C(i, j, k)] - fxz[C(i, j, k + 1)] - fxz[C(i - 1, j, k)] - fxz[C(i - 1, j, k + 1)]);
        s.ww[s.w(1, 8, i, j, k)] = e * (2.0 * fxy[C(i, j, k)] + fxy[C(i, j + 1, k)] + fxy[C(i, j - 1, k)] -
                                        fyx[C(i, j, k)] - fyx[C(i + 1, j, k)] - fyx[C(i, j - 1, k)] - fyx[C(i + 1, j - 1, k)]);
        s.ww[s.w(3, 8, i, j, k)] = e * (2.0 * fzy[C(i, j, k)] + fzy[C(i, j + 1, k)] + fzy[C(i, j - 1, k)] -
                                        fyz[C(i, j, k)] - fyz[C(i, j, k + 1)] - fyz[C(i, j - 1, k)] - fyz[C(i, j - 1, k + 1)]);
        s.ww[s.w(1, 9, i, j, k)] = e * (2.0 * fxz[C(i, j, k)] + fxz[C(i, j, k + 1)] + fxz[C(i, j, k - 1)] -
                                        fzx[C(i, j, k)] - fzx[C(i + 1, j, k)] - fzx[C(i, j, k - 1)] - fzx[C(i + 1, j, k - 1)]);
        s.ww[s.w(2, 9, i, j, k)] = e * (2.0 * fyz[C(i, j, k)] + fyz[C(i, j, k + 1)] + fyz[C(i, j, k - 1)] -
                                        fzy[C(i, j, k)] - fzy[C(i, j + 1, k)] - fzy[C(i, j, k - 1)] - fzy[C(i, j + 1, k - 1)]);
      }
}

// ct.f90:121-233 (mflct, Gardiner & Stone 2005): cell-centred EMFs from the
// face fluxes on nm0+1..n-nm0, then the flux-CT brackets weighted 1/4 plus
// averaged EMFs on nm1..n-nm1.
void mflct(State& s) {
  const int nm0 = s.nm0, nm1 = s.nm1;
  const size_t N = s.ncell;
  std::vector<double> fyx(N), fzx(N), fxy(N), fzy(N), fxz(N), fyz(N), exc(N), eyc(N), ezc(N);
  auto C = [&](int i, int j, int k) { return s.cell(i, j, k); };
#pragma omp parallel for schedule(static)
  for (int k = nm0; k <= s.kmax - nm0; ++k)
    for (int j = nm0; j <= s.jmax - nm0; ++j)
      for (int i = nm0; i <= s.imax - nm0; ++i) {
        const size_t c = C(i, j, k);
        fyx[c] = s.ww[s.w(2, 7, i, j, k)];
        fzx[c] = s.ww[s.w(3, 7, i, j, k)];
        fxy[c] = s.ww[s.w(1, 8, i, j, k)];
        fzy[c] = s.ww[s.w(3, 8, i, j, k)];
        fxz[c] = s.ww[s.w(1, 9, i, j, k)];
        fyz[c] = s.ww[s.w(2, 9, i, j, k)];
      }
#pragma omp parallel for schedule(static)
  for (int k = nm0 + 1; k <= s.kmax - nm0; ++k)
    for (int j = nm0 + 1; j <= s.jmax - nm0; ++j)
      for (int i = nm0 + 1; i <= s.imax - nm0; ++i) {
        const size_t c = C(i, j, k);
        ezc[c] = 0.25 * (-fxy[C(i - 1, j, k)] - fxy[c] + fyx[C(i, j - 1, k)] + fyx[c]);
        exc[c] = 0.25 * (-fyz[C(i, j - 1, k)] - fyz[c] + fzy[C(i, j, k - 1)] + fzy[c]);
        eyc[c] = 0.25 * (-fzx[C(i, j, k - 1)] - fzx[c] + fxz[C(i - 1, j, k)] + fxz[c]);
      }
  const double q = 1.0 / 4.0, h = 1.0 / 8.0;
#pragma omp parallel for schedule(static)
  for (int k = nm1; k <= s.kmax - nm1; ++k)
    for (int j = nm1; j <= s.jmax - nm1; ++j)
      for (int i = nm1; i <= s.imax - nm1; ++i) {
        const double fbyx = q * (2.0 * fyx[C(i, j, k)] + fyx[C(i + 1, j, k)] + fyx[C(i - 1, j, k)] - fxy[C(i, j, k)] -
                                 fxy[C(i, j + 1, k)] - fxy[C(i - 1, j, k)] - fxy[C(i - 1, j + 1, k)]);
        const double fbzx = q * (2.0 * fzx[C(i, j, k)] + fzx[C(i + 1, j, k)] + fzx[C(i - 1, j, k)] - fxz[C(i, j, k)] -
                                 fxz[C(i, j, k + 1)] - fxz[C(i - 1, j, k)] - fxz[C(i - 1, j, k + 1)]);
        const double fbxy = q * (2.0 * fxy[C(i, j, k)] + fxy[C(i, j + 1, k)] + fxy[C(i, j - 1, k)] - fyx[C(i, j, k)] -
                                 fyx[C(i + 1, j, k)] - fyx[C(i, j - 1, k)] - fyx[C(i + 1, j - 1, k)]);
        const double fbzy = q * (2.0 * fzy[C(i, j, k)] + fzy[C(i, j + 1, k)] + fzy[C(i, j - 1, k)] - fyz[C(i, j, k)] -
                                 fyz[C(i, j, k + 1)] - fyz[C(i, j - 1, k)] - fyz[C(i, j - 1, k + 1)]);
        const double fbxz = q * (2.0 * fxz[C(i, j, k)] + fxz[C(i, j, k + 1)] + fxz[C(i, j, k - 1)] - fzx[C(i, j, k)] -
                                 fzx[C(i + 1, j, k)] - fzx[C(i, j, k - 1)] - fzx[C(i + 1, j, k - 1)]);
        const double fbyz = q * (2.0 * fyz[C(i, j, k)] + fyz[C(i, j, k + 1)] + fyz[C(i, j, k - 1)] - fzy[C(i, j, k)] -
                                 fzy[C(i, j + 1, k)] - fzy[C(i, j, k - 1)] - fzy[C(i, j + 1, k - 1)]);
        const double fhyx = -h * (2. * ezc[C(i, j, k)] + 2. * ezc[C(i, j + 1, k)] + ezc[C(i + 1, j, k)] +
                                  ezc[C(i + 1, j + 1, k)] + ezc[C(i - 1, j, k)] + ezc[C(i - 1, j + 1, k)]);
        const double fhzx = h * (2. * eyc[C(i, j, k)] + 2. * eyc[C(i, j, k + 1)] + eyc[C(i + 1, j, k)] +
                                 eyc[C(i + 1, j, k + 1)] + eyc[C(i - 1, j, k)] + eyc[C(i - 1, j, k + 1)]);
        const double fhxy = h * (2. * ezc[C(i, j, k)] + 2. * ezc[C(i + 1, j, k)] + ezc[C(i, j + 1, k)] +
                                 ezc[C(i + 1, j + 1, k)] + ezc[C(i, j - 1, k)] + ezc[C(i + 1, j - 1, k)]);
        const double fhzy = -h * (2. * exc[C(i, j, k)] + 2. * exc[C(i, j, k + 1)] + exc[C(i, j + 1, k)] +
                                  exc[C(i, j + 1, k + 1)] + exc[C(i, j - 1, k)] + exc[C(i, j - 1, k + 1)]);
        const double fhxz = -h * (2. * eyc[C(i, j, k)] + 2. * eyc[C(i + 1, j, k)] + eyc[C(i, j, k + 1)] +
                                  eyc[C(i + 1, j, k + 1)] + eyc[C(i, j, k - 1)] + eyc[C(i + 1, j, k - 1)]);
        const double fhyz = h * (2. * exc[C(i, j, k)] + 2. * exc[C(i, j + 1, k)] + exc[C(i, j, k + 1)] +
                                 exc[C(i, j + 1, k + 1)] + exc[C(i, j, k - 1)] + exc[C(i, j + 1, k - 1)]);
        s.ww[s.w(2, 7, i, j, k)] = fbyx + fhyx;
        s.ww[s.w(3, 7, i, j, k)] = fbzx + fhzx;
        s.ww[s.w(1, 8, i, j, k)] = fbxy + fhxy;
        s.ww[s.w(3, 8, i, j, k)] = fbzy + fhzy;
        s.ww[s.w(1, 9, i, j, k)] = fbxz + fhxz;
        s.ww[s.w(2, 9, i, j, k)] = fbyz + fhyz;
      }
}

// ct.f90:236-445 (upflct, ict 3): upwinded corner EMFs.  Level 1 (on
// nm0+1..n-nm0-1): cell-centred EMFs e?c, face-pair EMFs e?b and 1/8 flux-CT
// brackets fb??; level 2 (on nm0+1..n-nm0-2): differences d?e? upwinded by
// the sign of the velocity uri(2..4) at the cell; level 3 (on nm1..n-nm1):
// corner EMFs averaged into the six induction fluxes.  Every index is the
// reference's as written: eyb reads fzx at j+1; each fb?? takes the 2-1-1
// average of its own flux along the direction that is neither its face
// normal nor its field component (fluxct takes it along the face normal);
// every elseif after dyez's tests uri(2); dzey's negative-velocity branch
// subtracts eyc(i), not eyc(i+1).
void upflct(State& s) {
  const int nm0 = s.nm0, nm1 = s.nm1, nm2 = nm0 + 1, nm3 = nm0 + 2;
  const size_t N = s.ncell;
  std::vector<double> fyx(N), fzx(N), fxy(N), fzy(N), fxz(N), fyz(N);
  std::vector<double> exc(N), eyc(N), ezc(N), exb(N), eyb(N), ezb(N);
  std::vector<double> fbyx(N), fbzx(N), fbxy(N), fbzy(N), fbxz(N), fbyz(N);
  std::vector<double> dyez(N), dxez(N), dyex(N), dzex(N), dxey(N), dzey(N);
  auto C = [&](int i, int j, int k) { return s.cell(i, j, k); };
#pragma omp parallel for schedule(static)
  for (int k = nm0; k <= s.kmax - nm0; ++k)
    for (int j = nm0; j <= s.jmax - nm0; ++j)
      for (int i = nm0; i <= s.imax - nm0; ++i) {
        const size_t c = C(i, j, k);
        fyx[c] = s.ww[s.w(2, 7, i, j, k)];
        fzx[c] = s.ww[s.w(3, 7, i, j, k)];
        fxy[c] = s.ww[s.w(1, 8, i, j, k)];
        fzy[c] = s.ww[s.w(3, 8, i, j, k)];
        fxz[c] = s.ww[s.w(1, 9, i, j, k)];
        fyz[c] = s.ww[s.w(2, 9, i, j, k)];
      }
  const double q = 0.25, e = 1.0 / 8.0, h = 0.5;
#pragma omp parallel for schedule(static)
  for (int k = nm2; k <= s.kmax - nm2; ++k)
    for (int j = nm2; j <= s.jmax - nm2; ++j)
      for (int i = nm2; i <= s.imax - nm2; ++i) {
        const size_t c = C(i, j, k);
        ezc[c] = q * (-fxy[C(i - 1, j, k)] - fxy[c] + fyx[C(i, j - 1, k)] + fyx[c]);
        exc[c] = q * (-fyz[C(i, j - 1, k)] - fyz[c] + fzy[C(i, j, k - 1)] + fzy[c]);
        eyc[c] = q * (-fzx[C(i, j, k - 1)] - fzx[c] + fxz[C(i - 1, j, k)] + fxz[c]);
        ezb[c] = q * (fyx[c] + fyx[C(i + 1, j, k)] - fxy[c] - fxy[C(i, j + 1, k)]);
        exb[c] = q * (fzy[c] + fzy[C(i, j + 1, k)] - fyz[c] - fyz[C(i, j, k + 1)]);
        eyb[c] = q * (fxz[c] + fxz[C(i + 1, j, k)] - fzx[c] - fzx[C(i, j + 1, k)]);
        fbyx[c] = e * (2.0 * fyx[c] + fyx[C(i, j, k + 1)] + fyx[C(i, j, k - 1)] - fxy[c] - fxy[C(i, j + 1, k)] -
                       fxy[C(i - 1, j, k)] - fxy[C(i - 1, j + 1, k)]);
        fbzx[c] = e * (2.0 * fzx[c] + fzx[C(i, j + 1, k)] + fzx[C(i, j - 1, k)] - fxz[c] - fxz[C(i, j, k + 1)] -
                       fxz[C(i - 1, j, k)] - fxz[C(i - 1, j, k + 1)]);
        fbxy[c] = e * (2.0 * fxy[c] + fxy[C(i, j, k + 1)] + fxy[C(i, j, k - 1)] - fyx[c] - fyx[C(i + 1, j, k)] -
                       fyx[C(i, j - 1, k)] - fyx[C(i + 1, j - 1, k)]);
        fbzy[c] = e * (2.0 * fzy[c] + fzy[C(i + 1, j, k)] + fzy[C(i - 1, j, k)] - fyz[c] - fyz[C(i, j, k + 1)] -
                       fyz[C(i, j - 1, k)] - fyz[C(i, j - 1, k + 1)]);
        fbxz[c] = e * (2.0 * fxz[c] + fxz[C(i, j + 1, k)] + fxz[C(i, j - 1, k)] - fzx[c] - fzx[C(i + 1, j, k)] -
                       fzx[C(i, j, k - 1)] - fzx[C(i + 1, j, k - 1)]);
        fbyz[c] = e * (2.0 * fyz[c] + fyz[C(i + 1, j, k)] + fyz[C(i - 1, j, k)] - fzy[c] - fzy[C(i, j + 1, k)] -
                       fzy[C(i, j, k - 1)] - fzy[C(i, j + 1, k - 1)]);
      }
  // upwinded differences: a(c) - b(c) when u > 0, a(n) - b(n) when u < 0
  // (n the neighbour up the direction), the mean of both otherwise
  auto up = [&](double u, double ul, const std::vector<double>& a, const std::vector<double>& b, size_t c, size_t n,
                size_t bneg) {
    if (u > 0.0) return a[c] - b[c];
    if (ul < 0.0) return a[n] - b[bneg];
    return h * (a[c] + a[n] - b[c] - b[n]);
  };
#pragma omp parallel for schedule(static)
  for (int k = nm2; k <= s.kmax - nm3; ++k)
    for (int j = nm2; j <= s.jmax - nm3; ++j)
      for (int i = nm2; i <= s.imax - nm3; ++i) {
        const size_t c = C(i, j, k), ci = C(i + 1, j, k), cj = C(i, j + 1, k), ck = C(i, j, k + 1);
        const double u1 = s.uri[s.a(2, i, j, k)], u2 = s.uri[s.a(3, i, j, k)], u3 = s.uri[s.a(4, i, j, k)];
        dyez[c] = up(u1, u1, fbyx, ezc, c, ci, ci);
        dxez[c] = up(u2, u1, fbxy, ezc, c, cj, cj);
        dyex[c] = up(u3, u1, fbyz, exc, c, ck, ck);
        dzex[c] = up(u2, u1, fbzy, exc, c, cj, cj);
        dxey[c] = up(u3, u1, fbxz, eyc, c, ck, ck);
        dzey[c] = up(u1, u1, fbzx, eyc, c, ci, c);
      }
#pragma omp parallel for schedule(static)
  for (int k = nm1; k <= s.kmax - nm1; ++k)
    for (int j = nm1; j <= s.jmax - nm1; ++j)
      for (int i = nm1; i <= s.imax - nm1; ++i) {
        const size_t c = C(i, j, k);
        const size_t im = C(i - 1, j, k), jm = C(i, j - 1, k), km = C(i, j, k - 1);
        const size_t ip = C(i + 1, j, k), jp = C(i, j + 1, k), kp = C(i, j, k + 1);
        const size_t imjp = C(i - 1, j + 1, k), ipjm = C(i + 1, j - 1, k), jmkp = C(i, j - 1, k + 1);
        const size_t jpkm = C(i, j + 1, k - 1), imkp = C(i - 1, j, k + 1), ipkm = C(i + 1, j, k - 1);
        const double ezh = ezb[c] + q * (dyez[c] - dyez[jp]) + q * (dxez[c] - dxez[ip]);
        const double ezhmi = ezb[im] + q * (dyez[im] - dyez[imjp]) + q * (dxez[im] - dxez[c]);
        const double ezhmj = ezb[jm] + q * (dyez[jm] - dyez[c]) + q * (dxez[jm] - dxez[ipjm]);
        const double exh = exb[c] + q * (dyex[c] - dyex[jp]) + q * (dzex[c] - dzex[kp]);
        const double exhmj = exb[jm] + q * (dyex[jm] - dyex[c]) + q * (dzex[jm] - dzex[jmkp]);
        const double exhmk = exb[km] + q * (dyex[km] - dyex[jpkm]) + q * (dzex[km] - dzex[c]);
        const double eyh = eyb[c] + q * (dxey[c] - dxey[ip]) + q * (dzey[c] - dzey[kp]);
        const double eyhmi = eyb[im] + q * (dxey[im] - dxey[c]) + q * (dzey[im] - dzey[imkp]);
        const double eyhmk = eyb[km] + q * (dxey[km] - dxey[ipkm]) + q * (dzey[km] - dzey[c]);
        s.ww[s.w(2, 7, i, j, k)] = h * (ezh + ezhmi);
        s.ww[s.w(3, 7, i, j, k)] = h * (-eyh - eyhmi);
        s.ww[s.w(1, 8, i, j, k)] = h * (-ezh - ezhmj);
        s.ww[s.w(3, 8, i, j, k)] = h * (exh + exhmj);
        s.ww[s.w(1, 9, i, j, k)] = h * (eyh + eyhmk);
        s.ww[s.w(2, 9, i, j, k)] = h * (-exh - exhmk);
      }
}
}  // namespace

// ct.f90:4-27: the constrained-transport scheme ict.  guard bit 2 (not in
// the reference) first zeroes the flux of each face's normal field
// component: the reference keeps the LLF diffusion -0.5 c (B^d_R - B^d_L) in
// ww(1,7), ww(2,8), ww(3,9) (hll.f90:109-111), which CT does not replace, so
// its corner divergence of B is not conserved.
void ct(State& s) {
  const int nm0 = s.nm0;
  if (s.p.guard & 2) {
#pragma omp parallel for schedule(static)
    for (int k = nm0; k <= s.kmax - nm0; ++k)
      for (int j = nm0; j <= s.jmax - nm0; ++j)
        for (int i = nm0; i <= s.imax - nm0; ++i)
          for (int d = 1; d <= 3; ++d) s.ww[s.w(d, 6 + d, i, j, k)] = 0.0;
  }
  if (s.p.ict == 1) fluxct(s);
  else if (s.p.ict == 2) mflct(s);
  else if (s.p.ict == 3) upflct(s);
}

// calsf.f90:6-151 (T^m_n at the cell and S_nu = sqrt(-g) T^m_n Gamma^n_{nu m}).
// The step computes it on the interior only, the only cells that read sf
// (rkt.f90); every_cell covers the reference's whole loop range.
void calsf_all(State& s, bool every_cell) {
  const double gam = s.p.gam;
  const int lo = every_cell ? 0 : s.nm1;
#pragma omp parallel for schedule(static)
  for (int k = lo + 1; k <= s.kmax - lo; ++k)
    for (int j = lo + 1; j <= s.jmax - lo; ++j)
      for (int i = lo + 1; i <= s.imax - lo; ++i) {
        const size_t q = s.ik(i, k);
        PS ps;
        pstate(&s.uri[s.a(1, i, j, k)], s.gcov[q], s.gcon[q], gam, ps);
        double t[4][4];  // t[m][n] = T^m_n
        const double a = ps.roh + ps.bbsq, b = ps.pr + 0.5 * ps.bbsq;
        for (int n = 0; n < 4; ++n)
          for (int m = 0; m < 4; ++m)
            t[m][n] = a * ps.ucon[m] * ps.ucov[n] + b * (m == n ? 1.0 : 0.0) - ps.bbcon[m] * ps.bbcov[n];
        const double* ch = &s.christ[q * 64];
        auto G = [&](int l, int m, int n) { return ch[l + 4 * m + 16 * n]; };
        double ta = 0, tb = 0, tc = 0, td = 0;
        for (int n = 0; n < 4; ++n)
          for (int m = 0; m < 4; ++m) {
            ta = ta + t[m][n] * G(n, 1, m);
            tb = tb + t[m][n] * G(n, 2, m);
            tc = tc + t[m][n] * G(n, 3, m);
            td = td + t[m][n] * G(n, 0, m);
          }
        double* o = &s.sf[4 * s.cell(i, j, k)];
        o[0] = s.detg[q] * ta;
        o[1] = s.detg[q] * tb;
        o[2] = s.detg[q] * tc;
        o[3] = s.detg[q] * td;
      }
}

// rkt.f90:2-320: rk2fst/rk3snd/rk3trd plus rk2adsff/rk3adsfs/rk3adsft.
// akap?b(i) = dt/dx?b(i) (main.f90:766-779); (1./3.) and (2./3.) are
// single-precision literals in the reference.
void rkstage(State& s, int stage) {
  const int nm1 = s.nm1;
  const double dt = s.dt;
  const double third = sp(1.0f / 3.0f), twothird = sp(2.0f / 3.0f);
  std::vector<double>& out = (stage == 1) ? s.uh : (stage == 2 ? s.us : s.un);
#pragma omp parallel for schedule(static)
  for (int k = nm1 + 1; k <= s.kmax - nm1; ++k)
    for (int j = nm1 + 1; j <= s.jmax - nm1; ++j)
      for (int i = nm1 + 1; i <= s.imax - nm1; ++i) {
        const double a1 = dt / s.dx1b[i], a2 = dt / s.dx2b[j], a3 = dt / s.dx3b[k];
        for (int m = 1; m <= NV; ++m) {
          const double d1 = s.ww[s.w(1, m, i, j, k)] - s.ww[s.w(1, m, i - 1, j, k)];
          const double d2 = s.ww[s.w(2, m, i, j, k)] - s.ww[s.w(2, m, i, j - 1, k)];
          const double d3 = s.ww[s.w(3, m, i, j, k)] - s.ww[s.w(3, m, i, j, k - 1)];
          const size_t o = s.a(m, i, j, k);
          if (stage == 1) {
            out[o] = s.uu[o] - a1 * d1 - a2 * d2 - a3 * d3;
          } else if (stage == 2) {
            out[o] = (3.0 * s.uo[o] + s.uh[o]) * 0.25 + (-(a1 * d1) - a2 * d2 - a3 * d3) * 0.25;
          } else {
            out[o] = (s.uo[o] + 2. * s.us[o]) * third + (-(a1 * d1) - a2 * d2 - a3 * d3) * twothird;
          }
        }
        const double* f = &s.sf[4 * s.cell(i, j, k)];
        for (int m = 2; m <= 5; ++m) {
          const size_t o = s.a(m, i, j, k);
          if (stage == 1) out[o] = out[o] + f[m - 2] * dt;
          else if (stage == 2) out[o] = out[o] + f[m - 2] * dt * 0.25;
          else out[o] = out[o] + f[m - 2] * dt * twothird;
        }
      }
}

// ------------------------------------------------------------------ recov1a
namespace {

constexpr int kRescaleCap = 1000;  // the reference's "go to 95" loop is unbounded

struct RecovResult {
  double wg_final;
  bool nr2, fail, cap;
};

// recov.f90:578-1228, one interior cell.  Returns false without touching the
// cell when both roots of the W quadratic are negative and no carried-in W
// was supplied (the reference then reuses the last cell's W, recov.f90:810-815).
bool recov_cell(const State& s, double* u, double* q, const M4& g, const M4& gc, double detg1,
                double x1i, const double* wg_carry, RecovResult& res) {
  const double gam = s.p.gam;
  const int iter = s.p.iter;
  const double safty = 1.0e-4, saftybig = 1.0e5, dv = 1.0e-2;
  const double gam1 = gam / (gam - 1.0), gam2 = 1.0 / gam1;
  double delta = 1.0, deltaend = 1.e-7;
  int irecov = 0;
  const double alpha1 = 1. / std::sqrt(-gc.a[0][0]);
  const double dro = alpha1 * u[0] * (1. / detg1);
  double qcov[4], qcon[4], bcon[4], bcov[4], oncov[4], oncon[4];
  qcov[0] = alpha1 * (u[4] - u[0]) * (1. / detg1);
  qcov[1] = alpha1 * u[1] * (1. / detg1);
  qcov[2] = alpha1 * u[2] * (1. / detg1);
  qcov[3] = alpha1 * u[3] * (1. / detg1);
  const double gss = alpha1 * u[5] * (1. / detg1);
  bcon[0] = 0.0;
  bcon[1] = alpha1 * u[6] * (1. / detg1);
  bcon[2] = alpha1 * u[7] * (1. / detg1);
  bcon[3] = alpha1 * u[8] * (1. / detg1);
  double ro = q[0];
  double util[4] = {0.0, q[1], q[2], q[3]};
  double pp = q[4];
  const double ro1 = q[0], pp1 = q[4];
  const double util1[4] = {0.0, q[1], q[2], q[3]};
  lower(bcon, bcov, g);
  upper(qcov, qcon, gc);
  const double bsq = bcon[1] * bcov[1] + bcon[2] * bcov[2] + bcon[3] * bcov[3];
  const double qdotb = qcov[0] * bcon[0] + qcov[1] * bcon[1] + qcov[2] * bcon[2] + qcov[3] * bcon[3];
  const double qdotbsq = qdotb * qdotb;
  oncov[0] = -1.0 * alpha1; oncov[1] = 0.0; oncov[2] = 0.0; oncov[3] = 0.0;
  upper(oncov, oncon, gc);
  const double qdotn = qcon[0] * oncov[0];
  const double qsq = qcov[0] * qcon[0] + qcov[1] * qcon[1] + qcov[2] * qcon[2] + qcov[3] * qcon[3];
  const double qtsq = qsq + (qdotn * qdotn);
  double utsq = 0.0;
  for (int m = 1; m <= 3; ++m)
    for (int n = 1; n <= 3; ++n) utsq = utsq + g.a[m][n] * util[m] * util[n];
  if (utsq < 0.0 && std::fabs(utsq) <= safty) utsq = std::fabs(utsq);
  if (std::fabs(utsq) > 1.e4) utsq = 1.e4;
  double gfsq = 1. + utsq;
  double gf = std::sqrt(gfsq);
  double vsq = (gfsq - 1.) * (1. / gfsq);
  const double vsq1 = vsq;
  const double tmp1a = 4. - vsq1;
  const double tmp1b = 4. * (bsq + qdotn);
  const double tmp1c = qtsq + bsq * bsq + 2. * bsq * qdotn;
  double tmp1d = (tmp1b * tmp1b) - 4. * tmp1a * tmp1c;
  if (tmp1d <= 0.0) tmp1d = std::fabs(tmp1d);
  const double wgp = (-tmp1b + std::sqrt(tmp1d)) * (1. / (2. * tmp1a));
  const double wgm = (-tmp1b - std::sqrt(tmp1d)) * (1. / (2. * tmp1a));
  double wg;
  if (wgp > 0.0) wg = wgp;
  else if (wgm >= 0.0) wg = wgm;
  else {
    if (!wg_carry) return false;
    wg = *wg_carry;
  }
  // "Make sure that W is large enough so that v^2 < 1" (recov.f90:823-850)
  bool cap = false;
  for (int cnt = 0;; ++cnt) {
    if (cnt >= kRescaleCap) { cap = true; break; }
    pp = gam2 * (wg * gf - dro * std::sqrt(gf));
    const double tmp3a = (wg * wg * wg) * (wg + 2. * bsq) - qdotbsq * (2. * wg + bsq);
    const double tmp3b = (wg * wg) * (qtsq - bsq * bsq);
    const double tmp3c = (wg * wg * wg) + (wg * wg) * (0.5 * bsq + qdotn - pp) - 0.5 * qdotbsq;
    if (tmp3a <= tmp3b) { wg = std::fabs(1.5 * wg); continue; }
    if (tmp3c > 0.0) { wg = std::fabs(sp(0.9f) * wg); continue; }
    break;
  }
  if (!cap) {
    double wsq = wg * wg;
    const double xsq = (bsq + wg) * (bsq + wg);
    vsq = std::fabs((wsq * qtsq + qdotbsq * (bsq + 2. * wg)) * (1. / (wsq * xsq)));
    if (vsq > 1.0) vsq = 1.0 - dv;
    const double vsqo = vsq;
    double xxn = wg, yyn = vsq;
    // 2D Newton-Raphson on (W, v^2) (recov.f90:877-960)
    for (int nnn = 1; nnn <= iter; ++nnn) {
      if (!(std::fabs(delta) >= deltaend && irecov == 0)) break;
      if (nnn == iter) { irecov = 1; break; }
      wg = xxn;
      vsq = yyn;
      wsq = wg * wg;
      const double w3 = wsq * wg;
      double gtmp = 1. - vsq;
      if (gtmp < 0.0 || gtmp < safty) { gtmp = safty; vsq = 1. - gtmp; }
      const double ptmp = gam2 * (wg * gtmp - dro * std::sqrt(gtmp));
      const double f1 = qtsq - vsq * (wg + bsq) * (wg + bsq) + (qdotbsq * (bsq + 2. * wg)) * (1. / wsq);
      const double g1 = -qdotn - 0.5 * bsq * (1. + vsq) + 0.5 * (qdotbsq * (1. / wsq)) - wg + ptmp;
      const double dpdw = gam2 * gtmp;
      const double dpdvsq = -(gam2 * wg) + 0.5 * gam2 * dro * (1. / (std::sqrt(gtmp)));
      const double dfx = -(2. * (wg + bsq) * (vsq + qdotbsq * (1. / w3)));
      const double dfy = -((wg + bsq) * (wg + bsq));
      const double dgx = -1. - (qdotbsq * (1. / w3)) + dpdw;
      const double dgy = -(0.5 * bsq) + dpdvsq;
      double det = dfx * dgy - dfy * dgx;
      if (det == 0.0) det = 1.0;
      const double dx = (-(dgy * f1) + dfy * g1) * (1. / det);
      const double dy = (dgx * f1 - dfx * g1) * (1. / det);
      delta = 0.5 * (std::fabs(dx) + std::fabs(dy));
      xxn = wg + dx;
      yyn = vsq + dy;
      if (xxn < 0.0) xxn = std::fabs(xxn);
      if (xxn > saftybig) xxn = saftybig;
      if (yyn < 0.0) yyn = std::fabs(yyn);
      if (std::fabs(yyn) > 1.0) yyn = 1.0 - dv;
    }
    if (irecov == 0) {
      wg = xxn;
      vsq = yyn;
      double gtmp = 1. - vsq;
      if (gtmp < 0.0 || gtmp < safty) { gtmp = safty; vsq = 1. - gtmp; }
      gf = 1. / std::sqrt(gtmp);
      ro = dro * (1. / gf);
      const double w2 = wg * (gtmp);
      pp = gam2 * (w2 - ro);
      if (ro < 0.0 || pp < 0.0) irecov = 1;
      if (irecov == 0) {
        for (int m = 1; m <= 3; ++m) {
          const double qt = qcon[m] + oncon[m] * qdotn;
          util[m] = (gf * (1. / (wg + bsq))) * (qt + qdotb * bcon[m] * (1. / wg));
        }
      }
      wg = xxn;
      vsq = yyn;
    }
    // entropy-based 1D Newton-Raphson on v^2 (recov.f90:1022-1147)
    if (irecov == 1) {
      res.nr2 = true;
      delta = 1.0;
      deltaend = 1.e-6;
      irecov = 0;
      xxn = vsqo;
      for (int nnn = 1; nnn <= iter; ++nnn) {
        if (!(std::fabs(delta) >= deltaend && irecov == 0)) break;
        if (nnn == iter) { irecov = 1; break; }
        vsq = xxn;
        double gtmp = 1. - vsq;
        if (gtmp < 0.0 || gtmp < safty) { gtmp = safty; vsq = 1. - gtmp; }
        gf = 1. / std::sqrt(gtmp);
        gfsq = gf * gf;
        ro = dro * (1. / gf);
        pp = (gss / dro) * fpow(ro, gam);
        const double roh = ro + gam1 * pp;
        wg = std::fabs(gfsq * roh);
        wsq = wg * wg;
        const double w3 = wsq * wg;
        const double dgfdvsq = 0.5 * fpow(gtmp, -1.5);
        const double dwdvsq = dro * dgfdvsq + gam1 * gss * fpow(dro, gam - 1.) * (2. - gam) *
                                                  fpow(gf, 1. - gam) * dgfdvsq;
        const double f = qtsq - vsq * (wg + bsq) * (wg + bsq) + (qdotbsq * (bsq + 2. * wg)) / wsq;
        const double ta = -((wg + bsq) * (wg + bsq));
        const double tb = -(2. * vsq * (wg + bsq));
        const double tc = -(2. * qdotbsq * (bsq + 2. * wg) * (1. / w3));
        const double td = 2. * qdotbsq * (1. / wsq);
        const double df = ta + (tb + tc + td) * dwdvsq;
        delta = f / df;
        xxn = vsq - delta;
        if (xxn < 0.0) xxn = std::fabs(xxn);
        if (std::fabs(xxn) >= 1.0) xxn = 1. - dv;
      }
      if (irecov == 0) {
        vsq = xxn;
        double gtmp = 1. - vsq;
        if (gtmp < 0.0 || gtmp < safty) gtmp = safty;
        gf = 1. / std::sqrt(gtmp);
        gfsq = gf * gf;
        ro = dro * (1. / gf);
        pp = (gss * (1. / gf)) * fpow(ro, gam - 1.);
        if (ro < 0.0) ro = s.p.dmin * fpow(x1i, -1.5);
        if (pp < 0.0) pp = (gam - 1.) * s.p.pmin * fpow(x1i, -2.5);
        const double roh = ro + gam1 * pp;
        wg = std::fabs(gfsq * roh);
        for (int m = 1; m <= 3; ++m) {
          const double qt = qcon[m] + oncon[m] * qdotn;
          util[m] = (gf / (wg + bsq)) * (qt + qdotb * bcon[m] * (1. / wg));
        }
      }
    }
  } else {
    irecov = 1;
  }
  res.cap = cap;
  res.fail = (irecov != 0);
  res.wg_final = wg;
  // set primitives (recov.f90:1174-1216)
  double ucon[4];
  if (irecov == 0) {
    q[0] = ro; q[1] = util[1]; q[2] = util[2]; q[3] = util[3]; q[4] = pp;
    q[5] = ro * pp / fpow(ro, gam - 1.);
    q[6] = u[6] * (1. / detg1); q[7] = u[7] * (1. / detg1); q[8] = u[8] * (1. / detg1);
    calucon(util, ucon, gf, gc);
    u[5] = detg1 * q[5] * ucon[0];
  } else {
    q[0] = ro1; q[1] = util1[1]; q[2] = util1[2]; q[3] = util1[3]; q[4] = pp1;
    q[5] = ro1 * pp1 / fpow(ro1, gam);
    q[6] = u[6] * (1. / detg1); q[7] = u[7] * (1. / detg1); q[8] = u[8] * (1. / detg1);
    calucon(util, ucon, gf, gc);
    u[5] = detg1 * ro1 * q[5] * ucon[0];
  }
  return true;
}

}  // namespace

namespace {
// recov.f90:1919-2456 (recov2, Mignone & McKinney 2007: one-variable
// Newton-Raphson on W' = W - D, gamma-law EoS), one interior cell, with the
// reference's own choices kept: D = alpha uu(1) / detg (a division where the
// other terms multiply by 1/detg), u~^2 < 0 beyond the tolerance reset to
// 1e4, the "make sure v^2 < 1" pressure p = (W gamma - D sqrt(gamma)) (gam-1)/gam,
// and p/rho^(gam-1) for uri(6).  As in recov1a the first guess of W is the
// previous cell's final W when the quadratic has no non-negative root (the
// caller supplies it, or the cell is reported pending), and the unbounded
// rescale loop (go to 95) is capped, a capped cell keeping its primitives.
bool recov2_cell(const State& s, const double* u, double* q, const M4& g, const M4& gc, double detg1,
                 double x1i, const double* wg_carry, RecovResult& res) {
  const double gam = s.p.gam;
  const int iter = s.p.iter;
  const double safty = 1.0e-5, dv = 1.0e-4;
  const double gam1 = gam / (gam - 1.0), gam2 = 1.0 / gam1;
  double delta = 1.0;
  const double deltaend = 1.e-8;
  int irecov = 0;
  const double alpha1 = 1. / std::sqrt(-gc.a[0][0]);
  const double dro = alpha1 * u[0] / detg1;
  double qcov[4], qcon[4], bcon[4], bcov[4], oncov[4], oncon[4];
  qcov[0] = alpha1 * (u[4] - u[0]) * (1. / detg1);
  qcov[1] = alpha1 * u[1] * (1. / detg1);
  qcov[2] = alpha1 * u[2] * (1. / detg1);
  qcov[3] = alpha1 * u[3] * (1. / detg1);
  bcon[0] = 0.0;
  bcon[1] = alpha1 * u[6] * (1. / detg1);
  bcon[2] = alpha1 * u[7] * (1. / detg1);
  bcon[3] = alpha1 * u[8] * (1. / detg1);
  double ro = q[0], pp = q[4];
  double util[4] = {0.0, q[1], q[2], q[3]};
  const double ro1 = q[0], pp1 = q[4];
  const double util1[4] = {0.0, q[1], q[2], q[3]};
  lower(bcon, bcov, g);
  upper(qcov, qcon, gc);
  const double bsq = bcon[1] * bcov[1] + bcon[2] * bcov[2] + bcon[3] * bcov[3];
  const double qdotb = qcov[0] * bcon[0] + qcov[1] * bcon[1] + qcov[2] * bcon[2] + qcov[3] * bcon[3];
  const double qdotbsq = qdotb * qdotb;
  oncov[0] = -1.0 * alpha1; oncov[1] = 0.0; oncov[2] = 0.0; oncov[3] = 0.0;
  upper(oncov, oncon, gc);
  const double qdotn = qcon[0] * oncov[0];
  const double qsq = qcov[0] * qcon[0] + qcov[1] * qcon[1] + qcov[2] * qcon[2] + qcov[3] * qcon[3];
  const double qtsq = qsq + (qdotn * qdotn);
  double utsq = 0.0;
  for (int m = 1; m <= 3; ++m)
    for (int n = 1; n <= 3; ++n) utsq = utsq + g.a[m][n] * util[m] * util[n];
  if (utsq < 0.0 && std::fabs(utsq) <= safty) utsq = std::fabs(utsq);
  if (utsq < 0.0 || std::fabs(utsq) > 1.e4) utsq = 1.e4;
  double gfsq = 1. + utsq;
  double gf = std::sqrt(gfsq);
  double vsq = (gfsq - 1.) * (1. / gfsq);
  const double tmp1a = 4. - vsq;
  const double tmp1b = 4. * (bsq + qdotn);
  const double tmp1c = qtsq + bsq * bsq + 2. * bsq * qdotn;
  double tmp1d = (tmp1b * tmp1b) - 4. * tmp1a * tmp1c;
  if (tmp1d <= 0.0) tmp1d = std::fabs(tmp1d);
  const double wgp = (-tmp1b + std::sqrt(tmp1d)) * (1. / (2. * tmp1a));
  const double wgm = (-tmp1b - std::sqrt(tmp1d)) * (1. / (2. * tmp1a));
  double wg;
  if (wgp > 0.0) wg = wgp;
  else if (wgm >= 0.0) wg = wgm;
  else {
    if (!wg_carry) return false;
    wg = *wg_carry;
  }
  bool cap = false;
  for (int cnt = 0;; ++cnt) {  // recov.f90:2147-2169
    if (cnt >= kRescaleCap) { cap = true; break; }
    pp = gam2 * (wg * gf - dro * std::sqrt(gf));
    const double tmp3a = (wg * wg * wg) * (wg + 2. * bsq) - qdotbsq * (2. * wg + bsq);
    const double tmp3b = (wg * wg) * (qtsq - bsq * bsq);
    const double tmp3c = (wg * wg * wg) + (wg * wg) * (0.5 * bsq + qdotn - pp) - 0.5 * qdotbsq;
    if (tmp3a <= tmp3b) { wg = std::fabs(1.5 * wg); continue; }
    if (tmp3c > 0.0) { wg = std::fabs(sp(0.9f) * wg); continue; }
    break;
  }
  if (cap) irecov = 1;
  // Newton-Raphson on W' (recov.f90:2174-2306)
  double wgd = wg - dro;
  double xxn = wgd;
  for (int nnn = 1; nnn <= iter; ++nnn) {
    if (!(std::fabs(delta) >= deltaend && irecov == 0)) continue;
    if (nnn == iter) { irecov = 1; continue; }
    wgd = xxn;
    wg = wgd + dro;
    const double wsq = wg * wg, w3 = wsq * wg, xsq = (bsq + wg) * (bsq + wg);
    vsq = std::fabs((wsq * qtsq + qdotbsq * (bsq + 2. * wg)) * (1. / (wsq * xsq)));
    if (std::fabs(vsq) > 1.0) vsq = 1.0 - dv;
    if (vsq < 0.0) vsq = std::fabs(vsq);
    double gtmp = 1. - vsq;
    if (gtmp < 0.0 || gtmp < safty) { gtmp = safty; vsq = 1. - gtmp; }
    const double usq = (1. - gtmp) / (gtmp);
    gf = std::sqrt(1. + usq);
    gfsq = gf * gf;
    ro = dro / gf;
    const double xi = (wg - dro * gf) * (1. / gfsq);
    pp = gam2 * xi;
    const double dpdxi = gam2, dpdro = 0.0;
    const double ta = (bsq + wg);
    const double tb = (bsq + wg) * (bsq + wg) * (bsq + wg);
    const double tc = (qtsq == 0.0) ? 0.0 : -2. * qtsq * (1. / tb);
    const double td = (qdotbsq == 0.0) ? 0.0 : -2. * qdotbsq * (3. * wg * ta + bsq * bsq) * (1. / (tb * w3));
    const double dvdwd = tc + td;
    const double dxidwd = (1. / gfsq) - 0.5 * gf * (dro + 2. * gf * xi) * dvdwd;
    const double drodwd = -0.5 * dro * gf * dvdwd;
    const double dpdwd = dpdxi * dxidwd + dpdro * drodwd;
    const double t5a = bsq * qtsq - qdotbsq;
    const double t5b = bsq + wgd + dro;
    double t5c = 0.0, t5d = 0.0;
    if (t5a != 0.0) {
      t5c = 0.5 * t5a * (1. / (t5b * t5b));
      t5d = t5a * (1. / (t5b * t5b * t5b));
    }
    const double f = -(qdotn + dro) - wgd + pp - 0.5 * bsq - t5c;
    const double df = -1. + dpdwd + t5d;
    delta = f / df;
    xxn = wgd - delta;
    if (xxn < 0.0) xxn = std::fabs(xxn);
    if (xxn > 1.e8) xxn = 1.e8;
  }
  if (irecov == 0) {  // recov.f90:2310-2377
    wgd = xxn;
    wg = wgd + dro;
    const double wsq = wg * wg, xsq = (bsq + wg) * (bsq + wg);
    vsq = std::fabs((wsq * qtsq + qdotbsq * (bsq + 2. * wg)) * (1. / (wsq * xsq)));
    if (vsq < 0.0) vsq = std::fabs(vsq);
    if (vsq > 1.0) vsq = 1.0 - dv;
    double gtmp = 1. - vsq;
    if (gtmp < safty) gtmp = safty;
    const double usq = (1. - gtmp) / gtmp;
    gf = std::sqrt(1. + usq);
    gfsq = gf * gf;
    ro = dro / gf;
    const double xi = wg * (1. / gfsq) - ro;
    pp = gam2 * xi;
    if (ro < 0.0) ro = s.p.dmin * fpow(x1i, -3. / 2.);
    if (pp < 0.0) pp = s.p.pmin * (gam - 1.) * fpow(x1i, -5. / 2.);
    for (int a = 1; a <= 3; ++a) {
      const double qt = qcon[a] + oncon[a] * qdotn;
      util[a] = (gf * (1. / (wg + bsq))) * (qt + qdotb * bcon[a] * (1. / wg));
    }
  }
  res.nr2 = false;
  res.cap = cap;
  res.fail = (irecov != 0);
  res.wg_final = wg;
  // recov.f90:2407-2441
  if (irecov == 0) {
    q[0] = ro; q[1] = util[1]; q[2] = util[2]; q[3] = util[3]; q[4] = pp;
    q[5] = pp / fpow(ro, gam - 1.);
  } else {
    q[0] = ro1; q[1] = util1[1]; q[2] = util1[2]; q[3] = util1[3]; q[4] = pp1;
    q[5] = pp1 / fpow(ro1, gam - 1.);
  }
  q[6] = u[6] * (1. / detg1); q[7] = u[7] * (1. / detg1); q[8] = u[8] * (1. / detg1);
  return true;
}
}  // namespace

// recov.f90:1919-2456 over the interior, with recov1a's treatment of the
// loop-order W carry (cells without a root redone in loop order).
void recov2(State& s, std::vector<double>& uu) {
  const int nm1 = s.nm1;
  const int i0 = nm1 + 1, i1 = s.imax - nm1, j0 = nm1 + 1, j1 = s.jmax - nm1, k0 = nm1 + 1, k1 = s.kmax - nm1;
  const int ni = i1 - i0 + 1, nj = j1 - j0 + 1, nk = k1 - k0 + 1;
  if (ni <= 0 || nj <= 0 || nk <= 0) return;
  const size_t nint = (size_t)ni * nj * nk;
  std::vector<double> wgfin(nint, 0.0);
  std::vector<unsigned char> pending(nint, 0);
  long long c_fail = 0, c_cap = 0;
  auto lin = [&](int i, int j, int k) { return (size_t)(i - i0) + (size_t)ni * ((size_t)(j - j0) + (size_t)nj * (k - k0)); };
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : c_fail, c_cap)
  for (int k = k0; k <= k1; ++k)
    for (int j = j0; j <= j1; ++j)
      for (int i = i0; i <= i1; ++i) {
        const size_t q = s.ik(i, k);
        RecovResult r{0, false, false, false};
        if (!recov2_cell(s, &uu[s.a(1, i, j, k)], &s.uri[s.a(1, i, j, k)], s.gcov[q], s.gcon[q], s.detg[q], s.x1[i],
                         nullptr, r)) {
          pending[lin(i, j, k)] = 1;
          continue;
        }
        wgfin[lin(i, j, k)] = r.wg_final;
        c_fail += r.fail; c_cap += r.cap;
      }
  long long c_carry = 0;
  for (size_t l = 0; l < nint; ++l) {
    if (!pending[l]) continue;
    const int i = i0 + (int)(l % ni), j = j0 + (int)((l / ni) % nj), k = k0 + (int)(l / ((size_t)ni * nj));
    const double wprev = (l == 0) ? 0.0 : wgfin[l - 1];
    const size_t q = s.ik(i, k);
    RecovResult r{0, false, false, false};
    recov2_cell(s, &uu[s.a(1, i, j, k)], &s.uri[s.a(1, i, j, k)], s.gcov[q], s.gcon[q], s.detg[q], s.x1[i], &wprev, r);
    wgfin[l] = r.wg_final;
    c_fail += r.fail; c_cap += r.cap;
    ++c_carry;
  }
  s.st.recov_calls += (long long)nint;
  s.st.recov_fail += c_fail;
  s.st.recov_cap += c_cap;
  s.st.recov_carry += c_carry;
}

void recov(State& s, std::vector<double>& uu) {
  if (s.p.iwvec == 2) recov2(s, uu);
  else recov1a(s, uu);
}

// recov.f90:578-1228 over the interior.  The reference carries W from one cell
// to the next in loop order when the quadratic has no non-negative root; the
// cells are computed in parallel first and those few cells are then redone
// in loop order with the previous cell's final W, which reproduces the
// sequential result exactly.  The first cell of a sweep starts from W = 0 as
// in the reference, where the rescale loop then never ends; here it is capped.
void recov1a(State& s, std::vector<double>& uu) {
  const int nm1 = s.nm1;
  const int i0 = nm1 + 1, i1 = s.imax - nm1, j0 = nm1 + 1, j1 = s.jmax - nm1, k0 = nm1 + 1, k1 = s.kmax - nm1;
  const int ni = i1 - i0 + 1, nj = j1 - j0 + 1, nk = k1 - k0 + 1;
  if (ni <= 0 || nj <= 0 || nk <= 0) return;
  const size_t nint = (size_t)ni * nj * nk;
  std::vector<double> wgfin(nint, 0.0);
  std::vector<unsigned char> pending(nint, 0);
  long long c_nr2 = 0, c_fail = 0, c_cap = 0;
  auto lin = [&](int i, int j, int k) { return (size_t)(i - i0) + (size_t)ni * ((size_t)(j - j0) + (size_t)nj * (k - k0)); };
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : c_nr2, c_fail, c_cap)
  for (int k = k0; k <= k1; ++k)
    for (int j = j0; j <= j1; ++j)
      for (int i = i0; i <= i1; ++i) {
        const size_t q = s.ik(i, k);
        RecovResult r{0, false, false, false};
        const bool ok = recov_cell(s, &uu[s.a(1, i, j, k)], &s.uri[s.a(1, i, j, k)], s.gcov[q], s.gcon[q],
                                   s.detg[q], s.x1[i], nullptr, r);
        if (!ok) { pending[lin(i, j, k)] = 1; continue; }
        wgfin[lin(i, j, k)] = r.wg_final;
        c_nr2 += r.nr2; c_fail += r.fail; c_cap += r.cap;
      }
  long long c_carry = 0;
  for (size_t l = 0; l < nint; ++l) {
    if (!pending[l]) continue;
    const int i = i0 + (int)(l % ni), j = j0 + (int)((l / ni) % nj), k = k0 + (int)(l / ((size_t)ni * nj));
    const double wprev = (l == 0) ? 0.0 : wgfin[l - 1];
    const size_t q = s.ik(i, k);
    RecovResult r{0, false, false, false};
    recov_cell(s, &uu[s.a(1, i, j, k)], &s.uri[s.a(1, i, j, k)], s.gcov[q], s.gcon[q], s.detg[q], s.x1[i],
               &wprev, r);
    wgfin[l] = r.wg_final;
    c_nr2 += r.nr2; c_fail += r.fail; c_cap += r.cap;
    ++c_carry;
  }
  s.st.recov_calls += (long long)nint;
  s.st.recov_nr2 += c_nr2;
  s.st.recov_fail += c_fail;
  s.st.recov_cap += c_cap;
  s.st.recov_carry += c_carry;
}

// ------------------------------------------------------------------- boundaries
// bnd.f90:26-381, single-rank periodic branches (iprocs = jprocs = kprocs = 1)
static void bndpefb4(State& s) {
  const int nm1 = s.nm1, imax = s.imax, jmax = s.jmax, kmax = s.kmax;
  auto& u = s.uri;
  const auto& B = s.p.ibc;
  {
    const int ib0 = 1 + nm1, ib1 = imax - nm1;
    for (int k = 1 + nm1; k <= kmax - nm1; ++k)
      for (int j = 1 + nm1; j <= jmax - nm1; ++j)
        for (int i = 1; i <= nm1; ++i)
          for (int m = 1; m <= NV; ++m)
            if (B[0][m - 1] == 1 || B[1][m - 1] == 1) {
              u[s.a(m, ib0 - i, j, k)] = u[s.a(m, ib1 + 1 - i, j, k)];
              u[s.a(m, ib1 + i, j, k)] = u[s.a(m, ib0 - 1 + i, j, k)];
            }
  }
  {
    const int ib0 = 1 + nm1, ib1 = jmax - nm1;
    for (int k = 1 + nm1; k <= kmax - nm1; ++k)
      for (int j = 1; j <= nm1; ++j)
        for (int i = 1 + nm1; i <= imax - nm1; ++i)
          for (int m = 1; m <= NV; ++m)
            if (B[2][m - 1] == 1 || B[3][m - 1] == 1) {
              u[s.a(m, i, ib0 - j, k)] = u[s.a(m, i, ib1 + 1 - j, k)];
              u[s.a(m, i, ib1 + j, k)] = u[s.a(m, i, ib0 - 1 + j, k)];
            }
  }
  {
    const int ib0 = 1 + nm1, ib1 = kmax - nm1;
    for (int k = 1; k <= nm1; ++k)
      for (int j = 1 + nm1; j <= jmax - nm1; ++j)
        for (int i = 1 + nm1; i <= imax - nm1; ++i)
          for (int m = 1; m <= NV; ++m)
            if (B[4][m - 1] == 1 || B[5][m - 1] == 1) {
              u[s.a(m, i, j, ib0 - k)] = u[s.a(m, i, j, ib1 + 1 - k)];
              u[s.a(m, i, j, ib1 + k)] = u[s.a(m, i, j, ib0 - 1 + k)];
            }
  }
}

// bnd.f90:384-1058 for one direction.  A(n) addresses layer n (1..len) with
// the two transverse indices fixed; uo is urio (the primitives at step start).
template <class Fn>
static void phys_side(int code, bool outer, int nm1, int len, Fn at, const std::vector<double>& uo,
                      std::vector<double>& u, bool x1_18_neg) {
  // at(n) -> flat index of layer n in the current direction for variable m
  if (!outer) {
    switch (code) {
      case 2: for (int n = 1; n <= nm1; ++n) u[at(n)] = uo[at(n)]; break;
      case 3: for (int n = nm1; n >= 1; --n) u[at(n)] = (4.0 * u[at(n + 1)] - u[at(n + 2)]) / 3.0; break;
      case 4: for (int n = nm1; n >= 1; --n) u[at(n)] = 2.0 * u[at(n + 1)] - u[at(n + 2)]; break;
      case 5: for (int n = nm1; n >= 1; --n) u[at(n)] = u[at(1 + nm1)]; break;
      case 12: for (int n = 1; n <= nm1; ++n) u[at(n)] = -u[at(2 * nm1 - n + 1)]; break;
      case 13: for (int n = 1; n <= nm1; ++n) u[at(n)] = 0.0; break;
      case 14: for (int n = 1; n <= nm1; ++n) u[at(n)] = u[at(2 * nm1 - n + 1)]; break;
      case 7:
        for (int n = nm1; n >= 1; --n) u[at(n)] = uo[at(n)] + u[at(n + 1)] - uo[at(n + 1)];
        break;
      default: break;
    }
  } else {
    const int L = len;
    switch (code) {
      case 2: for (int n = 0; n <= nm1 - 1; ++n) u[at(L - n)] = uo[at(L - n)]; break;
      case 3: for (int n = nm1 - 1; n >= 0; --n) u[at(L - n)] = (4.0 * u[at(L - n - 1)] - u[at(L - n - 2)]) / 3.0; break;
      case 4: for (int n = nm1 - 1; n >= 0; --n) u[at(L - n)] = 2.0 * u[at(L - n - 1)] - u[at(L - n - 2)]; break;
      case 5: for (int n = nm1 - 1; n >= 0; --n) u[at(L - n)] = u[at(L - nm1)]; break;
      case 12: for (int n = 0; n <= nm1 - 1; ++n) u[at(L - n)] = -u[at(L - 2 * nm1 + 1 + n)]; break;
      case 13: for (int n = 0; n <= nm1 - 1; ++n) u[at(L - n)] = 0.0; break;
      case 14: for (int n = 0; n <= nm1 - 1; ++n) u[at(L - n)] = u[at(L - 2 * nm1 + 1 + n)]; break;
      case 7:
        for (int n = nm1 - 1; n >= 0; --n) u[at(L - n)] = uo[at(L - n)] + u[at(L - n - 1)] - uo[at(L - n - 1)];
        break;
      case 18:  // x1 outer only (bnd.f90:598-610)
        for (int n = nm1 - 1; n >= 0; --n) u[at(L - n)] = x1_18_neg ? 0.0 : u[at(L - nm1)];
        break;
      default: break;
    }
  }
}

static void bndryfb4(State& s) {
  const int nm1 = s.nm1, imax = s.imax, jmax = s.jmax, kmax = s.kmax;
  auto& u = s.uri;
  const auto& uo = s.urio;
  const auto& B = s.p.ibc;
  for (int m = 1; m <= NV; ++m) {
    for (int k = 1; k <= kmax; ++k)
      for (int j = 1; j <= jmax; ++j) {
        auto at = [&](int n) { return s.a(m, n, j, k); };
        phys_side(B[0][m - 1], false, nm1, imax, at, uo, u, false);
      }
    for (int k = 1; k <= kmax; ++k)
      for (int j = 1; j <= jmax; ++j) {
        auto at = [&](int n) { return s.a(m, n, j, k); };
        const bool neg = u[s.a(2, imax - nm1, j, k)] < 0.0;
        phys_side(B[1][m - 1], true, nm1, imax, at, uo, u, neg);
      }
  }
  for (int m = 1; m <= NV; ++m) {
    for (int k = 1; k <= kmax; ++k)
      for (int i = 1; i <= imax; ++i) {
        auto at = [&](int n) { return s.a(m, i, n, k); };
        phys_side(B[2][m - 1], false, nm1, jmax, at, uo, u, false);
      }
    for (int k = 1; k <= kmax; ++k)
      for (int i = 1; i <= imax; ++i) {
        auto at = [&](int n) { return s.a(m, i, n, k); };
        phys_side(B[3][m - 1] == 18 ? 0 : B[3][m - 1], true, nm1, jmax, at, uo, u, false);
      }
  }
  for (int m = 1; m <= NV; ++m) {
    for (int j = 1; j <= jmax; ++j)
      for (int i = 1; i <= imax; ++i) {
        auto at = [&](int n) { return s.a(m, i, j, n); };
        phys_side(B[4][m - 1], false, nm1, kmax, at, uo, u, false);
      }
    for (int j = 1; j <= jmax; ++j)
      for (int i = 1; i <= imax; ++i) {
        auto at = [&](int n) { return s.a(m, i, j, n); };
        phys_side(B[5][m - 1] == 18 ? 0 : B[5][m - 1], true, nm1, kmax, at, uo, u, false);
      }
  }
}

// bnd.f90:4-23
void bnd4(State& s) {
  bndpefb4(s);
  bndryfb4(s);
}

// bnd.f90:1636-1824 (the inner branch writes nothing and is omitted)
void infchk(State& s) {
  const double gflmax = 10.0;
  const int nm1 = s.nm1, imax = s.imax;
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= s.kmax; ++k)
    for (int j = 1; j <= s.jmax; ++j)
      for (int n = 0; n <= nm1 - 1; ++n) {
        const int i = imax - n;
        double* q = &s.uri[s.a(1, i, j, k)];
        const size_t c = s.ik(i, k);
        const M4& g = s.gcov[c];
        const M4& gc = s.gcon[c];
        const double util[4] = {0.0, q[1], q[2], q[3]};
        double gfl;
        calgfl(util, gfl, g);
        double vel[4] = {0.0, util[1] * (1. / gfl), util[2] * (1. / gfl), util[3] * (1. / gfl)};
        if (vel[1] < 0.0) {
          const double alpha1 = 1. / std::sqrt(-gc.a[0][0]);
          const double b1 = alpha1 * alpha1 * gc.a[0][1];
          vel[1] = b1 * (1. / alpha1);
          double vsq = 0.0;
          for (int m = 1; m <= 3; ++m)
            for (int nn = 1; nn <= 3; ++nn) vsq = vsq + g.a[m][nn] * vel[m] * vel[nn];
          if (vsq >= 1.0) vsq = 1. - 1. / (gflmax * gflmax);
          gfl = 1. / std::sqrt(1. - vsq);
          q[1] = vel[1] * gfl;
          q[2] = vel[2] * gfl;
          q[3] = vel[3] * gfl;
        }
      }
}

// correction.f90:226-447 (all cells; "de<dthe .or. (pr<dthe1 .and. bsq<=1e-20)")
void atmosphere1a(State& s) {
  const double epsilon = 1.e-2, gflmax = 10.0;
  const double gam = s.p.gam;
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= s.kmax; ++k)
    for (int j = 1; j <= s.jmax; ++j)
      for (int i = 1; i <= s.imax; ++i) {
        double* q = &s.uri[s.a(1, i, j, k)];
        const M4& g = s.gcov[s.ik(i, k)];
        const double rr = s.x1[i];
        double de = q[0], pr = q[4];
        double util[4] = {0.0, q[1], q[2], q[3]};
        const double b1 = q[6], b2 = q[7], b3 = q[8];
        const double demin = s.p.dmin * fpow(rr, -1.5);
        const double prmin = (gam - 1.) * s.p.pmin * fpow(rr, -2.5);
        const double dthe = 1.0 * (1. + epsilon) * demin;
        const double dthe1 = 1.0 * (1. + epsilon) * prmin;
        const double bsq = b1 * b1 + b2 * b2 + b3 * b3;
        if (de < dthe || (pr < dthe1 && bsq <= 1.e-20)) {
          de = demin;
          pr = prmin;
          const double vel[4] = {0.0, 0.0, 0.0, 0.0};
          double vsq = 0.0;
          for (int m = 1; m <= 3; ++m)
            for (int n = 1; n <= 3; ++n) vsq = vsq + g.a[m][n] * vel[m] * vel[n];
          if (vsq >= 1.0) vsq = 1. - 1. / (gflmax * gflmax);
          const double gfl = 1. / std::sqrt(1. - vsq);
          util[1] = vel[1] * gfl; util[2] = vel[2] * gfl; util[3] = vel[3] * gfl;
        }
        q[0] = de; q[1] = util[1]; q[2] = util[2]; q[3] = util[3]; q[4] = pr;
        q[5] = 0.0;
      }
}

// correction.f90:744-999.  Only rho is stored when rho changed in the rescale
// loop (the "elseif" at correction.f90:887-893), as in the reference.
void pminmax2b(State& s) {
  const double gflmax = 20.0;
  const double gam = s.p.gam;
  const double f105 = sp(1.05f), f005 = sp(0.05f);
  long long caps = 0;
#pragma omp parallel for schedule(static) reduction(+ : caps)
  for (int k = 1; k <= s.kmax; ++k)
    for (int j = 1; j <= s.jmax; ++j)
      for (int i = 1; i <= s.imax; ++i) {
        double* q = &s.uri[s.a(1, i, j, k)];
        const size_t c = s.ik(i, k);
        const M4& g = s.gcov[c];
        const M4& gc = s.gcon[c];
        const double rr = s.x1[i];
        double de = q[0], pr = q[4];
        double util[4] = {0.0, q[1], q[2], q[3]};
        const double bcon[4] = {0.0, q[6], q[7], q[8]};
        double g3[4][4], gc3[4][4];
        cal3met(g, gc, g3, gc3);
        double gfl;
        calgfl(util, gfl, g);
        const double vel[4] = {0.0, util[1] * (1. / gfl), util[2] * (1. / gfl), util[3] * (1. / gfl)};
        double vsq = 0.0;
        for (int m = 1; m <= 3; ++m)
          for (int n = 1; n <= 3; ++n) vsq = vsq + g3[m][n] * vel[m] * vel[n];
        if (vsq >= 1.0 || gfl > gflmax) vsq = 1. - 1. / (gflmax * gflmax);
        gfl = 1. / std::sqrt(1. - vsq);
        util[1] = vel[1] * gfl; util[2] = vel[2] * gfl; util[3] = vel[3] * gfl;
        calgfl(util, gfl, g);
        double ucon[4], ucov[4], bbcon[4], bbcov[4];
        calucon(util, ucon, gfl, gc);
        lower(ucon, ucov, g);
        calbbcon(bcon, bbcon, ucov, ucon);
        lower(bbcon, bbcov, g);
        const double bbsq = calbbsq(bbcon, bbcov);
        double bcov1[4];
        lower(bcon, bcov1, g);
        const double bsq = bcon[1] * bcov1[1] + bcon[2] * bcov1[2] + bcon[3] * bcov1[3];
        for (int cnt = 0;; ++cnt) {
          if (cnt >= 100000) { ++caps; break; }
          const double roh = de + (gam / (gam - 1.0)) * pr;
          const double tmp1a = roh * gfl * gfl - pr;
          const double tmp1b = std::fabs(f005 * bsq);
          if (tmp1a <= tmp1b) { de = f105 * de; pr = f105 * pr; continue; }
          break;
        }
        if (de != q[0]) q[0] = de;
        else if (pr != q[4]) q[4] = pr;
        const double demin = s.p.dmin * fpow(rr, -1.5);
        const double prmin = (gam - 1.) * s.p.pmin * fpow(rr, -2.5);
        const double bbromax = 50.0, bbprmax = 2.e3, prromax = 1.e6;
        if (pr < prmin) q[4] = prmin;
        if (pr > s.p.pmax) q[4] = s.p.pmax;
        if (de < demin) q[0] = demin;
        const double prro = q[4] * (1. / q[0]);
        if (prro > prromax) q[0] = q[4] / prromax;
        const double bbro = bbsq * (1. / q[0]);
        const double bbpr = bbsq * (1. / q[4]);
        if (bbro > bbromax) q[0] = bbsq / bbromax;
        if (bbpr > bbprmax) q[4] = bbsq / bbprmax;
      }
  s.st.floor_cap += caps;
}

// cdtcfl.f90:2-129 with calcha4 (calcha.f90:129-367); dx? are the dx?b arrays
// (main.f90:753).  The unused vmin sweep is omitted.
double cdtcfl4(State& s) {
  const double gam = s.p.gam, small = 1.e-12;
  const int nm1 = s.nm1;
  const int nmax = nm1 * 2 + (nm1 - 1);
  double dtcfl = 1.0;
#pragma omp parallel for schedule(static) reduction(min : dtcfl)
  for (int k = 2; k <= s.kmax - 1; ++k)
    for (int j = 2; j <= s.jmax - 1; ++j)
      for (int i = 2; i <= s.imax - 1; ++i) {
        const size_t c = s.ik(i, k);
        const double* q = &s.uri[s.a(1, i, j, k)];
        double vp[4], vm[4];
        for (int d = 1; d <= 3; ++d) calcha4d(q, s.gcov[c], s.gcon[c], gam, d, vp[d], vm[d]);
        double vfi = fmax3(0.0, std::fabs(vp[1]), std::fabs(vm[1]));
        double vfj = fmax3(0.0, std::fabs(vp[2]), std::fabs(vm[2]));
        double vfk = fmax3(0.0, std::fabs(vp[3]), std::fabs(vm[3]));
        double d1, d2, d3;
        if (s.imax > nmax && vfi > 0.0) { if (vfi > 1.0) vfi = 1.0; d1 = std::fabs(s.dx1b[i] / (vfi + small)); }
        else d1 = 1.e10;
        if (s.jmax > nmax && vfj > 0.0) { if (vfj > 1.0) vfj = 1.0; d2 = std::fabs(s.dx2b[j] / (vfj + small)); }
        else d2 = 1.e10;
        if (s.kmax > nmax && vfk > 0.0) { if (vfk > 1.0) vfk = 1.0; d3 = std::fabs(s.dx3b[k] / (vfk + small)); }
        else d3 = 1.e10;
        dtcfl = std::min(dtcfl, d1);
        dtcfl = std::min(dtcfl, d2);
        dtcfl = std::min(dtcfl, d3);
      }
  return dtcfl;
}

// main.f90:586-1147: one pass of the time loop (loop-top time update, dt,
// three RK stages).  Output/restart I/O is not part of the hot path.
void step(State& s) {
  s.time = s.timeh;
  s.uo = s.uu;
  s.urio = s.uri;
  s.dtcfl = cdtcfl4(s);
  s.dt = s.p.cfl * s.dtcfl;
  s.timeh = s.time + s.dt;
  const bool torus = (s.p.model >= 7 && s.p.model <= 15);
  const bool inflow = (s.p.model >= 7 && s.p.model <= 20);
  for (int stage = 1; stage <= 3; ++stage) {
    rec2(s);
    calcha(s);
    hlle(s);
    ct(s);
    calsf_all(s);
    rkstage(s, stage);
    std::vector<double>& un = (stage == 1) ? s.uh : (stage == 2 ? s.us : s.un);
    recov(s, un);
    bnd4(s);
    if (inflow) infchk(s);
    if (torus) atmosphere1a(s);
    pminmax2b(s);
    caluu1(s, s.uri, un);
    s.uu = un;
  }
  ++s.it;
}

}  // namespace orc
