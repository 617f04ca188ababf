// Test infrastructure only: the CPU restatement of the output converter's
// per-cell derived quantities (convert_vtk2dn1.f90:254-371, with
// transmks2ks1 / transks2bl1 at convert_vtk2dn1.f90:1399-1554 and its own
// calgfl / calucon / calbbcon / calbbsq / lower at 1158-1331), the oracle for
// rg_run_derived.  The converter re-evaluates the run's metric from the
// coord.f90 formulas; this restatement takes it from the oracle's cell-centre
// metric, which is the same evaluation.
#include <cmath>

#include "oracle.hpp"

namespace orc {

namespace {

// convert_vtk2dn1.f90:1158-1197 (clamp |u~^2| > 1e10 to 1e9)
double conv_calgfl(const double util[3], const M4& g) {
  double utsq = 0.0;
  for (int m = 1; m <= 3; ++m)
    for (int n = 1; n <= 3; ++n) utsq = utsq + g.a[m][n] * util[m - 1] * util[n - 1];
  if (utsq < 0.0) {
    if (std::fabs(utsq) <= 1.0e-10) utsq = std::fabs(utsq);
    else utsq = 1.e-10;
  }
  if (std::fabs(utsq) > 1.0e10) utsq = 1.0e9;
  return std::sqrt(1. + utsq);
}

// convert_vtk2dn1.f90:1200-1233
void conv_calucon(const double util[3], double gfl, const M4& gc, double ucon[4]) {
  const double alpha1 = 1. / std::sqrt(-gc.a[0][0]);
  const double beta1[3] = {alpha1 * alpha1 * gc.a[0][1], alpha1 * alpha1 * gc.a[0][2], alpha1 * alpha1 * gc.a[0][3]};
  ucon[0] = gfl * (1. / alpha1);
  for (int m = 1; m <= 3; ++m) ucon[m] = util[m - 1] - gfl * beta1[m - 1] * (1. / alpha1);
}

// convert_vtk2dn1.f90:1295-1329
void conv_lower(const double v[4], double o[4], const M4& g) {
  for (int m = 0; m < 4; ++m) o[m] = g.a[m][0] * v[0] + g.a[m][1] * v[1] + g.a[m][2] * v[2] + g.a[m][3] * v[3];
}

}  // namespace

void derived(State& s, const std::vector<double>& uri, int jslice, double* out) {
  const orc_params& p = s.p;
  const double akm = p.akm;
  const double rbh1 = 1. + std::sqrt(1. - akm * akm);
  for (int k = 1; k <= s.kmax; ++k)
    for (int j = (jslice ? jslice : 1); j <= (jslice ? jslice : s.jmax); ++j)
      for (int i = 1; i <= s.imax; ++i) {
        // coordinates (convert_vtk2dn1.f90:138-161)
        double rr, th, x1t = 0.0, x3t = 0.0;
        if (p.metric == 403) {
          x1t = s.x1b[i];
          rr = (p.ix1 == 2) ? p.R0 + std::exp(x1t) : x1t;
          x3t = s.x3b[k];
          th = (p.ix3 == 2) ? x3t + 0.5 * (1. - p.hslope) * std::sin(2. * x3t) : x3t;
        } else {
          rr = s.x1[i];
          th = s.x3[k];
        }
        const size_t q = s.ik(i, k);
        const M4& g = s.gcov[q];
        const M4& gc = s.gcon[q];
        double u[9];
        for (int n = 0; n < 9; ++n) u[n] = uri[s.a(n + 1, i, j, k)];
        const double de = u[0], pr = u[4];
        const double roh = de + (p.gam / (p.gam - 1.0)) * pr;
        for (int n = 6; n < 9; ++n)
          if (std::fabs(u[n]) < 1.e-20) u[n] = 0.0;
        const double util[3] = {u[1], u[2], u[3]};
        const double gfl = conv_calgfl(util, g);
        double ucon[4], ucov[4], bbcon[4], bbcov[4];
        conv_calucon(util, gfl, gc, ucon);
        conv_lower(ucon, ucov, g);
        // calbbcon / calbbsq (convert_vtk2dn1.f90:1236-1275)
        bbcon[0] = u[6] * ucov[1] + u[7] * ucov[2] + u[8] * ucov[3];
        for (int m = 1; m <= 3; ++m) bbcon[m] = (u[5 + m] + bbcon[0] * ucon[m]) * (1. / ucon[0]);
        conv_lower(bbcon, bbcov, g);
        const double bbsq = bbcon[0] * bbcov[0] + bbcon[1] * bbcov[1] + bbcon[2] * bbcov[2] + bbcon[3] * bbcov[3];
        double o[7];
        o[2] = bbsq;
        o[3] = -(roh / de) * ucov[0];
        if (rr > rbh1) {
          // transmks2ks1 (convert_vtk2dn1.f90:1524-1554)
          double ut[3] = {util[0], util[1], util[2]};
          if (p.metric == 403) {
            const double rfac = (p.ix1 == 2) ? std::exp(x1t) : 1.0;
            const double hfac = (p.ix3 == 2) ? 1. + (1. - p.hslope) * std::cos(2. * x3t) : 1.0;
            ut[0] = rfac * util[0];
            ut[1] = 1.0 * util[1];
            ut[2] = hfac * util[2];
          }
          // transks2bl1 (convert_vtk2dn1.f90:1399-1521): KS metric at (rr, th)
          const double sth = std::sin(th), cth = std::cos(th);
          const double del = rr * rr - (2. * rr) + akm * akm;
          const double sig = rr * rr + akm * cth * akm * cth;
          const double aa = ((rr * rr + akm * akm) * (rr * rr + akm * akm)) - akm * akm * del * sth * sth;
          M4 kg{}, kc{};
          kg.a[0][0] = -1. + 2. * rr / sig;
          kg.a[0][1] = 2. * rr / sig;
          kg.a[0][2] = -2. * akm * rr * sth * sth / sig;
          kg.a[1][0] = kg.a[0][1];
          kg.a[1][1] = 1. + 2. * rr / sig;
          kg.a[1][2] = -1. * akm * sth * sth * (1. + 2. * rr / sig);
          kg.a[2][0] = kg.a[0][2];
          kg.a[2][1] = kg.a[1][2];
          kg.a[2][2] = aa * sth * sth / sig;
          kg.a[3][3] = sig;
          kc.a[0][0] = -1. - 2. * rr / sig;
          kc.a[0][1] = 2. * rr / sig;
          kc.a[1][0] = kc.a[0][1];
          kc.a[1][1] = del / sig;
          kc.a[1][2] = akm / sig;
          kc.a[2][1] = kc.a[1][2];
          kc.a[2][2] = 1. / (sig * sth * sth);
          kc.a[3][3] = 1. / sig;
          const double gks = conv_calgfl(ut, kg);
          double uks[4];
          conv_calucon(ut, gks, kc, uks);
          double trans[4][4] = {};
          const double tmp2 = rr * rr - (2. * rr) + akm * akm;
          if (tmp2 > 0.0) {
            trans[0][0] = 1.0;
            trans[0][1] = -2. * rr * (1. / tmp2);
            trans[1][1] = 1.0;
            trans[2][2] = 1.0;
            trans[2][1] = -akm * (1. / tmp2);
            trans[3][3] = 1.0;
          }
          double ubl[4] = {0.0, 0.0, 0.0, 0.0};
          for (int n = 0; n < 4; ++n)
            for (int m = 0; m < 4; ++m) ubl[m] = ubl[m] + trans[m][n] * uks[n];
          // BL lapse and shift (convert_vtk2dn1.f90:325-348)
          const double gcon1a00 = -aa / (sig * del);
          const double gcon1a01 = 0.0, gcon1a02 = -(2. * akm * rr) / (sig * del), gcon1a03 = 0.0;
          const double gcov1a00 = -(sig - 2. * rr) / sig;
          const double alpha1 = 1. / std::sqrt(-gcon1a00);
          const double beta1[3] = {alpha1 * alpha1 * gcon1a01, alpha1 * alpha1 * gcon1a02, alpha1 * alpha1 * gcon1a03};
          o[0] = alpha1 * ubl[0];
          o[1] = ubl[0] * std::sqrt(-gcov1a00);
          for (int m = 1; m <= 3; ++m) o[3 + m] = ubl[m] + o[0] * beta1[m - 1] * (1. / alpha1);
        } else {
          o[0] = 1.0; o[1] = 1.0; o[4] = 0.0; o[5] = 0.0; o[6] = 0.0;
        }
        const size_t pt = jslice ? (size_t)(i - 1) + (size_t)s.imax * (size_t)(k - 1)
                                 : (size_t)(i - 1) + (size_t)s.imax * ((size_t)(j - 1) + (size_t)s.jmax * (size_t)(k - 1));
        for (int f = 0; f < 7; ++f) out[7 * pt + f] = o[f];
      }
}

}  // namespace orc
