// rg_geometry.cpp -- host-side setup of one run: the grid of grid.f90, the
// metric cache of coord1 (coord.f90:5-146) and the Christoffel symbols of
// calchrist (coord.f90:1089-1321).  This is init-time work done once per run;
// the arrays are uploaded into the device caches read by the kernels.
#include <cmath>
#include <cstring>

#include "rg_host.h"

namespace rg {

namespace {

constexpr double kPi = 3.14159265358979323;  // pram.f90:30
using Mat = double[4][4];

void zero(Mat m) { std::memset(m, 0, sizeof(double) * 16); }

// Clamp |x| < 1e-12 away from zero keeping its side (coord.f90:556-571).
double clamp_small(double v) {
  const double small = 1.e-12;
  if (std::fabs(v) < small) return (v > 0.0) ? small : -small;
  return v;
}

// Modified Kerr-Schild covariant metric (coord.f90:693-792); with rfac = hfac
// = 1 this is the Kerr-Schild metric of kshcov1 (coord.f90:535-613).
void mks_cov(const rg_run_params& p, Mat g, double r, double th_ks, double th_mks, bool modified) {
  const double a = p.akm;
  const double theta = (th_ks > kPi) ? 2. * kPi - th_ks : th_ks;
  const double sth = clamp_small(std::sin(theta));
  const double s2 = sth * sth;
  const double cth = clamp_small(std::cos(theta));
  const double a2 = a * a, r2 = r * r;
  const double del = r2 - (2. * r) + a2;
  const double sig = r2 + a2 * cth * cth;
  const double aa = ((r2 + a2) * (r2 + a2)) - a2 * del * s2;
  const double rfac = (modified && p.ix1 == 2) ? r : 1.0;
  const double hfac = (modified && p.ix3 == 2) ? 1. + (1. - p.hslope) * std::cos(2. * th_mks) : 1.0;
  zero(g);
  if (modified) {
    g[0][0] = (-1. + 2. * r / sig) * 1.0 * 1.0;
    g[0][1] = (2. * r / sig) * 1.0 * rfac;
    g[0][2] = (-(2. * a * r * s2 * (1. / sig))) * 1.0 * 1.0;
    g[1][1] = (1. + 2. * r / sig) * rfac * rfac;
    g[1][2] = (-(1. * a * s2 * (1. + 2. * r / sig))) * rfac * 1.0;
    g[2][2] = (aa * s2 * (1. / sig)) * 1.0 * 1.0;
    g[3][3] = sig * hfac * hfac;
  } else {
    g[0][0] = -1. + 2. * r / sig;
    g[0][1] = 2. * r / sig;
    g[0][2] = -(2. * a * r * s2 * (1. / sig));
    g[1][1] = 1. + 2. * r / sig;
    g[1][2] = -(1. * a * s2 * (1. + 2. * r / sig));
    g[2][2] = aa * s2 * (1. / sig);
    g[3][3] = sig;
  }
  g[1][0] = g[0][1];
  g[2][0] = g[0][2];
  g[2][1] = g[1][2];
}

// Analytic Kerr-Schild contravariant metric (coord.f90:616-690).
void ks_con(const rg_run_params& p, Mat g, double r, double th) {
  const double a = p.akm;
  const double theta = (th > kPi) ? 2. * kPi - th : th;
  const double sth = clamp_small(std::sin(theta));
  const double s2 = sth * sth;
  const double cth = clamp_small(std::cos(theta));
  const double a2 = a * a, r2 = r * r;
  const double del = r2 - (2. * r) + a2;
  const double sig = r2 + a2 * cth * cth;
  zero(g);
  g[0][0] = -1. - 2. * r / sig;
  g[0][1] = 2. * r / sig;
  g[1][0] = g[0][1];
  g[1][1] = del / sig;
  g[1][2] = a * (1. / sig);
  g[2][1] = g[1][2];
  g[2][2] = 1. / (sig * s2);
  g[3][3] = 1. / sig;
}

void minkowski(Mat g) {
  zero(g);
  g[0][0] = -1.0; g[1][1] = 1.0; g[2][2] = 1.0; g[3][3] = 1.0;
}

// Inverse by Crout LU with implicit pivoting and back substitution, the
// numerics of invert_matrix2/ludcmp/lubksb (coord.f90:1504-1689).  The
// reference's first inner loop starts at row 0 and rewrites a(0,j) with its own
// value, which changes nothing; it starts at row 1 here.
void lu_inverse(const Mat in, Mat out) {
  double a[5][5], vv[5];
  int indx[5];
  for (int r = 1; r <= 4; ++r)
    for (int c = 1; c <= 4; ++c) a[r][c] = in[r - 1][c - 1];
  for (int r = 1; r <= 4; ++r) {
    double big = 0.0;
    for (int c = 1; c <= 4; ++c) big = (std::fabs(a[r][c]) > big) ? std::fabs(a[r][c]) : big;
    vv[r] = 1. / big;
  }
  int piv = 1;
  for (int c = 1; c <= 4; ++c) {
    for (int r = 1; r < c; ++r) {
      double s = a[r][c];
      for (int t = 1; t < r; ++t) s = s - a[r][t] * a[t][c];
      a[r][c] = s;
    }
    double big = 0.0;
    for (int r = c; r <= 4; ++r) {
      double s = a[r][c];
      for (int t = 1; t < c; ++t) s = s - a[r][t] * a[t][c];
      a[r][c] = s;
      const double fig = vv[r] * std::fabs(s);
      if (fig >= big) { piv = r; big = fig; }
    }
    if (c != piv) {
      for (int t = 1; t <= 4; ++t) {
        const double tmp = a[piv][t];
        a[piv][t] = a[c][t];
        a[c][t] = tmp;
      }
      vv[piv] = vv[c];
    }
    indx[c] = piv;
    if (a[c][c] == 0.0) a[c][c] = (double)1.e-20f;
    if (c != 4) {
      const double inv = 1. / a[c][c];
      for (int r = c + 1; r <= 4; ++r) a[r][c] = a[r][c] * inv;
    }
  }
  for (int col = 1; col <= 4; ++col) {
    double b[5];
    for (int r = 1; r <= 4; ++r) b[r] = (r == col) ? 1.0 : 0.0;
    int ii = 0;
    for (int r = 1; r <= 4; ++r) {
      const int ll = indx[r];
      double s = b[ll];
      b[ll] = b[r];
      if (ii != 0) {
        for (int t = ii; t < r; ++t) s = s - a[r][t] * b[t];
      } else if (s != 0) {
        ii = r;
      }
      b[r] = s;
    }
    for (int r = 4; r >= 1; --r) {
      double s = b[r];
      for (int t = r + 1; t <= 4; ++t) s = s - a[r][t] * b[t];
      b[r] = s / a[r][r];
    }
    for (int r = 1; r <= 4; ++r) out[r - 1][col - 1] = b[r];
  }
}

// sqrt(-g) by cofactor expansion along the first column (coord.f90:1016-1086).
double sqrt_minus_det(const Mat g) {
  auto d3 = [](double aa, double bb, double cc, double pp, double qq, double rr, double xx, double yy,
               double zz) {
    return aa * qq * zz + bb * rr * xx + cc * pp * yy - cc * qq * xx - bb * pp * zz - aa * rr * yy;
  };
  const double t1 = d3(g[1][1], g[1][2], g[1][3], g[2][1], g[2][2], g[2][3], g[3][1], g[3][2], g[3][3]);
  const double t2 = d3(g[0][1], g[0][2], g[0][3], g[2][1], g[2][2], g[2][3], g[3][1], g[3][2], g[3][3]);
  const double t3 = d3(g[0][1], g[0][2], g[0][3], g[1][1], g[1][2], g[1][3], g[3][1], g[3][2], g[3][3]);
  const double t4 = d3(g[0][1], g[0][2], g[0][3], g[1][1], g[1][2], g[1][3], g[2][1], g[2][2], g[2][3]);
  return std::sqrt(-1. * (g[0][0] * t1 - g[1][0] * t2 + g[2][0] * t3 - g[3][0] * t4));
}

// Covariant and contravariant metric of the run's coordinates at (r, theta)
// with theta_MKS used by hfac (coord.f90:59-122).
void metric_at(const rg_run_params& p, double r, double th, double th_mks, Mat g, Mat gc) {
  if (p.metric == 1) {
    minkowski(g);
    minkowski(gc);
  } else if (p.metric == 303) {
    mks_cov(p, g, r, th, th_mks, false);
    ks_con(p, gc, r, th);
  } else {
    mks_cov(p, g, r, th, th_mks, true);
    lu_inverse(g, gc);
  }
}

// Compact cache of one point: gcov (t,r,phi) block + g_thth, the full
// (t,r,phi) block of gcon (not symmetric to the last bit) + g^thth, sqrt(-g).
// Returns false if an entry coupling theta to (t,r,phi) is nonzero or gcov is
// not symmetric, which the compact kernels do not represent.
bool store_met(std::vector<double>& dst, size_t nik, size_t q, const Mat g, const Mat gc) {
  const double v[kMetBase] = {g[0][0], g[0][1], g[0][2], g[1][1], g[1][2], g[2][2], g[3][3],
                               gc[0][0], gc[0][1], gc[0][2], gc[1][0], gc[1][1], gc[1][2],
                               gc[2][0], gc[2][1], gc[2][2], gc[3][3], sqrt_minus_det(g)};
  for (int c = 0; c < kMetBase; ++c) dst[(size_t)c * nik + q] = v[c];
  bool ok = g[1][0] == g[0][1] && g[2][0] == g[0][2] && g[2][1] == g[1][2];
  for (int a = 0; a < 3; ++a) ok = ok && g[a][3] == 0.0 && g[3][a] == 0.0 && gc[a][3] == 0.0 && gc[3][a] == 0.0;
  return ok;
}

}  // namespace

// grid.f90:2-266 for one direction.  kind 1 uniform, 2 logarithmic (x1) or
// MKS theta (x3).  "log" and "mks" select the x1 and x3 variants.
static void make_axis(int n, double lo, double hi, int kind, bool is_x1, bool is_x3, bool mks, double R0,
                      double hslope, Axis& ax) {
  ax.x.assign(n + 2, 0.0); ax.xa.assign(n + 2, 0.0); ax.xb.assign(n + 2, 0.0);
  ax.xab.assign(n + 2, 0.0); ax.dx.assign(n + 2, 0.0); ax.dxb.assign(n + 2, 0.0);
  if (kind == 1) {
    for (int i = 1; i <= n; ++i) {
      ax.dx[i] = (hi - lo) / (double)(float)(n - 1);
      ax.x[i] = lo + ax.dx[i] * (double)(float)(i - 1);
      ax.xb[i] = ax.x[i];
    }
  } else if (is_x1) {  // logarithmic r (grid.f90:33-50)
    const double s0 = std::log(lo - R0), s1 = std::log(hi - R0);
    const double ds = (s1 - s0) * (double)(1.0f / (float)(n - 1));
    for (int i = 1; i <= n; ++i) {
      const double s = s0 + (double)(float)(i - 1) * ds;
      ax.x[i] = std::exp(s) + R0;
      ax.xb[i] = s;
    }
    for (int i = 2; i <= n; ++i) ax.dx[i] = mks ? ax.xb[i] - ax.xb[i - 1] : ax.x[i] - ax.x[i - 1];
    ax.dx[1] = ax.dx[2];
  } else if (is_x3) {  // theta(x3) of MKS (grid.f90:195-218)
    const double t0 = lo / kPi, t1 = hi / kPi;
    const double dt = (t1 - t0) / (double)(float)(n - 1);
    for (int k = 1; k <= n; ++k) {
      const double xt = kPi * (t0 + (double)(float)(k - 1) * dt);
      ax.x[k] = xt + 0.5 * (1. - hslope) * std::sin(2. * xt);
      ax.xb[k] = xt;
    }
    for (int k = 2; k <= n; ++k) ax.dx[k] = mks ? ax.xb[k] - ax.xb[k - 1] : ax.x[k] - ax.x[k - 1];
    ax.dx[1] = ax.dx[2];
  }
  for (int i = 1; i <= n - 1; ++i) ax.xa[i] = 0.5 * (ax.x[i] + ax.x[i + 1]);
  ax.xa[n] = ax.xa[n - 1] + ax.dx[n];
  const bool mid_b = mks || (!is_x1 && !is_x3);  // x2ab = x2a (grid.f90:173-176)
  if (mks && (is_x1 || is_x3)) {
    for (int i = 1; i <= n - 1; ++i) ax.xab[i] = 0.5 * (ax.xb[i] + ax.xb[i + 1]);
    ax.xab[n] = ax.xab[n - 1] + ax.dx[n];
  } else if (mid_b) {
    for (int i = 1; i <= n; ++i) ax.xab[i] = ax.xa[i];
  }
  // dx?b(n) is written one past the reference's declared extent (grid.f90:139)
  for (int i = 2; i <= n; ++i) ax.dxb[i] = (mks && (is_x1 || is_x3)) ? ax.xab[i] - ax.xab[i - 1] : ax.xa[i] - ax.xa[i - 1];
  ax.dxb[1] = ax.dxb[2];
}

void build_geometry(const rg_run_params& p, HostGeom& G, int krow) {
  const bool mks = (p.metric == 403);
  make_axis(p.imax, p.xmin, p.xmax, p.ix1, true, false, mks, p.R0, p.hslope, G.ax[0]);
  make_axis(p.jmax, p.ymin, p.ymax, 1, false, false, mks, p.R0, p.hslope, G.ax[1]);
  make_axis(p.kmax, p.zmin, p.zmax, p.ix3, false, true, mks, p.R0, p.hslope, G.ax[2]);
  const int imax = p.imax, kmax = p.kmax;
  // krow > 0: one theta row (a theta slab in Minkowski space, where every row is the same)
  const size_t nik = (size_t)imax * (krow > 0 ? 1 : kmax);
  G.nik = nik;
  G.mc.assign(kMetComps * nik, 0.0);
  G.mi.assign(kMetComps * nik, 0.0);
  G.mk.assign(kMetComps * nik, 0.0);
  G.compact_ok = true;
  G.chr.assign(64 * nik, 0.0);
  const Axis& X1 = G.ax[0];
  const Axis& X3 = G.ax[2];
  // every (i, k) point is independent: OpenMP over points (bit-identical to a serial loop)
  const int k0 = (krow > 0 ? krow : 1), nk = (krow > 0 ? 1 : kmax);
  bool ok = true;
#pragma omp parallel for schedule(static) reduction(&& : ok) if ((long long)nk * imax > 4096)
  for (long long pt = 0; pt < (long long)nk * imax; ++pt) {
      const int k = k0 + (int)(pt / imax), i = 1 + (int)(pt % imax);
      const size_t q = (size_t)(i - 1) + (krow > 0 ? 0 : (size_t)imax * (k - 1));
      Mat g, gc;
      metric_at(p, X1.x[i], X3.x[k], X3.xb[k], g, gc);
      ok = store_met(G.mc, nik, q, g, gc) && ok;
      metric_at(p, X1.xa[i], X3.x[k], X3.xb[k], g, gc);
      ok = store_met(G.mi, nik, q, g, gc) && ok;
      metric_at(p, X1.x[i], X3.xa[k], X3.xb[k], g, gc);  // hfac at the centre theta_MKS (coord.f90:96-98)
      ok = store_met(G.mk, nik, q, g, gc) && ok;
      // Minkowski: the central differences of the constant metric vanish exactly,
      // so every Christoffel symbol is 0 (the array is zero-initialised)
      if (p.metric == 1) continue;
      // Christoffel symbols by central differences, delta = 1e-5 (coord.f90:1134-1317)
      const double delta = 1.0e-5, small = 1.e-12;
      double r0 = X1.x[i], th0 = X3.x[k], thm = X3.xb[k];
      double rp = r0 + delta, rm = r0 - delta, sp = 0, sm = 0;
      double tp = th0 + delta, tm = th0 - delta, tbp = 0, tbm = 0, thm_p = thm, thm_m = thm;
      if (mks) {
        sp = X1.xb[i] + delta; sm = X1.xb[i] - delta;
        rp = (p.ix1 == 1) ? sp : std::exp(sp);
        rm = (p.ix1 == 1) ? sm : std::exp(sm);
        tbp = X3.xb[k] + delta; tbm = X3.xb[k] - delta;
        if (p.ix3 == 1) { tp = tbp; tm = tbm; }
        else {
          tp = tbp + 0.5 * (1. - p.hslope) * std::sin(2. * tbp);
          tm = tbm + 0.5 * (1. - p.hslope) * std::sin(2. * tbm);
        }
        thm_p = tbp; thm_m = tbm;
      }
      Mat gip, gim, gkp, gkm, g0, gcon, dummy;
      metric_at(p, rp, th0, thm, gip, dummy);
      metric_at(p, rm, th0, thm, gim, dummy);
      metric_at(p, r0, tp, thm_p, gkp, dummy);
      metric_at(p, r0, tm, thm_m, gkm, dummy);
      metric_at(p, r0, th0, thm, g0, gcon);
      double dg[4][4][4];  // dg[l][m][n] = g_{lm,n}; phi derivative 0 (metric phi independent)
      for (int m = 0; m < 4; ++m)
        for (int l = 0; l < 4; ++l) {
          dg[l][m][0] = 0.0;
          dg[l][m][1] = mks ? (gip[l][m] - gim[l][m]) / (sp - sm + small) : (gip[l][m] - gim[l][m]) / (rp - rm + small);
          dg[l][m][2] = 0.0 / (2.0 * delta + small);
          dg[l][m][3] = mks ? (gkp[l][m] - gkm[l][m]) / (tbp - tbm + small) : (gkp[l][m] - gkm[l][m]) / (tp - tm + small);
        }
      double low[4][4][4];
      for (int n = 0; n < 4; ++n)
        for (int m = 0; m < 4; ++m)
          for (int l = 0; l < 4; ++l) low[l][m][n] = 0.5 * (dg[m][l][n] + dg[n][l][m] - dg[n][m][l]);
      for (int n = 0; n < 4; ++n)
        for (int m = 0; m < 4; ++m)
          for (int l = 0; l < 4; ++l)
            G.chr[(size_t)(l + 4 * m + 16 * n) * nik + q] = gcon[l][0] * low[0][m][n] + gcon[l][1] * low[1][m][n] +
                                                            gcon[l][2] * low[2][m][n] + gcon[l][3] * low[3][m][n];
    }
  G.compact_ok = ok;
}

}  // namespace rg

// ------------------------------------------------------------ initial data
namespace rg {

namespace {

// Boyer-Lindquist Kerr covariant metric (coord.f90:378-463), IC only.
void bl_cov(double akm, Mat g, double r, double th) {
  const double theta = (th > kPi) ? 2. * kPi - th : th;
  const double sth = clamp_small(std::sin(theta));
  const double s2 = sth * sth;
  const double cth = clamp_small(std::cos(theta));
  const double a2 = akm * akm, r2 = r * r;
  const double del = 1. - (2. / r) + (a2 * (1. / r2));
  const double sig = 1. + a2 * cth * cth * (1. / r2);
  zero(g);
  g[0][0] = -(1. - 2. * (1. / (r * sig)));
  g[0][2] = -(2. * akm * s2 * (1. / (r * sig)));
  g[1][1] = sig / del;
  g[2][0] = g[0][2];
  g[2][2] = r2 * s2 * (1. + (a2 * (1. / r2)) + 2. * a2 * s2 * (1. / (r2 * r * sig)));
  g[3][3] = r2 * sig;
}

// Inverse by the column-pivoted LU of invert_matrix (coord.f90:1324-1501),
// used by the Boyer-Lindquist -> MKS velocity transform.  out(i,j) is the
// j-th entry of the i-th solve, as in the reference.
bool lu_inverse_cols(const Mat in, Mat out) {
  double A[5][5];
  int p[5];
  for (int i = 1; i <= 4; ++i) p[i] = i;
  for (int c = 1; c <= 4; ++c)
    for (int r = 1; r <= 4; ++r) A[r][c] = in[r - 1][c - 1];
  for (int t = 1; t <= 4; ++t) {
    int mj = t;
    for (int c = t + 1; c <= 4; ++c)
      if (std::fabs(A[t][c]) > std::fabs(A[t][mj])) mj = c;
    if (mj != t) {
      for (int r = 1; r <= 4; ++r) { const double x = A[r][mj]; A[r][mj] = A[r][t]; A[r][t] = x; }
      const int x = p[mj]; p[mj] = p[t]; p[t] = x;
    }
    if (std::fabs(A[t][t]) < 1e-10) return false;
    for (int c = t + 1; c <= 4; ++c) {
      A[t][c] = A[t][c] / A[t][t];
      for (int r = t + 1; r <= 4; ++r) A[r][c] = A[r][c] - A[t][c] * A[r][t];
    }
  }
  for (int i = 1; i <= 4; ++i) {
    double b[5] = {0, 0, 0, 0, 0};
    b[i] = 1.0;
    for (int c = 1; c <= 4; ++c)
      if (c != p[c] && c < p[c]) { const double x = b[c]; b[c] = b[p[c]]; b[p[c]] = x; }
    for (int c = 1; c <= 4; ++c) {
      double s = b[c];
      for (int r = 1; r < c; ++r) s = s - A[r][c] * b[r];
      b[c] = s;
    }
    for (int c = 4; c >= 1; --c) {
      double s = b[c];
      for (int r = 4; r > c; --r) s = s - A[r][c] * b[r];
      b[c] = s / A[c][c];
    }
    for (int c = 1; c <= 4; ++c) out[i - 1][c - 1] = b[c];
  }
  return true;
}

// transbl2ks (physfunc.f90:366-505): BL 4-velocity -> (M)KS u-tilde.
void bl_to_ks(const rg_run_params& p, const double util[4], double out[4], double r, double th, double thm) {
  const double akm = p.akm;
  const double rbh1 = 1. + std::sqrt(1. - akm * akm);
  Mat g, gc;
  zero(gc);
  auto con = [&](void) {
    if (p.metric == 303) {
      ks_con(p, gc, r, th);
    } else {
      mks_cov(p, g, r, th, thm, true);
      lu_inverse_cols(g, gc);
    }
  };
  if (r > rbh1) {
    bl_cov(akm, g, r, th);
    double u[4] = {0.0, util[1], util[2], util[3]};
    const double aa = g[0][0];
    const double bb = 2. * (g[0][1] * u[1] + g[0][2] * u[2] + g[0][3] * u[3]);
    const double cc = 1. + g[1][1] * u[1] * u[1] + g[2][2] * u[2] * u[2] + g[3][3] * u[3] * u[3] +
                      2. * (g[1][2] * u[1] * u[2] + g[1][3] * u[1] * u[3] + g[2][3] * u[2] * u[3]);
    const double disc = bb * bb - 4. * aa * cc;
    u[0] = (-bb - std::sqrt(disc)) * (1. / (2. * aa));
    Mat tr;
    zero(tr);
    const double del = r * r - (2. * r) + akm * akm;
    if (del > 0.0) {
      tr[0][0] = 1.0; tr[0][1] = 2. * r * (1. / del); tr[1][1] = 1.0;
      tr[2][2] = 1.0; tr[2][1] = akm * (1. / del); tr[3][3] = 1.0;
    }
    double v[4] = {0, 0, 0, 0};
    for (int n = 0; n < 4; ++n)
      for (int m = 0; m < 4; ++m) v[m] = v[m] + tr[m][n] * u[n];
    if (p.metric == 403) {
      if (p.ix1 == 2) v[1] = v[1] * (1. / (r));
      if (p.ix3 == 2) v[3] = v[3] * (1. / (1. + (1. - p.hslope) * std::cos(2. * thm)));
    }
    con();
    const double alpha = 1. / std::sqrt(-gc[0][0]);
    const double gfl = v[0] * alpha;
    for (int m = 1; m <= 3; ++m) out[m] = v[m] + gfl * (alpha * alpha * gc[0][m]) * (1. / alpha);
  } else {
    con();
    const double alpha = 1. / std::sqrt(-gc[0][0]);
    for (int m = 1; m <= 3; ++m) out[m] = alpha * alpha * gc[0][m] * (1. / alpha);
  }
}

// Counter-based uniform in [0,1) keyed by (seed, cell): splitmix64 finaliser.
double uniform01(uint64_t seed, uint64_t idx) {
  uint64_t z = seed * 0x9E3779B97F4A7C15ULL + idx + 0x632BE59BD9B4E019ULL;
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z = z ^ (z >> 31);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

// Angular momentum of the Fishbone-Moncrief torus (mdgrmhd.f90:808-832).
double fm_ell(double a, double r) {
  const double sr = std::sqrt(r);
  const double t1a = ((a * a) - 2. * a * sr + (r * r));
  const double t1b = (-2. * a * r) * t1a;
  const double t1c = std::sqrt(2. * a * sr + (-3. + r) * r);
  const double t1d = (a + (-2. + r) * sr);
  const double t1e = ((r * r * r) + (a * a) * (2. + r));
  const double t1f = std::sqrt(1. + (2. * a / std::pow(r, 1.5)) - (3. / r));
  const double t2a = (r * r * r) * std::sqrt(2. * a * sr + (-3. + r) * r);
  const double t2b = ((a * a) + (-2. + r) * r);
  return (t1a * ((t1b / t1c) + t1d * t1e / t1f)) / (t2a * t2b);
}

}  // namespace

// Seeded 1D RMHD Riemann problem in the pattern of mdshoctub
// (mdgrmhd.f90:56-118): state[0] fills i <= imax/2, state[1] the rest.  The
// states are drawn with uniform01 keyed by (seed, 16*tube + field): field 0
// the shared B^x in [0, 5]; per side s (fields 1+7s ..) rho log-uniform in
// [0.1, 10], p log-uniform in [0.01, 100], v^x, v^y, v^z uniform in
// [-0.9, 0.9] (scaled down to |v| = 0.9 when larger), B^y, B^z uniform in
// [-5, 5].  Primitives: util = gamma*v (Minkowski), uri(6) = p/rho**(gam-1).
void tube_states(uint64_t seed, uint64_t tube, double gam, double state[2][9]) {
  auto U = [&](int f) { return uniform01(seed, 16 * tube + (uint64_t)f); };
  const double bx = 5.0 * U(0);
  for (int side = 0; side < 2; ++side) {
    const int f0 = 1 + 7 * side;
    const double rho = std::pow(10.0, -1.0 + 2.0 * U(f0));
    const double pg = std::pow(10.0, -2.0 + 4.0 * U(f0 + 1));
    double v[3];
    for (int a = 0; a < 3; ++a) v[a] = 0.9 * (2.0 * U(f0 + 2 + a) - 1.0);
    const double v2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    if (v2 > 0.81) {
      const double scale = 0.9 / std::sqrt(v2);
      for (double& x : v) x *= scale;
    }
    const double lor = 1.0 / std::sqrt(1.0 - (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
    double* q = state[side];
    q[0] = rho;
    for (int a = 0; a < 3; ++a) q[1 + a] = lor * v[a];
    q[4] = pg;
    q[5] = pg * (1. / std::pow(rho, gam - 1.));
    q[6] = bx;
    q[7] = 5.0 * (2.0 * U(f0 + 5) - 1.0);
    q[8] = 5.0 * (2.0 * U(f0 + 6) - 1.0);
  }
}

void torus_ic(const rg_run_params& p, const HostGeom& G, uint64_t seed, double amp, double rin, double rmax,
              double beta, double kappa, std::vector<double>& P, bool plane_only) {
  const int imax = p.imax, jmax = p.jmax, kmax = p.kmax;
  // Every phi plane of the torus is the same except for the perturbation,
  // which a 2D phi slab keys by its interior plane: a run that stores the slab
  // as one plane needs only that plane (the others stay zero).
  const int nm1_pl = ghost_nm1(p);
  const int jlo = plane_only ? nm1_pl + 1 : 1, jhi = plane_only ? nm1_pl + 1 : jmax;
  const size_t N = (size_t)imax * jmax * kmax, nik = G.nik;
  const double gam = p.gam, a = p.akm;
  const Axis& X1 = G.ax[0];
  const Axis& X3 = G.ax[2];
  P.assign(9 * N, 0.0);
  auto at = [&](int v, int i, int j, int k) -> double& {
    return P[(size_t)v * N + (size_t)(i - 1) + (size_t)imax * ((size_t)(j - 1) + (size_t)jmax * (k - 1))];
  };
  auto cidx = [&](int i, int j, int k) { return (size_t)(i - 1) + (size_t)imax * ((size_t)(j - 1) + (size_t)jmax * (k - 1)); };
  const double edge0 = (double)0.02f * kPi, edge1 = (double)0.98f * kPi;
  const double ell = fm_ell(a, rmax);
  std::vector<double> lnh(N, 0.0), apot(N, 0.0);
  // floor atmosphere everywhere (mdgrmhd.f90:964-1021)
  for (int k = 1; k <= kmax; ++k)
    for (int j = jlo; j <= jhi; ++j)
      for (int i = 1; i <= imax; ++i) {
        const double r = X1.x[i];
        const double de = p.dmin * std::pow(r, -1.5), pr = p.pmin * (gam - 1.) * std::pow(r, -2.5);
        at(0, i, j, k) = de;
        at(4, i, j, k) = pr;
        at(5, i, j, k) = pr * (1. / std::pow(de, gam - 1.));
      }
  // ln h relative to the inner edge (mdgrmhd.f90:1027-1103)
  const double dl = rin * rin - 2.0 * rin + a * a;
  const double al = (rin * rin + a * a) * (rin * rin + a * a) - dl * a * a;
  const double sl = rin * rin;
  const double e2a = 4.0 * (ell * ell * sl * sl) * dl * (1.0 / (al * al));
  const double e2c = sl * dl * (1.0 / al);
  const double h_in = 0.5 * std::log((1.0 + std::sqrt(1. + e2a)) * (1.0 / e2c)) - 0.5 * std::sqrt(1.0 + e2a) -
                      2.0 * a * rin * ell * (1.0 / al);
  double rhomax = 0.0;
  for (int k = 1; k <= kmax; ++k)
    for (int j = jlo; j <= jhi; ++j)
      for (int i = 1; i <= imax; ++i) {
        const double r = X1.x[i], th = X3.x[k];
        double sth = std::sin(th);
        if (std::fabs(sth) < 1.e-12) sth = (sth >= 0.0) ? 1.e-12 : -1.e-12;
        const double cth = std::cos(th);
        const double del = (r * r) - (2.0 * r) + (a * a);
        const double aa = (r * r + a * a) * (r * r + a * a) - del * a * a * sth * sth;
        const double sig = r * r + a * a * cth * cth;
        const bool inside = (r >= rin && th >= edge0 && th <= edge1);
        double lh = 0.0;
        if (inside) {
          const double t1a = 4.0 * (ell * ell * sig * sig) * del * (1.0 / (aa * sth * aa * sth));
          const double t1c = sig * del * (1.0 / aa);
          const double t1d = 0.5 * std::log((1.0 + std::sqrt(1. + t1a)) * (1.0 / t1c));
          const double t1e = 0.5 * std::sqrt(1.0 + t1a);
          const double t1f = 2.0 * a * r * ell * (1.0 / aa);
          lh = t1d - t1e - t1f - h_in;
          if (lh <= 0.0) lh = 0.0;
        }
        lnh[cidx(i, j, k)] = lh;
        const double hm1 = std::exp(lh) - 1.0;
        if (hm1 > 0.0 && inside) {
          const double de = std::pow(hm1 * (gam - 1.0) / (kappa * gam), 1.0 / (gam - 1.0));
          const double pr = kappa * std::pow(de, gam);
          const double e2chi = sig * sig * del * (1.0 / (aa * aa * sth * sth));
          const double uphi = std::sqrt((-1.0 + std::sqrt(1.0 + 4.0 * ell * ell * e2chi)) / 2.0);
          const double t3a = 2.0 * a * r * std::sqrt(1. + uphi * uphi);
          const double t3b = std::sqrt(aa * sig * del);
          const double t3c = std::sqrt(sig * (1.0 / aa)) * uphi * (1.0 / sth);
          double util[4] = {0.0, 0.0, t3a * (1.0 / t3b) + t3c, 0.0};
          if (de > rhomax) rhomax = de;
          if (p.metric == 303 || p.metric == 403) {
            double un[4];
            bl_to_ks(p, util, un, r, th, X3.xb[k]);
            util[1] = un[1]; util[2] = un[2]; util[3] = un[3];
          }
          at(0, i, j, k) = de;
          at(1, i, j, k) = util[1];
          at(2, i, j, k) = util[2];
          at(3, i, j, k) = util[3];
          at(4, i, j, k) = pr;
          at(5, i, j, k) = pr * (1.0 / std::pow(de, gam - 1.));
        }
      }
  // normalise rho_max to 1, perturb p (mdgrmhd.f90:1198-1320).  In a 2D phi
  // slab (jmax = 2*nm1+1) the draw is keyed by the (r, theta) cell of the
  // interior phi index, so that the slab holds one axisymmetric state.
  const int nm1_ic = ghost_nm1(p);
  const bool phi_slab = (jmax == 2 * nm1_ic + 1);
  for (int k = 1; k <= kmax; ++k)
    for (int j = jlo; j <= jhi; ++j)
      for (int i = 1; i <= imax; ++i) {
        const double r = X1.x[i], th = X3.x[k];
        const size_t c = cidx(i, j, k);
        if (std::exp(lnh[c]) - 1.0 > 0.0 && r >= rin && th >= edge0 && th <= edge1) {
          const double rmin1 = p.dmin * std::pow(r, -1.5), pmin1 = p.pmin * (gam - 1.) * std::pow(r, -2.5);
          double de = at(0, i, j, k) * (1.0 / rhomax);
          double pr = at(4, i, j, k) * (1.0 / rhomax);
          pr = pr * (1.0 + amp * (uniform01(seed, phi_slab ? cidx(i, nm1_ic + 1, k) : c) - 0.5));
          if (de <= rmin1 || pr <= pmin1) {
            de = rmin1;
            pr = pmin1;
            at(1, i, j, k) = 0.0; at(2, i, j, k) = 0.0; at(3, i, j, k) = 0.0;
          }
          at(0, i, j, k) = de;
          at(4, i, j, k) = pr;
          at(5, i, j, k) = pr * (1.0 / std::pow(de, gam - 1.0));
        }
      }
  // A_phi ~ max(<rho> - 0.2, 0) at cell corners (mdgrmhd.f90:1335-1368)
  for (int k = 2; k <= kmax; ++k)
    for (int j = jlo; j <= jhi; ++j)
      for (int i = 2; i <= imax; ++i) {
        const double av = 0.25 * (at(0, i, j, k) + at(0, i - 1, j, k) + at(0, i, j, k - 1) + at(0, i - 1, j, k - 1));
        const double a1 = (av != 0.0) ? ((av * (1. / 1.0)) - 0.2) : 0.0;
        if (a1 > 0.0) apot[cidx(i, j, k)] = a1;
      }
  for (int j = jlo; j <= jhi; ++j)
    for (int i = 1; i <= imax; ++i) apot[cidx(i, j, 1)] = apot[cidx(i, j, 2)];
  for (int k = 1; k <= kmax; ++k)
    for (int j = jlo; j <= jhi; ++j) apot[cidx(1, j, k)] = apot[cidx(2, j, k)];
  const bool mks = (p.metric == 403);
  for (int k = 2; k <= kmax - 1; ++k)
    for (int j = jlo; j <= jhi; ++j)
      for (int i = 2; i <= imax - 1; ++i) {
        auto A = [&](int ii, int kk) { return apot[cidx(ii, j, kk)]; };
        const double dg = G.mc[(size_t)(kMetBase - 1) * nik + (size_t)(i - 1) + (size_t)imax * (k - 1)];
        const double c1 = 0.5 * (A(i + 1, k + 1) + A(i, k + 1) - A(i + 1, k) - A(i, k));
        const double h3 = mks ? 0.5 * (X3.xb[k + 1] + X3.xb[k]) - 0.5 * (X3.xb[k] + X3.xb[k - 1])
                              : 0.5 * (X3.x[k + 1] + X3.x[k]) - 0.5 * (X3.x[k] + X3.x[k - 1]);
        const double c3 = 0.5 * (A(i + 1, k + 1) + A(i + 1, k) - A(i, k + 1) - A(i, k));
        const double h1 = mks ? 0.5 * (X1.xb[i + 1] + X1.xb[i]) - 0.5 * (X1.xb[i] + X1.xb[i - 1])
                              : 0.5 * (X1.x[i + 1] + X1.x[i]) - 0.5 * (X1.x[i] + X1.x[i - 1]);
        at(6, i, j, k) = (c1 != 0.0) ? -(c1 * (1.0 / (h3 * dg))) : 0.0;
        at(8, i, j, k) = (c3 != 0.0) ? c3 * (1.0 / (h1 * dg)) : 0.0;
      }
  for (int j = jlo; j <= jhi; ++j)
    for (int i = 1; i <= imax; ++i) {
      at(6, i, j, 1) = at(6, i, j, 2); at(6, i, j, kmax) = at(6, i, j, kmax - 1);
      at(8, i, j, 1) = at(8, i, j, 2); at(8, i, j, kmax) = at(8, i, j, kmax - 1);
    }
  for (int k = 1; k <= kmax; ++k)
    for (int j = jlo; j <= jhi; ++j) {
      at(6, 1, j, k) = at(6, 2, j, k); at(6, imax, j, k) = at(6, imax - 1, j, k);
      at(8, 1, j, k) = at(8, 2, j, k); at(8, imax, j, k) = at(8, imax - 1, j, k);
    }
  // scale B to the target minimum plasma beta (mdgrmhd.f90:1424-1540)
  double beta_min = 1.e5;
  for (int k = 1; k <= kmax; ++k)
    for (int j = jlo; j <= jhi; ++j)
      for (int i = 1; i <= imax; ++i) {
        const size_t q = (size_t)(i - 1) + (size_t)imax * (k - 1);
        Mat g, gc;
        metric_at(p, X1.x[i], X3.x[k], X3.xb[k], g, gc);
        const double u1 = at(1, i, j, k), u2 = at(2, i, j, k), u3 = at(3, i, j, k);
        const double ut[4] = {0.0, u1, u2, u3};
        double utsq = 0.0;
        for (int x = 1; x <= 3; ++x)
          for (int y = 1; y <= 3; ++y) utsq = utsq + g[x][y] * ut[x] * ut[y];
        if (utsq < 0.0) utsq = (std::fabs(utsq) <= 1.0e-10) ? std::fabs(utsq) : 1.e-10;
        if (std::fabs(utsq) > 5.e2) utsq = 5.0e2;
        const double gfl = std::sqrt(1. + utsq);
        const double alpha = 1. / std::sqrt(-gc[0][0]);
        double uc[4], ul[4], bc[4], bl[4];
        uc[0] = gfl * (1. / alpha);
        for (int m = 1; m <= 3; ++m) uc[m] = ut[m] - gfl * (alpha * alpha * gc[0][m]) * (1. / alpha);
        for (int x = 0; x < 4; ++x) ul[x] = g[x][0] * uc[0] + g[x][1] * uc[1] + g[x][2] * uc[2] + g[x][3] * uc[3];
        const double B1 = at(6, i, j, k), B2 = at(7, i, j, k), B3 = at(8, i, j, k);
        bc[0] = B1 * ul[1] + B2 * ul[2] + B3 * ul[3];
        bc[1] = (B1 + bc[0] * uc[1]) * (1. / uc[0]);
        bc[2] = (B2 + bc[0] * uc[2]) * (1. / uc[0]);
        bc[3] = (B3 + bc[0] * uc[3]) * (1. / uc[0]);
        for (int x = 0; x < 4; ++x) bl[x] = g[x][0] * bc[0] + g[x][1] * bc[1] + g[x][2] * bc[2] + g[x][3] * bc[3];
        const double bsq = bc[0] * bl[0] + bc[1] * bl[1] + bc[2] * bl[2] + bc[3] * bl[3];
        const double pb = (bsq != 0.0) ? 2. * at(4, i, j, k) / bsq : 1.e5;
        if (pb < beta_min) beta_min = pb;
      }
  const double bnorm = (beta == 0.0) ? 0.0 : std::sqrt(beta_min / beta);
  for (size_t c = 0; c < N; ++c)
    for (int v = 6; v <= 8; ++v) P[(size_t)v * N + c] = P[(size_t)v * N + c] * bnorm;
}

void torus_tables(const rg_run_params& p, const HostGeom& G, double rin, double rmax, TorusTables& T) {
  const int imax = p.imax, kmax = p.kmax;
  const double gam = p.gam, a = p.akm;
  const Axis& X1 = G.ax[0];
  const Axis& X3 = G.ax[2];
  const bool mks = (p.metric == 403);
  T.tab.assign((size_t)kIcTabI * imax + (size_t)kIcTabK * kmax, 0.0);
  auto ti = [&](int f, int i) -> double& { return T.tab[(size_t)f * imax + (i - 1)]; };
  auto tk = [&](int f, int k) -> double& { return T.tab[(size_t)kIcTabI * imax + (size_t)f * kmax + (k - 1)]; };
  for (int i = 1; i <= imax; ++i) {
    const double r = X1.x[i];
    ti(IC_R, i) = r;
    ti(IC_DE, i) = p.dmin * std::pow(r, -1.5);
    ti(IC_PR, i) = p.pmin * (gam - 1.) * std::pow(r, -2.5);
    if (i >= 2 && i <= imax - 1)
      ti(IC_H1, i) = mks ? 0.5 * (X1.xb[i + 1] + X1.xb[i]) - 0.5 * (X1.xb[i] + X1.xb[i - 1])
                         : 0.5 * (X1.x[i + 1] + X1.x[i]) - 0.5 * (X1.x[i] + X1.x[i - 1]);
  }
  for (int k = 1; k <= kmax; ++k) {
    const double th = X3.x[k];
    double sth = std::sin(th);
    if (std::fabs(sth) < 1.e-12) sth = (sth >= 0.0) ? 1.e-12 : -1.e-12;
    tk(IC_TH, k) = th;
    tk(IC_STH, k) = sth;
    tk(IC_CTH, k) = std::cos(th);
    const double thb = (th > kPi) ? 2. * kPi - th : th;  // bl_cov's theta
    tk(IC_SBL, k) = clamp_small(std::sin(thb));
    tk(IC_CBL, k) = clamp_small(std::cos(thb));
    tk(IC_HDEN, k) = 1. + (1. - p.hslope) * std::cos(2. * X3.xb[k]);
    if (k >= 2 && k <= kmax - 1)
      tk(IC_H3, k) = mks ? 0.5 * (X3.xb[k + 1] + X3.xb[k]) - 0.5 * (X3.xb[k] + X3.xb[k - 1])
                         : 0.5 * (X3.x[k + 1] + X3.x[k]) - 0.5 * (X3.x[k] + X3.x[k - 1]);
  }
  T.edge0 = (double)0.02f * kPi;
  T.edge1 = (double)0.98f * kPi;
  T.ell = fm_ell(a, rmax);
  const double ell = T.ell;
  const double dl = rin * rin - 2.0 * rin + a * a;
  const double al = (rin * rin + a * a) * (rin * rin + a * a) - dl * a * a;
  const double sl = rin * rin;
  const double e2a = 4.0 * (ell * ell * sl * sl) * dl * (1.0 / (al * al));
  const double e2c = sl * dl * (1.0 / al);
  T.h_in = 0.5 * std::log((1.0 + std::sqrt(1. + e2a)) * (1.0 / e2c)) - 0.5 * std::sqrt(1.0 + e2a) -
           2.0 * a * rin * ell * (1.0 / al);
}

}  // namespace rg
