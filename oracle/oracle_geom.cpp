// oracle_geom.cpp -- grid, metric, Christoffel symbols and the pointwise GR
// helpers of the reference, restated for the CPU oracle (test infrastructure
// only; see oracle.hpp).
#include <cmath>
#include <cstdio>
#include <cstring>

#include "oracle.hpp"

namespace orc {

// grid.f90:2-266 (ix1 in {1,2}, ix2 = 1, ix3 in {1,2}).
void grid(State& s) {
  const orc_params& p = s.p;
  const int imax = p.imax, jmax = p.jmax, kmax = p.kmax;
  auto alloc = [](std::vector<double>& v, int n) { v.assign(n + 2, 0.0); };
  alloc(s.x1, imax); alloc(s.x1a, imax); alloc(s.x1b, imax); alloc(s.x1ab, imax);
  alloc(s.x2, jmax); alloc(s.x2a, jmax); alloc(s.x2b, jmax); alloc(s.x2ab, jmax);
  alloc(s.x3, kmax); alloc(s.x3a, kmax); alloc(s.x3b, kmax); alloc(s.x3ab, kmax);
  alloc(s.dx1, imax); alloc(s.dx2, jmax); alloc(s.dx3, kmax);
  alloc(s.dx1b, imax); alloc(s.dx2b, jmax); alloc(s.dx3b, kmax);
  const bool mks = (p.metric == 403);

  // x1 (grid.f90:25-50)
  if (p.ix1 == 1) {
    for (int i = 1; i <= imax; ++i) {
      s.dx1[i] = (p.xmax - p.xmin) / (double)(float)(imax - 1);
      s.x1[i] = p.xmin + s.dx1[i] * (double)(float)(i - 1);
      s.x1b[i] = s.x1[i];
    }
  } else {  // ix1 == 2, logarithmic (grid.f90:33-50)
    const double xx0 = p.R0;
    const double x1stat = std::log(p.xmin - xx0);
    const double x1end = std::log(p.xmax - xx0);
    const double dx1t = (x1end - x1stat) * sp(1.0f / (float)(imax - 1));
    for (int i = 1; i <= imax; ++i) {
      const double x1t = x1stat + (double)(float)(i - 1) * dx1t;
      s.x1[i] = std::exp(x1t) + xx0;
      s.x1b[i] = x1t;
    }
    for (int i = 2; i <= imax; ++i) s.dx1[i] = mks ? s.x1b[i] - s.x1b[i - 1] : s.x1[i] - s.x1[i - 1];
    s.dx1[1] = s.dx1[2];
  }
  // cell boundaries (grid.f90:124-145)
  for (int i = 1; i <= imax - 1; ++i) s.x1a[i] = 0.5 * (s.x1[i] + s.x1[i + 1]);
  s.x1a[imax] = s.x1a[imax - 1] + s.dx1[imax];
  if (mks) {
    for (int i = 1; i <= imax - 1; ++i) s.x1ab[i] = 0.5 * (s.x1b[i] + s.x1b[i + 1]);
    s.x1ab[imax] = s.x1ab[imax - 1] + s.dx1[imax];
  }
  // grid.f90:139 writes dx1b(imax) one past the declared dx1b(imax-1).
  for (int i = 2; i <= imax; ++i) s.dx1b[i] = mks ? s.x1ab[i] - s.x1ab[i - 1] : s.x1a[i] - s.x1a[i - 1];
  s.dx1b[1] = s.dx1b[2];

  // x2 uniform (grid.f90:150-181)
  for (int j = 1; j <= jmax; ++j) {
    s.dx2[j] = (p.ymax - p.ymin) / (double)(float)(jmax - 1);
    s.x2[j] = p.ymin + s.dx2[j] * (double)(float)(j - 1);
    s.x2b[j] = s.x2[j];
  }
  for (int j = 1; j <= jmax - 1; ++j) s.x2a[j] = 0.5 * (s.x2[j] + s.x2[j + 1]);
  s.x2a[jmax] = s.x2a[jmax - 1] + s.dx2[jmax];
  for (int j = 1; j <= jmax; ++j) s.x2ab[j] = s.x2a[j];
  for (int j = 2; j <= jmax; ++j) s.dx2b[j] = s.x2a[j] - s.x2a[j - 1];
  s.dx2b[1] = s.dx2b[2];

  // x3 (grid.f90:185-264)
  if (p.ix3 == 1) {
    for (int k = 1; k <= kmax; ++k) {
      s.dx3[k] = (p.zmax - p.zmin) / (double)(float)(kmax - 1);
      s.x3[k] = p.zmin + s.dx3[k] * (double)(float)(k - 1);
      s.x3b[k] = s.x3[k];
    }
  } else {  // ix3 == 2 (grid.f90:195-218)
    const double x3stat = p.zmin / PI;
    const double x3end = p.zmax / PI;
    const double dx3t = (x3end - x3stat) / (double)(float)(kmax - 1);
    for (int k = 1; k <= kmax; ++k) {
      const double x3t = PI * (x3stat + (double)(float)(k - 1) * dx3t);
      s.x3[k] = x3t + 0.5 * (1. - p.hslope) * std::sin(2. * x3t);
      s.x3b[k] = x3t;
    }
    for (int k = 2; k <= kmax; ++k) s.dx3[k] = mks ? s.x3b[k] - s.x3b[k - 1] : s.x3[k] - s.x3[k - 1];
    s.dx3[1] = s.dx3[2];
  }
  for (int k = 1; k <= kmax - 1; ++k) s.x3a[k] = 0.5 * (s.x3[k] + s.x3[k + 1]);
  s.x3a[kmax] = s.x3a[kmax - 1] + s.dx3[kmax];
  if (mks) {
    for (int k = 1; k <= kmax - 1; ++k) s.x3ab[k] = 0.5 * (s.x3b[k] + s.x3b[k + 1]);
    s.x3ab[kmax] = s.x3ab[kmax - 1] + s.dx3[kmax];
  }
  for (int k = 2; k <= kmax; ++k) s.dx3b[k] = mks ? s.x3ab[k] - s.x3ab[k - 1] : s.x3a[k] - s.x3a[k - 1];
  s.dx3b[1] = s.dx3b[2];
}

static inline void clamp_small(double& v) {
  const double small = 1.e-12;
  if (std::fabs(v) < small) v = (v > 0.0) ? small : -small;
}

// coord.f90:149-171
void mincov1(M4& g) {
  std::memset(&g, 0, sizeof(g));
  g.a[0][0] = -1.0; g.a[1][1] = 1.0; g.a[2][2] = 1.0; g.a[3][3] = 1.0;
}

// coord.f90:535-613 (KS covariant metric; index 2 = phi, 3 = theta)
void kshcov1(const State& s, M4& g, double x1aa, double x3aa) {
  const double akm = s.p.akm;
  const double rr = x1aa;
  const double theta = (x3aa > PI) ? 2. * PI - x3aa : x3aa;
  double sth = std::sin(theta); clamp_small(sth);
  const double s2 = sth * sth;
  double cth = std::cos(theta); clamp_small(cth);
  const double a2 = akm * akm, r2 = rr * rr;
  const double del = r2 - (2. * rr) + a2;
  const double sig = r2 + a2 * cth * cth;
  const double aa = ((r2 + a2) * (r2 + a2)) - a2 * del * s2;
  std::memset(&g, 0, sizeof(g));
  g.a[0][0] = -1. + 2. * rr / sig;
  g.a[0][1] = 2. * rr / sig;
  g.a[0][2] = -(2. * akm * rr * s2 * (1. / sig));
  g.a[1][0] = g.a[0][1];
  g.a[1][1] = 1. + 2. * rr / sig;
  g.a[1][2] = -(1. * akm * s2 * (1. + 2. * rr / sig));
  g.a[2][0] = g.a[0][2];
  g.a[2][1] = g.a[1][2];
  g.a[2][2] = aa * s2 * (1. / sig);
  g.a[3][3] = sig;
}

// coord.f90:616-690 (analytic KS contravariant metric)
void kshcon1(const State& s, M4& g, double x1aa, double x3aa) {
  const double akm = s.p.akm;
  const double rr = x1aa;
  const double theta = (x3aa > PI) ? 2. * PI - x3aa : x3aa;
  double sth = std::sin(theta); clamp_small(sth);
  const double s2 = sth * sth;
  double cth = std::cos(theta); clamp_small(cth);
  const double a2 = akm * akm, r2 = rr * rr;
  const double del = r2 - (2. * rr) + a2;
  const double sig = r2 + a2 * cth * cth;
  std::memset(&g, 0, sizeof(g));
  g.a[0][0] = -1. - 2. * rr / sig;
  g.a[0][1] = 2. * rr / sig;
  g.a[1][0] = g.a[0][1];
  g.a[1][1] = del / sig;
  g.a[1][2] = akm * (1. / sig);
  g.a[2][1] = g.a[1][2];
  g.a[2][2] = 1. / (sig * s2);
  g.a[3][3] = 1. / sig;
}

// coord.f90:693-792 (modified KS: r = exp(x1) for ix1 = 2, theta(x3) for ix3 = 2)
void mkshcov1(const State& s, M4& g, double x1aa, double x3aa, double x3t) {
  const double akm = s.p.akm;
  const double rr = x1aa;
  const double theta = (x3aa > PI) ? 2. * PI - x3aa : x3aa;
  double sth = std::sin(theta); clamp_small(sth);
  const double s2 = sth * sth;
  double cth = std::cos(theta); clamp_small(cth);
  const double a2 = akm * akm, r2 = rr * rr;
  const double del = r2 - (2. * rr) + a2;
  const double sig = r2 + a2 * cth * cth;
  const double aa = ((r2 + a2) * (r2 + a2)) - a2 * del * s2;
  const double tfac = 1.0, pfac = 1.0;
  const double rfac = (s.p.ix1 == 2) ? rr : 1.0;
  const double hfac = (s.p.ix3 == 2) ? 1. + (1. - s.p.hslope) * std::cos(2. * x3t) : 1.0;
  std::memset(&g, 0, sizeof(g));
  g.a[0][0] = (-1. + 2. * rr / sig) * tfac * tfac;
  g.a[0][1] = (2. * rr / sig) * tfac * rfac;
  g.a[0][2] = (-(2. * akm * rr * s2 * (1. / sig))) * tfac * pfac;
  g.a[1][0] = g.a[0][1];
  g.a[1][1] = (1. + 2. * rr / sig) * rfac * rfac;
  g.a[1][2] = (-(1. * akm * s2 * (1. + 2. * rr / sig))) * rfac * pfac;
  g.a[2][0] = g.a[0][2];
  g.a[2][1] = g.a[1][2];
  g.a[2][2] = (aa * s2 * (1. / sig)) * pfac * pfac;
  g.a[3][3] = sig * hfac * hfac;
}

// coord.f90:378-463 (Boyer-Lindquist Kerr covariant metric; IC only)
void kercov1(const State& s, M4& g, double x1aa, double x3aa) {
  const double akm = s.p.akm;
  const double rr = x1aa;
  const double theta = (x3aa > PI) ? 2. * PI - x3aa : x3aa;
  double sth = std::sin(theta); clamp_small(sth);
  const double s2 = sth * sth;
  double cth = std::cos(theta); clamp_small(cth);
  const double a2 = akm * akm, r2 = rr * rr;
  const double del = 1. - (2. / rr) + (a2 * (1. / r2));
  const double sig = 1. + a2 * cth * cth * (1. / r2);
  std::memset(&g, 0, sizeof(g));
  g.a[0][0] = -(1. - 2. * (1. / (rr * sig)));
  g.a[0][2] = -(2. * akm * s2 * (1. / (rr * sig)));
  g.a[1][1] = sig / del;
  g.a[2][0] = g.a[0][2];
  g.a[2][2] = r2 * s2 * (1. + (a2 * (1. / r2)) + 2. * a2 * s2 * (1. / (r2 * rr * sig)));
  g.a[3][3] = r2 * sig;
}

// coord.f90:1558-1645 (Crout LU with implicit pivoting; 1-based a[1..4][1..4]).
// The reference loop "do i=0,j-1" reads and writes back a(0,j) unchanged; the
// i = 0 pass is therefore a no-op and is skipped here.
static void ludcmp(double a[5][5], int n, int indx[5], double& d) {
  const double tiny = sp(1.e-20f);
  double vv[5];
  d = 1.0;
  for (int i = 1; i <= n; ++i) {
    double aamax = 0.0;
    for (int j = 1; j <= n; ++j)
      if (std::fabs(a[i][j]) > aamax) aamax = std::fabs(a[i][j]);
    vv[i] = 1. / aamax;
  }
  int imax = 1;
  for (int j = 1; j <= n; ++j) {
    for (int i = 1; i <= j - 1; ++i) {
      double sum = a[i][j];
      for (int k = 1; k <= i - 1; ++k) sum = sum - a[i][k] * a[k][j];
      a[i][j] = sum;
    }
    double aamax = 0.0;
    for (int i = j; i <= n; ++i) {
      double sum = a[i][j];
      for (int k = 1; k <= j - 1; ++k) sum = sum - a[i][k] * a[k][j];
      a[i][j] = sum;
      const double dum = vv[i] * std::fabs(sum);
      if (dum >= aamax) { imax = i; aamax = dum; }
    }
    if (j != imax) {
      for (int k = 1; k <= n; ++k) {
        const double dum = a[imax][k];
        a[imax][k] = a[j][k];
        a[j][k] = dum;
      }
      d = -d;
      vv[imax] = vv[j];
    }
    indx[j] = imax;
    if (a[j][j] == 0.0) a[j][j] = tiny;
    if (j != n) {
      const double dum = 1. / a[j][j];
      for (int i = j + 1; i <= n; ++i) a[i][j] = a[i][j] * dum;
    }
  }
}

// coord.f90:1647-1689
static void lubksb(const double a[5][5], int n, const int indx[5], double b[5]) {
  int ii = 0;
  for (int i = 1; i <= n; ++i) {
    const int ll = indx[i];
    double sum = b[ll];
    b[ll] = b[i];
    if (ii != 0) {
      for (int j = ii; j <= i - 1; ++j) sum = sum - a[i][j] * b[j];
    } else if (sum != 0) {
      ii = i;
    }
    b[i] = sum;
  }
  for (int i = n; i >= 1; --i) {
    double sum = b[i];
    for (int j = i + 1; j <= n; ++j) sum = sum - a[i][j] * b[j];
    b[i] = sum / a[i][i];
  }
}

// coord.f90:1504-1555
void invert_matrix2(const M4& g, M4& out) {
  double an[5][5];
  for (int i = 1; i <= 4; ++i)
    for (int j = 1; j <= 4; ++j) an[i][j] = g.a[i - 1][j - 1];
  int indx[5];
  double d;
  ludcmp(an, 4, indx, d);
  for (int j = 1; j <= 4; ++j) {
    double b[5];
    for (int i = 1; i <= 4; ++i) b[i] = (i == j) ? 1.0 : 0.0;
    lubksb(an, 4, indx, b);
    for (int i = 1; i <= 4; ++i) out.a[i - 1][j - 1] = b[i];
  }
}

// coord.f90:1403-1461.  A(i,j) is 1-based, column-major in the reference;
// here A[i][j] with the same index meaning.
static bool lu_decompose(double A[5][5], int N, int p[5], double& d) {
  const double Eps = 1e-10;
  for (int t = 1; t <= N; ++t) {
    int mj = t;
    for (int j = t + 1; j <= N; ++j)
      if (std::fabs(A[t][j]) > std::fabs(A[t][mj])) mj = j;
    if (mj != t) {
      for (int i = 1; i <= N; ++i) {
        const double tmp = A[i][mj];
        A[i][mj] = A[i][t];
        A[i][t] = tmp;
      }
      const int tmp2 = p[mj]; p[mj] = p[t]; p[t] = tmp2;
      d = -d;
    }
    if (std::fabs(A[t][t]) < Eps) return false;
    for (int j = t + 1; j <= N; ++j) {
      A[t][j] = A[t][j] / A[t][t];
      for (int i = t + 1; i <= N; ++i) A[i][j] = A[i][j] - A[t][j] * A[i][t];
    }
  }
  return true;
}

// coord.f90:1463-1501
static void lu_solve(const double A[5][5], int N, const int p[5], double b[5]) {
  for (int j = 1; j <= N; ++j) {
    if (j != p[j] && j < p[j]) {
      const double tmp = b[j];
      b[j] = b[p[j]];
      b[p[j]] = tmp;
    }
  }
  for (int j = 1; j <= N; ++j) {
    double sum = b[j];
    for (int i = 1; i <= j - 1; ++i) sum = sum - A[i][j] * b[i];
    b[j] = sum;
  }
  for (int j = N; j >= 1; --j) {
    double sum = b[j];
    for (int i = N; i >= j + 1; --i) sum = sum - A[i][j] * b[i];
    b[j] = sum / A[j][j];
  }
}

// coord.f90:1324-1400 (A_inv(i,j) = col(j) of the i-th solve)
void invert_matrix(const M4& g, M4& out) {
  double A[5][5];
  int p[5];
  for (int i = 1; i <= 4; ++i) p[i] = i;
  for (int j = 1; j <= 4; ++j)
    for (int i = 1; i <= 4; ++i) A[i][j] = g.a[i - 1][j - 1];
  double d = 1.0;
  if (!lu_decompose(A, 4, p, d)) return;  // reference leaves A_inv untouched
  for (int i = 1; i <= 4; ++i) {
    double col[5] = {0, 0, 0, 0, 0};
    col[i] = 1.0;
    lu_solve(A, 4, p, col);
    for (int j = 1; j <= 4; ++j) out.a[i - 1][j - 1] = col[j];
  }
}

// coord.f90:1016-1086
static double caldetg(const M4& g) {
  auto det3 = [](double aa, double bb, double cc, double pp, double qq, double rr, double xx,
                 double yy, double zz) {
    return aa * qq * zz + bb * rr * xx + cc * pp * yy - cc * qq * xx - bb * pp * zz - aa * rr * yy;
  };
  const auto& G = g.a;
  const double tmp1 = det3(G[1][1], G[1][2], G[1][3], G[2][1], G[2][2], G[2][3], G[3][1], G[3][2], G[3][3]);
  const double tmp2 = det3(G[0][1], G[0][2], G[0][3], G[2][1], G[2][2], G[2][3], G[3][1], G[3][2], G[3][3]);
  const double tmp3 = det3(G[0][1], G[0][2], G[0][3], G[1][1], G[1][2], G[1][3], G[3][1], G[3][2], G[3][3]);
  const double tmp4 = det3(G[0][1], G[0][2], G[0][3], G[1][1], G[1][2], G[1][3], G[2][1], G[2][2], G[2][3]);
  return std::sqrt(-1. * (G[0][0] * tmp1 - G[1][0] * tmp2 + G[2][0] * tmp3 - G[3][0] * tmp4));
}

// coord.f90:5-146 for metric 1, 303 and 403 (j-independent, stored per (i,k))
void coord1(State& s) {
  const int imax = s.imax, kmax = s.kmax;
  const size_t nik = (size_t)imax * kmax;
  s.gcov.resize(nik); s.gcon.resize(nik); s.gcovi.resize(nik); s.gconi.resize(nik);
  s.gcovk.resize(nik); s.gconk.resize(nik);
  s.detg.resize(nik); s.detgi.resize(nik); s.detgk.resize(nik);
  for (int k = 1; k <= kmax; ++k) {
    for (int i = 1; i <= imax; ++i) {
      const size_t q = s.ik(i, k);
      const double x1aa = s.x1[i], x1ai = s.x1a[i], x3aa = s.x3[k], x3ak = s.x3a[k], x3t = s.x3b[k];
      M4 g, gi, gk, c, ci, ck;
      if (s.p.metric == 1) {
        mincov1(g); mincov1(gi); mincov1(gk);
        mincov1(c); mincov1(ci); mincov1(ck);   // mincon1 has the same entries
      } else if (s.p.metric == 303) {
        kshcov1(s, g, x1aa, x3aa); kshcov1(s, gi, x1ai, x3aa); kshcov1(s, gk, x1aa, x3ak);
        kshcon1(s, c, x1aa, x3aa); kshcon1(s, ci, x1ai, x3aa); kshcon1(s, ck, x1aa, x3ak);
      } else {  // 403
        mkshcov1(s, g, x1aa, x3aa, x3t);
        mkshcov1(s, gi, x1ai, x3aa, x3t);
        mkshcov1(s, gk, x1aa, x3ak, x3t);
        invert_matrix2(g, c); invert_matrix2(gi, ci); invert_matrix2(gk, ck);
      }
      s.gcov[q] = g; s.gcovi[q] = gi; s.gcovk[q] = gk;
      s.gcon[q] = c; s.gconi[q] = ci; s.gconk[q] = ck;
      s.detg[q] = caldetg(g); s.detgi[q] = caldetg(gi); s.detgk[q] = caldetg(gk);
    }
  }
}

// coord.f90:1089-1321 (Christoffel symbols by central differences, delta=1e-5)
void calchrist(State& s) {
  const int imax = s.imax, kmax = s.kmax;
  s.christ.assign((size_t)imax * kmax * 64, 0.0);
  const double delta = 1.0e-5, small = 1.e-12;
  const int metric = s.p.metric;
  for (int k = 1; k <= kmax; ++k) {
    for (int i = 1; i <= imax; ++i) {
      double x1aa = s.x1[i], x1ia = s.x1[i] + delta, x1ib = s.x1[i] - delta;
      double x3aa = s.x3[k], x3ka = s.x3[k] + delta, x3kb = s.x3[k] - delta;
      double x1iab = 0, x1ibb = 0, x3kab = 0, x3kbb = 0, x3t = 0;
      if (metric == 403) {
        x1iab = s.x1b[i] + delta;
        x1ibb = s.x1b[i] - delta;
        if (s.p.ix1 == 1) { x1ia = x1iab; x1ib = x1ibb; }
        else { x1ia = std::exp(x1iab); x1ib = std::exp(x1ibb); }
        x3kab = s.x3b[k] + delta;
        x3kbb = s.x3b[k] - delta;
        if (s.p.ix3 == 1) { x3ka = x3kab; x3kb = x3kbb; }
        else {
          x3ka = x3kab + 0.5 * (1. - s.p.hslope) * std::sin(2. * x3kab);
          x3kb = x3kbb + 0.5 * (1. - s.p.hslope) * std::sin(2. * x3kbb);
        }
        x3t = s.x3b[k];
      }
      M4 gia, gib, gja, gjb, gka, gkb, g, gc;
      if (metric == 1) {
        mincov1(gia); mincov1(gib); mincov1(gja); mincov1(gjb); mincov1(gka); mincov1(gkb);
        mincov1(gc);
      } else if (metric == 303) {
        kshcov1(s, gia, x1ia, x3aa); kshcov1(s, gib, x1ib, x3aa);
        kshcov1(s, gja, x1aa, x3aa); kshcov1(s, gjb, x1aa, x3aa);
        kshcov1(s, gka, x1aa, x3ka); kshcov1(s, gkb, x1aa, x3kb);
        kshcon1(s, gc, x1aa, x3aa);
      } else {
        mkshcov1(s, gia, x1ia, x3aa, x3t); mkshcov1(s, gib, x1ib, x3aa, x3t);
        mkshcov1(s, gja, x1aa, x3aa, x3t); mkshcov1(s, gjb, x1aa, x3aa, x3t);
        mkshcov1(s, gka, x1aa, x3ka, x3kab); mkshcov1(s, gkb, x1aa, x3kb, x3kbb);
        mkshcov1(s, g, x1aa, x3aa, x3t);
        invert_matrix2(g, gc);
      }
      // phi positions x2(j) +- delta: every supported metric is phi independent,
      // so g(phi+delta) - g(phi-delta) == 0 exactly (coord.f90:1249-1251).
      const double x2ja_minus_x2jb = 2.0 * delta;  // only divides a zero numerator
      double dg[4][4][4];  // dg[l][m][n] = g_{lm,n}
      for (int m = 0; m < 4; ++m) {
        for (int l = 0; l < 4; ++l) {
          dg[l][m][0] = 0.0;
          const double t1i = gia.a[l][m] - gib.a[l][m];
          dg[l][m][1] = (metric == 403) ? t1i / (x1iab - x1ibb + small) : t1i / (x1ia - x1ib + small);
          const double t1j = gja.a[l][m] - gjb.a[l][m];
          dg[l][m][2] = t1j / (x2ja_minus_x2jb + small);
          const double t1k = gka.a[l][m] - gkb.a[l][m];
          dg[l][m][3] = (metric == 403) ? t1k / (x3kab - x3kbb + small) : t1k / (x3ka - x3kb + small);
        }
      }
      double t2[4][4][4];
      for (int n = 0; n < 4; ++n)
        for (int m = 0; m < 4; ++m)
          for (int l = 0; l < 4; ++l)
            t2[l][m][n] = 0.5 * (dg[m][l][n] + dg[n][l][m] - dg[n][m][l]);
      double* ch = &s.christ[s.ik(i, k) * 64];
      for (int n = 0; n < 4; ++n)
        for (int m = 0; m < 4; ++m)
          for (int l = 0; l < 4; ++l)
            ch[l + 4 * m + 16 * n] = gc.a[l][0] * t2[0][m][n] + gc.a[l][1] * t2[1][m][n] +
                                     gc.a[l][2] * t2[2][m][n] + gc.a[l][3] * t2[3][m][n];
    }
  }
}

// ---------------------------------------------------------------- physfunc.f90
// physfunc.f90:2-42
void calgfl(const double util[4], double& gfl, const M4& g) {
  double utsq = 0.0;
  for (int m = 1; m <= 3; ++m)
    for (int n = 1; n <= 3; ++n) utsq = utsq + g.a[m][n] * util[m] * util[n];
  if (utsq < 0.0) {
    if (std::fabs(utsq) <= 1.0e-10) utsq = std::fabs(utsq);
    else utsq = 1.e-10;
  }
  if (std::fabs(utsq) > 5.e2) utsq = 5.0e2;
  gfl = std::sqrt(1. + utsq);
}

// physfunc.f90:45-78
void calucon(const double util[4], double ucon[4], double gfl, const M4& gc) {
  const double alpha1 = 1. / std::sqrt(-gc.a[0][0]);
  const double b1 = alpha1 * alpha1 * gc.a[0][1];
  const double b2 = alpha1 * alpha1 * gc.a[0][2];
  const double b3 = alpha1 * alpha1 * gc.a[0][3];
  ucon[0] = gfl * (1. / alpha1);
  ucon[1] = util[1] - gfl * b1 * (1. / alpha1);
  ucon[2] = util[2] - gfl * b2 * (1. / alpha1);
  ucon[3] = util[3] - gfl * b3 * (1. / alpha1);
}

// physfunc.f90:161-195
void lower(const double v[4], double o[4], const M4& g) {
  for (int m = 0; m < 4; ++m)
    o[m] = g.a[m][0] * v[0] + g.a[m][1] * v[1] + g.a[m][2] * v[2] + g.a[m][3] * v[3];
}

// physfunc.f90:198-232
void upper(const double v[4], double o[4], const M4& gc) {
  for (int m = 0; m < 4; ++m)
    o[m] = gc.a[m][0] * v[0] + gc.a[m][1] * v[1] + gc.a[m][2] * v[2] + gc.a[m][3] * v[3];
}

// physfunc.f90:81-100 (bcon indexed 1..3)
void calbbcon(const double bcon[4], double bbcon[4], const double ucov[4], const double ucon[4]) {
  bbcon[0] = bcon[1] * ucov[1] + bcon[2] * ucov[2] + bcon[3] * ucov[3];
  bbcon[1] = (bcon[1] + bbcon[0] * ucon[1]) * (1. / ucon[0]);
  bbcon[2] = (bcon[2] + bbcon[0] * ucon[2]) * (1. / ucon[0]);
  bbcon[3] = (bcon[3] + bbcon[0] * ucon[3]) * (1. / ucon[0]);
}

// physfunc.f90:103-119
double calbbsq(const double bbcon[4], const double bbcov[4]) {
  return bbcon[0] * bbcov[0] + bbcon[1] * bbcov[1] + bbcon[2] * bbcov[2] + bbcon[3] * bbcov[3];
}

// coord.f90:970-1013 (spatial 3-metric; indices 1..3 used)
void cal3met(const M4& g, const M4& gc, double g3[4][4], double gc3[4][4]) {
  const double alpha1 = 1. / std::sqrt(-gc.a[0][0]);
  const double beta[4] = {0.0, alpha1 * alpha1 * gc.a[0][1], alpha1 * alpha1 * gc.a[0][2],
                          alpha1 * alpha1 * gc.a[0][3]};
  const double oncon[4] = {1. / alpha1, beta[1] / alpha1, beta[2] / alpha1, beta[3] / alpha1};
  const double oncov[4] = {-alpha1, 0.0, 0.0, 0.0};
  for (int m = 1; m <= 3; ++m)
    for (int n = 1; n <= 3; ++n) {
      g3[m][n] = g.a[m][n] + (oncov[m] * oncov[n]);
      gc3[m][n] = gc.a[m][n] + (oncon[m] * oncon[n]);
    }
}

// physfunc.f90:366-505 (Boyer-Lindquist -> (modified) Kerr-Schild 4-velocity; IC only)
void transbl2ks(const State& s, const double util[4], double utiln[4], double x1aa, double x3aa,
                double x3t) {
  const double akm = s.p.akm;
  const double rbh1 = 1. + std::sqrt(1. - akm * akm);
  const double rr = x1aa;
  M4 gcov1, gcon1;
  std::memset(&gcon1, 0, sizeof(gcon1));
  if (rr > rbh1) {
    kercov1(s, gcov1, x1aa, x3aa);
    double ucon[4] = {0.0, util[1], util[2], util[3]};
    const double aa = gcov1.a[0][0];
    const double bb = 2. * (gcov1.a[0][1] * ucon[1] + gcov1.a[0][2] * ucon[2] + gcov1.a[0][3] * ucon[3]);
    const double cc = 1. + gcov1.a[1][1] * ucon[1] * ucon[1] + gcov1.a[2][2] * ucon[2] * ucon[2] +
                      gcov1.a[3][3] * ucon[3] * ucon[3] +
                      2. * (gcov1.a[1][2] * ucon[1] * ucon[2] + gcov1.a[1][3] * ucon[1] * ucon[3] +
                            gcov1.a[2][3] * ucon[2] * ucon[3]);
    const double discr = bb * bb - 4. * aa * cc;
    ucon[0] = (-bb - std::sqrt(discr)) * (1. / (2. * aa));
    double trans[4][4];
    std::memset(trans, 0, sizeof(trans));
    const double tmp2 = rr * rr - (2. * rr) + akm * akm;
    if (tmp2 > 0.0) {
      trans[0][0] = 1.0;
      trans[0][1] = 2. * rr * (1. / tmp2);
      trans[1][1] = 1.0;
      trans[2][2] = 1.0;
      trans[2][1] = akm * (1. / tmp2);
      trans[3][3] = 1.0;
    }
    double t1[4] = {0, 0, 0, 0};
    for (int n = 0; n < 4; ++n)
      for (int m = 0; m < 4; ++m) t1[m] = t1[m] + trans[m][n] * ucon[n];
    double ucon1[4] = {t1[0], t1[1], t1[2], t1[3]};
    if (s.p.metric == 403) {
      if (s.p.ix1 == 2) ucon1[1] = ucon1[1] * (1. / (rr));
      if (s.p.ix3 == 2) ucon1[3] = ucon1[3] * (1. / (1. + (1. - s.p.hslope) * std::cos(2. * x3t)));
    }
    if (s.p.metric == 303) {
      kshcon1(s, gcon1, x1aa, x3aa);
    } else {
      mkshcov1(s, gcov1, x1aa, x3aa, x3t);
      invert_matrix(gcov1, gcon1);
    }
    const double alpha1 = 1. / std::sqrt(-gcon1.a[0][0]);
    const double gfl = ucon1[0] * alpha1;
    const double b1 = alpha1 * alpha1 * gcon1.a[0][1];
    const double b2 = alpha1 * alpha1 * gcon1.a[0][2];
    const double b3 = alpha1 * alpha1 * gcon1.a[0][3];
    utiln[1] = ucon1[1] + gfl * b1 * (1. / alpha1);
    utiln[2] = ucon1[2] + gfl * b2 * (1. / alpha1);
    utiln[3] = ucon1[3] + gfl * b3 * (1. / alpha1);
  } else {
    if (s.p.metric == 303) {
      kshcon1(s, gcon1, x1aa, x3aa);
    } else {
      mkshcov1(s, gcov1, x1aa, x3aa, x3t);
      invert_matrix(gcov1, gcon1);
    }
    const double alpha1 = 1. / std::sqrt(-gcon1.a[0][0]);
    utiln[1] = alpha1 * alpha1 * gcon1.a[0][1] * (1. / alpha1);
    utiln[2] = alpha1 * alpha1 * gcon1.a[0][2] * (1. / alpha1);
    utiln[3] = alpha1 * alpha1 * gcon1.a[0][3] * (1. / alpha1);
  }
}

}  // namespace orc
