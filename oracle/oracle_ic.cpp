// oracle_ic.cpp -- Fishbone-Moncrief torus initial data (mdgrmhd.f90:808-1654)
// restated for the CPU oracle (test infrastructure only; see oracle.hpp).
#include <cmath>
#include <cstdint>
#include <vector>

#include "oracle.hpp"

namespace orc {

// Counter-based uniform draw in [0,1) keyed by (seed, cell index).  The
// reference calls the unseeded random_number once per torus cell in loop order
// (mdgrmhd.f90:1279), which no other program can reproduce; keying the draw by
// the cell makes the perturbation reproducible and order independent.
double ic_uniform(uint64_t seed, uint64_t idx) {
  uint64_t z = seed * 0x9E3779B97F4A7C15ULL + idx + 0x632BE59BD9B4E019ULL;
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z = z ^ (z >> 31);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

// mdgrmhd.f90:808-832
double callfish(double akm, double rmax) {
  const double tmp1a = ((akm * akm) - 2. * akm * std::sqrt(rmax) + (rmax * rmax));
  const double tmp1b = (-2. * akm * rmax) * tmp1a;
  const double tmp1c = std::sqrt(2. * akm * std::sqrt(rmax) + (-3. + rmax) * rmax);
  const double tmp1d = (akm + (-2. + rmax) * std::sqrt(rmax));
  const double tmp1e = ((rmax * rmax * rmax) + (akm * akm) * (2. + rmax));
  const double tmp1f = std::sqrt(1. + (2. * akm / std::pow(rmax, 1.5)) - (3. / rmax));
  const double tmp2a = (rmax * rmax * rmax) * std::sqrt(2. * akm * std::sqrt(rmax) + (-3. + rmax) * rmax);
  const double tmp2b = ((akm * akm) + (-2. + rmax) * rmax);
  const double tmp3a = tmp1a * ((tmp1b / tmp1c) + tmp1d * tmp1e / tmp1f);
  const double tmp3b = tmp2a * tmp2b;
  return tmp3a / tmp3b;
}

// mdgrmhd.f90:879-1654 on one rank.  The pressure perturbation is
// p *= 1 + amp*(U - 0.5) with U from ic_uniform (the reference uses amp = 0.05
// with an unseeded generator).
void mdtorus1(State& s, uint64_t seed, double amp, double rin, double rmax, double beta,
              double kappa) {
  const int imax = s.imax, jmax = s.jmax, kmax = s.kmax;
  const double gam = s.p.gam, akm = s.p.akm;
  const double thedge = sp(0.02f) * PI, thedge1 = sp(0.98f) * PI;
  const double kpol1 = kappa;
  const double rhomin = s.p.dmin, prmin = s.p.pmin, small = 1.e-12;
  auto& u = s.uri;
  std::vector<double> alnh(s.ncell, 0.0), pom(s.ncell, 0.0);
  const double clm = callfish(akm, rmax);
  double rhomax1 = 0.0, prmax1 = 0.0;
  // atmosphere everywhere (mdgrmhd.f90:964-1021)
  for (int k = 1; k <= kmax; ++k)
    for (int j = 1; j <= jmax; ++j)
      for (int i = 1; i <= imax; ++i) {
        const double rr = s.x1[i];
        const double de = rhomin * std::pow(rr, -1.5);
        const double pr = prmin * (gam - 1.) * std::pow(rr, -2.5);
        double* q = &u[s.a(1, i, j, k)];
        q[0] = de; q[1] = 0.0; q[2] = 0.0; q[3] = 0.0; q[4] = pr;
        q[5] = pr * (1. / std::pow(de, gam - 1.));
        q[6] = 0.0; q[7] = 0.0; q[8] = 0.0;
      }
  // ln h at the inner edge (mdgrmhd.f90:1027-1043)
  const double delin = rin * rin - 2.0 * rin + akm * akm;
  const double aain = (rin * rin + akm * akm) * (rin * rin + akm * akm) - delin * akm * akm;
  const double sigin = rin * rin;
  const double tmp2a = 4.0 * (clm * clm * sigin * sigin) * delin * (1.0 / (aain * aain));
  const double tmp2c = sigin * delin * (1.0 / aain);
  const double tmp2d = 0.5 * std::log((1.0 + std::sqrt(1. + tmp2a)) * (1.0 / tmp2c));
  const double tmp2e = 0.5 * std::sqrt(1.0 + tmp2a);
  const double tmp2f = 2.0 * akm * rin * clm * (1.0 / aain);
  // torus interior (mdgrmhd.f90:1045-1190)
  for (int k = 1; k <= kmax; ++k)
    for (int j = 1; j <= jmax; ++j)
      for (int i = 1; i <= imax; ++i) {
        const double rr = s.x1[i], th = s.x3[k];
        double sth = std::sin(th);
        if (std::fabs(sth) < small) sth = (sth >= 0.0) ? small : -small;
        const double cth = std::cos(th);
        const double del = (rr * rr) - (2.0 * rr) + (akm * akm);
        const double aa = (rr * rr + akm * akm) * (rr * rr + akm * akm) - del * akm * akm * sth * sth;
        const double sig = rr * rr + akm * akm * cth * cth;
        const size_t c = s.cell(i, j, k);
        const bool inside = (rr >= rin && th >= thedge && th <= thedge1);
        if (inside) {
          const double tmp1a = 4.0 * (clm * clm * sig * sig) * del * (1.0 / (aa * sth * aa * sth));
          const double tmp1c = sig * del * (1.0 / aa);
          const double tmp1d = 0.5 * std::log((1.0 + std::sqrt(1. + tmp1a)) * (1.0 / tmp1c));
          const double tmp1e = 0.5 * std::sqrt(1.0 + tmp1a);
          const double tmp1f = 2.0 * akm * rr * clm * (1.0 / aa);
          alnh[c] = tmp1d - tmp1e - tmp1f - (tmp2d - tmp2e - tmp2f);
          if (alnh[c] <= 0.0) alnh[c] = 0.0;
        } else {
          alnh[c] = 0.0;
        }
        const double hm1 = std::exp(alnh[c]) - 1.0;
        if (hm1 > 0.0 && inside) {
          const double de = std::pow(hm1 * (gam - 1.0) / (kpol1 * gam), 1.0 / (gam - 1.0));
          const double pr = kpol1 * std::pow(de, gam);
          double util[4] = {0.0, 0.0, 0.0, 0.0};
          const double expm2chi = sig * sig * del * (1.0 / (aa * aa * sth * sth));
          const double uphi1 = std::sqrt((-1.0 + std::sqrt(1.0 + 4.0 * clm * clm * expm2chi)) / 2.0);
          const double tmp3a = 2.0 * akm * rr * std::sqrt(1. + uphi1 * uphi1);
          const double tmp3b = std::sqrt(aa * sig * del);
          const double tmp3c = std::sqrt(sig * (1.0 / aa)) * uphi1 * (1.0 / sth);
          util[2] = tmp3a * (1.0 / tmp3b) + tmp3c;
          if (de > rhomax1) rhomax1 = de;
          if (pr > prmax1) prmax1 = pr;
          if (s.p.metric == 303 || s.p.metric == 403) {
            double utiln[4];
            transbl2ks(s, util, utiln, s.x1[i], s.x3[k], s.x3b[k]);
            util[1] = utiln[1]; util[2] = utiln[2]; util[3] = utiln[3];
          }
          double* q = &u[s.a(1, i, j, k)];
          q[0] = de; q[1] = util[1]; q[2] = util[2]; q[3] = util[3]; q[4] = pr;
          q[5] = pr * (1.0 / std::pow(de, gam - 1.));
        }
      }
  // normalise to rho_max = 1 and perturb p (mdgrmhd.f90:1198-1320).  In a 2D
  // phi slab (jmax = 2*nm1+1) the draw is keyed by the (r, theta) cell of the
  // interior phi index: the slab then holds one axisymmetric state.
  const double rhomax1a = rhomax1;
  const bool phi_slab = (jmax == 2 * s.nm1 + 1);
  for (int k = 1; k <= kmax; ++k)
    for (int j = 1; j <= jmax; ++j)
      for (int i = 1; i <= imax; ++i) {
        const double rr = s.x1[i], th = s.x3[k];
        const double rhomin1 = rhomin * std::pow(rr, -1.5);
        const double prmin1 = prmin * (gam - 1.) * std::pow(rr, -2.5);
        const size_t c = s.cell(i, j, k);
        const double hm1 = std::exp(alnh[c]) - 1.0;
        if (hm1 > 0.0 && rr >= rin && th >= thedge && th <= thedge1) {
          double* q = &u[s.a(1, i, j, k)];
          double de = q[0] * (1.0 / rhomax1a);
          double pr = q[4] * (1.0 / rhomax1a);
          const double r01 = ic_uniform(seed, (uint64_t)(phi_slab ? s.cell(i, s.nm1 + 1, k) : c));
          pr = pr * (1.0 + amp * (r01 - 0.5));
          if (de <= rhomin1) { de = rhomin1; q[1] = 0.0; q[2] = 0.0; q[3] = 0.0; pr = prmin1; }
          if (pr <= prmin1) { de = rhomin1; q[1] = 0.0; q[2] = 0.0; q[3] = 0.0; pr = prmin1; }
          q[0] = de;
          q[4] = pr;
          q[5] = pr * (1.0 / std::pow(de, gam - 1.0));
        }
      }
  // vector potential A_phi ~ max(rho/rho_max - 0.2, 0) on corners (mdgrmhd.f90:1335-1361)
  const double rhomax_n = 1.0;
  for (int k = 2; k <= kmax; ++k)
    for (int j = 1; j <= jmax; ++j)
      for (int i = 2; i <= imax; ++i) {
        const double rhoav = 0.25 * (u[s.a(1, i, j, k)] + u[s.a(1, i - 1, j, k)] + u[s.a(1, i, j, k - 1)] +
                                     u[s.a(1, i - 1, j, k - 1)]);
        const double pom1 = (rhoav != 0.0) ? ((rhoav * (1. / rhomax_n)) - 0.2) : 0.0;
        if (pom1 > 0.0) pom[s.cell(i, j, k)] = pom1;
      }
  for (int j = 1; j <= jmax; ++j)
    for (int i = 1; i <= imax; ++i) pom[s.cell(i, j, 1)] = pom[s.cell(i, j, 2)];
  for (int k = 1; k <= kmax; ++k)
    for (int j = 1; j <= jmax; ++j) pom[s.cell(1, j, k)] = pom[s.cell(2, j, k)];
  // B^r and B^theta from the curl of A_phi (mdgrmhd.f90:1374-1420)
  const bool mks = (s.p.metric == 403);
  for (int k = 2; k <= kmax - 1; ++k)
    for (int j = 1; j <= jmax; ++j)
      for (int i = 2; i <= imax - 1; ++i) {
        auto P = [&](int ii, int kk) { return pom[s.cell(ii, j, kk)]; };
        const double dg = s.detg[s.ik(i, k)];
        const double tmp1a = 0.5 * (P(i + 1, k + 1) + P(i, k + 1) - P(i + 1, k) - P(i, k));
        const double dx3a = mks ? 0.5 * (s.x3b[k + 1] + s.x3b[k]) - 0.5 * (s.x3b[k] + s.x3b[k - 1])
                                : 0.5 * (s.x3[k + 1] + s.x3[k]) - 0.5 * (s.x3[k] + s.x3[k - 1]);
        const double b1 = (tmp1a != 0.0) ? -(tmp1a * (1.0 / (dx3a * dg))) : 0.0;
        const double tmp1b = 0.5 * (P(i + 1, k + 1) + P(i + 1, k) - P(i, k + 1) - P(i, k));
        const double dx1a = mks ? 0.5 * (s.x1b[i + 1] + s.x1b[i]) - 0.5 * (s.x1b[i] + s.x1b[i - 1])
                                : 0.5 * (s.x1[i + 1] + s.x1[i]) - 0.5 * (s.x1[i] + s.x1[i - 1]);
        const double b3 = (tmp1b != 0.0) ? tmp1b * (1.0 / (dx1a * dg)) : 0.0;
        u[s.a(7, i, j, k)] = b1;
        u[s.a(9, i, j, k)] = b3;
      }
  for (int j = 1; j <= jmax; ++j)
    for (int i = 1; i <= imax; ++i) {
      u[s.a(7, i, j, 1)] = u[s.a(7, i, j, 2)];
      u[s.a(7, i, j, kmax)] = u[s.a(7, i, j, kmax - 1)];
      u[s.a(9, i, j, 1)] = u[s.a(9, i, j, 2)];
      u[s.a(9, i, j, kmax)] = u[s.a(9, i, j, kmax - 1)];
    }
  for (int k = 1; k <= kmax; ++k)
    for (int j = 1; j <= jmax; ++j) {
      u[s.a(7, 1, j, k)] = u[s.a(7, 2, j, k)];
      u[s.a(7, imax, j, k)] = u[s.a(7, imax - 1, j, k)];
      u[s.a(9, 1, j, k)] = u[s.a(9, 2, j, k)];
      u[s.a(9, imax, j, k)] = u[s.a(9, imax - 1, j, k)];
    }
  // normalise to the target minimum plasma beta (mdgrmhd.f90:1424-1540)
  double pbeta_min = 1.e5;
  for (int k = 1; k <= kmax; ++k)
    for (int j = 1; j <= jmax; ++j)
      for (int i = 1; i <= imax; ++i) {
        const double* q = &u[s.a(1, i, j, k)];
        const size_t c = s.ik(i, k);
        const double util[4] = {0.0, q[1], q[2], q[3]};
        const double bcon[4] = {0.0, q[6], q[7], q[8]};
        double gfl, ucon[4], ucov[4], bbcon[4], bbcov[4];
        calgfl(util, gfl, s.gcov[c]);
        calucon(util, ucon, gfl, s.gcon[c]);
        lower(ucon, ucov, s.gcov[c]);
        calbbcon(bcon, bbcon, ucov, ucon);
        lower(bbcon, bbcov, s.gcov[c]);
        const double bbsq = calbbsq(bbcon, bbcov);
        const double pbeta = (bbsq != 0.0) ? 2. * q[4] / bbsq : 1.e5;
        if (pbeta < pbeta_min) pbeta_min = pbeta;
      }
  const double bnorm = (beta == 0.0) ? 0.0 : std::sqrt(pbeta_min / beta);
  for (size_t c = 0; c < s.ncell; ++c) {
    u[NV * c + 6] = u[NV * c + 6] * bnorm;
    u[NV * c + 7] = u[NV * c + 7] * bnorm;
    u[NV * c + 8] = u[NV * c + 8] * bnorm;
  }
}

// Seeded 1D RMHD Riemann problem in the pattern of mdshoctub
// (mdgrmhd.f90:56-118): the left state fills i <= imax/2, the right state the
// rest, in every cell (ghosts included); util is the spatial 4-velocity
// gamma*v (Minkowski) and uri(6) = p / rho**(gam-1).  The two states are drawn
// with ic_uniform keyed by (seed, 16*tube + field): field 0 the shared B^x in
// [0, 5]; per side s (base 1 + 7s) rho log-uniform in [0.1, 10], p
// log-uniform in [0.01, 100], v^x, v^y, v^z uniform in [-0.9, 0.9] (scaled
// down to |v| = 0.9 when larger), B^y and B^z uniform in [-5, 5].
void tube_states(uint64_t seed, uint64_t tube, double gam, double q[2][9]) {
  auto U = [&](int f) { return ic_uniform(seed, 16 * tube + (uint64_t)f); };
  const double bx = 5.0 * U(0);
  for (int sd = 0; sd < 2; ++sd) {
    const int b = 1 + 7 * sd;
    const double de = std::pow(10.0, -1.0 + 2.0 * U(b));
    const double pr = std::pow(10.0, -2.0 + 4.0 * U(b + 1));
    double v[3] = {0.9 * (2.0 * U(b + 2) - 1.0), 0.9 * (2.0 * U(b + 3) - 1.0), 0.9 * (2.0 * U(b + 4) - 1.0)};
    const double vv = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    if (vv > 0.81) {
      const double f = 0.9 / std::sqrt(vv);
      v[0] *= f; v[1] *= f; v[2] *= f;
    }
    const double g = 1.0 / std::sqrt(1.0 - (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
    q[sd][0] = de;
    q[sd][1] = g * v[0];
    q[sd][2] = g * v[1];
    q[sd][3] = g * v[2];
    q[sd][4] = pr;
    q[sd][5] = pr * (1. / std::pow(de, gam - 1.));
    q[sd][6] = bx;
    q[sd][7] = 5.0 * (2.0 * U(b + 5) - 1.0);
    q[sd][8] = 5.0 * (2.0 * U(b + 6) - 1.0);
  }
}

void mdtube(State& s, uint64_t seed, uint64_t tube) {
  double q[2][9];
  tube_states(seed, tube, s.p.gam, q);
  for (int k = 1; k <= s.kmax; ++k)
    for (int j = 1; j <= s.jmax; ++j)
      for (int i = 1; i <= s.imax; ++i) {
        const double* src = q[i <= s.imax / 2 ? 0 : 1];
        for (int n = 1; n <= NV; ++n) s.uri[s.a(n, i, j, k)] = src[n - 1];
      }
}

}  // namespace orc
