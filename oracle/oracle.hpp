// oracle.hpp -- CPU restatement of RAISHIN's GRMHD update (test infrastructure).
//
// THIS IS THE ORACLE.  It exists only so that tests, the smoke check and the
// CPU baseline leg of the benchmark can check the CUDA product against a
// line-faithful restatement of the reference Fortran.  Nothing in the product
// (raishinsource_b200/) links, imports or calls it.
//
// Parity status: UNPINNED.  The reference (Fortran 90 + MPI) ships no tests,
// golden vectors or fixtures, and no Fortran compiler exists on this machine,
// so this restatement could not be checked against outputs of the reference
// itself.  It follows the reference routine by routine (file:line cited at
// each function), keeps the reference's loop order, 1-based index arithmetic,
// single-precision literals and known quirks, and is compiled with
// -ffp-contract=off so that, like gfortran -O2 on x86-64, no FMA contraction
// or reassociation happens.
//
// Arrays keep the reference layout a(nv,i,j,k) (variable fastest, then i, j,
// k) with 1-based indices.  Metric quantities, which the reference stores per
// (i,j,k) but which depend only on (r,theta) for every metric this build
// supports, are stored per (i,k); this changes no arithmetic.
#pragma once
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <vector>

#include "../include/rg_pow.h"

extern "C" {

// Mirrors module pram (pram.f90:1-80) as a runtime block.
typedef struct {
  int imax, jmax, kmax;       // grid incl. ghosts (pram.f90:11)
  int metric;                 // 1 Minkowski, 303 KS, 403 MKS (pram.f90:67)
  int ix1, ix2, ix3;          // grid spacing kinds (pram.f90:59)
  int irec;                   // 1 MC, 2 minmod, 3 MUSCL, 4 CENO, 5 PPM, 6 MP5, 7 WENO5, 8 MP-WENO,
                              // 9 WENO-Z, 10 WENO-M, 11 LimO3, 12 MVL, 13 Koren (pram.f90:122-131)
  int model;                  // 2 shock tube, 7 FM torus (pram.f90:66)
  int iter;                   // NR iteration cap (pram.f90:27)
  double xmin, xmax, ymin, ymax, zmin, zmax;   // (pram.f90:52-57)
  double R0, hslope, akm, gam;                  // (pram.f90:40,45,60)
  double cfl, dmin, pmin, pmax, tmax, dtmin;    // (pram.f90:22-36)
  int ibc[6][9];              // iboux1in, 1ot, 2in, 2ot, 3in, 3ot (pram.f90:75-80)
  int guard;                  // 0: reference semantics.  Bit 1: first-order fallback for a
                              // reconstructed face state with rho <= 0 or p <= 0; bit 2: zero
                              // flux of the normal B component before flux-CT.  Neither is in
                              // the reference (see face_guard and fluxct in oracle_step.cpp).
  int ict;                    // constrained transport (pram.f90:148-151): 0 none, 1 fluxct,
                              // 2 mflct, 3 upflct
  int iwvec;                  // primitive recovery (pram.f90:160-161): 1 recov1a, 2 recov2
} orc_params;

typedef struct {
  long long recov_calls;      // interior cells inverted
  long long recov_nr2;        // cells that fell back to the entropy NR
  long long recov_fail;       // cells that kept the previous primitives
  long long recov_carry;      // cells whose W guess came from the previous cell
  long long recov_cap;        // rescale-loop caps hit (reference: unbounded)
  long long floor_cap;        // pminmax2b rescale caps hit (reference: unbounded)
} orc_stats;

}  // extern "C"

namespace orc {

constexpr int NV = 9;
constexpr double PI = 3.14159265358979323;   // pram.f90:30

// Fortran single-precision literal as the double gfortran produces from it.
inline double sp(float f) { return (double)f; }

// x**y in the step.  Mode 0 (the default): the C library's pow, which
// gfortran calls for the reference's ** with a real exponent.  Mode 1: the
// library's own power function (include/rg_pow.h), which the uncontracted GPU
// build evaluates to the same bits on the device; with it, that build and
// this restatement carry out one and the same sequence of IEEE operations.
// Both are accurate to about half a unit in the last place and differ in the
// last bit of a small fraction of results.  Set once before stepping.
extern int g_pow_mode;
inline double fpow(double x, double y) { return g_pow_mode ? rgm::pow(x, y) : std::pow(x, y); }

struct M4 { double a[4][4]; };   // a[m][n] == gcov(m,n)

struct State {
  orc_params p;
  int nm0 = 0, nm1 = 0;
  int imax = 0, jmax = 0, kmax = 0;
  size_t ncell = 0;
  // grid (grid.f90); 1-based, element 0 unused.  dx?b has imax entries because
  // grid.f90:139 writes dx1b(imax) past the declared extent dx1b(imax-1).
  std::vector<double> x1, x2, x3, x1a, x2a, x3a, x1b, x2b, x3b, x1ab, x2ab, x3ab;
  std::vector<double> dx1, dx2, dx3, dx1b, dx2b, dx3b;
  // metric per (i,k): centre, i-face (x1a), k-face (x3a); j-face == centre.
  std::vector<M4> gcov, gcon, gcovi, gconi, gcovk, gconk;
  std::vector<double> detg, detgi, detgk;
  std::vector<double> christ;   // 64 per (i,k): christ(l,m,n) at l+4m+16n
  // state arrays a(nv,i,j,k)
  std::vector<double> uu, uo, uh, us, un, uri, urio;
  std::vector<double> uriir, uriil, urijr, urijl, urikr, urikl;
  std::vector<double> uuir, uuil, uujr, uujl, uukr, uukl;
  std::vector<double> wwir, wwil, wwjr, wwjl, wwkr, wwkl;
  std::vector<double> ww;       // ww(3,nv,i,j,k)
  std::vector<double> sf;       // sf(2:5,i,j,k) -> 4 per cell
  std::vector<double> cmaxi, cmini, cmaxj, cminj, cmaxk, cmink;
  double time = 0, timeh = 0, dt = 0.01, dtcfl = 1;
  long long it = 0;
  orc_stats st{};

  size_t cell(int i, int j, int k) const {
    return (size_t)(i - 1) + (size_t)imax * ((size_t)(j - 1) + (size_t)jmax * (size_t)(k - 1));
  }
  size_t a(int n, int i, int j, int k) const { return (size_t)(n - 1) + NV * cell(i, j, k); }
  size_t ik(int i, int k) const { return (size_t)(i - 1) + (size_t)imax * (size_t)(k - 1); }
  size_t w(int d, int n, int i, int j, int k) const {
    return (size_t)(d - 1) + 3 * ((size_t)(n - 1) + NV * cell(i, j, k));
  }
};

// geometry (oracle_geom.cpp)
void grid(State& s);
void coord1(State& s);
void calchrist(State& s);
void mkshcov1(const State& s, M4& g, double x1aa, double x3aa, double x3t);
void kshcov1(const State& s, M4& g, double x1aa, double x3aa);
void kshcon1(const State& s, M4& g, double x1aa, double x3aa);
void kercov1(const State& s, M4& g, double x1aa, double x3aa);
void mincov1(M4& g);
void invert_matrix2(const M4& a, M4& out);
void invert_matrix(const M4& a, M4& out);

// pointwise helpers (physfunc.f90)
void calgfl(const double util[4], double& gfl, const M4& g);
void calucon(const double util[4], double ucon[4], double gfl, const M4& gc);
void lower(const double vcon[4], double vcov[4], const M4& g);
void upper(const double vcov[4], double vcon[4], const M4& gc);
void calbbcon(const double bcon[4], double bbcon[4], const double ucov[4], const double ucon[4]);
double calbbsq(const double bbcon[4], const double bbcov[4]);
void cal3met(const M4& g, const M4& gc, double g3[4][4], double gc3[4][4]);
void transbl2ks(const State& s, const double util[4], double utiln[4], double x1aa, double x3aa,
                double x3t);

// step pieces (oracle_step.cpp)
void caluu1(State& s, const std::vector<double>& uri, std::vector<double>& uu);
void rec2(State& s);
void calcha(State& s);
void hlle(State& s);
void ct(State& s);
void calsf_all(State& s, bool every_cell = false);
void derived(State& s, const std::vector<double>& uri, int jslice, double* out);
void rkstage(State& s, int stage);
void recov1a(State& s, std::vector<double>& uu);
void recov2(State& s, std::vector<double>& uu);
void recov(State& s, std::vector<double>& uu);  // recov.f90:2-47: recov1a or recov2 by iwvec
void bnd4(State& s);
void infchk(State& s);
void atmosphere1a(State& s);
void pminmax2b(State& s);
double cdtcfl4(State& s);
void step(State& s);

// initial conditions (oracle_ic.cpp)
void mdtorus1(State& s, uint64_t seed, double amp, double rin, double rmax, double beta,
              double kappa);
double callfish(double akm, double rmax);
double ic_uniform(uint64_t seed, uint64_t idx);
void tube_states(uint64_t seed, uint64_t tube, double gam, double q[2][9]);
void mdtube(State& s, uint64_t seed, uint64_t tube);

}  // namespace orc
