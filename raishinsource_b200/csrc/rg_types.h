// rg_types.h -- device-side description of one run (passed to every kernel by
// value) and the host-side run record.
#pragma once
#include <cstddef>
#include <cstdint>

#include "../../include/raishin_gpu.h"

#ifdef __CUDACC__
#define RG_HD __host__ __device__
#else
#define RG_HD
#endif

namespace rg {

constexpr int NV = 9;

// Metric cache components per (i,k) point: the host stores the first
// kMetBase (gcov, gcon blocks, sqrt(-g)); k_met_derive fills the rest.
constexpr int kMetBase = 18;
constexpr int kMetComps = 26;

// Planes of the torus initial-data table (TorusTables): per radial index,
// then per theta index.
enum IcTabI { IC_R = 0, IC_DE, IC_PR, IC_H1, kIcTabI };
enum IcTabK { IC_TH = 0, IC_STH, IC_CTH, IC_SBL, IC_CBL, IC_HDEN, IC_H3, kIcTabK };

// Device scalars of a run (one small block of device memory).
struct Scal {
  unsigned long long dtcfl_bits;  // min-reduced CFL time step (bits of a positive double)
  double dt;                      // cfl * dtcfl of the current step
  double time;                    // loop-top time of the current step
  double timeh;                   // time + dt
  int active;                     // 0 once time > tmax: every kernel of the step returns early
  int carry_count;                // cells queued for the loop-order W carry fix-up
  int cur;                        // index of P^n among the run's three primitive buffers
  int strag_count;                // cells whose primitive recovery was deferred this stage
};

// Counters (device, atomically accumulated).
enum Counter {
  C_STEPS = 0, C_RECOV, C_NR2, C_FAIL, C_CARRY, C_CAP, C_FLOORCAP, C_CARRY_OVF,
  C_TMAWAIT,  // blocks whose TMA wait ran out (k_flux_tma); never expected
  C_NCOUNTERS
};

// Everything a kernel needs, by value.  Arrays are structure-of-arrays with
// the cell index c = (i-1) + sj*(j-1) + sk*(k-1) (1-based i, j, k; sj = imax,
// sk = imax*jmax unless a direction is a slab) and variable v at offset v*N.
// Metric caches are per (i,k) point q = (i-1) + imax*(k-1), kMetComps
// components each (see MetT in rg_device.cuh).
struct DevRun {
  int imax, jmax, kmax;  // logical extents incl. ghosts (the reference's array bounds)
  // Slab directions.  A direction of extent 2*nm1+1 (one interior cell) whose
  // boundaries copy the interior cell (periodic or copy codes) and on which the
  // metric does not depend holds the same state in every one of its cells after
  // each ghost fill: the reference's 2D phi slab and the transverse directions
  // of a 1D tube.  Such a direction is stored as a single plane; kernels compute
  // only its interior index jfix/kfix and read neighbours in it at stride 0.
  int jfix, kfix;        // the computed index of a slab direction, 0 otherwise
  int kmet;              // metric caches hold one theta row (a theta slab), 0 otherwise
  int jpl, kpl;          // stored planes in j and k (1 along a slab direction)
  size_t sj, sk;         // storage strides of j and k neighbours (0 along a slab direction)
  int nm0, nm1;
  int irec, model, guard, iter;
  int mixed;             // 1: FP32 reconstruction/fluxes/CT/RK combine (RG_MIXED)
  int gkind;             // x**gam form: 1 gam == 4/3, 2 gam == 5/3 (cube roots), 0 pow
  int i_fp64;            // radial cells 1..i_fp64 (r < 2 r_H) keep FP64 in the mixed path
  int nmax_cfl;          // nm1*2 + (nm1-1) (cdtcfl.f90:38)
  size_t N;              // stored cells (imax * jpl * kpl)
  size_t nik;            // (i,k) points of the metric caches (imax for a theta slab)
  double gam, cfl, dmin, pmin, pmax, tmax;
  const double* mc;      // metric at cell centres (also the phi faces)
  const double* mi;      // metric at the r faces x1a(i)
  const double* mk;      // metric at the theta faces x3a(k)
  const double* chr;     // Christoffel symbols, 64 per point: christ(l,m,n) at l+4m+16n
  const double* x1;      // cell-centre r, index i-1
  const double* dx1b;    // dx1b(i) at index i-1 (grid.f90:134-141)
  const double* dx2b;
  const double* dx3b;
  const double* x2;      // phi centres (PPM contact detection)
  const double* x3;      // theta centres
  const double* fl_de;   // density floor dmin * x1(i)**(-1.5) (correction.f90:897), index i-1
  const double* fl_pr;   // pressure floor (gam-1) * pmin * x1(i)**(-2.5) (correction.f90:898), index i-1
  double* Un;            // conserved variables of the step's initial primitives (9*N), written in stage 1
  // FP32 arrays of the mixed path (null for FP64 runs)
  const float* mc32;     // FP32 copies of the metric caches
  const float* mi32;
  const float* mk32;
  const float* chr32;    // FP32 copy of the Christoffel symbols
  float* P32;            // FP32 copy of the current primitives (written by the floor pass)
  float* F32[3];         // FP32 face fluxes per direction, 9*N each
  float* CT32;           // FP32 flux-CT values, 6*N
  const double* dx1s;    // rec2's shifted dx1b: dummy dx1b(i) = actual dx1b(i-1), index i-1
  const double* dx2s;
  const double* dx3s;
  // Limiter coefficients per direction d (MC, minmod, LimO3, MVL, Koren,
  // CENO): ten planes of n_d values at index m-1 of the cell's coordinate
  // spacings, as limiter_state and ceno_state in rg_recon.cuh read them.
  const double* lim[3];
  int ict;               // constrained transport: 0 none, 1 flux-CT, 2 modified flux-CT, 3 upwind flux-CT
  double* ctd;           // ict 3: six planes (6*N) of upflct's upwinded EMF differences
  int iwvec;             // primitive recovery: 1 recov1a, 2 recov2
  int ibc[6][9];
  double* P[3];          // the run's rotating primitive buffers (P^n = P[scal->cur])
  double* F[3];          // FP64 face fluxes per direction
  double* CT;            // FP64 flux-CT values
  Scal* scal;
  unsigned long long* cnt;
  int* carry_list;       // interior cells queued for the W carry fix-up
  int* carry_sorted;     // the same cells in loop order (carry_cap entries of scratch)
  int carry_cap;
  int* strag_list;       // interior cells whose Newton-Raphson passed kDeferIter iterations
  int strag_cap;

  RG_HD size_t cell(int i, int j, int k) const {
    return (size_t)(i - 1) + sj * (size_t)(j - 1) + sk * (size_t)(k - 1);
  }
  // index of cell (i,j,k) in the reference's full array (imax*jmax*kmax cells)
  RG_HD size_t cell_full(int i, int j, int k) const {
    return (size_t)(i - 1) + (size_t)imax * ((size_t)(j - 1) + (size_t)jmax * (size_t)(k - 1));
  }
  // metric-cache point of (i, k); a theta slab (Minkowski only, so the metric
  // is the same at every k) keeps one row, also in the full-layout view
  RG_HD size_t ik(int i, int k) const { return (size_t)(i - 1) + (kmet ? 0 : (size_t)imax * (size_t)(k - 1)); }
};

}  // namespace rg
