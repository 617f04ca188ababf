// rg_host.h -- host-side setup shared by the C ABI: grid/metric construction
// and initial data.
#pragma once
#include <cstdint>
#include <vector>

#include "../../include/raishin_gpu.h"
#include "rg_types.h"

namespace rg {

// One grid direction (grid.f90): values at 1-based index, entries 0 and n+1 unused.
struct Axis {
  std::vector<double> x, xa, xb, xab, dx, dxb;
};


struct HostGeom {
  Axis ax[3];                      // i = r, j = phi, k = theta
  size_t nik = 0;
  bool compact_ok = false;         // every point has the (t,r,phi)+theta block structure
  std::vector<double> mc, mi, mk;  // kMetComps components per (i,k) point, SoA
  std::vector<double> chr;         // 64 components per point, SoA
};

// krow > 0 computes the single theta row krow (theta slab in Minkowski space).
// Ghost widths (main.f90:179-199): nm0 = 2 for the second-order schemes
// (irec 1-3, 11-13), 3 for the five-point schemes, 4 for PPM; constrained
// transport adds ict layers.
inline int ghost_nm0(int irec) {
  return (irec == 1 || irec == 2 || irec == 3 || irec == 11 || irec == 12 || irec == 13) ? 2 : (irec == 5 ? 4 : 3);
}
inline int ghost_nm1(const rg_run_params& p) { return ghost_nm0(p.irec) + p.ict; }

void build_geometry(const rg_run_params& p, HostGeom& g, int krow = 0);

// mdtorus1 (mdgrmhd.f90:879-1654) into SoA primitives prim[v*N + c].
void torus_ic(const rg_run_params& p, const HostGeom& g, uint64_t seed, double amp, double rin, double rmax,
              double beta, double kappa, std::vector<double>& prim, bool plane_only = false);

// Inputs of the device torus construction (rg_ic.cu), evaluated on the host
// with the libm calls torus_ic makes: per radial index r, the floors
// dmin r^-1.5 and pmin (gam-1) r^-2.5 and the corner spacing h1; per theta
// index theta, its clamped sine and cosine, bl_cov's clamped sine and cosine,
// the MKS factor 1 + (1-hslope) cos(2 theta_MKS) and the spacing h3; and the
// run's scalars (angular momentum, ln h at the inner edge, polar edges).
struct TorusTables {
  std::vector<double> tab;  // kIcTabI planes of imax, then kIcTabK planes of kmax (rg_types.h)
  double ell = 0, h_in = 0, edge0 = 0, edge1 = 0;
};
void torus_tables(const rg_run_params& p, const HostGeom& g, double rin, double rmax, TorusTables& out);

// Left/right primitive states of the seeded Riemann tube `tube` (mdshoctub pattern).
void tube_states(uint64_t seed, uint64_t tube, double gam, double state[2][9]);

}  // namespace rg
