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
void build_geometry(const rg_run_params& p, HostGeom& g, int krow = 0);

// mdtorus1 (mdgrmhd.f90:879-1654) into SoA primitives prim[v*N + c].
void torus_ic(const rg_run_params& p, const HostGeom& g, uint64_t seed, double amp, double rin, double rmax,
              double beta, double kappa, std::vector<double>& prim, bool plane_only = false);

// Left/right primitive states of the seeded Riemann tube `tube` (mdshoctub pattern).
void tube_states(uint64_t seed, uint64_t tube, double gam, double state[2][9]);

}  // namespace rg
