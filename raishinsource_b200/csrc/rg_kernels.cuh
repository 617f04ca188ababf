// rg_kernels.cuh -- kernel declarations and launch helpers shared by the C ABI.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "rg_types.h"

namespace rg {

// Buffers of one run on the device.
struct DevBufs {
  double* P[3];   // rotating primitive buffers, 9*N each (SoA)
  double* F[3];   // raw LLF face fluxes per direction, 9*N each
  double* CT;     // 6*N flux-CT averaged induction fluxes
  double* stage;  // 9*N staging buffer (layout conversion, per-routine entry points)
  double* stage2; // 9*N second staging buffer
  double* ctd;    // 6*N upwinded EMF differences of upflct (ict 3 only)
  double* r2;     // recov2 runs: 22*N of stage scratch (Uc 9N, SF 4N, Unew 9N)
};

cudaError_t launch_cfl(const DevRun& r, const double* P, cudaStream_t s);
cudaError_t launch_step_begin(const DevRun& r, cudaStream_t s);
cudaError_t launch_dt(const DevRun& r, cudaStream_t s);
cudaError_t launch_step_end(const DevRun& r, cudaStream_t s);
cudaError_t launch_flux(const DevRun& r, int dir, const double* P, double* F, cudaStream_t s);
// Faces (PPM, MP5, WENO5, WENO-Z, WENO-M) of a run stored in full (no slab
// direction, imax a multiple of 4) with the stencil staged in shared memory
// by TMA: tmap64 is the
// CUtensorMap of the FP64 primitive buffer, tmap32 that of P32 (mixed runs;
// 4D: i, j, k, v; box flux_tma_box(dir, element bytes, irec))
bool flux_tma_eligible(const DevRun& r);
void flux_tma_box(int dir, int elem_bytes, int irec, unsigned box[4]);
// tmapm: the FP64 face-metric map of direction dir (3D: i, k, component; box
// flux_tma_met_box), staged with the stencil
cudaError_t launch_flux_tma(const DevRun& r, int dir, const void* tmap64, const void* tmap32, const void* tmapm,
                            double* F, cudaStream_t s);
void flux_tma_met_box(unsigned box[3]);
// P: the stage's primitives (upflct's upwinding reads their velocities)
cudaError_t launch_ct(const DevRun& r, const double* P, const double* F1, const double* F2, const double* F3,
                      double* CT, cudaStream_t s);
// umaps: the run's five update tensor maps (F1, F2, F3, CT, U^n; CUtensorMap[5])
// for the TMA-staged update where update_tma_eligible, else nullptr;
// umaps_mix: those of a mixed run's FP32 region (F32[0..2], CT32, U^n) where
// update_tma_mix_eligible, else nullptr
cudaError_t launch_update(const DevRun& r, int stage, const double* Pn, const double* Pc, double* Pw,
                          const double* F1, const double* F2, const double* F3, const double* CT, cudaStream_t s,
                          const void* umaps = nullptr, const void* umaps_mix = nullptr);
// TMA-staged FP32 region of a mixed run's update: stored in full, recov1a, imax a multiple of 4
bool update_tma_mix_eligible(const DevRun& r);
void update_tma_mix_box(int which, unsigned box[4]);
// TMA-staged update: runs stored in full, FP64, recov1a, imax even
bool update_tma_eligible(const DevRun& r);
// box of update tensor map `which` (0 F1, 1 F2, 2 F3, 3 CT, 4 U^n) as (x, y, z, variables)
void update_tma_box(int which, unsigned box[4]);
// shared-memory attributes of the staged update kernels (on the current device)
cudaError_t prepare_update_tma();
cudaError_t launch_bc(const DevRun& r, double* P, const double* Po, cudaStream_t s);
cudaError_t launch_floor(const DevRun& r, double* P, cudaStream_t s);
// one floor routine alone: part 1 infchk, 2 atmosphere1a, 4 pminmax2b
cudaError_t launch_floor_part(const DevRun& r, int part, double* P, cudaStream_t s);
// per-routine entry points
cudaError_t launch_recov_only(const DevRun& r, const double* U, const double* Pold, double* Pw, cudaStream_t s);
// One RK stage of a recov2 run after its fluxes and CT: the CT values are
// written into F1-F3; Uc, SF, Unew are 9N, 4N and 9N of scratch.
cudaError_t launch_stage_recov2(const DevRun& r, int stage, const double* Pc, double* Pw, double* F1, double* F2,
                                double* F3, const double* CT, double* Uc, double* SF, double* Unew, cudaStream_t s);
cudaError_t launch_p2c(const DevRun& r, const double* P, double* U, cudaStream_t s);
cudaError_t launch_calsf(const DevRun& r, const double* P, double* SF, cudaStream_t s);
// per-routine rec2 / calcha / hll / ct on the full layout: q/u/w[0] (L) and
// [1] (R) are the face primitives, conserved variables and fluxes of one
// direction (9 planes of N each); F receives the LLF fluxes (rec2: scratch)
cudaError_t launch_rec2(const DevRun& r, int dir, const double* P, double* F, double* const q[2], double* const u[2],
                        double* const w[2], cudaStream_t s);
cudaError_t launch_calcha(const DevRun& r, int dir, const double* QL, const double* QR, double* cmax, double* cmin,
                          cudaStream_t s);
cudaError_t launch_hll(const DevRun& r, int dir, const double* UL, const double* UR, const double* WL,
                       const double* WR, const double* CX, const double* CN, double* F, cudaStream_t s);
// m values per cell (value fastest) <-> m planes of N
cudaError_t launch_aos_planes(double* aos, double* planes, size_t N, int m, bool to_planes, cudaStream_t s);
// ww(3,nv,i,j,k) <-> flux planes F1..F3 (9 planes of N each)
cudaError_t launch_ww_layout(double* ww, double* F1, double* F2, double* F3, size_t N, bool to_planes,
                             cudaStream_t s);
// guard bit 2's zero normal-field fluxes and the CT values into the flux planes
cudaError_t launch_ct_apply(const DevRun& r, const double* CT, double* F1, double* F2, double* F3, cudaStream_t s);
// corner-centred div(sqrt(-g) B) of P over the interior: red[0] = max |D|,
// red[1] = max |sqrt(-g) B^d| / dx_d (bit patterns of doubles)
cudaError_t launch_divb(const DevRun& r, const double* P, unsigned long long* red, cudaStream_t s);
// records rec0 .. rec0+nrec-1 of output1's data (restar.f90:160-167) as the file's bytes, 112 per record
cudaError_t launch_output1(const DevRun& r, const double* P, const double* cx, const double* cy, const double* cz,
                           size_t rec0, size_t nrec, unsigned* out, cudaStream_t s);
cudaError_t launch_derived(const DevRun& r, const double* P, const double* geo_i, const double* geo_k, double akm,
                           int jslice, double* out, cudaStream_t s);
cudaError_t launch_rkt(const DevRun& r, int stage, const double* W1, const double* W2, const double* W3,
                       const double* Uo, const double* Uc, const double* SF, double* Unew, double dt, cudaStream_t s);
// reference layout a(nv,i,j,k) of the full array <-> the run's stored SoA
// (bad, if given, is set non-zero when the data are not uniform along a slab direction)
cudaError_t launch_aos_to_soa(const DevRun& r, const double* aos, double* soa, int* bad, cudaStream_t s);
cudaError_t launch_soa_to_aos(const DevRun& r, const double* soa, double* aos, cudaStream_t s);
cudaError_t launch_fill(double* p, double v, size_t n, cudaStream_t s);
int n_flux_launches(const DevRun& r);
int n_ct_launches(const DevRun& r);
int n_update_launches(const DevRun& r);
int n_bc_launches(const DevRun& r);
cudaError_t launch_to_f32(const double* a, float* b, size_t n, cudaStream_t s);
// derived metric fields of the three caches and the radial floor profiles (run setup)
cudaError_t launch_geom_derive(const DevRun& r, double* mc, double* mi, double* mk, double* fl_de, double* fl_pr,
                               cudaStream_t s);

// Fishbone-Moncrief torus initial data on the device (rg_ic.cu).
struct IcTorusArgs {
  const double* tab;        // TorusTables::tab on the device
  unsigned long long* red;  // two reduction words: rho_max bits, ordered key of beta_min
  uint64_t seed;
  double amp, rin, kappa, beta, akm, ell, h_in, edge0, edge1;
  int metric, ix1, ix3;
  int phi_slab, slab_j;     // jmax == 2*nm1+1: the draw is keyed by the plane slab_j = nm1+1
};
cudaError_t launch_ic_torus(const DevRun& r, const IcTorusArgs& a, double* P, cudaStream_t s);

// Batched steps of runs of one class (rg_batch.cuh).
struct BatchPlan;
int batch_build(const std::vector<DevRun>& runs, int width, int group, BatchPlan** out);
void batch_destroy(BatchPlan* B);
int batch_launch_count(const BatchPlan* B);
void batch_set_grid(BatchPlan* B, int factor);
cudaError_t batch_issue(const BatchPlan* B, int idx, cudaStream_t s);
cudaError_t batch_step(const BatchPlan* B, cudaStream_t s);
int batch_launch_kind(const BatchPlan* B, int idx, int* dir);

}  // namespace rg
