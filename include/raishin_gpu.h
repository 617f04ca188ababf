/* raishin_gpu.h -- C ABI of the B200-native RAISHIN GRMHD update.
 *
 * The reference (gustavo689/raishinsource) is Fortran 90: main.f90 drives one
 * RK3 step per pass of its time loop (main.f90:586-1151) by calling the
 * routines of rec.f90, calcha.f90, hll.f90, ct.f90, calsf.f90, rkt.f90,
 * recov.f90, bnd.f90, correction.f90 and cdtcfl.f90 on whole local blocks
 * uri(nv,is1:ie1,js1:je1,ks1:ke1).  This library replaces those calls with
 * sm_100a kernels on one GPU.  Every entry point is extern "C" with plain
 * pointers and sizes so that the Fortran driver can bind it with
 * ISO_C_BINDING (bind(C) interfaces with value integers and type(c_ptr) or
 * real(c_double) arrays).
 *
 * Conventions
 *  - Host arrays of primitives/conserved variables use the reference layout
 *    a(nv,i,j,k), nv = 9, variable fastest, then i, j, k, ghosts included
 *    (imax*jmax*kmax cells).  Flux arrays use ww(3,nv,i,j,k).
 *  - Every function returns an rg_status (0 = RG_OK).  Nothing aborts the
 *    process and no kernel traps; CUDA errors are returned as RG_ECUDA.
 *  - The library owns device memory.  Host buffers are only read or written
 *    during the call.  One host thread per rg_ctx.
 */
#ifndef RAISHIN_GPU_H
#define RAISHIN_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  RG_OK = 0,
  RG_EINVAL_CONFIG = 1, /* parameters outside what the kernels support */
  RG_ENOMEM_ADMIT = 2,  /* the run's device footprint does not fit */
  RG_ECUDA = 3,         /* a CUDA call failed (message in rg_last_error) */
  RG_ENR_CAP = 4,       /* an unbounded reference loop hit its cap (see stats) */
  RG_ENAN = 5,          /* non-finite primitives found */
  RG_ENOTFOUND = 6,     /* unknown run id */
  RG_EOVERFLOW = 7      /* a bounded device list overflowed (see stats) */
} rg_status;

typedef enum { RG_FP64 = 0, RG_MIXED = 1 } rg_precision;

/* One run's parameters: the runtime form of module pram (pram.f90:1-80). */
typedef struct rg_run_params {
  int imax, jmax, kmax; /* cells incl. ghosts; i = r, j = phi, k = theta (pram.f90:11) */
  int metric;           /* 1 Minkowski, 303 Kerr-Schild, 403 modified KS (pram.f90:67) */
  int ix1, ix2, ix3;    /* grid kinds: ix1 1 uniform / 2 log; ix3 1 uniform / 2 MKS theta */
  int irec;             /* 5 PPM, 6 MP5, 7 WENO5 (pram.f90:73) */
  int model;            /* 2 shock tube, 7 Fishbone-Moncrief torus (pram.f90:66) */
  int iter;             /* Newton-Raphson iteration cap, 5000 in the reference */
  double xmin, xmax, ymin, ymax, zmin, zmax; /* first/last cell centres (grid.f90) */
  double R0, hslope, akm, gam;
  double cfl, dmin, pmin, pmax, tmax, dtmin;
  int ibc[6][9]; /* iboux1in, iboux1ot, iboux2in, iboux2ot, iboux3in, iboux3ot */
  int guard;     /* 0 reference semantics.  Bit 1: first-order fallback for reconstructed face
                    states with rho<=0 or p<=0 (MP5/WENO5 undershoot at a torus surface);
                    bit 2: zero flux of the normal B component before flux-CT (Toth 2000),
                    which the reference's LLF term breaks (hll.f90:109).  Not in the reference. */
  int precision; /* rg_precision */
  int flags;     /* RG_FLAG_* bits */
  int ict;       /* constrained transport as pram.f90's ict (pram.f90:148-151, ct.f90:4-27):
                    0 none, 1 flux-CT (Toth 2000; the reference's setting), 2 modified flux-CT
                    (Gardiner & Stone 2005, mflct), 3 upwind flux-CT (upflct; FP64 precision
                    only; in rg_step_batch such a run takes its own launches; rg_calflx_static
                    refuses it).
                    Ghost width nm1 = nm0 + ict (main.f90:192-199). */
  int iwvec;     /* primitive recovery as pram.f90's iwvec (pram.f90:160-161, recov.f90:2-47):
                    1 (or 0) recov1a, the reference's setting; 2 recov2 (Mignone & McKinney,
                    one-variable W; FP64 precision only; in rg_step_batch such a run takes
                    its own launches). */
} rg_run_params;

/* rg_run_params.flags.  A direction of extent 2*nm1+1 (one interior cell)
 * whose ghost fills copy that cell (periodic or copy codes) and on which the
 * metric does not depend (phi; theta in Minkowski space) holds one state along
 * it: the reference's 2D phi slab and the transverse directions of a 1D tube.
 * The library stores such a direction as one plane and computes its interior
 * cell only, with results equal to computing every cell; uploaded primitives
 * must then be uniform along it.  RG_FLAG_FULL computes every cell instead. */
#define RG_FLAG_FULL 1

typedef struct rg_step_stats {
  long long steps;        /* full RK3 steps taken */
  long long recov_calls;  /* interior cells inverted */
  long long recov_nr2;    /* cells that needed the entropy Newton-Raphson (recov.f90:1022) */
  long long recov_fail;   /* cells that kept their previous primitives (recov.f90:1196) */
  long long recov_carry;  /* cells whose W guess came from the previous cell (recov.f90:810) */
  long long recov_cap;    /* capped W rescale loops (unbounded "go to 95", recov.f90:823) */
  long long floor_cap;    /* capped pminmax2b loops (unbounded "go to 95", correction.f90:870) */
  long long carry_overflow; /* carry cells beyond the device list capacity */
  double time;            /* simulation time at the loop top of the next step */
  double dt;              /* dt of the last step */
} rg_step_stats;

typedef struct rg_ctx rg_ctx;

/* Library / context ------------------------------------------------------ */
const char* rg_last_error(void);
/* A context on one device with its own stream.  The environment variables
 * RAISHIN_FLUX_TMA=0 and RAISHIN_UPDATE_TMA=0, read here, make the context's
 * runs use the face and stage-update kernels that read global memory
 * directly instead of the TMA-staged ones (for comparisons; the results are
 * the same operations on the same values). */
int rg_ctx_create(int device, rg_ctx** out);
int rg_ctx_destroy(rg_ctx* ctx);
int rg_sync(rg_ctx* ctx);
/* Marks on the context stream, for a host that keeps work queued while it
 * prepares more: rg_ctx_mark records a point in the stream in slot
 * 0..RG_MAX_MARKS-1 (re-marking a slot moves it); rg_ctx_wait_mark blocks
 * until the work before the mark has completed (block != 0) or only reports
 * it in *done (block = 0).  No counterpart in the reference. */
#define RG_MAX_MARKS 8
int rg_ctx_mark(rg_ctx* ctx, int slot);
int rg_ctx_wait_mark(rg_ctx* ctx, int slot, int block, int* done);
/* Run all later work of ctx on a caller-owned cudaStream_t (passed as void*) of
 * the same device, e.g. the stream of an enclosing framework; the context
 * then no longer owns or destroys a stream. */
int rg_ctx_set_stream(rg_ctx* ctx, void* stream);

/* Runs ------------------------------------------------------------------- */
/* Admit a run: checks the parameters, computes grid (grid.f90:2-266), metric
 * (coord.f90:5-146) and Christoffel symbols (coord.f90:1089-1321) and
 * allocates the device state.  RG_ENOMEM_ADMIT if it does not fit. */
int rg_run_admit(rg_ctx* ctx, const rg_run_params* p, int* run_id);
int rg_run_release(rg_ctx* ctx, int run);
/* Admission in two parts, for schedulers that prepare runs on other threads
 * while their context keeps the GPU busy: rg_prep_create checks the
 * parameters and computes the grid, metric and Christoffel symbols on the
 * host (no context, no GPU; any thread), rg_prep_ic_torus adds the torus
 * initial data of rg_run_ic_torus, and rg_run_admit_prep allocates the run on
 * the context and uploads both (the run then starts at time 0).  The
 * preparation stays valid for further admissions until rg_prep_destroy. */
typedef struct rg_prep rg_prep;
int rg_prep_create(const rg_run_params* p, rg_prep** out);
int rg_prep_ic_torus(rg_prep* prep, uint64_t seed, double amp, double rin, double rmax, double beta, double kappa);
int rg_run_admit_prep(rg_ctx* ctx, rg_prep* prep, int* run_id);
int rg_prep_destroy(rg_prep* prep);
/* Device bytes a run with these parameters needs (admission by footprint). */
int rg_run_footprint(const rg_run_params* p, size_t* bytes);

/* Initial data: Fishbone-Moncrief torus of mdtorus1 (mdgrmhd.f90:879-1654);
 * the pressure perturbation is p *= 1 + amp*(U-0.5) with U a counter-based
 * uniform keyed by (seed, cell).  Also sets time = 0 (main.f90:530-548). */
int rg_run_ic_torus(rg_ctx* ctx, int run, uint64_t seed, double amp, double rin, double rmax,
                    double beta, double kappa);
/* The same initial data computed on the device (the step's stream; the call
 * returns when it is in place): only per-index tables cross to the device,
 * so large 3D runs start without the host pass over every cell.  Agrees with
 * rg_run_ic_torus to a few units in the last place (CUDA's exp/log/pow in
 * the per-cell terms).  Not for theta slabs (RG_EINVAL_CONFIG). */
int rg_run_ic_torus_device(rg_ctx* ctx, int run, uint64_t seed, double amp, double rin, double rmax,
                           double beta, double kappa);
/* Initial data: seeded 1D RMHD Riemann problem number `tube` in the pattern
 * of mdshoctub (mdgrmhd.f90:56-118): a left state for i <= imax/2 and a right
 * state beyond, drawn from a counter-based uniform keyed by (seed, tube):
 * rho log-uniform in [0.1, 10], p log-uniform in [0.01, 100], |v| <= 0.9,
 * B^x in [0, 5] shared by both sides, B^y, B^z in [-5, 5].  Sets time = 0. */
int rg_run_ic_tube(rg_ctx* ctx, int run, uint64_t seed, uint64_t tube);
/* Host <-> device primitives, layout a(nv,i,j,k).  Upload also sets time = t0. */
int rg_run_upload_prims(rg_ctx* ctx, int run, const double* uri, double t0);
int rg_run_download_prims(rg_ctx* ctx, int run, double* uri);

/* The run's stored layout (a slab direction holds one plane): ncells stored
 * cells, jplanes and kplanes stored planes in j and k; rg_run_download_stored
 * copies the primitives as stored, variable v of stored cell
 * c = (i-1) + imax*((j-1) + jplanes*(k-1)) at v*ncells + c (9*ncells doubles),
 * j and k counted within the stored planes. */
int rg_run_layout(rg_ctx* ctx, int run, size_t* ncells, int* jplanes, int* kplanes);
int rg_run_download_stored(rg_ctx* ctx, int run, double* soa);

/* Advance nsteps full RK3 steps of main.f90:586-1147 on the device (CFL
 * reduction, three stages, ghost fill, floors).  Stops early once the loop-top
 * time exceeds tmax.  Asynchronous on the context stream unless stats != NULL.
 * A run with a slab direction steps as a batch of one (rg_step_batch), unless
 * it uses upwind flux-CT or recov2, which have no batched kernels. */
int rg_step(rg_ctx* ctx, int run, int nsteps, rg_step_stats* stats);
int rg_run_stats(rg_ctx* ctx, int run, rg_step_stats* stats);

/* Advance nruns runs together by nsteps full RK3 steps.  Runs with a slab
 * direction that share reconstruction, precision and slab class (see
 * RG_FLAG_FULL) form one batch, whose step is one launch per kernel kind over
 * a per-run tile table (persistent grid), captured once in a CUDA graph and
 * replayed each step: many small runs (2D slabs, 1D tubes).  Runs without a
 * slab direction (3D runs, which fill the GPU alone) and runs with upwind
 * flux-CT or recov2 take each step with their own launches, after the
 * batches of that step, exactly as rg_step steps them.  The launch shape (block width, cells per tile
 * along i, persistent grid size) is tuned per batch class and context: a new
 * class starts with a default shape and, at the first segment boundary after
 * 32 steps of its batch, times every candidate shape on trial steps from a
 * snapshot of the runs' state (which it restores) and keeps the fastest.
 * Each run's result equals its result stepped alone.  stats, if given,
 * receives nruns records.  Replaces the reference's one-run-per-job time loop
 * (main.f90:586-1151) for ensembles. */
int rg_step_batch(rg_ctx* ctx, const int* runs, int nruns, int nsteps, rg_step_stats* stats);
/* The shape of the batch of exactly these runs: block width of the cell
 * kernels, persistent blocks per SM (0: one block per tile), launches per
 * step, the step time measured by the tuner (ms; 0 while tuning is still
 * pending) and the cells along i of one tile of the cell kernels. */
int rg_batch_info(rg_ctx* ctx, const int* runs, int nruns, int* width, int* grid_factor, int* launches,
                  double* tuned_ms, int* tile_cells);

/* Kernel timing: rg_profile(ctx, 1) clears the counters and brackets every
 * following launch of rg_step with CUDA events on the context stream;
 * rg_profile_read returns accumulated milliseconds and launch counts per kind:
 * 0 cfl, 1 flux r, 2 flux phi, 3 flux theta, 4 flux-CT, 5 update (+ W carry),
 * 6 ghost fill, 7 floors, 8 scalar bookkeeping.  Launch counts are kept with
 * profiling off too.  No counterpart in the reference (cpu_time only). */
int rg_profile(rg_ctx* ctx, int enable);
int rg_profile_read(rg_ctx* ctx, double* ms, long long* launches, int nkinds);

/* Reference-interface entry points (arrays in the reference layout); each
 * runs the named routine(s) on the GPU for per-routine parity and swap-in.
 * Their arrays may be host memory or device memory (unified addressing: the
 * library copies with cudaMemcpyDefault), so a driver that keeps its arrays
 * on the device passes device pointers; scalar outputs (rg_cdtcfl's dtcfl)
 * are host memory. */
/* caluu1 (caluu.f90:2-126) */
int rg_caluu1(rg_ctx* ctx, int run, const double* uri, double* uu);
/* rec2 + calcha + hll + ct (rec.f90:2-142, calflx.f90:391-795, calcha.f90:2-126,
 * hll.f90:47-192, ct.f90:30-118): ww(3,nv,i,j,k) on the hll range */
int rg_calflx(rg_ctx* ctx, int run, const double* uri, double* ww);
/* The four calls of rg_calflx one at a time, as the reference makes them
 * (main.f90:807-831), for a driver that swaps in one routine at a time.
 * Face arrays come in sixes in the order ?l, ?r for ? = i, j, k, each
 * a(nv,i,j,k) holding at cell f the state of the face f+1/2 (rec.f90's
 * uriil(f) from cell f and uriir(f) from cell f+1); speeds come in the order
 * cmaxi, cmini, cmaxj, cminj, cmaxk, cmink, one value per cell.  Only the hll
 * range nm0..n-nm0 is written; rg_rec2 leaves its other entries 0, rg_hll and
 * rg_ct leave the other entries of ww as given.
 *  rg_rec2: rec2 with caluu3 and calflx3 (rec.f90:2-142): face primitives,
 *    and, unless NULL, face conserved variables and face fluxes;
 *  rg_calcha: calcha (calcha.f90:2-126, with cmink from the R state's plus
 *    speed, calcha.f90:107) from face primitives;
 *  rg_hll: hll (hll.f90:47-192) from face conserved variables, face fluxes and
 *    speeds, into ww(3,nv,i,j,k) in place;
 *  rg_ct: ct (ct.f90:4-27, the run's ict; guard bit 2 first zeroes the
 *    normal-field fluxes) on ww in place, with the primitives uri. */
int rg_rec2(rg_ctx* ctx, int run, const double* uri, double* face_prims, double* face_cons, double* face_flux);
int rg_calcha(rg_ctx* ctx, int run, const double* face_prims, double* cha);
int rg_hll(rg_ctx* ctx, int run, const double* face_cons, const double* face_flux, const double* cha, double* ww);
int rg_ct(rg_ctx* ctx, int run, const double* uri, double* ww);
/* recov1a (recov.f90:578-1228) on the interior: uu in (conserved), uri in/out */
int rg_recov(rg_ctx* ctx, int run, const double* uu, double* uri);
/* cdtcfl4 (cdtcfl.f90:2-129): dtcfl before the cfl factor */
int rg_cdtcfl(rg_ctx* ctx, int run, const double* uri, double* dtcfl);
/* bnd4 + infchk + atmosphere1a + pminmax2b (bnd.f90, correction.f90) on uri in/out */
int rg_bnd_floor(rg_ctx* ctx, int run, double* uri, const double* urio);
/* The same four one at a time (main.f90:860-878), uri in/out: bnd4
 * (bnd.f90:4-1058, single-rank branches; urio the previous state), infchk
 * (bnd.f90:1636-1824, for models 7-20), atmosphere1a (correction.f90:226-447,
 * models 7-15) and pminmax2b (correction.f90:744-999), each with the model
 * condition the reference's driver applies. */
int rg_bnd4(rg_ctx* ctx, int run, double* uri, const double* urio);
int rg_infchk(rg_ctx* ctx, int run, double* uri);
int rg_atmosphere1a(rg_ctx* ctx, int run, double* uri);
int rg_pminmax2b(rg_ctx* ctx, int run, double* uri);
/* caltenr + calsf (calsf.f90:6-151) on every cell: sf(2:5,i,j,k), 4 doubles
 * per cell */
int rg_calsf(rg_ctx* ctx, int run, const double* uri, double* sf);
/* One RK3 stage of rkt.f90 on the interior (is1+nm1..ie1-nm1 in each
 * direction) with akap?b = dt/dx?b (main.f90:766-779): stage 1 = rk2fst +
 * rk2adsff, unew = uh from ucur = uu; stage 2 = rk3snd + rk3adsfs, unew = us
 * from uo and ucur = uh; stage 3 = rk3trd + rk3adsft, unew = un from uo and
 * ucur = us (rkt.f90:2-42, 91-180, 183-215, 253-320).  ww(3,nv,i,j,k) with flux-CT
 * applied (rg_calflx), sf(2:5,i,j,k) (rg_calsf); uo may be NULL in stage 1;
 * unew is in/out (cells outside the interior keep their values). */
int rg_rkt(rg_ctx* ctx, int run, int stage, double dt, const double* ww, const double* uo, const double* ucur,
           const double* sf, double* unew);

/* Restart files byte-compatible with store1 / restar2 (restar.f90:5-88,
 * 273-346) for one rank: gfortran sequential unformatted records (4-byte
 * lengths) (myrank = 0, nd), (it0, ih0), (time), then per cell in (k, j, i)
 * order uu, u0, uri, uri0 (9 doubles each).  rg_run_store writes the run's
 * current primitives, their conserved variables (caluu1) and the initial state
 * uri0 (NULL: the current primitives) with its conserved variables;
 * rg_run_restore reads a file of this grid, uploads uri with time = the
 * stored time (icres = 1, main.f90:560-571) and returns it0, ih0, nd and,
 * if uri0 is not NULL, the stored initial primitives. */
int rg_run_store(rg_ctx* ctx, int run, const char* path, int it0, int ih0, int nd, const double* uri0);
int rg_run_restore(rg_ctx* ctx, int run, const char* path, int* it0, int* ih0, int* nd, double* uri0);

/* Snapshot file of output1 (restar.f90:91-185) for one rank holding the
 * whole grid, byte-compatible with structrNNNN-MMMM.outdat (the caller passes
 * the file name): gfortran sequential unformatted records with 4-byte length
 * markers, (time, myrank, npe), (is, ie, js, je, ks, ke) = (1, imax, 1,
 * jmax, 1, kmax), then for i, j, k (k fastest) the 13 doubles x1(i), x2(j),
 * x3(k), uri(1:9,i,j,k), detg(i,j,k); the coordinates are the MKS x?b for
 * metric 403 and x? otherwise (main.f90:711-717), time the loop-top time.
 * The records are formatted on the device and copied chunk by chunk into
 * pinned host memory, overlapping the file writes. */
int rg_run_output(rg_ctx* ctx, int run, const char* path, int myrank, int npe);

/* Accretion rates through the inner edge of the interior (the radial face
 * nm1+1/2, just outside the horizon for the torus grids): mdot = -sum of the
 * radial flux of sqrt(-g) rho u^r over the interior (phi, theta) faces times
 * dx2*dx3, edot the same of the energy variable sqrt(-g)(T^r_t + rho u^r)
 * (calflx.f90:391-528), from FP64 fluxes of the run's current primitives.
 * The reference has no such diagnostic; it is how the mixed-precision path's
 * effect on the accretion is measured. */
int rg_run_horizon_flux(rg_ctx* ctx, int run, double* mdot, double* edot);
/* The same rates through the radial face iface+1/2 (iface in nm0..imax-nm0,
 * 1-based cell index; rg_run_horizon_flux is iface = nm1): a shell at any
 * radius, e.g. inside the FP32 region of a mixed run (r > 2 r_H), where the
 * mixed path's effect on the flow is measured. */
int rg_run_radial_flux(rg_ctx* ctx, int run, int iface, double* mdot, double* edot);

/* Corner-centred divergence of sqrt(-g) B of the run's current primitives:
 * at each corner between interior cells, D = sum over d of the four
 * differences of sqrt(-g) B^d across the corner along d, divided by 4 dx_d.
 * Toth's flux-CT (ct.f90:30-118) keeps D constant when the flux of the normal
 * field component is zero (guard bit 2); the reference's LLF term
 * (hll.f90:109-111) lets it drift.  *divb_max = max |D| (NaN if any D is);
 * *b_scale = max |sqrt(-g) B^d| / dx_d over the same cells, the natural unit
 * of D.  No counterpart in the reference. */
int rg_run_divb(rg_ctx* ctx, int run, double* divb_max, double* b_scale);

/* Derived quantities of the output converter (convert_vtk2dn1.f90:254-371,
 * with transmks2ks1 / transks2bl1, convert_vtk2dn1.f90:1399-1554) from the
 * run's current primitives, 7 doubles per point: the Lorentz factors of the
 * Boyer-Lindquist ZAMO (gfa) and of the static observer at infinity (gfb),
 * b^2, the Bernoulli parameter -h u_t, and the BL velocity u^i + gfa
 * beta^i/alpha (i = r, phi, theta); inside r_H gfa = gfb = 1 and the velocity
 * is 0.  jslice = 0: every cell, out[7*((i-1) + imax*((j-1) + jmax*(k-1))) + f];
 * jslice = j: the meridional plane at phi index j (the converter's 2D cut),
 * out[7*((i-1) + imax*(k-1)) + f], only that plane crossing to the host.
 * Kerr metrics (303, 403) only.  Replaces the per-rank files read by the
 * converter; the VTK writing itself stays with the caller. */
int rg_run_derived(rg_ctx* ctx, int run, int jslice, double* out);

/* The power function of the uncontracted build (rg_pow, include/rg_pow.h),
 * evaluated on the device: out[i] = x[i]**y[i] for n host values.  A host
 * program that evaluates rg_pow itself gets the same bits; this entry point
 * lets it check that.  The reference's x**y is gfortran's call of the C
 * library's pow (calflx.f90:474, caluu.f90:303, recov.f90:1044-1186). */
int rg_pow_eval(rg_ctx* ctx, const double* x, const double* y, double* out, size_t n);

/* Allocation-free variant of rg_calflx.  No counterpart in the reference.
 * For host programs that cannot let the library call cudaMalloc when they need
 * the fluxes: a framework or driver whose device memory comes only from its
 * own pool or arena, where an allocation behind its back would synchronise the
 * device and take memory its pool does not account for.  The caller passes
 * device buffers: d_prims, the primitives in structure-of-arrays order
 * (variable v of cell c at v*N + c, c = (i-1) + imax*((j-1) + jmax*(k-1))),
 * and d_ww, 27*N doubles receiving ww(d,v) of cell c at ((d-1)*9 + v)*N + c on
 * the hll range, with flux-CT applied on its range.  The flux-CT intermediate
 * lives in a file-scope device array that holds grids of at most 262144 cells
 * (larger grids return RG_EINVAL_CONFIG); every GPU that loads the library
 * keeps that array (about 12.6 MB) until exit.  The run's geometry, allocated
 * by rg_run_admit beforehand, is read; the call itself allocates and frees
 * nothing, with one exception: a device's first call looks up the array's
 * device address (cudaGetSymbolAddress), which with CUDA's lazy module loading
 * may load the module and so allocate the array.  Make that first call during
 * set-up, before any stream capture and before the program restricts itself to
 * its own pool.  All calls share the one array and each starts by clearing
 * it: calls whose work overlaps on the GPU (other contexts or streams) race,
 * so callers must serialise them.  The call returns after its work has
 * completed on the context stream. */
int rg_calflx_static(rg_ctx* ctx, int run, const double* d_prims, double* d_ww);

#ifdef __cplusplus
}
#endif
#endif /* RAISHIN_GPU_H */
