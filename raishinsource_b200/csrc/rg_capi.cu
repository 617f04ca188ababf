// rg_capi.cu -- the C ABI of include/raishin_gpu.h: contexts, run admission
// by device footprint, host<->device layout conversion, the device-resident
// RK3 step driver and the per-routine entry points.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <iterator>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/raishin_gpu.h"
#include "../../include/rg_pow.h"
#include "rg_host.h"
#include "rg_kernels.cuh"
#include "rg_types.h"

using namespace rg;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define RG_CUDA(call)                                                                                  \
  do {                                                                                                 \
    cudaError_t e_ = (call);                                                                           \
    if (e_ != cudaSuccess) return fail(RG_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

constexpr int kCarryCap = 1 << 16;

struct Run {
  rg_run_params p{};
  DevRun d{};
  DevBufs b{};             // stored-layout buffers of the step (stage/stage2 unused)
  DevBufs fb{};            // full-layout buffers of the per-routine entry points (allocated on first use)
  bool fb_ready = false;
  double* aos = nullptr;   // 9*Nfull staging buffer in the reference layout (allocated on first use)
  double* unew = nullptr;  // 9*Nfull output of rg_rkt (allocated on first use)
  double* wwaos = nullptr; // 27*Nfull staging of ww(3,nv,i,j,k) (allocated on first use)
  // scalar block and counters of the per-routine entry points, so that those
  // calls never touch the run's own time state, buffer rotation or statistics
  Scal* fscal = nullptr;
  unsigned long long* fcnt = nullptr;
  int* bad = nullptr;      // device flag: uploaded data not uniform along a slab direction
  size_t nfull = 0;        // imax*jmax*kmax
  int cur = 0;             // index of P^n in b.P
  std::vector<void*> allocs;
  size_t bytes = 0;
  HostGeom geom;
  // TMA tensor maps of the primitive buffers b.P[buffer] for the staged face
  // kernel, per direction (flux_tma_box); tma is set when all nine exist
  CUtensorMap tmap[3][3];
  CUtensorMap tmap32[3];   // the FP32 copy P32 of a mixed run, per direction
  CUtensorMap tmapm[3];    // the FP64 face metric per direction (mi, mc, mk; flux_tma_met_box)
  bool tma = false;
  // tensor maps of the staged update (F1, F2, F3, CT, U^n; update_tma_box) and
  // of a mixed run's FP32 region (F32[0..2], CT32, U^n; update_tma_mix_box)
  CUtensorMap umap[5];
  CUtensorMap umap32[5];
  bool utma = false;
  bool utma32 = false;
};

}  // namespace

// Host-side preparation of a run (geometry, initial data), built without a context.
struct rg_prep {
  rg_run_params p{};
  int krow = 0;        // geometry of one theta row (theta slab)
  bool plane = false;  // initial data of the interior phi plane only (phi slab)
  HostGeom geom;
  std::vector<double> ic;  // full-layout SoA primitives, empty if none
};

// Kernel kinds timed by the profiling mode (rg_profile).
enum Kind { K_CFL = 0, K_FLUX1, K_FLUX2, K_FLUX3, K_CT, K_UPDATE, K_BC, K_FLOOR, K_SCALAR, K_NKINDS };

// A batched step of one class of runs: its tile plan, the tuned launch
// shape and the CUDA graph of one step.
struct BatchEntry {
  std::vector<int> ids;        // member runs, sorted
  BatchPlan* plan = nullptr;
  cudaGraphExec_t graph = nullptr;
  int width = 128, group = 1, grid_factor = 0;
  double tuned_ms = 0.0;       // step time of the chosen shape
  bool tune_pending = false;   // the class has no tuned shape yet: tune once kTuneAfter steps have run
  long long steps_run = 0;     // batched steps taken by this entry
};

struct rg_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::map<int, Run*> runs;
  std::map<std::vector<int>, BatchEntry*> batches;
  struct Tuned { int width, group, grid_factor; double ms; };
  std::map<long long, Tuned> tuned;  // batch class -> shape chosen by the tuner and its step time
  int next_id = 1;
  long long launches[K_NKINDS] = {};   // kernel launches issued, per kind
  bool prof = false;                   // bracket every launch with CUDA events
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
  std::vector<cudaEvent_t> pool;
  double ms[K_NKINDS] = {};
  bool own_stream = true;              // false after rg_ctx_set_stream
  cudaEvent_t marks[RG_MAX_MARKS] = {};  // rg_ctx_mark / rg_ctx_wait_mark
  bool tma = true;                     // staged face kernel where a run allows it (RAISHIN_FLUX_TMA=0: off)
  bool utma = true;                    // staged update kernel where a run allows it (RAISHIN_UPDATE_TMA=0: off)
};

namespace {

int dalloc(Run* R, void** ptr, size_t bytes) {
  cudaError_t e = cudaMalloc(ptr, bytes);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return fail(RG_ENOMEM_ADMIT, std::string("cudaMalloc failed: ") + cudaGetErrorString(e));
  }
  R->allocs.push_back(*ptr);
  R->bytes += bytes;
  return RG_OK;
}

void free_run(Run* R) {
  for (void* p : R->allocs) cudaFree(p);
  R->allocs.clear();
  delete R;
}

// cuTensorMapEncodeTiled from the driver (no link-time dependency on libcuda).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
    else
      (void)cudaGetLastError();
  });
  return fn;
}

// Tensor maps of the three primitive buffers (and of P32 for a mixed run) as
// 4D arrays (i, j, k, v) with the boxes of the staged face kernel, and of the
// update's flux, flux-CT and U^n arrays with the boxes of the staged update;
// a run they do not fit keeps the generic kernels.
void make_tmaps(Run* R) {
  R->tma = false;
  R->utma = false;
  R->utma32 = false;
  const DevRun& d = R->d;
  EncodeTiledFn enc = encode_tiled();
  if (!enc) return;
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  auto encode = [&](CUtensorMap* tm, void* base, int eb, int nv, const unsigned box[4]) {
    const cuuint64_t dims[4] = {(cuuint64_t)d.imax, (cuuint64_t)d.jmax, (cuuint64_t)d.kmax, (cuuint64_t)nv};
    const cuuint64_t strides[3] = {(cuuint64_t)d.imax * eb, (cuuint64_t)d.imax * d.jmax * eb, (cuuint64_t)d.N * eb};
    const cuuint32_t bx[4] = {box[0], box[1], box[2], box[3]};
    return enc(tm, eb == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, base, dims,
               strides, bx, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
  };
  if (flux_tma_eligible(d)) {
    bool ok = true;
    for (int dir = 1; dir <= 3 && ok; ++dir) {
      unsigned box[4];
      flux_tma_box(dir, 8, d.irec, box);
      for (int b = 0; b < 3 && ok; ++b) ok = encode(&R->tmap[b][dir - 1], R->b.P[b], 8, 9, box);
      if (ok && d.mixed) {
        flux_tma_box(dir, 4, d.irec, box);
        ok = encode(&R->tmap32[dir - 1], d.P32, 4, 9, box);
      }
    }
    // face metric (i, k, component): kMetComps components nik apart
    const double* met[3] = {d.mi, d.mc, d.mk};
    unsigned mb[3];
    flux_tma_met_box(mb);
    for (int dir = 1; dir <= 3 && ok; ++dir) {
      const cuuint64_t dims[3] = {(cuuint64_t)d.imax, (cuuint64_t)d.kmax, (cuuint64_t)kMetComps};
      const cuuint64_t strides[2] = {(cuuint64_t)d.imax * 8, (cuuint64_t)d.nik * 8};
      const cuuint32_t bx[3] = {mb[0], mb[1], mb[2]};
      ok = enc(&R->tmapm[dir - 1], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double*>(met[dir - 1]), dims,
               strides, bx, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
    }
    R->tma = ok;
  }
  if (update_tma_eligible(d) && prepare_update_tma() == cudaSuccess) {
    void* bases[5] = {R->b.F[0], R->b.F[1], R->b.F[2], R->b.CT, d.Un};
    bool ok = true;
    for (int w = 0; w < 5 && ok; ++w) {
      unsigned box[4];
      update_tma_box(w, box);
      ok = encode(&R->umap[w], bases[w], 8, (int)box[3], box);
    }
    R->utma = ok;
  } else {
    (void)cudaGetLastError();
  }
  if (update_tma_mix_eligible(d)) {
    void* bases[5] = {d.F32[0], d.F32[1], d.F32[2], d.CT32, d.Un};
    bool ok = true;
    for (int w = 0; w < 5 && ok; ++w) {
      unsigned box[4];
      update_tma_mix_box(w, box);
      ok = encode(&R->umap32[w], bases[w], w == 4 ? 8 : 4, (int)box[3], box);
    }
    R->utma32 = ok;
  }
}

// Ghost widths of the reconstruction (main.f90:179-190): nm0 = 2 for the
// second-order schemes, 3 for the five-point schemes, 4 for PPM; constrained
// transport adds ict layers, nm1 = nm0 + ict (main.f90:192-199).
int nm0_of(int irec) { return ghost_nm0(irec); }
int nm1_of(const rg_run_params* p) { return ghost_nm1(*p); }

int check_params(const rg_run_params* p) {
  if (!p) return fail(RG_EINVAL_CONFIG, "null parameters");
  static const int built[] = {1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13};
  if (std::find(std::begin(built), std::end(built), p->irec) == std::end(built))
    return fail(RG_EINVAL_CONFIG,
                "irec must be 1 (MC), 2 (minmod), 3 (MUSCL), 4 (CENO), 5 (PPM), 6 (MP5), 7 (WENO5), 8 (MP-WENO), 9 (WENO-Z), "
                "10 (WENO-M), 11 (LimO3), 12 (MVL) or 13 (Koren)");
  if (p->ict < 0 || p->ict > 3)
    return fail(RG_EINVAL_CONFIG, "ict must be 0 (none), 1 (flux-CT), 2 (modified flux-CT) or 3 (upwind flux-CT)");
  if (p->ict == 3 && p->precision == RG_MIXED)
    return fail(RG_EINVAL_CONFIG, "upwind flux-CT (ict 3) runs in FP64 only");
  if (p->iwvec < 0 || p->iwvec > 2)
    return fail(RG_EINVAL_CONFIG, "iwvec must be 1 (recov1a; 0 means 1) or 2 (recov2)");
  if (p->iwvec == 2 && p->precision == RG_MIXED)
    return fail(RG_EINVAL_CONFIG, "recov2 (iwvec 2) runs in FP64 only");
  if (p->metric != 1 && p->metric != 303 && p->metric != 403)
    return fail(RG_EINVAL_CONFIG, "metric must be 1, 303 or 403");
  if (p->ix1 != 1 && p->ix1 != 2) return fail(RG_EINVAL_CONFIG, "ix1 must be 1 or 2");
  if (p->ix2 != 1) return fail(RG_EINVAL_CONFIG, "ix2 must be 1");
  if (p->ix3 != 1 && p->ix3 != 2) return fail(RG_EINVAL_CONFIG, "ix3 must be 1 or 2");
  if (p->precision != RG_FP64 && p->precision != RG_MIXED) return fail(RG_EINVAL_CONFIG, "unknown precision mode");
  const int nm1 = nm1_of(p);
  if (p->imax <= 2 * nm1 || p->jmax <= 2 * nm1 || p->kmax <= 2 * nm1)
    return fail(RG_EINVAL_CONFIG, "every extent must exceed 2*nm1 (main.f90:247-254)");
  const double n = (double)p->imax * p->jmax * p->kmax;
  if (n > 1.9e9) return fail(RG_EINVAL_CONFIG, "grid too large for 32-bit interior indices");
  for (int s = 0; s < 6; ++s)
    for (int v = 0; v < 9; ++v) {
      const int c = p->ibc[s][v];
      const bool ok = c == 1 || c == 2 || c == 3 || c == 4 || c == 5 || c == 7 || c == 12 || c == 13 || c == 14 ||
                      (c == 18 && s == 1) || c == 0;
      if (!ok) return fail(RG_EINVAL_CONFIG, "unsupported boundary code");
    }
  if (p->iter < 2) return fail(RG_EINVAL_CONFIG, "iter must be >= 2");
  return RG_OK;
}

// A direction that holds one interior cell, whose ghost fills copy that cell
// (periodic or copy codes for every variable on both sides) and on which the
// metric does not depend (phi always; theta only in Minkowski space) keeps the
// same state in all its cells after each ghost fill, provided every other
// direction's boundary codes are physical ones (bnd.f90:384-1058), whose
// passes cover all columns: the single-rank periodic pass covers only columns
// with interior transverse indices (bnd.f90:50-70, 160-180, 272-292), so with
// two periodic directions the cells that are ghosts in both are never
// refreshed.  Such a direction is stored as one plane.
bool all_physical(const rg_run_params* p, int dir) {
  for (int sd = 2 * (dir - 1); sd <= 2 * (dir - 1) + 1; ++sd)
    for (int v = 0; v < 9; ++v)
      if (p->ibc[sd][v] == 1 || p->ibc[sd][v] == 0) return false;
  return true;
}

bool slab_direction(const rg_run_params* p, int dir, int nm1) {
  const int n = dir == 2 ? p->jmax : p->kmax;
  if (n != 2 * nm1 + 1) return false;
  if (dir == 3 && p->metric != 1) return false;
  for (int sd = 2 * (dir - 1); sd <= 2 * (dir - 1) + 1; ++sd)
    for (int v = 0; v < 9; ++v)
      if (p->ibc[sd][v] != 1 && p->ibc[sd][v] != 5) return false;
  for (int e = 1; e <= 3; ++e)
    if (e != dir && !all_physical(p, e)) return false;
  return true;
}

// Capacity of a run's list of deferred recoveries (cells per stage whose
// Newton-Raphson passes kDeferIter iterations; a few per 10^4 in practice).
int straggler_cap(size_t N) { return (int)std::max<size_t>(1024, std::min<size_t>(N / 64, (size_t)1 << 20)); }

size_t stored_cells(const rg_run_params* p) {
  const int nm1 = nm1_of(p);
  const bool full = (p->flags & RG_FLAG_FULL) != 0;
  const size_t jpl = (!full && slab_direction(p, 2, nm1)) ? 1 : (size_t)p->jmax;
  const size_t kpl = (!full && slab_direction(p, 3, nm1)) ? 1 : (size_t)p->kmax;
  return (size_t)p->imax * jpl * kpl;
}

// Device bytes of a run's step state, geometry and FP32 copies (the
// per-routine entry points' full-layout buffers are allocated on first use).
size_t footprint_bytes(const rg_run_params* p) {
  const size_t N = stored_cells(p);
  const int nm1 = nm1_of(p);
  const bool kslab = !(p->flags & RG_FLAG_FULL) && slab_direction(p, 3, nm1);
  const size_t nik = (size_t)p->imax * (kslab ? 1 : p->kmax);
  const size_t state = (3 * 9 + 3 * 9 + 6 + 9) * N * sizeof(double);
  const size_t geom = (3 * kMetComps + 64) * nik * sizeof(double) + 16 * (size_t)(p->imax + p->jmax + p->kmax) * sizeof(double);
  size_t mixed = 0;
  if (p->precision == RG_MIXED)  // P32, F32 x3, CT32; FP32 metric caches and Christoffels
    mixed = (9 + 27 + 6) * N * sizeof(float) + (3 * kMetComps + 64) * nik * sizeof(float);
  const size_t upct = (p->ict == 3) ? 6 * N * sizeof(double) : 0;  // upflct's EMF differences
  const size_t rec2 = (p->iwvec == 2) ? 22 * N * sizeof(double) : 0;  // recov2 stage scratch
  return state + geom + mixed + upct + rec2 + sizeof(Scal) + C_NCOUNTERS * 8 + (2 * kCarryCap + straggler_cap(N)) * sizeof(int);
}

Run* find(rg_ctx* ctx, int id) {
  if (!ctx) return nullptr;
  auto it = ctx->runs.find(id);
  return it == ctx->runs.end() ? nullptr : it->second;
}

int upload(const std::vector<double>& h, const double** dst, Run* R, cudaStream_t s) {
  void* p = nullptr;
  int rc = dalloc(R, &p, h.size() * sizeof(double));
  if (rc) return rc;
  RG_CUDA(cudaMemcpyAsync(p, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  *dst = static_cast<const double*>(p);
  return RG_OK;
}

// values of a 1-based axis array at 0-based index i-1
std::vector<double> zero_based(const std::vector<double>& v, int n) {
  return std::vector<double>(v.begin() + 1, v.begin() + 1 + n);
}

// Per-index coefficients of the second-order limiters and of CENO along one
// axis, up to ten planes of n values at index m-1 for the cells m = 2..n-1 (zero at the ends,
// which the limiters never reconstruct), computed in FP64 as the reference
// writes them, from the MKS coordinates x?b, x?ab for metric 403 and from x?,
// x?a otherwise.  With small = 1e-12, a = x(m+1) - x(m) + small,
// b = x(m) - x(m-1) + small, c = xa(m) - x(m) + small, d = x(m) - xa(m-1) + small:
//   mclim, minlim, lim03a (rec.f90:267-285, 629-646, 4108-4145): 1/a, 1/b, 0, 0, xa(m) - x(m), x(m) - xa(m-1)
//   koren (rec.f90:4543-4579):  1/a, 1/b, a (1/c), b (1/d), xa(m) - x(m), x(m) - xa(m-1)
//   mvllim (rec.f90:4334-4365): a, b, a/c, b/d, c, d
//   ceno (rec.f90:861-881, 945-951, physical x in every metric): x(m+1) - x(m),
//     x(m) - x(m-1), half of each, and the quadratic candidates' offsets
//     (xf - x(m-1), xf - x(m), xf - x(m+1)) / (x(m+1) - x(m)) with
//     xf = (x(m+1) + x(m))/2, and the same about (x(m) + x(m-1))/2 over x(m) - x(m-1)
std::vector<double> limiter_coefs(const Axis& ax, int n, bool mks, int irec) {
  const double small = 1.0e-12;
  std::vector<double> o(10 * (size_t)n, 0.0);
  if (irec == 4) {
    const std::vector<double>& x = ax.x;
    for (int m = 2; m <= n - 1; ++m) {
      double* q = o.data() + m - 1;
      const double dp = x[m + 1] - x[m], dm = x[m] - x[m - 1];
      const double fp = 0.5 * (x[m + 1] + x[m]), fm = 0.5 * (x[m] + x[m - 1]);
      q[0] = dp; q[n] = dm; q[2 * n] = 0.5 * dp; q[3 * n] = 0.5 * dm;
      q[4 * n] = (fp - x[m - 1]) / dp; q[5 * n] = (fp - x[m]) / dp; q[6 * n] = (fp - x[m + 1]) / dp;
      q[7 * n] = (fm - x[m - 1]) / dm; q[8 * n] = (fm - x[m]) / dm; q[9 * n] = (fm - x[m + 1]) / dm;
    }
    return o;
  }
  const std::vector<double>& x = mks ? ax.xb : ax.x;
  const std::vector<double>& xa = mks ? ax.xab : ax.xa;
  for (int m = 2; m <= n - 1; ++m) {
    const double a = x[m + 1] - x[m] + small, b = x[m] - x[m - 1] + small;
    const double c = xa[m] - x[m] + small, d = x[m] - xa[m - 1] + small;
    double* q = o.data() + m - 1;
    if (irec == 12) {
      q[0] = a; q[n] = b; q[2 * n] = a / c; q[3 * n] = b / d; q[4 * n] = c; q[5 * n] = d;
    } else {
      q[0] = 1.0 / a; q[n] = 1.0 / b;
      if (irec == 13) { q[2 * n] = a * (1.0 / c); q[3 * n] = b * (1.0 / d); }
      q[4 * n] = xa[m] - x[m];
      q[5 * n] = x[m] - xa[m - 1];
    }
  }
  return o;
}

// rec2's dummy dx?b(2:n-1) receives actual dx?b(1:n-1) (rec.f90:58, main.f90:120):
// dummy index m holds actual m-1; dummy 1 (outside the actual array) is taken as actual 1.
std::vector<double> shifted(const std::vector<double>& v, int n) {
  std::vector<double> o(n, 0.0);
  for (int m = 2; m <= n; ++m) o[m - 1] = v[m - 1];
  o[0] = v[1];
  return o;
}

// The per-routine entry points compute in FP64 on the reference's full
// array layout, whatever the run's precision and slab directions.
DevRun full_view(const Run* R) {
  DevRun d = R->d;
  d.mixed = 0;
  d.P32 = nullptr;
  d.jfix = d.kfix = 0;
  d.jpl = d.jmax;
  d.kpl = d.kmax;
  d.sj = (size_t)d.imax;
  d.sk = (size_t)d.imax * d.jmax;
  d.N = R->nfull;
  d.Un = nullptr;
  d.scal = R->fscal;
  d.cnt = R->fcnt;
  return d;
}

// A fresh scalar block for one per-routine call: active, empty queues and the
// given initial CFL bound (cdtcfl4 starts from dtcfl = 1, cdtcfl.f90:30).
int reset_fscal(rg_ctx* ctx, Run* R, double dtcfl0 = 0.0) {
  Scal sc{};
  sc.active = 1;
  std::memcpy(&sc.dtcfl_bits, &dtcfl0, sizeof(double));
  RG_CUDA(cudaMemcpyAsync(R->fscal, &sc, sizeof(Scal), cudaMemcpyHostToDevice, ctx->stream));
  return RG_OK;
}

// Full-layout work buffers of the per-routine entry points, allocated on first use.
int full_bufs(Run* R, cudaStream_t s, DevBufs** out) {
  if (!R->fb_ready) {
    const size_t N = R->nfull;
    void* p = nullptr;
    int rc;
    for (int k = 0; k < 3; ++k) {
      if ((rc = dalloc(R, &p, 9 * N * sizeof(double)))) return rc;
      R->fb.F[k] = static_cast<double*>(p);
      if (cudaMemsetAsync(p, 0, 9 * N * sizeof(double), s) != cudaSuccess) return fail(RG_ECUDA, "memset failed");
    }
    if ((rc = dalloc(R, &p, 6 * N * sizeof(double)))) return rc;
    R->fb.CT = static_cast<double*>(p);
    if (cudaMemsetAsync(p, 0, 6 * N * sizeof(double), s) != cudaSuccess) return fail(RG_ECUDA, "memset failed");
    if ((rc = dalloc(R, &p, 9 * N * sizeof(double)))) return rc;
    R->fb.stage = static_cast<double*>(p);
    if ((rc = dalloc(R, &p, 9 * N * sizeof(double)))) return rc;
    R->fb.stage2 = static_cast<double*>(p);
    if (R->d.ict == 3) {
      if ((rc = dalloc(R, &p, 6 * N * sizeof(double)))) return rc;
      R->fb.ctd = static_cast<double*>(p);
    }
    R->fb_ready = true;
  }
  *out = &R->fb;
  return RG_OK;
}

// Values of a full-layout SoA array (v*Nfull + full cell) at the stored cells of d.
std::vector<double> stored_from_full(const DevRun& d, const std::vector<double>& full, size_t nfull) {
  if (!d.jfix && !d.kfix) return full;
  std::vector<double> out(9 * d.N);
  for (int k = 1; k <= d.kmax; ++k) {
    if (d.kfix && k != d.kfix) continue;
    for (int j = 1; j <= d.jmax; ++j) {
      if (d.jfix && j != d.jfix) continue;
      for (int i = 1; i <= d.imax; ++i)
        for (int v = 0; v < 9; ++v) out[(size_t)v * d.N + d.cell(i, j, k)] = full[(size_t)v * nfull + d.cell_full(i, j, k)];
    }
  }
  return out;
}

int set_time(rg_ctx* ctx, Run* R, double t0) {
  Scal s{};
  s.dtcfl_bits = 0;
  s.dt = 0.01;  // main.f90:358
  s.time = t0;
  s.timeh = t0;
  s.active = 1;
  s.carry_count = 0;
  RG_CUDA(cudaMemcpyAsync(R->d.scal, &s, sizeof(Scal), cudaMemcpyHostToDevice, ctx->stream));
  return RG_OK;
}

int ensure_aos(Run* R) {
  if (R->aos) return RG_OK;
  void* p = nullptr;
  int rc = dalloc(R, &p, 9 * R->nfull * sizeof(double));
  if (rc) return rc;
  R->aos = static_cast<double*>(p);
  return RG_OK;
}

// Host reference-layout array -> device SoA in the layout of view v (the run's
// stored layout, or the full layout of the per-routine entry points).  With
// check, data that are not uniform along a slab direction are refused.
int to_soa(rg_ctx* ctx, Run* R, const double* host_aos, double* dev_soa, const DevRun& v, bool check) {
  int rc = ensure_aos(R);
  if (rc) return rc;
  // cudaMemcpyDefault: the caller's array may be host memory or device memory (unified addressing)
  RG_CUDA(cudaMemcpyAsync(R->aos, host_aos, 9 * R->nfull * sizeof(double), cudaMemcpyDefault, ctx->stream));
  const bool slab = v.jfix || v.kfix;
  if (check && slab) RG_CUDA(cudaMemsetAsync(R->bad, 0, sizeof(int), ctx->stream));
  RG_CUDA(launch_aos_to_soa(v, R->aos, dev_soa, (check && slab) ? R->bad : nullptr, ctx->stream));
  if (check && slab) {
    int bad = 0;
    RG_CUDA(cudaMemcpyAsync(&bad, R->bad, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    RG_CUDA(cudaStreamSynchronize(ctx->stream));
    if (bad)
      return fail(RG_EINVAL_CONFIG,
                  "primitives differ along a slab direction (the run stores one plane of it); admit the run "
                  "with flags bit 0 (RG_FLAG_FULL) to compute every cell");
  }
  return RG_OK;
}

int from_soa(rg_ctx* ctx, Run* R, const double* dev_soa, double* host_aos, const DevRun& v) {
  int rc = ensure_aos(R);
  if (rc) return rc;
  RG_CUDA(launch_soa_to_aos(v, dev_soa, R->aos, ctx->stream));
  RG_CUDA(cudaMemcpyAsync(host_aos, R->aos, 9 * R->nfull * sizeof(double), cudaMemcpyDefault, ctx->stream));
  RG_CUDA(cudaStreamSynchronize(ctx->stream));
  return RG_OK;
}

// ww(3,nv,i,j,k) (host or device array) <-> the full-layout flux planes B->F.
int ww_scratch(Run* R, double** out) {
  if (!R->wwaos) {
    void* p = nullptr;
    const int rc = dalloc(R, &p, 27 * R->nfull * sizeof(double));
    if (rc) return rc;
    R->wwaos = static_cast<double*>(p);
  }
  *out = R->wwaos;
  return RG_OK;
}
int ww_in(rg_ctx* ctx, Run* R, DevBufs* B, const double* ww) {
  double* a = nullptr;
  int rc = ww_scratch(R, &a);
  if (rc) return rc;
  RG_CUDA(cudaMemcpyAsync(a, ww, 27 * R->nfull * sizeof(double), cudaMemcpyDefault, ctx->stream));
  RG_CUDA(launch_ww_layout(a, B->F[0], B->F[1], B->F[2], R->nfull, true, ctx->stream));
  return RG_OK;
}
int ww_out(rg_ctx* ctx, Run* R, DevBufs* B, double* ww) {
  double* a = nullptr;
  int rc = ww_scratch(R, &a);
  if (rc) return rc;
  RG_CUDA(launch_ww_layout(a, B->F[0], B->F[1], B->F[2], R->nfull, false, ctx->stream));
  RG_CUDA(cudaMemcpyAsync(ww, a, 27 * R->nfull * sizeof(double), cudaMemcpyDefault, ctx->stream));
  RG_CUDA(cudaStreamSynchronize(ctx->stream));
  return RG_OK;
}

cudaEvent_t take_event(rg_ctx* ctx) {
  if (!ctx->pool.empty()) {
    cudaEvent_t e = ctx->pool.back();
    ctx->pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// Issue one kernel launch of the given kind; with profiling on it is bracketed
// by CUDA events on the context stream (the stream the kernel runs on).
template <class Fn>
cudaError_t issue(rg_ctx* ctx, int kind, int nlaunch, Fn&& fn) {
  ctx->launches[kind] += nlaunch;
  if (!ctx->prof) return fn();
  cudaEvent_t a = take_event(ctx), b = take_event(ctx);
  cudaEventRecord(a, ctx->stream);
  const cudaError_t e = fn();
  cudaEventRecord(b, ctx->stream);
  ctx->pending.push_back({kind, {a, b}});
  return e;
}

int drain_events(rg_ctx* ctx) {
  if (ctx->pending.empty()) return RG_OK;
  RG_CUDA(cudaStreamSynchronize(ctx->stream));
  for (auto& pe : ctx->pending) {
    float t = 0.f;
    cudaEventElapsedTime(&t, pe.second.first, pe.second.second);
    ctx->ms[pe.first] += t;
    ctx->pool.push_back(pe.second.first);
    ctx->pool.push_back(pe.second.second);
  }
  ctx->pending.clear();
  return RG_OK;
}

// One RK3 stage (main.f90:807-911 / 919-1032 / 1043-1147).
int run_stage(rg_ctx* ctx, Run* R, int stage, const double* Pn, const double* Pc, double* Pw) {
  const DevRun& d = R->d;
  cudaStream_t s = ctx->stream;
  const int nf = n_flux_launches(d);
  // the faces with the stencil staged by TMA where the run allows it
  const int bi = (Pc == R->b.P[0]) ? 0 : (Pc == R->b.P[1] ? 1 : 2);
  const bool tma = R->tma && ctx->tma && Pc == R->b.P[bi];
  auto faces = [&](int dir) {
    return tma ? launch_flux_tma(d, dir, &R->tmap[bi][dir - 1], &R->tmap32[dir - 1], &R->tmapm[dir - 1],
                                 R->b.F[dir - 1], s)
               : launch_flux(d, dir, Pc, R->b.F[dir - 1], s);
  };
  RG_CUDA(issue(ctx, K_FLUX1, nf, [&] { return faces(1); }));
  RG_CUDA(issue(ctx, K_FLUX2, nf, [&] { return faces(2); }));
  RG_CUDA(issue(ctx, K_FLUX3, nf, [&] { return faces(3); }));
  RG_CUDA(issue(ctx, K_CT, n_ct_launches(d), [&] { return launch_ct(d, Pc, R->b.F[0], R->b.F[1], R->b.F[2], R->b.CT, s); }));
  if (d.iwvec == 2) {
    const size_t N = d.N;
    RG_CUDA(issue(ctx, K_UPDATE, 6, [&] {
      return launch_stage_recov2(d, stage, Pc, Pw, R->b.F[0], R->b.F[1], R->b.F[2], R->b.CT, R->b.r2,
                                 R->b.r2 + 9 * N, R->b.r2 + 13 * N, s);
    }));
  } else {
    RG_CUDA(issue(ctx, K_UPDATE, n_update_launches(d), [&] {
      return launch_update(d, stage, Pn, Pc, Pw, R->b.F[0], R->b.F[1], R->b.F[2], R->b.CT, s,
                           (R->utma && ctx->utma) ? static_cast<const void*>(R->umap) : nullptr,
                           (R->utma32 && ctx->utma) ? static_cast<const void*>(R->umap32) : nullptr);
    }));
  }
  RG_CUDA(issue(ctx, K_BC, n_bc_launches(d), [&] { return launch_bc(d, Pw, Pn, s); }));
  RG_CUDA(issue(ctx, K_FLOOR, 1, [&] { return launch_floor(d, Pw, s); }));
  return RG_OK;
}

int read_stats(rg_ctx* ctx, Run* R, rg_step_stats* st) {
  unsigned long long c[C_NCOUNTERS];
  Scal sc;
  RG_CUDA(cudaMemcpyAsync(c, R->d.cnt, sizeof(c), cudaMemcpyDeviceToHost, ctx->stream));
  RG_CUDA(cudaMemcpyAsync(&sc, R->d.scal, sizeof(Scal), cudaMemcpyDeviceToHost, ctx->stream));
  RG_CUDA(cudaStreamSynchronize(ctx->stream));
  const long long ni = (long long)(R->p.imax - 2 * R->d.nm1) * (R->p.jmax - 2 * R->d.nm1) * (R->p.kmax - 2 * R->d.nm1);
  st->steps = (long long)c[C_STEPS];
  st->recov_calls = 3 * ni * (long long)c[C_STEPS];
  st->recov_nr2 = (long long)c[C_NR2];
  st->recov_fail = (long long)c[C_FAIL];
  st->recov_carry = (long long)c[C_CARRY];
  st->recov_cap = (long long)c[C_CAP];
  st->floor_cap = (long long)c[C_FLOORCAP];
  st->carry_overflow = (long long)c[C_CARRY_OVF];
  st->time = sc.timeh;
  st->dt = sc.dt;
  if (c[C_TMAWAIT]) return fail(RG_ECUDA, "a TMA wait of a staged face or update kernel ran out");
  if (c[C_CARRY_OVF]) return fail(RG_EOVERFLOW, "W-carry list overflowed");
  if (c[C_CAP] || c[C_FLOORCAP]) return fail(RG_ENR_CAP, "a capped rescale loop was hit");
  return RG_OK;
}

void free_batch(BatchEntry* E) {
  if (E->graph) cudaGraphExecDestroy(E->graph);
  batch_destroy(E->plan);
  delete E;
}

// Forget every batch a run belongs to (its buffers are about to be freed).
void drop_batches(rg_ctx* ctx, int run) {
  for (auto it = ctx->batches.begin(); it != ctx->batches.end();) {
    if (std::find(it->first.begin(), it->first.end(), run) != it->first.end()) {
      free_batch(it->second);
      it = ctx->batches.erase(it);
    } else {
      ++it;
    }
  }
}

// Runs of one batch class share reconstruction, precision and slab class.
long long batch_class(const Run* R) {
  const DevRun& d = R->d;
  return (long long)d.ict * 100000 + (long long)d.irec * 1000 + d.mixed * 100 + (d.jfix ? 10 : 0) + (d.kfix ? 1 : 0);
}

int kind_of(const BatchPlan* B, int idx) {
  int dir = 0;
  switch (batch_launch_kind(B, idx, &dir)) {
    case 1: return K_CFL;
    case 3: return K_FLUX1 + dir - 1;
    case 4: return K_CT;
    case 5: case 6: return K_UPDATE;
    case 7: case 8: return K_BC;
    case 9: return K_FLOOR;
    case 11: return K_UPDATE;
    default: return K_SCALAR;
  }
}

// Device state of the member runs that a trial step changes: P^n, its FP32
// copy, the scalar block and the counters.
struct Snapshot {
  std::vector<void*> bufs;
  int save(std::vector<Run*>& rs, cudaStream_t s) {
    for (Run* R : rs) {
      const DevRun& d = R->d;
      const size_t sizes[4] = {9 * d.N * sizeof(double), d.P32 ? 9 * d.N * sizeof(float) : 0, sizeof(Scal),
                               C_NCOUNTERS * sizeof(unsigned long long)};
      const void* srcs[4] = {R->b.P[R->cur], d.P32, d.scal, d.cnt};
      for (int a = 0; a < 4; ++a) {
        void* p = nullptr;
        if (sizes[a]) {
          if (cudaMalloc(&p, sizes[a]) != cudaSuccess) return fail(RG_ENOMEM_ADMIT, "autotune snapshot");
          if (cudaMemcpyAsync(p, srcs[a], sizes[a], cudaMemcpyDeviceToDevice, s) != cudaSuccess)
            return fail(RG_ECUDA, "autotune snapshot copy");
        }
        bufs.push_back(p);
      }
    }
    return RG_OK;
  }
  int restore(std::vector<Run*>& rs, cudaStream_t s) {
    size_t a = 0;
    for (Run* R : rs) {
      const DevRun& d = R->d;
      const size_t sizes[4] = {9 * d.N * sizeof(double), d.P32 ? 9 * d.N * sizeof(float) : 0, sizeof(Scal),
                               C_NCOUNTERS * sizeof(unsigned long long)};
      void* dsts[4] = {R->b.P[R->cur], d.P32, d.scal, d.cnt};
      for (int k = 0; k < 4; ++k, ++a)
        if (sizes[k] && cudaMemcpyAsync(dsts[k], bufs[a], sizes[k], cudaMemcpyDeviceToDevice, s) != cudaSuccess)
          return fail(RG_ECUDA, "autotune restore copy");
    }
    return RG_OK;
  }
  ~Snapshot() {
    for (void* p : bufs) cudaFree(p);
  }
};

// Build and capture the batched step of runs of one class.  A class that
// has been tuned in this context (e.g. a serving batch whose members changed)
// gets its tuned shape at once; otherwise the batch starts with the default
// shape (128-thread blocks, one block per tile, one block per tile along i)
// and is tuned by tune_batch once it has run kTuneAfter steps, so that the
// trial steps see the evolved state (shocks, deferred Newton-Raphson cells)
// rather than the initial data.  The one-step launch sequence is captured in
// a CUDA graph.
int capture_batch(BatchEntry* E);
constexpr int kTuneAfter = 32;

int make_batch(rg_ctx* ctx, std::vector<Run*>& rs, const std::vector<int>& ids, BatchEntry** out) {
  std::vector<DevRun> dr;
  for (Run* R : rs) dr.push_back(R->d);
  const long long cls = batch_class(rs[0]);
  auto tk = ctx->tuned.find(cls);
  BatchEntry* E = new BatchEntry();
  E->ids = ids;
  if (tk != ctx->tuned.end()) {
    E->width = tk->second.width;
    E->group = tk->second.group;
    E->grid_factor = tk->second.grid_factor;
    E->tuned_ms = tk->second.ms;
  } else {
    E->tune_pending = true;
  }
  if (batch_build(dr, E->width, E->group, &E->plan)) {
    delete E;
    return fail(RG_ENOMEM_ADMIT, "batch tables do not fit");
  }
  batch_set_grid(E->plan, E->grid_factor);
  const int rc = capture_batch(E);
  if (rc) return rc;
  *out = E;
  return RG_OK;
}

// The tuner: times every candidate shape -- block width 64 or 128 along i,
// tiles of 1, 2 or 4 blocks along i, and persistent grids of one block per
// tile or 2, 4 or 8 blocks per SM -- on trial steps (one warm-up, two timed)
// that start from a snapshot of the members' current state, restores the
// state after each, and keeps the fastest.  The shape decides which block
// computes which cells, never a cell's arithmetic.  The choice is kept per
// batch class for later batches of the context.
int tune_batch(rg_ctx* ctx, BatchEntry* E) {
  cudaStream_t s = ctx->stream;
  std::vector<Run*> rs;
  std::vector<DevRun> dr;
  for (int id : E->ids) {
    Run* R = find(ctx, id);
    rs.push_back(R);
    dr.push_back(R->d);
  }
  Snapshot snap;
  int rc = snap.save(rs, s);
  if (rc) return rc;
  cudaEvent_t e0, e1;
  RG_CUDA(cudaEventCreate(&e0));
  RG_CUDA(cudaEventCreate(&e1));
  struct Shape { int width, group; };
  const Shape shapes[4] = {{64, 1}, {128, 1}, {128, 2}, {128, 4}};
  const int factors[4] = {0, 2, 4, 8};
  double best = 1e30;
  Shape keep{E->width, E->group};
  int keep_factor = E->grid_factor;
  for (const Shape& sh : shapes) {
    BatchPlan* P = nullptr;
    if (batch_build(dr, sh.width, sh.group, &P)) return fail(RG_ENOMEM_ADMIT, "batch tables do not fit");
    for (int f : factors) {
      batch_set_grid(P, f);
      float ms = 0.f;
      cudaError_t e = cudaSuccess;
      for (int rep = 0; rep < 3 && e == cudaSuccess; ++rep) {  // one warm-up step, two timed
        if (rep == 1) e = cudaEventRecord(e0, s);
        if (e == cudaSuccess) e = batch_step(P, s);
      }
      if (e == cudaSuccess) e = cudaEventRecord(e1, s);
      if (e == cudaSuccess) e = cudaEventSynchronize(e1);
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
      if (e != cudaSuccess) {
        batch_destroy(P);
        return fail(RG_ECUDA, std::string("batch tuner: ") + cudaGetErrorString(e));
      }
      if ((rc = snap.restore(rs, s))) {
        batch_destroy(P);
        return rc;
      }
      if (ms < best) {
        best = ms;
        keep = sh;
        keep_factor = f;
      }
    }
    batch_destroy(P);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  RG_CUDA(cudaStreamSynchronize(s));
  BatchPlan* P = nullptr;
  if (batch_build(dr, keep.width, keep.group, &P)) return fail(RG_ENOMEM_ADMIT, "batch tables do not fit");
  batch_set_grid(P, keep_factor);
  if (E->graph) cudaGraphExecDestroy(E->graph);
  E->graph = nullptr;
  batch_destroy(E->plan);
  E->plan = P;
  E->width = keep.width;
  E->group = keep.group;
  E->grid_factor = keep_factor;
  E->tuned_ms = best / 2.0;
  E->tune_pending = false;
  ctx->tuned[batch_class(rs[0])] = {E->width, E->group, E->grid_factor, E->tuned_ms};
  return capture_batch(E);
}

int capture_batch(BatchEntry* E) {
  // one step captured as a graph (the rotation is read on the device, so it replays for every step)
  // (captured on a private stream: the context stream may be the legacy default stream)
  cudaGraph_t g = nullptr;
  cudaStream_t cs = nullptr;
  RG_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  RG_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  const cudaError_t ce = batch_step(E->plan, cs);
  const cudaError_t ee = cudaStreamEndCapture(cs, &g);
  cudaStreamDestroy(cs);
  if (ce != cudaSuccess || ee != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    free_batch(E);
    return fail(RG_ECUDA, "capturing the batched step failed");
  }
  const cudaError_t ie = cudaGraphInstantiate(&E->graph, g, 0);
  cudaGraphDestroy(g);
  if (ie != cudaSuccess) {
    E->graph = nullptr;
    free_batch(E);
    return fail(RG_ECUDA, "instantiating the batched step graph failed");
  }
  return RG_OK;
}

}  // namespace

extern "C" {

const char* rg_last_error(void) { return g_err.c_str(); }

int rg_ctx_create(int device, rg_ctx** out) {
  if (!out) return fail(RG_EINVAL_CONFIG, "null output pointer");
  int n = 0;
  RG_CUDA(cudaGetDeviceCount(&n));
  if (device < 0 || device >= n) return fail(RG_EINVAL_CONFIG, "no such CUDA device");
  RG_CUDA(cudaSetDevice(device));
  rg_ctx* c = new rg_ctx();
  c->device = device;
  if (const char* t = std::getenv("RAISHIN_FLUX_TMA")) c->tma = std::strcmp(t, "0") != 0;
  if (const char* t = std::getenv("RAISHIN_UPDATE_TMA")) c->utma = std::strcmp(t, "0") != 0;
  cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    return fail(RG_ECUDA, cudaGetErrorString(e));
  }
  *out = c;
  return RG_OK;
}

int rg_ctx_destroy(rg_ctx* ctx) {
  if (!ctx) return RG_OK;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  for (auto& kv : ctx->batches) free_batch(kv.second);
  for (auto& kv : ctx->runs) free_run(kv.second);
  for (auto& pe : ctx->pending) ctx->pool.push_back(pe.second.first), ctx->pool.push_back(pe.second.second);
  for (cudaEvent_t e : ctx->pool) cudaEventDestroy(e);
  for (cudaEvent_t e : ctx->marks)
    if (e) cudaEventDestroy(e);
  if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return RG_OK;
}

int rg_ctx_set_stream(rg_ctx* ctx, void* stream) {
  if (!ctx) return fail(RG_EINVAL_CONFIG, "null context");
  RG_CUDA(cudaStreamSynchronize(ctx->stream));
  if (ctx->own_stream) RG_CUDA(cudaStreamDestroy(ctx->stream));
  ctx->stream = static_cast<cudaStream_t>(stream);
  ctx->own_stream = false;
  return RG_OK;
}

int rg_sync(rg_ctx* ctx) {
  if (!ctx) return fail(RG_EINVAL_CONFIG, "null context");
  RG_CUDA(cudaStreamSynchronize(ctx->stream));
  return RG_OK;
}

int rg_ctx_mark(rg_ctx* ctx, int slot) {
  if (!ctx) return fail(RG_EINVAL_CONFIG, "null context");
  if (slot < 0 || slot >= RG_MAX_MARKS) return fail(RG_EINVAL_CONFIG, "mark slot out of range");
  if (!ctx->marks[slot]) RG_CUDA(cudaEventCreateWithFlags(&ctx->marks[slot], cudaEventDisableTiming));
  RG_CUDA(cudaEventRecord(ctx->marks[slot], ctx->stream));
  return RG_OK;
}

int rg_ctx_wait_mark(rg_ctx* ctx, int slot, int block, int* done) {
  if (!ctx) return fail(RG_EINVAL_CONFIG, "null context");
  if (slot < 0 || slot >= RG_MAX_MARKS) return fail(RG_EINVAL_CONFIG, "mark slot out of range");
  if (!ctx->marks[slot]) {  // never marked: nothing to wait for
    if (done) *done = 1;
    return RG_OK;
  }
  if (block) {
    RG_CUDA(cudaEventSynchronize(ctx->marks[slot]));
    if (done) *done = 1;
    return RG_OK;
  }
  const cudaError_t e = cudaEventQuery(ctx->marks[slot]);
  if (e == cudaErrorNotReady) {
    (void)cudaGetLastError();
    if (done) *done = 0;
    return RG_OK;
  }
  RG_CUDA(e);
  if (done) *done = 1;
  return RG_OK;
}

int rg_run_footprint(const rg_run_params* p, size_t* bytes) {
  const int rc = check_params(p);
  if (rc) return rc;
  if (bytes) *bytes = footprint_bytes(p);
  return RG_OK;
}

int rg_prep_create(const rg_run_params* p, rg_prep** out) {
  if (!out) return fail(RG_EINVAL_CONFIG, "null argument");
  int rc = check_params(p);
  if (rc) return rc;
  rg_prep* P = new rg_prep();
  P->p = *p;
  const int nm1 = nm1_of(p);
  const bool full = (p->flags & RG_FLAG_FULL) != 0;
  P->krow = (!full && slab_direction(p, 3, nm1)) ? nm1 + 1 : 0;  // theta slab: one metric row
  P->plane = !full && slab_direction(p, 2, nm1);                   // phi slab: one initial-data plane
  build_geometry(*p, P->geom, P->krow);
  if (!P->geom.compact_ok) {
    delete P;
    return fail(RG_EINVAL_CONFIG, "metric couples theta to (t,r,phi): not representable by the compact cache");
  }
  *out = P;
  return RG_OK;
}

int rg_prep_ic_torus(rg_prep* P, uint64_t seed, double amp, double rin, double rmax, double beta, double kappa) {
  if (!P) return fail(RG_EINVAL_CONFIG, "null preparation");
  if (P->krow) return fail(RG_EINVAL_CONFIG, "torus initial data needs a Kerr metric (this run is a Minkowski slab)");
  torus_ic(P->p, P->geom, seed, amp, rin, rmax, beta, kappa, P->ic, P->plane);
  return RG_OK;
}

int rg_prep_destroy(rg_prep* P) {
  delete P;
  return RG_OK;
}

int rg_run_admit(rg_ctx* ctx, const rg_run_params* p, int* run_id) {
  rg_prep* P = nullptr;
  int rc = rg_prep_create(p, &P);
  if (rc) return rc;
  rc = rg_run_admit_prep(ctx, P, run_id);
  delete P;
  return rc;
}

int rg_run_admit_prep(rg_ctx* ctx, rg_prep* prep, int* run_id) {
  if (!ctx || !run_id || !prep) return fail(RG_EINVAL_CONFIG, "null argument");
  const rg_run_params* p = &prep->p;
  int rc = RG_OK;
  RG_CUDA(cudaSetDevice(ctx->device));
  size_t free_b = 0, total_b = 0;
  RG_CUDA(cudaMemGetInfo(&free_b, &total_b));
  const size_t need = footprint_bytes(p);
  if (need + (size_t)256 * 1024 * 1024 > free_b)
    return fail(RG_ENOMEM_ADMIT, "run footprint " + std::to_string(need) + " B exceeds free device memory");
  Run* R = new Run();
  R->p = *p;
  R->geom = prep->geom;
  DevRun& d = R->d;
  d.imax = p->imax; d.jmax = p->jmax; d.kmax = p->kmax;
  d.nm0 = nm0_of(p->irec);
  d.nm1 = d.nm0 + p->ict;
  d.ict = p->ict;
  d.iwvec = (p->iwvec == 2) ? 2 : 1;
  d.irec = p->irec; d.model = p->model; d.guard = p->guard; d.iter = p->iter;
  d.mixed = (p->precision == RG_MIXED);
#ifdef RG_EXACT_ARITH
  d.gkind = 0;  // every power through pow(), as the reference writes it
#else
  d.gkind = (p->gam == 4.0 / 3.0) ? 1 : (p->gam == 5.0 / 3.0 ? 2 : 0);
#endif
  // cells inside r < 2 r_H keep FP64 in the mixed path (Kerr metrics only)
  d.i_fp64 = 0;
  if (p->metric == 303 || p->metric == 403) {
    const double r2h = 2.0 * (1.0 + std::sqrt(1.0 - p->akm * p->akm));
    for (int i = 1; i <= p->imax; ++i)
      if (R->geom.ax[0].x[i] < r2h) d.i_fp64 = i;
  }
  d.nmax_cfl = d.nm1 * 2 + (d.nm1 - 1);
  const bool full = (p->flags & RG_FLAG_FULL) != 0;
  d.jfix = (!full && slab_direction(p, 2, d.nm1)) ? d.nm1 + 1 : 0;
  d.kfix = (!full && slab_direction(p, 3, d.nm1)) ? d.nm1 + 1 : 0;
  d.jpl = d.jfix ? 1 : p->jmax;
  d.kpl = d.kfix ? 1 : p->kmax;
  d.sj = d.jfix ? 0 : (size_t)p->imax;
  d.sk = d.kfix ? 0 : (size_t)p->imax * d.jpl;
  d.N = (size_t)p->imax * d.jpl * d.kpl;
  R->nfull = (size_t)p->imax * p->jmax * p->kmax;
  d.kmet = d.kfix;
  d.nik = (size_t)p->imax * (d.kfix ? 1 : p->kmax);
  d.gam = p->gam; d.cfl = p->cfl; d.dmin = p->dmin; d.pmin = p->pmin; d.pmax = p->pmax; d.tmax = p->tmax;
  std::memcpy(d.ibc, p->ibc, sizeof(d.ibc));
  d.carry_cap = kCarryCap;
  cudaStream_t s = ctx->stream;
  const size_t N = d.N;
  void* ptr = nullptr;
  auto bail = [&](int code) {
    cudaStreamSynchronize(s);
    free_run(R);
    return code;
  };
  for (int k = 0; k < 3; ++k) {
    if ((rc = dalloc(R, &ptr, 9 * N * sizeof(double)))) return bail(rc);
    R->b.P[k] = static_cast<double*>(ptr);
    d.P[k] = R->b.P[k];
    if ((rc = dalloc(R, &ptr, 9 * N * sizeof(double)))) return bail(rc);
    R->b.F[k] = static_cast<double*>(ptr);
  }
  if ((rc = dalloc(R, &ptr, 6 * N * sizeof(double)))) return bail(rc);
  R->b.CT = static_cast<double*>(ptr);
  for (int k = 0; k < 3; ++k) d.F[k] = R->b.F[k];
  d.CT = R->b.CT;
  if (d.ict == 3) {
    if ((rc = dalloc(R, &ptr, 6 * N * sizeof(double)))) return bail(rc);
    R->b.ctd = static_cast<double*>(ptr);
    d.ctd = R->b.ctd;
  }
  if (d.iwvec == 2) {
    if ((rc = dalloc(R, &ptr, 22 * N * sizeof(double)))) return bail(rc);
    R->b.r2 = static_cast<double*>(ptr);
  }
  if ((rc = dalloc(R, &ptr, 9 * N * sizeof(double)))) return bail(rc);
  d.Un = static_cast<double*>(ptr);
  if ((rc = dalloc(R, &ptr, sizeof(int)))) return bail(rc);
  R->bad = static_cast<int*>(ptr);
  if (!d.jfix && !d.kfix) {  // the full layout is the stored one: share the step's flux buffers
    R->fb.F[0] = R->b.F[0]; R->fb.F[1] = R->b.F[1]; R->fb.F[2] = R->b.F[2]; R->fb.CT = R->b.CT;
  }
  if ((rc = dalloc(R, &ptr, 2 * (size_t)p->imax * sizeof(double)))) return bail(rc);
  d.fl_de = static_cast<double*>(ptr);
  d.fl_pr = d.fl_de + p->imax;
  if ((rc = dalloc(R, &ptr, sizeof(Scal)))) return bail(rc);
  d.scal = static_cast<Scal*>(ptr);
  if ((rc = dalloc(R, &ptr, sizeof(Scal)))) return bail(rc);
  R->fscal = static_cast<Scal*>(ptr);
  if ((rc = dalloc(R, &ptr, C_NCOUNTERS * sizeof(unsigned long long)))) return bail(rc);
  R->fcnt = static_cast<unsigned long long*>(ptr);
  if (cudaMemsetAsync(R->fcnt, 0, C_NCOUNTERS * sizeof(unsigned long long), s) != cudaSuccess) return bail(RG_ECUDA);
  if ((rc = dalloc(R, &ptr, C_NCOUNTERS * sizeof(unsigned long long)))) return bail(rc);
  d.cnt = static_cast<unsigned long long*>(ptr);
  if ((rc = dalloc(R, &ptr, 2 * (size_t)kCarryCap * sizeof(int)))) return bail(rc);
  d.carry_list = static_cast<int*>(ptr);
  d.carry_sorted = d.carry_list + kCarryCap;
  d.strag_cap = straggler_cap(N);
  if ((rc = dalloc(R, &ptr, (size_t)d.strag_cap * sizeof(int)))) return bail(rc);
  d.strag_list = static_cast<int*>(ptr);
  if (cudaMemsetAsync(d.cnt, 0, C_NCOUNTERS * sizeof(unsigned long long), s) != cudaSuccess) return bail(RG_ECUDA);
  for (int k = 0; k < 3; ++k) {
    if (cudaMemsetAsync(R->b.P[k], 0, 9 * N * sizeof(double), s) != cudaSuccess) return bail(RG_ECUDA);
    if (cudaMemsetAsync(R->b.F[k], 0, 9 * N * sizeof(double), s) != cudaSuccess) return bail(RG_ECUDA);
  }
  if (cudaMemsetAsync(R->b.CT, 0, 6 * N * sizeof(double), s) != cudaSuccess) return bail(RG_ECUDA);
  const HostGeom& G = R->geom;
  // (a theta slab's geometry holds the one metric row of its computed index)
  if (G.nik != d.nik) return bail(fail(RG_EINVAL_CONFIG, "geometry prepared for another slab layout"));
  if ((rc = upload(G.mc, &d.mc, R, s))) return bail(rc);
  if ((rc = upload(G.mi, &d.mi, R, s))) return bail(rc);
  if ((rc = upload(G.mk, &d.mk, R, s))) return bail(rc);
  if ((rc = upload(G.chr, &d.chr, R, s))) return bail(rc);
  std::vector<double> t;
  if ((rc = upload(zero_based(G.ax[0].x, p->imax), &d.x1, R, s))) return bail(rc);
  if ((rc = upload(zero_based(G.ax[0].dxb, p->imax), &d.dx1b, R, s))) return bail(rc);
  if ((rc = upload(zero_based(G.ax[1].dxb, p->jmax), &d.dx2b, R, s))) return bail(rc);
  if ((rc = upload(zero_based(G.ax[2].dxb, p->kmax), &d.dx3b, R, s))) return bail(rc);
  if ((rc = upload(zero_based(G.ax[1].x, p->jmax), &d.x2, R, s))) return bail(rc);
  if ((rc = upload(zero_based(G.ax[2].x, p->kmax), &d.x3, R, s))) return bail(rc);
  if ((rc = upload(shifted(G.ax[0].dxb, p->imax), &d.dx1s, R, s))) return bail(rc);
  if ((rc = upload(shifted(G.ax[1].dxb, p->jmax), &d.dx2s, R, s))) return bail(rc);
  if ((rc = upload(shifted(G.ax[2].dxb, p->kmax), &d.dx3s, R, s))) return bail(rc);
  const int ext[3] = {p->imax, p->jmax, p->kmax};
  for (int a = 0; a < 3; ++a)
    if ((rc = upload(limiter_coefs(G.ax[a], ext[a], p->metric == 403, p->irec), &d.lim[a], R, s))) return bail(rc);
  // the caches and floor tables are this run's own allocations: fill their derived parts
  if (launch_geom_derive(d, const_cast<double*>(d.mc), const_cast<double*>(d.mi), const_cast<double*>(d.mk),
                         const_cast<double*>(d.fl_de), const_cast<double*>(d.fl_pr), s) != cudaSuccess)
    return bail(fail(RG_ECUDA, "geometry setup kernel failed"));
  if (d.mixed) {
    const size_t nik = d.nik;
    float* f = nullptr;
    auto falloc = [&](size_t n) -> int {
      void* q = nullptr;
      int e = dalloc(R, &q, n * sizeof(float));
      f = static_cast<float*>(q);
      return e;
    };
    if ((rc = falloc(9 * N))) return bail(rc);
    d.P32 = f;
    for (int k = 0; k < 3; ++k) {
      if ((rc = falloc(9 * N))) return bail(rc);
      d.F32[k] = f;
      if (cudaMemsetAsync(f, 0, 9 * N * sizeof(float), s) != cudaSuccess) return bail(RG_ECUDA);
    }
    if ((rc = falloc(6 * N))) return bail(rc);
    d.CT32 = f;
    if (cudaMemsetAsync(f, 0, 6 * N * sizeof(float), s) != cudaSuccess) return bail(RG_ECUDA);
    const double* src[4] = {d.mc, d.mi, d.mk, d.chr};
    const float** dst[4] = {&d.mc32, &d.mi32, &d.mk32, &d.chr32};
    for (int a = 0; a < 4; ++a) {
      const size_t n = (a < 3 ? (size_t)kMetComps : (size_t)64) * nik;
      if ((rc = falloc(n))) return bail(rc);
      if (launch_to_f32(src[a], f, n, s) != cudaSuccess) return bail(fail(RG_ECUDA, "FP32 cache setup failed"));
      *dst[a] = f;
    }
  }
  if ((rc = set_time(ctx, R, 0.0))) return bail(rc);
  make_tmaps(R);
  if (!prep->ic.empty()) {  // initial data computed with the preparation
    const std::vector<double> Ps = stored_from_full(d, prep->ic, R->nfull);
    if (cudaMemcpyAsync(R->b.P[0], Ps.data(), Ps.size() * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess)
      return bail(fail(RG_ECUDA, "initial data upload failed"));
    if (d.P32 && launch_to_f32(R->b.P[0], d.P32, 9 * d.N, s) != cudaSuccess)
      return bail(fail(RG_ECUDA, "initial data upload failed"));
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) return bail(fail(RG_ECUDA, "setup failed"));
  const int id = ctx->next_id++;
  ctx->runs[id] = R;
  *run_id = id;
  return RG_OK;
}

int rg_run_release(rg_ctx* ctx, int run) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  cudaStreamSynchronize(ctx->stream);
  drop_batches(ctx, run);
  free_run(R);
  ctx->runs.erase(run);
  return RG_OK;
}

int rg_run_ic_torus(rg_ctx* ctx, int run, uint64_t seed, double amp, double rin, double rmax, double beta,
                    double kappa) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  std::vector<double> P;
  if (R->d.kmet) return fail(RG_EINVAL_CONFIG, "torus initial data needs a Kerr metric (this run is a Minkowski slab)");
  torus_ic(R->p, R->geom, seed, amp, rin, rmax, beta, kappa, P, R->d.jfix != 0);
  const std::vector<double> Ps = stored_from_full(R->d, P, R->nfull);
  R->cur = 0;
  RG_CUDA(cudaMemcpyAsync(R->b.P[0], Ps.data(), Ps.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  if (R->d.P32) RG_CUDA(launch_to_f32(R->b.P[0], R->d.P32, 9 * R->d.N, ctx->stream));
  int rc = set_time(ctx, R, 0.0);
  if (rc) return rc;
  RG_CUDA(cudaStreamSynchronize(ctx->stream));
  return RG_OK;
}

int rg_run_ic_torus_device(rg_ctx* ctx, int run, uint64_t seed, double amp, double rin, double rmax, double beta,
                           double kappa) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  const DevRun& d = R->d;
  if (d.kmet || d.kfix) return fail(RG_EINVAL_CONFIG, "torus initial data needs a Kerr metric on a full theta range");
  if (d.imax < 3 || d.kmax < 3) return fail(RG_EINVAL_CONFIG, "torus initial data needs imax, kmax >= 3");
  TorusTables T;
  torus_tables(R->p, R->geom, rin, rmax, T);
  void* buf = nullptr;
  const size_t tab_bytes = T.tab.size() * sizeof(double);
  RG_CUDA(cudaMalloc(&buf, tab_bytes + 2 * sizeof(unsigned long long)));
  IcTorusArgs a{};
  a.tab = static_cast<const double*>(buf);
  a.red = reinterpret_cast<unsigned long long*>(static_cast<char*>(buf) + tab_bytes);
  a.seed = seed; a.amp = amp; a.rin = rin; a.kappa = kappa; a.beta = beta; a.akm = R->p.akm;
  a.ell = T.ell; a.h_in = T.h_in; a.edge0 = T.edge0; a.edge1 = T.edge1;
  a.metric = R->p.metric; a.ix1 = R->p.ix1; a.ix3 = R->p.ix3;
  const int nm1 = nm1_of(&R->p);
  a.phi_slab = (d.jmax == 2 * nm1 + 1);
  a.slab_j = nm1 + 1;
  cudaError_t e = cudaMemcpyAsync(buf, T.tab.data(), tab_bytes, cudaMemcpyHostToDevice, ctx->stream);
  R->cur = 0;
  if (e == cudaSuccess) e = launch_ic_torus(d, a, R->b.P[0], ctx->stream);
  if (e == cudaSuccess && d.P32) e = launch_to_f32(R->b.P[0], d.P32, 9 * d.N, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(buf);
  if (e != cudaSuccess) return fail(RG_ECUDA, cudaGetErrorString(e));
  return set_time(ctx, R, 0.0);
}

int rg_run_ic_tube(rg_ctx* ctx, int run, uint64_t seed, uint64_t tube) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  const DevRun& d = R->d;
  double q[2][9];
  tube_states(seed, tube, d.gam, q);
  std::vector<double> P(9 * d.N);
  for (int k = 1; k <= d.kmax; ++k) {
    if (d.kfix && k != d.kfix) continue;
    for (int j = 1; j <= d.jmax; ++j) {
      if (d.jfix && j != d.jfix) continue;
      for (int i = 1; i <= d.imax; ++i)
        for (int v = 0; v < 9; ++v) P[(size_t)v * d.N + d.cell(i, j, k)] = q[i <= d.imax / 2 ? 0 : 1][v];
    }
  }
  R->cur = 0;
  RG_CUDA(cudaMemcpyAsync(R->b.P[0], P.data(), P.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  if (d.P32) RG_CUDA(launch_to_f32(R->b.P[0], d.P32, 9 * d.N, ctx->stream));
  int rc = set_time(ctx, R, 0.0);
  if (rc) return rc;
  RG_CUDA(cudaStreamSynchronize(ctx->stream));
  return RG_OK;
}

int rg_run_upload_prims(rg_ctx* ctx, int run, const double* uri, double t0) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  if (!uri) return fail(RG_EINVAL_CONFIG, "null array");
  R->cur = 0;
  int rc = to_soa(ctx, R, uri, R->b.P[0], R->d, true);
  if (rc) return rc;
  if (R->d.P32) RG_CUDA(launch_to_f32(R->b.P[0], R->d.P32, 9 * R->d.N, ctx->stream));
  return set_time(ctx, R, t0);
}

int rg_run_download_prims(rg_ctx* ctx, int run, double* uri) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  if (!uri) return fail(RG_EINVAL_CONFIG, "null array");
  return from_soa(ctx, R, R->b.P[R->cur], uri, R->d);
}

int rg_run_layout(rg_ctx* ctx, int run, size_t* ncells, int* jplanes, int* kplanes) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  if (ncells) *ncells = R->d.N;
  if (jplanes) *jplanes = R->d.jpl;
  if (kplanes) *kplanes = R->d.kpl;
  return RG_OK;
}

int rg_run_download_stored(rg_ctx* ctx, int run, double* soa) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  if (!soa) return fail(RG_EINVAL_CONFIG, "null array");
  RG_CUDA(cudaMemcpyAsync(soa, R->b.P[R->cur], 9 * R->d.N * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  RG_CUDA(cudaStreamSynchronize(ctx->stream));
  return RG_OK;
}

// One full step of a run with its own launches (CFL, three stages, scalars).
static int step_alone(rg_ctx* ctx, Run* R) {
  cudaStream_t s = ctx->stream;
  double* Pn = R->b.P[R->cur];
  double* P1 = R->b.P[(R->cur + 1) % 3];
  double* P2 = R->b.P[(R->cur + 2) % 3];
  RG_CUDA(issue(ctx, K_SCALAR, 1, [&] { return launch_step_begin(R->d, s); }));
  RG_CUDA(issue(ctx, K_CFL, 1, [&] { return launch_cfl(R->d, Pn, s); }));
  RG_CUDA(issue(ctx, K_SCALAR, 1, [&] { return launch_dt(R->d, s); }));
  int rc;
  if ((rc = run_stage(ctx, R, 1, Pn, Pn, P1))) return rc;
  if ((rc = run_stage(ctx, R, 2, Pn, P1, P2))) return rc;
  if ((rc = run_stage(ctx, R, 3, Pn, P2, P1))) return rc;
  RG_CUDA(issue(ctx, K_SCALAR, 1, [&] { return launch_step_end(R->d, s); }));
  R->cur = (R->cur + 1) % 3;
  return RG_OK;
}

// Runs that a batch steps with their own launches: no slab direction (they
// fill the GPU alone, and the single-run kernels stage their stencils and
// rows by TMA), or a scheme without batched kernels (upwind flux-CT, recov2).
static bool steps_alone(const Run* R) {
  return !(R->d.jfix || R->d.kfix) || R->d.ict == 3 || R->d.iwvec == 2;
}

int rg_step(rg_ctx* ctx, int run, int nsteps, rg_step_stats* stats) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  // A run with a slab direction steps as a batch of one: it then runs the same
  // compiled kernels alone as in any batch, so its results do not depend on
  // the company it keeps, and its step is replayed from a CUDA graph.
  if (!steps_alone(R)) return rg_step_batch(ctx, &run, 1, nsteps, stats);
  for (int n = 0; n < nsteps; ++n) {
    const int rc = step_alone(ctx, R);
    if (rc) return rc;
  }
  if (ctx->prof) {
    int rc = drain_events(ctx);
    if (rc) return rc;
  }
  if (stats) return read_stats(ctx, R, stats);
  return RG_OK;
}

int rg_step_batch(rg_ctx* ctx, const int* runs, int nruns, int nsteps, rg_step_stats* stats) {
  if (!ctx || !runs || nruns <= 0) return fail(RG_EINVAL_CONFIG, "empty batch");
  std::map<long long, std::vector<int>> groups;
  std::vector<Run*> alone;  // stepped with their own launches, after the batch classes of each step
  {
    std::vector<int> all(runs, runs + nruns);
    std::sort(all.begin(), all.end());
    if (std::adjacent_find(all.begin(), all.end()) != all.end())
      return fail(RG_EINVAL_CONFIG, "a run appears twice in the batch");
  }
  for (int a = 0; a < nruns; ++a) {
    Run* R = find(ctx, runs[a]);
    if (!R) return fail(RG_ENOTFOUND, "unknown run in batch");
    if (steps_alone(R)) alone.push_back(R);
    else groups[batch_class(R)].push_back(runs[a]);
  }
  std::vector<BatchEntry*> es;
  for (auto& kv : groups) {
    std::vector<int> ids = kv.second;
    std::sort(ids.begin(), ids.end());
    if (std::adjacent_find(ids.begin(), ids.end()) != ids.end())
      return fail(RG_EINVAL_CONFIG, "a run appears twice in the batch");
    auto it = ctx->batches.find(ids);
    if (it == ctx->batches.end()) {
      std::vector<Run*> rs;
      for (int id : ids) rs.push_back(find(ctx, id));
      BatchEntry* E = nullptr;
      int rc = make_batch(ctx, rs, ids, &E);
      if (rc) return rc;
      it = ctx->batches.emplace(ids, E).first;
    }
    es.push_back(it->second);
  }
  cudaStream_t s = ctx->stream;
  // Steps run in segments whose ends keep the host-side buffer rotation up
  // to date, so that an entry due for tuning is tuned between segments.
  for (int done = 0; done < nsteps;) {
    int seg = nsteps - done;
    for (BatchEntry* E : es) {
      if (E->tune_pending && E->steps_run >= kTuneAfter) {
        const int rc = tune_batch(ctx, E);
        if (rc) return rc;
      }
      if (E->tune_pending) seg = std::min<long long>(seg, kTuneAfter - E->steps_run);
    }
    for (int n = 0; n < seg; ++n) {
      for (BatchEntry* E : es) {
        const int nl = batch_launch_count(E->plan);
        if (!ctx->prof) {
          RG_CUDA(cudaGraphLaunch(E->graph, s));
          for (int a = 0; a < nl; ++a) ctx->launches[kind_of(E->plan, a)] += 1;
        } else {
          for (int a = 0; a < nl; ++a)
            RG_CUDA(issue(ctx, kind_of(E->plan, a), 1, [&] { return batch_issue(E->plan, a, s); }));
        }
        E->steps_run += 1;
      }
      for (Run* R : alone) {  // advances its own buffer rotation
        const int rc = step_alone(ctx, R);
        if (rc) return rc;
      }
    }
    for (int a = 0; a < nruns; ++a) {
      Run* R = find(ctx, runs[a]);
      if (!steps_alone(R)) R->cur = (R->cur + seg) % 3;
    }
    done += seg;
  }
  if (ctx->prof) {
    int rc = drain_events(ctx);
    if (rc) return rc;
  }
  if (stats) {
    int worst = RG_OK;
    for (int a = 0; a < nruns; ++a) {
      const int rc = read_stats(ctx, find(ctx, runs[a]), stats + a);
      if (rc == RG_ECUDA) return rc;
      if (rc && !worst) worst = rc;
    }
    return worst;
  }
  return RG_OK;
}

int rg_batch_info(rg_ctx* ctx, const int* runs, int nruns, int* width, int* grid_factor, int* launches,
                  double* tuned_ms, int* tile_cells) {
  if (!ctx || !runs || nruns <= 0) return fail(RG_EINVAL_CONFIG, "empty batch");
  std::vector<int> ids(runs, runs + nruns);
  std::sort(ids.begin(), ids.end());
  auto it = ctx->batches.find(ids);
  if (it == ctx->batches.end()) return fail(RG_ENOTFOUND, "no batch of exactly these runs has been stepped");
  if (width) *width = it->second->width;
  if (grid_factor) *grid_factor = it->second->grid_factor;
  if (launches) *launches = batch_launch_count(it->second->plan);
  if (tuned_ms) *tuned_ms = it->second->tune_pending ? 0.0 : it->second->tuned_ms;
  if (tile_cells) *tile_cells = it->second->width * it->second->group;
  return RG_OK;
}

int rg_profile(rg_ctx* ctx, int enable) {
  if (!ctx) return fail(RG_EINVAL_CONFIG, "null context");
  int rc = drain_events(ctx);
  if (rc) return rc;
  ctx->prof = (enable != 0);
  for (int k = 0; k < K_NKINDS; ++k) {
    ctx->ms[k] = 0.0;
    ctx->launches[k] = 0;
  }
  return RG_OK;
}

int rg_profile_read(rg_ctx* ctx, double* ms, long long* launches, int nkinds) {
  if (!ctx) return fail(RG_EINVAL_CONFIG, "null context");
  int rc = drain_events(ctx);
  if (rc) return rc;
  for (int k = 0; k < nkinds && k < K_NKINDS; ++k) {
    if (ms) ms[k] = ctx->ms[k];
    if (launches) launches[k] = ctx->launches[k];
  }
  return RG_OK;
}

int rg_run_stats(rg_ctx* ctx, int run, rg_step_stats* stats) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  if (!stats) return fail(RG_EINVAL_CONFIG, "null stats");
  return read_stats(ctx, R, stats);
}

int rg_caluu1(rg_ctx* ctx, int run, const double* uri, double* uu) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  if (!uri || !uu) return fail(RG_EINVAL_CONFIG, "null array");
  const DevRun d = full_view(R);
  DevBufs* B = nullptr;
  int rc = full_bufs(R, ctx->stream, &B);
  if (rc || (rc = to_soa(ctx, R, uri, B->stage, d, false))) return rc;
  RG_CUDA(launch_p2c(d, B->stage, B->stage2, ctx->stream));
  return from_soa(ctx, R, B->stage2, uu, d);
}

int rg_calflx(rg_ctx* ctx, int run, const double* uri, double* ww) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  if (!uri || !ww) return fail(RG_EINVAL_CONFIG, "null array");
  DevRun d = full_view(R);
  DevBufs* B = nullptr;
  int rc = full_bufs(R, ctx->stream, &B);
  if (rc || (rc = to_soa(ctx, R, uri, B->stage, d, false)) || (rc = reset_fscal(ctx, R))) return rc;
  d.ctd = B->ctd;
  for (int dir = 1; dir <= 3; ++dir) RG_CUDA(launch_flux(d, dir, B->stage, B->F[dir - 1], ctx->stream));
  RG_CUDA(launch_ct(d, B->stage, B->F[0], B->F[1], B->F[2], B->CT, ctx->stream));
  RG_CUDA(launch_ct_apply(d, B->CT, B->F[0], B->F[1], B->F[2], ctx->stream));
  return ww_out(ctx, R, B, ww);
}

int rg_calsf(rg_ctx* ctx, int run, const double* uri, double* sf) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  if (!uri || !sf) return fail(RG_EINVAL_CONFIG, "null array");
  const DevRun d = full_view(R);
  const size_t N = d.N;
  DevBufs* B = nullptr;
  int rc = full_bufs(R, ctx->stream, &B);
  if (rc || (rc = to_soa(ctx, R, uri, B->stage, d, false))) return rc;
  RG_CUDA(launch_calsf(d, B->stage, B->CT, ctx->stream));
  // sf(2:5,i,j,k): the four planes into the reference layout in the ww staging buffer
  double* a = nullptr;
  if ((rc = ww_scratch(R, &a))) return rc;
  RG_CUDA(launch_aos_planes(a, B->CT, N, 4, false, ctx->stream));
  RG_CUDA(cudaMemcpyAsync(sf, a, 4 * N * sizeof(double), cudaMemcpyDefault, ctx->stream));
  RG_CUDA(cudaStreamSynchronize(ctx->stream));
  return RG_OK;
}

int rg_rkt(rg_ctx* ctx, int run, int stage, double dt, const double* ww, const double* uo, const double* ucur,
           const double* sf, double* unew) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  if (stage < 1 || stage > 3) return fail(RG_EINVAL_CONFIG, "stage must be 1, 2 or 3");
  if (!ww || !ucur || !sf || !unew || (stage > 1 && !uo)) return fail(RG_EINVAL_CONFIG, "null array");
  const DevRun d = full_view(R);
  const size_t N = d.N;
  DevBufs* B = nullptr;
  int rc = full_bufs(R, ctx->stream, &B);
  if (rc) return rc;
  if (!R->unew) {
    void* p = nullptr;
    if ((rc = dalloc(R, &p, 9 * N * sizeof(double)))) return rc;
    R->unew = static_cast<double*>(p);
  }
  // ww(3,nv,i,j,k) and sf(2:5,i,j,k) to planes on the device
  if ((rc = ww_in(ctx, R, B, ww))) return rc;
  RG_CUDA(cudaStreamSynchronize(ctx->stream));  // the staging buffer is reused for sf
  double* a = nullptr;
  if ((rc = ww_scratch(R, &a))) return rc;
  RG_CUDA(cudaMemcpyAsync(a, sf, 4 * N * sizeof(double), cudaMemcpyDefault, ctx->stream));
  RG_CUDA(launch_aos_planes(a, B->CT, N, 4, true, ctx->stream));
  if ((rc = to_soa(ctx, R, ucur, B->stage, d, false))) return rc;
  if (stage > 1 && (rc = to_soa(ctx, R, uo, B->stage2, d, false))) return rc;
  if ((rc = to_soa(ctx, R, unew, R->unew, d, false))) return rc;
  RG_CUDA(launch_rkt(d, stage, B->F[0], B->F[1], B->F[2], stage > 1 ? B->stage2 : nullptr, B->stage, B->CT, R->unew,
                     dt, ctx->stream));
  return from_soa(ctx, R, R->unew, unew, d);
}

int rg_run_derived(rg_ctx* ctx, int run, int jslice, double* out) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  if (!out) return fail(RG_EINVAL_CONFIG, "null array");
  const rg_run_params& p = R->p;
  if (p.metric != 303 && p.metric != 403)
    return fail(RG_EINVAL_CONFIG, "derived quantities are defined for the Kerr metrics 303 and 403");
  if (jslice < 0 || jslice > p.jmax) return fail(RG_EINVAL_CONFIG, "jslice must be 0 or a phi index 1..jmax");
  // the converter's coordinates (convert_vtk2dn1.f90:138-161) and the
  // MKS -> KS factors of transmks2ks1 (convert_vtk2dn1.f90:1524-1554)
  const Axis& a1 = R->geom.ax[0];
  const Axis& a3 = R->geom.ax[2];
  std::vector<double> gi(2 * (size_t)p.imax), gk(3 * (size_t)p.kmax);
  for (int i = 1; i <= p.imax; ++i) {
    double rr = a1.x[i], rfac = 1.0;
    if (p.metric == 403) {
      const double x1t = a1.xb[i];
      rr = (p.ix1 == 2) ? p.R0 + std::exp(x1t) : x1t;
      if (p.ix1 == 2) rfac = std::exp(x1t);
    }
    gi[2 * (i - 1)] = rr;
    gi[2 * (i - 1) + 1] = rfac;
  }
  for (int k = 1; k <= p.kmax; ++k) {
    double th = a3.x[k], hfac = 1.0;
    if (p.metric == 403) {
      const double x3t = a3.xb[k];
      th = (p.ix3 == 2) ? x3t + 0.5 * (1. - p.hslope) * std::sin(2. * x3t) : x3t;
      if (p.ix3 == 2) hfac = 1. + (1. - p.hslope) * std::cos(2. * x3t);
    }
    gk[3 * (k - 1)] = std::sin(th);
    gk[3 * (k - 1) + 1] = std::cos(th);
    gk[3 * (k - 1) + 2] = hfac;
  }
  const size_t npt = (size_t)p.imax * (size_t)p.kmax * (jslice ? 1 : (size_t)p.jmax);
  double* buf = nullptr;
  const size_t nbuf = gi.size() + gk.size() + 7 * npt;
  RG_CUDA(cudaMalloc(&buf, nbuf * sizeof(double)));
  double* dgi = buf;
  double* dgk = buf + gi.size();
  double* dout = dgk + gk.size();
  cudaError_t e = cudaMemcpyAsync(dgi, gi.data(), gi.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dgk, gk.data(), gk.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = launch_derived(R->d, R->b.P[R->cur], dgi, dgk, p.akm, jslice, dout, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out, dout, 7 * npt * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(buf);
  RG_CUDA(e);
  return RG_OK;
}

// ------------------------------------------------------------ restart files
// ------------------------------------------------------------ restart files
// store1 / restar2 (restar.f90:5-88, 273-346) write and read one rank's state
// as gfortran sequential unformatted records (a 4-byte length before and
// after each record): (myrank, nd), (it0, ih0), (time), then for every cell in
// (k, j, i) order four records of nv = 9 doubles: uu, u0, uri, uri0.
namespace {

bool put_record(FILE* f, const void* data, uint32_t n) {
  return fwrite(&n, 4, 1, f) == 1 && (n == 0 || fwrite(data, n, 1, f) == 1) && fwrite(&n, 4, 1, f) == 1;
}
bool get_record(FILE* f, void* data, uint32_t n) {
  uint32_t a = 0, b = 0;
  if (fread(&a, 4, 1, f) != 1 || a != n) return false;
  if (n && fread(data, n, 1, f) != 1) return false;
  return fread(&b, 4, 1, f) == 1 && b == n;
}

}  // namespace

int rg_run_store(rg_ctx* ctx, int run, const char* path, int it0, int ih0, int nd, const double* uri0) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  if (!path) return fail(RG_EINVAL_CONFIG, "null path");
  const size_t nf = R->nfull;
  std::vector<double> uri(9 * nf), uu(9 * nf), u0(9 * nf), p0;
  int rc = rg_run_download_prims(ctx, run, uri.data());
  if (rc) return rc;
  if ((rc = rg_caluu1(ctx, run, uri.data(), uu.data()))) return rc;
  const double* pr0 = uri0 ? uri0 : uri.data();
  if ((rc = rg_caluu1(ctx, run, pr0, u0.data()))) return rc;
  Scal sc{};
  RG_CUDA(cudaMemcpyAsync(&sc, R->d.scal, sizeof(Scal), cudaMemcpyDeviceToHost, ctx->stream));
  RG_CUDA(cudaStreamSynchronize(ctx->stream));
  FILE* f = std::fopen(path, "wb");
  if (!f) return fail(RG_EINVAL_CONFIG, std::string("cannot open ") + path);
  const int32_t h1[2] = {0, nd}, h2[2] = {it0, ih0};
  const double time = sc.timeh;
  bool ok = put_record(f, h1, 8) && put_record(f, h2, 8) && put_record(f, &time, 8);
  for (size_t c = 0; ok && c < nf; ++c)
    ok = put_record(f, &uu[9 * c], 72) && put_record(f, &u0[9 * c], 72) && put_record(f, &uri[9 * c], 72) &&
         put_record(f, &pr0[9 * c], 72);
  ok = (std::fclose(f) == 0) && ok;
  return ok ? RG_OK : fail(RG_EINVAL_CONFIG, std::string("write failed: ") + path);
}

int rg_run_restore(rg_ctx* ctx, int run, const char* path, int* it0, int* ih0, int* nd, double* uri0) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  if (!path) return fail(RG_EINVAL_CONFIG, "null path");
  FILE* f = std::fopen(path, "rb");
  if (!f) return fail(RG_EINVAL_CONFIG, std::string("cannot open ") + path);
  const size_t nf = R->nfull;
  int32_t h1[2], h2[2];
  double time = 0.0;
  std::vector<double> uri(9 * nf), rec(9);
  bool ok = get_record(f, h1, 8) && get_record(f, h2, 8) && get_record(f, &time, 8);
  for (size_t c = 0; ok && c < nf; ++c) {
    ok = get_record(f, rec.data(), 72) && get_record(f, rec.data(), 72) && get_record(f, &uri[9 * c], 72) &&
         get_record(f, uri0 ? uri0 + 9 * c : rec.data(), 72);
  }
  std::fclose(f);
  if (!ok) return fail(RG_EINVAL_CONFIG, std::string("not a restart file of this grid: ") + path);
  if (it0) *it0 = h2[0];
  if (ih0) *ih0 = h2[1];
  if (nd) *nd = h1[1];
  return rg_run_upload_prims(ctx, run, uri.data(), time);  // restart at timeh (main.f90:560-571)
}

int rg_run_horizon_flux(rg_ctx* ctx, int run, double* mdot, double* edot) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  return rg_run_radial_flux(ctx, run, R->d.nm1, mdot, edot);
}

int rg_run_radial_flux(rg_ctx* ctx, int run, int iface, double* mdot, double* edot) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  if (!mdot || !edot) return fail(RG_EINVAL_CONFIG, "null output");
  if (iface < R->d.nm0 || iface > R->d.imax - R->d.nm0)
    return fail(RG_EINVAL_CONFIG, "radial face index outside the hll range nm0..imax-nm0");
  const DevRun d = full_view(R);
  DevBufs* B = nullptr;
  int rc = full_bufs(R, ctx->stream, &B);
  if (rc) return rc;
  // the run's current primitives in the full layout
  RG_CUDA(launch_soa_to_aos(R->d, R->b.P[R->cur], B->stage2, ctx->stream));
  int* nobad = nullptr;
  RG_CUDA(launch_aos_to_soa(d, B->stage2, B->stage, nobad, ctx->stream));
  // fluxes on the per-routine scalar block: the run's own time state is left alone
  if ((rc = reset_fscal(ctx, R))) return rc;
  RG_CUDA(launch_flux(d, 1, B->stage, B->F[0], ctx->stream));
  // radial face iface+1/2: F1 of rho u^r and of the energy variable
  const int i = iface;
  std::vector<double> f0((size_t)d.jmax * d.kmax), f4((size_t)d.jmax * d.kmax);
  // in the full layout the faces (i, j, k) of fixed i lie imax values apart
  const size_t rows = (size_t)d.jmax * d.kmax, pitch = (size_t)d.imax * sizeof(double);
  RG_CUDA(cudaMemcpy2DAsync(f0.data(), sizeof(double), B->F[0] + d.cell(i, 1, 1), pitch, sizeof(double), rows,
                            cudaMemcpyDeviceToHost, ctx->stream));
  RG_CUDA(cudaMemcpy2DAsync(f4.data(), sizeof(double), B->F[0] + 4 * d.N + d.cell(i, 1, 1), pitch, sizeof(double),
                            rows, cudaMemcpyDeviceToHost, ctx->stream));
  RG_CUDA(cudaStreamSynchronize(ctx->stream));
  const Axis& X2 = R->geom.ax[1];
  const Axis& X3 = R->geom.ax[2];
  double m = 0.0, e = 0.0;
  for (int k = d.nm1 + 1; k <= d.kmax - d.nm1; ++k)
    for (int j = d.nm1 + 1; j <= d.jmax - d.nm1; ++j) {
      const size_t o = (size_t)(j - 1) + (size_t)d.jmax * (k - 1);
      const double area = X2.dx[j] * X3.dx[k];
      m += f0[o] * area;
      e += f4[o] * area;
    }
  *mdot = -m;
  *edot = -e;
  return RG_OK;
}

// output1 (restar.f90:91-185): the records are formatted on the device in
// chunks, each copied by one cudaMemcpyAsync into one of two pinned host
// buffers, so that the formatting and copy of a chunk overlap the file write
// of the previous one.
int rg_run_output(rg_ctx* ctx, int run, const char* path, int myrank, int npe) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  if (!path) return fail(RG_EINVAL_CONFIG, "null path");
  RG_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  Scal sc{};
  RG_CUDA(cudaMemcpyAsync(&sc, R->d.scal, sizeof(Scal), cudaMemcpyDeviceToHost, s));
  RG_CUDA(cudaStreamSynchronize(s));
  const DevRun& d = R->d;
  // the coordinates output1 carries: x?b for metric 403, x? otherwise (main.f90:711-717)
  const bool mks = (R->p.metric == 403);
  std::vector<double> axes;
  const int ext[3] = {d.imax, d.jmax, d.kmax};
  for (int a = 0; a < 3; ++a) {
    const std::vector<double>& x = mks ? R->geom.ax[a].xb : R->geom.ax[a].x;
    for (int m = 1; m <= ext[a]; ++m) axes.push_back(x[m]);
  }
  const size_t nrec = (size_t)d.imax * d.jmax * d.kmax;
  const size_t chunk = std::min<size_t>(nrec, (size_t)1 << 19);  // records per chunk (56 MB)
  const size_t cbytes = chunk * 112;
  double* dax = nullptr;
  unsigned* dbuf = nullptr;
  unsigned char* hbuf = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  FILE* f = nullptr;
  int rc = RG_OK;
  auto cleanup = [&]() {
    if (f) std::fclose(f);
    for (cudaEvent_t e : ev)
      if (e) cudaEventDestroy(e);
    cudaFree(dax);
    cudaFree(dbuf);
    cudaFreeHost(hbuf);
  };
  cudaError_t e = cudaMalloc(&dax, axes.size() * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&dbuf, 2 * cbytes);
  if (e == cudaSuccess) e = cudaMallocHost(&hbuf, 2 * cbytes);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dax, axes.data(), axes.size() * sizeof(double), cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) {
    cleanup();
    return fail(RG_ECUDA, std::string("rg_run_output: ") + cudaGetErrorString(e));
  }
  f = std::fopen(path, "wb");
  if (!f) {
    cleanup();
    return fail(RG_EINVAL_CONFIG, std::string("cannot open ") + path);
  }
  unsigned char h1[16];
  std::memcpy(h1, &sc.timeh, 8);
  std::memcpy(h1 + 8, &myrank, 4);
  std::memcpy(h1 + 12, &npe, 4);
  const int32_t h2[6] = {1, d.imax, 1, d.jmax, 1, d.kmax};
  bool ok = put_record(f, h1, 16) && put_record(f, h2, 24);
  const size_t nchunks = (nrec + chunk - 1) / chunk;
  for (size_t c = 0; ok && c <= nchunks; ++c) {
    if (c < nchunks) {  // format and copy chunk c
      const int b = (int)(c % 2);
      const size_t r0 = c * chunk, n = std::min(chunk, nrec - r0);
      unsigned* db = dbuf + (size_t)b * (cbytes / 4);
      e = launch_output1(d, R->b.P[R->cur], dax, dax + d.imax, dax + d.imax + d.jmax, r0, n, db, s);
      if (e == cudaSuccess) e = cudaMemcpyAsync(hbuf + (size_t)b * cbytes, db, n * 112, cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaEventRecord(ev[b], s);
      if (e != cudaSuccess) break;
    }
    if (c >= 1) {  // write chunk c-1 while chunk c is formatted and copied
      const int b = (int)((c - 1) % 2);
      const size_t n = std::min(chunk, nrec - (c - 1) * chunk);
      e = cudaEventSynchronize(ev[b]);
      if (e != cudaSuccess) break;
      ok = std::fwrite(hbuf + (size_t)b * cbytes, n * 112, 1, f) == 1;
    }
  }
  if (e != cudaSuccess) rc = fail(RG_ECUDA, std::string("rg_run_output: ") + cudaGetErrorString(e));
  else if (!ok) rc = fail(RG_EINVAL_CONFIG, std::string("write failed: ") + path);
  if (std::fclose(f) != 0 && rc == RG_OK) rc = fail(RG_EINVAL_CONFIG, std::string("write failed: ") + path);
  f = nullptr;
  cudaStreamSynchronize(s);
  cleanup();
  return rc;
}

int rg_run_divb(rg_ctx* ctx, int run, double* divb_max, double* b_scale) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  if (!divb_max || !b_scale) return fail(RG_EINVAL_CONFIG, "null output");
  RG_CUDA(cudaSetDevice(ctx->device));
  unsigned long long* red = nullptr;
  RG_CUDA(cudaMalloc(&red, 2 * sizeof(unsigned long long)));
  unsigned long long h[2] = {0, 0};
  cudaError_t e = launch_divb(R->d, R->b.P[R->cur], red, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, red, sizeof h, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(red);
  if (e != cudaSuccess) return fail(RG_ECUDA, std::string("rg_run_divb: ") + cudaGetErrorString(e));
  std::memcpy(divb_max, &h[0], sizeof(double));
  std::memcpy(b_scale, &h[1], sizeof(double));
  return RG_OK;
}

// ---- rec2, calcha, hll and ct one at a time (the reference's separate calls,
// main.f90:807-831).  Arrays in the reference layout, host or device memory.
namespace {
// Device scratch of the per-routine calls below, freed on return.
struct Scratch {
  double* p = nullptr;
  ~Scratch() { cudaFree(p); }
  int alloc(size_t n) {
    if (cudaMalloc(&p, n * sizeof(double)) != cudaSuccess) {
      (void)cudaGetLastError();
      return fail(RG_ENOMEM_ADMIT, "per-routine scratch does not fit");
    }
    return RG_OK;
  }
};
}  // namespace

int rg_rec2(rg_ctx* ctx, int run, const double* uri, double* face_prims, double* face_cons, double* face_flux) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  if (!uri || !face_prims) return fail(RG_EINVAL_CONFIG, "null array");
  const DevRun d = full_view(R);
  const size_t N = d.N, n9 = 9 * N;
  DevBufs* B = nullptr;
  int rc = full_bufs(R, ctx->stream, &B);
  if (rc || (rc = to_soa(ctx, R, uri, B->stage, d, false)) || (rc = reset_fscal(ctx, R))) return rc;
  Scratch S;  // 18 face arrays: prims, cons, flux x (il, ir, jl, jr, kl, kr)
  if ((rc = S.alloc(18 * n9))) return rc;
  RG_CUDA(cudaMemsetAsync(S.p, 0, 18 * n9 * sizeof(double), ctx->stream));
  for (int dir = 1; dir <= 3; ++dir) {
    double* const q[2] = {S.p + (2 * (dir - 1)) * n9, S.p + (2 * (dir - 1) + 1) * n9};
    double* const u[2] = {q[0] + 6 * n9, q[1] + 6 * n9};
    double* const w[2] = {q[0] + 12 * n9, q[1] + 12 * n9};
    RG_CUDA(launch_rec2(d, dir, B->stage, B->F[dir - 1], q, u, w, ctx->stream));
  }
  double* outs[3] = {face_prims, face_cons, face_flux};
  for (int a = 0; a < 3; ++a) {
    if (!outs[a]) continue;
    for (int m = 0; m < 6; ++m)
      if ((rc = from_soa(ctx, R, S.p + (size_t)(6 * a + m) * n9, outs[a] + (size_t)m * n9, d))) return rc;
  }
  return RG_OK;
}

int rg_calcha(rg_ctx* ctx, int run, const double* face_prims, double* cha) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  if (!face_prims || !cha) return fail(RG_EINVAL_CONFIG, "null array");
  const DevRun d = full_view(R);
  const size_t N = d.N, n9 = 9 * N;
  Scratch S;  // 6 face arrays, then 6 speed arrays
  int rc = S.alloc(6 * n9 + 6 * N);
  if (rc) return rc;
  for (int m = 0; m < 6; ++m)
    if ((rc = to_soa(ctx, R, face_prims + (size_t)m * n9, S.p + (size_t)m * n9, d, false))) return rc;
  double* C = S.p + 6 * n9;
  RG_CUDA(cudaMemsetAsync(C, 0, 6 * N * sizeof(double), ctx->stream));
  for (int dir = 1; dir <= 3; ++dir)
    RG_CUDA(launch_calcha(d, dir, S.p + (2 * (dir - 1)) * n9, S.p + (2 * (dir - 1) + 1) * n9,
                          C + (2 * (dir - 1)) * N, C + (2 * (dir - 1) + 1) * N, ctx->stream));
  RG_CUDA(cudaMemcpyAsync(cha, C, 6 * N * sizeof(double), cudaMemcpyDefault, ctx->stream));
  RG_CUDA(cudaStreamSynchronize(ctx->stream));
  return RG_OK;
}

int rg_hll(rg_ctx* ctx, int run, const double* face_cons, const double* face_flux, const double* cha, double* ww) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  if (!face_cons || !face_flux || !cha || !ww) return fail(RG_EINVAL_CONFIG, "null array");
  const DevRun d = full_view(R);
  const size_t N = d.N, n9 = 9 * N;
  DevBufs* B = nullptr;
  int rc = full_bufs(R, ctx->stream, &B);
  if (rc) return rc;
  Scratch S;  // 6 conserved, 6 flux face arrays, 6 speed arrays
  if ((rc = S.alloc(12 * n9 + 6 * N))) return rc;
  for (int m = 0; m < 6; ++m) {
    if ((rc = to_soa(ctx, R, face_cons + (size_t)m * n9, S.p + (size_t)m * n9, d, false))) return rc;
    if ((rc = to_soa(ctx, R, face_flux + (size_t)m * n9, S.p + (size_t)(6 + m) * n9, d, false))) return rc;
  }
  double* C = S.p + 12 * n9;
  RG_CUDA(cudaMemcpyAsync(C, cha, 6 * N * sizeof(double), cudaMemcpyDefault, ctx->stream));
  if ((rc = ww_in(ctx, R, B, ww))) return rc;
  for (int dir = 1; dir <= 3; ++dir) {
    const size_t l = 2 * (dir - 1), rr = l + 1;
    RG_CUDA(launch_hll(d, dir, S.p + l * n9, S.p + rr * n9, S.p + (6 + l) * n9, S.p + (6 + rr) * n9, C + l * N,
                       C + rr * N, B->F[dir - 1], ctx->stream));
  }
  return ww_out(ctx, R, B, ww);
}

int rg_ct(rg_ctx* ctx, int run, const double* uri, double* ww) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  if (!uri || !ww) return fail(RG_EINVAL_CONFIG, "null array");
  DevRun d = full_view(R);
  DevBufs* B = nullptr;
  int rc = full_bufs(R, ctx->stream, &B);
  if (rc || (rc = to_soa(ctx, R, uri, B->stage, d, false)) || (rc = reset_fscal(ctx, R))) return rc;
  d.ctd = B->ctd;
  if ((rc = ww_in(ctx, R, B, ww))) return rc;
  if (d.guard & 2) {  // the zero normal-field fluxes come before the CT averages read the planes
    DevRun z = d;
    z.ict = 0;  // zeroing only
    RG_CUDA(launch_ct_apply(z, B->CT, B->F[0], B->F[1], B->F[2], ctx->stream));
  }
  RG_CUDA(launch_ct(d, B->stage, B->F[0], B->F[1], B->F[2], B->CT, ctx->stream));
  RG_CUDA(launch_ct_apply(d, B->CT, B->F[0], B->F[1], B->F[2], ctx->stream));
  return ww_out(ctx, R, B, ww);
}

int rg_recov(rg_ctx* ctx, int run, const double* uu, double* uri) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  if (!uu || !uri) return fail(RG_EINVAL_CONFIG, "null array");
  const DevRun d = full_view(R);
  DevBufs* B = nullptr;
  int rc = full_bufs(R, ctx->stream, &B);
  if (rc || (rc = to_soa(ctx, R, uu, B->stage, d, false))) return rc;
  if ((rc = to_soa(ctx, R, uri, B->stage2, d, false)) || (rc = reset_fscal(ctx, R))) return rc;
  RG_CUDA(launch_recov_only(d, B->stage, B->stage2, B->F[0], ctx->stream));
  return from_soa(ctx, R, B->F[0], uri, d);
}

int rg_cdtcfl(rg_ctx* ctx, int run, const double* uri, double* dtcfl) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  if (!uri || !dtcfl) return fail(RG_EINVAL_CONFIG, "null array");
  const DevRun d = full_view(R);
  DevBufs* B = nullptr;
  int rc = full_bufs(R, ctx->stream, &B);
  if (rc || (rc = to_soa(ctx, R, uri, B->stage, d, false)) || (rc = reset_fscal(ctx, R, 1.0))) return rc;
  Scal sc{};
  RG_CUDA(launch_cfl(d, B->stage, ctx->stream));
  RG_CUDA(cudaMemcpyAsync(&sc, d.scal, sizeof(Scal), cudaMemcpyDeviceToHost, ctx->stream));
  RG_CUDA(cudaStreamSynchronize(ctx->stream));
  std::memcpy(dtcfl, &sc.dtcfl_bits, sizeof(double));
  return RG_OK;
}

int rg_bnd4(rg_ctx* ctx, int run, double* uri, const double* urio) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  if (!uri || !urio) return fail(RG_EINVAL_CONFIG, "null array");
  const DevRun d = full_view(R);
  DevBufs* B = nullptr;
  int rc = full_bufs(R, ctx->stream, &B);
  if (rc || (rc = to_soa(ctx, R, uri, B->stage, d, false))) return rc;
  if ((rc = to_soa(ctx, R, urio, B->stage2, d, false)) || (rc = reset_fscal(ctx, R))) return rc;
  RG_CUDA(launch_bc(d, B->stage, B->stage2, ctx->stream));
  return from_soa(ctx, R, B->stage, uri, d);
}

namespace {
int floor_part(rg_ctx* ctx, int run, int part, double* uri) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  if (!uri) return fail(RG_EINVAL_CONFIG, "null array");
  const DevRun d = full_view(R);
  DevBufs* B = nullptr;
  int rc = full_bufs(R, ctx->stream, &B);
  if (rc || (rc = to_soa(ctx, R, uri, B->stage, d, false)) || (rc = reset_fscal(ctx, R))) return rc;
  RG_CUDA(launch_floor_part(d, part, B->stage, ctx->stream));
  return from_soa(ctx, R, B->stage, uri, d);
}
}  // namespace

int rg_infchk(rg_ctx* ctx, int run, double* uri) { return floor_part(ctx, run, 1, uri); }
int rg_atmosphere1a(rg_ctx* ctx, int run, double* uri) { return floor_part(ctx, run, 2, uri); }
int rg_pminmax2b(rg_ctx* ctx, int run, double* uri) { return floor_part(ctx, run, 4, uri); }

int rg_bnd_floor(rg_ctx* ctx, int run, double* uri, const double* urio) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  if (!uri || !urio) return fail(RG_EINVAL_CONFIG, "null array");
  const DevRun d = full_view(R);
  DevBufs* B = nullptr;
  int rc = full_bufs(R, ctx->stream, &B);
  if (rc || (rc = to_soa(ctx, R, uri, B->stage, d, false))) return rc;
  if ((rc = to_soa(ctx, R, urio, B->stage2, d, false)) || (rc = reset_fscal(ctx, R))) return rc;
  RG_CUDA(launch_bc(d, B->stage, B->stage2, ctx->stream));
  RG_CUDA(launch_floor(d, B->stage, ctx->stream));
  return from_soa(ctx, R, B->stage, uri, d);
}

}  // extern "C"

// ------------------------------------------------------ the step's power function
namespace {
__global__ void k_pow_eval(const double* __restrict__ x, const double* __restrict__ y, double* __restrict__ o,
                           size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) o[i] = rgm::pow(x[i], y[i]);
}
}  // namespace

extern "C" int rg_pow_eval(rg_ctx* ctx, const double* x, const double* y, double* out, size_t n) {
  if (!ctx) return fail(RG_EINVAL_CONFIG, "null context");
  if (n == 0) return RG_OK;
  if (!x || !y || !out) return fail(RG_EINVAL_CONFIG, "null array");
  RG_CUDA(cudaSetDevice(ctx->device));
  double* d = nullptr;
  RG_CUDA(cudaMalloc(&d, 3 * n * sizeof(double)));
  cudaStream_t s = ctx->stream;
  cudaError_t e = cudaMemcpyAsync(d, x, n * sizeof(double), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d + n, y, n * sizeof(double), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) {
    k_pow_eval<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(d, d + n, d + 2 * n, n);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, d + 2 * n, n * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(d);
  if (e != cudaSuccess) return fail(RG_ECUDA, std::string("rg_pow_eval: ") + cudaGetErrorString(e));
  return RG_OK;
}

// ------------------------------------------------------ allocation-free fluxes
// rg_calflx_static serves callers that cannot let the library call cudaMalloc
// when they need the fluxes: a host program whose device memory comes only
// from its own pool or arena (a framework's caching allocator, a driver given
// a fixed memory budget), where a cudaMalloc behind its back would
// synchronise the device and take memory the pool does not know about.  The
// caller owns the input and output device buffers; the flux-CT intermediate
// (the six averaged induction fluxes) and the kernels' scalar block live in
// the file-scope device arrays below, sized for grids of at most
// kStaticMaxCells cells.  Every GPU that loads this library holds these
// arrays (about 12.6 MB) until the process exits; with CUDA's lazy module
// loading the module, and with it the arrays, is typically loaded by a
// device's first call, which is therefore the one call that may allocate.
namespace {

constexpr size_t kStaticMaxCells = (size_t)1 << 18;
__device__ __align__(256) double g_static_ct[6 * kStaticMaxCells];
__device__ __align__(256) Scal g_static_scal;

constexpr int kMaxDevices = 64;
double* g_static_ct_addr[kMaxDevices] = {};
Scal* g_static_scal_addr[kMaxDevices] = {};
std::mutex g_static_mu;  // guards the per-device address look-up above

// Copy the flux-CT values from the static array into the caller's fluxes over
// the CT range nm1..n-nm1 (ct.f90:60-109); elsewhere the raw LLF fluxes stay.
__global__ void k_ct_scatter(DevRun r, const double* __restrict__ ct, double* __restrict__ ww) {
  const int nm1 = r.nm1;
  const int i = blockIdx.x * blockDim.x + threadIdx.x + nm1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + nm1;
  const int k = blockIdx.z * blockDim.z + threadIdx.z + nm1;
  if (i > r.imax - nm1 || j > r.jmax - nm1 || k > r.kmax - nm1) return;
  const size_t N = r.N, c = r.cell(i, j, k);
  // (direction, variable) of the six replaced fluxes: ww(2,7) ww(3,7) ww(1,8) ww(3,8) ww(1,9) ww(2,9)
  const int dir[6] = {1, 2, 0, 2, 0, 1}, var[6] = {6, 6, 7, 7, 8, 8};
#pragma unroll
  for (int q = 0; q < 6; ++q) ww[((size_t)dir[q] * 9 + var[q]) * N + c] = ct[(size_t)q * N + c];
}

// Reset the static scalar block: zero, then mark the kernels' work as active.
__global__ void k_static_scal_reset(Scal* s) {
  Scal z{};
  z.active = 1;
  *s = z;
}

}  // namespace

extern "C" int rg_calflx_static(rg_ctx* ctx, int run, const double* d_prims, double* d_ww) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  if (!d_prims || !d_ww) return fail(RG_EINVAL_CONFIG, "null device buffer");
  if (R->d.ict == 3)
    return fail(RG_EINVAL_CONFIG, "rg_calflx_static: upwind flux-CT (ict 3) needs its difference planes (rg_calflx)");
  const size_t N = R->nfull;
  if (N > kStaticMaxCells)
    return fail(RG_EINVAL_CONFIG, "rg_calflx_static: grid of " + std::to_string(N) +
                                      " cells exceeds the static scratch maximum of " +
                                      std::to_string(kStaticMaxCells) + " cells");
  if (ctx->device < 0 || ctx->device >= kMaxDevices) return fail(RG_EINVAL_CONFIG, "device index out of range");
  RG_CUDA(cudaSetDevice(ctx->device));
  // Set-up once per device, with that device current: the host-side names of
  // the arrays are not device addresses, so their addresses are looked up here
  // (under a lock, so that threads making their first calls on one device at
  // the same time do not race on the table).
  double* ct = nullptr;
  Scal* scal = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_static_mu);
    if (!g_static_ct_addr[ctx->device]) {
      void* a = nullptr;
      void* b = nullptr;
      RG_CUDA(cudaGetSymbolAddress(&a, g_static_ct));
      RG_CUDA(cudaGetSymbolAddress(&b, g_static_scal));
      g_static_ct_addr[ctx->device] = static_cast<double*>(a);
      g_static_scal_addr[ctx->device] = static_cast<Scal*>(b);
    }
    ct = g_static_ct_addr[ctx->device];
    scal = g_static_scal_addr[ctx->device];
  }
  DevRun d = full_view(R);
  d.scal = scal;  // the run's own time state is not touched
  cudaStream_t s = ctx->stream;
  // The arrays keep the previous call's contents: clear them first.
  RG_CUDA(cudaMemsetAsync(ct, 0, 6 * N * sizeof(double), s));
  k_static_scal_reset<<<1, 1, 0, s>>>(d.scal);
  RG_CUDA(cudaGetLastError());
  for (int dir = 1; dir <= 3; ++dir) RG_CUDA(launch_flux(d, dir, d_prims, d_ww + (size_t)(dir - 1) * 9 * N, s));
  RG_CUDA(launch_ct(d, d_prims, d_ww, d_ww + 9 * N, d_ww + 18 * N, ct, s));
  const dim3 b(64, 4, 1);
  const int n = d.imax - 2 * d.nm1 + 1, m = d.jmax - 2 * d.nm1 + 1, l = d.kmax - 2 * d.nm1 + 1;
  k_ct_scatter<<<dim3((n + 63) / 64, (m + 3) / 4, l), b, 0, s>>>(d, ct, d_ww);
  RG_CUDA(cudaGetLastError());
  RG_CUDA(cudaStreamSynchronize(s));
  return RG_OK;
}
