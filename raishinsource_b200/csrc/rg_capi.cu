// rg_capi.cu -- the C ABI of include/raishin_gpu.h: contexts, run admission
// by device footprint, host<->device layout conversion, the device-resident
// RK3 step driver and the per-routine entry points.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/raishin_gpu.h"
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
  DevBufs b{};
  double* aos = nullptr;   // 9*N staging buffer in the reference layout
  int cur = 0;             // index of P^n in b.P
  std::vector<void*> allocs;
  size_t bytes = 0;
  HostGeom geom;
};

}  // namespace

// Kernel kinds timed by the profiling mode (rg_profile).
enum Kind { K_CFL = 0, K_FLUX1, K_FLUX2, K_FLUX3, K_CT, K_UPDATE, K_BC, K_FLOOR, K_SCALAR, K_NKINDS };

struct rg_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::map<int, Run*> runs;
  int next_id = 1;
  long long launches[K_NKINDS] = {};   // kernel launches issued, per kind
  bool prof = false;                   // bracket every launch with CUDA events
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
  std::vector<cudaEvent_t> pool;
  double ms[K_NKINDS] = {};
  bool own_stream = true;              // false after rg_ctx_set_stream
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

int check_params(const rg_run_params* p) {
  if (!p) return fail(RG_EINVAL_CONFIG, "null parameters");
  if (p->irec != 5 && p->irec != 6 && p->irec != 7)
    return fail(RG_EINVAL_CONFIG, "irec must be 5 (PPM), 6 (MP5) or 7 (WENO5)");
  if (p->metric != 1 && p->metric != 303 && p->metric != 403)
    return fail(RG_EINVAL_CONFIG, "metric must be 1, 303 or 403");
  if (p->ix1 != 1 && p->ix1 != 2) return fail(RG_EINVAL_CONFIG, "ix1 must be 1 or 2");
  if (p->ix2 != 1) return fail(RG_EINVAL_CONFIG, "ix2 must be 1");
  if (p->ix3 != 1 && p->ix3 != 2) return fail(RG_EINVAL_CONFIG, "ix3 must be 1 or 2");
  if (p->precision != RG_FP64 && p->precision != RG_MIXED) return fail(RG_EINVAL_CONFIG, "unknown precision mode");
  const int nm1 = (p->irec == 5) ? 5 : 4;
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

size_t footprint_bytes(const rg_run_params* p) {
  const size_t N = (size_t)p->imax * p->jmax * p->kmax;
  const size_t nik = (size_t)p->imax * p->kmax;
  const size_t state = (3 * 9 + 3 * 9 + 6 + 2 * 9 + 9 + 9) * N * sizeof(double);
  const size_t geom = (3 * kMetComps + 64) * nik * sizeof(double) + 16 * (size_t)(p->imax + p->jmax + p->kmax) * sizeof(double);
  size_t mixed = 0;
  if (p->precision == RG_MIXED)  // P32, F32 x3, CT32; FP32 metric caches and Christoffels
    mixed = (9 + 27 + 6) * N * sizeof(float) + (3 * kMetComps + 64) * nik * sizeof(float);
  return state + geom + mixed + sizeof(Scal) + C_NCOUNTERS * 8 + kCarryCap * sizeof(int);
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

// rec2's dummy dx?b(2:n-1) receives actual dx?b(1:n-1) (rec.f90:58, main.f90:120):
// dummy index m holds actual m-1; dummy 1 (outside the actual array) is taken as actual 1.
std::vector<double> shifted(const std::vector<double>& v, int n) {
  std::vector<double> o(n, 0.0);
  for (int m = 2; m <= n; ++m) o[m - 1] = v[m - 1];
  o[0] = v[1];
  return o;
}

// The per-routine entry points compute in FP64 whatever the run's precision.
DevRun fp64_view(const Run* R) {
  DevRun d = R->d;
  d.mixed = 0;
  d.P32 = nullptr;
  return d;
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

int to_soa(rg_ctx* ctx, Run* R, const double* host_aos, double* dev_soa) {
  const size_t N = R->d.N;
  RG_CUDA(cudaMemcpyAsync(R->aos, host_aos, 9 * N * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  RG_CUDA(launch_aos_to_soa(R->aos, dev_soa, N, ctx->stream));
  return RG_OK;
}

int from_soa(rg_ctx* ctx, Run* R, const double* dev_soa, double* host_aos) {
  const size_t N = R->d.N;
  RG_CUDA(launch_soa_to_aos(dev_soa, R->aos, N, ctx->stream));
  RG_CUDA(cudaMemcpyAsync(host_aos, R->aos, 9 * N * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
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

int bc_launches(const DevRun& r) {
  int n = 0;
  for (int side0 = 0; side0 <= 4; side0 += 2) {
    bool per = false, phys = false;
    for (int sd = side0; sd <= side0 + 1; ++sd)
      for (int v = 0; v < 9; ++v) {
        per = per || r.ibc[sd][v] == 1;
        phys = phys || (r.ibc[sd][v] != 1 && r.ibc[sd][v] != 0);
      }
    n += per + phys;
  }
  return n;
}

// One RK3 stage (main.f90:807-911 / 919-1032 / 1043-1147).
int run_stage(rg_ctx* ctx, Run* R, int stage, const double* Pn, const double* Pc, double* Pw) {
  const DevRun& d = R->d;
  cudaStream_t s = ctx->stream;
  const int nf = n_flux_launches(d);
  RG_CUDA(issue(ctx, K_FLUX1, nf, [&] { return launch_flux(d, 1, Pc, R->b.F[0], s); }));
  RG_CUDA(issue(ctx, K_FLUX2, nf, [&] { return launch_flux(d, 2, Pc, R->b.F[1], s); }));
  RG_CUDA(issue(ctx, K_FLUX3, nf, [&] { return launch_flux(d, 3, Pc, R->b.F[2], s); }));
  RG_CUDA(issue(ctx, K_CT, n_ct_launches(d), [&] { return launch_ct(d, R->b.F[0], R->b.F[1], R->b.F[2], R->b.CT, s); }));
  RG_CUDA(issue(ctx, K_UPDATE, n_update_launches(d), [&] {
    return launch_update(d, stage, Pn, Pc, Pw, R->b.F[0], R->b.F[1], R->b.F[2], R->b.CT, s);
  }));
  RG_CUDA(issue(ctx, K_BC, bc_launches(d), [&] { return launch_bc(d, Pw, Pn, s); }));
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
  if (c[C_CARRY_OVF]) return fail(RG_EOVERFLOW, "W-carry list overflowed");
  if (c[C_CAP] || c[C_FLOORCAP]) return fail(RG_ENR_CAP, "a capped rescale loop was hit");
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
  for (auto& kv : ctx->runs) free_run(kv.second);
  for (auto& pe : ctx->pending) ctx->pool.push_back(pe.second.first), ctx->pool.push_back(pe.second.second);
  for (cudaEvent_t e : ctx->pool) cudaEventDestroy(e);
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

int rg_run_footprint(const rg_run_params* p, size_t* bytes) {
  const int rc = check_params(p);
  if (rc) return rc;
  if (bytes) *bytes = footprint_bytes(p);
  return RG_OK;
}

int rg_run_admit(rg_ctx* ctx, const rg_run_params* p, int* run_id) {
  if (!ctx || !run_id) return fail(RG_EINVAL_CONFIG, "null argument");
  int rc = check_params(p);
  if (rc) return rc;
  RG_CUDA(cudaSetDevice(ctx->device));
  size_t free_b = 0, total_b = 0;
  RG_CUDA(cudaMemGetInfo(&free_b, &total_b));
  const size_t need = footprint_bytes(p);
  if (need + (size_t)256 * 1024 * 1024 > free_b)
    return fail(RG_ENOMEM_ADMIT, "run footprint " + std::to_string(need) + " B exceeds free device memory");
  Run* R = new Run();
  R->p = *p;
  build_geometry(*p, R->geom);
  if (!R->geom.compact_ok) {
    delete R;
    return fail(RG_EINVAL_CONFIG, "metric couples theta to (t,r,phi): not representable by the compact cache");
  }
  DevRun& d = R->d;
  d.imax = p->imax; d.jmax = p->jmax; d.kmax = p->kmax;
  d.nm0 = (p->irec == 5) ? 4 : 3;
  d.nm1 = d.nm0 + 1;
  d.irec = p->irec; d.model = p->model; d.guard = p->guard; d.iter = p->iter;
  d.mixed = (p->precision == RG_MIXED);
  d.gkind = (p->gam == 4.0 / 3.0) ? 1 : (p->gam == 5.0 / 3.0 ? 2 : 0);
  // cells inside r < 2 r_H keep FP64 in the mixed path (Kerr metrics only)
  d.i_fp64 = 0;
  if (p->metric == 303 || p->metric == 403) {
    const double r2h = 2.0 * (1.0 + std::sqrt(1.0 - p->akm * p->akm));
    for (int i = 1; i <= p->imax; ++i)
      if (R->geom.ax[0].x[i] < r2h) d.i_fp64 = i;
  }
  d.nmax_cfl = d.nm1 * 2 + (d.nm1 - 1);
  d.N = (size_t)p->imax * p->jmax * p->kmax;
  d.nik = (size_t)p->imax * p->kmax;
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
    if ((rc = dalloc(R, &ptr, 9 * N * sizeof(double)))) return bail(rc);
    R->b.F[k] = static_cast<double*>(ptr);
  }
  if ((rc = dalloc(R, &ptr, 6 * N * sizeof(double)))) return bail(rc);
  R->b.CT = static_cast<double*>(ptr);
  if ((rc = dalloc(R, &ptr, 9 * N * sizeof(double)))) return bail(rc);
  R->b.stage = static_cast<double*>(ptr);
  if ((rc = dalloc(R, &ptr, 9 * N * sizeof(double)))) return bail(rc);
  R->b.stage2 = static_cast<double*>(ptr);
  if ((rc = dalloc(R, &ptr, 9 * N * sizeof(double)))) return bail(rc);
  R->aos = static_cast<double*>(ptr);
  if ((rc = dalloc(R, &ptr, 9 * N * sizeof(double)))) return bail(rc);
  d.Un = static_cast<double*>(ptr);
  if ((rc = dalloc(R, &ptr, 2 * (size_t)p->imax * sizeof(double)))) return bail(rc);
  d.fl_de = static_cast<double*>(ptr);
  d.fl_pr = d.fl_de + p->imax;
  if ((rc = dalloc(R, &ptr, sizeof(Scal)))) return bail(rc);
  d.scal = static_cast<Scal*>(ptr);
  if ((rc = dalloc(R, &ptr, C_NCOUNTERS * sizeof(unsigned long long)))) return bail(rc);
  d.cnt = static_cast<unsigned long long*>(ptr);
  if ((rc = dalloc(R, &ptr, kCarryCap * sizeof(int)))) return bail(rc);
  d.carry_list = static_cast<int*>(ptr);
  if (cudaMemsetAsync(d.cnt, 0, C_NCOUNTERS * sizeof(unsigned long long), s) != cudaSuccess) return bail(RG_ECUDA);
  for (int k = 0; k < 3; ++k) {
    if (cudaMemsetAsync(R->b.P[k], 0, 9 * N * sizeof(double), s) != cudaSuccess) return bail(RG_ECUDA);
    if (cudaMemsetAsync(R->b.F[k], 0, 9 * N * sizeof(double), s) != cudaSuccess) return bail(RG_ECUDA);
  }
  if (cudaMemsetAsync(R->b.CT, 0, 6 * N * sizeof(double), s) != cudaSuccess) return bail(RG_ECUDA);
  const HostGeom& G = R->geom;
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
  free_run(R);
  ctx->runs.erase(run);
  return RG_OK;
}

int rg_run_ic_torus(rg_ctx* ctx, int run, uint64_t seed, double amp, double rin, double rmax, double beta,
                    double kappa) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  std::vector<double> P;
  torus_ic(R->p, R->geom, seed, amp, rin, rmax, beta, kappa, P);
  R->cur = 0;
  RG_CUDA(cudaMemcpyAsync(R->b.P[0], P.data(), P.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  if (R->d.P32) RG_CUDA(launch_to_f32(R->b.P[0], R->d.P32, 9 * R->d.N, ctx->stream));
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
  int rc = to_soa(ctx, R, uri, R->b.P[0]);
  if (rc) return rc;
  if (R->d.P32) RG_CUDA(launch_to_f32(R->b.P[0], R->d.P32, 9 * R->d.N, ctx->stream));
  return set_time(ctx, R, t0);
}

int rg_run_download_prims(rg_ctx* ctx, int run, double* uri) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  if (!uri) return fail(RG_EINVAL_CONFIG, "null array");
  return from_soa(ctx, R, R->b.P[R->cur], uri);
}

int rg_step(rg_ctx* ctx, int run, int nsteps, rg_step_stats* stats) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  cudaStream_t s = ctx->stream;
  for (int n = 0; n < nsteps; ++n) {
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
  }
  if (ctx->prof) {
    int rc = drain_events(ctx);
    if (rc) return rc;
  }
  if (stats) return read_stats(ctx, R, stats);
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
  int rc = to_soa(ctx, R, uri, R->b.stage);
  if (rc) return rc;
  RG_CUDA(launch_p2c(fp64_view(R), R->b.stage, R->b.stage2, ctx->stream));
  return from_soa(ctx, R, R->b.stage2, uu);
}

int rg_calflx(rg_ctx* ctx, int run, const double* uri, double* ww) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  const DevRun d = fp64_view(R);
  const size_t N = d.N;
  int rc = to_soa(ctx, R, uri, R->b.stage);
  if (rc) return rc;
  Scal sc{};
  sc.active = 1;
  RG_CUDA(cudaMemcpyAsync(d.scal, &sc, sizeof(Scal), cudaMemcpyHostToDevice, ctx->stream));
  for (int dir = 1; dir <= 3; ++dir) RG_CUDA(launch_flux(d, dir, R->b.stage, R->b.F[dir - 1], ctx->stream));
  RG_CUDA(launch_ct(d, R->b.F[0], R->b.F[1], R->b.F[2], R->b.CT, ctx->stream));
  std::vector<double> F(27 * N), CT(6 * N);
  for (int dir = 0; dir < 3; ++dir)
    RG_CUDA(cudaMemcpyAsync(F.data() + (size_t)dir * 9 * N, R->b.F[dir], 9 * N * sizeof(double),
                            cudaMemcpyDeviceToHost, ctx->stream));
  RG_CUDA(cudaMemcpyAsync(CT.data(), R->b.CT, 6 * N * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  RG_CUDA(cudaStreamSynchronize(ctx->stream));
  const int nm1 = d.nm1;
  for (int k = 1; k <= d.kmax; ++k)
    for (int j = 1; j <= d.jmax; ++j)
      for (int i = 1; i <= d.imax; ++i) {
        const size_t c = d.cell(i, j, k);
        const bool in_ct = i >= nm1 && i <= d.imax - nm1 && j >= nm1 && j <= d.jmax - nm1 && k >= nm1 && k <= d.kmax - nm1;
        for (int v = 0; v < 9; ++v)
          for (int dir = 0; dir < 3; ++dir) {
            double w = F[(size_t)dir * 9 * N + (size_t)v * N + c];
            if (in_ct) {
              if (dir == 1 && v == 6) w = CT[0 * N + c];
              if (dir == 2 && v == 6) w = CT[1 * N + c];
              if (dir == 0 && v == 7) w = CT[2 * N + c];
              if (dir == 2 && v == 7) w = CT[3 * N + c];
              if (dir == 0 && v == 8) w = CT[4 * N + c];
              if (dir == 1 && v == 8) w = CT[5 * N + c];
            }
            ww[dir + 3 * (v + 9 * c)] = w;
          }
      }
  return RG_OK;
}

int rg_recov(rg_ctx* ctx, int run, const double* uu, double* uri) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  int rc = to_soa(ctx, R, uu, R->b.stage);
  if (rc) return rc;
  if ((rc = to_soa(ctx, R, uri, R->b.stage2))) return rc;
  RG_CUDA(launch_recov_only(fp64_view(R), R->b.stage, R->b.stage2, R->b.F[0], ctx->stream));
  return from_soa(ctx, R, R->b.F[0], uri);
}

int rg_cdtcfl(rg_ctx* ctx, int run, const double* uri, double* dtcfl) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  int rc = to_soa(ctx, R, uri, R->b.stage);
  if (rc) return rc;
  Scal sc{};
  sc.active = 1;
  const double one = 1.0;
  std::memcpy(&sc.dtcfl_bits, &one, sizeof(double));
  RG_CUDA(cudaMemcpyAsync(R->d.scal, &sc, sizeof(Scal), cudaMemcpyHostToDevice, ctx->stream));
  RG_CUDA(launch_cfl(fp64_view(R), R->b.stage, ctx->stream));
  RG_CUDA(cudaMemcpyAsync(&sc, R->d.scal, sizeof(Scal), cudaMemcpyDeviceToHost, ctx->stream));
  RG_CUDA(cudaStreamSynchronize(ctx->stream));
  std::memcpy(dtcfl, &sc.dtcfl_bits, sizeof(double));
  return RG_OK;
}

int rg_bnd_floor(rg_ctx* ctx, int run, double* uri, const double* urio) {
  Run* R = find(ctx, run);
  if (!R) return fail(RG_ENOTFOUND, "unknown run");
  int rc = to_soa(ctx, R, uri, R->b.stage);
  if (rc) return rc;
  if ((rc = to_soa(ctx, R, urio, R->b.stage2))) return rc;
  Scal sc{};
  sc.active = 1;
  RG_CUDA(cudaMemcpyAsync(R->d.scal, &sc, sizeof(Scal), cudaMemcpyHostToDevice, ctx->stream));
  const DevRun d = fp64_view(R);
  RG_CUDA(launch_bc(d, R->b.stage, R->b.stage2, ctx->stream));
  RG_CUDA(launch_floor(d, R->b.stage, ctx->stream));
  return from_soa(ctx, R, R->b.stage, uri);
}

}  // extern "C"

// ------------------------------------------------------ allocation-free fluxes
// rg_calflx_static serves callers that cannot call cudaMalloc when they need
// the fluxes: a driver running inside a CUDA stream capture, or a host code
// whose device memory comes only from its own pool or arena.  The caller owns
// the input and output device buffers; the flux-CT intermediate (the six
// averaged induction fluxes) and the kernels' scalar block live in the
// file-scope device arrays below, sized for grids of at most
// kStaticMaxCells cells.  Every GPU that loads this library holds these
// arrays (about 12.6 MB) until the process exits.
namespace {

constexpr size_t kStaticMaxCells = (size_t)1 << 18;
__device__ __align__(256) double g_static_ct[6 * kStaticMaxCells];
__device__ __align__(256) Scal g_static_scal;

constexpr int kMaxDevices = 64;
double* g_static_ct_addr[kMaxDevices] = {};
Scal* g_static_scal_addr[kMaxDevices] = {};

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
  const size_t N = R->d.N;
  if (N > kStaticMaxCells)
    return fail(RG_EINVAL_CONFIG, "rg_calflx_static: grid of " + std::to_string(N) +
                                      " cells exceeds the static scratch maximum of " +
                                      std::to_string(kStaticMaxCells) + " cells");
  if (ctx->device < 0 || ctx->device >= kMaxDevices) return fail(RG_EINVAL_CONFIG, "device index out of range");
  RG_CUDA(cudaSetDevice(ctx->device));
  // Set-up once per device, with that device current: the host-side names of
  // the arrays are not device addresses, so their addresses are looked up here.
  if (!g_static_ct_addr[ctx->device]) {
    void* a = nullptr;
    void* b = nullptr;
    RG_CUDA(cudaGetSymbolAddress(&a, g_static_ct));
    RG_CUDA(cudaGetSymbolAddress(&b, g_static_scal));
    g_static_ct_addr[ctx->device] = static_cast<double*>(a);
    g_static_scal_addr[ctx->device] = static_cast<Scal*>(b);
  }
  double* ct = g_static_ct_addr[ctx->device];
  DevRun d = fp64_view(R);
  d.scal = g_static_scal_addr[ctx->device];  // the run's own time state is not touched
  cudaStream_t s = ctx->stream;
  // The arrays keep the previous call's contents: clear them first.
  RG_CUDA(cudaMemsetAsync(ct, 0, 6 * N * sizeof(double), s));
  k_static_scal_reset<<<1, 1, 0, s>>>(d.scal);
  RG_CUDA(cudaGetLastError());
  for (int dir = 1; dir <= 3; ++dir) RG_CUDA(launch_flux(d, dir, d_prims, d_ww + (size_t)(dir - 1) * 9 * N, s));
  RG_CUDA(launch_ct(d, d_ww, d_ww + 9 * N, d_ww + 18 * N, ct, s));
  const dim3 b(64, 4, 1);
  const int n = d.imax - 2 * d.nm1 + 1, m = d.jmax - 2 * d.nm1 + 1, l = d.kmax - 2 * d.nm1 + 1;
  k_ct_scatter<<<dim3((n + 63) / 64, (m + 3) / 4, l), b, 0, s>>>(d, ct, d_ww);
  RG_CUDA(cudaGetLastError());
  RG_CUDA(cudaStreamSynchronize(s));
  return RG_OK;
}
