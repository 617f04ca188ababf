// rg_batch.cuh -- batched steps of many runs (part of the rg_kernels.cu
// translation unit: it reuses that file's kernel bodies).
//
// A batch advances runs that share the reconstruction scheme, the precision
// mode and the slab class (which directions are stored as one plane) by one
// RK3 step with one launch per kernel kind of the step, whatever the number
// of runs.  Each launch walks a tile table: tile t is block (bx, by, bz) of
// run `run` in that run's own single-run grid, with the run's index range
// [ilo, ihi] for kernels that cover part of the radial range (the FP64 and
// FP32 halves of the mixed path).  The grid is persistent: `grid` blocks
// stride over the tiles.  Each block copies its run's DevRun into shared
// memory and calls the same body as the single-run kernel, so a run gives the
// same result alone and in any batch.  The run's buffer rotation lives on the
// device (Scal::cur), which makes one step's launch sequence valid for every
// step: the host captures it once in a CUDA graph and replays it.

namespace {

// nsub: the tile covers blocks bx .. bx+nsub-1 of the run's grid (the tile
// shape along i is nsub blocks of the cell kernels' width).
struct Tile {
  int run, bx, by, bz;
  int ilo, ihi, aux, nsub;
};

// P^n, the stage input and the stage output of a run (stage 0: CFL, P^n only).
__device__ __forceinline__ void stage_ptrs(const DevRun& r, int stage, double*& Pn, double*& Pc, double*& Pw) {
  const int cur = r.scal->cur;
  Pn = r.P[cur];
  if (stage <= 1) { Pc = Pn; Pw = r.P[(cur + 1) % 3]; }
  else if (stage == 2) { Pc = r.P[(cur + 1) % 3]; Pw = r.P[(cur + 2) % 3]; }
  else { Pc = r.P[(cur + 2) % 3]; Pw = r.P[(cur + 1) % 3]; }
}

template <class Body, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) kb(const DevRun* __restrict__ runs, const Tile* __restrict__ tiles,
                                               int ntiles, Body body) {
  __shared__ DevRun sr;
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nt = blockDim.x * blockDim.y * blockDim.z;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const unsigned* src = reinterpret_cast<const unsigned*>(runs + tl.run);
    unsigned* dst = reinterpret_cast<unsigned*>(&sr);
    for (int w = tid; w < (int)(sizeof(DevRun) / 4); w += nt) dst[w] = src[w];
    __syncthreads();
    for (int u = 0; u < tl.nsub; ++u) {
      Tile su = tl;
      su.bx = tl.bx + u;
      body(sr, su);
      __syncthreads();
    }
  }
}

template <int D, int IREC, typename T, typename S>
struct FluxB {
  int stage;
  __device__ void operator()(const DevRun& r, const Tile& t) const {
    double *Pn, *Pc, *Pw;
    stage_ptrs(r, stage, Pn, Pc, Pw);
    if constexpr (sizeof(S) == 8)
      flux_body<D, IREC, T, S>(r, Pc, r.F[D - 1], r.mixed ? r.F32[D - 1] : nullptr, t.aux, t.ilo, t.ihi,
                               make_uint3(t.bx, t.by, t.bz));
    else
      flux_body<D, IREC, T, S>(r, r.P32, r.F32[D - 1], nullptr, 0, t.ilo, t.ihi, make_uint3(t.bx, t.by, t.bz));
  }
};

template <int ICT, typename T, typename S>
struct CtB {
  __device__ void operator()(const DevRun& r, const Tile& t) const {
    if constexpr (sizeof(S) == 8)
      ct_body<ICT, T, S>(r, r.F[0], r.F[1], r.F[2], r.CT, r.mixed ? r.CT32 : nullptr, t.ilo, t.ihi,
                         make_uint3(t.bx, t.by, t.bz));
    else
      ct_body<ICT, T, S>(r, r.F32[0], r.F32[1], r.F32[2], r.CT32, nullptr, t.ilo, t.ihi,
                         make_uint3(t.bx, t.by, t.bz));
  }
};

template <int STAGE, bool MIX>
struct UpdateB {
  __device__ void operator()(const DevRun& r, const Tile& t) const {
    double *Pn, *Pc, *Pw;
    stage_ptrs(r, STAGE, Pn, Pc, Pw);
    update_body<STAGE, MIX>(r, Pn, Pc, Pw, r.F[0], r.F[1], r.F[2], r.CT, t.ilo, t.ihi, make_uint3(t.bx, t.by, t.bz));
  }
};

template <int STAGE>
struct CarryB {
  __device__ void operator()(const DevRun& r, const Tile&) const {
    double *Pn, *Pc, *Pw;
    stage_ptrs(r, STAGE, Pn, Pc, Pw);
    carry_fix_body<0, STAGE>(r, Pn, Pc, Pw, r.F[0], r.F[1], r.F[2], r.CT, nullptr);
  }
};

template <int STAGE>
struct StragB {
  __device__ void operator()(const DevRun& r, const Tile& t) const {
    double *Pn, *Pc, *Pw;
    stage_ptrs(r, STAGE, Pn, Pc, Pw);
    straggler_body<STAGE>(r, Pn, Pc, Pw, r.F[0], r.F[1], r.F[2], r.CT, make_uint3(t.bx, 0, 0));
  }
};

template <int D, bool PERIODIC>
struct BcB {
  int stage;
  __device__ void operator()(const DevRun& r, const Tile& t) const {
    double *Pn, *Pc, *Pw;
    stage_ptrs(r, stage, Pn, Pc, Pw);
    if (PERIODIC) bc_periodic_body<D>(r, Pw, make_uint3(t.bx, t.by, t.bz));
    else bc_phys_body<D>(r, Pw, Pn, make_uint3(t.bx, t.by, t.bz));
  }
};

struct FloorB {
  int stage;
  __device__ void operator()(const DevRun& r, const Tile& t) const {
    double *Pn, *Pc, *Pw;
    stage_ptrs(r, stage, Pn, Pc, Pw);
    floor_body(r, Pw, make_uint3(t.bx, t.by, t.bz));
  }
};

struct CflB {
  __device__ void operator()(const DevRun& r, const Tile& t) const {
    double *Pn, *Pc, *Pw;
    stage_ptrs(r, 0, Pn, Pc, Pw);
    cfl_body(r, Pn, make_uint3(t.bx, t.by, t.bz));
  }
};

// kind 0 step_begin, 1 dt, 2 step_end
template <int KIND>
struct ScalarB {
  __device__ void operator()(const DevRun& r, const Tile&) const {
    if (threadIdx.x != 0) return;
    if (KIND == 0) step_begin_body(r);
    else if (KIND == 1) dt_body(r);
    else step_end_body(r);
  }
};

}  // namespace

// ------------------------------------------------------------- host side
// One launch of a batched step: the kernel to run and its tile range.
enum BKind {
  BK_BEGIN, BK_CFL, BK_DT, BK_FLUX, BK_CT, BK_UPDATE, BK_CARRY, BK_BCPER, BK_BCPHYS, BK_FLOOR, BK_END, BK_STRAG
};
struct BLaunch {
  int kind;
  int stage, dir;   // stage 1..3; direction 1..3 (flux, boundaries)
  int fp32;         // FP32 half of a mixed run (flux, CT) / mixed update
  dim3 block;
  int tile0, ntiles;
  int grid;         // persistent blocks (autotuned)
};

struct BatchPlan {
  int nruns = 0;
  int irec = 6;
  int ict = 1;
  int width = 128;            // threads per block of the cell kernels
  int group = 1;              // blocks along i per tile of the cell kernels
  DevRun* d_runs = nullptr;
  Tile* d_tiles = nullptr;
  std::vector<BLaunch> launches;
  int sm_count = 148;
};

namespace {

inline void add_tiles(std::vector<Tile>& T, int run, dim3 g, int ilo, int ihi, int aux, int group = 1) {
  for (unsigned z = 0; z < g.z; ++z)
    for (unsigned y = 0; y < g.y; ++y)
      for (unsigned x = 0; x < g.x; x += (unsigned)group)
        T.push_back(Tile{run, (int)x, (int)y, (int)z, ilo, ihi, aux, (int)std::min<unsigned>(group, g.x - x)});
}

// Block shape of a cell kernel in a batch of slab runs: `width` threads along i.
inline dim3 wblock(const DevRun& r, dim3 b, int width) {
  dim3 o = sblock(r, b);
  if (o.y == 1 && o.z == 1) o.x = (unsigned)width;
  return o;
}

void plan_append(BatchPlan& B, std::vector<Tile>& T, BLaunch L, const std::vector<DevRun>& runs,
                 const std::function<void(int, const DevRun&, std::vector<Tile>&)>& gen) {
  L.tile0 = (int)T.size();
  for (int a = 0; a < (int)runs.size(); ++a) gen(a, runs[a], T);
  L.ntiles = (int)T.size() - L.tile0;
  L.grid = L.ntiles;
  if (L.ntiles > 0) B.launches.push_back(L);
}

}  // namespace

// Tile tables of one batched step for runs of one class (same irec,
// precision, slab class); `width` is the block width of the cell kernels
// along i (64 or 128: the batched kernels are compiled for at most 128, the
// CT kernel for 2 * 128) and `group` the blocks along i of one tile, so a
// tile of a cell kernel covers width * group cells along i.
int batch_build(const std::vector<DevRun>& runs, int width, int group, BatchPlan** out) {
  if (width != 64 && width != 128) return 1;
  if (group < 1) group = 1;
  BatchPlan* B = new BatchPlan();
  B->nruns = (int)runs.size();
  B->irec = runs.empty() ? 6 : runs[0].irec;
  B->ict = runs.empty() ? 1 : runs[0].ict;
  B->width = width;
  B->group = group;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&B->sm_count, cudaDevAttrMultiProcessorCount, dev);
  std::vector<Tile> T;
  const DevRun& r0 = runs[0];
  const bool mixed = r0.mixed != 0;
  auto one = [](int a, const DevRun&, std::vector<Tile>& t) { add_tiles(t, a, dim3(1, 1, 1), 0, 0, 0); };
  BLaunch L{};
  L.block = dim3(32, 1, 1);
  L.kind = BK_BEGIN;
  plan_append(*B, T, L, runs, one);
  L.kind = BK_CFL;
  L.block = wblock(r0, dim3(64, 2, 1), width);
  plan_append(*B, T, L, runs, [&](int a, const DevRun& r, std::vector<Tile>& t) {
    add_tiles(t, a, sgrid(r, r.imax - 2, r.jmax - 2, r.kmax - 2, L.block), 0, 0, 0, group);
  });
  L.kind = BK_DT;
  L.block = dim3(32, 1, 1);
  plan_append(*B, T, L, runs, one);
  for (int stage = 1; stage <= 3; ++stage) {
    L.stage = stage;
    for (int dir = 1; dir <= 3; ++dir) {
      L.kind = BK_FLUX;
      L.dir = dir;
      L.block = wblock(r0, dim3(64, 2, 1), width);
      for (int part = 0; part < 2; ++part) {
        L.fp32 = part;
        plan_append(*B, T, L, runs, [&](int a, const DevRun& r, std::vector<Tile>& t) {
          const int lo = r.nm0, hi = r.imax - r.nm0, m = r.jmax - 2 * r.nm0 + 1, l = r.kmax - 2 * r.nm0 + 1;
          int ilo = lo, ihi = hi, aux = 0;
          if (!r.mixed) {
            if (part == 1) return;
          } else {
            const int split = fp64_split(r, lo, hi);
            if (part == 0) {
              if (split < lo) return;
              ihi = split < hi ? split + 1 : hi;
              aux = split;
            } else {
              if (split >= hi) return;
              ilo = split + 1;
            }
          }
          add_tiles(t, a, sgrid(r, 2 * (ihi - ilo + 1), m, l, L.block), ilo, ihi, aux, group);
        });
      }
    }
    L.kind = BK_CT;
    L.dir = 0;
    L.block = wblock(r0, dim3(64, 4, 1), 2 * width);
    for (int part = 0; part < 2; ++part) {
      L.fp32 = part;
      plan_append(*B, T, L, runs, [&](int a, const DevRun& r, std::vector<Tile>& t) {
        const int lo = r.nm1, hi = r.imax - r.nm1, m = r.jmax - 2 * r.nm1 + 1, l = r.kmax - 2 * r.nm1 + 1;
        int ilo = lo, ihi = hi;
        if (!r.mixed) {
          if (part == 1) return;
        } else {
          const int split = fp64_split(r, lo, hi);
          if (part == 0) { if (split < lo) return; ihi = split; }
          else { if (split >= hi) return; ilo = split + 1; }
        }
        add_tiles(t, a, sgrid(r, ihi - ilo + 1, m, l, L.block), ilo, ihi, 0, group);
      });
    }
    L.kind = BK_UPDATE;
    L.block = wblock(r0, dim3(64, 2, 1), width);
    for (int part = 0; part < 2; ++part) {
      L.fp32 = part;
      plan_append(*B, T, L, runs, [&](int a, const DevRun& r, std::vector<Tile>& t) {
        int ilo = 1, ihi = r.imax;
        if (!r.mixed) {
          if (part == 1) return;
        } else {
          const int split = fp64_split(r, 1, r.imax);
          if (part == 0) { if (split < 1) return; ihi = split; }
          else { if (split >= r.imax) return; ilo = split + 1; }
        }
        add_tiles(t, a, sgrid(r, ihi - ilo + 1, r.jmax, r.kmax, L.block), ilo, ihi, 0, group);
      });
    }
    L.fp32 = 0;
    L.kind = BK_STRAG;
    L.block = dim3(128, 1, 1);
    plan_append(*B, T, L, runs, [&](int a, const DevRun& r, std::vector<Tile>& t) {
      if (r.strag_list) add_tiles(t, a, dim3((unsigned)((r.strag_cap + 127) / 128), 1, 1), 0, 0, 0);
    });
    L.kind = BK_CARRY;
    L.block = dim3(128, 1, 1);
    plan_append(*B, T, L, runs, one);
    for (int per = 1; per >= 0; --per)
      for (int dir = 1; dir <= 3; ++dir) {
        L.kind = per ? BK_BCPER : BK_BCPHYS;
        L.dir = dir;
        dim3 g, b;
        const bool jf = r0.jfix != 0, kf = r0.kfix != 0;
        const bool slab = (dir == 2 && jf) || (dir == 3 && kf);
        if (slab) continue;
        const bool fix1 = (dir == 1) ? jf : false, fix2 = (dir == 3) ? jf : kf;
        bc_shape(8, 8, fix1, fix2, g, b);
        L.block = b;
        plan_append(*B, T, L, runs, [&](int a, const DevRun& r, std::vector<Tile>& t) {
          if (!any_code(r, 2 * (dir - 1), per != 0)) return;
          const int nm1 = r.nm1;
          int n1, n2;
          if (dir == 1) { n1 = r.jmax; n2 = r.kmax; }
          else if (dir == 2) { n1 = r.imax; n2 = r.kmax; }
          else { n1 = r.imax; n2 = r.jmax; }
          if (per) { n1 -= 2 * nm1; n2 -= 2 * nm1; }
          dim3 gg, bb;
          bc_shape(n1, n2, fix1, fix2, gg, bb);
          add_tiles(t, a, gg, 0, 0, 0);
        });
      }
    L.kind = BK_FLOOR;
    L.dir = 0;
    L.block = wblock(r0, dim3(64, 2, 1), width);
    plan_append(*B, T, L, runs, [&](int a, const DevRun& r, std::vector<Tile>& t) {
      add_tiles(t, a, sgrid(r, r.imax, r.jmax, r.kmax, L.block), 0, 0, 0, group);
    });
  }
  L = BLaunch{};
  L.kind = BK_END;
  L.block = dim3(32, 1, 1);
  plan_append(*B, T, L, runs, one);
  (void)mixed;
  if (cudaMalloc(&B->d_runs, runs.size() * sizeof(DevRun)) != cudaSuccess ||
      cudaMalloc(&B->d_tiles, T.size() * sizeof(Tile)) != cudaSuccess) {
    cudaFree(B->d_runs);
    delete B;
    return 1;
  }
  if (cudaMemcpy(B->d_runs, runs.data(), runs.size() * sizeof(DevRun), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(B->d_tiles, T.data(), T.size() * sizeof(Tile), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(B->d_runs);
    cudaFree(B->d_tiles);
    delete B;
    return 1;
  }
  *out = B;
  return 0;
}

void batch_destroy(BatchPlan* B) {
  if (!B) return;
  cudaFree(B->d_runs);
  cudaFree(B->d_tiles);
  delete B;
}

int batch_launch_count(const BatchPlan* B) { return (int)B->launches.size(); }
int batch_launch_kind(const BatchPlan* B, int idx, int* dir) {
  if (dir) *dir = B->launches[idx].dir;
  return B->launches[idx].kind;
}

// Persistent grid sizes: every launch gets min(tiles, factor * SMs) blocks
// (factor 0: one block per tile).
void batch_set_grid(BatchPlan* B, int factor) {
  for (BLaunch& L : B->launches) L.grid = factor <= 0 ? L.ntiles : std::min(L.ntiles, factor * B->sm_count);
}

namespace {

template <class Body, int NT, int MINB>
cudaError_t kb_go(const BatchPlan* B, const BLaunch& L, Body body, cudaStream_t s) {
  kb<Body, NT, MINB><<<L.grid, L.block, 0, s>>>(B->d_runs, B->d_tiles + L.tile0, L.ntiles, body);
  return cudaGetLastError();
}

// Cell kernels run 128-thread blocks (the CT kernel 256) whatever the batch,
// so a run's cells go through the same compiled code alone and in any mix;
// MINB keeps each kernel's register budget of the single-run launch (FP64
// faces 96, FP32 faces 64, update 168 registers).
template <int D, int IREC, typename T, typename S>
cudaError_t go_flux(const BatchPlan* B, const BLaunch& L, cudaStream_t s) {
  const FluxB<D, IREC, T, S> b{L.stage};
  return kb_go<FluxB<D, IREC, T, S>, 128, sizeof(T) == 8 ? RG_FLUX_MINB64 : 8>(B, L, b, s);
}

template <int D, typename T, typename S>
cudaError_t go_flux_irec(const BatchPlan* B, const BLaunch& L, cudaStream_t s) {
  switch (B->irec) {
    case 1: return go_flux<D, 1, T, S>(B, L, s);
    case 2: return go_flux<D, 2, T, S>(B, L, s);
    case 3: return go_flux<D, 3, T, S>(B, L, s);
    case 4: return go_flux<D, 4, T, S>(B, L, s);
    case 8: return go_flux<D, 8, T, S>(B, L, s);
    case 10: return go_flux<D, 10, T, S>(B, L, s);
    case 11: return go_flux<D, 11, T, S>(B, L, s);
    case 12: return go_flux<D, 12, T, S>(B, L, s);
    case 13: return go_flux<D, 13, T, S>(B, L, s);
    case 5: return go_flux<D, 5, T, S>(B, L, s);
    case 6: return go_flux<D, 6, T, S>(B, L, s);
    case 7: return go_flux<D, 7, T, S>(B, L, s);
    default: return go_flux<D, 9, T, S>(B, L, s);
  }
}

template <typename T, typename S>
cudaError_t go_flux_dir(const BatchPlan* B, const BLaunch& L, cudaStream_t s) {
  if (L.dir == 1) return go_flux_irec<1, T, S>(B, L, s);
  if (L.dir == 2) return go_flux_irec<2, T, S>(B, L, s);
  return go_flux_irec<3, T, S>(B, L, s);
}

template <int STAGE, bool MIX>
cudaError_t go_update(const BatchPlan* B, const BLaunch& L, cudaStream_t s) {
  return kb_go<UpdateB<STAGE, MIX>, 128, RG_UPDATE_MINB>(B, L, UpdateB<STAGE, MIX>{}, s);
}

template <int D>
cudaError_t go_bc(const BatchPlan* B, const BLaunch& L, cudaStream_t s) {
  if (L.kind == BK_BCPER) return kb_go<BcB<D, true>, 128, 1>(B, L, BcB<D, true>{L.stage}, s);
  return kb_go<BcB<D, false>, 128, 1>(B, L, BcB<D, false>{L.stage}, s);
}

template <class Body>
cudaError_t go_cell(const BatchPlan* B, const BLaunch& L, Body b, cudaStream_t s) {
  if (L.block.x * L.block.y * L.block.z == 256) return kb_go<Body, 256, 1>(B, L, b, s);
  return kb_go<Body, 128, 1>(B, L, b, s);
}

}  // namespace

cudaError_t batch_issue(const BatchPlan* B, int idx, cudaStream_t s) {
  const BLaunch& L = B->launches[idx];
  switch (L.kind) {
    case BK_BEGIN: return kb_go<ScalarB<0>, 32, 1>(B, L, ScalarB<0>{}, s);
    case BK_DT: return kb_go<ScalarB<1>, 32, 1>(B, L, ScalarB<1>{}, s);
    case BK_END: return kb_go<ScalarB<2>, 32, 1>(B, L, ScalarB<2>{}, s);
    case BK_CFL: return go_cell(B, L, CflB{}, s);
    case BK_FLUX:
      return L.fp32 ? go_flux_dir<float, float>(B, L, s) : go_flux_dir<double, double>(B, L, s);
    case BK_CT:
      if (B->ict == 0)
        return L.fp32 ? go_cell(B, L, CtB<0, float, float>{}, s) : go_cell(B, L, CtB<0, double, double>{}, s);
      if (B->ict == 2)
        return L.fp32 ? go_cell(B, L, CtB<2, float, float>{}, s) : go_cell(B, L, CtB<2, double, double>{}, s);
      return L.fp32 ? go_cell(B, L, CtB<1, float, float>{}, s) : go_cell(B, L, CtB<1, double, double>{}, s);
    case BK_UPDATE:
      if (L.stage == 1) return L.fp32 ? go_update<1, true>(B, L, s) : go_update<1, false>(B, L, s);
      if (L.stage == 2) return L.fp32 ? go_update<2, true>(B, L, s) : go_update<2, false>(B, L, s);
      return L.fp32 ? go_update<3, true>(B, L, s) : go_update<3, false>(B, L, s);
    case BK_STRAG:
      if (L.stage == 1) return kb_go<StragB<1>, 128, 1>(B, L, StragB<1>{}, s);
      if (L.stage == 2) return kb_go<StragB<2>, 128, 1>(B, L, StragB<2>{}, s);
      return kb_go<StragB<3>, 128, 1>(B, L, StragB<3>{}, s);
    case BK_CARRY:
      if (L.stage == 1) return kb_go<CarryB<1>, 128, 1>(B, L, CarryB<1>{}, s);
      if (L.stage == 2) return kb_go<CarryB<2>, 128, 1>(B, L, CarryB<2>{}, s);
      return kb_go<CarryB<3>, 128, 1>(B, L, CarryB<3>{}, s);
    case BK_BCPER:
    case BK_BCPHYS:
      if (L.dir == 1) return go_bc<1>(B, L, s);
      if (L.dir == 2) return go_bc<2>(B, L, s);
      return go_bc<3>(B, L, s);
    case BK_FLOOR: return go_cell(B, L, FloorB{L.stage}, s);
    default: return cudaErrorInvalidValue;
  }
}

// One full RK3 step of every run of the batch.
cudaError_t batch_step(const BatchPlan* B, cudaStream_t s) {
  for (int a = 0; a < (int)B->launches.size(); ++a) {
    const cudaError_t e = batch_issue(B, a, s);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}
