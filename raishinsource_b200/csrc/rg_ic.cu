// rg_ic.cu -- Fishbone-Moncrief torus initial data computed on the device:
// the construction of mdtorus1 (mdgrmhd.f90:879-1654) that torus_ic in
// rg_geometry.cpp also states, in four passes over the run's stored cells.
//
//   pass 0  ln h, rho and the maximum of rho over the torus (mdgrmhd.f90:1027-1197)
//   pass 1  every primitive: floor atmosphere outside the torus; inside it rho
//           and p normalised by that maximum, p perturbed by the seeded draw,
//           BL -> (M)KS velocity, floors (mdgrmhd.f90:964-1021, 1198-1320)
//   pass 2  B^r, B^theta from the corner vector potential A_phi ~ max(<rho> -
//           0.2, 0) (mdgrmhd.f90:1335-1423), and the minimum plasma beta
//           (mdgrmhd.f90:1424-1540)
//   pass 3  B scaled to the target minimum beta
//
// Pass 1 recomputes the torus state of pass 0 instead of storing it, and
// pass 2 evaluates A_phi at the four corners of a cell from rho, so the
// construction needs no scratch array beyond two reduction words.  The
// host-side copies of the corner and edge loops reduce to: A_phi at corner
// (i, k) is the corner value at (max(i, 2), max(k, 2)), and the field of cell
// (i, k) is the field computed at (clamp(i, 2, imax-1), clamp(k, 2, kmax-1)).
//
// Every per-index transcendental (floors, sines, cosines, spacings) and the
// run's scalars come from the host table (TorusTables), evaluated there with
// the calls torus_ic makes; the per-cell exp, log and pow are CUDA's, so the
// result agrees with the host construction to a few units in the last place.
#include <cstdint>

#include "rg_kernels.cuh"

namespace rg {

namespace {

constexpr int kIcThreads = 256;

// splitmix64 finaliser keyed by (seed, cell): the draw of uniform01 in rg_geometry.cpp.
__device__ double ic_uniform01(uint64_t seed, uint64_t idx) {
  uint64_t z = seed * 0x9E3779B97F4A7C15ULL + idx + 0x632BE59BD9B4E019ULL;
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z = z ^ (z >> 31);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

// Order-preserving map of a double onto unsigned integers (for atomicMin).
__device__ __forceinline__ unsigned long long ordered_key(double x) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(x);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ULL);
}
__device__ __forceinline__ double from_ordered_key(unsigned long long k) {
  return __longlong_as_double((long long)((k >> 63) ? (k & 0x7FFFFFFFFFFFFFFFULL) : ~k));
}

struct IcView {
  DevRun d;
  IcTorusArgs a;
  __device__ double ti(int f, int i) const { return a.tab[(size_t)f * d.imax + (i - 1)]; }
  __device__ double tk(int f, int k) const { return a.tab[(size_t)kIcTabI * d.imax + (size_t)f * d.kmax + (k - 1)]; }
  __device__ double met(int c, int i, int k) const { return d.mc[(size_t)c * d.nik + d.ik(i, k)]; }
  // (i, j, k) of stored cell c (a phi slab stores the plane j = jfix)
  __device__ void decode(size_t c, int& i, int& j, int& k) const {
    i = (int)(c % (size_t)d.imax) + 1;
    const size_t t = c / (size_t)d.imax;
    if (d.jfix) {
      j = d.jfix;
      k = (int)t + 1;
    } else {
      j = (int)(t % (size_t)d.jmax) + 1;
      k = (int)(t / (size_t)d.jmax) + 1;
    }
  }
};

// Covariant metric at the cell centre (i, k) from the cache (gcov block + g_thth).
__device__ void cached_gcov(const IcView& v, int i, int k, double g[4][4]) {
  g[0][0] = v.met(0, i, k); g[0][1] = v.met(1, i, k); g[0][2] = v.met(2, i, k);
  g[1][1] = v.met(3, i, k); g[1][2] = v.met(4, i, k); g[2][2] = v.met(5, i, k);
  g[3][3] = v.met(6, i, k);
  g[1][0] = g[0][1]; g[2][0] = g[0][2]; g[2][1] = g[1][2];
  g[0][3] = g[1][3] = g[2][3] = g[3][0] = g[3][1] = g[3][2] = 0.0;
}

// Row 0 of the inverse by invert_matrix's column-pivoted LU (coord.f90:1324-1501),
// the inverse lu_inverse_cols in rg_geometry.cpp computes; row 0 of
// the result is the first solve.  Leaves out untouched for a pivot below 1e-10.
__device__ void lu_inverse_cols_row0(const double in[4][4], double out[4]) {
  double A[5][5];
  int p[5];
  for (int i = 1; i <= 4; ++i) p[i] = i;
  for (int c = 1; c <= 4; ++c)
    for (int r = 1; r <= 4; ++r) A[r][c] = in[r - 1][c - 1];
  for (int t = 1; t <= 4; ++t) {
    int mj = t;
    for (int c = t + 1; c <= 4; ++c)
      if (fabs(A[t][c]) > fabs(A[t][mj])) mj = c;
    if (mj != t) {
      for (int r = 1; r <= 4; ++r) { const double x = A[r][mj]; A[r][mj] = A[r][t]; A[r][t] = x; }
      const int x = p[mj]; p[mj] = p[t]; p[t] = x;
    }
    if (fabs(A[t][t]) < 1e-10) return;
    for (int c = t + 1; c <= 4; ++c) {
      A[t][c] = A[t][c] / A[t][t];
      for (int r = t + 1; r <= 4; ++r) A[r][c] = A[r][c] - A[t][c] * A[r][t];
    }
  }
  double b[5] = {0, 1.0, 0, 0, 0};
  for (int c = 1; c <= 4; ++c)
    if (c != p[c] && c < p[c]) { const double x = b[c]; b[c] = b[p[c]]; b[p[c]] = x; }
  for (int c = 1; c <= 4; ++c) {
    double s = b[c];
    for (int r = 1; r < c; ++r) s = s - A[r][c] * b[r];
    b[c] = s;
  }
  for (int c = 4; c >= 1; --c) {
    double s = b[c];
    for (int r = 4; r > c; --r) s = s - A[r][c] * b[r];
    b[c] = s / A[c][c];
  }
  for (int c = 1; c <= 4; ++c) out[c - 1] = b[c];
}

// transbl2ks (physfunc.f90:366-505): BL 4-velocity util -> (M)KS u-tilde at (i, k).
__device__ void ic_bl_to_ks(const IcView& v, int i, int k, double r, const double util[4], double out[4]) {
  const double akm = v.a.akm;
  const double rbh1 = 1. + sqrt(1. - akm * akm);
  double gc0[4] = {0.0, 0.0, 0.0, 0.0};  // row 0 of the contravariant metric
  auto con = [&]() {
    if (v.a.metric == 303) {
      gc0[0] = v.met(7, i, k); gc0[1] = v.met(8, i, k); gc0[2] = v.met(9, i, k); gc0[3] = 0.0;
    } else {
      double g[4][4];
      cached_gcov(v, i, k, g);
      lu_inverse_cols_row0(g, gc0);
    }
  };
  if (r > rbh1) {
    // bl_cov (coord.f90:378-463)
    const double sth = v.tk(IC_SBL, k), cth = v.tk(IC_CBL, k);
    const double s2 = sth * sth;
    const double a2 = akm * akm, r2 = r * r;
    const double bdel = 1. - (2. / r) + (a2 * (1. / r2));
    const double bsig = 1. + a2 * cth * cth * (1. / r2);
    double g[4][4] = {};
    g[0][0] = -(1. - 2. * (1. / (r * bsig)));
    g[0][2] = -(2. * akm * s2 * (1. / (r * bsig)));
    g[1][1] = bsig / bdel;
    g[2][0] = g[0][2];
    g[2][2] = r2 * s2 * (1. + (a2 * (1. / r2)) + 2. * a2 * s2 * (1. / (r2 * r * bsig)));
    g[3][3] = r2 * bsig;
    double u[4] = {0.0, util[1], util[2], util[3]};
    const double aa = g[0][0];
    const double bb = 2. * (g[0][1] * u[1] + g[0][2] * u[2] + g[0][3] * u[3]);
    const double cc = 1. + g[1][1] * u[1] * u[1] + g[2][2] * u[2] * u[2] + g[3][3] * u[3] * u[3] +
                      2. * (g[1][2] * u[1] * u[2] + g[1][3] * u[1] * u[3] + g[2][3] * u[2] * u[3]);
    const double disc = bb * bb - 4. * aa * cc;
    u[0] = (-bb - sqrt(disc)) * (1. / (2. * aa));
    double tr[4][4] = {};
    const double del = r * r - (2. * r) + akm * akm;
    if (del > 0.0) {
      tr[0][0] = 1.0; tr[0][1] = 2. * r * (1. / del); tr[1][1] = 1.0;
      tr[2][2] = 1.0; tr[2][1] = akm * (1. / del); tr[3][3] = 1.0;
    }
    double w[4] = {0, 0, 0, 0};
    for (int n = 0; n < 4; ++n)
      for (int m = 0; m < 4; ++m) w[m] = w[m] + tr[m][n] * u[n];
    if (v.a.metric == 403) {
      if (v.a.ix1 == 2) w[1] = w[1] * (1. / (r));
      if (v.a.ix3 == 2) w[3] = w[3] * (1. / v.tk(IC_HDEN, k));
    }
    con();
    const double alpha = 1. / sqrt(-gc0[0]);
    const double gfl = w[0] * alpha;
    for (int m = 1; m <= 3; ++m) out[m] = w[m] + gfl * (alpha * alpha * gc0[m]) * (1. / alpha);
  } else {
    con();
    const double alpha = 1. / sqrt(-gc0[0]);
    for (int m = 1; m <= 3; ++m) out[m] = alpha * alpha * gc0[m] * (1. / alpha);
  }
}

// Unnormalised torus state at (i, k) (mdgrmhd.f90:1027-1197); false outside the torus.
__device__ bool torus_point(const IcView& v, int i, int k, double& de, double& pr, double util[4]) {
  const IcTorusArgs& a = v.a;
  const double r = v.ti(IC_R, i), th = v.tk(IC_TH, k);
  if (!(r >= a.rin && th >= a.edge0 && th <= a.edge1)) return false;
  const double sth = v.tk(IC_STH, k), cth = v.tk(IC_CTH, k);
  const double am = a.akm, ell = a.ell, gam = v.d.gam;
  const double del = (r * r) - (2.0 * r) + (am * am);
  const double aa = (r * r + am * am) * (r * r + am * am) - del * am * am * sth * sth;
  const double sig = r * r + am * am * cth * cth;
  const double t1a = 4.0 * (ell * ell * sig * sig) * del * (1.0 / (aa * sth * aa * sth));
  const double t1c = sig * del * (1.0 / aa);
  const double t1d = 0.5 * log((1.0 + sqrt(1. + t1a)) * (1.0 / t1c));
  const double t1e = 0.5 * sqrt(1.0 + t1a);
  const double t1f = 2.0 * am * r * ell * (1.0 / aa);
  double lh = t1d - t1e - t1f - a.h_in;
  if (lh <= 0.0) lh = 0.0;
  const double hm1 = exp(lh) - 1.0;
  if (!(hm1 > 0.0)) return false;
  de = pow(hm1 * (gam - 1.0) / (a.kappa * gam), 1.0 / (gam - 1.0));
  pr = a.kappa * pow(de, gam);
  const double e2chi = sig * sig * del * (1.0 / (aa * aa * sth * sth));
  const double uphi = sqrt((-1.0 + sqrt(1.0 + 4.0 * ell * ell * e2chi)) / 2.0);
  const double t3a = 2.0 * am * r * sqrt(1. + uphi * uphi);
  const double t3b = sqrt(aa * sig * del);
  const double t3c = sqrt(sig * (1.0 / aa)) * uphi * (1.0 / sth);
  util[0] = 0.0; util[1] = 0.0; util[2] = t3a * (1.0 / t3b) + t3c; util[3] = 0.0;
  return true;
}

__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long x) {
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long y = __shfl_xor_sync(0xffffffffu, x, o);
    x = y > x ? y : x;
  }
  return x;
}
__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long x) {
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long y = __shfl_xor_sync(0xffffffffu, x, o);
    x = y < x ? y : x;
  }
  return x;
}

__global__ void k_ic_init(unsigned long long* red) {
  red[0] = 0ULL;                   // bits of rho_max (non-negative)
  red[1] = ordered_key(1.e5);      // beta_min starts at 1e5 (mdgrmhd.f90:1424)
}

__global__ void __launch_bounds__(kIcThreads) k_ic_rhomax(IcView v) {
  const size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long key = 0ULL;
  if (c < v.d.N) {
    int i, j, k;
    v.decode(c, i, j, k);
    double de, pr, util[4];
    if (torus_point(v, i, k, de, pr, util) && de > 0.0) key = (unsigned long long)__double_as_longlong(de);
  }
  key = warp_max_u64(key);
  if ((threadIdx.x & 31) == 0 && key) atomicMax(v.a.red, key);
}

__global__ void __launch_bounds__(kIcThreads) k_ic_state(IcView v, double* __restrict__ P) {
  const size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= v.d.N) return;
  int i, j, k;
  v.decode(c, i, j, k);
  const size_t N = v.d.N;
  const double gam = v.d.gam;
  const double rmin1 = v.ti(IC_DE, i), pmin1 = v.ti(IC_PR, i);
  double de = rmin1, pr = pmin1, u[4] = {0.0, 0.0, 0.0, 0.0};
  if (torus_point(v, i, k, de, pr, u)) {
    const int mt = v.a.metric;
    if (mt == 303 || mt == 403) {
      double un[4];
      ic_bl_to_ks(v, i, k, v.ti(IC_R, i), u, un);
      u[1] = un[1]; u[2] = un[2]; u[3] = un[3];
    }
    const double rhomax = __longlong_as_double((long long)v.a.red[0]);
    de = de * (1.0 / rhomax);
    pr = pr * (1.0 / rhomax);
    // a phi slab keys its draw by the (r, theta) cell of the interior phi index
    const size_t key = v.a.phi_slab ? v.d.cell_full(i, v.a.slab_j, k) : v.d.cell_full(i, j, k);
    pr = pr * (1.0 + v.a.amp * (ic_uniform01(v.a.seed, key) - 0.5));
    if (de <= rmin1 || pr <= pmin1) {
      de = rmin1;
      pr = pmin1;
      u[1] = 0.0; u[2] = 0.0; u[3] = 0.0;
    }
  }
  P[0 * N + c] = de;
  P[1 * N + c] = u[1];
  P[2 * N + c] = u[2];
  P[3 * N + c] = u[3];
  P[4 * N + c] = pr;
  P[5 * N + c] = pr * (1.0 / pow(de, gam - 1.0));
  P[6 * N + c] = 0.0;
  P[7 * N + c] = 0.0;
  P[8 * N + c] = 0.0;
}

__global__ void __launch_bounds__(kIcThreads) k_ic_field(IcView v, double* __restrict__ P) {
  const size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long key = ordered_key(1.e5);
  if (c < v.d.N) {
    int i, j, k;
    v.decode(c, i, j, k);
    const DevRun& d = v.d;
    const size_t N = d.N;
    auto rho = [&](int ii, int kk) { return P[d.cell(ii, j, kk)]; };
    auto apot = [&](int ii, int kk) {
      ii = ii < 2 ? 2 : ii;
      kk = kk < 2 ? 2 : kk;
      const double av = 0.25 * (rho(ii, kk) + rho(ii - 1, kk) + rho(ii, kk - 1) + rho(ii - 1, kk - 1));
      const double a1 = (av != 0.0) ? ((av * (1. / 1.0)) - 0.2) : 0.0;
      return a1 > 0.0 ? a1 : 0.0;
    };
    const int ci = i < 2 ? 2 : (i > d.imax - 1 ? d.imax - 1 : i);
    const int ck = k < 2 ? 2 : (k > d.kmax - 1 ? d.kmax - 1 : k);
    const double a11 = apot(ci + 1, ck + 1), a01 = apot(ci, ck + 1), a10 = apot(ci + 1, ck), a00 = apot(ci, ck);
    const double dg = v.met(kMetBase - 1, ci, ck);
    const double c1 = 0.5 * (a11 + a01 - a10 - a00);
    const double c3 = 0.5 * (a11 + a10 - a01 - a00);
    const double B1 = (c1 != 0.0) ? -(c1 * (1.0 / (v.tk(IC_H3, ck) * dg))) : 0.0;
    const double B3 = (c3 != 0.0) ? c3 * (1.0 / (v.ti(IC_H1, ci) * dg)) : 0.0;
    const double B2 = 0.0;
    P[6 * N + c] = B1;
    P[8 * N + c] = B3;
    // plasma beta of this cell (mdgrmhd.f90:1424-1540)
    double g[4][4];
    cached_gcov(v, i, k, g);
    const double gc00 = v.met(7, i, k), gc0[4] = {gc00, v.met(8, i, k), v.met(9, i, k), 0.0};
    const double ut[4] = {0.0, P[1 * N + c], P[2 * N + c], P[3 * N + c]};
    double utsq = 0.0;
    for (int x = 1; x <= 3; ++x)
      for (int y = 1; y <= 3; ++y) utsq = utsq + g[x][y] * ut[x] * ut[y];
    if (utsq < 0.0) utsq = (fabs(utsq) <= 1.0e-10) ? fabs(utsq) : 1.e-10;
    if (fabs(utsq) > 5.e2) utsq = 5.0e2;
    const double gfl = sqrt(1. + utsq);
    const double alpha = 1. / sqrt(-gc00);
    double uc[4], ul[4], bc[4], bl[4];
    uc[0] = gfl * (1. / alpha);
    for (int m = 1; m <= 3; ++m) uc[m] = ut[m] - gfl * (alpha * alpha * gc0[m]) * (1. / alpha);
    for (int x = 0; x < 4; ++x) ul[x] = g[x][0] * uc[0] + g[x][1] * uc[1] + g[x][2] * uc[2] + g[x][3] * uc[3];
    bc[0] = B1 * ul[1] + B2 * ul[2] + B3 * ul[3];
    bc[1] = (B1 + bc[0] * uc[1]) * (1. / uc[0]);
    bc[2] = (B2 + bc[0] * uc[2]) * (1. / uc[0]);
    bc[3] = (B3 + bc[0] * uc[3]) * (1. / uc[0]);
    for (int x = 0; x < 4; ++x) bl[x] = g[x][0] * bc[0] + g[x][1] * bc[1] + g[x][2] * bc[2] + g[x][3] * bc[3];
    const double bsq = bc[0] * bl[0] + bc[1] * bl[1] + bc[2] * bl[2] + bc[3] * bl[3];
    const double pb = (bsq != 0.0) ? 2. * P[4 * N + c] / bsq : 1.e5;
    if (pb < 1.e5) key = ordered_key(pb);
  }
  key = warp_min_u64(key);
  if ((threadIdx.x & 31) == 0) atomicMin(v.a.red + 1, key);
}

__global__ void __launch_bounds__(kIcThreads) k_ic_scale(IcView v, double* __restrict__ P) {
  const size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= v.d.N) return;
  const double beta_min = from_ordered_key(v.a.red[1]);
  const double bnorm = (v.a.beta == 0.0) ? 0.0 : sqrt(beta_min / v.a.beta);
  const size_t N = v.d.N;
  for (int q = 6; q <= 8; ++q) P[q * N + c] = P[q * N + c] * bnorm;
}

}  // namespace

cudaError_t launch_ic_torus(const DevRun& r, const IcTorusArgs& a, double* P, cudaStream_t s) {
  const IcView v{r, a};
  const unsigned blocks = (unsigned)((r.N + kIcThreads - 1) / kIcThreads);
  k_ic_init<<<1, 1, 0, s>>>(a.red);
  k_ic_rhomax<<<blocks, kIcThreads, 0, s>>>(v);
  k_ic_state<<<blocks, kIcThreads, 0, s>>>(v, P);
  k_ic_field<<<blocks, kIcThreads, 0, s>>>(v, P);
  k_ic_scale<<<blocks, kIcThreads, 0, s>>>(v, P);
  return cudaGetLastError();
}

}  // namespace rg
