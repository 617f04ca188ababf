// rg_kernels.cu -- sm_100a kernels of one RK3 stage of the RAISHIN GRMHD
// update (main.f90:807-911) on one GPU.
//
// Per stage:  k_flux<1..3>  reconstruction + face state + LLF flux per face
//             k_ct          flux-CT averaging of the induction fluxes
//             k_update      RK combine + geometric source + primitive recovery
//             k_carry_fix   loop-order W carry of recov1a (only when queued)
//             k_bc_*        ghost fill in the reference's pass order
//             k_floor       infchk + atmosphere1a + pminmax2b (pointwise)
// Per step:   k_step_begin, k_cfl (block min + atomicMin), k_dt, k_step_end.
// All state is FP64 structure-of-arrays; a step never synchronises the host.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <functional>
#include <vector>

#include "rg_device.cuh"
#include "rg_kernels.cuh"

namespace rg {

namespace {

__device__ __forceinline__ void count_event(const DevRun& r, int which, bool flag) {
  const unsigned mask = __activemask();
  const unsigned b = __ballot_sync(mask, flag);
  if (b && (threadIdx.x & 31) == (unsigned)(__ffs(mask) - 1)) atomicAdd(r.cnt + which, (unsigned long long)__popc(b));
}

__device__ __forceinline__ void load9(const double* __restrict__ P, size_t N, size_t c, double q[9]) {
#pragma unroll
  for (int v = 0; v < 9; ++v) q[v] = P[(size_t)v * N + c];
}

// j and k of this thread for a kernel whose j (k) range starts at lo: the
// slab index when the direction is a slab (one stored plane), otherwise from
// the grid's y (z) coordinate.
__device__ __forceinline__ int jidx(const DevRun& r, int lo, uint3 bid) {
  return r.jfix ? r.jfix : (int)(bid.y * blockDim.y + threadIdx.y) + lo;
}
__device__ __forceinline__ int kidx(const DevRun& r, int lo, uint3 bid) {
  return r.kfix ? r.kfix : (int)(bid.z * blockDim.z + threadIdx.z) + lo;
}

// ----------------------------------------------------------------- recov1a
struct RecovOut {
  double wg;
  bool nr2, fail, cap;
  bool deferred;  // the iteration passed `defer` steps unconverged: nothing written, redo without limit
};

constexpr int kRescaleCap = 1000;  // the reference's "go to 95" loop (recov.f90:823-850) is unbounded

// recov.f90:578-1228 for one interior cell.  u: conserved (sqrt(-g) scaled),
// q: previous primitives (initial guess and failure fallback), out: new
// primitives.  Returns false, touching nothing, when the W quadratic has no
// non-negative root and no carried-in W is given: the reference then keeps W
// from the previous cell of its loop (recov.f90:810-815), which the caller
// resolves in loop order.
__device__ bool recov_cell(const double u[9], const double q[9], double out[9], const Met& m, double gam, int gkind,
                           int iter, double demin_i, double prmin_i, const double* wg_carry, RecovOut& res,
                           int defer = 0x7fffffff) {
  const double safty = 1.0e-4, saftybig = 1.0e5, dv = 1.0e-2;
  const double gam1 = gam / (gam - 1.0), gam2 = 1.0 / gam1;
  const double idetg1 = m.idetg;  // 1. / detg1
  double delta = 1.0, deltaend = 1.e-7;
  int irecov = 0;
  const double alpha1 = m.al;
  const double dro = alpha1 * u[0] * idetg1;
  double qcov[4], qcon[4], bcon[4], bcov[4], oncov[4], oncon[4];
  qcov[0] = alpha1 * (u[4] - u[0]) * idetg1;
  qcov[1] = alpha1 * u[1] * idetg1;
  qcov[2] = alpha1 * u[2] * idetg1;
  qcov[3] = alpha1 * u[3] * idetg1;
  const double gss = alpha1 * u[5] * idetg1;
  bcon[0] = 0.0;
  bcon[1] = alpha1 * u[6] * idetg1;
  bcon[2] = alpha1 * u[7] * idetg1;
  bcon[3] = alpha1 * u[8] * idetg1;
  double ro = q[0], pp = q[4];
  double util[4] = {0.0, q[1], q[2], q[3]};
  lower_g(bcon, bcov, m);
  upper_gc(qcov, qcon, m);
  const double bsq = bcon[1] * bcov[1] + bcon[2] * bcov[2] + bcon[3] * bcov[3];
  const double qdotb = qcov[0] * bcon[0] + qcov[1] * bcon[1] + qcov[2] * bcon[2] + qcov[3] * bcon[3];
  const double qdotbsq = qdotb * qdotb;
  oncov[0] = -1.0 * alpha1; oncov[1] = 0.0; oncov[2] = 0.0; oncov[3] = 0.0;
  upper_gc(oncov, oncon, m);
  const double qdotn = qcon[0] * oncov[0];
  const double qsq = qcov[0] * qcon[0] + qcov[1] * qcon[1] + qcov[2] * qcon[2] + qcov[3] * qcon[3];
  const double qtsq = qsq + (qdotn * qdotn);
  double utsq = qform3(m, util[1], util[2], util[3]);
  if (utsq < 0.0 && fabs(utsq) <= safty) utsq = fabs(utsq);
  if (fabs(utsq) > 1.e4) utsq = 1.e4;
  double gfsq = 1. + utsq;
  double gf = sqrt(gfsq);
  double vsq = (gfsq - 1.) * (1. / gfsq);
  const double t1a = 4. - vsq;
  const double t1b = 4. * (bsq + qdotn);
  const double t1c = qtsq + bsq * bsq + 2. * bsq * qdotn;
  double t1d = (t1b * t1b) - 4. * t1a * t1c;
  if (t1d <= 0.0) t1d = fabs(t1d);
  const double wgp = (-t1b + sqrt(t1d)) * (1. / (2. * t1a));
  const double wgm = (-t1b - sqrt(t1d)) * (1. / (2. * t1a));
  double wg;
  if (wgp > 0.0) wg = wgp;
  else if (wgm >= 0.0) wg = wgm;
  else {
    if (!wg_carry) return false;
    wg = *wg_carry;
  }
  bool cap = false;
  for (int cnt = 0;; ++cnt) {
    if (cnt >= kRescaleCap) { cap = true; break; }
    pp = gam2 * (wg * gf - dro * sqrt(gf));
    const double t3a = (wg * wg * wg) * (wg + 2. * bsq) - qdotbsq * (2. * wg + bsq);
    const double t3b = (wg * wg) * (qtsq - bsq * bsq);
    const double t3c = (wg * wg * wg) + (wg * wg) * (0.5 * bsq + qdotn - pp) - 0.5 * qdotbsq;
    if (t3a <= t3b) { wg = fabs(1.5 * wg); continue; }
    if (t3c > 0.0) { wg = fabs((double)0.9f * wg); continue; }
    break;
  }
  res.nr2 = false;
  if (!cap) {
    double wsq = wg * wg;
    const double xsq = (bsq + wg) * (bsq + wg);
    vsq = fabs((wsq * qtsq + qdotbsq * (bsq + 2. * wg)) * (1. / (wsq * xsq)));
    if (vsq > 1.0) vsq = 1.0 - dv;
    const double vsqo = vsq;
    double xxn = wg, yyn = vsq;
    // 2D Newton-Raphson on (W, v^2) (recov.f90:877-960)
    // Brent's cycle detection on the iterate (xxn, yyn), compared bit for bit:
    // the step is a function of the iterate alone, so once an iterate repeats
    // while the current step is still above the tolerance, every later step
    // repeats a step already found too large and the reference's loop runs to
    // iter without converging.  Its outcome (irecov = 1) is taken at once; the
    // 2D iterate is not used after a failure.
    long long cyc_x = __double_as_longlong(xxn), cyc_y = __double_as_longlong(yyn);
    int cyc_pow = 1, cyc_lam = 0;
    for (int nnn = 1; nnn <= iter; ++nnn) {
      if (!(fabs(delta) >= deltaend && irecov == 0)) break;
      if (nnn == iter) { irecov = 1; break; }
      if (nnn > 1 && __double_as_longlong(xxn) == cyc_x && __double_as_longlong(yyn) == cyc_y) {
        irecov = 1;
        break;
      }
      if (++cyc_lam == cyc_pow) {
        cyc_x = __double_as_longlong(xxn);
        cyc_y = __double_as_longlong(yyn);
        cyc_pow <<= 1;
        cyc_lam = 0;
      }
      if (nnn > defer) { res.deferred = true; return true; }
      wg = xxn;
      vsq = yyn;
      wsq = wg * wg;
      const double w3 = wsq * wg;
      double gtmp = 1. - vsq;
      if (gtmp < 0.0 || gtmp < safty) { gtmp = safty; vsq = 1. - gtmp; }
      const double ptmp = gam2 * (wg * gtmp - dro * sqrt(gtmp));
      const double f1 = qtsq - vsq * (wg + bsq) * (wg + bsq) + (qdotbsq * (bsq + 2. * wg)) * (1. / wsq);
      const double g1 = -qdotn - 0.5 * bsq * (1. + vsq) + 0.5 * (qdotbsq * (1. / wsq)) - wg + ptmp;
      const double dpdw = gam2 * gtmp;
      const double dpdvsq = -(gam2 * wg) + 0.5 * gam2 * dro * (1. / (sqrt(gtmp)));
      const double dfx = -(2. * (wg + bsq) * (vsq + qdotbsq * (1. / w3)));
      const double dfy = -((wg + bsq) * (wg + bsq));
      const double dgx = -1. - (qdotbsq * (1. / w3)) + dpdw;
      const double dgy = -(0.5 * bsq) + dpdvsq;
      double det = dfx * dgy - dfy * dgx;
      if (det == 0.0) det = 1.0;
      const double dx = (-(dgy * f1) + dfy * g1) * (1. / det);
      const double dy = (dgx * f1 - dfx * g1) * (1. / det);
      delta = 0.5 * (fabs(dx) + fabs(dy));
      xxn = wg + dx;
      yyn = vsq + dy;
      if (xxn < 0.0) xxn = fabs(xxn);
      if (xxn > saftybig) xxn = saftybig;
      if (yyn < 0.0) yyn = fabs(yyn);
      if (fabs(yyn) > 1.0) yyn = 1.0 - dv;
    }
    if (irecov == 0) {
      wg = xxn;
      vsq = yyn;
      double gtmp = 1. - vsq;
      if (gtmp < 0.0 || gtmp < safty) { gtmp = safty; vsq = 1. - gtmp; }
      gf = 1. / sqrt(gtmp);
      ro = dro * (1. / gf);
      const double w2 = wg * (gtmp);
      pp = gam2 * (w2 - ro);
      if (ro < 0.0 || pp < 0.0) irecov = 1;
      if (irecov == 0) {
#pragma unroll
        for (int a = 1; a <= 3; ++a) {
          const double qt = qcon[a] + oncon[a] * qdotn;
          util[a] = (gf * (1. / (wg + bsq))) * (qt + qdotb * bcon[a] * (1. / wg));
        }
      }
      wg = xxn;
      vsq = yyn;
    }
    // entropy Newton-Raphson on v^2 (recov.f90:1022-1147)
    if (irecov == 1) {
      res.nr2 = true;
      delta = 1.0;
      deltaend = 1.e-6;
      irecov = 0;
      xxn = vsqo;
      // Cycle detection as in the 2D iteration; here the last iterate's W is
      // kept on failure (the carried-in guess of a following cell), so on a
      // repeat the loop counter advances by whole cycles and the remaining
      // (fewer than one cycle of) iterations run as in the reference.
      long long cyc_s = __double_as_longlong(xxn);
      int cyc_pow2 = 1, cyc_lam2 = 0, cyc_at = 1;
      bool cyc_on = true;
      const double dro_g1 = spow(dro, gam - 1.);  // loop-invariant factor of dW/dv^2
      for (int nnn = 1; nnn <= iter; ++nnn) {
        if (!(fabs(delta) >= deltaend && irecov == 0)) break;
        if (nnn == iter) { irecov = 1; break; }
        if (cyc_on && nnn > 1 && __double_as_longlong(xxn) == cyc_s) {
          const int L = nnn - cyc_at;  // the iterate at the start of iteration cyc_at recurred
          nnn += ((iter - nnn) / L) * L;
          cyc_on = false;
          if (nnn == iter) { irecov = 1; break; }
        }
        if (cyc_on && ++cyc_lam2 == cyc_pow2) {
          cyc_s = __double_as_longlong(xxn);
          cyc_at = nnn;
          cyc_pow2 <<= 1;
          cyc_lam2 = 0;
        }
        if (nnn > defer) { res.deferred = true; return true; }
        vsq = xxn;
        double gtmp = 1. - vsq;
        if (gtmp < 0.0 || gtmp < safty) { gtmp = safty; vsq = 1. - gtmp; }
        gf = 1. / sqrt(gtmp);
        gfsq = gf * gf;
        ro = dro * (1. / gf);
        pp = (gss / dro) * pow_gam(ro, gam, gkind);
        const double roh = ro + gam1 * pp;
        wg = fabs(gfsq * roh);
        wsq = wg * wg;
        const double w3 = wsq * wg;
#ifdef RG_EXACT_ARITH
        const double dgfdvsq = 0.5 * spow(gtmp, -1.5);  // as recov.f90 writes it
#else
        const double dgfdvsq = 0.5 * (gfsq * gf);  // 0.5 gtmp^-1.5 with gf = gtmp^-1/2
#endif
        const double dwdvsq =
            dro * dgfdvsq + gam1 * gss * dro_g1 * (2. - gam) * pow_1mgam(gf, gam, gkind) * dgfdvsq;
        const double f = qtsq - vsq * (wg + bsq) * (wg + bsq) + (qdotbsq * (bsq + 2. * wg)) / wsq;
        const double ta = -((wg + bsq) * (wg + bsq));
        const double tb = -(2. * vsq * (wg + bsq));
        const double tc = -(2. * qdotbsq * (bsq + 2. * wg) * (1. / w3));
        const double td = 2. * qdotbsq * (1. / wsq);
        const double df = ta + (tb + tc + td) * dwdvsq;
        delta = f / df;
        xxn = vsq - delta;
        if (xxn < 0.0) xxn = fabs(xxn);
        if (fabs(xxn) >= 1.0) xxn = 1. - dv;
      }
      if (irecov == 0) {
        vsq = xxn;
        double gtmp = 1. - vsq;
        if (gtmp < 0.0 || gtmp < safty) gtmp = safty;
        gf = 1. / sqrt(gtmp);
        gfsq = gf * gf;
        ro = dro * (1. / gf);
        pp = (gss * (1. / gf)) * pow_gam1(ro, gam, gkind);
        if (ro < 0.0) ro = demin_i;
        if (pp < 0.0) pp = prmin_i;
        const double roh = ro + gam1 * pp;
        wg = fabs(gfsq * roh);
#pragma unroll
        for (int a = 1; a <= 3; ++a) {
          const double qt = qcon[a] + oncon[a] * qdotn;
          util[a] = (gf / (wg + bsq)) * (qt + qdotb * bcon[a] * (1. / wg));
        }
      }
    }
  } else {
    irecov = 1;
  }
  res.cap = cap;
  res.fail = (irecov != 0);
  res.wg = wg;
  // recov.f90:1174-1216 (the uu(6) rewrite is overwritten by caluu1 and is not kept)
  if (irecov == 0) {
    out[0] = ro; out[1] = util[1]; out[2] = util[2]; out[3] = util[3]; out[4] = pp;
    out[5] = ro * pp / pow_gam1(ro, gam, gkind);
  } else {
    out[0] = q[0]; out[1] = q[1]; out[2] = q[2]; out[3] = q[3]; out[4] = q[4];
    out[5] = q[0] * q[4] / pow_gam(q[0], gam, gkind);
  }
  out[6] = u[6] * idetg1;
  out[7] = u[7] * idetg1;
  out[8] = u[8] * idetg1;
  return true;
}

// recov.f90:1919-2456 (recov2, iwvec 2: Mignone & McKinney's one-variable
// Newton-Raphson on W' = W - D, gamma-law EoS), one interior cell, with the
// interface of recov_cell: the first W guess of a cell whose quadratic has no
// non-negative root comes from the previous cell in loop order (wg_carry, or
// false without one), and the unbounded rescale loop is capped (the capped
// cell keeps its primitives).  The reference's own choices are kept: D =
// alpha uu(1)/detg by division, u~^2 < 0 beyond the tolerance reset to 1e4,
// p = (W gamma - D sqrt(gamma)) (gam-1)/gam in the rescale loop, and
// p/rho^(gam-1) for uri(6).  No deferral: the iteration is one-dimensional.
__device__ bool recov2_cell(const double u[9], const double q[9], double out[9], const Met& m, double gam, int gkind,
                            int iter, double demin_i, double prmin_i, const double* wg_carry, RecovOut& res) {
  const double safty = 1.0e-5, dv = 1.0e-4;
  const double gam1 = gam / (gam - 1.0), gam2 = 1.0 / gam1;
  const double idetg1 = m.idetg;
  double delta = 1.0;
  const double deltaend = 1.e-8;
  int irecov = 0;
  const double alpha1 = m.al;
  const double dro = alpha1 * u[0] / m.detg;
  double qcov[4], qcon[4], bcon[4], bcov[4], oncov[4], oncon[4];
  qcov[0] = alpha1 * (u[4] - u[0]) * idetg1;
  qcov[1] = alpha1 * u[1] * idetg1;
  qcov[2] = alpha1 * u[2] * idetg1;
  qcov[3] = alpha1 * u[3] * idetg1;
  bcon[0] = 0.0;
  bcon[1] = alpha1 * u[6] * idetg1;
  bcon[2] = alpha1 * u[7] * idetg1;
  bcon[3] = alpha1 * u[8] * idetg1;
  double ro = q[0], pp = q[4];
  double util[4] = {0.0, q[1], q[2], q[3]};
  lower_g(bcon, bcov, m);
  upper_gc(qcov, qcon, m);
  const double bsq = bcon[1] * bcov[1] + bcon[2] * bcov[2] + bcon[3] * bcov[3];
  const double qdotb = qcov[0] * bcon[0] + qcov[1] * bcon[1] + qcov[2] * bcon[2] + qcov[3] * bcon[3];
  const double qdotbsq = qdotb * qdotb;
  oncov[0] = -1.0 * alpha1; oncov[1] = 0.0; oncov[2] = 0.0; oncov[3] = 0.0;
  upper_gc(oncov, oncon, m);
  const double qdotn = qcon[0] * oncov[0];
  const double qsq = qcov[0] * qcon[0] + qcov[1] * qcon[1] + qcov[2] * qcon[2] + qcov[3] * qcon[3];
  const double qtsq = qsq + (qdotn * qdotn);
  double utsq = qform3(m, util[1], util[2], util[3]);
  if (utsq < 0.0 && fabs(utsq) <= safty) utsq = fabs(utsq);
  if (utsq < 0.0 || fabs(utsq) > 1.e4) utsq = 1.e4;
  double gfsq = 1. + utsq;
  double gf = sqrt(gfsq);
  double vsq = (gfsq - 1.) * (1. / gfsq);
  const double t1a = 4. - vsq;
  const double t1b = 4. * (bsq + qdotn);
  const double t1c = qtsq + bsq * bsq + 2. * bsq * qdotn;
  double t1d = (t1b * t1b) - 4. * t1a * t1c;
  if (t1d <= 0.0) t1d = fabs(t1d);
  const double wgp = (-t1b + sqrt(t1d)) * (1. / (2. * t1a));
  const double wgm = (-t1b - sqrt(t1d)) * (1. / (2. * t1a));
  double wg;
  if (wgp > 0.0) wg = wgp;
  else if (wgm >= 0.0) wg = wgm;
  else {
    if (!wg_carry) return false;
    wg = *wg_carry;
  }
  bool cap = false;
  for (int cnt = 0;; ++cnt) {  // recov.f90:2147-2169
    if (cnt >= kRescaleCap) { cap = true; break; }
    pp = gam2 * (wg * gf - dro * sqrt(gf));
    const double t3a = (wg * wg * wg) * (wg + 2. * bsq) - qdotbsq * (2. * wg + bsq);
    const double t3b = (wg * wg) * (qtsq - bsq * bsq);
    const double t3c = (wg * wg * wg) + (wg * wg) * (0.5 * bsq + qdotn - pp) - 0.5 * qdotbsq;
    if (t3a <= t3b) { wg = fabs(1.5 * wg); continue; }
    if (t3c > 0.0) { wg = fabs((double)0.9f * wg); continue; }
    break;
  }
  if (cap) irecov = 1;
  // Newton-Raphson on W' (recov.f90:2174-2306)
  double wgd = wg - dro;
  double xxn = wgd;
  for (int nnn = 1; nnn <= iter; ++nnn) {
    if (!(fabs(delta) >= deltaend && irecov == 0)) break;  // nothing changes in the remaining iterations
    if (nnn == iter) { irecov = 1; break; }
    wgd = xxn;
    wg = wgd + dro;
    const double wsq = wg * wg, w3 = wsq * wg, xsq = (bsq + wg) * (bsq + wg);
    vsq = fabs((wsq * qtsq + qdotbsq * (bsq + 2. * wg)) * (1. / (wsq * xsq)));
    if (fabs(vsq) > 1.0) vsq = 1.0 - dv;
    if (vsq < 0.0) vsq = fabs(vsq);
    double gtmp = 1. - vsq;
    if (gtmp < 0.0 || gtmp < safty) { gtmp = safty; vsq = 1. - gtmp; }
    const double usq = (1. - gtmp) / (gtmp);
    gf = sqrt(1. + usq);
    gfsq = gf * gf;
    ro = dro / gf;
    const double xi = (wg - dro * gf) * (1. / gfsq);
    pp = gam2 * xi;
    const double dpdxi = gam2, dpdro = 0.0;
    const double ta = (bsq + wg);
    const double tb = (bsq + wg) * (bsq + wg) * (bsq + wg);
    const double tc = (qtsq == 0.0) ? 0.0 : -2. * qtsq * (1. / tb);
    const double td = (qdotbsq == 0.0) ? 0.0 : -2. * qdotbsq * (3. * wg * ta + bsq * bsq) * (1. / (tb * w3));
    const double dvdwd = tc + td;
    const double dxidwd = (1. / gfsq) - 0.5 * gf * (dro + 2. * gf * xi) * dvdwd;
    const double drodwd = -0.5 * dro * gf * dvdwd;
    const double dpdwd = dpdxi * dxidwd + dpdro * drodwd;
    const double t5a = bsq * qtsq - qdotbsq;
    const double t5b = bsq + wgd + dro;
    double t5c = 0.0, t5d = 0.0;
    if (t5a != 0.0) {
      t5c = 0.5 * t5a * (1. / (t5b * t5b));
      t5d = t5a * (1. / (t5b * t5b * t5b));
    }
    const double f = -(qdotn + dro) - wgd + pp - 0.5 * bsq - t5c;
    const double df = -1. + dpdwd + t5d;
    delta = f / df;
    xxn = wgd - delta;
    if (xxn < 0.0) xxn = fabs(xxn);
    if (xxn > 1.e8) xxn = 1.e8;
  }
  if (irecov == 0) {  // recov.f90:2310-2377
    wgd = xxn;
    wg = wgd + dro;
    const double wsq = wg * wg, xsq = (bsq + wg) * (bsq + wg);
    vsq = fabs((wsq * qtsq + qdotbsq * (bsq + 2. * wg)) * (1. / (wsq * xsq)));
    if (vsq < 0.0) vsq = fabs(vsq);
    if (vsq > 1.0) vsq = 1.0 - dv;
    double gtmp = 1. - vsq;
    if (gtmp < safty) gtmp = safty;
    const double usq = (1. - gtmp) / gtmp;
    gf = sqrt(1. + usq);
    gfsq = gf * gf;
    ro = dro / gf;
    const double xi = wg * (1. / gfsq) - ro;
    pp = gam2 * xi;
    if (ro < 0.0) ro = demin_i;
    if (pp < 0.0) pp = prmin_i;
#pragma unroll
    for (int a = 1; a <= 3; ++a) {
      const double qt = qcon[a] + oncon[a] * qdotn;
      util[a] = (gf * (1. / (wg + bsq))) * (qt + qdotb * bcon[a] * (1. / wg));
    }
  }
  res.nr2 = false;
  res.cap = cap;
  res.fail = (irecov != 0);
  res.wg = wg;
  if (irecov == 0) {  // recov.f90:2407-2441
    out[0] = ro; out[1] = util[1]; out[2] = util[2]; out[3] = util[3]; out[4] = pp;
    out[5] = pp / pow_gam1(ro, gam, gkind);
  } else {
    out[0] = q[0]; out[1] = q[1]; out[2] = q[2]; out[3] = q[3]; out[4] = q[4];
    out[5] = q[4] / pow_gam1(q[0], gam, gkind);
  }
  out[6] = u[6] * idetg1;
  out[7] = u[7] * idetg1;
  out[8] = u[8] * idetg1;
  return true;
}

// recov1a (IWVEC 1) or recov2 (IWVEC 2) of one cell.
template <int IWVEC>
__device__ __forceinline__ bool recov_any(const double u[9], const double q[9], double out[9], const Met& m, double gam,
                                          int gkind, int iter, double demin_i, double prmin_i,
                                          const double* wg_carry, RecovOut& res) {
  if constexpr (IWVEC == 2) return recov2_cell(u, q, out, m, gam, gkind, iter, demin_i, prmin_i, wg_carry, res);
  else return recov_cell(u, q, out, m, gam, gkind, iter, demin_i, prmin_i, wg_carry, res);
}

// ------------------------------------------------------------ stage update
// calsf.f90:107-151 with caltenr's T^m_n (calsf.f90:6-104): the source
// S_nu = sqrt(-g) sum_{n,m} T^m_n Gamma^n_{nu m} of one cell from its
// 4-vectors and the Christoffel cache at metric point q, summed in the
// reference's (n, m) order; sf[0..3] = sf(2:5) (nu = 1, 2, 3, 0).
// The cache holds Gamma^l_{mn} at l + 4m + 16n, symmetric in (m, n) bit for
// bit (the geometry builds it from a symmetric metric), so the 40 distinct
// values of a point are loaded and the 64-term sum reads them in the
// reference's order.
template <typename T>
__device__ __forceinline__ void load_christ_row(const T* __restrict__ chr, size_t nik, size_t q, int n, T g[4][4]) {
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = a; b < 4; ++b) g[a][b] = g[b][a] = __ldg(chr + (size_t)(n + 4 * a + 16 * b) * nik + q);
}

__device__ __forceinline__ void geom_source(const DevRun& r, const PS& s, size_t q, double detg, double sf[4]) {
  const double a = s.roh + s.bbsq, b = s.pr + 0.5 * s.bbsq;
  double ta = 0.0, tb = 0.0, tc = 0.0, td = 0.0;
  const size_t nik = r.nik;
#pragma unroll
  for (int n = 0; n < 4; ++n) {
    double g[4][4];  // g[nu][m] = Gamma^n_{nu m}
    load_christ_row(r.chr, nik, q, n, g);
#pragma unroll
    for (int mm = 0; mm < 4; ++mm) {
      const double t = a * s.ucon[mm] * s.ucov[n] + b * (mm == n ? 1.0 : 0.0) - s.bbcon[mm] * s.bbcov[n];
      ta = ta + t * g[1][mm];
      tb = tb + t * g[2][mm];
      tc = tc + t * g[3][mm];
      td = td + t * g[0][mm];
    }
  }
  sf[0] = detg * ta; sf[1] = detg * tb; sf[2] = detg * tc; sf[3] = detg * td;
}

// rk2fst (rkt.f90:2-42), rk3snd (rkt.f90:91-134) and rk3trd (rkt.f90:137-180)
// for one variable: uo = U^n, uc = the stage input (uu, uh or us), a? = dt/dx?b
// and d? the flux differences; (1./3.) and (2./3.) are single-precision
// literals in the reference.
template <int STAGE>
__device__ __forceinline__ double rk_combine(double uo, double uc, double a1, double d1, double a2, double d2,
                                             double a3, double d3) {
  if (STAGE == 1) return uc - a1 * d1 - a2 * d2 - a3 * d3;
  if (STAGE == 2) return (3.0 * uo + uc) * 0.25 + (-(a1 * d1) - a2 * d2 - a3 * d3) * 0.25;
  return (uo + 2. * uc) * (double)(1.0f / 3.0f) + (-(a1 * d1) - a2 * d2 - a3 * d3) * (double)(2.0f / 3.0f);
}
// rk2adsff / rk3adsfs / rk3adsft (rkt.f90:183-215, 253-320) for one of variables 2-5.
template <int STAGE>
__device__ __forceinline__ double rk_add_source(double u, double sf, double dt) {
  if (STAGE == 1) return u + sf * dt;
  if (STAGE == 2) return u + sf * dt * 0.25;
  return u + sf * dt * (double)(2.0f / 3.0f);
}

// Conserved state after the RK combine and source (rkt.f90:2-320) of one
// interior cell.  U = P2C(P) always holds in the reference (caluu1 runs after
// every stage, main.f90:899), so the stage inputs uu/uo/uh/us are recomputed
// from the stored primitives here.  Two halves: stage_pre (P2C of the stage
// input, U^n stored in stage 1, the geometric source) and stage_combine (the
// RK combine with the flux differences and the source), which reads the flux
// differences through an accessor: FluxDiffGlobal from the flux arrays, or
// the shared-memory rows of the TMA-staged update.
template <int STAGE>
__device__ __forceinline__ void stage_pre(const DevRun& r, int i, int j, int k, const Met& m,
                                          const double* __restrict__ Pc, double ucur[9], double sf[4]) {
  const size_t N = r.N, c = r.cell(i, j, k), q = r.ik(i, k);
  const double gam = r.gam;
  double qc[9];
  load9(Pc, N, c, qc);
  PS s;
  pstate(qc, m, gam, s);
  p2c(s, gam, r.gkind, m.detg, ucur);
  // U^n = P2C(P^n) is this stage's ucur in stage 1; stages 2 and 3 read it back
  if (STAGE == 1)
#pragma unroll
    for (int v = 0; v < 9; ++v) r.Un[(size_t)v * N + c] = ucur[v];
  // geometric source (calsf.f90:6-151): S_nu = sqrt(-g) T^m_n Gamma^n_{nu m}
  geom_source(r, s, q, m.detg, sf);
}

// Flux differences of variable v along the three directions at cell c from
// the flux arrays; flux-CT replaces ww(2,7) ww(3,7) ww(1,8) ww(3,8) ww(1,9)
// ww(2,9) (ct.f90:98-109).
struct FluxDiffGlobal {
  const double* __restrict__ F1;
  const double* __restrict__ F2;
  const double* __restrict__ F3;
  const double* __restrict__ CT;
  size_t N, c, ci, cj, ck;
  __device__ __forceinline__ void operator()(int v, double& d1, double& d2, double& d3) const {
    if (v == 7) d1 = CT[2 * N + c] - CT[2 * N + ci];
    else if (v == 8) d1 = CT[4 * N + c] - CT[4 * N + ci];
    else d1 = F1[(size_t)v * N + c] - F1[(size_t)v * N + ci];
    if (v == 6) d2 = CT[0 * N + c] - CT[0 * N + cj];
    else if (v == 8) d2 = CT[5 * N + c] - CT[5 * N + cj];
    else d2 = F2[(size_t)v * N + c] - F2[(size_t)v * N + cj];
    if (v == 6) d3 = CT[1 * N + c] - CT[1 * N + ck];
    else if (v == 7) d3 = CT[3 * N + c] - CT[3 * N + ck];
    else d3 = F3[(size_t)v * N + c] - F3[(size_t)v * N + ck];
  }
};

template <int STAGE, typename Diff>
__device__ __forceinline__ void stage_combine(const DevRun& r, int i, int j, int k, const double ucur[9],
                                              const double sf[4], const double uo[9], double dt, const Diff& diff,
                                              double u[9]) {
  const double a1 = dt / __ldg(r.dx1b + i - 1), a2 = dt / __ldg(r.dx2b + j - 1), a3 = dt / __ldg(r.dx3b + k - 1);
#pragma unroll
  for (int v = 0; v < 9; ++v) {
    double d1, d2, d3;
    diff(v, d1, d2, d3);
    u[v] = rk_combine<STAGE>(STAGE > 1 ? uo[v] : 0.0, ucur[v], a1, d1, a2, d2, a3, d3);
  }
#pragma unroll
  for (int v = 1; v <= 4; ++v) u[v] = rk_add_source<STAGE>(u[v], sf[v - 1], dt);
}

template <int STAGE>
__device__ void stage_rhs(const DevRun& r, int i, int j, int k, const Met& m, const double* __restrict__ Pn,
                          const double* __restrict__ Pc, const double* __restrict__ F1, const double* __restrict__ F2,
                          const double* __restrict__ F3, const double* __restrict__ CT, double dt, double u[9]) {
  const size_t N = r.N, c = r.cell(i, j, k);
  double ucur[9], sf[4];
  stage_pre<STAGE>(r, i, j, k, m, Pc, ucur, sf);
  double uo[9];
  if (STAGE > 1) load9(r.Un, N, c, uo);
  const FluxDiffGlobal diff{F1, F2, F3, CT, N, c, c - 1, c - r.sj, c - r.sk};
  stage_combine<STAGE>(r, i, j, k, ucur, sf, uo, dt, diff, u);
}

// Compensated FP32 accumulation (Kahan/Knuth two-sum, FMA two-product):
// the running sum keeps its rounding error in a second float.
struct Acc32 {
  float s = 0.f, c = 0.f;
  __device__ __forceinline__ void add(float t) {
    const float x = s + t;
    const float bb = x - s;
    c += (s - (x - bb)) + (t - bb);
    s = x;
  }
  // coef * (hi + lo) with the product's rounding error kept (fmaf)
  __device__ __forceinline__ void add_scaled(float coef, float hi, float lo) {
    const float p = coef * hi;
    const float e = fmaf(coef, hi, -p);
    add(p);
    c += e + coef * lo;
  }
  __device__ __forceinline__ double value() const { return (double)s + (double)c; }
};

__device__ __forceinline__ void split(double x, float& hi, float& lo) {
  hi = (float)x;
  lo = (float)(x - (double)hi);
}

// Mixed-precision counterpart of stage_rhs for cells beyond r = 2 r_H: the
// flux divergence (FP32 face fluxes and flux-CT values), the geometric source
// (FP32 Christoffel cache, FP32 copy of the cell's 4-vectors) and the RK
// combine run in FP32; the combine accumulates with compensation (Acc32), so
// the conserved state keeps the FP64 precision of its inputs U^n and
// P2C(P).  Those inputs, the stored-state stand-ins of the reference's uu/uo
// arrays, stay FP64, as does the primitive recovery that follows.
template <int STAGE>
__device__ __forceinline__ void stage_pre_mixed(const DevRun& r, int i, int j, int k, const Met& m,
                                                const double* __restrict__ Pc, double ucur[9], float sf[4]) {
  const size_t N = r.N, c = r.cell(i, j, k), q = r.ik(i, k);
  const double gam = r.gam;
  double qc[9];
  load9(Pc, N, c, qc);
  PS s;
  pstate(qc, m, gam, s);
  p2c(s, gam, r.gkind, m.detg, ucur);
  if (STAGE == 1)
#pragma unroll
    for (int v = 0; v < 9; ++v) r.Un[(size_t)v * N + c] = ucur[v];
  const size_t nik = r.nik;
  const float a = (float)(s.roh + s.bbsq), b = (float)(s.pr + 0.5 * s.bbsq);
  float uc[4], ul[4], bc[4], bl[4];
#pragma unroll
  for (int n = 0; n < 4; ++n) {
    uc[n] = (float)s.ucon[n]; ul[n] = (float)s.ucov[n]; bc[n] = (float)s.bbcon[n]; bl[n] = (float)s.bbcov[n];
  }
  float ta = 0.f, tb = 0.f, tc = 0.f, td = 0.f;
#pragma unroll
  for (int n = 0; n < 4; ++n) {
    float g[4][4];
    load_christ_row(r.chr32, nik, q, n, g);
#pragma unroll
    for (int mm = 0; mm < 4; ++mm) {
      const float t = a * uc[mm] * ul[n] + (mm == n ? b : 0.f) - bc[mm] * bl[n];
      ta = ta + t * g[1][mm];
      tb = tb + t * g[2][mm];
      tc = tc + t * g[3][mm];
      td = td + t * g[0][mm];
    }
  }
  const float dg = (float)m.detg;
  sf[0] = dg * ta; sf[1] = dg * tb; sf[2] = dg * tc; sf[3] = dg * td;
}

// FP32 flux differences of variable v from the FP32 face fluxes and flux-CT
// values (global arrays).
struct FluxDiffGlobal32 {
  const float* __restrict__ F1;
  const float* __restrict__ F2;
  const float* __restrict__ F3;
  const float* __restrict__ CT;
  size_t N, c, ci, cj, ck;
  __device__ __forceinline__ void operator()(int v, float& d1, float& d2, float& d3) const {
    auto fd = [&](const float* A, size_t x, size_t xm) { return A[x] - A[xm]; };
    if (v == 7) d1 = fd(CT + 2 * N, c, ci);
    else if (v == 8) d1 = fd(CT + 4 * N, c, ci);
    else d1 = fd(F1 + (size_t)v * N, c, ci);
    if (v == 6) d2 = fd(CT, c, cj);
    else if (v == 8) d2 = fd(CT + 5 * N, c, cj);
    else d2 = fd(F2 + (size_t)v * N, c, cj);
    if (v == 6) d3 = fd(CT + 1 * N, c, ck);
    else if (v == 7) d3 = fd(CT + 3 * N, c, ck);
    else d3 = fd(F3 + (size_t)v * N, c, ck);
  }
};

// The compensated FP32 combine of the mixed path (uo = U^n in stages 2, 3).
template <int STAGE, typename Diff>
__device__ __forceinline__ void stage_combine_mixed(const DevRun& r, int i, int j, int k, const double ucur[9],
                                                    const float sf[4], const double uo[9], double dt,
                                                    const Diff& diff, double u[9]) {
  const float a1 = (float)(dt / __ldg(r.dx1b + i - 1)), a2 = (float)(dt / __ldg(r.dx2b + j - 1)),
              a3 = (float)(dt / __ldg(r.dx3b + k - 1));
  const float fdt = (float)dt;
  // stage weights: U = wo*uo + wc*ucur + wf*(flux divergence + dt*S)
  const float wo = (STAGE == 1) ? 0.f : (STAGE == 2 ? 0.75f : 1.0f / 3.0f);
  const float wc = (STAGE == 1) ? 1.f : (STAGE == 2 ? 0.25f : 2.0f / 3.0f);
  const float wf = wc;
#pragma unroll
  for (int v = 0; v < 9; ++v) {
    float d1, d2, d3;
    diff(v, d1, d2, d3);
    Acc32 acc;
    float hi, lo;
    if (STAGE > 1) {
      split(uo[v], hi, lo);
      acc.add_scaled(wo, hi, lo);
    }
    split(ucur[v], hi, lo);
    acc.add_scaled(wc, hi, lo);
    float inc = -(a1 * d1) - a2 * d2 - a3 * d3;
    if (v >= 1 && v <= 4) inc = inc + sf[v - 1] * fdt;
    acc.add(wf * inc);
    u[v] = acc.value();
  }
}

template <int STAGE>
__device__ void stage_rhs_mixed(const DevRun& r, int i, int j, int k, const Met& m, const double* __restrict__ Pc,
                                double dt, double u[9]) {
  const size_t N = r.N, c = r.cell(i, j, k);
  double ucur[9];
  float sf[4];
  stage_pre_mixed<STAGE>(r, i, j, k, m, Pc, ucur, sf);
  double uo[9];
  if (STAGE > 1) load9(r.Un, N, c, uo);
  const FluxDiffGlobal32 diff{r.F32[0], r.F32[1], r.F32[2], r.CT32, N, c, c - 1, c - r.sj, c - r.sk};
  stage_combine_mixed<STAGE>(r, i, j, k, ucur, sf, uo, dt, diff, u);
}

__device__ __forceinline__ bool is_interior(const DevRun& r, int i, int j, int k) {
  return i > r.nm1 && i <= r.imax - r.nm1 && j > r.nm1 && j <= r.jmax - r.nm1 && k > r.nm1 && k <= r.kmax - r.nm1;
}

__device__ __forceinline__ void queue_carry(const DevRun& r, int i, int j, int k) {
  const int ni = r.imax - 2 * r.nm1, nj = r.jmax - 2 * r.nm1;
  const int lin = (i - r.nm1 - 1) + ni * ((j - r.nm1 - 1) + nj * (k - r.nm1 - 1));
  const int slot = atomicAdd(&r.scal->carry_count, 1);
  if (slot < r.carry_cap) r.carry_list[slot] = lin;
  else atomicAdd(r.cnt + C_CARRY_OVF, 1ull);
}

// Divergence-aware recovery: a cell whose Newton-Raphson has not converged
// after kDeferIter iterations (the usual count is 2-10; the reference allows
// `iter` = 5000 per loop) is queued instead of holding its warp, and the
// straggler pass recomputes the queued cells from scratch, packed one per
// thread, so a slow cell costs one thread's time rather than 32.  The result
// is the same as the undeferred computation.
constexpr int kDeferIter = 64;

// Queue a deferred cell; false if the list is full (the caller then finishes it in place).
__device__ __forceinline__ bool queue_straggler(const DevRun& r, int i, int j, int k) {
  const int ni = r.imax - 2 * r.nm1, nj = r.jmax - 2 * r.nm1;
  const int lin = (i - r.nm1 - 1) + ni * ((j - r.nm1 - 1) + nj * (k - r.nm1 - 1));
  const int slot = atomicAdd(&r.scal->strag_count, 1);
  if (slot >= r.strag_cap) return false;
  r.strag_list[slot] = lin;
  return true;
}

#ifndef RG_UPDATE_MINB
#define RG_UPDATE_MINB 3
#endif
// Block of the stage update: RG_UPDATE_BX cells along i times 128 / RG_UPDATE_BX
// rows along j (the rows share the metric of their (i, k) points; 32 x 4
// measured 0.4% faster than 64 x 2 and 16 x 8 on the 256x128x128 torus).
#ifndef RG_UPDATE_BX
#define RG_UPDATE_BX 32
#endif

// recov1a of one interior cell from its stage conserved state u, with
// straggler deferral (the cell is queued for k_straggler when its iteration
// count passes kDeferIter and the list has room) and the loop-order W carry
// for cells without a root; the primitives go to Pw.
__device__ __forceinline__ void update_recov(const DevRun& r, int i, int j, int k, const Met& m,
                                             const double* __restrict__ Pc, double* __restrict__ Pw,
                                             const double u[9]) {
  const size_t N = r.N, c = r.cell(i, j, k);
  double qo[9], qn[9];
  load9(Pc, N, c, qo);
  RecovOut o{0.0, false, false, false};
  const double dei = __ldg(r.fl_de + i - 1), pri = __ldg(r.fl_pr + i - 1);
  bool ok = recov_cell(u, qo, qn, m, r.gam, r.gkind, r.iter, dei, pri, nullptr, o, r.strag_list ? kDeferIter : 0x7fffffff);
  if (o.deferred) {
    if (queue_straggler(r, i, j, k)) return;
    o = RecovOut{0.0, false, false, false};
    ok = recov_cell(u, qo, qn, m, r.gam, r.gkind, r.iter, dei, pri, nullptr, o);
  }
  if (!ok) {
    queue_carry(r, i, j, k);
  } else {
#pragma unroll
    for (int v = 0; v < 9; ++v) Pw[(size_t)v * N + c] = qn[v];
  }
  count_event(r, C_NR2, ok && o.nr2);
  count_event(r, C_FAIL, ok && o.fail);
  count_event(r, C_CAP, ok && o.cap);
}

// One stage of every cell with radial index in [ilo, ihi]: interior cells get
// the RK combine (FP64, or MIX = mixed precision for the cells beyond
// r = 2 r_H) and recov1a; ghost cells copy their primitives through.
template <int STAGE, bool MIX>
__device__ __forceinline__ void update_body(const DevRun& r, const double* __restrict__ Pn, const double* __restrict__ Pc,
                                                double* __restrict__ Pw, const double* __restrict__ F1,
                                                const double* __restrict__ F2, const double* __restrict__ F3,
                                                const double* __restrict__ CT, int ilo, int ihi, const uint3 bid) {
  const int i = bid.x * blockDim.x + threadIdx.x + ilo;
  const int j = jidx(r, 1, bid);
  const int k = kidx(r, 1, bid);
  if (i > ihi || j > r.jmax || k > r.kmax) return;
  const size_t N = r.N, c = r.cell(i, j, k);
  // A finished run (time > tmax) copies its state through the stage so that the
  // host-side buffer rotation stays valid without a host synchronisation.
  if (!r.scal->active || !is_interior(r, i, j, k)) {
#pragma unroll
    for (int v = 0; v < 9; ++v) Pw[(size_t)v * N + c] = Pc[(size_t)v * N + c];
    return;
  }
  Met m;
  load_met(r.mc, r.nik, r.ik(i, k), m);
  double u[9];
  if (MIX) stage_rhs_mixed<STAGE>(r, i, j, k, m, Pc, r.scal->dt, u);
  else stage_rhs<STAGE>(r, i, j, k, m, Pn, Pc, F1, F2, F3, CT, r.scal->dt, u);
  update_recov(r, i, j, k, m, Pc, Pw, u);
}

// The straggler pass: slot t of the run's list, recomputed without deferral
// (stage combine, source, then recov1a), in the reference's arithmetic.
template <int STAGE>
__device__ __forceinline__ void straggler_body(const DevRun& r, const double* __restrict__ Pn,
                                               const double* __restrict__ Pc, double* __restrict__ Pw,
                                               const double* __restrict__ F1, const double* __restrict__ F2,
                                               const double* __restrict__ F3, const double* __restrict__ CT,
                                               const uint3 bid) {
  if (!r.scal->active) return;
  const int t = bid.x * blockDim.x + threadIdx.x;
  const int n = min(r.scal->strag_count, r.strag_cap);
  if (t >= n) return;
  const int lin = r.strag_list[t];
  const int ni = r.imax - 2 * r.nm1, nj = r.jmax - 2 * r.nm1;
  const int i = lin % ni + r.nm1 + 1, j = (lin / ni) % nj + r.nm1 + 1, k = lin / (ni * nj) + r.nm1 + 1;
  const size_t N = r.N, c = r.cell(i, j, k);
  Met m;
  load_met(r.mc, r.nik, r.ik(i, k), m);
  double u[9], qo[9], qn[9];
  if (r.mixed && i > r.i_fp64) stage_rhs_mixed<STAGE>(r, i, j, k, m, Pc, r.scal->dt, u);
  else stage_rhs<STAGE>(r, i, j, k, m, Pn, Pc, F1, F2, F3, CT, r.scal->dt, u);
  load9(Pc, N, c, qo);
  RecovOut o{0.0, false, false, false};
  const bool ok = recov_cell(u, qo, qn, m, r.gam, r.gkind, r.iter, __ldg(r.fl_de + i - 1), __ldg(r.fl_pr + i - 1),
                             nullptr, o);
  if (!ok) {
    queue_carry(r, i, j, k);
  } else {
#pragma unroll
    for (int v = 0; v < 9; ++v) Pw[(size_t)v * N + c] = qn[v];
  }
  count_event(r, C_NR2, ok && o.nr2);
  count_event(r, C_FAIL, ok && o.fail);
  count_event(r, C_CAP, ok && o.cap);
}

template <int STAGE>
__global__ void __launch_bounds__(128) k_straggler(DevRun r, const double* __restrict__ Pn,
                                                   const double* __restrict__ Pc, double* __restrict__ Pw,
                                                   const double* __restrict__ F1, const double* __restrict__ F2,
                                                   const double* __restrict__ F3, const double* __restrict__ CT) {
  straggler_body<STAGE>(r, Pn, Pc, Pw, F1, F2, F3, CT, blockIdx);
}
template <int STAGE, bool MIX>
__global__ void __launch_bounds__(128, RG_UPDATE_MINB) k_update(DevRun r, const double* __restrict__ Pn, const double* __restrict__ Pc,
                                                double* __restrict__ Pw, const double* __restrict__ F1,
                                                const double* __restrict__ F2, const double* __restrict__ F3,
                                                const double* __restrict__ CT, int ilo, int ihi) { update_body<STAGE, MIX>(r, Pn, Pc, Pw, F1, F2, F3, CT, ilo, ihi, blockIdx); }

// Resolve cells queued by k_update / k_recov in the reference's loop order
// (k, j, i over the interior): each takes the final W of its predecessor cell
// (recov.f90:810-815).  Runs only when cells were queued.  The whole block
// works on the run's list: the queued cells are ranked into loop order
// (carry_sorted), and every maximal chain of consecutive queued cells is one
// sequential task, given to one thread: its first cell takes the W of its
// unqueued predecessor (recomputed, it has a root of its own), every later
// cell the W its predecessor in the chain ends with.  That is the reference's
// sequence of W values, so the result equals a serial sweep over the list;
// chains proceed in parallel.  MODE 0: stage update; MODE 1: recov-only
// entry point.  Every thread of the block calls it.
template <int MODE, int STAGE, int IWVEC = 1>
__device__ void carry_fix_body(const DevRun& r, const double* __restrict__ Pn, const double* __restrict__ Pc,
                               double* __restrict__ Pw, const double* __restrict__ F1, const double* __restrict__ F2,
                               const double* __restrict__ F3, const double* __restrict__ CT,
                               const double* __restrict__ U) {
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nt = blockDim.x * blockDim.y * blockDim.z;
  const bool active = MODE != 0 || r.scal->active;
  int n = r.scal->carry_count;
  __syncthreads();  // every thread has read the scalars before thread 0 resets them
  if (MODE == 0 && tid == 0) r.scal->strag_count = 0;  // the straggler pass of this stage has run
  if (!active || n <= 0) {
    if (tid == 0 && n > 0) r.scal->carry_count = 0;
    return;
  }
  if (n > r.carry_cap) n = r.carry_cap;
  const int* L = r.carry_list;
  int* S = r.carry_sorted;
  for (int a = tid; a < n; a += nt) {  // rank of each queued cell in loop order (indices are distinct)
    const int x = L[a];
    int rank = 0;
    for (int b = 0; b < n; ++b) rank += (L[b] < x);
    S[rank] = x;
  }
  __syncthreads();
  const int ni = r.imax - 2 * r.nm1, nj = r.jmax - 2 * r.nm1;
  const double dt = (MODE == 0) ? r.scal->dt : 0.0;
  auto run_cell = [&](int lin, const double* carry, double& wg_out, bool write, RecovOut& o) -> bool {
    const int i = lin % ni + r.nm1 + 1, j = (lin / ni) % nj + r.nm1 + 1, k = lin / (ni * nj) + r.nm1 + 1;
    const size_t c = r.cell(i, j, k);
    Met m;
    load_met(r.mc, r.nik, r.ik(i, k), m);
    double u[9], qo[9], qn[9];
    if (MODE == 0 && r.mixed && i > r.i_fp64) stage_rhs_mixed<STAGE>(r, i, j, k, m, Pc, dt, u);
    else if (MODE == 0) stage_rhs<STAGE>(r, i, j, k, m, Pn, Pc, F1, F2, F3, CT, dt, u);
    else load9(U, r.N, c, u);
    load9(Pc, r.N, c, qo);
    const bool ok = recov_any<IWVEC>(u, qo, qn, m, r.gam, r.gkind, r.iter, r.fl_de[i - 1], r.fl_pr[i - 1], carry, o);
    if (ok) {
      wg_out = o.wg;
      if (write)
        for (int v = 0; v < 9; ++v) Pw[(size_t)v * r.N + c] = qn[v];
    }
    return ok;
  };
  for (int p = tid; p < n; p += nt) {
    if (p > 0 && S[p - 1] == S[p] - 1) continue;  // inside a chain: its head's thread takes it
    double wg_in = 0.0;  // the first cell of the sweep starts from W = 0 (recov.f90:642)
    if (S[p] > 0) {
      RecovOut po{0.0, false, false, false};
      run_cell(S[p] - 1, nullptr, wg_in, false, po);  // the predecessor has a root of its own
    }
    for (int q = p; q < n && (q == p || S[q] == S[q - 1] + 1); ++q) {
      RecovOut o{0.0, false, false, false};
      double w = 0.0;
      run_cell(S[q], &wg_in, w, true, o);
      wg_in = w;
      atomicAdd(r.cnt + C_CARRY, 1ull);
      if (o.nr2) atomicAdd(r.cnt + C_NR2, 1ull);
      if (o.fail) atomicAdd(r.cnt + C_FAIL, 1ull);
      if (o.cap) atomicAdd(r.cnt + C_CAP, 1ull);
    }
  }
  __syncthreads();
  if (tid == 0) r.scal->carry_count = 0;
}
constexpr int kCarryThreads = 128;
template <int MODE, int STAGE, int IWVEC = 1>
__global__ void __launch_bounds__(kCarryThreads) k_carry_fix(DevRun r, const double* __restrict__ Pn, const double* __restrict__ Pc,
                            double* __restrict__ Pw, const double* __restrict__ F1, const double* __restrict__ F2,
                            const double* __restrict__ F3, const double* __restrict__ CT, const double* __restrict__ U) {
  // one block: every thread takes part (the body ranks the queued cells and
  // runs the chains with the whole block, with block barriers)
  carry_fix_body<MODE, STAGE, IWVEC>(r, Pn, Pc, Pw, F1, F2, F3, CT, U);
}

// ------------------------------------------------------------- face fluxes
// Face f+1/2 in direction D over the hll range nm0..n-nm0 in every dimension
// (hll.f90:83-85).  Two neighbouring lanes share a face: the even lane
// builds the left state from cell f (uriil(f)), the odd lane the right state
// from cell f+1 (uriir(f), rec.f90:2138); each evaluates its state's conserved
// variables, flux and wave speeds in arithmetic type T, and the pair exchanges
// them by warp shuffle for the LLF flux.  Lanes past the edge of the range work
// on the last face and store nothing.  Both lanes of a pair always take the
// same branch, so the shuffles run on the active mask.  S is the storage type
// of the primitives, metric cache and fluxes (double, or float for the FP32
// half of the mixed path, which then reads and writes no FP64 array).  Fcopy,
// if given, receives an FP32 copy of the fluxes of faces i <= icopy (the FP64
// faces next to the FP32 region of the mixed path).
template <int D, typename S>
__device__ __forceinline__ const S* met_of(const DevRun& r);
template <>
__device__ __forceinline__ const double* met_of<1, double>(const DevRun& r) { return r.mi; }
template <>
__device__ __forceinline__ const double* met_of<2, double>(const DevRun& r) { return r.mc; }
template <>
__device__ __forceinline__ const double* met_of<3, double>(const DevRun& r) { return r.mk; }
template <>
__device__ __forceinline__ const float* met_of<1, float>(const DevRun& r) { return r.mi32; }
template <>
__device__ __forceinline__ const float* met_of<2, float>(const DevRun& r) { return r.mc32; }
template <>
__device__ __forceinline__ const float* met_of<3, float>(const DevRun& r) { return r.mk32; }

//
// VIEW: the stencil (and the positivity fallback) is read from a staged copy
// of the primitives instead of P: variable v of the lane's cell at
// Vp[v * Vn + Vc], neighbours along D Vst apart (the shared-memory box of
// k_flux_tma).  Stores, metric and coordinates stay global.
//
// OUT (the per-routine rg_rec2): the lane also stores its face state, face
// conserved variables and face flux, all nine variables (the sixth included),
// into fo->q/u/w[side] at the face's cell index (rec.f90's uri?l/uri?r,
// uu?l/uu?r, ww?l/ww?r of face f+1/2 at index f).
struct FaceOut {
  double* q[2];
  double* u[2];
  double* w[2];
};
template <int D, int IREC, typename T, typename S, bool VIEW = false, bool OUT = false>
__device__ __forceinline__ void face_lane(const DevRun& r, const S* __restrict__ P, S* __restrict__ F,
                                          float* __restrict__ Fcopy, int icopy, int i, int j, int k, int side,
                                          bool valid, const S* Vp = nullptr, size_t Vn = 0, size_t Vc = 0,
                                          long long Vst = 0, const FaceOut* fo = nullptr,
                                          const S* Mv = nullptr, int Mst = 0) {
  const unsigned mask = __activemask();
  const size_t N = r.N, c = r.cell(i, j, k);
  const long long st = (D == 1) ? 1 : (D == 2 ? (long long)r.sj : (long long)r.sk);
  const S* Pv = VIEW ? Vp : P;
  const size_t Nv = VIEW ? Vn : N, cv = VIEW ? Vc : c;
  const long long sv = VIEW ? Vst : st;
  T q[9];
  if (IREC == 5) {
    const int f = ((D == 1) ? i : (D == 2 ? j : k)) + side;  // owner cell of this lane's state
    const double* dxs = (D == 1) ? r.dx1s : (D == 2 ? r.dx2s : r.dx3s);
    const double* xs = (D == 1) ? r.x1 : (D == 2 ? r.x2 : r.x3);
    T dx[9], xx[9], other[9];
#pragma unroll
    for (int o = -2; o <= 2; ++o) dx[o + 4] = T(__ldg(dxs + f - 1 + o));
#pragma unroll
    for (int o = -1; o <= 1; ++o) xx[o + 4] = T(__ldg(xs + f - 1 + o));
    if (side == 0) ppm_cell<D, T, S, OUT>(Pv + cv, Nv, sv, dx, xx, T(r.gam), other, q);  // uriil(f)
    else ppm_cell<D, T, S, OUT>(Pv + cv + sv, Nv, sv, dx, xx, T(r.gam), q, other);       // uriir(f)
  } else if (IREC == 1 || IREC == 2 || IREC == 11 || IREC == 12 || IREC == 13) {
    // owner cell f of this lane's state and its coordinate's coefficients
    const int f = ((D == 1) ? i : (D == 2 ? j : k)) + side;
    const int n = (D == 1) ? r.imax : (D == 2 ? r.jmax : r.kmax);
    const double* lc = r.lim[D - 1];
    T co[6];
#pragma unroll
    for (int a = 0; a < 6; ++a) co[a] = T(__ldg(lc + a * n + f - 1));
    // koren's j sweep takes the i-direction slope sign in its backward state
    const bool cross = (IREC == 13 && D == 2 && side == 1);
    const T hpi = cross ? T(__ldg(r.lim[0] + i - 1)) : T(0);
#pragma unroll
    for (int v = 0; v < 9; ++v) {
      if (v == 5 && !OUT) { q[v] = T(0); continue; }  // var 6 faces are never read downstream
      const S* p = Pv + (size_t)v * Nv + cv + side * sv;
      const T u0 = T(p[0]);
      T tmp_b = T(0);
      if (cross) tmp_b = ((T(p[1]) - u0) * hpi < T(0)) ? T(-1) : T(1);
      else if (IREC == 13) tmp_b = ((T(p[sv]) - u0) * co[0] < T(0)) ? T(-1) : T(1);
      q[v] = limiter_state<IREC>(T(p[-sv]), u0, T(p[sv]), co, side, tmp_b);
    }
  } else if (IREC == 4) {
    const int f = ((D == 1) ? i : (D == 2 ? j : k)) + side;
    const int n = (D == 1) ? r.imax : (D == 2 ? r.jmax : r.kmax);
    const double* lc = r.lim[D - 1];
    T co[10];
#pragma unroll
    for (int a = 0; a < 10; ++a) co[a] = T(__ldg(lc + a * n + f - 1));
#pragma unroll
    for (int v = 0; v < 9; ++v) {
      if (v == 5 && !OUT) { q[v] = T(0); continue; }  // var 6 faces are never read downstream
      const S* p = Pv + (size_t)v * Nv + cv + side * sv;
      q[v] = ceno_state(T(p[-2 * sv]), T(p[-sv]), T(p[0]), T(p[sv]), T(p[2 * sv]), co, side, D == 3 && side == 0);
    }
  } else if (IREC == 3) {
#pragma unroll
    for (int v = 0; v < 9; ++v) {
      if (v == 5 && !OUT) { q[v] = T(0); continue; }  // var 6 faces are never read downstream
      const S* p = Pv + (size_t)v * Nv + cv + side * sv;
      q[v] = muscl_state(T(p[-sv]), T(p[0]), T(p[sv]), side);
    }
  } else {
#pragma unroll
    for (int v = 0; v < 9; ++v) {
      if (v == 5 && !OUT) { q[v] = T(0); continue; }  // var 6 faces are never read downstream
      // owner cell f + side; the right state reads its stencil mirrored
      const long long sd = side ? -sv : sv;
      const S* p = Pv + (size_t)v * Nv + cv + side * sv;
      const T a2 = T(p[-2 * sd]), a1 = T(p[-sd]), u0 = T(p[0]), b1 = T(p[sd]), b2 = T(p[2 * sd]);
      if (IREC == 6) q[v] = mp5_state(a2, a1, u0, b1, b2, side ? T(-1) : T(1));
      else if (IREC == 8) {
        // mpweno5: WENO5-JS limited by MP5's bounds (rec.f90:2645-3158).  Its
        // radial right state reads uri(n,i-11,j,k) for uri(n,i-1,j,k) in beta_1
        // (rec.f90:2757); Fortran addresses it in the column-major array, so
        // below i = 1 it is cell (imax + i - 11, j - 1, k).
        T b1s = b1;
        if (D == 1 && side == 1) {
          const int f = i + 1;
          const size_t ct = (f - 11 >= 1) ? r.cell(f - 11, j, k) : r.cell(r.imax + f - 11, j - 1, k);
          b1s = T(P[(size_t)v * N + ct]);
        }
        q[v] = mp_limit(weno5_js(a2, a1, u0, b1, b2, b1s), a2, a1, u0, b1, b2, side ? T(-1) : T(1));
      } else if (IREC == 9) q[v] = weno5z_state(a2, a1, u0, b1, b2);
      else if (IREC == 10) q[v] = weno5m_state(a2, a1, u0, b1, b2);
      else q[v] = weno5_state(a2, a1, u0, b1, b2);
    }
  }
  if ((r.guard & 1) && !(q[0] > T(0) && q[4] > T(0))) {
#pragma unroll
    for (int v = 0; v < 9; ++v) q[v] = T(Pv[(size_t)v * Nv + cv + side * sv]);
  }
  MetT<T> m;
  if (VIEW && Mv) load_met<T, S, false>(Mv, (size_t)Mst, 0, m);  // the face metric staged with the stencil
  else load_met(met_of<D, S>(r), r.nik, r.ik(i, k), m);
  const T gam = T(r.gam);
  T u[9], w[9], vp, vm;
  {
    PST<T> s;
    pstate(q, m, gam, s);
    const T sr = ent_ratio(s, gam, r.gkind);
    p2c(s, gam, m.detg, u, sr);
    flux<D>(s, gam, m.detg, w, sr);
    wavespeed<D>(q, s, m, gam, vp, vm);
  }
  if constexpr (OUT) {
    if (valid) {
#pragma unroll
      for (int v = 0; v < 9; ++v) {
        fo->q[side][(size_t)v * N + c] = double(q[v]);
        fo->u[side][(size_t)v * N + c] = double(u[v]);
        fo->w[side][(size_t)v * N + c] = double(w[v]);
      }
    }
  }
  const T vpo = __shfl_xor_sync(mask, vp, 1), vmo = __shfl_xor_sync(mask, vm, 1);
  const T vpL = side ? vpo : vp, vpR = side ? vp : vpo;
  const T vmL = side ? vmo : vm, vmR = side ? vm : vmo;
  // calcha.f90:96-120 (cmink uses the R-state plus speed, calcha.f90:107)
  const T cmax = fmax3(T(0), vpR, vpL);
  const T cmin = (D == 3) ? fmin3(T(0), vpR, vmL) : fmin3(T(0), vmR, vmL);
  const bool copy = Fcopy != nullptr && i <= icopy;
  // hll.f90:83-183
#pragma unroll
  for (int v = 0; v < 9; ++v) {
    const T uo = __shfl_xor_sync(mask, u[v], 1), wo = __shfl_xor_sync(mask, w[v], 1);
    if (!valid || (v & 1) != side) continue;
    const T uL = side ? uo : u[v], uR = side ? u[v] : uo;
    const T wL = side ? wo : w[v], wR = side ? w[v] : wo;
    T f;
    if (cmin > T(0)) f = wL;
    else if (cmin <= T(0) && cmax > T(0)) {
      const T c1 = dmax2(mabs(cmax), mabs(cmin));
      f = T(0.5) * (wL + wR - c1 * (uR - uL));
    } else if (cmax <= T(0)) f = wR;
    else continue;  // NaN speeds: the reference keeps the previous ww
    if (mabs(f) < T(1.0e-40)) f = T(0);
    if ((r.guard & 2) && v == 5 + D) f = T(0);  // Toth: no flux of the normal field component
    F[(size_t)v * N + c] = S(f);
    if (copy) Fcopy[(size_t)v * N + c] = float(f);
  }
}

// Resident blocks of 128 threads per SM the FP64 face kernel is compiled for
// (registers per thread <= 65536 / (128 * blocks), in steps of 8).
#ifndef RG_FLUX_MINB64
#define RG_FLUX_MINB64 5
#endif

// Faces with radial index i in [ilo, ihi] (and the hll range in j, k) in
// arithmetic type T on storage S.  The FP64 path launches it once over the
// whole range; the mixed path launches FP64 for r < 2 r_H (faces i <=
// i_fp64 + 1, copied to FP32 up to i_fp64) and FP32 beyond.
template <int D, int IREC, typename T, typename S>
__device__ __forceinline__ void flux_body(const DevRun& r, const S* __restrict__ P, S* __restrict__ F,
                                              float* __restrict__ Fcopy, int icopy, int ilo, int ihi, const uint3 bid) {
  if (!r.scal->active) return;
  const int nm0 = r.nm0;
  const int side = threadIdx.x & 1;
  const int i0 = (int)((bid.x * blockDim.x + threadIdx.x) >> 1) + ilo;
  const int j0 = jidx(r, nm0, bid);
  const int k0 = kidx(r, nm0, bid);
  const bool valid = i0 <= ihi && j0 <= r.jmax - nm0 && k0 <= r.kmax - nm0;
  const int i = min(i0, ihi), j = min(j0, r.jmax - nm0), k = min(k0, r.kmax - nm0);
  face_lane<D, IREC, T, S>(r, P, F, Fcopy, icopy, i, j, k, side, valid);
}
template <int D, int IREC, typename T, typename S>
__global__ void __launch_bounds__(128, sizeof(T) == 8 ? RG_FLUX_MINB64 : 8) k_flux(DevRun r, const S* __restrict__ P, S* __restrict__ F,
                                              float* __restrict__ Fcopy, int icopy, int ilo, int ihi) { flux_body<D, IREC, T, S>(r, P, F, Fcopy, icopy, ilo, ihi, blockIdx); }

// The face kernel (PPM, MP5, WENO5, WENO-Z, WENO-M) with its stencil staged in shared memory by one TMA
// tile load per block (cp.async.bulk.tensor, this GPU's own buffer, no
// multicast), in FP64 (S = double) or for the FP32 half of the mixed path
// (S = float, over P32).  A block takes the same 32 x 2 faces as k_flux (32
// along i, two rows along j, one k); the tensor map views the primitives as
// the 4D array (i, j, k, v) and the box covers the block's stencil for all
// nine variables: 40 x 2 x 1 cells for r faces (i-2 .. i+3 of 32 faces), X x
// 7 x 1 for phi faces (two rows, j-2 .. j+3 each), X x 2 x 6 for theta faces,
// with X = 34 (FP64) or 36 (FP32).  The box starts on a 16-byte boundary
// along i (the TMA's rule): its origin is rounded down to an even (FP64) or
// a multiple-of-four (FP32) index and the view offsets the lanes by the
// remainder.  Cells past the array read as zeros (the TMA's out-of-bounds
// fill); only lanes working on a clamped face could reach them, and those
// store nothing.  The wait on the transaction barrier is bounded: if the copy
// has not landed after kTmaWaitCap polls or kTmaWaitNs of the global timer,
// the block counts C_TMAWAIT, waits once more (bounded) for the copy and
// returns without computing; the host reports RG_ECUDA.  A block still
// waiting after 1024 polls also gives up once the run's count is set, so a
// launch whose copies never land ends after about one timed-out wave.  (The
// count is read only there: the normal path issues its copy at once.)
constexpr int kTmaWaitCap = 1 << 22;
constexpr unsigned long long kTmaWaitNs = 50000000ull;  // 50 ms

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// LO: cells a face's state reads beyond its owner cell on either side (2
// for the five-point schemes; 3 for PPM, whose flattening reads the pressure
// three cells out), so the faces f of a block need cells f-LO .. f+1+LO.
template <int D, typename S, int LO>
struct TmaBox {
  static constexpr int ALIGN = 16 / (int)sizeof(S);  // elements per 16 bytes
  __host__ __device__ static constexpr int up(int n) { return (n + ALIGN - 1) / ALIGN * ALIGN; }
  // along D: 32 faces + 2 LO + 1 cells, plus the alignment slack; across: 32 faces plus slack
  static constexpr int X = (D == 1) ? up(33 + 2 * LO + ALIGN - 1) : up(32 + ALIGN - 1);
  static constexpr int Y = (D == 2) ? 2 + 2 * LO + 1 : 2;
  static constexpr int Z = (D == 3) ? 1 + 2 * LO + 1 : 1;
  static constexpr int PLANE = X * Y * Z;                                   // cells per variable
  static constexpr unsigned BYTES = (unsigned)PLANE * 9u * (unsigned)sizeof(S);  // whole box
  // FP64 runs also stage the face metric of the block's faces (MetT's
  // components at each face's (i, k) point): MX points along i from the
  // block's first face rounded down to 16 bytes, one k, kMetComps components,
  // placed after the stencil box at MOFF -- where five blocks per SM still fit
  // (at most 45 KB each; PPM's theta box leaves no room and reads the metric
  // through L1)
  static constexpr int MX = up(32 + ALIGN - 1);
  static constexpr unsigned MOFF = (BYTES + 127u) / 128u * 128u;
  static constexpr unsigned MSIZE = (unsigned)MX * (unsigned)kMetComps * (unsigned)sizeof(S);
  static constexpr bool MET = sizeof(S) == 8 && MOFF + MSIZE <= 45u * 1024u;
  static constexpr unsigned MBYTES = MET ? MSIZE : 0u;
  static constexpr unsigned SMEM = MET ? MOFF + MBYTES : BYTES;
};
template <int IREC>
__host__ __device__ constexpr int tma_lo() { return IREC == 5 ? 3 : 2; }

// abandon: the run's C_TMAWAIT counter (nullptr: wait the full bound).  The
// polls run in rounds of 1024, so the clock and the counter are read only by a
// block that has waited a whole round.
__device__ __forceinline__ bool tma_wait(unsigned bar, const unsigned long long* abandon) {
  unsigned done = 0;
  unsigned long long t0 = 0;
  for (int round = 0; round < kTmaWaitCap / 1024; ++round) {
    for (int it = 0; it < 1024 && !done; ++it)
      asm volatile(
          "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
          : "=r"(done)
          : "r"(bar), "r"(0)
          : "memory");
    if (done) break;
    if (abandon && *reinterpret_cast<volatile const unsigned long long*>(abandon) != 0ull) break;
    const unsigned long long t = global_ns();
    if (t0 == 0) t0 = t;
    else if (t - t0 > kTmaWaitNs) break;
  }
  return done != 0;
}

template <int D, int IREC, typename T, typename S>
__global__ void __launch_bounds__(128, sizeof(T) == 8 ? RG_FLUX_MINB64 : 8)
    k_flux_tma(const __grid_constant__ CUtensorMap tm, const __grid_constant__ CUtensorMap tmm, DevRun r,
               S* __restrict__ F, float* __restrict__ Fcopy, int icopy, int ilo, int ihi) {
  extern __shared__ __align__(128) unsigned char box_raw[];
  __shared__ __align__(8) unsigned long long bar;
  if (!r.scal->active) return;
  using B = TmaBox<D, S, tma_lo<IREC>()>;
  S* box = reinterpret_cast<S*>(box_raw);
  const int nm0 = r.nm0;
  const int fi0 = ilo + (int)blockIdx.x * 32, fj0 = nm0 + 2 * (int)blockIdx.y, fk0 = nm0 + (int)blockIdx.z;
  // 0-based origin of the box: the first stencil cell along D, the block's
  // first face elsewhere; along i rounded down to a 16-byte boundary
  constexpr int LO = tma_lo<IREC>();
  const int x0 = ((D == 1) ? fi0 - 1 - LO : fi0 - 1) & ~(B::ALIGN - 1);
  const int y0 = (D == 2) ? fj0 - 1 - LO : fj0 - 1;
  const int z0 = (D == 3) ? fk0 - 1 - LO : fk0 - 1;
  const int mx0 = (fi0 - 1) & ~(B::ALIGN - 1);  // first metric point (0-based i) of the metric box
  const unsigned bar_a = (unsigned)__cvta_generic_to_shared(&bar);
  const unsigned box_a = (unsigned)__cvta_generic_to_shared(box_raw);
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a), "r"(B::BYTES + B::MBYTES)
                 : "memory");
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];" ::"r"(box_a),
        "l"(reinterpret_cast<unsigned long long>(&tm)), "r"(x0), "r"(y0), "r"(z0), "r"(0), "r"(bar_a)
        : "memory");
    if (B::MET)
      asm volatile(
          "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
          "%4}], [%5];" ::"r"(box_a + B::MOFF),
          "l"(reinterpret_cast<unsigned long long>(&tmm)), "r"(mx0), "r"(fk0 - 1), "r"(0), "r"(bar_a)
          : "memory");
  }
  __syncthreads();
  if (!tma_wait(bar_a, r.cnt + C_TMAWAIT)) {
    if (tid == 0) atomicAdd(r.cnt + C_TMAWAIT, 1ull);
    tma_wait(bar_a, nullptr);  // the copy in flight writes this block's shared memory: give it one more bounded wait
    return;
  }
  const int side = threadIdx.x & 1;
  const int i0 = fi0 + (int)(threadIdx.x >> 1), j0 = fj0 + (int)threadIdx.y;
  const bool valid = i0 <= ihi && j0 <= r.jmax - nm0 && fk0 <= r.kmax - nm0;
  const int i = min(i0, ihi), j = min(j0, r.jmax - nm0), k = min(fk0, r.kmax - nm0);
  const size_t vc = (size_t)((i - 1 - x0) + B::X * ((j - 1 - y0) + B::Y * (k - 1 - z0)));
  const long long vst = (D == 1) ? 1 : (D == 2 ? B::X : B::X * B::Y);
  const S* met = B::MET ? reinterpret_cast<const S*>(box_raw + B::MOFF) + (i - 1 - mx0) : nullptr;
  face_lane<D, IREC, T, S, true>(r, nullptr, F, Fcopy, icopy, i, j, k, side, valid, box, B::PLANE, vc, vst, nullptr,
                                 met, B::MX);
}

// ------------------------------------------------ TMA-staged stage update
// k_update with the rows its RK combine reads staged in shared memory: a
// block of BX cells along i, BY rows along j and one k issues, when it
// starts, one 4D tile load (cp.async.bulk.tensor, this GPU's own buffers, no
// multicast) per array -- the three face-flux arrays, the flux-CT components
// and, in stages 2 and 3, U^n -- each box covering the block's cells and the
// lower neighbours the flux differences need (i-1 for F1 and CT, j-1 for F2
// and CT, k-1 for F3 and CT).  While the copies travel the threads load the
// metric, compute P2C of the stage input and the geometric source
// (stage_pre); they then wait on the transaction barrier (bounded, as in
// k_flux_tma) and take the flux differences from shared memory.  The values
// and the operations are those of k_update.  The box origins along i are
// even (16-byte aligned in FP64): the F1 and CT boxes start two cells before
// the block, the others at its first cell; cells before index 0 or past the
// array read as zeros and are never used.
template <int BX, int BY>
struct UpdBox {
  // (x, y, z) extents per array; variables are the 4th dimension
  static constexpr int X1 = BX + 2, Y1 = BY, Z1 = 1;      // F1: i-2 .. i+BX-1
  static constexpr int X2 = BX, Y2 = BY + 1, Z2 = 1;      // F2: rows j-1 .. j+BY-1
  static constexpr int X3 = BX, Y3 = BY, Z3 = 2;          // F3: planes k-1, k
  static constexpr int XC = BX + 2, YC = BY + 1, ZC = 2;  // CT: all three neighbours
  static constexpr int XU = BX, YU = BY, ZU = 1;          // U^n
  static constexpr unsigned up128(unsigned n) { return (n + 127u) / 128u * 128u; }
  static constexpr unsigned B1 = X1 * Y1 * Z1 * 9 * 8, B2 = X2 * Y2 * Z2 * 9 * 8, B3 = X3 * Y3 * Z3 * 9 * 8;
  static constexpr unsigned BC = XC * YC * ZC * 6 * 8, BU = XU * YU * ZU * 9 * 8;
  static constexpr unsigned O1 = 0, O2 = up128(O1 + B1), O3 = up128(O2 + B2), OC = up128(O3 + B3),
                            OU = up128(OC + BC), BYTES = up128(OU + BU);
};
using UpdB = UpdBox<RG_UPDATE_BX, 128 / RG_UPDATE_BX>;

// The five tensor maps of a run's update (F1, F2, F3, CT, U^n).
struct UpdMaps {
  CUtensorMap m[5];
};

__device__ __forceinline__ void tma_load4(unsigned dst, const CUtensorMap* tm, int x, int y, int z, unsigned bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
      "%5}], [%6];" ::"r"(dst),
      "l"(reinterpret_cast<unsigned long long>(tm)), "r"(x), "r"(y), "r"(z), "r"(0), "r"(bar)
      : "memory");
}

// Flux differences from the staged rows of one thread's cell (pointers at the
// cell in each box; neighbours one element, one row or one plane back).
struct FluxDiffStaged {
  const double* f1;
  const double* f2;
  const double* f3;
  const double* ct;
  __device__ __forceinline__ void operator()(int v, double& d1, double& d2, double& d3) const {
    using B = UpdB;
    constexpr int P1 = B::X1 * B::Y1 * B::Z1, P2 = B::X2 * B::Y2 * B::Z2, P3 = B::X3 * B::Y3 * B::Z3;
    constexpr int PC = B::XC * B::YC * B::ZC, SJC = B::XC, SKC = B::XC * B::YC, SK3 = B::X3 * B::Y3;
    if (v == 7) d1 = ct[2 * PC] - ct[2 * PC - 1];
    else if (v == 8) d1 = ct[4 * PC] - ct[4 * PC - 1];
    else d1 = f1[v * P1] - f1[v * P1 - 1];
    if (v == 6) d2 = ct[0 * PC] - ct[0 * PC - SJC];
    else if (v == 8) d2 = ct[5 * PC] - ct[5 * PC - SJC];
    else d2 = f2[v * P2] - f2[v * P2 - B::X2];
    if (v == 6) d3 = ct[1 * PC] - ct[1 * PC - SKC];
    else if (v == 7) d3 = ct[3 * PC] - ct[3 * PC - SKC];
    else d3 = f3[v * P3] - f3[v * P3 - SK3];
  }
};

template <int STAGE>
__global__ void __launch_bounds__(128, RG_UPDATE_MINB)
    k_update_tma(const __grid_constant__ UpdMaps tm, DevRun r, const double* __restrict__ Pc, double* __restrict__ Pw) {
  using B = UpdB;
  extern __shared__ __align__(128) unsigned char upd_raw[];
  __shared__ __align__(8) unsigned long long bar;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + RG_UPDATE_BX * ty;
  const int x0 = (int)blockIdx.x * RG_UPDATE_BX, y0 = (int)blockIdx.y * (128 / RG_UPDATE_BX), z0 = (int)blockIdx.z;
  const int i = x0 + tx + 1, j = y0 + ty + 1, k = z0 + 1;
  const bool inr = i <= r.imax && j <= r.jmax && k <= r.kmax;
  const size_t N = r.N, c = inr ? r.cell(i, j, k) : 0;
  if (!r.scal->active) {  // a finished run copies its state through (as k_update)
    if (inr)
#pragma unroll
      for (int v = 0; v < 9; ++v) Pw[(size_t)v * N + c] = Pc[(size_t)v * N + c];
    return;
  }
  const unsigned bar_a = (unsigned)__cvta_generic_to_shared(&bar);
  const unsigned base = (unsigned)__cvta_generic_to_shared(upd_raw);
  if (tid == 0) {
    const unsigned bytes = B::B1 + B::B2 + B::B3 + B::BC + (STAGE > 1 ? B::BU : 0u);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a), "r"(bytes) : "memory");
    tma_load4(base + B::O1, &tm.m[0], x0 - 2, y0, z0, bar_a);
    tma_load4(base + B::O2, &tm.m[1], x0, y0 - 1, z0, bar_a);
    tma_load4(base + B::O3, &tm.m[2], x0, y0, z0 - 1, bar_a);
    tma_load4(base + B::OC, &tm.m[3], x0 - 2, y0 - 1, z0 - 1, bar_a);
    if (STAGE > 1) tma_load4(base + B::OU, &tm.m[4], x0, y0, z0, bar_a);
  }
  __syncthreads();
  const bool interior = inr && is_interior(r, i, j, k);
  if (inr && !interior)
#pragma unroll
    for (int v = 0; v < 9; ++v) Pw[(size_t)v * N + c] = Pc[(size_t)v * N + c];
  Met m;
  double ucur[9], sf[4];
  if (interior) {
    load_met(r.mc, r.nik, r.ik(i, k), m);
    stage_pre<STAGE>(r, i, j, k, m, Pc, ucur, sf);
  }
  if (!tma_wait(bar_a, r.cnt + C_TMAWAIT)) {
    if (tid == 0) atomicAdd(r.cnt + C_TMAWAIT, 1ull);
    tma_wait(bar_a, nullptr);  // the copies in flight write this block's shared memory: one more bounded wait
    return;
  }
  if (!interior) return;
  const double* sm = reinterpret_cast<const double*>(upd_raw);
  const FluxDiffStaged diff{sm + B::O1 / 8 + (tx + 2) + B::X1 * ty,
                            sm + B::O2 / 8 + tx + B::X2 * (ty + 1),
                            sm + B::O3 / 8 + tx + B::X3 * ty + B::X3 * B::Y3,
                            sm + B::OC / 8 + (tx + 2) + B::XC * (ty + 1) + B::XC * B::YC};
  double uo[9];
  if (STAGE > 1) {
    const double* un = sm + B::OU / 8 + tx + B::XU * ty;
#pragma unroll
    for (int v = 0; v < 9; ++v) uo[v] = un[v * B::XU * B::YU];
  }
  double u[9];
  stage_combine<STAGE>(r, i, j, k, ucur, sf, uo, r.scal->dt, diff, u);
  update_recov(r, i, j, k, m, Pc, Pw, u);
}

// The same staging for the FP32 region of a mixed run (cells i >= ilo, the
// first cell beyond r = 2 r_H): FP32 face fluxes and flux-CT values, FP64 U^n.
// The region starts at any i, so each box starts at the 16-byte boundary at
// or below its first cell (a multiple of 4 cells in FP32, of 2 in FP64) and
// a thread's cell sits `off` cells into it.
constexpr unsigned round_up128(unsigned n) { return (n + 127u) / 128u * 128u; }
struct UpdBoxMix {
  static constexpr int BX = RG_UPDATE_BX, BY = 128 / RG_UPDATE_BX;
  static constexpr int X1 = BX + 4, Y1 = BY, Z1 = 1;      // F1 (FP32): from i0-1 rounded down to 4
  static constexpr int X2 = BX + 4, Y2 = BY + 1, Z2 = 1;  // F2 (FP32): from i0 rounded down
  static constexpr int X3 = BX + 4, Y3 = BY, Z3 = 2;      // F3 (FP32)
  static constexpr int XC = BX + 4, YC = BY + 1, ZC = 2;  // CT (FP32): from i0-1 rounded down
  static constexpr int XU = BX + 2, YU = BY, ZU = 1;      // U^n (FP64): from i0 rounded down to 2
  static constexpr unsigned B1 = X1 * Y1 * Z1 * 9 * 4, B2 = X2 * Y2 * Z2 * 9 * 4, B3 = X3 * Y3 * Z3 * 9 * 4;
  static constexpr unsigned BC = XC * YC * ZC * 6 * 4, BU = XU * YU * ZU * 9 * 8;
  static constexpr unsigned O1 = 0, O2 = round_up128(O1 + B1), O3 = round_up128(O2 + B2),
                            OC = round_up128(O3 + B3), OU = round_up128(OC + BC), BYTES = round_up128(OU + BU);
};

struct FluxDiffStaged32 {
  const float* f1;
  const float* f2;
  const float* f3;
  const float* ct;
  __device__ __forceinline__ void operator()(int v, float& d1, float& d2, float& d3) const {
    using B = UpdBoxMix;
    constexpr int P1 = B::X1 * B::Y1 * B::Z1, P2 = B::X2 * B::Y2 * B::Z2, P3 = B::X3 * B::Y3 * B::Z3;
    constexpr int PC = B::XC * B::YC * B::ZC, SJC = B::XC, SKC = B::XC * B::YC, SK3 = B::X3 * B::Y3;
    if (v == 7) d1 = ct[2 * PC] - ct[2 * PC - 1];
    else if (v == 8) d1 = ct[4 * PC] - ct[4 * PC - 1];
    else d1 = f1[v * P1] - f1[v * P1 - 1];
    if (v == 6) d2 = ct[0 * PC] - ct[0 * PC - SJC];
    else if (v == 8) d2 = ct[5 * PC] - ct[5 * PC - SJC];
    else d2 = f2[v * P2] - f2[v * P2 - B::X2];
    if (v == 6) d3 = ct[1 * PC] - ct[1 * PC - SKC];
    else if (v == 7) d3 = ct[3 * PC] - ct[3 * PC - SKC];
    else d3 = f3[v * P3] - f3[v * P3 - SK3];
  }
};

template <int STAGE>
__global__ void __launch_bounds__(128, RG_UPDATE_MINB)
    k_update_tma_mix(const __grid_constant__ UpdMaps tm, DevRun r, const double* __restrict__ Pc,
                     double* __restrict__ Pw, int ilo) {
  using B = UpdBoxMix;
  extern __shared__ __align__(128) unsigned char upd_raw[];
  __shared__ __align__(8) unsigned long long bar;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + B::BX * ty;
  const int i0 = ilo + (int)blockIdx.x * B::BX, y0 = (int)blockIdx.y * B::BY, z0 = (int)blockIdx.z;
  const int i = i0 + tx, j = y0 + ty + 1, k = z0 + 1;
  const bool inr = i <= r.imax && j <= r.jmax && k <= r.kmax;
  const size_t N = r.N, c = inr ? r.cell(i, j, k) : 0;
  if (!r.scal->active) {  // a finished run copies its state through (as k_update)
    if (inr)
#pragma unroll
      for (int v = 0; v < 9; ++v) Pw[(size_t)v * N + c] = Pc[(size_t)v * N + c];
    return;
  }
  // 0-based box origins along i: F1 and CT start at or below cell i0-1, the others at or below i0
  const int xa = (i0 - 2) & ~3, xb = (i0 - 1) & ~3, xu = (i0 - 1) & ~1;
  const unsigned bar_a = (unsigned)__cvta_generic_to_shared(&bar);
  const unsigned base = (unsigned)__cvta_generic_to_shared(upd_raw);
  if (tid == 0) {
    const unsigned bytes = B::B1 + B::B2 + B::B3 + B::BC + (STAGE > 1 ? B::BU : 0u);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a), "r"(bytes) : "memory");
    tma_load4(base + B::O1, &tm.m[0], xa, y0, z0, bar_a);
    tma_load4(base + B::O2, &tm.m[1], xb, y0 - 1, z0, bar_a);
    tma_load4(base + B::O3, &tm.m[2], xb, y0, z0 - 1, bar_a);
    tma_load4(base + B::OC, &tm.m[3], xa, y0 - 1, z0 - 1, bar_a);
    if (STAGE > 1) tma_load4(base + B::OU, &tm.m[4], xu, y0, z0, bar_a);
  }
  __syncthreads();
  const bool interior = inr && is_interior(r, i, j, k);
  if (inr && !interior)
#pragma unroll
    for (int v = 0; v < 9; ++v) Pw[(size_t)v * N + c] = Pc[(size_t)v * N + c];
  Met m;
  double ucur[9];
  float sf[4];
  if (interior) {
    load_met(r.mc, r.nik, r.ik(i, k), m);
    stage_pre_mixed<STAGE>(r, i, j, k, m, Pc, ucur, sf);
  }
  if (!tma_wait(bar_a, r.cnt + C_TMAWAIT)) {
    if (tid == 0) atomicAdd(r.cnt + C_TMAWAIT, 1ull);
    tma_wait(bar_a, nullptr);  // the copies in flight write this block's shared memory: one more bounded wait
    return;
  }
  if (!interior) return;
  const float* sm = reinterpret_cast<const float*>(upd_raw);
  const int oa = (i - 1) - xa, ob = (i - 1) - xb;  // the cell's index along i in each box
  const FluxDiffStaged32 diff{sm + B::O1 / 4 + oa + B::X1 * ty,
                              sm + B::O2 / 4 + ob + B::X2 * (ty + 1),
                              sm + B::O3 / 4 + ob + B::X3 * ty + B::X3 * B::Y3,
                              sm + B::OC / 4 + oa + B::XC * (ty + 1) + B::XC * B::YC};
  double uo[9];
  if (STAGE > 1) {
    const double* un = reinterpret_cast<const double*>(upd_raw + B::OU) + ((i - 1) - xu) + B::XU * ty;
#pragma unroll
    for (int v = 0; v < 9; ++v) uo[v] = un[v * B::XU * B::YU];
  }
  double u[9];
  stage_combine_mixed<STAGE>(r, i, j, k, ucur, sf, uo, r.scal->dt, diff, u);
  update_recov(r, i, j, k, m, Pc, Pw, u);
}

// ------------------------------------------- per-routine rec2 / calcha / hll
// rec2 with caluu3 and calflx3 (rec.f90:2-142) for one direction: the face
// lanes of k_flux with their states, conserved variables and fluxes stored
// (FaceOut); the LLF fluxes go to F, which the caller discards.
template <int D, int IREC>
__global__ void __launch_bounds__(128, RG_FLUX_MINB64) k_rec2(DevRun r, const double* __restrict__ P,
                                                             double* __restrict__ F, FaceOut fo) {
  const int nm0 = r.nm0, ilo = nm0, ihi = r.imax - nm0;
  const int side = threadIdx.x & 1;
  const int i0 = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 1) + ilo;
  const int j0 = jidx(r, nm0, blockIdx);
  const int k0 = kidx(r, nm0, blockIdx);
  const bool valid = i0 <= ihi && j0 <= r.jmax - nm0 && k0 <= r.kmax - nm0;
  const int i = min(i0, ihi), j = min(j0, r.jmax - nm0), k = min(k0, r.kmax - nm0);
  face_lane<D, IREC, double, double, false, true>(r, P, F, nullptr, 0, i, j, k, side, valid, nullptr, 0, 0, 0, &fo);
}

// calcha (calcha.f90:2-126, with cmink built from the R state's plus speed,
// calcha.f90:107) from given face primitives QL (uri?l) and QR (uri?r) of
// direction D, over the hll range nm0..n-nm0.
template <int D>
__global__ void __launch_bounds__(128) k_calcha(DevRun r, const double* __restrict__ QL, const double* __restrict__ QR,
                                                double* __restrict__ cmax, double* __restrict__ cmin) {
  const int nm0 = r.nm0;
  const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x) + nm0;
  const int j = (int)(blockIdx.y * blockDim.y + threadIdx.y) + nm0;
  const int k = (int)(blockIdx.z * blockDim.z + threadIdx.z) + nm0;
  if (i > r.imax - nm0 || j > r.jmax - nm0 || k > r.kmax - nm0) return;
  const size_t N = r.N, c = r.cell(i, j, k);
  Met m;
  load_met(met_of<D, double>(r), r.nik, r.ik(i, k), m);
  double qL[9], qR[9], vpL, vmL, vpR, vmR;
  load9(QL, N, c, qL);
  load9(QR, N, c, qR);
  {
    PS s;
    pstate(qL, m, r.gam, s);
    wavespeed<D>(qL, s, m, r.gam, vpL, vmL);
  }
  {
    PS s;
    pstate(qR, m, r.gam, s);
    wavespeed<D>(qR, s, m, r.gam, vpR, vmR);
  }
  cmax[c] = fmax3(0.0, vpR, vpL);
  cmin[c] = (D == 3) ? fmin3(0.0, vpR, vmL) : fmin3(0.0, vmR, vmL);
}

// hll (hll.f90:83-183) for direction D from given face conserved variables,
// face fluxes and speeds: the fluxes F of the hll range, in place (a face with
// NaN speeds keeps its value, as the reference's ww does).
template <int D>
__global__ void __launch_bounds__(128) k_hll(DevRun r, const double* __restrict__ UL, const double* __restrict__ UR,
                                             const double* __restrict__ WL, const double* __restrict__ WR,
                                             const double* __restrict__ CX, const double* __restrict__ CN,
                                             double* __restrict__ F) {
  const int nm0 = r.nm0;
  const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x) + nm0;
  const int j = (int)(blockIdx.y * blockDim.y + threadIdx.y) + nm0;
  const int k = (int)(blockIdx.z * blockDim.z + threadIdx.z) + nm0;
  if (i > r.imax - nm0 || j > r.jmax - nm0 || k > r.kmax - nm0) return;
  const size_t N = r.N, c = r.cell(i, j, k);
  const double cmin = CN[c], cmax = CX[c];
#pragma unroll
  for (int v = 0; v < 9; ++v) {
    const size_t o = (size_t)v * N + c;
    double f;
    if (cmin > 0.0) f = WL[o];
    else if (cmin <= 0.0 && cmax > 0.0) {
      const double c1 = dmax2(fabs(cmax), fabs(cmin));
      f = 0.5 * (WL[o] + WR[o] - c1 * (UR[o] - UL[o]));
    } else if (cmax <= 0.0) f = WR[o];
    else continue;
    if (fabs(f) < 1.0e-40) f = 0.0;
    F[o] = f;
  }
}

// ww(3,nv,i,j,k) of the reference (direction fastest) <-> the three flux
// planes F[d][v*N + c] of the full layout.
__global__ void k_ww_layout(double* __restrict__ ww, double* __restrict__ F1, double* __restrict__ F2,
                            double* __restrict__ F3, size_t N, int to_planes) {
  const size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  double* F[3] = {F1, F2, F3};
#pragma unroll
  for (int v = 0; v < 9; ++v)
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      double& a = ww[d + 3 * (v + 9 * c)];
      double& b = F[d][(size_t)v * N + c];
      if (to_planes) b = a;
      else a = b;
    }
}

// ct's results into the flux planes: with guard bit 2 the normal-field
// fluxes ww(1,7), ww(2,8), ww(3,9) are zero on the hll range (the oracle's ct
// does that first); the six CT values replace the transverse induction fluxes
// on the CT range nm1..n-nm1 (ct.f90:98-109).
__global__ void k_ct_apply(DevRun r, const double* __restrict__ CT, double* __restrict__ F1, double* __restrict__ F2,
                           double* __restrict__ F3) {
  const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x) + 1;
  const int j = (int)(blockIdx.y * blockDim.y + threadIdx.y) + 1;
  const int k = (int)(blockIdx.z * blockDim.z + threadIdx.z) + 1;
  if (i > r.imax || j > r.jmax || k > r.kmax) return;
  const size_t N = r.N, c = r.cell(i, j, k);
  const int nm0 = r.nm0, nm1 = r.nm1;
  double* F[3] = {F1, F2, F3};
  if ((r.guard & 2) && i >= nm0 && i <= r.imax - nm0 && j >= nm0 && j <= r.jmax - nm0 && k >= nm0 &&
      k <= r.kmax - nm0)
#pragma unroll
    for (int d = 0; d < 3; ++d) F[d][(size_t)(6 + d) * N + c] = 0.0;
  if (r.ict == 0 || i < nm1 || i > r.imax - nm1 || j < nm1 || j > r.jmax - nm1 || k < nm1 || k > r.kmax - nm1) return;
  // (direction, variable) of the six replaced fluxes: ww(2,7) ww(3,7) ww(1,8) ww(3,8) ww(1,9) ww(2,9)
  const int dir[6] = {1, 2, 0, 2, 0, 1}, var[6] = {6, 6, 7, 7, 8, 8};
#pragma unroll
  for (int q = 0; q < 6; ++q) F[dir[q]][(size_t)var[q] * N + c] = CT[(size_t)q * N + c];
}

// ---------------------------------------------------------------- flux-CT
// ct.f90:30-118 (flux-CT, ict 1), ct.f90:121-233 (mflct, ict 2),
// ct.f90:236-445 (upflct, ict 3: its last level) or none (ict 0) on nm1..n-nm1 in every dimension (edges with i in [ilo, ihi]),
// in arithmetic type T on flux storage S.  CTcopy, if given, receives an FP32
// copy (the FP64 edges next to the FP32 region of the mixed path).
template <int ICT, typename T, typename S>
__device__ __forceinline__ void ct_body(const DevRun& r, const S* __restrict__ F1, const S* __restrict__ F2,
                                            const S* __restrict__ F3, S* __restrict__ CT,
                                            float* __restrict__ CTcopy, int ilo, int ihi, const uint3 bid) {
  if (!r.scal->active) return;
  const int nm1 = r.nm1;
  const int i = bid.x * blockDim.x + threadIdx.x + ilo;
  const int j = jidx(r, nm1, bid);
  const int k = kidx(r, nm1, bid);
  if (i > ihi || j > r.jmax - nm1 || k > r.kmax - nm1) return;
  const size_t N = r.N, c = r.cell(i, j, k);
  const size_t di = 1, dj = r.sj, dk = r.sk;
  const S* fyx = F2 + 6 * N;  // ww(2,7)
  const S* fzx = F3 + 6 * N;  // ww(3,7)
  const S* fxy = F1 + 7 * N;  // ww(1,8)
  const S* fzy = F3 + 7 * N;  // ww(3,8)
  const S* fxz = F1 + 8 * N;  // ww(1,9)
  const S* fyz = F2 + 8 * N;  // ww(2,9)
  auto L = [](const S* a, size_t x) { return T(a[x]); };
  const T e = T(1.0) / T(8.0), two = T(2.0);
  T o[6];
  if constexpr (ICT == 0) {  // no constrained transport: the induction fluxes stay as hll left them
    o[0] = L(fyx, c); o[1] = L(fzx, c); o[2] = L(fxy, c); o[3] = L(fzy, c); o[4] = L(fxz, c); o[5] = L(fyz, c);
  } else if constexpr (ICT == 2) {
    // mflct (ct.f90:121-233): the cell-centred EMFs of its second pass
    // (ct.f90:174-176), evaluated where the corner formulas need them, and
    // the flux-CT brackets with weight 1/4 plus the averaged EMFs (ct.f90:191-224)
    const T q = T(0.25), h = T(1.0) / T(8.0);
    auto ez = [&](size_t x) { return q * (-L(fxy, x - di) - L(fxy, x) + L(fyx, x - dj) + L(fyx, x)); };
    auto ex = [&](size_t x) { return q * (-L(fyz, x - dj) - L(fyz, x) + L(fzy, x - dk) + L(fzy, x)); };
    auto ey = [&](size_t x) { return q * (-L(fzx, x - dk) - L(fzx, x) + L(fxz, x - di) + L(fxz, x)); };
    const T fbyx = q * (two * L(fyx, c) + L(fyx, c + di) + L(fyx, c - di) - L(fxy, c) - L(fxy, c + dj) -
                        L(fxy, c - di) - L(fxy, c - di + dj));
    const T fbzx = q * (two * L(fzx, c) + L(fzx, c + di) + L(fzx, c - di) - L(fxz, c) - L(fxz, c + dk) -
                        L(fxz, c - di) - L(fxz, c - di + dk));
    const T fbxy = q * (two * L(fxy, c) + L(fxy, c + dj) + L(fxy, c - dj) - L(fyx, c) - L(fyx, c + di) -
                        L(fyx, c - dj) - L(fyx, c + di - dj));
    const T fbzy = q * (two * L(fzy, c) + L(fzy, c + dj) + L(fzy, c - dj) - L(fyz, c) - L(fyz, c + dk) -
                        L(fyz, c - dj) - L(fyz, c - dj + dk));
    const T fbxz = q * (two * L(fxz, c) + L(fxz, c + dk) + L(fxz, c - dk) - L(fzx, c) - L(fzx, c + di) -
                        L(fzx, c - dk) - L(fzx, c + di - dk));
    const T fbyz = q * (two * L(fyz, c) + L(fyz, c + dk) + L(fyz, c - dk) - L(fzy, c) - L(fzy, c + dj) -
                        L(fzy, c - dk) - L(fzy, c + dj - dk));
    const T fhyx = -(h * (two * ez(c) + two * ez(c + dj) + ez(c + di) + ez(c + di + dj) + ez(c - di) + ez(c - di + dj)));
    const T fhzx = h * (two * ey(c) + two * ey(c + dk) + ey(c + di) + ey(c + di + dk) + ey(c - di) + ey(c - di + dk));
    const T fhxy = h * (two * ez(c) + two * ez(c + di) + ez(c + dj) + ez(c + di + dj) + ez(c - dj) + ez(c + di - dj));
    const T fhzy = -(h * (two * ex(c) + two * ex(c + dk) + ex(c + dj) + ex(c + dj + dk) + ex(c - dj) + ex(c - dj + dk)));
    const T fhxz = -(h * (two * ey(c) + two * ey(c + di) + ey(c + dk) + ey(c + di + dk) + ey(c - dk) + ey(c + di - dk)));
    const T fhyz = h * (two * ex(c) + two * ex(c + dj) + ex(c + dk) + ex(c + dj + dk) + ex(c - dk) + ex(c + dj - dk));
    o[0] = fbyx + fhyx; o[1] = fbzx + fhzx; o[2] = fbxy + fhxy;
    o[3] = fbzy + fhzy; o[4] = fbxz + fhxz; o[5] = fbyz + fhyz;
  } else if constexpr (ICT == 3) {
    // upflct's corner EMFs (ct.f90:391-433) from the face-pair EMFs e?b,
    // evaluated here, and the upwinded differences of k_upct_diff
    const T q = T(0.25), h = T(0.5);
    const double* D = r.ctd;
    const double *dyez = D, *dxez = D + N, *dyex = D + 2 * N, *dzex = D + 3 * N, *dxey = D + 4 * N, *dzey = D + 5 * N;
    auto ezb = [&](size_t x) { return q * (L(fyx, x) + L(fyx, x + di) - L(fxy, x) - L(fxy, x + dj)); };
    auto exb = [&](size_t x) { return q * (L(fzy, x) + L(fzy, x + dj) - L(fyz, x) - L(fyz, x + dk)); };
    auto eyb = [&](size_t x) { return q * (L(fxz, x) + L(fxz, x + di) - L(fzx, x) - L(fzx, x + dj)); };
    const size_t im = c - di, jm = c - dj, km = c - dk, ip = c + di, jp = c + dj, kp = c + dk;
    const T ezh = ezb(c) + q * (L(dyez, c) - L(dyez, jp)) + q * (L(dxez, c) - L(dxez, ip));
    const T ezhmi = ezb(im) + q * (L(dyez, im) - L(dyez, im + dj)) + q * (L(dxez, im) - L(dxez, c));
    const T ezhmj = ezb(jm) + q * (L(dyez, jm) - L(dyez, c)) + q * (L(dxez, jm) - L(dxez, ip - dj));
    const T exh = exb(c) + q * (L(dyex, c) - L(dyex, jp)) + q * (L(dzex, c) - L(dzex, kp));
    const T exhmj = exb(jm) + q * (L(dyex, jm) - L(dyex, c)) + q * (L(dzex, jm) - L(dzex, jm + dk));
    const T exhmk = exb(km) + q * (L(dyex, km) - L(dyex, jp - dk)) + q * (L(dzex, km) - L(dzex, c));
    const T eyh = eyb(c) + q * (L(dxey, c) - L(dxey, ip)) + q * (L(dzey, c) - L(dzey, kp));
    const T eyhmi = eyb(im) + q * (L(dxey, im) - L(dxey, c)) + q * (L(dzey, im) - L(dzey, im + dk));
    const T eyhmk = eyb(km) + q * (L(dxey, km) - L(dxey, ip - dk)) + q * (L(dzey, km) - L(dzey, c));
    o[0] = h * (ezh + ezhmi);
    o[1] = h * (-eyh - eyhmi);
    o[2] = h * (-ezh - ezhmj);
    o[3] = h * (exh + exhmj);
    o[4] = h * (eyh + eyhmk);
    o[5] = h * (-exh - exhmk);
  } else {
  o[0] = e * (two * L(fyx, c) + L(fyx, c + di) + L(fyx, c - di) - L(fxy, c) - L(fxy, c + dj) - L(fxy, c - di) -
              L(fxy, c - di + dj));
  o[1] = e * (two * L(fzx, c) + L(fzx, c + di) + L(fzx, c - di) - L(fxz, c) - L(fxz, c + dk) - L(fxz, c - di) -
              L(fxz, c - di + dk));
  o[2] = e * (two * L(fxy, c) + L(fxy, c + dj) + L(fxy, c - dj) - L(fyx, c) - L(fyx, c + di) - L(fyx, c - dj) -
              L(fyx, c + di - dj));
  o[3] = e * (two * L(fzy, c) + L(fzy, c + dj) + L(fzy, c - dj) - L(fyz, c) - L(fyz, c + dk) - L(fyz, c - dj) -
              L(fyz, c - dj + dk));
  o[4] = e * (two * L(fxz, c) + L(fxz, c + dk) + L(fxz, c - dk) - L(fzx, c) - L(fzx, c + di) - L(fzx, c - dk) -
              L(fzx, c + di - dk));
  o[5] = e * (two * L(fyz, c) + L(fyz, c + dk) + L(fyz, c - dk) - L(fzy, c) - L(fzy, c + dj) - L(fzy, c - dk) -
              L(fzy, c + dj - dk));
  }
#pragma unroll
  for (int a = 0; a < 6; ++a) {
    CT[(size_t)a * N + c] = S(o[a]);
    if (CTcopy) CTcopy[(size_t)a * N + c] = float(o[a]);
  }
}
template <int ICT, typename T, typename S>
__global__ void __launch_bounds__(256) k_ct(DevRun r, const S* __restrict__ F1, const S* __restrict__ F2,
                                            const S* __restrict__ F3, S* __restrict__ CT,
                                            float* __restrict__ CTcopy, int ilo, int ihi) { ct_body<ICT, T, S>(r, F1, F2, F3, CT, CTcopy, ilo, ihi, blockIdx); }

// upflct's first two levels (ct.f90:300-389, ict 3) on nm0+1..n-nm0-2 in
// every dimension: the six upwinded EMF differences d?e? of each cell, from
// the cell-centred EMFs e?c and the 1/8 brackets fb?? at the cell and at its
// upper neighbour, both evaluated from the face fluxes where needed; the sign
// tests read the cell's velocity uri(2..4).  Every index is the
// reference's as written: each fb?? averages its own flux along the direction
// that is neither its face normal nor its field component, every test after
// dyez's falls back on uri(2) < 0, and dzey's negative-velocity branch
// subtracts eyc at the cell itself.  Written to r.ctd (six planes of N).
__global__ void __launch_bounds__(256) k_upct_diff(DevRun r, const double* __restrict__ P,
                                                   const double* __restrict__ F1, const double* __restrict__ F2,
                                                   const double* __restrict__ F3, int hi_i, int hi_j, int hi_k) {
  if (!r.scal->active) return;
  const int lo = r.nm0 + 1;
  const int i = blockIdx.x * blockDim.x + threadIdx.x + lo;
  const int j = jidx(r, lo, blockIdx);
  const int k = kidx(r, lo, blockIdx);
  if (i > hi_i || j > hi_j || k > hi_k) return;
  const size_t N = r.N, c = r.cell(i, j, k);
  const size_t di = 1, dj = r.sj, dk = r.sk;
  const double* fyx = F2 + 6 * N;
  const double* fzx = F3 + 6 * N;
  const double* fxy = F1 + 7 * N;
  const double* fzy = F3 + 7 * N;
  const double* fxz = F1 + 8 * N;
  const double* fyz = F2 + 8 * N;
  auto L = [](const double* a, size_t x) { return __ldg(a + x); };
  const double q = 0.25, e = 1.0 / 8.0, two = 2.0, h = 0.5;
  auto ezc = [&](size_t x) { return q * (-L(fxy, x - di) - L(fxy, x) + L(fyx, x - dj) + L(fyx, x)); };
  auto exc = [&](size_t x) { return q * (-L(fyz, x - dj) - L(fyz, x) + L(fzy, x - dk) + L(fzy, x)); };
  auto eyc = [&](size_t x) { return q * (-L(fzx, x - dk) - L(fzx, x) + L(fxz, x - di) + L(fxz, x)); };
  auto fbyx = [&](size_t x) {
    return e * (two * L(fyx, x) + L(fyx, x + dk) + L(fyx, x - dk) - L(fxy, x) - L(fxy, x + dj) - L(fxy, x - di) -
                L(fxy, x - di + dj));
  };
  auto fbzx = [&](size_t x) {
    return e * (two * L(fzx, x) + L(fzx, x + dj) + L(fzx, x - dj) - L(fxz, x) - L(fxz, x + dk) - L(fxz, x - di) -
                L(fxz, x - di + dk));
  };
  auto fbxy = [&](size_t x) {
    return e * (two * L(fxy, x) + L(fxy, x + dk) + L(fxy, x - dk) - L(fyx, x) - L(fyx, x + di) - L(fyx, x - dj) -
                L(fyx, x + di - dj));
  };
  auto fbzy = [&](size_t x) {
    return e * (two * L(fzy, x) + L(fzy, x + di) + L(fzy, x - di) - L(fyz, x) - L(fyz, x + dk) - L(fyz, x - dj) -
                L(fyz, x - dj + dk));
  };
  auto fbxz = [&](size_t x) {
    return e * (two * L(fxz, x) + L(fxz, x + dj) + L(fxz, x - dj) - L(fzx, x) - L(fzx, x + di) - L(fzx, x - dk) -
                L(fzx, x + di - dk));
  };
  auto fbyz = [&](size_t x) {
    return e * (two * L(fyz, x) + L(fyz, x + di) + L(fyz, x - di) - L(fzy, x) - L(fzy, x + dj) - L(fzy, x - dk) -
                L(fzy, x + dj - dk));
  };
  // a(c) - b(c) for u > 0, a(n) - b(m) for ul < 0, else the mean over c and n
  auto up = [&](double u, double ul, auto a, auto b, size_t n, size_t m) {
    if (u > 0.0) return a(c) - b(c);
    if (ul < 0.0) return a(n) - b(m);
    return h * (a(c) + a(n) - b(c) - b(n));
  };
  const double u1 = P[1 * N + c], u2 = P[2 * N + c], u3 = P[3 * N + c];
  double* D = r.ctd;
  D[0 * N + c] = up(u1, u1, fbyx, ezc, c + di, c + di);  // dyez
  D[1 * N + c] = up(u2, u1, fbxy, ezc, c + dj, c + dj);  // dxez
  D[2 * N + c] = up(u3, u1, fbyz, exc, c + dk, c + dk);  // dyex
  D[3 * N + c] = up(u2, u1, fbzy, exc, c + dj, c + dj);  // dzex
  D[4 * N + c] = up(u3, u1, fbxz, eyc, c + dk, c + dk);  // dxey
  D[5 * N + c] = up(u1, u1, fbzx, eyc, c + di, c);       // dzey
}

// ------------------------------------------------------------ boundaries
// Transverse indices of a column of direction D: (j,k) for D = 1, (i,k) for
// D = 2, (i,j) for D = 3; a slab direction contributes its fixed index.
template <int D>
__device__ __forceinline__ int col_fix1(const DevRun& r) { return D == 1 ? r.jfix : 0; }
template <int D>
__device__ __forceinline__ int col_fix2(const DevRun& r) { return D == 3 ? r.jfix : r.kfix; }

// Layer n (1-based) along direction D of column (t1, t2).
template <int D>
__device__ __forceinline__ size_t col_cell(const DevRun& r, int t1, int t2, int n) {
  if (D == 1) return r.cell(n, t1, t2);
  if (D == 2) return r.cell(t1, n, t2);
  return r.cell(t1, t2, n);
}

// bnd.f90:45-70, 156-180, 266-292: single-rank periodic copy for columns whose
// transverse indices are interior.
template <int D>
__device__ __forceinline__ void bc_periodic_body(const DevRun& r, double* __restrict__ P, const uint3 bid,
                                                 int vlo = 0, int vhi = 9) {
  if (!r.scal->active) return;
  const int nm1 = r.nm1;
  const int n1 = (D == 1) ? r.jmax : r.imax;
  const int n2 = (D == 3) ? r.jmax : r.kmax;
  const int t1 = col_fix1<D>(r) ? col_fix1<D>(r) : (int)(bid.x * blockDim.x + threadIdx.x) + nm1 + 1;
  const int t2 = col_fix2<D>(r) ? col_fix2<D>(r) : (int)(bid.y * blockDim.y + threadIdx.y) + nm1 + 1;
  if (t1 > n1 - nm1 || t2 > n2 - nm1) return;
  const int len = (D == 1) ? r.imax : (D == 2 ? r.jmax : r.kmax);
  const int ib0 = 1 + nm1, ib1 = len - nm1;
  const size_t N = r.N;
  for (int n = 1; n <= nm1; ++n)
    for (int v = vlo; v < vhi; ++v) {
      if (r.ibc[2 * (D - 1)][v] == 1 || r.ibc[2 * (D - 1) + 1][v] == 1) {
        double* p = P + (size_t)v * N;
        p[col_cell<D>(r, t1, t2, ib0 - n)] = p[col_cell<D>(r, t1, t2, ib1 + 1 - n)];
        p[col_cell<D>(r, t1, t2, ib1 + n)] = p[col_cell<D>(r, t1, t2, ib0 - 1 + n)];
      }
    }
}
// The standalone passes take one variable per grid z index (the variables of
// a column are independent: each code reads only its own variable, and the
// outflow check of code 18 an interior cell).
template <int D>
__global__ void k_bc_periodic(DevRun r, double* __restrict__ P) {
  bc_periodic_body<D>(r, P, blockIdx, (int)blockIdx.z, (int)blockIdx.z + 1);
}

// bnd.f90:384-1058: physical boundary codes for every column of direction D.
template <int D>
__device__ __forceinline__ void bc_phys_body(const DevRun& r, double* __restrict__ P, const double* __restrict__ Po,
                                             const uint3 bid, int vlo = 0, int vhi = 9) {
  if (!r.scal->active) return;
  const int n1 = (D == 1) ? r.jmax : r.imax;
  const int n2 = (D == 3) ? r.jmax : r.kmax;
  const int t1 = col_fix1<D>(r) ? col_fix1<D>(r) : (int)(bid.x * blockDim.x + threadIdx.x) + 1;
  const int t2 = col_fix2<D>(r) ? col_fix2<D>(r) : (int)(bid.y * blockDim.y + threadIdx.y) + 1;
  if (t1 > n1 || t2 > n2) return;
  const int nm1 = r.nm1;
  const int L = (D == 1) ? r.imax : (D == 2 ? r.jmax : r.kmax);
  const size_t N = r.N;
  for (int v = vlo; v < vhi; ++v) {
    double* u = P + (size_t)v * N;
    const double* uo = Po + (size_t)v * N;
    auto at = [&](int n) { return col_cell<D>(r, t1, t2, n); };
    switch (r.ibc[2 * (D - 1)][v]) {  // inner side
      case 2: for (int n = 1; n <= nm1; ++n) u[at(n)] = uo[at(n)]; break;
      case 3: for (int n = nm1; n >= 1; --n) u[at(n)] = (4.0 * u[at(n + 1)] - u[at(n + 2)]) / 3.0; break;
      case 4: for (int n = nm1; n >= 1; --n) u[at(n)] = 2.0 * u[at(n + 1)] - u[at(n + 2)]; break;
      case 5: for (int n = nm1; n >= 1; --n) u[at(n)] = u[at(1 + nm1)]; break;
      case 12: for (int n = 1; n <= nm1; ++n) u[at(n)] = -u[at(2 * nm1 - n + 1)]; break;
      case 13: for (int n = 1; n <= nm1; ++n) u[at(n)] = 0.0; break;
      case 14: for (int n = 1; n <= nm1; ++n) u[at(n)] = u[at(2 * nm1 - n + 1)]; break;
      case 7: for (int n = nm1; n >= 1; --n) u[at(n)] = uo[at(n)] + u[at(n + 1)] - uo[at(n + 1)]; break;
      default: break;
    }
    switch (r.ibc[2 * (D - 1) + 1][v]) {  // outer side
      case 2: for (int n = 0; n <= nm1 - 1; ++n) u[at(L - n)] = uo[at(L - n)]; break;
      case 3: for (int n = nm1 - 1; n >= 0; --n) u[at(L - n)] = (4.0 * u[at(L - n - 1)] - u[at(L - n - 2)]) / 3.0; break;
      case 4: for (int n = nm1 - 1; n >= 0; --n) u[at(L - n)] = 2.0 * u[at(L - n - 1)] - u[at(L - n - 2)]; break;
      case 5: for (int n = nm1 - 1; n >= 0; --n) u[at(L - n)] = u[at(L - nm1)]; break;
      case 12: for (int n = 0; n <= nm1 - 1; ++n) u[at(L - n)] = -u[at(L - 2 * nm1 + 1 + n)]; break;
      case 13: for (int n = 0; n <= nm1 - 1; ++n) u[at(L - n)] = 0.0; break;
      case 14: for (int n = 0; n <= nm1 - 1; ++n) u[at(L - n)] = u[at(L - 2 * nm1 + 1 + n)]; break;
      case 7:
        for (int n = nm1 - 1; n >= 0; --n) u[at(L - n)] = uo[at(L - n)] + u[at(L - n - 1)] - uo[at(L - n - 1)];
        break;
      case 18:  // x1 outer only (bnd.f90:598-610): zero when u^r of the last interior cell is negative
        if (D == 1) {
          const bool neg = P[(size_t)1 * N + at(L - nm1)] < 0.0;
          for (int n = nm1 - 1; n >= 0; --n) u[at(L - n)] = neg ? 0.0 : u[at(L - nm1)];
        }
        break;
      default: break;
    }
  }
}
template <int D>
__global__ void k_bc_phys(DevRun r, double* __restrict__ P, const double* __restrict__ Po) {
  bc_phys_body<D>(r, P, Po, blockIdx, (int)blockIdx.z, (int)blockIdx.z + 1);
}

// ----------------------------------------------------------------- floors
// infchk (bnd.f90:1636-1824, outer radial ghosts), atmosphere1a
// (correction.f90:226-447) and pminmax2b (correction.f90:744-999) over every
// cell, in place.  pminmax2b stores rho alone when its rescale loop changed rho
// (the "elseif" at correction.f90:887-893).
// PARTS selects the routines (bit 0 infchk, 1 atmosphere1a, 2 pminmax2b) for
// the per-routine entry points; the step runs all three.
template <int PARTS = 7>
__device__ __forceinline__ void floor_body(const DevRun& r, double* __restrict__ P, const uint3 bid) {
  if (!r.scal->active) return;
  const int i = bid.x * blockDim.x + threadIdx.x + 1;
  const int j = jidx(r, 1, bid);
  const int k = kidx(r, 1, bid);
  if (i > r.imax || j > r.jmax || k > r.kmax) return;
  const size_t N = r.N, c = r.cell(i, j, k);
  double q[9];
  load9(P, N, c, q);
  Met m;
  load_met(r.mc, r.nik, r.ik(i, k), m);
  const double gam = r.gam;
  if ((PARTS & 1) && r.model >= 7 && r.model <= 20 && i > r.imax - r.nm1) {
    const double gflmax = 10.0;
    double gfl = calgfl(q[1], q[2], q[3], m);
    double vel[4] = {0.0, q[1] * (1. / gfl), q[2] * (1. / gfl), q[3] * (1. / gfl)};
    if (vel[1] < 0.0) {
      vel[1] = m.be1 * m.ial;  // beta^r / alpha
      double vsq = qform3(m, vel[1], vel[2], vel[3]);
      if (vsq >= 1.0) vsq = 1. - 1. / (gflmax * gflmax);
      gfl = 1. / sqrt(1. - vsq);
      q[1] = vel[1] * gfl; q[2] = vel[2] * gfl; q[3] = vel[3] * gfl;
    }
  }
  if ((PARTS & 2) && r.model >= 7 && r.model <= 15) {
    const double epsilon = 1.e-2, gflmax = 10.0;
    const double demin = __ldg(r.fl_de + i - 1);
    const double prmin = __ldg(r.fl_pr + i - 1);
    const double dthe = 1.0 * (1. + epsilon) * demin;
    const double dthe1 = 1.0 * (1. + epsilon) * prmin;
    const double bsq = q[6] * q[6] + q[7] * q[7] + q[8] * q[8];
    if (q[0] < dthe || (q[4] < dthe1 && bsq <= 1.e-20)) {
      q[0] = demin;
      q[4] = prmin;
      const double vel[4] = {0.0, 0.0, 0.0, 0.0};
      double vsq = qform3(m, vel[1], vel[2], vel[3]);
      if (vsq >= 1.0) vsq = 1. - 1. / (gflmax * gflmax);
      const double gfl = 1. / sqrt(1. - vsq);
      q[1] = vel[1] * gfl; q[2] = vel[2] * gfl; q[3] = vel[3] * gfl;
    }
    q[5] = 0.0;
  }
  if (PARTS & 4) {  // pminmax2b
    const double gflmax = 20.0;
    double de = q[0], pr = q[4];
    double gfl = calgfl(q[1], q[2], q[3], m);
    const double vel[4] = {0.0, q[1] * (1. / gfl), q[2] * (1. / gfl), q[3] * (1. / gfl)};
    double vsq = qform3(m, vel[1], vel[2], vel[3]);
    if (vsq >= 1.0 || gfl > gflmax) vsq = 1. - 1. / (gflmax * gflmax);
    gfl = 1. / sqrt(1. - vsq);
    double lim[9];
#pragma unroll
    for (int v = 0; v < 9; ++v) lim[v] = q[v];
    lim[1] = vel[1] * gfl; lim[2] = vel[2] * gfl; lim[3] = vel[3] * gfl;
    PS s;
    pstate(lim, m, gam, s);
    const double bbsq = s.bbsq;
    gfl = s.gfl;
    const double bcon[4] = {0.0, q[6], q[7], q[8]};
    double bcov[4];
    lower_g(bcon, bcov, m);
    const double bsq = bcon[1] * bcov[1] + bcon[2] * bcov[2] + bcon[3] * bcov[3];
    const double f105 = (double)1.05f, f005 = (double)0.05f;
    bool capped = false;
    for (int cnt = 0;; ++cnt) {
      if (cnt >= 100000) { capped = true; break; }
      const double roh = de + (gam / (gam - 1.0)) * pr;
      const double t1a = roh * gfl * gfl - pr;
      const double t1b = fabs(f005 * bsq);
      if (t1a <= t1b) { de = f105 * de; pr = f105 * pr; continue; }
      break;
    }
    if (capped) atomicAdd(r.cnt + C_FLOORCAP, 1ull);
    if (de != q[0]) q[0] = de;
    else if (pr != q[4]) q[4] = pr;
    const double demin = __ldg(r.fl_de + i - 1);
    const double prmin = __ldg(r.fl_pr + i - 1);
    const double bbromax = 50.0, bbprmax = 2.e3, prromax = 1.e6;
    if (pr < prmin) q[4] = prmin;
    if (pr > r.pmax) q[4] = r.pmax;
    if (de < demin) q[0] = demin;
    const double prro = q[4] * (1. / q[0]);
    if (prro > prromax) q[0] = q[4] / prromax;
    const double bbro = bbsq * (1. / q[0]);
    const double bbpr = bbsq * (1. / q[4]);
    if (bbro > bbromax) q[0] = bbsq / bbromax;
    if (bbpr > bbprmax) q[4] = bbsq / bbprmax;
  }
#pragma unroll
  for (int v = 0; v < 6; ++v) P[(size_t)v * N + c] = q[v];
  if (r.P32)  // FP32 copy of the final primitives for the next stage's FP32 faces
#pragma unroll
    for (int v = 0; v < 9; ++v) r.P32[(size_t)v * N + c] = (float)q[v];
}
// Resident blocks per SM the floor and CFL passes are compiled for: 8 (64 registers,
// 28-44 B of spills) measured 15% (floors) and 8% (CFL) faster than 6-7 blocks at 72-82.
#ifndef RG_CELL_MINB
#define RG_CELL_MINB 8
#endif
__global__ void __launch_bounds__(128, RG_CELL_MINB) k_floor(DevRun r, double* __restrict__ P) { floor_body(r, P, blockIdx); }
template <int PARTS>
__global__ void __launch_bounds__(128) k_floor_part(DevRun r, double* __restrict__ P) {
  floor_body<PARTS>(r, P, blockIdx);
}

// FP32 copy of a primitive array (mixed runs, after initial data or upload).
__global__ void k_to_f32(const double* __restrict__ a, float* __restrict__ b, size_t n) {
  const size_t x = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (x < n) b[x] = (float)a[x];
}

// ------------------------------------------------------------------- CFL
// cdtcfl4 (cdtcfl.f90:2-129) with calcha4 (calcha.f90:129-367) over
// is1+1..ie1-1 (every dimension); min over cells, then over blocks with an
// atomicMin on the bit pattern (positive doubles order like their bits).
__device__ __forceinline__ void cfl_body(const DevRun& r, const double* __restrict__ P, const uint3 bid) {
  if (!r.scal->active) return;
  const int i = bid.x * blockDim.x + threadIdx.x + 2;
  const int j = jidx(r, 2, bid);
  const int k = kidx(r, 2, bid);
  double dtc = 1.0;
  if (i <= r.imax - 1 && j <= r.jmax - 1 && k <= r.kmax - 1) {
    const size_t c = r.cell(i, j, k);
    double q[9];
    load9(P, r.N, c, q);
    Met m;
    load_met(r.mc, r.nik, r.ik(i, k), m);
    PS s;
    pstate(q, m, r.gam, s);
    double vp1, vm1, vp2, vm2, vp3, vm3;
    wavespeed<1>(q, s, m, r.gam, vp1, vm1);
    wavespeed<2>(q, s, m, r.gam, vp2, vm2);
    wavespeed<3>(q, s, m, r.gam, vp3, vm3);
    const double small = 1.e-12;
    double vfi = fmax3(0.0, fabs(vp1), fabs(vm1));
    double vfj = fmax3(0.0, fabs(vp2), fabs(vm2));
    double vfk = fmax3(0.0, fabs(vp3), fabs(vm3));
    double d1 = 1.e10, d2 = 1.e10, d3 = 1.e10;
    if (r.imax > r.nmax_cfl && vfi > 0.0) { if (vfi > 1.0) vfi = 1.0; d1 = fabs(__ldg(r.dx1b + i - 1) / (vfi + small)); }
    if (r.jmax > r.nmax_cfl && vfj > 0.0) { if (vfj > 1.0) vfj = 1.0; d2 = fabs(__ldg(r.dx2b + j - 1) / (vfj + small)); }
    if (r.kmax > r.nmax_cfl && vfk > 0.0) { if (vfk > 1.0) vfk = 1.0; d3 = fabs(__ldg(r.dx3b + k - 1) / (vfk + small)); }
    dtc = dmin2(dtc, d1);
    dtc = dmin2(dtc, d2);
    dtc = dmin2(dtc, d3);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) dtc = dmin2(dtc, __shfl_xor_sync(0xffffffffu, dtc, o));
  __shared__ double red[32];
  const int t = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nt = blockDim.x * blockDim.y * blockDim.z;
  if ((t & 31) == 0) red[t >> 5] = dtc;
  __syncthreads();
  if (t < 32) {
    double x = (t < (nt + 31) / 32) ? red[t] : 1.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = dmin2(x, __shfl_xor_sync(0xffffffffu, x, o));
    if (t == 0 && x > 0.0) atomicMin(&r.scal->dtcfl_bits, (unsigned long long)__double_as_longlong(x));
  }
}
__global__ void __launch_bounds__(128, RG_CELL_MINB) k_cfl(DevRun r, const double* __restrict__ P) { cfl_body(r, P, blockIdx); }

__device__ __forceinline__ void step_begin_body(const DevRun& r) {
  Scal* s = r.scal;
  if (!s->active) return;
  s->time = s->timeh;  // main.f90:617-620
  if (s->time > r.tmax) { s->active = 0; return; }
  s->dtcfl_bits = (unsigned long long)__double_as_longlong(1.0);
}
__device__ __forceinline__ void dt_body(const DevRun& r) {
  Scal* s = r.scal;
  if (!s->active) return;
  const double dtcfl = __longlong_as_double((long long)s->dtcfl_bits);
  s->dt = r.cfl * dtcfl;  // main.f90:763
  s->timeh = s->time + s->dt;
}
// The buffer rotation advances every step (a finished run copies its state
// through the stages), the step count only while the run is active.
__device__ __forceinline__ void step_end_body(const DevRun& r) {
  Scal* s = r.scal;
  s->cur = (s->cur + 1) % 3;
  if (s->active) atomicAdd(r.cnt + C_STEPS, 1ull);
}
__global__ void k_step_begin(DevRun r) { step_begin_body(r); }
__global__ void k_dt(DevRun r) { dt_body(r); }
__global__ void k_step_end(DevRun r) { step_end_body(r); }

// ------------------------------------------------------ snapshot output
// The byte image of output1's data records (restar.f90:160-167): record
// rec0 + t, for (i, j, k) with k fastest, then j, then i, is 13 doubles
// x1(i), x2(j), x3(k), uri(1:9,i,j,k), detg(i,j,k) framed by the 4-byte
// record length 104 of gfortran's sequential unformatted files: 28 words of
// 4 bytes, so that the image is the file's bytes.  cx/cy/cz are the three
// coordinate axes the file carries (index i-1 etc.).
__global__ void __launch_bounds__(128) k_output1(DevRun r, const double* __restrict__ P, const double* __restrict__ cx,
                                                 const double* __restrict__ cy, const double* __restrict__ cz,
                                                 size_t rec0, size_t nrec, unsigned* __restrict__ out) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nrec) return;
  const size_t rr = rec0 + t;
  const int k = (int)(rr % (size_t)r.kmax) + 1;
  const int j = (int)((rr / (size_t)r.kmax) % (size_t)r.jmax) + 1;
  const int i = (int)(rr / ((size_t)r.kmax * (size_t)r.jmax)) + 1;
  const size_t c = r.cell(i, j, k);
  double v[13];
  v[0] = cx[i - 1];
  v[1] = cy[j - 1];
  v[2] = cz[k - 1];
#pragma unroll
  for (int n = 0; n < 9; ++n) v[3 + n] = P[(size_t)n * r.N + c];
  v[12] = r.mc[17 * r.nik + r.ik(i, k)];
  unsigned* o = out + t * 28;
  o[0] = 104u;
#pragma unroll
  for (int m = 0; m < 13; ++m) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(v[m]);
    o[1 + 2 * m] = (unsigned)(b & 0xffffffffull);
    o[2 + 2 * m] = (unsigned)(b >> 32);
  }
  o[27] = 104u;
}

// ------------------------------------------------------ div B diagnostic
// Corner-centred divergence of sqrt(-g) B (the quantity Toth's flux-CT,
// ct.f90:30-118, keeps constant when the normal-field flux is zero): at the
// corner between cells (i..i+1, j..j+1, k..k+1) of the interior,
//   D = sum_d (1/(4 dx_d)) sum of the four differences along d
//       of [sqrt(-g) B^d](cell + e_d) - [sqrt(-g) B^d](cell),
// with dx_d the spacing of the lower cell.  A slab direction (one interior
// cell, uniform along it) has one corner plane and no difference along it.
// red[0] receives max |D|, red[1] max |sqrt(-g) B^d| / dx_d over the same
// cells, both as bit patterns of non-negative doubles (atomicMax).
__global__ void __launch_bounds__(256) k_divb(DevRun r, const double* __restrict__ P,
                                              unsigned long long* __restrict__ red) {
  const int nm1 = r.nm1;
  const int i0 = nm1 + 1, j0 = r.jfix ? r.jfix : nm1 + 1, k0 = r.kfix ? r.kfix : nm1 + 1;
  const int ni = r.imax - 2 * nm1 - 1;
  const int nj = r.jfix ? 1 : r.jmax - 2 * nm1 - 1;
  const int nk = r.kfix ? 1 : r.kmax - 2 * nm1 - 1;
  const long long total = (long long)ni * nj * nk;
  const size_t N = r.N;
  double dmax = 0.0, bmax = 0.0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = i0 + (int)(t % ni);
    const int j = j0 + (int)((t / ni) % nj);
    const int k = k0 + (int)(t / ((long long)ni * nj));
    double b[2][2][2][3];
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
      for (int bb = 0; bb < 2; ++bb)
#pragma unroll
        for (int a = 0; a < 2; ++a) {
          const size_t cell = r.cell(i + a, j + bb, k + c);
          const double g = __ldg(r.mc + 17 * r.nik + r.ik(i + a, k + c));
#pragma unroll
          for (int d = 0; d < 3; ++d) b[c][bb][a][d] = g * P[(size_t)(6 + d) * N + cell];
        }
    const double dx1 = r.dx1b[i - 1], dx2 = r.dx2b[j - 1], dx3 = r.dx3b[k - 1];
    double d1 = 0.0, d2 = 0.0, d3 = 0.0;
#pragma unroll
    for (int u = 0; u < 2; ++u)
#pragma unroll
      for (int v = 0; v < 2; ++v) {
        d1 += b[u][v][1][0] - b[u][v][0][0];
        d2 += b[u][1][v][1] - b[u][0][v][1];
        d3 += b[1][u][v][2] - b[0][u][v][2];
      }
    const double D = d1 / (4.0 * dx1) + (r.jfix ? 0.0 : d2 / (4.0 * dx2)) + (r.kfix ? 0.0 : d3 / (4.0 * dx3));
    dmax = fmax(dmax, fabs(D));
    if (D != D) dmax = D;
    bmax = fmax(bmax, fmax(fabs(b[0][0][0][0]) / dx1, fmax(fabs(b[0][0][0][1]) / dx2, fabs(b[0][0][0][2]) / dx3)));
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double x = __shfl_xor_sync(0xffffffffu, dmax, o), y = __shfl_xor_sync(0xffffffffu, bmax, o);
    dmax = (x != x) ? x : fmax(dmax, x);
    bmax = fmax(bmax, y);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(red, (unsigned long long)__double_as_longlong(fabs(dmax)));
    atomicMax(red + 1, (unsigned long long)__double_as_longlong(bmax));
  }
}

// ------------------------------------------------- per-routine entry points
// recov (recov.f90:2-47) of every interior cell; other cells, and every cell
// of a run that has passed tmax, keep Pc.
template <int IWVEC>
__global__ void __launch_bounds__(128) k_recov(DevRun r, const double* __restrict__ U, const double* __restrict__ Pc,
                                               double* __restrict__ Pw) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = jidx(r, 1, blockIdx);
  const int k = kidx(r, 1, blockIdx);
  if (i > r.imax || j > r.jmax || k > r.kmax) return;
  const size_t N = r.N, c = r.cell(i, j, k);
  if (!r.scal->active || !is_interior(r, i, j, k)) {
#pragma unroll
    for (int v = 0; v < 9; ++v) Pw[(size_t)v * N + c] = Pc[(size_t)v * N + c];
    return;
  }
  Met m;
  load_met(r.mc, r.nik, r.ik(i, k), m);
  double u[9], qo[9], qn[9];
  load9(U, N, c, u);
  load9(Pc, N, c, qo);
  RecovOut o{0.0, false, false, false};
  const bool ok =
      recov_any<IWVEC>(u, qo, qn, m, r.gam, r.gkind, r.iter, __ldg(r.fl_de + i - 1), __ldg(r.fl_pr + i - 1), nullptr, o);
  if (!ok) queue_carry(r, i, j, k);
  else
#pragma unroll
    for (int v = 0; v < 9; ++v) Pw[(size_t)v * N + c] = qn[v];
  count_event(r, C_NR2, ok && o.nr2);
  count_event(r, C_FAIL, ok && o.fail);
  count_event(r, C_CAP, ok && o.cap);
}

// caluu1 (caluu.f90:2-126) on every cell
__global__ void __launch_bounds__(128) k_p2c(DevRun r, const double* __restrict__ P, double* __restrict__ U) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = jidx(r, 1, blockIdx);
  const int k = kidx(r, 1, blockIdx);
  if (i > r.imax || j > r.jmax || k > r.kmax) return;
  const size_t N = r.N, c = r.cell(i, j, k);
  double q[9], u[9];
  load9(P, N, c, q);
  Met m;
  load_met(r.mc, r.nik, r.ik(i, k), m);
  PS s;
  pstate(q, m, r.gam, s);
  p2c(s, r.gam, r.gkind, m.detg, u);
#pragma unroll
  for (int v = 0; v < 9; ++v) U[(size_t)v * N + c] = u[v];
}

// caltenr + calsf (calsf.f90:6-151) on every cell: sf(2:5) as four planes
// SF[n*N + c].
__global__ void __launch_bounds__(128) k_calsf(DevRun r, const double* __restrict__ P, double* __restrict__ SF) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = jidx(r, 1, blockIdx);
  const int k = kidx(r, 1, blockIdx);
  if (i > r.imax || j > r.jmax || k > r.kmax) return;
  const size_t N = r.N, c = r.cell(i, j, k), q = r.ik(i, k);
  double p[9];
  load9(P, N, c, p);
  Met m;
  load_met(r.mc, r.nik, q, m);
  PS s;
  pstate(p, m, r.gam, s);
  double sf[4];
  geom_source(r, s, q, m.detg, sf);
#pragma unroll
  for (int n = 0; n < 4; ++n) SF[(size_t)n * N + c] = sf[n];
}

// calgfl of the output converter (convert_vtk2dn1.f90:1158-1197): the same
// quadratic form as physfunc's, clamped at |u~^2| > 1e10 to 1e9.
__device__ __forceinline__ double calgfl_conv(double u1, double u2, double u3, const Met& m) {
  double utsq = qform3(m, u1, u2, u3);
  if (utsq < 0.0) utsq = (fabs(utsq) <= 1.0e-10) ? fabs(utsq) : 1.e-10;
  if (fabs(utsq) > 1.0e10) utsq = 1.0e9;
  return sqrt(1. + utsq);
}

// Derived quantities of one cell as convert_vtk2dn1.f90:254-371 computes them
// for its output: out = (gfa, gfb, b^2, -h u_t, v1, v2, v3), the Lorentz
// factors of the Boyer-Lindquist ZAMO and of the static observer at infinity,
// the field strength, the Bernoulli parameter and the BL velocity
// u^i + gfa beta^i / alpha; inside r_H = 1 + sqrt(1 - a^2) gfa = gfb = 1 and
// v = 0.  The run's metric comes from the cell-centre cache (the converter
// re-evaluates the same coord.f90 formulas); transmks2ks1 and transks2bl1
// (convert_vtk2dn1.f90:1399-1554) use the Kerr-Schild formulas at
// (rr, th) with rfac = dr/dx1, hfac = dtheta/dx3 and sin/cos of th given.
__device__ void derived_cell(const DevRun& r, double akm, const double qin[9], const Met& m, double rr, double rfac,
                             double sth, double cth, double hfac, double out[7]) {
  double q[9];
#pragma unroll
  for (int v = 0; v < 9; ++v) q[v] = qin[v];
  // minimum magnetic field (bmin1 = 1e-20)
  for (int v = 6; v < 9; ++v)
    if (fabs(q[v]) < 1.e-20) q[v] = 0.0;
  PS s;
  pstate_gfl(q, m, r.gam, calgfl_conv(q[1], q[2], q[3], m), s);
  out[2] = s.bbsq;
  out[3] = -(s.roh / s.de) * s.ucov[0];
  const double rbh1 = 1. + sqrt(1. - akm * akm);
  if (!(rr > rbh1)) {
    out[0] = 1.0; out[1] = 1.0; out[4] = 0.0; out[5] = 0.0; out[6] = 0.0;
    return;
  }
  // MKS -> KS 3-velocity, then the KS 4-velocity (Kerr-Schild metric at (rr, th))
  const double ut1 = rfac * q[1], ut2 = q[2], ut3 = hfac * q[3];
  const double del = rr * rr - (2. * rr) + akm * akm;
  const double sig = rr * rr + akm * cth * akm * cth;
  const double aa = ((rr * rr + akm * akm) * (rr * rr + akm * akm)) - akm * akm * del * sth * sth;
  Met ks{};
  ks.g11 = 1. + 2. * rr / sig;
  ks.g12 = -1. * akm * sth * sth * (1. + 2. * rr / sig);
  ks.g22 = aa * sth * sth / sig;
  ks.g33 = sig;
  const double gfl = calgfl_conv(ut1, ut2, ut3, ks);
  const double gc00 = -1. - 2. * rr / sig, gc01 = 2. * rr / sig;
  const double alpha1 = 1. / sqrt(-gc00);
  const double beta1 = alpha1 * alpha1 * gc01;
  const double u0 = gfl * (1. / alpha1);
  const double u1 = ut1 - gfl * beta1 * (1. / alpha1);
  const double u2 = ut2 - gfl * (alpha1 * alpha1 * 0.0) * (1. / alpha1);
  const double u3 = ut3 - gfl * (alpha1 * alpha1 * 0.0) * (1. / alpha1);
  // KS -> BL (transks2bl1): t and phi pick up -2r/Delta u^r and -a/Delta u^r
  const double tmp2 = rr * rr - (2. * rr) + akm * akm;
  double b0 = 0.0, b1 = 0.0, b2 = 0.0, b3 = 0.0;
  if (tmp2 > 0.0) {
    b0 = u0 + (-2. * rr * (1. / tmp2)) * u1;
    b1 = u1;
    b2 = (-akm * (1. / tmp2)) * u1 + u2;
    b3 = u3;
  }
  // Boyer-Lindquist lapse and shift at (rr, th)
  const double gcon1a00 = -aa / (sig * del);
  const double gcon1a02 = -(2. * akm * rr) / (sig * del);
  const double gcov1a00 = -(sig - 2. * rr) / sig;
  const double al = 1. / sqrt(-gcon1a00);
  const double bt2 = al * al * gcon1a02;
  out[0] = al * b0;
  out[1] = b0 * sqrt(-gcov1a00);
  out[4] = b1 + out[0] * (al * al * 0.0) * (1. / al);
  out[5] = b2 + out[0] * bt2 * (1. / al);
  out[6] = b3 + out[0] * (al * al * 0.0) * (1. / al);
}

// Derived quantities of every cell (jslice = 0, out[7*c_full + f]) or of the
// phi plane jslice (out[7*((i-1) + imax*(k-1)) + f]); geo_i holds (rr, rfac)
// per radial index, geo_k (sin th, cos th, hfac) per theta index.
__global__ void __launch_bounds__(128) k_derived(DevRun r, const double* __restrict__ P,
                                                 const double* __restrict__ geo_i,
                                                 const double* __restrict__ geo_k, double akm, int jslice,
                                                 double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int jj = (int)(blockIdx.y * blockDim.y + threadIdx.y) + 1;
  const int k = (int)(blockIdx.z * blockDim.z + threadIdx.z) + 1;
  const int j = jslice ? jslice : jj;
  if (i > r.imax || jj > (jslice ? 1 : r.jmax) || k > r.kmax) return;
  const size_t N = r.N, c = r.cell(i, j, k);
  double q[9], o[7];
  load9(P, N, c, q);
  Met m;
  load_met(r.mc, r.nik, r.ik(i, k), m);
  derived_cell(r, akm, q, m, geo_i[2 * (i - 1)], geo_i[2 * (i - 1) + 1], geo_k[3 * (k - 1)], geo_k[3 * (k - 1) + 1],
               geo_k[3 * (k - 1) + 2], o);
  const size_t pt = jslice ? (size_t)(i - 1) + (size_t)r.imax * (size_t)(k - 1)
                           : (size_t)(i - 1) + (size_t)r.imax * ((size_t)(j - 1) + (size_t)r.jmax * (size_t)(k - 1));
#pragma unroll
  for (int f = 0; f < 7; ++f) out[7 * pt + f] = o[f];
}

// One RK stage of rkt.f90 (rk2fst, rk3snd or rk3trd, then the matching
// rk*ads*) on the interior: W[d] holds ww(d, m) of cell c at m*N + c (flux-CT
// already applied), Uo = uo (stages 2 and 3), Uc = the stage input (uu, uh or
// us), SF = sf(2:5) as four planes; Unew keeps its values outside the interior.
template <int STAGE>
__global__ void __launch_bounds__(128) k_rkt(DevRun r, const double* __restrict__ W1, const double* __restrict__ W2,
                                             const double* __restrict__ W3, const double* __restrict__ Uo,
                                             const double* __restrict__ Uc, const double* __restrict__ SF,
                                             double* __restrict__ Unew, double dt, bool step_dt = false) {
  if (step_dt) dt = r.scal->dt;  // inside a step: the step's dt (main.f90:763)
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = jidx(r, 1, blockIdx);
  const int k = kidx(r, 1, blockIdx);
  if (i > r.imax || j > r.jmax || k > r.kmax || !is_interior(r, i, j, k)) return;
  const size_t N = r.N, c = r.cell(i, j, k);
  const size_t ci = c - 1, cj = c - r.sj, ck = c - r.sk;
  const double a1 = dt / __ldg(r.dx1b + i - 1), a2 = dt / __ldg(r.dx2b + j - 1), a3 = dt / __ldg(r.dx3b + k - 1);
  double u[9];
#pragma unroll
  for (int v = 0; v < 9; ++v) {
    const size_t o = (size_t)v * N;
    const double d1 = W1[o + c] - W1[o + ci], d2 = W2[o + c] - W2[o + cj], d3 = W3[o + c] - W3[o + ck];
    u[v] = rk_combine<STAGE>(STAGE > 1 ? Uo[o + c] : 0.0, Uc[o + c], a1, d1, a2, d2, a3, d3);
  }
#pragma unroll
  for (int v = 1; v <= 4; ++v) u[v] = rk_add_source<STAGE>(u[v], SF[(size_t)(v - 1) * N + c], dt);
#pragma unroll
  for (int v = 0; v < 9; ++v) Unew[(size_t)v * N + c] = u[v];
}

// a(nv, cell) of the reference's full array <-> stored SoA.  Upload reads the
// stored cells' values and flags (bad != 0) any full-array cell whose value
// differs from the stored cell it maps to: a slab direction holds one plane,
// so its data must be uniform along it.  Download writes every full cell.
__global__ void k_aos_to_soa(DevRun r, const double* __restrict__ a, double* __restrict__ s, int* bad) {
  const size_t f = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t nfull = (size_t)r.imax * r.jmax * r.kmax;
  if (f >= nfull) return;
  const int i = (int)(f % r.imax) + 1;
  const int j = (int)((f / r.imax) % r.jmax) + 1;
  const int k = (int)(f / ((size_t)r.imax * r.jmax)) + 1;
  const bool owner = (!r.jfix || j == r.jfix) && (!r.kfix || k == r.kfix);
  const size_t c = r.cell(i, j, k);
  if (owner) {
#pragma unroll
    for (int v = 0; v < 9; ++v) s[(size_t)v * r.N + c] = a[9 * f + v];
  } else if (bad) {
    const size_t o = r.cell_full(i, r.jfix ? r.jfix : j, r.kfix ? r.kfix : k);
    bool same = true;
#pragma unroll
    for (int v = 0; v < 9; ++v)
      same = same && (__double_as_longlong(a[9 * f + v]) == __double_as_longlong(a[9 * o + v]));
    if (!same) atomicOr(bad, 1);
  }
}
__global__ void k_soa_to_aos(DevRun r, const double* __restrict__ s, double* __restrict__ a) {
  const size_t f = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t nfull = (size_t)r.imax * r.jmax * r.kmax;
  if (f >= nfull) return;
  const int i = (int)(f % r.imax) + 1;
  const int j = (int)((f / r.imax) % r.jmax) + 1;
  const int k = (int)(f / ((size_t)r.imax * r.jmax)) + 1;
  const size_t c = r.cell(i, j, k);
#pragma unroll
  for (int v = 0; v < 9; ++v) a[9 * f + v] = s[(size_t)v * r.N + c];
}
__global__ void k_fill(double* p, double v, size_t n) {
  const size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c < n) p[c] = v;
}

// Derived metric fields (met_derive) of every point of the three caches and
// the radial floor profiles of atmosphere1a/pminmax2b (correction.f90:897-898).
__global__ void k_geom_derive(DevRun r, double* mc, double* mi, double* mk, double* fl_de, double* fl_pr) {
  const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < r.nik) {
    double* caches[3] = {mc, mi, mk};
#pragma unroll 1
    for (int a = 0; a < 3; ++a) {
      double base[kMetBase], d[kMetComps - kMetBase];
      for (int c = 0; c < kMetBase; ++c) base[c] = caches[a][(size_t)c * r.nik + q];
      met_derive(base, d);
      for (int c = 0; c < kMetComps - kMetBase; ++c) caches[a][(size_t)(kMetBase + c) * r.nik + q] = d[c];
    }
  }
  if (q < (size_t)r.imax) {
    const double rr = r.x1[q];
    fl_de[q] = r.dmin * spow(rr, -1.5);
    fl_pr[q] = (r.gam - 1.) * r.pmin * spow(rr, -2.5);
  }
}

inline dim3 grid3(int nx, int ny, int nz, dim3 b) {
  return dim3((unsigned)((nx + (int)b.x - 1) / (int)b.x), (unsigned)((ny + (int)b.y - 1) / (int)b.y),
              (unsigned)((nz + (int)b.z - 1) / (int)b.z));
}
// Block shape and grid of a cell kernel over (nx, ny, nz): a slab direction
// has one index, so its block and grid extent fold to 1 (its threads move to x).
inline dim3 sblock(const DevRun& r, dim3 b) {
  if (r.jfix) { b.x *= b.y; b.y = 1; }
  if (r.kfix) { b.x *= b.z; b.z = 1; }
  return b;
}
inline dim3 sgrid(const DevRun& r, int nx, int ny, int nz, dim3 b) {
  return grid3(nx, r.jfix ? 1 : ny, r.kfix ? 1 : nz, b);
}

}  // namespace

// ------------------------------------------------------------- launchers
cudaError_t launch_step_begin(const DevRun& r, cudaStream_t s) {
  k_step_begin<<<1, 1, 0, s>>>(r);
  return cudaGetLastError();
}
cudaError_t launch_dt(const DevRun& r, cudaStream_t s) {
  k_dt<<<1, 1, 0, s>>>(r);
  return cudaGetLastError();
}
cudaError_t launch_step_end(const DevRun& r, cudaStream_t s) {
  k_step_end<<<1, 1, 0, s>>>(r);
  return cudaGetLastError();
}

// Block of the CFL and floor passes: RG_CELL_BX cells along i times
// 128 / RG_CELL_BX rows along j (rows share their (i, k) metric points).
#ifndef RG_CELL_BX
#define RG_CELL_BX 32
#endif
cudaError_t launch_cfl(const DevRun& r, const double* P, cudaStream_t s) {
  const dim3 b = sblock(r, dim3(RG_CELL_BX, 128 / RG_CELL_BX, 1));
  k_cfl<<<sgrid(r, r.imax - 2, r.jmax - 2, r.kmax - 2, b), b, 0, s>>>(r, P);
  return cudaGetLastError();
}

template <int IREC, typename T, typename S>
static void flux_dir(const DevRun& r, int dir, dim3 g, dim3 b, const S* P, S* F, float* Fcopy, int icopy, int ilo,
                     int ihi, cudaStream_t s) {
  if (dir == 1) k_flux<1, IREC, T, S><<<g, b, 0, s>>>(r, P, F, Fcopy, icopy, ilo, ihi);
  else if (dir == 2) k_flux<2, IREC, T, S><<<g, b, 0, s>>>(r, P, F, Fcopy, icopy, ilo, ihi);
  else k_flux<3, IREC, T, S><<<g, b, 0, s>>>(r, P, F, Fcopy, icopy, ilo, ihi);
}

template <typename T, typename S>
static void launch_flux_t(const DevRun& r, int dir, const S* P, S* F, float* Fcopy, int icopy, int ilo, int ihi,
                          cudaStream_t s) {
  if (ihi < ilo) return;
  const int n = ihi - ilo + 1, m = r.jmax - 2 * r.nm0 + 1, l = r.kmax - 2 * r.nm0 + 1;
  const dim3 b = sblock(r, dim3(64, 2, 1));
  const dim3 g = sgrid(r, 2 * n, m, l, b);  // two lanes per face
  switch (r.irec) {
    case 1: flux_dir<1, T, S>(r, dir, g, b, P, F, Fcopy, icopy, ilo, ihi, s); break;
    case 2: flux_dir<2, T, S>(r, dir, g, b, P, F, Fcopy, icopy, ilo, ihi, s); break;
    case 3: flux_dir<3, T, S>(r, dir, g, b, P, F, Fcopy, icopy, ilo, ihi, s); break;
    case 4: flux_dir<4, T, S>(r, dir, g, b, P, F, Fcopy, icopy, ilo, ihi, s); break;
    case 8: flux_dir<8, T, S>(r, dir, g, b, P, F, Fcopy, icopy, ilo, ihi, s); break;
    case 10: flux_dir<10, T, S>(r, dir, g, b, P, F, Fcopy, icopy, ilo, ihi, s); break;
    case 11: flux_dir<11, T, S>(r, dir, g, b, P, F, Fcopy, icopy, ilo, ihi, s); break;
    case 12: flux_dir<12, T, S>(r, dir, g, b, P, F, Fcopy, icopy, ilo, ihi, s); break;
    case 13: flux_dir<13, T, S>(r, dir, g, b, P, F, Fcopy, icopy, ilo, ihi, s); break;
    case 5: flux_dir<5, T, S>(r, dir, g, b, P, F, Fcopy, icopy, ilo, ihi, s); break;
    case 6: flux_dir<6, T, S>(r, dir, g, b, P, F, Fcopy, icopy, ilo, ihi, s); break;
    case 7: flux_dir<7, T, S>(r, dir, g, b, P, F, Fcopy, icopy, ilo, ihi, s); break;
    default: flux_dir<9, T, S>(r, dir, g, b, P, F, Fcopy, icopy, ilo, ihi, s); break;
  }
}

// Radial index of the last FP64 cell of a mixed run, clamped to [lo-1, hi].
static int fp64_split(const DevRun& r, int lo, int hi) {
  return r.i_fp64 < lo ? lo - 1 : (r.i_fp64 > hi ? hi : r.i_fp64);
}

// The staged kernel covers the reconstructions whose lanes read their
// stencil alone, at most two cells either side of the owner cell (the box
// holds i-2 .. i+3 of its faces): PPM, MP5, WENO5, WENO-Z and WENO-M, whose
// ghost widths (nm0 = 3, 4) keep the box origin at or above index 0.  MP-WENO
// also reads a cell eleven away, the second-order schemes are cheap to read.
bool flux_tma_eligible(const DevRun& r) {
  const bool scheme = r.irec == 5 || r.irec == 6 || r.irec == 7 || r.irec == 9 || r.irec == 10;
  return scheme && r.nm0 >= 3 && !r.jfix && !r.kfix && !r.kmet && (r.imax % 4) == 0 &&
         r.N == (size_t)r.imax * r.jmax * r.kmax;
}

template <int IREC, typename T, typename S>
static void launch_flux_tma_irec(const DevRun& r, int dir, const CUtensorMap& tm, const CUtensorMap& tmm, S* F,
                                 float* Fcopy, int icopy, int ilo, int ihi, dim3 g, dim3 b, cudaStream_t s) {
  constexpr int LO = tma_lo<IREC>();
  if (dir == 1)
    k_flux_tma<1, IREC, T, S><<<g, b, TmaBox<1, S, LO>::SMEM, s>>>(tm, tmm, r, F, Fcopy, icopy, ilo, ihi);
  else if (dir == 2)
    k_flux_tma<2, IREC, T, S><<<g, b, TmaBox<2, S, LO>::SMEM, s>>>(tm, tmm, r, F, Fcopy, icopy, ilo, ihi);
  else
    k_flux_tma<3, IREC, T, S><<<g, b, TmaBox<3, S, LO>::SMEM, s>>>(tm, tmm, r, F, Fcopy, icopy, ilo, ihi);
}
template <typename T, typename S>
static void launch_flux_tma_t(const DevRun& r, int dir, const CUtensorMap& tm, const CUtensorMap& tmm, S* F,
                              float* Fcopy, int icopy, int ilo, int ihi, cudaStream_t s) {
  if (ihi < ilo) return;
  const int n = ihi - ilo + 1, m = r.jmax - 2 * r.nm0 + 1, l = r.kmax - 2 * r.nm0 + 1;
  const dim3 b(64, 2, 1);
  const dim3 g((unsigned)((n + 31) / 32), (unsigned)((m + 1) / 2), (unsigned)l);
  switch (r.irec) {
    case 5: launch_flux_tma_irec<5, T, S>(r, dir, tm, tmm, F, Fcopy, icopy, ilo, ihi, g, b, s); break;
    case 7: launch_flux_tma_irec<7, T, S>(r, dir, tm, tmm, F, Fcopy, icopy, ilo, ihi, g, b, s); break;
    case 9: launch_flux_tma_irec<9, T, S>(r, dir, tm, tmm, F, Fcopy, icopy, ilo, ihi, g, b, s); break;
    case 10: launch_flux_tma_irec<10, T, S>(r, dir, tm, tmm, F, Fcopy, icopy, ilo, ihi, g, b, s); break;
    default: launch_flux_tma_irec<6, T, S>(r, dir, tm, tmm, F, Fcopy, icopy, ilo, ihi, g, b, s); break;
  }
}

cudaError_t launch_flux_tma(const DevRun& r, int dir, const void* tmap64, const void* tmap32, const void* tmapm,
                            double* F, cudaStream_t s) {
  const int lo = r.nm0, hi = r.imax - r.nm0;
  const CUtensorMap& t64 = *static_cast<const CUtensorMap*>(tmap64);
  const CUtensorMap& tm = *static_cast<const CUtensorMap*>(tmapm);
  if (!r.mixed) {
    launch_flux_tma_t<double, double>(r, dir, t64, tm, F, nullptr, 0, lo, hi, s);
  } else {
    // as launch_flux: FP64 faces up to i_fp64 + 1, copied to FP32 up to i_fp64; FP32 faces beyond
    const int split = fp64_split(r, lo, hi);
    if (split >= lo)
      launch_flux_tma_t<double, double>(r, dir, t64, tm, F, r.F32[dir - 1], split, lo, split < hi ? split + 1 : hi,
                                        s);
    launch_flux_tma_t<float, float>(r, dir, *static_cast<const CUtensorMap*>(tmap32), tm, r.F32[dir - 1], nullptr,
                                    0, split + 1, hi, s);
  }
  return cudaGetLastError();
}

// Box of the face-metric tensor map (i, k, component) of the staged FP64 face kernel.
void flux_tma_met_box(unsigned box[3]) {
  box[0] = TmaBox<1, double, 2>::MX;
  box[1] = 1;
  box[2] = kMetComps;
}

template <typename S, int LO>
static void tma_box_of(int dir, unsigned box[4]) {
  box[0] = dir == 1 ? TmaBox<1, S, LO>::X : (dir == 2 ? TmaBox<2, S, LO>::X : TmaBox<3, S, LO>::X);
  box[1] = dir == 1 ? TmaBox<1, S, LO>::Y : (dir == 2 ? TmaBox<2, S, LO>::Y : TmaBox<3, S, LO>::Y);
  box[2] = dir == 1 ? TmaBox<1, S, LO>::Z : (dir == 2 ? TmaBox<2, S, LO>::Z : TmaBox<3, S, LO>::Z);
  box[3] = 9;
}
void flux_tma_box(int dir, int elem_bytes, int irec, unsigned box[4]) {
  const bool ppm = (irec == 5);
  if (elem_bytes == 8) {
    if (ppm) tma_box_of<double, tma_lo<5>()>(dir, box);
    else tma_box_of<double, tma_lo<6>()>(dir, box);
  } else {
    if (ppm) tma_box_of<float, tma_lo<5>()>(dir, box);
    else tma_box_of<float, tma_lo<6>()>(dir, box);
  }
}

cudaError_t launch_flux(const DevRun& r, int dir, const double* P, double* F, cudaStream_t s) {
  const int lo = r.nm0, hi = r.imax - r.nm0;
  if (!r.mixed) {
    launch_flux_t<double, double>(r, dir, P, F, nullptr, 0, lo, hi, s);
  } else {
    // FP64 faces up to i_fp64 + 1 (flux-CT of the last FP64 edges reads them),
    // copied to FP32 up to i_fp64; FP32 faces from i_fp64 + 1 on.
    const int split = fp64_split(r, lo, hi);
    if (split >= lo)
      launch_flux_t<double, double>(r, dir, P, F, r.F32[dir - 1], split, lo, split < hi ? split + 1 : hi, s);
    launch_flux_t<float, float>(r, dir, r.P32, r.F32[dir - 1], nullptr, 0, split + 1, hi, s);
  }
  return cudaGetLastError();
}

template <int ICT>
static void launch_ct_t(const DevRun& r, const double* F1, const double* F2, const double* F3, double* CT,
                        cudaStream_t s) {
  const int lo = r.nm1, hi = r.imax - r.nm1, m = r.jmax - 2 * r.nm1 + 1, l = r.kmax - 2 * r.nm1 + 1;
  const dim3 b = sblock(r, dim3(64, 4, 1));
  if (!r.mixed) {
    k_ct<ICT, double, double><<<sgrid(r, hi - lo + 1, m, l, b), b, 0, s>>>(r, F1, F2, F3, CT, nullptr, lo, hi);
  } else {
    const int split = fp64_split(r, lo, hi);
    if (split >= lo)
      k_ct<ICT, double, double><<<sgrid(r, split - lo + 1, m, l, b), b, 0, s>>>(r, F1, F2, F3, CT, r.CT32, lo,
                                                                                  split);
    if (split < hi)
      k_ct<ICT, float, float><<<sgrid(r, hi - split, m, l, b), b, 0, s>>>(r, r.F32[0], r.F32[1], r.F32[2],
                                                                              r.CT32, nullptr, split + 1, hi);
  }
}

cudaError_t launch_ct(const DevRun& r, const double* P, const double* F1, const double* F2, const double* F3,
                      double* CT, cudaStream_t s) {
  if (r.ict == 0) {
    launch_ct_t<0>(r, F1, F2, F3, CT, s);
  } else if (r.ict == 2) {
    launch_ct_t<2>(r, F1, F2, F3, CT, s);
  } else if (r.ict == 3) {  // FP64 only (the run parameters exclude the mixed path)
    const int lo = r.nm0 + 1, hi_i = r.imax - r.nm0 - 2, hi_j = r.jmax - r.nm0 - 2, hi_k = r.kmax - r.nm0 - 2;
    const dim3 b = sblock(r, dim3(64, 4, 1));
    k_upct_diff<<<sgrid(r, hi_i - lo + 1, hi_j - lo + 1, hi_k - lo + 1, b), b, 0, s>>>(r, P, F1, F2, F3, hi_i,
                                                                                      hi_j, hi_k);
    const int clo = r.nm1, chi = r.imax - r.nm1, m = r.jmax - 2 * r.nm1 + 1, l = r.kmax - 2 * r.nm1 + 1;
    k_ct<3, double, double><<<sgrid(r, chi - clo + 1, m, l, b), b, 0, s>>>(r, F1, F2, F3, CT, nullptr, clo, chi);
  } else {
    launch_ct_t<1>(r, F1, F2, F3, CT, s);
  }
  return cudaGetLastError();
}

template <bool MIX>
static void launch_update_t(const DevRun& r, int stage, const double* Pn, const double* Pc, double* Pw,
                            const double* F1, const double* F2, const double* F3, const double* CT, int ilo,
                            int ihi, cudaStream_t s) {
  if (ihi < ilo) return;
  const dim3 b = sblock(r, dim3(RG_UPDATE_BX, 128 / RG_UPDATE_BX, 1));
  const dim3 g = sgrid(r, ihi - ilo + 1, r.jmax, r.kmax, b);
  if (stage == 1) k_update<1, MIX><<<g, b, 0, s>>>(r, Pn, Pc, Pw, F1, F2, F3, CT, ilo, ihi);
  else if (stage == 2) k_update<2, MIX><<<g, b, 0, s>>>(r, Pn, Pc, Pw, F1, F2, F3, CT, ilo, ihi);
  else k_update<3, MIX><<<g, b, 0, s>>>(r, Pn, Pc, Pw, F1, F2, F3, CT, ilo, ihi);
}

bool update_tma_eligible(const DevRun& r) {
  return !r.mixed && !r.jfix && !r.kfix && r.iwvec != 2 && (r.imax % 2) == 0 &&
         r.N == (size_t)r.imax * r.jmax * r.kmax;
}

void update_tma_box(int which, unsigned box[4]) {
  using B = UpdB;
  const unsigned x[5] = {B::X1, B::X2, B::X3, B::XC, B::XU}, y[5] = {B::Y1, B::Y2, B::Y3, B::YC, B::YU};
  const unsigned z[5] = {B::Z1, B::Z2, B::Z3, B::ZC, B::ZU};
  box[0] = x[which];
  box[1] = y[which];
  box[2] = z[which];
  box[3] = which == 3 ? 6 : 9;
}

cudaError_t prepare_update_tma() {
  const void* fns[3] = {reinterpret_cast<const void*>(k_update_tma<1>), reinterpret_cast<const void*>(k_update_tma<2>),
                        reinterpret_cast<const void*>(k_update_tma<3>)};
  for (const void* f : fns) {
    cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)UpdB::BYTES);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

bool update_tma_mix_eligible(const DevRun& r) {
  return r.mixed && !r.jfix && !r.kfix && r.iwvec != 2 && (r.imax % 4) == 0 &&
         r.N == (size_t)r.imax * r.jmax * r.kmax;
}

void update_tma_mix_box(int which, unsigned box[4]) {
  using B = UpdBoxMix;
  const unsigned x[5] = {B::X1, B::X2, B::X3, B::XC, B::XU}, y[5] = {B::Y1, B::Y2, B::Y3, B::YC, B::YU};
  const unsigned z[5] = {B::Z1, B::Z2, B::Z3, B::ZC, B::ZU};
  box[0] = x[which];
  box[1] = y[which];
  box[2] = z[which];
  box[3] = which == 3 ? 6 : 9;
}

template <int STAGE>
static void launch_update_tma_mix(const DevRun& r, const UpdMaps& maps, const double* Pc, double* Pw, int ilo,
                                  cudaStream_t s) {
  if (ilo > r.imax) return;
  const dim3 b(RG_UPDATE_BX, 128 / RG_UPDATE_BX, 1);
  const dim3 g = grid3(r.imax - ilo + 1, r.jmax, r.kmax, b);
  k_update_tma_mix<STAGE><<<g, b, UpdBoxMix::BYTES, s>>>(maps, r, Pc, Pw, ilo);
}

cudaError_t launch_update(const DevRun& r, int stage, const double* Pn, const double* Pc, double* Pw,
                          const double* F1, const double* F2, const double* F3, const double* CT, cudaStream_t s,
                          const void* umaps, const void* umaps_mix) {
  if (umaps && update_tma_eligible(r)) {
    UpdMaps maps;
    memcpy(&maps, umaps, sizeof maps);
    const dim3 b(RG_UPDATE_BX, 128 / RG_UPDATE_BX, 1);
    const dim3 g = grid3(r.imax, r.jmax, r.kmax, b);
    if (stage == 1) k_update_tma<1><<<g, b, UpdB::BYTES, s>>>(maps, r, Pc, Pw);
    else if (stage == 2) k_update_tma<2><<<g, b, UpdB::BYTES, s>>>(maps, r, Pc, Pw);
    else k_update_tma<3><<<g, b, UpdB::BYTES, s>>>(maps, r, Pc, Pw);
  } else if (!r.mixed) {
    launch_update_t<false>(r, stage, Pn, Pc, Pw, F1, F2, F3, CT, 1, r.imax, s);
  } else {
    const int split = fp64_split(r, 1, r.imax);
    launch_update_t<false>(r, stage, Pn, Pc, Pw, F1, F2, F3, CT, 1, split, s);
    if (umaps_mix && update_tma_mix_eligible(r)) {
      UpdMaps maps;
      memcpy(&maps, umaps_mix, sizeof maps);
      if (stage == 1) launch_update_tma_mix<1>(r, maps, Pc, Pw, split + 1, s);
      else if (stage == 2) launch_update_tma_mix<2>(r, maps, Pc, Pw, split + 1, s);
      else launch_update_tma_mix<3>(r, maps, Pc, Pw, split + 1, s);
    } else {
      launch_update_t<true>(r, stage, Pn, Pc, Pw, F1, F2, F3, CT, split + 1, r.imax, s);
    }
  }
  if (r.strag_list) {
    const unsigned gs = (unsigned)((r.strag_cap + 127) / 128);
    if (stage == 1) k_straggler<1><<<gs, 128, 0, s>>>(r, Pn, Pc, Pw, F1, F2, F3, CT);
    else if (stage == 2) k_straggler<2><<<gs, 128, 0, s>>>(r, Pn, Pc, Pw, F1, F2, F3, CT);
    else k_straggler<3><<<gs, 128, 0, s>>>(r, Pn, Pc, Pw, F1, F2, F3, CT);
  }
  if (stage == 1) k_carry_fix<0, 1><<<1, kCarryThreads, 0, s>>>(r, Pn, Pc, Pw, F1, F2, F3, CT, nullptr);
  else if (stage == 2) k_carry_fix<0, 2><<<1, kCarryThreads, 0, s>>>(r, Pn, Pc, Pw, F1, F2, F3, CT, nullptr);
  else k_carry_fix<0, 3><<<1, kCarryThreads, 0, s>>>(r, Pn, Pc, Pw, F1, F2, F3, CT, nullptr);
  return cudaGetLastError();
}

// Launches issued by launch_flux (per direction), launch_ct and launch_update.
int n_flux_launches(const DevRun& r) {
  if (!r.mixed) return 1;
  const int lo = r.nm0, hi = r.imax - r.nm0, split = fp64_split(r, lo, hi);
  return (split >= lo) + (split < hi);
}
int n_ct_launches(const DevRun& r) {
  if (r.ict == 3) return 2;
  if (!r.mixed) return 1;
  const int lo = r.nm1, hi = r.imax - r.nm1, split = fp64_split(r, lo, hi);
  return (split >= lo) + (split < hi);
}
int n_update_launches(const DevRun& r) {
  const int extra = 1 + (r.strag_list ? 1 : 0);  // carry fix, straggler pass
  if (!r.mixed) return 1 + extra;
  const int split = fp64_split(r, 1, r.imax);
  return (split >= 1) + (split < r.imax) + extra;
}

cudaError_t launch_to_f32(const double* a, float* b, size_t n, cudaStream_t s) {
  k_to_f32<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a, b, n);
  return cudaGetLastError();
}

static bool any_code(const DevRun& r, int side0, bool periodic) {
  for (int sd = side0; sd <= side0 + 1; ++sd)
    for (int v = 0; v < 9; ++v) {
      const int c = r.ibc[sd][v];
      if (periodic ? (c == 1) : (c != 1 && c != 0)) return true;
    }
  return false;
}

// Columns (n1 x n2) of a boundary pass; a transverse slab direction has one column.
static void bc_shape(int n1, int n2, bool fix1, bool fix2, dim3& g, dim3& b) {
  b = dim3(fix1 ? 1 : (fix2 ? 128 : 32), fix2 ? 1 : (fix1 ? 128 : 4), 1);
  g = grid3(fix1 ? 1 : n1, fix2 ? 1 : n2, 1, b);
}
// The standalone passes: one variable per grid z index.
static void bc_shape9(int n1, int n2, bool fix1, bool fix2, dim3& g, dim3& b) {
  bc_shape(n1, n2, fix1, fix2, g, b);
  g.z = 9;
}

int n_bc_launches(const DevRun& r) {
  int n = 0;
  for (int d = 0; d < 3; ++d) {
    const bool slab = (d == 1 && r.jfix) || (d == 2 && r.kfix);  // ghost fill of a slab plane is a no-op
    if (slab) continue;
    n += any_code(r, 2 * d, true) + any_code(r, 2 * d, false);
  }
  return n;
}

cudaError_t launch_bc(const DevRun& r, double* P, const double* Po, cudaStream_t s) {
  const int nm1 = r.nm1;
  const bool jf = r.jfix != 0, kf = r.kfix != 0;
  dim3 g, b;
  // periodic passes on interior columns (bndpefb4), then physical passes on all
  // columns (bndryfb4); a slab direction's own passes copy its plane onto itself
  if (any_code(r, 0, true)) {
    bc_shape9(r.jmax - 2 * nm1, r.kmax - 2 * nm1, jf, kf, g, b);
    k_bc_periodic<1><<<g, b, 0, s>>>(r, P);
  }
  if (!jf && any_code(r, 2, true)) {
    bc_shape9(r.imax - 2 * nm1, r.kmax - 2 * nm1, false, kf, g, b);
    k_bc_periodic<2><<<g, b, 0, s>>>(r, P);
  }
  if (!kf && any_code(r, 4, true)) {
    bc_shape9(r.imax - 2 * nm1, r.jmax - 2 * nm1, false, jf, g, b);
    k_bc_periodic<3><<<g, b, 0, s>>>(r, P);
  }
  if (any_code(r, 0, false)) {
    bc_shape9(r.jmax, r.kmax, jf, kf, g, b);
    k_bc_phys<1><<<g, b, 0, s>>>(r, P, Po);
  }
  if (!jf && any_code(r, 2, false)) {
    bc_shape9(r.imax, r.kmax, false, kf, g, b);
    k_bc_phys<2><<<g, b, 0, s>>>(r, P, Po);
  }
  if (!kf && any_code(r, 4, false)) {
    bc_shape9(r.imax, r.jmax, false, jf, g, b);
    k_bc_phys<3><<<g, b, 0, s>>>(r, P, Po);
  }
  return cudaGetLastError();
}

cudaError_t launch_floor(const DevRun& r, double* P, cudaStream_t s) {
  const dim3 b = sblock(r, dim3(RG_CELL_BX, 128 / RG_CELL_BX, 1));
  k_floor<<<sgrid(r, r.imax, r.jmax, r.kmax, b), b, 0, s>>>(r, P);
  return cudaGetLastError();
}

cudaError_t launch_recov_only(const DevRun& r, const double* U, const double* Pold, double* Pw, cudaStream_t s) {
  const dim3 b = sblock(r, dim3(64, 2, 1));
  if (r.iwvec == 2) {
    k_recov<2><<<sgrid(r, r.imax, r.jmax, r.kmax, b), b, 0, s>>>(r, U, Pold, Pw);
    k_carry_fix<1, 1, 2><<<1, kCarryThreads, 0, s>>>(r, nullptr, Pold, Pw, nullptr, nullptr, nullptr, nullptr, U);
  } else {
    k_recov<1><<<sgrid(r, r.imax, r.jmax, r.kmax, b), b, 0, s>>>(r, U, Pold, Pw);
    k_carry_fix<1, 1><<<1, kCarryThreads, 0, s>>>(r, nullptr, Pold, Pw, nullptr, nullptr, nullptr, nullptr, U);
  }
  return cudaGetLastError();
}

// A stage of a recov2 run in the reference's sequence (main.f90:807-899):
// the CT values written into the face fluxes (ct edits ww in place), the
// conserved variables of the stage's primitives (caluu1; those of P^n, the
// step's uo, kept from stage 1), the geometric source, the RK combine with
// the step's dt, then recov2 with its loop-order carry pass.
__global__ void k_ct_into_fluxes(DevRun r, const double* __restrict__ CT, double* __restrict__ F1,
                                 double* __restrict__ F2, double* __restrict__ F3) {
  const int nm1 = r.nm1;
  const int i = blockIdx.x * blockDim.x + threadIdx.x + nm1;
  const int j = jidx(r, nm1, blockIdx);
  const int k = kidx(r, nm1, blockIdx);
  if (i > r.imax - nm1 || j > r.jmax - nm1 || k > r.kmax - nm1) return;
  const size_t N = r.N, c = r.cell(i, j, k);
  // ww(2,7) ww(3,7) ww(1,8) ww(3,8) ww(1,9) ww(2,9)
  F2[6 * N + c] = CT[0 * N + c];
  F3[6 * N + c] = CT[1 * N + c];
  F1[7 * N + c] = CT[2 * N + c];
  F3[7 * N + c] = CT[3 * N + c];
  F1[8 * N + c] = CT[4 * N + c];
  F2[8 * N + c] = CT[5 * N + c];
}

cudaError_t launch_stage_recov2(const DevRun& r, int stage, const double* Pc, double* Pw, double* F1, double* F2,
                                double* F3, const double* CT, double* Uc, double* SF, double* Unew, cudaStream_t s) {
  const dim3 bc = sblock(r, dim3(64, 4, 1));
  const int n = r.imax - 2 * r.nm1 + 1, m = r.jmax - 2 * r.nm1 + 1, l = r.kmax - 2 * r.nm1 + 1;
  k_ct_into_fluxes<<<sgrid(r, n, m, l, bc), bc, 0, s>>>(r, CT, F1, F2, F3);
  const dim3 b = sblock(r, dim3(64, 2, 1));
  const dim3 g = sgrid(r, r.imax, r.jmax, r.kmax, b);
  double* Ucur = (stage == 1) ? r.Un : Uc;
  k_p2c<<<g, b, 0, s>>>(r, Pc, Ucur);
  k_calsf<<<g, b, 0, s>>>(r, Pc, SF);
  if (stage == 1) k_rkt<1><<<g, b, 0, s>>>(r, F1, F2, F3, r.Un, Ucur, SF, Unew, 0.0, true);
  else if (stage == 2) k_rkt<2><<<g, b, 0, s>>>(r, F1, F2, F3, r.Un, Ucur, SF, Unew, 0.0, true);
  else k_rkt<3><<<g, b, 0, s>>>(r, F1, F2, F3, r.Un, Ucur, SF, Unew, 0.0, true);
  k_recov<2><<<g, b, 0, s>>>(r, Unew, Pc, Pw);
  k_carry_fix<1, 1, 2><<<1, kCarryThreads, 0, s>>>(r, nullptr, Pc, Pw, nullptr, nullptr, nullptr, nullptr, Unew);
  return cudaGetLastError();
}

cudaError_t launch_p2c(const DevRun& r, const double* P, double* U, cudaStream_t s) {
  const dim3 b = sblock(r, dim3(64, 2, 1));
  k_p2c<<<sgrid(r, r.imax, r.jmax, r.kmax, b), b, 0, s>>>(r, P, U);
  return cudaGetLastError();
}

cudaError_t launch_output1(const DevRun& r, const double* P, const double* cx, const double* cy, const double* cz,
                           size_t rec0, size_t nrec, unsigned* out, cudaStream_t s) {
  if (nrec == 0) return cudaSuccess;
  k_output1<<<(unsigned)((nrec + 127) / 128), 128, 0, s>>>(r, P, cx, cy, cz, rec0, nrec, out);
  return cudaGetLastError();
}
template <int D>
static void launch_rec2_d(const DevRun& r, const double* P, double* F, const FaceOut& fo, dim3 g, dim3 b,
                          cudaStream_t s) {
  switch (r.irec) {
    case 1: k_rec2<D, 1><<<g, b, 0, s>>>(r, P, F, fo); break;
    case 2: k_rec2<D, 2><<<g, b, 0, s>>>(r, P, F, fo); break;
    case 3: k_rec2<D, 3><<<g, b, 0, s>>>(r, P, F, fo); break;
    case 4: k_rec2<D, 4><<<g, b, 0, s>>>(r, P, F, fo); break;
    case 5: k_rec2<D, 5><<<g, b, 0, s>>>(r, P, F, fo); break;
    case 6: k_rec2<D, 6><<<g, b, 0, s>>>(r, P, F, fo); break;
    case 7: k_rec2<D, 7><<<g, b, 0, s>>>(r, P, F, fo); break;
    case 8: k_rec2<D, 8><<<g, b, 0, s>>>(r, P, F, fo); break;
    case 9: k_rec2<D, 9><<<g, b, 0, s>>>(r, P, F, fo); break;
    case 10: k_rec2<D, 10><<<g, b, 0, s>>>(r, P, F, fo); break;
    case 11: k_rec2<D, 11><<<g, b, 0, s>>>(r, P, F, fo); break;
    case 12: k_rec2<D, 12><<<g, b, 0, s>>>(r, P, F, fo); break;
    default: k_rec2<D, 13><<<g, b, 0, s>>>(r, P, F, fo); break;
  }
}

cudaError_t launch_rec2(const DevRun& r, int dir, const double* P, double* F, double* const q[2], double* const u[2],
                        double* const w[2], cudaStream_t s) {
  const int n = r.imax - 2 * r.nm0 + 1, m = r.jmax - 2 * r.nm0 + 1, l = r.kmax - 2 * r.nm0 + 1;
  const dim3 b(64, 2, 1);
  const dim3 g = grid3(2 * n, m, l, b);
  const FaceOut fo{{q[0], q[1]}, {u[0], u[1]}, {w[0], w[1]}};
  if (dir == 1) launch_rec2_d<1>(r, P, F, fo, g, b, s);
  else if (dir == 2) launch_rec2_d<2>(r, P, F, fo, g, b, s);
  else launch_rec2_d<3>(r, P, F, fo, g, b, s);
  return cudaGetLastError();
}

cudaError_t launch_calcha(const DevRun& r, int dir, const double* QL, const double* QR, double* cmax, double* cmin,
                          cudaStream_t s) {
  const dim3 b(64, 2, 1);
  const dim3 g = grid3(r.imax - 2 * r.nm0 + 1, r.jmax - 2 * r.nm0 + 1, r.kmax - 2 * r.nm0 + 1, b);
  if (dir == 1) k_calcha<1><<<g, b, 0, s>>>(r, QL, QR, cmax, cmin);
  else if (dir == 2) k_calcha<2><<<g, b, 0, s>>>(r, QL, QR, cmax, cmin);
  else k_calcha<3><<<g, b, 0, s>>>(r, QL, QR, cmax, cmin);
  return cudaGetLastError();
}

cudaError_t launch_hll(const DevRun& r, int dir, const double* UL, const double* UR, const double* WL,
                       const double* WR, const double* CX, const double* CN, double* F, cudaStream_t s) {
  const dim3 b(64, 2, 1);
  const dim3 g = grid3(r.imax - 2 * r.nm0 + 1, r.jmax - 2 * r.nm0 + 1, r.kmax - 2 * r.nm0 + 1, b);
  if (dir == 1) k_hll<1><<<g, b, 0, s>>>(r, UL, UR, WL, WR, CX, CN, F);
  else if (dir == 2) k_hll<2><<<g, b, 0, s>>>(r, UL, UR, WL, WR, CX, CN, F);
  else k_hll<3><<<g, b, 0, s>>>(r, UL, UR, WL, WR, CX, CN, F);
  return cudaGetLastError();
}

__global__ void k_aos_planes(double* __restrict__ aos, double* __restrict__ planes, size_t N, int m, int to_planes) {
  const size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  for (int a = 0; a < m; ++a) {
    if (to_planes) planes[(size_t)a * N + c] = aos[(size_t)m * c + a];
    else aos[(size_t)m * c + a] = planes[(size_t)a * N + c];
  }
}
cudaError_t launch_aos_planes(double* aos, double* planes, size_t N, int m, bool to_planes, cudaStream_t s) {
  k_aos_planes<<<(unsigned)((N + 127) / 128), 128, 0, s>>>(aos, planes, N, m, to_planes ? 1 : 0);
  return cudaGetLastError();
}
cudaError_t launch_ww_layout(double* ww, double* F1, double* F2, double* F3, size_t N, bool to_planes,
                             cudaStream_t s) {
  k_ww_layout<<<(unsigned)((N + 127) / 128), 128, 0, s>>>(ww, F1, F2, F3, N, to_planes ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_ct_apply(const DevRun& r, const double* CT, double* F1, double* F2, double* F3, cudaStream_t s) {
  const dim3 b(64, 2, 1);
  k_ct_apply<<<grid3(r.imax, r.jmax, r.kmax, b), b, 0, s>>>(r, CT, F1, F2, F3);
  return cudaGetLastError();
}

cudaError_t launch_floor_part(const DevRun& r, int part, double* P, cudaStream_t s) {
  const dim3 b = sblock(r, dim3(64, 2, 1));
  const dim3 g = sgrid(r, r.imax, r.jmax, r.kmax, b);
  if (part == 1) k_floor_part<1><<<g, b, 0, s>>>(r, P);
  else if (part == 2) k_floor_part<2><<<g, b, 0, s>>>(r, P);
  else k_floor_part<4><<<g, b, 0, s>>>(r, P);
  return cudaGetLastError();
}

cudaError_t launch_divb(const DevRun& r, const double* P, unsigned long long* red, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(red, 0, 2 * sizeof(unsigned long long), s);
  if (e != cudaSuccess) return e;
  k_divb<<<148 * 4, 256, 0, s>>>(r, P, red);
  return cudaGetLastError();
}
cudaError_t launch_calsf(const DevRun& r, const double* P, double* SF, cudaStream_t s) {
  const dim3 b = sblock(r, dim3(64, 2, 1));
  k_calsf<<<sgrid(r, r.imax, r.jmax, r.kmax, b), b, 0, s>>>(r, P, SF);
  return cudaGetLastError();
}

cudaError_t launch_derived(const DevRun& r, const double* P, const double* geo_i, const double* geo_k, double akm,
                           int jslice, double* out, cudaStream_t s) {
  const dim3 b(64, 1, 2);
  const dim3 g = grid3(r.imax, jslice ? 1 : r.jmax, r.kmax, b);
  k_derived<<<g, b, 0, s>>>(r, P, geo_i, geo_k, akm, jslice, out);
  return cudaGetLastError();
}

cudaError_t launch_rkt(const DevRun& r, int stage, const double* W1, const double* W2, const double* W3,
                       const double* Uo, const double* Uc, const double* SF, double* Unew, double dt, cudaStream_t s) {
  const dim3 b = sblock(r, dim3(64, 2, 1));
  const dim3 g = sgrid(r, r.imax, r.jmax, r.kmax, b);
  if (stage == 1) k_rkt<1><<<g, b, 0, s>>>(r, W1, W2, W3, Uo, Uc, SF, Unew, dt);
  else if (stage == 2) k_rkt<2><<<g, b, 0, s>>>(r, W1, W2, W3, Uo, Uc, SF, Unew, dt);
  else k_rkt<3><<<g, b, 0, s>>>(r, W1, W2, W3, Uo, Uc, SF, Unew, dt);
  return cudaGetLastError();
}

cudaError_t launch_aos_to_soa(const DevRun& r, const double* aos, double* soa, int* bad, cudaStream_t s) {
  const size_t n = (size_t)r.imax * r.jmax * r.kmax;
  k_aos_to_soa<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(r, aos, soa, bad);
  return cudaGetLastError();
}
cudaError_t launch_soa_to_aos(const DevRun& r, const double* soa, double* aos, cudaStream_t s) {
  const size_t n = (size_t)r.imax * r.jmax * r.kmax;
  k_soa_to_aos<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(r, soa, aos);
  return cudaGetLastError();
}
cudaError_t launch_geom_derive(const DevRun& r, double* mc, double* mi, double* mk, double* fl_de, double* fl_pr,
                               cudaStream_t s) {
  const size_t n = r.nik > (size_t)r.imax ? r.nik : (size_t)r.imax;
  k_geom_derive<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(r, mc, mi, mk, fl_de, fl_pr);
  return cudaGetLastError();
}
cudaError_t launch_fill(double* p, double v, size_t n, cudaStream_t s) {
  k_fill<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(p, v, n);
  return cudaGetLastError();
}

#include "rg_batch.cuh"

}  // namespace rg
