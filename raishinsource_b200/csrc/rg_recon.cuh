// rg_recon.cuh -- face reconstruction of rec.f90 (MP5, WENO5, PPM) as device
// functions templated on the arithmetic type T (see rg_device.cuh).
#pragma once

namespace rg {

// rec.f90:2346-2370.  dmm = 0.5*(sign(1,x)+sign(1,y))*min(|x|,|y|) and
// dm4 = 0.125*(sw+sx)*|sw+sy|*(sw+sz)*min(|w|,|x|,|y|,|z|) (s = sign(1,.);
// note the reference's abs covers only the middle factor, so dm4 is +min
// when all four signs agree, whatever that sign).  The sign factors are
// +-1 or a signed zero, so the products are evaluated here as selects on the
// sign bits: the same values bit for bit (signed zeros and NaN included) with
// the FP64 arithmetic reduced to the min and one multiply.
template <typename T>
__device__ __forceinline__ T dmm(T xx, T yy) {
  const T mn = dmin2(mabs(xx), mabs(yy));
  // same signs: 0.5*(+-2)*mn = +-mn; otherwise 0.5*(+0)*mn = +0 (or NaN)
  return (signbit(xx) == signbit(yy)) ? copysign(mn, xx) : T(0) * mn;
}
template <typename T>
__device__ __forceinline__ T dm4(T ww, T xx, T yy, T zz) {
  T mn = mabs(ww);
  if (mabs(xx) < mn) mn = mabs(xx);
  if (mabs(yy) < mn) mn = mabs(yy);
  if (mabs(zz) < mn) mn = mabs(zz);
  const bool nw = signbit(ww);
  const bool az = nw != signbit(xx), bz = nw != signbit(yy), cz = nw != signbit(zz);
  if (!az && !bz && !cz) return mn;  // 0.125 * (2 sw) * 2 * (2 sw) = +1
  // a zero factor: the product ((0.125*A)*B)*C*mn is a zero with the sign of
  // A times the sign of C, where A = sw+sx and C = sw+sz are +0 when their
  // signs differ and 2 sw otherwise (B = |sw+sy| >= 0 keeps the sign)
  const bool neg = (!az && nw) != (!cz && nw);
  return (neg ? T(-0.0) : T(0)) * mn;
}

// rec.f90:2095-2178: MP5 face state of cell 0 from u(-2..+2) given in the
// order (a2, a1, u0, b1, b2): the left state at +1/2 takes
// (u-2, u-1, u0, u+1, u+2) and sg = +1; the right state at -1/2 takes the
// mirrored stencil (u+2, u+1, u0, u-1, u-2) and sg = -1, because the
// reference's right state flips the signs of the dm4 terms of md and lc
// (rec.f90:2172-2176).  Negation is exact, so both equal the reference's
// separate formulas bit for bit, and the two lanes of a face run one code path.
// The second differences are the exception: the reference evaluates them once
// per cell in stencil order, (u-2 - 2 u-1) + u0, (u-1 - 2 u0) + u+1 and
// (u0 - 2 u+1) + u+2, for both states, and a sum taken in the mirrored order
// can round differently; the right state therefore picks its operands so
// that each difference is summed as the reference sums it.
template <typename T>
__device__ __forceinline__ T mp_limit(T ul1, T a2, T a1, T u0, T b1, T b2, T sg) {
  const T tmp2 = T(4.0) / T(3.0), alpha = T(4.0), eps1 = T(1.0e-10);
  const T ulmp = u0 + dmm(b1 - u0, alpha * (u0 - a1));
  const T t = (ul1 - u0) * (ul1 - ulmp);
  if (t <= eps1) return ul1;
  const bool right = sg < T(0);
  // left: dim1 = (a2 - 2 a1) + u0, di1 = (a1 - 2 u0) + b1, dip1 = (u0 - 2 b1) + b2;
  // right (a = u+, b = u-): dim1 = (u0 - 2 a1) + a2, di1 = (b1 - 2 u0) + a1, dip1 = (b2 - 2 b1) + u0
  const T dim1 = (right ? u0 : a2) - T(2.) * a1 + (right ? a2 : u0);
  const T di1 = (right ? b1 : a1) - T(2.) * u0 + (right ? a1 : b1);
  const T dip1 = (right ? b2 : u0) - T(2.) * b1 + (right ? u0 : b2);
  const T dm4p = dm4(T(4.) * di1 - dip1, T(4.) * dip1 - di1, di1, dip1);
  const T dm4m = dm4(T(4.) * di1 - dim1, T(4.) * dim1 - di1, di1, dim1);
  const T ul = u0 + alpha * (u0 - a1);
  const T av = T(0.5) * (u0 + b1);
  const T md = av - (sg * T(0.5)) * dm4p;
  const T lc = u0 + T(0.5) * (u0 - a1) + (sg * tmp2) * dm4m;
  const T m1 = fmin3(u0, b1, md), m2 = fmin3(u0, ul, lc);
  const T m3 = fmax3(u0, b1, md), m4 = fmax3(u0, ul, lc);
  const T umax = dmax2(m1, m2), umin = dmin2(m3, m4);
  return ul1 + dmm(umin - ul1, umax - ul1);
}
template <typename T>
__device__ __forceinline__ T mp5_state(T a2, T a1, T u0, T b1, T b2, T sg) {
  const T tmp1 = T(1.0) / T(60.0);
  const T ul1 = tmp1 * (T(2.) * a2 - T(13.) * a1 + T(47.) * u0 + T(27.) * b1 - T(3.) * b2);
  return mp_limit(ul1, a2, a1, u0, b1, b2, sg);
}

// rec.f90:2373-2643 (WENO5-JS); the left state at +1/2 takes
// (u-2, u-1, u0, u+1, u+2), the right state at -1/2 the mirrored stencil.
// (13./12.) is a single-precision literal in the reference.
// b1s is the value the smoothness indicator beta_1 reads in place of b1: b1
// itself, except in mpweno5's radial right state (rec.f90:2757, see face_lane).
template <typename T>
__device__ __forceinline__ T weno5_js(T a2, T a1, T u0, T b1, T b2, T b1s) {
  const T cd0 = T(1.0 / 10.0), cd1 = T(6.0 / 10.0), cd2 = T(3.0 / 10.0);
  const T c00 = T(2.0 / 6.0), c01 = T(-7.0 / 6.0), c02 = T(11.0 / 6.0);
  const T c10 = T(-1.0 / 6.0), c11 = T(5.0 / 6.0), c12 = T(2.0 / 6.0);
  const T c20 = T(2.0 / 6.0), c21 = T(5.0 / 6.0), c22 = T(-1.0 / 6.0);
  const T epsi = T(1.0e-6), c1312 = T((double)(13.0f / 12.0f)), c14 = T(0.25);
  const T s0 = a2 - T(2.) * a1 + u0, t0 = a2 - T(4.) * a1 + T(3.) * u0;
  const T s1 = a1 - T(2.) * u0 + b1s, t1 = a1 - b1;
  const T s2 = u0 - T(2.) * b1 + b2, t2 = T(3.) * u0 - T(4.) * b1 + b2;
  const T be0 = c1312 * (s0 * s0) + c14 * (t0 * t0) + epsi;
  const T be1 = c1312 * (s1 * s1) + c14 * (t1 * t1) + epsi;
  const T be2 = c1312 * (s2 * s2) + c14 * (t2 * t2) + epsi;
  const T w0 = cd0 / (be0 * be0), w1 = cd1 / (be1 * be1), w2 = cd2 / (be2 * be2);
  const T wt = w0 + w1 + w2;
  const T o0 = w0 / wt, o1 = w1 / wt, o2 = w2 / wt;
  const T q0 = c00 * a2 + c01 * a1 + c02 * u0;
  const T q1 = c10 * a1 + c11 * u0 + c12 * b1;
  const T q2 = c20 * u0 + c21 * b1 + c22 * b2;
  return o0 * q0 + o1 * q1 + o2 * q2;
}
template <typename T>
__device__ __forceinline__ T weno5_state(T a2, T a1, T u0, T b1, T b2) {
  return weno5_js(a2, a1, u0, b1, b2, b1);
}

// rec.f90:3161-3436 (WENO-Z, Borges et al. 2008): WENO5 with the weights
// cd_m (1 + tau / (beta_m + eps)), tau = |beta_0 - beta_2|, the smoothness
// indicators without eps; p0 = 1 makes (beta + eps)**p0 the plain sum.
template <typename T>
__device__ __forceinline__ T weno5z_state(T a2, T a1, T u0, T b1, T b2) {
  const T cd0 = T(1.0 / 10.0), cd1 = T(6.0 / 10.0), cd2 = T(3.0 / 10.0);
  const T c00 = T(2.0 / 6.0), c01 = T(-7.0 / 6.0), c02 = T(11.0 / 6.0);
  const T c10 = T(-1.0 / 6.0), c11 = T(5.0 / 6.0), c12 = T(2.0 / 6.0);
  const T c20 = T(2.0 / 6.0), c21 = T(5.0 / 6.0), c22 = T(-1.0 / 6.0);
  const T epsi = T(1.0e-6), c1312 = T((double)(13.0f / 12.0f)), c14 = T(0.25);
  const T s0 = a2 - T(2.) * a1 + u0, t0 = a2 - T(4.) * a1 + T(3.) * u0;
  const T s1 = a1 - T(2.) * u0 + b1, t1 = a1 - b1;
  const T s2 = u0 - T(2.) * b1 + b2, t2 = T(3.) * u0 - T(4.) * b1 + b2;
  const T be0 = c1312 * (s0 * s0) + c14 * (t0 * t0);
  const T be1 = c1312 * (s1 * s1) + c14 * (t1 * t1);
  const T be2 = c1312 * (s2 * s2) + c14 * (t2 * t2);
  const T tau = mabs(be0 - be2);
  const T w0 = cd0 * (T(1.0) + tau / (be0 + epsi));
  const T w1 = cd1 * (T(1.0) + tau / (be1 + epsi));
  const T w2 = cd2 * (T(1.0) + tau / (be2 + epsi));
  const T wt = w0 + w1 + w2;
  const T o0 = w0 / wt, o1 = w1 / wt, o2 = w2 / wt;
  const T q0 = c00 * a2 + c01 * a1 + c02 * u0;
  const T q1 = c10 * a1 + c11 * u0 + c12 * b1;
  const T q2 = c20 * u0 + c21 * b1 + c22 * b2;
  return o0 * q0 + o1 * q1 + o2 * q2;
}

// rec.f90:3439-3793 (mapped WENO5, Henrick et al. 2005): the JS weights
// cd_m / (beta_m + eps)^2 with eps = 1e-40, normalised, mapped by
// g_m(w) = w (cd_m + cd_m^2 - 3 cd_m w + w^2) / (cd_m^2 + w (1 - 2 cd_m)) and
// normalised again.
template <typename T>
__device__ __forceinline__ T weno5m_state(T a2, T a1, T u0, T b1, T b2) {
  const T cd[3] = {T(1.0 / 10.0), T(6.0 / 10.0), T(3.0 / 10.0)};
  const T c00 = T(2.0 / 6.0), c01 = T(-7.0 / 6.0), c02 = T(11.0 / 6.0);
  const T c10 = T(-1.0 / 6.0), c11 = T(5.0 / 6.0), c12 = T(2.0 / 6.0);
  const T c20 = T(2.0 / 6.0), c21 = T(5.0 / 6.0), c22 = T(-1.0 / 6.0);
  const T epsi = T(1.0e-40), c1312 = T((double)(13.0f / 12.0f)), c14 = T(0.25);
  const T s0 = a2 - T(2.) * a1 + u0, t0 = a2 - T(4.) * a1 + T(3.) * u0;
  const T s1 = a1 - T(2.) * u0 + b1, t1 = a1 - b1;
  const T s2 = u0 - T(2.) * b1 + b2, t2 = T(3.) * u0 - T(4.) * b1 + b2;
  const T be[3] = {c1312 * (s0 * s0) + c14 * (t0 * t0), c1312 * (s1 * s1) + c14 * (t1 * t1),
                   c1312 * (s2 * s2) + c14 * (t2 * t2)};
  T wa[3], g[3];
#pragma unroll
  for (int m = 0; m < 3; ++m) wa[m] = cd[m] / ((be[m] + epsi) * (be[m] + epsi));
  const T wat = wa[0] + wa[1] + wa[2];
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    const T w = wa[m] / wat;
    g[m] = w * (cd[m] + cd[m] * cd[m] - T(3.) * cd[m] * w + w * w) / (cd[m] * cd[m] + w * (T(1.) - T(2.) * cd[m]));
  }
  const T gt = g[0] + g[1] + g[2];
  const T o0 = g[0] / gt, o1 = g[1] / gt, o2 = g[2] / gt;
  const T q0 = c00 * a2 + c01 * a1 + c02 * u0;
  const T q1 = c10 * a1 + c11 * u0 + c12 * b1;
  const T q2 = c20 * u0 + c21 * b1 + c22 * b2;
  return o0 * q0 + o1 * q1 + o2 * q2;
}

// The second-order limiters of rec.f90 on nonuniform coordinates: mclim
// (irec 1, rec.f90:208-367), minlim (2, 568-739), lim03a (11, 4037-4267),
// mvllim (12, 4269-4477) and koren (13, 4480-4697).  One cell's state on the
// side `side` (0: left state at its +1/2 face, 1: right state at its -1/2
// face) from its neighbours um, up and the per-index coefficients co[6] of
// its coordinate (small = 1e-12, a = x_p - x_c + small, b = x_c - x_m + small,
// c = xa_p - x_c + small, d = x_c - xa_m + small):
//   irec 1, 2, 11: (1/a, 1/b, -, -, xa_p - x_c, x_c - xa_m)
//   irec 13:       (1/a, 1/b, a (1/c), b (1/d), xa_p - x_c, x_c - xa_m)
//   irec 12:       (a, b, a/c, b/d, c, d)
// MAX/MIN follow Fortran's order (the first argument seeds the result).
// tmp_b is the sign used in koren's backward slope: the reference takes the
// i-direction sign there in its j sweep (rec.f90:4628), else the cell's own.
template <int IREC, typename T>
__device__ __forceinline__ T limiter_state(T um, T u0, T up, const T co[6], int side, T tmp_b) {
  const T s3 = T(1.0 / 3.0);
  if (IREC == 12) {
    const T sp = (up - u0) / co[0], sm = (u0 - um) / co[1];
    T dk = T(0);
    if (!(sp * sm <= T(0))) {
      const T t = sm * sm + (co[2] + co[3] - T(2)) * sm * sp + sp * sp;
      dk = (sm * sp * (co[2] * sm + co[3] * sp)) / (t + T(1.0e-12));
    }
    return side ? u0 - dk * co[5] : u0 + dk * co[4];
  }
  const T sp = (up - u0) * co[0], sm = (u0 - um) * co[1];
  const T tmp = (sp < T(0)) ? T(-1) : T(1);
  T dk;
  if (IREC == 1) {
    dk = tmp * dmax2(T(0), fmin3(T(2) * mabs(sp), tmp * T(2) * sm, tmp * T(0.5) * (sp + sm)));
  } else if (IREC == 2) {
    dk = tmp * dmax2(T(0), dmin2(mabs(sp), tmp * sm));
  } else if (IREC == 11) {
    const T al = T(0.5), be = T(2), ga = T(1.6);
    if (side) {
      const T e = (T(2) * mabs(sp) + tmp * sm) * s3;
      dk = dmax2(T(0), dmin2(e, dmax2(-al * sm * tmp, fmin3(be * sm * tmp, e, ga * mabs(sp)))));
    } else {
      const T e = (mabs(sp) + tmp * T(2) * sm) * s3;
      dk = dmax2(T(0), dmin2(e, dmax2(-al * mabs(sp), fmin3(be * mabs(sp), e, ga * tmp * sm))));
    }
  } else {  // 13
    const T e = side ? (mabs(sp) + T(2) * tmp_b * sm) * s3 : (T(2) * mabs(sp) + tmp * sm) * s3;
    dk = tmp * dmax2(T(0), fmin3(mabs(co[2] * sp), tmp * co[3] * sm, e));
  }
  return side ? u0 - dk * co[5] : u0 + dk * co[4];
}

// rec.f90:742-1258 (ceno, irec 4, convex ENO): one cell's state on side
// `side` from u(-2..+2) along the direction and the per-index coefficients
// co[10] of its physical coordinate x (rg_capi.cu, ceno_coefs): the minmod
// state u1, three quadratic candidates (centred at the cell before, at and
// after it), their deviations from u1 weighted by (1, 0.7, 1), and the
// candidate of smallest deviation when all three deviate the same way.
// kquirk drops the third candidate from the negative branch, as the
// reference's theta sweep compares |dklp| with itself there (rec.f90:1211).
template <typename T>
__device__ __forceinline__ T ceno_state(T um2, T um, T u0, T up, T up2, const T co[10], int side, bool kquirk) {
  const T sp = (up - u0) / co[0], sm = (u0 - um) / co[1];
  T dk = T(0);
  if (!(sp * sm <= T(0))) {
    const T tmp = (sp < T(0)) ? T(-1) : T(1);
    dk = tmp * dmin2(mabs(sp), mabs(sm));
  }
  const T u1 = side ? u0 - dk * co[3] : u0 + dk * co[2];
  const T d2m = T(0.5) * (u0 - um2), d20 = T(0.5) * (up - um), d2p = T(0.5) * (up2 - u0);
  const T d3m = u0 - T(2.0) * um + um2, d30 = up - T(2.0) * u0 + um, d3p = up2 - T(2.0) * up + u0;
  const T tm = side ? co[7] : co[4], t0 = side ? co[8] : co[5], tp = side ? co[9] : co[6];
  const T cm = u0 + d2m * tm + T(0.5) * d3m * (tm * tm);
  const T c0 = u0 + d20 * t0 + T(0.5) * d30 * (t0 * t0);
  const T cp = u0 + d2p * tp + T(0.5) * d3p * (tp * tp);
  const T dm = T(1.0) * (cm - u1), d0 = T(0.7) * (c0 - u1), dp = T(1.0) * (cp - u1);
  T out = u1;
  if (dp > T(0) && d0 > T(0) && dm > T(0)) {
    out = cm;
    if (mabs(d0) < mabs(dm) && mabs(d0) < mabs(dp)) out = c0;
    if (mabs(dp) < mabs(dm) && mabs(dp) < mabs(d0)) out = cp;
  }
  if (dm < T(0) && d0 < T(0) && dp < T(0)) {
    out = cm;
    if (mabs(d0) < mabs(dm) && mabs(d0) < mabs(dp)) out = c0;
    if (!kquirk && mabs(dp) < mabs(dm) && mabs(dp) < mabs(d0)) out = cp;
  }
  return out;
}

// rec.f90:145-205 (muscl, irec 3, beta = 1/3, no limiter): the left state of
// a cell at its +1/2 face (side 0) and its right state at its -1/2 face
// (side 1; the reference stores it as uriir of the face's left cell).
template <typename T>
__device__ __forceinline__ T muscl_state(T um, T u0, T up, int side) {
  const T beta = T(1.0 / 3.0);
  if (side) return u0 - T(0.25) * ((T(1.0) + beta) * (u0 - um) + (T(1.0) - beta) * (up - u0));
  return u0 + T(0.25) * ((T(1.0) + beta) * (up - u0) + (T(1.0) - beta) * (u0 - um));
}

// ------------------------------------------------------------------- PPM
// rPPM of Marti & Muller (1996) as restated by rec.f90:1261-2058.  The four
// passes (interp, detect, flaten, monoto) touch only the two face states of
// one cell each, so both states of cell c follow from the cells c-3..c+3:
// L = state at c-1/2 (the reference's uriir(c-1)), R = state at c+1/2
// (uriil(c)).  dx is rec2's shifted dx?b (dummy dx?b(m) = actual dx?b(m-1),
// rec.f90:58), x the cell centres (contact detection).

// interp Eq. (60)-(61) (rec.f90:1346-1418); the theta direction lacks the
// factor 2 of r and phi (rec.f90:1414).
template <typename T>
__device__ __forceinline__ T ppm_dma(T um, T u0, T up, T dxm, T dx0, T dxp, bool kdir) {
  const T t1a = dx0 / (dxm + dx0 + dxp);
  const T t1b = (T(2.0) * dxm + dx0) / (dxp + dx0);
  const T t1c = (dx0 + T(2.0) * dxp) / (dxm + dx0);
  const T sp1 = up - u0, sm1 = u0 - um;
  const T spm1 = sp1 * sm1;
  const T da = t1a * (t1b * sp1 + t1c * sm1);
  if (spm1 <= T(0)) return T(0);
  const T t1 = (da < T(0)) ? T(-1) : T(1);
  const T t1d = dmin2(mabs(sm1), mabs(sp1));
  return kdir ? t1 * dmin2(mabs(da), t1d) : t1 * dmin2(mabs(da), T(2.0) * t1d);
}

// interp Eq. (51) (rec.f90:1422-1468): interface value at c+1/2.
template <typename T>
__device__ __forceinline__ T ppm_face(T u0, T u1, T dma0, T dma1, T dxm, T dx0, T dx1, T dx2) {
  const T t2 = (dx0 / (dx0 + dx1)) * (u1 - u0);
  const T t3a = T(1.0) / (dxm + dx0 + dx1 + dx2);
  const T t3b = (T(2.0) * dx1 * dx0) / (dx0 + dx1);
  const T t3c = ((dxm + dx0) / (T(2.0) * dx0 + dx1)) - ((dx2 + dx1) / (T(2.0) * dx1 + dx0));
  const T t3 = t3a * t3b * t3c * (u1 - u0);
  const T t4 = t3a * dx0 * ((dxm + dx0) / (T(2.0) * dx0 + dx1));
  const T t5 = t3a * dx1 * ((dx1 + dx2) / (dx0 + T(2.0) * dx1));
  return u0 + t2 + t3 - t4 * dma1 + t5 * dma0;
}

// Both face states of the cell at p (primitive v at p[v*N], storage type S),
// stride st along direction D; dx[o+4], x[o+4] are the shifted spacing and
// centre at offset o from the cell.  gam enters the contact test (rec.f90:1623).
// ALL: also the sixth variable (the per-routine rec2 outputs every face state).
template <int D, typename T, typename S, bool ALL = false>
__device__ void ppm_cell(const S* __restrict__ p, size_t N, long long st, const T dx[9], const T x[9], T gam,
                         T L[9], T R[9]) {
  auto U = [&](int v, int o) { return T(p[(size_t)v * N + o * st]); };
  auto DX = [&](int o) { return dx[o + 4]; };
  // detect (rec.f90:1479-1686): contact steepening factor eta on density
  T eta;
  {
    const T eta1 = T(5.0), eta2 = T(0.05), eps1 = T(0.1), ak0 = T(1.0);
    auto dda = [&](int o) {
      const T t0a = T(1.0) / (DX(o - 1) + DX(o) + DX(o + 1));
      const T t0b = (U(0, o + 1) - U(0, o)) / (DX(o + 1) + DX(o));
      const T t0c = (U(0, o) - U(0, o - 1)) / (DX(o) + DX(o - 1));
      return t0a * (t0b - t0c);
    };
    const T ddp = dda(1), ddm = dda(-1);
    const T rp = U(0, 1), rm = U(0, -1);
    const T t1 = ddp * ddm;
    const T t2 = mabs(rp - rm) - eps1 * dmin2(mabs(rp), mabs(rm));
    T etatil;
    if (t1 >= T(0) && t2 <= T(0)) {
      etatil = T(0);
    } else {
      const T t2a = -(ddp - ddm) / (x[5] - x[3]);
      const T a = x[4] - x[3], b = x[5] - x[4];
      const T t2b = (a * a * a + b * b * b) / (rp - rm);
      etatil = t2a * t2b;
    }
    eta = dmax2(T(0), dmin2(eta1 * (etatil - eta2), T(1)));
    const T pp = U(4, 1), pm = U(4, -1);
    const T t3 = mabs(rp - rm) / dmin2(rp, rm);
    const T t4 = mabs(pp - pm) / dmin2(pp, pm);
    if (gam * ak0 * t3 < t4) eta = T(0);
  }
  // flaten (rec.f90:1689-1884): shock flattening f2a from p and u^D
  T f2a;
  {
    const T eps2 = T(1.0), omg2 = T(0.52), omg3 = T(10.0);
    auto f1a = [&](int o) {
      const T pp1 = U(4, o + 1), pm1 = U(4, o - 1);
      const T t3a = mabs(pp1 - pm1);
      const T t1 = eps2 * dmin2(pp1, pm1) - t3a;
      const T t2 = U(D, o + 1) - U(D, o - 1);
      const T omg1 = (t1 < T(0) && t2 < T(0)) ? T(1) : T(0);
      const T t3b = U(4, o + 2) - U(4, o - 2);
      T t4;
      if (t3b == T(0)) t4 = (t3a == T(0)) ? -omg2 : T(1.0) - omg2;
      else t4 = (t3a / t3b) - omg2;
      return dmin2(T(1), omg1 * dmax2(T(0), t4 * omg3));
    };
    const T f1b = (U(4, 1) - U(4, -1) < T(0)) ? f1a(1) : f1a(-1);
    f2a = dmax2(f1a(0), f1b);
  }
#pragma unroll 1
  for (int v = 0; v < 9; ++v) {
    if (v == 5 && !ALL) { L[v] = T(0); R[v] = T(0); continue; }  // var 6 faces are never read downstream
    const T um2 = U(v, -2), um1 = U(v, -1), u0 = U(v, 0), up1 = U(v, 1), up2 = U(v, 2);
    const T dm = ppm_dma(um2, um1, u0, DX(-2), DX(-1), DX(0), D == 3);
    const T d0 = ppm_dma(um1, u0, up1, DX(-1), DX(0), DX(1), D == 3);
    const T dp = ppm_dma(u0, up1, up2, DX(0), DX(1), DX(2), D == 3);
    T l = ppm_face(um1, u0, dm, d0, DX(-2), DX(-1), DX(0), DX(1));
    T r = ppm_face(u0, up1, d0, dp, DX(-1), DX(0), DX(1), DX(2));
    if (v == 0) {
      r = r * (T(1.0) - eta) + (up1 - T(0.5) * dp) * eta;
      l = l * (T(1.0) - eta) + (um1 + T(0.5) * dm) * eta;
    }
    r = u0 * f2a + r * (T(1.0) - f2a);
    l = u0 * f2a + l * (T(1.0) - f2a);
    // monoto (rec.f90:1887-2056)
    if ((r - u0) * (l - u0) >= T(0)) { r = u0; l = u0; }
    const T t3 = T(6.0) * (r - l) * (u0 - T(0.5) * (r + l));
    const T t4 = (r - l) * (r - l);
    if (t3 > t4) l = T(3.0) * u0 - T(2.0) * r;
    if (-t3 > t4) r = T(3.0) * u0 - T(2.0) * l;
    L[v] = l;
    R[v] = r;
  }
}

}  // namespace rg
