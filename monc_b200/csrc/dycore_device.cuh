// Device functions of the dynamical core: one function per MONC component, evaluated at a
// single grid point of an x-fastest [nz][ny][nx] field with periodic horizontal indexing.
//
// The same functions serve the per-component kernels (drop-in replacements of MONC's column
// callbacks) and the fused step kernels.  Expression trees follow the Fortran so that the FP64
// instantiation reproduces MONC's rounding; T = float gives the FP32 stencil path.
// Vertical indices k are MONC's 1-based levels; horizontal indices i, j are 0-based and may lie
// up to 2 points outside [0, n) (wrapped periodically).
#pragma once

#include <type_traits>

#include "mgpu_internal.h"

namespace mgpu {

struct Geo {
  int nx, ny, nz;
  long long plane;
  __device__ __forceinline__ int wi(int i) const { return i < 0 ? i + nx : (i >= nx ? i - nx : i); }
  __device__ __forceinline__ int wj(int j) const { return j < 0 ? j + ny : (j >= ny ? j - ny : j); }
  __device__ __forceinline__ long long at(int k, int j, int i) const {
    return (long long)(k - 1) * plane + (long long)wj(j) * nx + wi(i);
  }
};

// read-only field view bound to a geometry
template <typename T>
struct View {
  const T* __restrict__ p;
  Geo g;
  __device__ __forceinline__ T operator()(int k, int j, int i) const { return __ldg(p + g.at(k, j, i)); }
};

// profile accessor (FP64 in memory, converted to the compute type)
template <typename T>
struct Prof {
  const double* __restrict__ base;
  int stride;
  __device__ __forceinline__ T operator()(int id, int k) const { return (T)__ldg(base + id * stride + k); }
};

template <typename T> __device__ __forceinline__ T tsign(T a, T b) { return copysign(fabs(a), b); }
template <typename T> __device__ __forceinline__ T tmax(T a, T b) { return a > b ? a : b; }  // Fortran MAX
template <typename T> __device__ __forceinline__ T tmin(T a, T b) { return a < b ? a : b; }
template <typename T> __device__ __forceinline__ T sqr(T a) { return a * a; }
// 1/x rounded to nearest: the same value IEEE division 1.0/x produces, with a shorter sequence
__device__ __forceinline__ double rcp(double x) { return __drcp_rn(x); }
__device__ __forceinline__ float rcp(float x) { return __frcp_rn(x); }
// IEEE division (the instruction `x / r` compiles to) written as PTX, so that the compiler cannot
// fold `c ? x : x / r` into an unconditional x / (c ? 1 : r)
__device__ __forceinline__ double div_rn(double x, double r) {
  double q;
  asm("div.rn.f64 %0, %1, %2;" : "=d"(q) : "d"(x), "d"(r));
  return q;
}
__device__ __forceinline__ float div_rn(float x, float r) {
  float q;
  asm("div.rn.f32 %0, %1, %2;" : "=f"(q) : "f"(x), "f"(r));
  return q;
}
// x / r where r is a reference density; Boussinesq runs have r == 1 exactly and x/1 == x
template <typename T> __device__ __forceinline__ T div_rho(const Scalars& s, T x, T r) { return s.rho_unity ? x : div_rn(x, r); }
template <typename T> __device__ __forceinline__ T cub(T a) { return a * a * a; }
// 1/(fdels + 1e-30) of the TVD limiter.  In FP32 an advected perturbation of order 1e-30 can
// cancel the 1e-30 exactly and make the reciprocal infinite (then 0*inf = NaN downstream); the
// FP32 path returns 1e30 there.  FP64 keeps MONC's expression unchanged.
template <typename T> __device__ __forceinline__ T rcp_limiter(T x) { return rcp(x); }
__device__ __forceinline__ float rcp_limiter(float x) { return x == 0.0f ? 1.0e30f : rcp(x); }

// ------------------------------------------------------------------------------------------
// lower_bc, prescribed surface fluxes (lowerbc.F90:221-305, 601-768; look :645-666)
// ------------------------------------------------------------------------------------------
template <typename T>
__device__ T lookup_ustr(const Scalars& s, T vel) {
  T posn = (T)1.0 + (T)(float)(s.lookup_entries - 1) * log(vel / (T)s.velmin) * (T)s.aloginv;
  int ip = (int)posn;
  if (ip >= 1) {
    if (ip < s.lookup_entries) {
      T a = (T)__ldg(s.lookup + ip), b = (T)__ldg(s.lookup + ip + 1);
      return a + (posn - (T)(float)ip) * (b - a);
    }
    return vel * (T)s.cneut;
  }
  return pow(vel, -(T)s.convective_limit) * (T)s.cfc;
}

// Level-1 eddy coefficients and scalar ghost value of one column.
//   zu_state : current_state%zu (always), zu_a/zv_a: u,v on the forward step else zu,zv,
//   th_a     : th on the forward step else zth (level 2 read, level 1 written by the caller).
template <typename T, class A, class PA>
__device__ void lower_bc_column(const Scalars& s, const PA& P, const A& zu_state, const A& zu_a, const A& zv_a,
                                const A& th_a, const A* qv_a, int j, int i, T& vis1, T& diff1, T& th1, T& qv1) {
  T hv = sqr((T)0.5 * (zu_state(2, j, i) + zu_a(2, j, i - 1)) + (T)s.ugal);
  hv = hv + sqr((T)0.5 * (zv_a(2, j, i) + zv_a(2, j - 1, i)) + (T)s.vgal);
  hv = sqrt(hv) + (T)s.smallp;
  const T fbuoy = (T)s.fbuoy, vk = (T)s.vk, czn = (T)s.czn, zn2 = (T)s.zn2;
  T v1, d1;
  bool set_scalars = true;
  if (fbuoy > (T)0.0) {
    // convective surface layer (lowerbc.F90:601-633)
    T ustr = lookup_ustr<T>(s, hv);
    v1 = czn * sqr(ustr) / hv;
    d1 = (vk * czn * ustr / (T)s.alphah) /
         ((T)s.zlogth - (T)2. * log(((T)1. + sqrt((T)1. + (T)s.gammah * vk * fbuoy * (zn2 + (T)s.z0) / cub(ustr))) /
                                    ((T)1. + sqrt((T)1. + (T)s.gammah * vk * fbuoy * (T)s.z0th / cub(ustr)))));
  } else if (fbuoy == (T)0.0) {
    // neutral (lowerbc.F90:672-702)
    T ustr = hv * (T)s.vk_on_zlogm;
    v1 = czn * sqr(ustr) / hv;
    d1 = v1 * (T)s.zlogm / ((T)s.alphah * (T)s.zlogth);
  } else {
    // stable surface layer (lowerbc.F90:708-768)
    T ustr = hv * (T)s.vk_on_zlogm;
    if ((fbuoy - (T)1.E-9) < (T)-4.0 * sqr(vk) * cub(hv) / ((T)27.0 * (T)s.betam * zn2 * sqr((T)s.zlogm))) {
      v1 = (T)0.0;
      d1 = (T)0.0;
      set_scalars = false;
    } else {
      ustr = ustr / (T)3.0 *
             ((T)1.0 - (T)2.0 * cos((acos((T)-27.0 * (T)s.betam * vk * zn2 * fbuoy / ((T)s.zlogm * (T)2.0 * cub(ustr)) - (T)1.0) +
                                     (T)2.0 * (T)s.pi) / (T)3.0));
      v1 = czn * sqr(ustr) / hv;
      d1 = v1 * ((T)s.zlogm - (T)s.betam * zn2 * vk * fbuoy / cub(ustr)) /
           ((T)s.alphah * (T)s.zlogth - (T)s.betah * vk * fbuoy * (zn2 + (T)s.z0 - (T)s.z0th) / cub(ustr));
    }
  }
  v1 = tmin<T>(v1, (T)s.max_diff_or_visc);
  d1 = tmin<T>(d1, (T)s.max_diff_or_visc);
  vis1 = v1;
  diff1 = d1;
  if (set_scalars) {
    if constexpr (sizeof(T) == 4) {
      // FP32: thref(2) - thref(1) as the FP64 profile difference.  MONC's order, th(2) - thref(1)
      // + thref(2), rounds th(2) to the spacing of thref (~290 K, ulp 3e-5 K) and turns the ghost
      // value into a staircase of th(2) that drives the surface-layer buoyancy every step
      th1 = th_a(2, j, i) + (((T)s.surface_temperature_flux * P(P_DZN, 2) / d1) + P(P_DTHREF, 1));
    } else
      th1 = ((T)s.surface_temperature_flux * P(P_DZN, 2) / d1) + th_a(2, j, i) - P(P_THREF, 1) + P(P_THREF, 2);
    qv1 = qv_a ? (*qv_a)(2, j, i) + (T)s.surface_vapour_flux * P(P_DZN, 2) / d1 : (T)0;
  } else {
    th1 = th_a(2, j, i);
    qv1 = qv_a ? (*qv_a)(2, j, i) : (T)0;
  }
}

// ------------------------------------------------------------------------------------------
// smagorinsky (smagorinsky.F90:180-304 setfri + dry Ri, :316-402 moist Ri, :487-696 strain)
// ------------------------------------------------------------------------------------------
// The parts of the strain rate that belong to one level kk (smagorinsky.F90:487-696): the squared
// x and y differences of u and v at kk, the squared vertical difference of w below kk, and the
// four squared horizontal-shear terms at kk.  half_squared_strain at level k combines the parts
// of levels k and k+1, so a kernel marching up the levels carries the k+1 parts to the next level.
template <typename T>
struct StrainLevel {
  T a11, a22, a33, g12;
};

template <typename T, class A, class PA>
__device__ __forceinline__ StrainLevel<T> strain_level(const Scalars& s, const PA& P, const A& U, const A& V,
                                                       const A& W, int kk, int j, int i) {
  const T cx = (T)s.cx, cy = (T)s.cy;
  StrainLevel<T> r;
  r.a11 = sqr(U(kk, j, i) - U(kk, j, i - 1));
  r.a22 = sqr(V(kk, j, i) - V(kk, j - 1, i));
  r.a33 = sqr((W(kk, j, i) - W(kk - 1, j, i)) * P(P_RDZ, kk));
  r.g12 = (sqr((U(kk, j, i - 1) - U(kk, j - 1, i - 1)) * cy + (V(kk, j - 1, i) - V(kk, j - 1, i - 1)) * cx) +
           sqr((U(kk, j + 1, i - 1) - U(kk, j, i - 1)) * cy + (V(kk, j, i) - V(kk, j, i - 1)) * cx)) +
          (sqr((U(kk, j, i) - U(kk, j - 1, i)) * cy + (V(kk, j - 1, i + 1) - V(kk, j - 1, i)) * cx) +
           sqr((U(kk, j + 1, i) - U(kk, j, i)) * cy + (V(kk, j, i + 1) - V(kk, j, i)) * cx));
  return r;
}

// half the squared strain rate at level k from the level parts lo (level k) and hi (level k+1)
template <typename T, class A, class PA>
__device__ __forceinline__ T half_squared_strain_parts(const Scalars& s, const PA& P, const A& U, const A& V,
                                                       const A& W, int k, int j, int i, const StrainLevel<T>& lo,
                                                       const StrainLevel<T>& hi) {
  const T cx = (T)s.cx, cy = (T)s.cy, cx2 = (T)s.cx2, cy2 = (T)s.cy2;
  const T rdzn1 = P(P_RDZN, k + 1);
  T ssq11 = cx2 * (hi.a11 + lo.a11);
  T ssq22 = cy2 * (hi.a22 + lo.a22);
  T ssq33 = lo.a33 + hi.a33;
  T ssq13 = (sqr((U(k + 1, j, i) - U(k, j, i)) * rdzn1 + (W(k, j, i + 1) - W(k, j, i)) * cx) +
             sqr((U(k + 1, j, i - 1) - U(k, j, i - 1)) * rdzn1 + (W(k, j, i) - W(k, j, i - 1)) * cx)) * (T)0.5;
  T ssq23 = (sqr((W(k, j, i) - W(k, j - 1, i)) * cy + (V(k + 1, j - 1, i) - V(k, j - 1, i)) * rdzn1) +
             sqr((W(k, j + 1, i) - W(k, j, i)) * cy + (V(k + 1, j, i) - V(k, j, i)) * rdzn1)) * (T)0.5;
  T ssq12 = (lo.g12 + hi.g12) * (T)0.125;
  return ssq11 + ssq22 + ssq33 + ssq13 + ssq23 + ssq12 + (T)s.smallp;
}

template <typename T, class A, class PA>
__device__ T half_squared_strain(const Scalars& s, const PA& P, const A& U, const A& V,
                                 const A& W, int k, int j, int i) {
  const StrainLevel<T> lo = strain_level<T, A, PA>(s, P, U, V, W, k, j, i);
  const StrainLevel<T> hi = strain_level<T, A, PA>(s, P, U, V, W, k + 1, j, i);
  return half_squared_strain_parts<T, A, PA>(s, P, U, V, W, k, j, i, lo, hi);
}

// moist_ri_2 for one level (RICHARDSON_NUMBER_CALCULATION = 2); with NUM, ri * ssq (the number
// without its 1/ssq factor)
template <typename T, class A, class PA, bool NUM = false>
__device__ T moist_ri(const Scalars& s, const PA& P, T ssq, const A& TH, const A& QV, const A& QL, int k, int j, int i) {
  T tmpinv = NUM ? (T)1.0 : rcp(ssq);
  T scltmp = P(P_RDZN, k + 1) * P(P_BUOY_CO, k);
  const T rl = (T)s.rlvap_over_cp, eps = (T)s.eps;
  const T qsat = P(P_QSAT, k), dq = P(P_DQSATDT, k), rpr = P(P_RPREFRCP, k), tst = P(P_TSTARPR, k), fac = P(P_QSATFAC, k);
  const T pr = P(P_PREFRCP, k), thr = P(P_THREF, k), thr1 = P(P_THREF, k + 1), tref = P(P_TREF, k);
  T qt_k = QV(k, j, i) + QL(k, j, i);
  T qt_kp1 = QV(k + 1, j, i) + QL(k + 1, j, i);
  T thlpr_k = TH(k, j, i) - rl * QL(k, j, i) * pr;
  T thlpr_kp1 = TH(k + 1, j, i) - rl * QL(k + 1, j, i) * pr;
  if constexpr (sizeof(T) == 4) {
    // FP32: the same quantities with the reference-state offsets (thref ~ 290 K) cancelled
    // analytically -- thv(ln) - thv(li) = eps dth + (rl pr - thcona)(ql(ln) - ql(li)) -- and the
    // temperature offset rpr thref(k+1) - tstarpr - tref taken from an FP64 profile
    const T toff = P(P_TOFF, k);
    T dth = (thlpr_kp1 - thlpr_k + P(P_DTHREF, k));
    T qtun = qt_kp1 - eps * (qt_kp1 - qt_k);
    T qtln = qt_k + eps * (qt_kp1 - qt_k);
    T qlli = tmax<T>((T)0.0, (qt_k - (qsat + dq * (rpr * thlpr_k - tst))) * fac);
    T qlui = tmax<T>((T)0.0, (qt_kp1 - (qsat + dq * (rpr * thlpr_kp1 + toff))) * fac);
    T qlln = tmax<T>((T)0.0, (qtln - (qsat + dq * (rpr * (thlpr_k + eps * dth) - tst))) * fac);
    T qlun = tmax<T>((T)0.0, (qtun - (qsat + dq * (rpr * (thlpr_kp1 - eps * dth) + toff))) * fac);
    T dl = eps * dth + (rl * pr - (T)s.thcona) * (qlln - qlli);
    T du = -eps * dth + (rl * pr - (T)s.thconap1) * (qlun - qlui);
    (void)thr;
    (void)thr1;
    (void)tref;
    if constexpr (NUM) return scltmp * ((T)s.thconb * (qt_kp1 - qt_k) + (dl - du) * (T)s.repsh);
    else return scltmp * tmpinv * ((T)s.thconb * (qt_kp1 - qt_k) + (dl - du) * (T)s.repsh);
  }
  T qlli = tmax<T>((T)0.0, (qt_k - (qsat + dq * (rpr * thlpr_k - tst))) * fac);
  T qlui = tmax<T>((T)0.0, (qt_kp1 - (qsat + dq * (rpr * (thlpr_kp1 + thr1) - tst - tref))) * fac);
  T thvli = thlpr_k + thr + (rl * pr - (T)s.thcona) * qlli;
  T thvui = thlpr_kp1 + thr1 + (rl * pr - (T)s.thconap1) * qlui;
  T dth = (thlpr_kp1 - thlpr_k + P(P_DTHREF, k));
  T thlpr_un = thlpr_kp1 - eps * dth;
  T thlpr_ln = thlpr_k + eps * dth;
  T qtun = qt_kp1 - eps * (qt_kp1 - qt_k);
  T qtln = qt_k + eps * (qt_kp1 - qt_k);
  T qlln = tmax<T>((T)0.0, (qtln - (qsat + dq * (rpr * thlpr_ln - tst))) * fac);
  T qlun = tmax<T>((T)0.0, (qtun - (qsat + dq * (rpr * (thlpr_un + thr1) - tst - tref))) * fac);
  T thvln = thlpr_ln + thr + (rl * pr - (T)s.thcona) * qlln;
  T thvun = thlpr_un + thr1 + (rl * pr - (T)s.thconap1) * qlun;
  if constexpr (NUM) return scltmp * ((T)s.thconb * (qt_kp1 - qt_k) + ((thvln - thvli) - (thvun - thvui)) * (T)s.repsh);
  else return scltmp * tmpinv * ((T)s.thconb * (qt_kp1 - qt_k) + ((thvln - thvli) - (thvun - thvui)) * (T)s.repsh);
}

// vis/diff at level 2 <= k <= nz-1 from the strain rate and Richardson number
template <typename T, class PA, class ATC, class AT>
__device__ void smagorinsky_from_strain(const Scalars& s, const PA& P, T ssq, const ATC& THcur, const AT& THarg,
                                        const AT* QV, const AT* QL, int k, int j, int i, T& vis, T& diff) {
#ifdef MGPU_CONTRACTED
  // The contracted build folds the neutral factor sqrt(ssq) into the unstable branch's stability
  // functions: with X = ri ssq (the Richardson number's numerator), sqrt(1 - c ri) sqrt(ssq) =
  // sqrt(ssq - c X), so that branch, the common one in a convective layer, takes two square roots
  // and no division where MONC's order takes three and one.  The branches are the same (ri and X
  // have one sign); the values agree to rounding.
  T X = (T)0.0;
  if (!s.passive_th) {
    if (!s.passive_q) X = moist_ri<T, AT, PA, true>(s, P, ssq, THarg, *QV, *QL, k, j, i);
    else X = (P(P_DTHREF, k) + THcur(k + 1, j, i) - THcur(k, j, i)) * P(P_RDZN, k + 1) * P(P_BUOY_CO, k);
  }
  const T rn = P(P_RNEUTML_SQ, k);
  if (X <= (T)0.0) {
    vis = rn * sqrt(ssq - (T)s.subc * X);
    diff = rn * ((T)s.suba * sqrt(ssq - (T)s.subb * X));
  } else {
    const T ri = X / ssq;
    if (ri < (T)s.ric) {
      T t = (T)1. - ri * (T)s.ricinv;
      t = t * t;
      const T rifac = t * t;
      const T sctmp = rn * sqrt(ssq);
      vis = (rifac * ((T)1. - (T)s.subh * ri)) * sctmp;
      diff = (rifac * (T)s.suba * ((T)1. - (T)s.subg * ri)) * sctmp;
    } else {
      vis = (T)0.0;
      diff = (T)0.0;
    }
  }
#else
  T ri = (T)0.0;
  if (!s.passive_th) {
    if (!s.passive_q) ri = moist_ri<T, AT>(s, P, ssq, THarg, *QV, *QL, k, j, i);
    else  // the dry branch reads current_state%th in both stepping modes
      ri = (P(P_DTHREF, k) + THcur(k + 1, j, i) - THcur(k, j, i)) * P(P_RDZN, k + 1) * P(P_BUOY_CO, k) / ssq;
  }
  T vs, df;
  if (ri <= (T)0.0) {
    vs = sqrt((T)1.0 - (T)s.subc * ri);
    df = (T)s.suba * sqrt((T)1. - (T)s.subb * ri);
  } else if (ri > (T)0.0 && ri < (T)s.ric) {
    T t = (T)1. - ri * (T)s.ricinv;
    t = t * t;
    T rifac = t * t;
    vs = rifac * ((T)1. - (T)s.subh * ri);
    df = rifac * (T)s.suba * ((T)1. - (T)s.subg * ri);
  } else {
    vs = (T)0.0;
    df = (T)0.0;
  }
  T sctmp = P(P_RNEUTML_SQ, k) * sqrt(ssq);
  vis = vs * sctmp;
  diff = df * sctmp;
#endif
}

template <typename T, class A, class PA, class AT>
__device__ void smagorinsky_point(const Scalars& s, const PA& P, const A& U, const A& V, const A& W, const AT& THcur,
                                  const AT& THarg, const AT* QV, const AT* QL, int k, int j, int i, T& vis, T& diff) {
  T ssq = half_squared_strain<T, A>(s, P, U, V, W, k, j, i);
  smagorinsky_from_strain<T, PA, AT, AT>(s, P, ssq, THcur, THarg, QV, QL, k, j, i, vis, diff);
}

// ------------------------------------------------------------------------------------------
// pw_advection advect_flow_fields (pwadvection.F90:466-610): assigned sources, 2<=k<=nz
// ------------------------------------------------------------------------------------------
template <typename T, class A, class PA>
__device__ void pw_point(const Scalars& s, const PA& P, const A& U, const A& V, const A& W,
                         int k, int j, int i, T& su, T& sv, T& sw) {
  const T tcx = (T)s.tcx, tcy = (T)s.tcy;
  const T u0 = U(k, j, i), v0 = V(k, j, i);
  if (k < s.nz) {
    const T w0 = W(k, j, i);
    T a = tcx * (U(k, j, i - 1) * (u0 + U(k, j, i - 1)) - U(k, j, i + 1) * (u0 + U(k, j, i + 1)));
    a = a + tcy * (U(k, j - 1, i) * (V(k, j - 1, i) + V(k, j - 1, i + 1)) - U(k, j + 1, i) * (v0 + V(k, j, i + 1)));
    a = a + (P(P_TZC1, k) * U(k - 1, j, i) * (W(k - 1, j, i) + W(k - 1, j, i + 1)) -
             P(P_TZC2, k) * U(k + 1, j, i) * (w0 + W(k, j, i + 1)));
    su = a;
    T b = tcy * (V(k, j - 1, i) * (v0 + V(k, j - 1, i)) - V(k, j + 1, i) * (v0 + V(k, j + 1, i)));
    b = b + tcx * (V(k, j, i - 1) * (U(k, j, i - 1) + U(k, j + 1, i - 1)) - V(k, j, i + 1) * (u0 + U(k, j + 1, i)));
    b = b + (P(P_TZC1, k) * V(k - 1, j, i) * (W(k - 1, j, i) + W(k - 1, j + 1, i)) -
             P(P_TZC2, k) * V(k + 1, j, i) * (w0 + W(k, j + 1, i)));
    sv = b;
    T c = (P(P_TZD1, k) * W(k - 1, j, i) * (w0 + W(k - 1, j, i)) - P(P_TZD2, k) * W(k + 1, j, i) * (w0 + W(k + 1, j, i)));
    c = c + tcx * (W(k, j, i - 1) * (U(k, j, i - 1) + U(k + 1, j, i - 1)) - W(k, j, i + 1) * (u0 + U(k + 1, j, i)));
    c = c + tcy * (W(k, j - 1, i) * (V(k, j - 1, i) + V(k + 1, j - 1, i)) - W(k, j + 1, i) * (v0 + V(k + 1, j, i)));
    sw = c;
  } else {
    T a = tcx * (U(k, j, i - 1) * (u0 + U(k, j, i - 1)) - U(k, j, i + 1) * (u0 + U(k, j, i + 1)));
    a = a + tcy * (U(k, j - 1, i) * (V(k, j - 1, i) + V(k, j - 1, i + 1)) - U(k, j + 1, i) * (v0 + V(k, j, i + 1)));
    a = a + P(P_TZC1, k) * U(k - 1, j, i) * (W(k - 1, j, i) + W(k - 1, j, i + 1));
    su = a;
    T b = tcy * (V(k, j - 1, i) * (v0 + V(k, j - 1, i)) - V(k, j + 1, i) * (v0 + V(k, j + 1, i)));
    b = b + tcx * (V(k, j, i - 1) * (U(k, j, i - 1) + U(k, j + 1, i - 1)) - V(k, j, i + 1) * (u0 + U(k, j + 1, i)));
    b = b + P(P_TZC1, k) * V(k - 1, j, i) * (W(k - 1, j, i) + W(k - 1, j + 1, i));
    sv = b;
    sw = (T)0.0;  // sw(nz) is left at its cleared value
  }
}

// ------------------------------------------------------------------------------------------
// viscosity (viscosity.F90:293-498): increments of su, sv (2<=k<=nz) and sw (2<=k<=nz-1)
// ------------------------------------------------------------------------------------------
template <typename T>
struct Tau13 {
  T t13, t13m1, t23, t23m1;
};

template <typename T, class A, class PA>
__device__ Tau13<T> tau_13_23(const Scalars& s, const PA& P, const A& ZU, const A& ZV,
                              const A& ZW, const A& VIS, int k, int j, int i) {
  Tau13<T> t;
  if (k >= s.nz) { t.t13 = t.t13m1 = t.t23 = t.t23m1 = (T)0.0; return t; }
  const T cx = (T)s.cx, cy = (T)s.cy, rdzn = P(P_RDZN, k + 1), rho = P(P_RHO, k);
  T vis13 = (T)0.5 * (VIS(k, j, i) + VIS(k, j, i + 1));
  T a = (ZU(k + 1, j, i) - ZU(k, j, i)) * rdzn;
  a = a + (ZW(k, j, i + 1) - ZW(k, j, i)) * cx;
  t.t13 = a * rho * vis13;
  vis13 = (T)0.5 * (VIS(k, j, i - 1) + VIS(k, j, i));
  a = (ZU(k + 1, j, i - 1) - ZU(k, j, i - 1)) * rdzn;
  a = a + (ZW(k, j, i) - ZW(k, j, i - 1)) * cx;
  t.t13m1 = a * rho * vis13;
  T vis23 = (T)0.5 * (VIS(k, j, i) + VIS(k, j + 1, i));
  a = (ZW(k, j + 1, i) - ZW(k, j, i)) * cy;
  a = a + (ZV(k + 1, j, i) - ZV(k, j, i)) * rdzn;
  t.t23 = a * rho * vis23;
  vis23 = (T)0.5 * (VIS(k, j - 1, i) + VIS(k, j, i));
  a = (ZW(k, j, i) - ZW(k, j - 1, i)) * cy;
  a = a + (ZV(k + 1, j - 1, i) - ZV(k, j - 1, i)) * rdzn;
  t.t23m1 = a * rho * vis23;
  return t;
}

template <typename T, class A, class PA>
__device__ T tau33_at(const Scalars& s, const PA& P, const A& ZW, const A& VIS, int k, int j, int i) {
  if (k <= 1) return (T)0.0;
  T visonp2 = P(P_RHON, k) * (VIS(k, j, i) + VIS(k - 1, j, i));
  return visonp2 * (ZW(k, j, i) - ZW(k - 1, j, i)) * P(P_RDZ, k);
}

// Viscous increments at level k from this level's stresses and the level-below values tm13, tm23
// (tau_13_23(k-1).t13, .t23) and t33 (tau33_at(k)); t13, t23 and t33p return this level's
// tau_13_23(k).t13, .t23 and tau33_at(k+1), which a kernel marching up the levels carries to the
// level above instead of recomputing them.
template <typename T, class A, class PA>
__device__ void viscosity_core(const Scalars& s, const PA& P, const A& ZU, const A& ZV, const A& ZW,
                               const A& ZU_state, const A& VIS, int k, int j, int i, T tm13, T tm23, T t33, T& du,
                               T& dv, T& dw, T& t13, T& t23, T& t33p) {
  const T cx = (T)s.cx, cy = (T)s.cy, rhon = P(P_RHON, k);
  // horizontal stresses at level k (k >= 2)
  T vistmp = VIS(k, j, i) + VIS(k, j + 1, i) + VIS(k - 1, j, i) + VIS(k - 1, j + 1, i);
  T vis12 = (T)0.125 * (vistmp + VIS(k, j, i + 1) + VIS(k, j + 1, i + 1) + VIS(k - 1, j, i + 1) + VIS(k - 1, j + 1, i + 1));
  T tau12 = (ZU(k, j + 1, i) - ZU(k, j, i)) * cy;
  tau12 = tau12 + (ZV(k, j, i + 1) - ZV(k, j, i)) * cx;
  tau12 = tau12 * rhon * vis12;
  T vis12a = (T)0.125 * (vistmp + VIS(k, j, i - 1) + VIS(k, j + 1, i - 1) + VIS(k - 1, j, i - 1) + VIS(k - 1, j + 1, i - 1));
  T tau12m1 = (ZU(k, j + 1, i - 1) - ZU(k, j, i - 1)) * cy;
  tau12m1 = tau12m1 + (ZV(k, j, i) - ZV(k, j, i - 1)) * cx;
  tau12m1 = tau12m1 * rhon * vis12a;
  vistmp = VIS(k, j - 1, i) + VIS(k, j, i) + VIS(k - 1, j - 1, i) + VIS(k - 1, j, i);
  vis12 = (T)0.125 * (vistmp + VIS(k, j - 1, i + 1) + VIS(k, j, i + 1) + VIS(k - 1, j - 1, i + 1) + VIS(k - 1, j, i + 1));
  T tau12_ym1 = (ZU(k, j, i) - ZU(k, j - 1, i)) * cy;
  tau12_ym1 = tau12_ym1 + (ZV(k, j - 1, i + 1) - ZV(k, j - 1, i)) * cx;
  tau12_ym1 = tau12_ym1 * rhon * vis12;
  T visonp2 = rhon * (VIS(k, j, i) + VIS(k - 1, j, i));
  T tau11 = visonp2 * (ZU(k, j, i) - ZU(k, j, i - 1)) * cx;
  T tau22 = visonp2 * (ZV(k, j, i) - ZV(k, j - 1, i)) * cy;
  visonp2 = rhon * (VIS(k, j + 1, i) + VIS(k - 1, j + 1, i));
  T tau22_yp1 = visonp2 * (ZV(k, j + 1, i) - ZV(k, j, i)) * cy;
  T visonp2a = rhon * (VIS(k, j, i + 1) + VIS(k - 1, j, i + 1));
  T tau11p1 = visonp2a * (ZU_state(k, j, i + 1) - ZU(k, j, i)) * cx;  // reads current_state%zu at x+1
  Tau13<T> t0 = tau_13_23<T, A>(s, P, ZU, ZV, ZW, VIS, k, j, i);
  du = div_rho<T>(s, (tau11p1 - tau11) * cx + (tau12 - tau12_ym1) * cy + (t0.t13 - tm13) * P(P_RDZ, k), rhon);
  dv = div_rho<T>(s, (tau12 - tau12m1) * cx + (tau22_yp1 - tau22) * cy + (t0.t23 - tm23) * P(P_RDZ, k), rhon);
  if (k < s.nz) {
    t33p = tau33_at<T, A>(s, P, ZW, VIS, k + 1, j, i);
    dw = div_rho<T>(s, (t0.t13 - t0.t13m1) * cx + (t0.t23 - t0.t23m1) * cy + (t33p - t33) * P(P_RDZN, k + 1), P(P_RHO, k));
  } else {
    t33p = (T)0.0;
    dw = (T)0.0;
  }
  t13 = t0.t13;
  t23 = t0.t23;
}

template <typename T, class A, class PA>
__device__ void viscosity_point(const Scalars& s, const PA& P, const A& ZU, const A& ZV,
                                const A& ZW, const A& ZU_state, const A& VIS, int k, int j, int i,
                                T& du, T& dv, T& dw) {
  const Tau13<T> tm = tau_13_23<T, A>(s, P, ZU, ZV, ZW, VIS, k - 1, j, i);
  const T t33 = k < s.nz ? tau33_at<T, A>(s, P, ZW, VIS, k, j, i) : (T)0.0;
  T t13, t23, t33p;
  viscosity_core<T, A, PA>(s, P, ZU, ZV, ZW, ZU_state, VIS, k, j, i, tm.t13, tm.t23, t33, du, dv, dw, t13, t23, t33p);
}

// ------------------------------------------------------------------------------------------
// coriolis (coriolis.F90:243-258), buoyancy (buoyancy.F90:229-262)
// ------------------------------------------------------------------------------------------
template <typename T, class A, class PA>
__device__ void coriolis_point(const Scalars& s, const PA& P, const A& U, const A& V, int k, int j,
                               int i, T& su, T& sv) {
  const T f = (T)s.fcoriol;
  su = su + f * ((T)0.25 * (V(k, j, i) + V(k, j, i + 1) + V(k, j - 1, i) + V(k, j - 1, i + 1)) + (T)s.vgal - P(P_GWY, k));
  sv = sv - f * ((T)0.25 * (U(k, j, i) + U(k, j, i - 1) + U(k, j + 1, i) + U(k, j + 1, i - 1)) + (T)s.ugal - P(P_GWX, k));
}

template <typename T>
__device__ T buoyancy_point(const Scalars& s, const Prof<T>& P, const View<T>& TH, const View<T>* Q, int k, int j,
                            int i, T sw) {
  // with s.bmean the horizontal means are taken out first: a horizontally uniform part of sw only
  // moves the mean pressure, which the projection removes again (the projected mean w is zero)
  const int st = s.nz + 2;
  if (!s.passive_th) {
    if (s.bmean) sw = sw + ((T)0.5 * P(P_BUOY_CO, k)) * ((TH(k, j, i) - (T)s.bmean[k]) + (TH(k + 1, j, i) - (T)s.bmean[k + 1]));
    else sw = sw + ((T)0.5 * P(P_BUOY_CO, k)) * (TH(k, j, i) + TH(k + 1, j, i));
  }
  if (!s.passive_q) {
    const T g2 = (T)(0.5 * s.G);
    for (int n = 0; n < s.nq; ++n) {
      if (s.bmean)
        sw = sw + g2 * (T)s.cq[n] * ((Q[n](k, j, i) - (T)s.bmean[(1 + n) * st + k]) +
                                    (Q[n](k + 1, j, i) - (T)s.bmean[(1 + n) * st + k + 1]));
      else
        sw = sw + g2 * (T)s.cq[n] * (Q[n](k, j, i) + Q[n](k + 1, j, i));
    }
  }
  return sw;
}

// ------------------------------------------------------------------------------------------
// damping (damping.F90:367-404), levels kdmpmin..nz (w: ..nz-1): Newtonian relaxation of zu, zv
// towards the mean profiles (in the Galilean frame), of zw towards 0, of scalars towards theirs
// ------------------------------------------------------------------------------------------
template <typename T, class PA>
__device__ __forceinline__ void damping_flow_point(const Scalars& s, const PA& P, int k, T zu, T zv, T zw, T& su,
                                                   T& sv, T& sw) {
  if (k < s.kdmpmin) return;
  const int st = s.nz + 2;
  su = su - P(P_DMPCO, k) * (zu - (T)(s.olz[k] - s.ugal));
  sv = sv - P(P_DMPCO, k) * (zv - (T)(s.olz[st + k] - s.vgal));
  if (k <= s.nz - 1) sw = sw - P(P_DMPCOZ, k) * zw;
}

// row 2 of s.olz for theta, 3 + n for q(n)
template <typename T, class PA>
__device__ __forceinline__ T damping_scalar_point(const Scalars& s, const PA& P, int k, T zf, int row, T sf) {
  if (k < s.kdmpmin) return sf;
  return sf - P(P_DMPCO, k) * (zf - (T)s.olz[row * (s.nz + 2) + k]);
}

// ------------------------------------------------------------------------------------------
// forcing: subsidence (forcing.F90:1052-1166), levels 2..nz.  With subsidence_local_* the
// gradients are the column's; otherwise every column gets the mean-profile tendencies in
// s.subs_tend (k_subsidence_tendencies).
// ------------------------------------------------------------------------------------------
template <typename T, class A, class PA>
__device__ __forceinline__ void subsidence_flow_point(const Scalars& s, const PA& P, const A& ZU, const A& ZV, int k,
                                                      int j, int i, T& su, T& sv) {
  if (!s.subs_local_th) {
    su = su - (T)s.subs_tend[k];
    sv = sv - (T)s.subs_tend[(s.nz + 2) + k];
    return;
  }
  T usub, vsub;
  if (k < s.nz) {
    usub = (T)2.0 * (P(P_WSUBS, k - 1) * P(P_TZC1, k) * (ZU(k, j, i) - ZU(k - 1, j, i)) +
                     P(P_WSUBS, k) * P(P_TZC2, k) * (ZU(k + 1, j, i) - ZU(k, j, i)));
    vsub = (T)2.0 * (P(P_WSUBS, k - 1) * P(P_TZC1, k) * (ZV(k, j, i) - ZV(k - 1, j, i)) +
                     P(P_WSUBS, k) * P(P_TZC2, k) * (ZV(k + 1, j, i) - ZV(k, j, i)));
  } else {
    usub = (T)2.0 * (P(P_WSUBS, k - 1) * P(P_TZC1, k) * (ZU(k, j, i) - ZU(k - 1, j, i)));
    vsub = (T)2.0 * (P(P_WSUBS, k - 1) * P(P_TZC1, k) * (ZV(k, j, i) - ZV(k - 1, j, i)));
  }
  su = su - usub;
  sv = sv - vsub;
}

template <typename T, class A, class PA>
__device__ __forceinline__ T subsidence_theta_point(const Scalars& s, const PA& P, const A& ZTH, int k, int j, int i,
                                                    T sth) {
  if (!s.subs_local_th) return sth - (T)s.subs_tend[2 * (s.nz + 2) + k];
  const int ka = k < s.nz ? k + 1 : k, kb = ka - 1;  // the upper and lower level of the difference
  T thsub;
  if constexpr (sizeof(T) == 4) {
    // FP32: (zth + thref) differenced as dzth + dthref; thref (~290 K) would round zth to its
    // 3e-5 K spacing
    thsub = P(P_WSUBS, k) * ((ZTH(ka, j, i) - ZTH(kb, j, i)) + P(P_DTHREF, kb)) * P(P_RDZN, ka);
  } else {
    thsub = P(P_WSUBS, k) * ((ZTH(ka, j, i) + P(P_THREF, ka)) - (ZTH(kb, j, i) + P(P_THREF, kb))) * P(P_RDZN, ka);
  }
  return sth - thsub;
}

template <typename T, class A, class PA>
__device__ __forceinline__ T subsidence_q_point(const Scalars& s, const PA& P, const A& ZQ, int n, int k, int j, int i,
                                                T sq) {
  if (!s.subs_local_q) return sq - (T)s.subs_tend[(3 + n) * (s.nz + 2) + k];
  const int ka = k < s.nz ? k + 1 : k, kb = ka - 1;
  return sq - P(P_WSUBS, k) * (ZQ(ka, j, i) - ZQ(kb, j, i)) * P(P_RDZN, ka);
}

// ------------------------------------------------------------------------------------------
// simplecloud saturation adjustment (simplecloud.F90:262-379, saturation.F90 qsaturation and
// dqwsatdt), one point 2 <= k <= nz.  q_v, q_l, th are the state (forward step) or z-fields;
// zq_l is always the z-field (the evaporation branch tests scalar_stepping, which is centred).
// Above k_cloudmax the Fortran reuses one_over_exner from the last adjusted level.
// ------------------------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T qsaturation(T temperature, T pressure) {
  const T tk0c = (T)273.15, qsa1 = (T)3.8, qsa2 = (T)-17.2693882, qsa3 = (T)35.86, qsa4 = (T)6.109;
  return qsa1 / (pressure * exp(qsa2 * (temperature - tk0c) / (temperature - qsa3)) - qsa4);
}
template <typename T>
__device__ __forceinline__ T dqwsatdt(T qs, T temperature) {
  const T tk0c = (T)273.15, qsa1 = (T)3.8, qsa2 = (T)-17.2693882, qsa3 = (T)35.86, qsa4 = (T)6.109;
  return -qsa2 * (tk0c - qsa3) * ((T)1.0 + qsa4 * qs / qsa1) * qs * pow(temperature - qsa3, (T)-2.0);
}

template <typename T, class PA>
__device__ void simplecloud_point(const Scalars& s, const PA& P, int k, T q_v, T q_l, T th, T zq_l, T& sth, T& sqv,
                                  T& sql) {
  const T dtm = s.forward ? (T)s.dtm : (T)(s.dtm * 2.0);
  const T rl = (T)s.rlvap_over_cp;
  if (k <= s.k_cloudmax) {
    const T exner = P(P_RPREFRCP, k), one_over_exner = P(P_PREFRCP, k);
    const T Pmb = P(P_PREFN, k) / (T)100.;
    const T qv = q_v + sqv * dtm;
    const T qc = q_l + sql * dtm;
    T qs, dqsdT_ = (T)0.0;
    if constexpr (sizeof(T) == 4) {
      // FP32: the temperature as its departure from 273.15 K, built from an FP64 reference
      // offset, so that exp() and the pole of Tetens' formula see it without cancellation
      const T tc = (th + sth * dtm) * exner + P(P_TC0, k);
      const T tq = tc + (T)(273.15 - 35.86);  // temperature - qsa3
      qs = (T)3.8 / (Pmb * exp((T)-17.2693882 * tc / tq) - (T)6.109);
      dqsdT_ = (T)17.2693882 * (T)(273.15 - 35.86) * ((T)1.0 + (T)6.109 * qs / (T)3.8) * qs / (tq * tq);
    } else {
      const T tk = (th + sth * dtm + P(P_THREF, k)) * exner;
      qs = qsaturation<T>(tk, Pmb);
      dqsdT_ = dqwsatdt<T>(qs, tk);
    }
    if (qv > qs || qc > (T)0.0) {
      const T dqsdT = dqsdT_;
      const T qsatfac = (T)1.0 / ((T)1.0 + rl * dqsdT);
      const T dmass = tmax<T>(-qc, (qv - qs) * qsatfac) / dtm;
      sqv = sqv - dmass;
      sql = sql + dmass;
      sth = sth + rl * dmass * one_over_exner;
    }
  } else {
    const T one_over_exner = s.k_cloudmax >= 2 ? P(P_PREFRCP, s.k_cloudmax) : (T)0.0;
    const T qc = zq_l + sql * dtm;
    if (qc > (T)0.0) {
      const T dmass = -qc / dtm;
      sqv = sqv - dmass;
      sql = sql + dmass;
      sth = sth + rl * dmass * one_over_exner;
    }
  }
}

// ------------------------------------------------------------------------------------------
// TVD advection: ULTIMATE-QUICKEST face values (ultimateflux.F90) and their divergence
// (tvdadvection.F90:911-960).  dt is 2*dtm in both stepping modes.
//
// The vertical metrics ultflx is called with (tvdadvection.F90:722-908): scalars, u and v take
// rdz, rdzn, dzn and kdof = 0; w takes rdzn, rdz, dz and kdof = 1, which shifts the rdz of the
// gradient and central terms up one level.
// ------------------------------------------------------------------------------------------
struct TvdMetricScalar {
  static constexpr int RDZ = P_RDZ, RDZN = P_RDZN, DZN = P_DZN, KDOF = 0, TZ1 = P_TZC1, TZ2 = P_TZC2;
};
struct TvdMetricW {
  static constexpr int RDZ = P_RDZN, RDZN = P_RDZ, DZN = P_DZ, KDOF = 1, TZ1 = P_TZD1, TZ2 = P_TZD2;
};
// Branch recorders of the face functions: NoRec (the kernels) records nothing and compiles away;
// BitRec appends each decision's bits to a code, so that a gradient check can count where two
// nearby trajectories take different branches (the kinks that finite differences straddle).
struct NoRec {
  __device__ __forceinline__ void operator()(unsigned, int) const {}
};
struct BitRec {
  unsigned* code;
  __device__ __forceinline__ void operator()(unsigned v, int nbits) const { *code = (*code << nbits) | v; }
};

// which of fncs, fnfs, fnrefs and 1 the limiter max(fncs, min(min(fnfs, fnrefs), 1)) takes
template <typename T>
__device__ __forceinline__ unsigned limiter_choice(T fncs, T fnfs, T fnrefs) {
  const T m = tmin<T>(fnfs, fnrefs);
  return fncs > tmin<T>(m, (T)1.0) ? 0u : (m < (T)1.0 ? (fnfs < fnrefs ? 1u : 2u) : 3u);
}

// The limited face value fu + fdels max(fncs, min(fnfs, fnrefs, 1)), fncs = (fc - fu) / fdels',
// fnfs = (ffs - fu) / fdels', fnrefs = fncs hrcfl, fdels' = fdels + 1e-30 (calculate_flux_in_x /
// _y / _w), with the branch recorded.  Where |fdels| is far above the 1e-30 offset, the
// contracted build multiplies the limiter through by fdels: max(fc - fu, min(ffs - fu,
// (fc - fu) hrcfl, fdels)) for fdels > 0, min and max exchanged for fdels < 0.  That needs no
// reciprocal of fdels; the values agree to rounding.
template <typename T, class Rec = NoRec>
__device__ __forceinline__ T limited_face(T ffs, T fc, T fu, T fdels, T hrcfl, const Rec& rec = Rec()) {
#ifdef MGPU_CONTRACTED
  if constexpr (std::is_same<Rec, NoRec>::value) {
    if (fabs(fdels) > (T)1.e-20) {
      const T a = fc - fu, b = ffs - fu, ah = a * hrcfl;
      const T x = fdels > (T)0.0 ? tmax<T>(a, tmin<T>(tmin<T>(b, ah), fdels))
                                 : tmin<T>(a, tmax<T>(tmax<T>(b, ah), fdels));
      return x + fu;
    }
  }
#endif
  T rfdels = rcp_limiter(fdels + (T)1.e-30);
  T fnfs = (ffs - fu) * rfdels;
  T fncs = (fc - fu) * rfdels;
  T fnrefs = fncs * hrcfl;
  T ftemp = tmax<T>(fncs, tmin<T>(tmin<T>(fnfs, fnrefs), (T)1.0));
  rec(limiter_choice<T>(fncs, fnfs, fnrefs), 2);
  return ftemp * fdels + fu;
}

template <typename T, class Rec = NoRec>
__device__ __forceinline__ T limit_face(T data_value, T c, T dt, T sum_cfl_out, T fdels, T fd, T fc, T fu, T fgt1, T fgt2,
                                        T curv_term, const Rec& rec = Rec()) {
  const T r6 = (T)(1.0 / 6.0);
  T cflmod = fabs(data_value * c * dt);
  T hrcfl = rcp(sum_cfl_out + (T)1.e-30);
  T hcfl = (T)0.5 * cflmod;
  T cflcoef = r6 * ((T)1.0 - cflmod * cflmod);
  T ffs = (T)0.5 * (fd + fc) - hcfl * (fd - fc) - cflcoef * curv_term - fgt1 - fgt2;
  return limited_face<T, Rec>(ffs, fc, fu, fdels, hrcfl, rec);
}

// Sum of the outgoing Courant numbers of cell (k, j, i) without the factor dt: the sum_cfl_out
// that ultimateflux.F90's face routines form for the upwind cell of a face (calculate_flux_in_x,
// _y, _w and their callers), one term per face of the cell through which the flow leaves it.
// Written once for every face direction: the x routine's u0 + |min(0, u(i-1))| (u0 > 0) and
// max(0, u(i+1)) - u0 (u0 <= 0) are the same values as this cell formula for cells i and i+1.
template <typename T, class A, class PA, class M = TvdMetricScalar>
__device__ __forceinline__ T cell_cfl_out(const Scalars& s, const PA& P, const A& U, const A& V, const A& W, int k,
                                          int j, int i) {
  const T cx = (T)s.cx, cy = (T)s.cy;
  T sum = (T)0.0;
  sum = sum + P(M::RDZ, k) * (tmax<T>((T)0.0, W(k, j, i)) + fabs(tmin<T>((T)0.0, W(k - 1, j, i))));
  sum = sum + cy * (tmax<T>((T)0.0, V(k, j, i)) + fabs(tmin<T>((T)0.0, V(k, j - 1, i))));
  sum = sum + cx * (tmax<T>((T)0.0, U(k, j, i)) + fabs(tmin<T>((T)0.0, U(k, j, i - 1))));
  return sum;
}

// The cell sums evaluated from the advecting flow where a face needs them
template <typename T, class A, class PA, class M>
struct CflInline {
  const Scalars& s;
  const PA& P;
  const A& U;
  const A& V;
  const A& W;
  __device__ __forceinline__ T operator()(int k, int j, int i) const {
    return cell_cfl_out<T, A, PA, M>(s, P, U, V, W, k, j, i);
  }
};

// face x+1/2 of cell (k, j, i): flux_previous_x(k) of ultflx; cfl(k, j, i) gives cell_cfl_out
template <typename T, class A, class AF, class PA, class M, class CS, class Rec = NoRec>
__device__ T tvd_face_x_g(const Scalars& s, const PA& P, const A& U, const A& V, const A& W,
                          const AF& ZF, T dt, int k, int j, int i, const CS& cfl, const Rec& rec = Rec()) {
  const int nz = s.nz;
  const T cx = (T)s.cx, cy = (T)s.cy;
  const int kp1 = k + 1 < nz ? k + 1 : nz;
  const int kp0 = kp1 - 1;
  const T u0 = U(k, j, i);
  T sm = tsign<T>((T).5, u0);
  T advpos = (T)0.5 + sm, advneg = (T)0.5 - sm;
  T fu = ZF(k, j, i - 1) * advpos + ZF(k, j, i + 2) * advneg;
  T fc = ZF(k, j, i) * advpos + ZF(k, j, i + 1) * advneg;
  T fd = ZF(k, j, i + 1) * advpos + ZF(k, j, i) * advneg;
  T fdels = fd - fu;
  T fcurvs = fd - (T)2.0 * fc + fu;
  rec(signbit(u0) ? 1u : 0u, 1);
  rec(fabs(fcurvs) >= fabs(fdels) ? 1u : 0u, 1);
  if (fabs(fcurvs) >= fabs(fdels)) return fc;
  // the upwind cell: i when u0 > 0, otherwise i + 1 (u0 = 0 included, as ultflx tests u > 0)
  rec(u0 > (T)0.0 ? 1u : 0u, 1);
  T sum = cfl(k, j, u0 > (T)0.0 ? i : i + 1) * dt;
  // gradient term in z (calculate_gradient_term_in_z with two source columns)
  T fgt1;
  {
    T sf = (T)0.125 * (W(k, j, i) + W(k - 1, j, i) + W(k, j, i + 1) + W(k - 1, j, i + 1));
    bool pos = !signbit(sf);
    rec(pos ? 1u : 0u, 1);
    int ksu = pos ? k - 1 : kp1;
    int ksl = pos ? k : kp0;
    T ts = ZF(ksl, j, i) - ZF(ksu, j, i);
    ts = ts * advpos + (ZF(ksl, j, i + 1) - ZF(ksu, j, i + 1)) * advneg;
    fgt1 = fabs(sf) * P(M::RDZ, k + M::KDOF) * dt * ts;
  }
  // gradient term in y with two v columns
  T fgt2;
  {
    T sf = (T)0.125 * (V(k, j, i + 1) + V(k, j, i) + V(k, j - 1, i + 1) + V(k, j - 1, i));
    rec(signbit(sf) ? 1u : 0u, 1);
    int jsu = signbit(sf) ? j + 1 : j - 1;
    T t1 = ZF(k, jsu, i) * advpos;
    T t2 = ZF(k, jsu, i + 1) * advneg;
    t1 = t1 + t2;
    fgt2 = fabs(sf) * cy * dt * (fc - t1);
  }
  return limit_face<T, Rec>(u0, cx, dt, sum, fdels, fd, fc, fu, fgt1, fgt2, fcurvs, rec);
}

template <typename T, class A, class AF, class PA, class M = TvdMetricScalar>
__device__ T tvd_face_x(const Scalars& s, const PA& P, const A& U, const A& V, const A& W,
                        const AF& ZF, T dt, int k, int j, int i) {
  return tvd_face_x_g<T, A, AF, PA, M>(s, P, U, V, W, ZF, dt, k, j, i, CflInline<T, A, PA, M>{s, P, U, V, W});
}

// face y+1/2 of cell (k, j, i): flux_y(k) of ultflx
template <typename T, class A, class AF, class PA, class M, class CS, class Rec = NoRec>
__device__ T tvd_face_y_g(const Scalars& s, const PA& P, const A& U, const A& V, const A& W,
                          const AF& ZF, T dt, int k, int j, int i, const CS& cfl, const Rec& rec = Rec()) {
  const int nz = s.nz;
  const T cx = (T)s.cx, cy = (T)s.cy;
  const int kp1 = k + 1 < nz ? k + 1 : nz;
  const int kp0 = kp1 - 1;
  const T v0 = V(k, j, i);
  T sm = tsign<T>((T)0.5, v0);
  T advpos = (T)0.5 + sm, advneg = (T)0.5 - sm;
  int jo = signbit(v0) ? 1 : 0;  // jofset = nint(advneg)
  T fu = ZF(k, j - 1, i) * advpos + ZF(k, j + 2, i) * advneg;
  T fc = ZF(k, j, i) * advpos + ZF(k, j + 1, i) * advneg;
  T fd = ZF(k, j + 1, i) * advpos + ZF(k, j, i) * advneg;
  T fdels = fd - fu;
  T fcurvs = fd - (T)2.0 * fc + fu;
  rec((unsigned)jo, 1);
  rec(fabs(fcurvs) >= fabs(fdels) ? 1u : 0u, 1);
  if (fabs(fcurvs) >= fabs(fdels)) return fc;
  T sum = cfl(k, j + jo, i) * dt;
  T fgt1;
  {
    T sf = (T)0.125 * (W(k, j, i) + W(k - 1, j, i) + W(k, j + 1, i) + W(k - 1, j + 1, i));
    bool pos = !signbit(sf);
    rec(pos ? 1u : 0u, 1);
    int ksu = pos ? k - 1 : kp1;
    int ksl = pos ? k : kp0;
    T ts = ZF(ksl, j + jo, i) - ZF(ksu, j + jo, i);
    fgt1 = fabs(sf) * P(M::RDZ, k + M::KDOF) * dt * ts;
  }
  T fgt2;
  {
    T sf = (T)0.125 * (U(k, j, i - 1) + U(k, j, i) + U(k, j + 1, i - 1) + U(k, j + 1, i));
    rec(signbit(sf) ? 1u : 0u, 1);
    T posuf = (T)0.5 + tsign<T>((T).5, sf);
    fgt2 = fabs(sf) * cx * dt * (fc - (ZF(k, j + jo, i + 1) * ((T)1. - posuf) + ZF(k, j + jo, i - 1) * posuf));
  }
  return limit_face<T, Rec>(v0, cy, dt, sum, fdels, fd, fc, fu, fgt1, fgt2, fcurvs, rec);
}

template <typename T, class A, class AF, class PA, class M = TvdMetricScalar>
__device__ T tvd_face_y(const Scalars& s, const PA& P, const A& U, const A& V, const A& W,
                        const AF& ZF, T dt, int k, int j, int i) {
  return tvd_face_y_g<T, A, AF, PA, M>(s, P, U, V, W, ZF, dt, k, j, i, CflInline<T, A, PA, M>{s, P, U, V, W});
}

// flux_z(k+1): face above level k (2 <= k <= nz-1); the top routine handles k = nz-1
template <typename T, class A, class AF, class PA, class M, class CS, class Rec = NoRec>
__device__ T tvd_face_z_g(const Scalars& s, const PA& P, const A& U, const A& V, const A& W,
                          const AF& ZF, T dt, int k, int j, int i, const CS& cfl, const Rec& rec = Rec()) {
  const int nz = s.nz;
  const T cx = (T)s.cx, cy = (T)s.cy;
  const T w0 = W(k, j, i);
  T fu, fc, fd, rdu, rdc, sum, fgt1, fgt2;
  int kf;  // level of the upwind-side values used by the gradient terms
  if (k == nz - 1) {
    bool up = w0 >= (T)0.0;
    if (up) { fu = ZF(k - 1, j, i); fc = ZF(k, j, i); fd = ZF(k + 1, j, i); }
    else { fu = (T)2.0 * ZF(k + 1, j, i) - ZF(k, j, i); fc = ZF(k + 1, j, i); fd = ZF(k, j, i); }
    T fcurvs = fd - (T)2.0 * fc + fu;
    T fdels = fd - fu;
    rec(up ? 1u : 0u, 1);
    rec(fabs(fcurvs) >= fabs(fdels) ? 1u : 0u, 1);
    if (fabs(fcurvs) >= fabs(fdels)) return fc;
    if (up) {
      sum = (T)0.0;
      sum = sum + P(M::RDZ, k + M::KDOF) * (w0 + fabs(tmin<T>((T)0.0, W(k - 1, j, i))));
      sum = sum + cy * (tmax<T>((T)0.0, V(k, j, i)) + fabs(tmin<T>((T)0.0, V(k, j - 1, i))));
      sum = sum + cx * (tmax<T>((T)0.0, U(k, j, i)) + fabs(tmin<T>((T)0.0, U(k, j, i - 1))));
      sum = sum * dt;
      kf = k;
      rdu = P(M::RDZN, k);
      rdc = P(M::RDZ, k + M::KDOF);
    } else {
      sum = (T)0.0;
      sum = sum + (-w0 * P(M::RDZ, nz < k + 1 + M::KDOF ? nz : k + 1 + M::KDOF));
      sum = sum + cy * (tmax<T>((T)0.0, V(k + 1, j, i)) + fabs(tmin<T>((T)0.0, V(k + 1, j - 1, i))));
      sum = sum + cx * (tmax<T>((T)0.0, U(k + 1, j, i)) + fabs(tmin<T>((T)0.0, U(k + 1, j, i - 1))));
      sum = sum * dt;
      kf = k + 1;
      rdu = P(M::RDZN, nz);
      rdc = P(M::RDZ, nz < k + 1 + M::KDOF ? nz : k + 1 + M::KDOF);
    }
    {
      T sf = (T)0.125 * (V(k, j - 1, i) + V(k, j, i) + V(k + 1, j - 1, i) + V(k + 1, j, i));
      rec(signbit(sf) ? 1u : 0u, 1);
      int jsu = signbit(sf) ? j + 1 : j - 1;
      fgt1 = fabs(sf) * cy * dt * (fc - ZF(kf, jsu, i));
    }
    {
      T sf = (T)0.125 * (U(k, j, i - 1) + U(k, j, i) + U(k + 1, j, i - 1) + U(k + 1, j, i));
      rec(signbit(sf) ? 1u : 0u, 1);
      T posuf = (T)0.5 + tsign<T>((T).5, sf);
      fgt2 = fabs(sf) * cx * dt * (fc - (ZF(kf, j, i + 1) * ((T)1. - posuf) + ZF(kf, j, i - 1) * posuf));
    }
    // calculate_flux_in_w
    T dd = P(M::DZN, k + 1), rdd = P(M::RDZN, k + 1);
    T cflmod = fabs(w0 * rdd * dt);
    T hrcfl = rcp(sum + (T)1.e-30);
    T hcfl = (T)0.5 * cflmod;
    T cflcoef = (T)(1.0 / 6.0) * ((T)1.0 - cflmod * cflmod) * (dd * dd * rdc);
    T ffs = (T)0.5 * (fd + fc) - hcfl * (fd - fc) - cflcoef * ((fd - fc) * rdd - (fc - fu) * rdu) - fgt1 - fgt2;
    return limited_face<T, Rec>(ffs, fc, fu, fdels, hrcfl, rec);
  }
  // middle of the column
  T sm = tsign<T>((T).5, w0);
  T advpos = (T)0.5 + sm, advneg = (T)0.5 - sm;
  int ko = signbit(w0) ? 1 : 0;  // kofset
  fu = ZF(k - 1, j, i) * advpos + ZF(k + 2, j, i) * advneg;
  fc = ZF(k + ko, j, i);
  fd = ZF(k + 1, j, i) * advpos + ZF(k, j, i) * advneg;
  T fcurvs = fd - (T)2.0 * fc + fu;
  T fdels = fd - fu;
  rec((unsigned)ko, 1);
  rec(fabs(fcurvs) >= fabs(fdels) ? 1u : 0u, 1);
  if (fabs(fcurvs) >= fabs(fdels)) return fc;
  sum = cfl(k + ko, j, i) * dt;
  {
    T sf = (T)0.125 * (V(k, j - 1, i) + V(k, j, i) + V(k + 1, j - 1, i) + V(k + 1, j, i));
    rec(signbit(sf) ? 1u : 0u, 1);
    int jsu = signbit(sf) ? j + 1 : j - 1;
    fgt1 = fabs(sf) * cy * dt * (fc - ZF(k + ko, jsu, i));
  }
  {
    T sf = (T)0.125 * (U(k, j, i - 1) + U(k, j, i) + U(k + 1, j, i - 1) + U(k + 1, j, i));
    rec(signbit(sf) ? 1u : 0u, 1);
    T posuf = (T)0.5 + tsign<T>((T).5, sf);
    fgt2 = fabs(sf) * cx * dt * (fc - (ZF(k + ko, j, i + 1) * ((T)1. - posuf) + ZF(k + ko, j, i - 1) * posuf));
  }
  rdu = P(M::RDZN, k) * advpos + P(M::RDZN, k + 2) * advneg;
  rdc = P(M::RDZ, k + M::KDOF) * advpos + P(M::RDZ, k + 1 + M::KDOF) * advneg;
  T dd = P(M::DZN, k + 1), rdd = P(M::RDZN, k + 1);
  T cflmod = fabs(w0 * rdd * dt);
  T hrcfl = rcp(sum + (T)1.e-30);
  T hcfl = (T)0.5 * cflmod;
  T cflcoef = (T)(1.0 / 6.0) * ((T)1.0 - cflmod * cflmod) * (dd * dd * rdc);
  T ffs = (T)0.5 * (fd + fc) - hcfl * (fd - fc) - cflcoef * ((fd - fc) * rdd - (fc - fu) * rdu) - fgt1 - fgt2;
  return limited_face<T, Rec>(ffs, fc, fu, fdels, hrcfl, rec);
}

template <typename T, class A, class AF, class PA, class M = TvdMetricScalar>
__device__ T tvd_face_z(const Scalars& s, const PA& P, const A& U, const A& V, const A& W,
                        const AF& ZF, T dt, int k, int j, int i) {
  return tvd_face_z_g<T, A, AF, PA, M>(s, P, U, V, W, ZF, dt, k, j, i, CflInline<T, A, PA, M>{s, P, U, V, W});
}


// TVD source of cell (k, j, i), 2 <= k <= nz, from the six face values
// acc0 is the source value before the callback (MONC accumulates into it below the top level
// and zeroes it at the top level)
template <typename T, class A, class PA, class M = TvdMetricScalar>
__device__ T tvd_source(const Scalars& s, const PA& P, const A& U, const A& V, const A& W,
                        T fx_m, T fx_p, T fy_m, T fy_p, T fz_m, T fz_p, int k, int j, int i, T acc0) {
  const T cx = (T)s.cx, cy = (T)s.cy;
  T acc = (k < s.nz) ? acc0 : (T)0.0;
  if (k < s.nz) {
    acc = acc + (V(k, j - 1, i) * fy_m - V(k, j, i) * fy_p) * cy;
    acc = acc + (T)4.0 * (W(k - 1, j, i) * fz_m * P(M::TZ1, k) - W(k, j, i) * fz_p * P(M::TZ2, k));
    acc = acc + (U(k, j, i - 1) * fx_m - U(k, j, i) * fx_p) * cx;
  } else {
    acc = acc + (V(k, j - 1, i) * fy_m - V(k, j, i) * fy_p) * cy;
    acc = acc + (T)4.0 * P(M::TZ1, k) * W(k - 1, j, i) * fz_m;
    acc = acc + (U(k, j, i - 1) * fx_m - U(k, j, i) * fx_p) * cx;
  }
  return acc;
}

template <typename T, class A, class PA>
__device__ T tvd_point(const Scalars& s, const PA& P, const A& U, const A& V, const A& W,
                       const A& ZF, int k, int j, int i, T acc0) {
  const T dt = (T)(s.dtm * 2.0);
  T fxm = tvd_face_x<T, A>(s, P, U, V, W, ZF, dt, k, j, i - 1);
  T fxp = tvd_face_x<T, A>(s, P, U, V, W, ZF, dt, k, j, i);
  T fym = tvd_face_y<T, A>(s, P, U, V, W, ZF, dt, k, j - 1, i);
  T fyp = tvd_face_y<T, A>(s, P, U, V, W, ZF, dt, k, j, i);
  T fzm = (k == 2) ? (T)0.0 : tvd_face_z<T, A>(s, P, U, V, W, ZF, dt, k - 1, j, i);
  T fzp = (k < s.nz) ? tvd_face_z<T, A>(s, P, U, V, W, ZF, dt, k, j, i) : (T)0.0;
  return tvd_source<T, A>(s, P, U, V, W, fxm, fxp, fym, fyp, fzm, fzp, k, j, i, acc0);
}

// ------------------------------------------------------------------------------------------
// TVD advection of the flow fields (tvdadvection.F90:603-908, advection_flow_fields = tvd)
// ------------------------------------------------------------------------------------------
// The advecting flow of u, v or w: interpolate_to_dual (stencil.F90:87-169) averages each flow
// component with its neighbour one point along the direction in which the advected field sits on
// the primal grid -- x for u, y for v, z for w (simplesetup.F90:70-85) -- and keeps the top level
// as it is for w.  MONC also keeps the value where that neighbour lies outside its local arrays,
// the outermost halo column or row; the faces of interior points never read those.
template <typename T, class A, int DIM>
struct DualFlow {
  A a;
  int nz;
  __device__ __forceinline__ T operator()(int k, int j, int i) const {
    if (DIM == 0) return (T)0.5 * (a(k, j, i) + a(k, j, i + 1));
    if (DIM == 1) return (T)0.5 * (a(k, j, i) + a(k, j + 1, i));
    return k == nz ? a(k, j, i) : (T)0.5 * (a(k, j, i) + a(k + 1, j, i));
  }
};

// flux_z(2) of w's advection: handle_vertical_fluxes_bottomofcolumn (ultimateflux.F90:307-412),
// the face above level 1 (only w's metrics reach it: kmin = 1)
template <typename T, class A, class AF, class PA, class M>
__device__ T tvd_face_z_bottom(const Scalars& s, const PA& P, const A& U, const A& V, const A& W, const AF& ZF, T dt,
                               int j, int i) {
  const int k = 1;
  const T cx = (T)s.cx, cy = (T)s.cy;
  const T w0 = W(k, j, i);
  const bool up = w0 >= (T)0.0;
  T fu, fc, fd;
  if (up) { fu = ZF(1, j, i); fc = ZF(k, j, i); fd = ZF(k + 1, j, i); }
  else { fu = ZF(k + 2, j, i); fc = ZF(k + 1, j, i); fd = ZF(k, j, i); }
  T fcurvs = fd - (T)2.0 * fc + fu;
  T fdels = fd - fu;
  if (fabs(fcurvs) >= fabs(fdels)) return fc;
  T sum, rdu, rdc;
  const int kf = up ? k : k + 1;  // level of the values the gradient terms take
  if (up) {
    sum = (T)0.0;
    sum = sum + w0 * P(M::RDZ, k + M::KDOF);
    sum = sum + cy * (tmax<T>((T)0.0, V(k, j, i)) + fabs(tmin<T>((T)0.0, V(k, j - 1, i))));
    sum = sum + cx * (tmax<T>((T)0.0, U(k, j, i)) + fabs(tmin<T>((T)0.0, U(k, j, i - 1))));
    sum = sum * dt;
    rdu = P(M::RDZN, 2);
    rdc = P(M::RDZ, k + M::KDOF);
  } else {
    sum = (T)0.0;
    sum = sum + P(M::RDZ, k + 1 + M::KDOF) * (tmax<T>((T)0.0, W(k + 1, j, i)) - w0);
    sum = sum + cy * (tmax<T>((T)0.0, V(k + 1, j, i)) + fabs(tmin<T>((T)0.0, V(k + 1, j - 1, i))));
    sum = sum + cx * (tmax<T>((T)0.0, U(k + 1, j, i)) + fabs(tmin<T>((T)0.0, U(k + 1, j, i - 1))));
    sum = sum * dt;
    rdu = P(M::RDZN, k + 2);
    rdc = P(M::RDZ, k + 1 + M::KDOF);
  }
  T fgt1, fgt2;
  {
    T sf = (T)0.125 * (V(k, j - 1, i) + V(k, j, i) + V(k + 1, j - 1, i) + V(k + 1, j, i));
    int jsu = signbit(sf) ? j + 1 : j - 1;
    fgt1 = fabs(sf) * cy * dt * (fc - ZF(kf, jsu, i));
  }
  {
    T sf = (T)0.125 * (U(k, j, i - 1) + U(k, j, i) + U(k + 1, j, i - 1) + U(k + 1, j, i));
    T posuf = (T)0.5 + tsign<T>((T).5, sf);
    fgt2 = fabs(sf) * cx * dt * (fc - (ZF(kf, j, i + 1) * ((T)1. - posuf) + ZF(kf, j, i - 1) * posuf));
  }
  T dd = P(M::DZN, k + 1), rdd = P(M::RDZN, k + 1);
  T cflmod = fabs(w0 * rdd * dt);
  T hrcfl = rcp(sum + (T)1.e-30);
  T hcfl = (T)0.5 * cflmod;
  T cflcoef = (T)(1.0 / 6.0) * ((T)1.0 - cflmod * cflmod) * (dd * dd * rdc);
  T ffs = (T)0.5 * (fd + fc) - hcfl * (fd - fc) - cflcoef * ((fd - fc) * rdd - (fc - fu) * rdu) - fgt1 - fgt2;
  return limited_face<T>(ffs, fc, fu, fdels, hrcfl);
}

// TVD sources of u, v (2 <= k <= nz) and w (2 <= k <= nz-1) at (k, j, i), added to su_in, sv_in,
// sw_in as differentiate_face_values adds them (u and v restart from 0 at the top level; w has no
// top-level source).  U, V, W are the current flow fields, ZU, ZV, ZW the advected ones.
template <typename T, class A, class PA>
__device__ void tvd_flow_point(const Scalars& s, const PA& P, const A& U, const A& V, const A& W, const A& ZU,
                               const A& ZV, const A& ZW, int k, int j, int i, T su_in, T sv_in, T sw_in, T& su, T& sv,
                               T& sw) {
  const T dt = (T)(s.dtm * 2.0);  // momentum_stepping is always centred (steppingdirection.F90:32)
  const int nz = s.nz;
  {
    typedef DualFlow<T, A, 0> F;
    const F IU{U, nz}, IV{V, nz}, IW{W, nz};
    T fxm = tvd_face_x<T, F, A, PA, TvdMetricScalar>(s, P, IU, IV, IW, ZU, dt, k, j, i - 1);
    T fxp = tvd_face_x<T, F, A, PA, TvdMetricScalar>(s, P, IU, IV, IW, ZU, dt, k, j, i);
    T fym = tvd_face_y<T, F, A, PA, TvdMetricScalar>(s, P, IU, IV, IW, ZU, dt, k, j - 1, i);
    T fyp = tvd_face_y<T, F, A, PA, TvdMetricScalar>(s, P, IU, IV, IW, ZU, dt, k, j, i);
    T fzm = (k == 2) ? (T)0.0 : tvd_face_z<T, F, A, PA, TvdMetricScalar>(s, P, IU, IV, IW, ZU, dt, k - 1, j, i);
    T fzp = (k < nz) ? tvd_face_z<T, F, A, PA, TvdMetricScalar>(s, P, IU, IV, IW, ZU, dt, k, j, i) : (T)0.0;
    su = tvd_source<T, F, PA, TvdMetricScalar>(s, P, IU, IV, IW, fxm, fxp, fym, fyp, fzm, fzp, k, j, i, su_in);
  }
  {
    typedef DualFlow<T, A, 1> F;
    const F IU{U, nz}, IV{V, nz}, IW{W, nz};
    T fxm = tvd_face_x<T, F, A, PA, TvdMetricScalar>(s, P, IU, IV, IW, ZV, dt, k, j, i - 1);
    T fxp = tvd_face_x<T, F, A, PA, TvdMetricScalar>(s, P, IU, IV, IW, ZV, dt, k, j, i);
    T fym = tvd_face_y<T, F, A, PA, TvdMetricScalar>(s, P, IU, IV, IW, ZV, dt, k, j - 1, i);
    T fyp = tvd_face_y<T, F, A, PA, TvdMetricScalar>(s, P, IU, IV, IW, ZV, dt, k, j, i);
    T fzm = (k == 2) ? (T)0.0 : tvd_face_z<T, F, A, PA, TvdMetricScalar>(s, P, IU, IV, IW, ZV, dt, k - 1, j, i);
    T fzp = (k < nz) ? tvd_face_z<T, F, A, PA, TvdMetricScalar>(s, P, IU, IV, IW, ZV, dt, k, j, i) : (T)0.0;
    sv = tvd_source<T, F, PA, TvdMetricScalar>(s, P, IU, IV, IW, fxm, fxp, fym, fyp, fzm, fzp, k, j, i, sv_in);
  }
  sw = sw_in;
  if (k <= nz - 1) {
    typedef DualFlow<T, A, 2> F;
    const F IU{U, nz}, IV{V, nz}, IW{W, nz};
    T fxm = tvd_face_x<T, F, A, PA, TvdMetricW>(s, P, IU, IV, IW, ZW, dt, k, j, i - 1);
    T fxp = tvd_face_x<T, F, A, PA, TvdMetricW>(s, P, IU, IV, IW, ZW, dt, k, j, i);
    T fym = tvd_face_y<T, F, A, PA, TvdMetricW>(s, P, IU, IV, IW, ZW, dt, k, j - 1, i);
    T fyp = tvd_face_y<T, F, A, PA, TvdMetricW>(s, P, IU, IV, IW, ZW, dt, k, j, i);
    T fzm = (k == 2) ? tvd_face_z_bottom<T, F, A, PA, TvdMetricW>(s, P, IU, IV, IW, ZW, dt, j, i)
                     : tvd_face_z<T, F, A, PA, TvdMetricW>(s, P, IU, IV, IW, ZW, dt, k - 1, j, i);
    T fzp = tvd_face_z<T, F, A, PA, TvdMetricW>(s, P, IU, IV, IW, ZW, dt, k, j, i);
    sw = tvd_source<T, F, PA, TvdMetricW>(s, P, IU, IV, IW, fxm, fxp, fym, fyp, fzm, fzp, k, j, i, sw_in);
  }
}

// ------------------------------------------------------------------------------------------
// th_advection (thadvection.F90:196-216): the advection of the mean baroclinicity, Boussinesq
// form, added to the theta source at 2 <= k <= nz; u, v are the current flow fields
// ------------------------------------------------------------------------------------------
template <typename T, class A>
__device__ __forceinline__ T th_baroclinic_point(const Scalars& s, const A& U, const A& V, int k, int j, int i) {
  return (V(k, j, i) + (T)s.vgal) * (T)s.mfx - (U(k, j, i) + (T)s.ugal) * (T)s.mfy;
}

// ------------------------------------------------------------------------------------------
// diffusion general_diffusion (diffusion.F90:501-545), 2 <= k <= nz
// ------------------------------------------------------------------------------------------
template <typename T, class AF, class AD, class PA>
__device__ T diffusion_point(const Scalars& s, const PA& P, const AF& F, const AD& D, int k, int j, int i) {
  const T f0 = F(k, j, i), d0 = D(k, j, i), dm = D(k - 1, j, i);
  T term = (T)s.cx2 * (T)0.25 *
               (((d0 + D(k, j, i - 1)) + (dm + D(k - 1, j, i - 1))) * (F(k, j, i - 1) - f0) -
                ((D(k, j, i + 1) + d0) + (D(k - 1, j, i + 1) + dm)) * (f0 - F(k, j, i + 1))) +
           (T)s.cy2 * (T)0.25 *
               (((d0 + D(k, j - 1, i)) + (dm + D(k - 1, j - 1, i))) * (F(k, j - 1, i) - f0) -
                ((D(k, j + 1, i) + d0) + (D(k - 1, j + 1, i) + dm)) * (f0 - F(k, j + 1, i))) +
           (P(P_CZB, k) * dm * (F(k - 1, j, i) - f0));
  if (k < s.nz) term = term - P(P_CZA, k) * d0 * (f0 - F(k + 1, j, i));
  return term;
}

}  // namespace mgpu
