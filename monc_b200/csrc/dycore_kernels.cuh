// Dynamical-core kernels: MONC's column callbacks as whole-domain CUDA kernels.
//
// Two families share the device functions of dycore_device.cuh:
//  * component kernels (k_c_*): one MONC component each, reading and writing the same
//    fields as the Fortran callback (sources su/sv/sw/sth explicit), for drop-in use;
//  * fused step kernels (k_f_*): the whole timestep in five passes over memory
//      1. subgrid   : lower_bc + smagorinsky                        -> vis, diff, th(1)/zth(1)
//      2. dynamics  : pw + tvd + diffusion + viscosity + coriolis + buoyancy + stepfields
//                     (+ swap_smooth of theta)                     -> z-velocities, th, zth
//      3. pressure source: diverr + psrce from the stepped z-velocities -> p
//      4. pressure solve (fft.cu)
//      5. pstep + swap_smooth of the velocities
//    Sources live in registers and never reach memory.
// MONC's per-column ordering (stepfields lagging two columns, TVD carrying face fluxes, psrce
// deferring the first column's faces) is equivalent to this whole-field ordering on a periodic
// domain; the CPU oracle keeps MONC's column order and the parity tests compare the two.
#pragma once
#include <cuda_runtime.h>

#include "dycore.h"
#include "dycore_device.cuh"

namespace mgpu {

static inline dim3 pt_block() { return dim3(32, 8, 1); }
static inline dim3 pt_grid(const Scalars& s, int kcount) {
  return dim3((s.nx + 31) / 32, (s.ny + 7) / 8, kcount);
}

template <typename T>
__device__ __forceinline__ View<T> view(const T* p, const Scalars& s) {
  View<T> v;
  v.p = p;
  v.g.nx = s.nx;
  v.g.ny = s.ny;
  v.g.nz = s.nz;
  v.g.plane = s.plane;
  return v;
}

template <typename T>
__device__ __forceinline__ Prof<T> prof(const Scalars& s) {
  Prof<T> P;
  P.base = s.prof;
  P.stride = s.nz + 2;
  return P;
}

__device__ __forceinline__ long long lin(const Scalars& s, int k, int j, int i) {
  return (long long)(k - 1) * s.plane + (long long)j * s.nx + i;
}

// ==========================================================================================
// Component kernels
// ==========================================================================================

// lower_bc: one thread per column
template <typename T>
__global__ void k_c_lower_bc(Scalars s, DevState<T> d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= s.nx || j >= s.ny) return;
  Prof<T> P = prof<T>(s);
  bool fwd = s.forward;
  View<T> zus = view<T>(d.zu, s);
  View<T> zua = view<T>(fwd ? d.u : d.zu, s);
  View<T> zva = view<T>(fwd ? d.v : d.zv, s);
  T* tha = fwd ? d.th : d.zth;
  View<T> thv = view<T>(tha, s);
  View<T> qv;
  T* qa = nullptr;
  if (s.nq > 0) {
    qa = fwd ? d.q[s.iqv] : d.zq[s.iqv];
    qv = view<T>(qa, s);
  }
  T vis1, diff1, th1, qv1;
  lower_bc_column<T>(s, P, zus, zua, zva, thv, s.nq > 0 ? &qv : nullptr, j, i, vis1, diff1, th1, qv1);
  long long o = lin(s, 1, j, i);
  d.vis[o] = vis1;
  d.diff[o] = diff1;
  tha[o] = th1;
  if (qa) qa[o] = qv1;
}

// smagorinsky: levels 2..nz (top level zeroed)
template <typename T>
__global__ void k_c_smagorinsky(Scalars s, DevState<T> d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z + 2;
  if (i >= s.nx || j >= s.ny || k > s.nz) return;
  long long o = lin(s, k, j, i);
  if (k == s.nz) { d.vis[o] = (T)0.0; d.diff[o] = (T)0.0; return; }
  Prof<T> P = prof<T>(s);
  bool fwd = s.forward;
  View<T> U = view<T>(fwd ? d.u : d.zu, s), V = view<T>(fwd ? d.v : d.zv, s), W = view<T>(fwd ? d.w : d.zw, s);
  View<T> THc = view<T>(d.th, s), THa = view<T>(fwd ? d.th : d.zth, s);
  View<T> QV, QL;
  if (!s.passive_q && s.nq > 1) {
    QV = view<T>(fwd ? d.q[s.iqv] : d.zq[s.iqv], s);
    QL = view<T>(fwd ? d.q[s.iql] : d.zq[s.iql], s);
  }
  T vis, diff;
  smagorinsky_point<T>(s, P, U, V, W, THc, THa, &QV, &QL, k, j, i, vis, diff);
  d.vis[o] = vis;
  d.diff[o] = diff;
}

template <typename T>
__global__ void k_c_pw(Scalars s, DevState<T> d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z + 2;
  if (i >= s.nx || j >= s.ny || k > s.nz) return;
  Prof<T> P = prof<T>(s);
  View<T> U = view<T>(d.u, s), V = view<T>(d.v, s), W = view<T>(d.w, s);
  T su, sv, sw;
  pw_point<T>(s, P, U, V, W, k, j, i, su, sv, sw);
  long long o = lin(s, k, j, i);
  d.su[o] = su;
  d.sv[o] = sv;
  if (k < s.nz) d.sw[o] = sw;
}

template <typename T>
__global__ void k_c_tvd(Scalars s, DevState<T> d, const T* zf_th, T* sth, int n_extra) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z + 2;
  if (i >= s.nx || j >= s.ny || k > s.nz) return;
  Prof<T> P = prof<T>(s);
  View<T> U = view<T>(d.u, s), V = view<T>(d.v, s), W = view<T>(d.w, s);
  long long o = lin(s, k, j, i);
  bool fwd = s.forward;
  // theta, then each q field (advect_theta, advect_q_fields)
  {
    View<T> ZF = view<T>(fwd ? d.th : d.zth, s);
    d.sth[o] = tvd_point<T>(s, P, U, V, W, ZF, k, j, i, d.sth[o]);
  }
  for (int n = 0; n < s.nq; ++n) {
    View<T> ZF = view<T>(fwd ? d.q[n] : d.zq[n], s);
    d.sq[n][o] = tvd_point<T>(s, P, U, V, W, ZF, k, j, i, d.sq[n][o]);
  }
  (void)zf_th; (void)sth; (void)n_extra;
}

template <typename T>
__global__ void k_c_diffusion(Scalars s, DevState<T> d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z + 2;
  if (i >= s.nx || j >= s.ny || k > s.nz) return;
  Prof<T> P = prof<T>(s);
  View<T> D = view<T>(d.diff, s);
  long long o = lin(s, k, j, i);
  d.sth[o] = d.sth[o] + diffusion_point<T>(s, P, view<T>(d.zth, s), D, k, j, i);
  for (int n = 0; n < s.nq; ++n) d.sq[n][o] = d.sq[n][o] + diffusion_point<T>(s, P, view<T>(d.zq[n], s), D, k, j, i);
}

template <typename T>
__global__ void k_c_viscosity(Scalars s, DevState<T> d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z + 2;
  if (i >= s.nx || j >= s.ny || k > s.nz) return;
  Prof<T> P = prof<T>(s);
  bool fwd = s.forward;
  View<T> ZU = view<T>(fwd ? d.u : d.zu, s), ZV = view<T>(fwd ? d.v : d.zv, s), ZW = view<T>(fwd ? d.w : d.zw, s);
  T du, dv, dw;
  viscosity_point<T>(s, P, ZU, ZV, ZW, view<T>(d.zu, s), view<T>(d.vis, s), k, j, i, du, dv, dw);
  long long o = lin(s, k, j, i);
  d.su[o] = d.su[o] + du;
  d.sv[o] = d.sv[o] + dv;
  if (k < s.nz) d.sw[o] = d.sw[o] + dw;
}

template <typename T>
__global__ void k_c_coriolis(Scalars s, DevState<T> d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z + 2;
  if (i >= s.nx || j >= s.ny || k > s.nz) return;
  Prof<T> P = prof<T>(s);
  long long o = lin(s, k, j, i);
  T su = d.su[o], sv = d.sv[o];
  coriolis_point<T>(s, P, view<T>(d.u, s), view<T>(d.v, s), k, j, i, su, sv);
  d.su[o] = su;
  d.sv[o] = sv;
}

template <typename T>
__global__ void k_c_buoyancy(Scalars s, DevState<T> d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z + 2;
  if (i >= s.nx || j >= s.ny || k >= s.nz) return;
  Prof<T> P = prof<T>(s);
  View<T> Q[MGPU_MAX_Q];
  for (int n = 0; n < s.nq; ++n) Q[n] = view<T>(d.q[n], s);
  long long o = lin(s, k, j, i);
  d.sw[o] = buoyancy_point<T>(s, P, view<T>(d.th, s), Q, k, j, i, d.sw[o]);
}

template <typename T>
__global__ void k_c_set_consistent_lowbc(Scalars s, DevState<T> d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= s.nx || j >= s.ny) return;
  long long o1 = lin(s, 1, j, i), o2 = lin(s, 2, j, i);
  if (s.use_vd && s.surface_bcs) { d.su[o1] = -d.su[o2]; d.sv[o1] = -d.sv[o2]; }
  else { d.su[o1] = d.su[o2]; d.sv[o1] = d.sv[o2]; }
  if (s.surface_bcs) d.sth[o1] = d.sth[o2];  // prescribed surface fluxes
  for (int n = 0; n < s.nq; ++n) d.sq[n][o1] = d.sq[n][o2];
}

// diverr: p from the divergence of the (z-)velocities; |p| max into *divmax (bit pattern)
template <typename T>
__global__ void k_c_diverr(Scalars s, DevState<T> d, unsigned long long* divmax) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z + 1;
  if (i >= s.nx || j >= s.ny || k > s.nz) return;
  long long o = lin(s, k, j, i);
  if (k == 1) { d.p[o] = (T)0.0; return; }
  Prof<T> P = prof<T>(s);
  bool fwd = s.forward;
  T timec = fwd ? (T)(1.0 / s.dtm) : (T)(1.0 / (2.0 * s.dtm));
  View<T> U = view<T>(fwd ? d.u : d.zu, s), V = view<T>(fwd ? d.v : d.zv, s), W = view<T>(fwd ? d.w : d.zw, s);
  T pp = (T)0.0;
  pp = pp + (T)s.cx * (U(k, j, i) - U(k, j, i - 1));
  pp = pp + (T)s.cy * (V(k, j, i) - V(k, j - 1, i));
  pp = pp + (T)4.0 * (P(P_TZC2, k) * W(k, j, i) - P(P_TZC1, k) * W(k - 1, j, i));
  pp = pp * timec;
  d.p[o] = pp;
  double a = fabs((double)pp);
  atomicMax(divmax, (unsigned long long)__double_as_longlong(a));
}

// psrce including the deferred first-row / first-column faces (fftsolver.F90:215-250)
template <typename T>
__global__ void k_c_psrce(Scalars s, DevState<T> d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z + 2;
  if (i >= s.nx || j >= s.ny || k > s.nz) return;
  Prof<T> P = prof<T>(s);
  View<T> SU = view<T>(d.su, s), SV = view<T>(d.sv, s), SW = view<T>(d.sw, s);
  long long o = lin(s, k, j, i);
  T pp = d.p[o];
  pp = pp + (T)4.0 * (P(P_TZC2, k) * SW(k, j, i) - P(P_TZC1, k) * SW(k - 1, j, i));
  pp = pp + (T)s.cx * SU(k, j, i);
  pp = pp + (T)s.cy * SV(k, j, i);
  pp = pp - (T)s.cx * SU(k, j, i - 1);
  pp = pp - (T)s.cy * SV(k, j - 1, i);
  d.p[o] = pp;
}

// stepfields: step_field + perform_timesmooth_for_field + negative-q clipping, pointwise
template <typename T>
__global__ void k_c_stepfields(Scalars s, DevState<T> d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z + 1;
  if (i >= s.nx || j >= s.ny || k > s.nz) return;
  long long o = lin(s, k, j, i);
  const bool fwd = s.forward;
  const T dtm = (T)s.dtm, dtm_x2 = (T)(2.0 * s.dtm);
  const T c1 = (T)(1.0 - 2.0 * s.tsmth), c2 = (T)s.tsmth;
  auto step = [&](T* f, T* zf, T* sf, bool flow, T gal, T* sav, bool ts) {
    T sv = (k == 1) ? (T)0.0 : sf[o];
    if (k == 1) sf[o] = (T)0.0;
    T fv = f[o], zv = zf[o];
    if (ts) { fv = c1 * fv + c2 * zv; f[o] = fv; }
    if (sav && !fwd) sav[o] = zv + (flow ? gal : (T)0.0);
    T ag = flow ? gal : (T)0.0;
    if (flow) { fv = ag + fv; f[o] = fv; }
    if (fwd) zf[o] = fv + dtm * sv;
    else zf[o] = ag + zv + dtm_x2 * sv;
  };
  step(d.u, d.zu, d.su, true, (T)s.ugal, d.savu, false);
  step(d.v, d.zv, d.sv, true, (T)s.vgal, d.savv, false);
  step(d.w, d.zw, d.sw, false, (T)0.0, d.savw, false);
  step(d.th, d.zth, d.sth, false, (T)0.0, nullptr, !fwd);
  for (int n = 0; n < s.nq; ++n) {
    step(d.q[n], d.zq[n], d.sq[n], false, (T)0.0, nullptr, !fwd);
    if (d.zq[n][o] < (T)0.0) d.zq[n][o] = (T)0.0;
  }
}

// pstep: one thread per column (level 1 depends on the updated level 2)
template <typename T>
__global__ void k_c_pstep(Scalars s, DevState<T> d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= s.nx || j >= s.ny) return;
  Prof<T> P = prof<T>(s);
  View<T> Pv = view<T>(d.p, s);
  T dtmtmp = s.forward ? (T)(0.5 * s.dtm) : (T)s.dtm;
  for (int k = 2; k <= s.nz; ++k) {
    long long o = lin(s, k, j, i);
    T p0 = Pv(k, j, i);
    d.zu[o] = d.zu[o] + (T)2.0 * (T)s.cx * dtmtmp * (p0 - Pv(k, j, i + 1));
    d.zv[o] = d.zv[o] + (T)2.0 * (T)s.cy * dtmtmp * (p0 - Pv(k, j + 1, i));
    if (k < s.nz) d.zw[o] = d.zw[o] + (T)2.0 * P(P_RDZN, k + 1) * dtmtmp * (p0 - Pv(k + 1, j, i));
  }
  long long o1 = lin(s, 1, j, i), o2 = lin(s, 2, j, i);
  if (s.use_vd && s.surface_bcs) {
    d.zu[o1] = -d.zu[o2] - (T)2.0 * (T)s.ugal;
    d.zv[o1] = -d.zv[o2] - (T)2.0 * (T)s.vgal;
  } else {
    d.zu[o1] = d.zu[o2];
    d.zv[o1] = d.zv[o2];
  }
}

template <typename T>
__global__ void k_c_swap_smooth(Scalars s, DevState<T> d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z + 1;
  if (i >= s.nx || j >= s.ny || k > s.nz) return;
  long long o = lin(s, k, j, i);
  if (s.forward) {
    const T c1 = (T)1.0, c2 = (T)-1.0;
    auto sw = [&](T* f, T* zf) {
      T ev = f[o] + zf[o];
      T nf = ev * c1 + f[o] * c2;
      f[o] = nf;
      zf[o] = ev - nf;
    };
    sw(d.u, d.zu); sw(d.v, d.zv); sw(d.w, d.zw); sw(d.th, d.zth);
    for (int n = 0; n < s.nq; ++n) sw(d.q[n], d.zq[n]);
  } else {
    const T c1 = (T)(1.0 - 2.0 * s.tsmth), c2 = (T)s.tsmth;
    auto rf = [&](T* f, T* zf, T* sav, T gal) {
      T ev = f[o];
      T nf = zf[o];
      f[o] = nf;
      zf[o] = c1 * ev + c2 * (nf + sav[o] - gal);
    };
    rf(d.u, d.zu, d.savu, (T)s.ugal);
    rf(d.v, d.zv, d.savv, (T)s.vgal);
    {
      T ev = d.w[o];
      T nf = d.zw[o];
      d.w[o] = nf;
      d.zw[o] = c1 * ev + c2 * (nf + d.savw[o]);
    }
    auto sc = [&](T* f, T* zf) {
      T ev = zf[o];
      zf[o] = f[o] + (T)s.tsmth * ev;
      f[o] = ev;
    };
    sc(d.th, d.zth);
    for (int n = 0; n < s.nq; ++n) sc(d.q[n], d.zq[n]);
  }
}

template <typename T>
__global__ void k_zero(T* p, long long n) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  for (; t < n; t += (long long)gridDim.x * blockDim.x) p[t] = (T)0.0;
}

// ==========================================================================================
// Fused step kernels
// ==========================================================================================

// 1. subgrid: lower_bc (level 1) + smagorinsky (levels 2..nz)
template <typename T>
__global__ void k_f_subgrid(Scalars s, DevState<T> d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z + 1;
  if (i >= s.nx || j >= s.ny || k > s.nz) return;
  Prof<T> P = prof<T>(s);
  bool fwd = s.forward;
  long long o = lin(s, k, j, i);
  if (k == 1) {
    View<T> zus = view<T>(d.zu, s), zua = view<T>(fwd ? d.u : d.zu, s), zva = view<T>(fwd ? d.v : d.zv, s);
    T* tha = fwd ? d.th : d.zth;
    View<T> qv;
    T* qa = nullptr;
    if (s.nq > 0) { qa = fwd ? d.q[s.iqv] : d.zq[s.iqv]; qv = view<T>(qa, s); }
    T vis1, diff1, th1, qv1;
    lower_bc_column<T>(s, P, zus, zua, zva, view<T>(tha, s), s.nq > 0 ? &qv : nullptr, j, i, vis1, diff1, th1, qv1);
    d.vis[o] = vis1;
    d.diff[o] = diff1;
    tha[o] = th1;
    if (qa) qa[o] = qv1;
    return;
  }
  if (k == s.nz) { d.vis[o] = (T)0.0; d.diff[o] = (T)0.0; return; }
  View<T> U = view<T>(fwd ? d.u : d.zu, s), V = view<T>(fwd ? d.v : d.zv, s), W = view<T>(fwd ? d.w : d.zw, s);
  View<T> QV, QL;
  if (!s.passive_q && s.nq > 1) {
    QV = view<T>(fwd ? d.q[s.iqv] : d.zq[s.iqv], s);
    QL = view<T>(fwd ? d.q[s.iql] : d.zq[s.iql], s);
  }
  T vis, diff;
  smagorinsky_point<T>(s, P, U, V, W, view<T>(d.th, s), view<T>(fwd ? d.th : d.zth, s), &QV, &QL, k, j, i, vis, diff);
  d.vis[o] = vis;
  d.diff[o] = diff;
}

// 2. dynamics + stepfields + swap_smooth of the scalars
template <typename T>
__global__ void __launch_bounds__(256) k_f_dynamics(Scalars s, DevState<T> d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z + 1;
  if (i >= s.nx || j >= s.ny || k > s.nz) return;
  Prof<T> P = prof<T>(s);
  const bool fwd = s.forward;
  long long o = lin(s, k, j, i);
  View<T> U = view<T>(d.u, s), V = view<T>(d.v, s), W = view<T>(d.w, s);
  T su = (T)0.0, sv = (T)0.0, sw = (T)0.0, sth = (T)0.0;
  T sq[MGPU_MAX_Q];
  for (int n = 0; n < s.nq; ++n) sq[n] = (T)0.0;
  if (k >= 2) {
    // pw_advection (assigns), viscosity, coriolis, buoyancy: the order MONC adds them in
    pw_point<T>(s, P, U, V, W, k, j, i, su, sv, sw);
    if (s.use_vd) {
      View<T> ZU = view<T>(fwd ? d.u : d.zu, s), ZV = view<T>(fwd ? d.v : d.zv, s), ZW = view<T>(fwd ? d.w : d.zw, s);
      T du, dv, dw;
      viscosity_point<T>(s, P, ZU, ZV, ZW, view<T>(d.zu, s), view<T>(d.vis, s), k, j, i, du, dv, dw);
      su = su + du;
      sv = sv + dv;
      if (k < s.nz) sw = sw + dw;
    }
    if (s.coriolis) coriolis_point<T>(s, P, U, V, k, j, i, su, sv);
    if (k < s.nz) {
      View<T> Q[MGPU_MAX_Q];
      for (int n = 0; n < s.nq; ++n) Q[n] = view<T>(d.q[n], s);
      sw = buoyancy_point<T>(s, P, view<T>(d.th, s), Q, k, j, i, sw);
    }
    // tvd_advection then diffusion of theta and q
    sth = tvd_point<T>(s, P, U, V, W, view<T>(fwd ? d.th : d.zth, s), k, j, i, (T)0.0);
    if (s.use_vd) sth = sth + diffusion_point<T>(s, P, view<T>(d.zth, s), view<T>(d.diff, s), k, j, i);
    for (int n = 0; n < s.nq; ++n) {
      sq[n] = tvd_point<T>(s, P, U, V, W, view<T>(fwd ? d.q[n] : d.zq[n], s), k, j, i, (T)0.0);
      if (s.use_vd) sq[n] = sq[n] + diffusion_point<T>(s, P, view<T>(d.zq[n], s), view<T>(d.diff, s), k, j, i);
    }
  }
  // stepfields (source at level 1 is zeroed there) and, for scalars, swap_smooth
  const T dtm = (T)s.dtm, dtm_x2 = (T)(2.0 * s.dtm);
  const T c1 = (T)(1.0 - 2.0 * s.tsmth), c2 = (T)s.tsmth;
  auto step_flow = [&](const T* f, const T* zf, T src, T gal, T* out) {
    T fv = gal + f[o];
    if (fwd) out[o] = fv + dtm * src;
    else out[o] = gal + zf[o] + dtm_x2 * src;
  };
  step_flow(d.u, d.zu, su, (T)s.ugal, d.zu_n);
  step_flow(d.v, d.zv, sv, (T)s.vgal, d.zv_n);
  {
    T wv = d.w[o];
    if (fwd) d.zw_n[o] = wv + dtm * sw;
    else d.zw_n[o] = (T)0.0 + d.zw[o] + dtm_x2 * sw;
  }
  auto step_scalar = [&](const T* f, const T* zf, T src, T* f_out, T* zf_out, bool clip) {
    T fv = f[o], zv = zf[o];
    if (fwd) {
      T zn = fv + dtm * src;
      if (clip && zn < (T)0.0) zn = (T)0.0;
      T ev = fv + zn;
      T nf = ev * (T)1.0 + fv * (T)-1.0;
      f_out[o] = nf;
      zf_out[o] = ev - nf;
    } else {
      T sm = c1 * fv + c2 * zv;
      T zn = (T)0.0 + zv + dtm_x2 * src;
      if (clip && zn < (T)0.0) zn = (T)0.0;
      zf_out[o] = sm + (T)s.tsmth * zn;
      f_out[o] = zn;
    }
  };
  step_scalar(d.th, d.zth, sth, d.th_n, d.zth_n, false);
  for (int n = 0; n < s.nq; ++n) step_scalar(d.q[n], d.zq[n], sq[n], d.q_n[n], d.zq_n[n], true);
}

// 3. pressure source from the stepped z-velocities (diverr + psrce)
template <typename T>
__global__ void k_f_pressure_source(Scalars s, DevState<T> d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z + 1;
  if (i >= s.nx || j >= s.ny || k > s.nz) return;
  long long o = lin(s, k, j, i);
  if (k == 1) { d.p[o] = (T)0.0; return; }
  Prof<T> P = prof<T>(s);
  T timec = s.forward ? (T)(1.0 / s.dtm) : (T)(1.0 / (2.0 * s.dtm));
  View<T> U = view<T>(d.zu_n, s), V = view<T>(d.zv_n, s), W = view<T>(d.zw_n, s);
  T pp = (T)0.0;
  pp = pp + (T)s.cx * (U(k, j, i) - U(k, j, i - 1));
  pp = pp + (T)s.cy * (V(k, j, i) - V(k, j - 1, i));
  pp = pp + (T)4.0 * (P(P_TZC2, k) * W(k, j, i) - P(P_TZC1, k) * W(k - 1, j, i));
  d.p[o] = pp * timec;
}

// 5. pstep + swap_smooth of u, v, w
template <typename T>
__global__ void k_f_pstep_swap(Scalars s, DevState<T> d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z + 1;
  if (i >= s.nx || j >= s.ny || k > s.nz) return;
  Prof<T> P = prof<T>(s);
  View<T> Pv = view<T>(d.p, s);
  const bool fwd = s.forward;
  const T dtmtmp = fwd ? (T)(0.5 * s.dtm) : (T)s.dtm;
  long long o = lin(s, k, j, i);
  const bool bc = s.use_vd && s.surface_bcs;
  auto pu = [&](int kk) {
    return d.zu_n[lin(s, kk, j, i)] + (T)2.0 * (T)s.cx * dtmtmp * (Pv(kk, j, i) - Pv(kk, j, i + 1));
  };
  auto pv = [&](int kk) {
    return d.zv_n[lin(s, kk, j, i)] + (T)2.0 * (T)s.cy * dtmtmp * (Pv(kk, j, i) - Pv(kk, j + 1, i));
  };
  T zu_p, zv_p, zw_p;
  if (k >= 2) {
    zu_p = pu(k);
    zv_p = pv(k);
  } else if (bc) {
    zu_p = -pu(2) - (T)2.0 * (T)s.ugal;
    zv_p = -pv(2) - (T)2.0 * (T)s.vgal;
  } else {
    zu_p = pu(2);
    zv_p = pv(2);
  }
  zw_p = d.zw_n[o];
  if (k >= 2 && k < s.nz) zw_p = zw_p + (T)2.0 * P(P_RDZN, k + 1) * dtmtmp * (Pv(k, j, i) - Pv(k + 1, j, i));
  if (fwd) {
    auto cl = [&](T* f, T* zf, T fv, T zn) {
      T ev = fv + zn;
      T nf = ev * (T)1.0 + fv * (T)-1.0;
      f[o] = nf;
      zf[o] = ev - nf;
    };
    cl(d.u, d.zu, (T)s.ugal + d.u[o], zu_p);
    cl(d.v, d.zv, (T)s.vgal + d.v[o], zv_p);
    cl(d.w, d.zw, d.w[o], zw_p);
  } else {
    const T c1 = (T)(1.0 - 2.0 * s.tsmth), c2 = (T)s.tsmth;
    T ev = (T)s.ugal + d.u[o];
    T sav = d.zu[o] + (T)s.ugal;
    d.u[o] = zu_p;
    d.zu[o] = c1 * ev + c2 * (zu_p + sav - (T)s.ugal);
    ev = (T)s.vgal + d.v[o];
    sav = d.zv[o] + (T)s.vgal;
    d.v[o] = zv_p;
    d.zv[o] = c1 * ev + c2 * (zv_p + sav - (T)s.vgal);
    ev = d.w[o];
    sav = d.zw[o] + (T)0.0;
    d.w[o] = zw_p;
    d.zw[o] = c1 * ev + c2 * (zw_p + sav);
  }
}

// ==========================================================================================
// host launchers
// ==========================================================================================
template <typename T>
int launch_component(int cid, const Scalars& s, DevState<T>& d, cudaStream_t st, unsigned long long* divmax,
                     int64_t* launches) {
  dim3 b = pt_block();
  dim3 gcol((s.nx + 31) / 32, (s.ny + 7) / 8, 1);
  int nl = 1;
  switch (cid) {
    case MGPU_C_LOWER_BC: k_c_lower_bc<T><<<gcol, b, 0, st>>>(s, d); break;
    case MGPU_C_SMAGORINSKY: k_c_smagorinsky<T><<<pt_grid(s, s.nz - 1), b, 0, st>>>(s, d); break;
    case MGPU_C_PW_ADVECTION: k_c_pw<T><<<pt_grid(s, s.nz - 1), b, 0, st>>>(s, d); break;
    case MGPU_C_TVD_ADVECTION: k_c_tvd<T><<<pt_grid(s, s.nz - 1), b, 0, st>>>(s, d, nullptr, nullptr, 0); break;
    case MGPU_C_DIFFUSION: k_c_diffusion<T><<<pt_grid(s, s.nz - 1), b, 0, st>>>(s, d); break;
    case MGPU_C_VISCOSITY: k_c_viscosity<T><<<pt_grid(s, s.nz - 1), b, 0, st>>>(s, d); break;
    case MGPU_C_CORIOLIS: k_c_coriolis<T><<<pt_grid(s, s.nz - 1), b, 0, st>>>(s, d); break;
    case MGPU_C_BUOYANCY: k_c_buoyancy<T><<<pt_grid(s, s.nz - 2), b, 0, st>>>(s, d); break;
    case MGPU_C_SET_CONSISTENT_LOWBC: k_c_set_consistent_lowbc<T><<<gcol, b, 0, st>>>(s, d); break;
    case MGPU_C_DIVERR: k_c_diverr<T><<<pt_grid(s, s.nz), b, 0, st>>>(s, d, divmax); break;
    case MGPU_C_PSRCE: k_c_psrce<T><<<pt_grid(s, s.nz - 1), b, 0, st>>>(s, d); break;
    case MGPU_C_STEPFIELDS: k_c_stepfields<T><<<pt_grid(s, s.nz), b, 0, st>>>(s, d); break;
    case MGPU_C_PSTEP: k_c_pstep<T><<<gcol, b, 0, st>>>(s, d); break;
    case MGPU_C_SWAP_SMOOTH: k_c_swap_smooth<T><<<pt_grid(s, s.nz), b, 0, st>>>(s, d); break;
    case MGPU_C_CLEARSOURCETERMS: {
      long long n = (long long)s.nz * s.plane;
      T* arr[4] = {d.su, d.sv, d.sw, d.sth};
      nl = 0;
      for (T* a : arr) { k_zero<T><<<592, 256, 0, st>>>(a, n); ++nl; }
      for (int q = 0; q < s.nq; ++q) { k_zero<T><<<592, 256, 0, st>>>(d.sq[q], n); ++nl; }
      break;
    }
    default: return MGPU_ERR_UNSUPPORTED;
  }
  *launches += nl;
  return MGPU_OK;
}

template <typename T>
void launch_fused_subgrid(const Scalars& s, DevState<T>& d, cudaStream_t st) {
  k_f_subgrid<T><<<pt_grid(s, s.nz), pt_block(), 0, st>>>(s, d);
}
template <typename T>
void launch_fused_dynamics(const Scalars& s, DevState<T>& d, cudaStream_t st) {
  k_f_dynamics<T><<<pt_grid(s, s.nz), pt_block(), 0, st>>>(s, d);
}
template <typename T>
void launch_fused_pressure_source(const Scalars& s, DevState<T>& d, cudaStream_t st) {
  k_f_pressure_source<T><<<pt_grid(s, s.nz), pt_block(), 0, st>>>(s, d);
}
template <typename T>
void launch_fused_pstep_swap(const Scalars& s, DevState<T>& d, cudaStream_t st) {
  k_f_pstep_swap<T><<<pt_grid(s, s.nz), pt_block(), 0, st>>>(s, d);
}

}  // namespace mgpu
