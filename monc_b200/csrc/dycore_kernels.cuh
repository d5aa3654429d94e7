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

#include <type_traits>

#include "dycore.h"
#include "dycore_device.cuh"

#ifndef KVARIANT
#define KVARIANT exact
#endif

namespace mgpu {
namespace KVARIANT {

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
  if (s.tvd_flow) return;  // the flow is advected by tvd_advection (advect_flow is false here)
  Prof<T> P = prof<T>(s);
  View<T> U = view<T>(d.u, s), V = view<T>(d.v, s), W = view<T>(d.w, s);
  T su, sv, sw;
  pw_point<T, View<T>>(s, P, U, V, W, k, j, i, su, sv, sw);
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
  // the flow fields (advect_flow_fields), then theta, then each q field (advect_theta, advect_q_fields)
  if (s.tvd_flow) {
    T su, sv, sw;
    tvd_flow_point<T, View<T>>(s, P, U, V, W, view<T>(fwd ? d.u : d.zu, s), view<T>(fwd ? d.v : d.zv, s),
                               view<T>(fwd ? d.w : d.zw, s), k, j, i, d.su[o], d.sv[o], k < s.nz ? d.sw[o] : (T)0.0,
                               su, sv, sw);
    d.su[o] = su;
    d.sv[o] = sv;
    if (k < s.nz) d.sw[o] = sw;
  }
  {
    View<T> ZF = view<T>(fwd ? d.th : d.zth, s);
    d.sth[o] = tvd_point<T, View<T>>(s, P, U, V, W, ZF, k, j, i, d.sth[o]);
  }
  for (int n = 0; n < s.nq; ++n) {
    View<T> ZF = view<T>(fwd ? d.q[n] : d.zq[n], s);
    d.sq[n][o] = tvd_point<T, View<T>>(s, P, U, V, W, ZF, k, j, i, d.sq[n][o]);
  }
  (void)zf_th; (void)sth; (void)n_extra;
}

// th_advection: the mean-baroclinicity term added to sth, levels 2..nz
template <typename T>
__global__ void k_c_th_advection(Scalars s, DevState<T> d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z + 2;
  if (i >= s.nx || j >= s.ny || k > s.nz) return;
  long long o = lin(s, k, j, i);
  d.sth[o] = d.sth[o] + th_baroclinic_point<T>(s, view<T>(d.u, s), view<T>(d.v, s), k, j, i);
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
  d.sth[o] = d.sth[o] + diffusion_point<T, View<T>>(s, P, view<T>(d.zth, s), D, k, j, i);
  for (int n = 0; n < s.nq; ++n) d.sq[n][o] = d.sq[n][o] + diffusion_point<T, View<T>>(s, P, view<T>(d.zq[n], s), D, k, j, i);
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
  viscosity_point<T, View<T>>(s, P, ZU, ZV, ZW, view<T>(d.zu, s), view<T>(d.vis, s), k, j, i, du, dv, dw);
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
  coriolis_point<T, View<T>>(s, P, view<T>(d.u, s), view<T>(d.v, s), k, j, i, su, sv);
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

// damping (damping.F90:301-409) over the levels kdmpmin..nz of every column
template <typename T>
__global__ void k_c_damping(Scalars s, DevState<T> d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z + 1;
  if (i >= s.nx || j >= s.ny || k > s.nz || k < s.kdmpmin) return;
  Prof<T> P = prof<T>(s);
  long long o = lin(s, k, j, i);
  T su = d.su[o], sv = d.sv[o], sw = d.sw[o];
  damping_flow_point<T>(s, P, k, d.zu[o], d.zv[o], d.zw[o], su, sv, sw);
  d.su[o] = su;
  d.sv[o] = sv;
  d.sw[o] = sw;
  if (!s.passive_th) d.sth[o] = damping_scalar_point<T>(s, P, k, d.zth[o], 2, d.sth[o]);
  for (int n = 0; n < s.nq; ++n) d.sq[n][o] = damping_scalar_point<T>(s, P, k, d.zq[n][o], 3 + n, d.sq[n][o]);
}

// forcing's subsidence (forcing.F90:1032-1166): u, v and theta, then q, levels 2..nz
template <typename T>
__global__ void k_c_forcing(Scalars s, DevState<T> d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z + 1;
  if (i >= s.nx || j >= s.ny || k > s.nz || k < 2) return;
  Prof<T> P = prof<T>(s);
  long long o = lin(s, k, j, i);
  if (s.subs_th) {
    T su = d.su[o], sv = d.sv[o];
    subsidence_flow_point<T>(s, P, view<T>(d.zu, s), view<T>(d.zv, s), k, j, i, su, sv);
    d.su[o] = su;
    d.sv[o] = sv;
    d.sth[o] = subsidence_theta_point<T>(s, P, view<T>(d.zth, s), k, j, i, d.sth[o]);
  }
  if (s.subs_q)
    for (int n = 0; n < s.nq; ++n) d.sq[n][o] = subsidence_q_point<T>(s, P, view<T>(d.zq[n], s), n, k, j, i, d.sq[n][o]);
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

// simplecloud: saturation adjustment of sth, sq(vapour), sq(liquid), levels 2..nz
template <typename T>
__global__ void k_c_simplecloud(Scalars s, DevState<T> d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z + 2;
  if (i >= s.nx || j >= s.ny || k > s.nz) return;
  Prof<T> P = prof<T>(s);
  const long long o = lin(s, k, j, i);
  const bool fwd = s.forward;
  const int iv = s.iqv, il = s.iql;
  T sth = d.sth[o], sqv = d.sq[iv][o], sql = d.sq[il][o];
  simplecloud_point<T>(s, P, k, (fwd ? d.q[iv] : d.zq[iv])[o], (fwd ? d.q[il] : d.zq[il])[o], (fwd ? d.th : d.zth)[o],
                       d.zq[il][o], sth, sqv, sql);
  d.sth[o] = sth;
  d.sq[iv][o] = sqv;
  d.sq[il][o] = sql;
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
  if (s.galilean)  // perform_galilean_transformation, every level, before the pressure step
    for (int k = 1; k <= s.nz; ++k) {
      long long o = lin(s, k, j, i);
      d.u[o] = d.u[o] - (T)s.ugal;
      d.zu[o] = d.zu[o] - (T)s.ugal;
      d.v[o] = d.v[o] - (T)s.vgal;
      d.zv[o] = d.zv[o] - (T)s.vgal;
    }
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
    // pw_advection (assigns) or the TVD advection of the flow (adds to the cleared sources),
    // viscosity, coriolis, buoyancy: the order MONC adds them in
    if (s.tvd_flow)
      tvd_flow_point<T, View<T>>(s, P, U, V, W, view<T>(fwd ? d.u : d.zu, s), view<T>(fwd ? d.v : d.zv, s),
                                 view<T>(fwd ? d.w : d.zw, s), k, j, i, (T)0.0, (T)0.0, (T)0.0, su, sv, sw);
    else
      pw_point<T, View<T>>(s, P, U, V, W, k, j, i, su, sv, sw);
    if (s.use_vd) {
      View<T> ZU = view<T>(fwd ? d.u : d.zu, s), ZV = view<T>(fwd ? d.v : d.zv, s), ZW = view<T>(fwd ? d.w : d.zw, s);
      T du, dv, dw;
      viscosity_point<T, View<T>>(s, P, ZU, ZV, ZW, view<T>(d.zu, s), view<T>(d.vis, s), k, j, i, du, dv, dw);
      su = su + du;
      sv = sv + dv;
      if (k < s.nz) sw = sw + dw;
    }
    if (s.coriolis) coriolis_point<T, View<T>>(s, P, U, V, k, j, i, su, sv);
    if (k < s.nz) {
      View<T> Q[MGPU_MAX_Q];
      for (int n = 0; n < s.nq; ++n) Q[n] = view<T>(d.q[n], s);
      sw = buoyancy_point<T>(s, P, view<T>(d.th, s), Q, k, j, i, sw);
    }
    // damping, then forcing's subsidence (both from timestep 3, so the z-fields are zu, zv, zw)
    if (s.damping) damping_flow_point<T>(s, P, k, d.zu[o], d.zv[o], d.zw[o], su, sv, sw);
    if (s.subs_th) subsidence_flow_point<T>(s, P, view<T>(d.zu, s), view<T>(d.zv, s), k, j, i, su, sv);
    // tvd_advection then diffusion of theta and q, then their damping and subsidence
    sth = tvd_point<T, View<T>>(s, P, U, V, W, view<T>(fwd ? d.th : d.zth, s), k, j, i, (T)0.0);
    if (s.th_baroclinic) sth = sth + th_baroclinic_point<T>(s, U, V, k, j, i);
    if (s.use_vd) sth = sth + diffusion_point<T, View<T>>(s, P, view<T>(d.zth, s), view<T>(d.diff, s), k, j, i);
    if (s.damping && !s.passive_th) sth = damping_scalar_point<T>(s, P, k, d.zth[o], 2, sth);
    if (s.subs_th) sth = subsidence_theta_point<T>(s, P, view<T>(d.zth, s), k, j, i, sth);
    for (int n = 0; n < s.nq; ++n) {
      sq[n] = tvd_point<T, View<T>>(s, P, U, V, W, view<T>(fwd ? d.q[n] : d.zq[n], s), k, j, i, (T)0.0);
      if (s.use_vd) sq[n] = sq[n] + diffusion_point<T, View<T>>(s, P, view<T>(d.zq[n], s), view<T>(d.diff, s), k, j, i);
      if (s.damping) sq[n] = damping_scalar_point<T>(s, P, k, d.zq[n][o], 3 + n, sq[n]);
      if (s.subs_q) sq[n] = subsidence_q_point<T>(s, P, view<T>(d.zq[n], s), n, k, j, i, sq[n]);
    }
    if (s.simplecloud) {
      const int iv = s.iqv, il = s.iql;
      simplecloud_point<T>(s, P, k, (fwd ? d.q[iv] : d.zq[iv])[o], (fwd ? d.q[il] : d.zq[il])[o], (fwd ? d.th : d.zth)[o],
                           d.zq[il][o], sth, sq[iv], sq[il]);
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

// 2'. Centred-step dynamics, shared-memory tiled, as two kernels that each march up the levels
//     of a TX x TY tile of columns:
//       k_f_momentum_tiled : pw_advection + viscosity + coriolis + buoyancy + stepfields of u, v, w
//       k_f_scalar_tiled   : tvd_advection + diffusion + stepfields + swap_smooth pre-smoothing of th
//     The planes each level needs (with a periodic halo of 2 points in y and one 16-byte chunk
//     in x) sit in per-field ring buffers in shared memory, filled one level ahead with 16-byte
//     cp.async copies whose source offsets each thread computes once.  Every TVD face flux is
//     computed once: x and y faces go through shared memory, the z face is carried in a
//     register from the level below.  The arithmetic is the device code the point kernel
//     runs, so the results are bit-identical to it.
namespace tiled {
constexpr int TX = 32, TY = 8, HY = 2, NT = TX * TY;
template <typename T>
struct G {
  static constexpr int V = 16 / (int)sizeof(T);  // elements per 16-byte chunk = x halo width
  static constexpr int PW = TX + 2 * V, PH = TY + 2 * HY, PLANE = PW * PH;
  static constexpr int CPR = PW / V;   // chunks per plane row
  static constexpr int NCH = CPR * PH;  // chunks per plane (<= NT)
  static_assert(NCH <= NT, "one chunk per thread and plane");
  static_assert((PLANE * sizeof(T)) % 16 == 0, "planes start on 16-byte boundaries");
};
constexpr int RM = 4;              // momentum rings: levels k-1..k+1 live, k+2 in flight
// Scalar kernel rings, each as deep as the levels it must hold (level k's faces, source and
// diffusion read u, v at k..k+1, w at k-1..k+1, diff at k-1..k and the scalar at k-1..k+2), plus
// the level in flight.  Slots are level mod depth.  With 18 planes the FP64 kernel fits three
// CTAs on an SM.  A ring slot whose level is not live is never read (a centred accessor's
// pointer to it aliases another slot).
// FP64 keeps the minimum depths; FP32, whose occupancy registers limit, keeps powers of two
// (slots by mask).
template <typename T>
struct ScalarRings {
  static constexpr bool F64 = sizeof(T) == 8;
  static constexpr int RUV = F64 ? 3 : 4, RW = 4, RD = F64 ? 3 : 4, RZF = F64 ? 5 : 8;
  static constexpr int PLANES = 2 * RUV + RW + RD + RZF;  // u v w diff + scalar
};
constexpr int RP = 8;              // profile ring: levels k-1..k+2 live, k+3 staged
// resident CTAs per SM the register budget is sized for (FP64: 2 x 256 threads x <= 128 registers)
template <typename T>
constexpr int min_ctas() { return sizeof(T) == 4 ? 3 : 2; }
// the scalar and Smagorinsky kernels fit 80 registers without spilling, and their shared memory
// allows three CTAs per SM in FP64 too
constexpr int min_ctas3() { return 3; }
// resident CTAs per SM of the centred-step kernels: FP32 fits all three in 64 registers (no
// spills) and four CTAs' shared memory; FP64 runs three scalar and Smagorinsky CTAs, two momentum
template <typename T>
constexpr int ctas_scalar() { return sizeof(T) == 4 ? 4 : 3; }
template <typename T>
constexpr int ctas_momentum() { return sizeof(T) == 4 ? 4 : 2; }
constexpr int M_PLANES = 7 * RM;   // u v w zu zv zw vis
template <typename T>
constexpr size_t smag_smem() { return sizeof(T) * ((size_t)3 * RM * G<T>::PLANE + (size_t)RP * P_COUNT); }
template <typename T>
constexpr size_t momentum_smem() { return sizeof(T) * ((size_t)M_PLANES * G<T>::PLANE + (size_t)RP * P_COUNT); }
// the scalar kernel's table of cell outflow Courant sums: rows j0-1 .. j0+TY, columns i0-1 .. i0+TX
constexpr int CW = TX + 2, CN = (TY + 2) * CW;
template <typename T>
constexpr size_t scalar_smem() {
  return sizeof(T) * ((size_t)ScalarRings<T>::PLANES * G<T>::PLANE + (size_t)RP * P_COUNT + (size_t)TY * (TX + 1) +
                      (size_t)(TY + 1) * TX + (size_t)2 * CN);
}
// TVD advection of a flow component (DIM 0: u, 1: v, 2: w).  The advecting velocities are
// interpolated to the component's dual grid, which for w averages levels k and k+1: its faces at
// level k read u, v up to k+2 and w up to k+2 (UPF = 2), the others up to k+1 (UPF = 1).  The
// rings hold those levels and the one in flight; the advected component's ring holds k-1..k+2.
template <int DIM>
struct FlowRings {
  static constexpr int UPF = DIM == 2 ? 2 : 1;
  static constexpr int RUV = UPF + 2, RW = UPF + 3, RZ = 5;
  static constexpr int PLANES = 2 * RUV + RW + RZ;
};
template <typename T, int DIM>
constexpr size_t flow_smem() {
  return sizeof(T) * ((size_t)FlowRings<DIM>::PLANES * G<T>::PLANE + (size_t)RP * P_COUNT + (size_t)TY * (TX + 1) +
                      (size_t)(TY + 1) * TX + (size_t)2 * CN);
}
// The moist centred step with vapour and liquid (theta and two q fields) in one kernel: the flow,
// diff and the cell Courant sums are staged and formed once for the three scalars; each scalar
// has its own ring (k-1..k+2 and the level in flight).  Two x/y face buffers alternate between
// the scalars.
struct MoistRings {
  static constexpr int NS = 3, RUV = 3, RW = 4, RD = 3, RZF = 5;
  static constexpr int PLANES = 2 * RUV + RW + RD + NS * RZF;
};
template <typename T>
constexpr size_t moist_smem() {
  return sizeof(T) * ((size_t)MoistRings::PLANES * G<T>::PLANE + (size_t)RP * P_COUNT +
                      (size_t)2 * (TY * (TX + 1) + (TY + 1) * TX) + (size_t)2 * CN);
}
}  // namespace tiled

// A column's values at levels k0 and k0+1 held in registers, read through the accessor interface
template <typename T>
struct ColPair {
  T v0, v1;
  int k0;
  __device__ __forceinline__ T operator()(int k, int, int) const { return k == k0 ? v0 : v1; }
};

// Centred ring view: the thread's own point at levels kc-1 .. kc+2 through four slot pointers.
// Every access the device functions make at k +- const, j +- const, i +- const folds to one
// shared-memory load with an immediate offset; data-dependent levels select among the four.
template <typename T>
struct CRing {
  const T* pm;
  const T* p0;
  const T* p1;
  const T* p2;
  int kc, jc, ic;
  __device__ __forceinline__ const T* lvl(int dk) const { return dk <= -1 ? pm : (dk == 0 ? p0 : (dk == 1 ? p1 : p2)); }
  __device__ __forceinline__ T operator()(int k, int j, int i) const {
    return lvl(k - kc)[(j - jc) * tiled::G<T>::PW + (i - ic)];
  }
};

// profile values of levels kc-1 .. kc+2, staged per level in shared memory (P_COUNT per level)
template <typename T>
struct CProf {
  const T* pm;
  const T* p0;
  const T* p1;
  const T* p2;
  int kc;
  __device__ __forceinline__ T operator()(int id, int k) const {
    const int dk = k - kc;
    return (dk <= -1 ? pm : (dk == 0 ? p0 : (dk == 1 ? p1 : p2)))[id];
  }
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// slot of level k (>= 0) in a ring of R planes: a mask for powers of two, an unsigned remainder
// by a constant otherwise (a multiply and a shift)
template <int R>
__device__ __forceinline__ int ring_slot(int k) {
  if constexpr ((R & (R - 1)) == 0) return k & (R - 1);
  else return (int)((unsigned)k % (unsigned)R);
}
// One thread's share of staging a plane: a single 16-byte chunk.  The x halo is one whole
// chunk on each side and nx is a multiple of the chunk, so no chunk straddles the periodic wrap.
template <typename T>
struct Stager {
  int soff;       // element offset of the chunk inside a plane
  long long goff; // element offset of the chunk inside a global level
  bool on;
  __device__ void init(const Scalars& s, int j0, int i0, int tid) {
    using Gt = tiled::G<T>;
    on = tid < Gt::NCH;
    const int c = on ? tid : 0;
    const int row = c / Gt::CPR, cc = c - row * Gt::CPR;
    soff = row * Gt::PW + cc * Gt::V;
    int gj = j0 - tiled::HY + row, gi = i0 - Gt::V + cc * Gt::V;
    gj = gj < 0 ? gj + s.ny : (gj >= s.ny ? gj - s.ny : gj);
    gi = gi < 0 ? gi + s.nx : (gi >= s.nx ? gi - s.nx : gi);
    goff = (long long)gj * s.nx + gi;
  }
  // copy level k of field f into slot (k mod R) of the ring at `ring`
  template <int R>
  __device__ __forceinline__ void stage(T* ring, const T* __restrict__ f, long long plane, int k) const {
    if (on) cp_async16(ring + ring_slot<R>(k) * tiled::G<T>::PLANE + soff, f + (long long)(k - 1) * plane + goff);
  }
};

// profile ring: RP levels x P_COUNT values, converted to the compute type when staged
template <typename T>
__device__ __forceinline__ T load_profile(const Scalars& s, int id, int k) {
  return (T)__ldg(s.prof + id * (s.nz + 2) + k);
}
template <typename T>
__device__ __forceinline__ CProf<T> cprof(const T* ring, int k) {
  using namespace tiled;
  return CProf<T>{ring + ((k - 1) & (RP - 1)) * P_COUNT, ring + (k & (RP - 1)) * P_COUNT,
                  ring + ((k + 1) & (RP - 1)) * P_COUNT, ring + ((k + 2) & (RP - 1)) * P_COUNT, k};
}
// the four centred slot pointers of a ring of R planes for level k at plane offset `co`
template <typename T, int R>
__device__ __forceinline__ CRing<T> cring(const T* ring, int k, int co, int j, int i) {
  using Gt = tiled::G<T>;
  // one remainder per ring and level; the neighbouring slots follow by wrapping
  const int m0 = ring_slot<R>(k);
  const int mm = m0 == 0 ? R - 1 : m0 - 1, m1 = m0 + 1 == R ? 0 : m0 + 1, m2 = m1 + 1 == R ? 0 : m1 + 1;
  return CRing<T>{ring + mm * Gt::PLANE + co, ring + m0 * Gt::PLANE + co, ring + m1 * Gt::PLANE + co,
                  ring + m2 * Gt::PLANE + co, k, j, i};
}

// Each CTA runs the levels kb..ke of its tile, kb = 2 + blockIdx.z * kchunk: splitting the level
// range gives enough CTAs to fill every SM on grids with few tiles.
template <typename T, bool TVD>
__global__ void __launch_bounds__(tiled::NT, tiled::ctas_momentum<T>()) k_f_momentum_tiled(Scalars s, DevState<T> d,
                                                                                      int kchunk) {
  using namespace tiled;
  using Gt = G<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sm = reinterpret_cast<T*>(smem_raw);
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  const int i = i0 + tx, j = j0 + ty;
  const int nz = s.nz;
  const int kb = 2 + (int)blockIdx.z * kchunk;
  const int ke = min(nz, kb + kchunk - 1);
  const long long plane = s.plane;
  constexpr int FS = RM * Gt::PLANE;  // field stride inside the shared ring block
  T* rU = sm;
  T* rV = rU + FS;
  T* rW = rV + FS;
  T* rZU = rW + FS;
  T* rZV = rZU + FS;
  T* rZW = rZV + FS;
  T* rVIS = rZW + FS;
  T* rP = rVIS + FS;  // profile ring
  const int co = (ty + HY) * Gt::PW + (tx + Gt::V);
  Stager<T> sg;
  sg.init(s, j0, i0, tid);
  auto stage_level = [&](int kk) {
    sg.template stage<RM>(rU, d.u, plane, kk);
    sg.template stage<RM>(rV, d.v, plane, kk);
    sg.template stage<RM>(rW, d.w, plane, kk);
    sg.template stage<RM>(rZU, d.zu, plane, kk);
    sg.template stage<RM>(rZV, d.zv, plane, kk);
    sg.template stage<RM>(rZW, d.zw, plane, kk);
    sg.template stage<RM>(rVIS, d.vis, plane, kk);
  };
  // level k reads levels k-1 .. k+1 of every ring and profiles k-1 .. k+2
  for (int kk = kb - 1; kk <= kb + 1 && kk <= nz; ++kk) stage_level(kk);
  if (tid < P_COUNT)
    for (int kk = kb - 1; kk <= kb + 2 && kk <= nz; ++kk) rP[(kk & (RP - 1)) * P_COUNT + tid] = load_profile<T>(s, tid, kk);
  const T dtm_x2 = (T)(2.0 * s.dtm);
  if (kb == 2) {
    // level 1: the sources are zero there (stepfields zeroes them)
    const long long o = lin(s, 1, j, i);
    d.zu_n[o] = (T)s.ugal + d.zu[o] + dtm_x2 * (T)0.0;
    d.zv_n[o] = (T)s.vgal + d.zv[o] + dtm_x2 * (T)0.0;
    d.zw_n[o] = (T)0.0 + d.zw[o] + dtm_x2 * (T)0.0;
  }
  const T* __restrict__ th = d.th;
  T th_hi = th[lin(s, kb, j, i)];
  cp_async_wait_all();
  __syncthreads();
  // the viscous stresses of the level below (tau13, tau23 at kb-1 and tau33 at kb), carried up
  // the column from then on
  T tm13 = (T)0.0, tm23 = (T)0.0, t33 = (T)0.0;
  if (s.use_vd) {
    const CProf<T> P = cprof<T>(rP, kb);
    const CRing<T> ZU = cring<T, RM>(rZU, kb, co, j, i), ZV = cring<T, RM>(rZV, kb, co, j, i),
                   ZW = cring<T, RM>(rZW, kb, co, j, i), VIS = cring<T, RM>(rVIS, kb, co, j, i);
    const Tau13<T> tm = tau_13_23<T>(s, P, ZU, ZV, ZW, VIS, kb - 1, j, i);
    tm13 = tm.t13;
    tm23 = tm.t23;
    if (kb < nz) t33 = tau33_at<T>(s, P, ZW, VIS, kb, j, i);
  }
  for (int k = kb; k <= ke; ++k) {
    if (k + 2 <= min(nz, ke + 1)) stage_level(k + 2);
    const bool pstage = tid < P_COUNT && k + 3 <= min(nz, ke + 2);
    T pnext = pstage ? load_profile<T>(s, tid, k + 3) : (T)0;
    const long long o = lin(s, k, j, i);
    const T th_lo = th_hi;
    if (k < nz) th_hi = __ldg(th + o + plane);
    const CProf<T> P = cprof<T>(rP, k);
    const CRing<T> U = cring<T, RM>(rU, k, co, j, i), V = cring<T, RM>(rV, k, co, j, i),
                   W = cring<T, RM>(rW, k, co, j, i);
    const CRing<T> ZU = cring<T, RM>(rZU, k, co, j, i), ZV = cring<T, RM>(rZV, k, co, j, i),
                   ZW = cring<T, RM>(rZW, k, co, j, i), VIS = cring<T, RM>(rVIS, k, co, j, i);
    T su, sv, sw;
    if constexpr (TVD) {
      // the TVD advective sources k_f_flow_tvd_tiled wrote (they start the sums, as PW's do)
      su = d.su[o];
      sv = d.sv[o];
      sw = d.sw[o];
    } else {
      pw_point<T>(s, P, U, V, W, k, j, i, su, sv, sw);
    }
    if (s.use_vd) {
      T du, dv, dw;
      viscosity_core<T>(s, P, ZU, ZV, ZW, ZU, VIS, k, j, i, tm13, tm23, t33, du, dv, dw, tm13, tm23, t33);
      su = su + du;
      sv = sv + dv;
      if (k < nz) sw = sw + dw;
    }
    if (s.coriolis) coriolis_point<T>(s, P, U, V, k, j, i, su, sv);
    // as buoyancy_point, with the horizontal means removed when s.bmean is set
    if (k < nz && !s.passive_th) {
      if (s.bmean) sw = sw + ((T)0.5 * P(P_BUOY_CO, k)) * ((th_lo - (T)s.bmean[k]) + (th_hi - (T)s.bmean[k + 1]));
      else sw = sw + ((T)0.5 * P(P_BUOY_CO, k)) * (th_lo + th_hi);
    }
    if (k < nz && !s.passive_q) {
      const T g2 = (T)(0.5 * s.G);
      const int st = nz + 2;
      for (int n = 0; n < s.nq; ++n) {
        if (s.bmean)
          sw = sw + g2 * (T)s.cq[n] * ((__ldg(d.q[n] + o) - (T)s.bmean[(1 + n) * st + k]) +
                                      (__ldg(d.q[n] + o + plane) - (T)s.bmean[(1 + n) * st + k + 1]));
        else
          sw = sw + g2 * (T)s.cq[n] * (__ldg(d.q[n] + o) + __ldg(d.q[n] + o + plane));
      }
    }
    if (s.damping) damping_flow_point<T>(s, P, k, ZU(k, j, i), ZV(k, j, i), ZW(k, j, i), su, sv, sw);
    if (s.subs_th) subsidence_flow_point<T>(s, P, ZU, ZV, k, j, i, su, sv);
    d.zu_n[o] = (T)s.ugal + ZU(k, j, i) + dtm_x2 * su;
    d.zv_n[o] = (T)s.vgal + ZV(k, j, i) + dtm_x2 * sv;
    d.zw_n[o] = (T)0.0 + ZW(k, j, i) + dtm_x2 * sw;
    if (pstage) rP[((k + 3) & (RP - 1)) * P_COUNT + tid] = pnext;
    cp_async_wait_all();
    __syncthreads();
  }
}

// One scalar of the centred step: `zf` is advected and diffused; with `src` null the kernel also
// steps it (stepfields + the Robert pre-smoothing of swap_smooth, with the negative clip for q
// fields) into out_f / out_zf, otherwise it writes the source (levels 2..nz) for the cloud step.
template <typename T>
struct ScalarJob {
  const T* f;   // state field (th or q)
  const T* zf;  // z-field (zth or zq)
  T* out_f;
  T* out_zf;
  T* src;
  int clip;
  int row;  // the field's row in the mean profiles: 2 for theta, 3 + n for q(n)
};

template <typename T>
__global__ void __launch_bounds__(tiled::NT, tiled::ctas_scalar<T>()) k_f_scalar_tiled(Scalars s, DevState<T> d,
                                                                                    int kchunk, ScalarJob<T> job) {
  using namespace tiled;
  using Gt = G<T>;
  typedef ScalarRings<T> SR;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sm = reinterpret_cast<T*>(smem_raw);
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  const int i = i0 + tx, j = j0 + ty;
  const int nz = s.nz;
  const int kb = 2 + (int)blockIdx.z * kchunk;
  const int ke = min(nz, kb + kchunk - 1);
  const long long plane = s.plane;
  T* rU = sm;
  T* rV = rU + SR::RUV * Gt::PLANE;
  T* rW = rV + SR::RUV * Gt::PLANE;
  T* rD = rW + SR::RW * Gt::PLANE;
  T* rF = rD + SR::RD * Gt::PLANE;
  T* rP = rF + SR::RZF * Gt::PLANE;  // profile ring
  T* FX = rP + RP * P_COUNT;     // [TY][TX+1]: x-faces of columns i0-1 .. i0+TX-1
  T* FY = FX + TY * (TX + 1);    // [TY+1][TX]: y-faces of rows j0-1 .. j0+TY-1
  T* CT = FY + (TY + 1) * TX;    // [2][TY+2][TX+2]: cell_cfl_out of levels of parity 0 and 1
  const int co = (ty + HY) * Gt::PW + (tx + Gt::V);
  // Each face's limiter needs the outflow Courant sum of its upwind cell.  The sums of one level
  // go into a table once (each thread its own cell, the first 2*CW + 2*TY threads one border cell
  // each), one level ahead of the faces that read them.
  const int own_cell = (ty + 1) * CW + tx + 1;
  int hr = -1, hc = -1;
  if (tid < CW) { hr = 0; hc = tid; }
  else if (tid < 2 * CW) { hr = TY + 1; hc = tid - CW; }
  else if (tid < 2 * CW + TY) { hr = tid - 2 * CW + 1; hc = 0; }
  else if (tid < 2 * CW + 2 * TY) { hr = tid - 2 * CW - TY + 1; hc = TX + 1; }
  Stager<T> sg;
  sg.init(s, j0, i0, tid);
  // level k reads the scalar at k-1 .. k+2, u v w at k-1 .. k+1, diff at k-1 .. k and profiles
  // at k-1 .. k+2; a chunk above level 2 also needs the z face below it (level kb-1).
  const int k0 = kb == 2 ? 1 : kb - 2;
  for (int kk = k0; kk <= kb + 2 && kk <= nz; ++kk) sg.template stage<SR::RZF>(rF, job.zf, plane, kk);
  // (the z face below the chunk reads w from level kb-2 but u and v from kb-1 up)
  for (int kk = k0; kk <= kb + 1 && kk <= nz; ++kk) {
    if (kk >= kb - 1) {
      sg.template stage<SR::RUV>(rU, d.u, plane, kk);
      sg.template stage<SR::RUV>(rV, d.v, plane, kk);
    }
    sg.template stage<SR::RW>(rW, d.w, plane, kk);
  }
  for (int kk = kb - 1; kk <= kb; ++kk) sg.template stage<SR::RD>(rD, d.diff, plane, kk);
  if (tid < P_COUNT)
    for (int kk = k0; kk <= kb + 2 && kk <= nz; ++kk) rP[(kk & (RP - 1)) * P_COUNT + tid] = load_profile<T>(s, tid, kk);
  const T dtm_x2 = (T)(2.0 * s.dtm);
  const T c1 = (T)(1.0 - 2.0 * s.tsmth), c2 = (T)s.tsmth;
  const T* __restrict__ th = job.f;
  if (kb == 2) {
    // level 1: zero source
    const long long o = lin(s, 1, j, i);
    if (job.src) {
      job.src[o] = (T)0.0;
    } else {
      T fv = th[o], zv = job.zf[o];
      T sm1 = c1 * fv + c2 * zv;
      T zn = (T)0.0 + zv + dtm_x2 * (T)0.0;
      if (job.clip && zn < (T)0.0) zn = (T)0.0;
      job.out_zf[o] = sm1 + (T)s.tsmth * zn;
      job.out_f[o] = zn;
    }
  }
  cp_async_wait_all();
  __syncthreads();
  const T dt = (T)(s.dtm * 2.0);
  T fz_lo = (T)0.0;  // flux_z(2) = 0
  if (kb > 2) {
    const int kz = kb - 1;
    const CProf<T> P = cprof<T>(rP, kz);
    const CRing<T> U = cring<T, SR::RUV>(rU, kz, co, j, i), V = cring<T, SR::RUV>(rV, kz, co, j, i),
                   W = cring<T, SR::RW>(rW, kz, co, j, i);
    const CRing<T> ZF = cring<T, SR::RZF>(rF, kz, co, j, i);
    fz_lo = tvd_face_z<T>(s, P, U, V, W, ZF, dt, kz, j, i);
  }
  {
    // the cell sums of level kb
    const CProf<T> P = cprof<T>(rP, kb);
    const CRing<T> U = cring<T, SR::RUV>(rU, kb, co, j, i), V = cring<T, SR::RUV>(rV, kb, co, j, i),
                   W = cring<T, SR::RW>(rW, kb, co, j, i);
    T* C = CT + (kb & 1) * CN;
    C[own_cell] = cell_cfl_out<T>(s, P, U, V, W, kb, j, i);
    if (hr >= 0) C[hr * CW + hc] = cell_cfl_out<T>(s, P, U, V, W, kb, j0 - 1 + hr, i0 - 1 + hc);
  }
  // the table is complete; the first prefetch overwrites the slots of levels kb-1 (u, v) and kb-2 (w)
  __syncthreads();
  for (int k = kb; k <= ke; ++k) {
    if (k + 3 <= min(nz, ke + 2)) sg.template stage<SR::RZF>(rF, job.zf, plane, k + 3);
    if (k + 2 <= min(nz, ke + 1)) {
      sg.template stage<SR::RUV>(rU, d.u, plane, k + 2);
      sg.template stage<SR::RUV>(rV, d.v, plane, k + 2);
      sg.template stage<SR::RW>(rW, d.w, plane, k + 2);
    }
    if (k + 1 <= min(nz, ke)) sg.template stage<SR::RD>(rD, d.diff, plane, k + 1);
    const bool pstage = tid < P_COUNT && k + 3 <= min(nz, ke + 2);
    T pnext = pstage ? load_profile<T>(s, tid, k + 3) : (T)0;
    const long long o = lin(s, k, j, i);
    const T fv = job.src ? (T)0.0 : __ldg(th + o);
    const CProf<T> P = cprof<T>(rP, k);
    const CRing<T> U = cring<T, SR::RUV>(rU, k, co, j, i), V = cring<T, SR::RUV>(rV, k, co, j, i),
                   W = cring<T, SR::RW>(rW, k, co, j, i), DIFF = cring<T, SR::RD>(rD, k, co, j, i);
    const CRing<T> ZF = cring<T, SR::RZF>(rF, k, co, j, i);
    // the cell sums of level k+1: the own cell's for the z face above, the table for the next level
    T c_hi = (T)0.0;
    if (k < nz) {
      c_hi = cell_cfl_out<T>(s, P, U, V, W, k + 1, j, i);
      if (k + 1 <= ke) {
        T* C = CT + ((k + 1) & 1) * CN;
        C[own_cell] = c_hi;
        if (hr >= 0) C[hr * CW + hc] = cell_cfl_out<T>(s, P, U, V, W, k + 1, j0 - 1 + hr, i0 - 1 + hc);
      }
    }
    const T* Ck = CT + (k & 1) * CN;
    auto cfl = [&](int kk, int jj, int ii) -> T { return kk == k ? Ck[(jj - j0 + 1) * CW + (ii - i0 + 1)] : c_hi; };
    // TVD faces of this level: own x+1/2 and y+1/2 faces, then the tile's low-side faces
    FX[ty * (TX + 1) + tx + 1] =
        tvd_face_x_g<T, CRing<T>, CRing<T>, CProf<T>, TvdMetricScalar>(s, P, U, V, W, ZF, dt, k, j, i, cfl);
    FY[(ty + 1) * TX + tx] =
        tvd_face_y_g<T, CRing<T>, CRing<T>, CProf<T>, TvdMetricScalar>(s, P, U, V, W, ZF, dt, k, j, i, cfl);
    T fz_hi = (k < nz) ? tvd_face_z_g<T, CRing<T>, CRing<T>, CProf<T>, TvdMetricScalar>(s, P, U, V, W, ZF, dt, k, j, i, cfl)
                       : (T)0.0;
    if (tid < TX)
      FY[tid] = tvd_face_y_g<T, CRing<T>, CRing<T>, CProf<T>, TvdMetricScalar>(s, P, U, V, W, ZF, dt, k, j0 - 1,
                                                                               i0 + tid, cfl);
    else if (tid < TX + TY)
      FX[(tid - TX) * (TX + 1)] = tvd_face_x_g<T, CRing<T>, CRing<T>, CProf<T>, TvdMetricScalar>(
          s, P, U, V, W, ZF, dt, k, j0 + tid - TX, i0 - 1, cfl);
    __syncthreads();
    T sth = tvd_source<T>(s, P, U, V, W, FX[ty * (TX + 1) + tx], FX[ty * (TX + 1) + tx + 1], FY[ty * TX + tx],
                          FY[(ty + 1) * TX + tx], fz_lo, fz_hi, k, j, i, (T)0.0);
    if (s.th_baroclinic && job.row == 2) sth = sth + th_baroclinic_point<T>(s, U, V, k, j, i);
    if (s.use_vd) sth = sth + diffusion_point<T>(s, P, ZF, DIFF, k, j, i);
    // damping, then forcing's subsidence (the dynamics group's order)
    if (s.damping && (job.row > 2 || !s.passive_th)) sth = damping_scalar_point<T>(s, P, k, ZF(k, j, i), job.row, sth);
    if (job.row == 2 ? s.subs_th : s.subs_q)
      sth = job.row == 2 ? subsidence_theta_point<T>(s, P, ZF, k, j, i, sth)
                         : subsidence_q_point<T>(s, P, ZF, job.row - 3, k, j, i, sth);
    fz_lo = fz_hi;
    if (job.src) {
      job.src[o] = sth;
    } else {
      T zv = ZF(k, j, i);
      T smo = c1 * fv + c2 * zv;
      T zn = (T)0.0 + zv + dtm_x2 * sth;
      if (job.clip && zn < (T)0.0) zn = (T)0.0;
      job.out_zf[o] = smo + (T)s.tsmth * zn;
      job.out_f[o] = zn;
    }
    if (pstage) rP[((k + 3) & (RP - 1)) * P_COUNT + tid] = pnext;
    cp_async_wait_all();
    __syncthreads();
  }
}

// TVD advection of one flow component on a centred step (advection_flow_fields = tvd): the
// advective source of u (DIM 0), v (1) or w (2) into `src`, levels 2..nz (w: 2..nz-1, 0 at nz),
// which the momentum kernel then takes in place of pw_advection's.  Tiled like the scalar
// kernel: the same face functions on the component's dual-grid velocities (`DualFlow`), each
// x and y face computed once and shared through shared memory, the z face carried up the column;
// the faces and the source are tvd_flow_point's, so the result is bit-identical to it.
template <typename T, int DIM>
__global__ void __launch_bounds__(tiled::NT, tiled::min_ctas3()) k_f_flow_tvd_tiled(Scalars s, DevState<T> d,
                                                                                   int kchunk, T* __restrict__ src) {
  using namespace tiled;
  using Gt = G<T>;
  typedef FlowRings<DIM> R;
  typedef typename std::conditional<DIM == 2, TvdMetricW, TvdMetricScalar>::type M;
  typedef DualFlow<T, CRing<T>, DIM> F;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sm = reinterpret_cast<T*>(smem_raw);
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  const int i = i0 + tx, j = j0 + ty;
  const int nz = s.nz;
  const int ktop = DIM == 2 ? nz - 1 : nz;  // the last level with a source
  const int kb = 2 + (int)blockIdx.z * kchunk;
  const int ke = min(nz, kb + kchunk - 1);
  const long long plane = s.plane;
  T* rU = sm;
  T* rV = rU + R::RUV * Gt::PLANE;
  T* rW = rV + R::RUV * Gt::PLANE;
  T* rZ = rW + R::RW * Gt::PLANE;
  T* rP = rZ + R::RZ * Gt::PLANE;
  T* FX = rP + RP * P_COUNT;   // [TY][TX+1]: x-faces of columns i0-1 .. i0+TX-1
  T* FY = FX + TY * (TX + 1);  // [TY+1][TX]: y-faces of rows j0-1 .. j0+TY-1
  T* CT = FY + (TY + 1) * TX;  // [2][TY+2][TX+2]: cell Courant sums of levels of parity 0 and 1
  const int co = (ty + HY) * Gt::PW + (tx + Gt::V);
  // the cell sums each face's limiter needs, once per cell and level, as the scalar kernel forms
  // them (own cell per thread, the tile's border cells by the first 2*CW + 2*TY threads)
  const int own_cell = (ty + 1) * CW + tx + 1;
  int hr = -1, hc = -1;
  if (tid < CW) { hr = 0; hc = tid; }
  else if (tid < 2 * CW) { hr = TY + 1; hc = tid - CW; }
  else if (tid < 2 * CW + TY) { hr = tid - 2 * CW + 1; hc = 0; }
  else if (tid < 2 * CW + 2 * TY) { hr = tid - 2 * CW - TY + 1; hc = TX + 1; }
  const T* zf = DIM == 0 ? d.zu : (DIM == 1 ? d.zv : d.zw);
  Stager<T> sg;
  sg.init(s, j0, i0, tid);
  // the chunk starts with the z face below level kb (at kb-1): w from kb-2, u and v from kb-1
  const int k0 = kb == 2 ? 1 : kb - 2;
  for (int kk = k0; kk <= kb + 2 && kk <= nz; ++kk) sg.template stage<R::RZ>(rZ, zf, plane, kk);
  for (int kk = k0; kk <= kb + R::UPF && kk <= nz; ++kk) {
    if (kk >= kb - 1) {
      sg.template stage<R::RUV>(rU, d.u, plane, kk);
      sg.template stage<R::RUV>(rV, d.v, plane, kk);
    }
    sg.template stage<R::RW>(rW, d.w, plane, kk);
  }
  if (tid < P_COUNT)
    for (int kk = k0; kk <= kb + 2 && kk <= nz; ++kk) rP[(kk & (RP - 1)) * P_COUNT + tid] = load_profile<T>(s, tid, kk);
  cp_async_wait_all();
  __syncthreads();
  const T dt = (T)(s.dtm * 2.0);  // momentum_stepping is always centred
  T fz_lo = (T)0.0;               // u, v: no flux through the face above level 1
  {
    const int kz = kb - 1;
    const CProf<T> P = cprof<T>(rP, kz);
    const CRing<T> U = cring<T, R::RUV>(rU, kz, co, j, i), V = cring<T, R::RUV>(rV, kz, co, j, i),
                   W = cring<T, R::RW>(rW, kz, co, j, i), ZF = cring<T, R::RZ>(rZ, kz, co, j, i);
    const F IU{U, nz}, IV{V, nz}, IW{W, nz};
    if (kb > 2) fz_lo = tvd_face_z<T, F, CRing<T>, CProf<T>, M>(s, P, IU, IV, IW, ZF, dt, kz, j, i);
    else if (DIM == 2) fz_lo = tvd_face_z_bottom<T, F, CRing<T>, CProf<T>, M>(s, P, IU, IV, IW, ZF, dt, j, i);
  }
  if (kb <= ktop) {
    // the cell sums of level kb
    const CProf<T> P = cprof<T>(rP, kb);
    const CRing<T> U = cring<T, R::RUV>(rU, kb, co, j, i), V = cring<T, R::RUV>(rV, kb, co, j, i),
                   W = cring<T, R::RW>(rW, kb, co, j, i);
    const F IU{U, nz}, IV{V, nz}, IW{W, nz};
    T* C = CT + (kb & 1) * CN;
    C[own_cell] = cell_cfl_out<T, F, CProf<T>, M>(s, P, IU, IV, IW, kb, j, i);
    if (hr >= 0) C[hr * CW + hc] = cell_cfl_out<T, F, CProf<T>, M>(s, P, IU, IV, IW, kb, j0 - 1 + hr, i0 - 1 + hc);
  }
  // The first prefetch below overwrites the slot of level kb-1 that this face read.  The copy is
  // an asm statement without a memory clobber, so without the barrier the compiler may sink the
  // face's shared-memory loads past it (a race that showed as run-to-run differences in w's
  // lowest source).
  __syncthreads();
  for (int k = kb; k <= ke; ++k) {
    if (k + 3 <= min(nz, ke + 2)) sg.template stage<R::RZ>(rZ, zf, plane, k + 3);
    if (k + R::UPF + 1 <= min(nz, ke + R::UPF)) {
      sg.template stage<R::RUV>(rU, d.u, plane, k + R::UPF + 1);
      sg.template stage<R::RUV>(rV, d.v, plane, k + R::UPF + 1);
      sg.template stage<R::RW>(rW, d.w, plane, k + R::UPF + 1);
    }
    const bool pstage = tid < P_COUNT && k + 3 <= min(nz, ke + 2);
    T pnext = pstage ? load_profile<T>(s, tid, k + 3) : (T)0;
    const long long o = lin(s, k, j, i);
    if (k <= ktop) {
      const CProf<T> P = cprof<T>(rP, k);
      const CRing<T> U = cring<T, R::RUV>(rU, k, co, j, i), V = cring<T, R::RUV>(rV, k, co, j, i),
                     W = cring<T, R::RW>(rW, k, co, j, i), ZF = cring<T, R::RZ>(rZ, k, co, j, i);
      const F IU{U, nz}, IV{V, nz}, IW{W, nz};
      // the cell sums of level k+1: the own cell's for the z face above, the table for the next level
      T c_hi = (T)0.0;
      if (k < nz) {
        c_hi = cell_cfl_out<T, F, CProf<T>, M>(s, P, IU, IV, IW, k + 1, j, i);
        if (k + 1 <= min(ke, ktop)) {
          T* C = CT + ((k + 1) & 1) * CN;
          C[own_cell] = c_hi;
          if (hr >= 0) C[hr * CW + hc] = cell_cfl_out<T, F, CProf<T>, M>(s, P, IU, IV, IW, k + 1, j0 - 1 + hr, i0 - 1 + hc);
        }
      }
      const T* Ck = CT + (k & 1) * CN;
      auto cfl = [&](int kk, int jj, int ii) -> T { return kk == k ? Ck[(jj - j0 + 1) * CW + (ii - i0 + 1)] : c_hi; };
      typedef decltype(cfl) CS;
      FX[ty * (TX + 1) + tx + 1] = tvd_face_x_g<T, F, CRing<T>, CProf<T>, M, CS>(s, P, IU, IV, IW, ZF, dt, k, j, i, cfl);
      FY[(ty + 1) * TX + tx] = tvd_face_y_g<T, F, CRing<T>, CProf<T>, M, CS>(s, P, IU, IV, IW, ZF, dt, k, j, i, cfl);
      // u, v have no z face above the top level; w's top level (nz-1) has one
      const T fz_hi = (DIM == 2 || k < nz)
                          ? tvd_face_z_g<T, F, CRing<T>, CProf<T>, M, CS>(s, P, IU, IV, IW, ZF, dt, k, j, i, cfl)
                          : (T)0.0;
      if (tid < TX)
        FY[tid] = tvd_face_y_g<T, F, CRing<T>, CProf<T>, M, CS>(s, P, IU, IV, IW, ZF, dt, k, j0 - 1, i0 + tid, cfl);
      else if (tid < TX + TY)
        FX[(tid - TX) * (TX + 1)] = tvd_face_x_g<T, F, CRing<T>, CProf<T>, M, CS>(s, P, IU, IV, IW, ZF, dt, k,
                                                                                 j0 + tid - TX, i0 - 1, cfl);
      __syncthreads();
      src[o] = tvd_source<T, F, CProf<T>, M>(s, P, IU, IV, IW, FX[ty * (TX + 1) + tx], FX[ty * (TX + 1) + tx + 1],
                                            FY[ty * TX + tx], FY[(ty + 1) * TX + tx], fz_lo, fz_hi, k, j, i, (T)0.0);
      fz_lo = fz_hi;
    } else {
      src[o] = (T)0.0;  // w at the top level
    }
    if (pstage) rP[((k + 3) & (RP - 1)) * P_COUNT + tid] = pnext;
    cp_async_wait_all();
    __syncthreads();
  }
}

// The whole moist centred step of theta, vapour and liquid in one pass (number_q_fields = 2):
// for each scalar the TVD faces, source, diffusion, damping and subsidence of k_f_scalar_tiled,
// then simplecloud and stepfields (with swap_smooth's pre-smoothing and the negative-q clip) of
// k_f_cloud_step, at each point as soon as its three sources are known.  The sources never go
// to memory, the flow, diff and the Courant sums are staged once for the three scalars, and the
// results are those of the point kernel, to the bit.
template <typename T>
__global__ void __launch_bounds__(tiled::NT, sizeof(T) == 4 ? 3 : 2) k_f_moist_tiled(Scalars s, DevState<T> d, int kchunk) {
  using namespace tiled;
  using Gt = G<T>;
  typedef MoistRings R;
  constexpr int NS = R::NS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sm = reinterpret_cast<T*>(smem_raw);
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  const int i = i0 + tx, j = j0 + ty;
  const int nz = s.nz;
  const int kb = 2 + (int)blockIdx.z * kchunk;
  const int ke = min(nz, kb + kchunk - 1);
  const long long plane = s.plane;
  T* rU = sm;
  T* rV = rU + R::RUV * Gt::PLANE;
  T* rW = rV + R::RUV * Gt::PLANE;
  T* rD = rW + R::RW * Gt::PLANE;
  T* rF[NS];
  rF[0] = rD + R::RD * Gt::PLANE;
  for (int n = 1; n < NS; ++n) rF[n] = rF[n - 1] + R::RZF * Gt::PLANE;
  T* rP = rF[NS - 1] + R::RZF * Gt::PLANE;
  T* FXs[2];
  T* FYs[2];
  FXs[0] = rP + RP * P_COUNT;
  FYs[0] = FXs[0] + TY * (TX + 1);
  FXs[1] = FYs[0] + (TY + 1) * TX;
  FYs[1] = FXs[1] + TY * (TX + 1);
  T* CT = FYs[1] + (TY + 1) * TX;
  const int co = (ty + HY) * Gt::PW + (tx + Gt::V);
  const int own_cell = (ty + 1) * CW + tx + 1;
  int hr = -1, hc = -1;
  if (tid < CW) { hr = 0; hc = tid; }
  else if (tid < 2 * CW) { hr = TY + 1; hc = tid - CW; }
  else if (tid < 2 * CW + TY) { hr = tid - 2 * CW + 1; hc = 0; }
  else if (tid < 2 * CW + 2 * TY) { hr = tid - 2 * CW - TY + 1; hc = TX + 1; }
  // scalar n: 0 theta, 1 + m the q field m; its state, z-field, outputs and mean-profile row
  const T* fs[NS] = {d.th, d.q[0], d.q[1]};
  const T* zfs[NS] = {d.zth, d.zq[0], d.zq[1]};
  T* fo[NS] = {d.th_n, d.q_n[0], d.q_n[1]};
  T* zfo[NS] = {d.zth_n, d.zq_n[0], d.zq_n[1]};
  Stager<T> sg;
  sg.init(s, j0, i0, tid);
  const int k0 = kb == 2 ? 1 : kb - 2;
  for (int kk = k0; kk <= kb + 2 && kk <= nz; ++kk)
#pragma unroll
    for (int n = 0; n < NS; ++n) sg.template stage<R::RZF>(rF[n], zfs[n], plane, kk);
  for (int kk = k0; kk <= kb + 1 && kk <= nz; ++kk) {
    if (kk >= kb - 1) {
      sg.template stage<R::RUV>(rU, d.u, plane, kk);
      sg.template stage<R::RUV>(rV, d.v, plane, kk);
    }
    sg.template stage<R::RW>(rW, d.w, plane, kk);
  }
  for (int kk = kb - 1; kk <= kb; ++kk) sg.template stage<R::RD>(rD, d.diff, plane, kk);
  if (tid < P_COUNT)
    for (int kk = k0; kk <= kb + 2 && kk <= nz; ++kk) rP[(kk & (RP - 1)) * P_COUNT + tid] = load_profile<T>(s, tid, kk);
  const T dtm_x2 = (T)(2.0 * s.dtm);
  const T c1 = (T)(1.0 - 2.0 * s.tsmth), c2 = (T)s.tsmth;
  // stepfields with the pre-smoothing of swap_smooth (k_f_cloud_step's `step`)
  auto step = [&](int n, long long o, T zv, T src) {
    const T fv = fs[n][o];
    const T smo = c1 * fv + c2 * zv;
    T zn = (T)0.0 + zv + dtm_x2 * src;
    if (n > 0 && zn < (T)0.0) zn = (T)0.0;
    zfo[n][o] = smo + (T)s.tsmth * zn;
    fo[n][o] = zn;
  };
  if (kb == 2) {
    // level 1: zero sources
    const long long o = lin(s, 1, j, i);
#pragma unroll
    for (int n = 0; n < NS; ++n) step(n, o, zfs[n][o], (T)0.0);
  }
  cp_async_wait_all();
  __syncthreads();
  const T dt = (T)(s.dtm * 2.0);
  T fz_lo[NS];
#pragma unroll
  for (int n = 0; n < NS; ++n) fz_lo[n] = (T)0.0;  // flux_z(2) = 0
  if (kb > 2) {
    const int kz = kb - 1;
    const CProf<T> P = cprof<T>(rP, kz);
    const CRing<T> U = cring<T, R::RUV>(rU, kz, co, j, i), V = cring<T, R::RUV>(rV, kz, co, j, i),
                   W = cring<T, R::RW>(rW, kz, co, j, i);
#pragma unroll
    for (int n = 0; n < NS; ++n) {
      const CRing<T> ZF = cring<T, R::RZF>(rF[n], kz, co, j, i);
      fz_lo[n] = tvd_face_z<T>(s, P, U, V, W, ZF, dt, kz, j, i);
    }
  }
  {
    const CProf<T> P = cprof<T>(rP, kb);
    const CRing<T> U = cring<T, R::RUV>(rU, kb, co, j, i), V = cring<T, R::RUV>(rV, kb, co, j, i),
                   W = cring<T, R::RW>(rW, kb, co, j, i);
    T* C = CT + (kb & 1) * CN;
    C[own_cell] = cell_cfl_out<T>(s, P, U, V, W, kb, j, i);
    if (hr >= 0) C[hr * CW + hc] = cell_cfl_out<T>(s, P, U, V, W, kb, j0 - 1 + hr, i0 - 1 + hc);
  }
  // the first prefetch overwrites the slots of levels kb-1 (u, v) and kb-2 (w, the scalars)
  __syncthreads();
  for (int k = kb; k <= ke; ++k) {
    if (k + 3 <= min(nz, ke + 2))
#pragma unroll
      for (int n = 0; n < NS; ++n) sg.template stage<R::RZF>(rF[n], zfs[n], plane, k + 3);
    if (k + 2 <= min(nz, ke + 1)) {
      sg.template stage<R::RUV>(rU, d.u, plane, k + 2);
      sg.template stage<R::RUV>(rV, d.v, plane, k + 2);
      sg.template stage<R::RW>(rW, d.w, plane, k + 2);
    }
    if (k + 1 <= min(nz, ke)) sg.template stage<R::RD>(rD, d.diff, plane, k + 1);
    const bool pstage = tid < P_COUNT && k + 3 <= min(nz, ke + 2);
    T pnext = pstage ? load_profile<T>(s, tid, k + 3) : (T)0;
    const long long o = lin(s, k, j, i);
    const CProf<T> P = cprof<T>(rP, k);
    const CRing<T> U = cring<T, R::RUV>(rU, k, co, j, i), V = cring<T, R::RUV>(rV, k, co, j, i),
                   W = cring<T, R::RW>(rW, k, co, j, i), DIFF = cring<T, R::RD>(rD, k, co, j, i);
    // the cell sums of level k+1: the own cell's for the z faces above, the table for the next level
    T c_hi = (T)0.0;
    if (k < nz) {
      c_hi = cell_cfl_out<T>(s, P, U, V, W, k + 1, j, i);
      if (k + 1 <= ke) {
        T* C = CT + ((k + 1) & 1) * CN;
        C[own_cell] = c_hi;
        if (hr >= 0) C[hr * CW + hc] = cell_cfl_out<T>(s, P, U, V, W, k + 1, j0 - 1 + hr, i0 - 1 + hc);
      }
    }
    const T* Ck = CT + (k & 1) * CN;
    auto cfl = [&](int kk, int jj, int ii) -> T { return kk == k ? Ck[(jj - j0 + 1) * CW + (ii - i0 + 1)] : c_hi; };
    typedef decltype(cfl) CS;
    T src[NS], zv[NS];
#pragma unroll
    for (int n = 0; n < NS; ++n) {
      // faces of scalar n into buffer n & 1; the barrier also ends the reads of that buffer by
      // scalar n - 2's source
      T* FX = FXs[n & 1];
      T* FY = FYs[n & 1];
      const CRing<T> ZF = cring<T, R::RZF>(rF[n], k, co, j, i);
      FX[ty * (TX + 1) + tx + 1] =
          tvd_face_x_g<T, CRing<T>, CRing<T>, CProf<T>, TvdMetricScalar, CS>(s, P, U, V, W, ZF, dt, k, j, i, cfl);
      FY[(ty + 1) * TX + tx] =
          tvd_face_y_g<T, CRing<T>, CRing<T>, CProf<T>, TvdMetricScalar, CS>(s, P, U, V, W, ZF, dt, k, j, i, cfl);
      const T fz_hi = (k < nz) ? tvd_face_z_g<T, CRing<T>, CRing<T>, CProf<T>, TvdMetricScalar, CS>(
                                     s, P, U, V, W, ZF, dt, k, j, i, cfl)
                               : (T)0.0;
      if (tid < TX)
        FY[tid] = tvd_face_y_g<T, CRing<T>, CRing<T>, CProf<T>, TvdMetricScalar, CS>(s, P, U, V, W, ZF, dt, k, j0 - 1,
                                                                                    i0 + tid, cfl);
      else if (tid < TX + TY)
        FX[(tid - TX) * (TX + 1)] = tvd_face_x_g<T, CRing<T>, CRing<T>, CProf<T>, TvdMetricScalar, CS>(
            s, P, U, V, W, ZF, dt, k, j0 + tid - TX, i0 - 1, cfl);
      __syncthreads();
      const int row = n == 0 ? 2 : 2 + n;
      T sf = tvd_source<T>(s, P, U, V, W, FX[ty * (TX + 1) + tx], FX[ty * (TX + 1) + tx + 1], FY[ty * TX + tx],
                           FY[(ty + 1) * TX + tx], fz_lo[n], fz_hi, k, j, i, (T)0.0);
      if (n == 0 && s.th_baroclinic) sf = sf + th_baroclinic_point<T>(s, U, V, k, j, i);
      if (s.use_vd) sf = sf + diffusion_point<T>(s, P, ZF, DIFF, k, j, i);
      if (s.damping && (row > 2 || !s.passive_th)) sf = damping_scalar_point<T>(s, P, k, ZF(k, j, i), row, sf);
      if (n == 0 ? s.subs_th : s.subs_q)
        sf = n == 0 ? subsidence_theta_point<T>(s, P, ZF, k, j, i, sf)
                    : subsidence_q_point<T>(s, P, ZF, n - 1, k, j, i, sf);
      fz_lo[n] = fz_hi;
      src[n] = sf;
      zv[n] = ZF(k, j, i);
    }
    // simplecloud and stepfields (k_f_cloud_step)
    if (s.simplecloud) {
      // vapour and liquid are q fields iqv and iql, scalars 1 + iqv and 1 + iql (selected, so
      // that the arrays stay in registers)
      const bool v0 = s.iqv == 0;
      const T zqv = v0 ? zv[1] : zv[2], zql = v0 ? zv[2] : zv[1];
      T sqv = v0 ? src[1] : src[2], sql = v0 ? src[2] : src[1];
      simplecloud_point<T>(s, P, k, zqv, zql, zv[0], zql, src[0], sqv, sql);
      src[1] = v0 ? sqv : sql;
      src[2] = v0 ? sql : sqv;
    }
#pragma unroll
    for (int n = 0; n < NS; ++n) step(n, o, zv[n], src[n]);
    if (pstage) rP[((k + 3) & (RP - 1)) * P_COUNT + tid] = pnext;
    cp_async_wait_all();
    __syncthreads();
  }
}

// Moist centred step after the tiled scalar kernels have written the advective + diffusive
// sources: simplecloud (when enabled), then stepfields with the Robert pre-smoothing of
// swap_smooth for theta and every q field (negative q clipped), as the point kernel does.
template <typename T>
__global__ void __launch_bounds__(256) k_f_cloud_step(Scalars s, DevState<T> d) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z + 1;
  if (i >= s.nx || j >= s.ny || k > s.nz) return;
  const long long o = lin(s, k, j, i);
  T sth = k >= 2 ? d.sth[o] : (T)0.0;
  T sq[MGPU_MAX_Q];
  for (int n = 0; n < s.nq; ++n) sq[n] = k >= 2 ? d.sq[n][o] : (T)0.0;
  if (s.simplecloud && k >= 2) {
    Prof<T> P = prof<T>(s);
    const int iv = s.iqv, il = s.iql;
    simplecloud_point<T>(s, P, k, d.zq[iv][o], d.zq[il][o], d.zth[o], d.zq[il][o], sth, sq[iv], sq[il]);
  }
  const T dtm_x2 = (T)(2.0 * s.dtm);
  const T c1 = (T)(1.0 - 2.0 * s.tsmth), c2 = (T)s.tsmth;
  auto step = [&](const T* f, const T* zf, T src, T* f_out, T* zf_out, bool clip) {
    T fv = f[o], zv = zf[o];
    T sm = c1 * fv + c2 * zv;
    T zn = (T)0.0 + zv + dtm_x2 * src;
    if (clip && zn < (T)0.0) zn = (T)0.0;
    zf_out[o] = sm + (T)s.tsmth * zn;
    f_out[o] = zn;
  };
  step(d.th, d.zth, sth, d.th_n, d.zth_n, false);
  for (int n = 0; n < s.nq; ++n) step(d.q[n], d.zq[n], sq[n], d.q_n[n], d.zq_n[n], true);
}

// Smagorinsky of levels kb..ke (2 <= k <= nz-1) of a tile, shared-memory tiled like the
// dynamics kernels: u, v, w (the z-fields on centred steps) in rings of four planes, profiles in a
// ring, the Richardson-number inputs (th, q) read at the column itself.  The chunk holding level
// nz-1 also zeroes vis and diff at the top level.  Level 1 (lower_bc) is k_c_lower_bc.
template <typename T>
__global__ void __launch_bounds__(tiled::NT, tiled::ctas_scalar<T>()) k_f_smag_tiled(Scalars s, DevState<T> d,
                                                                                  int kchunk) {
  using namespace tiled;
  using Gt = G<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sm = reinterpret_cast<T*>(smem_raw);
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  const int i = i0 + tx, j = j0 + ty;
  const int nz = s.nz;
  const int kb = 2 + (int)blockIdx.z * kchunk;
  const int ke = min(nz - 1, kb + kchunk - 1);
  const long long plane = s.plane;
  const bool fwd = s.forward;
  constexpr int FS = RM * Gt::PLANE;
  T* rU = sm;
  T* rV = rU + FS;
  T* rW = rV + FS;
  T* rP = rW + FS;
  const int co = (ty + HY) * Gt::PW + (tx + Gt::V);
  const T* gu = fwd ? d.u : d.zu;
  const T* gv = fwd ? d.v : d.zv;
  const T* gw = fwd ? d.w : d.zw;
  Stager<T> sg;
  sg.init(s, j0, i0, tid);
  auto stage_level = [&](int kk) {
    sg.template stage<RM>(rU, gu, plane, kk);
    sg.template stage<RM>(rV, gv, plane, kk);
    sg.template stage<RM>(rW, gw, plane, kk);
  };
  for (int kk = kb - 1; kk <= kb + 1 && kk <= nz; ++kk) stage_level(kk);
  if (tid < P_COUNT)
    for (int kk = kb - 1; kk <= kb + 2 && kk <= nz; ++kk) rP[(kk & (RP - 1)) * P_COUNT + tid] = load_profile<T>(s, tid, kk);
  const View<T> THc = view<T>(d.th, s), THa = view<T>(fwd ? d.th : d.zth, s);
  View<T> QV, QL;
  const bool moist = !s.passive_q && s.nq > 1;
  if (moist) {
    QV = view<T>(fwd ? d.q[s.iqv] : d.zq[s.iqv], s);
    QL = view<T>(fwd ? d.q[s.iql] : d.zq[s.iql], s);
  }
  if (ke == nz - 1) {
    const long long o = lin(s, nz, j, i);
    d.vis[o] = (T)0.0;
    d.diff[o] = (T)0.0;
  }
  cp_async_wait_all();
  __syncthreads();
  // the dry Richardson number reads th at k and k+1 of the column: kept in registers, the level
  // k+2 value loaded one level ahead so that its latency overlaps the strain rate
  const T* __restrict__ thg = d.th;
  T th0 = (T)0.0, th1 = (T)0.0;
  if (!moist) {
    th0 = __ldg(thg + lin(s, kb, j, i));
    th1 = __ldg(thg + lin(s, kb + 1, j, i));
  }
  // the strain-rate parts of level k come from the level below, where they were level k+1's
  StrainLevel<T> lo;
  {
    const CProf<T> P = cprof<T>(rP, kb);
    const CRing<T> U = cring<T, RM>(rU, kb, co, j, i), V = cring<T, RM>(rV, kb, co, j, i),
                   W = cring<T, RM>(rW, kb, co, j, i);
    lo = strain_level<T>(s, P, U, V, W, kb, j, i);
  }
  for (int k = kb; k <= ke; ++k) {
    if (k + 2 <= min(nz, ke + 1)) stage_level(k + 2);
    const bool pstage = tid < P_COUNT && k + 3 <= min(nz, ke + 2);
    T pnext = pstage ? load_profile<T>(s, tid, k + 3) : (T)0;
    const CProf<T> P = cprof<T>(rP, k);
    const CRing<T> U = cring<T, RM>(rU, k, co, j, i), V = cring<T, RM>(rV, k, co, j, i),
                   W = cring<T, RM>(rW, k, co, j, i);
    const T th2 = (!moist && k + 2 <= nz) ? __ldg(thg + lin(s, k + 2, j, i)) : (T)0.0;
    const StrainLevel<T> hi = strain_level<T>(s, P, U, V, W, k + 1, j, i);
    const T ssq = half_squared_strain_parts<T>(s, P, U, V, W, k, j, i, lo, hi);
    lo = hi;
    T vis, diff;
    if (moist)
      smagorinsky_from_strain<T, CProf<T>, View<T>, View<T>>(s, P, ssq, THc, THa, &QV, &QL, k, j, i, vis, diff);
    else
      smagorinsky_from_strain<T, CProf<T>, ColPair<T>, View<T>>(s, P, ssq, ColPair<T>{th0, th1, k}, THa,
                                                                (const View<T>*)nullptr, (const View<T>*)nullptr, k, j,
                                                                i, vis, diff);
    th0 = th1;
    th1 = th2;
    const long long o = lin(s, k, j, i);
    d.vis[o] = vis;
    d.diff[o] = diff;
    if (pstage) rP[((k + 3) & (RP - 1)) * P_COUNT + tid] = pnext;
    cp_async_wait_all();
    __syncthreads();
  }
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

// 5. pstep + swap_smooth of u, v, w.  Every input is loaded before the first store so that the
//    loads of a thread are in flight together (the outputs overwrite u, v, w, zu, zv, zw in place).
template <typename T>
__global__ void __launch_bounds__(256) k_f_pstep_swap(Scalars s, DevState<T> d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y * blockDim.y + threadIdx.y;
  int k = blockIdx.z + 1;
  if (i >= s.nx || j >= s.ny || k > s.nz) return;
  Prof<T> P = prof<T>(s);
  const bool fwd = s.forward;
  const T dtmtmp = fwd ? (T)(0.5 * s.dtm) : (T)s.dtm;
  const long long o = lin(s, k, j, i);
  const bool bc = s.use_vd && s.surface_bcs;
  const int kp = (k >= 2) ? k : 2;  // level whose pressure gradient sets zu, zv (level 1 mirrors level 2)
  const long long op = lin(s, kp, j, i);
  const int ie = (i + 1 == s.nx) ? 0 : i + 1, jn = (j + 1 == s.ny) ? 0 : j + 1;
  const T* __restrict__ p = d.p;
  const T p0 = __ldg(p + op);
  const T pe = __ldg(p + lin(s, kp, j, ie));
  const T pn = __ldg(p + lin(s, kp, jn, i));
  const T pz0 = __ldg(p + o);
  const T pz1 = (k >= 2 && k < s.nz) ? __ldg(p + o + s.plane) : (T)0;
  const T zun = __ldg(d.zu_n + op), zvn = __ldg(d.zv_n + op), zwn = __ldg(d.zw_n + o);
  const T u0 = d.u[o], v0 = d.v[o], w0 = d.w[o], zu0 = d.zu[o], zv0 = d.zv[o], zw0 = d.zw[o];
  // u, v as stepfields leaves them (the frame velocity of the stepping added), then moved into the
  // frame of the pressure-terms group by the Galilean transformation
  const T ugp = (T)s.ugal_p, vgp = (T)s.vgal_p;
  T ua = (T)s.ugal + u0, va = (T)s.vgal + v0, zua = zun, zva = zvn;
  if (s.galilean) {
    ua = ua - ugp;
    va = va - vgp;
    zua = zua - ugp;
    zva = zva - vgp;
  }
  T zu_p = zua + (T)2.0 * (T)s.cx * dtmtmp * (p0 - pe);
  T zv_p = zva + (T)2.0 * (T)s.cy * dtmtmp * (p0 - pn);
  if (k == 1) {
    if (bc) {
      zu_p = -zu_p - (T)2.0 * ugp;
      zv_p = -zv_p - (T)2.0 * vgp;
    }
  }
  T zw_p = zwn;
  if (k >= 2 && k < s.nz) zw_p = zw_p + (T)2.0 * P(P_RDZN, k + 1) * dtmtmp * (pz0 - pz1);
  T nu, nzu, nv, nzv, nw, nzw;
  if (fwd) {
    T ev = ua + zu_p;
    nu = ev * (T)1.0 + ua * (T)-1.0;
    nzu = ev - nu;
    ev = va + zv_p;
    nv = ev * (T)1.0 + va * (T)-1.0;
    nzv = ev - nv;
    ev = w0 + zw_p;
    nw = ev * (T)1.0 + w0 * (T)-1.0;
    nzw = ev - nw;
  } else {
    // savu = zu + ugal of the stepping (stepfields.F90:609-610)
    const T c1 = (T)(1.0 - 2.0 * s.tsmth), c2 = (T)s.tsmth;
    nu = zu_p;
    nzu = c1 * ua + c2 * (zu_p + (zu0 + (T)s.ugal) - ugp);
    nv = zv_p;
    nzv = c1 * va + c2 * (zv_p + (zv0 + (T)s.vgal) - vgp);
    nw = zw_p;
    nzw = c1 * w0 + c2 * (zw_p + (zw0 + (T)0.0));
  }
  d.u[o] = nu;
  d.zu[o] = nzu;
  d.v[o] = nv;
  d.zv[o] = nzv;
  d.w[o] = nw;
  d.zw[o] = nzw;
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
    case MGPU_C_TH_ADVECTION:
      if (s.th_baroclinic) k_c_th_advection<T><<<pt_grid(s, s.nz - 1), b, 0, st>>>(s, d);
      else nl = 0;
      break;
    case MGPU_C_VISCOSITY: k_c_viscosity<T><<<pt_grid(s, s.nz - 1), b, 0, st>>>(s, d); break;
    case MGPU_C_CORIOLIS: k_c_coriolis<T><<<pt_grid(s, s.nz - 1), b, 0, st>>>(s, d); break;
    case MGPU_C_BUOYANCY: k_c_buoyancy<T><<<pt_grid(s, s.nz - 2), b, 0, st>>>(s, d); break;
    case MGPU_C_SET_CONSISTENT_LOWBC: k_c_set_consistent_lowbc<T><<<gcol, b, 0, st>>>(s, d); break;
    case MGPU_C_DAMPING: if (s.damping) k_c_damping<T><<<pt_grid(s, s.nz), b, 0, st>>>(s, d); break;
    case MGPU_C_FORCING: if (s.subs_th || s.subs_q) k_c_forcing<T><<<pt_grid(s, s.nz), b, 0, st>>>(s, d); break;
    case MGPU_C_SIMPLECLOUD:
      if (!s.simplecloud) return MGPU_ERR_UNSUPPORTED;
      k_c_simplecloud<T><<<pt_grid(s, s.nz - 1), b, 0, st>>>(s, d);
      break;
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

// Number of level chunks for a grid of `tiles` tiles: the count (chunks of at least 8 levels) whose
// CTAs fill the resident slots most evenly; each extra chunk costs a few staged levels, weighed
// by `per_chunk` against the fill.  The scalar kernel takes a smaller weight: its CTAs vary in
// duration with the limiter's path, so more and shorter chunks balance the SMs better, and
// staging is a small part of its level.
static inline int choose_level_chunks(int tiles, int slots, int levels, double per_chunk = 0.01) {
  int best = 1;
  double best_score = -1.0;
  for (int n = 1; n <= 16 && levels / n >= 8; ++n) {
    const long long ctas = (long long)tiles * n;
    const long long waves = (ctas + slots - 1) / slots;
    const double score = (double)ctas / (double)(waves * slots) - per_chunk * n;
    if (score > best_score + 1e-9) { best_score = score; best = n; }
  }
  return best;
}

// the TVD advection of flow component DIM on the centred step, into src (one launch)
template <typename T, int DIM>
static int launch_flow_tvd(const Scalars& s, DevState<T>& d, T* src, int tiles, int nsm, int levels,
                           cudaStream_t st) {
  const size_t smem = tiled::flow_smem<T, DIM>();
  static int occ = 0;
  if (!occ) {
    cudaFuncSetAttribute(k_f_flow_tvd_tiled<T, DIM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(k_f_flow_tvd_tiled<T, DIM>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_f_flow_tvd_tiled<T, DIM>, tiled::NT, smem);
    if (occ < 1) occ = 1;
  }
  const int nc = s.level_chunks > 0 ? s.level_chunks : choose_level_chunks(tiles, occ * nsm, levels);
  const int kc = (levels + nc - 1) / nc;
  dim3 grid(s.nx / tiled::TX, s.ny / tiled::TY, (levels + kc - 1) / kc);
  k_f_flow_tvd_tiled<T, DIM><<<grid, dim3(tiled::TX, tiled::TY, 1), smem, st>>>(s, d, kc, src);
  return 1;
}

// the moist scalar step of theta and two q fields (one launch)
template <typename T>
static int launch_moist(const Scalars& s, DevState<T>& d, int tiles, int nsm, int levels, cudaStream_t st) {
  const size_t smem = tiled::moist_smem<T>();
  static int occ = 0;
  if (!occ) {
    cudaFuncSetAttribute(k_f_moist_tiled<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(k_f_moist_tiled<T>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_f_moist_tiled<T>, tiled::NT, smem);
    if (occ < 1) occ = 1;
  }
  const int nc = s.level_chunks > 0 ? s.level_chunks : choose_level_chunks(tiles, occ * nsm, levels);
  const int kc = (levels + nc - 1) / nc;
  dim3 grid(s.nx / tiled::TX, s.ny / tiled::TY, (levels + kc - 1) / kc);
  k_f_moist_tiled<T><<<grid, dim3(tiled::TX, tiled::TY, 1), smem, st>>>(s, d, kc);
  return 1;
}

// returns the number of kernels launched; `mid` (may be null) is recorded before the momentum kernel
// returns the number of kernels launched
template <typename T>
int launch_fused_subgrid(const Scalars& s, DevState<T>& d, cudaStream_t st) {
  const bool tiled_ok = !s.point_dynamics && (s.nx % tiled::TX) == 0 &&
                        (s.ny % tiled::TY) == 0 && s.nz >= 4;
  if (!tiled_ok) {
    k_f_subgrid<T><<<pt_grid(s, s.nz), pt_block(), 0, st>>>(s, d);
    return 1;
  }
  const size_t smem = tiled::smag_smem<T>();
  static int occ = 0, nsm = 0;
  if (!nsm) {
    cudaFuncSetAttribute(k_f_smag_tiled<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(k_f_smag_tiled<T>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_f_smag_tiled<T>, tiled::NT, smem);
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (occ < 1) occ = 1;
    if (nsm < 1) nsm = 1;
  }
  k_c_lower_bc<T><<<dim3((s.nx + 31) / 32, (s.ny + 7) / 8, 1), pt_block(), 0, st>>>(s, d);
  const int tiles = (s.nx / tiled::TX) * (s.ny / tiled::TY), levels = s.nz - 2;
  const int nc = s.level_chunks > 0 ? s.level_chunks : choose_level_chunks(tiles, occ * nsm, levels);
  const int kc = (levels + nc - 1) / nc;
  dim3 grid(s.nx / tiled::TX, s.ny / tiled::TY, (levels + kc - 1) / kc);
  k_f_smag_tiled<T><<<grid, dim3(tiled::TX, tiled::TY, 1), smem, st>>>(s, d, kc);
  return 2;
}
template <typename T>
int launch_fused_dynamics(const Scalars& s, DevState<T>& d, cudaStream_t st, cudaEvent_t mid) {
  // the tiled kernels cover centred dry steps; the first (forward) step and moist runs use the
  // point kernel
  const bool moist = s.nq > 0;
  const bool tiled_ok = !s.forward && !s.point_dynamics && (s.nx % tiled::TX) == 0 && (s.ny % tiled::TY) == 0 &&
                        s.nz >= 4 && (!moist || (d.sth && d.sq[s.nq - 1])) && (!s.tvd_flow || (d.su && d.sv && d.sw));
  if (!tiled_ok) {
    k_f_dynamics<T><<<pt_grid(s, s.nz), pt_block(), 0, st>>>(s, d);
    if (mid) cudaEventRecord(mid, st);
    return 1;
  }
  const size_t sm_m = tiled::momentum_smem<T>(), sm_s = tiled::scalar_smem<T>();
  static int occ_m = 0, occ_s = 0, nsm = 0;
  if (!nsm) {
    cudaFuncSetAttribute(k_f_momentum_tiled<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_m);
    cudaFuncSetAttribute(k_f_momentum_tiled<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_m);
    cudaFuncSetAttribute(k_f_scalar_tiled<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_s);
    cudaFuncSetAttribute(k_f_momentum_tiled<T, false>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    cudaFuncSetAttribute(k_f_momentum_tiled<T, true>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    cudaFuncSetAttribute(k_f_scalar_tiled<T>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_m, k_f_momentum_tiled<T, false>, tiled::NT, sm_m);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_s, k_f_scalar_tiled<T>, tiled::NT, sm_s);
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (occ_m < 1) occ_m = 1;
    if (occ_s < 1) occ_s = 1;
    if (nsm < 1) nsm = 1;
  }
  const int tiles = (s.nx / tiled::TX) * (s.ny / tiled::TY), levels = s.nz - 1;
  const int nc_s = s.level_chunks > 0 ? s.level_chunks : choose_level_chunks(tiles, occ_s * nsm, levels, 0.002);
  const int nc_m = s.level_chunks > 0 ? s.level_chunks : choose_level_chunks(tiles, occ_m * nsm, levels);
  const int kc_s = (levels + nc_s - 1) / nc_s, kc_m = (levels + nc_m - 1) / nc_m;
  dim3 block(tiled::TX, tiled::TY, 1);
  dim3 grid_s(s.nx / tiled::TX, s.ny / tiled::TY, (levels + kc_s - 1) / kc_s);
  dim3 grid_m(s.nx / tiled::TX, s.ny / tiled::TY, (levels + kc_m - 1) / kc_m);
  int nscal = moist ? s.nq + 2 : 1;  // launches of the scalar part
  if (!moist) {
    k_f_scalar_tiled<T><<<grid_s, block, sm_s, st>>>(s, d, kc_s, ScalarJob<T>{d.th, d.zth, d.th_n, d.zth_n, nullptr, 0, 2});
  } else if (s.nq == 2) {
    // theta, vapour and liquid in one pass, sources, cloud and stepping included
    nscal = launch_moist<T>(s, d, tiles, nsm, levels, st);
  } else {
    // one launch per scalar writing its source, then saturation adjustment and stepping
    k_f_scalar_tiled<T><<<grid_s, block, sm_s, st>>>(s, d, kc_s, ScalarJob<T>{d.th, d.zth, nullptr, nullptr, d.sth, 0, 2});
    for (int n = 0; n < s.nq; ++n)
      k_f_scalar_tiled<T><<<grid_s, block, sm_s, st>>>(s, d, kc_s, ScalarJob<T>{d.q[n], d.zq[n], nullptr, nullptr, d.sq[n], 1, 3 + n});
    k_f_cloud_step<T><<<pt_grid(s, s.nz), pt_block(), 0, st>>>(s, d);
  }
  if (mid) cudaEventRecord(mid, st);
  int flow = 0;
  if (s.tvd_flow) {
    flow += launch_flow_tvd<T, 0>(s, d, d.su, tiles, nsm, levels, st);
    flow += launch_flow_tvd<T, 1>(s, d, d.sv, tiles, nsm, levels, st);
    flow += launch_flow_tvd<T, 2>(s, d, d.sw, tiles, nsm, levels, st);
  }
  if (s.tvd_flow) k_f_momentum_tiled<T, true><<<grid_m, block, sm_m, st>>>(s, d, kc_m);
  else k_f_momentum_tiled<T, false><<<grid_m, block, sm_m, st>>>(s, d, kc_m);
  return nscal + 1 + flow;
}
template <typename T>
void launch_fused_pressure_source(const Scalars& s, DevState<T>& d, cudaStream_t st) {
  k_f_pressure_source<T><<<pt_grid(s, s.nz), pt_block(), 0, st>>>(s, d);
}
template <typename T>
void launch_fused_pstep_swap(const Scalars& s, DevState<T>& d, cudaStream_t st) {
  k_f_pstep_swap<T><<<pt_grid(s, s.nz), pt_block(), 0, st>>>(s, d);
}

}  // namespace KVARIANT
}  // namespace mgpu
