// Tangent-linear and adjoint passes of the dry FP64 timestep.
//
// The fused step is five passes (subgrid, dynamics, pressure source, pressure solve, pstep +
// swap_smooth).  Each pass except the solve is a pointwise map of a stencil of input arrays,
// written here once as an evaluation function templated on its number type, on the same device
// functions the forward kernels run:
//   * the tangent-linear kernels evaluate it with ad::Dual, reading value and tangent arrays;
//   * the adjoint kernels evaluate it with ad::TV on a per-thread tape whose leaves are the
//     input reads, seed the outputs with their adjoints, sweep the tape backwards and add each
//     leaf's adjoint into the adjoint array of its input (atomicAdd, FP64).
// TVD faces are taped one at a time: the divergence is taped with the six face values as leaves,
// then each face is re-evaluated on its own tape and seeded with its adjoint.  Limiter branches
// are those the forward evaluation takes.  The pressure solve is linear; its adjoint is the same
// FFT pipeline with the transposed tridiagonal (fft_solve(..., transpose=true)).
#include <cstdio>

#include "ad.cuh"
#include "dycore.h"
#include "dycore_device.cuh"

namespace mgpu {
namespace tlad {

using ad::Dual;
using ad::Tape;
using ad::TV;

__device__ __forceinline__ Geo geo(const Scalars& s) { return Geo{s.nx, s.ny, s.nz, s.plane}; }

// ---- accessors ---------------------------------------------------------------------------
struct DView {
  const double* v;
  const double* t;
  Geo g;
  __device__ __forceinline__ Dual operator()(int k, int j, int i) const {
    const long long o = g.at(k, j, i);
    return Dual(v[o], t[o]);
  }
};
struct DProf {
  const double* base;
  int stride;
  const double* drsq;  // d rneutml_sq / d rmlmax per level, or null
  double dpar;         // tangent of rmlmax
  __device__ __forceinline__ Dual operator()(int id, int k) const {
    const double val = base[id * stride + k];
    return (drsq && id == P_RNEUTML_SQ) ? Dual(val, drsq[k] * dpar) : Dual(val);
  }
};
struct TView {
  const double* v;
  Geo g;
  int field;
  Tape* t;
  __device__ __forceinline__ TV operator()(int k, int j, int i) const {
    const long long o = g.at(k, j, i);
    return TV(v[o], t->leaf(field, o), t);
  }
};
struct TProf {
  const double* base;
  int stride;
  Tape* t;
  __device__ __forceinline__ TV operator()(int id, int k) const {
    const double val = base[id * stride + k];
    if (id == P_RNEUTML_SQ) return TV(val, t->leaf(F_PROF, k), t);
    return TV(val);
  }
};
struct VView {  // plain values
  const double* v;
  Geo g;
  __device__ __forceinline__ double operator()(int k, int j, int i) const { return v[g.at(k, j, i)]; }
};

// ---- evaluation functions (mirror k_f_subgrid, k_f_dynamics, k_f_pressure_source and
//      k_f_pstep_swap) --------------------------------------------------------------------
template <class X, class A, class PA>
__device__ void eval_subgrid(const Scalars& s, const PA& P, const A& u, const A& v, const A& w, const A& th,
                             const A& zu, const A& zv, const A& zw, const A& zth, int k, int j, int i, X& vis,
                             X& diff, X& th1) {
  const bool fwd = s.forward;
  if (k == 1) {
    X qv1;
    lower_bc_column<X>(s, P, zu, fwd ? u : zu, fwd ? v : zv, fwd ? th : zth, (const A*)nullptr, j, i, vis, diff, th1,
                       qv1);
    return;
  }
  if (k == s.nz) {
    vis = X(0.0);
    diff = X(0.0);
    return;
  }
  smagorinsky_point<X>(s, P, fwd ? u : zu, fwd ? v : zv, fwd ? w : zw, th, fwd ? th : zth, (const A*)nullptr,
                       (const A*)nullptr, k, j, i, vis, diff);
}

template <class X, class A, class PA>
__device__ void eval_momentum(const Scalars& s, const PA& P, const A& u, const A& v, const A& w, const A& th,
                              const A& zu, const A& zv, const A& zw, const A& vis, int k, int j, int i, X& zun,
                              X& zvn, X& zwn) {
  const bool fwd = s.forward;
  X su(0.0), sv(0.0), sw(0.0);
  if (k >= 2) {
    pw_point<X>(s, P, u, v, w, k, j, i, su, sv, sw);
    if (s.use_vd) {
      X du, dv, dw;
      viscosity_point<X>(s, P, fwd ? u : zu, fwd ? v : zv, fwd ? w : zw, zu, vis, k, j, i, du, dv, dw);
      su = su + du;
      sv = sv + dv;
      if (k < s.nz) sw = sw + dw;
    }
    if (s.coriolis) coriolis_point<X>(s, P, u, v, k, j, i, su, sv);
    if (k < s.nz && !s.passive_th) sw = sw + (X(0.5) * P(P_BUOY_CO, k)) * (th(k, j, i) + th(k + 1, j, i));
  }
  const X dtm(s.dtm), dtm_x2(2.0 * s.dtm);
  if (fwd) {
    zun = (X(s.ugal) + u(k, j, i)) + dtm * su;
    zvn = (X(s.vgal) + v(k, j, i)) + dtm * sv;
    zwn = w(k, j, i) + dtm * sw;
  } else {
    zun = X(s.ugal) + zu(k, j, i) + dtm_x2 * su;
    zvn = X(s.vgal) + zv(k, j, i) + dtm_x2 * sv;
    zwn = X(0.0) + zw(k, j, i) + dtm_x2 * sw;
  }
}

// the six TVD faces of cell (k, j, i): x-, x+, y-, y+, z-, z+ (tvd_point)
template <class X, class A, class PA>
__device__ X eval_face(const Scalars& s, const PA& P, const A& u, const A& v, const A& w, const A& zf, int m, int k,
                       int j, int i) {
  const X dt(s.dtm * 2.0);
  switch (m) {
    case 0: return tvd_face_x<X>(s, P, u, v, w, zf, dt, k, j, i - 1);
    case 1: return tvd_face_x<X>(s, P, u, v, w, zf, dt, k, j, i);
    case 2: return tvd_face_y<X>(s, P, u, v, w, zf, dt, k, j - 1, i);
    case 3: return tvd_face_y<X>(s, P, u, v, w, zf, dt, k, j, i);
    case 4: return k == 2 ? X(0.0) : tvd_face_z<X>(s, P, u, v, w, zf, dt, k - 1, j, i);
    default: return k < s.nz ? tvd_face_z<X>(s, P, u, v, w, zf, dt, k, j, i) : X(0.0);
  }
}

template <class X, class A, class PA>
__device__ void eval_scalar(const Scalars& s, const PA& P, const A& u, const A& v, const A& w, const A& th,
                            const A& zth, const A& diff, const X (&f)[6], int k, int j, int i, X& thn, X& zthn) {
  const bool fwd = s.forward;
  X src(0.0);
  if (k >= 2) {
    src = tvd_source<X>(s, P, u, v, w, f[0], f[1], f[2], f[3], f[4], f[5], k, j, i, X(0.0));
    if (s.use_vd) src = src + diffusion_point<X>(s, P, zth, diff, k, j, i);
  }
  const X fv = th(k, j, i), zv = zth(k, j, i);
  if (fwd) {
    const X zn = fv + X(s.dtm) * src;
    const X ev = fv + zn;
    const X nf = ev * X(1.0) + fv * X(-1.0);
    thn = nf;
    zthn = ev - nf;
  } else {
    const X sm = X(1.0 - 2.0 * s.tsmth) * fv + X(s.tsmth) * zv;
    const X zn = X(0.0) + zv + X(2.0 * s.dtm) * src;
    zthn = sm + X(s.tsmth) * zn;
    thn = zn;
  }
}

template <class X, class A, class PA>
__device__ X eval_psrc(const Scalars& s, const PA& P, const A& zun, const A& zvn, const A& zwn, int k, int j, int i) {
  if (k == 1) return X(0.0);
  const X timec = s.forward ? X(1.0 / s.dtm) : X(1.0 / (2.0 * s.dtm));
  X pp(0.0);
  pp = pp + X(s.cx) * (zun(k, j, i) - zun(k, j, i - 1));
  pp = pp + X(s.cy) * (zvn(k, j, i) - zvn(k, j - 1, i));
  pp = pp + X(4.0) * (P(P_TZC2, k) * zwn(k, j, i) - P(P_TZC1, k) * zwn(k - 1, j, i));
  return pp * timec;
}

template <class X, class A, class PA>
__device__ void eval_pstep(const Scalars& s, const PA& P, const A& p, const A& u, const A& v, const A& w, const A& zu,
                           const A& zv, const A& zw, const A& zun_a, const A& zvn_a, const A& zwn_a, int k, int j,
                           int i, X (&out)[6]) {
  const bool fwd = s.forward;
  const X dtmtmp = fwd ? X(0.5 * s.dtm) : X(s.dtm);
  const bool bc = s.use_vd && s.surface_bcs;
  const int kp = (k >= 2) ? k : 2;
  const X p0 = p(kp, j, i), pe = p(kp, j, i + 1), pn = p(kp, j + 1, i);
  const X zun = zun_a(kp, j, i), zvn = zvn_a(kp, j, i), zwn = zwn_a(k, j, i);
  const X u0 = u(k, j, i), v0 = v(k, j, i), w0 = w(k, j, i), zu0 = zu(k, j, i), zv0 = zv(k, j, i), zw0 = zw(k, j, i);
  X zu_p = zun + X(2.0) * X(s.cx) * dtmtmp * (p0 - pe);
  X zv_p = zvn + X(2.0) * X(s.cy) * dtmtmp * (p0 - pn);
  if (k == 1 && bc) {
    zu_p = -zu_p - X(2.0) * X(s.ugal);
    zv_p = -zv_p - X(2.0) * X(s.vgal);
  }
  X zw_p = zwn;
  if (k >= 2 && k < s.nz) zw_p = zw_p + X(2.0) * P(P_RDZN, k + 1) * dtmtmp * (p(k, j, i) - p(k + 1, j, i));
  if (fwd) {
    X ev = (X(s.ugal) + u0) + zu_p;
    out[0] = ev * X(1.0) + (X(s.ugal) + u0) * X(-1.0);
    out[1] = ev - out[0];
    ev = (X(s.vgal) + v0) + zv_p;
    out[2] = ev * X(1.0) + (X(s.vgal) + v0) * X(-1.0);
    out[3] = ev - out[2];
    ev = w0 + zw_p;
    out[4] = ev * X(1.0) + w0 * X(-1.0);
    out[5] = ev - out[4];
  } else {
    const X c1(1.0 - 2.0 * s.tsmth), c2(s.tsmth);
    out[0] = zu_p;
    out[1] = c1 * (X(s.ugal) + u0) + c2 * (zu_p + (zu0 + X(s.ugal)) - X(s.ugal));
    out[2] = zv_p;
    out[3] = c1 * (X(s.vgal) + v0) + c2 * (zv_p + (zv0 + X(s.vgal)) - X(s.vgal));
    out[4] = zw_p;
    out[5] = c1 * w0 + c2 * (zw_p + (zw0 + X(0.0)));
  }
}

// ---- tangent-linear kernels --------------------------------------------------------------
struct TlArgs {
  DevState<double> d;  // values
  DevState<double> t;  // tangents, same roles
  const double* drsq;
  double dpar;
};

#define POINT_INDEX                                       \
  const int i = blockIdx.x * blockDim.x + threadIdx.x;    \
  const int j = blockIdx.y * blockDim.y + threadIdx.y;    \
  const int k = blockIdx.z + 1;                           \
  if (i >= s.nx || j >= s.ny || k > s.nz) return;         \
  const long long o = (long long)(k - 1) * s.plane + (long long)j * s.nx + i;

__global__ void __launch_bounds__(128) k_tl_subgrid(Scalars s, TlArgs a) {
  POINT_INDEX
  const Geo g = geo(s);
  const DProf P{s.prof, s.nz + 2, a.drsq, a.dpar};
  const DevState<double>& d = a.d;
  const DevState<double>& t = a.t;
  Dual vis, diff, th1;
  eval_subgrid<Dual>(s, P, DView{d.u, t.u, g}, DView{d.v, t.v, g}, DView{d.w, t.w, g}, DView{d.th, t.th, g},
                     DView{d.zu, t.zu, g}, DView{d.zv, t.zv, g}, DView{d.zw, t.zw, g}, DView{d.zth, t.zth, g}, k, j, i,
                     vis, diff, th1);
  t.vis[o] = vis.d;
  t.diff[o] = diff.d;
  if (k == 1) (s.forward ? t.th : t.zth)[o] = th1.d;
}

__global__ void __launch_bounds__(128) k_tl_dynamics(Scalars s, TlArgs a) {
  POINT_INDEX
  const Geo g = geo(s);
  const DProf P{s.prof, s.nz + 2, a.drsq, a.dpar};
  const DevState<double>& d = a.d;
  const DevState<double>& t = a.t;
  const DView u{d.u, t.u, g}, v{d.v, t.v, g}, w{d.w, t.w, g}, th{d.th, t.th, g}, zth{d.zth, t.zth, g};
  Dual zun, zvn, zwn;
  eval_momentum<Dual>(s, P, u, v, w, th, DView{d.zu, t.zu, g}, DView{d.zv, t.zv, g}, DView{d.zw, t.zw, g},
                      DView{d.vis, t.vis, g}, k, j, i, zun, zvn, zwn);
  t.zu_n[o] = zun.d;
  t.zv_n[o] = zvn.d;
  t.zw_n[o] = zwn.d;
  Dual f[6];
  if (k >= 2)
    for (int m = 0; m < 6; ++m) f[m] = eval_face<Dual>(s, P, u, v, w, s.forward ? th : zth, m, k, j, i);
  Dual thn, zthn;
  eval_scalar<Dual>(s, P, u, v, w, th, zth, DView{d.diff, t.diff, g}, f, k, j, i, thn, zthn);
  t.th_n[o] = thn.d;
  t.zth_n[o] = zthn.d;
}

__global__ void __launch_bounds__(128) k_tl_pressure_source(Scalars s, TlArgs a) {
  POINT_INDEX
  const Geo g = geo(s);
  const DProf P{s.prof, s.nz + 2, nullptr, 0.0};
  const Dual p = eval_psrc<Dual>(s, P, DView{a.d.zu_n, a.t.zu_n, g}, DView{a.d.zv_n, a.t.zv_n, g},
                                 DView{a.d.zw_n, a.t.zw_n, g}, k, j, i);
  a.t.p[o] = p.d;
}

__global__ void __launch_bounds__(128) k_tl_pstep_swap(Scalars s, TlArgs a) {
  POINT_INDEX
  const Geo g = geo(s);
  const DProf P{s.prof, s.nz + 2, nullptr, 0.0};
  const DevState<double>& d = a.d;
  const DevState<double>& t = a.t;
  Dual out[6];
  eval_pstep<Dual>(s, P, DView{d.p, t.p, g}, DView{d.u, t.u, g}, DView{d.v, t.v, g}, DView{d.w, t.w, g},
                   DView{d.zu, t.zu, g}, DView{d.zv, t.zv, g}, DView{d.zw, t.zw, g}, DView{d.zu_n, t.zu_n, g},
                   DView{d.zv_n, t.zv_n, g}, DView{d.zw_n, t.zw_n, g}, k, j, i, out);
  // each thread reads its own u..zw tangents only, so the outputs may overwrite them in place
  t.u[o] = out[0].d;
  t.zu[o] = out[1].d;
  t.v[o] = out[2].d;
  t.zv[o] = out[3].d;
  t.w[o] = out[4].d;
  t.zw[o] = out[5].d;
}

// ---- adjoint kernels ---------------------------------------------------------------------
struct AdjArgs {
  DevState<double> d;     // values of the recomputed step (post-subgrid state and intermediates)
  double* tg[F_COUNT];    // adjoint arrays the leaves of each field add into
  const double* seed[8];  // adjoints of the next state: u v w th zu zv zw zth
  int* overflow;
};

// add each leaf's adjoint into its field's adjoint array; face leaves are collected instead
__device__ __forceinline__ void scatter(Tape& tp, double* const* tg, double (*face)) {
  for (int l = 0; l < tp.nleaf; ++l) {
    const double g = tp.adj[tp.lf_node[l]];
    if (g == 0.0) continue;
    const int f = tp.lf_field[l];
    if (f >= F_FACE0) face[f - F_FACE0] += g;
    else atomicAdd(tg[f] + tp.lf_off[l], g);
  }
}
__device__ __forceinline__ void seed(Tape& tp, const TV& x, double g) {
  if (x.id >= 0) tp.adj[x.id] += g;
}

__global__ void __launch_bounds__(128) k_adj_pstep_swap(Scalars s, AdjArgs a) {
  POINT_INDEX
  double sd[6] = {a.seed[0][o], a.seed[4][o], a.seed[1][o], a.seed[5][o], a.seed[2][o], a.seed[6][o]};
  if (sd[0] == 0.0 && sd[1] == 0.0 && sd[2] == 0.0 && sd[3] == 0.0 && sd[4] == 0.0 && sd[5] == 0.0) return;
  Tape tp;
  tp.reset();
  tp.overflow = 0;
  const Geo g = geo(s);
  const TProf P{s.prof, s.nz + 2, &tp};
  const DevState<double>& d = a.d;
  TV out[6];
  eval_pstep<TV>(s, P, TView{d.p, g, F_P, &tp}, TView{d.u, g, F_U, &tp}, TView{d.v, g, F_V, &tp},
                 TView{d.w, g, F_W, &tp}, TView{d.zu, g, F_ZU, &tp}, TView{d.zv, g, F_ZV, &tp},
                 TView{d.zw, g, F_ZW, &tp}, TView{d.zu_n, g, F_ZUN, &tp}, TView{d.zv_n, g, F_ZVN, &tp},
                 TView{d.zw_n, g, F_ZWN, &tp}, k, j, i, out);
  tp.clear_adj();
  for (int q = 0; q < 6; ++q) seed(tp, out[q], sd[q]);
  tp.sweep();
  double face[6] = {};
  scatter(tp, a.tg, face);
  if (tp.overflow) atomicOr(a.overflow, 1);
}

__global__ void __launch_bounds__(128) k_adj_pressure_source(Scalars s, AdjArgs a, const double* pbar) {
  POINT_INDEX
  const double sd = pbar[o];
  if (sd == 0.0 || k == 1) return;
  Tape tp;
  tp.reset();
  tp.overflow = 0;
  const Geo g = geo(s);
  const TProf P{s.prof, s.nz + 2, &tp};
  const DevState<double>& d = a.d;
  const TV p = eval_psrc<TV>(s, P, TView{d.zu_n, g, F_ZUN, &tp}, TView{d.zv_n, g, F_ZVN, &tp},
                             TView{d.zw_n, g, F_ZWN, &tp}, k, j, i);
  tp.clear_adj();
  seed(tp, p, sd);
  tp.sweep();
  double face[6] = {};
  scatter(tp, a.tg, face);
  if (tp.overflow) atomicOr(a.overflow, 1);
}

__global__ void __launch_bounds__(128) k_adj_momentum(Scalars s, AdjArgs a) {
  POINT_INDEX
  const double s0 = a.tg[F_ZUN][o], s1 = a.tg[F_ZVN][o], s2 = a.tg[F_ZWN][o];
  if (s0 == 0.0 && s1 == 0.0 && s2 == 0.0) return;
  Tape tp;
  tp.reset();
  tp.overflow = 0;
  const Geo g = geo(s);
  const TProf P{s.prof, s.nz + 2, &tp};
  const DevState<double>& d = a.d;
  TV zun, zvn, zwn;
  eval_momentum<TV>(s, P, TView{d.u, g, F_U, &tp}, TView{d.v, g, F_V, &tp}, TView{d.w, g, F_W, &tp},
                    TView{d.th, g, F_TH, &tp}, TView{d.zu, g, F_ZU, &tp}, TView{d.zv, g, F_ZV, &tp},
                    TView{d.zw, g, F_ZW, &tp}, TView{d.vis, g, F_VIS, &tp}, k, j, i, zun, zvn, zwn);
  tp.clear_adj();
  seed(tp, zun, s0);
  seed(tp, zvn, s1);
  seed(tp, zwn, s2);
  tp.sweep();
  double face[6] = {};
  scatter(tp, a.tg, face);
  if (tp.overflow) atomicOr(a.overflow, 1);
}

__global__ void __launch_bounds__(128) k_adj_scalar(Scalars s, AdjArgs a) {
  POINT_INDEX
  const double s_th = a.seed[3][o], s_zth = a.seed[7][o];
  if (s_th == 0.0 && s_zth == 0.0) return;
  const Geo g = geo(s);
  const DevState<double>& d = a.d;
  const bool fwd = s.forward;
  // face values
  double fv[6] = {0, 0, 0, 0, 0, 0};
  if (k >= 2) {
    const Prof<double> Pv{s.prof, s.nz + 2};
    const VView u{d.u, g}, v{d.v, g}, w{d.w, g}, zf{fwd ? d.th : d.zth, g};
    for (int m = 0; m < 6; ++m) fv[m] = eval_face<double>(s, Pv, u, v, w, zf, m, k, j, i);
  }
  Tape tp;
  tp.reset();
  tp.overflow = 0;
  const TProf P{s.prof, s.nz + 2, &tp};
  TV f[6];
  for (int m = 0; m < 6; ++m) f[m] = (k >= 2) ? TV(fv[m], tp.leaf(F_FACE0 + m, 0), &tp) : TV(0.0);
  TV thn, zthn;
  eval_scalar<TV>(s, P, TView{d.u, g, F_U, &tp}, TView{d.v, g, F_V, &tp}, TView{d.w, g, F_W, &tp},
                  TView{d.th, g, F_TH, &tp}, TView{d.zth, g, F_ZTH, &tp}, TView{d.diff, g, F_DIFF, &tp}, f, k, j, i,
                  thn, zthn);
  tp.clear_adj();
  seed(tp, thn, s_th);
  seed(tp, zthn, s_zth);
  tp.sweep();
  double face[6] = {0, 0, 0, 0, 0, 0};
  scatter(tp, a.tg, face);
  int ovf = tp.overflow;
  for (int m = 0; m < 6; ++m) {
    if (face[m] == 0.0) continue;
    tp.reset();
    const TProf Pm{s.prof, s.nz + 2, &tp};
    const TV fm = eval_face<TV>(s, Pm, TView{d.u, g, F_U, &tp}, TView{d.v, g, F_V, &tp}, TView{d.w, g, F_W, &tp},
                                TView{fwd ? d.th : d.zth, g, fwd ? F_TH : F_ZTH, &tp}, m, k, j, i);
    tp.clear_adj();
    seed(tp, fm, face[m]);
    tp.sweep();
    double unused[6] = {};
    scatter(tp, a.tg, unused);
    ovf |= tp.overflow;
  }
  if (ovf) atomicOr(a.overflow, 1);
}

// k == 1: lower_bc overwrote th(1) (forward step) or zth(1); its adjoint there is the seed and
// then zero, since the old value is read by nothing
__global__ void __launch_bounds__(128) k_adj_subgrid(Scalars s, AdjArgs a) {
  POINT_INDEX
  const bool fwd = s.forward;
  double* tha_bar = fwd ? a.tg[F_TH] : a.tg[F_ZTH];
  const double s_vis = a.tg[F_VIS][o], s_diff = a.tg[F_DIFF][o];
  const double s_th1 = k == 1 ? tha_bar[o] : 0.0;
  if (k == 1) tha_bar[o] = 0.0;
  if (s_vis == 0.0 && s_diff == 0.0 && s_th1 == 0.0) return;
  Tape tp;
  tp.reset();
  tp.overflow = 0;
  const Geo g = geo(s);
  const TProf P{s.prof, s.nz + 2, &tp};
  const DevState<double>& d = a.d;
  TV vis, diff, th1;
  eval_subgrid<TV>(s, P, TView{d.u, g, F_U, &tp}, TView{d.v, g, F_V, &tp}, TView{d.w, g, F_W, &tp},
                   TView{d.th, g, F_TH, &tp}, TView{d.zu, g, F_ZU, &tp}, TView{d.zv, g, F_ZV, &tp},
                   TView{d.zw, g, F_ZW, &tp}, TView{d.zth, g, F_ZTH, &tp}, k, j, i, vis, diff, th1);
  tp.clear_adj();
  seed(tp, vis, s_vis);
  seed(tp, diff, s_diff);
  if (k == 1) seed(tp, th1, s_th1);
  tp.sweep();
  double face[6] = {};
  scatter(tp, a.tg, face);
  if (tp.overflow) atomicOr(a.overflow, 1);
}

}  // namespace tlad

// ---- launchers ---------------------------------------------------------------------------
static dim3 ad_grid(const Scalars& s) { return dim3((s.nx + 31) / 32, (s.ny + 3) / 4, s.nz); }
static dim3 ad_block() { return dim3(32, 4, 1); }

void adj_lower_bc(const Scalars& s, const DevState<double>& d, double* const* tg, const double* const* seed,
                  int* overflow, cudaStream_t st) {
  tlad::AdjArgs a;
  a.d = d;
  for (int f = 0; f < F_COUNT; ++f) a.tg[f] = tg[f];
  for (int q = 0; q < 8; ++q) a.seed[q] = seed[q];
  a.overflow = overflow;
  dim3 grid = ad_grid(s);
  grid.z = 1;  // k = 1 only
  tlad::k_adj_subgrid<<<grid, ad_block(), 0, st>>>(s, a);
}

// ---- branch decisions of two states (a gradient-check diagnostic) -------------------------
// For every point: the branch codes of the theta TVD faces x+1/2, y+1/2 and z+1/2 (upwind side,
// the smooth-region early return, the limiter's choice among fncs, fnfs, fnrefs and 1, the signs
// that pick the gradient-term stencils) and the Smagorinsky regime of the dry Richardson number
// (ri <= 0, 0 < ri < ric, ri >= ric), evaluated on the state each model would step next.  The
// kernel counts the decisions that differ between the two models.
__device__ __forceinline__ unsigned smag_regime(const Scalars& s, const Prof<double>& P, const View<double>& U,
                                                const View<double>& V, const View<double>& W, const View<double>& TH,
                                                int k, int j, int i) {
  const double ssq = half_squared_strain<double>(s, P, U, V, W, k, j, i);
  const double ri = (P(P_DTHREF, k) + TH(k + 1, j, i) - TH(k, j, i)) * P(P_RDZN, k + 1) * P(P_BUOY_CO, k) / ssq;
  return ri <= 0.0 ? 0u : (ri < s.ric ? 1u : 2u);
}

__global__ void k_branch_flips(Scalars s, DevState<double> a, DevState<double> b, unsigned long long* count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z + 2;
  unsigned n = 0;
  if (i < s.nx && j < s.ny && k <= s.nz) {
    const Geo g{s.nx, s.ny, s.nz, s.plane};
    Prof<double> P;
    P.base = s.prof;
    P.stride = s.nz + 2;
    const double dt = s.dtm * 2.0;
    unsigned code[2][4];
    const DevState<double>* st[2] = {&a, &b};
    for (int q = 0; q < 2; ++q) {
      const DevState<double>& d = *st[q];
      const View<double> U{d.u, g}, V{d.v, g}, W{d.w, g}, ZF{s.forward ? d.th : d.zth, g};
      const CflInline<double, View<double>, Prof<double>, TvdMetricScalar> cfl{s, P, U, V, W};
      for (int c = 0; c < 4; ++c) code[q][c] = 0;
      tvd_face_x_g<double, View<double>, View<double>, Prof<double>, TvdMetricScalar>(s, P, U, V, W, ZF, dt, k, j, i,
                                                                                     cfl, BitRec{&code[q][0]});
      tvd_face_y_g<double, View<double>, View<double>, Prof<double>, TvdMetricScalar>(s, P, U, V, W, ZF, dt, k, j, i,
                                                                                     cfl, BitRec{&code[q][1]});
      if (k < s.nz) {
        tvd_face_z_g<double, View<double>, View<double>, Prof<double>, TvdMetricScalar>(s, P, U, V, W, ZF, dt, k, j, i,
                                                                                       cfl, BitRec{&code[q][2]});
        const View<double> SU{s.forward ? d.u : d.zu, g}, SV{s.forward ? d.v : d.zv, g}, SW{s.forward ? d.w : d.zw, g};
        code[q][3] = smag_regime(s, P, SU, SV, SW, View<double>{d.th, g}, k, j, i);
      }
    }
    for (int c = 0; c < 4; ++c) n += code[0][c] != code[1][c] ? 1u : 0u;
  }
  // one atomic per warp
  for (int off = 16; off > 0; off >>= 1) n += __shfl_down_sync(0xffffffffu, n, off);
  if ((threadIdx.x & 31) == 0 && n) atomicAdd(count, (unsigned long long)n);
}

void branch_flips(const Scalars& s, const DevState<double>& a, const DevState<double>& b, unsigned long long* count,
                  cudaStream_t st) {
  dim3 block(32, 4, 1), grid((s.nx + 31) / 32, (s.ny + 3) / 4, s.nz - 1);
  k_branch_flips<<<grid, block, 0, st>>>(s, a, b, count);
}

void tl_pass(int pass, const Scalars& s, const DevState<double>& d, const DevState<double>& t, const double* drsq,
             double dpar, cudaStream_t st) {
  tlad::TlArgs a{d, t, drsq, dpar};
  switch (pass) {
    case 0: tlad::k_tl_subgrid<<<ad_grid(s), ad_block(), 0, st>>>(s, a); break;
    case 1: tlad::k_tl_dynamics<<<ad_grid(s), ad_block(), 0, st>>>(s, a); break;
    case 2: tlad::k_tl_pressure_source<<<ad_grid(s), ad_block(), 0, st>>>(s, a); break;
    default: tlad::k_tl_pstep_swap<<<ad_grid(s), ad_block(), 0, st>>>(s, a); break;
  }
}

void adj_pass(int pass, const Scalars& s, const DevState<double>& d, double* const* tg, const double* const* seed,
              int* overflow, cudaStream_t st) {
  tlad::AdjArgs a;
  a.d = d;
  for (int f = 0; f < F_COUNT; ++f) a.tg[f] = tg[f];
  for (int q = 0; q < 8; ++q) a.seed[q] = seed[q];
  a.overflow = overflow;
  switch (pass) {
    case 0: tlad::k_adj_subgrid<<<ad_grid(s), ad_block(), 0, st>>>(s, a); break;
    case 1: tlad::k_adj_momentum<<<ad_grid(s), ad_block(), 0, st>>>(s, a); break;
    case 2: tlad::k_adj_scalar<<<ad_grid(s), ad_block(), 0, st>>>(s, a); break;
    case 3: tlad::k_adj_pressure_source<<<ad_grid(s), ad_block(), 0, st>>>(s, a, tg[F_P]); break;
    default: tlad::k_adj_pstep_swap<<<ad_grid(s), ad_block(), 0, st>>>(s, a); break;
  }
}

}  // namespace mgpu
