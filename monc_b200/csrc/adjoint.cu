// Hand-written adjoints of the dry FP64 timestep's passes.
//
// Each kernel is the transpose of one pass of the fused step, derived statement by statement
// from the forward device functions (dycore_device.cuh) the pass runs:
//   * pressure step + swap_smooth and pressure source are linear with constant coefficients;
//     their adjoints are written in gather form: each thread forms the adjoint of its own inputs
//     from the output adjoints of the points that read them, with no atomics;
//   * momentum (PW advection, viscosity, Coriolis, buoyancy, stepping) is a bilinear stencil; its
//     adjoint is written in scatter form: each thread evaluates the partial derivatives of its
//     outputs in registers, sums the contributions that land on the same input point, and adds
//     them into the input adjoints with FP64 atomics.
// The adjoint arrays and seeds follow adj_pass (tlad.cu); the operator-overloading tape kernels
// there evaluate the same transposes and are the check these kernels are tested against.
#include "dycore.h"
#include "dycore_device.cuh"

namespace mgpu {
namespace hadj {

struct Args {
  DevState<double> d;     // values of the recomputed step
  double* tg[F_COUNT];    // adjoint arrays added into
  const double* seed[8];  // adjoints of the next state: u v w th zu zv zw zth
};

__device__ __forceinline__ Geo geo(const Scalars& s) { return Geo{s.nx, s.ny, s.nz, s.plane}; }

// scatter of one contribution into the adjoint of field f at (k, j, i)
struct Scatter {
  double* const* tg;
  Geo g;
  __device__ __forceinline__ void operator()(int f, int k, int j, int i, double v) const {
    atomicAdd(tg[f] + g.at(k, j, i), v);
  }
};

#define HADJ_POINT_INDEX                                  \
  const int i = blockIdx.x * blockDim.x + threadIdx.x;    \
  const int j = blockIdx.y * blockDim.y + threadIdx.y;    \
  const int k = blockIdx.z + 1;                           \
  if (i >= s.nx || j >= s.ny || k > s.nz) return;         \
  const long long o = (long long)(k - 1) * s.plane + (long long)j * s.nx + i;

// ---- pressure step + swap_smooth (eval_pstep / k_f_pstep_swap) -------------------------------
// Outputs of point n: u, zu, v, zv, w, zw of the next state.  The adjoint of the stepped
// velocities before swap_smooth:
//   forward step  : zu_p -> u (the new u), u -> zu
//   centred step  : zu_p -> u and tsmth zu_p -> zu, u -> (1 - 2 tsmth) zu, zu -> tsmth zu
// and at k = 1 with surface boundary conditions zu_p enters negated.
struct PstepSeeds {
  const double* const* seed;
  Geo g;
  int nz;
  bool fwd, bc;
  double c2;
  // adjoint of zun + 2 cx dtmtmp (p0 - pe) at (k, j, i) (after the k = 1 sign flip)
  __device__ __forceinline__ double zu_pre(int k, int j, int i) const {
    const long long n = g.at(k, j, i);
    double b = fwd ? seed[0][n] : seed[0][n] + c2 * seed[4][n];
    return (k == 1 && bc) ? -b : b;
  }
  __device__ __forceinline__ double zv_pre(int k, int j, int i) const {
    const long long n = g.at(k, j, i);
    double b = fwd ? seed[1][n] : seed[1][n] + c2 * seed[5][n];
    return (k == 1 && bc) ? -b : b;
  }
  __device__ __forceinline__ double zw_p(int k, int j, int i) const {
    const long long n = g.at(k, j, i);
    return fwd ? seed[2][n] : seed[2][n] + c2 * seed[6][n];
  }
  // the x- and y-pressure-gradient adjoints the points of level k put on p(kp): level 2 also
  // carries level 1's, which reads p and zun at kp = 2
  __device__ __forceinline__ double zu_at(int k, int j, int i) const {
    if (k == 1) return 0.0;
    return k == 2 ? zu_pre(2, j, i) + zu_pre(1, j, i) : zu_pre(k, j, i);
  }
  __device__ __forceinline__ double zv_at(int k, int j, int i) const {
    if (k == 1) return 0.0;
    return k == 2 ? zv_pre(2, j, i) + zv_pre(1, j, i) : zv_pre(k, j, i);
  }
};

__global__ void __launch_bounds__(128) k_hadj_pstep_swap(Scalars s, Args a) {
  HADJ_POINT_INDEX
  const Geo g = geo(s);
  const bool fwd = s.forward;
  const PstepSeeds S{a.seed, g, s.nz, fwd, s.use_vd && s.surface_bcs, s.tsmth};
  const double dtmtmp = fwd ? 0.5 * s.dtm : s.dtm;
  const double cxd = 2.0 * s.cx * dtmtmp, cyd = 2.0 * s.cy * dtmtmp;
  // own state inputs u, v, w (and zu, zv, zw on a centred step)
  const double g1 = a.seed[4][o], g3 = a.seed[5][o], g5 = a.seed[6][o];
  if (fwd) {
    a.tg[F_U][o] += g1;
    a.tg[F_V][o] += g3;
    a.tg[F_W][o] += g5;
  } else {
    const double c1 = 1.0 - 2.0 * s.tsmth, c2 = s.tsmth;
    a.tg[F_U][o] += c1 * g1;
    a.tg[F_ZU][o] += c2 * g1;
    a.tg[F_V][o] += c1 * g3;
    a.tg[F_ZV][o] += c2 * g3;
    a.tg[F_W][o] += c1 * g5;
    a.tg[F_ZW][o] += c2 * g5;
  }
  // zun, zvn (read at kp = max(k, 2)) and zwn (read at k)
  const double zu_k = S.zu_at(k, j, i), zv_k = S.zv_at(k, j, i), zw_k = S.zw_p(k, j, i);
  a.tg[F_ZUN][o] += zu_k;
  a.tg[F_ZVN][o] += zv_k;
  a.tg[F_ZWN][o] += zw_k;
  // p: +cxd at its own point and -cxd at the point west of it (which reads it as pe); the same
  // in y; vertically +cz(k) from level k's w and -cz(k-1) from level k-1's
  double pb = cxd * (zu_k - S.zu_at(k, j, i - 1)) + cyd * (zv_k - S.zv_at(k, j - 1, i));
  if (k >= 2 && k < s.nz) pb += 2.0 * s.prof[P_RDZN * (s.nz + 2) + k + 1] * dtmtmp * zw_k;
  if (k - 1 >= 2 && k - 1 < s.nz) pb -= 2.0 * s.prof[P_RDZN * (s.nz + 2) + k] * dtmtmp * S.zw_p(k - 1, j, i);
  a.tg[F_P][o] += pb;
}

// ---- pressure source (eval_psrc / k_f_pressure_source) ----------------------------------------
//   p(k) = timec (cx (zun(i) - zun(i-1)) + cy (zvn(j) - zvn(j-1)) + 4 (tzc2(k) zwn(k) - tzc1(k) zwn(k-1)))
// for k >= 2; p(1) = 0.
__global__ void __launch_bounds__(128) k_hadj_pressure_source(Scalars s, Args a) {
  HADJ_POINT_INDEX
  const Geo g = geo(s);
  const double* pb = a.tg[F_P];
  const double timec = s.forward ? 1.0 / s.dtm : 1.0 / (2.0 * s.dtm);
  const int st = s.nz + 2;
  if (k >= 2) {
    const double p0 = pb[o];
    a.tg[F_ZUN][o] += timec * s.cx * (p0 - pb[g.at(k, j, i + 1)]);
    a.tg[F_ZVN][o] += timec * s.cy * (p0 - pb[g.at(k, j + 1, i)]);
  }
  double zw = 0.0;
  if (k >= 2) zw += s.prof[P_TZC2 * st + k] * pb[o];
  if (k + 1 <= s.nz) zw -= s.prof[P_TZC1 * st + k + 1] * pb[o + s.plane];
  a.tg[F_ZWN][o] += timec * 4.0 * zw;
}

// ---- momentum (eval_momentum: pw_point, viscosity_point, coriolis_point, buoyancy, stepping) ---
struct VelAdj {
  int fu, fv, fw;  // adjoint targets of ZU, ZV, ZW (u, v, w on the forward step, else zu, zv, zw)
};

// adjoint of tau_13_23(kk) (the t13, t13m1, t23, t23m1 stresses) with the given bars
__device__ __forceinline__ void adj_tau13_23(const Scalars& s, const Prof<double>& P, const View<double>& ZU,
                                             const View<double>& ZV, const View<double>& ZW,
                                             const View<double>& VIS, const Scatter& S, const VelAdj& f, int kk,
                                             int j, int i, double b13, double b13m1, double b23, double b23m1) {
  const double cx = s.cx, cy = s.cy, rdzn = P(P_RDZN, kk + 1), rho = P(P_RHO, kk);
  if (b13 != 0.0) {
    const double vis13 = 0.5 * (VIS(kk, j, i) + VIS(kk, j, i + 1));
    const double gr = (ZU(kk + 1, j, i) - ZU(kk, j, i)) * rdzn + (ZW(kk, j, i + 1) - ZW(kk, j, i)) * cx;
    const double gb = b13 * rho * vis13, vb = 0.5 * b13 * gr * rho;
    S(f.fu, kk + 1, j, i, gb * rdzn);
    S(f.fu, kk, j, i, -gb * rdzn);
    S(f.fw, kk, j, i + 1, gb * cx);
    S(f.fw, kk, j, i, -gb * cx);
    S(F_VIS, kk, j, i, vb);
    S(F_VIS, kk, j, i + 1, vb);
  }
  if (b13m1 != 0.0) {
    const double vis13 = 0.5 * (VIS(kk, j, i - 1) + VIS(kk, j, i));
    const double gr = (ZU(kk + 1, j, i - 1) - ZU(kk, j, i - 1)) * rdzn + (ZW(kk, j, i) - ZW(kk, j, i - 1)) * cx;
    const double gb = b13m1 * rho * vis13, vb = 0.5 * b13m1 * gr * rho;
    S(f.fu, kk + 1, j, i - 1, gb * rdzn);
    S(f.fu, kk, j, i - 1, -gb * rdzn);
    S(f.fw, kk, j, i, gb * cx);
    S(f.fw, kk, j, i - 1, -gb * cx);
    S(F_VIS, kk, j, i - 1, vb);
    S(F_VIS, kk, j, i, vb);
  }
  if (b23 != 0.0) {
    const double vis23 = 0.5 * (VIS(kk, j, i) + VIS(kk, j + 1, i));
    const double gr = (ZW(kk, j + 1, i) - ZW(kk, j, i)) * cy + (ZV(kk + 1, j, i) - ZV(kk, j, i)) * rdzn;
    const double gb = b23 * rho * vis23, vb = 0.5 * b23 * gr * rho;
    S(f.fw, kk, j + 1, i, gb * cy);
    S(f.fw, kk, j, i, -gb * cy);
    S(f.fv, kk + 1, j, i, gb * rdzn);
    S(f.fv, kk, j, i, -gb * rdzn);
    S(F_VIS, kk, j, i, vb);
    S(F_VIS, kk, j + 1, i, vb);
  }
  if (b23m1 != 0.0) {
    const double vis23 = 0.5 * (VIS(kk, j - 1, i) + VIS(kk, j, i));
    const double gr = (ZW(kk, j, i) - ZW(kk, j - 1, i)) * cy + (ZV(kk + 1, j - 1, i) - ZV(kk, j - 1, i)) * rdzn;
    const double gb = b23m1 * rho * vis23, vb = 0.5 * b23m1 * gr * rho;
    S(f.fw, kk, j, i, gb * cy);
    S(f.fw, kk, j - 1, i, -gb * cy);
    S(f.fv, kk + 1, j - 1, i, gb * rdzn);
    S(f.fv, kk, j - 1, i, -gb * rdzn);
    S(F_VIS, kk, j - 1, i, vb);
    S(F_VIS, kk, j, i, vb);
  }
}

// adjoint of tau33_at(kk) = rhon(kk) (vis(kk) + vis(kk-1)) (zw(kk) - zw(kk-1)) rdz(kk)
__device__ __forceinline__ void adj_tau33(const Prof<double>& P, const View<double>& ZW, const View<double>& VIS,
                                          const Scatter& S, int fw, int kk, int j, int i, double b) {
  if (kk <= 1 || b == 0.0) return;
  const double rhon = P(P_RHON, kk), rdz = P(P_RDZ, kk);
  const double visonp2 = rhon * (VIS(kk, j, i) + VIS(kk - 1, j, i));
  const double dw = (ZW(kk, j, i) - ZW(kk - 1, j, i));
  S(fw, kk, j, i, b * visonp2 * rdz);
  S(fw, kk - 1, j, i, -b * visonp2 * rdz);
  const double vb = b * rhon * dw * rdz;
  S(F_VIS, kk, j, i, vb);
  S(F_VIS, kk - 1, j, i, vb);
}

// adjoint of viscosity_point with the bars du_b, dv_b, dw_b of its three increments
__device__ void adj_viscosity(const Scalars& s, const Prof<double>& P, const View<double>& ZU,
                              const View<double>& ZV, const View<double>& ZW, const View<double>& ZUs,
                              const View<double>& VIS, const Scatter& S, const VelAdj& f, int k, int j, int i,
                              double du_b, double dv_b, double dw_b) {
  const double cx = s.cx, cy = s.cy, rhon = P(P_RHON, k);
  const double xa = s.rho_unity ? du_b : du_b / rhon;
  const double xb = s.rho_unity ? dv_b : dv_b / rhon;
  const double xc = (k < s.nz) ? (s.rho_unity ? dw_b : dw_b / P(P_RHO, k)) : 0.0;
  const double rdz = P(P_RDZ, k);
  // bars of the stresses the three increments difference
  const double b11p1 = xa * cx, b11 = -xa * cx;
  const double b12 = xa * cy + xb * cx, b12ym1 = -xa * cy, b12m1 = -xb * cx;
  const double b22yp1 = xb * cy, b22 = -xb * cy;
  // tau12 at (j, i): columns i, i+1 of rows j, j+1 on levels k, k-1
  {
    const double gr = (ZU(k, j + 1, i) - ZU(k, j, i)) * cy + (ZV(k, j, i + 1) - ZV(k, j, i)) * cx;
    const double vis12 = 0.125 * (VIS(k, j, i) + VIS(k, j + 1, i) + VIS(k - 1, j, i) + VIS(k - 1, j + 1, i) +
                                  VIS(k, j, i + 1) + VIS(k, j + 1, i + 1) + VIS(k - 1, j, i + 1) +
                                  VIS(k - 1, j + 1, i + 1));
    const double gb = b12 * rhon * vis12, vb = 0.125 * b12 * gr * rhon;
    S(f.fu, k, j + 1, i, gb * cy);
    S(f.fu, k, j, i, -gb * cy);
    S(f.fv, k, j, i + 1, gb * cx);
    S(f.fv, k, j, i, -gb * cx);
    for (int kk = k - 1; kk <= k; ++kk)
      for (int jj = j; jj <= j + 1; ++jj)
        for (int ii = i; ii <= i + 1; ++ii) S(F_VIS, kk, jj, ii, vb);
  }
  // tau12m1: columns i-1, i of rows j, j+1
  {
    const double gr = (ZU(k, j + 1, i - 1) - ZU(k, j, i - 1)) * cy + (ZV(k, j, i) - ZV(k, j, i - 1)) * cx;
    const double vis12 = 0.125 * (VIS(k, j, i) + VIS(k, j + 1, i) + VIS(k - 1, j, i) + VIS(k - 1, j + 1, i) +
                                  VIS(k, j, i - 1) + VIS(k, j + 1, i - 1) + VIS(k - 1, j, i - 1) +
                                  VIS(k - 1, j + 1, i - 1));
    const double gb = b12m1 * rhon * vis12, vb = 0.125 * b12m1 * gr * rhon;
    S(f.fu, k, j + 1, i - 1, gb * cy);
    S(f.fu, k, j, i - 1, -gb * cy);
    S(f.fv, k, j, i, gb * cx);
    S(f.fv, k, j, i - 1, -gb * cx);
    for (int kk = k - 1; kk <= k; ++kk)
      for (int jj = j; jj <= j + 1; ++jj)
        for (int ii = i - 1; ii <= i; ++ii) S(F_VIS, kk, jj, ii, vb);
  }
  // tau12_ym1: columns i, i+1 of rows j-1, j
  {
    const double gr = (ZU(k, j, i) - ZU(k, j - 1, i)) * cy + (ZV(k, j - 1, i + 1) - ZV(k, j - 1, i)) * cx;
    const double vis12 = 0.125 * (VIS(k, j - 1, i) + VIS(k, j, i) + VIS(k - 1, j - 1, i) + VIS(k - 1, j, i) +
                                  VIS(k, j - 1, i + 1) + VIS(k, j, i + 1) + VIS(k - 1, j - 1, i + 1) +
                                  VIS(k - 1, j, i + 1));
    const double gb = b12ym1 * rhon * vis12, vb = 0.125 * b12ym1 * gr * rhon;
    S(f.fu, k, j, i, gb * cy);
    S(f.fu, k, j - 1, i, -gb * cy);
    S(f.fv, k, j - 1, i + 1, gb * cx);
    S(f.fv, k, j - 1, i, -gb * cx);
    for (int kk = k - 1; kk <= k; ++kk)
      for (int jj = j - 1; jj <= j; ++jj)
        for (int ii = i; ii <= i + 1; ++ii) S(F_VIS, kk, jj, ii, vb);
  }
  // tau11 and tau22 share visonp2 = rhon (vis(k) + vis(k-1)) at (j, i)
  {
    const double visonp2 = rhon * (VIS(k, j, i) + VIS(k - 1, j, i));
    const double du = (ZU(k, j, i) - ZU(k, j, i - 1)), dv = (ZV(k, j, i) - ZV(k, j - 1, i));
    S(f.fu, k, j, i, b11 * visonp2 * cx);
    S(f.fu, k, j, i - 1, -b11 * visonp2 * cx);
    S(f.fv, k, j, i, b22 * visonp2 * cy);
    S(f.fv, k, j - 1, i, -b22 * visonp2 * cy);
    const double vb = rhon * (b11 * du * cx + b22 * dv * cy);
    S(F_VIS, k, j, i, vb);
    S(F_VIS, k - 1, j, i, vb);
  }
  // tau22_yp1 at (j+1, i)
  {
    const double visonp2 = rhon * (VIS(k, j + 1, i) + VIS(k - 1, j + 1, i));
    const double dv = (ZV(k, j + 1, i) - ZV(k, j, i));
    S(f.fv, k, j + 1, i, b22yp1 * visonp2 * cy);
    S(f.fv, k, j, i, -b22yp1 * visonp2 * cy);
    const double vb = rhon * b22yp1 * dv * cy;
    S(F_VIS, k, j + 1, i, vb);
    S(F_VIS, k - 1, j + 1, i, vb);
  }
  // tau11p1 at (j, i+1): current_state%zu at x+1 minus ZU at x
  {
    const double visonp2 = rhon * (VIS(k, j, i + 1) + VIS(k - 1, j, i + 1));
    const double du = (ZUs(k, j, i + 1) - ZU(k, j, i));
    S(F_ZU, k, j, i + 1, b11p1 * visonp2 * cx);
    S(f.fu, k, j, i, -b11p1 * visonp2 * cx);
    const double vb = rhon * b11p1 * du * cx;
    S(F_VIS, k, j, i + 1, vb);
    S(F_VIS, k - 1, j, i + 1, vb);
  }
  // vertical stresses
  if (k < s.nz)
    adj_tau13_23(s, P, ZU, ZV, ZW, VIS, S, f, k, j, i, xa * rdz + xc * cx, -xc * cx, xb * rdz + xc * cy, -xc * cy);
  adj_tau13_23(s, P, ZU, ZV, ZW, VIS, S, f, k - 1, j, i, -xa * rdz, 0.0, -xb * rdz, 0.0);
  if (k < s.nz) {
    const double rdzn1 = P(P_RDZN, k + 1);
    adj_tau33(P, ZW, VIS, S, f.fw, k + 1, j, i, xc * rdzn1);
    adj_tau33(P, ZW, VIS, S, f.fw, k, j, i, -xc * rdzn1);
  }
}

// adjoint of pw_point with the bars a, b, c of su, sv, sw (c = 0 at k = nz, where sw is not set)
__device__ void adj_pw(const Scalars& s, const Prof<double>& P, const View<double>& U, const View<double>& V,
                       const View<double>& W, const Scatter& S, int k, int j, int i, double a, double b, double c) {
  const double tcx = s.tcx, tcy = s.tcy, tzc1 = P(P_TZC1, k);
  const double u0 = U(k, j, i), v0 = V(k, j, i);
  const double Uw = U(k, j, i - 1), Ue = U(k, j, i + 1), Us = U(k, j - 1, i), Un = U(k, j + 1, i), Ub = U(k - 1, j, i);
  const double Uwn = U(k, j + 1, i - 1);
  const double Vs = V(k, j - 1, i), Vse = V(k, j - 1, i + 1), Ve = V(k, j, i + 1), Vn = V(k, j + 1, i);
  const double Vw = V(k, j, i - 1), Vb = V(k - 1, j, i);
  const double Wb = W(k - 1, j, i), Wbe = W(k - 1, j, i + 1), Wbn = W(k - 1, j + 1, i);
  // terms present on every level 2 <= k <= nz
  double bu0 = a * tcx * (Uw - Ue) - b * tcx * Ve;
  double buw = a * tcx * (u0 + 2.0 * Uw) + b * tcx * Vw;
  const double bue = -a * tcx * (u0 + 2.0 * Ue);
  const double bus = a * tcy * (Vs + Vse);
  const double bun = -a * tcy * (v0 + Ve) - b * tcx * Ve;
  const double bub = a * tzc1 * (Wb + Wbe);
  const double buwn = b * tcx * Vw;
  double bv0 = -a * tcy * Un + b * tcy * (Vs - Vn);
  const double bve = -a * tcy * Un - b * tcx * (u0 + Un);
  double bvs = a * tcy * Us + b * tcy * (v0 + 2.0 * Vs);
  const double bvse = a * tcy * Us;
  const double bvn = -b * tcy * (v0 + 2.0 * Vn);
  const double bvw = b * tcx * (Uw + Uwn);
  const double bvb = b * tzc1 * (Wb + Wbn);
  double bwb = a * tzc1 * Ub + b * tzc1 * Vb;
  const double bwbe = a * tzc1 * Ub;
  const double bwbn = b * tzc1 * Vb;
  if (k < s.nz) {
    const double tzc2 = P(P_TZC2, k), tzd1 = P(P_TZD1, k), tzd2 = P(P_TZD2, k);
    const double w0 = W(k, j, i), We = W(k, j, i + 1), Wn = W(k, j + 1, i), Wt = W(k + 1, j, i);
    const double Ww = W(k, j, i - 1), Ws = W(k, j - 1, i);
    const double Ut = U(k + 1, j, i), Uwt = U(k + 1, j, i - 1), Vt = V(k + 1, j, i), Vst = V(k + 1, j - 1, i);
    bu0 += -c * tcx * We;
    buw += c * tcx * Ww;
    bv0 += -c * tcy * Wn;
    bvs += c * tcy * Ws;
    bwb += c * tzd1 * (w0 + 2.0 * Wb);
    S(F_U, k + 1, j, i, -a * tzc2 * (w0 + We) - c * tcx * We);
    S(F_U, k + 1, j, i - 1, c * tcx * Ww);
    S(F_V, k + 1, j, i, -b * tzc2 * (w0 + Wn) - c * tcy * Wn);
    S(F_V, k + 1, j - 1, i, c * tcy * Ws);
    S(F_W, k, j, i, -a * tzc2 * Ut - b * tzc2 * Vt + c * (tzd1 * Wb - tzd2 * Wt));
    S(F_W, k, j, i + 1, -a * tzc2 * Ut - c * tcx * (u0 + Ut));
    S(F_W, k, j + 1, i, -b * tzc2 * Vt - c * tcy * (v0 + Vt));
    S(F_W, k + 1, j, i, -c * tzd2 * (w0 + 2.0 * Wt));
    S(F_W, k, j, i - 1, c * tcx * (Uw + Uwt));
    S(F_W, k, j - 1, i, c * tcy * (Vs + Vst));
  }
  S(F_U, k, j, i, bu0);
  S(F_U, k, j, i - 1, buw);
  S(F_U, k, j, i + 1, bue);
  S(F_U, k, j - 1, i, bus);
  S(F_U, k, j + 1, i, bun);
  S(F_U, k - 1, j, i, bub);
  S(F_U, k, j + 1, i - 1, buwn);
  S(F_V, k, j, i, bv0);
  S(F_V, k, j, i + 1, bve);
  S(F_V, k, j - 1, i, bvs);
  S(F_V, k, j - 1, i + 1, bvse);
  S(F_V, k, j + 1, i, bvn);
  S(F_V, k, j, i - 1, bvw);
  S(F_V, k - 1, j, i, bvb);
  S(F_W, k - 1, j, i, bwb);
  S(F_W, k - 1, j, i + 1, bwbe);
  S(F_W, k - 1, j + 1, i, bwbn);
}

__global__ void __launch_bounds__(128) k_hadj_momentum(Scalars s, Args a) {
  HADJ_POINT_INDEX
  const double A = a.tg[F_ZUN][o], B = a.tg[F_ZVN][o], C = a.tg[F_ZWN][o];
  if (A == 0.0 && B == 0.0 && C == 0.0) return;
  const Geo g = geo(s);
  const Prof<double> P{s.prof, s.nz + 2};
  const Scatter S{a.tg, g};
  const DevState<double>& d = a.d;
  const bool fwd = s.forward;
  // stepping: zun = ugal + u + dtm su (forward) or ugal + zu + 2 dtm su (centred)
  if (fwd) {
    S(F_U, k, j, i, A);
    S(F_V, k, j, i, B);
    S(F_W, k, j, i, C);
  } else {
    S(F_ZU, k, j, i, A);
    S(F_ZV, k, j, i, B);
    S(F_ZW, k, j, i, C);
  }
  if (k < 2) return;
  const double cst = fwd ? s.dtm : 2.0 * s.dtm;
  const double sa = cst * A, sb = cst * B, sc = (k < s.nz) ? cst * C : 0.0;
  const View<double> U{d.u, g}, V{d.v, g}, W{d.w, g};
  if (k < s.nz && !s.passive_th) {
    const double hb = 0.5 * P(P_BUOY_CO, k) * sc;
    S(F_TH, k, j, i, hb);
    S(F_TH, k + 1, j, i, hb);
  }
  if (s.coriolis) {
    const double q = 0.25 * s.fcoriol * sa, r = -0.25 * s.fcoriol * sb;
    S(F_V, k, j, i, q);
    S(F_V, k, j, i + 1, q);
    S(F_V, k, j - 1, i, q);
    S(F_V, k, j - 1, i + 1, q);
    S(F_U, k, j, i, r);
    S(F_U, k, j, i - 1, r);
    S(F_U, k, j + 1, i, r);
    S(F_U, k, j + 1, i - 1, r);
  }
  if (s.use_vd) {
    const VelAdj f = fwd ? VelAdj{F_U, F_V, F_W} : VelAdj{F_ZU, F_ZV, F_ZW};
    const View<double> ZU{fwd ? d.u : d.zu, g}, ZV{fwd ? d.v : d.zv, g}, ZW{fwd ? d.w : d.zw, g};
    const View<double> ZUs{d.zu, g}, VIS{d.vis, g};
    adj_viscosity(s, P, ZU, ZV, ZW, ZUs, VIS, S, f, k, j, i, sa, sb, sc);
  }
  adj_pw(s, P, U, V, W, S, k, j, i, sa, sb, sc);
}


// ---- scalar pass (eval_scalar: TVD advection of theta, diffusion, stepping) --------------------
// derivatives of the limiter's building blocks as the forward evaluation branches them:
// tmax(0, x) = 0 > x ? 0 : x, |tmin(0, x)| with tmin(0, x) = 0 < x ? 0 : x, and |x|' = -1 where
// signbit(x)
__device__ __forceinline__ double d_max0(double x) { return (0.0 > x) ? 0.0 : 1.0; }
__device__ __forceinline__ double d_absmin0(double x) { return (0.0 < x) ? 0.0 : (signbit(x) ? -1.0 : 1.0); }
__device__ __forceinline__ double d_abs(double x) { return signbit(x) ? -1.0 : 1.0; }

// adjoint of the face limiter (limit_face, and calculate_flux_in_w's form of it with kcoef =
// dz^2 rdc and the curvature term supplied): bars of the limiter's inputs from the face's bar
struct LimBar {
  double dv, sum, fdels, fd, fc, fu, fgt1, fgt2, curv;
};
__device__ __forceinline__ LimBar limit_adj(double rb, double data_value, double c, double dt, double sum,
                                            double fdels, double fd, double fc, double fu, double fgt1,
                                            double fgt2, double curv, double kcoef, double& value) {
  const double r6 = 1.0 / 6.0;
  const double cflmod = fabs(data_value * c * dt);
  const double hrcfl = rcp(sum + 1.e-30);
  const double hcfl = 0.5 * cflmod;
  const double cflcoef = r6 * (1.0 - cflmod * cflmod) * kcoef;
  const double rfdels = rcp(fdels + 1.e-30);
  const double ffs = 0.5 * (fd + fc) - hcfl * (fd - fc) - cflcoef * curv - fgt1 - fgt2;
  const double fnfs = (ffs - fu) * rfdels;
  const double fncs = (fc - fu) * rfdels;
  const double fnrefs = fncs * hrcfl;
  const bool sel_nfs = fnfs < fnrefs;
  const double m1 = sel_nfs ? fnfs : fnrefs;
  const bool sel_m1 = m1 < 1.0;
  const double m2 = sel_m1 ? m1 : 1.0;
  const bool sel_ncs = fncs > m2;
  const double ftemp = sel_ncs ? fncs : m2;
  value = ftemp * fdels + fu;
  LimBar b;
  const double ftemp_b = rb * fdels;
  b.fdels = rb * ftemp;
  b.fu = rb;
  double fncs_b = 0.0, fnfs_b = 0.0, fnrefs_b = 0.0;
  if (sel_ncs) fncs_b = ftemp_b;
  else if (sel_m1) (sel_nfs ? fnfs_b : fnrefs_b) = ftemp_b;
  fncs_b += fnrefs_b * hrcfl;
  const double hrcfl_b = fnrefs_b * fncs;
  const double rfdels_b = fncs_b * (fc - fu) + fnfs_b * (ffs - fu);
  b.fc = fncs_b * rfdels;
  b.fu -= (fncs_b + fnfs_b) * rfdels;
  const double ffs_b = fnfs_b * rfdels;
  b.fdels -= rfdels_b * rfdels * rfdels;
  b.sum = -hrcfl_b * hrcfl * hrcfl;
  b.fd = ffs_b * (0.5 - hcfl);
  b.fc += ffs_b * (0.5 + hcfl);
  const double hcfl_b = -ffs_b * (fd - fc);
  const double cflcoef_b = -ffs_b * curv;
  b.curv = -ffs_b * cflcoef;
  b.fgt1 = -ffs_b;
  b.fgt2 = -ffs_b;
  const double cflmod_b = 0.5 * hcfl_b - cflcoef_b * r6 * 2.0 * cflmod * kcoef;
  b.dv = cflmod_b * d_abs(data_value * c * dt) * c * dt;
  return b;
}

struct TvdAcc {
  View<double> U, V, W, ZF;
  Scatter S;
  int fz;  // adjoint target of the advected field (th on the forward step, else zth)
};

// one pair of the advective Courant sum, coef (max(0, x_a) + |min(0, x_b)|): its adjoint scattered
__device__ __forceinline__ void sum_pair_adj(const TvdAcc& t, int f, const View<double>& X, int ka, int ja, int ia,
                                             int kb, int jb, int ib, double coef) {
  t.S(f, ka, ja, ia, coef * d_max0(X(ka, ja, ia)));
  t.S(f, kb, jb, ib, coef * d_absmin0(X(kb, jb, ib)));
}

// face x+1/2 of cell (k, j, i) (tvd_face_x): its value, and with bar fb its adjoint scattered
__device__ double face_x_adj(const Scalars& s, const Prof<double>& P, const TvdAcc& t, int k, int j, int i,
                             double fb) {
  const int nz = s.nz;
  const double cx = s.cx, cy = s.cy, dt = s.dtm * 2.0;
  const int kp1 = k + 1 < nz ? k + 1 : nz;
  const int kp0 = kp1 - 1;
  const double u0 = t.U(k, j, i);
  const double sm = tsign<double>(.5, u0);
  const double advpos = 0.5 + sm, advneg = 0.5 - sm;
  const bool pos = advpos == 1.0;
  const double fu = t.ZF(k, j, i - 1) * advpos + t.ZF(k, j, i + 2) * advneg;
  const double fc = t.ZF(k, j, i) * advpos + t.ZF(k, j, i + 1) * advneg;
  const double fd = t.ZF(k, j, i + 1) * advpos + t.ZF(k, j, i) * advneg;
  const double fdels = fd - fu;
  const double fcurvs = fd - 2.0 * fc + fu;
  // the points fu, fc, fd read
  const int iu = pos ? i - 1 : i + 2, ic = pos ? i : i + 1, id = pos ? i + 1 : i;
  if (fabs(fcurvs) >= fabs(fdels)) {
    if (fb != 0.0) t.S(t.fz, k, j, ic, fb);
    return fc;
  }
  double sum;
  if (u0 > 0.0) {
    sum = 0.0;
    sum = sum + P(P_RDZ, k) * (tmax<double>(0.0, t.W(k, j, i)) + fabs(tmin<double>(0.0, t.W(k - 1, j, i))));
    sum = sum + cy * (tmax<double>(0.0, t.V(k, j, i)) + fabs(tmin<double>(0.0, t.V(k, j - 1, i))));
    sum = sum + cx * (u0 + fabs(tmin<double>(0.0, t.U(k, j, i - 1))));
    sum = sum * dt;
  } else {
    sum = 0.0;
    sum = sum + P(P_RDZ, k) * (tmax<double>(0.0, t.W(k, j, i + 1)) + fabs(tmin<double>(0.0, t.W(k - 1, j, i + 1))));
    sum = sum + cy * (tmax<double>(0.0, t.V(k, j, i + 1)) + fabs(tmin<double>(0.0, t.V(k, j - 1, i + 1))));
    sum = sum + cx * (tmax<double>(0.0, t.U(k, j, i + 1)) - u0);
    sum = sum * dt;
  }
  // gradient term in z over the two source columns
  const double sf1 = 0.125 * (t.W(k, j, i) + t.W(k - 1, j, i) + t.W(k, j, i + 1) + t.W(k - 1, j, i + 1));
  const bool zpos = !signbit(sf1);
  const int ksu = zpos ? k - 1 : kp1, ksl = zpos ? k : kp0;
  double ts = t.ZF(ksl, j, i) - t.ZF(ksu, j, i);
  ts = ts * advpos + (t.ZF(ksl, j, i + 1) - t.ZF(ksu, j, i + 1)) * advneg;
  const double rdzg = P(P_RDZ, k);
  const double fgt1 = fabs(sf1) * rdzg * dt * ts;
  // gradient term in y over the two v columns
  const double sf2 = 0.125 * (t.V(k, j, i + 1) + t.V(k, j, i) + t.V(k, j - 1, i + 1) + t.V(k, j - 1, i));
  const int jsu = signbit(sf2) ? j + 1 : j - 1;
  double t1 = t.ZF(k, jsu, i) * advpos;
  const double t2 = t.ZF(k, jsu, i + 1) * advneg;
  t1 = t1 + t2;
  const double fgt2 = fabs(sf2) * cy * dt * (fc - t1);
  double value;
  const LimBar b = limit_adj(fb, u0, cx, dt, sum, fdels, fd, fc, fu, fgt1, fgt2, fcurvs, 1.0, value);
  if (fb == 0.0) return value;
  // curvature and spread back onto fd, fc, fu
  const double fd_b = b.fd + b.fdels + b.curv;
  double fc_b = b.fc - 2.0 * b.curv + b.fgt2 * fabs(sf2) * cy * dt;
  const double fu_b = b.fu - b.fdels + b.curv;
  const double t1_b = -b.fgt2 * fabs(sf2) * cy * dt;
  const double ts_b = b.fgt1 * fabs(sf1) * rdzg * dt;
  const int isrc = pos ? i : i + 1;  // the column fgt1's and fgt2's ZF reads are weighted onto
  t.S(t.fz, k, j, iu, fu_b);
  t.S(t.fz, k, j, ic, fc_b);
  t.S(t.fz, k, j, id, fd_b);
  t.S(t.fz, ksl, j, isrc, ts_b);
  t.S(t.fz, ksu, j, isrc, -ts_b);
  t.S(t.fz, k, jsu, isrc, t1_b);
  // flow: the Courant sum, |sf1|, |sf2| and cflmod
  const double sa = b.sum * dt;
  if (u0 > 0.0) {
    sum_pair_adj(t, F_W, t.W, k, j, i, k - 1, j, i, sa * P(P_RDZ, k));
    sum_pair_adj(t, F_V, t.V, k, j, i, k, j - 1, i, sa * cy);
    t.S(F_U, k, j, i - 1, sa * cx * d_absmin0(t.U(k, j, i - 1)));
    t.S(F_U, k, j, i, sa * cx + b.dv);
  } else {
    sum_pair_adj(t, F_W, t.W, k, j, i + 1, k - 1, j, i + 1, sa * P(P_RDZ, k));
    sum_pair_adj(t, F_V, t.V, k, j, i + 1, k, j - 1, i + 1, sa * cy);
    t.S(F_U, k, j, i + 1, sa * cx * d_max0(t.U(k, j, i + 1)));
    t.S(F_U, k, j, i, -sa * cx + b.dv);
  }
  const double sf1_b = 0.125 * b.fgt1 * d_abs(sf1) * rdzg * dt * ts;
  t.S(F_W, k, j, i, sf1_b);
  t.S(F_W, k - 1, j, i, sf1_b);
  t.S(F_W, k, j, i + 1, sf1_b);
  t.S(F_W, k - 1, j, i + 1, sf1_b);
  const double sf2_b = 0.125 * b.fgt2 * d_abs(sf2) * cy * dt * (fc - t1);
  t.S(F_V, k, j, i + 1, sf2_b);
  t.S(F_V, k, j, i, sf2_b);
  t.S(F_V, k, j - 1, i + 1, sf2_b);
  t.S(F_V, k, j - 1, i, sf2_b);
  return value;
}

// face y+1/2 of cell (k, j, i) (tvd_face_y)
__device__ double face_y_adj(const Scalars& s, const Prof<double>& P, const TvdAcc& t, int k, int j, int i,
                             double fb) {
  const int nz = s.nz;
  const double cx = s.cx, cy = s.cy, dt = s.dtm * 2.0;
  const int kp1 = k + 1 < nz ? k + 1 : nz;
  const int kp0 = kp1 - 1;
  const double v0 = t.V(k, j, i);
  const double sm = tsign<double>(0.5, v0);
  const double advpos = 0.5 + sm, advneg = 0.5 - sm;
  const bool pos = advpos == 1.0;
  const int jo = signbit(v0) ? 1 : 0;
  const double fu = t.ZF(k, j - 1, i) * advpos + t.ZF(k, j + 2, i) * advneg;
  const double fc = t.ZF(k, j, i) * advpos + t.ZF(k, j + 1, i) * advneg;
  const double fd = t.ZF(k, j + 1, i) * advpos + t.ZF(k, j, i) * advneg;
  const double fdels = fd - fu;
  const double fcurvs = fd - 2.0 * fc + fu;
  const int ju = pos ? j - 1 : j + 2, jc = pos ? j : j + 1, jd = pos ? j + 1 : j;
  if (fabs(fcurvs) >= fabs(fdels)) {
    if (fb != 0.0) t.S(t.fz, k, jc, i, fb);
    return fc;
  }
  const int jj = j + jo;
  double sum = 0.0;
  sum = sum + P(P_RDZ, k) * (tmax<double>(0.0, t.W(k, jj, i)) + fabs(tmin<double>(0.0, t.W(k - 1, jj, i))));
  sum = sum + cy * (tmax<double>(0.0, t.V(k, jj, i)) + fabs(tmin<double>(0.0, t.V(k, jj - 1, i))));
  sum = sum + cx * (tmax<double>(0.0, t.U(k, jj, i)) + fabs(tmin<double>(0.0, t.U(k, jj, i - 1))));
  sum = sum * dt;
  const double sf1 = 0.125 * (t.W(k, j, i) + t.W(k - 1, j, i) + t.W(k, j + 1, i) + t.W(k - 1, j + 1, i));
  const bool zpos = !signbit(sf1);
  const int ksu = zpos ? k - 1 : kp1, ksl = zpos ? k : kp0;
  const double ts = t.ZF(ksl, jj, i) - t.ZF(ksu, jj, i);
  const double rdzg = P(P_RDZ, k);
  const double fgt1 = fabs(sf1) * rdzg * dt * ts;
  const double sf2 = 0.125 * (t.U(k, j, i - 1) + t.U(k, j, i) + t.U(k, j + 1, i - 1) + t.U(k, j + 1, i));
  const double posuf = 0.5 + tsign<double>(.5, sf2);
  const double zr = t.ZF(k, jj, i + 1) * (1. - posuf) + t.ZF(k, jj, i - 1) * posuf;
  const double fgt2 = fabs(sf2) * cx * dt * (fc - zr);
  double value;
  const LimBar b = limit_adj(fb, v0, cy, dt, sum, fdels, fd, fc, fu, fgt1, fgt2, fcurvs, 1.0, value);
  if (fb == 0.0) return value;
  const double g2 = fabs(sf2) * cx * dt;
  t.S(t.fz, k, ju, i, b.fu - b.fdels + b.curv);
  t.S(t.fz, k, jc, i, b.fc - 2.0 * b.curv + b.fgt2 * g2);
  t.S(t.fz, k, jd, i, b.fd + b.fdels + b.curv);
  const double ts_b = b.fgt1 * fabs(sf1) * rdzg * dt;
  t.S(t.fz, ksl, jj, i, ts_b);
  t.S(t.fz, ksu, jj, i, -ts_b);
  t.S(t.fz, k, jj, posuf == 1.0 ? i - 1 : i + 1, -b.fgt2 * g2);
  const double sa = b.sum * dt;
  sum_pair_adj(t, F_W, t.W, k, jj, i, k - 1, jj, i, sa * P(P_RDZ, k));
  sum_pair_adj(t, F_V, t.V, k, jj, i, k, jj - 1, i, sa * cy);
  sum_pair_adj(t, F_U, t.U, k, jj, i, k, jj, i - 1, sa * cx);
  t.S(F_V, k, j, i, b.dv);
  const double sf1_b = 0.125 * b.fgt1 * d_abs(sf1) * rdzg * dt * ts;
  t.S(F_W, k, j, i, sf1_b);
  t.S(F_W, k - 1, j, i, sf1_b);
  t.S(F_W, k, j + 1, i, sf1_b);
  t.S(F_W, k - 1, j + 1, i, sf1_b);
  const double sf2_b = 0.125 * b.fgt2 * d_abs(sf2) * cx * dt * (fc - zr);
  t.S(F_U, k, j, i - 1, sf2_b);
  t.S(F_U, k, j, i, sf2_b);
  t.S(F_U, k, j + 1, i - 1, sf2_b);
  t.S(F_U, k, j + 1, i, sf2_b);
  return value;
}

// face above level k of cell (k, j, i), 2 <= k <= nz-1 (tvd_face_z; k = nz-1 is the top form)
__device__ double face_z_adj(const Scalars& s, const Prof<double>& P, const TvdAcc& t, int k, int j, int i,
                             double fb) {
  const int nz = s.nz;
  const double cx = s.cx, cy = s.cy, dt = s.dtm * 2.0;
  const double w0 = t.W(k, j, i);
  double fu, fc, fd, rdu, rdc, sum;
  int kf;                  // level of the gradient terms' upwind-side values
  int ku, kc, kd;          // levels fu, fc, fd read (fu = 2 ZF(k+1) - ZF(k) when top_down)
  bool top_down = false;
  int sw_k;                // level of the sum's w, v and u pairs
  double sw_coef;          // rdz of the sum's w pair (or of -w0 on the top form going down)
  if (k == nz - 1) {
    const bool up = w0 >= 0.0;
    if (up) { fu = t.ZF(k - 1, j, i); fc = t.ZF(k, j, i); fd = t.ZF(k + 1, j, i); ku = k - 1; kc = k; kd = k + 1; }
    else { fu = 2.0 * t.ZF(k + 1, j, i) - t.ZF(k, j, i); fc = t.ZF(k + 1, j, i); fd = t.ZF(k, j, i); ku = k + 1; kc = k + 1; kd = k; top_down = true; }
    const double fcurvs = fd - 2.0 * fc + fu;
    const double fdels = fd - fu;
    if (fabs(fcurvs) >= fabs(fdels)) {
      if (fb != 0.0) t.S(t.fz, kc, j, i, fb);
      return fc;
    }
    if (up) {
      sum = 0.0;
      sum = sum + P(P_RDZ, k) * (w0 + fabs(tmin<double>(0.0, t.W(k - 1, j, i))));
      sum = sum + cy * (tmax<double>(0.0, t.V(k, j, i)) + fabs(tmin<double>(0.0, t.V(k, j - 1, i))));
      sum = sum + cx * (tmax<double>(0.0, t.U(k, j, i)) + fabs(tmin<double>(0.0, t.U(k, j, i - 1))));
      sum = sum * dt;
      kf = k;
      rdu = P(P_RDZN, k);
      rdc = P(P_RDZ, k);
      sw_k = k;
      sw_coef = P(P_RDZ, k);
    } else {
      const int kr = nz < k + 1 ? nz : k + 1;
      sum = 0.0;
      sum = sum + (-w0 * P(P_RDZ, kr));
      sum = sum + cy * (tmax<double>(0.0, t.V(k + 1, j, i)) + fabs(tmin<double>(0.0, t.V(k + 1, j - 1, i))));
      sum = sum + cx * (tmax<double>(0.0, t.U(k + 1, j, i)) + fabs(tmin<double>(0.0, t.U(k + 1, j, i - 1))));
      sum = sum * dt;
      kf = k + 1;
      rdu = P(P_RDZN, nz);
      rdc = P(P_RDZ, kr);
      sw_k = k + 1;
      sw_coef = P(P_RDZ, kr);
    }
  } else {
    const double sm = tsign<double>(.5, w0);
    const double advpos = 0.5 + sm, advneg = 0.5 - sm;
    const bool pos = advpos == 1.0;
    const int ko = signbit(w0) ? 1 : 0;
    fu = t.ZF(k - 1, j, i) * advpos + t.ZF(k + 2, j, i) * advneg;
    fc = t.ZF(k + ko, j, i);
    fd = t.ZF(k + 1, j, i) * advpos + t.ZF(k, j, i) * advneg;
    ku = pos ? k - 1 : k + 2;
    kc = k + ko;
    kd = pos ? k + 1 : k;
    const double fcurvs = fd - 2.0 * fc + fu;
    const double fdels = fd - fu;
    if (fabs(fcurvs) >= fabs(fdels)) {
      if (fb != 0.0) t.S(t.fz, kc, j, i, fb);
      return fc;
    }
    sum = 0.0;
    sum = sum + P(P_RDZ, k + ko) * (tmax<double>(0.0, t.W(k + ko, j, i)) + fabs(tmin<double>(0.0, t.W(k - 1 + ko, j, i))));
    sum = sum + cy * (tmax<double>(0.0, t.V(k + ko, j, i)) + fabs(tmin<double>(0.0, t.V(k + ko, j - 1, i))));
    sum = sum + cx * (tmax<double>(0.0, t.U(k + ko, j, i)) + fabs(tmin<double>(0.0, t.U(k + ko, j, i - 1))));
    sum = sum * dt;
    kf = k + ko;
    rdu = P(P_RDZN, k) * advpos + P(P_RDZN, k + 2) * advneg;
    rdc = P(P_RDZ, k) * advpos + P(P_RDZ, k + 1) * advneg;
    sw_k = k + ko;
    sw_coef = P(P_RDZ, k + ko);
  }
  const double sf1 = 0.125 * (t.V(k, j - 1, i) + t.V(k, j, i) + t.V(k + 1, j - 1, i) + t.V(k + 1, j, i));
  const int jsu = signbit(sf1) ? j + 1 : j - 1;
  const double zg1 = t.ZF(kf, jsu, i);
  const double fgt1 = fabs(sf1) * cy * dt * (fc - zg1);
  const double sf2 = 0.125 * (t.U(k, j, i - 1) + t.U(k, j, i) + t.U(k + 1, j, i - 1) + t.U(k + 1, j, i));
  const double posuf = 0.5 + tsign<double>(.5, sf2);
  const double zr = t.ZF(kf, j, i + 1) * (1. - posuf) + t.ZF(kf, j, i - 1) * posuf;
  const double fgt2 = fabs(sf2) * cx * dt * (fc - zr);
  const double dd = P(P_DZN, k + 1), rdd = P(P_RDZN, k + 1);
  const double fdels = fd - fu;
  const double curv = (fd - fc) * rdd - (fc - fu) * rdu;
  double value;
  const LimBar b = limit_adj(fb, w0, rdd, dt, sum, fdels, fd, fc, fu, fgt1, fgt2, curv, dd * dd * rdc, value);
  if (fb == 0.0) return value;
  const double g1 = fabs(sf1) * cy * dt, g2 = fabs(sf2) * cx * dt;
  const double fu_b = b.fu - b.fdels + b.curv * rdu;
  const double fc_b = b.fc - b.curv * (rdd + rdu) + b.fgt1 * g1 + b.fgt2 * g2;
  const double fd_b = b.fd + b.fdels + b.curv * rdd;
  if (top_down) {
    t.S(t.fz, k + 1, j, i, 2.0 * fu_b);
    t.S(t.fz, k, j, i, -fu_b);
  } else {
    t.S(t.fz, ku, j, i, fu_b);
  }
  t.S(t.fz, kc, j, i, fc_b);
  t.S(t.fz, kd, j, i, fd_b);
  t.S(t.fz, kf, jsu, i, -b.fgt1 * g1);
  t.S(t.fz, kf, j, posuf == 1.0 ? i - 1 : i + 1, -b.fgt2 * g2);
  const double sa = b.sum * dt;
  if (k == nz - 1) {
    if (!top_down) {
      t.S(F_W, k, j, i, sa * sw_coef);
      t.S(F_W, k - 1, j, i, sa * sw_coef * d_absmin0(t.W(k - 1, j, i)));
    } else {
      t.S(F_W, k, j, i, -sa * sw_coef);
    }
  } else {
    sum_pair_adj(t, F_W, t.W, sw_k, j, i, sw_k - 1, j, i, sa * sw_coef);
  }
  sum_pair_adj(t, F_V, t.V, sw_k, j, i, sw_k, j - 1, i, sa * cy);
  sum_pair_adj(t, F_U, t.U, sw_k, j, i, sw_k, j, i - 1, sa * cx);
  t.S(F_W, k, j, i, b.dv);
  const double sf1_b = 0.125 * b.fgt1 * d_abs(sf1) * cy * dt * (fc - zg1);
  t.S(F_V, k, j - 1, i, sf1_b);
  t.S(F_V, k, j, i, sf1_b);
  t.S(F_V, k + 1, j - 1, i, sf1_b);
  t.S(F_V, k + 1, j, i, sf1_b);
  const double sf2_b = 0.125 * b.fgt2 * d_abs(sf2) * cx * dt * (fc - zr);
  t.S(F_U, k, j, i - 1, sf2_b);
  t.S(F_U, k, j, i, sf2_b);
  t.S(F_U, k + 1, j, i - 1, sf2_b);
  t.S(F_U, k + 1, j, i, sf2_b);
  return value;
}

// adjoint of diffusion_point (F = zth, D = diff) with the bar r of its value
__device__ void adj_diffusion(const Scalars& s, const Prof<double>& P, const View<double>& F,
                              const View<double>& D, const Scatter& S, int k, int j, int i, double r) {
  const double f0 = F(k, j, i), d0 = D(k, j, i), dm = D(k - 1, j, i);
  const double ax = r * s.cx2 * 0.25, ay = r * s.cy2 * 0.25;
  const double fw = F(k, j, i - 1), fe = F(k, j, i + 1), fs = F(k, j - 1, i), fn = F(k, j + 1, i);
  const double dw4 = (d0 + D(k, j, i - 1)) + (dm + D(k - 1, j, i - 1));
  const double de4 = (D(k, j, i + 1) + d0) + (D(k - 1, j, i + 1) + dm);
  const double ds4 = (d0 + D(k, j - 1, i)) + (dm + D(k - 1, j - 1, i));
  const double dn4 = (D(k, j + 1, i) + d0) + (D(k - 1, j + 1, i) + dm);
  double f0b = -ax * (dw4 + de4) - ay * (ds4 + dn4);
  S(F_ZTH, k, j, i - 1, ax * dw4);
  S(F_ZTH, k, j, i + 1, ax * de4);
  S(F_ZTH, k, j - 1, i, ay * ds4);
  S(F_ZTH, k, j + 1, i, ay * dn4);
  const double gw = ax * (fw - f0), ge = -ax * (f0 - fe), gs = ay * (fs - f0), gn = -ay * (f0 - fn);
  double d0b = gw + ge + gs + gn, dmb = gw + ge + gs + gn;
  S(F_DIFF, k, j, i - 1, gw);
  S(F_DIFF, k - 1, j, i - 1, gw);
  S(F_DIFF, k, j, i + 1, ge);
  S(F_DIFF, k - 1, j, i + 1, ge);
  S(F_DIFF, k, j - 1, i, gs);
  S(F_DIFF, k - 1, j - 1, i, gs);
  S(F_DIFF, k, j + 1, i, gn);
  S(F_DIFF, k - 1, j + 1, i, gn);
  const double czb = P(P_CZB, k);
  S(F_ZTH, k - 1, j, i, r * czb * dm);
  f0b -= r * czb * dm;
  dmb += r * czb * (F(k - 1, j, i) - f0);
  if (k < s.nz) {
    const double cza = P(P_CZA, k);
    f0b -= r * cza * d0;
    S(F_ZTH, k + 1, j, i, r * cza * d0);
    d0b -= r * cza * (f0 - F(k + 1, j, i));
  }
  S(F_ZTH, k, j, i, f0b);
  S(F_DIFF, k, j, i, d0b);
  S(F_DIFF, k - 1, j, i, dmb);
}

__global__ void __launch_bounds__(128) k_hadj_scalar(Scalars s, Args a) {
  HADJ_POINT_INDEX
  const Geo g = geo(s);
  const Prof<double> P{s.prof, s.nz + 2};
  const Scatter S{a.tg, g};
  const DevState<double>& d = a.d;
  const bool fwd = s.forward;
  // adjoint of the source of cell (kk, jj, ii) from the stepping: th_new = th + dtm src (forward),
  // zth + 2 dtm src (centred); zth_new = th (forward), (1-2 tsmth) th + tsmth (zth + th_new)
  auto rbar = [&](int kk, int jj, int ii) -> double {
    if (kk < 2 || kk > s.nz) return 0.0;
    const long long n = g.at(kk, jj, ii);
    return fwd ? s.dtm * a.seed[3][n] : 2.0 * s.dtm * (a.seed[3][n] + s.tsmth * a.seed[7][n]);
  };
  const double s_th = a.seed[3][o], s_zth = a.seed[7][o];
  if (fwd) {
    S(F_TH, k, j, i, s_th + s_zth);
  } else {
    S(F_ZTH, k, j, i, s_th + 2.0 * s.tsmth * s_zth);
    S(F_TH, k, j, i, (1.0 - 2.0 * s.tsmth) * s_zth);
  }
  if (k < 2) return;
  const double r0 = rbar(k, j, i);
  if (s.use_vd && r0 != 0.0) adj_diffusion(s, P, View<double>{d.zth, g}, View<double>{d.diff, g}, S, k, j, i, r0);
  const TvdAcc t{View<double>{d.u, g}, View<double>{d.v, g}, View<double>{d.w, g},
                 View<double>{fwd ? d.th : d.zth, g}, S, fwd ? F_TH : F_ZTH};
  // the three faces this cell owns; each face's bar is its weight in the two sources it enters
  {
    const double dr = rbar(k, j, i + 1) - r0;
    if (dr != 0.0) {
      const double u0 = t.U(k, j, i);
      const double f = face_x_adj(s, P, t, k, j, i, s.cx * u0 * dr);
      S(F_U, k, j, i, s.cx * f * dr);
    }
  }
  {
    const double dr = rbar(k, j + 1, i) - r0;
    if (dr != 0.0) {
      const double v0 = t.V(k, j, i);
      const double f = face_y_adj(s, P, t, k, j, i, s.cy * v0 * dr);
      S(F_V, k, j, i, s.cy * f * dr);
    }
  }
  if (k <= s.nz - 1) {
    const double dr = P(P_TZC1, k + 1) * rbar(k + 1, j, i) - P(P_TZC2, k) * r0;
    if (dr != 0.0) {
      const double w0 = t.W(k, j, i);
      const double f = face_z_adj(s, P, t, k, j, i, 4.0 * w0 * dr);
      S(F_W, k, j, i, 4.0 * f * dr);
    }
  }
}

// ---- subgrid pass, levels 2 <= k <= nz-1 (smagorinsky_point, dry Richardson number) ------------
// adjoint of half_squared_strain with the bar g of ssq
__device__ void adj_strain(const Scalars& s, const Prof<double>& P, const View<double>& U, const View<double>& V,
                           const View<double>& W, const Scatter& S, const VelAdj& f, int k, int j, int i,
                           double g) {
  const double cx = s.cx, cy = s.cy, cx2 = s.cx2, cy2 = s.cy2;
  const double rdzn1 = P(P_RDZN, k + 1), rdzk = P(P_RDZ, k), rdzk1 = P(P_RDZ, k + 1);
  {  // ssq11
    const double b1 = g * cx2 * 2.0 * (U(k + 1, j, i) - U(k + 1, j, i - 1));
    const double b2 = g * cx2 * 2.0 * (U(k, j, i) - U(k, j, i - 1));
    S(f.fu, k + 1, j, i, b1);
    S(f.fu, k + 1, j, i - 1, -b1);
    S(f.fu, k, j, i, b2);
    S(f.fu, k, j, i - 1, -b2);
  }
  {  // ssq22
    const double b1 = g * cy2 * 2.0 * (V(k + 1, j, i) - V(k + 1, j - 1, i));
    const double b2 = g * cy2 * 2.0 * (V(k, j, i) - V(k, j - 1, i));
    S(f.fv, k + 1, j, i, b1);
    S(f.fv, k + 1, j - 1, i, -b1);
    S(f.fv, k, j, i, b2);
    S(f.fv, k, j - 1, i, -b2);
  }
  {  // ssq33
    const double b1 = g * 2.0 * ((W(k, j, i) - W(k - 1, j, i)) * rdzk) * rdzk;
    const double b2 = g * 2.0 * ((W(k + 1, j, i) - W(k, j, i)) * rdzk1) * rdzk1;
    S(f.fw, k, j, i, b1 - b2);
    S(f.fw, k - 1, j, i, -b1);
    S(f.fw, k + 1, j, i, b2);
  }
  {  // ssq13
    const double x1 = (U(k + 1, j, i) - U(k, j, i)) * rdzn1 + (W(k, j, i + 1) - W(k, j, i)) * cx;
    const double x2 = (U(k + 1, j, i - 1) - U(k, j, i - 1)) * rdzn1 + (W(k, j, i) - W(k, j, i - 1)) * cx;
    const double b1 = g * x1, b2 = g * x2;
    S(f.fu, k + 1, j, i, b1 * rdzn1);
    S(f.fu, k, j, i, -b1 * rdzn1);
    S(f.fw, k, j, i + 1, b1 * cx);
    S(f.fw, k, j, i, (b2 - b1) * cx);
    S(f.fu, k + 1, j, i - 1, b2 * rdzn1);
    S(f.fu, k, j, i - 1, -b2 * rdzn1);
    S(f.fw, k, j, i - 1, -b2 * cx);
  }
  {  // ssq23
    const double y1 = (W(k, j, i) - W(k, j - 1, i)) * cy + (V(k + 1, j - 1, i) - V(k, j - 1, i)) * rdzn1;
    const double y2 = (W(k, j + 1, i) - W(k, j, i)) * cy + (V(k + 1, j, i) - V(k, j, i)) * rdzn1;
    const double b1 = g * y1, b2 = g * y2;
    S(f.fw, k, j, i, (b1 - b2) * cy);
    S(f.fw, k, j - 1, i, -b1 * cy);
    S(f.fv, k + 1, j - 1, i, b1 * rdzn1);
    S(f.fv, k, j - 1, i, -b1 * rdzn1);
    S(f.fw, k, j + 1, i, b2 * cy);
    S(f.fv, k + 1, j, i, b2 * rdzn1);
    S(f.fv, k, j, i, -b2 * rdzn1);
  }
  for (int kk = k; kk <= k + 1; ++kk) {  // ssq12: four horizontal shears on levels k and k+1
    const double z1 = (U(kk, j, i - 1) - U(kk, j - 1, i - 1)) * cy + (V(kk, j - 1, i) - V(kk, j - 1, i - 1)) * cx;
    const double z2 = (U(kk, j + 1, i - 1) - U(kk, j, i - 1)) * cy + (V(kk, j, i) - V(kk, j, i - 1)) * cx;
    const double z3 = (U(kk, j, i) - U(kk, j - 1, i)) * cy + (V(kk, j - 1, i + 1) - V(kk, j - 1, i)) * cx;
    const double z4 = (U(kk, j + 1, i) - U(kk, j, i)) * cy + (V(kk, j, i + 1) - V(kk, j, i)) * cx;
    const double b1 = 0.25 * g * z1, b2 = 0.25 * g * z2, b3 = 0.25 * g * z3, b4 = 0.25 * g * z4;
    S(f.fu, kk, j, i - 1, (b1 - b2) * cy);
    S(f.fu, kk, j - 1, i - 1, -b1 * cy);
    S(f.fu, kk, j + 1, i - 1, b2 * cy);
    S(f.fu, kk, j, i, (b3 - b4) * cy);
    S(f.fu, kk, j - 1, i, -b3 * cy);
    S(f.fu, kk, j + 1, i, b4 * cy);
    S(f.fv, kk, j - 1, i, (b1 - b3) * cx);
    S(f.fv, kk, j - 1, i - 1, -b1 * cx);
    S(f.fv, kk, j, i, (b2 - b4) * cx);
    S(f.fv, kk, j, i - 1, -b2 * cx);
    S(f.fv, kk, j - 1, i + 1, b3 * cx);
    S(f.fv, kk, j, i + 1, b4 * cx);
  }
}

// sum of v over the block (all of whose threads lie on one level), added to *dst by one thread
__device__ __forceinline__ void block_add(double v, double* dst) {
  __shared__ double part[4];
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  const int lane = threadIdx.x & 31, warp = (threadIdx.y * blockDim.x + threadIdx.x) >> 5;
  if (lane == 0) part[warp] = v;
  __syncthreads();
  if (warp == 0 && lane == 0) {
    const double t = (part[0] + part[1]) + (part[2] + part[3]);
    if (t != 0.0) atomicAdd(dst, t);
  }
}

// one block of 32 x 4 threads per (x, y) tile of one level: the rneutml_sq adjoint of the level is
// summed over the block before its single atomic (every point of a level adds to the same entry)
__global__ void __launch_bounds__(128) k_hadj_smagorinsky(Scalars s, Args a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z + 1;
  if (k < 2 || k >= s.nz) return;  // uniform over the block
  double prof_c = 0.0;
  if (i < s.nx && j < s.ny) {
    const long long o = (long long)(k - 1) * s.plane + (long long)j * s.nx + i;
    const double vb = a.tg[F_VIS][o], db = a.tg[F_DIFF][o];
    if (vb != 0.0 || db != 0.0) {
      const Geo g = geo(s);
      const Prof<double> P{s.prof, s.nz + 2};
      const Scatter S{a.tg, g};
      const DevState<double>& d = a.d;
      const bool fwd = s.forward;
      const View<double> U{fwd ? d.u : d.zu, g}, V{fwd ? d.v : d.zv, g}, W{fwd ? d.w : d.zw, g}, TH{d.th, g};
      const VelAdj f = fwd ? VelAdj{F_U, F_V, F_W} : VelAdj{F_ZU, F_ZV, F_ZW};
      // forward
      const double ssq = half_squared_strain<double>(s, P, U, V, W, k, j, i);
      double ri = 0.0;
      if (!s.passive_th)
        ri = (P(P_DTHREF, k) + TH(k + 1, j, i) - TH(k, j, i)) * P(P_RDZN, k + 1) * P(P_BUOY_CO, k) / ssq;
      double vs = 0.0, df = 0.0, ri_vs = 0.0, ri_df = 0.0;  // stability functions and their ri-derivatives
      if (ri <= 0.0) {
        const double x1 = 1.0 - s.subc * ri, x2 = 1.0 - s.subb * ri;
        vs = sqrt(x1);
        const double r2 = sqrt(x2);
        df = s.suba * r2;
        ri_vs = vs > 0.0 ? -s.subc * 0.5 / vs : 0.0;
        ri_df = r2 > 0.0 ? -s.subb * s.suba * 0.5 / r2 : 0.0;
      } else if (ri > 0.0 && ri < s.ric) {
        const double t1 = 1. - ri * s.ricinv;
        const double t = t1 * t1;
        const double rifac = t * t;
        const double ev = 1. - s.subh * ri, ed = 1. - s.subg * ri;
        vs = rifac * ev;
        df = rifac * s.suba * ed;
        const double rifac_ri = 2.0 * t * 2.0 * t1 * (-s.ricinv);
        ri_vs = rifac_ri * ev - rifac * s.subh;
        ri_df = rifac_ri * s.suba * ed - rifac * s.suba * s.subg;
      }
      const double rsq = P(P_RNEUTML_SQ, k), sq = sqrt(ssq);
      const double sctmp = rsq * sq;
      // reverse: vis = vs sctmp, diff = df sctmp, sctmp = rneutml_sq sqrt(ssq)
      const double sct_b = vb * vs + db * df;
      prof_c = sct_b * sq;
      double ssq_b = sq > 0.0 ? sct_b * rsq * 0.5 / sq : 0.0;
      const double ri_b = (vb * ri_vs + db * ri_df) * sctmp;
      if (!s.passive_th && ri_b != 0.0) {
        const double nb = ri_b * P(P_RDZN, k + 1) * P(P_BUOY_CO, k) / ssq;
        S(F_TH, k + 1, j, i, nb);
        S(F_TH, k, j, i, -nb);
        ssq_b -= ri_b * ri / ssq;
      }
      adj_strain(s, P, U, V, W, S, f, k, j, i, ssq_b);
    }
  }
  block_add(prof_c, a.tg[F_PROF] + k);
}
}  // namespace hadj

static dim3 hadj_grid(const Scalars& s) { return dim3((s.nx + 31) / 32, (s.ny + 3) / 4, s.nz); }
static dim3 hadj_block() { return dim3(32, 4, 1); }

bool hadj_pass(int pass, const Scalars& s, const DevState<double>& d, double* const* tg, const double* const* seed,
               cudaStream_t st) {
  hadj::Args a;
  a.d = d;
  for (int f = 0; f < F_COUNT; ++f) a.tg[f] = tg[f];
  for (int q = 0; q < 8; ++q) a.seed[q] = seed[q];
  switch (pass) {
    case 1: hadj::k_hadj_momentum<<<hadj_grid(s), hadj_block(), 0, st>>>(s, a); return true;
    case 2: hadj::k_hadj_scalar<<<hadj_grid(s), hadj_block(), 0, st>>>(s, a); return true;
    case 0: hadj::k_hadj_smagorinsky<<<hadj_grid(s), hadj_block(), 0, st>>>(s, a); return true;
    case 3: hadj::k_hadj_pressure_source<<<hadj_grid(s), hadj_block(), 0, st>>>(s, a); return true;
    case 4: hadj::k_hadj_pstep_swap<<<hadj_grid(s), hadj_block(), 0, st>>>(s, a); return true;
    default: return false;
  }
}

}  // namespace mgpu
