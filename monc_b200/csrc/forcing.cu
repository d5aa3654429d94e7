// Mean profiles (meanprofiles.F90), the mean-profile subsidence tendencies (forcing.F90) the
// damping and forcing components read, and the profile_diagnostics sums
// (profile_diagnostics.F90).
//
// MONC's mean_profiles runs in the solver group, after stepfields: olzubar, olzvbar, olzthbar and
// olzqbar are the horizontal means of the stepped fields before the pressure correction.  In the
// fused step those are zu_n, zv_n and the new theta and q; the next step's damping and forcing
// read them.  Each level of each field is summed by one block in a fixed order (deterministic),
// in FP64 whatever the field precision, and multiplied by rnhpts = 1 / real(nx ny) as MONC does.
#include "dycore.h"
#include "dycore_device.cuh"

namespace mgpu {

// field q of a mean: c[q] + p[q], or a[q] p[q] + b[q] p2[q] when p2[q] is set (theta after
// stepfields' time smoothing)
template <typename T>
struct MeanFields {
  const T* p[3 + MGPU_MAX_Q];
  const T* p2[3 + MGPU_MAX_Q];
  double a[3 + MGPU_MAX_Q], b[3 + MGPU_MAX_Q], c[3 + MGPU_MAX_Q];
};

// the level sums run over count points from row offset off of each plane (a slab's interior rows)
template <typename T>
__global__ void __launch_bounds__(256) k_plane_means(MeanFields<T> f, long long plane, long long off, long long count,
                                                     double rnhpts, double* out, int stride) {
  const int k = blockIdx.x + 1, q = blockIdx.y;
  const long long base = (long long)(k - 1) * plane + off;
  const T* __restrict__ p = f.p[q] + base;
  const T* __restrict__ p2 = f.p2[q] ? f.p2[q] + base : nullptr;
  const double a = f.a[q], b = f.b[q], c = f.c[q];
  double acc = 0.0;
  if (p2)
    for (long long t = threadIdx.x; t < count; t += blockDim.x) acc += a * (double)__ldg(p + t) + b * (double)__ldg(p2 + t);
  else
    for (long long t = threadIdx.x; t < count; t += blockDim.x) acc += c + (double)__ldg(p + t);
  __shared__ double sh[256];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[q * stride + k] = sh[0] * rnhpts;
}

// rnhpts of meanprofiles.F90:44: the point count converted at default (single) precision; a
// slab (halo rows above and below) averages its interior rows, which the slabs' driver averages
// again across the slabs (all slabs hold the same number of rows)
static long long interior(const Scalars& s, int halo) { return (long long)s.nx * (s.ny - 2 * halo); }
static double rnhpts(const Scalars& s, int halo) { return 1.0 / (double)(float)interior(s, halo); }

template <typename T>
int launch_mean_profiles(const Scalars& s, const T* zu, const T* zv, const T* th, const T* const* q, double* olz,
                         cudaStream_t st, int halo) {
  MeanFields<T> f{};
  f.p[0] = zu;
  f.p[1] = zv;
  f.p[2] = th;
  for (int n = 0; n < s.nq; ++n) f.p[3 + n] = q[n];
  k_plane_means<T><<<dim3(s.nz, 3 + s.nq), 256, 0, st>>>(f, s.plane, (long long)halo * s.nx, interior(s, halo),
                                                         rnhpts(s, halo), olz, s.nz + 2);
  return 1;
}
template int launch_mean_profiles<float>(const Scalars&, const float*, const float*, const float*, const float* const*,
                                         double*, cudaStream_t, int);
template int launch_mean_profiles<double>(const Scalars&, const double*, const double*, const double*,
                                          const double* const*, double*, cudaStream_t, int);

// olubar, olvbar, olthbar and olqbar(n): the means of ugal + u, vgal + v, theta and each q field,
// the scalars time-smoothed (c1 f + c2 zf) where their z-fields are given
template <typename T>
int launch_mean_profiles_state(const Scalars& s, const T* u, const T* v, const T* th, const T* zth,
                               const T* const* q, const T* const* zq, double ugal, double vgal, double c1, double c2,
                               double* olbar, cudaStream_t st, int halo) {
  MeanFields<T> f{};
  f.p[0] = u;
  f.c[0] = ugal;
  f.p[1] = v;
  f.c[1] = vgal;
  f.p[2] = th;
  f.p2[2] = zth;
  f.a[2] = c1;
  f.b[2] = c2;
  const int nq = q ? s.nq : 0;
  for (int n = 0; n < nq; ++n) {
    f.p[3 + n] = q[n];
    f.p2[3 + n] = zq ? zq[n] : nullptr;
    f.a[3 + n] = c1;
    f.b[3 + n] = c2;
  }
  k_plane_means<T><<<dim3(s.nz, 3 + nq), 256, 0, st>>>(f, s.plane, (long long)halo * s.nx, interior(s, halo),
                                                       rnhpts(s, halo), olbar, s.nz + 2);
  return 1;
}
template int launch_mean_profiles_state<float>(const Scalars&, const float*, const float*, const float*, const float*,
                                               const float* const*, const float* const*, double, double, double,
                                               double, double*, cudaStream_t, int);
template int launch_mean_profiles_state<double>(const Scalars&, const double*, const double*, const double*,
                                                const double*, const double* const*, const double* const*, double,
                                                double, double, double, double*, cudaStream_t, int);

// profile_diagnostics (profile_diagnostics.F90:311-636, PW flow and TVD scalars): one block per
// level sums the MGPU_PD_* quantities over the plane in FP64, in a fixed order
template <typename T>
__global__ void __launch_bounds__(256) k_profile_diagnostics(Scalars s, const T* __restrict__ u,
                                                             const T* __restrict__ v, const T* __restrict__ w,
                                                             const T* __restrict__ th, const T* __restrict__ qv,
                                                             const T* __restrict__ ql, const double* __restrict__ olbar,
                                                             int has_mean, int halo, double* __restrict__ out) {
  constexpr int NR = MGPU_PD_COUNT;
  const int k = blockIdx.x + 1, nz = s.nz, st = nz + 2;
  const Geo g{s.nx, s.ny, s.nz, s.plane};
  auto P = [&](int id, int kk) { return s.prof[id * st + kk]; };
  const bool moist = qv != nullptr;
  double acc[NR];
  for (int r = 0; r < NR; ++r) acc[r] = 0.0;
  const double ugal = s.ugal, vgal = s.vgal, thref = P(P_THREF, k);
  const double thbar = olbar[2 * st + k];
  const double umean = (k < nz && has_mean) ? 0.5 * (olbar[k] + olbar[k + 1]) : 0.0;
  const double vmean = (k < nz && has_mean) ? 0.5 * (olbar[st + k] + olbar[st + k + 1]) : 0.0;
  const long long count = (long long)s.nx * (s.ny - 2 * halo);
  for (long long t = threadIdx.x; t < count; t += blockDim.x) {
    const int j = halo + (int)(t / s.nx), i = (int)(t % s.nx);
    const long long o = g.at(k, j, i);
    const double w0 = (double)w[o], th0 = (double)th[o];
    acc[MGPU_PD_U_WIND] += (double)u[o] + ugal;
    acc[MGPU_PD_V_WIND] += (double)v[o] + vgal;
    acc[MGPU_PD_WW] += w0 * w0;
    if (k >= 2) {
      acc[MGPU_PD_W_WIND] += w0;
      acc[MGPU_PD_WWW] += w0 * w0 * w0;
      acc[MGPU_PD_WWWW] += (w0 * w0) * (w0 * w0);
    }
    acc[MGPU_PD_THETA] += th0 + thref;
    const double dth = th0 - thbar;
    acc[MGPU_PD_TH2] += dth * dth;
    if (k < nz) {
      const long long o1 = o + s.plane;
      if (k >= 2) acc[MGPU_PD_WTHETA_CN] += w0 * (0.5 * (th0 + (double)th[o1]));
      double up = 0.25 * ((double)u[o] + (double)u[g.at(k, j, i - 1)] + (double)u[o1] + (double)u[g.at(k + 1, j, i - 1)]) + ugal;
      up = up - umean;
      acc[MGPU_PD_UW] += up * w0;
      double vp = 0.25 * ((double)v[o] + (double)v[g.at(k, j - 1, i)] + (double)v[o1] + (double)v[g.at(k + 1, j - 1, i)]) + vgal;
      vp = vp - vmean;
      acc[MGPU_PD_VW] += vp * w0;
    }
    if (moist) {
      const double q0 = (double)qv[o], l0 = (double)ql[o];
      acc[MGPU_PD_VAPOUR] += q0;
      acc[MGPU_PD_LIQUID] += l0;
      if (k >= 2 && k < nz) {
        acc[MGPU_PD_WQV_CN] += 0.5 * (q0 + (double)qv[o + s.plane]) * w0;
        acc[MGPU_PD_WQL_CN] += 0.5 * (l0 + (double)ql[o + s.plane]) * w0;
      }
      const double tk = (th0 + thref) * P(P_RPREFRCP, k), pmb = P(P_PREFN, k) / 100.;
      acc[MGPU_PD_RH] += q0 / qsaturation<double>(tk, pmb);
    }
  }
  __shared__ double sh[256];
  const int nrows = moist ? NR : MGPU_PD_VAPOUR;
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    if (r >= nrows) break;  // uniform over the block
    sh[threadIdx.x] = acc[r];
    __syncthreads();
    for (int wdt = 128; wdt > 0; wdt >>= 1) {
      if (threadIdx.x < wdt) sh[threadIdx.x] += sh[threadIdx.x + wdt];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[(size_t)r * nz + k - 1] = sh[0];
    __syncthreads();
  }
}

template <typename T>
int launch_profile_diagnostics(const Scalars& s, const T* u, const T* v, const T* w, const T* th, const T* qv,
                               const T* ql, const double* olbar, bool has_mean, double* out, cudaStream_t st,
                               int halo) {
  k_profile_diagnostics<T><<<s.nz, 256, 0, st>>>(s, u, v, w, th, qv, ql, olbar, has_mean ? 1 : 0, halo, out);
  return 1;
}
template int launch_profile_diagnostics<float>(const Scalars&, const float*, const float*, const float*, const float*,
                                               const float*, const float*, const double*, bool, double*, cudaStream_t,
                                               int);
template int launch_profile_diagnostics<double>(const Scalars&, const double*, const double*, const double*,
                                                const double*, const double*, const double*, const double*, bool,
                                                double*, cudaStream_t, int);

// subsidence tendencies of the mean profiles (forcing.F90:1052-1166 with the profiles olzubar,
// olzvbar, olzthbar + thref and olzqbar), levels 2..nz: rows usub, vsub, thsub, qsub(n)
__global__ void k_subsidence_tendencies(Scalars s, const double* __restrict__ olz, double* __restrict__ tend,
                                        int flow_theta, int q) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int nz = s.nz, st = nz + 2;
  if (k > nz) return;
  auto P = [&](int id, int kk) { return s.prof[id * st + kk]; };
  if (flow_theta) {
    for (int r = 0; r < 2; ++r) {
      const double* prof = olz + r * st;
      double sub;
      if (k < nz)
        sub = 2.0 * (P(P_WSUBS, k - 1) * P(P_TZC1, k) * (prof[k] - prof[k - 1]) +
                     P(P_WSUBS, k) * P(P_TZC2, k) * (prof[k + 1] - prof[k]));
      else
        sub = 2.0 * (P(P_WSUBS, k - 1) * P(P_TZC1, k) * (prof[k] - prof[k - 1]));
      tend[r * st + k] = sub;
    }
    const double* th = olz + 2 * st;
    const int ka = k < nz ? k + 1 : k, kb = ka - 1;
    tend[2 * st + k] = P(P_WSUBS, k) * ((th[ka] + P(P_THREF, ka)) - (th[kb] + P(P_THREF, kb))) * P(P_RDZN, ka);
  }
  if (q)
    for (int n = 0; n < s.nq; ++n) {
      const double* qp = olz + (3 + n) * st;
      const int ka = k < nz ? k + 1 : k, kb = ka - 1;
      tend[(3 + n) * st + k] = P(P_WSUBS, k) * (qp[ka] - qp[kb]) * P(P_RDZN, ka);
    }
}

int launch_subsidence_tendencies(const Scalars& s, const double* olz, double* tend, bool flow_theta, bool q,
                                 cudaStream_t st) {
  const int n = s.nz - 1;
  k_subsidence_tendencies<<<(n + 127) / 128, 128, 0, st>>>(s, olz, tend, flow_theta ? 1 : 0, q ? 1 : 0);
  return 1;
}

}  // namespace mgpu
