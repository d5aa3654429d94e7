// Mean profiles (meanprofiles.F90) and the mean-profile subsidence tendencies (forcing.F90)
// the damping and forcing components read.
//
// MONC's mean_profiles runs in the solver group, after stepfields: olzubar, olzvbar, olzthbar and
// olzqbar are the horizontal means of the stepped fields before the pressure correction.  In the
// fused step those are zu_n, zv_n and the new theta and q; the next step's damping and forcing
// read them.  Each level of each field is summed by one block in a fixed order (deterministic),
// in FP64 whatever the field precision, and multiplied by rnhpts = 1 / real(nx ny) as MONC does.
#include "dycore.h"
#include "dycore_device.cuh"

namespace mgpu {

template <typename T>
struct MeanFields {
  const T* p[3 + MGPU_MAX_Q];
};

template <typename T>
__global__ void __launch_bounds__(256) k_plane_means(MeanFields<T> f, long long plane, double rnhpts, double* out,
                                                     int stride) {
  const int k = blockIdx.x + 1, q = blockIdx.y;
  const T* __restrict__ p = f.p[q] + (long long)(k - 1) * plane;
  double acc = 0.0;
  for (long long t = threadIdx.x; t < plane; t += blockDim.x) acc += (double)__ldg(p + t);
  __shared__ double sh[256];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[q * stride + k] = sh[0] * rnhpts;
}

// rnhpts of meanprofiles.F90:44: the point count converted at default (single) precision
static double rnhpts(const Scalars& s) { return 1.0 / (double)(float)((long long)s.nx * s.ny); }

template <typename T>
int launch_mean_profiles(const Scalars& s, const T* zu, const T* zv, const T* th, const T* const* q, double* olz,
                         cudaStream_t st) {
  MeanFields<T> f;
  f.p[0] = zu;
  f.p[1] = zv;
  f.p[2] = th;
  for (int n = 0; n < s.nq; ++n) f.p[3 + n] = q[n];
  k_plane_means<T><<<dim3(s.nz, 3 + s.nq), 256, 0, st>>>(f, s.plane, rnhpts(s), olz, s.nz + 2);
  return 1;
}
template int launch_mean_profiles<float>(const Scalars&, const float*, const float*, const float*, const float* const*,
                                         double*, cudaStream_t);
template int launch_mean_profiles<double>(const Scalars&, const double*, const double*, const double*,
                                          const double* const*, double*, cudaStream_t);

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
