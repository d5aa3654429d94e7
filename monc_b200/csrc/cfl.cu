// The reductions cfltest reads (cfltest.F90:62-128, 193-222).
//
// MONC gathers them column by column while it steps: stepfields (stepfields.F90:372-393) takes
// the extrema of zu and zv over levels 2..nz and the maximum |zw| per level 2..nz-1 before
// stepping, and smagorinsky (smagorinsky.F90:143-173) the maximum of
// max(vis, diff) * (rdzn(k+1)^2 + cx2 + cy2) over levels 2..nz-1.  cfltest then scales
// abswmax(k) by rdzn(k+1) and takes the maximum over k; since rdzn > 0 and rounding is monotonic,
// max_k(max|zw| * rdzn(k+1)) equals the maximum over points of |zw| * rdzn(k+1), which is what is
// reduced here.  Minimum and maximum are exact in any order, so the result does not depend on the
// launch shape.  Products and sums are written with explicit round-to-nearest intrinsics so that
// no multiply-add is contracted (MONC evaluates them separately rounded).
#include <cfloat>

#include "dycore.h"

namespace mgpu {

constexpr int CFL_THREADS = 256;

// part[b*6 + q]: q = 0 min zu, 1 max zu, 2 min zv, 3 max zv, 4 max |zw| rdzn(k+1),
// 5 max max(vis, diff) (rdzn(k+1)^2 + cx2 + cy2)
template <typename T>
__global__ void __launch_bounds__(CFL_THREADS) k_cfl_partial(Scalars s, const T* __restrict__ zu,
                                                             const T* __restrict__ zv, const T* __restrict__ zw,
                                                             const T* __restrict__ vis, const T* __restrict__ diff,
                                                             int with_vis, int halo, double* __restrict__ part) {
  const double* rdzn = s.prof + P_RDZN * (s.nz + 2);
  double r0 = DBL_MAX, r1 = -DBL_MAX, r2 = DBL_MAX, r3 = -DBL_MAX, r4 = 0.0, r5 = 0.0;
  // levels 2..nz of the rows halo..ny-halo-1 (a y-slab leaves its halo rows to its neighbours)
  const long long rows = (long long)(s.ny - 2 * halo) * s.nx;
  const long long n = (long long)(s.nz - 1) * rows;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += stride) {
    const long long lev = t / rows;
    const long long o = (lev + 1) * s.plane + (long long)halo * s.nx + (t - lev * rows);
    const int k = (int)lev + 2;
    const double u = (double)zu[o], v = (double)zv[o];
    r0 = u < r0 ? u : r0;
    r1 = u > r1 ? u : r1;
    r2 = v < r2 ? v : r2;
    r3 = v > r3 ? v : r3;
    if (k <= s.nz - 1) {
      const double rz = rdzn[k + 1];
      const double cz = __dmul_rn(fabs((double)zw[o]), rz);
      r4 = cz > r4 ? cz : r4;
      if (with_vis) {
        const double a = (double)vis[o], b = (double)diff[o];
        const double fac = __dadd_rn(__dadd_rn(__dmul_rn(rz, rz), s.cx2), s.cy2);
        const double cv = __dmul_rn(a > b ? a : b, fac);
        r5 = cv > r5 ? cv : r5;
      }
    }
  }
  __shared__ double sh[6][CFL_THREADS];
  const int t = threadIdx.x;
  sh[0][t] = r0; sh[1][t] = r1; sh[2][t] = r2; sh[3][t] = r3; sh[4][t] = r4; sh[5][t] = r5;
  __syncthreads();
  for (int h = CFL_THREADS / 2; h > 0; h >>= 1) {
    if (t < h) {
      sh[0][t] = sh[0][t + h] < sh[0][t] ? sh[0][t + h] : sh[0][t];
      sh[2][t] = sh[2][t + h] < sh[2][t] ? sh[2][t + h] : sh[2][t];
      sh[1][t] = sh[1][t + h] > sh[1][t] ? sh[1][t + h] : sh[1][t];
      sh[3][t] = sh[3][t + h] > sh[3][t] ? sh[3][t + h] : sh[3][t];
      sh[4][t] = sh[4][t + h] > sh[4][t] ? sh[4][t + h] : sh[4][t];
      sh[5][t] = sh[5][t + h] > sh[5][t] ? sh[5][t + h] : sh[5][t];
    }
    __syncthreads();
  }
  if (t < 6) part[(long long)blockIdx.x * 6 + t] = sh[t][0];
}

__global__ void __launch_bounds__(CFL_THREADS) k_cfl_final(const double* __restrict__ part, int nblk,
                                                           double* __restrict__ out) {
  __shared__ double sh[6][CFL_THREADS];
  const int t = threadIdx.x;
  double r[6] = {DBL_MAX, -DBL_MAX, DBL_MAX, -DBL_MAX, 0.0, 0.0};
  for (int b = t; b < nblk; b += CFL_THREADS)
    for (int q = 0; q < 6; ++q) {
      const double x = part[(long long)b * 6 + q];
      const bool lower = (q == 0 || q == 2);
      r[q] = lower ? (x < r[q] ? x : r[q]) : (x > r[q] ? x : r[q]);
    }
  for (int q = 0; q < 6; ++q) sh[q][t] = r[q];
  __syncthreads();
  for (int h = CFL_THREADS / 2; h > 0; h >>= 1) {
    if (t < h)
      for (int q = 0; q < 6; ++q) {
        const bool lower = (q == 0 || q == 2);
        const double a = sh[q][t], b = sh[q][t + h];
        sh[q][t] = lower ? (b < a ? b : a) : (b > a ? b : a);
      }
    __syncthreads();
  }
  if (t < 6) out[t] = sh[t][0];
}

// The six values in the form a maximum reduces: the minima negated (negation is exact, so
// -max(-a, -b) = min(a, b)).  Its own inverse.
__global__ void k_cfl_max_form(const double* __restrict__ src, double* __restrict__ dst) {
  const int q = threadIdx.x;
  if (q < 6) dst[q] = (q == 0 || q == 2) ? -src[q] : src[q];
}

template <typename T>
int launch_cfl_gather(const Scalars& s, const DevState<T>& d, bool with_vis, double* part, double* out,
                      cudaStream_t st, int halo) {
  k_cfl_partial<T><<<CFL_BLOCKS, CFL_THREADS, 0, st>>>(s, d.zu, d.zv, d.zw, d.vis, d.diff, with_vis ? 1 : 0, halo,
                                                       part);
  k_cfl_final<<<1, CFL_THREADS, 0, st>>>(part, CFL_BLOCKS, out);
  return 2;
}

int launch_cfl_max_form(const double* src, double* dst, cudaStream_t st) {
  k_cfl_max_form<<<1, 32, 0, st>>>(src, dst);
  return 1;
}

// diverr's divergence error (diverr.F90:69-82, 120-175): max |p| over levels 2..nz of the rows
// halo .. ny-halo-1, p = (cx du + cy dv + 4 (tzc2 w_k - tzc1 w_{k-1})) timec from the velocities the
// step starts from (u, v, w forward; zu, zv, zw centred).  A block maximum, then one atomicMax on
// the bit pattern (non-negative doubles order as their bits do).
template <typename T>
__global__ void __launch_bounds__(CFL_THREADS) k_divmax(Scalars s, const T* __restrict__ u, const T* __restrict__ v,
                                                        const T* __restrict__ w, int halo,
                                                        unsigned long long* __restrict__ out) {
  const double* tzc1 = s.prof + P_TZC1 * (s.nz + 2);
  const double* tzc2 = s.prof + P_TZC2 * (s.nz + 2);
  const T timec = s.forward ? (T)(1.0 / s.dtm) : (T)(1.0 / (2.0 * s.dtm));
  const long long rows = (long long)(s.ny - 2 * halo) * s.nx;
  const long long n = (long long)(s.nz - 1) * rows;
  double m = 0.0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const long long lev = t / rows, r = t - lev * rows;
    const int k = (int)lev + 2, j = halo + (int)(r / s.nx), i = (int)(r % s.nx);
    const int iw = i == 0 ? s.nx - 1 : i - 1, js = j == 0 ? s.ny - 1 : j - 1;
    const long long o = (long long)(k - 1) * s.plane + (long long)j * s.nx + i;
    T pp = (T)0.0;
    pp = pp + (T)s.cx * (u[o] - u[o - i + iw]);
    pp = pp + (T)s.cy * (v[o] - v[o + (long long)(js - j) * s.nx]);
    pp = pp + (T)4.0 * ((T)tzc2[k] * w[o] - (T)tzc1[k] * w[o - s.plane]);
    pp = pp * timec;
    const double a = fabs((double)pp);
    m = a > m ? a : m;
  }
  for (int off = 16; off; off >>= 1) {
    const double o2 = __shfl_down_sync(0xffffffffu, m, off);
    m = o2 > m ? o2 : m;
  }
  __shared__ double sh[CFL_THREADS / 32];
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 1; q < CFL_THREADS / 32; ++q) m = sh[q] > m ? sh[q] : m;
    atomicMax(out, (unsigned long long)__double_as_longlong(m));
  }
}

template <typename T>
int launch_divmax(const Scalars& s, const DevState<T>& d, unsigned long long* out, cudaStream_t st, int halo) {
  const bool fwd = s.forward != 0;
  k_divmax<T><<<CFL_BLOCKS, CFL_THREADS, 0, st>>>(s, fwd ? d.u : d.zu, fwd ? d.v : d.zv, fwd ? d.w : d.zw, halo, out);
  return 1;
}
template int launch_divmax<double>(const Scalars&, const DevState<double>&, unsigned long long*, cudaStream_t, int);
template int launch_divmax<float>(const Scalars&, const DevState<float>&, unsigned long long*, cudaStream_t, int);

template int launch_cfl_gather<double>(const Scalars&, const DevState<double>&, bool, double*, double*, cudaStream_t,
                                       int);
template int launch_cfl_gather<float>(const Scalars&, const DevState<float>&, bool, double*, double*, cudaStream_t,
                                      int);

}  // namespace mgpu
