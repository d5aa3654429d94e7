// Spectral pressure solve (fftsolver.F90:129-309): horizontal FFTs in shared memory and a
// column-per-thread FP64 Thomas solve per horizontal wavenumber.
//
//   forward x : pairs of real rows packed as one complex row, radix-2 FFT in shared memory,
//               split into the two half spectra (kx = 0..nx/2)
//   forward y : complex FFT along y of a tile of kx columns
//   tridiag   : per (kx, ky) column, b(k) = cos_x + cos_y + czg(k) with the Thomas pivots
//               precomputed in FP64 on the host exactly as fftsolver.F90:259-293 forms them;
//               the horizontal-mean mode is integrated upward (fftsolver.F90:294-308)
//   inverse y, inverse x (imaginary parts of the kx = 0 and kx = nx/2 bins are dropped, as the
//               Hermitian completion of fftnorth.F90:54-73 drops them)
// MONC transforms y first and stores real and imaginary parts separately ("real-interleaved",
// pencilfft.F90:276-332); the solve is linear with real coefficients that depend only on
// |kx|, |ky|, so this complex half-spectrum form gives the same field up to rounding.
// Level 1 is transformed too: its non-mean modes pass through unchanged, its mean is zeroed.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include <mutex>

#include "dycore.h"

namespace mgpu {

template <typename T> struct Cx;
template <> struct Cx<double> { typedef double2 t; };
template <> struct Cx<float> { typedef float2 t; };

template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  C r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { C r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { C r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }

static int ilog2(int n) { int l = 0; while ((1 << l) < n) ++l; return l; }

// ---- line FFTs: Stockham autosort passes, radix 16 in registers -----------------------------
// An N-point complex transform (N = 2^LOGN) of one line is done by G = N/E threads holding E =
// min(N, 16) points each.  Pass p has radix R_p (16, the last pass 2^(LOGN mod 4) when LOGN is
// not a multiple of 4) and span NS_p = R_0*...*R_{p-1}: a thread's butterflies are jb = j + G*b,
// b < E/R_p, each on the points x[jb + r*N/R_p] (r < R_p), multiplied by W_{NS*R}^{(jb mod NS)*r},
// transformed by an R_p-point DFT in registers and stored to y[(jb/NS)*NS*R + jb mod NS + r*NS]
// (the self-sorting Stockham form: the output of the last pass is in natural order).  The first
// pass reads the line from wherever the caller's accessor points (global memory or shared
// memory), passes in between go through a padded shared-memory copy of the line, and the last
// pass hands each result to the caller's accessor.  W_N^m = e^{-2 pi i m / N} (forward) or its
// conjugate (inverse); inverse transforms are unscaled.
template <int LOGN>
struct LineShape {
  static constexpr int N = 1 << LOGN;
  static constexpr int E = N < 16 ? N : 16;
  static constexpr int G = N / E;
  static constexpr int P = (LOGN + 3) / 4;
  static constexpr int RL = 1 << (LOGN - 4 * (P - 1));   // radix of the last pass
  static constexpr int R(int p) { return p < P - 1 ? 16 : RL; }
  static constexpr int NS(int p) { return p == 0 ? 1 : (p == 1 ? R(0) : R(0) * R(1)); }
  static constexpr int LPL = N + N / 16 + 1;  // padded line length in shared memory (elements)
};
// shared-memory index of point i of a line: one element of padding after every 16, so that the
// first pass's stores (stride 16 between threads) fall in different banks
__device__ __forceinline__ int lpad(int i) { return i + (i >> 4); }

__host__ __device__ constexpr int brev_c(int i, int r) {
  int o = 0;
  for (int b = 1; b < r; b <<= 1) { o = (o << 1) | (i & 1); i >>= 1; }
  return o;
}

// b * W16^t (t < 8), conjugated twiddle when INV; t is a constant after unrolling
template <typename C, bool INV>
__device__ __forceinline__ C mul_w16(C b, int t) {
  typedef decltype(b.x) T;
  const T c1 = (T)0.92387953251128675613, s1 = (T)0.38268343236508977173, r2 = (T)0.70710678118654752440;
  if (t == 0) return b;
  C o;
  if (t == 4) {  // W16^4 = -i
    if (!INV) { o.x = b.y; o.y = -b.x; } else { o.x = -b.y; o.y = b.x; }
    return o;
  }
  T wr, wi;
  switch (t) {
    case 1: wr = c1; wi = -s1; break;
    case 2: wr = r2; wi = -r2; break;
    case 3: wr = s1; wi = -c1; break;
    case 5: wr = -s1; wi = -c1; break;
    case 6: wr = -r2; wi = -r2; break;
    default: wr = -c1; wi = -s1; break;
  }
  if (INV) wi = -wi;
  o.x = b.x * wr - b.y * wi;
  o.y = b.x * wi + b.y * wr;
  return o;
}

// R-point DFT (R <= 16) of u[0..R-1] in registers, natural order in and out (radix-2 DIT)
template <typename C, int R, bool INV>
__device__ __forceinline__ void dft_reg(C* u) {
  C w[R];
#pragma unroll
  for (int i = 0; i < R; ++i) w[i] = u[brev_c(i, R)];
#pragma unroll
  for (int h = 1; h < R; h <<= 1)
#pragma unroll
    for (int s = 0; s < R; s += 2 * h)
#pragma unroll
      for (int q = 0; q < h; ++q) {
        const C a = w[s + q];
        const C b = mul_w16<C, INV>(w[s + q + h], q * (R / (2 * h)) * (16 / R));
        w[s + q] = cadd(a, b);
        w[s + q + h] = csub(a, b);
      }
#pragma unroll
  for (int i = 0; i < R; ++i) u[i] = w[i];
}

template <typename C, bool INV>
__device__ __forceinline__ C mul_tw(C a, C w) {
  if (INV) w.y = -w.y;
  return cmul(a, w);
}

template <int N, int G, int E, int R, class In, class C>
__device__ __forceinline__ void pass_load(int j, In in, C* v) {
#pragma unroll
  for (int b = 0; b < E / R; ++b)
#pragma unroll
    for (int r = 0; r < R; ++r) v[b * R + r] = in(j + G * b + r * (N / R));
}

template <int N, int G, int E, int R, int NS, bool INV, class Out, class C>
__device__ __forceinline__ void pass_compute_store(int j, const C* __restrict__ tw, C* v, Out out) {
#pragma unroll
  for (int b = 0; b < E / R; ++b) {
    const int jb = j + G * b, k = jb & (NS - 1);
    C* u = v + b * R;
    if (NS > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) u[r] = mul_tw<C, INV>(u[r], __ldg(tw + k * r * (N / (NS * R))));
    }
    dft_reg<C, R, INV>(u);
    const int base = (jb / NS) * NS * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) out(base + r * NS, u[r]);
  }
}

// The transform of one line by its G threads (thread j of the line).  in(i) returns point i of
// the input, out(i, z) receives point i of the result.  IN_SMEM / OUT_SMEM say that in / out
// touch this line's shared-memory copy `line`, so that the pass separates them from its own
// shared-memory traffic with barriers.  Every thread of the block must call it.
template <typename C, int LOGN, bool INV, bool IN_SMEM, bool OUT_SMEM, class In, class Out>
__device__ __forceinline__ void line_fft(int j, C* line, const C* __restrict__ tw, In in, Out out) {
  typedef LineShape<LOGN> S;
  constexpr int N = S::N, G = S::G, E = S::E, P = S::P;
  C v[E];
  auto sm_in = [&](int i) { return line[lpad(i)]; };
  auto sm_out = [&](int i, C z) { line[lpad(i)] = z; };
  pass_load<N, G, E, S::R(0)>(j, in, v);
  if constexpr (P == 1) {
    if (IN_SMEM && OUT_SMEM) __syncthreads();
    pass_compute_store<N, G, E, S::R(0), 1, INV>(j, tw, v, out);
  } else {
    if (IN_SMEM) __syncthreads();
    pass_compute_store<N, G, E, S::R(0), 1, INV>(j, tw, v, sm_out);
    __syncthreads();
    pass_load<N, G, E, S::R(1)>(j, sm_in, v);
    if constexpr (P == 2) {
      if (OUT_SMEM) __syncthreads();
      pass_compute_store<N, G, E, S::R(1), S::NS(1), INV>(j, tw, v, out);
    } else {
      __syncthreads();
      pass_compute_store<N, G, E, S::R(1), S::NS(1), INV>(j, tw, v, sm_out);
      __syncthreads();
      pass_load<N, G, E, S::R(2)>(j, sm_in, v);
      if (OUT_SMEM) __syncthreads();
      pass_compute_store<N, G, E, S::R(2), S::NS(2), INV>(j, tw, v, out);
    }
  }
}

// threads per block and lines per block of the line-FFT kernels
__host__ __device__ constexpr int line_block(int logn) {
  return ((1 << logn) / ((1 << logn) < 16 ? (1 << logn) : 16)) > 128 ? ((1 << logn) / 16) : 128;
}
__host__ __device__ constexpr int line_lines(int logn) {
  return line_block(logn) / ((1 << logn) / ((1 << logn) < 16 ? (1 << logn) : 16));
}

// Offset of wavenumber m of row j, level k in an x-spectrum split into nblk blocks of
// consecutive wavenumbers: the nxh wavenumbers are dealt out as evenly as possible, the first
// nxh % nblk blocks one wider.  Block q covers k0_q .. k0_q+w_q-1, is [nz][ny][w_q] and starts at
// k0_q*nz*ny, so the blocks lie end to end.  *w receives w_q (the row stride inside the block).
__device__ __forceinline__ long long spec_x_offset(int m, int nxh, int nblk, int ny, int nz, int k, int j, int* w) {
  int k0 = 0, c = m, wq = nxh;
  if (nblk > 1) {
    const int b = nxh / nblk, rem = nxh - b * nblk, split = rem * (b + 1);
    if (m < split) {
      const int q = m / (b + 1);
      k0 = q * (b + 1);
      wq = b + 1;
    } else {
      const int q = (m - split) / b;
      k0 = split + q * b;
      wq = b;
    }
    c = m - k0;
  }
  *w = wq;
  return (long long)k0 * nz * ny + ((long long)(k - 1) * ny + j) * wq + c;
}

// ---- forward x: real rows (k, j), (k, j+1) -> half spectra ------------------------------
// ny rows of each level are transformed: rows p_row0 .. p_row0+ny-1 of p, which holds p_rows rows
// per level (a y-slab with halo rows has p_rows > ny).  Two real rows are packed as the real and
// imaginary parts of one complex line and separated after the transform.  The spectrum is split
// into nblk blocks of consecutive wavenumbers (see spec_x_offset); nblk = 1 gives the plain
// [nz][ny][nx/2+1] layout.
template <typename T, int LOGN>
__global__ void __launch_bounds__(line_block(LOGN)) k_fft_x_fwd(const T* __restrict__ p, typename Cx<T>::t* __restrict__ spec,
                                                              const typename Cx<T>::t* __restrict__ tw, int ny, int nz,
                                                              int p_rows, int p_row0, int nblk) {
  typedef typename Cx<T>::t C;
  typedef LineShape<LOGN> S;
  constexpr int N = S::N, G = S::G, L = line_lines(LOGN);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int line = threadIdx.x / G, j = threadIdx.x - line * G;
  C* buf = reinterpret_cast<C*>(smem_raw) + line * S::LPL;
  const int pairs = ny / 2;
  const long long pr = (long long)blockIdx.x * L + line;
  const bool ok = pr < (long long)nz * pairs;
  const int k = ok ? (int)(pr / pairs) + 1 : 1, jr = ok ? 2 * (int)(pr % pairs) : 0;
  const T* row = p + ((long long)(k - 1) * p_rows + p_row0 + jr) * N;
  auto in = [&](int e) {
    C z;
    if (ok) { z.x = row[e]; z.y = row[N + e]; } else { z.x = (T)0; z.y = (T)0; }
    return z;
  };
  auto out = [&](int i, C z) { buf[lpad(i)] = z; };
  line_fft<C, LOGN, false, false, true>(j, buf, tw, in, out);
  __syncthreads();
  if (!ok) return;
  constexpr int nxh = N / 2 + 1;
  for (int m = j; m < nxh; m += G) {
    const C zm = buf[lpad(m)];
    const C zn = buf[lpad((N - m) & (N - 1))];
    C a, b;
    a.x = (T)0.5 * (zm.x + zn.x);
    a.y = (T)0.5 * (zm.y - zn.y);
    b.x = (T)0.5 * (zm.y + zn.y);
    b.y = (T)0.5 * (zn.x - zm.x);
    int w;
    C* o = spec + spec_x_offset(m, nxh, nblk, ny, nz, k, jr, &w);
    o[0] = a;
    o[w] = b;
  }
}

// ---- forward x of the pressure source, formed on the fly ------------------------------------
// The fused step's source p = (cx (zu(i) - zu(i-1)) + cy (zv(j) - zv(j-1)) + 4 (tzc2 zw(k) -
// tzc1 zw(k-1))) * timec (k_f_pressure_source, the same expression in the same order) is
// computed for a row pair straight into its shared-memory line, which the x transform then
// reads: the source never goes through global memory.  One domain (all ny rows), plain
// [nz][ny][nx/2+1] spectrum.
template <typename T, int LOGN>
__global__ void __launch_bounds__(line_block(LOGN)) k_fft_x_fwd_src(Scalars s, SourceFields<T> f,
                                                                  typename Cx<T>::t* __restrict__ spec,
                                                                  const typename Cx<T>::t* __restrict__ tw) {
  typedef typename Cx<T>::t C;
  typedef LineShape<LOGN> S;
  constexpr int N = S::N, G = S::G, L = line_lines(LOGN);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int line = threadIdx.x / G, j = threadIdx.x - line * G;
  C* buf = reinterpret_cast<C*>(smem_raw) + line * S::LPL;
  const int ny = s.ny, nz = s.nz, pairs = ny / 2;
  const long long pr = (long long)blockIdx.x * L + line;
  const bool ok = pr < (long long)nz * pairs;
  const int k = ok ? (int)(pr / pairs) + 1 : 1, jr = ok ? 2 * (int)(pr % pairs) : 0;
  const long long plane = s.plane;
  const T timec = s.forward ? (T)(1.0 / s.dtm) : (T)(1.0 / (2.0 * s.dtm));
  const T cx = (T)s.cx, cy = (T)s.cy;
  const T tzc1 = (T)__ldg(s.prof + P_TZC1 * (nz + 2) + k), tzc2 = (T)__ldg(s.prof + P_TZC2 * (nz + 2) + k);
  const long long lv = (long long)(k - 1) * plane;
  const int jm = jr == 0 ? ny - 1 : jr - 1;
  const T* __restrict__ u0 = f.zu + lv + (long long)jr * N;
  const T* __restrict__ u1 = u0 + N;
  const T* __restrict__ vm = f.zv + lv + (long long)jm * N;
  const T* __restrict__ v0 = f.zv + lv + (long long)jr * N;
  const T* __restrict__ v1 = v0 + N;
  const T* __restrict__ w0 = f.zw + lv + (long long)jr * N;
  const T* __restrict__ w1 = w0 + N;
  auto src = [&](const T* u, const T* vlo, const T* v, const T* w, int e) {
    const int em = e == 0 ? N - 1 : e - 1;
    T pp = (T)0.0;
    pp = pp + cx * (__ldg(u + e) - __ldg(u + em));
    pp = pp + cy * (__ldg(v + e) - __ldg(vlo + e));
    pp = pp + (T)4.0 * (tzc2 * __ldg(w + e) - tzc1 * __ldg(w - plane + e));
    return pp * timec;
  };
#pragma unroll 4
  for (int q = 0; q < N / G; ++q) {
    const int e = j + q * G;
    C z;
    if (ok && k > 1) {
      z.x = src(u0, vm, v0, w0, e);
      z.y = src(u1, v0, v1, w1, e);
    } else {
      z.x = (T)0;
      z.y = (T)0;
    }
    buf[lpad(e)] = z;
  }
  __syncthreads();  // the line's points come from all G threads of the line
  auto in = [&](int i) { return buf[lpad(i)]; };
  auto out = [&](int i, C z) { buf[lpad(i)] = z; };
  line_fft<C, LOGN, false, true, true>(j, buf, tw, in, out);
  __syncthreads();
  if (!ok) return;
  constexpr int nxh = N / 2 + 1;
  for (int m = j; m < nxh; m += G) {
    const C zm = buf[lpad(m)];
    const C zn = buf[lpad((N - m) & (N - 1))];
    C a, b;
    a.x = (T)0.5 * (zm.x + zn.x);
    a.y = (T)0.5 * (zm.y - zn.y);
    b.x = (T)0.5 * (zm.y + zn.y);
    b.y = (T)0.5 * (zn.x - zm.x);
    C* o = spec + ((long long)(k - 1) * ny + jr) * nxh + m;
    o[0] = a;
    o[nxh] = b;
  }
}

// ---- inverse x: half spectra -> real rows (k, j), (k, j+1) -----------------------------
// the inverse of k_fft_x_fwd, with the same row window and spectrum blocks; the imaginary parts
// of the kx = 0 and kx = nx/2 bins are dropped (the Hermitian completion of fftnorth.F90:54-73)
template <typename T, int LOGN>
__global__ void __launch_bounds__(line_block(LOGN)) k_fft_x_inv(T* __restrict__ p, const typename Cx<T>::t* __restrict__ spec,
                                                              const typename Cx<T>::t* __restrict__ tw, int ny, int nz,
                                                              int p_rows, int p_row0, int nblk) {
  typedef typename Cx<T>::t C;
  typedef LineShape<LOGN> S;
  constexpr int N = S::N, G = S::G, L = line_lines(LOGN);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int line = threadIdx.x / G, j = threadIdx.x - line * G;
  C* buf = reinterpret_cast<C*>(smem_raw) + line * S::LPL;
  const int pairs = ny / 2;
  const long long pr = (long long)blockIdx.x * L + line;
  const bool ok = pr < (long long)nz * pairs;
  const int k = ok ? (int)(pr / pairs) + 1 : 1, jr = ok ? 2 * (int)(pr % pairs) : 0;
  constexpr int nxh = N / 2 + 1, NM = (nxh + G - 1) / G;
  // every bin this thread needs is loaded before the first is used, so that the loads are in
  // flight together rather than one DRAM round trip per bin
  C av[NM], bv[NM];
#pragma unroll
  for (int q = 0; q < NM; ++q) {
    const int m = j + q * G;
    if (ok && m < nxh) {
      int w;
      const C* in = spec + spec_x_offset(m, nxh, nblk, ny, nz, k, jr, &w);
      av[q] = in[0];
      bv[q] = in[w];
    } else {
      av[q].x = av[q].y = bv[q].x = bv[q].y = (T)0;
    }
  }
#pragma unroll
  for (int q = 0; q < NM; ++q) {
    const int m = j + q * G;
    if (m >= nxh) break;
    C a = av[q], b = bv[q];
    if (m == 0 || m == N / 2) { a.y = (T)0; b.y = (T)0; }
    C z;
    z.x = a.x - b.y;
    z.y = a.y + b.x;
    buf[lpad(m)] = z;
    if (m > 0 && m < N / 2) {
      C zc;
      zc.x = a.x + b.y;
      zc.y = b.x - a.y;
      buf[lpad(N - m)] = zc;
    }
  }
  __syncthreads();
  T* row = p + ((long long)(k - 1) * p_rows + p_row0 + jr) * N;
  const T sc = (T)(1.0 / (double)N);
  auto in = [&](int i) { return buf[lpad(i)]; };
  auto out = [&](int e, C z) {
    if (ok) { row[e] = z.x * sc; row[N + e] = z.y * sc; }
  };
  line_fft<C, LOGN, true, true, false>(j, buf, tw, in, out);
}

// ---- complex FFT along y on a tile of kx columns ------------------------------------------
// The spectrum holds ncols kx columns per row (nx/2+1, or one block of them after a transpose) and
// its ny rows in blocks of rpb rows: block b is [nz][rpb][ncols] and starts at b*nz*rpb*ncols.
// rpb = ny gives the plain [nz][ny][ncols] layout.
__device__ __forceinline__ long long spec_row(int e, int k, int rpb, int ncols, int nz) {
  const int b = e < rpb ? 0 : e / rpb;
  return ((long long)b * nz + (k - 1)) * rpb * ncols + (long long)(e - b * rpb) * ncols;
}

// One block per (tile of kx columns, level); consecutive threads take consecutive columns, so
// the first pass's loads and the last pass's stores are coalesced across the tile.  The inverse
// transform is scaled by 1/ny.
template <typename T, int LOGN, bool INV>
__global__ void __launch_bounds__(line_block(LOGN)) k_fft_y(typename Cx<T>::t* __restrict__ spec,
                                                          const typename Cx<T>::t* __restrict__ tw, int ncols, int nz,
                                                          int rpb) {
  typedef typename Cx<T>::t C;
  typedef LineShape<LOGN> S;
  constexpr int N = S::N, COLS = line_lines(LOGN);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int c = threadIdx.x % COLS, j = threadIdx.x / COLS;
  C* buf = reinterpret_cast<C*>(smem_raw) + c * S::LPL;
  const int kx = blockIdx.x * COLS + c, k = blockIdx.y + 1;
  const bool ok = kx < ncols;
  C* col = spec + kx;
  auto in = [&](int e) {
    C z;
    if (ok) z = col[spec_row(e, k, rpb, ncols, nz)];
    else { z.x = (T)0; z.y = (T)0; }
    return z;
  };
  const T sc = INV ? (T)(1.0 / (double)N) : (T)1.0;
  auto out = [&](int e, C z) {
    if (!ok) return;
    if (INV) { z.x = z.x * sc; z.y = z.y * sc; }
    col[spec_row(e, k, rpb, ncols, nz)] = z;
  };
  line_fft<C, LOGN, INV, false, false>(j, buf, tw, in, out);
}

// ---- lengths that are not powers of two: mixed-radix Stockham passes in shared memory ---------
// MONC's FFTPACK factorises any length (cffti1.f90 tries 4, 2, 3, 5, then odd factors); the
// lengths with prime factors 2, 3 and 5 only (96, 384, 100, 360, ...) take these kernels.  A line
// of n points sits in shared memory (two buffers, ping-pong) and is transformed by the threads of
// its block: pass p of radix R (4, 2, 3 or 5) and span NS forms, for j < n/R, the R points
// x[j + r n/R], multiplies point r by W_{NS R}^{(j mod NS) r} = tw[(j mod NS) r n/(NS R)] (the
// same table of W_n^q the power-of-two kernels use), applies the R-point DFT and stores point r
// to y[(j/NS) NS R + j mod NS + r NS] -- the self-sorting form of the radix-16 passes above with
// the radix varying from pass to pass, so the last pass leaves the result in natural order.
struct GenFactors {
  int n, npass;
  int radix[16];
};

// factors of n in the order the passes use them (4s, then 2, 3s, 5s); false if n has another
// prime factor or is out of range
static bool gen_factor(int n, GenFactors& g) {
  g.n = n;
  g.npass = 0;
  if (n < 2 || n > 4096) return false;
  int m = n;
  while (m % 4 == 0) { g.radix[g.npass++] = 4; m /= 4; }
  while (m % 2 == 0) { g.radix[g.npass++] = 2; m /= 2; }
  while (m % 3 == 0) { g.radix[g.npass++] = 3; m /= 3; }
  while (m % 5 == 0) { g.radix[g.npass++] = 5; m /= 5; }
  return m == 1 && g.npass <= 16;
}

// the R-point DFTs; forward uses W_R = e^{-2 pi i / R}, inverse its conjugate.  The constants are
// cos and sin of 2 pi/3, 2 pi/5 and 4 pi/5 to 30 digits.
template <typename C>
__device__ __forceinline__ C cmul_i(C a, bool inv) {  // a * (-i) forward, a * (+i) inverse
  C r;
  if (inv) { r.x = -a.y; r.y = a.x; } else { r.x = a.y; r.y = -a.x; }
  return r;
}
template <typename C, typename T>
__device__ __forceinline__ C cscale(C a, T s) { C r; r.x = a.x * s; r.y = a.y * s; return r; }

template <typename T, typename C>
__device__ __forceinline__ void gen_dft(C* v, int R, bool inv) {
  if (R == 2) {
    const C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if (R == 4) {
    const C t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]), t2 = cadd(v[1], v[3]);
    const C t3 = cmul_i(csub(v[1], v[3]), inv);
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3);
    v[3] = csub(t1, t3);
  } else if (R == 3) {
    const T c = (T)-0.5;
    const T sn = inv ? (T)0.866025403784438646763723170753 : (T)-0.866025403784438646763723170753;
    const C t1 = cadd(v[1], v[2]);
    const C t2 = cadd(v[0], cscale(t1, c));
    const C d = cscale(csub(v[1], v[2]), sn);  // i * d is added to y1
    C y1, y2;
    y1.x = t2.x - d.y; y1.y = t2.y + d.x;
    y2.x = t2.x + d.y; y2.y = t2.y - d.x;
    v[0] = cadd(v[0], t1);
    v[1] = y1;
    v[2] = y2;
  } else {  // R == 5
    const T c1 = (T)0.309016994374947424102293417183, c2 = (T)-0.809016994374947424102293417183;
    const T s1 = inv ? (T)0.951056516295153572116439333379 : (T)-0.951056516295153572116439333379;
    const T s2 = inv ? (T)0.587785252292473129180916317273 : (T)-0.587785252292473129180916317273;
    const C a1 = cadd(v[1], v[4]), a2 = cadd(v[2], v[3]);
    const C b1 = csub(v[1], v[4]), b2 = csub(v[2], v[3]);
    const C x0 = v[0];
    const C r1 = cadd(x0, cadd(cscale(a1, c1), cscale(a2, c2)));
    const C r2 = cadd(x0, cadd(cscale(a1, c2), cscale(a2, c1)));
    const C q1 = cadd(cscale(b1, s1), cscale(b2, s2));   // y1 = r1 + i q1, y4 = r1 - i q1
    const C q2 = csub(cscale(b1, s2), cscale(b2, s1));   // y2 = r2 + i q2, y3 = r2 - i q2
    v[0] = cadd(x0, cadd(a1, a2));
    v[1].x = r1.x - q1.y; v[1].y = r1.y + q1.x;
    v[4].x = r1.x + q1.y; v[4].y = r1.y - q1.x;
    v[2].x = r2.x - q2.y; v[2].y = r2.y + q2.x;
    v[3].x = r2.x + q2.y; v[3].y = r2.y - q2.x;
  }
}

// Transform `nl` lines of n points held at a + l*n (l < nl) in shared memory; b is scratch of the
// same size.  Returns the buffer holding the result.  All threads of the block take part.
template <typename T, bool INV>
__device__ typename Cx<T>::t* gen_lines_fft(typename Cx<T>::t* a, typename Cx<T>::t* b, int nl, const GenFactors& g,
                                            const typename Cx<T>::t* __restrict__ tw) {
  typedef typename Cx<T>::t C;
  const int n = g.n;
  int ns = 1;
  for (int p = 0; p < g.npass; ++p) {
    const int R = g.radix[p], nb = n / R, step = n / (ns * R);
    for (int t = threadIdx.x; t < nl * nb; t += blockDim.x) {
      const int l = t / nb, j = t - l * nb;
      const C* x = a + l * n;
      C* y = b + l * n;
      const int jm = j % ns;
      C v[5];
      for (int r = 0; r < R; ++r) {
        C z = x[j + r * nb];
        if (r > 0 && jm > 0) {
          C w = tw[jm * r * step];
          if (INV) w.y = -w.y;
          z = cmul(z, w);
        }
        v[r] = z;
      }
      gen_dft<T, C>(v, R, INV);
      const int o = (j / ns) * ns * R + jm;
      for (int r = 0; r < R; ++r) y[o + r * ns] = v[r];
    }
    __syncthreads();
    C* tmp = a; a = b; b = tmp;
    ns *= R;
  }
  return a;
}

constexpr int GEN_BLOCK = 128;

// forward x of generic length: one block per row pair, packed, transformed and split as
// k_fft_x_fwd does it
template <typename T>
__global__ void __launch_bounds__(GEN_BLOCK) k_fftg_x_fwd(const T* __restrict__ p, typename Cx<T>::t* __restrict__ spec,
                                                          const typename Cx<T>::t* __restrict__ tw, GenFactors g, int ny,
                                                          int nz, int p_rows, int p_row0, int nblk) {
  typedef typename Cx<T>::t C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = g.n, nxh = n / 2 + 1, pairs = ny / 2;
  C* a = reinterpret_cast<C*>(smem_raw);
  C* b = a + n;
  const int pr = blockIdx.x;
  const int k = pr / pairs + 1, jr = 2 * (pr % pairs);
  const T* row = p + ((long long)(k - 1) * p_rows + p_row0 + jr) * n;
  for (int e = threadIdx.x; e < n; e += blockDim.x) {
    C z;
    z.x = row[e];
    z.y = row[n + e];
    a[e] = z;
  }
  __syncthreads();
  const C* zt = gen_lines_fft<T, false>(a, b, 1, g, tw);
  for (int m = threadIdx.x; m < nxh; m += blockDim.x) {
    const C zm = zt[m];
    const C zn = zt[(n - m) % n];
    C ra, rb;
    ra.x = (T)0.5 * (zm.x + zn.x);
    ra.y = (T)0.5 * (zm.y - zn.y);
    rb.x = (T)0.5 * (zm.y + zn.y);
    rb.y = (T)0.5 * (zn.x - zm.x);
    int w;
    C* o = spec + spec_x_offset(m, nxh, nblk, ny, nz, k, jr, &w);
    o[0] = ra;
    o[w] = rb;
  }
}

// inverse x of generic length, the inverse of k_fftg_x_fwd (imaginary parts of kx = 0 and, for
// even n, kx = n/2 dropped)
template <typename T>
__global__ void __launch_bounds__(GEN_BLOCK) k_fftg_x_inv(T* __restrict__ p, const typename Cx<T>::t* __restrict__ spec,
                                                          const typename Cx<T>::t* __restrict__ tw, GenFactors g, int ny,
                                                          int nz, int p_rows, int p_row0, int nblk) {
  typedef typename Cx<T>::t C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = g.n, nxh = n / 2 + 1, pairs = ny / 2;
  C* a = reinterpret_cast<C*>(smem_raw);
  C* b = a + n;
  const int pr = blockIdx.x;
  const int k = pr / pairs + 1, jr = 2 * (pr % pairs);
  for (int m = threadIdx.x; m < nxh; m += blockDim.x) {
    int w;
    const C* in = spec + spec_x_offset(m, nxh, nblk, ny, nz, k, jr, &w);
    C ra = in[0], rb = in[w];
    const bool nyquist = 2 * m == n;
    if (m == 0 || nyquist) { ra.y = (T)0; rb.y = (T)0; }
    C z;
    z.x = ra.x - rb.y;
    z.y = ra.y + rb.x;
    a[m] = z;
    if (m > 0 && !nyquist) {
      C zc;
      zc.x = ra.x + rb.y;
      zc.y = rb.x - ra.y;
      a[n - m] = zc;
    }
  }
  __syncthreads();
  const C* zt = gen_lines_fft<T, true>(a, b, 1, g, tw);
  T* row = p + ((long long)(k - 1) * p_rows + p_row0 + jr) * n;
  const T sc = (T)(1.0 / (double)n);
  for (int e = threadIdx.x; e < n; e += blockDim.x) {
    row[e] = zt[e].x * sc;
    row[n + e] = zt[e].y * sc;
  }
}

// columns per block of the generic y kernel: as many as keep the two buffers within 64 KB of
// FP64 lines (at least one)
static int gen_y_cols(int n) { return std::max(1, std::min(8, 2048 / n)); }

// y of generic length on a tile of kx columns of one level, the layout of k_fft_y; the inverse
// is scaled by 1/n
template <typename T, bool INV>
__global__ void __launch_bounds__(GEN_BLOCK) k_fftg_y(typename Cx<T>::t* __restrict__ spec,
                                                      const typename Cx<T>::t* __restrict__ tw, GenFactors g, int ncols,
                                                      int nz, int rpb, int tc) {
  typedef typename Cx<T>::t C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = g.n;
  C* a = reinterpret_cast<C*>(smem_raw);
  C* b = a + (size_t)tc * n;
  const int kx0 = blockIdx.x * tc, k = blockIdx.y + 1;
  const int nc = min(tc, ncols - kx0);
  for (int t = threadIdx.x; t < nc * n; t += blockDim.x) {
    const int e = t / nc, c = t - e * nc;  // consecutive threads take consecutive columns
    a[c * n + e] = spec[spec_row(e, k, rpb, ncols, nz) + kx0 + c];
  }
  __syncthreads();
  const C* zt = gen_lines_fft<T, INV>(a, b, nc, g, tw);
  const T sc = INV ? (T)(1.0 / (double)n) : (T)1.0;
  for (int t = threadIdx.x; t < nc * n; t += blockDim.x) {
    const int e = t / nc, c = t - e * nc;
    C z = zt[c * n + e];
    if (INV) { z.x = z.x * sc; z.y = z.y * sc; }
    spec[spec_row(e, k, rpb, ncols, nz) + kx0 + c] = z;
  }
}

template <typename T>
static void ensure_gen_attr() {
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
  std::lock_guard<std::mutex> lock(mu);
  if (done[dev]) return;
  const int mx = (int)(2 * 4096 * sizeof(typename Cx<T>::t));
  cudaFuncSetAttribute(k_fftg_x_fwd<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_fftg_x_inv<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_fftg_y<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_fftg_y<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  done[dev] = true;
}

// ---- launches: one kernel instantiation per transform length (4 .. 4096 points) ----------------
template <typename T>
static size_t line_smem(int logn) {
  return (size_t)line_lines(logn) * ((1 << logn) + (1 << logn) / 16 + 1) * sizeof(typename Cx<T>::t);
}

#define MGPU_LOGN_CASES(X) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12)

// the largest line needs more than the default 48 KB of dynamic shared memory: raise the limit
// of every line kernel once per device
template <typename T>
static void ensure_line_attr() {
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
  std::lock_guard<std::mutex> lock(mu);
  if (done[dev]) return;
#define MGPU_SET_ATTR(L)                                                                                  \
  cudaFuncSetAttribute(k_fft_x_fwd<T, L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)line_smem<T>(L)); \
  cudaFuncSetAttribute(k_fft_x_inv<T, L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)line_smem<T>(L)); \
  cudaFuncSetAttribute(k_fft_x_fwd_src<T, L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)line_smem<T>(L)); \
  cudaFuncSetAttribute(k_fft_y<T, L, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)line_smem<T>(L)); \
  cudaFuncSetAttribute(k_fft_y<T, L, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)line_smem<T>(L));
  MGPU_LOGN_CASES(MGPU_SET_ATTR)
#undef MGPU_SET_ATTR
  done[dev] = true;
}

static bool is_pow2(int n) { return n >= 4 && n <= 4096 && (n & (n - 1)) == 0; }

// x-FFT of the nz * ny/2 row pairs of length n, forward or inverse
template <typename T>
static void launch_fft_x(bool inverse, int n, T* p, typename Cx<T>::t* spec, const typename Cx<T>::t* tw, int ny,
                         int nz, int p_rows, int p_row0, int nblk, cudaStream_t st) {
  if (!is_pow2(n)) {
    GenFactors g;
    if (!gen_factor(n, g)) return;
    ensure_gen_attr<T>();
    const unsigned grid = (unsigned)((long long)nz * (ny / 2));
    const size_t smem = 2 * (size_t)n * sizeof(typename Cx<T>::t);
    if (inverse) k_fftg_x_inv<T><<<grid, GEN_BLOCK, smem, st>>>(p, spec, tw, g, ny, nz, p_rows, p_row0, nblk);
    else k_fftg_x_fwd<T><<<grid, GEN_BLOCK, smem, st>>>(p, spec, tw, g, ny, nz, p_rows, p_row0, nblk);
    return;
  }
  const int logn = ilog2(n);
  ensure_line_attr<T>();
  const long long pairs = (long long)nz * (ny / 2);
  const int L = line_lines(logn);
  const unsigned grid = (unsigned)((pairs + L - 1) / L);
  const int block = line_block(logn);
  const size_t smem = line_smem<T>(logn);
  switch (logn) {
#define MGPU_X_CASE(LG)                                                                                     \
  case LG:                                                                                                  \
    if (inverse) k_fft_x_inv<T, LG><<<grid, block, smem, st>>>(p, spec, tw, ny, nz, p_rows, p_row0, nblk);  \
    else k_fft_x_fwd<T, LG><<<grid, block, smem, st>>>(p, spec, tw, ny, nz, p_rows, p_row0, nblk);          \
    break;
    MGPU_LOGN_CASES(MGPU_X_CASE)
#undef MGPU_X_CASE
    default: break;
  }
}

// forward x-FFT of the pressure source formed from zu, zv, zw (power-of-two nx, one domain)
template <typename T>
static void launch_fft_x_src(const Scalars& s, const SourceFields<T>& f, typename Cx<T>::t* spec,
                             const typename Cx<T>::t* tw, cudaStream_t st) {
  const int logn = ilog2(s.nx);
  ensure_line_attr<T>();
  const long long pairs = (long long)s.nz * (s.ny / 2);
  const int L = line_lines(logn);
  const unsigned grid = (unsigned)((pairs + L - 1) / L);
  const int block = line_block(logn);
  const size_t smem = line_smem<T>(logn);
  switch (logn) {
#define MGPU_XS_CASE(LG)                                                        \
  case LG:                                                                      \
    k_fft_x_fwd_src<T, LG><<<grid, block, smem, st>>>(s, f, spec, tw);          \
    break;
    MGPU_LOGN_CASES(MGPU_XS_CASE)
#undef MGPU_XS_CASE
    default: break;
  }
}

// y-FFT of ncols columns of n rows on each of nz levels (rows in blocks of rpb)
template <typename T>
static void launch_fft_y(bool inverse, int n, typename Cx<T>::t* spec, const typename Cx<T>::t* tw, int ncols, int nz,
                         int rpb, cudaStream_t st) {
  if (!is_pow2(n)) {
    GenFactors g;
    if (!gen_factor(n, g)) return;
    ensure_gen_attr<T>();
    const int tc = gen_y_cols(n);
    dim3 grid((unsigned)((ncols + tc - 1) / tc), (unsigned)nz);
    const size_t smem = 2 * (size_t)tc * n * sizeof(typename Cx<T>::t);
    if (inverse) k_fftg_y<T, true><<<grid, GEN_BLOCK, smem, st>>>(spec, tw, g, ncols, nz, rpb, tc);
    else k_fftg_y<T, false><<<grid, GEN_BLOCK, smem, st>>>(spec, tw, g, ncols, nz, rpb, tc);
    return;
  }
  const int logn = ilog2(n);
  ensure_line_attr<T>();
  const int cols = line_lines(logn);
  dim3 grid((unsigned)((ncols + cols - 1) / cols), (unsigned)nz);
  const int block = line_block(logn);
  const size_t smem = line_smem<T>(logn);
  switch (logn) {
#define MGPU_Y_CASE(LG)                                                                        \
  case LG:                                                                                     \
    if (inverse) k_fft_y<T, LG, true><<<grid, block, smem, st>>>(spec, tw, ncols, nz, rpb);    \
    else k_fft_y<T, LG, false><<<grid, block, smem, st>>>(spec, tw, ncols, nz, rpb);           \
    break;
    MGPU_LOGN_CASES(MGPU_Y_CASE)
#undef MGPU_Y_CASE
    default: break;
  }
}

// ---- cp.async staging (each thread copies and later reads its own shared-memory slots) -------
__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void cp_async_16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_elem(double2* dst, const double2* src) { cp_async_16(dst, src); }
__device__ __forceinline__ void cp_async_elem(float2* dst, const float2* src) { cp_async_8(dst, src); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// tridiagonal launch shape: TRI_TB columns (threads) per block, TRI_KC levels per staged chunk,
// TRI_NS chunks in the ring (TRI_NS - 1 of them in flight while one is used).  Two blocks of 112
// fit an SM, so the 33,024 columns of a 256 x 256 grid are one wave on 148 SMs.
constexpr int TRI_TB = 112, TRI_KC = 8, TRI_NS = 4;
constexpr size_t TRI_SMEM = (size_t)TRI_NS * TRI_KC * TRI_TB * (sizeof(double2) + sizeof(double));
// the staging ring (or the mean mode's column), then czb, cza, czg of levels 0 .. nz+1
template <typename C>
__host__ __device__ constexpr size_t tri_coef_off(int nz) {
  return ((TRI_SMEM > (size_t)nz * sizeof(C) ? TRI_SMEM : (size_t)nz * sizeof(C)) + 15) & ~(size_t)15;
}
template <typename C>
static size_t tri_smem_bytes(int nz) { return tri_coef_off<C>(nz) + 3 * (size_t)(nz + 2) * sizeof(double); }
constexpr size_t TRI_SMEM_MAX = TRI_SMEM + 3 * (size_t)(MGPU_MAX_NZ + 2) * sizeof(double);
template <typename T>
__global__ void k_tridiag(typename Cx<T>::t* __restrict__ spec, double2* __restrict__ s1buf, const double* __restrict__ b1,
                          const double* __restrict__ prof, int prof_stride, int nx, int ny, int nz, int transpose,
                          int ncols, int kx0, int rpb);
// the staging buffers exceed the default 48 KB of dynamic shared memory: raise the limit once per
// device (the largest column, nz = MGPU_MAX_NZ levels for the mean mode, stays below TRI_SMEM)
static void ensure_tri_attr() {
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
  std::lock_guard<std::mutex> lock(mu);
  if (done[dev]) return;
  cudaFuncSetAttribute(k_tridiag<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TRI_SMEM_MAX);
  cudaFuncSetAttribute(k_tridiag<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TRI_SMEM_MAX);
  done[dev] = true;
}
__device__ __forceinline__ unsigned char* tri_smem() {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  return smem_raw;
}

// ---- vertical tridiagonal per (ky, kx) in FP64 ----------------------------------------------
// The horizontal-mean mode (kx = ky = 0) of one column, held at col[0], col[1], ... (level k at
// col[k-1]): p(1) = p(2) = 0 and an upward recurrence, or with transpose the transposed recurrence
// from the top.
template <typename T>
__device__ void mean_mode_column(typename Cx<T>::t* col, int nz, const double* czb, const double* cza,
                                 const double* czg, int transpose) {
  typedef typename Cx<T>::t C;
  C zero;
  zero.x = (T)0;
  zero.y = (T)0;
  if (transpose) {
    // the rows r = 2..nz-1 of cza(r) p(r+1) + czg(r) p(r) + czb(r) p(r-1) = b(r), p(1) = p(2) = 0,
    // transposed and solved from the top
    double zr1 = 0.0, zi1 = 0.0, zr2 = 0.0, zi2 = 0.0;  // z(u), z(u+1)
    C ynext = col[nz - 1];                              // y(nz)
    for (int u = nz; u >= 3; --u) {
      const C yu = ynext;
      if (u >= 4) ynext = col[u - 2];  // y(u-1), read before z(u-1) overwrites it
      double yr = (double)yu.x, yi = (double)yu.y;
      if (u <= nz - 1) { yr -= czg[u] * zr1; yi -= czg[u] * zi1; }
      if (u + 1 <= nz - 1) { yr -= czb[u + 1] * zr2; yi -= czb[u + 1] * zi2; }
      const double zr = yr / cza[u - 1], zi = yi / cza[u - 1];  // z(u-1)
      zr2 = zr1; zi2 = zi1; zr1 = zr; zi1 = zi;
      C o;
      o.x = (T)zr;
      o.y = (T)zi;
      col[u - 2] = o;
    }
    col[0] = zero;
    col[nz - 1] = zero;
    return;
  }
  C v2 = col[1];
  double sr_prev = (double)v2.x, si_prev = (double)v2.y;
  double pr2 = 0.0, pi2 = 0.0, pr1 = 0.0, pi1 = 0.0;  // p(k-2), p(k-1)
  col[0] = zero;  // p(1) = p(2) = 0 for the mean mode
  col[1] = zero;
  for (int k = 3; k <= nz; ++k) {
    C vk = col[k - 1];
    double pr = (sr_prev - czg[k - 1] * pr1 - czb[k - 1] * pr2) / cza[k - 1];
    double pi = (si_prev - czg[k - 1] * pi1 - czb[k - 1] * pi2) / cza[k - 1];
    sr_prev = (double)vk.x;
    si_prev = (double)vk.y;
    C o;
    o.x = (T)pr;
    o.y = (T)pi;
    col[k - 1] = o;
    pr2 = pr1; pi2 = pi1; pr1 = pr; pi1 = pi;
  }
}

template <typename T>
// The spectrum holds ncols kx columns per row, the global wavenumbers kx0 .. kx0+ncols-1 (all
// nx/2+1 of them, or one rank's block after a transpose), and its rows in blocks of rpb as in
// k_fft_y.  s1buf is [nz][ny][ncols] whatever the spectrum layout.  One thread per column; when
// the block holds kx = 0 (kx0 == 0) the launch has one extra block, the last, for the mean mode.
__global__ void k_tridiag(typename Cx<T>::t* __restrict__ spec, double2* __restrict__ s1buf, const double* __restrict__ b1,
                          const double* __restrict__ prof, int prof_stride, int nx, int ny, int nz, int transpose,
                          int ncols, int kx0, int rpb) {
  typedef typename Cx<T>::t C;
  const int nxh = nx / 2 + 1;
  const long long lstride = (long long)rpb * ncols;   // level stride of the spectrum
  // the three coefficient profiles, read at every level of every column, from shared memory
  const int cs = nz + 2;
  double* cf = reinterpret_cast<double*>(tri_smem() + tri_coef_off<C>(nz));
  for (int q = threadIdx.x; q < 3 * cs; q += blockDim.x) {
    const int r = q / cs, kk = q - r * cs;
    cf[q] = prof[(r == 0 ? P_CZB : (r == 1 ? P_CZA : P_CZG)) * prof_stride + kk];
  }
  __syncthreads();
  const double* czb = cf;
  const double* cza = cf + cs;
  const double* czg = cf + 2 * cs;
  if (kx0 == 0 && blockIdx.x == gridDim.x - 1) {
    // the mean mode is one sequential recurrence over the levels: stage its column (row 0,
    // column 0 of every level) in shared memory so that no step of it waits on a global load
    C* colv = reinterpret_cast<C*>(tri_smem());
    for (int k = threadIdx.x; k < nz; k += blockDim.x) colv[k] = spec[(long long)k * lstride];
    __syncthreads();
    if (threadIdx.x == 0) mean_mode_column<T>(colv, nz, czb, cza, czg, transpose);
    __syncthreads();
    for (int k = threadIdx.x; k < nz; k += blockDim.x) spec[(long long)k * lstride] = colv[k];
    return;
  }
  long long col = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= (long long)ny * ncols) return;
  const int ky = (int)(col / ncols), c = (int)(col - (long long)ky * ncols), kx = kx0 + c;
  if (kx == 0 && ky == 0) return;  // the mean-mode block's column
  const long long plane = (long long)ny * ncols;      // level stride of s1buf
  C* sp = spec + spec_row(ky, 1, rpb, ncols, nz) + c;
  // the transposed tridiagonal has the same pivots (they depend on czb(k)*cza(k-1) only) with
  // the off-diagonals exchanged: cza(k-1) below the diagonal, czb(k+1) above it
  const double* lo = transpose ? cza - 1 : czb;  // lo[k]: coefficient of s(k-1) in row k
  const double* up = transpose ? czb + 1 : cza;  // up[k]: coefficient of p(k+1) in row k
  const int kyi = ky <= ny / 2 ? ky : ny - ky;
  const long long bstride = (long long)(ny / 2 + 1) * nxh;
  const double* bcol = b1 + (long long)kyi * nxh + kx;
  // Every level a thread needs (spectrum or s1, and the pivot) is staged in shared memory by
  // cp.async, TRI_KC levels per chunk, TRI_NS - 1 chunks in flight while one is used.  Each
  // thread copies and reads only its own slots, so no block barrier is involved.
  // Slots are 16 bytes whatever the spectrum type, so that a thread's forward slots (spectrum)
  // and backward slots (s1) are the same bytes and no thread's slot overlaps another's.
  unsigned char* raw = tri_smem();
  double2* sbuf = reinterpret_cast<double2*>(raw);    // [TRI_NS][TRI_KC][TRI_TB] 16-byte slots
  double* bbuf = reinterpret_cast<double*>(raw + (size_t)TRI_NS * TRI_KC * TRI_TB * sizeof(double2));
  const int t = threadIdx.x;
  auto slot = [&](int ch, int q) { return ((ch % TRI_NS) * TRI_KC + q) * TRI_TB + t; };
  auto fslot = [&](int ch, int q) { return reinterpret_cast<C*>(sbuf + slot(ch, q)); };
  // forward elimination s1(k) = pt(k) - czb(k)*s1(k-1)*b1(k-1) for k = 3..nz.  An FP64 spectrum
  // takes s1(k) in place of pt(k), which the sweep has read by then: the column's one array then
  // stays in L2 between the two sweeps, where a separate s1 array would double the footprint.  An
  // FP32 spectrum keeps s1 in FP64 in s1buf.
  constexpr bool in_place = sizeof(C) == sizeof(double2);
  auto s1_at = [&](int k) -> double2* {
    return in_place ? reinterpret_cast<double2*>(sp + (long long)(k - 1) * lstride) : s1buf + col + (long long)(k - 1) * plane;
  };
  C v = sp[lstride];
  double sr = (double)v.x, si = (double)v.y;
  if (!in_place) *s1_at(2) = make_double2(sr, si);
  const int nch = (nz - 2 + TRI_KC - 1) / TRI_KC;
  auto issue_fwd = [&](int ch) {
    for (int q = 0; q < TRI_KC; ++q) {
      const int k = 3 + ch * TRI_KC + q;
      if (k <= nz) {
        cp_async_elem(fslot(ch, q), sp + (long long)(k - 1) * lstride);
        cp_async_8(bbuf + slot(ch, q), bcol + (long long)(k - 1) * bstride);
      }
    }
    cp_async_commit();
  };
  for (int c = 0; c < TRI_NS - 1; ++c) {
    if (c < nch) issue_fwd(c);
    else cp_async_commit();
  }
  for (int ch = 0; ch < nch; ++ch) {
    if (ch + TRI_NS - 1 < nch) issue_fwd(ch + TRI_NS - 1);
    else cp_async_commit();
    cp_async_wait<TRI_NS - 1>();
#pragma unroll 4
    for (int q = 0; q < TRI_KC; ++q) {
      const int k = 3 + ch * TRI_KC + q;
      if (k <= nz) {
        const C vq = *fslot(ch, q);
        const double bq = bbuf[slot(ch, q)];
        sr = (double)vq.x - lo[k] * sr * bq;
        si = (double)vq.y - lo[k] * si * bq;
        *s1_at(k) = make_double2(sr, si);
      }
    }
  }
  cp_async_wait_0();
  // back substitution pt(k) = (s1(k) - cza(k)*pt(k+1))*b1(k) for k = nz-1 down to 2
  double pr = sr * __ldg(bcol + (long long)nz * bstride);
  double pi = si * __ldg(bcol + (long long)nz * bstride);
  C o;
  o.x = (T)pr;
  o.y = (T)pi;
  sp[(long long)(nz - 1) * lstride] = o;
  auto issue_bwd = [&](int ch) {
    for (int q = 0; q < TRI_KC; ++q) {
      const int k = nz - 1 - ch * TRI_KC - q;
      if (k >= 2) {
        cp_async_16(sbuf + slot(ch, q), s1_at(k));
        cp_async_8(bbuf + slot(ch, q), bcol + (long long)k * bstride);
      }
    }
    cp_async_commit();
  };
  for (int c = 0; c < TRI_NS - 1; ++c) {
    if (c < nch) issue_bwd(c);
    else cp_async_commit();
  }
  for (int ch = 0; ch < nch; ++ch) {
    if (ch + TRI_NS - 1 < nch) issue_bwd(ch + TRI_NS - 1);
    else cp_async_commit();
    cp_async_wait<TRI_NS - 1>();
#pragma unroll 4
    for (int q = 0; q < TRI_KC; ++q) {
      const int k = nz - 1 - ch * TRI_KC - q;
      if (k >= 2) {
        const double2 sq = sbuf[slot(ch, q)];
        const double bq = bbuf[slot(ch, q)];
        pr = (sq.x - up[k] * pr) * bq;
        pi = (sq.y - up[k] * pi) * bq;
        o.x = (T)pr;
        o.y = (T)pi;
        sp[(long long)(k - 1) * lstride] = o;
      }
    }
  }
  cp_async_wait_0();
}

// The column solve of ncols kx columns (global kx0 ..) on ny rows
template <typename T>
static void launch_tridiag(typename Cx<T>::t* spec, double2* s1, const double* b1, const double* prof, int prof_stride,
                           int nx, int ny, int nz, bool transpose, int ncols, int kx0, int rpb, cudaStream_t st) {
  typedef typename Cx<T>::t C;
  const long long ncol = (long long)ny * ncols;
  ensure_tri_attr();
  k_tridiag<T><<<(unsigned)((ncol + TRI_TB - 1) / TRI_TB + (kx0 == 0 ? 1 : 0)), TRI_TB, tri_smem_bytes<C>(nz), st>>>(
      spec, s1, b1, prof, prof_stride, nx, ny, nz, transpose ? 1 : 0, ncols, kx0, rpb);
}

// Pivots and twiddles of the (pl.nx, pl.ny, pl.nz) grid; pl.spec and pl.s1 are left to the caller.
static int plan_tables(FftPlanDev& pl, const RefState& rs) {
  // Thomas pivots per (|ky|, kx), built exactly as fftsolver.F90:259-280 and :72-90
  const int nyh = pl.ny / 2 + 1;
  std::vector<double> b1((size_t)(pl.nz + 1) * nyh * pl.nxh, 0.0);
  const double PI = 4.0 * std::atan(1.0);
  std::vector<double> cosx(pl.nxh), cosy(nyh);
  for (int m = 0; m < pl.nxh; ++m) cosx[m] = (2.0 / (rs.dx * rs.dx)) * (std::cos(2.0 * PI * (double)m / (double)pl.nx) - 1.0);
  for (int m = 0; m < nyh; ++m) cosy[m] = (2.0 / (rs.dy * rs.dy)) * (std::cos(2.0 * PI * (double)m / (double)pl.ny) - 1.0);
  for (int ky = 0; ky < nyh; ++ky)
    for (int kx = 0; kx < pl.nxh; ++kx) {
      double cij = cosx[kx] + cosy[ky];
      double b = cij - rs.cza[2];
      double prev = 1.0 / b;
      b1[((size_t)2 * nyh + ky) * pl.nxh + kx] = prev;
      for (int k = 3; k <= pl.nz; ++k) {
        double bk = cij + rs.czg[k];
        prev = 1.0 / (bk - rs.czh[k] * prev);
        b1[((size_t)k * nyh + ky) * pl.nxh + kx] = prev;
      }
    }
  if (cudaMalloc(&pl.b1, b1.size() * sizeof(double)) != cudaSuccess) return MGPU_ERR_CUDA;
  cudaMemcpy(pl.b1, b1.data(), b1.size() * sizeof(double), cudaMemcpyHostToDevice);
  // twiddles W_n^q = e^{-2 pi i q / n}, q < n (interleaved complex), and the same rounded to FP32
  auto twiddles = [&](int n, double** dd, float** df) {
    std::vector<double> t(2 * (size_t)n);
    std::vector<float> tf(2 * (size_t)n);
    for (int q = 0; q < n; ++q) {
      double a = 2.0 * PI * (double)q / (double)n;
      t[2 * q] = std::cos(a);
      t[2 * q + 1] = -std::sin(a);
      tf[2 * q] = (float)t[2 * q];
      tf[2 * q + 1] = (float)t[2 * q + 1];
    }
    cudaMalloc(dd, 2 * (size_t)n * sizeof(double));
    cudaMalloc(df, 2 * (size_t)n * sizeof(float));
    cudaMemcpy(*dd, t.data(), 2 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(*df, tf.data(), 2 * (size_t)n * sizeof(float), cudaMemcpyHostToDevice);
  };
  twiddles(pl.nx, &pl.twx, &pl.twx_f);
  twiddles(pl.ny, &pl.twy, &pl.twy_f);
  return cudaGetLastError() == cudaSuccess ? MGPU_OK : MGPU_ERR_CUDA;
}

// Horizontal transform lengths the solve supports: 4 .. 4096 points with prime factors 2, 3, 5
bool fft_length_ok(int n) {
  GenFactors g;
  return n >= 4 && gen_factor(n, g);
}

int fft_plan_create(FftPlanDev& pl, const Scalars& s, const RefState& rs, bool fp32) {
  pl.nx = s.nx;
  pl.ny = s.ny;
  pl.nz = s.nz;
  pl.nxh = s.nx / 2 + 1;
  if (!fft_length_ok(s.nx) || !fft_length_ok(s.ny) || (s.ny % 2)) return MGPU_ERR_UNSUPPORTED;
  const size_t plane = (size_t)s.ny * pl.nxh;
  const size_t cs = fp32 ? sizeof(float2) : sizeof(double2);
  if (cudaMalloc(&pl.spec, cs * plane * s.nz) != cudaSuccess) return MGPU_ERR_CUDA;
  // an FP64 spectrum holds the Thomas forward-elimination values in place (k_tridiag)
  if (fp32 && cudaMalloc(&pl.s1, sizeof(double2) * plane * s.nz) != cudaSuccess) return MGPU_ERR_CUDA;
  return plan_tables(pl, rs);
}

int fft_slab_plan_create(FftPlanDev& pl, const Scalars& s, const RefState& rs, int ny_global, int max_cols) {
  pl.nx = s.nx;
  pl.ny = ny_global;
  pl.nz = s.nz;
  pl.nxh = s.nx / 2 + 1;
  if (!fft_length_ok(s.nx) || !fft_length_ok(ny_global) || max_cols < 1 || max_cols > pl.nxh)
    return MGPU_ERR_UNSUPPORTED;
  if (cudaMalloc(&pl.s1, sizeof(double2) * (size_t)ny_global * max_cols * s.nz) != cudaSuccess) return MGPU_ERR_CUDA;
  return plan_tables(pl, rs);
}

void fft_plan_destroy(FftPlanDev& pl) {
  cudaFree(pl.spec);
  cudaFree(pl.s1);
  cudaFree(pl.b1);
  cudaFree(pl.twx);
  cudaFree(pl.twy);
  cudaFree(pl.twx_f);
  cudaFree(pl.twy_f);
  pl = FftPlanDev{};
}

template <typename T>
void fft_solve(const FftPlanDev& pl, const Scalars& s, T* p, cudaStream_t st, int64_t* launches, cudaEvent_t* evs,
               bool transpose, const SourceFields<T>* src) {
  typedef typename Cx<T>::t C;
  const bool f32 = sizeof(T) == 4;
  C* spec = reinterpret_cast<C*>(pl.spec);
  const C* twx = reinterpret_cast<const C*>(f32 ? (void*)pl.twx_f : (void*)pl.twx);
  const C* twy = reinterpret_cast<const C*>(f32 ? (void*)pl.twy_f : (void*)pl.twy);
  const int logx = s.nx, logy = s.ny;  // transform lengths
  double2* s1 = pl.s1;
  auto mark = [&](int q) { if (evs) cudaEventRecord(evs[q], st); };
  mark(0);
  if (src && is_pow2(s.nx)) launch_fft_x_src<T>(s, *src, spec, twx, st);
  else launch_fft_x<T>(false, logx, p, spec, twx, s.ny, s.nz, s.ny, 0, 1, st);
  mark(1);
  launch_fft_y<T>(false, logy, spec, twy, pl.nxh, s.nz, s.ny, st);
  mark(2);
  launch_tridiag<T>(spec, s1, pl.b1, s.prof, s.nz + 2, s.nx, s.ny, s.nz, transpose, pl.nxh, 0, s.ny, st);
  mark(3);
  launch_fft_y<T>(true, logy, spec, twy, pl.nxh, s.nz, s.ny, st);
  mark(4);
  launch_fft_x<T>(true, logx, p, spec, twx, s.ny, s.nz, s.ny, 0, 1, st);
  mark(5);
  *launches += 5;
}

template void fft_solve<double>(const FftPlanDev&, const Scalars&, double*, cudaStream_t, int64_t*, cudaEvent_t*, bool,
                                const SourceFields<double>*);
template void fft_solve<float>(const FftPlanDev&, const Scalars&, float*, cudaStream_t, int64_t*, cudaEvent_t*, bool,
                               const SourceFields<float>*);

// ---- y-slab decomposition: the solve split at the two transposes -------------------------
template <typename T>
void slab_fft_x(const FftPlanDev& pl, const Scalars& s, T* p, int halo, int nblk, void* spec, bool inverse,
                cudaStream_t st, int64_t* launches) {
  typedef typename Cx<T>::t C;
  const bool f32 = sizeof(T) == 4;
  const C* twx = reinterpret_cast<const C*>(f32 ? (void*)pl.twx_f : (void*)pl.twx);
  C* sp = reinterpret_cast<C*>(spec);
  const int nyl = s.ny - 2 * halo;
  launch_fft_x<T>(inverse, s.nx, p, sp, twx, nyl, s.nz, s.ny, halo, nblk, st);
  *launches += 1;
}

template <typename T>
void slab_solve_columns(const FftPlanDev& pl, const Scalars& s, void* spec, int kx0, int nkx, int rpb, bool transpose,
                        cudaStream_t st, int64_t* launches) {
  typedef typename Cx<T>::t C;
  const bool f32 = sizeof(T) == 4;
  const C* twy = reinterpret_cast<const C*>(f32 ? (void*)pl.twy_f : (void*)pl.twy);
  C* sp = reinterpret_cast<C*>(spec);
  const int logy = pl.ny;  // transform length
  launch_fft_y<T>(false, logy, sp, twy, nkx, s.nz, rpb, st);
  launch_tridiag<T>(sp, pl.s1, pl.b1, s.prof, s.nz + 2, pl.nx, pl.ny, s.nz, transpose, nkx, kx0, rpb, st);
  launch_fft_y<T>(true, logy, sp, twy, nkx, s.nz, rpb, st);
  *launches += 3;
}

template void slab_fft_x<double>(const FftPlanDev&, const Scalars&, double*, int, int, void*, bool, cudaStream_t, int64_t*);
template void slab_fft_x<float>(const FftPlanDev&, const Scalars&, float*, int, int, void*, bool, cudaStream_t, int64_t*);
template void slab_solve_columns<double>(const FftPlanDev&, const Scalars&, void*, int, int, int, bool, cudaStream_t,
                                         int64_t*);
template void slab_solve_columns<float>(const FftPlanDev&, const Scalars&, void*, int, int, int, bool, cudaStream_t,
                                        int64_t*);

// ---- horizontal-mean diagnostics: one block per level, FP64 accumulation in a fixed order ----
// Level sums split over a cluster of PSPLIT blocks (one cluster per level): block r sums its
// contiguous share of the level's points, each thread in a fixed stride order and the block by a
// tree; block 0 then adds the PSPLIT partial sums in rank order through distributed shared memory.
// Deterministic, and a level keeps PSPLIT blocks busy where one block per level left most of the
// GPU idle.
constexpr int PSPLIT = 8, PRED_T = 256;

template <int NV>
__device__ __forceinline__ void block_tree(double (*sh)[PRED_T]) {
  __syncthreads();
  for (int h = PRED_T / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h)
#pragma unroll
      for (int q = 0; q < NV; ++q) sh[q][threadIdx.x] += sh[q][threadIdx.x + h];
    __syncthreads();
  }
}

// the cluster's total of sh[q][0] over its blocks, valid in block 0 (thread 0)
template <int NV>
__device__ __forceinline__ void cluster_total(double (*sh)[PRED_T], double* tot) {
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  cluster.sync();
  if (cluster.block_rank() == 0 && threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) tot[q] = 0.0;
    for (int r = 0; r < PSPLIT; ++r) {
      double(*rs)[PRED_T] = cluster.map_shared_rank(sh, r);
#pragma unroll
      for (int q = 0; q < NV; ++q) tot[q] += rs[q][0];
    }
  }
  cluster.sync();  // no block leaves while block 0 reads its partial sums
}

template <typename T>
__global__ void __cluster_dims__(PSPLIT, 1, 1) __launch_bounds__(PRED_T)
    k_diagnostics(const T* __restrict__ th, const T* __restrict__ w, const double* __restrict__ prof, int prof_stride,
                  long long plane, long long first, long long count, double* out_th, double* out_w2) {
  // the `count` points from `first` of each level: the whole plane, or a y-slab's interior rows
  const int k = blockIdx.y + 1, r = blockIdx.x;
  const long long chunk = (count + PSPLIT - 1) / PSPLIT;
  const long long t0 = r * chunk, t1 = min(count, t0 + chunk);
  const T* thk = th + (long long)(k - 1) * plane + first;
  const T* wk = w + (long long)(k - 1) * plane + first;
  double a = 0.0, b = 0.0;
#pragma unroll 4
  for (long long t = t0 + threadIdx.x; t < t1; t += PRED_T) {
    a += (double)thk[t];
    double wv = (double)wk[t];
    b += wv * wv;
  }
  __shared__ double sh[2][PRED_T];
  sh[0][threadIdx.x] = a;
  sh[1][threadIdx.x] = b;
  block_tree<2>(sh);
  double tot[2];
  cluster_total<2>(sh, tot);
  if (r == 0 && threadIdx.x == 0) {
    if (out_th) out_th[k - 1] = tot[0] / (double)count + prof[P_THREF * prof_stride + k];
    if (out_w2) out_w2[k - 1] = tot[1] / (double)count;
  }
}

template <typename T>
void launch_diagnostics(const Scalars& s, const T* th, const T* w, double* out_th, double* out_w2, cudaStream_t st,
                        int halo) {
  const long long first = (long long)halo * s.nx, count = (long long)(s.ny - 2 * halo) * s.nx;
  k_diagnostics<T><<<dim3(PSPLIT, s.nz), PRED_T, 0, st>>>(th, w, s.prof, s.nz + 2, s.plane, first, count, out_th,
                                                          out_w2);
}
template void launch_diagnostics<double>(const Scalars&, const double*, const double*, double*, double*, cudaStream_t,
                                         int);

// ---- horizontal means of th and the q fields per level (FP64 sums in a fixed order) ----------
template <typename T>
struct MeanFields {
  const T* f[1 + MGPU_MAX_Q];
};
// the mean over `count` points of each level starting `off` points into the level
template <typename T>
__global__ void __cluster_dims__(PSPLIT, 1, 1) __launch_bounds__(PRED_T)
    k_level_means(MeanFields<T> mf, long long plane, long long off, long long count, int stride, double* out) {
  const int k = blockIdx.y + 1, row = blockIdx.z, r = blockIdx.x;
  const long long chunk = (count + PSPLIT - 1) / PSPLIT;
  const long long t0 = r * chunk, t1 = min(count, t0 + chunk);
  const T* fk = mf.f[row] + (long long)(k - 1) * plane + off;
  double a = 0.0;
#pragma unroll 4
  for (long long t = t0 + threadIdx.x; t < t1; t += PRED_T) a += (double)fk[t];
  __shared__ double sh[1][PRED_T];
  sh[0][threadIdx.x] = a;
  block_tree<1>(sh);
  double tot[1];
  cluster_total<1>(sh, tot);
  if (r == 0 && threadIdx.x == 0) out[(long long)row * stride + k] = tot[0] / (double)count;
}
template <typename T>
void launch_level_means(const Scalars& s, const T* th, T* const* q, int nq, double* out, cudaStream_t st, int halo) {
  MeanFields<T> mf{};
  mf.f[0] = th;
  for (int n = 0; n < nq; ++n) mf.f[1 + n] = q[n];
  k_level_means<T><<<dim3(PSPLIT, s.nz, 1 + nq), PRED_T, 0, st>>>(mf, s.plane, (long long)halo * s.nx,
                                                                  (long long)(s.ny - 2 * halo) * s.nx, s.nz + 2, out);
}
template void launch_level_means<double>(const Scalars&, const double*, double* const*, int, double*, cudaStream_t, int);
template void launch_level_means<float>(const Scalars&, const float*, float* const*, int, double*, cudaStream_t, int);
template void launch_diagnostics<float>(const Scalars&, const float*, const float*, double*, double*, cudaStream_t,
                                        int);

}  // namespace mgpu

// =============================================================================================
// Poisson solve without device allocation.
//
// Some host models cannot call cudaMalloc: their device memory is owned by another allocator (a
// caching allocator or a pool sized at start-up to most of HBM) and may not grow during a run, or
// their step loop must not meet the device-wide synchronisation that cudaFree implies.  They can
// still solve for the pressure: the caller passes the right-hand side (overwritten with the
// solution) and the vertical coefficients, all in device memory it owns, and every piece of
// working storage (the spectrum, pivots, twiddles, the coefficient block) lives in the
// fixed file-scope array below.  That array is part of the library image: every GPU that loads
// the library holds MGPU_NOALLOC_SCRATCH_BYTES until the process exits.
// =============================================================================================

#include "../../include/monc_gpu.h"

namespace mgpu {

static __device__ __align__(256) unsigned char g_noalloc_scratch[MGPU_NOALLOC_SCRATCH_BYTES];

// host-side device address of g_noalloc_scratch, looked up once per device
static void* noalloc_scratch_address(int* status) {
  static std::mutex mu;
  static void* addr[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) { *status = MGPU_ERR_CUDA; return nullptr; }
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) { *status = MGPU_ERR_CUDA; return nullptr; }
    addr[dev] = p;
  }
  *status = MGPU_OK;
  return addr[dev];
}

static size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// twiddles e^{-2 pi i q / n}, q < n
__global__ void k_noalloc_twiddles(double2* tw, int n) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  double sv, cv;
  sincospi(2.0 * (double)q / (double)n, &sv, &cv);
  tw[q] = make_double2(cv, -sv);
}

// the caller's vertical coefficients (device arrays, element k-1 = level k) into the scratch
// profile block, level k at index k as the tridiagonal kernels read it
__global__ void k_noalloc_coeffs(double* prof, int stride, int nz, const double* __restrict__ czb,
                                 const double* __restrict__ cza, const double* __restrict__ czg,
                                 const double* __restrict__ czh) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (k > nz) return;
  prof[(size_t)P_CZB * stride + k] = czb[k - 1];
  prof[(size_t)P_CZA * stride + k] = cza[k - 1];
  prof[(size_t)P_CZG * stride + k] = czg[k - 1];
  prof[(size_t)P_CZH * stride + k] = czh[k - 1];
}

// Thomas pivots per (|ky|, kx), formed as fftsolver.F90:72-90 and :259-280 form them
__global__ void k_noalloc_pivots(double* b1, const double* __restrict__ prof, int stride, int nx, int ny, int nz,
                                 double dx, double dy) {
  const int nxh = nx / 2 + 1, nyh = ny / 2 + 1;
  int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= nyh * nxh) return;
  int ky = col / nxh, kx = col - ky * nxh;
  const double PI = 4.0 * atan(1.0);
  double cosx = (2.0 / (dx * dx)) * (cos(2.0 * PI * (double)kx / (double)nx) - 1.0);
  double cosy = (2.0 / (dy * dy)) * (cos(2.0 * PI * (double)ky / (double)ny) - 1.0);
  double cij = cosx + cosy;
  const double* cza = prof + P_CZA * stride;
  const double* czg = prof + P_CZG * stride;
  const double* czh = prof + P_CZH * stride;
  double prev = 1.0 / (cij - cza[2]);
  b1[((size_t)2 * nyh + ky) * nxh + kx] = prev;
  for (int k = 3; k <= nz; ++k) {
    double bk = cij + czg[k];
    prev = 1.0 / (bk - czh[k] * prev);
    b1[((size_t)k * nyh + ky) * nxh + kx] = prev;
  }
}

}  // namespace mgpu

extern "C" int mgpu_poisson_fft_noalloc(double* p, int32_t nx, int32_t ny, int32_t nz, double dx, double dy,
                                        const double* czb, const double* cza, const double* czg, const double* czh,
                                        void* stream) {
  using namespace mgpu;
  auto pow2 = [](int n) { return n >= 4 && n <= 4096 && (n & (n - 1)) == 0; };
  if (!p || !czb || !cza || !czg || !czh || !pow2(nx) || !pow2(ny) || nz < 4 || nz > MGPU_MAX_NZ || !(dx > 0) ||
      !(dy > 0))
    return MGPU_ERR_ARGUMENT;
  const int nxh = nx / 2 + 1, nyh = ny / 2 + 1;
  const size_t plane = (size_t)ny * nxh;
  const int stride = nz + 2;
  const size_t b_spec = align256(sizeof(double2) * plane * nz);
  const size_t b_s1 = 0;  // the FP64 column solve keeps its elimination values in the spectrum
  const size_t b_b1 = align256(sizeof(double) * (size_t)(nz + 1) * nyh * nxh);
  const size_t b_twx = align256(sizeof(double2) * nx);
  const size_t b_twy = align256(sizeof(double2) * ny);
  const size_t b_prof = align256(sizeof(double) * (size_t)P_COUNT * stride);
  const size_t need = b_spec + b_s1 + b_b1 + b_twx + b_twy + b_prof;
  if (need > (size_t)MGPU_NOALLOC_SCRATCH_BYTES) {
    std::fprintf(stderr,
                 "mgpu_poisson_fft_noalloc: a %d x %d x %d grid needs %zu bytes of scratch, more than the "
                 "%zu-byte maximum\n",
                 nx, ny, nz, need, (size_t)MGPU_NOALLOC_SCRATCH_BYTES);
    return MGPU_ERR_ARGUMENT;
  }
  // an error left pending by earlier, unrelated work is reported as such and not as this call's
  const cudaError_t earlier = cudaGetLastError();
  if (earlier != cudaSuccess)
    std::fprintf(stderr, "mgpu_poisson_fft_noalloc: a CUDA error was pending before this call: %s\n",
                 cudaGetErrorString(earlier));
  int status = MGPU_OK;
  unsigned char* base = reinterpret_cast<unsigned char*>(noalloc_scratch_address(&status));
  if (status != MGPU_OK) {
    std::fprintf(stderr, "mgpu_poisson_fft_noalloc: cudaGetSymbolAddress of the scratch array failed\n");
    return status;
  }
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  double2* spec = reinterpret_cast<double2*>(base);
  double2* s1 = nullptr;
  double* b1 = reinterpret_cast<double*>(base + b_spec + b_s1);
  double2* twx = reinterpret_cast<double2*>(base + b_spec + b_s1 + b_b1);
  double2* twy = reinterpret_cast<double2*>(base + b_spec + b_s1 + b_b1 + b_twx);
  double* prof = reinterpret_cast<double*>(base + b_spec + b_s1 + b_b1 + b_twx + b_twy);
  k_noalloc_coeffs<<<(nz + 127) / 128, 128, 0, st>>>(prof, stride, nz, czb, cza, czg, czh);
  k_noalloc_twiddles<<<(nx + 127) / 128, 128, 0, st>>>(twx, nx);
  k_noalloc_twiddles<<<(ny + 127) / 128, 128, 0, st>>>(twy, ny);
  k_noalloc_pivots<<<(nyh * nxh + 127) / 128, 128, 0, st>>>(b1, prof, stride, nx, ny, nz, dx, dy);
  // the five solve kernels of fft_solve, on the scratch buffers
  launch_fft_x<double>(false, nx, p, spec, twx, ny, nz, ny, 0, 1, st);
  launch_fft_y<double>(false, ny, spec, twy, nxh, nz, ny, st);
  ensure_tri_attr();
  k_tridiag<double><<<(unsigned)((plane + TRI_TB - 1) / TRI_TB + 1), TRI_TB, tri_smem_bytes<double2>(nz), st>>>(
      spec, s1, b1, prof, stride, nx, ny, nz, 0, nxh, 0, ny);
  launch_fft_y<double>(true, ny, spec, twy, nxh, nz, ny, st);
  launch_fft_x<double>(true, nx, p, spec, twx, ny, nz, ny, 0, 1, st);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    std::fprintf(stderr, "mgpu_poisson_fft_noalloc: kernel launch failed: %s\n", cudaGetErrorString(e));
    return MGPU_ERR_CUDA;
  }
  return MGPU_OK;
}
