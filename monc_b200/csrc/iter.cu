// Iterative pressure solve: preconditioned BiCGStab or conjugate gradients on MONC's 7-point
// Poisson operator (iterativesolver.F90:140-248 bicgstab, :255-321 cg_solver, :329-380 precond,
// :400-493 calc_Ax, :500-553 inner products, :559-602 set_matrix_for_poisson).
//
// One BiCGStab iteration is five kernels over the resident work arrays:
//   k_bicg_direction  : t = r - bet*omg*v; s = M^-1 t; pp = s + bet*pp   (pp = M^-1 r on it 1)
//   k_bicg_apply_dot  : v = A pp,  nrm = <cr, v>, alf = rho / nrm
//   k_bicg_half_step  : s = r - alf*v,  cs = M^-1 s
//   k_bicg_apply_dots : t = A cs,  tt, ts, ss,  omg = ts / tt,  err
//   k_bicg_update     : x += alf*pp + omg*cs,  r = s - omg*t,  rho = <r, cr>,  convergence
// One CG iteration (solver_type MGPU_ITER_CG, MONC's symm_prob: the symmetric form of the operator,
// A_vol = dz, and a right-hand side scaled by A_vol) is three kernels:
//   k_cg_precond      : z = M^-1 r,  <z, r>,  bet = <z, r> / rho,  rho = <z, r>
//   k_cg_apply        : p' = z + bet*p (each point computes its neighbours' p' itself, so p' goes to
//                       a second buffer and no point waits for another),  Ap',  alf = rho / <p', Ap'>
//   k_cg_update       : x += alf*p',  r -= alf*Ap',  err = |r| / sc_err,  convergence
// M^-1 is MONC's column LU solve of the vertical part (preconditioner_iterations = 0).  Dot
// products accumulate in FP64 whatever the work precision: warp shuffles, one partial per block,
// and the last block to finish sums the partials in a fixed order (deterministic) and updates the
// solver scalars, which stay in device memory.  Every kernel returns at once when the solve has
// converged, so the host launches iterations in batches and reads the state back once a batch.
//
// The FP32-mixed model solves in FP64 by iterative refinement: r = b - A x in FP64, an FP32
// BiCGStab solve of A e = r to a relative residual set by the FP64 one (inner_tolerance), x += e,
// until the FP64 residual meets the tolerance.
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <vector>

#include "dycore.h"

namespace mgpu {

struct IterScalars {
  double rho, rho_prev, nrm, alf, omg, err, sc_err, tol, shift, bet;
  int it, done, it_done;
  int ext;  // 1: the dot products are summed outside (over y-slabs): the last block leaves them in loc
  unsigned int counter, pad;
  double loc[3];
};

namespace {

constexpr int BX = 32, BY = 8, NTH = BX * BY;
// A_u, A_d, A_p, lu_d, lu_u, vol = rhon*dz, A_vol (dz for the symmetric form, else 1), each nz+2
// long (1-based)
constexpr int NCOEF = 7;

struct Geom {
  int nx, ny, nz, symm;
  long long plane;
  double A_n, A_e;
  const double* coef;  // [NCOEF][nz+2]
  int j0, j1;          // rows solved: all (0, ny), or a y-slab's interior rows between its halo rows
  int ny_total;        // rows of the whole domain (the compatibility shift's point count)
  __device__ __forceinline__ double au(int k) const { return coef[k]; }
  __device__ __forceinline__ double ad(int k) const { return coef[(nz + 2) + k]; }
  __device__ __forceinline__ double ap(int k) const { return coef[2 * (nz + 2) + k]; }
  __device__ __forceinline__ double lud(int k) const { return coef[3 * (nz + 2) + k]; }
  __device__ __forceinline__ double luu(int k) const { return coef[4 * (nz + 2) + k]; }
  __device__ __forceinline__ double vol(int k) const { return coef[5 * (nz + 2) + k]; }
  __device__ __forceinline__ double avol(int k) const { return coef[6 * (nz + 2) + k]; }
  __device__ __forceinline__ long long at(int k, int j, int i) const { return (long long)(k - 1) * plane + (long long)j * nx + i; }
};

template <int NV>
__device__ __forceinline__ void block_partials(double (&v)[NV], double* partials, int nblocks, int bid) {
  __shared__ double sh[NV][NTH / 32];
  const int tid = threadIdx.y * BX + threadIdx.x, lane = tid & 31, wid = tid >> 5;
#pragma unroll
  for (int q = 0; q < NV; ++q)
    for (int off = 16; off; off >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], off);
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < NV; ++q) sh[q][wid] = v[q];
  __syncthreads();
  if (tid == 0)
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double a = 0.0;
      for (int w = 0; w < NTH / 32; ++w) a += sh[q][w];
      partials[(long long)q * nblocks + bid] = a;
    }
}

// True in thread 0 of the last block to finish; `out` then holds the sums over all blocks.
template <int NV>
__device__ bool last_block_sums(IterScalars* st, const double* partials, int nblocks, double (&out)[NV]) {
  __shared__ bool am_last;
  __shared__ double sh[NV][NTH / 32];
  const int tid = threadIdx.y * BX + threadIdx.x, lane = tid & 31, wid = tid >> 5;
  __threadfence();
  __syncthreads();
  if (tid == 0) am_last = atomicAdd(&st->counter, 1u) == (unsigned)nblocks - 1u;
  __syncthreads();
  if (!am_last) return false;
  __threadfence();
  double v[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    // the loads are independent of the running sum: unrolled, eight of them are in flight at once
    // instead of one L2 round trip per step of the ~60-step loop
    double a = 0.0;
#pragma unroll 8
    for (int b = tid; b < nblocks; b += NTH) a += __ldcg(partials + (long long)q * nblocks + b);
    v[q] = a;
  }
#pragma unroll
  for (int q = 0; q < NV; ++q)
    for (int off = 16; off; off >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], off);
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < NV; ++q) sh[q][wid] = v[q];
  __syncthreads();
  if (tid != 0) return false;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double a = 0.0;
    for (int w = 0; w < NTH / 32; ++w) a += sh[q][w];
    out[q] = a;
  }
  st->counter = 0u;
  if (st->ext) {
    // this slab's sums; the scalars are updated once the sums over all slabs are back
#pragma unroll
    for (int q = 0; q < NV; ++q) st->loc[q] = out[q];
    return false;
  }
  return true;
}

// The scalar updates that close each reduction (the same code for one domain, where the last
// block runs them, and for y-slabs, where k_iter_finish runs them on the sums over the slabs).
__device__ void finish_init(IterScalars* st, const double* s, double sc_floor) {
  st->sc_err = fmax(sqrt(s[1]), sc_floor);
  st->rho = s[0];
  st->rho_prev = 1.0;
  st->nrm = 1.0;
  st->alf = 1.0;
  st->omg = 1.0;
  st->err = sqrt(s[0]) / st->sc_err;
  st->it = 1;
  st->it_done = 0;
  st->done = st->err < st->tol ? 1 : 0;
}
__device__ void finish_apply_dot(IterScalars* st, const double* s) {
  st->nrm = s[0];
  st->alf = st->rho / s[0];
}
__device__ void finish_apply_dots(IterScalars* st, const double* s) {
  const double omg = s[1] / s[0];
  st->omg = omg;
  st->err = sqrt(s[2] - 2 * omg * s[1] + omg * omg * s[0]) / st->sc_err;
}
__device__ void finish_update(IterScalars* st, const double* s, int max_it) {
  st->rho_prev = st->rho;
  st->rho = s[0];
  st->it_done = st->it;
  st->done = (st->err < st->tol || st->it >= max_it) ? 1 : 0;
  st->it += 1;
}
// conjugate gradients: sums <b, b>, <r, r> (MONC's loop runs at least one iteration, so init
// never marks the solve done)
__device__ void finish_cg_init(IterScalars* st, const double* s, double sc_floor) {
  st->sc_err = fmax(sqrt(s[0]), sc_floor);
  st->err = sqrt(s[1]) / st->sc_err;
  st->rho = 0.0;
  st->alf = 0.0;
  st->bet = 0.0;
  st->it = 1;
  st->it_done = 0;
  st->done = 0;
}
// <z, r>: bet = <z, r> / rho and rho = <z, r> (iteration 1: rho = <z, r>)
__device__ void finish_cg_precond(IterScalars* st, const double* s) {
  st->bet = st->it == 1 ? 0.0 : s[0] / st->rho;
  st->rho = s[0];
  st->alf = s[0];
}
// <p', Ap'>: alf = rho / <p', Ap'>
__device__ void finish_cg_apply(IterScalars* st, const double* s) { st->alf = st->alf / s[0]; }
// |r|^2: err, convergence
__device__ void finish_cg_update(IterScalars* st, const double* s, int max_it) {
  st->err = sqrt(s[0]) / st->sc_err;
  st->it_done = st->it;
  st->done = (st->err < st->tol || st->it >= max_it) ? 1 : 0;
  st->it += 1;
}
// the refinement's compatibility shift: sum_k vol(k) sum_ij b over the volume of the domain
__device__ void finish_compat(IterScalars* st, const double* s, const Geom& g) {
  double w = 0.0;
  for (int kk = 2; kk <= g.nz; ++kk) w += g.vol(kk);
  st->shift = s[0] / (w * (double)g.nx * (double)g.ny_total);
}
// the refinement's FP64 residual: <r, r>, <b, b>
__device__ void finish_refine(IterScalars* st, const double* s) {
  st->sc_err = fmax(sqrt(s[1]), 0.0001);
  st->rho = s[0];
  st->err = sqrt(s[0]) / st->sc_err;
  st->done = st->err < st->tol ? 1 : 0;
}

// (A x)(k, j, i) for 2 <= k <= nz (calc_Ax); x(o) gives the value at offset o.  The symmetric
// form scales the horizontal part by A_vol(k).
template <typename W, class X>
__device__ __forceinline__ W apply_A_fn(const Geom& g, X x, int k, int j, int i) {
  const int ie = i + 1 == g.nx ? 0 : i + 1, iw = i == 0 ? g.nx - 1 : i - 1;
  const int jn = j + 1 == g.ny ? 0 : j + 1, js = j == 0 ? g.ny - 1 : j - 1;
  const long long o = g.at(k, j, i);
  const W xc = x(o);
  W h = (W)g.A_n * (x(g.at(k, j, ie)) + x(g.at(k, j, iw))) + (W)g.A_e * (x(g.at(k, jn, i)) + x(g.at(k, js, i)));
  if (g.symm) h = (W)g.avol(k) * h;
  if (k == 2) return h + (W)g.au(k) * x(o + g.plane) + (W)g.ap(k) * xc;
  if (k < g.nz) return h + (W)g.au(k) * x(o + g.plane) + (W)g.ad(k) * x(o - g.plane) + (W)g.ap(k) * xc;
  return h + (W)g.ad(k) * x(o - g.plane) + (W)g.ap(k) * xc;
}
template <typename W>
__device__ __forceinline__ W apply_A(const Geom& g, const W* __restrict__ x, int k, int j, int i) {
  return apply_A_fn<W>(g, [&](long long o) { return x[o]; }, k, j, i);
}

__device__ __forceinline__ int block_id() { return blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z); }

// The point kernels give each thread KZ consecutive levels of its column (blockIdx.z picks the
// group), so that a reduction closes over a quarter as many block partials: with one level per
// thread, the per-block fence, atomic and partial of ~16,000 blocks (256 x 256 x 64) made the
// dot-product kernels three times slower than their memory traffic.
constexpr int KZ = 4;
__device__ __forceinline__ int kz_lo() { return 2 + (int)blockIdx.z * KZ; }
__device__ __forceinline__ int kz_hi(const Geom& g) { return min(g.nz, kz_lo() + KZ - 1); }

// r = b - A x, cr = r; sums <r, r> and <b, b>; initial scalars
template <typename W>
__global__ void __launch_bounds__(NTH) k_bicg_init(Geom g, const W* __restrict__ x, const W* __restrict__ b, W* r, W* cr,
                                                    double* partials, int nblocks, IterScalars* st, double sc_floor) {
  const int i = blockIdx.x * BX + threadIdx.x, j = g.j0 + blockIdx.y * BY + threadIdx.y;
  double v[2] = {0.0, 0.0};
  if (i < g.nx && j < g.j1)
    for (int k = kz_lo(); k <= kz_hi(g); ++k) {
      const long long o = g.at(k, j, i);
      const W rv = b[o] - apply_A<W>(g, x, k, j, i);
      r[o] = rv;
      cr[o] = rv;
      v[0] += (double)rv * (double)rv;
      v[1] += (double)b[o] * (double)b[o];
    }
  block_partials<2>(v, partials, nblocks, block_id());
  double s[2];
  if (last_block_sums<2>(st, partials, nblocks, s)) finish_init(st, s, sc_floor);
}

// column LU solve of the vertical operator: out = M^-1 in (precond); `tmp` holds the forward sweep.
// A thread walks its column level by level; CH levels of its input are loaded before the first of
// them is used, so that the loads are in flight together instead of one round trip per level
// (one thread per column leaves too few warps to hide the latency otherwise).
constexpr int CH = 8;
template <typename W, class In>
__device__ __forceinline__ void column_precond(const Geom& g, In in, W* tmp, int j, int i) {
  long long o = g.at(2, j, i);
  W sp = in(o) * (W)g.lud(2);
  tmp[o] = sp;
  for (int k0 = 3; k0 <= g.nz; k0 += CH) {
    W x[CH];
#pragma unroll
    for (int q = 0; q < CH; ++q)
      if (k0 + q <= g.nz) x[q] = in(o + (long long)(q + 1) * g.plane);
#pragma unroll
    for (int q = 0; q < CH; ++q)
      if (k0 + q <= g.nz) {
        o += g.plane;
        sp = (x[q] - (W)g.ad(k0 + q) * sp) * (W)g.lud(k0 + q);
        tmp[o] = sp;
      }
  }
}

// back substitution sk(k) = tmp(k) - luu(k) sk(k+1) from the top level down to level 2;
// out(o, sk) receives each level's value
template <typename W, class Out>
__device__ __forceinline__ void column_back(const Geom& g, const W* tmp, int j, int i, Out out) {
  long long o = g.at(g.nz, j, i);
  W sk = tmp[o];
  out(o, sk);
  for (int k0 = g.nz - 1; k0 >= 2; k0 -= CH) {
    W t[CH];
#pragma unroll
    for (int q = 0; q < CH; ++q)
      if (k0 - q >= 2) t[q] = tmp[o - (long long)(q + 1) * g.plane];
#pragma unroll
    for (int q = 0; q < CH; ++q)
      if (k0 - q >= 2) {
        o -= g.plane;
        sk = t[q] - (W)g.luu(k0 - q) * sk;
        out(o, sk);
      }
  }
}

// iteration step 1: search direction pp
template <typename W>
__global__ void __launch_bounds__(NTH) k_bicg_direction(Geom g, const W* __restrict__ r, const W* __restrict__ v, W* pp,
                                                         W* tmp, const IterScalars* st) {
  if (st->done) return;
  const int i = blockIdx.x * BX + threadIdx.x, j = g.j0 + blockIdx.y * BY + threadIdx.y;
  if (i >= g.nx || j >= g.j1) return;
  const bool first = st->it == 1;
  const double bet_d = (st->rho / st->rho_prev) * (st->alf / st->omg);
  const W bet = (W)bet_d, bo = (W)(bet_d * st->omg);
  if (first) column_precond<W>(g, [&](long long o) { return r[o]; }, tmp, j, i);
  else column_precond<W>(g, [&](long long o) { return r[o] - bo * v[o]; }, tmp, j, i);
  // back substitution, then pp = s + bet*pp
  column_back<W>(g, tmp, j, i, [&](long long o, W sk) { pp[o] = first ? sk : sk + bet * pp[o]; });
}

// iteration step 2: v = A pp, alf = rho / <cr, v>
template <typename W>
__global__ void __launch_bounds__(NTH) k_bicg_apply_dot(Geom g, const W* __restrict__ pp, const W* __restrict__ cr, W* v,
                                                         double* partials, int nblocks, IterScalars* st) {
  if (st->done) return;
  const int i = blockIdx.x * BX + threadIdx.x, j = g.j0 + blockIdx.y * BY + threadIdx.y;
  double a[1] = {0.0};
  if (i < g.nx && j < g.j1)
    for (int k = kz_lo(); k <= kz_hi(g); ++k) {
      const long long o = g.at(k, j, i);
      const W vv = apply_A<W>(g, pp, k, j, i);
      v[o] = vv;
      a[0] += (double)cr[o] * (double)vv;
    }
  block_partials<1>(a, partials, nblocks, block_id());
  double s[1];
  if (last_block_sums<1>(st, partials, nblocks, s)) finish_apply_dot(st, s);
}

// iteration step 3: s = r - alf*v, cs = M^-1 s
template <typename W>
__global__ void __launch_bounds__(NTH) k_bicg_half_step(Geom g, const W* __restrict__ r, const W* __restrict__ v, W* s_,
                                                         W* cs, W* tmp, const IterScalars* st) {
  if (st->done) return;
  const int i = blockIdx.x * BX + threadIdx.x, j = g.j0 + blockIdx.y * BY + threadIdx.y;
  if (i >= g.nx || j >= g.j1) return;
  const W alf = (W)st->alf;
  column_precond<W>(g, [&](long long o) {
    const W sv = r[o] - alf * v[o];
    s_[o] = sv;
    return sv;
  }, tmp, j, i);
  column_back<W>(g, tmp, j, i, [&](long long o, W ck) { cs[o] = ck; });
}

// iteration step 4: t = A cs; tt, ts, ss; omg, err
template <typename W>
__global__ void __launch_bounds__(NTH) k_bicg_apply_dots(Geom g, const W* __restrict__ cs, const W* __restrict__ s_, W* t,
                                                          double* partials, int nblocks, IterScalars* st) {
  if (st->done) return;
  const int i = blockIdx.x * BX + threadIdx.x, j = g.j0 + blockIdx.y * BY + threadIdx.y;
  double a[3] = {0.0, 0.0, 0.0};
  if (i < g.nx && j < g.j1)
    for (int k = kz_lo(); k <= kz_hi(g); ++k) {
      const long long o = g.at(k, j, i);
      const W tv = apply_A<W>(g, cs, k, j, i);
      t[o] = tv;
      const double td = (double)tv, sd = (double)s_[o];
      a[0] += td * td;
      a[1] += td * sd;
      a[2] += sd * sd;
    }
  block_partials<3>(a, partials, nblocks, block_id());
  double s[3];
  if (last_block_sums<3>(st, partials, nblocks, s)) finish_apply_dots(st, s);
}

// iteration step 5: x += alf*pp + omg*cs, r = s - omg*t, rho = <r, cr>, convergence test
template <typename W>
__global__ void __launch_bounds__(NTH) k_bicg_update(Geom g, W* x, const W* __restrict__ pp, const W* __restrict__ cs,
                                                      const W* __restrict__ s_, const W* __restrict__ t, W* r,
                                                      const W* __restrict__ cr, double* partials, int nblocks,
                                                      IterScalars* st, int max_it) {
  if (st->done) return;
  const int i = blockIdx.x * BX + threadIdx.x, j = g.j0 + blockIdx.y * BY + threadIdx.y;
  double a[1] = {0.0};
  if (i < g.nx && j < g.j1) {
    const W alf = (W)st->alf, omg = (W)st->omg;
    for (int k = kz_lo(); k <= kz_hi(g); ++k) {
      const long long o = g.at(k, j, i);
      x[o] = x[o] + alf * pp[o] + omg * cs[o];
      const W rv = s_[o] - omg * t[o];
      r[o] = rv;
      a[0] += (double)rv * (double)cr[o];
    }
  }
  block_partials<1>(a, partials, nblocks, block_id());
  double s[1];
  if (last_block_sums<1>(st, partials, nblocks, s)) finish_update(st, s, max_it);
}

// y-slabs: close reduction `which` with the sums over all slabs: BiCGStab 0 init, 1 apply_dot,
// 2 apply_dots, 3 update; conjugate gradients 4 init, 5 precond, 6 apply, 7 update; the FP32-mixed
// refinement 8 compatibility sum, 9 FP64 residual
__global__ void k_iter_finish(IterScalars* st, const double* __restrict__ sums, int which, double sc_floor,
                              int max_it, Geom g) {
  if (threadIdx.x != 0) return;
  const double s[3] = {sums[0], sums[1], sums[2]};
  if (which == 0) { finish_init(st, s, sc_floor); return; }
  if (which == 4) { finish_cg_init(st, s, sc_floor); return; }
  if (which == 8) { finish_compat(st, s, g); return; }
  if (which == 9) { finish_refine(st, s); return; }
  if (st->done) return;
  switch (which) {
    case 1: finish_apply_dot(st, s); break;
    case 2: finish_apply_dots(st, s); break;
    case 3: finish_update(st, s, max_it); break;
    case 5: finish_cg_precond(st, s); break;
    case 6: finish_cg_apply(st, s); break;
    default: finish_cg_update(st, s, max_it); break;
  }
}


// ---- conjugate gradients (cg_solver, symmetric form) -------------------------------------------
// r = b*A_vol - A x (b*A_vol when scale_rhs, else b), sc_err = max(|b*A_vol|, sc_floor); MONC's
// loop runs at least one iteration, so the solve is never marked done here
template <typename W>
__global__ void __launch_bounds__(NTH) k_cg_init(Geom g, const W* __restrict__ x, const W* __restrict__ b, W* r,
                                                  double* partials, int nblocks, IterScalars* st, double sc_floor,
                                                  int scale_rhs) {
  const int i = blockIdx.x * BX + threadIdx.x, j = g.j0 + blockIdx.y * BY + threadIdx.y;
  double v[2] = {0.0, 0.0};
  if (i < g.nx && j < g.j1)
    for (int k = kz_lo(); k <= kz_hi(g); ++k) {
      const long long o = g.at(k, j, i);
      const W bv = scale_rhs ? b[o] * (W)g.avol(k) : b[o];
      const W rv = bv - apply_A<W>(g, x, k, j, i);
      r[o] = rv;
      v[0] += (double)bv * (double)bv;
      v[1] += (double)rv * (double)rv;
    }
  block_partials<2>(v, partials, nblocks, block_id());
  double s[2];
  if (last_block_sums<2>(st, partials, nblocks, s)) finish_cg_init(st, s, sc_floor);
}

// z = M^-1 r per column, <z, r>; bet = <z, r> / rho and rho = <z, r> (iteration 1: rho = <z, r>)
template <typename W>
__global__ void __launch_bounds__(NTH) k_cg_precond(Geom g, const W* __restrict__ r, W* z, W* tmp, double* partials,
                                                     int nblocks, IterScalars* st) {
  if (st->done) return;
  const int i = blockIdx.x * BX + threadIdx.x, j = g.j0 + blockIdx.y * BY + threadIdx.y;
  double a[1] = {0.0};
  if (i < g.nx && j < g.j1) {
    column_precond<W>(g, [&](long long o) { return r[o]; }, tmp, j, i);
    column_back<W>(g, tmp, j, i, [&](long long o, W zk) {
      z[o] = zk;
      a[0] += (double)zk * (double)r[o];
    });
  }
  block_partials<1>(a, partials, nblocks, block_id());
  double s[1];
  if (last_block_sums<1>(st, partials, nblocks, s)) finish_cg_precond(st, s);
}

// p' = z + bet*p (p' = z on iteration 1) into p_new, Ap' into Ax, alf = rho / <p', Ap'>.  Every
// point forms p' at its stencil neighbours from z and the old p itself, with the same rounding as
// the neighbour's own store, so the kernel needs no second pass.
template <typename W>
__device__ __forceinline__ W axpy_rn(W a, W x, W y) {
  if constexpr (sizeof(W) == 8) return __dadd_rn(y, __dmul_rn(a, x));
  else return __fadd_rn(y, __fmul_rn(a, x));
}
template <typename W>
__global__ void __launch_bounds__(NTH) k_cg_apply(Geom g, const W* __restrict__ z, const W* __restrict__ p_old,
                                                   W* p_new, W* Ax, double* partials, int nblocks, IterScalars* st) {
  if (st->done) return;
  const int i = blockIdx.x * BX + threadIdx.x, j = g.j0 + blockIdx.y * BY + threadIdx.y;
  const bool first = st->it == 1;
  const W bet = (W)st->bet;
  auto pn = [&](long long o) { return first ? z[o] : axpy_rn<W>(bet, p_old[o], z[o]); };
  double a[1] = {0.0};
  if (i < g.nx && j < g.j1)
    for (int k = kz_lo(); k <= kz_hi(g); ++k) {
      const long long o = g.at(k, j, i);
      const W pc = pn(o);
      p_new[o] = pc;
      const W av = apply_A_fn<W>(g, pn, k, j, i);
      Ax[o] = av;
      a[0] += (double)pc * (double)av;
    }
  block_partials<1>(a, partials, nblocks, block_id());
  double s[1];
  if (last_block_sums<1>(st, partials, nblocks, s)) finish_cg_apply(st, s);
}

// x += alf*p', r -= alf*Ap', err = |r| / sc_err, convergence
template <typename W>
__global__ void __launch_bounds__(NTH) k_cg_update(Geom g, W* x, const W* __restrict__ p, const W* __restrict__ Ax, W* r,
                                                    double* partials, int nblocks, IterScalars* st, int max_it) {
  if (st->done) return;
  const int i = blockIdx.x * BX + threadIdx.x, j = g.j0 + blockIdx.y * BY + threadIdx.y;
  double a[1] = {0.0};
  if (i < g.nx && j < g.j1) {
    const W alf = (W)st->alf;
    for (int k = kz_lo(); k <= kz_hi(g); ++k) {
      const long long o = g.at(k, j, i);
      x[o] = x[o] + alf * p[o];
      const W rv = r[o] - alf * Ax[o];
      r[o] = rv;
      a[0] += (double)rv * (double)rv;
    }
  }
  block_partials<1>(a, partials, nblocks, block_id());
  double s[1];
  if (last_block_sums<1>(st, partials, nblocks, s)) finish_cg_update(st, s, max_it);
}

// FP64 residual of the refinement: r = b - A x (levels 2..nz) with <r, r>, <b, b>
__global__ void __launch_bounds__(NTH) k_refine_residual(Geom g, const double* __restrict__ x, const double* __restrict__ b,
                                                          double* r, float* r32, double* partials, int nblocks,
                                                          IterScalars* st) {
  const int i = blockIdx.x * BX + threadIdx.x, j = g.j0 + blockIdx.y * BY + threadIdx.y;
  double v[2] = {0.0, 0.0};
  if (i < g.nx && j < g.j1)
    for (int k = kz_lo(); k <= kz_hi(g); ++k) {
      const long long o = g.at(k, j, i);
      const double bv = g.symm ? b[o] * g.avol(k) : b[o];
      const double rv = bv - apply_A<double>(g, x, k, j, i);
      r[o] = rv;
      r32[o] = (float)rv;
      v[0] += rv * rv;
      v[1] += bv * bv;
    }
  block_partials<2>(v, partials, nblocks, block_id());
  double s[2];
  if (last_block_sums<2>(st, partials, nblocks, s)) finish_refine(st, s);
}

// The horizontal-mean problem is singular: sum_k rhon(k) dz(k) sum_ij (A x)(k, j, i) = 0 for any x.
// A right-hand side rounded to FP32 carries an incompatible part of that size, which an FP32
// solve cannot remove; the refinement takes it out of b first (a constant shift of levels 2..nz).
__global__ void __launch_bounds__(NTH) k_compat_sum(Geom g, const double* __restrict__ b, double* partials, int nblocks,
                                                     IterScalars* st) {
  const int i = blockIdx.x * BX + threadIdx.x, j = g.j0 + blockIdx.y * BY + threadIdx.y;
  double v[1] = {0.0};
  if (i < g.nx && j < g.j1)
    for (int k = kz_lo(); k <= kz_hi(g); ++k) v[0] += g.vol(k) * b[g.at(k, j, i)];
  block_partials<1>(v, partials, nblocks, block_id());
  double s[1];
  if (last_block_sums<1>(st, partials, nblocks, s)) finish_compat(st, s, g);
}
__global__ void k_compat_shift(Geom g, double* b, const IterScalars* st) {
  const double c = st->shift;
  const long long n = (long long)g.nz * g.plane;
  for (long long q = g.plane + blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    b[q] = b[q] - c;
}

template <typename A, typename B>
__global__ void k_convert_levels(const A* __restrict__ a, B* b, long long n) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    b[q] = (B)a[q];
}
__global__ void k_add_correction(double* x, const float* __restrict__ e, long long plane, long long n, double sign) {
  for (long long q = plane + blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    x[q] = x[q] + sign * (double)e[q];
}

template <typename W>
struct Work {
  W *x, *b, *r, *cr, *pp, *v, *t, *s, *cs, *tmp;
};

}  // namespace

struct IterSolverDev {
  Geom g;
  bool fp32 = false;
  bool symm = false;  // conjugate gradients on the symmetric form (MGPU_ITER_CG)
  int max_it = 0;
  double tol = 0.0;
  double* coef = nullptr;
  double* partials = nullptr;
  int nblocks = 0;
  IterScalars* st = nullptr;
  IterScalars* st_host = nullptr;
  Work<double> w64{};
  Work<float> w32{};
  double* r64 = nullptr;  // refinement residual (FP32-mixed model)
  int pending = -1;       // y-slab steps: the reduction iter_slab_finish closes next
  int cg_n = 0;           // y-slab conjugate gradients: iterations done (which direction buffer is old)
  bool inner32 = false;   // y-slab FP32-mixed: the FP32 correction solve is running
  double sc_floor = 0.0001;
  bool scale_rhs = true;
  int inner_its = 0;      // y-slab FP32-mixed: FP32 iterations of this solve
  double slab_err = 0.0, slab_prev_err = 0.0;  // y-slab FP32-mixed: the last two FP64 residuals
  std::vector<void*> allocs;
  dim3 grid_pt, grid_col, block;
};

static int dev_alloc(IterSolverDev* it, void** p, size_t bytes) {
  if (cudaMalloc(p, bytes) != cudaSuccess) return MGPU_ERR_CUDA;
  cudaMemset(*p, 0, bytes);
  it->allocs.push_back(*p);
  return MGPU_OK;
}

IterSolverDev* iter_create(const Scalars& s, const RefState& rs, const mgpu_config& cfg, bool fp32, int* status, int j0,
                           int j1, int ny_total) {
  *status = MGPU_OK;
  if (j1 < 0) j1 = s.ny;
  if (ny_total < 0) ny_total = s.ny;
  if (cfg.solver_type != MGPU_ITER_BICGSTAB && cfg.solver_type != MGPU_ITER_CG) {
    std::fprintf(stderr, "iterative solver: unknown solver_type %d\n", cfg.solver_type);
    *status = MGPU_ERR_UNSUPPORTED;
    return nullptr;
  }
  auto* it = new IterSolverDev();
  const int nz = s.nz;
  it->fp32 = fp32;
  it->symm = cfg.solver_type == MGPU_ITER_CG;
  it->max_it = cfg.max_iterations > 0 ? cfg.max_iterations : 1;
  it->tol = cfg.tolerance;
  // set_matrix_for_poisson (iterativesolver.F90:559-602): BiCGStab form (A_vol = 1,
  // d_sc = rdz/rhon) or, for conjugate gradients, the symmetric form (A_vol = dz, d_sc = 1/rhon)
  const double A_n = rs.cx * rs.cx, A_e = rs.cy * rs.cy;
  const double concat = A_n + A_n + A_e + A_e;
  std::vector<double> c((size_t)NCOEF * (nz + 2), 0.0);
  double* Au = c.data();
  double* Ad = Au + (nz + 2);
  double* Ap = Ad + (nz + 2);
  double* lud = Ap + (nz + 2);
  double* luu = lud + (nz + 2);
  double* vol = luu + (nz + 2);
  double* avol = vol + (nz + 2);
  for (int k = 2; k <= nz; ++k) vol[k] = rs.rhon[k] * rs.dz[k];
  for (int k = 2; k <= nz; ++k) {
    avol[k] = it->symm ? rs.dz[k] : 1.0;
    const double d_sc = it->symm ? 1.0 / rs.rhon[k] : rs.rdz[k] / rs.rhon[k];
    Au[k] = (k == nz) ? 0.0 : rs.rho[k] * rs.rdzn[k + 1];
    Ad[k] = (k == 2) ? 0.0 : rs.rho[k - 1] * rs.rdzn[k];
    Ap[k] = d_sc * (-(Au[k] + Ad[k])) - concat * avol[k];
    Au[k] = d_sc * Au[k];
    Ad[k] = d_sc * Ad[k];
  }
  lud[2] = 1.0 / Ap[2];
  luu[2] = lud[2] * Au[2];
  for (int k = 3; k <= nz; ++k) {
    lud[k] = 1.0 / (Ap[k] - Ad[k] * luu[k - 1]);
    luu[k] = Au[k] * lud[k];
  }
  auto fail = [&](int code) {
    iter_destroy(it);
    *status = code;
    return (IterSolverDev*)nullptr;
  };
  if (dev_alloc(it, (void**)&it->coef, c.size() * sizeof(double))) return fail(MGPU_ERR_CUDA);
  cudaMemcpy(it->coef, c.data(), c.size() * sizeof(double), cudaMemcpyHostToDevice);
  it->g = Geom{s.nx, s.ny, nz, it->symm ? 1 : 0, s.plane, A_n, A_e, it->coef, j0, j1, ny_total};
  it->block = dim3(BX, BY, 1);
  it->grid_col = dim3((s.nx + BX - 1) / BX, (j1 - j0 + BY - 1) / BY, 1);
  it->grid_pt = dim3(it->grid_col.x, it->grid_col.y, (nz - 1 + KZ - 1) / KZ);
  it->nblocks = (int)(it->grid_pt.x * it->grid_pt.y * it->grid_pt.z);
  if (dev_alloc(it, (void**)&it->partials, sizeof(double) * 3 * (size_t)it->nblocks)) return fail(MGPU_ERR_CUDA);
  if (dev_alloc(it, (void**)&it->st, sizeof(IterScalars))) return fail(MGPU_ERR_CUDA);
  if (cudaMallocHost((void**)&it->st_host, sizeof(IterScalars)) != cudaSuccess) return fail(MGPU_ERR_CUDA);
  const size_t n = (size_t)nz * s.plane;
  // FP64 arrays: the solve itself (FP64 model) or the refinement's x, b, r (FP32-mixed model)
  double** f64[] = {&it->w64.x, &it->w64.b, &it->w64.r, &it->w64.cr, &it->w64.pp, &it->w64.v,
                    &it->w64.t, &it->w64.s, &it->w64.cs, &it->w64.tmp};
  const int n64 = fp32 ? 2 : 10;
  for (int q = 0; q < n64; ++q)
    if (dev_alloc(it, (void**)f64[q], n * sizeof(double))) return fail(MGPU_ERR_CUDA);
  if (fp32) {
    if (dev_alloc(it, (void**)&it->r64, n * sizeof(double))) return fail(MGPU_ERR_CUDA);
    float** f32[] = {&it->w32.x, &it->w32.b, &it->w32.r, &it->w32.cr, &it->w32.pp, &it->w32.v,
                     &it->w32.t, &it->w32.s, &it->w32.cs, &it->w32.tmp};
    for (float** pp : f32)
      if (dev_alloc(it, (void**)pp, n * sizeof(float))) return fail(MGPU_ERR_CUDA);
  }
  if (cudaDeviceSynchronize() != cudaSuccess) return fail(MGPU_ERR_CUDA);
  return it;
}

void iter_destroy(IterSolverDev* it) {
  if (!it) return;
  for (void* p : it->allocs) cudaFree(p);
  if (it->st_host) cudaFreeHost(it->st_host);
  delete it;
}

// BiCGStab on work arrays w (x is the initial guess and the result); returns the iterations done
template <typename W>
static int run_bicgstab(IterSolverDev* it, Work<W>& w, double tol, double sc_floor, cudaStream_t st, int64_t* launches,
                        int* iterations, double* residual) {
  IterScalars init{};
  init.tol = tol;
  it->st_host[0] = init;
  if (cudaMemcpyAsync(it->st, it->st_host, sizeof(IterScalars), cudaMemcpyHostToDevice, st) != cudaSuccess)
    return MGPU_ERR_CUDA;
  const Geom& g = it->g;
  k_bicg_init<W><<<it->grid_pt, it->block, 0, st>>>(g, w.x, w.b, w.r, w.cr, it->partials, it->nblocks, it->st, sc_floor);
  *launches += 1;
  constexpr int BATCH = 4;
  for (int done = 0; done < it->max_it;) {
    // the first batch checks convergence of the initial guess after one iteration's launches
    for (int q = 0; q < BATCH; ++q) {
      k_bicg_direction<W><<<it->grid_col, it->block, 0, st>>>(g, w.r, w.v, w.pp, w.tmp, it->st);
      k_bicg_apply_dot<W><<<it->grid_pt, it->block, 0, st>>>(g, w.pp, w.cr, w.v, it->partials, it->nblocks, it->st);
      k_bicg_half_step<W><<<it->grid_col, it->block, 0, st>>>(g, w.r, w.v, w.s, w.cs, w.tmp, it->st);
      k_bicg_apply_dots<W><<<it->grid_pt, it->block, 0, st>>>(g, w.cs, w.s, w.t, it->partials, it->nblocks, it->st);
      k_bicg_update<W><<<it->grid_pt, it->block, 0, st>>>(g, w.x, w.pp, w.cs, w.s, w.t, w.r, w.cr, it->partials,
                                                          it->nblocks, it->st, it->max_it);
      *launches += 5;
    }
    done += BATCH;
    if (cudaMemcpyAsync(it->st_host, it->st, sizeof(IterScalars), cudaMemcpyDeviceToHost, st) != cudaSuccess)
      return MGPU_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return MGPU_ERR_CUDA;
    if (it->st_host->done) break;
  }
  if (cudaGetLastError() != cudaSuccess) return MGPU_ERR_CUDA;
  *iterations = it->st_host->it_done;
  *residual = it->st_host->err;
  return it->st_host->err < tol ? MGPU_OK : MGPU_ERR_NOT_CONVERGED;
}

// conjugate gradients on work arrays w: x (initial guess, result), b, r, z in s, p in pp / cs
// (alternating), A p in v, column scratch in tmp
template <typename W>
static int run_cg(IterSolverDev* it, Work<W>& w, double tol, double sc_floor, bool scale_rhs, cudaStream_t st,
                  int64_t* launches, int* iterations, double* residual) {
  IterScalars init{};
  init.tol = tol;
  it->st_host[0] = init;
  if (cudaMemcpyAsync(it->st, it->st_host, sizeof(IterScalars), cudaMemcpyHostToDevice, st) != cudaSuccess)
    return MGPU_ERR_CUDA;
  const Geom& g = it->g;
  const int ncol = (int)(it->grid_col.x * it->grid_col.y);
  k_cg_init<W><<<it->grid_pt, it->block, 0, st>>>(g, w.x, w.b, w.r, it->partials, it->nblocks, it->st, sc_floor,
                                                   scale_rhs ? 1 : 0);
  *launches += 1;
  W* pbuf[2] = {w.pp, w.cs};
  int n = 0;
  constexpr int BATCH = 4;
  for (int done = 0; done < it->max_it;) {
    for (int q = 0; q < BATCH; ++q, ++n) {
      W* p_old = pbuf[n & 1];
      W* p_new = pbuf[(n + 1) & 1];
      k_cg_precond<W><<<it->grid_col, it->block, 0, st>>>(g, w.r, w.s, w.tmp, it->partials, ncol, it->st);
      k_cg_apply<W><<<it->grid_pt, it->block, 0, st>>>(g, w.s, p_old, p_new, w.v, it->partials, it->nblocks, it->st);
      k_cg_update<W><<<it->grid_pt, it->block, 0, st>>>(g, w.x, p_new, w.v, w.r, it->partials, it->nblocks, it->st,
                                                        it->max_it);
      *launches += 3;
    }
    done += BATCH;
    if (cudaMemcpyAsync(it->st_host, it->st, sizeof(IterScalars), cudaMemcpyDeviceToHost, st) != cudaSuccess)
      return MGPU_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return MGPU_ERR_CUDA;
    if (it->st_host->done) break;
  }
  if (cudaGetLastError() != cudaSuccess) return MGPU_ERR_CUDA;
  *iterations = it->st_host->it_done;
  *residual = it->st_host->err;
  return it->st_host->err < tol ? MGPU_OK : MGPU_ERR_NOT_CONVERGED;
}

static int solve_fp64(IterSolverDev* it, const Scalars& s, double* p, cudaStream_t st, int64_t* launches,
                      int* iterations, double* residual) {
  if (!it || it->fp32) return MGPU_ERR_ARGUMENT;
  // psource = p; the initial guess is the previous solution (iterativesolver.F90:95-106)
  const size_t bytes = (size_t)s.nz * s.plane * sizeof(double);
  if (cudaMemcpyAsync(it->w64.b, p, bytes, cudaMemcpyDeviceToDevice, st) != cudaSuccess) return MGPU_ERR_CUDA;
  int rc = it->symm ? run_cg<double>(it, it->w64, it->tol, 0.0001, true, st, launches, iterations, residual)
                    : run_bicgstab<double>(it, it->w64, it->tol, 0.0001, st, launches, iterations, residual);
  if (rc != MGPU_OK && rc != MGPU_ERR_NOT_CONVERGED) return rc;
  // p = x, level 1 included (the solution keeps the previous solve's level 1)
  if (cudaMemcpyAsync(p, it->w64.x, bytes, cudaMemcpyDeviceToDevice, st) != cudaSuccess) return MGPU_ERR_CUDA;
  return rc;
}

// The relative residual reduction asked of an FP32 correction solve: enough to bring the FP64
// residual err to half the tolerance, but no more than a factor 1e-3, which the FP32 iteration
// reaches in a few tens of iterations.  A fixed 1e-5 over-solved at loose tolerances and, on large
// grids (512 x 512 x 160), ran into the FP32 iteration's attainable accuracy and the iteration cap.
static double inner_tolerance(double err, double tol) {
  const double t = 0.5 * tol / err;
  return t < 1e-3 ? 1e-3 : (t > 0.5 ? 0.5 : t);
}

static int solve_mixed(IterSolverDev* it, const Scalars& s, float* p, cudaStream_t st, int64_t* launches,
                       int* iterations, double* residual) {
  if (!it || !it->fp32) return MGPU_ERR_ARGUMENT;
  const long long n = (long long)s.nz * s.plane;
  const Geom& g = it->g;
  double* x64 = it->w64.x;
  double* b64 = it->w64.b;
  k_convert_levels<float, double><<<592, 256, 0, st>>>(p, b64, n);
  {
    IterScalars init{};
    it->st_host[0] = init;
    if (cudaMemcpyAsync(it->st, it->st_host, sizeof(IterScalars), cudaMemcpyHostToDevice, st) != cudaSuccess)
      return MGPU_ERR_CUDA;
  }
  k_compat_sum<<<it->grid_pt, it->block, 0, st>>>(g, b64, it->partials, it->nblocks, it->st);
  k_compat_shift<<<592, 256, 0, st>>>(g, b64, it->st);
  *launches += 3;
  int total = 0;
  double err = 0.0, prev_err = 0.0;
  constexpr int MAX_REFINE = 8;
  int rc = MGPU_ERR_NOT_CONVERGED;
  for (int outer = 0; outer < MAX_REFINE; ++outer) {
    IterScalars init{};
    init.tol = it->tol;
    it->st_host[0] = init;
    if (cudaMemcpyAsync(it->st, it->st_host, sizeof(IterScalars), cudaMemcpyHostToDevice, st) != cudaSuccess)
      return MGPU_ERR_CUDA;
    k_refine_residual<<<it->grid_pt, it->block, 0, st>>>(g, x64, b64, it->r64, it->w32.b, it->partials, it->nblocks,
                                                        it->st);
    *launches += 1;
    if (cudaMemcpyAsync(it->st_host, it->st, sizeof(IterScalars), cudaMemcpyDeviceToHost, st) != cudaSuccess)
      return MGPU_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return MGPU_ERR_CUDA;
    err = it->st_host->err;
    if (it->st_host->done) { rc = MGPU_OK; break; }
    if (outer > 0 && !(err < prev_err)) {
      // the last correction did not reduce the FP64 residual: take it back and stop
      k_add_correction<<<592, 256, 0, st>>>(x64, it->w32.x, s.plane, n, -1.0);
      *launches += 1;
      err = prev_err;
      break;
    }
    prev_err = err;
    // FP32 correction solve A e = r, from e = 0, to the relative residual inner_tolerance asks
    if (cudaMemsetAsync(it->w32.x, 0, (size_t)n * sizeof(float), st) != cudaSuccess) return MGPU_ERR_CUDA;
    int its = 0;
    double inner = 0.0;
    const double itol = inner_tolerance(err, it->tol);
    int irc = it->symm ? run_cg<float>(it, it->w32, itol, 1e-300, false, st, launches, &its, &inner)
                       : run_bicgstab<float>(it, it->w32, itol, 1e-300, st, launches, &its, &inner);
    if (irc != MGPU_OK && irc != MGPU_ERR_NOT_CONVERGED) return irc;
    total += its;
    k_add_correction<<<592, 256, 0, st>>>(x64, it->w32.x, s.plane, n, 1.0);
    *launches += 1;
  }
  k_convert_levels<double, float><<<592, 256, 0, st>>>(x64, p, n);
  *launches += 1;
  if (cudaGetLastError() != cudaSuccess) return MGPU_ERR_CUDA;
  *iterations = total;
  *residual = err;
  return rc;
}

// ---- the iterative solve over y-slabs, one step at a time --------------------------------------
// The driver runs the iterations of run_bicgstab / run_cg (and, for FP32-mixed models, the
// refinement of solve_mixed around them) step by step: it exchanges the halo rows of the vectors A
// is applied to before the steps that apply it, and sums each reducing step's dot products over
// the slabs before iter_slab_finish closes the reduction with the update the single-domain
// kernel's last block makes.
static void slab_scalars(IterSolverDev* it, double tol, cudaStream_t st) {
  IterScalars init{};
  init.tol = tol;
  init.ext = 1;
  it->st_host[0] = init;
  cudaMemcpyAsync(it->st, it->st_host, sizeof(IterScalars), cudaMemcpyHostToDevice, st);
}

int iter_slab_begin(IterSolverDev* it, const void* p, size_t n, cudaStream_t st) {
  if (!it) return MGPU_ERR_ARGUMENT;
  if (it->fp32) {
    // the refinement's FP64 right-hand side; x (FP64) keeps the last solution
    k_convert_levels<float, double><<<592, 256, 0, st>>>(static_cast<const float*>(p), it->w64.b, (long long)n);
  } else {
    // psource = p; the initial guess is the previous solution (iterativesolver.F90:95-106)
    if (cudaMemcpyAsync(it->w64.b, p, n * sizeof(double), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
      return MGPU_ERR_CUDA;
  }
  slab_scalars(it, it->tol, st);
  it->pending = -1;
  it->cg_n = 0;
  it->inner32 = false;
  it->sc_floor = 0.0001;
  it->scale_rhs = true;
  return cudaGetLastError() == cudaSuccess ? MGPU_OK : MGPU_ERR_CUDA;
}

// the two search-direction buffers of conjugate gradients alternate: p_old = pbuf[n & 1]
template <typename W>
static W* cg_p(Work<W>& w, int n) { return (n & 1) ? w.cs : w.pp; }

template <typename W>
static int solver_step(IterSolverDev* it, Work<W>& w, int step, int* nsum, cudaStream_t st) {
  const Geom& g = it->g;
  if (it->symm) {
    const int ncol = (int)(it->grid_col.x * it->grid_col.y);
    switch (step) {
      case MGPU_SLAB_ITER_INIT:
        // MONC's symmetric form: the FP64 solve scales the right-hand side by A_vol (run_cg)
        k_cg_init<W><<<it->grid_pt, it->block, 0, st>>>(g, w.x, w.b, w.r, it->partials, it->nblocks, it->st,
                                                         it->sc_floor, it->scale_rhs ? 1 : 0);
        it->pending = 4; *nsum = 2; return MGPU_OK;
      case MGPU_SLAB_ITER_PRECOND:
        k_cg_precond<W><<<it->grid_col, it->block, 0, st>>>(g, w.r, w.s, w.tmp, it->partials, ncol, it->st);
        it->pending = 5; *nsum = 1; return MGPU_OK;
      case MGPU_SLAB_ITER_APPLY:
        k_cg_apply<W><<<it->grid_pt, it->block, 0, st>>>(g, w.s, cg_p(w, it->cg_n), cg_p(w, it->cg_n + 1), w.v,
                                                          it->partials, it->nblocks, it->st);
        it->pending = 6; *nsum = 1; return MGPU_OK;
      case MGPU_SLAB_ITER_UPDATE:
        k_cg_update<W><<<it->grid_pt, it->block, 0, st>>>(g, w.x, cg_p(w, it->cg_n + 1), w.v, w.r, it->partials,
                                                           it->nblocks, it->st, it->max_it);
        it->cg_n += 1;
        it->pending = 7; *nsum = 1; return MGPU_OK;
    }
    return MGPU_ERR_ARGUMENT;
  }
  switch (step) {
    case MGPU_SLAB_ITER_INIT:
      k_bicg_init<W><<<it->grid_pt, it->block, 0, st>>>(g, w.x, w.b, w.r, w.cr, it->partials, it->nblocks, it->st,
                                                        it->sc_floor);
      it->pending = 0; *nsum = 2; return MGPU_OK;
    case MGPU_SLAB_ITER_DIRECTION:
      k_bicg_direction<W><<<it->grid_col, it->block, 0, st>>>(g, w.r, w.v, w.pp, w.tmp, it->st);
      return MGPU_OK;
    case MGPU_SLAB_ITER_APPLY:
      k_bicg_apply_dot<W><<<it->grid_pt, it->block, 0, st>>>(g, w.pp, w.cr, w.v, it->partials, it->nblocks, it->st);
      it->pending = 1; *nsum = 1; return MGPU_OK;
    case MGPU_SLAB_ITER_HALF_STEP:
      k_bicg_half_step<W><<<it->grid_col, it->block, 0, st>>>(g, w.r, w.v, w.s, w.cs, w.tmp, it->st);
      return MGPU_OK;
    case MGPU_SLAB_ITER_APPLY2:
      k_bicg_apply_dots<W><<<it->grid_pt, it->block, 0, st>>>(g, w.cs, w.s, w.t, it->partials, it->nblocks, it->st);
      it->pending = 2; *nsum = 3; return MGPU_OK;
    case MGPU_SLAB_ITER_UPDATE:
      k_bicg_update<W><<<it->grid_pt, it->block, 0, st>>>(g, w.x, w.pp, w.cs, w.s, w.t, w.r, w.cr, it->partials,
                                                          it->nblocks, it->st, it->max_it);
      it->pending = 3; *nsum = 1; return MGPU_OK;
  }
  return MGPU_ERR_ARGUMENT;
}

int iter_slab_step(IterSolverDev* it, int step, double* d_sums, cudaStream_t st, int64_t* launches) {
  const Geom& g = it->g;
  const long long n = (long long)g.nz * g.plane;
  int nsum = 0;
  switch (step) {
    // the FP32-mixed refinement (solve_mixed)
    case MGPU_SLAB_ITER_COMPAT:
      if (!it->fp32) return MGPU_ERR_ARGUMENT;
      k_compat_sum<<<it->grid_pt, it->block, 0, st>>>(g, it->w64.b, it->partials, it->nblocks, it->st);
      it->pending = 8;
      nsum = 1;
      break;
    case MGPU_SLAB_ITER_SHIFT:
      if (!it->fp32) return MGPU_ERR_ARGUMENT;
      k_compat_shift<<<592, 256, 0, st>>>(g, it->w64.b, it->st);
      break;
    case MGPU_SLAB_ITER_REFINE:
      if (!it->fp32) return MGPU_ERR_ARGUMENT;
      slab_scalars(it, it->tol, st);
      k_refine_residual<<<it->grid_pt, it->block, 0, st>>>(g, it->w64.x, it->w64.b, it->r64, it->w32.b, it->partials,
                                                          it->nblocks, it->st);
      it->inner32 = false;
      it->pending = 9;
      nsum = 2;
      break;
    case MGPU_SLAB_ITER_INNER:
      // the FP32 correction solve A e = r, from e = 0, to the relative residual inner_tolerance asks
      if (!it->fp32) return MGPU_ERR_ARGUMENT;
      if (cudaMemsetAsync(it->w32.x, 0, (size_t)n * sizeof(float), st) != cudaSuccess) return MGPU_ERR_CUDA;
      slab_scalars(it, inner_tolerance(it->slab_err, it->tol), st);
      it->inner32 = true;
      it->sc_floor = 1e-300;
      it->scale_rhs = false;
      it->cg_n = 0;
      break;
    case MGPU_SLAB_ITER_CORRECT:
    case MGPU_SLAB_ITER_UNCORRECT:
      if (!it->fp32) return MGPU_ERR_ARGUMENT;
      k_add_correction<<<592, 256, 0, st>>>(it->w64.x, it->w32.x, g.plane, n,
                                            step == MGPU_SLAB_ITER_CORRECT ? 1.0 : -1.0);
      // taking back a correction that did not reduce the residual: the previous one stands
      if (step == MGPU_SLAB_ITER_UNCORRECT) it->slab_err = it->slab_prev_err;
      it->inner32 = false;
      break;
    default: {
      if (it->fp32 && !it->inner32) return MGPU_ERR_ARGUMENT;
      const int rc = it->fp32 ? solver_step<float>(it, it->w32, step, &nsum, st)
                              : solver_step<double>(it, it->w64, step, &nsum, st);
      if (rc) return rc;
    }
  }
  *launches += 1;
  if (nsum) {
    // this slab's sums (zeros past nsum), for the driver to add over the slabs
    if (cudaMemsetAsync(d_sums, 0, 3 * sizeof(double), st) != cudaSuccess ||
        cudaMemcpyAsync(d_sums, reinterpret_cast<const char*>(it->st) + offsetof(IterScalars, loc),
                        nsum * sizeof(double), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
      return MGPU_ERR_CUDA;
  }
  return cudaGetLastError() == cudaSuccess ? MGPU_OK : MGPU_ERR_CUDA;
}

int iter_slab_finish(IterSolverDev* it, const double* d_sums, cudaStream_t st, int64_t* launches, int* done,
                     double* err) {
  const int which = it->pending;
  if (which < 0) return MGPU_ERR_ARGUMENT;
  k_iter_finish<<<1, 32, 0, st>>>(it->st, d_sums, which, it->sc_floor, it->max_it, it->g);
  *launches += 1;
  it->pending = -1;
  if (cudaMemcpyAsync(it->st_host, it->st, sizeof(IterScalars), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return MGPU_ERR_CUDA;
  *done = it->st_host->done;
  *err = it->st_host->err;
  if (it->inner32 && it->st_host->done) it->inner_its += it->st_host->it_done;
  if (which == 9) {
    it->slab_prev_err = it->slab_err;
    it->slab_err = it->st_host->err;
  }
  return MGPU_OK;
}

int iter_slab_end(IterSolverDev* it, void* p, size_t n, cudaStream_t st, int* iterations, double* residual) {
  if (it->fp32) {
    k_convert_levels<double, float><<<592, 256, 0, st>>>(it->w64.x, static_cast<float*>(p), (long long)n);
    *iterations = it->inner_its;
    it->inner_its = 0;
    *residual = it->slab_err;
    return cudaGetLastError() == cudaSuccess ? MGPU_OK : MGPU_ERR_CUDA;
  }
  if (cudaMemcpyAsync(p, it->w64.x, n * sizeof(double), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return MGPU_ERR_CUDA;
  *iterations = it->st_host->it_done;
  *residual = it->st_host->err;
  return it->st_host->err < it->tol ? MGPU_OK : MGPU_ERR_NOT_CONVERGED;
}

int iter_slab_vectors(IterSolverDev* it, int set, void** f) {
  if (!it) return -1;
  if (set == MGPU_HALO_ITER_X64) {
    // the refinement's FP64 iterate of an FP32-mixed model
    if (!it->fp32) return -1;
    f[0] = it->w64.x;
    return 1;
  }
  auto pick = [&](auto& w) -> int {
    switch (set) {
      case MGPU_HALO_ITER_X: f[0] = w.x; return 1;
      case MGPU_HALO_ITER_PP: f[0] = w.pp; return 1;
      case MGPU_HALO_ITER_CS: f[0] = w.cs; return 1;
      case MGPU_HALO_ITER_CG:
        // conjugate gradients: z and the old direction, from which k_cg_apply forms p' at the
        // neighbours of each interior point
        f[0] = w.s;
        f[1] = cg_p(w, it->cg_n);
        return 2;
    }
    return -1;
  };
  return it->fp32 ? pick(it->w32) : pick(it->w64);
}

template <typename T>
int iter_solve(IterSolverDev* it, const Scalars& s, T* p, cudaStream_t st, int64_t* launches, int* iterations,
               double* residual) {
  if constexpr (sizeof(T) == 8) return solve_fp64(it, s, p, st, launches, iterations, residual);
  else return solve_mixed(it, s, p, st, launches, iterations, residual);
}
template int iter_solve<double>(IterSolverDev*, const Scalars&, double*, cudaStream_t, int64_t*, int*, double*);
template int iter_solve<float>(IterSolverDev*, const Scalars&, float*, cudaStream_t, int64_t*, int*, double*);

}  // namespace mgpu
