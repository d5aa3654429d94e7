// Device state and kernel launchers of the dynamical core.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "mgpu_internal.h"

namespace mgpu {

// Device field pointers ([nz][ny][nx], x fastest).  The *_n fields receive the fused
// dynamics kernel's stepped values; s* and sav* are only allocated for component calls.
template <typename T>
struct DevState {
  T *u, *v, *w, *th, *zu, *zv, *zw, *zth, *p, *vis, *diff;
  T *su, *sv, *sw, *sth, *savu, *savv, *savw;
  T *zu_n, *zv_n, *zw_n, *th_n, *zth_n;
  T* q[MGPU_MAX_Q];
  T* zq[MGPU_MAX_Q];
  T* sq[MGPU_MAX_Q];
  T* q_n[MGPU_MAX_Q];
  T* zq_n[MGPU_MAX_Q];
};

// Kernel launchers, built twice: `exact` compiles every multiply and add separately rounded
// (MONC's x86-64 arithmetic, bit-reproducible against the CPU oracle), `fast` lets nvcc contract
// multiply-adds into FMAs.  Component kernels always come from `exact`.
#define MGPU_DECLARE_LAUNCHERS                                                                            \
  template <typename T>                                                                                   \
  int launch_component(int cid, const Scalars& s, DevState<T>& d, cudaStream_t st, unsigned long long* divmax, \
                       int64_t* launches);                                                                \
  template <typename T> int launch_fused_subgrid(const Scalars& s, DevState<T>& d, cudaStream_t st);      \
  template <typename T> int launch_fused_dynamics(const Scalars& s, DevState<T>& d, cudaStream_t st, cudaEvent_t mid); \
  template <typename T> void launch_fused_pressure_source(const Scalars& s, DevState<T>& d, cudaStream_t st); \
  template <typename T> void launch_fused_pstep_swap(const Scalars& s, DevState<T>& d, cudaStream_t st);
namespace exact { MGPU_DECLARE_LAUNCHERS }
namespace fast { MGPU_DECLARE_LAUNCHERS }

// Spectral pressure solve (fftsolver): p (levels 1..nz) -> p.
struct FftPlanDev {
  int nx = 0, ny = 0, nz = 0, nxh = 0;
  void* spec = nullptr;            // complex [nz][ny][nxh], same precision as p
  double* b1 = nullptr;            // [nz+1][ny/2+1][nxh] Thomas pivots 1/(b - czh*b1), FP64
  double2* s1 = nullptr;           // forward-elimination values of the Thomas solve, FP64
  double* twx = nullptr;           // e^{-2 pi i p / nx}, p < nx/2 (complex FP64)
  double* twy = nullptr;
  float* twx_f = nullptr;          // the same twiddles rounded to FP32
  float* twy_f = nullptr;
};
// horizontal transform lengths of the spectral solve: 4 .. 4096 points with prime factors 2, 3, 5
bool fft_length_ok(int n);
int fft_plan_create(FftPlanDev& plan, const Scalars& s, const RefState& rs, bool fp32);
void fft_plan_destroy(FftPlanDev& plan);
// The stepped z-velocities from which the fused step forms the pressure source.
template <typename T>
struct SourceFields {
  const T* zu;
  const T* zv;
  const T* zw;
};
// evs: NULL, or 6 events recorded before, between and after the five kernels.  transpose: apply
// the transpose of the solve (the adjoint of the pressure solve) instead.  src: when given (and
// nx is a power of two), the forward x transform forms the pressure source from these fields
// itself and p's input is not read; the solution is written to p as always.
template <typename T>
void fft_solve(const FftPlanDev& plan, const Scalars& s, T* p, cudaStream_t st, int64_t* launches,
               cudaEvent_t* evs = nullptr, bool transpose = false, const SourceFields<T>* src = nullptr);

// horizontal means of th (row 0) and q[0..nq-1] (rows 1..nq) per level into out[row*(nz+2) + k],
// over the rows halo .. ny-halo-1 (all rows for halo 0)
template <typename T>
void launch_level_means(const Scalars& s, const T* th, T* const* q, int nq, double* out, cudaStream_t st,
                        int halo = 0);

// y-slab decomposition.  A slab plan holds the pivots and twiddles of the global grid (nx,
// ny_global) and Thomas scratch for max_cols kx columns; the spectra are the caller's.
int fft_slab_plan_create(FftPlanDev& plan, const Scalars& s, const RefState& rs, int ny_global, int max_cols);
// x-FFT between the slab's interior rows halo .. ny-halo-1 of p and a spectrum split into nblk
// blocks of consecutive wavenumbers, the first (nx/2+1) % nblk one wider than the rest: block q
// covers k0_q .. k0_q+w_q-1, is [nz][ny-2*halo][w_q] and starts at k0_q*nz*(ny-2*halo)
template <typename T>
void slab_fft_x(const FftPlanDev& plan, const Scalars& s, T* p, int halo, int nblk, void* spec, bool inverse,
                cudaStream_t st, int64_t* launches);
// forward y-FFT, vertical solve (or its transpose) and inverse y-FFT of the global wavenumbers
// kx0 .. kx0+nkx-1 over all plan.ny rows, held in row blocks of rpb rows: block b is [nz][rpb][nkx]
template <typename T>
void slab_solve_columns(const FftPlanDev& plan, const Scalars& s, void* spec, int kx0, int nkx, int rpb, bool transpose,
                        cudaStream_t st, int64_t* launches);
// rows [r_lo, r_lo+depth) and [r_hi, r_hi+depth) of every level of the n fields f[] to (pack) or
// from (unpack) the buffers lo and hi, each [n][nz][depth][nx]
template <typename T>
void launch_halo_rows(const Scalars& s, T* const* f, int n, int depth, int r_lo, int r_hi, T* lo, T* hi, bool unpack,
                      cudaStream_t st);

template <typename T>
void launch_diagnostics(const Scalars& s, const T* th, const T* w, double* out_th, double* out_w2, cudaStream_t st,
                        int halo = 0);

// cfltest's reductions of the current zu, zv, zw (and vis, diff when with_vis) into out[0..5]:
// min zu, max zu, min zv, max zv (levels 2..nz), max |zw| rdzn(k+1), max max(vis, diff) (rdzn(k+1)^2
// + cx2 + cy2) (levels 2..nz-1).  part holds CFL_BLOCKS*6 doubles.  Returns the launch count.
constexpr int CFL_BLOCKS = 296;
template <typename T>
int launch_cfl_gather(const Scalars& s, const DevState<T>& d, bool with_vis, double* part, double* out,
                      cudaStream_t st, int halo = 0);
// src -> dst with the two minima negated (the form a maximum all-reduce combines); its own inverse
int launch_cfl_max_form(const double* src, double* dst, cudaStream_t st);
// diverr's max |p| of the velocities the step starts from, atomically maxed into *out (double bits)
template <typename T>
int launch_divmax(const Scalars& s, const DevState<T>& d, unsigned long long* out, cudaStream_t st, int halo = 0);

// mean profiles (olzubar, olzvbar, olzthbar, olzqbar) of zu, zv, th and q into olz (rows of nz+2),
// and the mean-profile subsidence tendencies (forcing.cu)
template <typename T>
int launch_mean_profiles(const Scalars& s, const T* zu, const T* zv, const T* th, const T* const* q, double* olz,
                         cudaStream_t st, int halo = 0);
int launch_subsidence_tendencies(const Scalars& s, const double* olz, double* tend, bool flow_theta, bool q,
                                 cudaStream_t st);
// olubar, olvbar, olthbar, olqbar(n) from u, v, theta and the q fields (q may be null: no olqbar);
// zth, zq given: the scalars after time smoothing c1 f + c2 zf
template <typename T>
int launch_mean_profiles_state(const Scalars& s, const T* u, const T* v, const T* th, const T* zth,
                               const T* const* q, const T* const* zq, double ugal, double vgal, double c1, double c2,
                               double* olbar, cudaStream_t st, int halo = 0);
// profile_diagnostics sums into out (MGPU_PD_* rows of nz); qv, ql null for a dry model.  With halo
// > 0 (a y-slab) the means and sums run over the interior rows halo .. ny-1-halo
template <typename T>
int launch_profile_diagnostics(const Scalars& s, const T* u, const T* v, const T* w, const T* th, const T* qv,
                               const T* ql, const double* olbar, bool has_mean, double* out, cudaStream_t st,
                               int halo = 0);

// BiCGStab pressure solve (iterativesolver)
struct IterSolverDev;
IterSolverDev* iter_create(const Scalars& s, const RefState& rs, const mgpu_config& cfg, bool fp32, int* status,
                           int j0 = 0, int j1 = -1, int ny_total = -1);
// BiCGStab and conjugate gradients over y-slabs, with the FP32-mixed refinement around them, one
// step at a time (iter.cu); p holds n elements of the model's type
int iter_slab_begin(IterSolverDev* it, const void* p, size_t n, cudaStream_t st);
int iter_slab_step(IterSolverDev* it, int step, double* d_sums, cudaStream_t st, int64_t* launches);
int iter_slab_finish(IterSolverDev* it, const double* d_sums, cudaStream_t st, int64_t* launches, int* done,
                     double* err);
int iter_slab_end(IterSolverDev* it, void* p, size_t n, cudaStream_t st, int* iterations, double* residual);
// the halo set's solver vectors into f (at most 2; float for the FP32 inner solve, double for
// MGPU_HALO_ITER_X64 and FP64 models); returns their number, or -1
int iter_slab_vectors(IterSolverDev* it, int set, void** f);
void iter_destroy(IterSolverDev* it);
template <typename T>
int iter_solve(IterSolverDev* it, const Scalars& s, T* p, cudaStream_t st, int64_t* launches, int* iterations,
               double* residual);

// Tangent-linear and adjoint passes of the dry FP64 step (tlad.cu).  Adjoint arrays are indexed
// by these ids; F_FACE0.. are tape-internal (TVD face values).
enum AdField { F_U, F_V, F_W, F_TH, F_ZU, F_ZV, F_ZW, F_ZTH, F_VIS, F_DIFF, F_ZUN, F_ZVN, F_ZWN, F_P, F_PROF, F_COUNT,
               F_FACE0 = 64 };
// pass 0 subgrid, 1 dynamics, 2 pressure source, 3 pstep + swap_smooth; t holds the tangents
// the number of branch decisions (TVD faces of theta, Smagorinsky regime) in which two models'
// next steps differ, added to *count (device)
void branch_flips(const Scalars& s, const DevState<double>& a, const DevState<double>& b, unsigned long long* count,
                  cudaStream_t st);
void tl_pass(int pass, const Scalars& s, const DevState<double>& d, const DevState<double>& t, const double* drsq,
             double dpar, cudaStream_t st);
// pass 0 subgrid, 1 momentum, 2 scalars, 3 pressure source, 4 pstep + swap_smooth; seed[0..7] are
// the adjoints of the next state (u v w th zu zv zw zth), tg[F_*] the adjoint arrays added into
void adj_pass(int pass, const Scalars& s, const DevState<double>& d, double* const* tg, const double* const* seed,
              int* overflow, cudaStream_t st);
// the subgrid pass's adjoint on level 1 only (lower_bc), on the tape
void adj_lower_bc(const Scalars& s, const DevState<double>& d, double* const* tg, const double* const* seed,
                  int* overflow, cudaStream_t st);
// the hand-written adjoint of the same pass (adjoint.cu; the subgrid pass covers levels 2..nz, with
// level 1 left to adj_lower_bc); false when the pass has none
bool hadj_pass(int pass, const Scalars& s, const DevState<double>& d, double* const* tg, const double* const* seed,
               cudaStream_t st);

}  // namespace mgpu
