/*
 * monc_gpu.h -- C ABI of the B200 dynamical-core library (libmoncgpu.so).
 *
 * The library replaces MONC's per-column dynamical-core components with whole-domain
 * CUDA kernels that keep every prognostic field resident in GPU memory.  A MONC build
 * binds these entry points from a Fortran `bind(C)` component module; Python binds them
 * with ctypes (monc_b200/api.py).  Signatures use plain pointers, sizes and C structs.
 *
 * Reference interfaces replaced (paths inside the MONC source tree):
 *   component descriptor / callbacks    model_core/src/components/monc_component.F90:62-118
 *   group execution of callbacks        model_core/src/components/timestepper.F90:40-102
 *   state container                     model_core/src/state.F90:55-141
 *   prognostic field (z,y,x with halo)  model_core/src/grid/prognostics.F90:13-20
 *
 * Every function returns MGPU_OK (0) or a negative MGPU_ERR_* code; the message of the
 * last failure on a handle is returned by mgpu_last_error().  Nothing traps on the device.
 */
#ifndef MONC_GPU_H
#define MONC_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MGPU_MAX_NZ   1024
#define MGPU_MAX_KGD  16
#define MGPU_MAX_Q    8

/* status codes */
#define MGPU_OK                 0
#define MGPU_ERR_ARGUMENT      -1   /* bad size, id or pointer */
#define MGPU_ERR_CUDA          -2   /* a CUDA runtime call failed */
#define MGPU_ERR_NOT_CONVERGED -3   /* iterative solver stopped at max_iterations */
#define MGPU_ERR_TIMEOUT       -4   /* a bounded device-side wait gave up */
#define MGPU_ERR_UNSUPPORTED   -5   /* option not implemented on this path */
#define MGPU_ERR_NO_DEVICE     -6   /* no CUDA device visible */
#define MGPU_ERR_CFL           -7   /* cfltest: the new timestep fell below cfl_dtmmin (MONC stops) */

/* precision modes */
#define MGPU_FP64        0  /* every field and every operation in FP64 (MONC's DEFAULT_PRECISION) */
#define MGPU_FP32_MIXED  1  /* FP32 fields and stencils; FP64 tridiagonal, solver reductions, profiles */

/* pressure solvers (fftsolver / iterativesolver components) */
#define MGPU_SOLVER_FFT        0
#define MGPU_SOLVER_ITERATIVE  1
#define MGPU_SOLVER_EXTERNAL   2  /* one y-slab of a decomposed domain: the caller drives the solve */

/* advection of the flow fields (advection_flow_fields, pwadvection.F90 / tvdadvection.F90:603-908) */
#define MGPU_ADVECT_PW   0  /* Piacsek-Williams centred flux form (the benchmark configurations) */
#define MGPU_ADVECT_TVD  1  /* TVD (ULTIMATE-QUICKEST) on the dual grids of u, v, w */

/* subsidence input (forcing.F90:40-41, subsidence_input_type): the f_subs_pl nodes are a
 * divergence (w_subs = -div z) or the subsidence velocity itself */
#define MGPU_SUBS_DIVERGENCE 0
#define MGPU_SUBS_VELOCITY   1
#define MGPU_MAX_SUBS_NODES  32

/* iterative solver types (iterativesolver.F90 solver_type) */
#define MGPU_ITER_BICGSTAB 0
#define MGPU_ITER_CG       1

/* array layouts accepted by upload/download */
#define MGPU_LAYOUT_XFAST    0  /* C order [nz][ny][nx], interior only (the device layout) */
#define MGPU_LAYOUT_MONC     1  /* Fortran data(nz, ny+4, nx+4): z fastest, 2-deep x/y halo */
#define MGPU_LAYOUT_DEVICE   2  /* as MGPU_LAYOUT_XFAST, but a pointer to FP64 device memory of the
                                   handle's GPU: the copy stays on the device */

/* field identifiers (state.F90:86-92 names) */
enum mgpu_field_id {
  MGPU_U = 0, MGPU_V, MGPU_W, MGPU_TH,
  MGPU_ZU, MGPU_ZV, MGPU_ZW, MGPU_ZTH,
  MGPU_P,
  MGPU_SU, MGPU_SV, MGPU_SW, MGPU_STH,
  MGPU_VIS, MGPU_DIFF,
  MGPU_SAVU, MGPU_SAVV, MGPU_SAVW,
  MGPU_Q0 = 32,   /* q(n)  = MGPU_Q0  + n, n < MGPU_MAX_Q */
  MGPU_ZQ0 = 48,  /* zq(n) = MGPU_ZQ0 + n */
  MGPU_SQ0 = 64   /* sq(n) = MGPU_SQ0 + n */
};

/* component identifiers: the registered names of the MONC components this library replaces */
enum mgpu_component_id {
  MGPU_C_CLEARSOURCETERMS = 0,  /* clearsourceterms.F90:25-56 */
  MGPU_C_STEPPING_DIRECTION,    /* steppingdirection.F90:41-49 */
  MGPU_C_HALO_SWAPPER,          /* haloswapper.F90:62-71 */
  MGPU_C_LOWER_BC,              /* lowerbc.F90:194-305 */
  MGPU_C_SMAGORINSKY,           /* smagorinsky.F90:99-130 */
  MGPU_C_PW_ADVECTION,          /* pwadvection.F90:258-610 */
  MGPU_C_TVD_ADVECTION,         /* tvdadvection.F90:528-762 */
  MGPU_C_DIFFUSION,             /* diffusion.F90:376-545 */
  MGPU_C_VISCOSITY,             /* viscosity.F90:237-498 */
  MGPU_C_CORIOLIS,              /* coriolis.F90:206-262 */
  MGPU_C_BUOYANCY,              /* buoyancy.F90:190-269 */
  MGPU_C_SET_CONSISTENT_LOWBC,  /* set_consistent_lowbc.F90:41-144 */
  MGPU_C_SIMPLECLOUD,           /* simplecloud.F90:262-379 */
  MGPU_C_DIVERR,                /* diverr.F90:44-175 */
  MGPU_C_PSRCE,                 /* pressuresource.F90:61-238 */
  MGPU_C_STEPFIELDS,            /* stepfields.F90:231-627 */
  MGPU_C_FFTSOLVER,             /* fftsolver.F90:129-309 */
  MGPU_C_ITERATIVESOLVER,       /* iterativesolver.F90:87-602 */
  MGPU_C_PSTEP,                 /* pstep.F90:310-469 */
  MGPU_C_SWAP_SMOOTH,           /* swapsmooth.F90:45-289 */
  MGPU_C_MEAN_PROFILES,         /* meanprofiles.F90:95-216: olzubar, olzvbar, olzthbar, olzqbar */
  MGPU_C_DAMPING,               /* damping.F90:301-409 */
  MGPU_C_FORCING,               /* forcing.F90:918-1166: subsidence of u, v, theta and q */
  MGPU_C_TH_ADVECTION,          /* thadvection.F90:129-219: advection of the mean baroclinicity */
  MGPU_C_COUNT
};

/* Model configuration: the option-database keys of MONC's global_config that the
 * dynamical core reads (names in comments).  mgpu_config_defaults() fills the
 * global_config defaults. */
typedef struct mgpu_config {
  int32_t nx, ny, nz;                 /* x_size, y_size, z_size */
  int32_t n_kgd;                      /* number of kgd/hgd entries */
  int32_t kgd[MGPU_MAX_KGD];          /* kgd */
  double  hgd[MGPU_MAX_KGD];          /* hgd */
  int32_t nsmth;                      /* nsmth (vertical grid smoothing passes) */
  int32_t explicit_z;                 /* 1: w-level heights given in z_levels[0..nz-1] */
  double  dxx, dyy, zztop;            /* dxx, dyy, zztop */
  double  z_levels[MGPU_MAX_NZ];
  double  thref0, rhobous;            /* thref0, rhobous */
  double  surface_pressure, surface_reference_pressure;
  double  rmlmax;                     /* rmlmax (<=0: 0.23*max(dxx,dyy), simplesetup.F90:234) */
  double  dtm;                        /* dtm (fixed timestep, s) */
  int32_t passive_th, passive_q;      /* passive_th, passive_q */
  int32_t number_q_fields;            /* number_q_fields */
  int32_t use_viscosity_and_diffusion;
  int32_t use_surface_boundary_conditions;
  int32_t type_of_surface_boundary_conditions;  /* 0 = prescribed flux */
  double  surface_sensible_heat_flux; /* W m-2 */
  double  surface_latent_heat_flux;   /* W m-2 */
  int32_t coriolis_enabled;
  double  fcoriol;
  double  surface_geostrophic_wind_x, surface_geostrophic_wind_y;
  double  smag_subb, smag_subc;       /* smag-subb, smag-subc */
  int32_t simplecloud_enabled;
  double  max_height_cloud;
  int32_t solver;                     /* MGPU_SOLVER_* */
  int32_t solver_type;                /* MGPU_ITER_* */
  double  tolerance;                  /* tolerance */
  int32_t max_iterations;             /* max_iterations */
  int32_t precision;                  /* MGPU_FP64 / MGPU_FP32_MIXED */
  int32_t reproducible;               /* 1: fused kernels without FMA contraction (bit-reproducible) */
  /* science constants (global_config:355-372) */
  double  von_karman_constant, z0, z0th, alphah, betam, betah, gammam, gammah;
  double  pi, cp, rlvap, r, G, convective_limit, ratio_mol_wts, rlargep;
  /* cfltest (cfltest.F90:44-58, global_config:19,113,137-143): adaptive dtm from the advective and
   * viscous Courant numbers, evaluated every cfl_frequency steps inside mgpu_step.  cfl_enabled = 0
   * keeps dtm fixed. */
  int32_t cfl_enabled;                /* cfltest_enabled */
  int32_t cfl_frequency;              /* cfl_frequency */
  double  cfl_tollerance, cfl_cvismax, cfl_cvelmax; /* cfl_tollerance, cfl_cvismax, cfl_cvelmax */
  double  cfl_dtmmax, cfl_dtmmin, cfl_rincmax;      /* cfl_dtmmax, cfl_dtmmin, cfl_rincmax */
  int32_t l_constant_dtm;             /* l_constant_dtm */
  int32_t advection_flow_fields;      /* MGPU_ADVECT_PW / MGPU_ADVECT_TVD (MONC's "any" would advect twice) */
  int32_t adjoint_taped;              /* 1: adjoint passes on the operator-overloading tape (the check
                                         path); 0: the hand-written adjoint kernels */
  /* damping (damping.F90:124-148, global_config:157-159): Newtonian relaxation of u, v, theta and q
   * towards their horizontal means, and of w towards 0, above zdmp; dmpco = dmptim (exp((zn -
   * zdmp)/hdmp) - 1).  Needs the mean profiles, which the library keeps on the device. */
  int32_t damping_enabled;            /* damping_enabled */
  double  dmptim, zdmp, hdmp;         /* dmptim, zdmp, hdmp */
  /* forcing: subsidence (forcing.F90:447-1166, global_config:313-317).  w_subs is the piecewise-
   * linear interpolation (interpolation.F90:15-58) of the n_subs_pl nodes onto the w levels z. */
  int32_t l_subs_pl_theta;            /* subsidence of u, v and theta */
  int32_t l_subs_pl_q;                /* subsidence of the q fields */
  int32_t subsidence_input_type;      /* MGPU_SUBS_DIVERGENCE / MGPU_SUBS_VELOCITY */
  int32_t subsidence_local_theta;     /* 1: theta (and u, v) gradients of the column, 0: of the mean profiles */
  int32_t subsidence_local_q;         /* the same for q */
  int32_t n_subs_pl;                  /* nodes in z_subs_pl / f_subs_pl (<= MGPU_MAX_SUBS_NODES) */
  double  z_subs_pl[MGPU_MAX_SUBS_NODES], f_subs_pl[MGPU_MAX_SUBS_NODES];
  /* profile_diagnostics (profile_diagnostics.F90:311-636): keeps the mean profiles it reads up to
   * date every step, so that mgpu_profile_diagnostics can be called between steps */
  int32_t profile_diagnostics_enabled;
  /* Galilean transformation (simplesetup.F90:239-245, cfltest.F90:184-230, pstep.F90:345-346,
   * 453-469): the flow is stepped in a frame moving at (ugal, vgal), set on each cfltest evaluation
   * to the middle of the domain's zu (zv) range unless fixed at ugal (vgal).  Off in MONC's
   * global_config; most of MONC's test cases switch it on. */
  int32_t galilean_transformation;
  int32_t fix_ugal, fix_vgal;
  double  ugal, vgal;                 /* the fixed frame velocities (fix_ugal, fix_vgal) */
  /* th_advection (thadvection.F90:129-219) and the geostrophic shear of coriolis
   * (coriolis.F90:140-163, global_config:52,147-154).  With baroclinicity_use_geostrophic_shear
   * the geostrophic wind grows with height, ug(k) = surface_geostrophic_wind_x +
   * geostrophic_wind_rate_of_change_in_x zn(k) (v likewise), and th_advection adds the advection
   * of the mean baroclinicity, ((v + vgal) mfx - (u + ugal) mfy) with mfx =
   * rate_change_geostrophic_wind_x thref0 fcoriol / G (mfy likewise), to the theta source at
   * levels 2..nz; MONC does the latter only with passive q.  The library is Boussinesq (rho =
   * rhobous), where thref is constant and th_advection's vertical advection of the reference
   * state is zero. */
  int32_t th_advection_enabled;       /* th_advection_enabled */
  int32_t baroclinicity_use_geostrophic_shear;
  double  rate_change_geostrophic_wind_x, rate_change_geostrophic_wind_y;          /* th_advection's keys */
  double  geostrophic_wind_rate_of_change_in_x, geostrophic_wind_rate_of_change_in_y; /* coriolis's keys */
} mgpu_config;

/* Diagnostic reductions computed on the device after a step. */
typedef struct mgpu_reductions {
  double  global_divmax;              /* max |p| from diverr (diverr.F90:84-93) */
  int32_t solver_iterations;          /* iterations of the last iterative solve */
  double  solver_residual;            /* relative residual of the last iterative solve */
  int32_t timestep;                   /* next MONC timestep number (1 = first, forward) */
  /* cfltest state after the last step (cfltest.F90:62-128, 135-191) */
  double  dtm;                        /* timestep of the last step */
  double  dtm_new;                    /* timestep of the next step */
  double  absolute_new_dtm;           /* target of the last CFL evaluation */
  double  cvel, cvis, cfl_number;     /* Courant numbers of the last evaluation (scaled by dtm) */
  double  cvel_x, cvel_y, cvel_z;     /* their advective parts before the dtm scaling */
  int32_t cfl_evaluations;            /* CFL evaluations so far */
  int32_t last_cfl_timestep;          /* timestep of the last evaluation */
  double  ugal, vgal;                 /* the Galilean frame velocities of the next step */
} mgpu_reductions;

typedef struct mgpu_handle mgpu_handle;

/* Fill a configuration with MONC's global_config defaults (global_config:100-372). */
void mgpu_config_defaults(mgpu_config* cfg);

/* Create a device-resident model: builds the vertical grid and reference state
 * (replaces gridmanager.F90:2008-2075 + simplesetup.F90:60-126 initialisation callbacks)
 * and allocates every field on the current CUDA device.
 * MGPU_ERR_ARGUMENT (checked on the host before any device call): nx, ny even and >= 4; with the
 * FFT solver nx and ny <= 4096 with no prime factor other than 2, 3 and 5 (FFTPACK's radix-2, 3, 4
 * and 5 passes, cffti1.f90:8; powers of two take the radix-16 kernels, the rest mixed-radix
 * ones); 3 <= nz <= MGPU_MAX_NZ; dtm > 0; known precision and solver.  MGPU_ERR_NO_DEVICE when no CUDA device is visible.  A model with solver
 * MGPU_SOLVER_EXTERNAL is one slab of a decomposed domain (see mgpu_slab_init below); mgpu_step
 * refuses it. */
int mgpu_create(const mgpu_config* cfg, mgpu_handle** out);

/* Release every device allocation (the finalisation callbacks). */
int mgpu_destroy(mgpu_handle* h);

/* Copy a field between host and device (host pointer to FP64 data), or, with
 * MGPU_LAYOUT_DEVICE, between the model and another FP64 device array.  In MONC layout the halo
 * is ignored on upload and filled periodically on download.  The call returns when the copy is
 * complete; a device source must be ready before the call (work on other streams finished). */
int mgpu_upload_field(mgpu_handle* h, int32_t field_id, const double* host, int32_t layout);
int mgpu_download_field(mgpu_handle* h, int32_t field_id, double* host, int32_t layout);

/* Read back a 1-D vertical-grid profile (names as in grids.F90:91-159, e.g. "rdz",
 * "tzc1", "czg", "rneutml_sq", "buoy_co"); n receives the length (nz). */
int mgpu_get_profile(mgpu_handle* h, const char* name, double* out, int32_t* n);

/* Host-only: build the reference state of a configuration without a device and return one
 * profile (same names as mgpu_get_profile), for setup checks on machines without a GPU. */
int mgpu_reference_profile(const mgpu_config* cfg, const char* name, double* out);

/* Run one or more complete MONC timesteps (timestepper.F90:40-54 over the start, subgrid,
 * dynamics, solver and pressure-terms groups) with the fused kernels. */
int mgpu_step(mgpu_handle* h, int32_t nsteps);

/* Run a single component's timestep callback over the whole domain (the `entire` group
 * form of a column callback), for drop-in use and component-level parity tests. */
int mgpu_component_timestep(mgpu_handle* h, int32_t component_id);

/* Select forward (first-step) or centred stepping for component calls
 * (steppingdirection.F90:41-49 sets this from the timestep number). */
int mgpu_set_timestep(mgpu_handle* h, int32_t timestep);

int mgpu_get_reductions(mgpu_handle* h, mgpu_reductions* out);

/* The flow and viscosity extrema cfltest reads, gathered on the device from the current fields
 * (replaces stepfields.F90:372-393 determine_local_flow_minmax and smagorinsky.F90:143-173
 * update_viscous_number, for a CPU cfltest driving GPU-resident fields): out[0..5] = min zu, max zu,
 * min zv, max zv (levels 2..nz), max over k = 2..nz-1 of |zw| rdzn(k+1), max over k = 2..nz-1 of
 * max(vis, diff) (rdzn(k+1)^2 + cx2 + cy2).  Synchronous; reads back 48 bytes. */
int mgpu_cfl_gather(mgpu_handle* h, double* out);

/* The Galilean frame velocities (current_state%ugal, vgal) the component kernels read:
 * stepfields adds them to u, v; pstep subtracts them from u, zu, v, zv when
 * galilean_transformation is on (pstep.F90:345-346, 453-469); lower_bc, coriolis, damping,
 * swap_smooth and the mean profiles read them.  For a CPU cfltest driving GPU-resident fields:
 * it sets the frame after each evaluation, before pstep.  mgpu_step moves the frame itself. */
int mgpu_set_galilean_velocity(mgpu_handle* h, double ugal, double vgal);

/* Horizontal-mean profile of a field (meanprofiles.F90:155-293 style sum / (nx*ny)). */
int mgpu_mean_profile(mgpu_handle* h, int32_t field_id, double* out);

/* CUDA stream used by the handle (cudaStream_t as void*), for callers that overlap work. */
void* mgpu_stream(mgpu_handle* h);

/* Number of kernels this handle has launched so far. */
int64_t mgpu_launch_count(mgpu_handle* h);

/* Horizontal-mean profiles computed on the device in FP64: mean theta (th + thref) and the
 * mean of w squared per level (the domain-mean theta and w'^2 profiles used to compare runs);
 * either pointer may be NULL.  Reads back 8*nz bytes per non-NULL pointer. */
int mgpu_diagnostics(mgpu_handle* h, double* mean_theta, double* mean_w2);

/* ---- Checkpoint files (checkpointer: writecheckpoint.F90:42-100, readcheckpoint.F90) ----------
 * MONC's checkpoint layout (checkpointcommon.F90:11-81 names: options_database, x/y_resolution,
 * z, zn, thref, olz*bar, q, zq, u_nogal, v_nogal, w, th, p, zu, zv, zw, zth, timestep, time, dtm,
 * dtm_new, ...) in NetCDF classic format with 64-bit offsets, the format a serial MONC writes and
 * nf90_open reads.  Fields are stored z fastest as MONC stores them. */
typedef struct mgpu_checkpoint_meta {
  int32_t timestep;            /* the last completed step (MONC's current_state%timestep) */
  int32_t last_cfl_timestep;
  double  time;                /* model time after that step */
  double  dtm, dtm_new, absolute_new_dtm, ugal, vgal;
} mgpu_checkpoint_meta;

/* Write / read a checkpoint of the model's state (all fields, the mean profiles when damping or
 * subsidence is on, the step count, time and dtm state).  Reading restarts the model at the step
 * after the checkpointed one; the file's x, y, zn sizes and q fields must match the model's. */
int mgpu_checkpoint_write(mgpu_handle* h, const char* path);
int mgpu_checkpoint_read(mgpu_handle* h, const char* path);

/* The step state a checkpoint carries, without a file: for a decomposed run, whose driver
 * gathers the slabs' fields into one global file with mgpu_checkpoint_write_host (MONC's ranks
 * write their parts of one file, writecheckpoint.F90) and restores every slab after reading it.
 * mean (may be NULL): the rows of mgpu_mean_profiles, 2 (3 + number_q_fields) rows of nz. */
int mgpu_checkpoint_state(mgpu_handle* h, mgpu_checkpoint_meta* meta);
int mgpu_restore_state(mgpu_handle* h, const mgpu_checkpoint_meta* meta, const double* mean);

/* The same without a GPU, on host arrays: fields[0..8] = u v w th zu zv zw zth p, then q(n) and
 * zq(n) for n < number_q_fields, each [nz][ny][nx] x fastest; mean = the rows of
 * mgpu_mean_profiles (2 (3 + number_q_fields) rows of nz) or null.  read sets *has_mean to 1 when
 * the file holds the olz*bar profiles, 2 when it also holds olubar, olvbar, olthbar and olqbar
 * (otherwise those rows are zero), 0 when it holds none. */
int mgpu_checkpoint_write_host(const mgpu_config* cfg, const char* path, const double* const* fields,
                               const double* mean, const mgpu_checkpoint_meta* meta);
int mgpu_checkpoint_read_host(const mgpu_config* cfg, const char* path, double* const* fields, double* mean,
                              int32_t* has_mean, mgpu_checkpoint_meta* meta);

/* The mean profiles (meanprofiles.F90:95-216, global_grid vertical olzubar, olzvbar, olzthbar,
 * olzqbar, olubar, olvbar, olthbar, olqbar): out receives 2 (3 + number_q_fields) rows of nz
 * values, k = 1..nz: olzubar, olzvbar, olzthbar, olzqbar(n), then olubar, olvbar, olthbar,
 * olqbar(n).  They are the means of the fields as MONC's solver group sees them: the stepped zu,
 * zv, zth, zq before the pressure step, u + ugal, v + vgal, and theta and q after stepfields'
 * time smoothing.  mgpu_step
 * refreshes them every step when damping, subsidence or profile_diagnostics reads them;
 * MGPU_C_MEAN_PROFILES refreshes them from the component fields. */
int mgpu_mean_profiles(mgpu_handle* h, double* out);

/* profile_diagnostics (profile_diagnostics.F90:311-636, published as <name>_total_local): the
 * per-level sums over the domain's columns that MONC's component accumulates in the next step's
 * dynamics group, from the current state and the mean profiles of the last step.  For PW flow
 * advection with TVD scalars (the flux terms of TVD flow advection are not provided: error).
 * Needs profile_diagnostics_enabled.  out receives *nrows rows of nz values, k = 1..nz, in the
 * order MGPU_PD_U_WIND .. MGPU_PD_RH (the last five only with active q fields). */
enum mgpu_profile_diagnostic {
  MGPU_PD_U_WIND = 0,  /* u_wind_total:    sum (u + ugal) */
  MGPU_PD_V_WIND,      /* v_wind_total:    sum (v + vgal) */
  MGPU_PD_W_WIND,      /* w_wind_total:    sum w, k >= 2 */
  MGPU_PD_WW,          /* ww_total:        sum w^2 */
  MGPU_PD_WWW,         /* www_total:       sum w^3, k >= 2 */
  MGPU_PD_WWWW,        /* wwww_total:      sum w^4, k >= 2 */
  MGPU_PD_THETA,       /* theta_total:     sum (th + thref) */
  MGPU_PD_TH2,         /* th2_total:       sum (th - olthbar)^2 */
  MGPU_PD_WTHETA_CN,   /* wtheta_cn_total: sum w (th(k) + th(k+1))/2, 2 <= k <= nz-1 */
  MGPU_PD_UW,          /* uw_total:        sum (u at w points + ugal - mean) w, k <= nz-1 */
  MGPU_PD_VW,          /* vw_total:        the same for v */
  MGPU_PD_VAPOUR,      /* vapour_mmr_total */
  MGPU_PD_LIQUID,      /* liquid_mmr_total */
  MGPU_PD_WQV_CN,      /* wqv_cn_total:    sum w (qv(k) + qv(k+1))/2, 2 <= k <= nz-1 */
  MGPU_PD_WQL_CN,      /* wql_cn_total */
  MGPU_PD_RH,          /* rh_total:        sum qv / qsat(T, p) */
  MGPU_PD_COUNT
};
int mgpu_profile_diagnostics(mgpu_handle* h, double* out, int32_t* nrows);

/* Per-stage device timing of mgpu_step (CUDA events on the handle's stream).  Stage order:
 * 0 subgrid, 1 dynamics, 2 pressure source, 3 fft x forward, 4 fft y forward, 5 tridiagonal,
 * 6 fft y inverse, 7 fft x inverse, 8 pstep + swap_smooth, 9 iterative solve, 10 the momentum
 * kernel of the dynamics stage alone (stage 1 minus stage 10 is the scalar kernels). */
#define MGPU_NSTAGES 11
int mgpu_set_profiling(mgpu_handle* h, int32_t on);
int mgpu_stage_times(mgpu_handle* h, double* ms_total, int64_t* launches);

/* Pressure solve that allocates nothing on the device (no counterpart in the reference).
 *
 * For host models that cannot call cudaMalloc: their device memory belongs to another allocator
 * (a caching allocator, or a pool sized at start-up to most of HBM) and may not grow during a
 * run, or their step loop must not meet the device-wide synchronisation that cudaFree implies.
 * The caller passes p (device pointer, FP64 [nz][ny][nx], x fastest): the right-hand side on
 * entry, the pressure on return, solved exactly as the fftsolver component solves it.  czb, cza,
 * czg, czh are DEVICE arrays of nz doubles owned by the caller, element k-1 holding MONC level k
 * (the values mgpu_get_profile / mgpu_reference_profile return), read during the call; dx, dy
 * the horizontal spacings; stream a cudaStream_t or NULL.  nx and ny must be powers of two.
 *
 * All working storage (the spectrum, pivots, twiddles, a copy of the coefficients) is one
 * file-scope device array of MGPU_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds
 * until exit; grids needing more (about 128 x 128 x 128 is the largest cube-like grid that fits)
 * are rejected with MGPU_ERR_ARGUMENT and a message on stderr.  The
 * first call on a device looks up the array's device address (cudaGetSymbolAddress); make that
 * first call before any stream capture.  Nothing in the array has to start at zero -- each call
 * writes every value it later reads -- but all calls share the array and keep the last call's
 * contents, so calls whose work overlaps on the GPU (different streams or devices sharing a
 * context) race and must be serialised by the caller.
 *
 * There is no handle, so mgpu_last_error does not apply: the call returns a status code and
 * writes its message to stderr.  A CUDA error left pending by earlier work is reported on stderr
 * as such and cleared; MGPU_ERR_CUDA means a launch of this call failed. */
#define MGPU_NOALLOC_SCRATCH_BYTES (24u * 1024u * 1024u)
int mgpu_poisson_fft_noalloc(double* p, int32_t nx, int32_t ny, int32_t nz, double dx, double dy,
                             const double* czb, const double* cza, const double* czg, const double* czh,
                             void* stream);

/* Tangent-linear and adjoint runs of the dry FP64 model with the FFT solver (no counterpart in
 * the reference, which has no adjoint).  The derivative is that of the discrete step as
 * computed, with the TVD limiter branches, the Richardson-number regimes and max/min choices of
 * the forward evaluation.  Tangents and adjoints of the state fields u v w th zu zv zw zth
 * (ids 0..7) move through mgpu_upload_field / mgpu_download_field with the ids below (XFAST
 * layout). */
#define MGPU_TANGENT0 1024 /* MGPU_TANGENT0 + id: tangent of state field id */
#define MGPU_ADJOINT0 2048 /* MGPU_ADJOINT0 + id: adjoint of state field id */

/* Transpose (adjoint) of the FFT pressure solve applied to p in place: the same transforms with
 * the transposed tridiagonal and the transposed horizontal-mean recurrence. */
int mgpu_fftsolver_adjoint(mgpu_handle* h);

/* Advance the state and its tangent nsteps steps; d_rmlmax is the tangent of the Smagorinsky
 * mixing length rmlmax (= Cs * dx). */
int mgpu_tl_step(mgpu_handle* h, int32_t nsteps, double d_rmlmax);

/* Adjoint of nsteps steps from the current state.  On entry the adjoint fields hold dJ/d(state
 * after nsteps); on return they hold dJ/d(current state), *rmlmax_bar holds dJ/d rmlmax, and the
 * model state is the state after nsteps.  The forward sweep stores a checkpoint every
 * checkpoint_interval steps; the reverse sweep recomputes each segment from its checkpoint. */
int mgpu_adjoint_run(mgpu_handle* h, int32_t nsteps, int32_t checkpoint_interval, double* rmlmax_bar);

/* Gradient-check diagnostic (no counterpart in the reference): the number of branch decisions in
 * which the next steps of two dry FP64 models of one grid differ -- for every point, the theta TVD
 * faces' upwind sides, smooth-region early returns, limiter choices and gradient-term stencil
 * signs, and the Smagorinsky regime of the Richardson number.  Stepping two models started at
 * x + eps d and x - eps d side by side and adding the counts shows whether a central difference
 * along d straddles a kink of the discrete step.  Sets *count. */
int mgpu_branch_flips(mgpu_handle* a, mgpu_handle* b, int64_t* count);

/* ---- y-slab domain decomposition ---------------------------------------------------------
 *
 * The horizontal domain split into y-slabs, one per GPU (MONC splits it into 2-D blocks,
 * decomposition.F90:57-123; slabs keep whole x rows, so the x halo stays periodic inside each
 * model and only y rows move).  Each rank creates a model with solver MGPU_SOLVER_EXTERNAL and
 * ny = nyl + 2*halo rows: its nyl interior rows of the global ny_global, with `halo` rows of the
 * neighbouring slabs below and above (halo >= 3 covers the step's stencils: the TVD and
 * viscosity stencils reach 2 rows, the pressure source 1 more).  A step is then
 *
 *   halo exchange of MGPU_HALO_STATE (depth halo)
 *   mgpu_step_phase(SUBGRID)
 *   FP32-mixed only: mgpu_slab_level_means, average the means over the slabs
 *   mgpu_step_phase(DYNAMICS)                   dynamics, scalar swap, pressure source
 *   mgpu_slab_fft_x(forward)                    x-FFT of the interior rows into kx blocks
 *   all-to-all: block q of every slab to rank q (perform_forward_3dfft, pencilfft.F90:126-138)
 *   mgpu_slab_solve_columns                     y-FFT, vertical solve, inverse y-FFT
 *   all-to-all back (perform_backwards_3dfft, pencilfft.F90:147-159)
 *   mgpu_slab_fft_x(inverse)                    pressure on the interior rows
 *   halo exchange of MGPU_HALO_PRESSURE (depth >= 1)
 *   mgpu_step_phase(PSTEP)                      pressure step, swap_smooth, timestep + 1
 *
 * which replaces the halo_swapper component (haloswapper.F90:62-71 over
 * halocommunication.F90:109-163) and fftsolver's pencil transposes.  All buffers are device
 * memory of the model's precision (double for MGPU_FP64, float for MGPU_FP32_MIXED; spectra are
 * interleaved complex of that type) and all work is queued on mgpu_stream(h).  The decomposed
 * step computes each interior point with the operations of the single-domain step; with
 * reproducible = 1 an FP64 decomposed run equals the single-domain run bit for bit. */

/* Set the slab geometry: ny_global rows in all (nx and ny_global as mgpu_create's FFT sizes), `halo` rows each side, at most
 * max_cols kx columns per mgpu_slab_solve_columns call.  Builds the pivots and twiddles of the
 * (nx, ny_global) solve.  Needs ny - 2*halo even, >= max(halo, 2). */
int mgpu_slab_init(mgpu_handle* h, int32_t ny_global, int32_t halo, int32_t max_cols);

#define MGPU_PHASE_SUBGRID   0
#define MGPU_PHASE_DYNAMICS  1
#define MGPU_PHASE_PSTEP     2
int mgpu_step_phase(mgpu_handle* h, int32_t phase);

/* Halo rows.  Sets: MGPU_HALO_STATE = u v w th zu zv zw zth, then q(n), zq(n) for each q field;
 * MGPU_HALO_PRESSURE = p.  Buffers lo and hi are [nfields][nz][depth][nx] (nfields from
 * mgpu_halo_fields).  Pack copies the first `depth` interior rows into lo (for the slab below)
 * and the last `depth` into hi (for the slab above); unpack writes lo (received from the slab
 * below) into the rows just under the interior and hi (from the slab above) into the rows just
 * over it.  One kernel launch each. */
#define MGPU_HALO_STATE     0
#define MGPU_HALO_PRESSURE  1
#define MGPU_HALO_ITER_X    2   /* BiCGStab on slabs: the iterate x (before MGPU_SLAB_ITER_INIT) */
#define MGPU_HALO_ITER_PP   3   /* the search direction pp (before MGPU_SLAB_ITER_APPLY) */
#define MGPU_HALO_ITER_CS   4   /* the preconditioned half step cs (before MGPU_SLAB_ITER_APPLY2) */
#define MGPU_HALO_ITER_CG   5   /* conjugate gradients: z and the old direction p (before APPLY) */
#define MGPU_HALO_ITER_X64  6   /* FP32-mixed: the refinement's FP64 iterate (double buffers) */
int mgpu_halo_fields(mgpu_handle* h, int32_t set);
int mgpu_halo_pack(mgpu_handle* h, int32_t set, int32_t depth, void* d_lo, void* d_hi);
int mgpu_halo_unpack(mgpu_handle* h, int32_t set, int32_t depth, const void* d_lo, const void* d_hi);

/* FP32-mixed: means of th and of each q field per level over the slab's interior rows into
 * d_means (device FP64 [1 + number_q_fields][nz + 2], level k at column k).  The next dynamics
 * phase reads d_means as the domain means, so the caller averages it over the slabs in place
 * (equal slabs: the mean of the slab means) before that phase. */
int mgpu_slab_level_means(mgpu_handle* h, double* d_means);

/* The mean profiles of a slab (mgpu_mean_profiles' rows; damping, subsidence and
 * profile_diagnostics read them).  The dynamics phase leaves this slab's means; the driver
 * fetches them into d_buf (put = 0: 2 (3 + number_q_fields) rows of nz + 2 doubles on the
 * device, olz*bar rows then olubar, olvbar, olthbar, olqbar(n)), averages them over the slabs
 * (all slabs hold the same number of rows: the average is the domain mean) and puts the result
 * back (put = 1) before the next dynamics phase. */
int mgpu_slab_mean_profiles(mgpu_handle* h, double* d_buf, int32_t put);

/* cfltest on slabs (cfltest.F90:62-128; MONC reduces the same extrema across its ranks with
 * MPI_MIN/MPI_MAX in get_global_values, cfltest.F90:184-264).  On an evaluation step the
 * subgrid phase gathers this slab's extrema over its interior rows; put = 0 then writes them to
 * d_buf (6 doubles on the device: -min zu, max zu, -min zv, max zv, max |zw| rdzn, max of the
 * viscous term -- every entry combined by a maximum), the driver all-reduces d_buf with a
 * maximum over the slabs, and put = 1 hands the result back before the pressure-step phase,
 * which runs cfltest and sets the next step's dtm.  *gathered (may be NULL) says whether this
 * step gathered; on other steps the call does nothing, and every slab takes the same steps. */
int mgpu_slab_cfl_extrema(mgpu_handle* h, double* d_buf, int32_t put, int32_t* gathered);

/* iterativesolver on slabs (bicgstab, iterativesolver.F90:140-248, and cg_solver, :255-321; MONC
 * sums the inner products over its ranks with MPI_Allreduce in inner_prod, :500-553), FP64 models,
 * in place of the FFT steps between the dynamics and pressure-step phases.  solver_type
 * MGPU_ITER_BICGSTAB:
 *
 *   BEGIN                                     psource = p; the iterate x keeps the last solution
 *   halo exchange of MGPU_HALO_ITER_X (depth 1)
 *   INIT, sum d_sums over the slabs, FINISH   r = b - A x; <r, r>, <b, b>
 *   until FINISH reports done:
 *     DIRECTION                               pp = M^-1 (r - bet omg v) + bet pp
 *     halo exchange of MGPU_HALO_ITER_PP (depth 1)
 *     APPLY, sum, FINISH                      v = A pp; <cr, v>
 *     HALF_STEP                               s = r - alf v; cs = M^-1 s
 *     halo exchange of MGPU_HALO_ITER_CS (depth 1)
 *     APPLY2, sum, FINISH                     t = A cs; <t, t>, <t, s>, <s, s>
 *     UPDATE, sum, FINISH                     x, r; <r, cr>; convergence
 *   END                                       p = x (then the MGPU_HALO_PRESSURE exchange)
 *
 * The reducing steps write this slab's sums over its interior rows to d_sums (3 doubles on the
 * device); the driver replaces them by their sum over the slabs and passes them to FINISH,
 * which updates the solver scalars and sets *done (every slab reaches the same decision from
 * the same sums).  As in mgpu_step, a solve that stops at max_iterations above the tolerance is
 * not an error (MONC only warns); mgpu_get_reductions reports its iterations and residual. */
#define MGPU_SLAB_ITER_BEGIN      0
#define MGPU_SLAB_ITER_INIT       1
#define MGPU_SLAB_ITER_DIRECTION  2
#define MGPU_SLAB_ITER_APPLY      3
#define MGPU_SLAB_ITER_HALF_STEP  4
#define MGPU_SLAB_ITER_APPLY2     5
#define MGPU_SLAB_ITER_UPDATE     6
#define MGPU_SLAB_ITER_FINISH     7
#define MGPU_SLAB_ITER_END        8
#define MGPU_SLAB_ITER_PRECOND    9
#define MGPU_SLAB_ITER_COMPAT    10
#define MGPU_SLAB_ITER_SHIFT     11
#define MGPU_SLAB_ITER_REFINE    12
#define MGPU_SLAB_ITER_INNER     13
#define MGPU_SLAB_ITER_CORRECT   14
#define MGPU_SLAB_ITER_UNCORRECT 15
/* solver_type MGPU_ITER_CG (MONC's default; the symmetric form of the operator):
 *
 *   BEGIN; halo exchange of MGPU_HALO_ITER_X; INIT, sum, FINISH     r = b A_vol - A x
 *   until FINISH after UPDATE reports done:
 *     PRECOND, sum, FINISH                    z = M^-1 r; <z, r>
 *     halo exchange of MGPU_HALO_ITER_CG (depth 1)
 *     APPLY, sum, FINISH                      p' = z + bet p; A p'; <p', A p'>
 *     UPDATE, sum, FINISH                     x, r; |r|^2; convergence
 *   END
 *
 * FP32-mixed models (iterative refinement: the FP64 residual, an FP32 correction solve, the FP64
 * iterate corrected; the single-domain solve's loop):
 *
 *   BEGIN                                     b (FP64) = p
 *   COMPAT, sum, FINISH; SHIFT                b minus its incompatible horizontal-mean part
 *   up to 8 times:
 *     halo exchange of MGPU_HALO_ITER_X64 (depth 1, double buffers)
 *     REFINE, sum, FINISH                     r = b - A x in FP64; stop when FINISH reports done
 *     if the residual did not fall below the last one: UNCORRECT (x -= e) and stop
 *     INNER                                   e = 0; then the BiCGStab or conjugate-gradient
 *                                             steps above on the FP32 vectors, to a relative
 *                                             residual of 0.5 tolerance / (the FP64 residual),
 *                                             kept within 1e-3 .. 0.5
 *     CORRECT                                 x += e
 *   END                                       p = x
 *
 * FINISH reports the solver's relative residual through mgpu_get_reductions as it goes. */
int mgpu_slab_iter(mgpu_handle* h, int32_t step, double* d_sums, int32_t* done);

/* x-FFT (fftsolver.F90:50-309 transforms, x pass) between the interior rows of p and d_spec,
 * which is split into nblocks (<= nx/2+1) blocks of consecutive wavenumbers dealt out as evenly
 * as possible: with b = (nx/2+1) / nblocks and r = (nx/2+1) % nblocks, block q has width
 * w_q = b + (q < r), first wavenumber k0_q = q*b + min(q, r), is [nz][nyl][w_q] complex and starts
 * at element k0_q*nz*nyl -- exactly the send buffer of an all-to-all that gives rank q the
 * wavenumbers of block q.  inverse = 1 runs the inverse transform from d_spec back into p's
 * interior rows. */
int mgpu_slab_fft_x(mgpu_handle* h, void* d_spec, int32_t nblocks, int32_t inverse);

/* The rest of the solve on the global wavenumbers kx0 .. kx0+nkx-1 (nkx <= max_cols): forward
 * y-FFT over all ny_global rows, the vertical tridiagonal solve per (kx, ky) (fftsolver.F90:
 * 259-309; transpose = 1 applies its transpose, as mgpu_fftsolver_adjoint does), inverse y-FFT.
 * d_spec holds the rows in blocks of row_block rows: block b is [nz][row_block][nkx] complex and
 * starts at element b*nz*row_block*nkx -- the receive buffer of the all-to-all, block b coming
 * from the slab with rows b*row_block .. (b+1)*row_block-1. */
int mgpu_slab_solve_columns(mgpu_handle* h, void* d_spec, int32_t kx0, int32_t nkx, int32_t row_block,
                            int32_t transpose);

const char* mgpu_last_error(mgpu_handle* h);

#ifdef __cplusplus
}
#endif
#endif /* MONC_GPU_H */
