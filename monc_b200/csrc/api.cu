// C ABI of libmoncgpu.so (include/monc_gpu.h): device-resident model state, host<->device
// transfers with the MONC <-> x-fastest layout change, the fused timestep driver and the
// per-component entry points.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "dycore.h"

using namespace mgpu;

// Tangent-linear and adjoint work arrays (dry FP64 models)
struct AdWork {
  DevState<double> t{};          // tangents of the state and of the step's intermediates
  double* adj[2][8] = {};        // adjoints of u v w th zu zv zw zth: adj[cur] is the current one
  int cur = 0;
  double* inter[6] = {};         // adjoints of vis, diff, zu_n, zv_n, zw_n, p
  double* prof_bar = nullptr;    // adjoint of rneutml_sq per level
  double* drsq = nullptr;        // d rneutml_sq / d rmlmax per level (device)
  std::vector<double> drsq_h;
  int* overflow = nullptr;
  std::vector<double*> ckpt, seg;  // checkpoint states and the states of one segment (8 arrays each)
  double* final_state[8] = {};
  std::vector<void*> allocs;
  bool tl = false, adj_ok = false;
};

struct mgpu_handle {
  mgpu_config cfg;
  RefState rs;
  Scalars sc;
  int timestep = 1;
  double time = 0.0;  // model time: the dtm of every completed step
  int device = 0;
  bool fp32 = false;
  cudaStream_t stream = nullptr;
  double* prof_d = nullptr;
  double* lookup_d = nullptr;
  DevState<double> d64;
  DevState<float> d32;
  std::vector<void*> allocations;
  bool component_fields = false;
  FftPlanDev fft;
  IterSolverDev* iter = nullptr;
  unsigned long long* divmax_d = nullptr;
  unsigned long long* flips_d = nullptr;  // mgpu_branch_flips' counter, allocated on first use
  double global_divmax = 0.0;
  bool divmax_step = false;  // the last mgpu_step left diverr's max in divmax_d (iterative solver)
  int solver_iterations = 0;
  double solver_residual = 0.0;
  int64_t launches = 0;
  double* xfer = nullptr;  // device staging buffer (FP64 field) for uploads/downloads
  double* diag_d = nullptr;  // 2*nz FP64 diagnostics
  double* bmean_d = nullptr; // FP32-mixed: horizontal means of th and q per level (1+nq rows of nz+2)
  double* olz_d = nullptr;       // mean profiles olzubar, olzvbar, olzthbar, olzqbar (3+MGPU_MAX_Q rows of nz+2)
  double* subs_tend_d = nullptr; // mean-profile subsidence tendencies, the same rows
  double* olbar_d = nullptr;     // olubar, olvbar, olthbar, olqbar (3+MGPU_MAX_Q rows of nz+2)
  double* pd_d = nullptr;        // profile_diagnostics sums (MGPU_PD_COUNT rows of nz)
  bool profiling = false;
  cudaEvent_t ev[16] = {};
  struct AdWork* ad = nullptr;  // tangent-linear / adjoint arrays, allocated on first use
  double stage_ms[MGPU_NSTAGES] = {};
  int64_t stage_n[MGPU_NSTAGES] = {};
  // y-slab of a decomposed domain (solver MGPU_SOLVER_EXTERNAL, set up by mgpu_slab_init)
  int slab_halo = 0, slab_ny_global = 0, slab_cols = 0;
  FftPlanDev slab;
  const double* bmean_ext = nullptr;  // FP32-mixed: the domain level means for the next dynamics phase
  // cfltest (cfltest.F90:62-191) when cfg.cfl_enabled: state carried between steps
  struct {
    int last_cfl_timestep = 0, evaluations = 0;
    bool update_dtm = false;
    bool gathered = false;  // y-slab: this step's subgrid phase gathered the slab's extrema
    double dtm_new = 0.0, absolute_new_dtm = 0.0, dtm_last = 0.0;
    double cvel = 0.0, cvis = 0.0, cfl_number = 0.0, cvel_x = 0.0, cvel_y = 0.0, cvel_z = 0.0;
    double* part_d = nullptr;  // CFL_BLOCKS*6 block partials
    double* out_d = nullptr;   // 6 reduced values
    double* out_h = nullptr;   // the same, pinned host copy
    cudaEvent_t ev = nullptr;  // recorded after the copy to out_h
  } cfl;
  std::string err;
};

static int fail(mgpu_handle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

#define CK(call)                                                                          \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess) return fail(h, MGPU_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

static size_t field_elems(const mgpu_handle* h) { return (size_t)h->cfg.nx * h->cfg.ny * h->cfg.nz; }

template <typename T>
static int alloc_field(mgpu_handle* h, T** p) {
  void* ptr = nullptr;
  cudaError_t e = cudaMalloc(&ptr, field_elems(h) * sizeof(T));
  if (e != cudaSuccess) return fail(h, MGPU_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  cudaMemsetAsync(ptr, 0, field_elems(h) * sizeof(T), h->stream);
  h->allocations.push_back(ptr);
  *p = reinterpret_cast<T*>(ptr);
  return MGPU_OK;
}

template <typename T>
static int alloc_state(mgpu_handle* h, DevState<T>& d) {
  std::memset(&d, 0, sizeof(d));
  T** core[] = {&d.u, &d.v, &d.w, &d.th, &d.zu, &d.zv, &d.zw, &d.zth, &d.p, &d.vis, &d.diff,
                &d.zu_n, &d.zv_n, &d.zw_n, &d.th_n, &d.zth_n};
  for (T** pp : core) {
    int rc = alloc_field<T>(h, pp);
    if (rc) return rc;
  }
  for (int n = 0; n < h->cfg.number_q_fields; ++n) {
    T** qq[] = {&d.q[n], &d.zq[n], &d.q_n[n], &d.zq_n[n], &d.sq[n]};
    for (T** pp : qq) {
      int rc = alloc_field<T>(h, pp);
      if (rc) return rc;
    }
  }
  // the moist centred step passes the scalar sources through memory (tiled kernels, one per scalar)
  if (h->cfg.number_q_fields > 0) {
    int rc = alloc_field<T>(h, &d.sth);
    if (rc) return rc;
  }
  // TVD advection of the flow: the tiled centred step passes its advective sources through su,
  // sv, sw to the momentum kernel
  if (h->cfg.advection_flow_fields == MGPU_ADVECT_TVD) {
    T** flow[] = {&d.su, &d.sv, &d.sw};
    for (T** pp : flow) {
      int rc = alloc_field<T>(h, pp);
      if (rc) return rc;
    }
  }
  return MGPU_OK;
}

template <typename T>
static int alloc_component_fields(mgpu_handle* h, DevState<T>& d) {
  if (h->component_fields) return MGPU_OK;
  T** extra[] = {&d.su, &d.sv, &d.sw, &d.sth, &d.savu, &d.savv, &d.savw};
  for (T** pp : extra) {
    if (*pp) continue;
    int rc = alloc_field<T>(h, pp);
    if (rc) return rc;
  }
  h->component_fields = true;
  return MGPU_OK;
}

static void fill_scalars(mgpu_handle* h) {
  const mgpu_config& c = h->cfg;
  const RefState& r = h->rs;
  Scalars& s = h->sc;
  std::memset(&s, 0, sizeof(s));
  s.nx = c.nx; s.ny = c.ny; s.nz = c.nz;
  s.plane = (long long)c.nx * c.ny;
  s.cx = r.cx; s.cy = r.cy; s.cx2 = r.cx2; s.cy2 = r.cy2; s.tcx = r.tcx; s.tcy = r.tcy;
  s.dtm = c.dtm; s.tsmth = 1e-2;
  // simplesetup.F90:239-245: the frame starts at rest unless fixed
  s.galilean = c.galilean_transformation ? 1 : 0;
  s.ugal = (c.galilean_transformation && c.fix_ugal) ? c.ugal : 0.0;
  s.vgal = (c.galilean_transformation && c.fix_vgal) ? c.vgal : 0.0;
  s.ugal_p = s.ugal; s.vgal_p = s.vgal;
  s.fcoriol = c.fcoriol; s.smallp = r.smallp;
  s.czn = r.czn; s.zn2 = r.zn[2]; s.zlogm = r.zlogm; s.zlogth = r.zlogth; s.vk_on_zlogm = r.vk_on_zlogm;
  s.vk = c.von_karman_constant; s.z0 = c.z0; s.z0th = c.z0th; s.alphah = c.alphah; s.betam = c.betam;
  s.betah = c.betah; s.gammah = c.gammah; s.pi = c.pi;
  s.surface_temperature_flux = r.surface_temperature_flux; s.surface_vapour_flux = r.surface_vapour_flux;
  s.fbuoy = r.fbuoy;
  s.max_diff_or_visc = 1.7976931348623157e308;  // huge(0.5_DEFAULT_PRECISION): no surface-exchange limit
  s.velmin = r.velmin; s.aloginv = r.aloginv; s.cneut = r.cneut; s.cfc = r.cfc;
  s.convective_limit = c.convective_limit;
  s.subb = c.smag_subb; s.subc = c.smag_subc; s.subg = 1.2; s.subh = 0.0;
  s.suba = 1.0 / 0.7; s.ric = 0.25; s.ricinv = 1.0 / 0.25;
  s.eps = 0.01; s.repsh = 0.5 / 0.01;
  s.thcona = c.ratio_mol_wts * c.thref0; s.thconb = s.thcona - c.thref0; s.thconap1 = s.thcona;
  s.rlvap_over_cp = r.rlvap_over_cp; s.G = c.G;
  for (int n = 0; n < MGPU_MAX_Q; ++n) s.cq[n] = n < (int)r.cq.size() ? r.cq[n] : 0.0;
  s.simplecloud = c.simplecloud_enabled;
  s.k_cloudmax = r.k_cloudmax;
  s.lookup_entries = r.lookup_entries;
  s.forward = 1;
  {
    const char* e = std::getenv("MGPU_POINT_DYNAMICS");
    s.point_dynamics = (e && e[0] == '1') ? 1 : 0;
  }
  {
    const char* e = std::getenv("MGPU_LEVEL_CHUNKS");
    s.level_chunks = e ? std::atoi(e) : 0;
    if (s.level_chunks < 0) s.level_chunks = 0;
  }
  s.passive_th = c.passive_th; s.passive_q = c.passive_q; s.nq = c.number_q_fields;
  s.iqv = 0; s.iql = c.number_q_fields > 1 ? 1 : 0;
  s.coriolis = c.coriolis_enabled; s.surface_bcs = c.use_surface_boundary_conditions;
  s.use_vd = c.use_viscosity_and_diffusion;
  s.tvd_flow = c.advection_flow_fields == MGPU_ADVECT_TVD ? 1 : 0;
  s.rho_unity = 1;
  for (int k = 1; k <= c.nz; ++k)
    if (r.rho[k] != 1.0 || r.rhon[k] != 1.0) s.rho_unity = 0;
  s.prof = h->prof_d;
  s.lookup = h->lookup_d;
  s.damping = s.subs_th = s.subs_q = 0;  // set per step (forcing_flags)
  s.kdmpmin = r.kdmpmin;
  s.subs_local_th = c.subsidence_local_theta;
  s.subs_local_q = c.subsidence_local_q;
  s.olz = h->olz_d;
  s.subs_tend = h->subs_tend_d;
  // thadvection.F90:63-78: the mean baroclinicity is advected with passive q only
  s.th_baroclinic = (c.th_advection_enabled && c.baroclinicity_use_geostrophic_shear && c.passive_q && !c.passive_th) ? 1 : 0;
  const double fcoriol_over_G = c.fcoriol / c.G;
  s.mfx = c.rate_change_geostrophic_wind_x * c.thref0 * fcoriol_over_G;
  s.mfy = c.rate_change_geostrophic_wind_y * c.thref0 * fcoriol_over_G;
}

// damping and forcing act from timestep 3 (damping.F90:329-330, forcing.F90:974-975)
static void forcing_flags(mgpu_handle* h) {
  const mgpu_config& c = h->cfg;
  const bool on = h->timestep >= 3;
  h->sc.damping = (c.damping_enabled && on) ? 1 : 0;
  h->sc.subs_th = (c.l_subs_pl_theta && on) ? 1 : 0;
  h->sc.subs_q = (c.l_subs_pl_q && c.number_q_fields > 0 && on) ? 1 : 0;
}
// the mean profiles are refreshed every step when damping or mean-profile subsidence reads them
static bool needs_mean_profiles(const mgpu_config& c) {
  return c.damping_enabled || c.profile_diagnostics_enabled || (c.l_subs_pl_theta && !c.subsidence_local_theta) ||
         (c.l_subs_pl_q && !c.subsidence_local_q && c.number_q_fields > 0);
}
// the mean-profile subsidence tendencies of this step, from the mean profiles of the last
static int subsidence_tendencies(mgpu_handle* h) {
  const bool ft = h->sc.subs_th && !h->sc.subs_local_th, q = h->sc.subs_q && !h->sc.subs_local_q;
  if (!ft && !q) return 0;
  return launch_subsidence_tendencies(h->sc, h->olz_d, h->subs_tend_d, ft, q, h->stream);
}

static const std::vector<double>* prof_vec(const RefState& r, int id) {
  switch (id) {
    case P_RDZ: return &r.rdz; case P_RDZN: return &r.rdzn; case P_DZN: return &r.dzn; case P_RHO: return &r.rho;
    case P_RHON: return &r.rhon; case P_DTHREF: return &r.dthref; case P_CZB: return &r.czb; case P_CZA: return &r.cza;
    case P_CZG: return &r.czg; case P_CZH: return &r.czh; case P_TZC1: return &r.tzc1; case P_TZC2: return &r.tzc2;
    case P_TZD1: return &r.tzd1; case P_TZD2: return &r.tzd2; case P_RNEUTML_SQ: return &r.rneutml_sq;
    case P_BUOY_CO: return &r.buoy_co; case P_THREF: return &r.thref; case P_PREFRCP: return &r.prefrcp;
    case P_RPREFRCP: return &r.rprefrcp; case P_TREF: return &r.tref; case P_TSTARPR: return &r.tstarpr;
    case P_QSAT: return &r.qsat; case P_DQSATDT: return &r.dqsatdt; case P_QSATFAC: return &r.qsatfac;
    case P_GWX: return &r.gwx; case P_GWY: return &r.gwy; case P_PREFN: return &r.prefn;
    case P_TOFF: return &r.moist_toff; case P_TC0: return &r.tc0; case P_DZ: return &r.dz;
    case P_DMPCO: return &r.dmpco; case P_DMPCOZ: return &r.dmpcoz; case P_WSUBS: return &r.w_subs;
  }
  return nullptr;
}

extern "C" {

int mgpu_create(const mgpu_config* cfg, mgpu_handle** out) {
  if (!cfg || !out) return MGPU_ERR_ARGUMENT;
  *out = nullptr;
  // host-side checks first, so a bad configuration is reported the same with or without a device
  if (cfg->nx < 4 || cfg->ny < 4 || (cfg->nx % 2) || (cfg->ny % 2) || cfg->nz < 3 || cfg->nz > MGPU_MAX_NZ ||
      cfg->number_q_fields < 0 || cfg->number_q_fields > MGPU_MAX_Q ||
      (cfg->precision != MGPU_FP64 && cfg->precision != MGPU_FP32_MIXED) ||
      (cfg->solver != MGPU_SOLVER_FFT && cfg->solver != MGPU_SOLVER_ITERATIVE && cfg->solver != MGPU_SOLVER_EXTERNAL) ||
      (cfg->solver == MGPU_SOLVER_FFT && (!fft_length_ok(cfg->nx) || !fft_length_ok(cfg->ny))) || !(cfg->dtm > 0.0))
    return MGPU_ERR_ARGUMENT;
  if (cfg->cfl_enabled && (cfg->cfl_frequency < 1 || !(cfg->cfl_cvismax > 0.0) || !(cfg->cfl_cvelmax > 0.0) ||
                           !(cfg->cfl_dtmmax > 0.0) || cfg->cfl_rincmax < 0.0))
    return MGPU_ERR_ARGUMENT;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return MGPU_ERR_NO_DEVICE;
  mgpu_handle* h = new mgpu_handle();
  h->cfg = *cfg;
  cudaGetDevice(&h->device);
  try {
    build_reference_state(h->cfg, h->rs);
  } catch (std::exception& e) {
    std::fprintf(stderr, "mgpu_create: %s\n", e.what());
    delete h;
    return MGPU_ERR_ARGUMENT;
  }
  h->fp32 = cfg->precision == MGPU_FP32_MIXED;
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) { delete h; return MGPU_ERR_CUDA; }
  // profiles
  const int stride = cfg->nz + 2;
  std::vector<double> prof((size_t)P_COUNT * stride, 0.0);
  for (int id = 0; id < P_COUNT; ++id) {
    const std::vector<double>* v = prof_vec(h->rs, id);
    for (int k = 0; k <= cfg->nz && k < (int)v->size(); ++k) prof[(size_t)id * stride + k] = (*v)[k];
  }
  int rc = MGPU_OK;
  auto cleanup = [&](int code) { mgpu_destroy(h); return code; };
  if (cudaMalloc(&h->prof_d, prof.size() * sizeof(double)) != cudaSuccess) return cleanup(MGPU_ERR_CUDA);
  cudaMemcpy(h->prof_d, prof.data(), prof.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (cudaMalloc(&h->lookup_d, (h->rs.lookup_ustr.size() + 1) * sizeof(double)) != cudaSuccess) return cleanup(MGPU_ERR_CUDA);
  cudaMemcpy(h->lookup_d, h->rs.lookup_ustr.data(), h->rs.lookup_ustr.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (cudaMalloc(&h->divmax_d, sizeof(unsigned long long)) != cudaSuccess) return cleanup(MGPU_ERR_CUDA);
  cudaMemset(h->divmax_d, 0, sizeof(unsigned long long));
  if (cudaMalloc(&h->xfer, field_elems(h) * sizeof(double)) != cudaSuccess) return cleanup(MGPU_ERR_CUDA);
  if (cudaMalloc(&h->diag_d, 2 * (size_t)cfg->nz * sizeof(double)) != cudaSuccess) return cleanup(MGPU_ERR_CUDA);
  if (cudaMalloc(&h->bmean_d, (size_t)(1 + MGPU_MAX_Q) * (cfg->nz + 2) * sizeof(double)) != cudaSuccess)
    return cleanup(MGPU_ERR_CUDA);
  cudaMemset(h->bmean_d, 0, (size_t)(1 + MGPU_MAX_Q) * (cfg->nz + 2) * sizeof(double));
  {
    const size_t nb = (size_t)(3 + MGPU_MAX_Q) * (cfg->nz + 2) * sizeof(double);
    if (cudaMalloc(&h->olz_d, nb) != cudaSuccess || cudaMalloc(&h->subs_tend_d, nb) != cudaSuccess)
      return cleanup(MGPU_ERR_CUDA);
    cudaMemset(h->olz_d, 0, nb);
    cudaMemset(h->subs_tend_d, 0, nb);
    const size_t nbar = (size_t)(3 + MGPU_MAX_Q) * (cfg->nz + 2) * sizeof(double),
                 npd = (size_t)MGPU_PD_COUNT * cfg->nz * sizeof(double);
    if (cudaMalloc(&h->olbar_d, nbar) != cudaSuccess || cudaMalloc(&h->pd_d, npd) != cudaSuccess)
      return cleanup(MGPU_ERR_CUDA);
    cudaMemset(h->olbar_d, 0, nbar);
  }
  for (cudaEvent_t& e : h->ev)
    if (cudaEventCreate(&e) != cudaSuccess) return cleanup(MGPU_ERR_CUDA);
  fill_scalars(h);
  h->cfl.dtm_last = cfg->dtm;
  h->cfl.dtm_new = cfg->dtm;
  h->cfl.absolute_new_dtm = cfg->dtm;
  if (cudaMalloc(&h->cfl.part_d, (size_t)CFL_BLOCKS * 6 * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&h->cfl.out_d, 6 * sizeof(double)) != cudaSuccess ||
      cudaMallocHost(&h->cfl.out_h, 6 * sizeof(double)) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->cfl.ev, cudaEventDisableTiming) != cudaSuccess)
    return cleanup(MGPU_ERR_CUDA);
  rc = h->fp32 ? alloc_state<float>(h, h->d32) : alloc_state<double>(h, h->d64);
  if (rc) return cleanup(rc);
  if (cfg->solver == MGPU_SOLVER_FFT) {
    rc = fft_plan_create(h->fft, h->sc, h->rs, h->fp32);
    if (rc) { std::fprintf(stderr, "mgpu_create: FFT solver needs power-of-two nx, ny\n"); return cleanup(rc); }
  } else if (cfg->solver == MGPU_SOLVER_ITERATIVE) {
    int st = MGPU_OK;
    h->iter = iter_create(h->sc, h->rs, h->cfg, h->fp32, &st);
    if (st) return cleanup(st);
  }
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return cleanup(MGPU_ERR_CUDA);
  *out = h;
  return MGPU_OK;
}

int mgpu_destroy(mgpu_handle* h) {
  if (!h) return MGPU_ERR_ARGUMENT;
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->ad) {
    for (void* p : h->ad->allocs) cudaFree(p);
    delete h->ad;
    h->ad = nullptr;
  }
  for (void* p : h->allocations) cudaFree(p);
  h->allocations.clear();
  if (h->fft.spec) fft_plan_destroy(h->fft);
  if (h->slab.b1) fft_plan_destroy(h->slab);
  if (h->iter) iter_destroy(h->iter);
  cudaFree(h->prof_d);
  cudaFree(h->lookup_d);
  cudaFree(h->divmax_d);
  cudaFree(h->flips_d);
  cudaFree(h->xfer);
  cudaFree(h->diag_d);
  cudaFree(h->bmean_d);
  cudaFree(h->olz_d);
  cudaFree(h->subs_tend_d);
  cudaFree(h->olbar_d);
  cudaFree(h->pd_d);
  cudaFree(h->cfl.part_d);
  cudaFree(h->cfl.out_d);
  if (h->cfl.out_h) cudaFreeHost(h->cfl.out_h);
  if (h->cfl.ev) cudaEventDestroy(h->cfl.ev);
  for (cudaEvent_t& e : h->ev)
    if (e) cudaEventDestroy(e);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return MGPU_OK;
}

void* mgpu_stream(mgpu_handle* h) { return h ? (void*)h->stream : nullptr; }
int64_t mgpu_launch_count(mgpu_handle* h) { return h ? h->launches : 0; }
const char* mgpu_last_error(mgpu_handle* h) { return h ? h->err.c_str() : "null handle"; }

}  // extern "C"

// ---- tangent-linear / adjoint work arrays ------------------------------------------------
static void state_ptrs(DevState<double>& d, double* out[8]) {
  double* p[8] = {d.u, d.v, d.w, d.th, d.zu, d.zv, d.zw, d.zth};
  for (int q = 0; q < 8; ++q) out[q] = p[q];
}

static int ad_alloc(mgpu_handle* h, double** p, size_t n) {
  if (cudaMalloc((void**)p, n * sizeof(double)) != cudaSuccess) return fail(h, MGPU_ERR_CUDA, "cudaMalloc (adjoint work)");
  cudaMemsetAsync(*p, 0, n * sizeof(double), h->stream);
  h->ad->allocs.push_back(*p);
  return MGPU_OK;
}

static int ad_supported(mgpu_handle* h) {
  if (h->cfg.advection_flow_fields != MGPU_ADVECT_PW)
    return fail(h, MGPU_ERR_UNSUPPORTED, "tangent-linear and adjoint runs differentiate the PW advection of the flow");
  if (h->cfg.cfl_enabled)
    return fail(h, MGPU_ERR_UNSUPPORTED, "tangent-linear and adjoint runs hold dtm fixed: disable cfltest");
  if (h->cfg.galilean_transformation || h->sc.ugal != 0.0 || h->sc.vgal != 0.0)
    return fail(h, MGPU_ERR_UNSUPPORTED, "tangent-linear and adjoint runs differentiate the step in a frame at rest");
  if (h->cfg.damping_enabled || h->cfg.l_subs_pl_theta || h->cfg.l_subs_pl_q)
    return fail(h, MGPU_ERR_UNSUPPORTED, "tangent-linear and adjoint runs differentiate the step without damping and forcing");
  if (h->sc.th_baroclinic)
    return fail(h, MGPU_ERR_UNSUPPORTED, "tangent-linear and adjoint runs differentiate the step without th_advection");
  if (h->fp32 || h->cfg.number_q_fields > 0 || h->cfg.solver != MGPU_SOLVER_FFT)
    return fail(h, MGPU_ERR_UNSUPPORTED, "tangent-linear and adjoint runs need a dry FP64 model with the FFT solver");
  return MGPU_OK;
}

// d rneutml_sq / d rmlmax: rneutml_sq = 1 / (1/(vk (z+z0))^2 + 1/rmlmax^2) (gridmanager.F90:2298-2310)
static int ensure_drsq(mgpu_handle* h) {
  AdWork* a = h->ad;
  if (a->drsq) return MGPU_OK;
  const int nz = h->cfg.nz;
  a->drsq_h.assign(nz + 2, 0.0);
  const double rm = h->rs.rmlmax;
  for (int k = 2; k <= nz - 1; ++k) {
    const double r2 = h->rs.rneutml_sq[k];
    a->drsq_h[k] = 2.0 * r2 * r2 / (rm * rm * rm);
  }
  if (ad_alloc(h, &a->drsq, nz + 2)) return MGPU_ERR_CUDA;
  if (cudaMemcpy(a->drsq, a->drsq_h.data(), (nz + 2) * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(h, MGPU_ERR_CUDA, "cudaMemcpy (drsq)");
  return MGPU_OK;
}

static int ensure_tl(mgpu_handle* h) {
  if (int rc = ad_supported(h)) return rc;
  if (!h->ad) h->ad = new AdWork();
  AdWork* a = h->ad;
  if (a->tl) return MGPU_OK;
  const size_t n = field_elems(h);
  double** f[] = {&a->t.u, &a->t.v, &a->t.w, &a->t.th, &a->t.zu, &a->t.zv, &a->t.zw, &a->t.zth, &a->t.p,
                  &a->t.vis, &a->t.diff, &a->t.zu_n, &a->t.zv_n, &a->t.zw_n, &a->t.th_n, &a->t.zth_n};
  for (double** pp : f)
    if (ad_alloc(h, pp, n)) return MGPU_ERR_CUDA;
  if (ensure_drsq(h)) return MGPU_ERR_CUDA;
  a->tl = true;
  return MGPU_OK;
}

static int ensure_adj(mgpu_handle* h) {
  if (int rc = ad_supported(h)) return rc;
  if (!h->ad) h->ad = new AdWork();
  AdWork* a = h->ad;
  if (a->adj_ok) return MGPU_OK;
  const size_t n = field_elems(h);
  for (int c = 0; c < 2; ++c)
    for (int q = 0; q < 8; ++q)
      if (ad_alloc(h, &a->adj[c][q], n)) return MGPU_ERR_CUDA;
  for (int q = 0; q < 6; ++q)
    if (ad_alloc(h, &a->inter[q], n)) return MGPU_ERR_CUDA;
  for (int q = 0; q < 8; ++q)
    if (ad_alloc(h, &a->final_state[q], n)) return MGPU_ERR_CUDA;
  if (ad_alloc(h, &a->prof_bar, h->cfg.nz + 2)) return MGPU_ERR_CUDA;
  double* ov = nullptr;
  if (ad_alloc(h, &ov, 1)) return MGPU_ERR_CUDA;
  a->overflow = reinterpret_cast<int*>(ov);
  if (ensure_drsq(h)) return MGPU_ERR_CUDA;
  a->adj_ok = true;
  return MGPU_OK;
}

// ---- field lookup -----------------------------------------------------------------------
template <typename T>
static T* field_ptr(mgpu_handle* h, DevState<T>& d, int id) {
  switch (id) {
    case MGPU_U: return d.u; case MGPU_V: return d.v; case MGPU_W: return d.w; case MGPU_TH: return d.th;
    case MGPU_ZU: return d.zu; case MGPU_ZV: return d.zv; case MGPU_ZW: return d.zw; case MGPU_ZTH: return d.zth;
    case MGPU_P: return d.p; case MGPU_VIS: return d.vis; case MGPU_DIFF: return d.diff;
    case MGPU_SU: case MGPU_SV: case MGPU_SW: case MGPU_STH: case MGPU_SAVU: case MGPU_SAVV: case MGPU_SAVW:
      if (alloc_component_fields<T>(h, d)) return nullptr;
      switch (id) {
        case MGPU_SU: return d.su; case MGPU_SV: return d.sv; case MGPU_SW: return d.sw; case MGPU_STH: return d.sth;
        case MGPU_SAVU: return d.savu; case MGPU_SAVV: return d.savv; default: return d.savw;
      }
    default: break;
  }
  int nq = h->cfg.number_q_fields;
  if (id >= MGPU_Q0 && id < MGPU_Q0 + nq) return d.q[id - MGPU_Q0];
  if (id >= MGPU_ZQ0 && id < MGPU_ZQ0 + nq) return d.zq[id - MGPU_ZQ0];
  if (id >= MGPU_SQ0 && id < MGPU_SQ0 + nq) {
    if (alloc_component_fields<T>(h, d)) return nullptr;
    return d.sq[id - MGPU_SQ0];
  }
  if (sizeof(T) == sizeof(double) && id >= MGPU_TANGENT0 && id < MGPU_TANGENT0 + 8) {
    if (ensure_tl(h)) return nullptr;
    double* t[8];
    state_ptrs(h->ad->t, t);
    return reinterpret_cast<T*>(t[id - MGPU_TANGENT0]);
  }
  if (sizeof(T) == sizeof(double) && id >= MGPU_ADJOINT0 && id < MGPU_ADJOINT0 + 8) {
    if (ensure_adj(h)) return nullptr;
    return reinterpret_cast<T*>(h->ad->adj[h->ad->cur][id - MGPU_ADJOINT0]);
  }
  return nullptr;
}

// layout conversion kernels between the FP64 staging buffer and a device field
template <typename T>
__global__ void k_from_monc(const double* __restrict__ src, T* __restrict__ dst, int nx, int ny, int nz) {
  // src: (nz, ny+4, nx+4) z fastest; dst: [nz][ny][nx]
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long n = (long long)nx * ny * nz;
  if (t >= n) return;
  int i = (int)(t % nx);
  long long r = t / nx;
  int j = (int)(r % ny);
  int k = (int)(r / ny);
  long long s = (long long)k + (long long)nz * ((long long)(j + 2) + (long long)(ny + 4) * (i + 2));
  dst[t] = (T)src[s];
}

template <typename T>
__global__ void k_to_monc(const T* __restrict__ src, double* __restrict__ dst, int nx, int ny, int nz) {
  // every halo point receives its periodic image
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long n = (long long)(nx + 4) * (ny + 4) * nz;
  if (t >= n) return;
  int k = (int)(t % nz);
  long long r = t / nz;
  int jj = (int)(r % (ny + 4));
  int ii = (int)(r / (ny + 4));
  int j = ((jj - 2) % ny + ny) % ny;
  int i = ((ii - 2) % nx + nx) % nx;
  dst[t] = (double)src[(long long)k * nx * ny + (long long)j * nx + i];
}

template <typename T>
__global__ void k_convert(const double* __restrict__ src, T* __restrict__ dst, long long n) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) dst[t] = (T)src[t];
}
template <typename T>
__global__ void k_convert_back(const T* __restrict__ src, double* __restrict__ dst, long long n) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) dst[t] = (double)src[t];
}

template <typename T>
static int upload(mgpu_handle* h, DevState<T>& d, int id, const double* host, int layout) {
  T* dst = field_ptr<T>(h, d, id);
  if (!dst) return fail(h, MGPU_ERR_ARGUMENT, "unknown field id");
  const int nx = h->cfg.nx, ny = h->cfg.ny, nz = h->cfg.nz;
  const long long n = (long long)nx * ny * nz;
  if (layout == MGPU_LAYOUT_XFAST || layout == MGPU_LAYOUT_DEVICE) {
    const cudaMemcpyKind kind = layout == MGPU_LAYOUT_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    if (sizeof(T) == sizeof(double)) {
      CK(cudaMemcpyAsync(dst, host, n * sizeof(double), kind, h->stream));
    } else if (layout == MGPU_LAYOUT_DEVICE) {
      k_convert<T><<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>(host, dst, n);
      h->launches++;
    } else {
      CK(cudaMemcpyAsync(h->xfer, host, n * sizeof(double), kind, h->stream));
      k_convert<T><<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>(h->xfer, dst, n);
      h->launches++;
    }
  } else if (layout == MGPU_LAYOUT_MONC) {
    long long nm = (long long)(nx + 4) * (ny + 4) * nz;
    double* stage = nullptr;
    CK(cudaMallocAsync((void**)&stage, nm * sizeof(double), h->stream));
    CK(cudaMemcpyAsync(stage, host, nm * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    k_from_monc<T><<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>(stage, dst, nx, ny, nz);
    h->launches++;
    CK(cudaFreeAsync(stage, h->stream));
  } else {
    return fail(h, MGPU_ERR_ARGUMENT, "unknown layout");
  }
  CK(cudaStreamSynchronize(h->stream));
  return MGPU_OK;
}

template <typename T>
static int download(mgpu_handle* h, DevState<T>& d, int id, double* host, int layout) {
  T* src = field_ptr<T>(h, d, id);
  if (!src) return fail(h, MGPU_ERR_ARGUMENT, "unknown field id");
  const int nx = h->cfg.nx, ny = h->cfg.ny, nz = h->cfg.nz;
  const long long n = (long long)nx * ny * nz;
  if (layout == MGPU_LAYOUT_XFAST || layout == MGPU_LAYOUT_DEVICE) {
    const cudaMemcpyKind kind = layout == MGPU_LAYOUT_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (sizeof(T) == sizeof(double)) {
      CK(cudaMemcpyAsync(host, src, n * sizeof(double), kind, h->stream));
    } else if (layout == MGPU_LAYOUT_DEVICE) {
      k_convert_back<T><<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>(src, host, n);
      h->launches++;
    } else {
      k_convert_back<T><<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>(src, h->xfer, n);
      h->launches++;
      CK(cudaMemcpyAsync(host, h->xfer, n * sizeof(double), kind, h->stream));
    }
  } else if (layout == MGPU_LAYOUT_MONC) {
    long long nm = (long long)(nx + 4) * (ny + 4) * nz;
    double* stage = nullptr;
    CK(cudaMallocAsync((void**)&stage, nm * sizeof(double), h->stream));
    k_to_monc<T><<<(unsigned)((nm + 255) / 256), 256, 0, h->stream>>>(src, stage, nx, ny, nz);
    h->launches++;
    CK(cudaMemcpyAsync(host, stage, nm * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaFreeAsync(stage, h->stream));
  } else {
    return fail(h, MGPU_ERR_ARGUMENT, "unknown layout");
  }
  CK(cudaStreamSynchronize(h->stream));
  return MGPU_OK;
}

// ---- timestep driver ----------------------------------------------------------------------
template <typename T>
static void swap_scalar_buffers(DevState<T>& d, int nq) {
  std::swap(d.th, d.th_n);
  std::swap(d.zth, d.zth_n);
  for (int n = 0; n < nq; ++n) {
    std::swap(d.q[n], d.q_n[n]);
    std::swap(d.zq[n], d.zq_n[n]);
  }
}

template <typename T>
static int pressure_solve(mgpu_handle* h, T* p, const SourceFields<T>* src = nullptr) {
  if (h->cfg.solver == MGPU_SOLVER_FFT) {
    fft_solve<T>(h->fft, h->sc, p, h->stream, &h->launches, h->profiling ? &h->ev[3] : nullptr, false, src);
    return MGPU_OK;
  }
  int rc = iter_solve<T>(h->iter, h->sc, p, h->stream, &h->launches, &h->solver_iterations, &h->solver_residual);
  if (rc == MGPU_ERR_NOT_CONVERGED) return MGPU_OK;  // MONC only warns (iterativesolver.F90:240-242)
  return rc;
}

// With profiling on, events ev[0..2] bracket subgrid / dynamics / pressure source, ev[3..8]
// the five FFT kernels (or ev[3], ev[8] the iterative solve) and ev[8..9] pstep + swap.
static void collect_stage_times(mgpu_handle* h) {
  cudaEventSynchronize(h->ev[9]);
  float t;
  auto acc = [&](int stage, int a, int b) {
    if (cudaEventElapsedTime(&t, h->ev[a], h->ev[b]) == cudaSuccess) { h->stage_ms[stage] += t; h->stage_n[stage] += 1; }
  };
  acc(0, 0, 1);
  acc(1, 1, 2);
  acc(10, 10, 2);
  acc(2, 2, 3);
  if (h->cfg.solver == MGPU_SOLVER_FFT)
    for (int q = 0; q < 5; ++q) acc(3 + q, 3 + q, 4 + q);
  else
    acc(9, 3, 8);
  acc(8, 8, 9);
}

// cfltest's evaluation test (cfltest.F90:80-82; the same test gates the gathers in
// stepfields.F90:249-256 and smagorinsky.F90:151-153): every step up to cfl_frequency, then every
// cfl_frequency steps (start_timestep = 1, no reconfiguration offset)
static bool cfl_evaluation_step(const mgpu_handle* h, int n) {
  const int f = h->cfg.cfl_frequency;
  return n % f == 1 || n - 1 <= f || n >= h->cfl.last_cfl_timestep + f;
}

// cfltest's timestep callback (cfltest.F90:62-128) and update_dtm_based_on_absolute (:135-191), on
// the host: `evaluate` when this step gathered the extrema into cfl.out_h.  The new dtm takes
// effect at the start of the next step (monc.F90:313).  An evaluation also sets the frame of the
// Galilean transformation (perform_cfl_and_galilean_transformation_calculation, :184-230) into
// sc.ugal_p, vgal_p: the pressure-terms group of this step and the stepping of the next read it.
// The output-time alignment of time_basis runs is not on this path.
static int cfltest_callback(mgpu_handle* h, bool evaluate) {
  auto& c = h->cfl;
  const mgpu_config& g = h->cfg;
  const double dtm = h->sc.dtm;
  c.dtm_last = dtm;
  c.update_dtm = false;
  if (evaluate) {
    if (cudaEventSynchronize(c.ev) != cudaSuccess) return fail(h, MGPU_ERR_CUDA, "cfltest read-back");
    const double* r = c.out_h;
    c.last_cfl_timestep = h->timestep;
    c.evaluations += 1;
    // the extrema are of the stepping frame's zu, zv: undo its transformation
    const double zumin = r[0] + h->sc.ugal, zumax = r[1] + h->sc.ugal;
    const double zvmin = r[2] + h->sc.vgal, zvmax = r[3] + h->sc.vgal;
    double ugal = 0.0, vgal = 0.0;
    if (g.galilean_transformation) {
      ugal = g.fix_ugal ? h->sc.ugal : 0.5 * (zumin + zumax);
      vgal = g.fix_vgal ? h->sc.vgal : 0.5 * (zvmin + zvmax);
    }
    h->sc.ugal_p = ugal;
    h->sc.vgal_p = vgal;
    c.cvel_z = r[4];
    c.cvel_x = std::max(std::fabs(zumax - ugal), std::fabs(zumin - ugal));
    c.cvel_y = std::max(std::fabs(zvmax - vgal), std::fabs(zvmin - vgal));
    c.cvel = (c.cvel_x * h->sc.cx + c.cvel_y * h->sc.cy + c.cvel_z) * dtm;
    c.cvis = r[5] * (dtm * 4);
    c.cfl_number = c.cvis / g.cfl_cvismax + c.cvel / g.cfl_cvelmax;
    c.absolute_new_dtm = dtm;
    if (c.cfl_number > 0.0 &&
        (c.cfl_number < (1.0 - g.cfl_tollerance) || c.cfl_number > (1.0 + g.cfl_tollerance)))
      c.absolute_new_dtm = dtm / c.cfl_number;
  }
  if (dtm != c.absolute_new_dtm && (dtm != g.cfl_dtmmax || c.absolute_new_dtm < g.cfl_dtmmax)) {
    c.update_dtm = true;
    c.dtm_new = std::min(std::min(dtm * (1.0 + g.cfl_rincmax), c.absolute_new_dtm), g.cfl_dtmmax);
    if (c.dtm_new < g.cfl_dtmmin && !g.l_constant_dtm)
      return fail(h, MGPU_ERR_CFL, "cfltest: timestep too small, dtm_new=" + std::to_string(c.dtm_new) +
                                       " < cfl_dtmmin=" + std::to_string(g.cfl_dtmmin));
  }
  if (g.l_constant_dtm) {
    h->sc.dtm = g.dtm;
    c.dtm_new = g.dtm;
    c.update_dtm = false;
  }
  return MGPU_OK;
}

template <typename T>
static int step_once(mgpu_handle* h, DevState<T>& d) {
  const bool cfl = h->cfg.cfl_enabled != 0;
  if (cfl && h->cfl.update_dtm) h->sc.dtm = h->cfl.dtm_new;  // monc.F90:313
  const bool cfl_gather = cfl && cfl_evaluation_step(h, h->timestep);
  h->sc.forward = (h->timestep == 1) ? 1 : 0;  // steppingdirection.F90:44-48
  forcing_flags(h);
  auto mark = [&](int q) { if (h->profiling) cudaEventRecord(h->ev[q], h->stream); };
  mark(0);
  h->launches += subsidence_tendencies(h);
  if (h->cfg.reproducible) h->launches += exact::launch_fused_subgrid<T>(h->sc, d, h->stream);
  else h->launches += fast::launch_fused_subgrid<T>(h->sc, d, h->stream);
  if (h->cfg.solver == MGPU_SOLVER_ITERATIVE) {
    // diverr's divergence error, which the iterative solver reduces to global_divmax
    // (iterativesolver.F90:102, 606-613)
    cudaMemsetAsync(h->divmax_d, 0, sizeof(unsigned long long), h->stream);
    h->launches += launch_divmax<T>(h->sc, d, h->divmax_d, h->stream);
    h->divmax_step = true;
  }
  if (cfl_gather) {
    // the extrema of the pre-step zu, zv, zw and of this step's vis, diff (zu..zw change only in
    // the pressure step at the end of the step)
    h->launches += launch_cfl_gather<T>(h->sc, d, h->cfg.use_viscosity_and_diffusion != 0, h->cfl.part_d,
                                        h->cfl.out_d, h->stream);
    cudaMemcpyAsync(h->cfl.out_h, h->cfl.out_d, 6 * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    cudaEventRecord(h->cfl.ev, h->stream);
  }
  mark(1);
  cudaEvent_t mid = h->profiling ? h->ev[10] : nullptr;
  if (sizeof(T) == 4) {
    // FP32-mixed: take the horizontal-mean buoyancy out (see buoyancy_point)
    launch_level_means<T>(h->sc, d.th, d.q, h->cfg.number_q_fields, h->bmean_d, h->stream);
    h->sc.bmean = h->bmean_d;
    h->launches += 1;
  }
  if (h->cfg.reproducible) h->launches += exact::launch_fused_dynamics<T>(h->sc, d, h->stream, mid);
  else h->launches += fast::launch_fused_dynamics<T>(h->sc, d, h->stream, mid);
  h->sc.bmean = nullptr;
  mark(2);
  swap_scalar_buffers<T>(d, h->cfg.number_q_fields);
  // mean_profiles (solver group): the stepped zu, zv and the new theta, q before the pressure step
  if (needs_mean_profiles(h->cfg)) {
    h->launches += launch_mean_profiles<T>(h->sc, d.zu_n, d.zv_n, d.th, d.q, h->olz_d, h->stream);
    // u + ugal, v + vgal (stepfields.F90 adds the Galilean velocity before the solver group) and
    // the old theta and q, time-smoothed on a centred step; the swap left the old th, zth, q, zq
    // in th_n, zth_n, q_n, zq_n
    const bool fwd = h->sc.forward != 0;
    h->launches += launch_mean_profiles_state<T>(h->sc, d.u, d.v, d.th_n, fwd ? nullptr : d.zth_n, d.q_n,
                                                 fwd ? nullptr : d.zq_n, h->sc.ugal, h->sc.vgal,
                                                 1.0 - 2.0 * h->sc.tsmth, h->sc.tsmth, h->olbar_d, h->stream);
  }
  // The FFT solve of a power-of-two nx forms the source inside its first transform (fast
  // build); the reproducible build keeps the source kernel, whose rounding the oracle matches.
  const bool src_in_fft = !h->cfg.reproducible && h->cfg.solver == MGPU_SOLVER_FFT && (h->cfg.nx & (h->cfg.nx - 1)) == 0;
  const SourceFields<T> src{d.zu_n, d.zv_n, d.zw_n};
  if (!src_in_fft) {
    if (h->cfg.reproducible) exact::launch_fused_pressure_source<T>(h->sc, d, h->stream);
    else fast::launch_fused_pressure_source<T>(h->sc, d, h->stream);
    h->launches += 1;
  }
  if (h->cfg.solver != MGPU_SOLVER_FFT) mark(3);
  int rc = pressure_solve<T>(h, d.p, src_in_fft ? &src : nullptr);
  if (rc) return rc;
  if (h->cfg.solver != MGPU_SOLVER_FFT) mark(8);
  // cfltest ends the solver group.  Where its evaluation can move the frame the pressure step
  // works in (the Galilean transformation, or a frame to bring to rest), it runs before the
  // pressure step is queued, waiting for the extrema; otherwise it only sets the next step's dtm
  // and runs after, while the GPU works.
  const bool frame = h->cfg.galilean_transformation || h->sc.ugal != 0.0 || h->sc.vgal != 0.0;
  bool cfl_done = false;
  if (cfl && frame) {
    if (int rc = cfltest_callback(h, cfl_gather)) return rc;
    cfl_done = true;
  }
  if (h->cfg.reproducible) exact::launch_fused_pstep_swap<T>(h->sc, d, h->stream);
  else fast::launch_fused_pstep_swap<T>(h->sc, d, h->stream);
  mark(9);
  h->launches += 1;
  if (cfl && !cfl_done)
    if (int rc = cfltest_callback(h, cfl_gather)) return rc;
  h->sc.ugal = h->sc.ugal_p;  // the next step steps in the frame the pressure step left
  h->sc.vgal = h->sc.vgal_p;
  h->time += h->sc.dtm;
  h->timestep += 1;
  if (h->profiling) collect_stage_times(h);
  return MGPU_OK;
}

// ---- tangent-linear and adjoint drivers (dry FP64) ----------------------------------------
static void launch_subgrid(mgpu_handle* h, DevState<double>& d) {
  if (h->cfg.reproducible) h->launches += exact::launch_fused_subgrid<double>(h->sc, d, h->stream);
  else h->launches += fast::launch_fused_subgrid<double>(h->sc, d, h->stream);
}
static int launch_dynamics(mgpu_handle* h, DevState<double>& d) {
  return h->cfg.reproducible ? exact::launch_fused_dynamics<double>(h->sc, d, h->stream, nullptr)
                             : fast::launch_fused_dynamics<double>(h->sc, d, h->stream, nullptr);
}
static void launch_pressure_source(mgpu_handle* h, DevState<double>& d) {
  if (h->cfg.reproducible) exact::launch_fused_pressure_source<double>(h->sc, d, h->stream);
  else fast::launch_fused_pressure_source<double>(h->sc, d, h->stream);
}
static void launch_pstep_swap(mgpu_handle* h, DevState<double>& d) {
  if (h->cfg.reproducible) exact::launch_fused_pstep_swap<double>(h->sc, d, h->stream);
  else fast::launch_fused_pstep_swap<double>(h->sc, d, h->stream);
}

// one step of the state and of its tangent (each tangent pass runs before the forward pass that
// overwrites its inputs)
static int tl_step_once(mgpu_handle* h, double dpar) {
  DevState<double>& d = h->d64;
  DevState<double>& t = h->ad->t;
  const double* drsq = h->ad->drsq;
  h->sc.forward = (h->timestep == 1) ? 1 : 0;
  tl_pass(0, h->sc, d, t, drsq, dpar, h->stream);
  launch_subgrid(h, d);
  tl_pass(1, h->sc, d, t, drsq, dpar, h->stream);
  h->launches += 3 + launch_dynamics(h, d);
  swap_scalar_buffers<double>(d, 0);
  std::swap(t.th, t.th_n);
  std::swap(t.zth, t.zth_n);
  tl_pass(2, h->sc, d, t, drsq, dpar, h->stream);
  launch_pressure_source(h, d);
  fft_solve<double>(h->fft, h->sc, t.p, h->stream, &h->launches);
  int rc = pressure_solve<double>(h, d.p);
  if (rc) return rc;
  tl_pass(3, h->sc, d, t, drsq, dpar, h->stream);
  launch_pstep_swap(h, d);
  h->launches += 4;
  h->timestep += 1;
  return MGPU_OK;
}

static void copy_state(mgpu_handle* h, double* const* dst, double* const* src) {
  const size_t bytes = field_elems(h) * sizeof(double);
  for (int q = 0; q < 8; ++q) cudaMemcpyAsync(dst[q], src[q], bytes, cudaMemcpyDeviceToDevice, h->stream);
}

// the adjoint of one step from state X (already in h->d64): adjoints of the next state in
// adj[cur] become adjoints of X in adj[1-cur]
static int adjoint_step(mgpu_handle* h) {
  AdWork* a = h->ad;
  DevState<double>& d = h->d64;
  h->sc.forward = (h->timestep == 1) ? 1 : 0;
  // recompute the step's intermediates.  The hand-written passes read only the step's input state
  // (with lower_bc's th(1) or zth(1)) and vis, diff: the pressure step and source are linear and
  // read no values, so the subgrid pass is all there is to recompute.  The tape re-evaluates every
  // pass on its values: post-subgrid state, vis, diff, zu_n..zth_n and p.
  launch_subgrid(h, d);
  if (h->cfg.adjoint_taped) {
    h->launches += 3 + launch_dynamics(h, d);
    launch_pressure_source(h, d);
    int rc = pressure_solve<double>(h, d.p);
    if (rc) return rc;
  }
  double* const* B = a->adj[a->cur];
  double* const* A = a->adj[1 - a->cur];
  const size_t bytes = field_elems(h) * sizeof(double);
  for (int q = 0; q < 8; ++q) CK(cudaMemsetAsync(A[q], 0, bytes, h->stream));
  for (int q = 0; q < 6; ++q) CK(cudaMemsetAsync(a->inter[q], 0, bytes, h->stream));
  double* tg[F_COUNT];
  for (int q = 0; q < 8; ++q) tg[F_U + q] = A[q];
  tg[F_VIS] = a->inter[0];
  tg[F_DIFF] = a->inter[1];
  tg[F_ZUN] = a->inter[2];
  tg[F_ZVN] = a->inter[3];
  tg[F_ZWN] = a->inter[4];
  tg[F_P] = a->inter[5];
  tg[F_PROF] = a->prof_bar;
  const double* seed[8];
  for (int q = 0; q < 8; ++q) seed[q] = B[q];
  auto pass = [&](int q) {
    if (h->cfg.adjoint_taped) {
      adj_pass(q, h->sc, d, tg, seed, a->overflow, h->stream);
      return;
    }
    if (q == 0) adj_lower_bc(h->sc, d, tg, seed, a->overflow, h->stream);
    if (!hadj_pass(q, h->sc, d, tg, seed, h->stream)) adj_pass(q, h->sc, d, tg, seed, a->overflow, h->stream);
  };
  pass(4);  // pstep + swap_smooth
  fft_solve<double>(h->fft, h->sc, a->inter[5], h->stream, &h->launches, nullptr, true);
  pass(3);  // pressure source
  pass(1);  // momentum
  pass(2);  // scalars
  pass(0);  // subgrid
  h->launches += 5;
  a->cur = 1 - a->cur;
  return MGPU_OK;
}

static int adjoint_run(mgpu_handle* h, int nsteps, int interval, double* rmlmax_bar) {
  AdWork* a = h->ad;
  DevState<double>& d = h->d64;
  const size_t n = field_elems(h);
  const int t0 = h->timestep;
  const int nck = (nsteps + interval - 1) / interval;
  while ((int)a->ckpt.size() < 8 * nck) {
    double* p = nullptr;
    if (ad_alloc(h, &p, n)) return MGPU_ERR_CUDA;
    a->ckpt.push_back(p);
  }
  while ((int)a->seg.size() < 8 * interval) {
    double* p = nullptr;
    if (ad_alloc(h, &p, n)) return MGPU_ERR_CUDA;
    a->seg.push_back(p);
  }
  double* X[8];
  // forward sweep, saving a checkpoint every `interval` steps
  for (int st = 0; st < nsteps; ++st) {
    state_ptrs(d, X);
    if (st % interval == 0) copy_state(h, &a->ckpt[8 * (st / interval)], X);
    int rc = step_once<double>(h, d);
    if (rc) return rc;
  }
  state_ptrs(d, X);
  copy_state(h, a->final_state, X);
  CK(cudaMemsetAsync(a->prof_bar, 0, (h->cfg.nz + 2) * sizeof(double), h->stream));
  CK(cudaMemsetAsync(a->overflow, 0, sizeof(int), h->stream));
  // reverse sweep, one checkpoint segment at a time
  for (int c = nck - 1; c >= 0; --c) {
    const int s0 = c * interval, s1 = std::min(nsteps, s0 + interval);
    state_ptrs(d, X);
    copy_state(h, X, &a->ckpt[8 * c]);
    h->timestep = t0 + s0;
    // the input states of steps s0 .. s1-1; the last step's own result is not needed
    for (int st = s0; st < s1; ++st) {
      state_ptrs(d, X);
      copy_state(h, &a->seg[8 * (st - s0)], X);
      if (st == s1 - 1) break;
      int rc = step_once<double>(h, d);
      if (rc) return rc;
    }
    for (int st = s1 - 1; st >= s0; --st) {
      state_ptrs(d, X);
      copy_state(h, X, &a->seg[8 * (st - s0)]);
      h->timestep = t0 + st;
      int rc = adjoint_step(h);
      if (rc) return rc;
    }
  }
  state_ptrs(d, X);
  copy_state(h, X, a->final_state);
  h->timestep = t0 + nsteps;
  int ovf = 0;
  std::vector<double> pb(h->cfg.nz + 2);
  CK(cudaMemcpyAsync(&ovf, a->overflow, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(pb.data(), a->prof_bar, pb.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  CK(cudaGetLastError());
  if (ovf) return fail(h, MGPU_ERR_UNSUPPORTED, "adjoint tape capacity exceeded");
  double acc = 0.0;
  for (int k = 1; k <= h->cfg.nz; ++k) acc += pb[k] * a->drsq_h[k];
  if (rmlmax_bar) *rmlmax_bar = acc;
  return MGPU_OK;
}

template <typename T>
static int component(mgpu_handle* h, DevState<T>& d, int cid) {
  h->sc.forward = (h->timestep == 1) ? 1 : 0;
  forcing_flags(h);
  int rc = alloc_component_fields<T>(h, d);
  if (rc) return rc;
  switch (cid) {
    case MGPU_C_STEPPING_DIRECTION: return MGPU_OK;
    case MGPU_C_MEAN_PROFILES:
      // the component fields already hold u + ugal and the time-smoothed theta, as MONC's do
      h->launches += launch_mean_profiles<T>(h->sc, d.zu, d.zv, d.zth, d.zq, h->olz_d, h->stream);
      h->launches += launch_mean_profiles_state<T>(h->sc, d.u, d.v, d.th, nullptr, d.q, nullptr, 0.0, 0.0, 1.0, 0.0,
                                                   h->olbar_d, h->stream);
      break;
    case MGPU_C_FORCING:
      h->launches += subsidence_tendencies(h);
      rc = exact::launch_component<T>(cid, h->sc, d, h->stream, h->divmax_d, &h->launches);
      if (rc) return fail(h, rc, "component failed");
      break;
    case MGPU_C_HALO_SWAPPER: return MGPU_OK;  // periodic indexing in every kernel replaces the swap
    case MGPU_C_FFTSOLVER:
      if (h->cfg.solver != MGPU_SOLVER_FFT) return fail(h, MGPU_ERR_UNSUPPORTED, "model not configured for the FFT solver");
      fft_solve<T>(h->fft, h->sc, d.p, h->stream, &h->launches);
      break;
    case MGPU_C_ITERATIVESOLVER:
      if (h->cfg.solver != MGPU_SOLVER_ITERATIVE)
        return fail(h, MGPU_ERR_UNSUPPORTED, "model not configured for the iterative solver");
      rc = pressure_solve<T>(h, d.p);
      if (rc) return fail(h, rc, "iterative solve failed");
      break;
    case MGPU_C_DIVERR:
      CK(cudaMemsetAsync(h->divmax_d, 0, sizeof(unsigned long long), h->stream));
      rc = exact::launch_component<T>(cid, h->sc, d, h->stream, h->divmax_d, &h->launches);
      if (rc) return fail(h, rc, "component failed");
      {
        unsigned long long bits = 0;
        CK(cudaMemcpyAsync(&bits, h->divmax_d, sizeof(bits), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        double v;
        std::memcpy(&v, &bits, sizeof(v));
        if (v > h->global_divmax) h->global_divmax = v;
      }
      break;
    default:
      rc = exact::launch_component<T>(cid, h->sc, d, h->stream, h->divmax_d, &h->launches);
      if (rc) return fail(h, rc, "unknown or unsupported component");
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(h->stream));
  return MGPU_OK;
}

extern "C" {

int mgpu_upload_field(mgpu_handle* h, int32_t id, const double* host, int32_t layout) {
  if (!h || !host) return MGPU_ERR_ARGUMENT;
  return h->fp32 ? upload<float>(h, h->d32, id, host, layout) : upload<double>(h, h->d64, id, host, layout);
}

int mgpu_download_field(mgpu_handle* h, int32_t id, double* host, int32_t layout) {
  if (!h || !host) return MGPU_ERR_ARGUMENT;
  return h->fp32 ? download<float>(h, h->d32, id, host, layout) : download<double>(h, h->d64, id, host, layout);
}

int mgpu_get_profile(mgpu_handle* h, const char* name, double* out, int32_t* n) {
  if (!h || !name) return MGPU_ERR_ARGUMENT;
  const std::vector<double>* v = profile_by_name(h->rs, name);
  if (!v) return fail(h, MGPU_ERR_ARGUMENT, std::string("unknown profile ") + name);
  if (n) *n = h->cfg.nz;
  if (out)
    for (int k = 1; k <= h->cfg.nz; ++k) out[k - 1] = (*v)[k];
  return MGPU_OK;
}

int mgpu_step(mgpu_handle* h, int32_t nsteps) {
  if (!h || nsteps < 0) return MGPU_ERR_ARGUMENT;
  if (h->cfg.solver == MGPU_SOLVER_EXTERNAL)
    return fail(h, MGPU_ERR_UNSUPPORTED, "the pressure solve of this model is external: step it with mgpu_step_phase");
  for (int s = 0; s < nsteps; ++s) {
    int rc = h->fp32 ? step_once<float>(h, h->d32) : step_once<double>(h, h->d64);
    if (rc) return rc;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(h, MGPU_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  return MGPU_OK;
}

int mgpu_component_timestep(mgpu_handle* h, int32_t cid) {
  if (!h || cid < 0 || cid >= MGPU_C_COUNT) return MGPU_ERR_ARGUMENT;
  return h->fp32 ? component<float>(h, h->d32, cid) : component<double>(h, h->d64, cid);
}

int mgpu_set_timestep(mgpu_handle* h, int32_t ts) {
  if (!h || ts < 1) return MGPU_ERR_ARGUMENT;
  h->timestep = ts;
  return MGPU_OK;
}

int mgpu_get_reductions(mgpu_handle* h, mgpu_reductions* out) {
  if (!h || !out) return MGPU_ERR_ARGUMENT;
  if (h->divmax_step) {
    unsigned long long bits = 0;
    CK(cudaMemcpyAsync(&bits, h->divmax_d, sizeof(bits), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    std::memcpy(&h->global_divmax, &bits, sizeof(bits));
    h->divmax_step = false;
  }
  out->global_divmax = h->global_divmax;
  out->solver_iterations = h->solver_iterations;
  out->solver_residual = h->solver_residual;
  out->timestep = h->timestep;
  out->dtm = h->cfl.dtm_last;
  out->dtm_new = h->cfl.update_dtm ? h->cfl.dtm_new : h->sc.dtm;
  out->absolute_new_dtm = h->cfl.absolute_new_dtm;
  out->cvel = h->cfl.cvel;
  out->cvis = h->cfl.cvis;
  out->cfl_number = h->cfl.cfl_number;
  out->cvel_x = h->cfl.cvel_x;
  out->cvel_y = h->cfl.cvel_y;
  out->cvel_z = h->cfl.cvel_z;
  out->cfl_evaluations = h->cfl.evaluations;
  out->last_cfl_timestep = h->cfl.last_cfl_timestep;
  out->ugal = h->sc.ugal;
  out->vgal = h->sc.vgal;
  return MGPU_OK;
}

int mgpu_set_galilean_velocity(mgpu_handle* h, double ugal, double vgal) {
  if (!h || !std::isfinite(ugal) || !std::isfinite(vgal)) return MGPU_ERR_ARGUMENT;
  h->sc.ugal = h->sc.ugal_p = ugal;
  h->sc.vgal = h->sc.vgal_p = vgal;
  return MGPU_OK;
}

// ---- checkpoints: the host codec (checkpoint.cpp) around downloads / uploads of the state ----
static int checkpoint_fields(mgpu_handle* h, std::vector<std::vector<double>>& buf, std::vector<int>& ids) {
  const int nq = h->cfg.number_q_fields;
  const int base[9] = {MGPU_U, MGPU_V, MGPU_W, MGPU_TH, MGPU_ZU, MGPU_ZV, MGPU_ZW, MGPU_ZTH, MGPU_P};
  ids.assign(base, base + 9);
  for (int n = 0; n < nq; ++n) ids.push_back(MGPU_Q0 + n);
  for (int n = 0; n < nq; ++n) ids.push_back(MGPU_ZQ0 + n);
  buf.assign(ids.size(), std::vector<double>(field_elems(h)));
  return MGPU_OK;
}

int mgpu_checkpoint_write(mgpu_handle* h, const char* path) {
  if (!h || !path) return MGPU_ERR_ARGUMENT;
  std::vector<std::vector<double>> buf;
  std::vector<int> ids;
  checkpoint_fields(h, buf, ids);
  std::vector<const double*> ptr;
  for (size_t q = 0; q < ids.size(); ++q) {
    int rc = h->fp32 ? download<float>(h, h->d32, ids[q], buf[q].data(), MGPU_LAYOUT_XFAST)
                     : download<double>(h, h->d64, ids[q], buf[q].data(), MGPU_LAYOUT_XFAST);
    if (rc) return rc;
    ptr.push_back(buf[q].data());
  }
  std::vector<double> mean;
  const bool with_mean = needs_mean_profiles(h->cfg);
  if (with_mean) {
    // (3 + nq) rows of olz*bar, then olubar, olvbar, olthbar, olqbar(n)
    mean.resize((size_t)(6 + 2 * h->cfg.number_q_fields) * h->cfg.nz);
    if (int rc = mgpu_mean_profiles(h, mean.data())) return rc;
  }
  mgpu_checkpoint_meta meta{};
  mgpu_checkpoint_state(h, &meta);
  std::string err;
  int rc = checkpoint_write_host(h->cfg, h->rs, path, ptr.data(), with_mean ? mean.data() : nullptr, meta, err);
  if (rc) return fail(h, rc, "checkpoint write: " + err);
  return MGPU_OK;
}

int mgpu_checkpoint_read(mgpu_handle* h, const char* path) {
  if (!h || !path) return MGPU_ERR_ARGUMENT;
  std::vector<std::vector<double>> buf;
  std::vector<int> ids;
  checkpoint_fields(h, buf, ids);
  std::vector<double*> ptr;
  for (auto& b : buf) ptr.push_back(b.data());
  std::vector<double> mean((size_t)(6 + 2 * h->cfg.number_q_fields) * h->cfg.nz);
  int has_mean = 0;
  mgpu_checkpoint_meta meta{};
  std::string err;
  int rc = checkpoint_read_host(h->cfg, path, ptr.data(), mean.data(), &has_mean, meta, err);
  if (rc) return fail(h, rc, "checkpoint read: " + err);
  for (size_t q = 0; q < ids.size(); ++q) {
    rc = h->fp32 ? upload<float>(h, h->d32, ids[q], buf[q].data(), MGPU_LAYOUT_XFAST)
                 : upload<double>(h, h->d64, ids[q], buf[q].data(), MGPU_LAYOUT_XFAST);
    if (rc) return rc;
  }
  return mgpu_restore_state(h, &meta, has_mean ? mean.data() : nullptr);
}

int mgpu_checkpoint_state(mgpu_handle* h, mgpu_checkpoint_meta* meta) {
  if (!h || !meta) return MGPU_ERR_ARGUMENT;
  *meta = mgpu_checkpoint_meta{};
  meta->timestep = h->timestep - 1;  // the last completed step
  meta->last_cfl_timestep = h->cfl.last_cfl_timestep;
  meta->time = h->time;
  meta->dtm = h->sc.dtm;
  meta->dtm_new = h->cfl.update_dtm ? h->cfl.dtm_new : h->sc.dtm;
  meta->absolute_new_dtm = h->cfl.absolute_new_dtm;
  meta->ugal = h->sc.ugal;
  meta->vgal = h->sc.vgal;
  return MGPU_OK;
}

int mgpu_restore_state(mgpu_handle* h, const mgpu_checkpoint_meta* meta, const double* mean) {
  if (!h || !meta) return MGPU_ERR_ARGUMENT;
  if (mean && h->olz_d) {
    // (3 + nq) rows of olz*bar, then (3 + nq) rows of olubar, olvbar, olthbar, olqbar(n)
    const int nz = h->cfg.nz, nr = 3 + h->cfg.number_q_fields;
    std::vector<double> rows((size_t)(3 + MGPU_MAX_Q) * (nz + 2), 0.0), bars(rows.size(), 0.0);
    for (int r = 0; r < nr; ++r)
      for (int k = 1; k <= nz; ++k) {
        rows[(size_t)r * (nz + 2) + k] = mean[(size_t)r * nz + k - 1];
        bars[(size_t)r * (nz + 2) + k] = mean[(size_t)(nr + r) * nz + k - 1];
      }
    CK(cudaMemcpyAsync(h->olz_d, rows.data(), rows.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->olbar_d, bars.data(), bars.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
  }
  // readcheckpoint.F90 load_misc: the run continues at the step after the checkpointed one
  h->timestep = meta->timestep + 1;
  h->time = meta->time;
  h->sc.dtm = meta->dtm;
  h->sc.ugal = h->sc.ugal_p = meta->ugal;  // readcheckpoint.F90:184
  h->sc.vgal = h->sc.vgal_p = meta->vgal;
  h->cfl.dtm_last = meta->dtm;
  h->cfl.dtm_new = meta->dtm_new;
  h->cfl.update_dtm = h->cfg.cfl_enabled && meta->dtm_new != meta->dtm;
  h->cfl.absolute_new_dtm = meta->absolute_new_dtm;
  h->cfl.last_cfl_timestep = meta->last_cfl_timestep;
  return MGPU_OK;
}

int mgpu_mean_profiles(mgpu_handle* h, double* out) {
  if (!h || !out) return MGPU_ERR_ARGUMENT;
  // (3 + nq) rows of olz*bar, then (3 + nq) rows of olubar, olvbar, olthbar, olqbar(n)
  const int nz = h->cfg.nz, rows = 3 + h->cfg.number_q_fields;
  std::vector<double> buf((size_t)rows * (nz + 2)), bar((size_t)rows * (nz + 2));
  CK(cudaMemcpyAsync(buf.data(), h->olz_d, buf.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(bar.data(), h->olbar_d, bar.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  for (int r = 0; r < rows; ++r)
    for (int k = 1; k <= nz; ++k) {
      out[(size_t)r * nz + k - 1] = buf[(size_t)r * (nz + 2) + k];
      out[(size_t)(rows + r) * nz + k - 1] = bar[(size_t)r * (nz + 2) + k];
    }
  return MGPU_OK;
}

int mgpu_profile_diagnostics(mgpu_handle* h, double* out, int32_t* nrows) {
  if (!h || !out) return MGPU_ERR_ARGUMENT;
  if (!h->cfg.profile_diagnostics_enabled)
    return fail(h, MGPU_ERR_ARGUMENT, "profile_diagnostics_enabled is off (the mean profiles it reads are not kept)");
  if (h->cfg.advection_flow_fields != MGPU_ADVECT_PW)
    return fail(h, MGPU_ERR_UNSUPPORTED, "profile diagnostics of TVD flow advection (its flux diagnostics) are not provided");
  const int nz = h->cfg.nz, nq = h->cfg.number_q_fields;
  const bool moist = !h->cfg.passive_q && nq >= 2;
  const int rows = moist ? MGPU_PD_COUNT : MGPU_PD_VAPOUR;
  const bool has_mean = needs_mean_profiles(h->cfg);
  if (h->fp32) {
    DevState<float>& d = h->d32;
    h->launches += launch_profile_diagnostics<float>(h->sc, d.u, d.v, d.w, d.th, moist ? d.q[h->sc.iqv] : nullptr,
                                                     moist ? d.q[h->sc.iql] : nullptr, h->olbar_d, has_mean, h->pd_d,
                                                     h->stream, h->slab_halo);
  } else {
    DevState<double>& d = h->d64;
    h->launches += launch_profile_diagnostics<double>(h->sc, d.u, d.v, d.w, d.th, moist ? d.q[h->sc.iqv] : nullptr,
                                                      moist ? d.q[h->sc.iql] : nullptr, h->olbar_d, has_mean, h->pd_d,
                                                      h->stream, h->slab_halo);
  }
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, h->pd_d, (size_t)rows * nz * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (nrows) *nrows = rows;
  return MGPU_OK;
}

int mgpu_diagnostics(mgpu_handle* h, double* mean_theta, double* mean_w2) {
  if (!h) return MGPU_ERR_ARGUMENT;
  const int nz = h->cfg.nz;
  // a y-slab's means are over its interior rows
  if (h->fp32) launch_diagnostics<float>(h->sc, h->d32.th, h->d32.w, h->diag_d, h->diag_d + nz, h->stream, h->slab_halo);
  else launch_diagnostics<double>(h->sc, h->d64.th, h->d64.w, h->diag_d, h->diag_d + nz, h->stream, h->slab_halo);
  h->launches += 1;
  if (mean_theta) CK(cudaMemcpyAsync(mean_theta, h->diag_d, nz * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  if (mean_w2) CK(cudaMemcpyAsync(mean_w2, h->diag_d + nz, nz * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return MGPU_OK;
}

int mgpu_set_profiling(mgpu_handle* h, int32_t on) {
  if (!h) return MGPU_ERR_ARGUMENT;
  h->profiling = on != 0;
  for (int q = 0; q < MGPU_NSTAGES; ++q) { h->stage_ms[q] = 0.0; h->stage_n[q] = 0; }
  return MGPU_OK;
}

int mgpu_stage_times(mgpu_handle* h, double* ms_total, int64_t* launches) {
  if (!h) return MGPU_ERR_ARGUMENT;
  for (int q = 0; q < MGPU_NSTAGES; ++q) {
    if (ms_total) ms_total[q] = h->stage_ms[q];
    if (launches) launches[q] = h->stage_n[q];
  }
  return MGPU_OK;
}

int mgpu_fftsolver_adjoint(mgpu_handle* h) {
  if (!h) return MGPU_ERR_ARGUMENT;
  if (h->cfg.solver != MGPU_SOLVER_FFT) return fail(h, MGPU_ERR_UNSUPPORTED, "model not configured for the FFT solver");
  if (h->fp32) fft_solve<float>(h->fft, h->sc, h->d32.p, h->stream, &h->launches, nullptr, true);
  else fft_solve<double>(h->fft, h->sc, h->d64.p, h->stream, &h->launches, nullptr, true);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(h, MGPU_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  return MGPU_OK;
}

int mgpu_tl_step(mgpu_handle* h, int32_t nsteps, double d_rmlmax) {
  if (!h || nsteps < 0) return MGPU_ERR_ARGUMENT;
  if (int rc = ensure_tl(h)) return rc;
  for (int q = 0; q < nsteps; ++q)
    if (int rc = tl_step_once(h, d_rmlmax)) return rc;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(h, MGPU_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  return MGPU_OK;
}

int mgpu_adjoint_run(mgpu_handle* h, int32_t nsteps, int32_t checkpoint_interval, double* rmlmax_bar) {
  if (!h || nsteps < 1 || checkpoint_interval < 1) return MGPU_ERR_ARGUMENT;
  if (int rc = ensure_adj(h)) return rc;
  return adjoint_run(h, nsteps, checkpoint_interval, rmlmax_bar);
}

int mgpu_branch_flips(mgpu_handle* a, mgpu_handle* b, int64_t* count) {
  if (!a || !b || !count) return MGPU_ERR_ARGUMENT;
  mgpu_handle* h = a;  // the model whose stream runs the comparison and which reports errors
  if (a->fp32 || b->fp32 || a->cfg.nx != b->cfg.nx || a->cfg.ny != b->cfg.ny || a->cfg.nz != b->cfg.nz ||
      a->cfg.number_q_fields > 0 || b->cfg.number_q_fields > 0)
    return fail(h, MGPU_ERR_ARGUMENT, "branch_flips compares two dry FP64 models of one grid");
  a->sc.forward = (a->timestep == 1) ? 1 : 0;
  if (!a->flips_d) CK(cudaMalloc(&a->flips_d, sizeof(unsigned long long)));
  CK(cudaMemsetAsync(a->flips_d, 0, sizeof(unsigned long long), a->stream));
  // b's queued steps must be complete before a's stream reads its fields
  CK(cudaStreamSynchronize(b->stream));
  branch_flips(a->sc, a->d64, b->d64, a->flips_d, a->stream);
  a->launches += 1;
  unsigned long long host = 0;
  CK(cudaMemcpyAsync(&host, a->flips_d, sizeof(host), cudaMemcpyDeviceToHost, a->stream));
  CK(cudaStreamSynchronize(a->stream));
  *count = (int64_t)host;
  return MGPU_OK;
}

}  // extern "C"

// ---- y-slab decomposition ----------------------------------------------------------------
template <typename T>
static int step_phase(mgpu_handle* h, DevState<T>& d, int phase) {
  h->sc.forward = (h->timestep == 1) ? 1 : 0;  // steppingdirection.F90:44-48
  const bool exact_k = h->cfg.reproducible != 0;
  switch (phase) {
    case MGPU_PHASE_SUBGRID: {
      const bool cfl = h->cfg.cfl_enabled != 0;
      if (cfl && h->cfl.update_dtm) h->sc.dtm = h->cfl.dtm_new;  // monc.F90:313
      h->cfl.gathered = cfl && cfl_evaluation_step(h, h->timestep);
      h->launches += exact_k ? exact::launch_fused_subgrid<T>(h->sc, d, h->stream)
                             : fast::launch_fused_subgrid<T>(h->sc, d, h->stream);
      // this slab's extrema; the driver combines them across the slabs (mgpu_slab_cfl_extrema)
      if (h->cfl.gathered)
        h->launches += launch_cfl_gather<T>(h->sc, d, h->cfg.use_viscosity_and_diffusion != 0, h->cfl.part_d,
                                            h->cfl.out_d, h->stream, h->slab_halo);
      return MGPU_OK;
    }
    case MGPU_PHASE_DYNAMICS:
      forcing_flags(h);
      h->launches += subsidence_tendencies(h);
      if (sizeof(T) == 4) {
        if (!h->bmean_ext)
          return fail(h, MGPU_ERR_ARGUMENT, "FP32-mixed slab: mgpu_slab_level_means must precede each dynamics phase");
        h->sc.bmean = h->bmean_ext;
      }
      h->launches += exact_k ? exact::launch_fused_dynamics<T>(h->sc, d, h->stream, nullptr)
                             : fast::launch_fused_dynamics<T>(h->sc, d, h->stream, nullptr);
      h->sc.bmean = nullptr;
      h->bmean_ext = nullptr;
      swap_scalar_buffers<T>(d, h->cfg.number_q_fields);
      if (needs_mean_profiles(h->cfg)) {
        // this slab's means; the driver averages them across the slabs (mgpu_slab_mean_profiles)
        const bool fwd = h->sc.forward != 0;
        h->launches += launch_mean_profiles<T>(h->sc, d.zu_n, d.zv_n, d.th, d.q, h->olz_d, h->stream, h->slab_halo);
        h->launches += launch_mean_profiles_state<T>(h->sc, d.u, d.v, d.th_n, fwd ? nullptr : d.zth_n, d.q_n,
                                                     fwd ? nullptr : d.zq_n, h->sc.ugal, h->sc.vgal,
                                                     1.0 - 2.0 * h->sc.tsmth, h->sc.tsmth, h->olbar_d, h->stream,
                                                     h->slab_halo);
      }
      if (exact_k) exact::launch_fused_pressure_source<T>(h->sc, d, h->stream);
      else fast::launch_fused_pressure_source<T>(h->sc, d, h->stream);
      h->launches += 1;
      return MGPU_OK;
    case MGPU_PHASE_PSTEP:
      // cfltest (the end of the solver group) on the domain extrema, then the pressure terms
      if (h->cfg.cfl_enabled) {
        const bool gathered = h->cfl.gathered;
        h->cfl.gathered = false;
        if (gathered) {
          CK(cudaMemcpyAsync(h->cfl.out_h, h->cfl.out_d, 6 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
          CK(cudaEventRecord(h->cfl.ev, h->stream));
        }
        if (int rc = cfltest_callback(h, gathered)) return rc;
      }
      if (exact_k) exact::launch_fused_pstep_swap<T>(h->sc, d, h->stream);
      else fast::launch_fused_pstep_swap<T>(h->sc, d, h->stream);
      h->launches += 1;
      h->sc.ugal = h->sc.ugal_p;
      h->sc.vgal = h->sc.vgal_p;
      h->time += h->sc.dtm;
      h->timestep += 1;
      return MGPU_OK;
  }
  return fail(h, MGPU_ERR_ARGUMENT, "unknown step phase");
}

template <typename T>
static int halo_set(mgpu_handle* h, DevState<T>& d, int set, T** f) {
  int n = 0;
  if (set == MGPU_HALO_STATE) {
    T* st[8] = {d.u, d.v, d.w, d.th, d.zu, d.zv, d.zw, d.zth};
    for (T* p : st) f[n++] = p;
    for (int q = 0; q < h->cfg.number_q_fields; ++q) {
      f[n++] = d.q[q];
      f[n++] = d.zq[q];
    }
    return n;
  }
  if (set == MGPU_HALO_PRESSURE) {
    f[n++] = d.p;
    return n;
  }
  if (set >= MGPU_HALO_ITER_X && set <= MGPU_HALO_ITER_CG && h->iter) {
    // the solver vectors in the model's type (FP32-mixed: the FP32 correction solve's)
    void* v[2] = {nullptr, nullptr};
    const int nv = iter_slab_vectors(h->iter, set, v);
    for (int q = 0; q < nv; ++q) f[q] = static_cast<T*>(v[q]);
    return nv;
  }
  return -1;
}

template <typename T>
static int halo_rows(mgpu_handle* h, DevState<T>& d, int set, int depth, void* lo, void* hi, bool unpack) {
  T* f[8 + 2 * MGPU_MAX_Q];
  const int n = halo_set<T>(h, d, set, f);
  if (n < 0) return fail(h, MGPU_ERR_ARGUMENT, "unknown halo set");
  const int H = h->slab_halo, ny = h->cfg.ny;
  // pack the first and last `depth` interior rows; unpack into the rows just outside them
  const int r_lo = unpack ? H - depth : H, r_hi = unpack ? ny - H : ny - H - depth;
  launch_halo_rows<T>(h->sc, f, n, depth, r_lo, r_hi, static_cast<T*>(lo), static_cast<T*>(hi), unpack, h->stream);
  h->launches += 1;
  return MGPU_OK;
}

static int check_launch(mgpu_handle* h) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(h, MGPU_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  return MGPU_OK;
}

extern "C" {

int mgpu_slab_init(mgpu_handle* h, int32_t ny_global, int32_t halo, int32_t max_cols) {
  if (!h) return MGPU_ERR_ARGUMENT;
  if (h->cfg.solver != MGPU_SOLVER_EXTERNAL)
    return fail(h, MGPU_ERR_UNSUPPORTED, "a slab model is created with solver MGPU_SOLVER_EXTERNAL");
  if (h->slab.b1) return fail(h, MGPU_ERR_ARGUMENT, "slab already initialised");
  const int nyl = h->cfg.ny - 2 * halo, nxh = h->cfg.nx / 2 + 1;
  if (halo < 1 || nyl < 2 || nyl < halo || (nyl % 2) || !fft_length_ok(h->cfg.nx) || !fft_length_ok(ny_global) || nyl > ny_global ||
      max_cols < 1 || max_cols > nxh)
    return fail(h, MGPU_ERR_ARGUMENT,
                "slab needs halo >= 1, an even number of interior rows (ny - 2*halo) >= max(halo, 2) and <= ny_global, "
                "nx and ny_global of 4..4096 points with prime factors 2, 3 and 5, and 1 <= max_cols <= nx/2+1");
  int rc = fft_slab_plan_create(h->slab, h->sc, h->rs, ny_global, max_cols);
  if (rc) {
    fft_plan_destroy(h->slab);
    return fail(h, rc, "slab plan");
  }
  h->slab_halo = halo;
  h->slab_ny_global = ny_global;
  h->slab_cols = max_cols;
  return MGPU_OK;
}

int mgpu_step_phase(mgpu_handle* h, int32_t phase) {
  if (!h) return MGPU_ERR_ARGUMENT;
  if (h->cfg.solver != MGPU_SOLVER_EXTERNAL)
    return fail(h, MGPU_ERR_UNSUPPORTED, "phases are for models with an external pressure solve");
  int rc = h->fp32 ? step_phase<float>(h, h->d32, phase) : step_phase<double>(h, h->d64, phase);
  return rc ? rc : check_launch(h);
}

int mgpu_halo_fields(mgpu_handle* h, int32_t set) {
  if (!h) return MGPU_ERR_ARGUMENT;
  if (set == MGPU_HALO_STATE) return 8 + 2 * h->cfg.number_q_fields;
  if (set == MGPU_HALO_PRESSURE) return 1;
  if (set >= MGPU_HALO_ITER_X && set <= MGPU_HALO_ITER_X64) {
    if (!h->iter) return fail(h, MGPU_ERR_ARGUMENT, "the solver vectors exist after MGPU_SLAB_ITER_BEGIN");
    if (set == MGPU_HALO_ITER_X64 && !h->fp32) return fail(h, MGPU_ERR_ARGUMENT, "MGPU_HALO_ITER_X64 is FP32-mixed only");
    return set == MGPU_HALO_ITER_CG ? 2 : 1;
  }
  return fail(h, MGPU_ERR_ARGUMENT, "unknown halo set");
}

static int halo_entry(mgpu_handle* h, int32_t set, int32_t depth, void* lo, void* hi, bool unpack) {
  if (!h || !lo || !hi) return MGPU_ERR_ARGUMENT;
  if (!h->slab_halo) return fail(h, MGPU_ERR_ARGUMENT, "mgpu_slab_init first");
  if (depth < 1 || depth > h->slab_halo) return fail(h, MGPU_ERR_ARGUMENT, "halo depth out of range");
  if (set == MGPU_HALO_ITER_X64) {
    // an FP64 vector of an FP32-mixed model
    void* v[2] = {nullptr, nullptr};
    if (!h->iter || !h->fp32 || iter_slab_vectors(h->iter, set, v) != 1)
      return fail(h, MGPU_ERR_ARGUMENT, "MGPU_HALO_ITER_X64 is the FP32-mixed refinement's iterate");
    double* f[1] = {static_cast<double*>(v[0])};
    const int H = h->slab_halo, ny = h->cfg.ny;
    launch_halo_rows<double>(h->sc, f, 1, depth, unpack ? H - depth : H, unpack ? ny - H : ny - H - depth,
                             static_cast<double*>(lo), static_cast<double*>(hi), unpack, h->stream);
    h->launches += 1;
    return check_launch(h);
  }
  int rc = h->fp32 ? halo_rows<float>(h, h->d32, set, depth, lo, hi, unpack)
                   : halo_rows<double>(h, h->d64, set, depth, lo, hi, unpack);
  return rc ? rc : check_launch(h);
}

int mgpu_halo_pack(mgpu_handle* h, int32_t set, int32_t depth, void* d_lo, void* d_hi) {
  return halo_entry(h, set, depth, d_lo, d_hi, false);
}

int mgpu_halo_unpack(mgpu_handle* h, int32_t set, int32_t depth, const void* d_lo, const void* d_hi) {
  return halo_entry(h, set, depth, const_cast<void*>(d_lo), const_cast<void*>(d_hi), true);
}

int mgpu_slab_level_means(mgpu_handle* h, double* d_means) {
  if (!h || !d_means) return MGPU_ERR_ARGUMENT;
  if (!h->slab_halo) return fail(h, MGPU_ERR_ARGUMENT, "mgpu_slab_init first");
  if (h->fp32) launch_level_means<float>(h->sc, h->d32.th, h->d32.q, h->cfg.number_q_fields, d_means, h->stream, h->slab_halo);
  else launch_level_means<double>(h->sc, h->d64.th, h->d64.q, h->cfg.number_q_fields, d_means, h->stream, h->slab_halo);
  h->launches += 1;
  h->bmean_ext = d_means;
  return check_launch(h);
}

int mgpu_slab_mean_profiles(mgpu_handle* h, double* d_buf, int32_t put) {
  if (!h || !d_buf) return MGPU_ERR_ARGUMENT;
  if (!h->slab_halo) return fail(h, MGPU_ERR_ARGUMENT, "mgpu_slab_init first");
  if (!needs_mean_profiles(h->cfg))
    return fail(h, MGPU_ERR_ARGUMENT, "no mean profiles are kept (no damping, mean-profile subsidence or profile diagnostics)");
  const size_t row = (size_t)(h->cfg.nz + 2) * sizeof(double);
  const size_t nz_rows = (size_t)(3 + h->cfg.number_q_fields) * row, bar = nz_rows;
  if (put) {
    CK(cudaMemcpyAsync(h->olz_d, d_buf, nz_rows, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(h->olbar_d, (const char*)d_buf + nz_rows, bar, cudaMemcpyDeviceToDevice, h->stream));
  } else {
    CK(cudaMemcpyAsync(d_buf, h->olz_d, nz_rows, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync((char*)d_buf + nz_rows, h->olbar_d, bar, cudaMemcpyDeviceToDevice, h->stream));
  }
  return MGPU_OK;
}

int mgpu_slab_cfl_extrema(mgpu_handle* h, double* d_buf, int32_t put, int32_t* gathered) {
  if (!h || !d_buf) return MGPU_ERR_ARGUMENT;
  if (!h->slab_halo) return fail(h, MGPU_ERR_ARGUMENT, "mgpu_slab_init first");
  if (!h->cfg.cfl_enabled) return fail(h, MGPU_ERR_ARGUMENT, "cfltest is off");
  if (gathered) *gathered = h->cfl.gathered ? 1 : 0;
  if (!h->cfl.gathered) return MGPU_OK;  // not an evaluation step: nothing to combine
  h->launches += put ? launch_cfl_max_form(d_buf, h->cfl.out_d, h->stream)
                     : launch_cfl_max_form(h->cfl.out_d, d_buf, h->stream);
  return check_launch(h);
}

int mgpu_slab_iter(mgpu_handle* h, int32_t step, double* d_sums, int32_t* done) {
  if (!h) return MGPU_ERR_ARGUMENT;
  if (!h->slab_halo) return fail(h, MGPU_ERR_ARGUMENT, "mgpu_slab_init first");
  const size_t n = field_elems(h);
  void* p = h->fp32 ? static_cast<void*>(h->d32.p) : static_cast<void*>(h->d64.p);
  if (step == MGPU_SLAB_ITER_BEGIN) {
    if (!h->iter) {
      int st = MGPU_OK;
      h->iter = iter_create(h->sc, h->rs, h->cfg, h->fp32, &st, h->slab_halo, h->cfg.ny - h->slab_halo,
                            h->slab_ny_global);
      if (st) return fail(h, st, "iterative solver setup");
    }
    if (int rc = iter_slab_begin(h->iter, p, n, h->stream)) return fail(h, rc, "slab iterative begin");
    return MGPU_OK;
  }
  if (!h->iter) return fail(h, MGPU_ERR_ARGUMENT, "MGPU_SLAB_ITER_BEGIN first");
  if (step == MGPU_SLAB_ITER_END) {
    int rc = iter_slab_end(h->iter, p, n, h->stream, &h->solver_iterations, &h->solver_residual);
    if (rc == MGPU_ERR_CUDA) return fail(h, rc, "slab iterative end");
    return MGPU_OK;  // not converged: MONC only warns (iterativesolver.F90:240-242); see mgpu_get_reductions
  }
  const bool reduces = step == MGPU_SLAB_ITER_INIT || step == MGPU_SLAB_ITER_APPLY || step == MGPU_SLAB_ITER_APPLY2 ||
                       step == MGPU_SLAB_ITER_UPDATE || step == MGPU_SLAB_ITER_FINISH ||
                       step == MGPU_SLAB_ITER_PRECOND || step == MGPU_SLAB_ITER_COMPAT || step == MGPU_SLAB_ITER_REFINE;
  if (reduces && !d_sums) return fail(h, MGPU_ERR_ARGUMENT, "this step needs d_sums");
  if (step == MGPU_SLAB_ITER_FINISH) {
    int dn = 0;
    double err = 0.0;
    int rc = iter_slab_finish(h->iter, d_sums, h->stream, &h->launches, &dn, &err);
    if (rc) return fail(h, rc, "slab iterative finish (no reduction pending?)");
    h->solver_residual = err;
    if (done) *done = dn;
    return MGPU_OK;
  }
  if (int rc = iter_slab_step(h->iter, step, d_sums, h->stream, &h->launches)) return fail(h, rc, "slab iterative step");
  return MGPU_OK;
}

int mgpu_slab_fft_x(mgpu_handle* h, void* d_spec, int32_t nblocks, int32_t inverse) {
  if (!h || !d_spec) return MGPU_ERR_ARGUMENT;
  if (!h->slab_halo) return fail(h, MGPU_ERR_ARGUMENT, "mgpu_slab_init first");
  if (nblocks < 1 || nblocks > h->cfg.nx / 2 + 1) return fail(h, MGPU_ERR_ARGUMENT, "nblocks out of range");
  if (h->fp32) slab_fft_x<float>(h->slab, h->sc, h->d32.p, h->slab_halo, nblocks, d_spec, inverse != 0, h->stream, &h->launches);
  else slab_fft_x<double>(h->slab, h->sc, h->d64.p, h->slab_halo, nblocks, d_spec, inverse != 0, h->stream, &h->launches);
  return check_launch(h);
}

int mgpu_slab_solve_columns(mgpu_handle* h, void* d_spec, int32_t kx0, int32_t nkx, int32_t row_block,
                            int32_t transpose) {
  if (!h || !d_spec) return MGPU_ERR_ARGUMENT;
  if (!h->slab_halo) return fail(h, MGPU_ERR_ARGUMENT, "mgpu_slab_init first");
  if (kx0 < 0 || nkx < 1 || nkx > h->slab_cols || kx0 + nkx > h->cfg.nx / 2 + 1 || row_block < 1 ||
      h->slab_ny_global % row_block)
    return fail(h, MGPU_ERR_ARGUMENT, "column block or row block out of range");
  if (h->fp32)
    slab_solve_columns<float>(h->slab, h->sc, d_spec, kx0, nkx, row_block, transpose != 0, h->stream, &h->launches);
  else
    slab_solve_columns<double>(h->slab, h->sc, d_spec, kx0, nkx, row_block, transpose != 0, h->stream, &h->launches);
  return check_launch(h);
}

int mgpu_cfl_gather(mgpu_handle* h, double* out) {
  if (!h || !out) return MGPU_ERR_ARGUMENT;
  const bool vd = h->cfg.use_viscosity_and_diffusion != 0;
  if (h->fp32)
    h->launches += launch_cfl_gather<float>(h->sc, h->d32, vd, h->cfl.part_d, h->cfl.out_d, h->stream, h->slab_halo);
  else
    h->launches += launch_cfl_gather<double>(h->sc, h->d64, vd, h->cfl.part_d, h->cfl.out_d, h->stream, h->slab_halo);
  if (cudaMemcpyAsync(out, h->cfl.out_d, 6 * sizeof(double), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
      cudaStreamSynchronize(h->stream) != cudaSuccess)
    return fail(h, MGPU_ERR_CUDA, "cfl gather");
  return MGPU_OK;
}

int mgpu_mean_profile(mgpu_handle* h, int32_t id, double* out) {
  if (!h || !out) return MGPU_ERR_ARGUMENT;
  // horizontal means via a download; diagnostics only, not on the timed path
  std::vector<double> buf(field_elems(h));
  int rc = mgpu_download_field(h, id, buf.data(), MGPU_LAYOUT_XFAST);
  if (rc) return rc;
  const size_t plane = (size_t)h->cfg.nx * h->cfg.ny;
  for (int k = 0; k < h->cfg.nz; ++k) {
    double s = 0.0;
    for (size_t t = 0; t < plane; ++t) s += buf[k * plane + t];
    out[k] = s / (double)plane;
  }
  return MGPU_OK;
}

}  // extern "C"
