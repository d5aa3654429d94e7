// Internal declarations of libmoncgpu: host-side reference state and device model.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/monc_gpu.h"

namespace mgpu {

// Vertical-grid and reference-state profiles, 1-based like MONC (element [k], k = 1..nz),
// plus the horizontal-grid scalars.  Built on the host in FP64 (grid.cpp).
struct RefState {
  int nz = 0;
  std::vector<double> z, zn, dz, dzn, rdz, rdzn, rho, rhon, thref, dthref, czb, cza, czg, czh, tzc1, tzc2, tzd1, tzd2;
  std::vector<double> rneutml, rneutml_sq, buoy_co, prefn, prefrcp, rprefrcp, tref, tstarpr, qsat, dqsatdt, qsatfac;
  std::vector<double> gwx, gwy;  // geostrophic wind profile
  std::vector<double> moist_toff, tc0;  // FP64 offsets of the FP32-mixed moist terms (grid.cpp)
  double czn = 0, zlogm = 0, zlogth = 0, vk_on_zlogm = 0;
  double dx = 0, dy = 0, cx = 0, cy = 0, cx2 = 0, cy2 = 0, tcx = 0, tcy = 0;
  double rmlmax = 0, smallp = 0, rlvap_over_cp = 0, r_over_cp = 0;
  // surface scheme (setfluxlook / lowerbc)
  double surface_temperature_flux = 0, surface_vapour_flux = 0, fbuoy = 0;
  std::vector<double> lookup_ustr;  // 1-based, 80 entries
  double velmin = 0, velmax = 0, aloginv = 0, cneut = 0, cfc = 0;
  int lookup_entries = 80;
  std::vector<double> cq;
  int k_cloudmax = 0;  // simplecloud: highest level of saturation adjustment
  // damping (damping.F90:124-148) and subsidence (forcing.F90:568-582)
  std::vector<double> dmpco, dmpcoz, w_subs;
  int kdmpmin = 0;
};

// Builds the reference state from a configuration (restates gridmanager.F90:2008-2642,
// simplesetup.F90:149-266, setfluxlook.F90:63-186).  Throws std::runtime_error on bad input.
void build_reference_state(const mgpu_config& cfg, RefState& rs);
const std::vector<double>* profile_by_name(const RefState& rs, const std::string& name);

// Checkpoint files in MONC's layout (checkpoint.cpp); fields and mean as in mgpu_checkpoint_write_host
int checkpoint_write_host(const mgpu_config& c, const RefState& rs, const std::string& path,
                          const double* const* fields, const double* mean, const mgpu_checkpoint_meta& meta,
                          std::string& err);
int checkpoint_read_host(const mgpu_config& c, const std::string& path, double* const* fields, double* mean,
                         int* has_mean, mgpu_checkpoint_meta& meta, std::string& err);

// Profiles copied to device memory, 1-based (index k), FP64.
enum ProfileId {
  P_RDZ = 0, P_RDZN, P_DZN, P_RHO, P_RHON, P_DTHREF, P_CZB, P_CZA, P_CZG, P_CZH, P_TZC1, P_TZC2, P_TZD1, P_TZD2,
  P_RNEUTML_SQ, P_BUOY_CO, P_THREF, P_PREFRCP, P_RPREFRCP, P_TREF, P_TSTARPR, P_QSAT, P_DQSATDT, P_QSATFAC,
  P_GWX, P_GWY, P_PREFN, P_TOFF, P_TC0, P_DZ, P_DMPCO, P_DMPCOZ, P_WSUBS, P_COUNT
};

// Scalars every dynamical-core kernel reads (passed by value as a kernel parameter).
struct Scalars {
  int nx, ny, nz;
  long long plane;  // nx*ny
  double cx, cy, cx2, cy2, tcx, tcy;
  double dtm, tsmth, ugal, vgal, fcoriol, smallp;
  double czn, zn2, zlogm, zlogth, vk_on_zlogm, vk, z0, z0th, alphah, betam, betah, gammah, pi;
  double surface_temperature_flux, surface_vapour_flux, fbuoy, max_diff_or_visc;
  double velmin, aloginv, cneut, cfc, convective_limit;
  double subb, subc, subg, subh, suba, ric, ricinv;
  double eps, repsh, thcona, thconb, thconap1, rlvap_over_cp, G;
  double cq[MGPU_MAX_Q];  // buoyancy loading of each q field
  int simplecloud, k_cloudmax;
  int lookup_entries;
  int forward;  // 1 on the first (forward) step
  int point_dynamics;  // 1: always use the untiled dynamics kernel (MGPU_POINT_DYNAMICS=1)
  int level_chunks;    // level chunks of the tiled dynamics kernels; 0 = chosen from the occupancy
                       // (MGPU_LEVEL_CHUNKS=n fixes it)
  int rho_unity;       // 1 when rho = rhon = 1 on every level (Boussinesq with rhobous = 1)
  int passive_th, passive_q, nq, iqv, iql;
  int coriolis, surface_bcs, use_vd;
  int tvd_flow;            // 1: u, v, w advected by TVD (advection_flow_fields = tvd) instead of PW
  const double* prof;      // device: P_COUNT profiles, each (nz+2) long, 1-based
  const double* bmean;     // FP32-mixed fused step: horizontal means of th (row 0) and q(n) (row 1+n) per
                           // level, (nz+2) per row, removed from the buoyancy; null elsewhere
  const double* lookup;    // device: lookup_ustr, 1-based
  // damping and subsidence (damping.F90, forcing.F90); the flags are set per step (MONC applies
  // both from timestep 3)
  int damping, kdmpmin;
  int subs_th, subs_q;             // subsidence of u, v and theta / of the q fields this step
  int subs_local_th, subs_local_q; // 1: gradients of the column; 0: the tendencies in subs_tend
  const double* olz;       // device: olzubar, olzvbar, olzthbar, olzqbar(n) rows, (nz+2) each
  const double* subs_tend; // device: mean-profile subsidence tendencies usub, vsub, thsub, qsub(n) rows
  // Galilean transformation (pstep.F90:345-346, 453-469): ugal, vgal above are the frame of this
  // step's stepping; ugal_p, vgal_p the frame after this step's cfltest, which the pressure step
  // moves u, zu (v, zv) into when galilean is set and which the surface condition and the Robert
  // filter of the pressure-terms group read.  Equal to ugal, vgal outside cfltest evaluations.
  int galilean;
  double ugal_p, vgal_p;
  // th_advection's advection of the mean baroclinicity (thadvection.F90:196-216, Boussinesq form):
  // sth += (v + vgal) mfx - (u + ugal) mfy at levels 2..nz
  int th_baroclinic;
  double mfx, mfy;
};

}  // namespace mgpu
