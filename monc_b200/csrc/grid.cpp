// Host-side construction of the vertical grid, reference state and surface-scheme tables.
//
// These are one-off FP64 computations on the host (MONC does them in the initialisation
// callbacks); the device receives the finished profiles.  The arithmetic follows the MONC
// routines cited beside each block so that the profiles agree bit for bit with MONC's.
#include <algorithm>
#include <cmath>
#include <stdexcept>

#include "mgpu_internal.h"

namespace mgpu {

static inline double sqr(double a) { return a * a; }
static inline double cub(double a) { return a * a * a; }

extern "C" void mgpu_config_defaults(mgpu_config* c) {
  *c = mgpu_config{};
  c->nx = c->ny = c->nz = 1;
  c->n_kgd = 1;
  c->kgd[0] = 10;
  c->hgd[0] = 10.0;
  c->nsmth = 40;
  c->dxx = c->dyy = 1.0;
  c->zztop = 1.0;
  c->thref0 = 288.0;
  c->rhobous = 1.0;
  c->surface_pressure = 100000.0;
  c->surface_reference_pressure = 100000.0;
  c->rmlmax = -1.0;
  c->dtm = 0.001;
  c->passive_th = 1;
  c->passive_q = 1;
  c->use_viscosity_and_diffusion = 1;
  c->smag_subb = 40.0;
  c->smag_subc = 16.0;
  c->max_height_cloud = 20000.0;
  c->solver = MGPU_SOLVER_FFT;
  c->solver_type = MGPU_ITER_BICGSTAB;
  c->tolerance = 1.0e-4;
  c->max_iterations = 500;
  c->precision = MGPU_FP64;
  c->von_karman_constant = 0.4;
  c->z0 = 2.0e-3;
  c->z0th = 2.0e-4;
  c->alphah = 1.0;
  c->betam = 4.8;
  c->betah = 7.8;
  c->gammam = 19.3;
  c->gammah = 12.0;
  c->pi = 3.14159;
  c->cp = 1005.0;
  c->rlvap = 2.501e6;
  c->r = 287.05;
  c->G = 9.81;
  c->convective_limit = -0.5;
  c->ratio_mol_wts = 1.608;
  c->rlargep = 1.0e37;
  c->cfl_enabled = 1;
  c->cfl_frequency = 10;
  c->cfl_tollerance = 0.1;
  c->cfl_cvismax = 0.2;
  c->cfl_cvelmax = 0.2;
  c->cfl_dtmmax = 100.0;
  c->cfl_dtmmin = 0.0001;
  c->cfl_rincmax = 0.05;
  c->l_constant_dtm = 0;
  c->advection_flow_fields = MGPU_ADVECT_PW;
  c->adjoint_taped = 0;
  c->damping_enabled = 0;
  c->dmptim = 0.0;
  c->zdmp = 0.0;
  c->hdmp = 0.0;
  c->l_subs_pl_theta = 0;
  c->l_subs_pl_q = 0;
  c->subsidence_input_type = MGPU_SUBS_VELOCITY;
  c->subsidence_local_theta = 1;
  c->subsidence_local_q = 1;
  c->n_subs_pl = 0;
  for (int q = 0; q < MGPU_MAX_SUBS_NODES; ++q) c->z_subs_pl[q] = c->f_subs_pl[q] = 0.0;
  c->profile_diagnostics_enabled = 0;
  c->galilean_transformation = 0;  // global_config:268-270
  c->fix_ugal = c->fix_vgal = 0;
  c->ugal = c->vgal = 0.0;
}

// w-level heights: piecewise-linear kgd/hgd grid smoothed nsmth times
// (gridmanager.F90:2466-2495, 2556-2592), or explicit heights.
static void vertical_levels(const mgpu_config& c, RefState& rs) {
  const int n = c.nz;
  std::vector<double>& z = rs.z;
  std::vector<double>& zn = rs.zn;
  if (c.explicit_z) {
    for (int k = 1; k <= n; ++k) z[k] = c.z_levels[k - 1];
  } else {
    std::vector<int> kgd(c.kgd, c.kgd + c.n_kgd);
    std::vector<double> hgd(c.hgd, c.hgd + c.n_kgd);
    if (!kgd.empty() && kgd[0] == 1) {  // a level at the surface is implied (simplesetup.F90:162-169)
      kgd.erase(kgd.begin());
      hgd.erase(hgd.begin());
    }
    z[1] = 0.0;
    int kmax = kgd.empty() ? 1 : kgd[0];
    double zmax = 0.0;
    if (!kgd.empty() && kgd[0] > 1) {
      for (int k = 1; k <= kgd[0] && k <= n; ++k) z[k] = (double)(k - 1) * hgd[0] / (double)(kgd[0] - 1);
      for (size_t s = 1; s < kgd.size(); ++s) {
        if (kgd[s] <= 0) continue;
        kmax = kgd[s];
        zmax = hgd[s];
        for (int k = kgd[s - 1] + 1; k <= kgd[s] && k <= n; ++k)
          z[k] = hgd[s - 1] + (hgd[s] - hgd[s - 1]) * (double)(k - kgd[s - 1]) / (double)(kgd[s] - kgd[s - 1]);
      }
    }
    if (kmax < n)
      for (int k = kmax; k <= n; ++k) z[k] = zmax + (c.zztop - zmax) * (double)(k - kmax) / (double)(n - kmax);
    z[1] = 0.0;
    z[n] = c.zztop;
    for (int it = 0; it < c.nsmth; ++it) {
      for (int k = 2; k <= n; ++k) zn[k] = 0.5 * (z[k] + z[k - 1]);
      for (int k = 2; k <= n - 1; ++k) z[k] = 0.5 * (zn[k] + zn[k + 1]);
    }
  }
  for (int k = 3; k <= n - 1; ++k) zn[k] = 0.0625 * (9.0 * (z[k - 1] + z[k]) - z[k + 1] - z[k - 2]);
  zn[2] = 0.5 * (z[1] + z[2]);
  zn[1] = -zn[2];
  zn[n] = 0.5 * (z[n - 1] + z[n]);
}

// saturation.F90:19-21
static double qsaturation(double temperature, double pressure) {
  const double tk0c = 273.15, qsa1 = 3.8, qsa2 = -17.2693882, qsa3 = 35.86, qsa4 = 6.109;
  return qsa1 / (pressure * std::exp(qsa2 * (temperature - tk0c) / (temperature - qsa3)) - qsa4);
}

static void damping_and_subsidence(const mgpu_config& c, RefState& rs);

void build_reference_state(const mgpu_config& c, RefState& rs) {
  const int n = c.nz;
  if (c.nx < 4 || c.ny < 4 || n < 4 || n > MGPU_MAX_NZ) throw std::runtime_error("grid sizes out of range");
  if (c.dxx <= 0 || c.dyy <= 0 || c.dtm <= 0) throw std::runtime_error("dxx, dyy and dtm must be positive");
  rs.nz = n;
  std::vector<double>* all[] = {&rs.z, &rs.zn, &rs.dz, &rs.dzn, &rs.rdz, &rs.rdzn, &rs.rho, &rs.rhon, &rs.thref,
                                &rs.dthref, &rs.czb, &rs.cza, &rs.czg, &rs.czh, &rs.tzc1, &rs.tzc2, &rs.tzd1, &rs.tzd2,
                                &rs.rneutml, &rs.rneutml_sq, &rs.buoy_co, &rs.prefn, &rs.prefrcp, &rs.rprefrcp,
                                &rs.tref, &rs.tstarpr, &rs.qsat, &rs.dqsatdt, &rs.qsatfac, &rs.gwx, &rs.gwy,
                                &rs.moist_toff, &rs.tc0};
  for (auto* v : all) v->assign(n + 2, 0.0);
  rs.smallp = (double)1.0e-14f;  // MONC declares smallp in FP64 but initialises it from a single literal
  rs.rlvap_over_cp = c.rlvap / c.cp;
  rs.r_over_cp = c.r / c.cp;
  rs.rmlmax = c.rmlmax > 0.0 ? c.rmlmax : (double)0.23f * std::max(c.dxx, c.dyy);
  vertical_levels(c, rs);
  for (int k = 2; k <= n; ++k) {
    rs.dz[k] = rs.z[k] - rs.z[k - 1];
    rs.dzn[k] = rs.zn[k] - rs.zn[k - 1];
    rs.rdz[k] = 1. / rs.dz[k];
    rs.rdzn[k] = 1. / rs.dzn[k];
    if (!(rs.dz[k] > 0.0)) throw std::runtime_error("vertical levels must increase");
  }
  rs.dzn[1] = 0.0;
  // Boussinesq reference state (gridmanager.F90:2402-2421, 2649-2710)
  for (int k = 1; k <= n; ++k) {
    rs.thref[k] = c.thref0;
    rs.rho[k] = c.rhobous;
    rs.rhon[k] = c.rhobous;
  }
  for (int k = 1; k <= n - 1; ++k) rs.dthref[k] = rs.thref[k + 1] - rs.thref[k];
  rs.dthref[n] = 0.0;
  if (!c.passive_th) {
    std::vector<double> pdiff(n + 2, 0.0);
    double ptop = 0.0;
    for (int pass = 1; pass <= 2; ++pass) {
      rs.prefn[n] = std::pow(ptop / c.surface_reference_pressure, rs.r_over_cp);
      for (int k = n - 1; k >= 1; --k) pdiff[k] = c.G * rs.dzn[k + 1] / (0.5 * c.cp * (rs.thref[k] + rs.thref[k + 1]));
      for (int k = n - 1; k >= 1; --k) rs.prefn[k] = rs.prefn[k + 1] + pdiff[k];
      for (int k = n; k >= 1; --k) rs.prefn[k] = c.surface_reference_pressure * std::pow(rs.prefn[k], 1.0 / rs.r_over_cp);
      double p0 = 0.5 * (rs.prefn[1] + rs.prefn[2]);
      if (pass == 1) {
        ptop = std::pow(c.surface_pressure, rs.r_over_cp) + std::pow(ptop, rs.r_over_cp) - std::pow(p0, rs.r_over_cp);
        if (ptop <= 0.0) throw std::runtime_error("negative ptop in the reference pressure profile");
        ptop = std::pow(ptop, 1.0 / rs.r_over_cp);
      }
    }
  }
  // finite-difference coefficients (gridmanager.F90:2038-2062)
  for (int k = 2; k <= n - 1; ++k) {
    rs.czb[k] = (rs.rho[k - 1] / rs.rhon[k]) / (rs.dz[k] * rs.dzn[k]);
    rs.cza[k] = (rs.rho[k] / rs.rhon[k]) / (rs.dz[k] * rs.dzn[k + 1]);
    rs.czg[k] = -rs.czb[k] - rs.cza[k];
    if (k > 2) rs.czh[k] = rs.czb[k] * rs.cza[k - 1];
    rs.tzc1[k] = 0.25 * rs.rdz[k] * rs.rho[k - 1] / rs.rhon[k];
    rs.tzc2[k] = 0.25 * rs.rdz[k] * rs.rho[k] / rs.rhon[k];
    rs.tzd1[k] = 0.25 * rs.rdzn[k + 1] * rs.rhon[k] / rs.rho[k];
    rs.tzd2[k] = 0.25 * rs.rdzn[k + 1] * rs.rhon[k + 1] / rs.rho[k];
  }
  rs.czb[n] = (rs.rho[n - 1] / rs.rhon[n]) / (rs.dz[n] * rs.dzn[n]);
  rs.cza[n] = 0.0;
  rs.czg[n] = -rs.czb[n];
  rs.czh[n] = rs.czb[n] * rs.cza[n - 1];
  rs.tzc2[n] = 0.25 * rs.rdz[n] * rs.rho[n] / rs.rhon[n];
  rs.tzc1[n] = 0.25 * rs.rdz[n] * rs.rho[n - 1] / rs.rhon[n];
  rs.czn = rs.dzn[2] * 0.5;
  rs.zlogm = std::log(1.0 + rs.zn[2] / c.z0);
  rs.zlogth = std::log((rs.zn[2] + c.z0) / c.z0th);
  rs.vk_on_zlogm = c.von_karman_constant / rs.zlogm;
  // reference temperature and saturation (gridmanager.F90:2343-2363)
  for (int k = 1; k <= n; ++k) {
    rs.tref[k] = rs.thref[k] * std::pow(rs.prefn[k] / c.surface_reference_pressure, rs.r_over_cp);
    rs.tstarpr[k] = 0.0;
  }
  if (!c.passive_th) {
    for (int k = 1; k <= n; ++k) {
      rs.prefrcp[k] = std::pow(c.surface_reference_pressure / rs.prefn[k], rs.r_over_cp);
      rs.rprefrcp[k] = 1.0 / rs.prefrcp[k];
      rs.qsat[k] = qsaturation(rs.tref[k], 0.01 * rs.prefn[k]);
      rs.dqsatdt[k] = (qsaturation(rs.tref[k] + 1.0, 0.01 * rs.prefn[k]) - qsaturation(rs.tref[k] - 1.0, 0.01 * rs.prefn[k])) /
                      (2.0 * 1.0);
      rs.qsatfac[k] = 1.0 / (1.0 + rs.rlvap_over_cp * rs.dqsatdt[k]);
    }
    // FP64 offsets for the FP32-mixed moist terms: temperature minus 273.15 K of the reference
    // state, and rprefrcp(k) thref(k+1) - tstarpr(k) - tref(k) of the moist Richardson number
    for (int k = 1; k <= n; ++k) rs.tc0[k] = rs.thref[k] * rs.rprefrcp[k] - 273.15;
    for (int k = 1; k <= n - 1; ++k) rs.moist_toff[k] = rs.rprefrcp[k] * rs.thref[k + 1] - rs.tstarpr[k] - rs.tref[k];
  }
  // neutral mixing length (gridmanager.F90:2298-2310)
  for (int k = 2; k <= n - 1; ++k) {
    rs.rneutml[k] = std::sqrt(1.0 / (1.0 / sqr(c.von_karman_constant * (rs.z[k] + c.z0)) + 1.0 / sqr(rs.rmlmax)));
    rs.rneutml_sq[k] = rs.rneutml[k] * rs.rneutml[k];
  }
  // Boussinesq buoyancy coefficient (gridmanager.F90:2316-2337)
  if (!c.passive_th) {
    for (int k = 1; k <= n - 1; ++k) rs.buoy_co[k] = c.G / c.thref0;
    rs.buoy_co[n] = 0.;
  }
  // horizontal grid (gridmanager.F90:2624-2642); dx is stored through a single-precision real()
  rs.dx = (double)(float)c.dxx;
  rs.dy = (double)(float)c.dyy;
  rs.cx = 1. / rs.dx;
  rs.cy = 1. / rs.dy;
  rs.cx2 = rs.cx * rs.cx;
  rs.cy2 = rs.cy * rs.cy;
  rs.tcx = 0.25 / rs.dx;
  rs.tcy = 0.25 / rs.dy;
  // geostrophic wind profile (coriolis.F90:155-163), growing with height under the shear
  for (int k = 1; k <= n; ++k) {
    rs.gwx[k] = c.surface_geostrophic_wind_x;
    rs.gwy[k] = c.surface_geostrophic_wind_y;
    if (c.baroclinicity_use_geostrophic_shear) {
      rs.gwx[k] = rs.gwx[k] + c.geostrophic_wind_rate_of_change_in_x * rs.zn[k];
      rs.gwy[k] = rs.gwy[k] + c.geostrophic_wind_rate_of_change_in_y * rs.zn[k];
    }
  }
  // water loading coefficient of the vapour field (setfluxlook.F90:70-76)
  rs.cq.assign(std::max(c.number_q_fields, 1), 0.0);
  if (!c.passive_q && c.number_q_fields > 0) rs.cq[0] = c.ratio_mol_wts - 1.0;
  if (c.simplecloud_enabled) {
    // simplecloud.F90:230-248
    if (c.number_q_fields < 2) throw std::runtime_error("simplecloud needs the vapour and liquid q fields");
    rs.cq[1] = -1.0;
    int k = 2;
    for (; k <= c.nz - 1; ++k)
      if (rs.zn[k] > c.max_height_cloud) break;
    rs.k_cloudmax = k - 1;
  }
  // prescribed surface fluxes and the Monin-Obukhov u* table (setfluxlook.F90:78-99, 150-186)
  rs.lookup_ustr.assign(rs.lookup_entries + 1, 0.0);
  if (c.use_surface_boundary_conditions) {
    if (c.type_of_surface_boundary_conditions != 0) throw std::runtime_error("only prescribed surface fluxes are supported");
    rs.surface_temperature_flux = c.surface_sensible_heat_flux / (rs.rho[1] * c.cp);
    rs.surface_vapour_flux = c.surface_latent_heat_flux / (rs.rho[1] * c.rlvap);
    rs.fbuoy = 0.;
    if (!c.passive_th) rs.fbuoy = rs.buoy_co[1] * rs.surface_temperature_flux;
    if (!c.passive_q && c.number_q_fields > 0) rs.fbuoy = rs.fbuoy + rs.cq[0] * rs.surface_vapour_flux * c.G;
    if (rs.fbuoy > 0.0) {
      std::vector<double> vel(rs.lookup_entries + 1, 0.0);
      rs.velmax = 100.0;
      rs.velmin = 0.1;
      rs.aloginv = 1.0 / std::log(rs.velmax / rs.velmin);
      const double smth = 0.1;
      for (int ik = 1; ik <= rs.lookup_entries; ++ik) {
        float e = (float)(ik - 1) / (float)(rs.lookup_entries - 1);  // single-precision ratio in MONC
        vel[ik] = rs.velmin * std::pow(rs.velmax / rs.velmin, (double)e);
        double ustr = vel[ik] * rs.vk_on_zlogm;
        for (int it = 0; it < 30; ++it) {
          double ob = -cub(ustr) / (c.von_karman_constant * rs.fbuoy);
          double x1 = std::sqrt(std::sqrt(1. - c.gammam * (rs.zn[2] + c.z0) / ob));
          double x0 = std::sqrt(std::sqrt(1. - c.gammam * c.z0 / ob));
          ustr = (1. - smth) * ustr + smth * (c.von_karman_constant * vel[ik]) /
                                          (rs.zlogm - (2.0 * std::log((x1 + 1.0) / (x0 + 1.0)) +
                                                       std::log((x1 * x1 + 1.0) / (x0 * x0 + 1.0)) +
                                                       2.0 * std::atan(x0) - 2.0 * std::atan(x1)));
        }
        rs.lookup_ustr[ik] = ustr;
      }
      rs.cneut = rs.lookup_ustr[rs.lookup_entries] / vel[rs.lookup_entries];
      rs.cfc = rs.lookup_ustr[1] * std::pow(vel[1], c.convective_limit);
    }
  }
  damping_and_subsidence(c, rs);
}

// piecewise_linear_1d (interpolation.F90:15-58): linear between the nodes, the first node's value
// below it, the last node's value at exactly its height.  MONC leaves the levels above the last
// node unset; here they stay 0.
static void piecewise_linear_1d(const double* zvals, const double* vals, int nnodes, const std::vector<double>& zgrid,
                                int n, std::vector<double>& field) {
  std::vector<double> init(nnodes + 2), zng(nnodes + 2);
  const double verylow = -1.0e5;
  init[1] = vals[0];
  zng[1] = verylow;
  for (int nn = 2; nn <= nnodes + 1; ++nn) {
    init[nn] = vals[nn - 2];
    zng[nn] = zvals[nn - 2];
  }
  for (int nn = 1; nn <= nnodes; ++nn)
    for (int k = 1; k <= n; ++k)
      if (zng[nn] <= zgrid[k] && zgrid[k] < zng[nn + 1])
        field[k] = init[nn] + (init[nn + 1] - init[nn]) * (zgrid[k] - zng[nn]) / (zng[nn + 1] - zng[nn]);
  if (zgrid[n] == zng[nnodes + 1]) field[n] = init[nnodes + 1];
}

// damping coefficients (damping.F90:124-148) and the subsidence velocity (forcing.F90:568-582)
static void damping_and_subsidence(const mgpu_config& c, RefState& rs) {
  const int n = c.nz;
  rs.dmpco.assign(n + 2, 0.0);
  rs.dmpcoz.assign(n + 2, 0.0);
  rs.w_subs.assign(n + 2, 0.0);
  rs.kdmpmin = n + 1;  // no level damped
  if (c.damping_enabled) {
    if (!(c.hdmp > 0.0)) throw std::runtime_error("damping needs hdmp > 0");
    for (int k = n; k >= 1; --k) {
      rs.kdmpmin = k;
      if (rs.zn[k] >= c.zdmp) rs.dmpco[k] = c.dmptim * (std::exp((rs.zn[k] - c.zdmp) / c.hdmp) - 1.0);
      if (rs.z[k] >= c.zdmp) rs.dmpcoz[k] = c.dmptim * (std::exp((rs.z[k] - c.zdmp) / c.hdmp) - 1.0);
      if (rs.zn[k] < c.zdmp) break;
    }
  }
  if (c.l_subs_pl_theta || c.l_subs_pl_q) {
    if (c.n_subs_pl < 1 || c.n_subs_pl > MGPU_MAX_SUBS_NODES)
      throw std::runtime_error("subsidence needs 1..MGPU_MAX_SUBS_NODES nodes in z_subs_pl / f_subs_pl");
    piecewise_linear_1d(c.z_subs_pl, c.f_subs_pl, c.n_subs_pl, rs.z, n, rs.w_subs);
    if (c.subsidence_input_type == MGPU_SUBS_DIVERGENCE)
      for (int k = 1; k <= n; ++k) rs.w_subs[k] = -1.0 * rs.w_subs[k] * rs.z[k];
  }
}

const std::vector<double>* profile_by_name(const RefState& rs, const std::string& nm) {
  struct Entry { const char* name; const std::vector<double>* v; };
  const Entry tab[] = {{"z", &rs.z}, {"zn", &rs.zn}, {"dz", &rs.dz}, {"dzn", &rs.dzn}, {"rdz", &rs.rdz},
                       {"rdzn", &rs.rdzn}, {"rho", &rs.rho}, {"rhon", &rs.rhon}, {"thref", &rs.thref},
                       {"dthref", &rs.dthref}, {"czb", &rs.czb}, {"cza", &rs.cza}, {"czg", &rs.czg},
                       {"czh", &rs.czh}, {"tzc1", &rs.tzc1}, {"tzc2", &rs.tzc2}, {"tzd1", &rs.tzd1},
                       {"tzd2", &rs.tzd2}, {"rneutml", &rs.rneutml}, {"rneutml_sq", &rs.rneutml_sq},
                       {"buoy_co", &rs.buoy_co}, {"prefn", &rs.prefn}, {"prefrcp", &rs.prefrcp},
                       {"rprefrcp", &rs.rprefrcp}, {"tref", &rs.tref}, {"qsat", &rs.qsat},
                       {"dqsatdt", &rs.dqsatdt}, {"qsatfac", &rs.qsatfac}, {"dmpco", &rs.dmpco},
                       {"dmpcoz", &rs.dmpcoz}, {"w_subs", &rs.w_subs}, {"geostrophic_wind_x", &rs.gwx},
                       {"geostrophic_wind_y", &rs.gwy}};
  for (const Entry& e : tab)
    if (nm == e.name) return e.v;
  return nullptr;
}

}  // namespace mgpu

extern "C" int mgpu_reference_profile(const mgpu_config* cfg, const char* name, double* out) {
  if (!cfg || !name || !out) return MGPU_ERR_ARGUMENT;
  mgpu::RefState rs;
  try {
    mgpu::build_reference_state(*cfg, rs);
  } catch (std::exception&) {
    return MGPU_ERR_ARGUMENT;
  }
  const std::vector<double>* v = mgpu::profile_by_name(rs, name);
  if (!v) return MGPU_ERR_ARGUMENT;
  for (int k = 1; k <= cfg->nz; ++k) out[k - 1] = (*v)[k];
  return MGPU_OK;
}
