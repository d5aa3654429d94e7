// Oracle (test infrastructure only -- never linked into libmoncgpu.so).
//
// CPU restatement, in C++ FP64, of MONC's dynamical-core timestep as MONC executes it:
// fields in MONC's own layout data(k,j,i) with a 2-deep periodic halo, column callbacks run
// column by column (x outer, y inner, halo columns included) in the configured group order,
// TVD face fluxes carried between columns, stepfields lagging two columns behind, psrce's
// deferred -1 faces, and the FFTPACK pressure solve.  Each routine cites the Fortran it follows;
// loop order and expression trees follow the Fortran (left-to-right evaluation, single-precision
// literals kept single where MONC writes them without a kind suffix).  Build with
// -ffp-contract=off so that no multiply-add is fused.
//
// Parity pinning: MONC's own tests hold no golden vectors for this arithmetic and MONC cannot be
// compiled here (no Fortran compiler), so this restatement is "parity unpinned" against MONC
// itself; it is pinned by known-answer tests (FFT vs direct DFT, tridiagonal residuals,
// conservation) in tests/test_oracle_kat.py.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "oracle_internal.h"

namespace oracle {

static const int FORWARD_STEPPING = 1, CENTRED_STEPPING = 0;  // state.F90
static const int PRESCRIBED_SURFACE_FLUXES = 0, PRESCRIBED_SURFACE_VALUES = 1;

static inline double sign_(double a, double b) { return std::copysign(std::fabs(a), b); }  // Fortran SIGN
static inline double sq(double a) { return a * a; }                                         // a**2
static inline double cube(double a) { return a * a * a; }                                   // a**3
static inline double pow4(double a) { double t = a * a; return t * t; }                     // a**4
static inline double fmin3(double a, double b, double c) { return std::min(std::min(a, b), c); }
static inline double fmax_(double a, double b) { return a > b ? a : b; }   // Fortran MAX (no NaNs here)
static inline double fmin_(double a, double b) { return a < b ? a : b; }

struct TvdFieldState {           // per-field carried face fluxes (prognostics.F90 flux_previous_*)
  std::vector<double> fpx;       // flux_previous_x(nz, ny+4), 1-based (k, j)
  std::vector<double> fpy;       // flux_previous_y(nz)
  std::vector<double> fyb;       // flux_y_buffer(nz)
  int nz = 0;
  void alloc(int nz_, int nyh) { nz = nz_; fpx.assign((size_t)(nz + 1) * (nyh + 1), 0.0); fpy.assign(nz + 2, 0.0); fyb.assign(nz + 2, 0.0); }
  double* fpx_col(int j) { return &fpx[(size_t)(nz + 1) * j]; }  // index [k]
};

struct Model {
  mgpu_config cfg;
  int nx, ny, nz, nxh, nyh, xs, xe, ys, ye;
  // vertical grid / reference state (grids.F90:91-159)
  Prof z, zn, dz, dzn, rdz, rdzn, rho, rhon, thref, dthref, czb, cza, czg, czh, tzc1, tzc2, tzd1, tzd2;
  Prof rneutml, rneutml_sq, buoy_co, prefn, pdiff, prefrcp, rprefrcp, tref, tstarpr, qsat, dqsatdt, qsatfac;
  Prof geostrophic_wind_x, geostrophic_wind_y;
  double czn = 0, zlogm = 0, zlogth = 0, vk_on_zlogm = 0;
  // horizontal grid (gridmanager.F90:2624-2642)
  double dx, dy, cx, cy, cx2, cy2, tcx, tcy;
  // constants
  double smallp, vk, z0, z0th, alphah, betam, betah, gammam, gammah, pi, cp, rlvap, r, G, convective_limit,
      ratio_mol_wts, rlargep, rlvap_over_cp, r_over_cp;
  // smagorinsky constants (smagorinsky.F90 initialisation)
  double eps, repsh, thcona, thconb, thconap1, subb, subc, subg, subh, subr, pr_n, suba, ric, ricinv;
  // fields
  Field u, v, w, th, zu, zv, zw, zth, p, su, sv, sw, sth, savu, savv, savw, vis, diff;
  std::vector<Field> q, zq, sq;
  std::vector<double> cq;
  int iqv = 0, iql = 0;  // 0-based indices of vapour / liquid (q_indices)
  int k_cloudmax = 0;    // simplecloud: highest level of saturation adjustment
  // time stepping
  int timestep = 1, start_timestep = 1, field_stepping = FORWARD_STEPPING;
  int scalar_stepping = CENTRED_STEPPING, momentum_stepping = CENTRED_STEPPING;
  double dtm, ugal = 0.0, vgal = 0.0, tsmth;
  // surface
  double surface_temperature_flux = 0, surface_vapour_flux = 0, fbuoy = 0;
  int lookup_table_entries = 80;
  std::vector<double> lookup_table_velocity, lookup_table_ustr;
  double velmax = 0, velmin = 0, aloginv = 0, cneut = 0, cfc = 0, max_diff_or_visc;
  double local_divmax = 0.0;
  // column iteration state (timestepper.F90:65-122)
  int col_x = 1, col_y = 1;
  bool halo_column = false, first_col = false, last_col = false;
  // tvd module state
  std::vector<double> flux_x, flux_y, flux_z;
  TvdFieldState tvd_th;
  std::vector<TvdFieldState> tvd_q;
  TvdFieldState tvd_u, tvd_v, tvd_w;  // TVD momentum advection (advection_flow_fields = tvd)
  Field iflow[3][3];                  // [advected u, v, w][interpolated u, v, w]
  // psrce buffers (pressuresource.F90)
  std::vector<double> send_x, send_y, recv_x, recv_y;  // (nz-1, ny) / (nz-1, nx), 1-based (k-1, idx)
  // fft solver
  FftPlan plan_x, plan_y;
  std::vector<double> cos_x, cos_y;
  std::vector<double> pt;  // (nz, ny+2, nx+2) 1-based
  // iterative solver state (iterativesolver.F90:20-40)
  int last_iterations = 0;
  double last_residual = 0.0;
  double A_n = 0, A_s = 0, A_e = 0, A_w = 0;
  std::vector<double> A_u, A_d, A_p, A_lu_d, A_lu_u, A_vol;
  Field psource, prev_p;
  bool first_run = true;
  // cfltest (cfltest.F90:23-28, state.F90:104-117) and the gathers feeding it
  bool determine_flow_minmax = false;
  int last_cfl_timestep = 0, cfl_evaluations = 0;
  bool update_dtm = false;
  double dtm_new = 0.0, absolute_new_dtm = 0.0, dtm_last = 0.0, cfl_number = 0.0;
  double cvis = 0.0, cvis_last = 0.0, cvel = 0.0, cvel_x = 0.0, cvel_y = 0.0, cvel_z = 0.0;
  double local_zumin = 0.0, local_zumax = 0.0, local_zvmin = 0.0, local_zvmax = 0.0, local_cvel_z = 0.0;
  std::vector<double> abswmax;  // 1-based k
  int cfl_error = 0;
  // damping (damping.F90:19-21, grids.F90 dmpco/dmpcoz/kdmpmin), subsidence velocity (forcing.F90)
  // and the mean profiles they read (meanprofiles.F90, grids.F90 olz*bar)
  Prof dmpco, dmpcoz, w_subs, olzubar, olzvbar, olzthbar, olubar, olvbar, olthbar;
  std::vector<Prof> olzqbar;
  int kdmpmin = 0;
};

static inline double& PT(Model& m, int k, int j, int i) {
  return m.pt[(size_t)(k - 1) + (size_t)m.nz * ((size_t)(j - 1) + (size_t)(m.ny + 2) * (size_t)(i - 1))];
}

// ---------------------------------------------------------------------------------------------
// Grid and reference state (gridmanager.F90:2431-2495 original_vertical_grid_setup,
// :2556-2592 create_linear_grid, :2447-2456 spacings, :2402-2421, :2027-2075, :2298-2337,
// :2649-2710 pressure profile; horizontal :2624-2642)
// ---------------------------------------------------------------------------------------------
static void build_grid(Model& m) {
  const mgpu_config& c = m.cfg;
  int kkp = m.nz;
  Prof* all[] = {&m.z, &m.zn, &m.dz, &m.dzn, &m.rdz, &m.rdzn, &m.rho, &m.rhon, &m.thref, &m.dthref, &m.czb, &m.cza,
                 &m.czg, &m.czh, &m.tzc1, &m.tzc2, &m.tzd1, &m.tzd2, &m.rneutml, &m.rneutml_sq, &m.buoy_co,
                 &m.prefn, &m.pdiff, &m.prefrcp, &m.rprefrcp, &m.tref, &m.tstarpr, &m.qsat, &m.dqsatdt,
                 &m.qsatfac, &m.geostrophic_wind_x, &m.geostrophic_wind_y};
  for (Prof* pp : all) pp->alloc(kkp);
  double zztop = c.zztop;
  if (c.explicit_z) {
    for (int k = 1; k <= kkp; ++k) m.z(k) = c.z_levels[k - 1];
  } else {
    // create_linear_grid (kgd(1)==1 with hgd(1)==0 is shifted away as simplesetup.F90:162-169 does)
    std::vector<int> kgd(c.kgd, c.kgd + c.n_kgd);
    std::vector<double> hgd(c.hgd, c.hgd + c.n_kgd);
    if (!kgd.empty() && kgd[0] == 1) { kgd.erase(kgd.begin()); hgd.erase(hgd.begin()); }
    int ninitp = (int)kgd.size();
    m.z(1) = 0.0;
    int kmax = ninitp > 0 ? kgd[0] : 1;
    double zmax = 0.0;
    if (ninitp > 0 && kgd[0] > 1) {
      for (int k = 1; k <= kgd[0]; ++k) m.z(k) = (double)(k - 1) * hgd[0] / (double)(kgd[0] - 1);
      for (int i = 2; i <= ninitp; ++i) {
        if (kgd[i - 1] > 0) {
          kmax = kgd[i - 1];
          zmax = hgd[i - 1];
          for (int k = kgd[i - 2] + 1; k <= kgd[i - 1]; ++k)
            m.z(k) = hgd[i - 2] + (hgd[i - 1] - hgd[i - 2]) * (double)(k - kgd[i - 2]) / (double)(kgd[i - 1] - kgd[i - 2]);
        }
      }
    }
    if (kmax < kkp)
      for (int k = kmax; k <= kkp; ++k) m.z(k) = zmax + (zztop - zmax) * (double)(k - kmax) / (double)(kkp - kmax);
    m.z(1) = 0.0;
    m.z(kkp) = zztop;
    for (int n = 1; n <= c.nsmth; ++n) {
      for (int k = 2; k <= kkp; ++k) m.zn(k) = 0.5 * (m.z(k) + m.z(k - 1));
      for (int k = 2; k <= kkp - 1; ++k) m.z(k) = 0.5 * (m.zn(k) + m.zn(k + 1));
    }
  }
  for (int k = 3; k <= kkp - 1; ++k) m.zn(k) = 0.0625 * (9.0 * (m.z(k - 1) + m.z(k)) - m.z(k + 1) - m.z(k - 2));
  m.zn(2) = 0.5 * (m.z(1) + m.z(2));
  m.zn(1) = -m.zn(2);
  m.zn(kkp) = 0.5 * (m.z(kkp - 1) + m.z(kkp));
  for (int k = 2; k <= kkp; ++k) {
    m.dz(k) = m.z(k) - m.z(k - 1);
    m.dzn(k) = m.zn(k) - m.zn(k - 1);
    m.rdz(k) = 1. / m.dz(k);
    m.rdzn(k) = 1. / m.dzn(k);
  }
  m.dzn(1) = 0.0;
  // reference state: thref = thref0 (no l_thref), prefn = 0, rho = rhon = rhobous
  for (int k = 1; k <= kkp; ++k) {
    m.thref(k) = c.thref0;
    m.prefn(k) = 0.0;
    m.pdiff(k) = 0.0;
    m.rho(k) = c.rhobous;
    m.rhon(k) = c.rhobous;
  }
  for (int k = 1; k <= kkp - 1; ++k) m.dthref(k) = m.thref(k + 1) - m.thref(k);
  m.dthref(kkp) = 0.0;
  // set_anelastic_pressure, Boussinesq branch: pressure profile only when theta is active
  if (!c.passive_th) {
    double ptop = 0.0, p0;
    m.pdiff(kkp) = 0.0;
    for (int ipass = 1; ipass <= 2; ++ipass) {
      m.prefn(kkp) = std::pow(ptop / c.surface_reference_pressure, m.r_over_cp);
      for (int k = kkp - 1; k >= 1; --k)
        m.pdiff(k) = m.G * m.dzn(k + 1) / (0.5 * m.cp * (m.thref(k) + m.thref(k + 1)));
      for (int k = kkp - 1; k >= 1; --k) m.prefn(k) = m.prefn(k + 1) + m.pdiff(k);
      for (int k = kkp; k >= 1; --k) m.prefn(k) = c.surface_reference_pressure * std::pow(m.prefn(k), 1.0 / m.r_over_cp);
      p0 = 0.5 * (m.prefn(1) + m.prefn(2));
      if (ipass == 1) {
        ptop = std::pow(c.surface_pressure, m.r_over_cp) + std::pow(ptop, m.r_over_cp) - std::pow(p0, m.r_over_cp);
        ptop = std::pow(ptop, 1.0 / m.r_over_cp);
      }
    }
  } else {
    for (int k = 1; k <= kkp; ++k) m.prefn(k) = 0.0;
  }
  for (int k = 1; k <= kkp; ++k) { m.rho(k) = c.rhobous; m.rhon(k) = c.rhobous; m.pdiff(k) = 0.0; }
  // set_vertical_reference_profile coefficients
  for (int k = 2; k <= kkp - 1; ++k) {
    m.czb(k) = (m.rho(k - 1) / m.rhon(k)) / (m.dz(k) * m.dzn(k));
    m.cza(k) = (m.rho(k) / m.rhon(k)) / (m.dz(k) * m.dzn(k + 1));
    m.czg(k) = -m.czb(k) - m.cza(k);
    if (k > 2) m.czh(k) = m.czb(k) * m.cza(k - 1);
  }
  for (int k = 2; k <= kkp - 1; ++k) {
    m.tzc1(k) = 0.25 * m.rdz(k) * m.rho(k - 1) / m.rhon(k);
    m.tzc2(k) = 0.25 * m.rdz(k) * m.rho(k) / m.rhon(k);
  }
  for (int k = 2; k <= kkp - 1; ++k) {
    m.tzd1(k) = 0.25 * m.rdzn(k + 1) * m.rhon(k) / m.rho(k);
    m.tzd2(k) = 0.25 * m.rdzn(k + 1) * m.rhon(k + 1) / m.rho(k);
  }
  {
    int k = kkp;
    m.czb(k) = (m.rho(k - 1) / m.rhon(k)) / (m.dz(k) * m.dzn(k));
    m.cza(k) = 0.0;
    m.czg(k) = -m.czb(k);
    m.czh(k) = m.czb(k) * m.cza(k - 1);
    m.tzc2(k) = 0.25 * m.rdz(k) * m.rho(k) / m.rhon(k);
    m.tzc1(k) = 0.25 * m.rdz(k) * m.rho(k - 1) / m.rhon(k);
  }
  m.czn = m.dzn(2) * 0.5;
  m.zlogm = std::log(1.0 + m.zn(2) / m.z0);
  m.zlogth = std::log((m.zn(2) + m.z0) / m.z0th);
  m.vk_on_zlogm = m.vk / m.zlogm;
  // setup_reference_state_liquid_water_temperature_and_saturation (dry part: tref, prefrcp)
  for (int k = 1; k <= kkp; ++k) {
    m.tref(k) = m.thref(k) * std::pow(m.prefn(k) / c.surface_reference_pressure, m.r_over_cp);
    m.tstarpr(k) = 0.0;
  }
  if (!c.passive_th) {
    for (int k = 1; k <= kkp; ++k) {
      m.prefrcp(k) = std::pow(c.surface_reference_pressure / m.prefn(k), m.r_over_cp);
      m.rprefrcp(k) = 1.0 / m.prefrcp(k);
      // qsaturation (saturation.F90) -- used by moist Ri only
      // saturation.F90 qsaturation
      auto qsaturation = [&](double temperature, double pressure) {
        const double tk0c = 273.15, qsa1 = 3.8, qsa2 = -17.2693882, qsa3 = 35.86, qsa4 = 6.109;
        return qsa1 / (pressure * std::exp(qsa2 * (temperature - tk0c) / (temperature - qsa3)) - qsa4);
      };
      double delta_t = 1.0;
      m.qsat(k) = qsaturation(m.tref(k), 0.01 * m.prefn(k));
      m.dqsatdt(k) = (qsaturation(m.tref(k) + delta_t, 0.01 * m.prefn(k)) - qsaturation(m.tref(k) - delta_t, 0.01 * m.prefn(k))) /
                     (2.0 * delta_t);
      m.qsatfac(k) = 1.0 / (1.0 + m.rlvap_over_cp * m.dqsatdt(k));
    }
  }
  // calculate_mixing_length_for_neutral_case
  for (int k = 2; k <= kkp - 1; ++k) {
    m.rneutml(k) = std::sqrt(1.0 / (1.0 / sq(m.vk * (m.z(k) + m.z0)) + 1.0 / sq(m.cfg.rmlmax)));
    m.rneutml_sq(k) = m.rneutml(k) * m.rneutml(k);
  }
  // set_buoyancy_coefficient (Boussinesq)
  if (!c.passive_th) {
    for (int k = 1; k <= kkp - 1; ++k) m.buoy_co(k) = m.G / c.thref0;
    m.buoy_co(kkp) = 0.;
  } else {
    for (int k = 1; k <= kkp; ++k) m.buoy_co(k) = 0.;
  }
  // horizontal (gridmanager.F90:2624-2642): dx = real(resolution) is a single-precision conversion
  m.dx = (double)(float)c.dxx;
  m.dy = (double)(float)c.dyy;
  m.cx = 1. / m.dx;
  m.cy = 1. / m.dy;
  m.cx2 = m.cx * m.cx;
  m.cy2 = m.cy * m.cy;
  m.tcx = 0.25 / m.dx;
  m.tcy = 0.25 / m.dy;
  // coriolis.F90:155-163 geostrophic profile, with the shear of baroclinicity_use_geostrophic_shear
  for (int k = 1; k <= kkp; ++k) {
    m.geostrophic_wind_x(k) = c.surface_geostrophic_wind_x;
    m.geostrophic_wind_y(k) = c.surface_geostrophic_wind_y;
    if (c.baroclinicity_use_geostrophic_shear) {
      m.geostrophic_wind_x(k) = m.geostrophic_wind_x(k) + c.geostrophic_wind_rate_of_change_in_x * m.zn(k);
      m.geostrophic_wind_y(k) = m.geostrophic_wind_y(k) + c.geostrophic_wind_rate_of_change_in_y * m.zn(k);
    }
  }
}

// setfluxlook.F90:150-186 set_look: Monin-Obukhov u* lookup table for unstable conditions
static void set_look(Model& m) {
  m.lookup_table_velocity.assign(m.lookup_table_entries + 1, 0.0);
  m.lookup_table_ustr.assign(m.lookup_table_entries + 1, 0.0);
  if (m.fbuoy <= 0.0) return;
  m.velmax = 100.0;
  m.velmin = 0.1;
  m.aloginv = 1.0 / std::log(m.velmax / m.velmin);
  double smth = 0.1;
  for (int ik = 1; ik <= m.lookup_table_entries; ++ik) {
    float expo = (float)(ik - 1) / (float)(m.lookup_table_entries - 1);  // real(ik-1)/real(entries-1)
    m.lookup_table_velocity[ik] = m.velmin * std::pow(m.velmax / m.velmin, (double)expo);
    m.lookup_table_ustr[ik] = m.lookup_table_velocity[ik] * m.vk_on_zlogm;
    if (m.fbuoy > 0.0) {
      for (int i = 1; i <= 30; ++i) {
        double ob = -cube(m.lookup_table_ustr[ik]) / (m.vk * m.fbuoy);
        double x1 = std::sqrt(std::sqrt(1. - m.gammam * (m.zn(2) + m.z0) / ob));
        double x0 = std::sqrt(std::sqrt(1. - m.gammam * m.z0 / ob));
        m.lookup_table_ustr[ik] = (1. - smth) * m.lookup_table_ustr[ik] +
            smth * (m.vk * m.lookup_table_velocity[ik]) /
                (m.zlogm - (2.0 * std::log((x1 + 1.0) / (x0 + 1.0)) + std::log((x1 * x1 + 1.0) / (x0 * x0 + 1.0)) +
                            2.0 * std::atan(x0) - 2.0 * std::atan(x1)));
      }
    }
  }
  m.cneut = m.lookup_table_ustr[m.lookup_table_entries] / m.lookup_table_velocity[m.lookup_table_entries];
  m.cfc = m.lookup_table_ustr[1] * std::pow(m.lookup_table_velocity[1], m.convective_limit);
}

// ---------------------------------------------------------------------------------------------
// Halo handling (halocommunication.F90:486-509,1121-1168): serial periodic wrap.
// ---------------------------------------------------------------------------------------------
static void periodic_wrap(Model& m, Field& f, int depth, bool corners) {
  int kmax = m.nz;
  auto copy_y = [&](int tj, int sj) {
    for (int i = m.xs; i <= m.xe; ++i)
      for (int k = 1; k <= kmax; ++k) f(k, tj, i) = f(k, sj, i);
  };
  auto copy_x = [&](int ti, int si) {
    for (int j = m.ys; j <= m.ye; ++j)
      for (int k = 1; k <= kmax; ++k) f(k, j, ti) = f(k, j, si);
  };
  if (depth == 2) { copy_y(1, m.ye - 1); copy_y(2, m.ye); copy_y(m.ye + 1, m.ys); copy_y(m.ye + 2, m.ys + 1); }
  else { copy_y(2, m.ye); copy_y(m.ye + 1, m.ys); }
  if (depth == 2) { copy_x(1, m.xe - 1); copy_x(2, m.xe); copy_x(m.xe + 1, m.xs); copy_x(m.xe + 2, m.xs + 1); }
  else { copy_x(2, m.xe); copy_x(m.xe + 1, m.xs); }
  if (corners) {
    int nxi = m.nx, nyi = m.ny;
    for (int i = 1; i <= m.nxh; ++i)
      for (int j = 1; j <= m.nyh; ++j) {
        bool hx = (i < m.xs || i > m.xe), hy = (j < m.ys || j > m.ye);
        if (!(hx && hy)) continue;
        if (depth == 1 && (i == 1 || i == m.nxh || j == 1 || j == m.nyh)) continue;
        int si = ((i - m.xs) % nxi + nxi) % nxi + m.xs;
        int sj = ((j - m.ys) % nyi + nyi) % nyi + m.ys;
        for (int k = 1; k <= kmax; ++k) f(k, j, i) = f(k, sj, si);
      }
  }
}

// haloswapper.F90:62-71 (all prognostics and their z fields, depth halo_depth=2, corners)
static void halo_swapper(Model& m) {
  Field* fl[] = {&m.u, &m.zu, &m.v, &m.zv, &m.w, &m.zw, &m.th, &m.zth};
  for (Field* f : fl)
    if (f->active) periodic_wrap(m, *f, 2, true);
  for (size_t n = 0; n < m.q.size(); ++n) { periodic_wrap(m, m.q[n], 2, true); periodic_wrap(m, m.zq[n], 2, true); }
}

// clearsourceterms.F90:25-56
static void clearsourceterms(Model& m) {
  std::fill(m.su.d.begin(), m.su.d.end(), 0.0);
  std::fill(m.sv.d.begin(), m.sv.d.end(), 0.0);
  std::fill(m.sw.d.begin(), m.sw.d.end(), 0.0);
  if (m.sth.active) std::fill(m.sth.d.begin(), m.sth.d.end(), 0.0);
  for (auto& f : m.sq) std::fill(f.d.begin(), f.d.end(), 0.0);
}

// steppingdirection.F90:41-49
static void stepping_direction(Model& m) {
  m.field_stepping = CENTRED_STEPPING;
  if (m.timestep == m.start_timestep) m.field_stepping = FORWARD_STEPPING;
}

// ---------------------------------------------------------------------------------------------
// lower_bc (lowerbc.F90:221-305 compute_lower_boundary_conditions, :601-633 convective,
// :645-666 look, :672-702 neutral, :708-768 stable, :325-440 periodic wrap of level 1)
// ---------------------------------------------------------------------------------------------
static double look(Model& m, double vel) {
  double lookup_real_posn = 1.0 + (double)(float)(m.lookup_table_entries - 1) * std::log(vel / m.velmin) * m.aloginv;
  int lookup_int_posn = (int)lookup_real_posn;
  if (lookup_int_posn >= 1) {
    if (lookup_int_posn < m.lookup_table_entries) {
      return m.lookup_table_ustr[lookup_int_posn] +
             (lookup_real_posn - (double)(float)lookup_int_posn) *
                 (m.lookup_table_ustr[lookup_int_posn + 1] - m.lookup_table_ustr[lookup_int_posn]);
    }
    return vel * m.cneut;
  }
  return std::pow(vel, -m.convective_limit) * m.cfc;
}

static void surface_fluxes_column(Model& m, int y, int x, double hv, Field& thf, std::vector<Field>& qf) {
  double& vis1 = m.vis(1, y, x);
  double& diff1 = m.diff(1, y, x);
  auto scalar_bc = [&]() {
    if (m.th.active)
      thf(1, y, x) = (m.surface_temperature_flux * m.dzn(2) / diff1) + thf(2, y, x) - m.thref(1) + m.thref(2);
    if (m.cfg.number_q_fields > 0) {
      int n = m.iqv;
      qf[n](1, y, x) = qf[n](2, y, x) + m.surface_vapour_flux * m.dzn(2) / diff1;
    }
  };
  if (m.fbuoy > 0.0) {
    double ustr = look(m, hv);
    vis1 = m.czn * sq(ustr) / hv;
    diff1 = (m.vk * m.czn * ustr / m.alphah) /
            (m.zlogth - 2. * std::log((1. + std::sqrt(1. + m.gammah * m.vk * m.fbuoy * (m.zn(2) + m.z0) / cube(ustr))) /
                                      (1. + std::sqrt(1. + m.gammah * m.vk * m.fbuoy * m.z0th / cube(ustr)))));
    vis1 = fmin_(vis1, m.max_diff_or_visc);
    diff1 = fmin_(diff1, m.max_diff_or_visc);
    scalar_bc();
  } else if (m.fbuoy == 0.0) {
    double ustr = hv * m.vk_on_zlogm;
    vis1 = m.czn * sq(ustr) / hv;
    diff1 = vis1 * m.zlogm / (m.alphah * m.zlogth);
    vis1 = fmin_(vis1, m.max_diff_or_visc);
    diff1 = fmin_(diff1, m.max_diff_or_visc);
    scalar_bc();
  } else {
    double ustr = hv * m.vk_on_zlogm;
    if ((m.fbuoy - 1.E-9) < -4.0 * sq(m.vk) * cube(hv) / (27.0 * m.betam * m.zn(2) * sq(m.zlogm))) {
      vis1 = 0.0;
      diff1 = 0.0;
      if (m.th.active) thf(1, y, x) = thf(2, y, x);
      for (int n = 0; n < m.cfg.number_q_fields; ++n) qf[n](1, y, x) = qf[n](2, y, x);
    } else {
      ustr = ustr / 3.0 *
             (1.0 - 2.0 * std::cos((std::acos(-27.0 * m.betam * m.vk * m.zn(2) * m.fbuoy / (m.zlogm * 2.0 * cube(ustr)) - 1.0) +
                                    2.0 * m.pi) / 3.0));
      vis1 = m.czn * sq(ustr) / hv;
      diff1 = vis1 * (m.zlogm - m.betam * m.zn(2) * m.vk * m.fbuoy / cube(ustr)) /
              (m.alphah * m.zlogth - m.betah * m.vk * m.fbuoy * (m.zn(2) + m.z0 - m.z0th) / cube(ustr));
      vis1 = fmin_(vis1, m.max_diff_or_visc);
      diff1 = fmin_(diff1, m.max_diff_or_visc);
      scalar_bc();
    }
  }
}

static void lower_bc_column(Model& m) {
  int y = m.col_y, x = m.col_x;
  bool fwd = m.field_stepping == FORWARD_STEPPING;
  Field& zu_a = fwd ? m.u : m.zu;
  Field& zv_a = fwd ? m.v : m.zv;
  Field& zth_a = fwd ? m.th : m.zth;
  Field& th_a = fwd ? m.th : m.zth;
  std::vector<Field>& q_a = fwd ? m.q : m.zq;
  if (!m.cfg.use_viscosity_and_diffusion || !m.cfg.use_surface_boundary_conditions)
    throw std::runtime_error("oracle: lower_bc without surface boundary conditions is not restated");
  if (!(y < m.ys - 1 || x < m.xs - 1 || y > m.ye + 1 || x > m.xe + 1)) {
    double hv = sq(0.5 * (m.zu(2, y, x) + zu_a(2, y, x - 1)) + m.ugal);
    hv = hv + sq(0.5 * (zv_a(2, y, x) + zv_a(2, y - 1, x)) + m.vgal);
    hv = std::sqrt(hv) + m.smallp;
    if (m.cfg.type_of_surface_boundary_conditions != PRESCRIBED_SURFACE_FLUXES)
      throw std::runtime_error("oracle: prescribed surface values are not restated");
    surface_fluxes_column(m, y, x, hv, th_a, q_a);
  } else if (x == 1 && y == 1) {
    // register_async_wrapping_recv_requests: nothing in serial
  } else if (x == m.xe + 2 && y == m.ye + 2) {
    // complete_async_wrapping: periodic copy of level 1 of zth / zq, y first then x
    auto wrap1 = [&](Field& f) {
      for (int i = 1; i <= m.nxh; ++i) {
        f(1, 1, i) = f(1, m.ye - 1, i);
        f(1, 2, i) = f(1, m.ye, i);
        f(1, m.ye + 1, i) = f(1, m.ys, i);
        f(1, m.ye + 2, i) = f(1, m.ys + 1, i);
      }
      for (int j = 1; j <= m.nyh; ++j) {
        f(1, j, 1) = f(1, j, m.xe - 1);
        f(1, j, 2) = f(1, j, m.xe);
        f(1, j, m.xe + 1) = f(1, j, m.xs);
        f(1, j, m.xe + 2) = f(1, j, m.xs + 1);
      }
    };
    if (m.th.active) wrap1(zth_a);
    for (int n = 0; n < m.cfg.number_q_fields; ++n) wrap1(q_a[n]);
  }
}

// ---------------------------------------------------------------------------------------------
// smagorinsky (smagorinsky.F90:99-130 timestep, :180-275 setfri, :281-309 Ri, :316-402 moist Ri,
// :487-696 half squared strain)
// ---------------------------------------------------------------------------------------------
static void half_squared_strain(Model& m, Field& U, Field& V, Field& W, std::vector<double>& ssq) {
  int y = m.col_y, x = m.col_x;
  const double cx = m.cx, cy = m.cy, cx2 = m.cx2, cy2 = m.cy2;
  for (int k = 2; k <= m.nz - 1; ++k) {
    double ssq11 = cx2 * (sq(U(k + 1, y, x) - U(k + 1, y, x - 1)) + sq(U(k, y, x) - U(k, y, x - 1)));
    double ssq22 = cy2 * (sq(V(k + 1, y, x) - V(k + 1, y - 1, x)) + sq(V(k, y, x) - V(k, y - 1, x)));
    double ssq33 = sq((W(k, y, x) - W(k - 1, y, x)) * m.rdz(k)) + sq((W(k + 1, y, x) - W(k, y, x)) * m.rdz(k + 1));
    double ssq13 = (sq((U(k + 1, y, x) - U(k, y, x)) * m.rdzn(k + 1) + (W(k, y, x + 1) - W(k, y, x)) * cx) +
                    sq((U(k + 1, y, x - 1) - U(k, y, x - 1)) * m.rdzn(k + 1) + (W(k, y, x) - W(k, y, x - 1)) * cx)) * 0.5;
    double ssq23 = (sq((W(k, y, x) - W(k, y - 1, x)) * cy + (V(k + 1, y - 1, x) - V(k, y - 1, x)) * m.rdzn(k + 1)) +
                    sq((W(k, y + 1, x) - W(k, y, x)) * cy + (V(k + 1, y, x) - V(k, y, x)) * m.rdzn(k + 1))) * 0.5;
    double ssq12 =
        (((sq((U(k, y, x - 1) - U(k, y - 1, x - 1)) * cy + (V(k, y - 1, x) - V(k, y - 1, x - 1)) * cx) +
           sq((U(k, y + 1, x - 1) - U(k, y, x - 1)) * cy + (V(k, y, x) - V(k, y, x - 1)) * cx)) +
          (sq((U(k, y, x) - U(k, y - 1, x)) * cy + (V(k, y - 1, x + 1) - V(k, y - 1, x)) * cx) +
           sq((U(k, y + 1, x) - U(k, y, x)) * cy + (V(k, y, x + 1) - V(k, y, x)) * cx))) +
         ((sq((U(k + 1, y, x - 1) - U(k + 1, y - 1, x - 1)) * cy + (V(k + 1, y - 1, x) - V(k + 1, y - 1, x - 1)) * cx) +
           sq((U(k + 1, y + 1, x - 1) - U(k + 1, y, x - 1)) * cy + (V(k + 1, y, x) - V(k + 1, y, x - 1)) * cx)) +
          (sq((U(k + 1, y, x) - U(k + 1, y - 1, x)) * cy + (V(k + 1, y - 1, x + 1) - V(k + 1, y - 1, x)) * cx) +
           sq((U(k + 1, y + 1, x) - U(k + 1, y, x)) * cy + (V(k + 1, y, x + 1) - V(k + 1, y, x)) * cx)))) *
        0.125;
    ssq[k] = ssq11 + ssq22 + ssq33 + ssq13 + ssq23 + ssq12 + m.smallp;
  }
}

static void moist_ri_2(Model& m, const std::vector<double>& ssq, Field& TH, std::vector<Field>& Q, std::vector<double>& ri) {
  int y = m.col_y, x = m.col_x;
  Field& qv = Q[m.iqv];
  Field& ql = Q[m.iql];
  for (int k = 2; k <= m.nz - 1; ++k) {
    double tmpinv = 1.0 / ssq[k];
    double scltmp = m.rdzn(k + 1) * m.buoy_co(k);
    double qt_k = qv(k, y, x) + ql(k, y, x);
    double qt_kp1 = qv(k + 1, y, x) + ql(k + 1, y, x);
    double thlpr_k = TH(k, y, x) - m.rlvap_over_cp * ql(k, y, x) * m.prefrcp(k);
    double thlpr_kp1 = TH(k + 1, y, x) - m.rlvap_over_cp * ql(k + 1, y, x) * m.prefrcp(k);
    double qlli = fmax_(0.0, (qt_k - (m.qsat(k) + m.dqsatdt(k) * (m.rprefrcp(k) * thlpr_k - m.tstarpr(k)))) * m.qsatfac(k));
    double qlui = fmax_(0.0, (qt_kp1 - (m.qsat(k) + m.dqsatdt(k) * (m.rprefrcp(k) * (thlpr_kp1 + m.thref(k + 1)) -
                                                                  m.tstarpr(k) - m.tref(k)))) * m.qsatfac(k));
    double thvli = thlpr_k + m.thref(k) + (m.rlvap_over_cp * m.prefrcp(k) - m.thcona) * qlli;
    double thvui = thlpr_kp1 + m.thref(k + 1) + (m.rlvap_over_cp * m.prefrcp(k) - m.thconap1) * qlui;
    double thlpr_un = thlpr_kp1 - m.eps * (thlpr_kp1 - thlpr_k + m.dthref(k));
    double thlpr_ln = thlpr_k + m.eps * (thlpr_kp1 - thlpr_k + m.dthref(k));
    double qtun = qt_kp1 - m.eps * (qt_kp1 - qt_k);
    double qtln = qt_k + m.eps * (qt_kp1 - qt_k);
    double qlln = fmax_(0.0, (qtln - (m.qsat(k) + m.dqsatdt(k) * (m.rprefrcp(k) * thlpr_ln - m.tstarpr(k)))) * m.qsatfac(k));
    double qlun = fmax_(0.0, (qtun - (m.qsat(k) + m.dqsatdt(k) * (m.rprefrcp(k) * (thlpr_un + m.thref(k + 1)) -
                                                                 m.tstarpr(k) - m.tref(k)))) * m.qsatfac(k));
    double thvln = thlpr_ln + m.thref(k) + (m.rlvap_over_cp * m.prefrcp(k) - m.thcona) * qlln;
    double thvun = thlpr_un + m.thref(k + 1) + (m.rlvap_over_cp * m.prefrcp(k) - m.thconap1) * qlun;
    ri[k] = scltmp * tmpinv * (m.thconb * (qt_kp1 - qt_k) + ((thvln - thvli) - (thvun - thvui)) * m.repsh);
  }
}

// cfltest's evaluation test (cfltest.F90:80-82, stepfields.F90:249-256, smagorinsky.F90:151-153)
static bool cfl_step(const Model& m) {
  const int n = m.timestep, f = m.cfg.cfl_frequency;
  return n % f == 1 || n - m.start_timestep <= f || n >= m.last_cfl_timestep + f;
}

// smagorinsky.F90:143-173 (non-IB)
static void update_viscous_number(Model& m) {
  if (!cfl_step(m)) return;
  int y = m.col_y, x = m.col_x;
  for (int k = 2; k <= m.nz - 1; ++k)
    m.cvis = std::max(m.cvis, std::max(m.vis(k, y, x), m.diff(k, y, x)) *
                                  (m.rdzn(k + 1) * m.rdzn(k + 1) + m.cx2 + m.cy2));
}

static void smagorinsky_column(Model& m) {
  int y = m.col_y, x = m.col_x;
  if (!m.halo_column) {
    if (!m.cfg.use_viscosity_and_diffusion) throw std::runtime_error("oracle: use_viscosity_and_diffusion=.false.");
    std::vector<double> ssq(m.nz + 2, 0.0), ri(m.nz + 2, 0.0);
    bool fwd = m.field_stepping == FORWARD_STEPPING;
    if (fwd) half_squared_strain(m, m.u, m.v, m.w, ssq);
    else half_squared_strain(m, m.zu, m.zv, m.zw, ssq);
    Field& THa = fwd ? m.th : m.zth;
    std::vector<Field>& Qa = fwd ? m.q : m.zq;
    if (!m.cfg.passive_th) {
      if (!m.cfg.passive_q) {
        moist_ri_2(m, ssq, THa, Qa, ri);  // RICHARDSON_NUMBER_CALCULATION=2
      } else {
        // the dry branch reads current_state%th in both stepping modes (smagorinsky.F90:298-304)
        for (int k = 2; k <= m.nz - 1; ++k)
          ri[k] = (m.dthref(k) + m.th(k + 1, y, x) - m.th(k, y, x)) * m.rdzn(k + 1) * m.buoy_co(k) / ssq[k];
      }
    }
    // setfri (non-IB)
    for (int k = 2; k <= m.nz - 1; ++k) {
      double& vs = m.vis(k, y, x);
      double& df = m.diff(k, y, x);
      if (ri[k] <= 0.0) {
        vs = std::sqrt(1.0 - m.subc * ri[k]);
        df = m.suba * std::sqrt(1. - m.subb * ri[k]);
      } else if (ri[k] > 0.0 && ri[k] < m.ric) {
        double rifac = pow4(1. - ri[k] * m.ricinv);
        vs = rifac * (1. - m.subh * ri[k]);
        df = rifac * m.suba * (1. - m.subg * ri[k]);
      } else {
        vs = 0.0;
        df = 0.0;
      }
      double sctmp = m.rneutml_sq(k) * std::sqrt(ssq[k]);
      vs = vs * sctmp;
      df = df * sctmp;
    }
    m.vis(m.nz, y, x) = 0.0;
    m.diff(m.nz, y, x) = 0.0;
    if (m.cfg.cfl_enabled) update_viscous_number(m);
  }
  if (m.last_col) {  // non-blocking halo swap of vis and diff, completed before first use
    periodic_wrap(m, m.diff, 2, true);
    periodic_wrap(m, m.vis, 2, true);
  }
}

// ---------------------------------------------------------------------------------------------
// pw_advection advect_flow_fields (pwadvection.F90:466-610)
// ---------------------------------------------------------------------------------------------
static void pw_advection_column(Model& m) {
  if (m.halo_column) return;
  if (m.cfg.advection_flow_fields == MGPU_ADVECT_TVD) return;  // advect_flow is false (pwadvection.F90)
  int y = m.col_y, x = m.col_x;
  Field &U = m.u, &V = m.v, &W = m.w;
  const double tcx = m.tcx, tcy = m.tcy;
  for (int k = 2; k <= m.nz - 1; ++k) {
    double& s_u = m.su(k, y, x);
    s_u = tcx * (U(k, y, x - 1) * (U(k, y, x) + U(k, y, x - 1)) - U(k, y, x + 1) * (U(k, y, x) + U(k, y, x + 1)));
    s_u = s_u + tcy * (U(k, y - 1, x) * (V(k, y - 1, x) + V(k, y - 1, x + 1)) - U(k, y + 1, x) * (V(k, y, x) + V(k, y, x + 1)));
    s_u = s_u + (m.tzc1(k) * U(k - 1, y, x) * (W(k - 1, y, x) + W(k - 1, y, x + 1)) -
                 m.tzc2(k) * U(k + 1, y, x) * (W(k, y, x) + W(k, y, x + 1)));
    double& s_v = m.sv(k, y, x);
    s_v = tcy * (V(k, y - 1, x) * (V(k, y, x) + V(k, y - 1, x)) - V(k, y + 1, x) * (V(k, y, x) + V(k, y + 1, x)));
    s_v = s_v + tcx * (V(k, y, x - 1) * (U(k, y, x - 1) + U(k, y + 1, x - 1)) - V(k, y, x + 1) * (U(k, y, x) + U(k, y + 1, x)));
    s_v = s_v + (m.tzc1(k) * V(k - 1, y, x) * (W(k - 1, y, x) + W(k - 1, y + 1, x)) -
                 m.tzc2(k) * V(k + 1, y, x) * (W(k, y, x) + W(k, y + 1, x)));
    double& s_w = m.sw(k, y, x);
    s_w = (m.tzd1(k) * W(k - 1, y, x) * (W(k, y, x) + W(k - 1, y, x)) - m.tzd2(k) * W(k + 1, y, x) * (W(k, y, x) + W(k + 1, y, x)));
    s_w = s_w + tcx * (W(k, y, x - 1) * (U(k, y, x - 1) + U(k + 1, y, x - 1)) - W(k, y, x + 1) * (U(k, y, x) + U(k + 1, y, x)));
    s_w = s_w + tcy * (W(k, y - 1, x) * (V(k, y - 1, x) + V(k + 1, y - 1, x)) - W(k, y + 1, x) * (V(k, y, x) + V(k + 1, y, x)));
  }
  int k = m.nz;  // l_toplevel
  double& s_u = m.su(k, y, x);
  s_u = tcx * (U(k, y, x - 1) * (U(k, y, x) + U(k, y, x - 1)) - U(k, y, x + 1) * (U(k, y, x) + U(k, y, x + 1)));
  s_u = s_u + tcy * (U(k, y - 1, x) * (V(k, y - 1, x) + V(k, y - 1, x + 1)) - U(k, y + 1, x) * (V(k, y, x) + V(k, y, x + 1)));
  s_u = s_u + m.tzc1(k) * U(k - 1, y, x) * (W(k - 1, y, x) + W(k - 1, y, x + 1));
  double& s_v = m.sv(k, y, x);
  s_v = tcy * (V(k, y - 1, x) * (V(k, y, x) + V(k, y - 1, x)) - V(k, y + 1, x) * (V(k, y, x) + V(k, y + 1, x)));
  s_v = s_v + tcx * (V(k, y, x - 1) * (U(k, y, x - 1) + U(k, y + 1, x - 1)) - V(k, y, x + 1) * (U(k, y, x) + U(k, y + 1, x)));
  s_v = s_v + m.tzc1(k) * V(k - 1, y, x) * (W(k - 1, y, x) + W(k - 1, y + 1, x));
}

// ---------------------------------------------------------------------------------------------
// tvd_advection (tvdadvection.F90:722-762 advect_scalar_field, :911-960 differentiate_face_values,
// :990-1055 y-flux wrap) with ultflx (ultimateflux.F90:23-761)
// ---------------------------------------------------------------------------------------------
static const double r6 = 1.0 / 6.0;

// The vertical metrics ultflx is called with (tvdadvection.F90:722-908): scalars, u and v use
// rdz, rdzn, dzn with kdof = 0 over k = 2..nz; w uses rdzn, rdz, dz with kdof = 1 over
// k = 1..nz-1 (its bottom face from handle_vertical_fluxes_bottomofcolumn)
struct TvdMetrics {
  const Prof* rdz;
  const Prof* rdzn;
  const Prof* dzn;
  int kdof, kmin, kmax;
};

static double flux_in_w(const TvdMetrics& M, int k, double data_value, double dt, double sum_cfl_out, double rdc,
                        double fdels, double fd, double fc, double fu, double rdu, double fgt1, double fgt2) {
  double dd = (*M.dzn)(k + 1);
  double rdd = (*M.rdzn)(k + 1);
  double cflmod = std::fabs(data_value * (*M.rdzn)(k + 1) * dt);
  double hrcfl = 1.0 / (sum_cfl_out + 1.e-30);
  double hcfl = 0.5 * cflmod;
  double cflcoef = r6 * (1.0 - cflmod * cflmod) * (dd * dd * rdc);
  double rfdels = 1.0 / (fdels + 1.e-30);
  double ffs = 0.5 * (fd + fc) - hcfl * (fd - fc) - cflcoef * ((fd - fc) * rdd - (fc - fu) * rdu) - fgt1 - fgt2;
  double fnfs = (ffs - fu) * rfdels;
  double fncs = (fc - fu) * rfdels;
  double fnrefs = fncs * hrcfl;
  double ftemp = fmax_(fncs, fmin3(fnfs, fnrefs, 1.0));
  return ftemp * fdels + fu;
}

static double flux_in_xy(double data_value, double c, double dt, double sum_cfl_out, double fdels, double fd,
                         double fc, double fu, double fgt1, double fgt2, double fcurvs) {
  double cflmod = std::fabs(data_value * c * dt);
  double hrcfl = 1.0 / (sum_cfl_out + 1.e-30);
  double hcfl = 0.5 * cflmod;
  double cflcoef = r6 * (1.0 - cflmod * cflmod);
  double rfdels = 1.0 / (fdels + 1.e-30);
  double ffs = 0.5 * (fd + fc) - hcfl * (fd - fc) - cflcoef * fcurvs - fgt1 - fgt2;
  double fnfs = (ffs - fu) * rfdels;
  double fncs = (fc - fu) * rfdels;
  double fnrefs = fncs * hrcfl;
  double ftemp = fmax_(fncs, fmin3(fnfs, fnrefs, 1.0));
  return ftemp * fdels + fu;
}

// calculate_gradient_term_in_z
static double grad_z(const TvdMetrics& M, int k, const double* col1, const double* col2, double dt, double advneg,
                     double advpos, int kdof, int kp0, int kp1, const double* src1, const double* src2) {
  double specific_face = 0.125 * (col1[k] + col1[k - 1] + col2[k] + col2[k - 1]);
  int kposwf = (int)std::lround(0.5 + sign_(0.5, specific_face));
  int ksu = kp1 * (1 - kposwf) + (k - 1) * kposwf;
  int ksl = kp0 * (1 - kposwf) + k * kposwf;
  double temp_src = src1[ksl] - src1[ksu];
  if (src2) temp_src = temp_src * advpos + (src2[ksl] - src2[ksu]) * advneg;
  return std::fabs(specific_face) * (*M.rdz)(k + kdof) * dt * temp_src;
}

// calculate_gradient_term_in_x
static double grad_x(int k, const double* c1, const double* c2, const double* c3, const double* c4, double cx,
                     double dt, double fc, double s1, double s2, int kpv) {
  double specific_face = 0.125 * (c1[k] + c2[k] + c3[k + kpv] + c4[k + kpv]);
  double posuf = 0.5 + sign_(.5, specific_face);
  return std::fabs(specific_face) * cx * dt * (fc - (s1 * (1. - posuf) + s2 * posuf));
}

// nint(sign(1.0, x)): +1 unless the sign bit of x is set (SIGN honours -0.0)
static inline int nint_sign1(double x) { return std::signbit(x) ? -1 : 1; }

static void ultflx(Model& m, int y, int x, Field& U, Field& V, Field& W, Field& zf, const TvdMetrics& M, double dt,
                   std::vector<double>& flux_y, std::vector<double>& flux_z, std::vector<double>& flux_x,
                   double* flux_previous_x) {
  const int nz = m.nz;
  const int kdof = M.kdof;
  const double cx = m.cx, cy = m.cy;
  auto rdz = [&](int k) { return (*M.rdz)(k); };
  auto rdzn = [&](int k) { return (*M.rdzn)(k); };
  // ---- handle_vertical_fluxes: bottom of column (kmin = 1, w only: flux_z(2))
  if (M.kmin == 1) {
    const int k = 1;
    double fu, fc, fd;
    if (W(k, y, x) >= 0.0) { fu = zf(1, y, x); fc = zf(k, y, x); fd = zf(k + 1, y, x); }
    else { fu = zf(k + 2, y, x); fc = zf(k + 1, y, x); fd = zf(k, y, x); }
    double fcurvs = fd - 2.0 * fc + fu;
    double fdels = fd - fu;
    if (std::fabs(fcurvs) >= std::fabs(fdels)) {
      flux_z[k + 1] = fc;
    } else {
      double sum_cfl_out, fgt1, fgt2, rdu, rdc;
      if (W(k, y, x) >= 0.0) {
        sum_cfl_out = 0.0;
        sum_cfl_out = sum_cfl_out + W(k, y, x) * rdz(k + kdof);
        sum_cfl_out = sum_cfl_out + cy * (fmax_(0.0, V(k, y, x)) + std::fabs(fmin_(0.0, V(k, y - 1, x))));
        sum_cfl_out = sum_cfl_out + cx * (fmax_(0.0, U(k, y, x)) + std::fabs(fmin_(0.0, U(k, y, x - 1))));
        sum_cfl_out = sum_cfl_out * dt;
        {
          double sf = 0.125 * (V(k, y - 1, x) + V(k, y, x) + V(k + 1, y - 1, x) + V(k + 1, y, x));
          int jsu = y - nint_sign1(sf);
          fgt1 = std::fabs(sf) * cy * dt * (fc - zf(k, jsu, x));
        }
        fgt2 = grad_x(k, U.col(y, x - 1), U.col(y, x), U.col(y, x - 1), U.col(y, x), cx, dt, fc, zf(k, y, x + 1), zf(k, y, x - 1), 1);
        rdu = rdzn(2);
        rdc = rdz(k + kdof);
      } else {
        sum_cfl_out = 0.0;
        sum_cfl_out = sum_cfl_out + rdz(k + 1 + kdof) * (fmax_(0.0, W(k + 1, y, x)) - W(k, y, x));
        sum_cfl_out = sum_cfl_out + cy * (fmax_(0.0, V(k + 1, y, x)) + std::fabs(fmin_(0.0, V(k + 1, y - 1, x))));
        sum_cfl_out = sum_cfl_out + cx * (fmax_(0.0, U(k + 1, y, x)) + std::fabs(fmin_(0.0, U(k + 1, y, x - 1))));
        sum_cfl_out = sum_cfl_out * dt;
        {
          double sf = 0.125 * (V(k, y - 1, x) + V(k, y, x) + V(k + 1, y - 1, x) + V(k + 1, y, x));
          int jsu = y - nint_sign1(sf);
          fgt1 = std::fabs(sf) * cy * dt * (fc - zf(k + 1, jsu, x));
        }
        fgt2 = grad_x(k, U.col(y, x - 1), U.col(y, x), U.col(y, x - 1), U.col(y, x), cx, dt, fc, zf(k + 1, y, x + 1), zf(k + 1, y, x - 1), 1);
        rdu = rdzn(k + 2);
        rdc = rdz(k + 1 + kdof);
      }
      flux_z[k + 1] = flux_in_w(M, k, W(k, y, x), dt, sum_cfl_out, rdc, fdels, fd, fc, fu, rdu, fgt1, fgt2);
    }
  }
  // ---- handle_vertical_fluxes: top of column (k = nz-1)
  {
    int k = nz - 1;
    double fu, fc, fd;
    double* zfc = zf.col(y, x);
    if (W(k, y, x) >= 0.0) { fu = zfc[k - 1]; fc = zfc[k]; fd = zfc[k + 1]; }
    else { fu = 2.0 * zfc[k + 1] - zfc[k]; fc = zfc[k + 1]; fd = zfc[k]; }
    double fcurvs = fd - 2.0 * fc + fu;
    double fdels = fd - fu;
    if (std::fabs(fcurvs) >= std::fabs(fdels)) {
      flux_z[k + 1] = fc;
    } else {
      double sum_cfl_out, fgt1, fgt2, rdu, rdc;
      if (W(k, y, x) >= 0.0) {
        sum_cfl_out = 0.0;
        sum_cfl_out = sum_cfl_out + rdz(k + kdof) * (W(k, y, x) + std::fabs(fmin_(0.0, W(k - 1, y, x))));
        sum_cfl_out = sum_cfl_out + cy * (fmax_(0.0, V(k, y, x)) + std::fabs(fmin_(0.0, V(k, y - 1, x))));
        sum_cfl_out = sum_cfl_out + cx * (fmax_(0.0, U(k, y, x)) + std::fabs(fmin_(0.0, U(k, y, x - 1))));
        sum_cfl_out = sum_cfl_out * dt;
        // gradient_term_in_y(k, v, y, x, cy, dt, fc, zf, y, x)
        {
          double sf = 0.125 * (V(k, y - 1, x) + V(k, y, x) + V(k + 1, y - 1, x) + V(k + 1, y, x));
          int jsu = y - nint_sign1(sf);
          fgt1 = std::fabs(sf) * cy * dt * (fc - zf(k, jsu, x));
        }
        fgt2 = grad_x(k, U.col(y, x - 1), U.col(y, x), U.col(y, x - 1), U.col(y, x), cx, dt, fc, zf(k, y, x + 1), zf(k, y, x - 1), 1);
        rdu = rdzn(k);
        rdc = rdz(k + kdof);
      } else {
        sum_cfl_out = 0.0;
        sum_cfl_out = sum_cfl_out + (-W(k, y, x) * rdz(std::min(nz, k + 1 + kdof)));
        sum_cfl_out = sum_cfl_out + cy * (fmax_(0.0, V(k + 1, y, x)) + std::fabs(fmin_(0.0, V(k + 1, y - 1, x))));
        sum_cfl_out = sum_cfl_out + cx * (fmax_(0.0, U(k + 1, y, x)) + std::fabs(fmin_(0.0, U(k + 1, y, x - 1))));
        sum_cfl_out = sum_cfl_out * dt;
        {
          double sf = 0.125 * (V(k, y - 1, x) + V(k, y, x) + V(k + 1, y - 1, x) + V(k + 1, y, x));
          int jsu = y - nint_sign1(sf);
          fgt1 = std::fabs(sf) * cy * dt * (fc - zf(k + 1, jsu, x));
        }
        fgt2 = grad_x(k, U.col(y, x - 1), U.col(y, x), U.col(y, x - 1), U.col(y, x), cx, dt, fc, zf(k + 1, y, x + 1), zf(k + 1, y, x - 1), 1);
        rdu = rdzn(nz);
        rdc = rdz(std::min(nz, k + 1 + kdof));
      }
      flux_z[k + 1] = flux_in_w(M, k, W(k, y, x), dt, sum_cfl_out, rdc, fdels, fd, fc, fu, rdu, fgt1, fgt2);
    }
  }
  // ---- middle of column (k = 2 .. nz-2 -> flux_z(k+1))
  for (int k = 2; k <= nz - 2; ++k) {
    double sm = sign_(.5, W(k, y, x));
    double advpos = 0.5 + sm, advneg = 0.5 - sm;
    int kofset = (int)std::lround(advneg);
    double fu = zf(k - 1, y, x) * advpos + zf(k + 2, y, x) * advneg;
    double fc = zf(k + kofset, y, x);
    double fd = zf(k + 1, y, x) * advpos + zf(k, y, x) * advneg;
    double fcurvs = fd - 2.0 * fc + fu;
    double fdels = fd - fu;
    if (std::fabs(fcurvs) >= std::fabs(fdels)) {
      flux_z[k + 1] = fc;
    } else {
      double sum_cfl_out = 0.0;
      sum_cfl_out = sum_cfl_out + rdz(k + kofset) * (fmax_(0.0, W(k + kofset, y, x)) + std::fabs(fmin_(0.0, W(k - 1 + kofset, y, x))));
      sum_cfl_out = sum_cfl_out + cy * (fmax_(0.0, V(k + kofset, y, x)) + std::fabs(fmin_(0.0, V(k + kofset, y - 1, x))));
      sum_cfl_out = sum_cfl_out + cx * (fmax_(0.0, U(k + kofset, y, x)) + std::fabs(fmin_(0.0, U(k + kofset, y, x - 1))));
      sum_cfl_out = sum_cfl_out * dt;
      double fgt1;
      {
        double sf = 0.125 * (V(k, y - 1, x) + V(k, y, x) + V(k + 1, y - 1, x) + V(k + 1, y, x));
        int jsu = y - nint_sign1(sf);
        fgt1 = std::fabs(sf) * cy * dt * (fc - zf(k + kofset, jsu, x));
      }
      double fgt2 = grad_x(k, U.col(y, x - 1), U.col(y, x), U.col(y, x - 1), U.col(y, x), cx, dt, fc,
                           zf(k + kofset, y, x + 1), zf(k + kofset, y, x - 1), 1);
      double rdu = rdzn(k) * advpos + rdzn(k + 2) * advneg;
      double rdc = rdz(k + kdof) * advpos + rdz(k + 1 + kdof) * advneg;
      flux_z[k + 1] = flux_in_w(M, k, W(k, y, x), dt, sum_cfl_out, rdc, fdels, fd, fc, fu, rdu, fgt1, fgt2);
    }
  }
  if (M.kmin > 1) flux_z[2] = 0.0;
  // ---- y direction (skipped on the last interior row of the last y-process)
  if (y != m.ye) {
    for (int k = 2; k <= M.kmax; ++k) {
      int kp1 = std::min(k + 1, nz);
      int kp0 = kp1 - 1;
      double sm = sign_(0.5, V(k, y, x));
      double advpos = 0.5 + sm, advneg = 0.5 - sm;
      int jofset = (int)std::lround(advneg);
      int jperiod = (y > 1) ? 0 : 1;
      double fu = zf(k, y - 1 + jperiod, x) * advpos + zf(k, y + 2, x) * advneg;
      double fc = zf(k, y, x) * advpos + zf(k, y + 1, x) * advneg;
      double fd = zf(k, y + 1, x) * advpos + zf(k, y, x) * advneg;
      double fdels = fd - fu;
      double fcurvs = fd - 2.0 * fc + fu;
      if (std::fabs(fcurvs) >= std::fabs(fdels)) {
        flux_y[k] = fc;
      } else {
        double sum_cfl_out = 0.0;
        sum_cfl_out = sum_cfl_out + rdz(k) * (fmax_(0.0, W(k, y + jofset, x)) + std::fabs(fmin_(0.0, W(k - 1, y + jofset, x))));
        sum_cfl_out = sum_cfl_out + cy * (fmax_(0.0, V(k, y + jofset, x)) + std::fabs(fmin_(0.0, V(k, y - 1 + jofset + jperiod, x))));
        sum_cfl_out = sum_cfl_out + cx * (fmax_(0.0, U(k, y + jofset, x)) + std::fabs(fmin_(0.0, U(k, y + jofset, x - 1))));
        sum_cfl_out = sum_cfl_out * dt;
        double fgt1 = grad_z(M, k, W.col(y, x), W.col(y + 1, x), dt, advneg, advpos, kdof, kp0, kp1, zf.col(y + jofset, x), nullptr);
        double fgt2 = grad_x(k, U.col(y, x - 1), U.col(y, x), U.col(y + 1, x - 1), U.col(y + 1, x), cx, dt, fc,
                             zf(k, y + jofset, x + 1), zf(k, y + jofset, x - 1), 0);
        flux_y[k] = flux_in_xy(V(k, y, x), cy, dt, sum_cfl_out, fdels, fd, fc, fu, fgt1, fgt2, fcurvs);
      }
    }
  }
  // ---- x direction: flux_x <- previous (face x-1/2); compute face x+1/2 into flux_previous_x
  for (int k = 1; k <= nz; ++k) flux_x[k] = flux_previous_x[k];
  for (int k = 2; k <= M.kmax; ++k) {
    int kp1 = std::min(k + 1, nz);
    int kp0 = kp1 - 1;
    double sm = sign_(.5, U(k, y, x));
    double advpos = 0.5 + sm, advneg = 0.5 - sm;
    double fu = zf(k, y, x - 1) * advpos + zf(k, y, x + 2) * advneg;
    double fc = zf(k, y, x) * advpos + zf(k, y, x + 1) * advneg;
    double fd = zf(k, y, x + 1) * advpos + zf(k, y, x) * advneg;
    double fdels = fd - fu;
    double fcurvs = fd - 2.0 * fc + fu;
    if (std::fabs(fcurvs) >= std::fabs(fdels)) {
      flux_previous_x[k] = fc;
    } else {
      double sum_cfl_out;
      if (U(k, y, x) > 0.0) {
        sum_cfl_out = 0.0;
        sum_cfl_out = sum_cfl_out + rdz(k) * (fmax_(0.0, W(k, y, x)) + std::fabs(fmin_(0.0, W(k - 1, y, x))));
        sum_cfl_out = sum_cfl_out + cy * (fmax_(0.0, V(k, y, x)) + std::fabs(fmin_(0.0, V(k, y - 1, x))));
        sum_cfl_out = sum_cfl_out + cx * (U(k, y, x) + std::fabs(fmin_(0.0, U(k, y, x - 1))));
        sum_cfl_out = sum_cfl_out * dt;
      } else {
        sum_cfl_out = 0.0;
        sum_cfl_out = sum_cfl_out + rdz(k) * (fmax_(0.0, W(k, y, x + 1)) + std::fabs(fmin_(0.0, W(k - 1, y, x + 1))));
        sum_cfl_out = sum_cfl_out + cy * (fmax_(0.0, V(k, y, x + 1)) + std::fabs(fmin_(0.0, V(k, y - 1, x + 1))));
        sum_cfl_out = sum_cfl_out + cx * (fmax_(0.0, U(k, y, x + 1)) - U(k, y, x));
        sum_cfl_out = sum_cfl_out * dt;
      }
      double fgt1 = grad_z(M, k, W.col(y, x), W.col(y, x + 1), dt, advneg, advpos, kdof, kp0, kp1, zf.col(y, x), zf.col(y, x + 1));
      double fgt2;
      {
        // calculate_gradient_term_in_y with data_two: v at (y, x+1) and (y, x)
        double sf = 0.125 * (V(k, y, x + 1) + V(k, y, x) + V(k, y - 1, x + 1) + V(k, y - 1, x));
        int jsu = y - nint_sign1(sf);
        double t1 = zf(k, jsu, x) * advpos;
        double t2 = zf(k, jsu, x + 1) * advneg;
        t1 = t1 + t2;
        fgt2 = std::fabs(sf) * cy * dt * (fc - t1);
      }
      flux_previous_x[k] = flux_in_xy(U(k, y, x), cx, dt, sum_cfl_out, fdels, fd, fc, fu, fgt1, fgt2, fcurvs);
    }
  }
}

static void differentiate_face_values(Model& m, int y, int x, Field& U, Field& V, Field& W, Field& S,
                                      const std::vector<double>& fyp, const double* fxp, const Prof& tz1,
                                      const Prof& tz2, bool differentiate_top) {
  const double cx = m.cx, cy = m.cy;
  for (int k = 2; k <= m.nz - 1; ++k) {
    double& s = S(k, y, x);
    s = s + (V(k, y - 1, x) * fyp[k] - V(k, y, x) * m.flux_y[k]) * cy;
    s = s + 4.0 * (W(k - 1, y, x) * m.flux_z[k] * tz1(k) - W(k, y, x) * m.flux_z[k + 1] * tz2(k));
    s = s + (U(k, y, x - 1) * m.flux_x[k] - U(k, y, x) * fxp[k]) * cx;
  }
  if (!differentiate_top) return;
  int k = m.nz;
  double& s = S(k, y, x);
  s = 0.0;
  s = s + (V(k, y - 1, x) * fyp[k] - V(k, y, x) * m.flux_y[k]) * cy;
  s = s + 4.0 * tz1(k) * W(k - 1, y, x) * m.flux_z[k];
  s = s + (U(k, y, x - 1) * m.flux_x[k] - U(k, y, x) * fxp[k]) * cx;
}

static void advect_scalar_field(Model& m, double dt, Field& zqf, Field& qf, Field& sf, TvdFieldState& st) {
  int y = m.col_y, x = m.col_x;
  Field& src = (m.field_stepping == FORWARD_STEPPING) ? qf : zqf;
  const TvdMetrics M{&m.rdz, &m.rdzn, &m.dzn, 0, 2, m.nz};
  ultflx(m, y, x, m.u, m.v, m.w, src, M, dt, m.flux_y, m.flux_z, m.flux_x, st.fpx_col(y));
  if (y == m.ye) {  // complete_y_flux_wrap_recv_if_required (serial: local copy)
    for (int k = 1; k <= m.nz; ++k) m.flux_y[k] = st.fyb[k];
  }
  if (!m.halo_column)
    differentiate_face_values(m, y, x, m.u, m.v, m.w, sf, st.fpy, st.fpx_col(y), m.tzc1, m.tzc2, true);
  if (y < m.ye)
    for (int k = 1; k <= m.nz; ++k) st.fpy[k] = m.flux_y[k];
  if (y == m.ys - 1)  // register_y_flux_wrap_send_if_required
    for (int k = 1; k <= m.nz; ++k) st.fyb[k] = m.flux_y[k];
}

// interpolate_to_dual (stencil.F90:87-169) for the advection of field c (0 u, 1 v, 2 w): u, v, w
// averaged with their neighbour one point along the direction in which c is on the primal grid
// (x for u, y for v, z for w; simplesetup.F90:70-85), left as they are where that neighbour is
// outside the local arrays and, for z, at the top level.  MONC caches these per column as it
// sweeps; stepfields lags two columns behind, so every cached value is a pre-step one and
// computing them all before the sweep gives the same numbers.
static void interpolate_flow(Model& m, int c) {
  Field* src[3] = {&m.u, &m.v, &m.w};
  for (int f = 0; f < 3; ++f) {
    Field& in = *src[f];
    Field& out = m.iflow[c][f];
    for (int i = 1; i <= m.nxh; ++i)
      for (int j = 1; j <= m.nyh; ++j)
        for (int k = 1; k <= m.nz; ++k) {
          const int jj = c == 1 ? j + 1 : j, ii = c == 0 ? i + 1 : i, kk = c == 2 ? k + 1 : k;
          if (jj > m.nyh || ii > m.nxh || (c == 2 && k == m.nz)) out(k, j, i) = in(k, j, i);
          else out(k, j, i) = 0.5 * (in(k, j, i) + in(kk, jj, ii));
        }
  }
}

// advect_u / advect_v / advect_w (tvdadvection.F90:765-908): field c advected by the interpolated
// flow; w with the swapped vertical metrics and kdof = 1, its sources on levels 2..nz-1 only
static void advect_flow_field(Model& m, int c, double dt, Field& f, Field& zf, Field& sf, TvdFieldState& st) {
  int y = m.col_y, x = m.col_x;
  Field& src = (m.field_stepping == FORWARD_STEPPING) ? f : zf;
  Field &IU = m.iflow[c][0], &IV = m.iflow[c][1], &IW = m.iflow[c][2];
  const TvdMetrics M = c == 2 ? TvdMetrics{&m.rdzn, &m.rdz, &m.dz, 1, 1, m.nz - 1}
                              : TvdMetrics{&m.rdz, &m.rdzn, &m.dzn, 0, 2, m.nz};
  ultflx(m, y, x, IU, IV, IW, src, M, dt, m.flux_y, m.flux_z, m.flux_x, st.fpx_col(y));
  if (y == m.ye)
    for (int k = 1; k <= m.nz; ++k) m.flux_y[k] = st.fyb[k];
  if (!m.halo_column) {
    if (c == 2) differentiate_face_values(m, y, x, IU, IV, IW, sf, st.fpy, st.fpx_col(y), m.tzd1, m.tzd2, false);
    else differentiate_face_values(m, y, x, IU, IV, IW, sf, st.fpy, st.fpx_col(y), m.tzc1, m.tzc2, true);
  }
  if (y < m.ye)
    for (int k = 1; k <= m.nz; ++k) st.fpy[k] = m.flux_y[k];
  if (y == m.ys - 1)
    for (int k = 1; k <= m.nz; ++k) st.fyb[k] = m.flux_y[k];
}

static void tvd_advection_column(Model& m) {
  int y = m.col_y, x = m.col_x;
  if (m.halo_column) {
    bool keep = (y == 2 && x <= m.xe && x >= m.xs - 1) || (x == 2 && y >= m.ys && y <= m.ye);
    if (!keep) return;
  }
  if (m.cfg.advection_flow_fields == MGPU_ADVECT_TVD) {
    // advect_flow_fields (tvdadvection.F90:603-646): momentum_stepping is always centred
    // (steppingdirection.F90:32), so dt = 2 dtm
    const double dtf = m.dtm * 2.0;
    advect_flow_field(m, 0, dtf, m.u, m.zu, m.su, m.tvd_u);
    advect_flow_field(m, 1, dtf, m.v, m.zv, m.sv, m.tvd_v);
    advect_flow_field(m, 2, dtf, m.w, m.zw, m.sw, m.tvd_w);
  }
  double dt = m.dtm * 2.0;  // scalar_stepping is always CENTRED_STEPPING (steppingdirection.F90:29-33)
  if (m.th.active) advect_scalar_field(m, dt, m.zth, m.th, m.sth, m.tvd_th);
  for (int n = 0; n < m.cfg.number_q_fields; ++n) advect_scalar_field(m, dt, m.zq[n], m.q[n], m.sq[n], m.tvd_q[n]);
}

// ---------------------------------------------------------------------------------------------
// th_advection (thadvection.F90:53-78 initialisation, :129-219 timestep).  The oracle is Boussinesq
// (use_anelastic_equations = .false.): vertical_advection_of_reference_state does nothing there,
// and advection_of_mean_baroclinicity takes its Boussinesq branch (:205-212).  The callback
// touches every column it is given, halo columns included.
// ---------------------------------------------------------------------------------------------
static void th_advection_column(Model& m) {
  const mgpu_config& c = m.cfg;
  if (!c.th_advection_enabled) return;
  // l_advect_mean_baroclinicity (:62-71): only with passive q
  if (!(c.baroclinicity_use_geostrophic_shear && c.passive_q)) return;
  if (!m.th.active) return;
  const double fcoriol_over_G = c.fcoriol / c.G;
  const double multiplicative_factor_x = c.rate_change_geostrophic_wind_x * c.thref0 * fcoriol_over_G;
  const double multiplicative_factor_y = c.rate_change_geostrophic_wind_y * c.thref0 * fcoriol_over_G;
  int y = m.col_y, x = m.col_x;
  for (int k = 2; k <= m.nz; ++k)
    m.sth(k, y, x) = m.sth(k, y, x) + ((m.v(k, y, x) + m.vgal) * multiplicative_factor_x -
                                       (m.u(k, y, x) + m.ugal) * multiplicative_factor_y);
}

// ---------------------------------------------------------------------------------------------
// diffusion (diffusion.F90:376-545)
// ---------------------------------------------------------------------------------------------
static void general_diffusion(Model& m, Field& f, Field& s) {
  int y = m.col_y, x = m.col_x;
  Field& d = m.diff;
  for (int k = 2; k <= m.nz; ++k) {
    double term =
        m.cx2 * 0.25 *
            (((d(k, y, x) + d(k, y, x - 1)) + (d(k - 1, y, x) + d(k - 1, y, x - 1))) * (f(k, y, x - 1) - f(k, y, x)) -
             ((d(k, y, x + 1) + d(k, y, x)) + (d(k - 1, y, x + 1) + d(k - 1, y, x))) * (f(k, y, x) - f(k, y, x + 1))) +
        m.cy2 * 0.25 *
            (((d(k, y, x) + d(k, y - 1, x)) + (d(k - 1, y, x) + d(k - 1, y - 1, x))) * (f(k, y - 1, x) - f(k, y, x)) -
             ((d(k, y + 1, x) + d(k, y, x)) + (d(k - 1, y + 1, x) + d(k - 1, y, x))) * (f(k, y, x) - f(k, y + 1, x))) +
        (m.czb(k) * d(k - 1, y, x) * (f(k - 1, y, x) - f(k, y, x)));
    if (k < m.nz) term = term - m.cza(k) * d(k, y, x) * (f(k, y, x) - f(k + 1, y, x));
    s(k, y, x) = s(k, y, x) + term;
  }
}

static void diffusion_column(Model& m) {
  if (!m.cfg.use_viscosity_and_diffusion || m.halo_column) return;
  if (m.th.active) general_diffusion(m, m.zth, m.sth);
  for (int n = 0; n < m.cfg.number_q_fields; ++n) general_diffusion(m, m.zq[n], m.sq[n]);
}

// ---------------------------------------------------------------------------------------------
// viscosity (viscosity.F90:237-498)
// ---------------------------------------------------------------------------------------------
static void viscosity_column(Model& m) {
  if (!m.cfg.use_viscosity_and_diffusion || m.halo_column) return;
  int y = m.col_y, x = m.col_x;
  bool fwd = m.field_stepping == FORWARD_STEPPING;
  Field& ZU = fwd ? m.u : m.zu;
  Field& ZV = fwd ? m.v : m.zv;
  Field& ZW = fwd ? m.w : m.zw;
  Field& vis = m.vis;
  const int nz = m.nz;
  const double cx = m.cx, cy = m.cy;
  std::vector<double> tau12(nz + 2), tau12_ym1(nz + 2), tau12m1(nz + 2), tau11(nz + 2), tau22(nz + 2), tau22_yp1(nz + 2),
      tau33(nz + 2), tau11p1(nz + 2), tau13(nz + 2), tau13m1(nz + 2), tau23(nz + 2), tau23_ym1(nz + 2);
  for (int k = 1; k <= nz; ++k) {
    if (k > 1) {
      double vistmp = vis(k, y, x) + vis(k, y + 1, x) + vis(k - 1, y, x) + vis(k - 1, y + 1, x);
      double vis12 = 0.125 * (vistmp + vis(k, y, x + 1) + vis(k, y + 1, x + 1) + vis(k - 1, y, x + 1) + vis(k - 1, y + 1, x + 1));
      tau12[k] = (ZU(k, y + 1, x) - ZU(k, y, x)) * cy;
      tau12[k] = tau12[k] + (ZV(k, y, x + 1) - ZV(k, y, x)) * cx;
      tau12[k] = tau12[k] * m.rhon(k) * vis12;
      double vis12a = 0.125 * (vistmp + vis(k, y, x - 1) + vis(k, y + 1, x - 1) + vis(k - 1, y, x - 1) + vis(k - 1, y + 1, x - 1));
      tau12m1[k] = (ZU(k, y + 1, x - 1) - ZU(k, y, x - 1)) * cy;
      tau12m1[k] = tau12m1[k] + (ZV(k, y, x) - ZV(k, y, x - 1)) * cx;
      tau12m1[k] = tau12m1[k] * m.rhon(k) * vis12a;
      vistmp = vis(k, y - 1, x) + vis(k, y, x) + vis(k - 1, y - 1, x) + vis(k - 1, y, x);
      vis12 = 0.125 * (vistmp + vis(k, y - 1, x + 1) + vis(k, y, x + 1) + vis(k - 1, y - 1, x + 1) + vis(k - 1, y, x + 1));
      tau12_ym1[k] = (ZU(k, y, x) - ZU(k, y - 1, x)) * cy;
      tau12_ym1[k] = tau12_ym1[k] + (ZV(k, y - 1, x + 1) - ZV(k, y - 1, x)) * cx;
      tau12_ym1[k] = tau12_ym1[k] * m.rhon(k) * vis12;
      double visonp2 = m.rhon(k) * (vis(k, y, x) + vis(k - 1, y, x));
      tau11[k] = visonp2 * (ZU(k, y, x) - ZU(k, y, x - 1)) * cx;
      tau22[k] = visonp2 * (ZV(k, y, x) - ZV(k, y - 1, x)) * cy;
      tau33[k] = visonp2 * (ZW(k, y, x) - ZW(k - 1, y, x)) * m.rdz(k);
      visonp2 = m.rhon(k) * (vis(k, y + 1, x) + vis(k - 1, y + 1, x));
      tau22_yp1[k] = visonp2 * (ZV(k, y + 1, x) - ZV(k, y, x)) * cy;
      double visonp2a = m.rhon(k) * (vis(k, y, x + 1) + vis(k - 1, y, x + 1));
      // tau11p1 reads current_state%zu at x+1 in both stepping modes (viscosity.F90:438-440)
      tau11p1[k] = visonp2a * (m.zu(k, y, x + 1) - ZU(k, y, x)) * cx;
    } else {
      tau12[k] = tau12_ym1[k] = tau12m1[k] = tau11[k] = tau22[k] = tau22_yp1[k] = tau33[k] = tau11p1[k] = 0.0;
    }
    if (k < nz) {
      double vis13 = 0.5 * (vis(k, y, x) + vis(k, y, x + 1));
      tau13[k] = (ZU(k + 1, y, x) - ZU(k, y, x)) * m.rdzn(k + 1);
      tau13[k] = tau13[k] + (ZW(k, y, x + 1) - ZW(k, y, x)) * cx;
      tau13[k] = tau13[k] * m.rho(k) * vis13;
      vis13 = 0.5 * (vis(k, y, x - 1) + vis(k, y, x));
      tau13m1[k] = (ZU(k + 1, y, x - 1) - ZU(k, y, x - 1)) * m.rdzn(k + 1);
      tau13m1[k] = tau13m1[k] + (ZW(k, y, x) - ZW(k, y, x - 1)) * cx;
      tau13m1[k] = tau13m1[k] * m.rho(k) * vis13;
      double vis23 = 0.5 * (vis(k, y, x) + vis(k, y + 1, x));
      tau23[k] = (ZW(k, y + 1, x) - ZW(k, y, x)) * cy;
      tau23[k] = tau23[k] + (ZV(k + 1, y, x) - ZV(k, y, x)) * m.rdzn(k + 1);
      tau23[k] = tau23[k] * m.rho(k) * vis23;
      vis23 = 0.5 * (vis(k, y - 1, x) + vis(k, y, x));
      tau23_ym1[k] = (ZW(k, y, x) - ZW(k, y - 1, x)) * cy;
      tau23_ym1[k] = tau23_ym1[k] + (ZV(k + 1, y - 1, x) - ZV(k, y - 1, x)) * m.rdzn(k + 1);
      tau23_ym1[k] = tau23_ym1[k] * m.rho(k) * vis23;
    } else {
      tau13[k] = tau13m1[k] = tau23[k] = tau23_ym1[k] = 0.0;
    }
  }
  for (int k = 2; k <= nz; ++k) {
    double uv = ((tau11p1[k] - tau11[k]) * cx + (tau12[k] - tau12_ym1[k]) * cy + (tau13[k] - tau13[k - 1]) * m.rdz(k)) / m.rhon(k);
    m.su(k, y, x) = m.su(k, y, x) + uv;
    double vv = ((tau12[k] - tau12m1[k]) * cx + (tau22_yp1[k] - tau22[k]) * cy + (tau23[k] - tau23[k - 1]) * m.rdz(k)) / m.rhon(k);
    m.sv(k, y, x) = m.sv(k, y, x) + vv;
  }
  for (int k = 2; k <= nz - 1; ++k) {
    double wv = ((tau13[k] - tau13m1[k]) * cx + (tau23[k] - tau23_ym1[k]) * cy + (tau33[k + 1] - tau33[k]) * m.rdzn(k + 1)) / m.rho(k);
    m.sw(k, y, x) = m.sw(k, y, x) + wv;
  }
}

// ---------------------------------------------------------------------------------------------
// coriolis (coriolis.F90:206-262), buoyancy (buoyancy.F90:190-269),
// set_consistent_lowbc (set_consistent_lowbc.F90:41-144)
// ---------------------------------------------------------------------------------------------
static void coriolis_column(Model& m) {
  if (!m.cfg.coriolis_enabled) return;
  int y = m.col_y, x = m.col_x;
  if (m.halo_column) {
    bool keep = (y == 2 && x <= m.xe && x >= m.xs - 1) || (x == 2 && y >= m.ys && y <= m.ye);
    if (!keep) return;
  }
  const double f = m.cfg.fcoriol;
  for (int k = 2; k <= m.nz; ++k) {
    m.su(k, y, x) = m.su(k, y, x) + f * (0.25 * (m.v(k, y, x) + m.v(k, y, x + 1) + m.v(k, y - 1, x) + m.v(k, y - 1, x + 1)) +
                                         m.vgal - m.geostrophic_wind_y(k));
    m.sv(k, y, x) = m.sv(k, y, x) - f * (0.25 * (m.u(k, y, x) + m.u(k, y, x - 1) + m.u(k, y + 1, x) + m.u(k, y + 1, x - 1)) +
                                         m.ugal - m.geostrophic_wind_x(k));
  }
}

static void buoyancy_column(Model& m) {
  int y = m.col_y, x = m.col_x;
  if (!m.cfg.passive_th && m.th.active) {
    for (int k = 2; k <= m.nz - 1; ++k) {
      double wb = (0.5 * m.buoy_co(k)) * (m.th(k, y, x) + m.th(k + 1, y, x));
      m.sw(k, y, x) = m.sw(k, y, x) + wb;
    }
  }
  if (!m.cfg.passive_q && m.cfg.number_q_fields > 0) {
    double G_over_2 = 0.5 * m.G;
    for (int n = 0; n < m.cfg.number_q_fields; ++n)
      for (int k = 2; k <= m.nz - 1; ++k)
        m.sw(k, y, x) = m.sw(k, y, x) + G_over_2 * m.cq[n] * (m.q[n](k, y, x) + m.q[n](k + 1, y, x));
  }
}

static void set_consistent_lowbc_column(Model& m) {
  if (m.halo_column) return;
  int y = m.col_y, x = m.col_x;
  if (m.cfg.use_viscosity_and_diffusion && m.cfg.use_surface_boundary_conditions) {
    m.su(1, y, x) = -m.su(2, y, x);
    m.sv(1, y, x) = -m.sv(2, y, x);
  } else {
    m.su(1, y, x) = m.su(2, y, x);
    m.sv(1, y, x) = m.sv(2, y, x);
  }
  if (m.th.active && m.cfg.use_surface_boundary_conditions) {
    if (m.cfg.type_of_surface_boundary_conditions == PRESCRIBED_SURFACE_FLUXES) m.sth(1, y, x) = m.sth(2, y, x);
    else m.sth(1, y, x) = -m.sth(2, y, x);
  }
  for (int n = 0; n < m.cfg.number_q_fields; ++n) m.sq[n](1, y, x) = m.sq[n](2, y, x);
  if (m.cfg.number_q_fields > 0 && m.cfg.use_surface_boundary_conditions &&
      m.cfg.type_of_surface_boundary_conditions == PRESCRIBED_SURFACE_VALUES)
    m.sq[m.iqv](1, y, x) = -(m.sq[m.iqv](2, y, x));
}

// ---------------------------------------------------------------------------------------------
// simplecloud (simplecloud.F90:262-379) with saturation.F90 qsaturation / dqwsatdt
// ---------------------------------------------------------------------------------------------
static double qsaturation_(double temperature, double pressure) {
  const double tk0c = 273.15, qsa1 = 3.8, qsa2 = -17.2693882, qsa3 = 35.86, qsa4 = 6.109;
  return qsa1 / (pressure * std::exp(qsa2 * (temperature - tk0c) / (temperature - qsa3)) - qsa4);
}
static double dqwsatdt_(double qs, double temperature) {
  const double tk0c = 273.15, qsa1 = 3.8, qsa2 = -17.2693882, qsa3 = 35.86, qsa4 = 6.109;
  return -qsa2 * (tk0c - qsa3) * (1.0 + qsa4 * qs / qsa1) * qs * std::pow(temperature - qsa3, -2.0);
}

static void simplecloud_column(Model& m) {
  if (m.halo_column) return;
  const int y = m.col_y, x = m.col_x, iqv = m.iqv, iql = m.iql;
  const bool fwd = m.field_stepping == FORWARD_STEPPING;
  double dtm = m.dtm * 2.0;
  if (fwd) dtm = m.dtm;
  Field& q_v = fwd ? m.q[iqv] : m.zq[iqv];
  Field& q_l = fwd ? m.q[iql] : m.zq[iql];
  Field& th = fwd ? m.th : m.zth;
  double exner = 0.0, one_over_exner = 0.0;
  for (int k = 2; k <= m.k_cloudmax; ++k) {
    exner = m.rprefrcp(k);
    one_over_exner = m.prefrcp(k);
    const double Pmb = m.prefn(k) / 100.;
    const double qv = q_v(k, y, x) + m.sq[iqv](k, y, x) * dtm;
    const double qc = q_l(k, y, x) + m.sq[iql](k, y, x) * dtm;
    const double TdegK = (th(k, y, x) + m.sth(k, y, x) * dtm + m.thref(k)) * exner;
    const double qs = qsaturation_(TdegK, Pmb);
    if (qv > qs || qc > 0.0) {
      const double dqsdT = dqwsatdt_(qs, TdegK);
      const double qsatfac = 1.0 / (1.0 + m.rlvap_over_cp * dqsdT);
      const double dmass = fmax_(-qc, (qv - qs) * qsatfac) / dtm;
      m.sq[iqv](k, y, x) = m.sq[iqv](k, y, x) - dmass;
      m.sq[iql](k, y, x) = m.sq[iql](k, y, x) + dmass;
      m.sth(k, y, x) = m.sth(k, y, x) + m.rlvap_over_cp * dmass * one_over_exner;
    }
  }
  // above k_cloudmax any cloud evaporates; the branch tests scalar_stepping (always centred) and
  // one_over_exner keeps its value from the last level of the loop above
  for (int k = m.k_cloudmax + 1; k <= m.nz; ++k) {
    const bool sfwd = m.scalar_stepping == FORWARD_STEPPING;
    const double qc = (sfwd ? m.q[iql] : m.zq[iql])(k, y, x) + m.sq[iql](k, y, x) * dtm;
    if (qc > 0.0) {
      const double dmass = -qc / dtm;
      m.sq[iqv](k, y, x) = m.sq[iqv](k, y, x) - dmass;
      m.sq[iql](k, y, x) = m.sq[iql](k, y, x) + dmass;
      m.sth(k, y, x) = m.sth(k, y, x) + m.rlvap_over_cp * dmass * one_over_exner;
    }
  }
}

// ---------------------------------------------------------------------------------------------
// diverr (diverr.F90:44-175) and psrce (pressuresource.F90:61-238)
// ---------------------------------------------------------------------------------------------
static void diverr_column(Model& m) {
  int y = m.col_y, x = m.col_x;
  for (int k = 1; k <= m.nz; ++k) m.p(k, y, x) = 0.0;
  if (m.halo_column) return;
  bool fwd = m.field_stepping == FORWARD_STEPPING;
  double timec = fwd ? 1.0 / m.dtm : 1.0 / (2.0 * m.dtm);
  Field& U = fwd ? m.u : m.zu;
  Field& V = fwd ? m.v : m.zv;
  Field& W = fwd ? m.w : m.zw;
  for (int k = 1; k <= m.nz; ++k) m.p(k, y, x) = 0.0;
  for (int k = 2; k <= m.nz; ++k) {
    double& pp = m.p(k, y, x);
    pp = pp + m.cx * (U(k, y, x) - U(k, y, x - 1));
    pp = pp + m.cy * (V(k, y, x) - V(k, y - 1, x));
    pp = pp + 4.0 * (m.tzc2(k) * W(k, y, x) - m.tzc1(k) * W(k - 1, y, x));
    pp = pp * timec;
  }
  for (int k = 2; k <= m.nz; ++k)
    if (std::fabs(m.p(k, y, x)) > m.local_divmax) m.local_divmax = std::fabs(m.p(k, y, x));
}

static inline double& BUF(std::vector<double>& b, int nzm1, int k1, int idx) { return b[(size_t)(k1 - 1) + (size_t)nzm1 * (idx - 1)]; }

static void psrce_column(Model& m) {
  int y = m.col_y, x = m.col_x;
  int nzm1 = m.nz - 1;
  if (!m.halo_column) {
    bool last_y = y == m.ye, last_x = x == m.xe;
    int corrected_x = x - 2, corrected_y = y - 2;
    for (int k = 2; k <= m.nz; ++k) {
      double& pp = m.p(k, y, x);
      pp = pp + 4.0 * (m.tzc2(k) * m.sw(k, y, x) - m.tzc1(k) * m.sw(k - 1, y, x));
      pp = pp + m.cx * m.su(k, y, x);
      pp = pp + m.cy * m.sv(k, y, x);
      if (x > 3) pp = pp - m.cx * m.su(k, y, x - 1);
      if (last_x) BUF(m.send_x, nzm1, k - 1, corrected_y) = m.cx * m.su(k, y, x);
      if (y > 3 && x > 3) pp = pp - m.cy * m.sv(k, y - 1, x);
      if (last_y) BUF(m.send_y, nzm1, k - 1, corrected_x) = m.cy * m.sv(k, y, x);
    }
  }
  if (m.last_col) { m.recv_x = m.send_x; m.recv_y = m.send_y; }  // send_neighbouring_pressure_data (self)
}

// fftsolver.F90:215-250 complete_psrce_calculation
static void complete_psrce(Model& m) {
  int nzm1 = m.nz - 1;
  for (int j = m.ys; j <= m.ye; ++j)
    for (int k = 2; k <= m.nz; ++k) {
      m.p(k, j, 3) = m.p(k, j, 3) - BUF(m.recv_x, nzm1, k - 1, j - 2);
      if (j > 3) m.p(k, j, 3) = m.p(k, j, 3) - m.cy * m.sv(k, j - 1, 3);
    }
  for (int i = m.xs; i <= m.xe; ++i)
    for (int k = 2; k <= m.nz; ++k) m.p(k, 3, i) = m.p(k, 3, i) - BUF(m.recv_y, nzm1, k - 1, i - 2);
}

// ---------------------------------------------------------------------------------------------
// stepfields (stepfields.F90:231-627)
// ---------------------------------------------------------------------------------------------
static void step_field(Model& m, int x, int y, Field& f, Field& zf, Field& sf, bool flow, double gal, Field* sav) {
  double dtm_x2 = 2.0 * m.dtm;
  double actual_gal = flow ? gal : 0.0;
  sf(1, y, x) = 0.0;
  for (int k = 1; k <= m.nz; ++k) {
    if (sav && m.field_stepping == CENTRED_STEPPING) (*sav)(k, y, x) = zf(k, y, x) + actual_gal;
    if (flow) f(k, y, x) = actual_gal + f(k, y, x);
    if (m.field_stepping == FORWARD_STEPPING) zf(k, y, x) = f(k, y, x) + m.dtm * sf(k, y, x);
    else zf(k, y, x) = actual_gal + zf(k, y, x) + dtm_x2 * sf(k, y, x);
  }
}

static void timesmooth(Model& m, Field& f, Field& zf, int x, int y, double c1, double c2) {
  for (int k = 1; k <= m.nz; ++k) f(k, y, x) = c1 * f(k, y, x) + c2 * zf(k, y, x);
}

static void step_column_in_slice(Model& m, int yl, int xp, int yp, Field& f, Field& zf, Field& sf, bool flow, double gal,
                                 double c1, double c2, bool ts, Field* sav) {
  if (yp >= m.ys) {
    if (ts) timesmooth(m, f, zf, xp, yp, c1, c2);
    step_field(m, xp, yp, f, zf, sf, flow, gal, sav);
  }
  if (yl == m.ye) {
    if (ts) timesmooth(m, f, zf, xp, yl, c1, c2);
    step_field(m, xp, yl, f, zf, sf, flow, gal, sav);
  }
}

static void step_single_field(Model& m, int xl, int yl, int xp, int yp, Field& f, Field& zf, Field& sf, bool flow, double gal,
                              double c1, double c2, bool ts, Field* sav) {
  if (xp >= m.xs) step_column_in_slice(m, yl, xp, yp, f, zf, sf, flow, gal, c1, c2, ts, sav);
  if (xl == m.xe) {
    if (xl > 1) step_column_in_slice(m, yl, xl - 1, yp, f, zf, sf, flow, gal, c1, c2, ts, sav);
    step_column_in_slice(m, yl, xl, yp, f, zf, sf, flow, gal, c1, c2, ts, sav);
  }
}

static void clip_slice(Model& m, int yl, int xp, int yp, Field& f) {
  auto clip = [&](int yy) {
    for (int k = 1; k <= m.nz; ++k)
      if (f(k, yy, xp) < 0.0) f(k, yy, xp) = 0.0;
  };
  if (yp >= m.ys) clip(yp);
  if (yl == m.ye) clip(yl);
}

// stepfields.F90:397-406
static void reset_local_minmax_values(Model& m) {
  m.local_zumin = m.rlargep;
  m.local_zumax = -m.rlargep;
  m.local_zvmin = m.rlargep;
  m.local_zvmax = -m.rlargep;
  m.abswmax.assign(m.nz + 1, -m.rlargep);
}

// stepfields.F90:372-393, before the column is stepped
static void determine_local_flow_minmax(Model& m, int y, int x) {
  for (int k = 2; k <= m.nz; ++k) {
    m.local_zumax = std::max(m.local_zumax, m.zu(k, y, x));
    m.local_zumin = std::min(m.local_zumin, m.zu(k, y, x));
    m.local_zvmax = std::max(m.local_zvmax, m.zv(k, y, x));
    m.local_zvmin = std::min(m.local_zvmin, m.zv(k, y, x));
    if (k < m.nz) m.abswmax[k] = std::max(m.abswmax[k], std::fabs(m.zw(k, y, x)));
  }
}

static void stepfields_column(Model& m) {
  int x = m.col_x, y = m.col_y;
  if (m.cfg.cfl_enabled && m.first_col) {  // stepfields.F90:249-256
    m.determine_flow_minmax = cfl_step(m);
    if (m.determine_flow_minmax) reset_local_minmax_values(m);
  }
  if (!m.halo_column) {
    if (m.cfg.cfl_enabled && m.determine_flow_minmax) determine_local_flow_minmax(m, y, x);
    int xp = x - 2, yp = y - 1;
    double c1 = 1.0 - 2.0 * m.tsmth, c2 = m.tsmth;
    step_single_field(m, x, y, xp, yp, m.u, m.zu, m.su, true, m.ugal, c1, c2, false, &m.savu);
    step_single_field(m, x, y, xp, yp, m.v, m.zv, m.sv, true, m.vgal, c1, c2, false, &m.savv);
    step_single_field(m, x, y, xp, yp, m.w, m.zw, m.sw, false, 0.0, c1, c2, false, &m.savw);
    bool centred = m.field_stepping == CENTRED_STEPPING;
    if (m.th.active) step_single_field(m, x, y, xp, yp, m.th, m.zth, m.sth, false, 0.0, c1, c2, centred, nullptr);
    for (int n = 0; n < m.cfg.number_q_fields; ++n)
      step_single_field(m, x, y, xp, yp, m.q[n], m.zq[n], m.sq[n], false, 0.0, c1, c2, centred, nullptr);
  }
  // remove_negative_rounding_errors_for_single_field (runs for every column)
  for (int n = 0; n < m.cfg.number_q_fields; ++n) {
    int xp = x - 2, yp = y - 1;
    if (xp >= m.xs) clip_slice(m, y, xp, yp, m.zq[n]);
    if (x == m.xe) {
      if (x > 1) clip_slice(m, y, x - 1, yp, m.zq[n]);
      clip_slice(m, y, x, yp, m.zq[n]);
    }
  }
}

// ---------------------------------------------------------------------------------------------
// fftsolver (fftsolver.F90:50-309, pencilfft.F90:126-159 single-rank path)
// ---------------------------------------------------------------------------------------------
static void fft_init(Model& m) {
  fft_plan_init(m.plan_x, m.nx);
  fft_plan_init(m.plan_y, m.ny);
  double PI = 4.0 * std::atan(1.0);
  int fx = m.nx + 2, fy = m.ny + 2;
  m.cos_x.assign(fx + 1, 0.0);
  m.cos_y.assign(fy + 1, 0.0);
  for (int i = 1; i <= fx; ++i)
    m.cos_x[i] = (2.0 / (m.dx * m.dx)) * (std::cos(2.0 * PI * (double)((i - 1) / 2) / (double)m.nx) - 1.0);
  for (int i = 1; i <= fy; ++i)
    m.cos_y[i] = (2.0 / (m.dy * m.dy)) * (std::cos(2.0 * PI * (double)((i - 1) / 2) / (double)m.ny) - 1.0);
  m.pt.assign((size_t)m.nz * fy * fx, 0.0);
}

static void forward_3dfft(Model& m) {
  const int nx = m.nx, ny = m.ny, nz = m.nz, fy = ny + 2, fx = nx + 2;
  std::vector<double> row(std::max(nx, ny)), outc(2 * (std::max(nx, ny) / 2 + 1)), data(2 * std::max(nx, ny) + 2),
      work(2 * std::max(nx, ny) + 2);
  std::vector<double> ry((size_t)nz * fy * nx);  // real_buffer1 values indexed (k, jj, i)
  auto RY = [&](int k, int jj, int i) -> double& { return ry[(size_t)(k - 1) + (size_t)nz * ((size_t)(jj - 1) + (size_t)fy * (i - 1))]; };
  for (int i = 1; i <= nx; ++i)
    for (int k = 1; k <= nz; ++k) {
      for (int j = 1; j <= ny; ++j) row[j - 1] = m.p(k, j + 2, i + 2);
      fftn_r2c(m.plan_y, row.data(), outc.data(), data.data(), work.data());
      for (int mm = 1; mm <= ny / 2 + 1; ++mm) { RY(k, 2 * mm - 1, i) = outc[2 * (mm - 1)]; RY(k, 2 * mm, i) = outc[2 * (mm - 1) + 1]; }
    }
  for (int jj = 1; jj <= fy; ++jj)
    for (int k = 1; k <= nz; ++k) {
      for (int i = 1; i <= nx; ++i) row[i - 1] = RY(k, jj, i);
      fftn_r2c(m.plan_x, row.data(), outc.data(), data.data(), work.data());
      for (int mm = 1; mm <= nx / 2 + 1; ++mm) { PT(m, k, jj, 2 * mm - 1) = outc[2 * (mm - 1)]; PT(m, k, jj, 2 * mm) = outc[2 * (mm - 1) + 1]; }
    }
  (void)fx;
}

static void backward_3dfft(Model& m) {
  const int nx = m.nx, ny = m.ny, nz = m.nz, fy = ny + 2;
  std::vector<double> row(std::max(nx, ny)), inc(2 * (std::max(nx, ny) / 2 + 1)), data(2 * std::max(nx, ny) + 2),
      work(2 * std::max(nx, ny) + 2);
  std::vector<double> ry((size_t)nz * fy * nx);
  auto RY = [&](int k, int jj, int i) -> double& { return ry[(size_t)(k - 1) + (size_t)nz * ((size_t)(jj - 1) + (size_t)fy * (i - 1))]; };
  for (int jj = 1; jj <= fy; ++jj)
    for (int k = 1; k <= nz; ++k) {
      for (int mm = 1; mm <= nx / 2 + 1; ++mm) { inc[2 * (mm - 1)] = PT(m, k, jj, 2 * mm - 1); inc[2 * (mm - 1) + 1] = PT(m, k, jj, 2 * mm); }
      fftn_c2r(m.plan_x, inc.data(), row.data(), data.data(), work.data());
      for (int i = 1; i <= nx; ++i) RY(k, jj, i) = row[i - 1];
    }
  for (int i = 1; i <= nx; ++i)
    for (int k = 1; k <= nz; ++k) {
      for (int mm = 1; mm <= ny / 2 + 1; ++mm) { inc[2 * (mm - 1)] = RY(k, 2 * mm - 1, i); inc[2 * (mm - 1) + 1] = RY(k, 2 * mm, i); }
      fftn_c2r(m.plan_y, inc.data(), row.data(), data.data(), work.data());
      for (int j = 1; j <= ny; ++j) m.p(k, j + 2, i + 2) = row[j - 1];
    }
}

static void tridiagonal_solver(Model& m) {
  const int fx = m.nx + 2, fy = m.ny + 2, nz = m.nz;
  std::vector<double> b(nz + 2), b1(nz + 2), s(nz + 2), s1(nz + 2);
  for (int i = 1; i <= fx; ++i) {
    int j_start = (i < 3) ? 3 : 1;
    for (int j = j_start; j <= fy; ++j) {
      double cij = m.cos_x[i] + m.cos_y[j];
      b[2] = cij - m.cza(2);
      b1[2] = 1.0 / b[2];
      s1[2] = PT(m, 2, j, i);
      for (int k = 3; k <= nz; ++k) {
        b[k] = cij + m.czg(k);
        b1[k] = 1.0 / (b[k] - m.czh(k) * b1[k - 1]);
        s1[k] = PT(m, k, j, i) - m.czb(k) * s1[k - 1] * b1[k - 1];
      }
      PT(m, nz, j, i) = s1[nz] * b1[nz];
      for (int k = nz - 1; k >= 2; --k) PT(m, k, j, i) = (s1[k] - m.cza(k) * PT(m, k + 1, j, i)) * b1[k];
    }
  }
  for (int i = 1; i <= 2; ++i)
    for (int j = 1; j <= 2; ++j) {
      s[2] = PT(m, 2, j, i);
      PT(m, 1, j, i) = 0.0;
      PT(m, 2, j, i) = 0.0;
      for (int k = 3; k <= nz; ++k) {
        s[k] = PT(m, k, j, i);
        PT(m, k, j, i) = (s[k - 1] - m.czg(k - 1) * PT(m, k - 1, j, i) - m.czb(k - 1) * PT(m, k - 2, j, i)) / m.cza(k - 1);
      }
    }
}

static void fftsolver_solve(Model& m) {
  forward_3dfft(m);
  tridiagonal_solver(m);
  backward_3dfft(m);
  periodic_wrap(m, m.p, 1, false);
}

static void fftsolver(Model& m) {
  complete_psrce(m);
  fftsolver_solve(m);
}

// ---------------------------------------------------------------------------------------------
// pstep (pstep.F90:359-447) and swap_smooth (swapsmooth.F90:45-187)
// ---------------------------------------------------------------------------------------------
static void pstep_column(Model& m) {
  int y = m.col_y, x = m.col_x;
  // perform_galilean_transformation (pstep.F90:345-346, 453-469), on every column
  if (m.cfg.galilean_transformation)
    for (int k = 1; k <= m.nz; ++k) {
      m.u(k, y, x) = m.u(k, y, x) - m.ugal;
      m.zu(k, y, x) = m.zu(k, y, x) - m.ugal;
      m.v(k, y, x) = m.v(k, y, x) - m.vgal;
      m.zv(k, y, x) = m.zv(k, y, x) - m.vgal;
    }
  if (m.halo_column) return;
  double dtmtmp = (m.field_stepping == CENTRED_STEPPING) ? m.dtm : 0.5 * m.dtm;
  for (int k = 2; k <= m.nz; ++k) {
    m.zu(k, y, x) = m.zu(k, y, x) + 2.0 * m.cx * dtmtmp * (m.p(k, y, x) - m.p(k, y, x + 1));
    m.zv(k, y, x) = m.zv(k, y, x) + 2.0 * m.cy * dtmtmp * (m.p(k, y, x) - m.p(k, y + 1, x));
    if (k < m.nz) m.zw(k, y, x) = m.zw(k, y, x) + 2.0 * m.rdzn(k + 1) * dtmtmp * (m.p(k, y, x) - m.p(k + 1, y, x));
  }
  if (m.cfg.use_viscosity_and_diffusion && m.cfg.use_surface_boundary_conditions) {
    m.zu(1, y, x) = -m.zu(2, y, x) - 2.0 * m.ugal;
    m.zv(1, y, x) = -m.zv(2, y, x) - 2.0 * m.vgal;
  } else {
    m.zu(1, y, x) = m.zu(2, y, x);
    m.zv(1, y, x) = m.zv(2, y, x);
  }
}

static void swap_smooth_column(Model& m) {
  if (m.halo_column) return;
  int y = m.col_y, x = m.col_x;
  if (m.field_stepping == FORWARD_STEPPING) {
    double c1 = 1.0, c2 = -1.0;
    auto swap = [&](Field& f, Field& zf) {
      for (int k = 1; k <= m.nz; ++k) {
        double ev = f(k, y, x) + zf(k, y, x);
        f(k, y, x) = ev * c1 + f(k, y, x) * c2;
        zf(k, y, x) = ev - f(k, y, x);
      }
    };
    // field order inside the k loop does not matter: each field touches only itself
    swap(m.u, m.zu); swap(m.v, m.zv); swap(m.w, m.zw);
    if (m.th.active) swap(m.th, m.zth);
    for (int n = 0; n < m.cfg.number_q_fields; ++n) swap(m.q[n], m.zq[n]);
  } else {
    double c1 = 1.0 - 2.0 * m.tsmth, c2 = m.tsmth;
    for (int k = 1; k <= m.nz; ++k) {
      double ev = m.u(k, y, x);
      m.u(k, y, x) = m.zu(k, y, x);
      m.zu(k, y, x) = c1 * ev + c2 * (m.u(k, y, x) + m.savu(k, y, x) - m.ugal);
      ev = m.v(k, y, x);
      m.v(k, y, x) = m.zv(k, y, x);
      m.zv(k, y, x) = c1 * ev + c2 * (m.v(k, y, x) + m.savv(k, y, x) - m.vgal);
      ev = m.w(k, y, x);
      m.w(k, y, x) = m.zw(k, y, x);
      m.zw(k, y, x) = c1 * ev + c2 * (m.w(k, y, x) + m.savw(k, y, x));
      if (m.th.active) {
        ev = m.zth(k, y, x);
        m.zth(k, y, x) = m.th(k, y, x) + m.tsmth * ev;
        m.th(k, y, x) = ev;
      }
      for (int n = 0; n < m.cfg.number_q_fields; ++n) {
        ev = m.zq[n](k, y, x);
        m.zq[n](k, y, x) = m.q[n](k, y, x) + m.tsmth * ev;
        m.q[n](k, y, x) = ev;
      }
    }
  }
}

// ---------------------------------------------------------------------------------------------
// Group driver (timestepper.F90:40-122, global_config:77-92)
// ---------------------------------------------------------------------------------------------
typedef void (*ColumnFn)(Model&);

// ---------------------------------------------------------------------------------------------
// damping (damping.F90:124-148 init, :301-409 timestep), mean_profiles (meanprofiles.F90:95-216,
// no immersed boundary), forcing's subsidence (forcing.F90:568-582 init, :918-1166 timestep)
// ---------------------------------------------------------------------------------------------
// interpolation.F90:15-58; the levels above the last node are left at 0 (MONC leaves them unset)
static void piecewise_linear_1d(const double* zvals, const double* vals, int nnodes, const Prof& zgrid, int nlev,
                                Prof& field) {
  std::vector<double> initgd(nnodes + 2), zngd(nnodes + 2);
  double verylow = -1.0e5;
  initgd[1] = vals[0];
  zngd[1] = verylow;
  for (int nn = 2; nn <= nnodes + 1; ++nn) {
    initgd[nn] = vals[nn - 2];
    zngd[nn] = zvals[nn - 2];
  }
  for (int nn = 1; nn <= nnodes; ++nn)
    for (int k = 1; k <= nlev; ++k)
      if (zngd[nn] <= zgrid(k) && zgrid(k) < zngd[nn + 1])
        field(k) = initgd[nn] + (initgd[nn + 1] - initgd[nn]) * (zgrid(k) - zngd[nn]) / (zngd[nn + 1] - zngd[nn]);
  if (zgrid(nlev) == zngd[nnodes + 1]) field(nlev) = initgd[nnodes + 1];
}

static void damping_and_forcing_init(Model& m) {
  const mgpu_config& c = m.cfg;
  const int nz = m.nz;
  m.dmpco.alloc(nz); m.dmpcoz.alloc(nz); m.w_subs.alloc(nz);
  m.olzubar.alloc(nz); m.olzvbar.alloc(nz); m.olzthbar.alloc(nz);
  m.olubar.alloc(nz); m.olvbar.alloc(nz); m.olthbar.alloc(nz);
  m.olzqbar.assign(c.number_q_fields, Prof());
  for (Prof& p : m.olzqbar) p.alloc(nz);
  m.kdmpmin = nz + 1;
  if (c.damping_enabled) {
    for (int k = nz; k >= 1; --k) {
      m.kdmpmin = k;
      if (m.zn(k) >= c.zdmp) m.dmpco(k) = c.dmptim * (std::exp((m.zn(k) - c.zdmp) / c.hdmp) - 1.0);
      if (m.z(k) >= c.zdmp) m.dmpcoz(k) = c.dmptim * (std::exp((m.z(k) - c.zdmp) / c.hdmp) - 1.0);
      if (m.zn(k) < c.zdmp) break;
    }
  }
  if (c.l_subs_pl_theta || c.l_subs_pl_q) {
    piecewise_linear_1d(c.z_subs_pl, c.f_subs_pl, c.n_subs_pl, m.z, nz, m.w_subs);
    if (c.subsidence_input_type == MGPU_SUBS_DIVERGENCE)
      for (int k = 1; k <= nz; ++k) m.w_subs(k) = -1.0 * m.w_subs(k) * m.z(k);
  }
}

static bool mean_profiles_enabled(const Model& m) {
  const mgpu_config& c = m.cfg;
  return c.damping_enabled || c.l_subs_pl_theta || c.l_subs_pl_q || c.profile_diagnostics_enabled;
}

// calculate_mean_profiles: sums of zu, zv, zth, zq over the interior of each level (one rank)
// times rnhpts = 1 / real(nx ny), real() at default (single) precision
static void mean_profiles(Model& m) {
  const double rnhpts = 1.0 / (double)(float)((long long)m.nx * m.ny);
  auto mean = [&](const Field& f, Prof& out) {
    for (int k = 1; k <= m.nz; ++k) {
      double sum = 0.0;
      for (int x = m.xs; x <= m.xe; ++x)
        for (int y = m.ys; y <= m.ye; ++y) sum += f(k, y, x);
      out(k) = sum * rnhpts;
    }
  };
  mean(m.u, m.olubar);
  mean(m.zu, m.olzubar);
  mean(m.v, m.olvbar);
  mean(m.zv, m.olzvbar);
  mean(m.th, m.olthbar);
  mean(m.zth, m.olzthbar);
  for (int n = 0; n < m.cfg.number_q_fields; ++n) mean(m.zq[n], m.olzqbar[n]);
}

// profile_diagnostics (profile_diagnostics.F90:311-636) for PW flow and TVD scalars: the column
// sums over the interior, from the current state and the last mean profiles (what the component
// accumulates in the next step's dynamics group).  out: MGPU_PD_* rows of nz.
static int profile_diagnostics(Model& m, double* out) {
  halo_swapper(m);  // the next step's start group refreshes the halos before the dynamics group
  const int nz = m.nz, nq = m.cfg.number_q_fields;
  const bool moist = !m.cfg.passive_q && nq >= 2;
  const int rows = moist ? MGPU_PD_COUNT : MGPU_PD_VAPOUR;
  const bool has_mean = mean_profiles_enabled(m);
  std::vector<double> tot((size_t)MGPU_PD_COUNT * (nz + 1), 0.0);
  auto T = [&](int r, int k) -> double& { return tot[(size_t)r * (nz + 1) + k]; };
  for (int x = m.xs; x <= m.xe; ++x)
    for (int y = m.ys; y <= m.ye; ++y) {
      for (int k = 1; k <= nz; ++k) {
        T(MGPU_PD_U_WIND, k) = T(MGPU_PD_U_WIND, k) + (m.u(k, y, x) + m.ugal);
        T(MGPU_PD_V_WIND, k) = T(MGPU_PD_V_WIND, k) + (m.v(k, y, x) + m.vgal);
        T(MGPU_PD_WW, k) = T(MGPU_PD_WW, k) + m.w(k, y, x) * m.w(k, y, x);
      }
      for (int k = 2; k <= nz; ++k) {
        const double w = m.w(k, y, x);
        T(MGPU_PD_WWW, k) = T(MGPU_PD_WWW, k) + w * w * w;
        T(MGPU_PD_WWWW, k) = T(MGPU_PD_WWWW, k) + (w * w) * (w * w);
        T(MGPU_PD_W_WIND, k) = T(MGPU_PD_W_WIND, k) + w;
      }
      for (int k = 1; k <= nz - 1; ++k) {
        double up = 0.25 * (m.u(k, y, x) + m.u(k, y, x - 1) + m.u(k + 1, y, x) + m.u(k + 1, y, x - 1)) + m.ugal;
        if (has_mean) up = up - 0.5 * (m.olubar(k) + m.olubar(k + 1));
        T(MGPU_PD_UW, k) = T(MGPU_PD_UW, k) + up * m.w(k, y, x);
        double vp = 0.25 * (m.v(k, y, x) + m.v(k, y - 1, x) + m.v(k + 1, y, x) + m.v(k + 1, y - 1, x)) + m.vgal;
        if (has_mean) vp = vp - 0.5 * (m.olvbar(k) + m.olvbar(k + 1));
        T(MGPU_PD_VW, k) = T(MGPU_PD_VW, k) + vp * m.w(k, y, x);
      }
      for (int k = 1; k <= nz; ++k) {
        T(MGPU_PD_THETA, k) = T(MGPU_PD_THETA, k) + (m.th(k, y, x) + m.thref(k));
        const double d = m.th(k, y, x) - m.olthbar(k);
        T(MGPU_PD_TH2, k) = T(MGPU_PD_TH2, k) + d * d;
      }
      for (int k = 2; k <= nz - 1; ++k)
        T(MGPU_PD_WTHETA_CN, k) = T(MGPU_PD_WTHETA_CN, k) + m.w(k, y, x) * (0.5 * (m.th(k, y, x) + m.th(k + 1, y, x)));
      if (moist) {
        const Field &qv = m.q[m.iqv], &ql = m.q[m.iql];
        for (int k = 1; k <= nz; ++k) {
          T(MGPU_PD_VAPOUR, k) = T(MGPU_PD_VAPOUR, k) + qv(k, y, x);
          T(MGPU_PD_LIQUID, k) = T(MGPU_PD_LIQUID, k) + ql(k, y, x);
          const double exner = m.rprefrcp(k), pmb = m.prefn(k) / 100.;
          const double tk = (m.th(k, y, x) + m.thref(k)) * exner;
          T(MGPU_PD_RH, k) = T(MGPU_PD_RH, k) + qv(k, y, x) / qsaturation_(tk, pmb);
        }
        for (int k = 2; k <= nz - 1; ++k) {
          T(MGPU_PD_WQV_CN, k) = T(MGPU_PD_WQV_CN, k) + 0.5 * (qv(k, y, x) + qv(k + 1, y, x)) * m.w(k, y, x);
          T(MGPU_PD_WQL_CN, k) = T(MGPU_PD_WQL_CN, k) + 0.5 * (ql(k, y, x) + ql(k + 1, y, x)) * m.w(k, y, x);
        }
      }
    }
  for (int r = 0; r < rows; ++r)
    for (int k = 1; k <= nz; ++k) out[(size_t)r * nz + k - 1] = T(r, k);
  return rows;
}

static void damping_column(Model& m) {
  if (!m.cfg.damping_enabled) return;
  if (m.halo_column || m.timestep < 3) return;
  const int y = m.col_y, x = m.col_x;
  for (int k = m.kdmpmin; k <= m.nz; ++k) {
    m.su(k, y, x) = m.su(k, y, x) - m.dmpco(k) * (m.zu(k, y, x) - (m.olzubar(k) - m.ugal));
    m.sv(k, y, x) = m.sv(k, y, x) - m.dmpco(k) * (m.zv(k, y, x) - (m.olzvbar(k) - m.vgal));
    if (!m.cfg.passive_th) m.sth(k, y, x) = m.sth(k, y, x) - m.dmpco(k) * (m.zth(k, y, x) - m.olzthbar(k));
    for (int n = 0; n < m.cfg.number_q_fields; ++n)
      m.sq[n](k, y, x) = m.sq[n](k, y, x) - m.dmpco(k) * (m.zq[n](k, y, x) - m.olzqbar[n](k));
  }
  for (int k = m.kdmpmin; k <= m.nz - 1; ++k) m.sw(k, y, x) = m.sw(k, y, x) - m.dmpcoz(k) * m.zw(k, y, x);
}

static void forcing_column(Model& m) {
  const mgpu_config& c = m.cfg;
  if (!(c.l_subs_pl_theta || c.l_subs_pl_q)) return;
  if (m.halo_column || m.timestep < 3) return;
  const int y = m.col_y, x = m.col_x, nz = m.nz;
  std::vector<double> prof(nz + 2);
  if (c.l_subs_pl_theta) {
    // apply_subsidence_to_flow_fields
    for (int f = 0; f < 2; ++f) {
      const Field& zf = f == 0 ? m.zu : m.zv;
      const Prof& bar = f == 0 ? m.olzubar : m.olzvbar;
      Field& sf = f == 0 ? m.su : m.sv;
      for (int k = 1; k <= nz; ++k) prof[k] = c.subsidence_local_theta ? zf(k, y, x) : bar(k);
      for (int k = 2; k <= nz - 1; ++k) {
        double sub = 2.0 * (m.w_subs(k - 1) * m.tzc1(k) * (prof[k] - prof[k - 1]) +
                            m.w_subs(k) * m.tzc2(k) * (prof[k + 1] - prof[k]));
        sf(k, y, x) = sf(k, y, x) - sub;
      }
      int k = nz;
      double sub = 2.0 * (m.w_subs(k - 1) * m.tzc1(k) * (prof[k] - prof[k - 1]));
      sf(k, y, x) = sf(k, y, x) - sub;
    }
    // apply_subsidence_to_theta
    for (int k = 1; k <= nz; ++k) prof[k] = (c.subsidence_local_theta ? m.zth(k, y, x) : m.olzthbar(k)) + m.thref(k);
    for (int k = 2; k <= nz - 1; ++k) {
      double thsub = m.w_subs(k) * (prof[k + 1] - prof[k]) * m.rdzn(k + 1);
      m.sth(k, y, x) = m.sth(k, y, x) - thsub;
    }
    int k = nz;
    double thsub = m.w_subs(k) * (prof[k] - prof[k - 1]) * m.rdzn(k);
    m.sth(k, y, x) = m.sth(k, y, x) - thsub;
  }
  if (c.l_subs_pl_q)
    for (int n = 0; n < c.number_q_fields; ++n) {
      for (int k = 1; k <= nz; ++k) prof[k] = c.subsidence_local_q ? m.zq[n](k, y, x) : m.olzqbar[n](k);
      for (int k = 2; k <= nz - 1; ++k) {
        double qsub = m.w_subs(k) * (prof[k + 1] - prof[k]) * m.rdzn(k + 1);
        m.sq[n](k, y, x) = m.sq[n](k, y, x) - qsub;
      }
      int k = nz;
      double qsub = m.w_subs(k) * (prof[k] - prof[k - 1]) * m.rdzn(k);
      m.sq[n](k, y, x) = m.sq[n](k, y, x) - qsub;
    }
}

static void column_group(Model& m, const std::vector<ColumnFn>& fns) {
  for (int x = 1; x <= m.nxh; ++x)
    for (int y = 1; y <= m.nyh; ++y) {
      m.col_x = x;
      m.col_y = y;
      m.first_col = (x == 1 && y == 1);
      m.last_col = (x == m.nxh && y == m.nyh);
      m.halo_column = y < m.ys || x < m.xs || y > m.ye || x > m.xe;
      for (ColumnFn f : fns) f(m);
    }
}

void iterative_solver(Model& m);  // defined below
void iterative_solver_solve(Model& m);

// cfltest timestep callback (cfltest.F90:62-128) with update_dtm_based_on_absolute (:135-191) on
// normal steps, single rank (the global reductions of get_global_values, :246-264, are the local
// values)
static void cfltest(Model& m) {
  const mgpu_config& g = m.cfg;
  m.update_dtm = false;
  m.dtm_last = m.dtm;
  if (cfl_step(m)) {
    m.last_cfl_timestep = m.timestep;
    m.cfl_evaluations += 1;
    m.cvel = 0.0;
    m.cvel_x = 0.0;
    m.cvel_y = 0.0;
    m.cvel_z = 0.0;
    // perform_cfl_and_galilean_transformation_calculation (:231-266)
    m.local_zumin = m.local_zumin + m.ugal;
    m.local_zumax = m.local_zumax + m.ugal;
    m.local_zvmin = m.local_zvmin + m.vgal;
    m.local_zvmax = m.local_zvmax + m.vgal;
    m.local_cvel_z = m.cvel_z;
    for (int k = 2; k <= m.nz - 1; ++k) m.local_cvel_z = std::max(m.local_cvel_z, m.abswmax[k] * m.rdzn(k + 1));
    if (g.galilean_transformation) {
      if (!g.fix_ugal) m.ugal = 0.5 * (m.local_zumin + m.local_zumax);
      if (!g.fix_vgal) m.vgal = 0.5 * (m.local_zvmin + m.local_zvmax);
    } else {
      m.ugal = 0.0;
      m.vgal = 0.0;
    }
    m.cvel_z = m.local_cvel_z;
    m.cvel_x = std::max(std::fabs(m.local_zumax - m.ugal), std::fabs(m.local_zumin - m.ugal));
    m.cvel_y = std::max(std::fabs(m.local_zvmax - m.vgal), std::fabs(m.local_zvmin - m.vgal));
    m.cvel = (m.cvel_x * m.cx + m.cvel_y * m.cy + m.cvel_z) * m.dtm;
    m.cvis = m.cvis * (m.dtm * 4);
    m.cvis_last = m.cvis;
    m.cfl_number = m.cvis / g.cfl_cvismax + m.cvel / g.cfl_cvelmax;
    m.absolute_new_dtm = m.dtm;
    if (m.cfl_number > 0.0)
      if (m.cfl_number < (1.0 - g.cfl_tollerance) || m.cfl_number > (1.0 + g.cfl_tollerance))
        m.absolute_new_dtm = m.dtm / m.cfl_number;
  }
  if (m.dtm != m.absolute_new_dtm && (m.dtm != g.cfl_dtmmax || m.absolute_new_dtm < g.cfl_dtmmax)) {
    m.update_dtm = true;
    m.dtm_new = std::min(std::min(m.dtm * (1.0 + g.cfl_rincmax), m.absolute_new_dtm), g.cfl_dtmmax);
    if (m.dtm_new < g.cfl_dtmmin && !g.l_constant_dtm) m.cfl_error = 1;  // MONC stops (LOG_ERROR)
  }
  if (g.l_constant_dtm) {
    m.dtm = g.dtm;
    m.dtm_new = m.dtm;
    m.update_dtm = false;
  }
  m.cvis = 0.0;
}

static void timestep(Model& m) {
  if (m.cfg.cfl_enabled && m.update_dtm) m.dtm = m.dtm_new;  // monc.F90:313
  // start: clearsourceterms, stepping_direction, halo_swapper, setfluxlook (no per-step work)
  clearsourceterms(m);
  stepping_direction(m);
  halo_swapper(m);
  // subgrid
  column_group(m, {lower_bc_column, smagorinsky_column});
  // dynamics
  if (m.cfg.advection_flow_fields == MGPU_ADVECT_TVD)
    for (int c = 0; c < 3; ++c) interpolate_flow(m, c);
  // global_config:88: pw_advection, tvd_advection, th_advection, diffusion, viscosity, coriolis, ...
  if (m.cfg.simplecloud_enabled)
    column_group(m, {pw_advection_column, tvd_advection_column, th_advection_column, diffusion_column,
                     viscosity_column, coriolis_column, buoyancy_column, damping_column, forcing_column,
                     set_consistent_lowbc_column, simplecloud_column, diverr_column, psrce_column, stepfields_column});
  else
    column_group(m, {pw_advection_column, tvd_advection_column, th_advection_column, diffusion_column,
                     viscosity_column, coriolis_column, buoyancy_column, damping_column, forcing_column,
                     set_consistent_lowbc_column, diverr_column, psrce_column, stepfields_column});
  // solver: mean_profiles, then the pressure solve
  if (mean_profiles_enabled(m)) mean_profiles(m);
  if (m.cfg.solver == MGPU_SOLVER_FFT) fftsolver(m);
  else iterative_solver(m);
  if (m.cfg.cfl_enabled) cfltest(m);
  // pressure-terms
  column_group(m, {pstep_column, swap_smooth_column});
  m.timestep += 1;
}

static Field* field_by_id(Model& m, int id) {
  switch (id) {
    case MGPU_U: return &m.u; case MGPU_V: return &m.v; case MGPU_W: return &m.w; case MGPU_TH: return &m.th;
    case MGPU_ZU: return &m.zu; case MGPU_ZV: return &m.zv; case MGPU_ZW: return &m.zw; case MGPU_ZTH: return &m.zth;
    case MGPU_P: return &m.p; case MGPU_SU: return &m.su; case MGPU_SV: return &m.sv; case MGPU_SW: return &m.sw;
    case MGPU_STH: return &m.sth; case MGPU_VIS: return &m.vis; case MGPU_DIFF: return &m.diff;
    case MGPU_SAVU: return &m.savu; case MGPU_SAVV: return &m.savv; case MGPU_SAVW: return &m.savw;
    default: break;
  }
  int nq = m.cfg.number_q_fields;
  if (id >= MGPU_Q0 && id < MGPU_Q0 + nq) return &m.q[id - MGPU_Q0];
  if (id >= MGPU_ZQ0 && id < MGPU_ZQ0 + nq) return &m.zq[id - MGPU_ZQ0];
  if (id >= MGPU_SQ0 && id < MGPU_SQ0 + nq) return &m.sq[id - MGPU_SQ0];
  return nullptr;
}

Prof* profile_by_name(Model& m, const std::string& n) {
  struct { const char* name; Prof* p; } tab[] = {
      {"z", &m.z}, {"zn", &m.zn}, {"dz", &m.dz}, {"dzn", &m.dzn}, {"rdz", &m.rdz}, {"rdzn", &m.rdzn},
      {"rho", &m.rho}, {"rhon", &m.rhon}, {"thref", &m.thref}, {"dthref", &m.dthref}, {"czb", &m.czb},
      {"cza", &m.cza}, {"czg", &m.czg}, {"czh", &m.czh}, {"tzc1", &m.tzc1}, {"tzc2", &m.tzc2}, {"tzd1", &m.tzd1},
      {"tzd2", &m.tzd2}, {"rneutml", &m.rneutml}, {"rneutml_sq", &m.rneutml_sq}, {"buoy_co", &m.buoy_co},
      {"prefn", &m.prefn}, {"prefrcp", &m.prefrcp}, {"rprefrcp", &m.rprefrcp}, {"tref", &m.tref},
      {"qsat", &m.qsat}, {"dqsatdt", &m.dqsatdt}, {"qsatfac", &m.qsatfac}, {"dmpco", &m.dmpco},
      {"dmpcoz", &m.dmpcoz}, {"w_subs", &m.w_subs}, {"olzubar", &m.olzubar}, {"olzvbar", &m.olzvbar},
      {"olzthbar", &m.olzthbar}, {"olubar", &m.olubar}, {"olvbar", &m.olvbar}, {"olthbar", &m.olthbar},
      {"geostrophic_wind_x", &m.geostrophic_wind_x}, {"geostrophic_wind_y", &m.geostrophic_wind_y}};
  for (auto& t : tab)
    if (n == t.name) return t.p;
  return nullptr;
}

void init_iterative(Model& m);  // defined below

static Model* create(const mgpu_config* cfg) {
  Model* mp = new Model();
  Model& m = *mp;
  m.cfg = *cfg;
  m.nx = cfg->nx; m.ny = cfg->ny; m.nz = cfg->nz;
  m.nxh = m.nx + 4; m.nyh = m.ny + 4;
  m.xs = 3; m.xe = m.nx + 2; m.ys = 3; m.ye = m.ny + 2;
  if (m.cfg.rmlmax <= 0.0) m.cfg.rmlmax = (double)0.23f * std::max(cfg->dxx, cfg->dyy);  // simplesetup.F90:234
  m.smallp = (double)1.0e-14f;  // scienceconstants.F90: real(DP) :: smallp=1.0e-14 (single literal)
  m.vk = cfg->von_karman_constant; m.z0 = cfg->z0; m.z0th = cfg->z0th; m.alphah = cfg->alphah;
  m.betam = cfg->betam; m.betah = cfg->betah; m.gammam = cfg->gammam; m.gammah = cfg->gammah; m.pi = cfg->pi;
  m.cp = cfg->cp; m.rlvap = cfg->rlvap; m.r = cfg->r; m.G = cfg->G; m.convective_limit = cfg->convective_limit;
  m.ratio_mol_wts = cfg->ratio_mol_wts; m.rlargep = cfg->rlargep;
  m.rlvap_over_cp = m.rlvap / m.cp;
  m.r_over_cp = m.r / m.cp;
  m.dtm = cfg->dtm;
  m.tsmth = 1e-2;
  // simplesetup.F90:239-245
  if (cfg->galilean_transformation && cfg->fix_ugal) m.ugal = cfg->ugal;
  if (cfg->galilean_transformation && cfg->fix_vgal) m.vgal = cfg->vgal;
  m.dtm_last = m.dtm;
  m.absolute_new_dtm = m.dtm;
  m.dtm_new = m.dtm;
  m.abswmax.assign(cfg->nz + 1, 0.0);
  if (cfg->cfl_enabled) reset_local_minmax_values(m);  // stepfields.F90:99-100 (initialisation)
  build_grid(m);
  int nz = m.nz, nyh = m.nyh, nxh = m.nxh;
  Field* fl[] = {&m.u, &m.v, &m.w, &m.zu, &m.zv, &m.zw, &m.p, &m.su, &m.sv, &m.sw, &m.savu, &m.savv, &m.savw, &m.vis, &m.diff};
  for (Field* f : fl) f->alloc(nz, nyh, nxh);
  if (!cfg->passive_th || true) { m.th.alloc(nz, nyh, nxh); m.zth.alloc(nz, nyh, nxh); m.sth.alloc(nz, nyh, nxh); }
  int nq = cfg->number_q_fields;
  m.q.resize(nq); m.zq.resize(nq); m.sq.resize(nq); m.tvd_q.resize(nq);
  for (int n = 0; n < nq; ++n) { m.q[n].alloc(nz, nyh, nxh); m.zq[n].alloc(nz, nyh, nxh); m.sq[n].alloc(nz, nyh, nxh); m.tvd_q[n].alloc(nz, nyh); }
  m.iqv = 0; m.iql = nq > 1 ? 1 : 0;
  m.cq.assign(std::max(nq, 1), 0.0);
  if (!cfg->passive_q && nq > 0) m.cq[m.iqv] = m.ratio_mol_wts - 1.0;  // setfluxlook.F90:95
  if (cfg->simplecloud_enabled) {
    // simplecloud.F90:230-248: liquid loading, and the highest level below max_height_cloud
    if (nq < 2) throw std::runtime_error("simplecloud needs the vapour and liquid q fields");
    m.cq[m.iql] = -1.0;
    int k = 2;
    for (; k <= nz - 1; ++k)
      if (m.zn(k) > cfg->max_height_cloud) break;
    m.k_cloudmax = k - 1;
  }
  m.tvd_th.alloc(nz, nyh);
  if (cfg->advection_flow_fields == MGPU_ADVECT_TVD) {
    m.tvd_u.alloc(nz, nyh);
    m.tvd_v.alloc(nz, nyh);
    m.tvd_w.alloc(nz, nyh);
    for (auto& row : m.iflow)
      for (Field& f : row) f.alloc(nz, nyh, nxh);
  }
  m.flux_x.assign(nz + 2, 0.0); m.flux_y.assign(nz + 2, 0.0); m.flux_z.assign(nz + 2, 0.0);
  m.send_x.assign((size_t)(nz - 1) * m.ny, 0.0); m.recv_x = m.send_x;
  m.send_y.assign((size_t)(nz - 1) * m.nx, 0.0); m.recv_y = m.send_y;
  // smagorinsky init
  m.eps = 0.01; m.repsh = 0.5 / m.eps;
  m.thcona = m.ratio_mol_wts * cfg->thref0; m.thconb = m.thcona - cfg->thref0; m.thconap1 = m.thcona;
  m.subb = cfg->smag_subb; m.subc = cfg->smag_subc; m.subg = 1.2; m.subh = 0.0; m.subr = 4.0; m.pr_n = 0.7;
  m.suba = 1.0 / m.pr_n; m.ric = 0.25; m.ricinv = 1.0 / m.ric;
  // lower bc init
  m.max_diff_or_visc = 1.7976931348623157e308;  // huge(0.5_DEFAULT_PRECISION)
  // setfluxlook init (prescribed constant fluxes)
  if (cfg->use_surface_boundary_conditions && cfg->type_of_surface_boundary_conditions == PRESCRIBED_SURFACE_FLUXES) {
    m.surface_temperature_flux = cfg->surface_sensible_heat_flux / (m.rho(1) * m.cp);
    m.surface_vapour_flux = cfg->surface_latent_heat_flux / (m.rho(1) * m.rlvap);
    m.fbuoy = 0.;
    if (!cfg->passive_th) m.fbuoy = m.buoy_co(1) * m.surface_temperature_flux;
    if (!cfg->passive_q && nq > 0) m.fbuoy = m.fbuoy + m.cq[m.iqv] * m.surface_vapour_flux * m.G;
    set_look(m);
  }
  damping_and_forcing_init(m);
  if (cfg->solver == MGPU_SOLVER_FFT) fft_init(m);
  else init_iterative(m);
  return mp;
}


// ---------------------------------------------------------------------------------------------
// iterativesolver (iterativesolver.F90:50-124 callbacks, :140-248 bicgstab, :255-321 cg,
// :329-380 precond, :400-493 calc_Ax, :500-553 inner products, :559-602 set_matrix_for_poisson)
// Work arrays are zero-initialised (MONC leaves them uninitialised; only interior values and the
// depth-1 halo refreshed by calc_Ax are ever read).
// ---------------------------------------------------------------------------------------------
void init_iterative(Model& m) {
  int nz = m.nz;
  m.A_n = m.cx * m.cx;
  m.A_s = m.A_n;
  m.A_e = m.cy * m.cy;
  m.A_w = m.A_e;
  double concat_scalars = m.A_n + m.A_s + m.A_e + m.A_w;
  m.A_u.assign(nz + 2, 0.0); m.A_d.assign(nz + 2, 0.0); m.A_p.assign(nz + 2, 0.0);
  m.A_lu_d.assign(nz + 2, 0.0); m.A_lu_u.assign(nz + 2, 0.0); m.A_vol.assign(nz + 2, 0.0);
  bool symm = m.cfg.solver_type == MGPU_ITER_CG;
  for (int k = 2; k <= nz; ++k) {
    double d_sc;
    if (symm) { m.A_vol[k] = m.dz(k); d_sc = 1.0 / m.rhon(k); }
    else { d_sc = m.rdz(k) / m.rhon(k); m.A_vol[k] = 1.0; }
    m.A_u[k] = (k == nz) ? 0.0 : m.rho(k) * m.rdzn(k + 1);
    m.A_d[k] = (k == 2) ? 0.0 : m.rho(k - 1) * m.rdzn(k);
    m.A_p[k] = d_sc * (-(m.A_u[k] + m.A_d[k])) - concat_scalars * m.A_vol[k];
    m.A_u[k] = d_sc * m.A_u[k];
    m.A_d[k] = d_sc * m.A_d[k];
  }
  m.A_lu_d[2] = 1.0 / m.A_p[2];
  m.A_lu_u[2] = m.A_lu_d[2] * m.A_u[2];
  for (int k = 3; k <= nz; ++k) {
    m.A_lu_d[k] = 1.0 / (m.A_p[k] - m.A_d[k] * m.A_lu_u[k - 1]);
    m.A_lu_u[k] = m.A_u[k] * m.A_lu_d[k];
  }
  m.psource.alloc(nz, m.nyh, m.nxh);
  m.prev_p.alloc(nz, m.nyh, m.nxh);
  m.first_run = true;
}

static void calc_Ax(Model& m, Field& x, Field& Ax) {
  periodic_wrap(m, x, 1, false);
  bool symm = m.cfg.solver_type == MGPU_ITER_CG;
  for (int i = 1; i <= m.nxh; ++i)
    for (int j = 1; j <= m.nyh; ++j) Ax(1, j, i) = 0.0;
  // the five interior / edge passes of calc_Ax cover every interior column once; the
  // arithmetic per column does not depend on the pass
  for (int i = m.xs; i <= m.xe; ++i)
    for (int j = m.ys; j <= m.ye; ++j) {
      const int nz = m.nz;
      for (int k = 2; k <= nz; ++k) {
        double h;
        if (symm) h = m.A_vol[k] * (m.A_n * (x(k, j, i + 1) + x(k, j, i - 1)) + m.A_e * (x(k, j + 1, i) + x(k, j - 1, i)));
        else h = m.A_n * (x(k, j, i + 1) + x(k, j, i - 1)) + m.A_e * (x(k, j + 1, i) + x(k, j - 1, i));
        if (k == 2) Ax(k, j, i) = h + m.A_u[k] * x(k + 1, j, i) + m.A_p[k] * x(k, j, i);
        else if (k < nz) Ax(k, j, i) = h + m.A_u[k] * x(k + 1, j, i) + m.A_d[k] * x(k - 1, j, i) + m.A_p[k] * x(k, j, i);
        else Ax(k, j, i) = h + m.A_d[k] * x(k - 1, j, i) + m.A_p[k] * x(k, j, i);
      }
    }
}

static double inner_prod(Model& m, Field& x, Field& y) {
  double local_sum = 0.0;
  for (int i = m.xs; i <= m.xe; ++i)
    for (int j = m.ys; j <= m.ye; ++j)
      for (int k = 2; k <= m.nz; ++k) local_sum = local_sum + x(k, j, i) * y(k, j, i);
  return local_sum;
}

static void precond(Model& m, Field& s, Field& r) {
  // preconditioner_iterations = 0 (global_config:182): one column LU solve
  for (int i = m.xs; i <= m.xe; ++i)
    for (int j = m.ys; j <= m.ye; ++j) {
      s(1, j, i) = 0.0;
      s(2, j, i) = r(2, j, i) * m.A_lu_d[2];
      for (int k = 3; k <= m.nz; ++k) s(k, j, i) = (r(k, j, i) - m.A_d[k] * s(k - 1, j, i)) * m.A_lu_d[k];
      for (int k = m.nz - 1; k >= 2; --k) s(k, j, i) = s(k, j, i) - m.A_lu_u[k] * s(k + 1, j, i);
    }
}

static void bicgstab(Model& m, Field& x, Field& b) {
  const int nz = m.nz;
  Field Ax, r, cr, pp, v, t, s, cs;
  Field* ws[] = {&Ax, &r, &cr, &pp, &v, &t, &s, &cs};
  for (Field* f : ws) f->alloc(nz, m.nyh, m.nxh);
  const double tolerance = m.cfg.tolerance;
  const double TINY = (double)1.0e-16f;
  (void)TINY;
  double sc_err = std::sqrt(inner_prod(m, b, b));
  sc_err = fmax_(sc_err, 0.0001);
  calc_Ax(m, x, Ax);
  for (int i = m.xs; i <= m.xe; ++i)
    for (int j = m.ys; j <= m.ye; ++j)
      for (int k = 2; k <= nz; ++k) { r(k, j, i) = b(k, j, i) - Ax(k, j, i); cr(k, j, i) = r(k, j, i); }
  double my_rho = inner_prod(m, r, r);
  double err = std::sqrt(my_rho) / sc_err;
  double alf = 1.0, omg = 1.0, nrm = 1.0;
  int it_done = 0;
  if (err >= tolerance) {
    for (int it = 1; it <= m.cfg.max_iterations; ++it) {
      it_done = it;
      if (it > 1) my_rho = inner_prod(m, r, cr);
      double bet = (my_rho / nrm) * (alf / omg);
      if (it == 1) {
        precond(m, pp, r);
      } else {
        for (int i = m.xs; i <= m.xe; ++i)
          for (int j = m.ys; j <= m.ye; ++j)
            for (int k = 2; k <= nz; ++k) t(k, j, i) = r(k, j, i) - bet * omg * v(k, j, i);
        precond(m, s, t);
        for (int i = m.xs; i <= m.xe; ++i)
          for (int j = m.ys; j <= m.ye; ++j)
            for (int k = 2; k <= nz; ++k) pp(k, j, i) = s(k, j, i) + bet * pp(k, j, i);
      }
      calc_Ax(m, pp, v);
      nrm = inner_prod(m, cr, v);
      alf = my_rho / nrm;
      for (int i = m.xs; i <= m.xe; ++i)
        for (int j = m.ys; j <= m.ye; ++j)
          for (int k = 2; k <= nz; ++k) s(k, j, i) = r(k, j, i) - alf * v(k, j, i);
      precond(m, cs, s);
      calc_Ax(m, cs, t);
      double tt = 0.0, ts = 0.0, ss = 0.0;
      for (int i = m.xs; i <= m.xe; ++i)
        for (int j = m.ys; j <= m.ye; ++j)
          for (int k = 2; k <= nz; ++k) {
            tt = tt + t(k, j, i) * t(k, j, i);
            ts = ts + t(k, j, i) * s(k, j, i);
            ss = ss + s(k, j, i) * s(k, j, i);
          }
      omg = ts / tt;
      // x = x + alf*pp + omg*cs (interior; halos refreshed below)
      for (int i = m.xs; i <= m.xe; ++i)
        for (int j = m.ys; j <= m.ye; ++j)
          for (int k = 1; k <= nz; ++k) x(k, j, i) = x(k, j, i) + alf * pp(k, j, i) + omg * cs(k, j, i);
      for (int i = m.xs; i <= m.xe; ++i)
        for (int j = m.ys; j <= m.ye; ++j)
          for (int k = 2; k <= nz; ++k) r(k, j, i) = s(k, j, i) - omg * t(k, j, i);
      nrm = my_rho;
      err = std::sqrt(ss - 2 * omg * ts + omg * omg * tt) / sc_err;
      if (err < tolerance) break;
    }
  }
  periodic_wrap(m, x, 1, false);
  m.last_iterations = it_done;
  m.last_residual = err;
}

// cg_solver (iterativesolver.F90:255-321): preconditioned conjugate gradients on the symmetric
// form of the operator (symm_prob: A_vol = dz), right-hand side scaled by A_vol; the loop always
// runs at least one iteration and tests convergence after the update
static void cg_solver(Model& m, Field& x, Field& b) {
  const int nz = m.nz;
  Field Ax, r, z, p;
  Field* ws[] = {&Ax, &r, &z, &p};
  for (Field* f : ws) f->alloc(nz, m.nyh, m.nxh);
  const double tolerance = m.cfg.tolerance;
  for (int i = m.xs; i <= m.xe; ++i)
    for (int j = m.ys; j <= m.ye; ++j) {
      r(1, j, i) = 0.0;
      for (int k = 2; k <= nz; ++k) r(k, j, i) = b(k, j, i) * m.A_vol[k];
    }
  calc_Ax(m, x, Ax);
  double sc_err = std::sqrt(inner_prod(m, r, r));
  sc_err = fmax_(sc_err, 0.0001);
  for (int i = m.xs; i <= m.xe; ++i)
    for (int j = m.ys; j <= m.ye; ++j)
      for (int k = 1; k <= nz; ++k) r(k, j, i) = r(k, j, i) - Ax(k, j, i);
  double err = std::sqrt(inner_prod(m, r, r)) / sc_err;  // init_err
  double rho = 0.0, alf = 0.0;
  int it_done = 0;
  for (int it = 1; it <= m.cfg.max_iterations; ++it) {
    it_done = it;
    if (it == 1) {
      precond(m, p, r);
      rho = inner_prod(m, p, r);
      alf = rho;
    } else {
      precond(m, z, r);
      alf = inner_prod(m, z, r);
      const double bet = alf / rho;
      rho = alf;
      for (int i = m.xs; i <= m.xe; ++i)
        for (int j = m.ys; j <= m.ye; ++j)
          for (int k = 1; k <= nz; ++k) p(k, j, i) = z(k, j, i) + bet * p(k, j, i);
    }
    calc_Ax(m, p, Ax);
    alf = alf / inner_prod(m, p, Ax);
    for (int i = m.xs; i <= m.xe; ++i)
      for (int j = m.ys; j <= m.ye; ++j)
        for (int k = 1; k <= nz; ++k) {
          x(k, j, i) = x(k, j, i) + alf * p(k, j, i);
          r(k, j, i) = r(k, j, i) - alf * Ax(k, j, i);
        }
    err = std::sqrt(inner_prod(m, r, r)) / sc_err;
    if (err < tolerance) break;
  }
  periodic_wrap(m, x, 1, false);
  m.last_iterations = it_done;
  m.last_residual = err;
}

void iterative_solver_solve(Model& m) {
  periodic_wrap(m, m.p, 1, false);
  m.psource.d = m.p.d;
  if (m.first_run) { periodic_wrap(m, m.prev_p, 1, false); m.first_run = false; }
  m.p.d = m.prev_p.d;
  if (m.cfg.solver_type == MGPU_ITER_CG) cg_solver(m, m.p, m.psource);
  else bicgstab(m, m.p, m.psource);
  m.prev_p.d = m.p.d;
}

void iterative_solver(Model& m) {
  complete_psrce(m);
  iterative_solver_solve(m);
}

}  // namespace oracle

using namespace oracle;

extern "C" {

void* orc_create(const mgpu_config* cfg) {
  try { return create(cfg); } catch (std::exception& e) { std::fprintf(stderr, "orc_create: %s\n", e.what()); return nullptr; }
}
void orc_destroy(void* h) { delete (Model*)h; }

// interior values in C order [nz][ny][nx]; halos are filled periodically
int orc_set_field(void* h, int id, const double* src) {
  Model& m = *(Model*)h;
  Field* f = field_by_id(m, id);
  if (!f) return -1;
  for (int k = 1; k <= m.nz; ++k)
    for (int j = 1; j <= m.ny; ++j)
      for (int i = 1; i <= m.nx; ++i) (*f)(k, j + 2, i + 2) = src[(size_t)(k - 1) * m.ny * m.nx + (size_t)(j - 1) * m.nx + (i - 1)];
  periodic_wrap(m, *f, 2, true);
  return 0;
}

int orc_get_field(void* h, int id, double* dst) {
  Model& m = *(Model*)h;
  Field* f = field_by_id(m, id);
  if (!f) return -1;
  for (int k = 1; k <= m.nz; ++k)
    for (int j = 1; j <= m.ny; ++j)
      for (int i = 1; i <= m.nx; ++i) dst[(size_t)(k - 1) * m.ny * m.nx + (size_t)(j - 1) * m.nx + (i - 1)] = (*f)(k, j + 2, i + 2);
  return 0;
}

// MONC layout with halos, z fastest: (nz, ny+4, nx+4)
int orc_get_field_monc(void* h, int id, double* dst) {
  Model& m = *(Model*)h;
  Field* f = field_by_id(m, id);
  if (!f) return -1;
  std::memcpy(dst, f->d.data(), f->d.size() * sizeof(double));
  return 0;
}

int orc_get_profile(void* h, const char* name, double* dst) {
  Model& m = *(Model*)h;
  Prof* p = profile_by_name(m, name);
  if (!p) return -1;
  for (int k = 1; k <= m.nz; ++k) dst[k - 1] = (*p)(k);
  return 0;
}

int orc_step(void* h, int nsteps) {
  Model& m = *(Model*)h;
  try {
    for (int s = 0; s < nsteps; ++s) {
      timestep(m);
      if (m.cfl_error) return MGPU_ERR_CFL;
    }
  } catch (std::exception& e) {
    std::fprintf(stderr, "orc_step: %s\n", e.what());
    return -1;
  }
  return 0;
}

// cfltest state: out[0..8] = dtm of the last step, dtm of the next step, absolute_new_dtm, cvel,
// cvis, cfl_number, cvel_x, cvel_y, cvel_z; iout[0..1] = evaluations, last_cfl_timestep
int orc_cfl_state(void* h, double* out, int* iout) {
  Model& m = *(Model*)h;
  const double next = m.update_dtm ? m.dtm_new : m.dtm;
  const double v[11] = {m.dtm_last, next, m.absolute_new_dtm, m.cvel, m.cvis_last, m.cfl_number,
                        m.cvel_x, m.cvel_y, m.cvel_z, m.ugal, m.vgal};
  for (int q = 0; q < 11; ++q) out[q] = v[q];
  iout[0] = m.cfl_evaluations;
  iout[1] = m.last_cfl_timestep;
  return 0;
}

int orc_set_timestep(void* h, int ts) {
  Model& m = *(Model*)h;
  m.timestep = ts;
  stepping_direction(m);
  return 0;
}

// Run one component's callback in its configured group form (column components over every
// column; entire components once).  Sources are not cleared; the caller controls that.
int orc_component(void* h, int cid) {
  Model& m = *(Model*)h;
  stepping_direction(m);
  try {
    switch (cid) {
      case MGPU_C_CLEARSOURCETERMS: clearsourceterms(m); break;
      case MGPU_C_STEPPING_DIRECTION: stepping_direction(m); break;
      case MGPU_C_HALO_SWAPPER: halo_swapper(m); break;
      case MGPU_C_LOWER_BC: column_group(m, {lower_bc_column}); break;
      case MGPU_C_SMAGORINSKY: column_group(m, {smagorinsky_column}); break;
      case MGPU_C_PW_ADVECTION: column_group(m, {pw_advection_column}); break;
      case MGPU_C_TVD_ADVECTION:
        if (m.cfg.advection_flow_fields == MGPU_ADVECT_TVD)
          for (int c = 0; c < 3; ++c) interpolate_flow(m, c);
        column_group(m, {tvd_advection_column});
        break;
      case MGPU_C_DIFFUSION: column_group(m, {diffusion_column}); break;
      case MGPU_C_VISCOSITY: column_group(m, {viscosity_column}); break;
      case MGPU_C_CORIOLIS: column_group(m, {coriolis_column}); break;
      case MGPU_C_BUOYANCY: column_group(m, {buoyancy_column}); break;
      case MGPU_C_SET_CONSISTENT_LOWBC: column_group(m, {set_consistent_lowbc_column}); break;
      case MGPU_C_SIMPLECLOUD: if (!m.cfg.simplecloud_enabled) return -5; column_group(m, {simplecloud_column}); break;
      case MGPU_C_DIVERR: column_group(m, {diverr_column}); break;
      // psrce with the deferred first-row/column faces the solver callbacks add (fftsolver.F90:215-250)
      case MGPU_C_PSRCE: column_group(m, {psrce_column}); complete_psrce(m); break;
      case MGPU_C_STEPFIELDS: column_group(m, {stepfields_column}); break;
      case MGPU_C_FFTSOLVER: if (m.plan_x.n == 0) return -5; fftsolver_solve(m); break;
      case MGPU_C_ITERATIVESOLVER: if (m.A_u.empty()) return -5; iterative_solver_solve(m); break;
      case MGPU_C_PSTEP: column_group(m, {pstep_column}); break;
      case MGPU_C_SWAP_SMOOTH: column_group(m, {swap_smooth_column}); break;
      case MGPU_C_MEAN_PROFILES: mean_profiles(m); break;
      case MGPU_C_DAMPING: column_group(m, {damping_column}); break;
      case MGPU_C_FORCING: column_group(m, {forcing_column}); break;
      case MGPU_C_TH_ADVECTION: column_group(m, {th_advection_column}); break;
      default: return -5;
    }
  } catch (std::exception& e) {
    std::fprintf(stderr, "orc_component: %s\n", e.what());
    return -1;
  }
  return 0;
}

double orc_divmax(void* h) { return ((Model*)h)->local_divmax; }
int orc_solver_iterations(void* h) { return ((Model*)h)->last_iterations; }
double orc_solver_residual(void* h) { return ((Model*)h)->last_residual; }

// Known-answer helpers for the FFTPACK restatement
int orc_fft_c2c(int n, double* c, int sign) {
  try {
    FftPlan plan;
    fft_plan_init(plan, n);
    std::vector<double> work(2 * n + 2);
    if (sign < 0) zfftf(plan, c, work.data()); else zfftb(plan, c, work.data());
  } catch (...) { return -1; }
  return 0;
}

double orc_lookup_ustr(void* h, double vel) { return look(*(Model*)h, vel); }

int orc_profile_diagnostics(void* h, double* out) { return profile_diagnostics(*(Model*)h, out); }

// olzqbar(:, n) of the mean profiles, levels 1..nz
int orc_mean_q_profile(void* h, int n, double* out) {
  Model& m = *(Model*)h;
  if (n < 0 || n >= (int)m.olzqbar.size()) return -1;
  for (int k = 1; k <= m.nz; ++k) out[k - 1] = m.olzqbar[n](k);
  return 0;
}

}  // extern "C"
