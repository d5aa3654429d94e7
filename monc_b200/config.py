"""Model configuration for the B200 dynamical core.

`MgpuConfig` mirrors `mgpu_config` in include/monc_gpu.h field for field.  Its defaults are
MONC's `global_config` values (global_config:100-372) for the keys the dynamical core reads.

`dry_cbl_config`, `moist_sc_config` ... build the synthetic workloads the benchmarks run
(dry convective boundary layer, moist stratocumulus-like layer, large moist convective layer).
"""
from __future__ import annotations

import ctypes as C

MAX_NZ = 1024
MAX_KGD = 16
MAX_Q = 8

FP64 = 0
FP32_MIXED = 1
ADVECT_PW, ADVECT_TVD = 0, 1
SOLVER_FFT = 0
SOLVER_ITERATIVE = 1
SOLVER_EXTERNAL = 2  # one y-slab of a decomposed domain; the slab driver runs the pressure solve
PHASE_SUBGRID, PHASE_DYNAMICS, PHASE_PSTEP = 0, 1, 2
HALO_STATE, HALO_PRESSURE = 0, 1
HALO_ITER_X, HALO_ITER_PP, HALO_ITER_CS, HALO_ITER_CG, HALO_ITER_X64 = 2, 3, 4, 5, 6
(SLAB_ITER_BEGIN, SLAB_ITER_INIT, SLAB_ITER_DIRECTION, SLAB_ITER_APPLY, SLAB_ITER_HALF_STEP, SLAB_ITER_APPLY2,
 SLAB_ITER_UPDATE, SLAB_ITER_FINISH, SLAB_ITER_END, SLAB_ITER_PRECOND, SLAB_ITER_COMPAT, SLAB_ITER_SHIFT,
 SLAB_ITER_REFINE, SLAB_ITER_INNER, SLAB_ITER_CORRECT, SLAB_ITER_UNCORRECT) = range(16)
ITER_BICGSTAB = 0
ITER_CG = 1
SUBS_DIVERGENCE, SUBS_VELOCITY = 0, 1  # subsidence_input_type (forcing.F90:40-41)
MAX_SUBS_NODES = 32


class MgpuConfig(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("n_kgd", C.c_int32),
        ("kgd", C.c_int32 * MAX_KGD),
        ("hgd", C.c_double * MAX_KGD),
        ("nsmth", C.c_int32),
        ("explicit_z", C.c_int32),
        ("dxx", C.c_double), ("dyy", C.c_double), ("zztop", C.c_double),
        ("z_levels", C.c_double * MAX_NZ),
        ("thref0", C.c_double), ("rhobous", C.c_double),
        ("surface_pressure", C.c_double), ("surface_reference_pressure", C.c_double),
        ("rmlmax", C.c_double),
        ("dtm", C.c_double),
        ("passive_th", C.c_int32), ("passive_q", C.c_int32),
        ("number_q_fields", C.c_int32),
        ("use_viscosity_and_diffusion", C.c_int32),
        ("use_surface_boundary_conditions", C.c_int32),
        ("type_of_surface_boundary_conditions", C.c_int32),
        ("surface_sensible_heat_flux", C.c_double),
        ("surface_latent_heat_flux", C.c_double),
        ("coriolis_enabled", C.c_int32),
        ("fcoriol", C.c_double),
        ("surface_geostrophic_wind_x", C.c_double), ("surface_geostrophic_wind_y", C.c_double),
        ("smag_subb", C.c_double), ("smag_subc", C.c_double),
        ("simplecloud_enabled", C.c_int32),
        ("max_height_cloud", C.c_double),
        ("solver", C.c_int32),
        ("solver_type", C.c_int32),
        ("tolerance", C.c_double),
        ("max_iterations", C.c_int32),
        ("precision", C.c_int32),
        ("reproducible", C.c_int32),
        ("von_karman_constant", C.c_double), ("z0", C.c_double), ("z0th", C.c_double),
        ("alphah", C.c_double), ("betam", C.c_double), ("betah", C.c_double),
        ("gammam", C.c_double), ("gammah", C.c_double),
        ("pi", C.c_double), ("cp", C.c_double), ("rlvap", C.c_double), ("r", C.c_double),
        ("G", C.c_double), ("convective_limit", C.c_double), ("ratio_mol_wts", C.c_double),
        ("rlargep", C.c_double),
        ("cfl_enabled", C.c_int32), ("cfl_frequency", C.c_int32),
        ("cfl_tollerance", C.c_double), ("cfl_cvismax", C.c_double), ("cfl_cvelmax", C.c_double),
        ("cfl_dtmmax", C.c_double), ("cfl_dtmmin", C.c_double), ("cfl_rincmax", C.c_double),
        ("l_constant_dtm", C.c_int32),
        ("advection_flow_fields", C.c_int32),
        ("adjoint_taped", C.c_int32),
        ("damping_enabled", C.c_int32),
        ("dmptim", C.c_double), ("zdmp", C.c_double), ("hdmp", C.c_double),
        ("l_subs_pl_theta", C.c_int32), ("l_subs_pl_q", C.c_int32),
        ("subsidence_input_type", C.c_int32),
        ("subsidence_local_theta", C.c_int32), ("subsidence_local_q", C.c_int32),
        ("n_subs_pl", C.c_int32),
        ("z_subs_pl", C.c_double * MAX_SUBS_NODES), ("f_subs_pl", C.c_double * MAX_SUBS_NODES),
        ("profile_diagnostics_enabled", C.c_int32),
        ("galilean_transformation", C.c_int32), ("fix_ugal", C.c_int32), ("fix_vgal", C.c_int32),
        ("ugal", C.c_double), ("vgal", C.c_double),
        ("th_advection_enabled", C.c_int32), ("baroclinicity_use_geostrophic_shear", C.c_int32),
        ("rate_change_geostrophic_wind_x", C.c_double), ("rate_change_geostrophic_wind_y", C.c_double),
        ("geostrophic_wind_rate_of_change_in_x", C.c_double), ("geostrophic_wind_rate_of_change_in_y", C.c_double),
    ]


def default_config() -> MgpuConfig:
    """A config holding MONC's global_config defaults (same values as mgpu_config_defaults)."""
    c = MgpuConfig()
    c.nx = c.ny = c.nz = 1
    c.n_kgd = 1
    c.kgd[0] = 10
    c.hgd[0] = 10.0
    c.nsmth = 40
    c.explicit_z = 0
    c.dxx = c.dyy = 1.0
    c.zztop = 1.0
    c.thref0 = 288.0
    c.rhobous = 1.0
    c.surface_pressure = 100000.0
    c.surface_reference_pressure = 100000.0
    c.rmlmax = -1.0
    c.dtm = 0.001
    c.passive_th = 1
    c.passive_q = 1
    c.number_q_fields = 0
    c.use_viscosity_and_diffusion = 1
    c.use_surface_boundary_conditions = 0
    c.type_of_surface_boundary_conditions = 0
    c.surface_sensible_heat_flux = 0.0
    c.surface_latent_heat_flux = 0.0
    c.coriolis_enabled = 0
    c.fcoriol = 0.0
    c.surface_geostrophic_wind_x = 0.0
    c.surface_geostrophic_wind_y = 0.0
    c.smag_subb = 40.0
    c.smag_subc = 16.0
    c.simplecloud_enabled = 0
    c.max_height_cloud = 20000.0
    c.solver = SOLVER_FFT
    c.solver_type = ITER_BICGSTAB
    c.tolerance = 1.0e-4
    c.max_iterations = 500
    c.precision = FP64
    c.reproducible = 0
    c.von_karman_constant = 0.4
    c.z0 = 2.0e-3
    c.z0th = 2.0e-4
    c.alphah = 1.0
    c.betam = 4.8
    c.betah = 7.8
    c.gammam = 19.3
    c.gammah = 12.0
    c.pi = 3.14159
    c.cp = 1005.0
    c.rlvap = 2.501e6
    c.r = 287.05
    c.G = 9.81
    c.convective_limit = -0.5
    c.ratio_mol_wts = 1.608
    c.rlargep = 1.0e37
    c.cfl_enabled = 1
    c.cfl_frequency = 10
    c.cfl_tollerance = 0.1
    c.cfl_cvismax = 0.2
    c.cfl_cvelmax = 0.2
    c.cfl_dtmmax = 100.0
    c.cfl_dtmmin = 0.0001
    c.cfl_rincmax = 0.05
    c.l_constant_dtm = 0
    c.advection_flow_fields = ADVECT_PW
    c.damping_enabled = 0
    c.dmptim = c.zdmp = c.hdmp = 0.0
    c.l_subs_pl_theta = c.l_subs_pl_q = 0
    c.subsidence_input_type = SUBS_VELOCITY
    c.subsidence_local_theta = c.subsidence_local_q = 1
    c.n_subs_pl = 0
    c.profile_diagnostics_enabled = 0
    c.galilean_transformation = c.fix_ugal = c.fix_vgal = 0
    c.ugal = c.vgal = 0.0
    return c


def dry_cbl_config(nx: int, ny: int, nz: int, dx: float, dz: float, dtm: float,
                   ug: float = 0.0, fcoriol: float = 0.0, shf_kms: float = 0.1,
                   cs: float = 0.23, thref0: float = 300.0, precision: int = FP64,
                   solver: int = SOLVER_FFT) -> MgpuConfig:
    """Dry convective boundary layer on a uniform vertical grid (dz, nz levels incl. level 1).

    The surface sensible heat flux is given kinematically (K m/s); MONC takes W m-2 and divides
    by rho(1)*cp (setfluxlook.F90:84-85), so the W m-2 value passed is shf_kms*rhobous*cp.
    Cs maps to MONC's rmlmax = Cs*max(dx,dy) (simplesetup.F90:234 uses 0.23 as the default).
    The timestep is fixed (cfltest off), as the benchmark cases run; enable_cfl() turns it on.
    """
    c = default_config()
    c.nx, c.ny, c.nz = nx, ny, nz
    c.dxx = c.dyy = float(dx)
    c.zztop = dz * (nz - 1)
    c.n_kgd = 1
    c.kgd[0] = nz
    c.hgd[0] = c.zztop
    c.nsmth = 40
    c.thref0 = thref0
    c.rmlmax = cs * max(dx, dx)
    c.dtm = dtm
    c.passive_th = 0
    c.passive_q = 1
    c.use_surface_boundary_conditions = 1
    c.type_of_surface_boundary_conditions = 0
    c.surface_sensible_heat_flux = shf_kms * c.rhobous * c.cp
    c.surface_latent_heat_flux = 0.0
    c.z0 = 0.1
    c.z0th = 0.1
    if fcoriol != 0.0:
        c.coriolis_enabled = 1
        c.fcoriol = fcoriol
        c.surface_geostrophic_wind_x = ug
    c.precision = precision
    c.solver = solver
    c.cfl_enabled = 0
    return c


def enable_cfl(c: MgpuConfig, frequency: int = 10, dtmmax: float = 100.0, dtmmin: float = 1e-4,
               rincmax: float = 0.05, tollerance: float = 0.1, cvismax: float = 0.2, cvelmax: float = 0.2,
               constant_dtm: bool = False) -> MgpuConfig:
    """Switch on cfltest with MONC's option names (global_config:137-143 defaults)."""
    c.cfl_enabled = 1
    c.cfl_frequency = frequency
    c.cfl_dtmmax, c.cfl_dtmmin, c.cfl_rincmax = dtmmax, dtmmin, rincmax
    c.cfl_tollerance, c.cfl_cvismax, c.cfl_cvelmax = tollerance, cvismax, cvelmax
    c.l_constant_dtm = 1 if constant_dtm else 0
    return c


def enable_galilean(c: MgpuConfig, ugal: float | None = None, vgal: float | None = None) -> MgpuConfig:
    """Switch on the Galilean transformation (simplesetup.F90:239-245): the frame velocity follows
    the middle of the zu (zv) range at each cfltest evaluation, or stays at a given ugal (vgal),
    MONC's fix_ugal (fix_vgal)."""
    c.galilean_transformation = 1
    c.fix_ugal, c.ugal = (0, 0.0) if ugal is None else (1, ugal)
    c.fix_vgal, c.vgal = (0, 0.0) if vgal is None else (1, vgal)
    return c


def enable_baroclinicity(c: MgpuConfig, rate_x: float, rate_y: float, shear_x: float | None = None,
                         shear_y: float | None = None) -> MgpuConfig:
    """Geostrophic shear and th_advection's advection of the mean baroclinicity, with MONC's keys
    (global_config:52,147-154): baroclinicity_use_geostrophic_shear, th_advection_enabled,
    rate_change_geostrophic_wind_x/_y (th_advection, thadvection.F90:73-78) and
    geostrophic_wind_rate_of_change_in_x/_y (coriolis, coriolis.F90:142-163), which default to the
    same rates.  MONC advects the mean baroclinicity only with passive q."""
    c.th_advection_enabled = 1
    c.baroclinicity_use_geostrophic_shear = 1
    c.rate_change_geostrophic_wind_x, c.rate_change_geostrophic_wind_y = rate_x, rate_y
    c.geostrophic_wind_rate_of_change_in_x = rate_x if shear_x is None else shear_x
    c.geostrophic_wind_rate_of_change_in_y = rate_y if shear_y is None else shear_y
    return c


def enable_damping(c: MgpuConfig, dmptim: float, zdmp: float, hdmp: float) -> MgpuConfig:
    """Switch on the damping layer with MONC's option names (damping.F90:124-148): relaxation at
    rate dmptim (exp((z - zdmp)/hdmp) - 1) above zdmp towards the mean profiles."""
    c.damping_enabled = 1
    c.dmptim, c.zdmp, c.hdmp = dmptim, zdmp, hdmp
    return c


def enable_subsidence(c: MgpuConfig, z_nodes, f_nodes, input_type: int = None, theta: bool = True,
                      q: bool = False, local_theta: bool = False, local_q: bool = False) -> MgpuConfig:
    """Subsidence forcing with MONC's option names (forcing.F90:447-582, global_config:313-317):
    w_subs interpolated from the (z_subs_pl, f_subs_pl) nodes, a velocity or, with
    input_type = SUBS_DIVERGENCE, a divergence (w_subs = -div z); applied to u, v and theta
    (l_subs_pl_theta) and the q fields (l_subs_pl_q), with the column's gradients (local) or those
    of the mean profiles."""
    if len(z_nodes) != len(f_nodes) or not 1 <= len(z_nodes) <= MAX_SUBS_NODES:
        raise ValueError(f"z_subs_pl and f_subs_pl need the same length, 1..{MAX_SUBS_NODES}")
    c.l_subs_pl_theta = 1 if theta else 0
    c.l_subs_pl_q = 1 if q else 0
    c.subsidence_input_type = SUBS_VELOCITY if input_type is None else input_type
    c.subsidence_local_theta = 1 if local_theta else 0
    c.subsidence_local_q = 1 if local_q else 0
    c.n_subs_pl = len(z_nodes)
    for n, (z, f) in enumerate(zip(z_nodes, f_nodes)):
        c.z_subs_pl[n] = z
        c.f_subs_pl[n] = f
    return c


def moist_config(nx: int, ny: int, z, dx: float, dtm: float, shf_wm2: float = 0.0, lhf_wm2: float = 0.0,
                 thref0: float = 289.0, cs: float = 0.23, max_height_cloud: float = 20000.0,
                 n_tracers: int = 0, precision: int = FP64, solver: int = SOLVER_FFT) -> MgpuConfig:
    """Moist layer on explicit w-levels z: q fields vapour (0) and liquid (1), plus n_tracers
    passive q fields, saturation adjustment by simplecloud, moist Richardson number in the
    Smagorinsky closure, surface fluxes in W m-2 (setfluxlook.F90:84-92)."""
    c = dry_cbl_config(nx, ny, len(z), dx, 1.0, dtm, cs=cs, thref0=thref0, precision=precision, solver=solver)
    set_explicit_levels(c, z)
    c.passive_q = 0
    c.number_q_fields = 2 + n_tracers
    c.simplecloud_enabled = 1
    c.max_height_cloud = max_height_cloud
    c.surface_sensible_heat_flux = shf_wm2
    c.surface_latent_heat_flux = lhf_wm2
    return c


def stretched_levels(nz: int, dz_bottom: float, dz_top: float, ztop: float | None = None):
    """w-level heights with spacing growing geometrically from dz_bottom to dz_top.

    When ztop is given the geometric ratio is solved so that the top level lands on ztop.
    """
    import numpy as np

    n = nz - 1
    if ztop is None:
        r = (dz_top / dz_bottom) ** (1.0 / max(n - 1, 1))
        dzs = dz_bottom * r ** np.arange(n)
    else:
        lo, hi = 1.0, 2.0
        for _ in range(200):
            mid = 0.5 * (lo + hi)
            dzs = np.minimum(dz_bottom * mid ** np.arange(n), dz_top)
            if dzs.sum() > ztop:
                hi = mid
            else:
                lo = mid
        dzs = np.minimum(dz_bottom * lo ** np.arange(n), dz_top)
        dzs *= ztop / dzs.sum()
    z = np.concatenate([[0.0], np.cumsum(dzs)])
    return z


def set_explicit_levels(c: MgpuConfig, z) -> None:
    c.explicit_z = 1
    c.nz = len(z)
    c.zztop = float(z[-1])
    for k, zk in enumerate(z):
        c.z_levels[k] = float(zk)


def config_dict(c: MgpuConfig) -> dict:
    out = {}
    for name, _ in MgpuConfig._fields_:
        v = getattr(c, name)
        if hasattr(v, "__len__"):
            continue
        out[name] = v
    return out
