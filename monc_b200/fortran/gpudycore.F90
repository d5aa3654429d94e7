!> GPU dynamical core as a MONC component: the Fortran side of libmoncgpu's C ABI.
!!
!! A MONC maintainer adds this file as components/gpudycore/src/gpudycore.F90 and lists the
!! component like any other, so that the autogenerated registration (components/makefile:27-30)
!! calls gpudycore_get_descriptor, which returns a component_descriptor_type
!! (model_core/src/components/monc_component.F90:62-71) named "gpu_dycore".  Its timestep
!! callback runs one whole timestep (subgrid, dynamics, solver and pressure-terms groups of
!! global_config:77-92) on the GPU through mgpu_step, so it goes in an `entire` group that
!! replaces those four groups.  The prognostic fields stay resident in GPU memory between
!! steps; they are copied back to current_state before checkpoints and diagnostics read them
!! (gpudycore_sync_to_host) and at finalisation.
!!
!! Everything that crosses the boundary is declared with ISO_C_BINDING kinds, in the order of
!! include/monc_gpu.h; tests/test_fortran_binding.py checks the bind(C) mgpu_config and
!! mgpu_reductions types below against the C structs field by field (name, kind, array length,
!! byte offset) so that a field added on one side only fails the test suite.
module gpudycore_mod
  use iso_c_binding
  use monc_component_mod, only : component_descriptor_type
  use state_mod, only : model_state_type
  use datadefn_mod, only : DEFAULT_PRECISION, STRING_LENGTH
  use optionsdatabase_mod, only : options_get_integer, options_get_real, options_get_logical, &
       options_get_string, options_has_key, options_get_array_size
  use logging_mod, only : LOG_ERROR, LOG_WARN, log_log
  implicit none
  private

  integer, parameter :: MGPU_MAX_NZ = 1024, MGPU_MAX_KGD = 16, MGPU_MAX_Q = 8, MGPU_MAX_SUBS_NODES = 32
  integer(c_int), parameter :: MGPU_OK = 0, MGPU_ERR_NOT_CONVERGED = -3, MGPU_ERR_CFL = -7
  integer(c_int32_t), parameter :: MGPU_FP64 = 0, MGPU_FP32_MIXED = 1
  integer(c_int32_t), parameter :: MGPU_SOLVER_FFT = 0, MGPU_SOLVER_ITERATIVE = 1
  integer(c_int32_t), parameter :: MGPU_ITER_BICGSTAB = 0, MGPU_ITER_CG = 1
  integer(c_int32_t), parameter :: MGPU_ADVECT_PW = 0, MGPU_ADVECT_TVD = 1
  integer(c_int32_t), parameter :: MGPU_LAYOUT_XFAST = 0, MGPU_LAYOUT_MONC = 1, MGPU_LAYOUT_DEVICE = 2
  integer(c_int32_t), parameter :: MGPU_U = 0, MGPU_V = 1, MGPU_W = 2, MGPU_TH = 3, MGPU_ZU = 4, &
       MGPU_ZV = 5, MGPU_ZW = 6, MGPU_ZTH = 7, MGPU_P = 8, MGPU_Q0 = 32, MGPU_ZQ0 = 48

  !> mgpu_config of include/monc_gpu.h, field for field
  type, bind(C) :: mgpu_config
    integer(c_int32_t) :: nx, ny, nz
    integer(c_int32_t) :: n_kgd
    integer(c_int32_t) :: kgd(MGPU_MAX_KGD)
    real(c_double)     :: hgd(MGPU_MAX_KGD)
    integer(c_int32_t) :: nsmth
    integer(c_int32_t) :: explicit_z
    real(c_double)     :: dxx, dyy, zztop
    real(c_double)     :: z_levels(MGPU_MAX_NZ)
    real(c_double)     :: thref0, rhobous
    real(c_double)     :: surface_pressure, surface_reference_pressure
    real(c_double)     :: rmlmax
    real(c_double)     :: dtm
    integer(c_int32_t) :: passive_th, passive_q
    integer(c_int32_t) :: number_q_fields
    integer(c_int32_t) :: use_viscosity_and_diffusion
    integer(c_int32_t) :: use_surface_boundary_conditions
    integer(c_int32_t) :: type_of_surface_boundary_conditions
    real(c_double)     :: surface_sensible_heat_flux
    real(c_double)     :: surface_latent_heat_flux
    integer(c_int32_t) :: coriolis_enabled
    real(c_double)     :: fcoriol
    real(c_double)     :: surface_geostrophic_wind_x, surface_geostrophic_wind_y
    real(c_double)     :: smag_subb, smag_subc
    integer(c_int32_t) :: simplecloud_enabled
    real(c_double)     :: max_height_cloud
    integer(c_int32_t) :: solver
    integer(c_int32_t) :: solver_type
    real(c_double)     :: tolerance
    integer(c_int32_t) :: max_iterations
    integer(c_int32_t) :: precision
    integer(c_int32_t) :: reproducible
    real(c_double)     :: von_karman_constant, z0, z0th, alphah, betam, betah, gammam, gammah
    real(c_double)     :: pi, cp, rlvap, r, G, convective_limit, ratio_mol_wts, rlargep
    integer(c_int32_t) :: cfl_enabled
    integer(c_int32_t) :: cfl_frequency
    real(c_double)     :: cfl_tollerance, cfl_cvismax, cfl_cvelmax
    real(c_double)     :: cfl_dtmmax, cfl_dtmmin, cfl_rincmax
    integer(c_int32_t) :: l_constant_dtm
    integer(c_int32_t) :: advection_flow_fields
    integer(c_int32_t) :: adjoint_taped
    integer(c_int32_t) :: damping_enabled
    real(c_double)     :: dmptim, zdmp, hdmp
    integer(c_int32_t) :: l_subs_pl_theta
    integer(c_int32_t) :: l_subs_pl_q
    integer(c_int32_t) :: subsidence_input_type
    integer(c_int32_t) :: subsidence_local_theta
    integer(c_int32_t) :: subsidence_local_q
    integer(c_int32_t) :: n_subs_pl
    real(c_double)     :: z_subs_pl(MGPU_MAX_SUBS_NODES), f_subs_pl(MGPU_MAX_SUBS_NODES)
    integer(c_int32_t) :: profile_diagnostics_enabled
    integer(c_int32_t) :: galilean_transformation
    integer(c_int32_t) :: fix_ugal, fix_vgal
    real(c_double)     :: ugal, vgal
    integer(c_int32_t) :: th_advection_enabled
    integer(c_int32_t) :: baroclinicity_use_geostrophic_shear
    real(c_double)     :: rate_change_geostrophic_wind_x, rate_change_geostrophic_wind_y
    real(c_double)     :: geostrophic_wind_rate_of_change_in_x, geostrophic_wind_rate_of_change_in_y
  end type mgpu_config

  !> mgpu_reductions of include/monc_gpu.h
  type, bind(C) :: mgpu_reductions
    real(c_double)     :: global_divmax
    integer(c_int32_t) :: solver_iterations
    real(c_double)     :: solver_residual
    integer(c_int32_t) :: timestep
    real(c_double)     :: dtm
    real(c_double)     :: dtm_new
    real(c_double)     :: absolute_new_dtm
    real(c_double)     :: cvel, cvis, cfl_number
    real(c_double)     :: cvel_x, cvel_y, cvel_z
    integer(c_int32_t) :: cfl_evaluations
    integer(c_int32_t) :: last_cfl_timestep
    real(c_double)     :: ugal, vgal
  end type mgpu_reductions

  interface
    subroutine mgpu_config_defaults(cfg) bind(C, name="mgpu_config_defaults")
      import :: mgpu_config
      type(mgpu_config), intent(inout) :: cfg
    end subroutine mgpu_config_defaults
    integer(c_int) function mgpu_create(cfg, h) bind(C, name="mgpu_create")
      import :: mgpu_config, c_int, c_ptr
      type(mgpu_config), intent(in) :: cfg
      type(c_ptr), intent(out) :: h
    end function mgpu_create
    integer(c_int) function mgpu_destroy(h) bind(C, name="mgpu_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function mgpu_destroy
    integer(c_int) function mgpu_upload_field(h, id, host, layout) bind(C, name="mgpu_upload_field")
      import :: c_int, c_int32_t, c_ptr, c_double
      type(c_ptr), value :: h
      integer(c_int32_t), value :: id, layout
      real(c_double), intent(in) :: host(*)
    end function mgpu_upload_field
    integer(c_int) function mgpu_download_field(h, id, host, layout) bind(C, name="mgpu_download_field")
      import :: c_int, c_int32_t, c_ptr, c_double
      type(c_ptr), value :: h
      integer(c_int32_t), value :: id, layout
      real(c_double), intent(inout) :: host(*)
    end function mgpu_download_field
    integer(c_int) function mgpu_step(h, nsteps) bind(C, name="mgpu_step")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: h
      integer(c_int32_t), value :: nsteps
    end function mgpu_step
    integer(c_int) function mgpu_component_timestep(h, component_id) bind(C, name="mgpu_component_timestep")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: h
      integer(c_int32_t), value :: component_id
    end function mgpu_component_timestep
    integer(c_int) function mgpu_set_timestep(h, timestep) bind(C, name="mgpu_set_timestep")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: h
      integer(c_int32_t), value :: timestep
    end function mgpu_set_timestep
    integer(c_int) function mgpu_get_reductions(h, out) bind(C, name="mgpu_get_reductions")
      import :: c_int, c_ptr, mgpu_reductions
      type(c_ptr), value :: h
      type(mgpu_reductions), intent(out) :: out
    end function mgpu_get_reductions
    integer(c_int) function mgpu_checkpoint_write(h, path) bind(C, name="mgpu_checkpoint_write")
      import :: c_int, c_ptr, c_char
      type(c_ptr), value :: h
      character(kind=c_char), intent(in) :: path(*)
    end function mgpu_checkpoint_write
    type(c_ptr) function mgpu_last_error(h) bind(C, name="mgpu_last_error")
      import :: c_ptr
      type(c_ptr), value :: h
    end function mgpu_last_error
    integer(c_size_t) function c_strlen(s) bind(C, name="strlen")
      import :: c_ptr, c_size_t
      type(c_ptr), value :: s
    end function c_strlen
  end interface

  type(c_ptr), save :: handle = c_null_ptr
  integer, save :: nq = 0

  public gpudycore_get_descriptor, gpudycore_sync_to_host, mgpu_config, mgpu_reductions
contains

  !> The component descriptor MONC's registry installs
  type(component_descriptor_type) function gpudycore_get_descriptor()
    gpudycore_get_descriptor%name = "gpu_dycore"
    gpudycore_get_descriptor%version = 0.1
    gpudycore_get_descriptor%initialisation => initialisation_callback
    gpudycore_get_descriptor%timestep => timestep_callback
    gpudycore_get_descriptor%finalisation => finalisation_callback
  end function gpudycore_get_descriptor

  !> Builds mgpu_config from the options database (the keys the components it replaces read),
  !! creates the device model and uploads the prognostic fields
  subroutine initialisation_callback(current_state)
    type(model_state_type), target, intent(inout) :: current_state
    type(mgpu_config) :: cfg
    integer :: n

    call mgpu_config_defaults(cfg)
    cfg%nx = int(current_state%global_grid%size(3), c_int32_t)
    cfg%ny = int(current_state%global_grid%size(2), c_int32_t)
    cfg%nz = int(current_state%global_grid%size(1), c_int32_t)
    cfg%dxx = options_get_real(current_state%options_database, "dxx")
    cfg%dyy = options_get_real(current_state%options_database, "dyy")
    cfg%zztop = options_get_real(current_state%options_database, "zztop")
    cfg%n_kgd = int(min(options_get_array_size(current_state%options_database, "kgd"), MGPU_MAX_KGD), c_int32_t)
    do n = 1, cfg%n_kgd
      cfg%kgd(n) = int(options_get_integer(current_state%options_database, "kgd", n), c_int32_t)
      cfg%hgd(n) = options_get_real(current_state%options_database, "hgd", n)
    end do
    cfg%nsmth = int(options_get_integer(current_state%options_database, "nsmth"), c_int32_t)
    cfg%thref0 = options_get_real(current_state%options_database, "thref0")
    cfg%rhobous = options_get_real(current_state%options_database, "rhobous")
    cfg%surface_pressure = options_get_real(current_state%options_database, "surface_pressure")
    cfg%surface_reference_pressure = options_get_real(current_state%options_database, "surface_reference_pressure")
    cfg%rmlmax = options_get_real(current_state%options_database, "rmlmax")
    cfg%dtm = current_state%dtm
    cfg%passive_th = logical_flag(options_get_logical(current_state%options_database, "passive_th"))
    cfg%passive_q = logical_flag(options_get_logical(current_state%options_database, "passive_q"))
    nq = current_state%number_q_fields
    cfg%number_q_fields = int(nq, c_int32_t)
    cfg%use_viscosity_and_diffusion = logical_flag(current_state%use_viscosity_and_diffusion)
    cfg%use_surface_boundary_conditions = logical_flag(current_state%use_surface_boundary_conditions)
    cfg%type_of_surface_boundary_conditions = int(current_state%type_of_surface_boundary_conditions, c_int32_t)
    cfg%surface_sensible_heat_flux = options_get_real(current_state%options_database, "surface_sensible_heat_flux", 1)
    cfg%surface_latent_heat_flux = options_get_real(current_state%options_database, "surface_latent_heat_flux", 1)
    cfg%coriolis_enabled = logical_flag(options_get_logical(current_state%options_database, "coriolis_enabled"))
    cfg%fcoriol = options_get_real(current_state%options_database, "fcoriol")
    cfg%surface_geostrophic_wind_x = options_get_real(current_state%options_database, "surface_geostrophic_wind_x")
    cfg%surface_geostrophic_wind_y = options_get_real(current_state%options_database, "surface_geostrophic_wind_y")
    cfg%smag_subb = options_get_real(current_state%options_database, "smag-subb")
    cfg%smag_subc = options_get_real(current_state%options_database, "smag-subc")
    cfg%simplecloud_enabled = logical_flag(options_get_logical(current_state%options_database, "simplecloud_enabled"))
    cfg%max_height_cloud = options_get_real(current_state%options_database, "max_height_cloud")
    if (options_get_logical(current_state%options_database, "iterativesolver_enabled")) then
      cfg%solver = MGPU_SOLVER_ITERATIVE
      cfg%tolerance = options_get_real(current_state%options_database, "tolerance")
      cfg%max_iterations = int(options_get_integer(current_state%options_database, "max_iterations"), c_int32_t)
      if (options_get_integer(current_state%options_database, "solver_type") == 1) cfg%solver_type = MGPU_ITER_CG
    else
      cfg%solver = MGPU_SOLVER_FFT
    end if
    if (options_has_key(current_state%options_database, "gpu_precision")) then
      if (trim(options_get_string(current_state%options_database, "gpu_precision")) == "fp32_mixed") &
           cfg%precision = MGPU_FP32_MIXED
    end if
    if (trim(options_get_string(current_state%options_database, "advection_flow_fields")) == "tvd") &
         cfg%advection_flow_fields = MGPU_ADVECT_TVD
    cfg%cfl_enabled = logical_flag(options_get_logical(current_state%options_database, "cfltest_enabled"))
    if (cfg%cfl_enabled /= 0) then
      cfg%cfl_frequency = int(options_get_integer(current_state%options_database, "cfl_frequency"), c_int32_t)
      cfg%cfl_tollerance = options_get_real(current_state%options_database, "cfl_tollerance")
      cfg%cfl_cvismax = options_get_real(current_state%options_database, "cfl_cvismax")
      cfg%cfl_cvelmax = options_get_real(current_state%options_database, "cfl_cvelmax")
      cfg%cfl_dtmmax = options_get_real(current_state%options_database, "cfl_dtmmax")
      cfg%cfl_dtmmin = options_get_real(current_state%options_database, "cfl_dtmmin")
      cfg%cfl_rincmax = options_get_real(current_state%options_database, "cfl_rincmax")
    end if
    cfg%damping_enabled = logical_flag(options_get_logical(current_state%options_database, "damping_enabled"))
    if (cfg%damping_enabled /= 0) then
      cfg%dmptim = options_get_real(current_state%options_database, "dmptim")
      cfg%zdmp = options_get_real(current_state%options_database, "zdmp")
      cfg%hdmp = options_get_real(current_state%options_database, "hdmp")
    end if
    cfg%galilean_transformation = logical_flag(options_get_logical(current_state%options_database, &
         "galilean_transformation"))
    cfg%fix_ugal = logical_flag(options_get_logical(current_state%options_database, "fix_ugal"))
    cfg%fix_vgal = logical_flag(options_get_logical(current_state%options_database, "fix_vgal"))
    cfg%ugal = options_get_real(current_state%options_database, "ugal")
    cfg%vgal = options_get_real(current_state%options_database, "vgal")
    cfg%th_advection_enabled = logical_flag(options_get_logical(current_state%options_database, "th_advection_enabled"))
    cfg%baroclinicity_use_geostrophic_shear = logical_flag(options_get_logical(current_state%options_database, &
         "baroclinicity_use_geostrophic_shear"))
    cfg%rate_change_geostrophic_wind_x = options_get_real(current_state%options_database, "rate_change_geostrophic_wind_x")
    cfg%rate_change_geostrophic_wind_y = options_get_real(current_state%options_database, "rate_change_geostrophic_wind_y")
    cfg%geostrophic_wind_rate_of_change_in_x = options_get_real(current_state%options_database, &
         "geostrophic_wind_rate_of_change_in_x")
    cfg%geostrophic_wind_rate_of_change_in_y = options_get_real(current_state%options_database, &
         "geostrophic_wind_rate_of_change_in_y")

    call check(mgpu_create(cfg, handle), "mgpu_create")
    call upload_state(current_state)
  end subroutine initialisation_callback

  !> One whole timestep on the GPU (MONC's forward step first, then centred steps)
  subroutine timestep_callback(current_state)
    type(model_state_type), target, intent(inout) :: current_state
    type(mgpu_reductions) :: red
    integer(c_int) :: rc

    call check(mgpu_set_timestep(handle, int(current_state%timestep, c_int32_t)), "mgpu_set_timestep")
    rc = mgpu_step(handle, 1_c_int32_t)
    if (rc == MGPU_ERR_NOT_CONVERGED) then
      ! iterativesolver.F90:240-242 only warns when the solve stops at max_iterations
      call log_log(LOG_WARN, "gpu_dycore: the iterative solver did not converge")
    else
      call check(rc, "mgpu_step")
    end if
    call check(mgpu_get_reductions(handle, red), "mgpu_get_reductions")
    current_state%global_divmax = red%global_divmax
    current_state%dtm = red%dtm
    current_state%dtm_new = red%dtm_new
    current_state%absolute_new_dtm = red%absolute_new_dtm
    current_state%cvel = red%cvel
    current_state%cvis = red%cvis
    current_state%ugal = red%ugal
    current_state%vgal = red%vgal
  end subroutine timestep_callback

  !> Copies the prognostic fields back and releases the device model
  subroutine finalisation_callback(current_state)
    type(model_state_type), target, intent(inout) :: current_state

    call gpudycore_sync_to_host(current_state)
    call check(mgpu_destroy(handle), "mgpu_destroy")
    handle = c_null_ptr
  end subroutine finalisation_callback

  !> Brings current_state's prognostic fields up to date from the device (before a checkpoint,
  !! a diagnostics sample or any CPU component that reads them)
  subroutine gpudycore_sync_to_host(current_state)
    type(model_state_type), target, intent(inout) :: current_state
    integer :: n

    call download(MGPU_U, current_state%u%data)
    call download(MGPU_V, current_state%v%data)
    call download(MGPU_W, current_state%w%data)
    call download(MGPU_TH, current_state%th%data)
    call download(MGPU_ZU, current_state%zu%data)
    call download(MGPU_ZV, current_state%zv%data)
    call download(MGPU_ZW, current_state%zw%data)
    call download(MGPU_ZTH, current_state%zth%data)
    call download(MGPU_P, current_state%p%data)
    do n = 1, nq
      call download(MGPU_Q0 + int(n - 1, c_int32_t), current_state%q(n)%data)
      call download(MGPU_ZQ0 + int(n - 1, c_int32_t), current_state%zq(n)%data)
    end do
  end subroutine gpudycore_sync_to_host

  subroutine upload_state(current_state)
    type(model_state_type), target, intent(inout) :: current_state
    integer :: n

    call upload(MGPU_U, current_state%u%data)
    call upload(MGPU_V, current_state%v%data)
    call upload(MGPU_W, current_state%w%data)
    call upload(MGPU_TH, current_state%th%data)
    call upload(MGPU_ZU, current_state%zu%data)
    call upload(MGPU_ZV, current_state%zv%data)
    call upload(MGPU_ZW, current_state%zw%data)
    call upload(MGPU_ZTH, current_state%zth%data)
    do n = 1, nq
      call upload(MGPU_Q0 + int(n - 1, c_int32_t), current_state%q(n)%data)
      call upload(MGPU_ZQ0 + int(n - 1, c_int32_t), current_state%zq(n)%data)
    end do
  end subroutine upload_state

  !> MONC's data(nz, ny+4, nx+4) arrays go through MGPU_LAYOUT_MONC without a temporary
  subroutine upload(id, field)
    integer(c_int32_t), intent(in) :: id
    real(kind=DEFAULT_PRECISION), intent(in), target, contiguous :: field(:,:,:)
    call check(mgpu_upload_field(handle, id, field, MGPU_LAYOUT_MONC), "mgpu_upload_field")
  end subroutine upload

  subroutine download(id, field)
    integer(c_int32_t), intent(in) :: id
    real(kind=DEFAULT_PRECISION), intent(inout), target, contiguous :: field(:,:,:)
    call check(mgpu_download_field(handle, id, field, MGPU_LAYOUT_MONC), "mgpu_download_field")
  end subroutine download

  integer(c_int32_t) function logical_flag(l)
    logical, intent(in) :: l
    logical_flag = merge(1_c_int32_t, 0_c_int32_t, l)
  end function logical_flag

  !> Non-zero status: MONC's convention, log_log(LOG_ERROR) (which aborts, logging.F90:53,86),
  !! with the library's message
  subroutine check(rc, what)
    integer(c_int), intent(in) :: rc
    character(len=*), intent(in) :: what
    character(kind=c_char), pointer :: msg(:)
    character(len=STRING_LENGTH) :: text
    type(c_ptr) :: p
    integer :: n, length

    if (rc == MGPU_OK) return
    text = ""
    p = mgpu_last_error(handle)
    if (c_associated(p)) then
      length = int(min(c_strlen(p), int(STRING_LENGTH - 1, c_size_t)))
      call c_f_pointer(p, msg, [length])
      do n = 1, length
        text(n:n) = msg(n)
      end do
    end if
    call log_log(LOG_ERROR, "gpu_dycore: "//what//" failed: "//trim(text))
  end subroutine check
end module gpudycore_mod
