! elmm_gpu.f90 -- Fortran 2008 interface module of libelmm_gpu.so, the
! iso_c_binding mirror of include/elmm_gpu.h for the ELMM host.
!
! The host calls these functions from the shims that keep its own routines'
! signatures: TMarchRK3 (src/tsteps.f90:24), PressureCorrection for the
! initial projection (src/pressure.f90:169, called at src/initial.f90:4290)
! and the PoisSolver module (src/poisson.f90:76-210).  Arrays are passed as
! their first element (U(-2,-2,-2), Pr(-1,-1,-1), RHS(0,0,0)): the library
! reads and writes the reference's full padded arrays.  A host built with
! prec=dp (real64) uses the plain entry points; the default prec=sp build
! (real32, src/make_release:2) uses the *_float ones, which take real32
! arrays in the same layouts.  Every function returns 0 (ELMM_OK) or an
! ELMM_ERR_* code; elmm_last_error() points to the message (a C string).
module elmm_gpu
  use iso_c_binding
  implicit none

  integer(c_int32_t), parameter :: ELMM_ABI_VERSION = 5

  integer(c_int), parameter :: ELMM_OK = 0, ELMM_ERR_INVALID_CONFIG = 1, ELMM_ERR_OOM = 2, &
                               ELMM_ERR_NAN = 3, ELMM_ERR_CUDA = 4, ELMM_ERR_TIMEOUT = 5, &
                               ELMM_ERR_INVALID_ARG = 6, ELMM_ERR_ADMISSION = 7

  ! BC codes: the values of src/parameters.f90:249-250
  integer(c_int32_t), parameter :: ELMM_BC_NOSLIP = 1, ELMM_BC_FREESLIP = 2, ELMM_BC_PERIODIC = 3, &
                                   ELMM_BC_DIRICHLET = 4, ELMM_BC_NEUMANN = 5, ELMM_BC_CONSTFLUX = 6

  integer(c_int32_t), parameter :: ELMM_PREC_FP64 = 0, ELMM_PREC_MIXED = 1

  integer(c_int32_t), parameter :: ELMM_FIELD_U = 0, ELMM_FIELD_V = 1, ELMM_FIELD_W = 2, ELMM_FIELD_PR = 3, &
                                   ELMM_FIELD_VISCOSITY = 4, ELMM_FIELD_U2 = 5, ELMM_FIELD_V2 = 6, &
                                   ELMM_FIELD_W2 = 7, ELMM_FIELD_USTAR = 8, ELMM_FIELD_VSTAR = 9, &
                                   ELMM_FIELD_WSTAR = 10, ELMM_FIELD_PHI = 11, ELMM_FIELD_TEMPERATURE = 12, &
                                   ELMM_FIELD_TDIFF = 13, ELMM_FIELD_TEMPERATURE_ADV = 14, &
                                   ELMM_FIELD_SCALAR = 16, ELMM_FIELD_SCALAR_ADV = 20

  type, bind(C) :: elmm_point_source        ! ScalarPointSource (src/pointsources.f90:8-13)
    integer(c_int32_t) :: scalar_number, reserved
    real(c_double)     :: position(3), flux
  end type

  type, bind(C) :: elmm_puff                ! PuffSource (src/puffs.f90:15-21)
    real(c_double)     :: start_time, end_time, period, duration
    integer(c_int32_t) :: clear, reserved
  end type

  type, bind(C) :: elmm_puff_volume         ! a ScalarFlVolume of a puff
    integer(c_int32_t) :: puff, scalar_number, xi, yj, zk, reserved   ! puff: 0-based
    real(c_double)     :: flux
  end type

  type, bind(C) :: elmm_ib_point            ! TIBPoint (src/immersedboundary.f90:552-564)
    integer(c_int32_t) :: xi, yj, zk, interp
    integer(c_int32_t) :: ii(6), jj(6), kk(6)
    real(c_double)     :: coef(6)
  end type

  type, bind(C) :: elmm_wm_point            ! WMPointUVW at a solid face
    integer(c_int32_t) :: component, direction, xi, yj, zk, reserved
    real(c_double)     :: dist(3), z0, temperature_flux
  end type

  type, bind(C) :: elmm_solids
    integer(c_int64_t) :: n_ib(3)
    type(c_ptr)        :: ib(3)              ! UIBPoints, VIBPoints, WIBPoints
    integer(c_int64_t) :: n_null(3)
    type(c_ptr)        :: null_ijk(3)        ! Unull(3,:), Vnull, Wnull
    integer(c_int64_t) :: n_scalfl
    type(c_ptr)        :: scalfl             ! ScalFlIBPoints
    integer(c_int64_t) :: n_wm
    type(c_ptr)        :: wm                 ! solid-face WMPointUVW
    integer(c_int64_t) :: n_bottom_skip(3)
    type(c_ptr)        :: bottom_skip_ij(3)
    integer(c_int64_t) :: n_solid_pr
    type(c_ptr)        :: solid_pr_ijk       ! Prtype > 0 cells (passive scalars)
    integer(c_int64_t) :: n_wm_pr
    type(c_ptr)        :: wm_pr_ijk          ! Pr wall-model points of the scalars
    integer(c_int64_t) :: n_heat_pr
    type(c_ptr)        :: heat_pr_ijk        ! heated Pr wall-model points at solid faces
    type(c_ptr)        :: heat_pr_q          ! their temperature_flux x area_factor
    integer(c_int64_t) :: n_wall_pr
    type(c_ptr)        :: wall_pr_ijk        ! wall points kept beside the bodies
  end type

  type, bind(C) :: elmm_config
    integer(c_int32_t) :: abi_version
    integer(c_int32_t) :: Prnx, Prny, Prnz
    integer(c_int32_t) :: Btype(6)
    real(c_double)     :: xmin, ymin, zmin
    real(c_double)     :: dxmin, dymin, dzmin
    type(c_ptr)        :: zW                 ! c_null_ptr: uniform z; else c_loc(zW(0)), zW(0:Prnz) real64
    real(c_double)     :: dt
    real(c_double)     :: molecular_viscosity
    real(c_double)     :: C_Smagorinsky
    real(c_double)     :: filter_ratio
    integer(c_int32_t) :: sgstype
    integer(c_int32_t) :: wallmodeltype
    real(c_double)     :: z0(6)
    integer(c_int32_t) :: enable_pr_gradient_x_uniform, enable_pr_gradient_y_uniform
    real(c_double)     :: pr_gradient_x, pr_gradient_y
    integer(c_int32_t) :: precision
    integer(c_int32_t) :: max_refine_sweeps
    real(c_double)     :: refine_tol
    integer(c_int32_t) :: enable_CFL_check
    integer(c_int32_t) :: device
    integer(c_int32_t) :: enable_buoyancy    ! potential temperature + buoyancy
    integer(c_int32_t) :: TempBtype(6)       ! periodic / ELMM_BC_CONSTFLUX with sideTemp = 0
    real(c_double)     :: sideTemp(6)
    real(c_double)     :: temperature_ref, grav_acc, molecular_diffusivity
    integer(c_int32_t) :: num_scalars        ! passive scalars, 0..4
    integer(c_int32_t) :: ScalBtype(6)       ! as TempBtype
    real(c_double)     :: sideScal(6)
    integer(c_int32_t) :: num_point_sources, reserved0
    type(elmm_point_source) :: point_sources(8)
    integer(c_int32_t) :: avg_slice_k, avg_slice_j   ! time-averaged slices of each scalar
    real(c_double)     :: avg_weight                 ! dt / (timeavg2 - timeavg1)
    integer(c_int32_t) :: variable_time_steps, reserved1   ! TimeStepLength's variable branch
    real(c_double)     :: CFL, dt_max, end_time
  end type

  type, bind(C) :: elmm_stats
    integer(c_int32_t) :: steps_done, nan_detected
    real(c_double)     :: time, dt, cfl, max_div
    integer(c_int32_t) :: refine_sweeps, kernels
    real(c_double)     :: elapsed_ms
  end type

  interface
    type(c_ptr) function elmm_version() bind(C)
      import
    end function
    type(c_ptr) function elmm_last_error() bind(C)
      import
    end function
    integer(c_int) function elmm_config_defaults(cfg, nx, ny, nz) bind(C)
      import
      type(elmm_config) :: cfg
      integer(c_int32_t), value :: nx, ny, nz
    end function
    integer(c_int) function elmm_create(cfg, h) bind(C)
      import
      type(elmm_config), intent(in) :: cfg
      type(c_ptr) :: h
    end function
    integer(c_int) function elmm_destroy(h) bind(C)
      import
      type(c_ptr), value :: h
    end function

    ! ---- state transfers, real64 host arrays (prec=dp)
    integer(c_int) function elmm_upload_state(h, U, V, W, Pr) bind(C)
      import
      type(c_ptr), value :: h
      real(c_double), intent(in) :: U(*), V(*), W(*), Pr(*)
    end function
    integer(c_int) function elmm_download_state(h, U, V, W, Pr) bind(C)
      import
      type(c_ptr), value :: h
      real(c_double) :: U(*), V(*), W(*), Pr(*)
    end function
    integer(c_int) function elmm_download_field(h, field, a) bind(C)
      import
      type(c_ptr), value :: h
      integer(c_int32_t), value :: field
      real(c_double) :: a(*)
    end function
    integer(c_int) function elmm_upload_temperature(h, T) bind(C)
      import
      type(c_ptr), value :: h
      real(c_double), intent(in) :: T(*)      ! Temperature(-2:Prnx+3,-2:Prny+3,-2:Prnz+3)
    end function
    integer(c_int) function elmm_upload_scalar(h, sc, S) bind(C)
      import
      type(c_ptr), value :: h
      integer(c_int32_t), value :: sc
      real(c_double), intent(in) :: S(*)      ! Scalar(-2:Prnx+3,-2:Prny+3,-2:Prnz+3,sc)
    end function
    integer(c_int) function elmm_march_host(h, U, V, W, Pr, T, nsteps, st) bind(C)
      import
      type(c_ptr), value :: h
      real(c_double) :: U(*), V(*), W(*), Pr(*)
      type(c_ptr), value :: T                 ! c_loc(Temperature(-2,-2,-2)), or c_null_ptr
      integer(c_int32_t), value :: nsteps
      type(elmm_stats) :: st
    end function

    ! ---- state transfers, real32 host arrays (the default prec=sp build)
    integer(c_int) function elmm_upload_state_float(h, U, V, W, Pr) bind(C)
      import
      type(c_ptr), value :: h
      real(c_float), intent(in) :: U(*), V(*), W(*), Pr(*)
    end function
    integer(c_int) function elmm_download_state_float(h, U, V, W, Pr) bind(C)
      import
      type(c_ptr), value :: h
      real(c_float) :: U(*), V(*), W(*), Pr(*)
    end function
    integer(c_int) function elmm_download_field_float(h, field, a) bind(C)
      import
      type(c_ptr), value :: h
      integer(c_int32_t), value :: field
      real(c_float) :: a(*)
    end function
    integer(c_int) function elmm_upload_temperature_float(h, T) bind(C)
      import
      type(c_ptr), value :: h
      real(c_float), intent(in) :: T(*)
    end function
    integer(c_int) function elmm_upload_scalar_float(h, sc, S) bind(C)
      import
      type(c_ptr), value :: h
      integer(c_int32_t), value :: sc
      real(c_float), intent(in) :: S(*)
    end function
    integer(c_int) function elmm_march_host_float(h, U, V, W, Pr, T, nsteps, st) bind(C)
      import
      type(c_ptr), value :: h
      real(c_float) :: U(*), V(*), W(*), Pr(*)
      type(c_ptr), value :: T                 ! c_loc(Temperature(-2,-2,-2)), or c_null_ptr
      integer(c_int32_t), value :: nsteps
      type(elmm_stats) :: st
    end function

    ! ---- scalars, sources, solid bodies, frames
    integer(c_int) function elmm_download_scalar_slices(h, sc, xy, xz) bind(C)
      import
      type(c_ptr), value :: h
      integer(c_int32_t), value :: sc
      real(c_double) :: xy(*), xz(*)          ! (1:Prnx,1:Prny) and (1:Prnx,1:Prnz)
    end function
    integer(c_int) function elmm_reset_scalar_averages(h) bind(C)
      import
      type(c_ptr), value :: h
    end function
    integer(c_int) function elmm_set_puffs(h, puffs, npuffs, vols, nvols) bind(C)
      import
      type(c_ptr), value :: h
      type(elmm_puff), intent(in) :: puffs(*)
      integer(c_int32_t), value :: npuffs
      type(elmm_puff_volume), intent(in) :: vols(*)
      integer(c_int32_t), value :: nvols
    end function
    integer(c_int) function elmm_set_solids(h, s) bind(C)
      import
      type(c_ptr), value :: h
      type(elmm_solids), intent(in) :: s
    end function
    integer(c_int) function elmm_frame_begin(h) bind(C)
      import
      type(c_ptr), value :: h
    end function
    integer(c_int) function elmm_frame_wait(h, U, V, W, Pr) bind(C)
      import
      type(c_ptr), value :: h
      real(c_double) :: U(*), V(*), W(*), Pr(*)
    end function

    ! ---- the time step and the projection
    integer(c_int) function elmm_project(h, coef, st) bind(C)
      import
      type(c_ptr), value :: h
      real(c_double), value :: coef
      type(elmm_stats) :: st
    end function
    integer(c_int) function elmm_step(h, nsteps, st) bind(C)
      import
      type(c_ptr), value :: h
      integer(c_int32_t), value :: nsteps
      type(elmm_stats) :: st
    end function
    integer(c_int) function elmm_run_stage(h, stage, stop) bind(C)
      import
      type(c_ptr), value :: h
      integer(c_int32_t), value :: stage, stop
    end function

    ! ---- PoisSolver (src/poisson.f90:76-210); one handle serves the uniform and
    !      the nonuniform-z execute / finalize
    integer(c_int) function elmm_poisson_solver_new(s, n, L, bcs, prec, dev) bind(C)
      import
      type(c_ptr) :: s
      integer(c_int32_t), intent(in) :: n(3), bcs(6)
      real(c_double), intent(in) :: L(3)
      integer(c_int32_t), value :: prec, dev
    end function
    integer(c_int) function elmm_poisson_solver_nonuniform_z_new(s, n, Lxy, zPr, zW, bcs, prec, dev) bind(C)
      import
      type(c_ptr) :: s
      integer(c_int32_t), intent(in) :: n(3), bcs(6)
      real(c_double), intent(in) :: Lxy(2), zPr(*), zW(*)
      integer(c_int32_t), value :: prec, dev
    end function
    integer(c_int) function elmm_poisson_solver_execute(s, Phi, RHS) bind(C)
      import
      type(c_ptr), value :: s
      real(c_double) :: Phi(*)
      real(c_double), intent(in) :: RHS(*)
    end function
    integer(c_int) function elmm_poisson_solver_finalize(s) bind(C)
      import
      type(c_ptr), value :: s
    end function
    integer(c_int) function elmm_poisson_solver_new_float(s, n, L, bcs, prec, dev) bind(C)
      import
      type(c_ptr) :: s
      integer(c_int32_t), intent(in) :: n(3), bcs(6)
      real(c_float), intent(in) :: L(3)
      integer(c_int32_t), value :: prec, dev
    end function
    integer(c_int) function elmm_poisson_solver_nonuniform_z_new_float(s, n, Lxy, zPr, zW, bcs, prec, dev) bind(C)
      import
      type(c_ptr) :: s
      integer(c_int32_t), intent(in) :: n(3), bcs(6)
      real(c_float), intent(in) :: Lxy(2), zPr(*), zW(*)
      integer(c_int32_t), value :: prec, dev
    end function
    integer(c_int) function elmm_poisson_solver_execute_float(s, Phi, RHS) bind(C)
      import
      type(c_ptr), value :: s
      real(c_float) :: Phi(*)
      real(c_float), intent(in) :: RHS(*)
    end function
    integer(c_int) function elmm_poisson_solver_finalize_float(s) bind(C)
      import
      type(c_ptr), value :: s
    end function
    ! one domain split into z-slabs over several GPUs (the host arrays are
    ! the whole domain's); devices and nz_slab may be c_null_ptr
    integer(c_int) function elmm_slabs_create(cfg, nslabs, devices, nz_slab, h) bind(C)
      import
      type(elmm_config), intent(in) :: cfg
      integer(c_int32_t), value :: nslabs
      type(c_ptr), value :: devices, nz_slab
      type(c_ptr) :: h
    end function
    integer(c_int) function elmm_slabs_destroy(h) bind(C)
      import
      type(c_ptr), value :: h
    end function
    integer(c_int) function elmm_slabs_upload_state(h, U, V, W, Pr) bind(C)
      import
      type(c_ptr), value :: h
      real(c_double), intent(in) :: U(*), V(*), W(*), Pr(*)
    end function
    integer(c_int) function elmm_slabs_download_state(h, U, V, W, Pr) bind(C)
      import
      type(c_ptr), value :: h
      real(c_double) :: U(*), V(*), W(*), Pr(*)
    end function
    integer(c_int) function elmm_slabs_upload_temperature(h, T) bind(C)
      import
      type(c_ptr), value :: h
      real(c_double), intent(in) :: T(*)
    end function
    integer(c_int) function elmm_slabs_upload_scalar(h, sc, S) bind(C)
      import
      type(c_ptr), value :: h
      integer(c_int32_t), value :: sc
      real(c_double), intent(in) :: S(*)
    end function
    integer(c_int) function elmm_slabs_download_field(h, field, host) bind(C)
      import
      type(c_ptr), value :: h
      integer(c_int32_t), value :: field
      real(c_double) :: host(*)
    end function
    integer(c_int) function elmm_slabs_set_puffs(h, puffs, npuffs, volumes, nvolumes) bind(C)
      import
      type(c_ptr), value :: h, puffs, volumes
      integer(c_int32_t), value :: npuffs, nvolumes
    end function
    integer(c_int) function elmm_slabs_download_scalar_slices(h, sc, xy, xz) bind(C)
      import
      type(c_ptr), value :: h
      integer(c_int32_t), value :: sc
      type(c_ptr), value :: xy, xz
    end function
    integer(c_int) function elmm_slabs_project(h, coef, st) bind(C)
      import
      type(c_ptr), value :: h
      real(c_double), value :: coef
      type(elmm_stats) :: st
    end function
    integer(c_int) function elmm_slabs_step(h, nsteps, st) bind(C)
      import
      type(c_ptr), value :: h
      integer(c_int32_t), value :: nsteps
      type(elmm_stats) :: st
    end function
    integer(c_int) function elmm_slabs_march_host(h, U, V, W, Pr, nsteps, st) bind(C)
      import
      type(c_ptr), value :: h
      real(c_double) :: U(*), V(*), W(*), Pr(*)
      integer(c_int32_t), value :: nsteps
      type(elmm_stats) :: st
    end function
    integer(c_int) function elmm_slabs_upload_state_float(h, U, V, W, Pr) bind(C)
      import
      type(c_ptr), value :: h
      real(c_float), intent(in) :: U(*), V(*), W(*), Pr(*)
    end function
    integer(c_int) function elmm_slabs_download_state_float(h, U, V, W, Pr) bind(C)
      import
      type(c_ptr), value :: h
      real(c_float) :: U(*), V(*), W(*), Pr(*)
    end function
    integer(c_int) function elmm_slabs_march_host_float(h, U, V, W, Pr, nsteps, st) bind(C)
      import
      type(c_ptr), value :: h
      real(c_float) :: U(*), V(*), W(*), Pr(*)
      integer(c_int32_t), value :: nsteps
      type(elmm_stats) :: st
    end function
  end interface
end module elmm_gpu
