! gitm_vert_iface.f90 -- iso_c_binding interface of libgitmvert for the
! GITM Fortran host.
!
! With this module the host replaces the column loop of advance_vertical_all
! (src/advance_vertical.f90:25-27) by one call per block:
!
!    use ModGitmVertGpu
!    ...
!    do iBlock = 1, nBlocks
!       call calc_rates(iBlock)
!       call calc_viscosity(iBlock)
!       call gitm_vert_gpu_block(iBlock)        ! was: do iLon; do iLat; advance_vertical
!    end do
!
! The library reads and writes the ModGITM arrays in place through strided
! descriptors (GitmFArray in include/gitm_vert.h), so nothing is copied on
! the Fortran side.  Status bits map to the reference's stop_gitm messages.
!
! This file was written where no Fortran compiler exists; it is not
! compile-tested.

module ModGitmVertC

  use iso_c_binding
  implicit none

  integer(c_int), parameter :: GITM_OK = 0
  integer(c_int), parameter :: GITM_ERR_COLUMN = -4

  type, bind(C) :: GitmVertParams
     integer(c_int32_t) :: solver, use_neutral_friction, use_coriolis, &
          use_ion_advection, use_improved_ion_advection, use_nighttime_ion_bcs, &
          use_damping, use_msis_bcs, compute_coefficients, compute_eddy
     real(c_double) :: beta_limiter, max_vertical_velocity, min_tec, omega_body, vert_tau
     real(c_double) :: thermal_diff_coef(6)
     real(c_double) :: eddy_coef, eddy_pressure0, eddy_pressure1
  end type GitmVertParams

  type, bind(C) :: GitmFArray
     type(c_ptr) :: data
     integer(c_int64_t) :: stride(5)
     integer(c_int32_t) :: lower(5)
  end type GitmFArray

  type, bind(C) :: GitmFortranState
     integer(c_int32_t) :: n_lons, n_lats, n_alts, n_blocks
     type(GitmFArray) :: ndensity_s, idensity_s, rho, temperature, velocity, &
          ivelocity, vertical_velocity, log_ns, ndensity, species_density, &
          species_density_old, gamma, mean_major_mass, temp_unit, cmax, &
          kappa_eddy, altitude, gravity, dalt, inv_r, cos_latitude, sza, mlatitude
  end type GitmFortranState

  interface
     subroutine gitm_vert_default_params(p) bind(C, name="gitm_vert_default_params")
       import :: GitmVertParams
       type(GitmVertParams), intent(out) :: p
     end subroutine gitm_vert_default_params

     integer(c_int) function gitm_vert_create(p, device, ctx) bind(C, name="gitm_vert_create")
       import :: GitmVertParams, c_int, c_ptr
       type(GitmVertParams), intent(in) :: p
       integer(c_int), value :: device
       type(c_ptr), intent(out) :: ctx
     end function gitm_vert_create

     integer(c_int) function gitm_vert_destroy(ctx) bind(C, name="gitm_vert_destroy")
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
     end function gitm_vert_destroy

     type(c_ptr) function gitm_vert_last_error(ctx) bind(C, name="gitm_vert_last_error")
       import :: c_ptr
       type(c_ptr), value :: ctx
     end function gitm_vert_last_error

     integer(c_int) function gitm_vert_advance_fortran(ctx, st, block_first, block_last, &
          dt, on_device) bind(C, name="gitm_vert_advance_fortran")
       import :: GitmFortranState, c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       type(GitmFortranState), intent(in) :: st
       integer(c_int), value :: block_first, block_last, on_device
       real(c_double), value :: dt
     end function gitm_vert_advance_fortran
  end interface

contains

  ! Descriptor of a real(8) array section: pass the array's first element
  ! and its lower bounds / shape in the order (lon, lat, alt, field, block);
  ! absent dimensions get extent 1 and stride 0.
  function farray(first, lower, extent, present_dims) result(a)
    real(c_double), target, intent(in) :: first
    integer, intent(in) :: lower(5), extent(5)
    logical, intent(in) :: present_dims(5)
    type(GitmFArray) :: a
    integer(c_int64_t) :: s
    integer :: d
    a%data = c_loc(first)
    s = 1
    do d = 1, 5
       a%lower(d) = int(lower(d), c_int32_t)
       if (present_dims(d)) then
          a%stride(d) = s
          s = s * int(extent(d), c_int64_t)
       else
          a%stride(d) = 0
       end if
    end do
  end function farray

end module ModGitmVertC

module ModGitmVertGpu

  use ModGitmVertC
  use iso_c_binding
  implicit none

  type(c_ptr), save :: gpu_ctx = c_null_ptr

contains

  subroutine gitm_vert_gpu_init
    use ModInputs
    type(GitmVertParams) :: p
    integer(c_int) :: rc
    call gitm_vert_default_params(p)
    p%solver = merge(1, 0, UseAUSMSolver)
    p%use_neutral_friction = merge(1, 0, UseNeutralFriction)
    p%use_coriolis = merge(1, 0, UseCoriolis)
    p%use_ion_advection = merge(1, 0, UseIonAdvection)
    p%use_improved_ion_advection = merge(1, 0, UseImprovedIonAdvection)
    p%use_nighttime_ion_bcs = merge(1, 0, UseNighttimeIonBCs)
    p%use_damping = merge(1, 0, UseDamping)
    p%use_msis_bcs = 0   ! the MSIS lower boundary is passed as a table (lbc) by the native API
    p%compute_coefficients = 0   ! calc_pressure / calc_timestep / calc_rates ran on the host
    p%compute_eddy = 0           ! calc_sources (KappaEddyDiffusion) runs on the host
    p%beta_limiter = BetaLimiter
    p%max_vertical_velocity = MaximumVerticalVelocity
    p%min_tec = MinTEC
    p%omega_body = OmegaBodyInput
    rc = gitm_vert_create(p, 0_c_int, gpu_ctx)
    if (rc /= GITM_OK) call stop_gitm("gitm_vert_create failed")
  end subroutine gitm_vert_gpu_init

  ! advance_vertical for every column of block iBlock (after calc_rates(iBlock))
  subroutine gitm_vert_gpu_block(iBlock)
    use ModGITM
    use ModSources, only: KappaEddyDiffusion
    use ModEUV, only: SZA
    use ModInputs, only: Dt_in => Dt
    integer, intent(in) :: iBlock
    type(GitmFortranState) :: st
    integer(c_int) :: rc
    integer :: hl(5), he(5)
    logical :: all5(5) = .true.

    if (.not. c_associated(gpu_ctx)) call gitm_vert_gpu_init
    st%n_lons = nLons; st%n_lats = nLats; st%n_alts = nAlts; st%n_blocks = nBlocks

    hl = (/ -1, -1, -1, 1, 1 /)
    he = (/ nLons+4, nLats+4, nAlts+4, nSpeciesTotal, nBlocks /)
    st%ndensity_s = farray(NDensityS(-1,-1,-1,1,1), hl, he, all5)
    he(4) = nIons
    st%idensity_s = farray(IDensityS(-1,-1,-1,1,1), hl, he, all5)
    he(4) = nSpecies
    st%log_ns = farray(LogNS(-1,-1,-1,1,1), hl, he, all5)
    st%vertical_velocity = farray(VerticalVelocity(-1,-1,-1,1,1), hl, he, all5)
    he(4) = 3
    st%velocity = farray(Velocity(-1,-1,-1,1,1), hl, he, all5)
    st%ivelocity = farray(IVelocity(-1,-1,-1,1,1), hl, he, all5)
    he(4) = nSpeciesAll
    st%species_density = farray(SpeciesDensity(-1,-1,-1,1,1), hl, he, all5)
    st%species_density_old = farray(SpeciesDensityOld(-1,-1,-1,1,1), hl, he, all5)
    he(4) = 1
    st%rho = farray(Rho(-1,-1,-1,1), hl, he, (/ .true., .true., .true., .false., .true. /))
    st%temperature = farray(Temperature(-1,-1,-1,1), hl, he, (/ .true., .true., .true., .false., .true. /))
    st%ndensity = farray(NDensity(-1,-1,-1,1), hl, he, (/ .true., .true., .true., .false., .true. /))
    st%gamma = farray(Gamma(-1,-1,-1,1), hl, he, (/ .true., .true., .true., .false., .true. /))
    st%altitude = farray(Altitude_GB(-1,-1,-1,1), hl, he, (/ .true., .true., .true., .false., .true. /))
    st%gravity = farray(Gravity_GB(-1,-1,-1,1), hl, he, (/ .true., .true., .true., .false., .true. /))
    st%dalt = farray(dAlt_GB(-1,-1,-1,1), hl, he, (/ .true., .true., .true., .false., .true. /))
    st%inv_r = farray(InvRadialDistance_GB(-1,-1,-1,1), hl, he, (/ .true., .true., .true., .false., .true. /))
    st%mlatitude = farray(MLatitude(-1,-1,-1,1), hl, he, (/ .true., .true., .true., .false., .true. /))
    ! MeanMajorMass / TempUnit hold block iBlock only (calc_rates(iBlock))
    st%mean_major_mass = farray(MeanMajorMass(-1,-1,-1), hl, he, (/ .true., .true., .true., .false., .false. /))
    st%temp_unit = farray(TempUnit(-1,-1,-1), hl, he, (/ .true., .true., .true., .false., .false. /))
    ! cMax_GDB(0:nLons+1, 0:nLats+1, 0:nAlts+1, 3, nBlocks)
    st%cmax = farray(cMax_GDB(0,0,0,1,1), (/ 0, 0, 0, 1, 1 /), (/ nLons+2, nLats+2, nAlts+2, 3, nBlocks /), all5)
    ! KappaEddyDiffusion(nLons, nLats, -1:nAlts+2, nBlocks)
    st%kappa_eddy = farray(KappaEddyDiffusion(1,1,-1,1), (/ 1, 1, -1, 1, 1 /), &
         (/ nLons, nLats, nAlts+4, 1, nBlocks /), (/ .true., .true., .true., .false., .true. /))
    ! CosLatitude(-1:nLats+2, nBlocksMax); SZA(nLons, nLats, nBlocks)
    st%cos_latitude = farray(CosLatitude(-1,1), (/ 1, -1, 1, 1, 1 /), (/ 1, nLats+4, 1, 1, nBlocksMax /), &
         (/ .false., .true., .false., .false., .true. /))
    st%sza = farray(SZA(1,1,1), (/ 1, 1, 1, 1, 1 /), (/ nLons, nLats, 1, 1, nBlocks /), &
         (/ .true., .true., .false., .false., .true. /))

    rc = gitm_vert_advance_fortran(gpu_ctx, st, int(iBlock, c_int), int(iBlock, c_int), &
         real(Dt, c_double), 0_c_int)
    if (rc == GITM_ERR_COLUMN) call stop_gitm("Can't Continue (vertical advance reported a column failure)")
    if (rc /= GITM_OK) call stop_gitm("gitm_vert_advance_fortran failed")
  end subroutine gitm_vert_gpu_block

end module ModGitmVertGpu
