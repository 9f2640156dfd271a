!#############################################################################
!#                                                                           #
!# fosite_gpu_bind.f90 -- ISO_C_BINDING interfaces of the B200 backend       #
!#                                                                           #
!# The derived types mirror the C structs of include/fosite_gpu.h field by   #
!# field (BIND(C) keeps the C layout); the interfaces bind the extern "C"    #
!# entry points a fosite timedisc calls (timedisc_gpu.f90).                  #
!#                                                                           #
!# Not compile-tested: no Fortran compiler exists where this backend is      #
!# built.  The ABI it binds is exercised through Python ctypes by the tests. #
!#                                                                           #
!#############################################################################
MODULE fosite_gpu_bind
  USE, INTRINSIC :: ISO_C_BINDING
  IMPLICIT NONE
  PRIVATE

  ! return codes
  INTEGER(C_INT), PARAMETER, PUBLIC :: FGPU_OK = 0, FGPU_BREAK = 1, FGPU_STOPTIME = 2, &
       FGPU_EBADCFG = -1, FGPU_ENOMEM = -2, FGPU_ECUDA = -3, FGPU_ETIMEOUT = -4, &
       FGPU_EUNSUPPORTED = -5, FGPU_EARG = -6
  ! selectors of fgpu_upload_state / fgpu_download
  INTEGER(C_INT), PARAMETER, PUBLIC :: FGPU_CVAR = 1, FGPU_PVAR = 2, FGPU_RHS = 3, FGPU_BCCSOUND = 4, &
       FGPU_XFLUX = 5, FGPU_YFLUX = 6, FGPU_ZFLUX = 7
  ! boundary faces (C indices 0..5 of fgpu_config%bc are Fortran 1..6)
  INTEGER, PARAMETER, PUBLIC :: FGPU_WEST = 1, FGPU_EAST = 2, FGPU_SOUTH = 3, FGPU_NORTH = 4, &
       FGPU_BOTTOM = 5, FGPU_TOP = 6

  TYPE, BIND(C), PUBLIC :: fgpu_config
    ! mesh
    INTEGER(C_INT32_T) :: inum, jnum, knum
    INTEGER(C_INT32_T) :: geometry
    REAL(C_DOUBLE)     :: xmin, xmax, ymin, ymax, zmin, zmax
    REAL(C_DOUBLE)     :: gparam
    ! physics
    INTEGER(C_INT32_T) :: physics
    REAL(C_DOUBLE)     :: gamma, csiso, gn
    ! fluxes / reconstruction
    INTEGER(C_INT32_T) :: fluxtype, order, variables, limiter
    REAL(C_DOUBLE)     :: theta
    ! boundary conditions
    INTEGER(C_INT32_T) :: bc(6)
    ! timedisc
    INTEGER(C_INT32_T) :: method, tdorder
    REAL(C_DOUBLE)     :: cfl, stoptime, dtlimit, tol_rel, tol_abs(5), beta
    INTEGER(C_INT32_T) :: maxiter, checkdata
    REAL(C_DOUBLE)     :: pmin, rhomin, tmin
    ! point mass
    INTEGER(C_INT32_T) :: pointmass
    REAL(C_DOUBLE)     :: pm_mass
    ! fargo
    INTEGER(C_INT32_T) :: fargo_method, fargo_direction
    REAL(C_DOUBLE)     :: tout
    ! accretion
    INTEGER(C_INT32_T) :: pm_outbound, pad_
    REAL(C_DOUBLE)     :: starttime
    ! viscosity
    INTEGER(C_INT32_T) :: vismodel, pad2_
    REAL(C_DOUBLE)     :: dynconst, bulkconst, vis_exponent, cvis
  END TYPE fgpu_config

  TYPE, BIND(C), PUBLIC :: fgpu_status
    REAL(C_DOUBLE)     :: time, dt, dtold, dtmin, maxerr
    INTEGER(C_INT64_T) :: iter, n_adj
    INTEGER(C_INT32_T) :: dtcause, brk, checkflags, pad
  END TYPE fgpu_status

  PUBLIC :: fgpu_config_init, fgpu_create, fgpu_destroy, fgpu_last_error, fgpu_state_size, &
       fgpu_set_sound_speeds, fgpu_set_fargo_velocity, fgpu_upload_state, fgpu_download, &
       fgpu_first_step, fgpu_step, fgpu_run, fgpu_compute_rhs, fgpu_calc_timestep, &
       fgpu_set_output_time, fgpu_get_status, fgpu_get_pointmass, fgpu_synchronize

  INTERFACE
    ! fosite's GetAttr defaults
    SUBROUTINE fgpu_config_init(cfg) BIND(C, NAME="fgpu_config_init")
      IMPORT :: fgpu_config
      TYPE(fgpu_config), INTENT(OUT) :: cfg
    END SUBROUTINE
    ! new_mesh/new_physics/new_fluxes/new_timedisc/new_boundary in one call
    INTEGER(C_INT) FUNCTION fgpu_create(cfg, device, h) BIND(C, NAME="fgpu_create")
      IMPORT :: fgpu_config, C_INT, C_PTR
      TYPE(fgpu_config), INTENT(IN) :: cfg
      INTEGER(C_INT), VALUE :: device
      TYPE(C_PTR), INTENT(OUT) :: h
    END FUNCTION
    SUBROUTINE fgpu_destroy(h) BIND(C, NAME="fgpu_destroy")
      IMPORT :: C_PTR
      TYPE(C_PTR), VALUE :: h
    END SUBROUTINE
    INTEGER(C_INT) FUNCTION fgpu_last_error(h, buf, len) BIND(C, NAME="fgpu_last_error")
      IMPORT :: C_PTR, C_CHAR, C_INT
      TYPE(C_PTR), VALUE :: h
      CHARACTER(KIND=C_CHAR), INTENT(OUT) :: buf(*)
      INTEGER(C_INT), VALUE :: len
    END FUNCTION
    INTEGER(C_INT64_T) FUNCTION fgpu_state_size(h) BIND(C, NAME="fgpu_state_size")
      IMPORT :: C_PTR, C_INT64_T
      TYPE(C_PTR), VALUE :: h
    END FUNCTION
    ! physics_eulerisotherm%SetSoundSpeeds: bccsound%data1d, fcsound%data1d
    INTEGER(C_INT) FUNCTION fgpu_set_sound_speeds(h, bcc, nb, fcs, nf) BIND(C, NAME="fgpu_set_sound_speeds")
      IMPORT :: C_PTR, C_DOUBLE, C_INT64_T, C_INT
      TYPE(C_PTR), VALUE :: h
      REAL(C_DOUBLE), INTENT(IN) :: bcc(*), fcs(*)
      INTEGER(C_INT64_T), VALUE :: nb, nf
    END FUNCTION
    ! Timedisc%w of FARGO type 2
    INTEGER(C_INT) FUNCTION fgpu_set_fargo_velocity(h, w, n) BIND(C, NAME="fgpu_set_fargo_velocity")
      IMPORT :: C_PTR, C_DOUBLE, C_INT64_T, C_INT
      TYPE(C_PTR), VALUE :: h
      REAL(C_DOUBLE), INTENT(IN) :: w(*)
      INTEGER(C_INT64_T), VALUE :: n
    END FUNCTION
    ! Timedisc%cvar%data1d / %pvar%data1d (ghost-padded, Fortran order) to the device
    INTEGER(C_INT) FUNCTION fgpu_upload_state(h, which, dat, n) BIND(C, NAME="fgpu_upload_state")
      IMPORT :: C_PTR, C_DOUBLE, C_INT64_T, C_INT
      TYPE(C_PTR), VALUE :: h
      INTEGER(C_INT), VALUE :: which
      REAL(C_DOUBLE), INTENT(IN) :: dat(*)
      INTEGER(C_INT64_T), VALUE :: n
    END FUNCTION
    ! cvar, pvar, rhs, bccsound or the x/y/z fluxes of the last fgpu_compute_rhs to the host
    INTEGER(C_INT) FUNCTION fgpu_download(h, which, out, n) BIND(C, NAME="fgpu_download")
      IMPORT :: C_PTR, C_DOUBLE, C_INT64_T, C_INT
      TYPE(C_PTR), VALUE :: h
      INTEGER(C_INT), VALUE :: which
      REAL(C_DOUBLE), INTENT(OUT) :: out(*)
      INTEGER(C_INT64_T), VALUE :: n
    END FUNCTION
    ! fosite%FirstStep: ComputeRHS(CHECK_ALL) + CalcTimestep
    INTEGER(C_INT) FUNCTION fgpu_first_step(h) BIND(C, NAME="fgpu_first_step")
      IMPORT :: C_PTR, C_INT
      TYPE(C_PTR), VALUE :: h
    END FUNCTION
    ! fosite%Step: stop test, output-time clip, IntegrationStep, CalcTimestep
    INTEGER(C_INT) FUNCTION fgpu_step(h) BIND(C, NAME="fgpu_step")
      IMPORT :: C_PTR, C_INT
      TYPE(C_PTR), VALUE :: h
    END FUNCTION
    INTEGER(C_INT) FUNCTION fgpu_run(h, n, done) BIND(C, NAME="fgpu_run")
      IMPORT :: C_PTR, C_INT64_T, C_INT
      TYPE(C_PTR), VALUE :: h
      INTEGER(C_INT64_T), VALUE :: n
      INTEGER(C_INT64_T), INTENT(OUT) :: done
    END FUNCTION
    ! ComputeRHS(CHECK_NOTHING) of the current state; rhs and fluxes via fgpu_download
    INTEGER(C_INT) FUNCTION fgpu_compute_rhs(h) BIND(C, NAME="fgpu_compute_rhs")
      IMPORT :: C_PTR, C_INT
      TYPE(C_PTR), VALUE :: h
    END FUNCTION
    INTEGER(C_INT) FUNCTION fgpu_calc_timestep(h, dt) BIND(C, NAME="fgpu_calc_timestep")
      IMPORT :: C_PTR, C_DOUBLE, C_INT
      TYPE(C_PTR), VALUE :: h
      REAL(C_DOUBLE), INTENT(OUT) :: dt
    END FUNCTION
    ! Datafile%time: the next output time that fgpu_step clips dt to
    INTEGER(C_INT) FUNCTION fgpu_set_output_time(h, tout) BIND(C, NAME="fgpu_set_output_time")
      IMPORT :: C_PTR, C_DOUBLE, C_INT
      TYPE(C_PTR), VALUE :: h
      REAL(C_DOUBLE), VALUE :: tout
    END FUNCTION
    INTEGER(C_INT) FUNCTION fgpu_get_status(h, st) BIND(C, NAME="fgpu_get_status")
      IMPORT :: C_PTR, C_INT, fgpu_status
      TYPE(C_PTR), VALUE :: h
      TYPE(fgpu_status), INTENT(OUT) :: st
    END FUNCTION
    INTEGER(C_INT) FUNCTION fgpu_get_pointmass(h, mass, mdot) BIND(C, NAME="fgpu_get_pointmass")
      IMPORT :: C_PTR, C_DOUBLE, C_INT
      TYPE(C_PTR), VALUE :: h
      REAL(C_DOUBLE), INTENT(OUT) :: mass, mdot
    END FUNCTION
    INTEGER(C_INT) FUNCTION fgpu_synchronize(h) BIND(C, NAME="fgpu_synchronize")
      IMPORT :: C_PTR, C_INT
      TYPE(C_PTR), VALUE :: h
    END FUNCTION
  END INTERFACE
END MODULE fosite_gpu_bind
