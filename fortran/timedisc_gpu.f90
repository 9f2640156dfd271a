!#############################################################################
!#                                                                           #
!# timedisc_gpu.f90 -- fosite timedisc class whose time step runs on a B200  #
!#                                                                           #
!# new_timedisc (timedisc/timedisc_generic.f90:55-85) allocates this class   #
!# instead of the CPU schemes when the timedisc Dict holds backend = 1:      #
!#                                                                           #
!#     CALL GetAttr(config, "backend", backend, 0)                           #
!#     IF (backend.EQ.1) THEN                                                #
!#       ALLOCATE(timedisc_gpu::Timedisc)                                    #
!#     ELSE                                                                  #
!#       SELECT CASE(method) ... (unchanged)                                 #
!#     END IF                                                                #
!#     ...                                                                   #
!#     TYPE IS (timedisc_gpu)                                                #
!#       CALL obj%InitTimedisc_gpu(Mesh,Physics,config,IO)                   #
!#                                                                           #
!# The class keeps fosite's own bookkeeping (time, dt, dtcause, n_adj, break,#
!# the cvar/pvar arrays that Datafile writes) and forwards the step methods  #
!# to the library: ComputeRHS (FirstStep's CHECK_ALL call and the others),   #
!# IntegrationStep (fgpu_step: IntegrationStep + CalcTimestep of the next    #
!# step, with the output-time clip fosite%Step applied before), and          #
!# CalcTimestep (returns the dt that fgpu_step or fgpu_first_step computed). #
!# There is no CPU fallback: an unsupported configuration is an error.       #
!#                                                                           #
!# Not compile-tested: no Fortran compiler exists where this backend is      #
!# built.  The calls it makes are exercised through Python ctypes by the     #
!# tests (tests/test_abi.py, tests/test_gpu_*.py).                           #
!#                                                                           #
!#############################################################################
MODULE timedisc_gpu_mod
  USE, INTRINSIC :: ISO_C_BINDING
  USE fosite_gpu_bind
  USE timedisc_base_mod
  USE mesh_base_mod
  USE physics_base_mod
  USE physics_eulerisotherm_mod
  USE fluxes_base_mod
  USE sources_base_mod
  USE marray_compound_mod
  USE common_dict
  IMPLICIT NONE
  PRIVATE

  TYPE, EXTENDS(timedisc_base) :: timedisc_gpu
    TYPE(C_PTR)       :: h = C_NULL_PTR      ! the library's handle (device state, streams)
    TYPE(fgpu_config) :: cfg
    LOGICAL           :: dt_ready = .FALSE.  ! dt of the last step/first step is current
    REAL              :: dt_next = 0.0
    INTEGER           :: dtcause_next = 0
  CONTAINS
    PROCEDURE :: InitTimedisc_gpu
    PROCEDURE :: ComputeRHS
    PROCEDURE :: IntegrationStep
    PROCEDURE :: CalcTimestep
    PROCEDURE :: SetOutputTime
    PROCEDURE :: SolveODE
    PROCEDURE :: Finalize
  END TYPE timedisc_gpu

  PUBLIC :: timedisc_gpu

CONTAINS
  !> Constructor: fosite's own timedisc set-up (arrays, time, dt bookkeeping), then the
  !! fgpu_config from the same Dict keys the CPU classes read, then the library handle.
  !! root is the whole fosite configuration (mesh/, physics/, fluxes/, boundary/,
  !! sources/, timedisc/ sub-dictionaries).
  SUBROUTINE InitTimedisc_gpu(this,Mesh,Physics,config,IO,root)
    CLASS(timedisc_gpu), INTENT(INOUT) :: this
    CLASS(mesh_base),    INTENT(IN)    :: Mesh
    CLASS(physics_base), INTENT(IN)    :: Physics
    TYPE(Dict_TYP),      POINTER       :: config,IO,root
    !------------------------------------------------------------------------!
    INTEGER        :: method, ival, rc
    REAL           :: rval
    INTEGER(C_INT) :: irc
    !------------------------------------------------------------------------!
    CALL GetAttr(config, "method", method)
    CALL this%InitTimedisc(Mesh,Physics,config,IO,method,"GPU (B200) time step")
    CALL fgpu_config_init(this%cfg)
    ! mesh (mesh/mesh_base.f90:351-380, geometry_base.f90:394-407)
    this%cfg%inum = Mesh%INUM
    this%cfg%jnum = Mesh%JNUM
    this%cfg%knum = Mesh%KNUM
    this%cfg%xmin = Mesh%xmin
    this%cfg%xmax = Mesh%xmax
    this%cfg%ymin = Mesh%ymin
    this%cfg%ymax = Mesh%ymax
    this%cfg%zmin = Mesh%zmin
    this%cfg%zmax = Mesh%zmax
    CALL GetAttr(root, "mesh/geometry", ival)
    this%cfg%geometry = ival
    CALL GetAttr(root, "mesh/gparam", rval, 1.0)
    this%cfg%gparam = rval
    ! physics (physics_generic.f90:56, physics_euler.f90:152, physics_eulerisotherm.f90:176)
    CALL GetAttr(root, "physics/problem", ival)
    this%cfg%physics = ival
    CALL GetAttr(root, "physics/gamma", rval, 1.4)
    this%cfg%gamma = rval
    CALL GetAttr(root, "physics/cs", rval, 0.0)
    this%cfg%csiso = rval
    ! fluxes and reconstruction (fluxes_generic.f90:56, reconstruction_base.f90:115-117,
    ! reconstruction_linear.f90:120-121)
    CALL GetAttr(root, "fluxes/fluxtype", ival)
    this%cfg%fluxtype = ival
    CALL GetAttr(root, "fluxes/order", ival, 2)
    this%cfg%order = ival
    CALL GetAttr(root, "fluxes/variables", ival, 2)
    this%cfg%variables = ival
    CALL GetAttr(root, "fluxes/limiter", ival, 1)
    this%cfg%limiter = ival
    CALL GetAttr(root, "fluxes/theta", rval, 1.0)
    this%cfg%theta = rval
    ! boundaries (boundary_generic.f90:145-150)
    CALL GetAttr(root, "boundary/western", ival);  this%cfg%bc(FGPU_WEST) = ival
    CALL GetAttr(root, "boundary/eastern", ival);  this%cfg%bc(FGPU_EAST) = ival
    CALL GetAttr(root, "boundary/southern", ival); this%cfg%bc(FGPU_SOUTH) = ival
    CALL GetAttr(root, "boundary/northern", ival); this%cfg%bc(FGPU_NORTH) = ival
    CALL GetAttr(root, "boundary/bottomer", ival); this%cfg%bc(FGPU_BOTTOM) = ival
    CALL GetAttr(root, "boundary/topper", ival);   this%cfg%bc(FGPU_TOP) = ival
    ! timedisc (timedisc_base.f90:295-359 and the schemes' "order")
    this%cfg%method    = method
    CALL GetAttr(config, "order", ival, 0)
    this%cfg%tdorder   = ival
    this%cfg%cfl       = this%cfl
    this%cfg%stoptime  = this%stoptime
    this%cfg%dtlimit   = this%dtlimit
    this%cfg%tol_rel   = this%tol_rel
    this%cfg%tol_abs(1:Physics%VNUM) = this%tol_abs(1:Physics%VNUM)
    this%cfg%beta      = this%beta
    this%cfg%maxiter   = this%maxiter
    this%cfg%checkdata = this%checkdatabm
    this%cfg%pmin      = this%pmin
    this%cfg%rhomin    = this%rhomin
    this%cfg%tmin      = this%tmin
    this%cfg%starttime = this%time
    ! sources: central point mass (gravity_pointmass.f90:173, 293-297) and viscosity
    ! (sources_viscosity.f90:147-165); fosite's default outbound WEST on curvilinear meshes
    ! is passed explicitly
    IF (HasKey(root, "sources/grav/pmass")) THEN
      this%cfg%pointmass = 1
      CALL GetAttr(root, "sources/grav/pmass/mass", rval, 1.0)
      this%cfg%pm_mass = rval
      IF (this%cfg%geometry.EQ.1) THEN
        CALL GetAttr(root, "sources/grav/pmass/outbound", ival, 0)
      ELSE
        CALL GetAttr(root, "sources/grav/pmass/outbound", ival, 1)
      END IF
      this%cfg%pm_outbound = ival
    END IF
    IF (HasKey(root, "sources/vis")) THEN
      CALL GetAttr(root, "sources/vis/vismodel", ival);      this%cfg%vismodel = ival
      CALL GetAttr(root, "sources/vis/dynconst", rval, 0.1);  this%cfg%dynconst = rval
      IF (HasKey(root, "sources/vis/bulkconst")) THEN
        CALL GetAttr(root, "sources/vis/bulkconst", rval);   this%cfg%bulkconst = rval
      END IF
      CALL GetAttr(root, "sources/vis/exponent", rval, 0.0);  this%cfg%vis_exponent = rval
      CALL GetAttr(root, "sources/vis/cvis", rval, 0.5);      this%cfg%cvis = rval
    END IF
    ! FARGO transport (timedisc_base.f90:369-452)
    CALL GetAttr(config, "fargo", ival, 0)
    this%cfg%fargo_method = ival
    CALL GetAttr(config, "shift", ival, 2)
    this%cfg%fargo_direction = ival
    irc = fgpu_create(this%cfg, -1_C_INT, this%h)
    IF (irc.NE.FGPU_OK) CALL this%Error("InitTimedisc_gpu", "fgpu_create failed: " // last_error(C_NULL_PTR))
  END SUBROUTINE InitTimedisc_gpu

  !> ComputeRHS (timedisc_base.f90:1073-1271).  fosite%FirstStep calls it on this%cvar with
  !! CHECK_ALL (fosite.f90:315-321): that call runs fgpu_first_step, which also evaluates
  !! CalcTimestep for the following CalcTimestep call.  Any other call (e.g. from
  !! GetCentrifugalVelocity) evaluates the right-hand side of the given state.  The state
  !! comes back with its ghost cells as CenterBoundary leaves them.
  SUBROUTINE ComputeRHS(this,Mesh,Physics,Sources,Fluxes,time,dt,pvar,cvar,checkdatabm,rhs)
    CLASS(timedisc_gpu),  INTENT(INOUT) :: this
    CLASS(mesh_base),     INTENT(IN)    :: Mesh
    CLASS(physics_base),  INTENT(INOUT) :: Physics
    CLASS(sources_list), ALLOCATABLE, INTENT(INOUT) :: Sources
    CLASS(fluxes_base),   INTENT(INOUT) :: Fluxes
    REAL,                 INTENT(IN)    :: time, dt
    CLASS(marray_compound), INTENT(INOUT) :: pvar,cvar,rhs
    INTEGER,              INTENT(IN)    :: checkdatabm
    !------------------------------------------------------------------------!
    INTEGER(C_INT)     :: irc
    INTEGER(C_INT64_T) :: n
    !------------------------------------------------------------------------!
    n = SIZE(cvar%data1d, KIND=C_INT64_T)
    SELECT TYPE(phys => Physics)
    CLASS IS(physics_eulerisotherm)
      IF (phys%csiso.LE.0.0) &
        CALL check(this, fgpu_set_sound_speeds(this%h, phys%bccsound%data1d, &
                   SIZE(phys%bccsound%data1d, KIND=C_INT64_T), phys%fcsound%data1d, &
                   SIZE(phys%fcsound%data1d, KIND=C_INT64_T)), "fgpu_set_sound_speeds")
    END SELECT
    CALL check(this, fgpu_upload_state(this%h, FGPU_CVAR, cvar%data1d, n), "fgpu_upload_state")
    IF (checkdatabm.EQ.CHECK_ALL .AND. .NOT.this%dt_ready) THEN
      irc = fgpu_first_step(this%h)
      IF (irc.LT.0) CALL check(this, irc, "fgpu_first_step")
      CALL sync_status(this)
      this%dt_ready = .TRUE.
    ELSE
      CALL check(this, fgpu_compute_rhs(this%h), "fgpu_compute_rhs")
      CALL check(this, fgpu_download(this%h, FGPU_RHS, rhs%data1d, n), "fgpu_download(rhs)")
    END IF
    CALL check(this, fgpu_download(this%h, FGPU_CVAR, cvar%data1d, n), "fgpu_download(cvar)")
    CALL check(this, fgpu_download(this%h, FGPU_PVAR, pvar%data1d, n), "fgpu_download(pvar)")
  END SUBROUTINE ComputeRHS

  !> IntegrationStep (timedisc_base.f90:649-750) with the CalcTimestep of the next step:
  !! one fgpu_step.  The library applies the same output-time clip as fosite%Step
  !! (io/fileio_base.f90:604-621) to the output time set with SetOutputTime; fosite%Step
  !! passes Datafile%time after each WriteDataset.  cvar/pvar are copied back every step
  !! so that Datafile%WriteDataset and the diagnostics see the current state.
  SUBROUTINE IntegrationStep(this,Mesh,Physics,Sources,Fluxes,iter,config,IO)
    CLASS(timedisc_gpu),  INTENT(INOUT) :: this
    CLASS(mesh_base),     INTENT(INOUT) :: Mesh
    CLASS(physics_base),  INTENT(INOUT) :: Physics
    CLASS(sources_list), ALLOCATABLE, INTENT(INOUT) :: Sources
    CLASS(fluxes_base),   INTENT(INOUT) :: Fluxes
    INTEGER,              INTENT(INOUT) :: iter
    TYPE(Dict_TYP),       POINTER       :: config,IO
    !------------------------------------------------------------------------!
    INTEGER(C_INT)     :: irc
    INTEGER(C_INT64_T) :: n
    TYPE(fgpu_status)  :: st
    !------------------------------------------------------------------------!
    irc = fgpu_step(this%h)
    IF (irc.LT.0) CALL check(this, irc, "fgpu_step")
    CALL sync_status(this)
    CALL check(this, fgpu_get_status(this%h, st), "fgpu_get_status")
    iter = INT(st%iter)
    n = SIZE(this%cvar%data1d, KIND=C_INT64_T)
    CALL check(this, fgpu_download(this%h, FGPU_CVAR, this%cvar%data1d, n), "fgpu_download(cvar)")
    CALL check(this, fgpu_download(this%h, FGPU_PVAR, this%pvar%data1d, n), "fgpu_download(pvar)")
    this%cold = this%cvar
  END SUBROUTINE IntegrationStep

  !> CalcTimestep (timedisc_base.f90:818-909): the step size the library computed at the end
  !! of the last fgpu_step / fgpu_first_step (CFL over all cells incl. ghosts, sources).
  REAL FUNCTION CalcTimestep(this,Mesh,Physics,Sources,Fluxes,time,dtcause) RESULT(dt)
    CLASS(timedisc_gpu),  INTENT(INOUT) :: this
    CLASS(mesh_base),     INTENT(IN)    :: Mesh
    CLASS(physics_base),  INTENT(INOUT) :: Physics
    CLASS(sources_list), ALLOCATABLE, INTENT(INOUT) :: Sources
    CLASS(fluxes_base),   INTENT(INOUT) :: Fluxes
    REAL,                 INTENT(IN)    :: time
    INTEGER,              INTENT(INOUT) :: dtcause
    !------------------------------------------------------------------------!
    dt = this%dt_next
    dtcause = this%dtcause_next
  END FUNCTION CalcTimestep

  !> The next output time (Datafile%time), for the library's output-time clip.
  SUBROUTINE SetOutputTime(this,tout)
    CLASS(timedisc_gpu), INTENT(INOUT) :: this
    REAL,                INTENT(IN)    :: tout
    CALL check(this, fgpu_set_output_time(this%h, REAL(tout, C_DOUBLE)), "fgpu_set_output_time")
  END SUBROUTINE SetOutputTime

  !> The ODE solvers run inside the library; SolveODE is never called for this class.
  SUBROUTINE SolveODE(this,Mesh,Physics,Sources,Fluxes,time,dt,err)
    CLASS(timedisc_gpu),  INTENT(INOUT) :: this
    CLASS(mesh_base),     INTENT(IN)    :: Mesh
    CLASS(physics_base),  INTENT(INOUT) :: Physics
    CLASS(sources_list), ALLOCATABLE, INTENT(INOUT) :: Sources
    CLASS(fluxes_base),   INTENT(INOUT) :: Fluxes
    REAL,                 INTENT(IN)    :: time
    REAL,                 INTENT(INOUT) :: dt, err
    CALL this%Error("SolveODE", "the GPU timedisc integrates inside the library")
  END SUBROUTINE SolveODE

  SUBROUTINE Finalize(this)
    CLASS(timedisc_gpu) :: this
    IF (C_ASSOCIATED(this%h)) CALL fgpu_destroy(this%h)
    this%h = C_NULL_PTR
    CALL this%Finalize_base()
  END SUBROUTINE Finalize

  !> Timedisc bookkeeping from the library's status (time, dt of the next step, dtold,
  !! dtmin, dtcause, n_adj, break).
  SUBROUTINE sync_status(this)
    CLASS(timedisc_gpu), INTENT(INOUT) :: this
    TYPE(fgpu_status) :: st
    CALL check(this, fgpu_get_status(this%h, st), "fgpu_get_status")
    this%time    = st%time
    this%dtold   = st%dtold
    this%dtmin   = st%dtmin
    this%n_adj   = INT(st%n_adj)
    this%break   = st%brk.NE.0
    this%dt_next = st%dt
    this%dtcause_next = st%dtcause
  END SUBROUTINE sync_status

  !> Hard library errors (negative codes) abort through this%Error, as fosite does; soft
  !! codes (FGPU_BREAK, FGPU_STOPTIME) are read from the status instead.
  SUBROUTINE check(this,irc,what)
    CLASS(timedisc_gpu), INTENT(INOUT) :: this
    INTEGER(C_INT),      INTENT(IN)    :: irc
    CHARACTER(LEN=*),    INTENT(IN)    :: what
    IF (irc.LT.0) CALL this%Error("timedisc_gpu", what // ": " // last_error(this%h))
  END SUBROUTINE check

  FUNCTION last_error(h) RESULT(msg)
    TYPE(C_PTR), INTENT(IN) :: h
    CHARACTER(LEN=256)      :: msg
    CHARACTER(KIND=C_CHAR)  :: buf(256)
    INTEGER(C_INT)          :: n
    INTEGER                 :: i
    n = fgpu_last_error(h, buf, 256_C_INT)
    msg = ""
    DO i = 1, MIN(INT(n), 255)
      msg(i:i) = buf(i)
    END DO
  END FUNCTION last_error

END MODULE timedisc_gpu_mod
