/*
 * fosite_gpu.h -- C ABI of the B200 (sm_100a) backend for fosite's explicit
 * finite-volume time step.
 *
 * The entry points below are what a Fortran 2008 caller binds with
 * ISO_C_BINDING (fortran/fosite_gpu_bind.f90 holds the BIND(C) interface block).  Every
 * call takes plain pointers and sizes; no C++ or torch type crosses the
 * boundary.  All state arrays exchanged with the caller use fosite's own
 * layout: Fortran order, i fastest, ghost-padded by two cells in every active
 * direction (mesh/marray_base.f90:146-290, mesh/marray_compound.f90:275-391),
 * i.e. data4d(IGMIN:IGMAX, JGMIN:JGMAX, KGMIN:KGMAX, 1:VNUM) flattened.
 *
 * Ownership: the library copies on upload and download and owns all device
 * memory for the lifetime of a handle.  One handle owns one CUDA stream;
 * calls on one handle must be serialised by the caller, distinct handles may
 * be used from different threads.
 *
 * Return codes: FGPU_OK (0); positive values are soft conditions that the
 * fosite shim maps onto Timedisc%break; negative values are hard errors that
 * it maps onto this%Error (fgpu_last_error() gives the message).  Nothing in
 * the library calls exit(), abort() or traps on the device.
 */
#ifndef FOSITE_GPU_H
#define FOSITE_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- fosite's own integer identifiers (same values as the Fortran code) ---- */
/* geometries: mesh/geometry_base.f90:345-361 */
#define FGPU_CARTESIAN        1
#define FGPU_CYLINDRICAL      30
#define FGPU_LOGCYLINDRICAL   31
/* physics: physics/physics_base.f90:496-498 */
#define FGPU_EULER_ISOTHERM   16
#define FGPU_EULER            17
/* fluxes: fluxes/fluxes_base.f90:104 */
#define FGPU_KT               1
/* reconstruction order: fluxes/reconstruction_base.f90:78-79 */
#define FGPU_CONSTANT         1
#define FGPU_LINEAR           2
/* reconstruction variables: physics/physics_base.f90:67 */
#define FGPU_PRIMITIVE        1
#define FGPU_CONSERVATIVE     2
/* limiters: fluxes/reconstruction_linear.f90:71-78 (PP=6 is rejected, as in fosite) */
#define FGPU_MINMOD           1
#define FGPU_MONOCENT         2
#define FGPU_SWEBY            3
#define FGPU_SUPERBEE         4
#define FGPU_OSPRE            5
#define FGPU_PP               6
#define FGPU_VANLEER          7
#define FGPU_NOLIMIT          8
/* boundary conditions: boundary/boundary_base.f90:110-126 */
#define FGPU_NO_GRADIENTS     0x01
#define FGPU_PERIODIC         0x02
#define FGPU_REFLECTING       0x03
#define FGPU_AXIS             0x04   /* reflecting, with the azimuthal velocity reflected too (boundary_axis.f90) */
#define FGPU_ABSORBING        0x0D
/* boundary orientation: mesh/mesh_base.f90:102-107 (1-based there, 0-based here) */
#define FGPU_WEST   0
#define FGPU_EAST   1
#define FGPU_SOUTH  2
#define FGPU_NORTH  3
#define FGPU_BOTTOM 4
#define FGPU_TOP    5
/* time integrators: timedisc/timedisc_base.f90:187-191 */
#define FGPU_MODIFIED_EULER   1
#define FGPU_RK_FEHLBERG      2
#define FGPU_CASH_KARP        3
#define FGPU_DORMAND_PRINCE   4
#define FGPU_SSPRK            5
/* checkdata bit mask: timedisc/timedisc_base.f90:197-204 */
#define FGPU_CHECK_NOTHING    0x00
#define FGPU_CHECK_CSOUND     0x01
#define FGPU_CHECK_PMIN       0x02
#define FGPU_CHECK_RHOMIN     0x04
#define FGPU_CHECK_INVALID    0x08
#define FGPU_CHECK_TMIN       0x10
#define FGPU_CHECK_ALL        0xFF
/* dtcause: timedisc/timedisc_base.f90:192-196 */
#define FGPU_DTCAUSE_CFL       0
#define FGPU_DTCAUSE_ERRADJ   -1
#define FGPU_DTCAUSE_SMALLERR -2
#define FGPU_DTCAUSE_FILEIO   -4
/* dtcause of a source term is its source type: sources/sources_generic.f90:71-80 */
#define FGPU_DTCAUSE_VISCOSITY 3
/* viscosity models: sources/sources_viscosity.f90:72-76 */
#define FGPU_VIS_MOLECULAR    1
#define FGPU_VIS_ALPHA        2
#define FGPU_VIS_BETA         3
#define FGPU_VIS_POWERLAW     4
#define FGPU_VIS_ALPHA_ALT    5

/* ---- return codes ---- */
#define FGPU_OK               0
#define FGPU_BREAK            1   /* soft: NaN/Inf error norm, dt < dtlimit or CheckData failure */
#define FGPU_STOPTIME         2   /* soft: |stoptime - time| <= 1e-5 stoptime, nothing was done */
#define FGPU_EBADCFG         -1
#define FGPU_ENOMEM          -2
#define FGPU_ECUDA           -3
#define FGPU_ETIMEOUT        -4
#define FGPU_EUNSUPPORTED    -5
#define FGPU_EARG            -6

#define FGPU_MAXVAR 5

/*
 * Flat POD mirror of the fosite Dict keys read on the time-step path.  Field
 * names follow the Dict keys (mesh/mesh_base.f90:31-63,
 * timedisc/timedisc_base.f90:30-48,285-350, fluxes/reconstruction_linear.f90:
 * 116-117, physics/physics_base.f90, sources/gravity_pointmass.f90:160-190,
 * boundary/boundary_generic.f90:145-245).  fgpu_config_init() fills fosite's
 * defaults; a Fortran shim translates the caller's Dict into this struct.
 */
typedef struct fgpu_config {
    /* mesh */
    int32_t inum, jnum, knum;      /* interior cells per direction (1 = collapsed) */
    int32_t geometry;              /* FGPU_CARTESIAN / _CYLINDRICAL / _LOGCYLINDRICAL */
    double  xmin, xmax, ymin, ymax, zmin, zmax;
    double  gparam;                /* logcylindrical scale, default 1.0 */
    /* physics */
    int32_t physics;               /* FGPU_EULER or FGPU_EULER_ISOTHERM */
    double  gamma;                 /* default 1.4 */
    double  csiso;                 /* isothermal sound speed; 0 = caller-supplied profile */
    double  gn;                    /* gravitational constant of the unit system (1 = geometrical) */
    /* fluxes / reconstruction */
    int32_t fluxtype;              /* FGPU_KT */
    int32_t order;                 /* FGPU_CONSTANT or FGPU_LINEAR */
    int32_t variables;             /* FGPU_PRIMITIVE or FGPU_CONSERVATIVE (default) */
    int32_t limiter;               /* default FGPU_MINMOD */
    double  theta;                 /* MC / Sweby parameter, default 1.0 */
    /* boundary conditions, indexed by FGPU_WEST..FGPU_TOP */
    int32_t bc[6];
    /* timedisc */
    int32_t method;                /* FGPU_MODIFIED_EULER, FGPU_DORMAND_PRINCE, ... */
    int32_t tdorder;               /* 0 = the method's default order */
    double  cfl;                   /* default 0.4 */
    double  stoptime;
    double  dtlimit;               /* default EPSILON*stoptime */
    double  tol_rel;               /* default 0.01 */
    double  tol_abs[FGPU_MAXVAR];  /* default 0.001 */
    double  beta;                  /* PI controller, default 0.08 */
    int32_t maxiter;
    int32_t checkdata;             /* default FGPU_CHECK_ALL */
    double  pmin, rhomin, tmin;    /* default TINY(1.0) */
    /* sources: central point mass (gravity/pointmass), 0 = off */
    int32_t pointmass;
    double  pm_mass;               /* default 1.0 */
    /* fargo transport (timedisc_base.f90:369-452): method 0 off, 1 background velocity
     * computed every step, 2 fixed user-supplied background velocity
     * (fgpu_set_fargo_velocity); 2D x-y meshes (isothermal or ideal gas without CHECK_PMIN)
     * with the fixed-step or embedded modified Euler scheme or an embedded Butcher scheme.
     * Type 3 (shearing box) is not available. */
    int32_t fargo_method;
    int32_t fargo_direction;       /* 1 transport along x, 2 along y */
    /* output clip time for AdjustTimestep (io/fileio_base.f90:604-621); 0 = stoptime */
    double  tout;
    /* point-mass accretion (gravity_pointmass.f90:287-297, 383-428): the boundary whose
     * accumulated mass flux feeds the point mass, in fosite's numbering 1 = WEST,
     * 2 = EAST; 0 = off.  fosite defaults to WEST on cylindrical meshes, this struct
     * to 0 (the caller passes the Dict value).  Fixed-step modified Euler only. */
    int32_t pm_outbound;
    int32_t pad_;
    /* Timedisc%time at FirstStep ("starttime", timedisc_base.f90:295), e.g. the time of a
     * restart file (examples/restart.f90); default 0 */
    double  starttime;
    /* viscosity source (sources/sources_viscosity.f90, keys vismodel, dynconst,
     * bulkconst, exponent, cvis): 0 = off.  FGPU_VIS_MOLECULAR (constant dynamic and
     * bulk viscosity) on 2D x-y and 3D meshes.  bulkconst NaN (the fgpu_config_init
     * value) takes fosite's default -2/3*dynconst. */
    int32_t vismodel;
    int32_t pad2_;
    double  dynconst;              /* default 0.1 */
    double  bulkconst;             /* default NaN = -2/3*dynconst */
    double  vis_exponent;          /* POWERLAW exponent, default 0 */
    double  cvis;                  /* viscous Courant number, default 0.5 */
} fgpu_config;

/* Step bookkeeping returned to the caller (mirrors Timedisc%time/dt/...). */
typedef struct fgpu_status {
    double  time;        /* Timedisc%time */
    double  dt;          /* Timedisc%dt: next step size */
    double  dtold;       /* Timedisc%dtold */
    double  dtmin;       /* Timedisc%dtmin */
    double  maxerr;      /* last error norm returned by SolveODE */
    int64_t iter;        /* accepted (sub-)steps, fosite%iter */
    int64_t n_adj;       /* rejected attempts, Timedisc%n_adj */
    int32_t dtcause;
    int32_t brk;         /* Timedisc%break */
    int32_t checkflags;  /* FGPU_CHECK_* bits that failed in CheckData */
    int32_t pad;
} fgpu_status;

typedef struct fgpu_handle fgpu_handle;

/* which-selectors for fgpu_download / fgpu_upload_state / fgpu_get_mesh */
#define FGPU_CVAR        1   /* conservative state, ghost-padded, ghosts as CenterBoundary leaves them */
#define FGPU_PVAR        2   /* primitive state, ghost-padded */
#define FGPU_RHS         3   /* right-hand side of the last fgpu_compute_rhs (interior cells valid) */
#define FGPU_BCCSOUND    4   /* cell-centre sound speed (ghost-padded) */
/* Fluxes%xfluxdydz / yfluxdzdx / zfluxdxdy of the last fgpu_compute_rhs (fluxes_base.f90:87-97,
 * fluxes_kt.f90:109-208): ghost-padded, VNUM variables; index i holds the flux through the
 * face between cells i and i+1 (x), likewise j (y) and k (z).  Valid on the faces the
 * right-hand side reads: i from IMIN-1 to IMAX with interior j and k (x), and so on. */
#define FGPU_XFLUX       5
#define FGPU_YFLUX       6
#define FGPU_ZFLUX       7
#define FGPU_MESH_X      10  /* curvilinear cell-centre coordinates, ghost-padded scalar arrays */
#define FGPU_MESH_Y      11
#define FGPU_MESH_Z      12
#define FGPU_MESH_RADIUS 13  /* Mesh%radius%bcenter */

/* Fill a config with fosite's defaults (the GetAttr default values). */
void fgpu_config_init(fgpu_config* cfg);

/* Replaces the factories new_mesh/new_physics/new_fluxes/new_reconstruction/
 * new_timedisc/new_boundary/InitSources (fosite.f90:184-248,
 * timedisc/timedisc_generic.f90:45-87, fluxes/fluxes_generic.f90:46-68,
 * boundary/boundary_generic.f90:104-283): validates the config, builds the
 * metric on the host (mesh/mesh_base.f90:446-729, mesh/mesh_midpoint.f90:
 * 97-145) and allocates device memory.  device < 0 uses the current device. */
int  fgpu_create(const fgpu_config* cfg, int device, fgpu_handle** out);
void fgpu_destroy(fgpu_handle* h);
/* Copies the last error message of h (or of the last failed create when h is
 * NULL) into buf; returns the message length. */
int  fgpu_last_error(const fgpu_handle* h, char* buf, int len);

/* Number of doubles of a ghost-padded state array (cells x VNUM) and of a
 * ghost-padded scalar mesh array (cells). */
int64_t fgpu_state_size(const fgpu_handle* h);
int64_t fgpu_cell_count(const fgpu_handle* h);
int     fgpu_vnum(const fgpu_handle* h);

/* Mesh arrays for building initial data (Mesh%center / Mesh%radius). */
int fgpu_get_mesh(fgpu_handle* h, int which, double* out, int64_t n);

/* physics_eulerisotherm%SetSoundSpeeds (physics/physics_eulerisotherm.f90:
 * 288-309): bccsound(IG,JG,KG) and fcsound(IG,JG,KG,NFACES).  The profiles
 * may vary with the first coordinate only (disk setups set cs(r)); other
 * profiles are rejected with FGPU_EUNSUPPORTED. */
int fgpu_set_sound_speeds(fgpu_handle* h, const double* bccsound, int64_t nb,
                          const double* fcsound, int64_t nf);

/* Upload Timedisc%cvar (which = FGPU_CVAR) or Timedisc%pvar (FGPU_PVAR, then
 * converted with Convert2Conservative).  Only interior cells are read.  With
 * FARGO transport, a state uploaded after fgpu_first_step is taken to be in
 * the co-moving frame, the frame fgpu_download returns. */
int fgpu_upload_state(fgpu_handle* h, int which, const double* data, int64_t n);
/* Download a ghost-padded array (FGPU_CVAR, FGPU_PVAR, FGPU_RHS, FGPU_BCCSOUND,
 * FGPU_XFLUX/YFLUX/ZFLUX). */
int fgpu_download(fgpu_handle* h, int which, double* out, int64_t n);

/* fosite%FirstStep (fosite.f90:258-348): full ComputeRHS with CHECK_ALL and
 * CalcTimestep.  Must be called once after the initial upload. */
int fgpu_first_step(fgpu_handle* h);
/* One fosite%Step (fosite.f90:367-464): stop-time test, dt clip to the
 * output time, IntegrationStep (timedisc_base.f90:649-750) and
 * CalcTimestep (timedisc_base.f90:818-909). */
int fgpu_step(fgpu_handle* h);
/* n consecutive fgpu_step calls; fixed-step schemes replay a captured CUDA
 * graph with dt kept on the device.  *done receives the steps taken. */
int fgpu_run(fgpu_handle* h, int64_t n, int64_t* done);
/* Timedisc%ComputeRHS (timedisc_base.f90:1073-1271) of the current state with
 * CHECK_NOTHING; the result is available through fgpu_download(FGPU_RHS). */
int fgpu_compute_rhs(fgpu_handle* h);
/* Timedisc%CalcTimestep of the current state (does not change the status). */
int fgpu_calc_timestep(fgpu_handle* h, double* dt);
/* Datafile%time, the next output time (io/fileio_base.f90:604-621): fgpu_step clips dt so
 * that a step ends there, as fosite%Step does through Datafile%AdjustTimestep; replaces
 * fgpu_config.tout after each output. */
int fgpu_set_output_time(fgpu_handle* h, double tout);
/* Measure every stage-kernel layout on this grid (reps RHS evaluations each into
 * a scratch array; the state is untouched) and keep the fastest for later
 * steps.  *variant receives the choice.  Decisions are cached per process by
 * (device, dimensionality, physics, reconstruction variables, limiter, geometry,
 * mesh size, features): a grid with a known key takes the cached layout without
 * probing; reps < 0 measures |reps| times anyway and refreshes the entry.  No
 * counterpart in the reference. */
int fgpu_autotune(fgpu_handle* h, int reps, int* variant);
/* The stage-kernel layout later steps use (the tuner's choice, FGPU_STAGE_VARIANT, or
 * the default 0) and, for 3D grids, the z extent one block marches through.  Either
 * pointer may be NULL.  No counterpart in the reference. */
int fgpu_stage_layout(const fgpu_handle* h, int* variant, int* kchunk);

/* ---- batched ensembles (no counterpart in the reference, which integrates one
 * grid per process) ---------------------------------------------------------
 * A batch advances many independent grids with one persistent launch per
 * Runge-Kutta stage over the flattened tile queue of all grids, plus one
 * ghost-cell / CFL / finalize launch.  Members are handles created, uploaded
 * and past fgpu_first_step, all with either the fixed-step modified Euler
 * scheme of time order 2 or 3, the embedded modified Euler scheme of one order,
 * or the same embedded Butcher scheme (Dormand-
 * Prince, Fehlberg, Cash-Karp, SSPRK; each member keeps its own tolerances,
 * error norm and step-size controller, advanced attempt by attempt on the
 * device), the same dimensionality, physics and reconstruction variables, no
 * accretion or viscosity, on one device; fixed-step members may use FARGO (one
 * transport direction per batch; such a member takes its first step after
 * fgpu_first_step alone, as that step has its own frame changes); mesh sizes, geometry, limiters,
 * boundaries and physical parameters may differ.  Each member keeps its own
 * dt, time and stop state (a member that reached its stop time idles), and its
 * results are bitwise those of stepping it alone.  The handles stay owned by
 * the caller and must outlive the batch; while a batch runs, do not step its
 * members individually. */
typedef struct fgpu_batch fgpu_batch;
int  fgpu_batch_create(fgpu_handle* const* members, int n, fgpu_batch** out);
void fgpu_batch_destroy(fgpu_batch* b);
int  fgpu_batch_last_error(const fgpu_batch* b, char* buf, int len);
/* number of members and of tiles in the flattened queue */
int  fgpu_batch_size(const fgpu_batch* b, int* members, int* tiles);
/* Advance every member by nsteps steps (replayed CUDA graphs of 16 steps);
 * the members' status (fgpu_get_status) is current on return.  *active
 * receives the number of members that have neither stopped nor broken. */
int  fgpu_batch_run(fgpu_batch* b, int64_t nsteps, int* active);
/* fgpu_batch_run in two halves, so that batches on different streams overlap:
 * enqueue returns without waiting; collect waits for everything enqueued and
 * updates the members' status. */
int  fgpu_batch_enqueue(fgpu_batch* b, int64_t nsteps);
int  fgpu_batch_collect(fgpu_batch* b, int* active);
/* fgpu_autotune for the batched stage kernel: times the shared-memory tile layouts
 * 0, 2, 3 and, for fixed-step 2D batches whose every stage it serves, the
 * TMA-staged layout 6 (the layout the batch starts with when its first member's
 * layout is 6 or 7), and keeps the fastest. */
int  fgpu_batch_autotune(fgpu_batch* b, int reps, int* variant);
/* the batch's current stage layout */
int  fgpu_batch_layout(const fgpu_batch* b, int* variant);

/* CalcTimestep for callers that cannot allocate device memory (no counterpart
 * in the reference).  Takes a config and a caller-owned device state in the
 * library's stored layout (interior cells only, one field of inum*jnum*knum
 * doubles per conservative variable, i fastest) and writes the CFL time step
 * to the caller's device double *d_dt, on the caller's stream.  It calls no
 * cudaMalloc/cudaFree: the mesh metric and the reduction slots live in a
 * 1 MiB file-scope __device__ array that every GPU loading the library holds
 * until exit.  Cartesian meshes, ideal-gas or constant-cs isothermal physics,
 * no point mass or fargo; meshes whose metric does not fit (inum above about
 * 5000) return FGPU_EARG.  Each call only enqueues work on the caller's stream
 * (a memset and four kernels; the host does not wait).  The first call on a
 * device looks up the array's device address, so make it before any stream
 * capture.  All calls share the array: calls that overlap on the GPU race. */
int fgpu_calc_timestep_noalloc(const fgpu_config* cfg, const double* d_cvar, double* d_dt, void* stream);
int fgpu_get_status(fgpu_handle* h, fgpu_status* st);
/* Timedisc%w for FARGO type 2 (a background velocity the user supplies, e.g. in
 * InitData; timedisc_base.f90:414-424): transport along y, one value per padded i
 * (inum+4 values, the interior i starting at index 2); along x, one per padded j
 * (jnum+4 values); call before fgpu_first_step. */
int fgpu_set_fargo_velocity(fgpu_handle* h, const double* w, int64_t n);
/* The central point mass and the accumulated boundary mass flux of its last update
 * (gravity_pointmass%mass, %mdot); the configured mass when accretion is off. */
int fgpu_get_pointmass(fgpu_handle* h, double* mass, double* mdot);
/* Block until all device work of h has finished. */
int fgpu_synchronize(fgpu_handle* h);
/* Enqueue all further work of h on a caller-owned CUDA stream (a cudaStream_t
 * passed as void*); NULL returns to the handle's own stream.  No counterpart
 * in the reference (host-only code); lets a caller order the solver with its
 * own device work and time it with its own events. */
int fgpu_set_stream(fgpu_handle* h, void* stream);

/* Instrumentation (no counterpart in the reference, which only prints wall
 * clock run times, fosite.f90:515-575).  With profiling on, every stage-kernel
 * launch is bracketed by CUDA events on the handle's stream and its algorithmic
 * HBM bytes (arrays read + written x VNUM x cells x 8) are accumulated;
 * captured graphs are bypassed so each launch can be timed. */
typedef struct fgpu_stats {
    int64_t launches;         /* kernels launched by the library since the last reset */
    int64_t stage_launches;   /* fused stage (RHS) kernels */
    int64_t attempts;         /* time-step attempts (accepted + rejected) */
    int64_t cell_updates;     /* interior cells x accepted steps */
    double  stage_ms;         /* summed CUDA-event time of the RHS stages (profiling on): stage
                                 kernels plus the passes that form their input states */
    double  stage_bytes;      /* algorithmic bytes of the timed stages */
    double  other_ms;         /* boundary / reduction kernels (profiling on) */
    double  form_ms;          /* the stage-state formation part of stage_ms */
} fgpu_stats;
int fgpu_set_profiling(fgpu_handle* h, int on);
int fgpu_get_stats(fgpu_handle* h, fgpu_stats* st);
int fgpu_reset_stats(fgpu_handle* h);
/* Read bandwidth (GB/s) of an L2-resident array of mb MB (at most 64) on the device:
 * one launch whose grid reads the array `passes` times (16-byte loads), timed with
 * CUDA events after a warm-up launch; the denominator of L2-relative roofline
 * fractions for grids whose working set stays in L2. */
int fgpu_measure_l2_read(int device, int mb, int passes, double* gbs);

#ifdef __cplusplus
}
#endif
#endif /* FOSITE_GPU_H */
