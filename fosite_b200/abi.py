"""ctypes mirror of include/fosite_gpu.h.

The structs and constants below are the Python view of the C ABI; the same
definitions are used to drive the CUDA library (``libfosite_gpu.so``) and,
from the tests only, the CPU oracle, because both take the same flat config.
"""
import ctypes as C

# fosite identifiers (same values as the Fortran code, see the header)
CARTESIAN, CYLINDRICAL, LOGCYLINDRICAL = 1, 30, 31
EULER_ISOTHERM, EULER = 16, 17
KT = 1
CONSTANT, LINEAR = 1, 2
PRIMITIVE, CONSERVATIVE = 1, 2
MINMOD, MONOCENT, SWEBY, SUPERBEE, OSPRE, PP, VANLEER, NOLIMIT = 1, 2, 3, 4, 5, 6, 7, 8
NO_GRADIENTS, PERIODIC, REFLECTING, ABSORBING = 0x01, 0x02, 0x03, 0x0D
AXIS = 0x04
WEST, EAST, SOUTH, NORTH, BOTTOM, TOP = 0, 1, 2, 3, 4, 5
MODIFIED_EULER, RK_FEHLBERG, CASH_KARP, DORMAND_PRINCE, SSPRK = 1, 2, 3, 4, 5
CHECK_NOTHING, CHECK_CSOUND, CHECK_PMIN, CHECK_RHOMIN, CHECK_INVALID, CHECK_TMIN, CHECK_ALL = \
    0x00, 0x01, 0x02, 0x04, 0x08, 0x10, 0xFF

OK, BREAK, STOPTIME = 0, 1, 2
EBADCFG, ENOMEM, ECUDA, ETIMEOUT, EUNSUPPORTED, EARG = -1, -2, -3, -4, -5, -6

DTCAUSE_CFL, DTCAUSE_ERRADJ, DTCAUSE_SMALLERR, DTCAUSE_FILEIO, DTCAUSE_VISCOSITY = 0, -1, -2, -4, 3
VIS_MOLECULAR, VIS_ALPHA, VIS_BETA, VIS_POWERLAW, VIS_ALPHA_ALT = 1, 2, 3, 4, 5

CVAR, PVAR, RHS, BCCSOUND = 1, 2, 3, 4
XFLUX, YFLUX, ZFLUX = 5, 6, 7     # interface fluxes of the last compute_rhs (fosite xfluxdydz ...)
MESH_X, MESH_Y, MESH_Z, MESH_RADIUS = 10, 11, 12, 13

MAXVAR = 5
TINY = 2.2250738585072014e-308
EPSILON = 2.220446049250313e-16


class Config(C.Structure):
    """fgpu_config: flat mirror of the fosite Dict keys on the step path."""
    _fields_ = [
        ("inum", C.c_int32), ("jnum", C.c_int32), ("knum", C.c_int32),
        ("geometry", C.c_int32),
        ("xmin", C.c_double), ("xmax", C.c_double), ("ymin", C.c_double),
        ("ymax", C.c_double), ("zmin", C.c_double), ("zmax", C.c_double),
        ("gparam", C.c_double),
        ("physics", C.c_int32),
        ("gamma", C.c_double), ("csiso", C.c_double), ("gn", C.c_double),
        ("fluxtype", C.c_int32), ("order", C.c_int32), ("variables", C.c_int32),
        ("limiter", C.c_int32),
        ("theta", C.c_double),
        ("bc", C.c_int32 * 6),
        ("method", C.c_int32), ("tdorder", C.c_int32),
        ("cfl", C.c_double), ("stoptime", C.c_double), ("dtlimit", C.c_double),
        ("tol_rel", C.c_double),
        ("tol_abs", C.c_double * MAXVAR),
        ("beta", C.c_double),
        ("maxiter", C.c_int32), ("checkdata", C.c_int32),
        ("pmin", C.c_double), ("rhomin", C.c_double), ("tmin", C.c_double),
        ("pointmass", C.c_int32),
        ("pm_mass", C.c_double),
        ("fargo_method", C.c_int32), ("fargo_direction", C.c_int32),
        ("tout", C.c_double),
        ("pm_outbound", C.c_int32), ("pad_", C.c_int32),
        ("starttime", C.c_double),
        ("vismodel", C.c_int32), ("pad2_", C.c_int32),
        ("dynconst", C.c_double), ("bulkconst", C.c_double),
        ("vis_exponent", C.c_double), ("cvis", C.c_double),
    ]


class Status(C.Structure):
    """fgpu_status: Timedisc bookkeeping after a step."""
    _fields_ = [
        ("time", C.c_double), ("dt", C.c_double), ("dtold", C.c_double),
        ("dtmin", C.c_double), ("maxerr", C.c_double),
        ("iter", C.c_int64), ("n_adj", C.c_int64),
        ("dtcause", C.c_int32), ("brk", C.c_int32), ("checkflags", C.c_int32),
        ("pad", C.c_int32),
    ]


class Stats(C.Structure):
    """fgpu_stats: launch counts and CUDA-event kernel timing."""
    _fields_ = [
        ("launches", C.c_int64), ("stage_launches", C.c_int64), ("attempts", C.c_int64),
        ("cell_updates", C.c_int64), ("stage_ms", C.c_double), ("stage_bytes", C.c_double),
        ("other_ms", C.c_double), ("form_ms", C.c_double),
    ]


def default_config():
    """fosite's GetAttr defaults (timedisc_base.f90:285-350 and friends)."""
    c = Config()
    c.inum = c.jnum = c.knum = 1
    c.geometry = CARTESIAN
    c.gparam = 1.0
    c.physics = EULER
    c.gamma = 1.4
    c.csiso = 0.0
    c.gn = 1.0
    c.fluxtype = KT
    c.order = LINEAR
    c.variables = CONSERVATIVE
    c.limiter = MINMOD
    c.theta = 1.0
    for f in range(6):
        c.bc[f] = PERIODIC
    c.method = MODIFIED_EULER
    c.tdorder = 0
    c.cfl = 0.4
    c.stoptime = 1.0
    c.dtlimit = 0.0        # filled as EPSILON*stoptime by finalize_config
    c.tol_rel = 0.01
    c.beta = 0.08
    for v in range(MAXVAR):
        c.tol_abs[v] = 0.001
    c.maxiter = 0
    c.checkdata = CHECK_ALL
    c.pmin = c.rhomin = c.tmin = TINY
    c.pointmass = 0
    c.pm_mass = 1.0
    c.fargo_method = 0
    c.fargo_direction = 0
    c.tout = 0.0
    c.vismodel = 0
    c.dynconst = 0.1
    c.bulkconst = float("nan")   # fosite's default -2/3*dynconst
    c.vis_exponent = 0.0
    c.cvis = 0.5
    return c


def finalize_config(c):
    """Apply defaults that depend on other keys (dtlimit = EPSILON*stoptime)."""
    if c.dtlimit <= 0.0:
        c.dtlimit = EPSILON * c.stoptime
    return c


def config_copy(c):
    n = Config()
    C.memmove(C.byref(n), C.byref(c), C.sizeof(Config))
    return n
