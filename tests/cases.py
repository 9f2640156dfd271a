"""Small seeded parity cases shared by the oracle and GPU tests.

Every case is a (name, builder) pair; builders return (cfg, pvar, extra) like
fosite_b200.problems.  Sizes are deliberately not multiples of the kernel
tiles so partial tiles and all boundary code paths are exercised.
"""
import numpy as np

from fosite_b200 import abi, problems


def _khi(n=(40, 36), limiter=abi.VANLEER, variables=abi.CONSERVATIVE, theta=1.0, order=abi.LINEAR,
         method=abi.MODIFIED_EULER, tdorder=3, bcs=None, seed=11, me_tol=None):
    c = abi.default_config()
    c.inum, c.jnum, c.knum = n[0], n[1], 1
    c.xmin, c.xmax, c.ymin, c.ymax = -0.5, 0.5, -0.5, 0.5
    c.physics = abi.EULER
    c.gamma = 1.4
    c.limiter = limiter
    c.theta = theta
    c.order = order
    c.variables = variables
    c.method = method
    c.tdorder = tdorder
    c.tol_rel = 10.0 if method == abi.MODIFIED_EULER else 1e-4
    if method != abi.MODIFIED_EULER:
        for v in range(abi.MAXVAR):
            c.tol_abs[v] = 1e-4
    if me_tol is not None:      # modified Euler with embedded error control
        c.tol_rel = me_tol
        for v in range(abi.MAXVAR):
            c.tol_abs[v] = me_tol
    c.cfl = 0.4
    c.stoptime = 1.0e3
    if bcs:
        for f, t in enumerate(bcs):
            c.bc[f] = t
    abi.finalize_config(c)
    X, Y, Z, _ = problems.centers(c)
    rng = np.random.default_rng(seed)
    p = np.zeros((4,) + X.shape)
    band = np.abs(Y) < 0.25
    p[0] = np.where(band, 2.0, 1.0)
    p[1] = np.where(band, 0.5, -0.5) + rng.uniform(-1e-2, 1e-2, X.shape)
    p[2] = 0.05 * np.sin(4 * np.pi * X) + rng.uniform(-1e-2, 1e-2, X.shape)
    p[3] = 2.5 + 0.1 * np.exp(-((X - 0.1) ** 2 + Y ** 2) / 0.01)
    return c, p, {}


def _gauss3d(n=(20, 18, 16), variables=abi.PRIMITIVE, limiter=abi.MONOCENT, method=abi.DORMAND_PRINCE, tdorder=5,
             bcs=None, tol=1e-5, seed=21):
    c = abi.default_config()
    c.inum, c.jnum, c.knum = n
    c.xmin, c.xmax, c.ymin, c.ymax, c.zmin, c.zmax = -0.5, 0.5, -0.5, 0.5, -0.5, 0.5
    for f in range(6):
        c.bc[f] = abi.REFLECTING if bcs is None else bcs[f]
    c.physics = abi.EULER
    c.gamma = 1.4
    c.limiter = limiter
    c.variables = variables
    c.method = method
    c.tdorder = tdorder
    c.tol_rel = tol if method != abi.MODIFIED_EULER else 10.0
    for v in range(abi.MAXVAR):
        c.tol_abs[v] = tol
    c.cfl = 0.4
    c.stoptime = 1.0e3
    abi.finalize_config(c)
    X, Y, Z, _ = problems.centers(c)
    rng = np.random.default_rng(seed)
    p = np.zeros((5,) + X.shape)
    p[0] = 1.0 + 1e-2 * rng.uniform(-1.0, 1.0, X.shape)
    p[1] = 0.05 * rng.uniform(-1.0, 1.0, X.shape)
    p[2] = 0.05 * rng.uniform(-1.0, 1.0, X.shape)
    p[3] = 0.05 * rng.uniform(-1.0, 1.0, X.shape)
    p[4] = 1.0 + 10.0 * np.exp(-((X - 0.05) ** 2 + Y ** 2 + (Z + 0.03) ** 2) / 0.01)
    return c, p, {}


def _disk(n=(32, 48), geometry=abi.LOGCYLINDRICAL, seed=31, hratio=0.05, variables=abi.PRIMITIVE, outbound=0,
          bcs=None, fargo=0):
    c, p, extra = problems.disk2d(nr=n[0], nphi=n[1], seed=seed, hratio=hratio, geometry=geometry, fargo=fargo)
    c.variables = variables
    c.pm_outbound = outbound
    if bcs:
        for f, t in enumerate(bcs):
            c.bc[f] = t
    rng = np.random.default_rng(seed + 1)
    p[1] = 0.01 * rng.uniform(-1, 1, p[1].shape)
    return c, p, extra


def _disk_fargo(n=(32, 48), geometry=abi.LOGCYLINDRICAL, seed=51, variables=abi.PRIMITIVE, tdorder=3,
                bcs=None, limiter=abi.VANLEER):
    c, p, extra = problems.disk2d(nr=n[0], nphi=n[1], seed=seed, geometry=geometry, fargo=1)
    c.variables = variables
    c.tdorder = tdorder
    c.limiter = limiter
    if bcs:
        for f, t in enumerate(bcs):
            c.bc[f] = t
    rng = np.random.default_rng(seed + 1)
    p[1] = 0.01 * rng.uniform(-1, 1, p[1].shape)
    p[2] = p[2] * (1.0 + 0.02 * rng.uniform(-1, 1, p[2].shape))
    return c, p, extra


def _butcher(case, method, tdorder, tol=1e-3):
    """Switch a case to an embedded Butcher scheme (timedisc_rkfehlberg.f90 and its tableaus)
    with relative and absolute tolerance tol."""
    c, p, extra = case
    c.method = method
    c.tdorder = tdorder
    c.tol_rel = tol
    for v in range(abi.MAXVAR):
        c.tol_abs[v] = tol
    return c, p, extra


def _disk_fargo2(n=(32, 40), geometry=abi.CYLINDRICAL, seed=61):
    """FARGO type 2: the user supplies w, here the Keplerian velocity at the cell centres."""
    c, p, extra = _disk_fargo(n=n, geometry=geometry, seed=seed,
                              bcs=[abi.NO_GRADIENTS, abi.REFLECTING, abi.PERIODIC, abi.PERIODIC])
    c.fargo_method = 2
    X, _, _, _ = problems.centers(c)
    x = X[0, 0, :]
    r = np.exp(x) if geometry == abi.LOGCYLINDRICAL else x
    extra["fargo_w"] = np.sqrt(1.0 / r)
    return c, p, extra


def _euler_fargo(n=(36, 40), geometry=abi.CARTESIAN, variables=abi.CONSERVATIVE, fargo=1, seed=71):
    """Ideal-gas FARGO: a sheared box (Cartesian) or an adiabatic disk around a point mass
    (cylindrical); CHECK_PMIN off (its round trip sits between the frame changes)."""
    if geometry == abi.CARTESIAN:
        c, p, extra = _khi(n=n, variables=variables, seed=seed,
                           bcs=[abi.REFLECTING, abi.NO_GRADIENTS, abi.PERIODIC, abi.PERIODIC])
        X, Y, _, _ = problems.centers(c)
        rng = np.random.default_rng(seed)
        p[2] = 1.5 + 0.8 * X + 0.01 * rng.uniform(-1, 1, X.shape)
        p[1] = 0.02 * rng.uniform(-1, 1, X.shape)
    else:
        c, p0, extra = problems.disk2d(nr=n[0], nphi=n[1], seed=seed, geometry=geometry, fargo=0)
        c.physics = abi.EULER
        c.gamma = 1.4
        c.variables = variables
        c.bc[abi.WEST] = abi.NO_GRADIENTS
        c.bc[abi.EAST] = abi.REFLECTING
        abi.finalize_config(c)
        X, _, _, _ = problems.centers(c)
        r = X
        rng = np.random.default_rng(seed)
        p = np.zeros((4,) + X.shape)
        p[0] = p0[0]
        p[1] = 0.01 * rng.uniform(-1, 1, X.shape)
        p[2] = p0[2]
        p[3] = p0[0] * (0.05 ** 2 / r)
        extra = {}
    c.fargo_method = fargo
    c.fargo_direction = 2
    c.checkdata = abi.CHECK_ALL & ~abi.CHECK_PMIN
    return c, p, extra


def _iso3d(n=(18, 16, 20), seed=41):
    c = abi.default_config()
    c.inum, c.jnum, c.knum = n
    c.xmin, c.xmax, c.ymin, c.ymax, c.zmin, c.zmax = 0.0, 1.0, 0.0, 1.2, 0.0, 0.8
    c.bc[:] = [abi.REFLECTING, abi.NO_GRADIENTS, abi.PERIODIC, abi.PERIODIC, abi.ABSORBING, abi.ABSORBING]
    c.physics = abi.EULER_ISOTHERM
    c.csiso = 0.7
    c.limiter = abi.MINMOD
    c.variables = abi.CONSERVATIVE
    c.method = abi.CASH_KARP
    c.tdorder = 5
    c.tol_rel = 1e-4
    for v in range(abi.MAXVAR):
        c.tol_abs[v] = 1e-4
    c.stoptime = 1.0e3
    abi.finalize_config(c)
    X, Y, Z, _ = problems.centers(c)
    rng = np.random.default_rng(seed)
    p = np.zeros((4,) + X.shape)
    p[0] = 1.0 + 0.5 * np.exp(-((X - 0.4) ** 2 + (Y - 0.6) ** 2 + (Z - 0.4) ** 2) / 0.02) + 1e-3 * rng.uniform(-1, 1, X.shape)
    p[1] = 0.1 * rng.uniform(-1, 1, X.shape)
    p[2] = 0.2
    p[3] = 0.1 * rng.uniform(-1, 1, X.shape)
    return c, p, {}


def khi3d(perm=(0, 1, 2), n=8, tsim=30.0, seed=17, re=1.0e4):
    """tests/KHI3D.f90: a periodic 3D shear layer (flow along axis a, density and velocity
    jump across axis b), Euler gamma 1.4, KT + MC(theta 1.2) on conservative variables,
    SSPRK3 with CFL 0.4 and the test's molecular viscosity for Reynolds number re
    (None: inviscid).  perm maps the base orientation (flow along x, jump across y) to
    another axis order; the same seeded velocity noise is permuted with it, so the six
    runs are images of each other.  Returns (cfg, pvar, perm)."""
    c = abi.default_config()
    c.inum = c.jnum = c.knum = n
    c.xmin, c.xmax, c.ymin, c.ymax, c.zmin, c.zmax = -0.5, 0.5, -0.5, 0.5, -0.5, 0.5
    for f in range(6):
        c.bc[f] = abi.PERIODIC
    c.physics = abi.EULER
    c.gamma = 1.4
    c.limiter = abi.MONOCENT
    c.theta = 1.2
    c.variables = abi.CONSERVATIVE
    c.method = abi.MODIFIED_EULER
    c.tdorder = 3
    c.tol_rel = 10.0
    c.cfl = 0.4
    c.stoptime = tsim
    c.dtlimit = 1e-10
    if re is not None:
        eta = khi_reynolds(re)
        c.vismodel = abi.VIS_MOLECULAR
        c.dynconst = eta
        c.bulkconst = -2. / 3. * eta
    abi.finalize_config(c)
    X, Y, Z, _ = problems.centers(c)
    rng = np.random.default_rng(seed)
    dv = rng.uniform(0.0, 1.0, (3,) + X.shape)
    # base orientation in [v, z, y, x] order: flow along x, jump across y
    inner = ~((Y < -0.25) | (Y > 0.25))
    base = np.zeros((5,) + X.shape)
    base[0] = np.where(inner, 2.0, 1.0)
    base[1] = np.where(inner, 0.5, -0.5)
    base[4] = 2.5
    base[1:4] = base[1:4] + (dv - 0.5) * 0.2
    return c, permute_state(base, perm), perm


def permute_state(p, perm):
    """Relabel axes: new axis a carries old axis perm[a] (coordinates and velocity
    components); arrays are [v, z, y, x]."""
    spatial = [2 - perm[2 - d] for d in range(3)]       # array axis order (z, y, x)
    q = p[:, :, :, :].transpose([0] + [1 + s for s in spatial])
    out = q.copy()
    for a in range(3):
        out[1 + a] = q[1 + perm[a]]
    return out


def inverse_perm(perm):
    inv = [0, 0, 0]
    for a, b in enumerate(perm):
        inv[b] = a
    return tuple(inv)


def _visc(case, dynconst, bulkconst=None, cvis=0.5):
    """Add the MOLECULAR viscosity source (sources_viscosity.f90); bulkconst None keeps
    fosite's default -2/3*dynconst."""
    c, p, extra = case
    c.vismodel = abi.VIS_MOLECULAR
    c.dynconst = dynconst
    if bulkconst is not None:
        c.bulkconst = bulkconst
    c.cvis = cvis
    return c, p, extra


def _visc_model(case, model, dynconst, exponent=0.0, cvis=0.5, **kw):
    """Add an ALPHA/BETA/POWERLAW viscosity (sources_viscosity.f90:359-453) and set other keys."""
    c, p, extra = case
    c.vismodel = model
    c.dynconst = dynconst
    c.vis_exponent = exponent
    c.cvis = cvis
    for k, v in kw.items():
        setattr(c, k, v)
    return c, p, extra


def khi_reynolds(re=1.0e4, rho0=1.0, xyzlen=1.0, v0=-0.5, v1=0.5):
    """Dynamic viscosity of tests/KHI2D.f90:236-239 and tests/KHI3D.f90:328-331."""
    return abs(rho0 * xyzlen * (v0 - v1) / re)


def _iso_fargo_x(n=(40, 30), fargo=1, seed=83):
    """Isothermal shear flow along x with FARGO transport along x (direction 1): periodic in
    x, reflecting in y, v_x = 1 + 0.8 y plus noise (a sheared background that FARGO follows)."""
    c = abi.default_config()
    c.inum, c.jnum, c.knum = n[0], n[1], 1
    c.xmin, c.xmax, c.ymin, c.ymax = 0.0, 2.0, -0.5, 0.5
    c.physics = abi.EULER_ISOTHERM
    c.csiso = 0.6
    c.limiter = abi.VANLEER
    c.variables = abi.PRIMITIVE
    c.method = abi.MODIFIED_EULER
    c.tdorder = 3
    c.tol_rel = 10.0
    c.cfl = 0.4
    c.stoptime = 1.0e3
    c.bc[:4] = [abi.PERIODIC, abi.PERIODIC, abi.REFLECTING, abi.REFLECTING]
    c.fargo_method = fargo
    c.fargo_direction = 1
    abi.finalize_config(c)
    X, Y, _, _ = problems.centers(c)
    rng = np.random.default_rng(seed)
    p = np.zeros((3,) + X.shape)
    p[0] = 1.0 + 0.1 * np.sin(np.pi * X) + 0.01 * rng.uniform(-1, 1, X.shape)
    p[1] = 1.0 + 0.8 * Y + 0.02 * rng.uniform(-1, 1, X.shape)
    p[2] = 0.02 * rng.uniform(-1, 1, X.shape)
    return c, p, {}


def _axis_disk(n=(28, 36), euler=False, seed=91):
    """A rotating gas on a cylindrical mesh reaching the axis: r in [0, 1] with the AXIS
    boundary at r = 0 (boundary_axis.f90), reflecting at r = 1, periodic in phi; no point mass."""
    c = abi.default_config()
    c.inum, c.jnum, c.knum = n[0], n[1], 1
    c.geometry = abi.CYLINDRICAL
    c.xmin, c.xmax, c.ymin, c.ymax = 0.0, 1.0, -np.pi, np.pi
    c.physics = abi.EULER if euler else abi.EULER_ISOTHERM
    c.gamma = 1.4
    c.csiso = 0.0 if euler else 0.5
    c.limiter = abi.VANLEER
    c.variables = abi.PRIMITIVE
    c.method = abi.MODIFIED_EULER
    c.tdorder = 3
    c.tol_rel = 10.0
    c.cfl = 0.4
    c.stoptime = 1.0e3
    c.bc[:4] = [abi.AXIS, abi.REFLECTING, abi.PERIODIC, abi.PERIODIC]
    abi.finalize_config(c)
    X, Y, _, _ = problems.centers(c)
    rng = np.random.default_rng(seed)
    p = np.zeros((4 if euler else 3,) + X.shape)
    p[0] = 1.0 + 0.3 * np.exp(-((X - 0.4) ** 2) / 0.02) * (1 + np.cos(Y)) + 0.01 * rng.uniform(-1, 1, X.shape)
    p[1] = 0.05 * rng.uniform(-1, 1, X.shape)
    p[2] = 0.5 * X * np.exp(-X ** 2) + 0.02 * rng.uniform(-1, 1, X.shape)
    if euler:
        p[3] = 1.0 + 0.2 * np.exp(-((X - 0.5) ** 2) / 0.01)
    return c, p, {}


def _axis_cyl3d(n=(16, 20, 12), seed=93):
    """A 3D cylindrical mesh (r, phi, z) reaching the axis: AXIS at r = 0, reflecting at r = 1,
    periodic in phi, reflecting in z; isothermal rotating gas with a density bump."""
    c = abi.default_config()
    c.inum, c.jnum, c.knum = n
    c.geometry = abi.CYLINDRICAL
    c.xmin, c.xmax, c.ymin, c.ymax, c.zmin, c.zmax = 0.0, 1.0, -np.pi, np.pi, 0.0, 1.0
    c.physics = abi.EULER_ISOTHERM
    c.csiso = 0.5
    c.limiter = abi.VANLEER
    c.variables = abi.PRIMITIVE
    c.method = abi.MODIFIED_EULER
    c.tdorder = 3
    c.tol_rel = 10.0
    c.cfl = 0.4
    c.stoptime = 1.0e3
    c.bc[:6] = [abi.AXIS, abi.REFLECTING, abi.PERIODIC, abi.PERIODIC, abi.REFLECTING, abi.REFLECTING]
    abi.finalize_config(c)
    X, Y, Z, _ = problems.centers(c)
    rng = np.random.default_rng(seed)
    p = np.zeros((4,) + X.shape)
    p[0] = (1.0 + 0.3 * np.exp(-((X - 0.4) ** 2 + (Z - 0.5) ** 2) / 0.02) * (1 + np.cos(Y))
            + 0.01 * rng.uniform(-1, 1, X.shape))
    p[1] = 0.05 * rng.uniform(-1, 1, X.shape)
    p[2] = 0.5 * X * np.exp(-X ** 2) + 0.02 * rng.uniform(-1, 1, X.shape)
    p[3] = 0.02 * rng.uniform(-1, 1, X.shape)
    return c, p, {}


def _axis_fargo(n=(28, 36), fargo=1, seed=95):
    """The axis disk with FARGO transport along phi (type 1: the background velocity includes
    the axis ghost columns)."""
    c, p, extra = _axis_disk(n=n, seed=seed)
    c.fargo_method = fargo
    c.fargo_direction = 2
    abi.finalize_config(c)
    return c, p, extra


def khi_fargo(fargo, direction=1, n=(24, 24), visc=False, seed=11):
    """tests/KHI2D.f90's FARGO legs (:81-150, config :168-245, InitData :300-360): ideal-gas KHI,
    KT + MONOCENT (theta 1.2) on conservative variables, periodic box, FARGO type 1 or 2 along
    x (direction 1: shear layer along x, bands in y) or, for the transposed run, along y
    (direction 2: everything transposed), optionally with the test's molecular viscosity.
    Type 2 takes the band velocity as background velocity (InitData :323-331); CHECK_PMIN off
    (its round trip sits between the frame changes)."""
    cfg, p, extra = _khi(n=n, limiter=abi.MONOCENT, theta=1.2, seed=seed)
    cfg.fargo_method = fargo
    cfg.fargo_direction = 1
    cfg.checkdata = abi.CHECK_ALL & ~abi.CHECK_PMIN
    if visc:
        eta = khi_reynolds()
        cfg, p, extra = _visc((cfg, p, extra), eta, bulkconst=-2. / 3. * eta)
    # background velocity by padded j: the band velocity at the padded cell centres
    dy = (cfg.ymax - cfg.ymin) / cfg.jnum
    y = cfg.ymin + (np.arange(cfg.jnum + 4) - 1.5) * dy
    w = np.where(np.abs(y) < 0.25, 0.5, -0.5)
    if fargo == 2:
        extra = dict(extra, fargo_w=w)
    if direction == 2:
        cfg.inum, cfg.jnum = cfg.jnum, cfg.inum
        cfg.xmin, cfg.xmax, cfg.ymin, cfg.ymax = cfg.ymin, cfg.ymax, cfg.xmin, cfg.xmax
        cfg.fargo_direction = 2
        abi.finalize_config(cfg)
        p = np.stack([p[0], p[2], p[1], p[3]]).transpose(0, 1, 3, 2).copy()
    return cfg, p, extra


def _with(case, **kw):
    c, p, extra = case
    for k, v in kw.items():
        setattr(c, k, v)
    return c, p, extra


CASES = {
    "khi_ssprk3_vanleer_cons": lambda: _khi(),
    "khi_ssprk3_mc_prim": lambda: _khi(limiter=abi.MONOCENT, variables=abi.PRIMITIVE, theta=1.2),
    "khi_superbee": lambda: _khi(limiter=abi.SUPERBEE, n=(33, 35)),
    "khi_sweby": lambda: _khi(limiter=abi.SWEBY, theta=1.5, n=(24, 40)),
    "khi_ospre": lambda: _khi(limiter=abi.OSPRE, n=(31, 17)),
    "khi_nolimit_order2": lambda: _khi(limiter=abi.NOLIMIT, tdorder=2),
    "khi_constant_order1": lambda: _khi(order=abi.CONSTANT, tdorder=1),
    "euler2d_absorbing": lambda: _khi(bcs=[abi.ABSORBING] * 4, variables=abi.PRIMITIVE, n=(36, 34)),
    "euler2d_reflect_nograd_ssprk5": lambda: _khi(bcs=[abi.REFLECTING, abi.REFLECTING, abi.NO_GRADIENTS, abi.NO_GRADIENTS],
                                                 method=abi.SSPRK, tdorder=5, n=(30, 26)),
    "euler2d_rkf45": lambda: _khi(method=abi.RK_FEHLBERG, tdorder=5, n=(28, 30)),
    "khi_modeuler_adaptive3": lambda: _khi(me_tol=1e-3),
    "khi_checkdata_no_pmin": lambda: _with(_khi(variables=abi.PRIMITIVE, n=(30, 28)),
                                           checkdata=abi.CHECK_ALL & ~abi.CHECK_PMIN),
    "gauss3d_dopri_no_pmin": lambda: _with(_gauss3d(n=(12, 14, 10)), checkdata=abi.CHECK_NOTHING),
    "khi_modeuler_adaptive2_mc_prim": lambda: _khi(tdorder=2, me_tol=1e-3, limiter=abi.MONOCENT,
                                                  variables=abi.PRIMITIVE, n=(34, 30)),
    "gauss3d_dopri_mc_prim": lambda: _gauss3d(),
    "gauss3d_rkf3_minmod_cons": lambda: _gauss3d(variables=abi.CONSERVATIVE, limiter=abi.MINMOD, method=abi.RK_FEHLBERG,
                                                tdorder=3, n=(17, 20, 14),
                                                bcs=[abi.REFLECTING, abi.REFLECTING, abi.NO_GRADIENTS, abi.NO_GRADIENTS,
                                                     abi.PERIODIC, abi.PERIODIC]),
    "gauss3d_ssprk3_absorbing": lambda: _gauss3d(method=abi.MODIFIED_EULER, tdorder=3, limiter=abi.VANLEER,
                                                bcs=[abi.ABSORBING] * 6, n=(16, 14, 18)),
    "disk_logcyl_pointmass": lambda: _disk(),
    "disk_cyl_pointmass_cons": lambda: _disk(geometry=abi.CYLINDRICAL, n=(40, 32), variables=abi.CONSERVATIVE),
    "iso3d_cashkarp_mixed_bc": lambda: _iso3d(),
    "disk_accretion_west_nograd": lambda: _disk(n=(36, 40), outbound=1,
                                                bcs=[abi.NO_GRADIENTS, abi.REFLECTING, abi.PERIODIC, abi.PERIODIC]),
    "disk_accretion_east_cyl_fargo": lambda: _disk(n=(30, 44), geometry=abi.CYLINDRICAL, outbound=2, fargo=1,
                                                   bcs=[abi.REFLECTING, abi.NO_GRADIENTS, abi.PERIODIC, abi.PERIODIC]),
    "disk_fargo_logcyl": lambda: _disk_fargo(),
    "disk_fargo_cyl_cons_reflect": lambda: _disk_fargo(geometry=abi.CYLINDRICAL, n=(36, 40), variables=abi.CONSERVATIVE,
                                                       bcs=[abi.REFLECTING, abi.NO_GRADIENTS, abi.PERIODIC, abi.PERIODIC],
                                                       limiter=abi.MONOCENT),
    "disk_fargo2_user_w": lambda: _disk_fargo2(),
    "euler_fargo_shear_cons": lambda: _euler_fargo(),
    "khi_fargo1_x": lambda: khi_fargo(1, n=(28, 24)),
    "iso_axis_cyl": lambda: _axis_disk(),
    "iso_axis_cyl3d": lambda: _axis_cyl3d(),
    "iso_axis_cyl_fargo": lambda: _axis_fargo(),
    "euler_axis_cyl_dopri": lambda: _butcher(_axis_disk(n=(24, 32), euler=True), abi.DORMAND_PRINCE, 5, 1e-4),
    "disk_fargo_ssprk5_logcyl": lambda: _butcher(_disk_fargo(), abi.SSPRK, 5),
    "disk_fargo2_dopri_cyl": lambda: _butcher(_disk_fargo2(), abi.DORMAND_PRINCE, 5, 1e-4),
    "euler_fargo_rkf5_shear": lambda: _butcher(_euler_fargo(), abi.RK_FEHLBERG, 5, 1e-4),
    "khi_fargo1_x_cashkarp": lambda: _butcher(khi_fargo(1, n=(24, 26)), abi.CASH_KARP, 5, 1e-4),
    "disk_fargo_me3_adaptive": lambda: _butcher(_disk_fargo(n=(30, 40)), abi.MODIFIED_EULER, 3, 1e-3),
    "khi_fargo2_x_me3_adaptive": lambda: _butcher(khi_fargo(2, n=(26, 24)), abi.MODIFIED_EULER, 3, 1e-4),
    "disk_fargo2_me2_adaptive": lambda: _butcher(_disk_fargo2(), abi.MODIFIED_EULER, 2, 1e-3),
    "khi_fargo2_x_visc": lambda: khi_fargo(2, n=(24, 26), visc=True),
    "iso_fargo1_x_shear": lambda: _iso_fargo_x(),
    "euler_fargo1_x_disk_cyl": lambda: _with(_euler_fargo(n=(24, 40), geometry=abi.CYLINDRICAL), fargo_direction=1),
    "euler_fargo_disk_cyl_prim": lambda: _euler_fargo(n=(24, 160), geometry=abi.CYLINDRICAL, variables=abi.PRIMITIVE),
    "disk_fargo_order1_minmod": lambda: _disk_fargo(n=(30, 44), tdorder=1, limiter=abi.MINMOD,
                                                    bcs=[abi.REFLECTING, abi.REFLECTING, abi.PERIODIC, abi.PERIODIC]),
    # molecular viscosity (sources_viscosity.f90); the first is the KHI2D test's set-up
    "khi_visc_re1e4_mc": lambda: _visc(_khi(limiter=abi.MONOCENT, theta=1.2, n=(32, 30)), khi_reynolds(),
                                       bulkconst=-2. / 3. * khi_reynolds()),
    "khi_visc_dominant_reflect_prim": lambda: _visc(_khi(variables=abi.PRIMITIVE, n=(30, 28),
                                                         bcs=[abi.REFLECTING, abi.REFLECTING, abi.NO_GRADIENTS,
                                                              abi.NO_GRADIENTS]), 0.05, cvis=0.4),
    "khi_visc_rkf45_absorbing": lambda: _visc(_khi(method=abi.RK_FEHLBERG, tdorder=5, n=(26, 24),
                                                   bcs=[abi.ABSORBING] * 4), 5e-3, bulkconst=1e-3),
    "khi_visc_adaptive_me": lambda: _visc(_khi(me_tol=1e-3, n=(28, 26)), 2e-3),
    "gauss3d_visc_dopri": lambda: _visc(_gauss3d(n=(14, 12, 10)), 2e-3),
    "iso3d_visc_ssprk3_mixed_bc": lambda: _visc(_with(_iso3d(n=(14, 12, 16)), method=abi.MODIFIED_EULER, tdorder=3,
                                                      tol_rel=10.0), 1e-2),
    "disk_visc_logcyl_pointmass": lambda: _visc(_disk(bcs=[abi.NO_GRADIENTS, abi.REFLECTING, abi.PERIODIC,
                                                           abi.PERIODIC]), 1e-3),
    "disk_visc_fargo_cyl_cons": lambda: _visc(_disk_fargo(geometry=abi.CYLINDRICAL, n=(30, 36),
                                                          variables=abi.CONSERVATIVE,
                                                          bcs=[abi.REFLECTING, abi.NO_GRADIENTS, abi.PERIODIC,
                                                               abi.PERIODIC]), 2e-3),
    "euler_disk_cyl_visc_prim": lambda: _visc(_euler_fargo(n=(24, 40), geometry=abi.CYLINDRICAL,
                                                           variables=abi.PRIMITIVE, fargo=0), 1e-3),
    # state-dependent viscosities with UpdateViscosity's time caching; the first is the
    # set-up of tests/pringle.f90 (cylindrical disk, POWERLAW q = 0, SSPRK, tolerances)
    "disk_powerlaw_pringle_ssprk5": lambda: _visc_model(
        _disk(geometry=abi.CYLINDRICAL, n=(30, 36), bcs=[abi.NO_GRADIENTS, abi.REFLECTING, abi.PERIODIC, abi.PERIODIC]),
        abi.VIS_POWERLAW, 1e-3, 0.0, cvis=0.3, method=abi.SSPRK, tdorder=5, tol_rel=0.01),
    "disk_beta_logcyl_me3": lambda: _visc_model(
        _disk(bcs=[abi.NO_GRADIENTS, abi.REFLECTING, abi.PERIODIC, abi.PERIODIC]), abi.VIS_BETA, 1e-3),
    "disk_alpha_cyl_me2": lambda: _visc_model(
        _disk(geometry=abi.CYLINDRICAL, n=(28, 40), bcs=[abi.REFLECTING, abi.NO_GRADIENTS, abi.PERIODIC, abi.PERIODIC]),
        abi.VIS_ALPHA, 1e-2, tdorder=2),
    "disk_powerlaw_q05_adaptive_me": lambda: _visc_model(
        _disk(geometry=abi.CYLINDRICAL, n=(26, 32), bcs=[abi.REFLECTING, abi.REFLECTING, abi.PERIODIC, abi.PERIODIC]),
        abi.VIS_POWERLAW, 2e-3, 0.5, tol_rel=1e-3),
    "khi_powerlaw_me1": lambda: _visc_model(_khi(order=abi.CONSTANT, tdorder=1, n=(30, 26)), abi.VIS_POWERLAW, 1e-3, 0.0),
    "iso3d_beta_dopri": lambda: _visc_model(
        _with(_iso3d(n=(12, 14, 10)), method=abi.DORMAND_PRINCE,
              bc=(abi.REFLECTING, abi.NO_GRADIENTS, abi.PERIODIC, abi.PERIODIC, abi.REFLECTING, abi.NO_GRADIENTS)),
        abi.VIS_BETA, 1e-2),
}


def fixed_step(cfg):
    return cfg.method == abi.MODIFIED_EULER


def fix_modeuler(c):
    if c.method == abi.MODIFIED_EULER:
        c.tol_rel = 10.0
    return c
