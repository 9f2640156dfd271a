"""Seeded synthetic initial data for the benchmark workloads.

Each builder returns ``(cfg, pvar, extra)``: a config, the ghost-padded
primitive state (fosite's Timedisc%pvar layout: [VNUM, KG, JG, IG]) and, for
locally isothermal disks, the sound-speed arrays of
physics_eulerisotherm%SetSoundSpeeds.  The data follow the recipes of the
fosite test/example programs they stand in for (tests/KHI2D.f90:285-375,
tests/gauss3d.f90, examples/mmsn.f90:255-300); noise is drawn from numpy's
PCG64 with the stated seed so every run sees the same input.
"""
import numpy as np

from . import abi


def padded_shape(cfg):
    g = lambda n: 2 if n > 1 else 0
    return (cfg.knum + 2 * g(cfg.knum), cfg.jnum + 2 * g(cfg.jnum), cfg.inum + 2 * g(cfg.inum))


def centers(cfg):
    """Curvilinear cell-centre coordinates, mesh_base.f90:648-660 (ghost-padded)."""
    def axis(n, lo, hi):
        d = (hi - lo) / n
        md = d if d >= 2 * abi.EPSILON else 0.0
        g = 2 if n > 1 else 0
        idx = np.arange(1 - g, n + g + 1, dtype=np.float64)   # fosite 1-based indices
        return lo + ((2 * idx - 1) * 0.5) * md, md
    x, mdx = axis(cfg.inum, cfg.xmin, cfg.xmax)
    y, mdy = axis(cfg.jnum, cfg.ymin, cfg.ymax)
    z, mdz = axis(cfg.knum, cfg.zmin, cfg.zmax)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    return X, Y, Z, (mdx, mdy, mdz)


def _base(n, nd):
    c = abi.default_config()
    c.inum = n[0]
    c.jnum = n[1]
    c.knum = n[2] if nd == 3 else 1
    return c


def with_viscosity(c, re, rho0=1.0, xyzlen=1.0, dv=1.0):
    """The molecular viscosity of tests/KHI2D.f90:236-239 / tests/KHI3D.f90:328-331:
    dynconst = |rho0 * L * (V0 - V1) / RE|, bulk viscosity -2/3 of it."""
    eta = abs(rho0 * xyzlen * (-dv) / re)
    c.vismodel = abi.VIS_MOLECULAR
    c.dynconst = eta
    c.bulkconst = -2. / 3. * eta
    return c


def khi2d(n=256, seed=1000, steps=1000, re=None):
    """2D Kelvin-Helmholtz, Euler gamma=1.4, periodic, KT + van Leer, SSPRK3 fixed CFL 0.4;
    re: Reynolds number of the molecular viscosity (None: inviscid)."""
    c = _base((n, n, 1), 2)
    c.xmin, c.xmax, c.ymin, c.ymax = -0.5, 0.5, -0.5, 0.5
    c.physics = abi.EULER
    c.gamma = 1.4
    c.limiter = abi.VANLEER
    c.variables = abi.CONSERVATIVE
    c.method = abi.MODIFIED_EULER
    c.tdorder = 3
    c.tol_rel = 10.0          # fixed step size (timedisc_modeuler.f90:146)
    c.cfl = 0.4
    c.stoptime = 1.0e3        # the run length is set by the step count
    abi.finalize_config(c)
    X, Y, Z, _ = centers(c)
    rng = np.random.default_rng(seed)
    p = np.zeros((4,) + X.shape)
    band = np.abs(Y) < 0.25
    p[0] = np.where(band, 2.0, 1.0)
    p[1] = np.where(band, 0.5, -0.5) + rng.uniform(-1e-3, 1e-3, X.shape)
    p[2] = 0.01 * np.sin(4 * np.pi * X) + rng.uniform(-1e-3, 1e-3, X.shape)
    p[3] = 2.5
    if re is not None:
        with_viscosity(c, re)
    return c, p, {"steps": steps}


def khi3d(n=128, seed=1500, re=1.0e4):
    """tests/KHI3D.f90: periodic 3D shear layer (flow along x, jump across y), Euler gamma 1.4,
    KT + MC(theta 1.2) on conservative variables, SSPRK3 fixed CFL 0.4, the test's molecular
    viscosity (RE = 1e4; None: inviscid) and seeded velocity noise of amplitude 0.1."""
    c = _base((n, n, n), 3)
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
    c.stoptime = 1.0e3
    if re is not None:
        with_viscosity(c, re)
    abi.finalize_config(c)
    X, Y, Z, _ = centers(c)
    rng = np.random.default_rng(seed)
    inner = np.abs(Y) <= 0.25
    p = np.zeros((5,) + X.shape)
    p[0] = np.where(inner, 2.0, 1.0)
    p[1] = np.where(inner, 0.5, -0.5) + (rng.uniform(0.0, 1.0, X.shape) - 0.5) * 0.2
    p[2] = (rng.uniform(0.0, 1.0, X.shape) - 0.5) * 0.2
    p[3] = (rng.uniform(0.0, 1.0, X.shape) - 0.5) * 0.2
    p[4] = 2.5
    return c, p, {}


def gauss3d(n=256, seed=2000, mc_theta=1.0, method=None):
    """3D Euler Gaussian pressure pulse, reflecting walls, KT + MC, Dormand-Prince (tol 1e-5).

    method=abi.MODIFIED_EULER gives the fixed-step SSPRK3 variant (CFL 0.4) that
    batched ensembles and the serving loop use.
    """
    c = _base((n, n, n), 3)
    c.xmin, c.xmax, c.ymin, c.ymax, c.zmin, c.zmax = -0.5, 0.5, -0.5, 0.5, -0.5, 0.5
    for f in range(6):
        c.bc[f] = abi.REFLECTING
    c.physics = abi.EULER
    c.gamma = 1.4
    c.limiter = abi.MONOCENT
    c.theta = mc_theta
    c.variables = abi.PRIMITIVE
    c.method = abi.DORMAND_PRINCE
    c.tdorder = 5
    c.tol_rel = 1e-5
    for v in range(abi.MAXVAR):
        c.tol_abs[v] = 1e-5
    if method == abi.MODIFIED_EULER:
        c.method = abi.MODIFIED_EULER
        c.tdorder = 3
        c.tol_rel = 10.0
    c.cfl = 0.4
    c.stoptime = 1.0e3
    abi.finalize_config(c)
    X, Y, Z, _ = centers(c)
    rng = np.random.default_rng(seed)
    p = np.zeros((5,) + X.shape)
    r2 = X * X + Y * Y + Z * Z
    p[0] = 1.0 + 1e-4 * rng.uniform(-1.0, 1.0, X.shape)
    p[4] = 1.0 + 10.0 * np.exp(-r2 / 0.01)
    return c, p, {}


def disk2d(nr=512, nphi=1024, seed=3000, hratio=0.05, sigma_index=-1.0, geometry=abi.LOGCYLINDRICAL,
           fargo=1, rmin=0.4, rmax=2.5):
    """2D locally isothermal Keplerian disk around a unit point mass (GM = 1)."""
    c = _base((nr, nphi, 1), 2)
    c.geometry = geometry
    if geometry == abi.LOGCYLINDRICAL:
        c.xmin, c.xmax = float(np.log(rmin)), float(np.log(rmax))
    else:
        c.xmin, c.xmax = rmin, rmax
    c.ymin, c.ymax = -np.pi, np.pi
    c.bc[abi.WEST] = abi.ABSORBING
    c.bc[abi.EAST] = abi.ABSORBING
    c.bc[abi.SOUTH] = abi.PERIODIC
    c.bc[abi.NORTH] = abi.PERIODIC
    c.physics = abi.EULER_ISOTHERM
    c.csiso = 0.0
    c.gn = 1.0
    c.pointmass = 1
    c.pm_mass = 1.0
    c.limiter = abi.VANLEER
    c.variables = abi.PRIMITIVE
    c.method = abi.MODIFIED_EULER
    c.tdorder = 3
    c.tol_rel = 10.0
    c.cfl = 0.4
    c.stoptime = 1.0e3
    if fargo:
        c.fargo_method = fargo
        c.fargo_direction = 2
    abi.finalize_config(c)
    X, Y, Z, (mdx, mdy, mdz) = centers(c)

    def radius(x):
        return np.exp(x) if geometry == abi.LOGCYLINDRICAL else x
    r = radius(X)
    cs_c = hratio * np.sqrt(1.0 / r)
    faces = []
    for off in (-0.5 * mdx, 0.5 * mdx):
        faces.append(hratio * np.sqrt(1.0 / radius(X + off)))
    faces.append(cs_c)   # south
    faces.append(cs_c)   # north
    fcs = np.stack(faces)
    rng = np.random.default_rng(seed)
    p = np.zeros((3,) + X.shape)
    p[0] = r ** sigma_index * (1.0 + 1e-3 * rng.uniform(-1.0, 1.0, X.shape))
    # Keplerian rotation, pressure corrected for sigma ~ r^s, cs^2 ~ 1/r: v^2 = GM/r (1 - (1 - s) h^2)
    p[2] = np.sqrt(1.0 / r) * np.sqrt(1.0 - (1.0 - sigma_index) * hratio * hratio)
    return c, p, {"bccsound": cs_c, "fcsound": fcs}


def sedov(nd=2, n=64, half=0.3, r0=3.0e-2, e1=1.0, p0=1.0e-5, rho0=1.0, gamma=1.4, method=abi.MODIFIED_EULER,
          tdorder=2, stoptime=0.05, variables=abi.CONSERVATIVE, limiter=abi.MONOCENT, theta=1.2, cfl=0.3,
          tol_rel=0.01, tol_abs=(0.0, 1e-3, 1e-3, 0.0), dtlimit=1.0e-15):
    """Sedov point explosion on a Cartesian box [-half, half]^nd with no-gradient boundaries:
    gas at rest, density rho0, pressure p0 outside r0 and p1 = 3 (gamma-1) e1 / ((nd+1) pi r0^nd)
    inside (tests/ode.f90:159-190 in 2D, tests/sedov3d.f90:270-300 with nd = 3).  The defaults
    are the ode test's (64^2, KT + MC(1.2) on conservative variables, CFL 0.3, tol_rel 0.01,
    tol_abs (0, 1e-3, 1e-3, 0), stoptime 0.05)."""
    c = _base((n, n, n), nd)
    c.xmin, c.xmax, c.ymin, c.ymax = -half, half, -half, half
    if nd == 3:
        c.zmin, c.zmax = -half, half
    for f in range(6):
        c.bc[f] = abi.NO_GRADIENTS
    c.physics = abi.EULER
    c.gamma = gamma
    c.variables = variables
    c.limiter = limiter
    c.theta = theta
    c.method = method
    c.tdorder = tdorder
    c.cfl = cfl
    c.stoptime = stoptime
    c.dtlimit = dtlimit
    c.tol_rel = tol_rel
    V = nd + 2
    for v in range(abi.MAXVAR):
        c.tol_abs[v] = tol_abs[min(v, len(tol_abs) - 1)] if v < V - 1 else tol_abs[-1]
    c.maxiter = 1000000
    abi.finalize_config(c)
    X, Y, Z, _ = centers(c)
    r = np.sqrt(X * X + Y * Y + Z * Z)
    p1 = 3.0 * (gamma - 1.0) * e1 / ((nd + 1) * np.pi * r0 ** nd)
    p = np.zeros((V,) + X.shape)
    p[0] = rho0
    p[V - 1] = np.where(r <= r0, p1, p0)
    return c, p, {}
