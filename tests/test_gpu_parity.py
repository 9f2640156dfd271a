"""GPU parity against the CPU oracle through the C ABI.

The --fmad=false build must agree with the oracle bit for bit (the only
exceptions are cases with absorbing boundaries or a POWERLAW viscosity exponent,
where CUDA's exp/log/pow may differ from glibc's by an ulp: tolerance 1e-13).  The product build (FMA on)
must stay within relative L1 <= 1e-12 after one step
and <= 1e-9 after many steps.
"""
import numpy as np
import pytest

from fosite_b200 import abi
from cases import CASES

pyoracle = pytest.importorskip("pyoracle")

ABSORB = abi.ABSORBING


def _interior(a, cfg):
    sl = [slice(None)]
    for n in (cfg.knum, cfg.jnum, cfg.inum):
        sl.append(slice(2, -2) if n > 1 else slice(None))
    return a[tuple(sl)]


def rel_l1(a, b):
    """Relative L1 norm of the state-vector difference: sum|a-b| / sum|b| over all cells and variables."""
    return float(np.abs(a - b).sum() / (np.abs(b).sum() + 1e-300))


def rel_l1_per_var(a, b):
    num = np.abs(a - b).reshape(a.shape[0], -1).sum(axis=1)
    den = np.abs(b).reshape(b.shape[0], -1).sum(axis=1) + 1e-300
    return float(np.max(num / den))


def _has_absorbing(cfg):
    return any(cfg.bc[f] == ABSORB for f in range(6 if cfg.knum > 1 else 4))


def _inexact(cfg):
    """Cases whose arithmetic calls a transcendental function of CUDA's libm (exp/log of the
    absorbing boundaries, pow of a POWERLAW viscosity with a non-zero exponent), which may
    differ from glibc's by an ulp: compared to 1e-13."""
    return _has_absorbing(cfg) or (cfg.vismodel == abi.VIS_POWERLAW and cfg.vis_exponent != 0.0)


def _pair(name, exact):
    from fosite_b200.sim import Simulation
    cfg, p, extra = CASES[name]()
    o = pyoracle.Oracle(cfg)
    g = Simulation(cfg, exact=exact)
    if "bccsound" in extra:
        shape = o.shape
        bcc = np.broadcast_to(extra["bccsound"], shape)
        fcs = np.broadcast_to(extra["fcsound"], (4,) + shape)
        o.set_sound_speeds(bcc, fcs)
        g.set_sound_speeds(bcc, fcs)
    if "fargo_w" in extra:
        o.set_fargo_velocity(extra["fargo_w"])
        g.set_fargo_velocity(extra["fargo_w"])
    o.set_state(abi.PVAR, p)
    g.set_state(abi.PVAR, p)
    return cfg, o, g


def _compare(cfg, o, g, tol, what):
    for which, nm in ((abi.CVAR, "cvar"), (abi.PVAR, "pvar")):
        a = _interior(g.get(which), cfg)
        b = _interior(o.get(which), cfg)
        if tol == 0.0:
            bad = np.argwhere(a != b)
            assert bad.size == 0, "%s %s: %d cells differ, first %s gpu=%r oracle=%r" % (
                what, nm, len(bad), bad[0], a[tuple(bad[0])], b[tuple(bad[0])])
        else:
            r = rel_l1(a, b)
            assert r <= tol, "%s %s rel L1 %.3e > %.1e" % (what, nm, r, tol)
            rv = rel_l1_per_var(a, b)
            assert rv <= 10 * tol, "%s %s per-variable rel L1 %.3e > %.1e" % (what, nm, rv, 10 * tol)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_rhs_matches_oracle(name):
    cfg, o, g = _pair(name, exact=True)
    tol = 1e-13 if _inexact(cfg) else 0.0
    o.compute_rhs()
    rg = _interior(g.compute_rhs(), cfg)
    ro = _interior(o.get(abi.RHS), cfg)
    if tol == 0.0:
        bad = np.argwhere(rg != ro)
        assert bad.size == 0, "rhs: %d cells differ, first %s gpu=%r oracle=%r" % (
            len(bad), bad[0], rg[tuple(bad[0])], ro[tuple(bad[0])])
    else:
        assert rel_l1(rg, ro) <= tol


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_steps_bitwise_exact_build(name):
    cfg, o, g = _pair(name, exact=True)
    tol = 1e-13 if _inexact(cfg) else 0.0
    assert o.first_step() == 0
    assert g.first_step() == 0
    so, sg = o.status(), g.status()
    if tol == 0.0:
        assert sg.dt == so.dt, (sg.dt, so.dt)
    else:
        assert abs(sg.dt - so.dt) <= tol * so.dt
    for s in range(4):
        ro, rg = o.step(), g.step()
        assert ro == rg
        so, sg = o.status(), g.status()
        assert sg.iter == so.iter and sg.n_adj == so.n_adj
        if tol == 0.0:
            assert sg.time == so.time and sg.dt == so.dt, (s, sg.time, so.time, sg.dt, so.dt)
        _compare(cfg, o, g, tol, "step %d" % s)
        assert sg.dtcause == so.dtcause, (s, sg.dtcause, so.dtcause)
        if cfg.pm_outbound:
            (mg, dg), (mo, do) = g.pointmass(), o.pointmass()
            if tol == 0.0:
                assert (mg, dg) == (mo, do), (s, mg, mo, dg, do)
            else:
                assert abs(mg - mo) <= 1e-13 * abs(mo) and abs(dg - do) <= 1e-11 * abs(mo)
    # full ghost-padded primitive state, ghost cells included (CenterBoundary + SetCornerEdges)
    pa, pb = g.get(abi.PVAR), o.get(abi.PVAR)
    if tol == 0.0:
        assert np.array_equal(pa, pb), np.argwhere(pa != pb)[:5]
    else:
        assert np.allclose(pa, pb, rtol=1e-12, atol=1e-14)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["khi_ssprk3_vanleer_cons", "gauss3d_dopri_mc_prim", "disk_logcyl_pointmass",
                                  "euler2d_absorbing", "iso3d_cashkarp_mixed_bc", "disk_fargo_logcyl",
                                  "khi_visc_re1e4_mc", "gauss3d_visc_dopri", "disk_visc_logcyl_pointmass",
                                  "khi_fargo2_x_visc", "iso_fargo1_x_shear", "disk_fargo_ssprk5_logcyl"])
def test_fast_build_tolerance(name):
    cfg, o, g = _pair(name, exact=False)
    o.first_step()
    g.first_step()
    o.step()
    g.step()
    _compare(cfg, o, g, 1e-12, "1 step")
    for _ in range(30):
        o.step()
        g.step()
    _compare(cfg, o, g, 1e-9, "31 steps")
    assert abs(g.status().time - o.status().time) <= 1e-9 * o.status().time


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["khi_ssprk3_vanleer_cons", "disk_beta_logcyl_me3", "disk_alpha_cyl_me2"])
def test_run_graph_matches_single_steps(name):
    """fgpu_run (graph-replayed device-clocked steps) equals n calls of fgpu_step, also with
    the viscosity update on the device clock."""
    _, _, a = _pair(name, exact=True)
    _, _, b = _pair(name, exact=True)
    a.first_step()
    b.first_step()
    rc, done = a.run(37)
    assert rc == 0 and done == 37
    for _ in range(37):
        b.step()
    assert a.status().time == b.status().time
    assert np.array_equal(a.get(abi.CVAR), b.get(abi.CVAR))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["disk_fargo_cyl_cons_reflect", "khi_fargo1_x", "iso_fargo1_x_shear"])
def test_fargo_graph_run_matches_single_steps(name):
    """FARGO (along y and along x): the first step after FirstStep runs outside the graph,
    later steps replay it."""
    sims = []
    for _ in range(2):
        _, _, s = _pair(name, exact=True)
        s.first_step()
        sims.append(s)
    a, b = sims
    rc, done = a.run(35)
    assert rc == 0 and done == 35
    for _ in range(35):
        assert b.step() == 0
    assert a.status().time == b.status().time
    assert np.array_equal(a.get(abi.CVAR), b.get(abi.CVAR))
    assert np.array_equal(a.get(abi.PVAR), b.get(abi.PVAR))


@pytest.mark.gpu
@pytest.mark.parametrize("visc", [False, True])
def test_khi_transposition_symmetry(visc):
    """tests/KHI2D.f90:81-150: the x<->y transposed run agrees exactly (RMS < TINY), also
    with the test's molecular viscosity (RE = 1e4)."""
    from fosite_b200.sim import Simulation
    from cases import _khi, _visc, khi_reynolds
    cfg, p, _ = _khi(n=(36, 36))
    if visc:
        cfg, p, _ = _visc((cfg, p, {}), khi_reynolds(), bulkconst=-2. / 3. * khi_reynolds())
    pt = np.stack([p[0].transpose(0, 2, 1), p[2].transpose(0, 2, 1), p[1].transpose(0, 2, 1), p[3].transpose(0, 2, 1)])
    # the --fmad=false build: FMA contraction of a*a + b*b is not symmetric in a, b
    a = Simulation(cfg, exact=True)
    b = Simulation(cfg, exact=True)
    a.set_state(abi.PVAR, p)
    b.set_state(abi.PVAR, pt)
    a.first_step()
    b.first_step()
    a.run(20)
    b.run(20)
    ra, rb = a.get(abi.PVAR), b.get(abi.PVAR)
    rbt = np.stack([rb[0].transpose(0, 2, 1), rb[2].transpose(0, 2, 1), rb[1].transpose(0, 2, 1), rb[3].transpose(0, 2, 1)])
    assert np.sqrt(np.mean((ra - rbt) ** 2)) < abi.TINY


@pytest.mark.gpu
@pytest.mark.parametrize("visc", [False, True])
@pytest.mark.parametrize("fargo", [1, 2])
def test_khi_fargo_transposition_symmetry(fargo, visc):
    """tests/KHI2D.f90:81-150, the FARGO legs on the device: FARGO type 1 or 2 along x and
    the transposed run with FARGO along y agree to TINY (RMS), with and without the test's
    molecular viscosity, and the run along x equals the oracle's bit for bit."""
    from fosite_b200.sim import Simulation
    from cases import khi_fargo
    runs = []
    for direction in (1, 2):
        cfg, p, extra = khi_fargo(fargo, direction=direction, visc=visc)
        g = Simulation(cfg, exact=True)
        if "fargo_w" in extra:
            g.set_fargo_velocity(extra["fargo_w"])
        g.set_state(abi.PVAR, p)
        g.first_step()
        rc, done = g.run(20)
        assert rc == 0 and done == 20
        runs.append((g, cfg, p, extra))
    (a, ca, pa, ea), (b, _, _, _) = runs
    rb = b.get(abi.PVAR)
    rbt = np.stack([rb[0], rb[2], rb[1], rb[3]]).transpose(0, 1, 3, 2)
    assert np.sqrt(np.mean((a.get(abi.PVAR) - rbt) ** 2)) < abi.TINY
    assert a.status().time == b.status().time
    o = pyoracle.Oracle(ca)
    if "fargo_w" in ea:
        o.set_fargo_velocity(ea["fargo_w"])
    o.set_state(abi.PVAR, pa)
    o.first_step()
    for _ in range(20):
        assert o.step() == 0
    assert np.array_equal(o.get(abi.PVAR), a.get(abi.PVAR))


@pytest.mark.gpu
def test_khi3d_orientation_symmetry_gpu():
    """tests/KHI3D.f90:260-266 on the device, with the test's molecular viscosity: six
    orientations, TSIM = 30, RMS < 4 EPSILON (the --fmad=false build; contraction of
    a*a + b*b is not symmetric in a, b), and the base orientation equal to the oracle's
    run bit for bit."""
    from fosite_b200.sim import Simulation
    from cases import khi3d, permute_state, inverse_perm
    runs = {}
    for perm in [(0, 1, 2), (1, 0, 2), (2, 1, 0), (0, 2, 1), (1, 2, 0), (2, 0, 1)]:
        cfg, p, _ = khi3d(perm)
        g = Simulation(cfg, exact=True)
        g.set_state(abi.PVAR, p)
        g.first_step()
        rc, done = g.run(100000)
        assert rc == abi.STOPTIME and done > 900
        runs[perm] = permute_state(g.get(abi.PVAR), inverse_perm(perm))
    base = runs[(0, 1, 2)]
    for perm, r in runs.items():
        assert np.sqrt(np.mean((r - base) ** 2)) < 4 * np.finfo(float).eps, perm
    cfg, p, _ = khi3d((0, 1, 2))
    o = pyoracle.Oracle(cfg)
    o.set_state(abi.PVAR, p)
    o.first_step()
    while o.step() == 0:
        pass
    assert np.array_equal(o.get(abi.PVAR), base)


def _face_region(cfg, d):
    """Slices of the faces a right-hand side reads in direction d (padded indexing: the face
    between cells i and i+1 sits at i, from IMIN-1 to IMAX; the other directions interior)."""
    sl = [slice(None)]
    for ax, n in zip((2, 1, 0), (cfg.knum, cfg.jnum, cfg.inum)):
        if n == 1:
            sl.append(slice(None))
        elif ax == d:
            sl.append(slice(1, n + 2))
        else:
            sl.append(slice(2, n + 2))
    return tuple(sl)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_interface_fluxes_match_oracle(name):
    """CalculateFluxes (fluxes_base.f90:87-97): the x/y/z interface fluxes of ComputeRHS, exact build."""
    cfg, o, g = _pair(name, exact=True)
    tol = 1e-13 if _inexact(cfg) else 0.0
    o.compute_rhs()
    g.compute_rhs()
    dirs = [abi.XFLUX, abi.YFLUX] + ([abi.ZFLUX] if cfg.knum > 1 else [])
    for d, which in enumerate(dirs):
        sl = _face_region(cfg, d)
        a, b = g.fluxes(which)[sl], o.get(which)[sl]
        if tol == 0.0:
            bad = np.argwhere(a != b)
            assert bad.size == 0, "dir %d: %d faces differ, first %s gpu=%r oracle=%r" % (
                d, len(bad), bad[0], a[tuple(bad[0])], b[tuple(bad[0])])
        else:
            assert rel_l1(a, b) <= tol, d
    g.close()
