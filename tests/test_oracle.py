"""CPU checks of the oracle against the reference's own test assertions.

The reference ships no golden vectors; its tests pin the scheme through
metamorphic properties, which are reproduced here on the restatement:
  * tests/KHI2D.f90:81-150 -- the x<->y transposed KHI run agrees to TINY;
  * conservation of mass, momentum and energy on periodic boxes;
  * the committed golden fixtures (tests/golden/) regenerate bit for bit.
"""
import os

import numpy as np
import pytest

from fosite_b200 import abi, problems
from cases import CASES, _khi

pyoracle = pytest.importorskip("pyoracle")
HERE = os.path.dirname(os.path.abspath(__file__))


def _run(cfg, p, steps, extra=None):
    o = pyoracle.Oracle(cfg)
    if extra and "bccsound" in extra:
        o.set_sound_speeds(np.broadcast_to(extra["bccsound"], o.shape),
                           np.broadcast_to(extra["fcsound"], (4,) + o.shape))
    if extra and "fargo_w" in extra:
        o.set_fargo_velocity(extra["fargo_w"])
    o.set_state(abi.PVAR, p)
    assert o.first_step() == 0
    for _ in range(steps):
        assert o.step() == 0
    return o


def _swap_xy(p):
    q = np.stack([p[0], p[2], p[1], p[3]])
    return q.transpose(0, 1, 3, 2).copy()


def test_khi_transposition_symmetry_exact():
    cfg, p, _ = _khi(n=(24, 24))
    a = _run(cfg, p, 15)
    b = _run(cfg, _swap_xy(p), 15)
    ra, rb = a.get(abi.PVAR), _swap_xy(b.get(abi.PVAR))
    sigma = np.sqrt(np.mean((ra - rb) ** 2))
    assert sigma < abi.TINY
    assert a.status().dt == b.status().dt


@pytest.mark.parametrize("visc", [False, True])
@pytest.mark.parametrize("fargo", [1, 2])
def test_khi_fargo_transposition_symmetry_exact(fargo, visc):
    """tests/KHI2D.f90:81-150, the FARGO legs: FARGO type 1 or 2 along x and the transposed
    run with FARGO along y agree to TINY (with and without the test's viscosity)."""
    from cases import khi_fargo
    ca, pa, ea = khi_fargo(fargo, direction=1, visc=visc)
    cb, pb, eb = khi_fargo(fargo, direction=2, visc=visc)
    a = _run(ca, pa, 15, ea)
    b = _run(cb, pb, 15, eb)
    ra, rb = a.get(abi.PVAR), _swap_xy(b.get(abi.PVAR))
    assert np.sqrt(np.mean((ra - rb) ** 2)) < abi.TINY
    assert a.status().dt == b.status().dt and a.status().time == b.status().time


def test_khi_conservation_periodic():
    cfg, p, _ = _khi(n=(32, 28))
    o = pyoracle.Oracle(cfg)
    o.set_state(abi.PVAR, p)
    c0 = o.get(abi.CVAR)[:, :, 2:-2, 2:-2].sum(axis=(1, 2, 3))
    o.first_step()
    for _ in range(25):
        o.step()
    c1 = o.get(abi.CVAR)[:, :, 2:-2, 2:-2].sum(axis=(1, 2, 3))
    scale = np.abs(o.get(abi.CVAR)[:, :, 2:-2, 2:-2]).sum(axis=(1, 2, 3))
    assert np.all(np.abs(c1 - c0) <= 1e-13 * scale)


def test_gauss3d_dopri_adapts_and_conserves_mass():
    cfg, p, _ = CASES["gauss3d_dopri_mc_prim"]()
    o = pyoracle.Oracle(cfg)
    o.set_state(abi.PVAR, p)
    m0 = o.get(abi.CVAR)[0, 2:-2, 2:-2, 2:-2].sum()
    o.first_step()
    for _ in range(3):
        assert o.step() == 0
    st = o.status()
    assert st.iter >= 3 and 0.0 <= st.maxerr < 1.0
    m1 = o.get(abi.CVAR)[0, 2:-2, 2:-2, 2:-2].sum()
    assert abs(m1 - m0) <= 1e-13 * m0


def test_mesh_coordinates_match_host_builder():
    cfg, _, _ = _khi(n=(20, 12))
    o = pyoracle.Oracle(cfg)
    X, Y, Z, _ = problems.centers(cfg)
    assert np.array_equal(o.mesh(abi.MESH_X), X)
    assert np.array_equal(o.mesh(abi.MESH_Y), Y)


@pytest.mark.parametrize("name", sorted(CASES))
def test_golden_fixture(name):
    path = os.path.join(HERE, "golden", name + ".npz")
    if not os.path.exists(path):
        pytest.skip("fixture not generated")
    g = np.load(path)
    cfg, p, extra = CASES[name]()
    o = _run(cfg, p, int(g["steps"]), extra)
    assert np.array_equal(o.get(abi.CVAR), g["cvar"])
    assert o.status().dt == float(g["dt"])


def test_khi3d_orientation_symmetry():
    """tests/KHI3D.f90:260-266: the six orientations of the 3D shear layer, with the test's
    molecular viscosity (RE = 1e4), agree to 4 EPSILON (RMS) once mapped back, after the
    reference's TSIM = 30 (about 1000 steps at 8^3)."""
    from cases import khi3d, permute_state, inverse_perm
    runs = {}
    for perm in [(0, 1, 2), (1, 0, 2), (2, 1, 0), (0, 2, 1), (1, 2, 0), (2, 0, 1)]:
        cfg, p, _ = khi3d(perm)
        o = pyoracle.Oracle(cfg)
        o.set_state(abi.PVAR, p)
        assert o.first_step() == 0
        while o.step() == 0:
            pass
        runs[perm] = permute_state(o.get(abi.PVAR), inverse_perm(perm))
    base = runs[(0, 1, 2)]
    for perm, r in runs.items():
        sigma = np.sqrt(np.mean((r - base) ** 2))
        assert sigma < 4 * np.finfo(float).eps, (perm, sigma)


def test_khi_visc_transposition_symmetry_exact():
    """tests/KHI2D.f90:81-150 with the test's own molecular viscosity (RE = 1e4, bulk
    viscosity -2/3 of it): the transposed run agrees to TINY."""
    from cases import _visc, khi_reynolds
    eta = khi_reynolds()
    cfg, p, _ = _visc(_khi(n=(24, 24), limiter=abi.MONOCENT, theta=1.2), eta, bulkconst=-2. / 3. * eta)
    a = _run(cfg, p, 15)
    b = _run(cfg, _swap_xy(p), 15)
    ra, rb = a.get(abi.PVAR), _swap_xy(b.get(abi.PVAR))
    assert np.sqrt(np.mean((ra - rb) ** 2)) < abi.TINY
    assert a.status().dt == b.status().dt


def test_khi_visc_conservation_periodic():
    """The viscous momentum and energy sources are divergences of face averages
    (mesh_midpoint.f90:283-323) and telescope over a periodic box -- except through the
    corner ghost cells, which SetCornerEdges averages even on periodic meshes
    (boundary_generic.f90:434-470; the reference notes the viscosity reads them).  With
    the velocity zero within two cells of every boundary the corners are consistent and
    one right-hand side conserves momentum and energy to rounding; mass stays conserved
    over a whole viscous run in any case."""
    from cases import _visc
    cfg, p, _ = _visc(_khi(n=(32, 28)), 5e-3)
    o = pyoracle.Oracle(cfg)
    o.set_state(abi.PVAR, p)
    m0 = o.get(abi.CVAR)[0, :, 2:-2, 2:-2].sum()
    o.first_step()
    for _ in range(25):
        assert o.step() == 0
    m1 = o.get(abi.CVAR)[0, :, 2:-2, 2:-2].sum()
    assert abs(m1 - m0) <= 1e-13 * abs(m0)
    q = p.copy()
    frame = np.ones(q.shape[1:], dtype=bool)
    frame[:, 4:-4, 4:-4] = False      # two boundary cells of the interior plus the ghosts
    q[1][frame] = 0.0
    q[2][frame] = 0.0
    rhs = []
    for visc in (False, True):
        c, _, _ = _khi(n=(32, 28))
        if visc:
            c, _, _ = _visc((c, None, {}), 5e-3)
        o = pyoracle.Oracle(c)
        o.set_state(abi.PVAR, q)
        o.compute_rhs()
        rhs.append(o.get(abi.RHS)[:, 0, 2:-2, 2:-2])
    src = rhs[0] - rhs[1]
    tot = src.sum(axis=(1, 2))
    mag = np.abs(src).sum(axis=(1, 2))
    assert tot[0] == 0.0
    assert np.all(np.abs(tot[1:]) <= 1e-13 * mag[1:]), (tot, mag)


def test_viscous_force_of_a_sine_shear():
    """Physics of the restated stress divergence: for v_x = U sin(2 pi y) at rest otherwise,
    the x force is eta d2v_x/dy2 = -eta (2 pi)^2 U sin(2 pi y) and the heating
    div(v.T) = eta d(v_x dv_x/dy)/dy, to second order in dy.  The viscous source is the
    difference of the right-hand sides with and without viscosity (rhs = ... - src)."""
    from cases import _visc
    ny, eta, U = 64, 0.01, 0.1
    base = _khi(n=(8, ny))
    cfg0, _, _ = base
    X, Y, Z, _ = problems.centers(cfg0)
    p = np.zeros((4,) + X.shape)
    p[0] = 1.0
    p[1] = U * np.sin(2 * np.pi * (Y + 0.5))
    p[3] = 1.0
    rhs = []
    for visc in (False, True):
        cfg, _, _ = _khi(n=(8, ny))
        if visc:
            cfg, _, _ = _visc((cfg, None, {}), eta)
        o = pyoracle.Oracle(cfg)
        o.set_state(abi.PVAR, p)
        o.compute_rhs()
        rhs.append(o.get(abi.RHS)[:, 0, 2:-2, 2:-2])
    src = rhs[0] - rhs[1]
    # the four corner cells read the averaged corner ghosts of SetCornerEdges
    keep = np.ones(src.shape[1:], dtype=bool)
    keep[0, 0] = keep[0, -1] = keep[-1, 0] = keep[-1, -1] = False
    y = Y[0, 2:-2, 2:-2] + 0.5
    k = 2 * np.pi
    fx = -eta * k * k * U * np.sin(k * y)
    heat = eta * U * U * k * k * np.cos(2 * k * y)     # d/dy (v dv/dy) = U^2 k^2 cos(2ky)
    assert np.abs(src[0]).max() == 0.0
    assert np.abs(src[1] - fx)[keep].max() < 5e-3 * np.abs(fx).max()
    assert np.abs(src[2])[keep].max() < 1e-14
    assert np.abs(src[3] - heat)[keep].max() < 2e-2 * np.abs(heat).max()     # O((k dy)^2)


def test_viscous_timestep_limit():
    """sources_viscosity.f90:511-581: dt = cvis / max over the padded mesh of
    sum_d (max wave speed_d + 2 kinvis/dl_d)/dl_d; the sources list marks dtcause = 3
    (sources_generic.f90:264-293) where it undercuts the CFL step."""
    cfg, p, extra = CASES["khi_visc_dominant_reflect_prim"]()
    o = pyoracle.Oracle(cfg)
    o.set_state(abi.PVAR, p)
    assert o.first_step() == 0
    st = o.status()
    assert st.dtcause == abi.DTCAUSE_VISCOSITY
    pv = o.get(abi.PVAR)[:, 0]
    dx = (cfg.xmax - cfg.xmin) / cfg.inum
    dy = (cfg.ymax - cfg.ymin) / cfg.jnum
    cs = np.sqrt(np.maximum(2 * abi.TINY, cfg.gamma * pv[3] / pv[0]))
    nu = cfg.dynconst / pv[0]
    ax = np.maximum(np.maximum(0.0, pv[1] + cs), -np.minimum(0.0, pv[1] - cs))
    ay = np.maximum(np.maximum(0.0, pv[2] + cs), -np.minimum(0.0, pv[2] - cs))
    inv = (ax + 2.0 * nu / dx) / dx + (ay + 2.0 * nu / dy) / dy
    assert st.dt == cfg.cvis / inv.max()
