"""Embedded Runge-Kutta schemes on the device clock (fgpu_run): the IntegrationStep
loop (timedisc_base.f90:649-750) runs as replayed attempt slots with the accept/reject
predicate and the PI controller evaluated on the device.  Results must equal the
oracle's steps (bit for bit with the --fmad=false build) and the host-controlled
fgpu_step sequence, rejections and sub-steps included."""
import numpy as np
import pytest

from fosite_b200 import abi
from cases import CASES

pyoracle = pytest.importorskip("pyoracle")

from test_gpu_parity import _pair, _interior, _inexact, rel_l1  # noqa: E402


def _embedded(cfg):
    return cfg.method != abi.MODIFIED_EULER or cfg.tol_rel < 1.0


EMBEDDED = sorted(n for n in CASES if _embedded(CASES[n]()[0]))


@pytest.mark.gpu
@pytest.mark.parametrize("name", EMBEDDED)
def test_device_clock_matches_oracle(name):
    cfg, o, g = _pair(name, exact=True)
    tol = 1e-13 if _inexact(cfg) else 0.0
    assert o.first_step() == 0 and g.first_step() == 0
    steps = 6
    for _ in range(steps):
        assert o.step() == 0
    rc, done = g.run(steps)
    assert rc == 0 and done == steps
    so, sg = o.status(), g.status()
    assert (sg.iter, sg.n_adj) == (so.iter, so.n_adj)
    assert sg.dtcause == so.dtcause
    if tol == 0.0:
        assert (sg.time, sg.dt, sg.dtmin, sg.maxerr) == (so.time, so.dt, so.dtmin, so.maxerr)
        assert np.array_equal(g.get(abi.PVAR), o.get(abi.PVAR))
        assert np.array_equal(g.get(abi.CVAR), o.get(abi.CVAR))
    else:
        assert abs(sg.time - so.time) <= tol * so.time and abs(sg.dt - so.dt) <= tol * so.dt
        for which in (abi.PVAR, abi.CVAR):
            assert rel_l1(_interior(g.get(which), cfg), _interior(o.get(which), cfg)) <= tol


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["gauss3d_dopri_mc_prim", "gauss3d_rkf3_minmod_cons", "khi_modeuler_adaptive2_mc_prim",
                                  "iso3d_cashkarp_mixed_bc", "disk_powerlaw_pringle_ssprk5", "disk_fargo_ssprk5_logcyl",
                                  "khi_fargo1_x_cashkarp", "disk_fargo_me3_adaptive", "disk_fargo2_me2_adaptive"])
def test_device_clock_equals_host_steps(name):
    """fgpu_run (device clock) and repeated fgpu_step (host-controlled loop) agree bitwise,
    also when the device run is continued by host steps and vice versa."""
    _, _, a = _pair(name, exact=True)
    _, _, b = _pair(name, exact=True)
    a.first_step()
    b.first_step()
    rc, done = a.run(9)
    assert rc == 0 and done == 9
    for _ in range(9):
        assert b.step() == 0
    for x, y in ((a, b),):
        sx, sy = x.status(), y.status()
        assert (sx.time, sx.dt, sx.iter, sx.n_adj, sx.dtmin) == (sy.time, sy.dt, sy.iter, sy.n_adj, sy.dtmin)
        assert np.array_equal(x.get(abi.CVAR), y.get(abi.CVAR))
    assert a.step() == 0          # host step after a device run
    rc, done = b.run(1)           # device run after host steps
    assert rc == 0 and done == 1
    assert a.status().time == b.status().time and a.status().dt == b.status().dt
    assert np.array_equal(a.get(abi.CVAR), b.get(abi.CVAR))


@pytest.mark.gpu
def test_device_clock_stops_at_stoptime():
    """The device loop ends at the stop time like fosite%Run: the last step is clipped to it
    (the output-time clip with tout = stoptime) and a further run does nothing."""
    from fosite_b200.sim import Simulation
    cfg, p, _ = CASES["gauss3d_dopri_mc_prim"]()
    cfg.stoptime = 0.02
    abi.finalize_config(cfg)
    g = Simulation(cfg, exact=True)
    g.set_state(abi.PVAR, p)
    g.first_step()
    rc, done = g.run(1000)
    assert rc == abi.STOPTIME and 0 < done < 1000
    assert abs(g.status().time - cfg.stoptime) <= 1e-5 * cfg.stoptime
    o = pyoracle.Oracle(cfg)
    o.set_state(abi.PVAR, p)
    o.first_step()
    k = 0
    while o.step() == 0:
        k += 1
    assert k == done and o.status().time == g.status().time
    assert np.array_equal(o.get(abi.CVAR), g.get(abi.CVAR))
    rc, done = g.run(5)
    assert rc == abi.STOPTIME and done == 0


@pytest.mark.gpu
@pytest.mark.parametrize("host", [False, True])
@pytest.mark.parametrize("name", ["gauss3d_dopri_mc_prim", "gauss3d_rkf3_minmod_cons", "iso3d_beta_dopri",
                                  "euler2d_rkf45", "disk_powerlaw_pringle_ssprk5", "gauss3d_visc_dopri"])
def test_fused_stage_state_equals_form_pass(name, host, monkeypatch):
    """Butcher stage states formed in the previous stage kernel's epilogue (the default)
    equal the ones a separate form pass writes (FGPU_FUSE_FORM=0), bit for bit, on the
    device clock and on the host-controlled loop (FGPU_BUTCHER_HOST=1)."""
    if host:
        monkeypatch.setenv("FGPU_BUTCHER_HOST", "1")
    sims = []
    for fuse in ("1", "0"):
        monkeypatch.setenv("FGPU_FUSE_FORM", fuse)
        _, _, g = _pair(name, exact=True)
        assert g.first_step() == 0
        rc, done = g.run(5)
        assert rc == 0 and done == 5
        sims.append(g)
    a, b = sims
    sa, sb = a.status(), b.status()
    assert (sa.time, sa.dt, sa.iter, sa.n_adj) == (sb.time, sb.dt, sb.iter, sb.n_adj)
    assert np.array_equal(a.get(abi.CVAR), b.get(abi.CVAR))


@pytest.mark.gpu
@pytest.mark.parametrize("host", [False, True])
def test_butcher_steps_with_shuffle_layout_forced(host, monkeypatch):
    """With the warp-shuffle stage layout forced (FGPU_STAGE_VARIANT=1), the stages that it
    cannot run (gated device-clock stages, stages forming the next stage's state) take the
    base tile: results still equal the oracle's bit for bit."""
    monkeypatch.setenv("FGPU_STAGE_VARIANT", "1")
    if host:
        monkeypatch.setenv("FGPU_BUTCHER_HOST", "1")
    cfg, o, g = _pair("gauss3d_dopri_mc_prim", exact=True)
    assert o.first_step() == 0 and g.first_step() == 0
    for _ in range(4):
        assert o.step() == 0
    rc, done = g.run(4)
    assert rc == 0 and done == 4
    assert g.status().time == o.status().time
    assert np.array_equal(g.get(abi.CVAR), o.get(abi.CVAR))


@pytest.mark.gpu
@pytest.mark.parametrize("host", [False, True])
@pytest.mark.parametrize("name,frac", [("gauss3d_dopri_mc_prim", 0.999), ("gauss3d_dopri_mc_prim", 0.99),
                                       ("khi_modeuler_adaptive2_mc_prim", 0.999), ("euler2d_rkf45", 0.999)])
def test_checkdata_break_matches_oracle(name, frac, host, monkeypatch):
    """CheckData breaks the step where fosite does: inside the step, at AcceptSolution's
    ComputeRHS (timedisc_base.f90:926-931; the step then ends without its closing, time and dt
    unchanged), or at the closing ComputeRHS.  CHECK_RHOMIN with rhomin just below the initial
    minimum density provokes either; the break step, the bookkeeping and the state equal the
    oracle's, on the device clock (fgpu_run) and on the host-controlled loop."""
    if host:
        monkeypatch.setenv("FGPU_BUTCHER_HOST", "1")
    from fosite_b200.sim import Simulation
    cfg, p, extra = CASES[name]()
    cfg.rhomin = float(p[0].min()) * frac
    o = pyoracle.Oracle(cfg)
    o.set_state(abi.PVAR, p)
    g = Simulation(cfg, exact=True)
    g.set_state(abi.PVAR, p)
    assert o.first_step() == 0 and g.first_step() == 0
    for s in range(12):
        ro = o.step()
        rc, done = g.run(1)
        assert rc == ro, (s, rc, ro)
        assert done == (1 if ro == 0 else 0)
        so, sg = o.status(), g.status()
        assert (sg.time, sg.dt, sg.iter, sg.n_adj) == (so.time, so.dt, so.iter, so.n_adj), s
        assert sg.checkflags == so.checkflags and sg.brk == so.brk
        if ro != 0:
            assert ro == abi.BREAK
            assert np.array_equal(g.get(abi.CVAR), o.get(abi.CVAR))
            break
    else:
        pytest.fail("no CheckData break")
