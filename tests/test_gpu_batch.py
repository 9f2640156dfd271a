"""Batched ensembles (fgpu_batch_*): one persistent launch per stage over the
tile queue of many independent grids must give every grid exactly the
results of stepping it alone, with its own dt, time and stop state."""
import numpy as np
import pytest

from fosite_b200 import abi, problems
from cases import _khi, _gauss3d

pytestmark = pytest.mark.gpu


def _disk_member(nr, nphi, geometry, hratio, sigma, seed, exact):
    from fosite_b200.sim import Simulation
    cfg, p, extra = problems.disk2d(nr=nr, nphi=nphi, seed=seed, hratio=hratio, sigma_index=sigma,
                                    geometry=geometry, fargo=0)
    s = Simulation(cfg, exact=exact)
    shape = (1, nphi + 4, nr + 4)
    s.set_sound_speeds(np.broadcast_to(extra["bccsound"], shape), np.broadcast_to(extra["fcsound"], (4,) + shape))
    s.set_state(abi.PVAR, p)
    assert s.first_step() == 0
    return s


def _disk_specs(n, seed=7):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        nr = int(rng.integers(1, 5)) * 16 + 8          # deliberately not tile multiples
        nphi = int(rng.integers(2, 6)) * 16 + 4
        geo = abi.CYLINDRICAL if k % 2 else abi.LOGCYLINDRICAL
        out.append((nr, nphi, geo, float(rng.uniform(0.03, 0.1)), float(rng.uniform(-1.5, -0.5)), 100 + k))
    return out


@pytest.mark.parametrize("exact", [True, False])
def test_disk_ensemble_matches_single_grids(exact):
    from fosite_b200.sim import Batch
    specs = _disk_specs(7)
    members = [_disk_member(*sp, exact=exact) for sp in specs]
    alone = [_disk_member(*sp, exact=exact) for sp in specs]
    b = Batch(members)
    assert b.tiles == sum(((sp[0] + 31) // 32) * ((sp[1] + 7) // 8) for sp in specs)
    assert b.run(21) == len(members)     # 16-step graph + 5 direct steps
    for s in alone:
        rc, done = s.run(21)
        assert rc == 0 and done == 21
    for m, s in zip(members, alone):
        assert m.status().iter == s.status().iter == 21
        assert m.status().time == s.status().time
        assert m.status().dt == s.status().dt
        assert np.array_equal(m.get(abi.CVAR), s.get(abi.CVAR))
    b.close()


@pytest.mark.parametrize("exact,tpb", [(True, None), (False, None), (True, 3)])
def test_disk_ensemble_tma_layout(exact, tpb, monkeypatch):
    """The TMA-staged batched layout (6, one block per column of tiles, tensor maps of every
    member's stage inputs in a device table): every member equals its lone run on the TMA
    layout bit for bit, and on the exact build also its lone run on the base tile."""
    from fosite_b200.sim import Batch
    monkeypatch.setenv("FGPU_STAGE_VARIANT", "6")
    if tpb:
        monkeypatch.setenv("FGPU_TMA_TPB", str(tpb))
    specs = _disk_specs(7)
    members = [_disk_member(*sp, exact=exact) for sp in specs]
    alone = [_disk_member(*sp, exact=exact) for sp in specs]
    monkeypatch.setenv("FGPU_STAGE_VARIANT", "0")
    base = [_disk_member(*sp, exact=exact) for sp in specs] if exact else []
    b = Batch(members)
    assert b.layout() == 6
    assert b.run(21) == len(members)
    for s in alone + base:
        rc, done = s.run(21)
        assert rc == 0 and done == 21
    for m, s in zip(members, alone):
        assert (m.status().time, m.status().dt) == (s.status().time, s.status().dt)
        assert np.array_equal(m.get(abi.CVAR), s.get(abi.CVAR))
    for m, s in zip(members, base):
        assert np.array_equal(m.get(abi.CVAR), s.get(abi.CVAR))
    b.close()


@pytest.mark.parametrize("limiters", [(abi.VANLEER, abi.VANLEER, abi.VANLEER),
                                      (abi.MINMOD, abi.MONOCENT, abi.VANLEER)])
def test_euler2d_tma_batch_limiters_and_autotune(limiters, monkeypatch):
    """Euler members on the TMA batched layout with one compiled-in limiter, and with mixed
    limiters (MC with theta 1.3 among them: the kernel reads limiter and theta per member);
    the tuner's pick keeps every result."""
    from fosite_b200.sim import Batch, Simulation
    monkeypatch.setenv("FGPU_STAGE_VARIANT", "6")
    sizes = [(40, 36), (64, 20), (34, 50)]

    def make():
        out = []
        for k, (n, lim) in enumerate(zip(sizes, limiters)):
            cfg, p, _ = _khi(n=n, limiter=lim, theta=1.3 if lim == abi.MONOCENT else 1.0,
                             variables=abi.PRIMITIVE, seed=80 + k)
            s = Simulation(cfg, exact=True)
            s.set_state(abi.PVAR, p)
            s.first_step()
            out.append(s)
        return out
    members, alone = make(), make()
    b = Batch(members)
    assert b.layout() == 6
    b.run(9)
    v = b.autotune(2)
    assert v in (0, 2, 3, 6)
    b.run(9)
    for s in alone:
        s.run(18)
    for m, s in zip(members, alone):
        assert np.array_equal(m.get(abi.CVAR), s.get(abi.CVAR))
    b.close()


def test_members_stop_independently():
    """A member that reaches its stop time idles while the others go on."""
    from fosite_b200.sim import Batch, Simulation
    sims = []
    for k, stop in enumerate((0.02, 1.0, 0.05)):
        cfg, p, _ = _khi(n=(40 + 8 * k, 36), seed=3 + k)
        cfg.stoptime = stop
        abi.finalize_config(cfg)
        s = Simulation(cfg, exact=True)
        s.set_state(abi.PVAR, p)
        s.first_step()
        sims.append(s)
    b = Batch(sims)
    active = b.run(200)
    st = [s.status() for s in sims]
    assert abs(st[0].time - 0.02) <= 1e-5 * 0.02
    assert abs(st[2].time - 0.05) <= 1e-5 * 0.05
    assert active == 1 and st[1].time < 1.0
    frozen = sims[0].get(abi.CVAR)
    b.run(16)
    assert np.array_equal(sims[0].get(abi.CVAR), frozen)
    # the stopped member took exactly the steps a lone run takes to its stop time
    cfg, p, _ = _khi(n=(40, 36), seed=3)
    cfg.stoptime = 0.02
    abi.finalize_config(cfg)
    lone = Simulation(cfg, exact=True)
    lone.set_state(abi.PVAR, p)
    lone.first_step()
    rc, done = lone.run(200)
    assert rc == abi.STOPTIME
    assert done == st[0].iter
    assert np.array_equal(lone.get(abi.CVAR), frozen)


def test_euler3d_ensemble_and_autotune():
    from fosite_b200.sim import Batch, Simulation
    sizes = [(12, 14, 10), (20, 9, 17), (16, 16, 16)]
    def make():
        out = []
        for k, n in enumerate(sizes):
            cfg, p, _ = _gauss3d(n=n, method=abi.MODIFIED_EULER, tdorder=3, limiter=abi.VANLEER, seed=60 + k)
            s = Simulation(cfg, exact=True)
            s.set_state(abi.PVAR, p)
            s.first_step()
            out.append(s)
        return out
    members, alone = make(), make()
    b = Batch(members)
    v = b.autotune(2)
    assert v in (0, 2, 3)
    b.run(18)
    for s in alone:
        s.run(18)
    for m, s in zip(members, alone):
        assert np.array_equal(m.get(abi.CVAR), s.get(abi.CVAR))
        assert np.array_equal(m.get(abi.PVAR), s.get(abi.PVAR))


def test_batch_rejects_mixed_or_unsupported_members():
    from fosite_b200.sim import Batch, FositeError, Simulation
    c1, p1, _ = _khi(n=(24, 24))
    c2, p2, _ = _khi(n=(24, 24), variables=abi.PRIMITIVE)
    a, b = Simulation(c1), Simulation(c2)
    for s, p in ((a, p1), (b, p2)):
        s.set_state(abi.PVAR, p)
    with pytest.raises(FositeError):
        Batch([a])                       # before first_step
    a.first_step()
    b.first_step()
    with pytest.raises(FositeError):
        Batch([a, b])                    # conservative and primitive reconstruction
    c3, p3, _ = _khi(n=(24, 24), method=abi.DORMAND_PRINCE, tdorder=5)
    d = Simulation(c3)
    d.set_state(abi.PVAR, p3)
    d.first_step()
    with pytest.raises(FositeError):
        Batch([a, d])                    # fixed-step and embedded members
    c4, p4, _ = _khi(n=(24, 24), me_tol=1e-3)
    e = Simulation(c4)
    e.set_state(abi.PVAR, p4)
    e.first_step()
    with pytest.raises(FositeError):
        Batch([e, d])                    # embedded modified Euler and Butcher members
    c5, p5, _ = _khi(n=(24, 24), method=abi.CASH_KARP, tdorder=5)
    f = Simulation(c5)
    f.set_state(abi.PVAR, p5)
    f.first_step()
    with pytest.raises(FositeError):
        Batch([d, f])                    # different tableaus


def test_single_grid_autotune_keeps_results():
    from fosite_b200.sim import Simulation
    cfg, p, _ = _khi(n=(64, 48))
    a, b = Simulation(cfg, exact=True), Simulation(cfg, exact=True)
    for s in (a, b):
        s.set_state(abi.PVAR, p)
        s.first_step()
    v = a.autotune(2)
    assert v in (0, 1, 2, 3, 4, 5)
    a.run(20)
    b.run(20)
    assert np.array_equal(a.get(abi.CVAR), b.get(abi.CVAR))


@pytest.mark.gpu
def test_autotune_3d_chunks_and_cache_keep_results():
    """The tuner also picks the z chunk of 3D grids; a second grid with the same tuning key
    takes the cached choice; neither changes any result."""
    import time
    from fosite_b200.sim import Simulation
    from cases import _gauss3d
    cfg, p, _ = _gauss3d(n=(24, 20, 18))
    a, b, c = (Simulation(cfg, exact=True) for _ in range(3))
    for s in (a, b, c):
        s.set_state(abi.PVAR, p)
        s.first_step()
    va = a.autotune(2)
    t0 = time.perf_counter()
    vb = b.autotune(2)
    assert vb == va
    assert time.perf_counter() - t0 < 0.05          # cached: no probes
    for s in (a, b, c):
        assert s.run(6)[0] == 0
    assert np.array_equal(a.get(abi.CVAR), c.get(abi.CVAR))
    assert np.array_equal(b.get(abi.CVAR), c.get(abi.CVAR))


def test_embedded_batch_equals_lone_runs_and_oracle():
    """Dormand-Prince members of different sizes and tolerances in one batch: one attempt slot
    per replay advances every member with its own controller (rejections and sub-steps
    included); each member equals its lone device-clock run and the oracle bit for bit."""
    import pyoracle
    from fosite_b200.sim import Batch, Simulation
    specs = [((14, 12, 10), 1e-5), ((20, 18, 16), 1e-4), ((12, 16, 14), 3e-5)]

    def make():
        out = []
        for n, tol in specs:
            cfg, p, _ = _gauss3d(n=n, tol=tol)
            s = Simulation(cfg, exact=True)
            s.set_state(abi.PVAR, p)
            s.first_step()
            out.append(s)
        return out
    members, alone = make(), make()
    b = Batch(members)
    b.autotune(2)
    assert b.run(7) == len(specs)
    for s in alone:
        assert s.run(7) == (0, 7)
    for m, s in zip(members, alone):
        sm, ss = m.status(), s.status()
        assert (sm.time, sm.dt, sm.iter, sm.n_adj) == (ss.time, ss.dt, ss.iter, ss.n_adj)
        assert np.array_equal(m.get(abi.CVAR), s.get(abi.CVAR))
    cfg, p, _ = _gauss3d(n=specs[1][0], tol=specs[1][1])
    o = pyoracle.Oracle(cfg)
    o.set_state(abi.PVAR, p)
    o.first_step()
    for _ in range(7):
        assert o.step() == 0
    assert o.status().n_adj == members[1].status().n_adj and o.status().time == members[1].status().time
    assert np.array_equal(o.get(abi.CVAR), members[1].get(abi.CVAR))
    # a second round continues from the members' state
    assert b.run(3) == len(specs)
    for s in alone:
        s.run(3)
    for m, s in zip(members, alone):
        assert np.array_equal(m.get(abi.CVAR), s.get(abi.CVAR))


def _fargo_member(sp, fargo, exact):
    """A disk with FARGO transport (type 1, or type 2 with the Keplerian w) after FirstStep and
    one step alone (the first step after FirstStep has its own frame changes)."""
    from fosite_b200.sim import Simulation
    nr, nphi, geometry, hratio, sigma, seed = sp
    cfg, p, extra = problems.disk2d(nr=nr, nphi=nphi, seed=seed, hratio=hratio, sigma_index=sigma,
                                    geometry=geometry, fargo=fargo)
    s = Simulation(cfg, exact=exact)
    shape = (1, nphi + 4, nr + 4)
    s.set_sound_speeds(np.broadcast_to(extra["bccsound"], shape), np.broadcast_to(extra["fcsound"], (4,) + shape))
    if fargo == 2:
        X, _, _, _ = problems.centers(cfg)
        x = X[0, 0, :]
        r = np.exp(x) if geometry == abi.LOGCYLINDRICAL else x
        s.set_fargo_velocity(np.sqrt(1.0 / r))
    s.set_state(abi.PVAR, p)
    assert s.first_step() == 0
    assert s.step() == 0
    return s


@pytest.mark.parametrize("exact", [True, False])
def test_fargo_disk_batch_matches_single_grids(exact):
    """FARGO members (types 1 and 2, cylindrical and logcylindrical, mixed with a member
    without FARGO): background velocity, advection and w update over the batch's tables give
    every member exactly its lone run."""
    from fosite_b200.sim import Batch
    specs = _disk_specs(6, seed=13)
    kinds = [1, 1, 2, 1, 0, 2]
    members = [_fargo_member(sp, f, exact) for sp, f in zip(specs, kinds)]
    alone = [_fargo_member(sp, f, exact) for sp, f in zip(specs, kinds)]
    b = Batch(members)
    assert b.run(21) == len(members)
    for s in alone:
        rc, done = s.run(21)
        assert rc == 0 and done == 21
    for m, s in zip(members, alone):
        assert (m.status().iter, m.status().time, m.status().dt) == (s.status().iter, s.status().time, s.status().dt)
        assert np.array_equal(m.get(abi.CVAR), s.get(abi.CVAR))
        assert np.array_equal(m.get(abi.PVAR), s.get(abi.PVAR))
    b.close()


def test_fargo_x_batch_and_rejections():
    """FARGO along x (the reference's KHI2D legs, ideal gas) in a batch equals the lone runs;
    members must have stepped once alone and share the transport direction."""
    from fosite_b200.sim import Batch, FositeError, Simulation
    from cases import khi_fargo

    def member(fargo, direction, step=True):
        cfg, p, extra = khi_fargo(fargo, direction=direction, n=(24, 26))
        s = Simulation(cfg, exact=True)
        if "fargo_w" in extra:
            s.set_fargo_velocity(extra["fargo_w"])
        s.set_state(abi.PVAR, p)
        assert s.first_step() == 0
        if step:
            assert s.step() == 0
        return s

    members = [member(1, 1), member(2, 1)]
    alone = [member(1, 1), member(2, 1)]
    b = Batch(members)
    assert b.run(19) == 2
    for m, s in zip(members, alone):
        assert s.run(19) == (0, 19)
        assert m.status().time == s.status().time
        assert np.array_equal(m.get(abi.CVAR), s.get(abi.CVAR))
    b.close()
    with pytest.raises(FositeError):
        Batch([member(1, 1, step=False)])        # first step after FirstStep not taken alone
    with pytest.raises(FositeError):
        Batch([member(1, 1), member(1, 2)])      # different transport directions


@pytest.mark.parametrize("order", [2, 3])
def test_adaptive_modified_euler_batch_equals_lone_runs(order):
    """Members with the embedded modified Euler scheme (fosite's default tol_rel < 1) of
    different sizes and tolerances in one batch: the per-member first-stage update, the stages
    with the embedded solution and each member's controller give every member exactly its
    lone device-clock run (rejections and sub-steps included) and the oracle's steps."""
    import pyoracle
    from fosite_b200.sim import Batch, Simulation
    specs = [((30, 28), 1e-3), ((24, 36), 3e-4), ((40, 20), 1e-3)]

    def make():
        out = []
        for n, tol in specs:
            cfg, p, _ = _khi(n=n, tdorder=order, me_tol=tol, limiter=abi.MONOCENT, variables=abi.PRIMITIVE)
            s = Simulation(cfg, exact=True)
            s.set_state(abi.PVAR, p)
            s.first_step()
            out.append(s)
        return out
    members, alone = make(), make()
    b = Batch(members)
    assert b.run(9) == len(specs)
    for s in alone:
        assert s.run(9) == (0, 9)
    for m, s in zip(members, alone):
        sm, ss = m.status(), s.status()
        assert (sm.time, sm.dt, sm.iter, sm.n_adj) == (ss.time, ss.dt, ss.iter, ss.n_adj)
        assert np.array_equal(m.get(abi.CVAR), s.get(abi.CVAR))
    assert sum(m.status().n_adj for m in members) > 0
    cfg, p, _ = _khi(n=specs[1][0], tdorder=order, me_tol=specs[1][1], limiter=abi.MONOCENT, variables=abi.PRIMITIVE)
    o = pyoracle.Oracle(cfg)
    o.set_state(abi.PVAR, p)
    o.first_step()
    for _ in range(9):
        assert o.step() == 0
    assert o.status().time == members[1].status().time
    assert np.array_equal(o.get(abi.CVAR), members[1].get(abi.CVAR))
    b.close()
