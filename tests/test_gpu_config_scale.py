"""The benchmark configurations at their full sizes against the oracle.

tests/golden/pin_*.npz hold what the oracle gives on the benchmark's own synthetic set-ups
(tests/golden/make_config_pins.py): the SHA-256 of the interior cvar block, per-variable sums
and, for the disk, every cell of the rows next to the stage tiles' y seams.  The --fmad=false
build must reproduce the hashes bit for bit (the exact build equals the oracle); the product
build is then compared with the exact build's state, which makes its relative L1 against the
oracle exact too.  Bars (relative L1 of the state vector, sum|a-b|/sum|b|): 1e-12 after one
step, 1e-9 after 1000 (KHI) or 2000 (disk) steps; mass, momentum and energy of the periodic
KHI box and the reflecting 3D box conserved to 1e-13 relative.
"""
import hashlib
import os

import numpy as np
import pytest

from fosite_b200 import abi, problems

pyoracle = pytest.importorskip("pyoracle")

HERE = os.path.dirname(os.path.abspath(__file__))


def _pin(name):
    return np.load(os.path.join(HERE, "golden", "pin_%s.npz" % name))


def _interior(a, cfg):
    sl = [slice(None)]
    for n in (cfg.knum, cfg.jnum, cfg.inum):
        sl.append(slice(2, -2) if n > 1 else slice(None))
    return np.ascontiguousarray(a[tuple(sl)])


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def rel_l1(a, b):
    return float(np.abs(a - b).sum() / np.abs(b).sum())


def _sim(cfg, p, extra, exact, variant=None, monkeypatch=None):
    from fosite_b200.sim import Simulation
    if variant is not None:
        monkeypatch.setenv("FGPU_STAGE_VARIANT", str(variant))
    g = Simulation(cfg, exact=exact)
    if "bccsound" in extra:
        shape = g.shape
        g.set_sound_speeds(np.broadcast_to(extra["bccsound"], shape), np.broadcast_to(extra["fcsound"], (4,) + shape))
    g.set_state(abi.PVAR, p)
    if variant is None:
        g.autotune(3)
    return g


def _check_status(g, pin, tag):
    st = g.status()
    assert (st.time, st.dt, st.iter, st.n_adj) == (float(pin[tag + "_time"]), float(pin[tag + "_dt"]),
                                                    int(pin[tag + "_iter"]), int(pin[tag + "_nadj"])), tag


@pytest.mark.gpu
@pytest.mark.parametrize("variant,tpb", [(None, None), (4, None), (6, None), (6, 4)])
def test_khi256_bitwise_1000_steps(variant, tpb, monkeypatch):
    """KHI 256^2, SSPRK3: the exact build's state after 1 and 1000 steps is the oracle's bit for
    bit (tuned layout, shared-memory tile, TMA-staged tile, TMA tiles in columns of four)."""
    pin = _pin("khi256")
    if tpb:
        monkeypatch.setenv("FGPU_TMA_TPB", str(tpb))
    cfg, p, extra = problems.khi2d(n=256)
    g = _sim(cfg, p, extra, True, variant, monkeypatch)
    g.first_step()
    assert g.step() == 0
    assert _sha(_interior(g.get(abi.CVAR), cfg)) == str(pin["s1_sha256"])
    _check_status(g, pin, "s1")
    assert g.run(999)[1] == 999
    assert _sha(_interior(g.get(abi.CVAR), cfg)) == str(pin["s1000_sha256"])
    _check_status(g, pin, "s1000")
    g.close()


@pytest.mark.gpu
def test_khi256_product_build_and_conservation():
    """KHI 256^2 product build: relative L1 <= 1e-12 after 1 step and <= 1e-9 after 1000 steps;
    mass, momentum and energy of the periodic box conserved to 1e-13 relative."""
    cfg, p, extra = problems.khi2d(n=256)
    ex = _sim(cfg, p, extra, True)
    fa = _sim(cfg, p, extra, False)
    for g in (ex, fa):
        g.first_step()
    c0 = _interior(fa.get(abi.CVAR), cfg).reshape(4, -1)
    for n, bar in ((1, 1e-12), (999, 1e-9)):
        assert ex.run(n)[1] == n and fa.run(n)[1] == n
        a, b = _interior(fa.get(abi.CVAR), cfg), _interior(ex.get(abi.CVAR), cfg)
        r = rel_l1(a, b)
        assert r <= bar, (n, r)
    c1 = a.reshape(4, -1)
    for v in range(4):
        scale = np.abs(c0[v]).sum()
        drift = abs(c1[v].sum() - c0[v].sum()) / scale
        assert drift <= 1e-13, (v, drift)
    ex.close()
    fa.close()


@pytest.mark.gpu
@pytest.mark.parametrize("exact,variant", [(True, None), (False, None), (True, 6), (False, 7)])
def test_disk512_fargo(exact, variant, monkeypatch):
    """Logcylindrical isothermal disk 512x1024 with FARGO and absorbing radial boundaries (tuned
    layout, and the TMA-staged tiles with their frame changes): one step against the oracle run
    here, 2000 steps against the pinned rows."""
    pin = _pin("disk512")
    cfg, p, extra = problems.disk2d(nr=512, nphi=1024, fargo=1)
    g = _sim(cfg, p, extra, exact, variant, monkeypatch)
    if variant is not None:
        assert g.stage_layout()[0] == variant
    o = pyoracle.Oracle(cfg)
    o.set_sound_speeds(np.broadcast_to(extra["bccsound"], o.shape), np.broadcast_to(extra["fcsound"], (4,) + o.shape))
    o.set_state(abi.PVAR, p)
    o.first_step()
    g.first_step()
    assert o.step() == 0 and g.step() == 0
    r1 = rel_l1(_interior(g.get(abi.CVAR), cfg), _interior(o.get(abi.CVAR), cfg))
    # the absorbing boundaries call CUDA's exp/log, within an ulp of glibc's
    assert r1 <= (1e-13 if exact else 1e-12), r1
    del o
    assert g.run(1999)[1] == 1999
    c = _interior(g.get(abi.CVAR), cfg)
    rows = pin["rows_j"]
    r = rel_l1(c[:, 0, rows, :], pin["s2000_rows"])
    assert r <= 1e-9, r
    sums = c.reshape(3, -1).sum(axis=1)
    assert np.all(np.abs(sums - pin["s2000_sum"]) <= 1e-9 * pin["s2000_abssum"]), (sums, pin["s2000_sum"])
    st = g.status()
    assert st.iter == int(pin["s2000_iter"])
    # dt follows the state: within the state's bar (the exact build's exp/log differ by an ulp)
    assert abs(st.time - float(pin["s2000_time"])) <= 1e-10 * float(pin["s2000_time"])
    g.close()


@pytest.mark.gpu
def test_gauss256_one_step():
    """3D Gaussian pulse 256^3, Dormand-Prince, the tuned layout: the exact build after FirstStep
    and one step is the oracle's state bit for bit; the product build within 1e-12; mass and
    energy of the reflecting box conserved to 1e-13 relative."""
    pin = _pin("gauss256")
    cfg, p, extra = problems.gauss3d(n=256)
    ex = _sim(cfg, p, extra, True)
    ex.first_step()
    c0 = _interior(ex.get(abi.CVAR), cfg).reshape(5, -1)
    assert ex.step() == 0
    b = _interior(ex.get(abi.CVAR), cfg)
    assert _sha(b) == str(pin["s1_sha256"])
    _check_status(ex, pin, "s1")
    ex.close()
    fa = _sim(cfg, p, extra, False)
    fa.first_step()
    assert fa.step() == 0
    a = _interior(fa.get(abi.CVAR), cfg)
    r = rel_l1(a, b)
    assert r <= 1e-12, r
    c1 = a.reshape(5, -1)
    for v in (0, 4):
        drift = abs(c1[v].sum() - c0[v].sum()) / np.abs(c0[v]).sum()
        assert drift <= 1e-13, (v, drift)
    fa.close()
