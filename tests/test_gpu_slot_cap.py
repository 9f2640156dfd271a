"""The no-progress guard of the device-clock loops.

Embedded Runge-Kutta schemes run on the device clock: the host replays captured attempt
slots and reads the control block every few slots, giving up with FGPU_ETIMEOUT once a
slot budget (64 per requested step + 64) is spent without the steps completing.
FGPU_SLOT_CAP replaces the budget so that these tests can make it run out: the call must
come back with FGPU_ETIMEOUT, the handle's bookkeeping must be the device's, and the state
must be a valid one from which stepping continues to the oracle's result.
"""
import numpy as np
import pytest

from fosite_b200 import abi
from cases import _gauss3d
from test_gpu_parity import _interior

pyoracle = pytest.importorskip("pyoracle")


@pytest.mark.gpu
def test_single_grid_timeout_then_resume(monkeypatch):
    from fosite_b200.sim import FositeError, Simulation
    # Dormand-Prince with tolerance 1e-2: every step of this run is one attempt
    cfg, p, _ = _gauss3d(tol=1e-2)
    o = pyoracle.Oracle(cfg)
    o.set_state(abi.PVAR, p)
    o.first_step()
    for _ in range(20):
        assert o.step() == 0
    so = o.status()
    # one attempt per step in this run: a slot boundary is a step boundary
    assert so.iter == 20 and so.n_adj == 0
    g = Simulation(cfg, exact=True)
    g.set_state(abi.PVAR, p)
    g.first_step()
    monkeypatch.setenv("FGPU_SLOT_CAP", "0")
    with pytest.raises(FositeError) as e:
        g.run(20)
    assert e.value.code == abi.ETIMEOUT
    done = g.status().iter
    assert 0 < done < 20
    c = g.get(abi.CVAR)
    assert np.all(np.isfinite(c))
    monkeypatch.delenv("FGPU_SLOT_CAP")
    rc, n = g.run(20 - done)
    assert n == 20 - done
    sg = g.status()
    assert (sg.iter, sg.n_adj, sg.time, sg.dt) == (so.iter, so.n_adj, so.time, so.dt)
    a, b = _interior(g.get(abi.CVAR), cfg), _interior(o.get(abi.CVAR), cfg)
    assert np.array_equal(a, b)
    g.close()


@pytest.mark.gpu
def test_batch_timeout_returns(monkeypatch):
    """Members with a tight error tolerance need several attempts per step; with no slot budget
    beyond the first replay the batched loop returns FGPU_ETIMEOUT, its members' bookkeeping
    taken from the device and their states finite."""
    from fosite_b200.sim import Batch, FositeError, Simulation
    sims = []
    for seed in (3, 4):
        cfg, p, _ = _gauss3d(n=(16, 12, 10), tol=1e-9, seed=seed)
        s = Simulation(cfg)
        s.set_state(abi.PVAR, p)
        s.first_step()
        sims.append(s)
    b = Batch(sims)
    monkeypatch.setenv("FGPU_SLOT_CAP", "0")
    with pytest.raises(FositeError) as e:
        b.run(4)
    assert e.value.code == abi.ETIMEOUT
    for s in sims:
        st = s.status()
        assert st.iter >= 0 and np.isfinite(st.time) and st.dt > 0
        assert np.all(np.isfinite(s.get(abi.CVAR)))
    b.close()
    for s in sims:
        s.close()
