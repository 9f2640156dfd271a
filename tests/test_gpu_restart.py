"""Restart through fosite's binary format: a GPU run is written, read back into a new
run with the file's start time, and that restarted run agrees with the oracle
restarted from the same file bit for bit."""
import numpy as np
import pytest

from fosite_b200 import abi, fileio
from cases import CASES

pyoracle = pytest.importorskip("pyoracle")
pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["khi_ssprk3_mc_prim", "gauss3d_dopri_mc_prim", "disk_fargo_cyl_cons_reflect"])
def test_restart_from_binary_file(tmp_path, name):
    from fosite_b200.sim import Simulation
    cfg, p, extra = CASES[name]()

    def cs(s, shape):
        if "bccsound" in extra:
            s.set_sound_speeds(np.broadcast_to(extra["bccsound"], shape), np.broadcast_to(extra["fcsound"], (4,) + shape))

    a = Simulation(cfg, exact=True)
    cs(a, a.shape)
    a.set_state(abi.PVAR, p)
    a.first_step()
    for _ in range(3):
        a.step()
    path = str(tmp_path / "snap.bin")
    fileio.save(a, path)
    data = fileio.read(path)
    assert data["/timedisc/time"] == a.status().time
    c2 = fileio.restart_config(cfg, data)
    q = fileio.restart_state(c2, data)
    g = Simulation(c2, exact=True)
    o = pyoracle.Oracle(c2)
    cs(g, g.shape)
    cs(o, o.shape)
    g.set_state(abi.PVAR, q)
    o.set_state(abi.PVAR, q)
    assert g.first_step() == 0 and o.first_step() == 0
    for _ in range(3):
        assert g.step() == o.step()
    assert g.status().time == o.status().time > c2.starttime
    sl = [slice(None)] + [slice(2, -2) if n > 1 else slice(None) for n in (cfg.knum, cfg.jnum, cfg.inum)]
    assert np.array_equal(g.get(abi.CVAR)[tuple(sl)], o.get(abi.CVAR)[tuple(sl)])
