"""GetCentrifugalVelocity through the GPU's ComputeRHS equals the oracle's, bit for bit."""
import numpy as np
import pytest

from fosite_b200 import abi, initdata, problems

pyoracle = pytest.importorskip("pyoracle")
pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("geometry", [abi.CYLINDRICAL, abi.LOGCYLINDRICAL])
def test_balance_rotation_matches_oracle(geometry):
    from fosite_b200.sim import Simulation
    cfg, p, extra = problems.disk2d(nr=40, nphi=48, seed=9, geometry=geometry, fargo=0)
    p[1] = 0.0
    p[2] = 0.0
    g = Simulation(cfg, exact=True)
    o = pyoracle.Oracle(cfg)
    for s in (g, o):
        s.set_sound_speeds(np.broadcast_to(extra["bccsound"], o.shape), np.broadcast_to(extra["fcsound"], (4,) + o.shape))
    with np.errstate(divide="ignore", invalid="ignore"):
        pg = initdata.balance_rotation(g, p)
        o.set_state(abi.PVAR, p)
        o.compute_rhs()
        vo = initdata.centrifugal_velocity(cfg, o.mesh, o.get(abi.RHS), p)
    sl = (slice(None), slice(None), slice(2, -2), slice(2, -2))
    assert np.array_equal(pg[1:3][sl], vo[sl])
    assert np.all(pg[2][:, 2:-2, 2:-2] > 0)
