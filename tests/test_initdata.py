"""GetCentrifugalVelocity (timedisc_base.f90:2355-2530) on the oracle's RHS: for a thin
isothermal disk around a point mass the balanced rotation is the pressure-corrected
Keplerian velocity, and the radial velocity is zero."""
import numpy as np
import pytest

from fosite_b200 import abi, initdata, problems

pyoracle = pytest.importorskip("pyoracle")


@pytest.mark.parametrize("geometry", [abi.CYLINDRICAL, abi.LOGCYLINDRICAL])
def test_centrifugal_velocity_of_a_disk(geometry):
    cfg, p, extra = problems.disk2d(nr=64, nphi=32, seed=5, hratio=0.05, geometry=geometry, fargo=0)
    p[0] = np.where(p[0] > 0, p[0], 1.0)
    X, _, _, _ = problems.centers(cfg)
    r = np.exp(X) if geometry == abi.LOGCYLINDRICAL else X
    p[0] = r ** -1.0                     # smooth sigma ~ 1/r (no noise)
    p[1] = 0.0                           # at rest: the RHS holds gravity and pressure only
    p[2] = 0.0
    o = pyoracle.Oracle(cfg)
    o.set_sound_speeds(np.broadcast_to(extra["bccsound"], o.shape), np.broadcast_to(extra["fcsound"], (4,) + o.shape))
    o.set_state(abi.PVAR, p)
    o.compute_rhs()
    with np.errstate(divide="ignore", invalid="ignore"):
        v = initdata.centrifugal_velocity(cfg, o.mesh, o.get(abi.RHS), p)
    sl = (slice(None), slice(2, -2), slice(4, -4))
    vk = np.sqrt(1.0 / r) * np.sqrt(1.0 - 2.0 * 0.05 ** 2)      # sigma ~ r^-1, cs^2 ~ 1/r
    assert np.all(v[0][sl] == 0.0)
    rel = np.abs(v[1][sl] - vk[sl]) / vk[sl]
    assert rel.max() < 5e-3, rel.max()
