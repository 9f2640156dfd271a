"""The allocation-free CFL entry point against the handle-based one.

Callers such as memory-capped services or real-time loops may be barred from
calling cudaMalloc after start-up; fgpu_calc_timestep_noalloc serves them from
a fixed file-scope device array.  This file is collected last so that a run
stopping at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from fosite_b200 import abi
from cases import CASES, _khi


def _entry():
    from fosite_b200.sim import lib
    L = lib()
    L.fgpu_calc_timestep_noalloc.argtypes = [C.POINTER(abi.Config), C.c_void_p, C.c_void_p, C.c_void_p]
    return L


def _noalloc_dt(cfg, state, dt_dev):
    import torch
    rc = _entry().fgpu_calc_timestep_noalloc(C.byref(cfg), C.c_void_p(state.data_ptr()),
                                             C.c_void_p(dt_dev.data_ptr()),
                                             C.c_void_p(torch.cuda.current_stream().cuda_stream))
    return rc


def _axis_cartesian():
    # a Cartesian box with an AXIS face (reflecting with the axis masks) at x = xmin
    return _khi(n=(28, 24), bcs=[abi.AXIS, abi.REFLECTING, abi.PERIODIC, abi.PERIODIC], seed=5)


CALLS = {name: CASES[name] for name in ("khi_ssprk3_vanleer_cons", "gauss3d_dopri_mc_prim",
                                        "iso3d_cashkarp_mixed_bc", "euler2d_absorbing")}
CALLS["khi_axis_cartesian"] = _axis_cartesian


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CALLS))
def test_calc_timestep_noalloc_matches_handle(name):
    """dt equals the handle's CalcTimestep bit for bit, on two calls in a row, and the calls
    take no device memory."""
    import torch
    from fosite_b200.sim import Simulation
    cfg, p, _ = CALLS[name]()
    sim = Simulation(cfg)
    sim.set_state(abi.PVAR, p)
    dt_ref = sim.calc_timestep()
    cv = sim.get(abi.CVAR)
    sl = [slice(None)] + [slice(2, -2) if n > 1 else slice(None) for n in (cfg.knum, cfg.jnum, cfg.inum)]
    interior = np.ascontiguousarray(cv[tuple(sl)])
    state = torch.from_numpy(interior).cuda()
    dt_dev = torch.zeros(1, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    free0 = None
    for call in range(3):
        dt_dev.fill_(-1.0)
        assert _noalloc_dt(sim.cfg, state, dt_dev) == 0
        torch.cuda.synchronize()
        assert float(dt_dev.item()) == dt_ref
        if call == 0:
            free0 = torch.cuda.mem_get_info()[0]
    assert torch.cuda.mem_get_info()[0] == free0
    sim.close()


@pytest.mark.gpu
def test_calc_timestep_noalloc_rejections():
    """A mesh whose metric does not fit the scratch array gives FGPU_EARG, a curvilinear mesh
    FGPU_EUNSUPPORTED; neither launches anything (the state pointer is never read)."""
    import torch
    state = torch.zeros(16, dtype=torch.float64, device="cuda")
    dt_dev = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    cfg, _, _ = _khi(n=(40, 36))
    big = abi.config_copy(cfg)
    big.inum = 6000
    assert _noalloc_dt(big, state, dt_dev) == abi.EARG
    cyl = abi.config_copy(cfg)
    cyl.geometry = abi.CYLINDRICAL
    assert _noalloc_dt(cyl, state, dt_dev) == abi.EUNSUPPORTED
    torch.cuda.synchronize()
    assert float(dt_dev.item()) == -1.0
