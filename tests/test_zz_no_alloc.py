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
from cases import CASES


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["khi_ssprk3_vanleer_cons", "gauss3d_dopri_mc_prim", "iso3d_cashkarp_mixed_bc"])
def test_calc_timestep_noalloc_matches_handle(name):
    import torch
    from fosite_b200.sim import Simulation, lib
    cfg, p, _ = CASES[name]()
    sim = Simulation(cfg)
    sim.set_state(abi.PVAR, p)
    dt_ref = sim.calc_timestep()
    cv = sim.get(abi.CVAR)
    sl = [slice(None)] + [slice(2, -2) if n > 1 else slice(None) for n in (cfg.knum, cfg.jnum, cfg.inum)]
    interior = np.ascontiguousarray(cv[tuple(sl)])
    state = torch.from_numpy(interior).cuda()
    dt_dev = torch.zeros(1, dtype=torch.float64, device="cuda")
    L = lib()
    L.fgpu_calc_timestep_noalloc.argtypes = [C.POINTER(abi.Config), C.c_void_p, C.c_void_p, C.c_void_p]
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        dt_dev.fill_(-1.0)
        rc = L.fgpu_calc_timestep_noalloc(C.byref(sim.cfg), C.c_void_p(state.data_ptr()),
                                          C.c_void_p(dt_dev.data_ptr()), C.c_void_p(stream))
        assert rc == 0
        torch.cuda.synchronize()
        assert float(dt_dev.item()) == dt_ref
    sim.close()
