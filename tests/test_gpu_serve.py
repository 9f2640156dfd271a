"""Serving loop: continuous batching over a request stream on one GPU."""
import numpy as np
import pytest

from fosite_b200 import abi
from fosite_b200.serve import Request, Server, build_problem, footprint_bytes

pytestmark = pytest.mark.gpu


def _requests():
    return [
        Request("khi", (48, 48), 0.01, seed=1, arrival=0.0),
        Request("disk", (40, 72), 0.004, seed=2, arrival=0.0),
        Request("disk", (64, 40), 0.006, seed=3, arrival=0.001),
        Request("pulse", (16, 16, 16), 0.004, seed=4, arrival=0.002),
        Request("khi", (64, 64), 0.006, seed=5, arrival=0.003),
        Request("pulse", (20, 20, 20), 0.003, seed=6, arrival=0.004),
        Request("disk", (32, 64), 0.005, seed=7, arrival=0.005),
    ]


def test_alone_and_mixed_results_are_identical():
    reqs = _requests()
    mixed = Server(hbm_budget_bytes=1 << 33, chunk=5, exact=True, keep_results=True)
    rep = mixed.serve(reqs, timeout_s=300)
    assert rep["requests"] == len(reqs)
    by_seed = {r.seed: r for r in mixed.done}
    for seed in (2, 4, 5):
        r0 = [r for r in _requests() if r.seed == seed][0]
        r0.arrival = 0.0
        alone = Server(hbm_budget_bytes=1 << 33, chunk=7, exact=True, keep_results=True)
        alone.serve([r0], timeout_s=300)
        ra = alone.done[0]
        rm = by_seed[seed]
        assert ra.status == rm.status == abi.STOPTIME
        assert ra.steps == rm.steps
        assert np.array_equal(ra.result, rm.result)


def test_batched_request_equals_plain_simulation():
    """A served request ends with exactly the state of a lone fgpu_run to its stop time."""
    from fosite_b200.sim import Simulation
    req = Request("disk", (40, 72), 0.004, seed=2)
    srv = Server(hbm_budget_bytes=1 << 33, chunk=3, exact=True, keep_results=True)
    srv.serve([req, Request("disk", (64, 40), 0.006, seed=3)], timeout_s=300)
    got = [r for r in srv.done if r.seed == 2][0]
    cfg, p, extra = build_problem(Request("disk", (40, 72), 0.004, seed=2))
    s = Simulation(cfg, exact=True)
    s.set_sound_speeds(np.broadcast_to(extra["bccsound"], s.shape), np.broadcast_to(extra["fcsound"], (4,) + s.shape))
    s.set_state(abi.PVAR, p)
    s.first_step()
    rc, done = s.run(100000)
    assert rc == abi.STOPTIME and done == got.steps
    assert np.array_equal(s.get(abi.CVAR), got.result)


def test_admission_respects_hbm_budget():
    reqs = _requests()
    fps = [footprint_bytes(build_problem(r)[0]) for r in reqs]
    budget = int(2.2 * max(fps))
    srv = Server(hbm_budget_bytes=budget, chunk=4, exact=False)
    peak = [0]
    orig = srv._admit

    def admit():
        orig()
        peak[0] = max(peak[0], srv.used)
    srv._admit = admit
    rep = srv.serve(reqs, timeout_s=300)
    assert rep["requests"] == len(reqs)
    assert 0 < peak[0] <= budget
    assert all(r.status == abi.STOPTIME for r in srv.done)
    assert rep["p99_s"] >= rep["p50_s"] > 0
