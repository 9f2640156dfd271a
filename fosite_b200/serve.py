"""Serving loop: solve requests arriving as a stream, packed into batched launches.

Each request is one fosite run (a 2D Kelvin-Helmholtz box, a 2D isothermal
disk or a 3D Gaussian pulse) integrated from its initial data to its stop time
``t_end``.  The server

  * admits waiting requests by HBM footprint (the sum of the admitted grids'
    device arrays stays below a budget; requests that do not fit wait, later
    smaller ones may pass them);
  * keeps every admitted grid resident on the device from its upload to its
    final download;
  * groups the running grids by kernel class (dimensionality, physics,
    reconstruction variables, time integrator) and advances each class as ONE
    batch (``fgpu_batch_*``): one persistent stage launch per Runge-Kutta stage
    over the tiles of all its grids (embedded schemes: one replayed attempt slot
    per round trip, every grid with its own step-size controller).  Membership changes between scheduling
    rounds (continuous batching): new grids join, finished ones leave;
  * records per request the arrival, admission and completion times.

A grid's result does not depend on what it was batched with: batched and lone
stepping are bitwise identical (tests/test_gpu_serve.py checks this).
"""
import time
from dataclasses import dataclass, field

import numpy as np

from . import abi, problems


@dataclass
class Request:
    kind: str          # "khi" | "disk" | "pulse"
    size: tuple        # (nx, ny) or (nx, ny, nz)
    t_end: float
    seed: int = 0
    arrival: float = 0.0        # seconds after the start of the run
    # filled by the server
    admitted: float = None
    finished: float = None
    steps: int = 0
    cells: int = 0
    result: np.ndarray = None
    status: int = 0
    rid: int = field(default=-1)
    # the request's initial data (cfg, pvar, extra) when it arrives with it; otherwise the
    # server generates it from kind/size/seed at admission
    payload: tuple = None


def build_problem(req):
    """(cfg, pvar, extra) of a request, with its stop time."""
    if req.payload is not None:
        return req.payload
    if req.kind == "khi":
        cfg, p, extra = problems.khi2d(n=req.size[0], seed=req.seed)
    elif req.kind == "disk":
        rng = np.random.default_rng(req.seed)
        cfg, p, extra = problems.disk2d(nr=req.size[0], nphi=req.size[1], seed=req.seed,
                                        hratio=float(rng.uniform(0.03, 0.1)),
                                        sigma_index=float(rng.uniform(-1.5, -0.5)),
                                        geometry=abi.LOGCYLINDRICAL if req.seed % 2 else abi.CYLINDRICAL,
                                        fargo=0)
    elif req.kind == "pulse":
        # Dormand-Prince 5(4) with tolerance 1e-5: an embedded-scheme batch class
        cfg, p, extra = problems.gauss3d(n=req.size[0], seed=req.seed)
    else:
        raise ValueError("unknown request kind %r" % req.kind)
    cfg.stoptime = float(req.t_end)
    cfg.dtlimit = 0.0
    abi.finalize_config(cfg)
    return cfg, p, extra


STAGES = {abi.DORMAND_PRINCE: 7, abi.RK_FEHLBERG: 6, abi.CASH_KARP: 6, abi.SSPRK: 5}


def footprint_bytes(cfg):
    """Device bytes of one admitted grid: its state arrays (stored state and two stage
    scratch arrays for the fixed-step scheme, with primitive reconstruction their primitive
    forms too; stored state, cold state, m k-arrays and the
    formed stage state for an embedded scheme of m stages), the padded download scratch, the
    metric and, with FARGO along y, the background-velocity terms."""
    nd = 3 if cfg.knum > 1 else 2
    vnum = 1 + nd + (1 if cfg.physics == abi.EULER else 0)
    n = cfg.inum * cfg.jnum * cfg.knum
    npad = (cfg.inum + 4) * (cfg.jnum + 4) * (cfg.knum + 4 if nd == 3 else 1)
    arrays = 3
    if cfg.method == abi.MODIFIED_EULER and cfg.variables == abi.PRIMITIVE and cfg.tol_rel >= 1.0:
        arrays += 2     # the primitive forms of the two scratch stage results
    if cfg.method != abi.MODIFIED_EULER:
        m = STAGES.get(cfg.method, 7)
        if cfg.method in (abi.RK_FEHLBERG, abi.SSPRK) and cfg.tdorder == 3:
            m = 3
        arrays = 3 + m
    fargo_terms = (cfg.inum + 4) * cfg.jnum if cfg.fargo_method and cfg.fargo_direction != 1 else 0
    return 8 * vnum * (arrays * n + 2 * npad) + 8 * 40 * (cfg.inum + 4) + 8 * fargo_terms + (1 << 16)


def kernel_class(cfg):
    nd = 3 if cfg.knum > 1 else 2
    return (nd, cfg.physics, cfg.variables, cfg.method, cfg.tdorder)


class Server:
    """Continuous-batching solver for a request stream on one GPU."""

    def __init__(self, hbm_budget_bytes, device=-1, chunk=8, exact=False, keep_results=False, autotune=False):
        self.budget = int(hbm_budget_bytes)
        self.device = device
        self.chunk = int(chunk)
        self.exact = exact
        self.keep = keep_results
        self.autotune = autotune
        self.used = 0
        self.waiting = []
        self.classes = {}      # key -> {"members": [(req, sim, fp)], "batch": Batch or None, "dirty": bool}
        self.done = []
        self.t0 = None
        self.rounds = 0
        self.cell_updates = 0

    def now(self):
        return time.perf_counter() - self.t0

    def _admit(self):
        from .sim import Simulation
        still = []
        for req in self.waiting:
            cfg, p, extra = build_problem(req)
            fp = footprint_bytes(cfg)
            if self.used + fp > self.budget:
                still.append(req)
                continue
            sim = Simulation(cfg, device=self.device, exact=self.exact)
            if "bccsound" in extra:
                shape = sim.shape
                sim.set_sound_speeds(np.broadcast_to(extra["bccsound"], shape),
                                     np.broadcast_to(extra["fcsound"], (sim.nfaces,) + shape))
            sim.set_state(abi.PVAR, p)
            rc = sim.first_step()
            req.admitted = self.now()
            req.cells = cfg.inum * cfg.jnum * cfg.knum
            if rc != 0:
                req.status = rc
                req.finished = self.now()
                self.done.append(req)
                sim.close()
                continue
            self.used += fp
            key = kernel_class(cfg)
            cl = self.classes.setdefault(key, {"members": [], "batch": None, "dirty": True})
            cl["members"].append((req, sim, fp))
            cl["dirty"] = True
        self.waiting = still

    def _retire(self, cl):
        keep = []
        for req, sim, fp in cl["members"]:
            st = sim.status()
            if st.brk or abs(req.t_end - st.time) <= 1e-5 * req.t_end:
                req.finished = self.now()
                req.steps = int(st.iter)
                req.status = abi.BREAK if st.brk else abi.STOPTIME
                if self.keep:
                    req.result = sim.get(abi.CVAR)
                self.cell_updates += req.steps * req.cells
                self.used -= fp
                sim.close()
                self.done.append(req)
                cl["dirty"] = True
            else:
                keep.append((req, sim, fp))
        cl["members"] = keep

    def round(self):
        """One scheduling round: (re)batch and enqueue chunk steps of every class, admit
        waiting requests while the GPU runs them (host-side set-up overlaps the
        batched launches), then wait and retire finished requests."""
        from .sim import Batch
        active = []
        for key, cl in self.classes.items():
            if not cl["members"]:
                if cl["batch"]:
                    cl["batch"].close()
                    cl["batch"] = None
                continue
            if cl["dirty"] or cl["batch"] is None:
                if cl["batch"]:
                    cl["batch"].close()
                cl["batch"] = Batch([s for _, s, _ in cl["members"]])
                if self.autotune:
                    cl["batch"].autotune(2)
                cl["dirty"] = False
            cl["batch"].enqueue(self.chunk)
            active.append(cl)
        self._admit()
        for cl in active:
            cl["batch"].collect()
        for cl in active:
            self._retire(cl)
        self.rounds += 1
        return len(active)

    def serve(self, requests, timeout_s=600.0):
        """Run a request stream (arrival times relative to the start) to completion."""
        pending = sorted(requests, key=lambda r: r.arrival)
        for k, r in enumerate(pending):
            r.rid = k
        self.t0 = time.perf_counter()
        i = 0
        while i < len(pending) or self.waiting or any(cl["members"] for cl in self.classes.values()):
            t = self.now()
            if t > timeout_s:
                raise TimeoutError("serving run exceeded %.0f s" % timeout_s)
            while i < len(pending) and pending[i].arrival <= t:
                self.waiting.append(pending[i])
                i += 1
            self.round()
            running = any(cl["members"] for cl in self.classes.values())
            if not running and not self.waiting and i < len(pending):
                time.sleep(max(0.0, min(0.01, pending[i].arrival - self.now())))
        for cl in self.classes.values():
            if cl["batch"]:
                cl["batch"].close()
                cl["batch"] = None
        return self.report()

    def report(self):
        lat = np.array([r.finished - r.arrival for r in self.done if r.finished is not None])
        span = max((r.finished for r in self.done), default=0.0)
        return {
            "requests": len(self.done),
            "p50_s": float(np.percentile(lat, 50)) if lat.size else None,
            "p99_s": float(np.percentile(lat, 99)) if lat.size else None,
            "mean_s": float(lat.mean()) if lat.size else None,
            "makespan_s": span,
            "cell_updates": int(self.cell_updates),
            "cell_updates_per_s": self.cell_updates / span if span > 0 else None,
            "rounds": self.rounds,
        }


def poisson_stream(rate, n, seed=0, t_scale=1.0, mix=("khi", "disk", "pulse"), size_cap=None):
    """n requests with exponential inter-arrival times at the given rate (1/s).

    Sizes are drawn from the ranges of the mixed serving workload (KHI 64^2 to
    1024^2, disks 64x128 to 512x1024, pulses 32^3 to 128^3, powers of two) and
    t_end uniformly in [0.1, 2] characteristic times, multiplied by t_scale
    (KHI: box crossing time 1; disk: inner orbit 2*pi*0.4**1.5; pulse: sound
    crossing time 1/sqrt(1.4*11)).  size_cap limits the largest size index.
    """
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for k in range(n):
        t += rng.exponential(1.0 / rate)
        kind = mix[int(rng.integers(0, len(mix)))]
        f = float(rng.uniform(0.1, 2.0)) * t_scale
        if kind == "khi":
            e = int(rng.integers(0, 5 if size_cap is None else min(5, size_cap + 1)))
            size, t_end = (64 << e, 64 << e), f * 1.0
        elif kind == "disk":
            e = int(rng.integers(0, 4 if size_cap is None else min(4, size_cap + 1)))
            size, t_end = (64 << e, 128 << e), f * 2 * np.pi * 0.4 ** 1.5
        else:
            e = int(rng.integers(0, 3 if size_cap is None else min(3, size_cap + 1)))
            size, t_end = (32 << e, 32 << e, 32 << e), f / np.sqrt(1.4 * 11.0)
        out.append(Request(kind=kind, size=size, t_end=t_end, seed=seed * 1000 + k, arrival=t))
    return out
