"""Benchmark: cell-updates/s of fosite's explicit finite-volume step on B200.

Workload (default): 3D Euler Gaussian pressure pulse on a 256^3 Cartesian
grid, reflecting walls, KT fluxes with MC-limited primitive reconstruction,
Dormand-Prince 5(4) with embedded error control (tol 1e-5), CFL 0.4.  A "step"
is one fosite%Step (possibly several accepted sub-steps or rejected attempts);
cell-updates = interior cells x accepted steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl fosite_b200|reference]

N > 1 runs as one process per GPU under torch.distributed.run; each rank
advances its own replica of the grid (fosite's step does not shard across
GPUs here), timing is the maximum over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

WORKLOADS = {
    "gauss3d": "3D Euler Gaussian pulse, reflecting, KT+MC(prim), Dormand-Prince 5(4) tol 1e-5, CFL 0.4",
    "khi2d": "2D Kelvin-Helmholtz, periodic, KT+van Leer(cons), SSPRK3 fixed CFL 0.4",
    "disk2d": "2D isothermal Keplerian disk, logcylindrical (r x phi = n x 2n), point mass GM=1, sigma~1/r, "
              "cs/vK=0.05, FARGO shift, KT+van Leer(prim), SSPRK3 fixed CFL 0.4, absorbing r / periodic phi",
    "khi2d_visc": "khi2d with the KHI2D test's molecular viscosity at Reynolds number 1e4",
    "khi3d_visc": "3D Kelvin-Helmholtz (tests/KHI3D.f90 set-up), periodic, KT+MC 1.2(cons), SSPRK3 fixed "
                  "CFL 0.4, molecular viscosity at Reynolds number 1e4",
}
# the grid of each description is the line's config.grid


def make_problem(name, size):
    from fosite_b200 import problems
    if name == "gauss3d":
        return problems.gauss3d(n=size or 256)
    if name == "disk2d":
        nr = size or 512
        return problems.disk2d(nr=nr, nphi=2 * nr, fargo=1)
    if name == "khi2d_visc":
        return problems.khi2d(n=size or 256, re=1.0e4)
    if name == "khi3d_visc":
        return problems.khi3d(n=size or 128, re=1.0e4)
    return problems.khi2d(n=size or 256)


def apply_extra(sim, cfg, extra):
    """Radial sound-speed profiles of the isothermal disk (cell centres and faces)."""
    if "bccsound" in extra:
        shape = (cfg.knum, cfg.jnum + 4, cfg.inum + 4)
        sim.set_sound_speeds(np.broadcast_to(extra["bccsound"], shape),
                             np.broadcast_to(extra["fcsound"], (4,) + shape))


def algorithmic_bytes_per_cell_update(name, vnum):
    """Compulsory HBM traffic per interior cell and accepted step (fused design).

    Dormand-Prince with CHECK_ALL: end-of-step RHS reads the state and writes
    k1 and the round-tripped base (1+2), stages m=2..7 read base+k1..k_{m-1}
    and write k_m (27+6), the last stage also writes the new state (1):
    37 arrays.  SSPRK3 (modified Euler): 3 stages read the stage input and the
    start state, write the stage output: 8 arrays.  With FARGO the background
    velocity pass reads the state (1), the last stage writes a scratch state
    and the transport reads it and writes the state (2): 11 arrays.
    """
    arrays = {"gauss3d": 37, "disk2d": 11}.get(name, 8)
    fields = arrays * vnum
    if name.endswith("_visc"):
        # per stage the viscous pass reads the state and writes ND momentum + energy sources,
        # which the stage kernel reads: V + 2 (V - 1) more fields
        fields += 3 * (vnum + 2 * (vnum - 1))
    return fields * 8.0


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) >= 9:
                for k, nm in enumerate(names):
                    if r[5 + k].lower().startswith("active"):
                        reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_traffic_profile(name):
    """DRAM bytes per stage launch per cell from the committed ncu summary, or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f).get(name)
    except Exception:
        return None


HEADLINE_SIZE = {"gauss3d": 256, "khi2d": 256, "disk2d": 512, "khi2d_visc": 256, "khi3d_visc": 128}
# host memory of the oracle (it keeps the reference's face-state arrays) per ghost-padded cell,
# measured on the 3D Dormand-Prince workload: 2.2 KB
ORACLE_BYTES_PER_PADDED_CELL = 2400.0


def _padded_cells(name, size):
    if name in ("gauss3d", "khi3d_visc"):
        return (size + 4) ** 3
    if name == "disk2d":
        return (size + 4) * (2 * size + 4)
    return (size + 4) ** 2


def _mem_available():
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return float(line.split()[1]) * 1024.0
    except Exception:
        pass
    return 0.0


def oracle_size(name, full):
    """The headline grid if the oracle fits in half the available host memory, else the largest
    grid (multiple of 16) that does."""
    avail = 0.5 * _mem_available()
    size = full
    while size > 16 and _padded_cells(name, size) * ORACLE_BYTES_PER_PADDED_CELL > avail:
        size -= 16
    return size


def time_oracle(name, size, threads, budget_s, max_steps=200):
    """The oracle (C++ restatement of the reference CPU path) on the workload at `size`: FirstStep
    untimed, then fosite steps until the budget is spent; cell-updates (accepted steps x interior
    cells) per second."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from fosite_b200 import abi
    used = pyoracle.set_threads(threads if threads > 0 else (os.cpu_count() or 1))
    cfg, p, extra = make_problem(name, size)
    o = pyoracle.Oracle(cfg)
    apply_extra(o, cfg, extra)
    o.set_state(abi.PVAR, p)
    o.first_step()
    t0 = time.perf_counter()
    it0 = o.status().iter
    steps = 0
    while True:
        o.step()
        steps += 1
        if time.perf_counter() - t0 > budget_s or steps >= max_steps:
            break
    el = time.perf_counter() - t0
    upd = (o.status().iter - it0) * cfg.inum * cfg.jnum * cfg.knum
    grid = [cfg.inum, cfg.jnum, cfg.knum]
    return {"value": upd / el, "unit": "cell-updates/s", "cores": used, "kind": "port", "grid": grid,
            "sample": "%d fosite steps of the workload on a %dx%dx%d grid (%.1f s, oracle on %d host thread%s)"
                      % (steps, grid[0], grid[1], grid[2], el, used, "" if used == 1 else "s")}


def cpu_baseline(name, budget_s=20.0):
    """Bounded samples of the oracle on this host: all threads on a reduced grid, and the serial
    restatement (1 thread) on a smaller one."""
    small = {"gauss3d": 96, "disk2d": 256, "khi3d_visc": 48}.get(name, 256)
    cb = time_oracle(name, small, 0, 0.6 * budget_s)
    tiny = {"gauss3d": 48, "disk2d": 128, "khi3d_visc": 32}.get(name, 128)
    cb["serial"] = time_oracle(name, tiny, 1, 0.4 * budget_s)
    return cb


def dist_setup():
    from fosite_b200 import replicas
    return replicas.init()


def allmax(x, world):
    from fosite_b200 import replicas
    return replicas.allmax(x) if world > 1 else x


def allsum(x, world):
    from fosite_b200 import replicas
    return replicas.allsum(x) if world > 1 else x


def barrier(world):
    from fosite_b200 import replicas
    if world > 1:
        replicas.barrier()


def run_reference(args, world, rank):
    """The reference CPU path (the oracle, all host threads) on the headline grid when it fits in
    host memory; FirstStep untimed, then fosite steps for at most --ref-budget seconds."""
    if rank != 0:
        return
    full = args.size or HEADLINE_SIZE.get(args.workload, 256)
    size = oracle_size(args.workload, full)
    cb = time_oracle(args.workload, size, 0, args.ref_budget, max_steps=max(1, args.steps))
    cfg, _, _ = make_problem(args.workload, full)
    grid = [cfg.inum, cfg.jnum, cfg.knum]
    conf = {"workload": args.workload, "description": WORKLOADS[args.workload], "grid": grid}
    if cb["grid"] != grid:
        conf["timed_grid"] = cb["grid"]
        conf["comparable"] = False
        conf["note"] = "the oracle at the headline grid needs more host memory than this box has"
    line = {"metric": "cell-updates/s", "value": cb["value"], "unit": "cell-updates/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": conf, "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_own(args, world, rank, local):
    import ctypes as C
    import torch
    from fosite_b200 import abi
    from fosite_b200.sim import Simulation

    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    cfg, p, extra = make_problem(args.workload, args.size)
    sim = Simulation(cfg, device=local)
    sim.set_stream(stream.cuda_stream)
    apply_extra(sim, cfg, extra)
    sim.set_state(abi.PVAR, p)
    sim.first_step()
    # stage-kernel layout: measured on this GPU by the library's tuner unless forced
    forced = os.environ.get("FGPU_STAGE_VARIANT")
    variant = int(forced) if forced is not None else sim.autotune(3)
    # warm-up (also captures the device-clock graphs: at least one 16-step graph when the timed
    # run replays one, so that no capture falls inside the timed region)
    sim.run(max(args.warmup, min(args.steps, 16)))
    n_cells = cfg.inum * cfg.jnum * cfg.knum

    # ---- device-resident timed region (no per-launch instrumentation)
    barrier(world)
    torch.cuda.synchronize()
    clk = ClockSampler(local)
    clk.start()
    sim.reset_stats()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.run(args.steps)          # device clock: fixed-step graphs / embedded attempt slots
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clocks = clk.stop()
    ms = e0.elapsed_time(e1)
    st = sim.stats()
    ms_max = allmax(ms, world)
    upd_total = allsum(float(st.cell_updates), world)
    value = upd_total / (ms_max * 1e-3)

    # ---- the same number of steps again with every launch bracketed by CUDA events on the
    # library's stream (direct launches, every one of which does its work): the stage
    # kernels' mean duration and algorithmic bytes (roofline)
    sim.reset_stats()
    sim.set_profiling(True)
    for _ in range(args.steps):
        sim.step()
    torch.cuda.synchronize()
    stp = sim.stats()
    sim.set_profiling(False)

    # ---- end to end through the C ABI with host buffers (fosite keeps Timedisc%cvar on the host)
    L = sim.L
    nstate = sim.ncells * sim.vnum
    host = torch.empty(nstate, dtype=torch.float64, pin_memory=True)
    hv = host.numpy()
    hv[:] = sim.get(abi.CVAR).ravel()
    ptr = C.c_void_p(host.data_ptr())
    sim.reset_stats()
    barrier(world)
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(args.steps):
        L.fgpu_upload_state(sim.h, abi.CVAR, ptr, nstate)
        sim.step()
        L.fgpu_download(sim.h, abi.CVAR, ptr, nstate)
    f1.record(stream)
    torch.cuda.synchronize()
    ems_max = allmax(f0.elapsed_time(f1), world)
    st2 = sim.stats()
    e2e_value = allsum(float(st2.cell_updates), world) / (ems_max * 1e-3)

    if rank != 0:
        sim.close()
        if not args.no_extras:
            run_ensemble(args, world, rank, local, emit=False, steps=ENSEMBLE_EXTRA_STEPS)   # as rank 0
            run_serve(args, world, rank, local, emit=False, rates=SERVE_EXTRA["rate"],
                      requests=SERVE_EXTRA["requests"], t_scale=1.0)
        return
    peak, peak_kind = peak_hbm()
    achieved = stp.stage_bytes / (stp.stage_ms * 1e-3) / 1e9 if stp.stage_ms > 0 else None
    prof = load_traffic_profile(args.workload)
    traffic = None
    if prof and stp.stage_launches:
        traffic = prof.get("by_layout", {}).get(str(variant), prof["dram_bytes_per_cell"]) * n_cells
    cb = cpu_baseline(args.workload, budget_s=args.cpu_budget) if world == 1 and not args.no_cpu else None
    bpc = algorithmic_bytes_per_cell_update(args.workload, sim.vnum)
    # where the time of a step goes: kernel time (every launch bracketed by events, direct
    # launches) against the graph-replayed step of the timed region; the rest is the gaps
    # between dependent kernels (launch latency, block ramp-up and drain)
    kern_ms = (stp.stage_ms + stp.other_ms) / args.steps
    breakdown = {"graph_ms_per_step": ms_max / args.steps, "kernels_ms_per_step": kern_ms,
                 "stage_ms_per_step": stp.stage_ms / args.steps, "other_ms_per_step": stp.other_ms / args.steps,
                 "launches_per_step": stp.launches / args.steps,
                 "gap_ms_per_step": ms_max / args.steps - kern_ms}
    # grids whose stage working set (the stage's algorithmic bytes) fits in L2: the fraction of
    # a measured L2-resident copy as well
    l2 = None
    per_launch = stp.stage_bytes / max(1, stp.stage_launches)
    if achieved and per_launch < 96e6:
        from fosite_b200.sim import l2_read_gbs
        l2peak = l2_read_gbs(local)
        l2 = {"achieved": achieved, "peak": l2peak, "unit": "GB/s", "frac": achieved / l2peak,
              "peak_kind": "measured live: one launch reading a 16 MB L2-resident array 512 times "
                           "(fgpu_measure_l2_read)",
              "working_set_mb": per_launch / 1e6}
    line = {
        "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded inputs of the workload's shapes and value distributions)",
        "config": {"workload": args.workload, "description": WORKLOADS[args.workload],
                   "grid": [cfg.inum, cfg.jnum, cfg.knum], "parallelism": "replicas x%d" % world,
                   "l2": "inputs larger than L2: each state array is %.0f MB" % (n_cells * sim.vnum * 8 / 1e6),
                   "accepted_steps_per_rank": int(st.cell_updates // n_cells), "attempts": int(st.attempts),
                   "stage_variant": variant, "stage_kchunk": sim.stage_layout()[1] if cfg.knum > 1 else None,
                   "stage_variant_source": "forced" if forced is not None else "autotuned"},
        "achieved_gbps_step": value / world * bpc / 1e9,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                     "kernel": "RHS stage: stage_kernel (fused RHS + stage update; a Butcher stage's epilogue "
                               "forms the next stage's input state, the form_kernel pass only stage 2's)",
                     "form_ms_per_launch": stp.form_ms / max(1, stp.stage_launches),
                     "peak_kind": peak_kind + " copy bandwidth (burst)",
                     "algorithmic_bytes_per_launch": stp.stage_bytes / max(1, stp.stage_launches),
                     "launch_ms_avg": stp.stage_ms / max(1, stp.stage_launches),
                     "timing": "CUDA events around each stage launch on the library's stream, in a second "
                               "run of the same number of steps (single steps) after the timed region"},
        "step_breakdown": breakdown,
        "l2_roofline": l2,
        "cpu_baseline": cb,
        "e2e": {"value": e2e_value, "unit": "cell-updates/s", "h2d_bytes_per_step": nstate * 8,
                "d2h_bytes_per_step": nstate * 8},
        "gpu_launches": int(st.launches),
        "clocks": clocks,
    }
    sim.close()
    if not args.no_extras:
        # the batched ensemble against the loop of plain per-grid runs (96 disks), same steps
        ens = run_ensemble(args, world, rank, local, emit=False, steps=ENSEMBLE_EXTRA_STEPS)
        line["ensemble"] = {k: ens[k] for k in ("value", "unit", "ms_per_step", "speedup_vs_plain",
                                                  "speedup_vs_plain_tuned", "identical_to_plain", "identity_check",
                                                  "plain_loop", "plain_loop_tuned", "member_steps_per_s")}
        line["ensemble"]["layout"] = ens["config"]["variant"]
        line["ensemble"]["steps"] = ens["steps"]
        line["ensemble"]["config"] = {k: ens["config"][k] for k in ("description", "members", "cells")}
        # one serving rate at the full problem times (t_scale 1): p50 / p99 time to solution
        srv = run_serve(args, world, rank, local, emit=False, rates=SERVE_EXTRA["rate"],
                        requests=SERVE_EXTRA["requests"], t_scale=1.0)
        r = srv["rates"][0]
        line["serve"] = {"rate_req_s": r["rate_req_s"], "requests": r["requests"], "p50_s": r["p50_s"],
                         "p99_s": r["p99_s"], "makespan_s": r["makespan_s"],
                         "cell_updates_per_s": r["cell_updates_per_s"], "t_scale": 1.0,
                         "mix": srv["config"]["mix"]}
    print(json.dumps(line), flush=True)


# steps of the ensemble comparison in the default line: two 16-step graphs for the batch and for
# every plain member, so that both loops replay captured graphs
ENSEMBLE_EXTRA_STEPS = 32
# the serving point of the default line: Poisson arrivals at 20 requests/s, 24 requests of the
# full mix integrated to their full end times
SERVE_EXTRA = {"rate": "20", "requests": 24}

ENSEMBLE_DESC = ("96 independent 2D isothermal disks, Nr in [64,384], Nphi in [128,768] (multiples of 32), "
                 "cs/vK in [0.03,0.1], sigma index in [-1.5,-0.5], mixed cylindrical/logcylindrical, SSPRK3, "
                 "point mass, one launch per stage over every member's tiles, CUDA-graph captured, autotuned; "
                 "the plain loops step each member alone (default stage layout / each member's layout autotuned)")


def ensemble_members(n=96, seed=4000):
    from fosite_b200 import abi, problems
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        nr = 32 * int(rng.integers(2, 13))
        nphi = 32 * int(rng.integers(4, 25))
        geo = abi.LOGCYLINDRICAL if k % 2 == 0 else abi.CYLINDRICAL
        out.append(problems.disk2d(nr=nr, nphi=nphi, seed=seed + k, hratio=float(rng.uniform(0.03, 0.1)),
                                   sigma_index=float(rng.uniform(-1.5, -0.5)), geometry=geo, fargo=0))
    return out


def run_ensemble(args, world=1, rank=0, local=0, emit=True, steps=None):
    """Batched ensemble against a loop of plain per-grid runs of the same members.

    With N ranks the members are dealt round-robin to the GPUs (no collective in the
    step); the job time is the slowest rank's.  emit=False returns rank 0's line instead
    of printing it (None on the other ranks); steps overrides --steps."""
    import copy
    if steps is not None:
        args = copy.copy(args)
        args.steps = steps
    import torch
    from fosite_b200 import abi, replicas
    from fosite_b200.sim import Batch, Simulation
    torch.cuda.set_device(local)
    all_probs = ensemble_members(args.members)
    probs = replicas.partition(all_probs, rank, world)

    def make():
        sims = []
        for cfg, p, extra in probs:
            s = Simulation(cfg, device=local)
            apply_extra(s, cfg, extra)
            s.set_state(abi.PVAR, p)
            s.first_step()
            sims.append(s)
        return sims
    forced = os.environ.get("FGPU_STAGE_VARIANT")
    members, plain, tuned = make(), make(), make()
    cells = sum(c.inum * c.jnum for c, _, _ in probs)
    b = Batch(members)
    variant = b.autotune(3)
    # warm-up of at least one 16-step graph, so that graph capture stays outside the timed loops
    wsteps = max(args.warmup, 16)
    b.run(wsteps)
    # the plain per-grid loop as the API gives it (default stage layout), and with every member's
    # stage layout autotuned
    tuned_layouts = {}
    for s in plain:
        s.run(wsteps)
    for s in tuned:
        v = s.autotune(3)
        tuned_layouts[v] = tuned_layouts.get(v, 0) + 1
        s.run(wsteps)
    clk = ClockSampler(local)
    clk.start()
    barrier(world)
    t0 = time.perf_counter()
    b.run(args.steps)                      # returns after the device finished (status read back)
    t_batch = time.perf_counter() - t0
    clocks = clk.stop()

    def loop(sims):
        barrier(world)
        t = time.perf_counter()
        for s in sims:
            s.run(args.steps)
        return allmax(time.perf_counter() - t, world)
    t_plain = loop(plain)
    t_tuned = loop(tuned)
    # identity: every member against its lone run on the batch's stage layout (the product
    # build's layouts may differ from one another in the last bit; each equals the oracle bit for
    # bit on the --fmad=false build)
    for s in plain + tuned:
        s.close()
    os.environ["FGPU_STAGE_VARIANT"] = str(b.layout())
    try:
        check = make()
    finally:
        if forced is None:
            os.environ.pop("FGPU_STAGE_VARIANT", None)
        else:
            os.environ["FGPU_STAGE_VARIANT"] = forced
    for s in check:
        s.run(wsteps + args.steps)
    same = all(np.array_equal(m.get(abi.CVAR), s.get(abi.CVAR)) for m, s in zip(members, check))
    for s in check:
        s.close()
    value, cells_all, ms_batch = replicas.job_throughput(cells * args.steps, 1e3 * t_batch) if world > 1 else \
        (cells * args.steps / t_batch, cells * args.steps, 1e3 * t_batch)
    t_batch = ms_batch * 1e-3
    same = allsum(0.0 if same else 1.0, world) == 0.0
    members_all = len(all_probs)
    cells = int(allsum(cells, world))
    if rank != 0:
        b.close()
        return None
    line = {"metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_batch / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)",
            "config": {"workload": "ensemble", "description": ENSEMBLE_DESC, "members": members_all,
                       "cells": cells, "tiles_rank0": b.tiles, "variant": variant,
                       "parallelism": "members dealt round-robin over %d GPU(s)" % world},
            "member_steps_per_s": members_all * args.steps / t_batch,
            "plain_loop": {"value": cells * args.steps / t_plain, "ms_per_step": 1e3 * t_plain / args.steps,
                           "layouts": "the library's default (shared-memory tile 0)"},
            "plain_loop_tuned": {"value": cells * args.steps / t_tuned, "ms_per_step": 1e3 * t_tuned / args.steps,
                                 "layouts_rank0": {str(k): v for k, v in sorted(tuned_layouts.items())}},
            "speedup_vs_plain": t_plain / t_batch, "speedup_vs_plain_tuned": t_tuned / t_batch,
            "identical_to_plain": bool(same),
            "identity_check": "every member's state against its lone run on the batch's stage layout",
            "clocks": clocks}
    b.close()
    if emit:
        print(json.dumps(line), flush=True)
    return line


def run_serve(args, world=1, rank=0, local=0, emit=True, rates=None, requests=None, t_scale=None):
    """Poisson request streams at swept rates through the continuous-batching server.

    With N ranks each GPU serves the requests dealt to it round-robin (the stream's
    arrival times are kept); latencies are gathered on rank 0.  rates / requests / t_scale
    override the command line; emit=False returns rank 0's line instead of printing it."""
    rates = args.rates if rates is None else rates
    requests = args.requests if requests is None else requests
    t_scale = args.t_scale if t_scale is None else t_scale
    from fosite_b200 import replicas
    from fosite_b200.serve import Server, poisson_stream
    import torch
    torch.cuda.set_device(local)
    free, total = torch.cuda.mem_get_info()
    out = []
    for rate in [float(r) for r in str(rates).split(",")]:
        reqs = replicas.partition(poisson_stream(rate, requests, seed=int(rate), t_scale=t_scale), rank, world)
        from fosite_b200.serve import build_problem
        for r in reqs:               # requests arrive with their initial data
            r.payload = build_problem(r)
        srv = Server(hbm_budget_bytes=int(0.8 * free), device=local, chunk=args.chunk, autotune=False)
        barrier(world)
        rep = srv.serve(reqs, timeout_s=900)
        if world > 1:
            import torch.distributed as dist
            lat = [r.finished - r.arrival for r in srv.done]
            parts = [None] * world
            dist.all_gather_object(parts, (lat, rep["cell_updates"], rep["makespan_s"]))
            lat = np.array([x for p in parts for x in p[0]])
            span = max(p[2] for p in parts)
            cu = sum(p[1] for p in parts)
            rep = {"requests": int(lat.size), "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
                   "mean_s": float(lat.mean()), "makespan_s": span, "cell_updates": int(cu),
                   "cell_updates_per_s": cu / span if span > 0 else None}
        rep["rate_req_s"] = rate
        out.append(rep)
    if rank != 0:
        return
    line = {"metric": "p50/p99 time-to-solution, cell-updates/s", "unit": "s", "n_gpus": world,
            "higher_is_better": False, "dtype": "f64", "data": "synthetic (seeded Poisson streams)",
            "config": {"workload": "serve", "requests_per_rate": requests, "t_scale": t_scale,
                       "chunk_steps": args.chunk, "payload": "initial data generated before the stream starts "
                                                             "(requests carry their data)",
                       "mix": "2D KHI 64^2-1024^2, 2D disks 64x128-512x1024, 3D pulses 32^3-128^3"},
            "rates": out}
    if emit:
        print(json.dumps(line), flush=True)
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="fosite_b200", choices=["fosite_b200", "reference"])
    ap.add_argument("--workload", default="gauss3d", choices=sorted(WORKLOADS) + ["ensemble", "serve"])
    ap.add_argument("--members", type=int, default=96)
    ap.add_argument("--rates", default="10,50,200,500")
    ap.add_argument("--requests", type=int, default=200)
    ap.add_argument("--t-scale", type=float, default=0.01)
    ap.add_argument("--chunk", type=int, default=8)
    ap.add_argument("--size", type=int, default=0)
    ap.add_argument("--ref-budget", type=float, default=120.0)
    ap.add_argument("--cpu-budget", type=float, default=25.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the ensemble comparison and the serving point of the default line")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    try:
        if args.workload in ("ensemble", "serve"):
            fn = run_ensemble if args.workload == "ensemble" else run_serve
            fn(args, world, rank, local)
        elif args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_own(args, world, rank, local)
    finally:
        if world > 1:
            from fosite_b200 import replicas
            replicas.finalize()


if __name__ == "__main__":
    main()
