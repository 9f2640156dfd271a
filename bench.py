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
    "gauss3d": "3D Euler Gaussian pulse 256^3, reflecting, KT+MC(prim), Dormand-Prince 5(4) tol 1e-5, CFL 0.4",
    "khi2d": "2D Kelvin-Helmholtz 256^2, periodic, KT+van Leer(cons), SSPRK3 fixed CFL 0.4",
}


def make_problem(name, size):
    from fosite_b200 import problems
    if name == "gauss3d":
        return problems.gauss3d(n=size or 256)
    return problems.khi2d(n=size or 256)


def algorithmic_bytes_per_cell_update(name, vnum):
    """Compulsory HBM traffic per interior cell and accepted step (fused design).

    Dormand-Prince with CHECK_ALL: end-of-step RHS reads the state and writes
    k1 and the round-tripped base (1+2), stages m=2..7 read base+k1..k_{m-1}
    and write k_m (27+6), the last stage also writes the new state (1):
    37 arrays.  SSPRK3 (modified Euler): 3 stages read the stage input and the
    start state, write the stage output: 8 arrays.
    """
    arrays = 37 if name == "gauss3d" else 8
    return arrays * vnum * 8.0


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


def cpu_baseline(name, budget_s=20.0):
    """The oracle (serial C++ restatement of the reference CPU path) on a bounded sample."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from fosite_b200 import abi
    size = 48 if name == "gauss3d" else 256
    cfg, p, _ = make_problem(name, size)
    o = pyoracle.Oracle(cfg)
    o.set_state(abi.PVAR, p)
    o.first_step()
    t0 = time.perf_counter()
    it0 = o.status().iter
    steps = 0
    while True:
        o.step()
        steps += 1
        if time.perf_counter() - t0 > budget_s or steps >= 200:
            break
    el = time.perf_counter() - t0
    upd = (o.status().iter - it0) * cfg.inum * cfg.jnum * cfg.knum
    return {"value": upd / el, "unit": "cell-updates/s", "cores": 1, "kind": "port",
            "sample": "%d fosite steps of the same problem on a %dx%dx%d grid (%.1f s, serial oracle)"
                      % (steps, cfg.inum, cfg.jnum, cfg.knum, el)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def allmax(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def allsum(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def run_reference(args, world, rank):
    if rank != 0:
        return
    cb = cpu_baseline(args.workload, budget_s=args.ref_budget)
    line = {"metric": "cell-updates/s", "value": cb["value"], "unit": "cell-updates/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": args.workload, "description": WORKLOADS[args.workload]},
            "cpu_baseline": cb, "e2e": {"value": cb["value"], "unit": "cell-updates/s",
                                        "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
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
    sim.set_state(abi.PVAR, p)
    sim.first_step()
    for _ in range(args.warmup):
        sim.step()
    n_cells = cfg.inum * cfg.jnum * cfg.knum

    # ---- device-resident timed region
    barrier(world)
    torch.cuda.synchronize()
    clk = ClockSampler(local)
    clk.start()
    sim.reset_stats()
    sim.set_profiling(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        sim.step()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clocks = clk.stop()
    ms = e0.elapsed_time(e1)
    st = sim.stats()
    sim.set_profiling(False)
    ms_max = allmax(ms, world)
    upd_total = allsum(float(st.cell_updates), world)
    value = upd_total / (ms_max * 1e-3)

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
        return
    peak, peak_kind = peak_hbm()
    achieved = st.stage_bytes / (st.stage_ms * 1e-3) / 1e9 if st.stage_ms > 0 else None
    prof = load_traffic_profile(args.workload)
    traffic = None
    if prof and st.stage_launches:
        traffic = prof["dram_bytes_per_cell"] * n_cells
    cb = cpu_baseline(args.workload, budget_s=args.ref_budget) if world == 1 and not args.no_cpu else None
    bpc = algorithmic_bytes_per_cell_update(args.workload, sim.vnum)
    line = {
        "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded, BASELINE config shapes)",
        "config": {"workload": args.workload, "description": WORKLOADS[args.workload],
                   "grid": [cfg.inum, cfg.jnum, cfg.knum], "parallelism": "replicas x%d" % world,
                   "l2": "inputs larger than L2: each state array is %.0f MB" % (n_cells * sim.vnum * 8 / 1e6),
                   "accepted_steps_per_rank": int(st.cell_updates // n_cells), "attempts": int(st.attempts)},
        "achieved_gbps_step": value / world * bpc / 1e9,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                     "kernel": "stage_kernel (fused RHS + stage update)", "peak_kind": peak_kind + " copy bandwidth"},
        "cpu_baseline": cb,
        "e2e": {"value": e2e_value, "unit": "cell-updates/s", "h2d_bytes_per_step": nstate * 8,
                "d2h_bytes_per_step": nstate * 8},
        "gpu_launches": int(st.launches),
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    sim.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="fosite_b200", choices=["fosite_b200", "reference"])
    ap.add_argument("--workload", default="gauss3d", choices=sorted(WORKLOADS))
    ap.add_argument("--size", type=int, default=0)
    ap.add_argument("--ref-budget", type=float, default=20.0)
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_own(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
