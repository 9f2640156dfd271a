"""Host plumbing of multi-GPU runs: one process per GPU, no data-path collective.

fosite's step is not sharded across GPUs here.  A multi-GPU run either advances
N independent replicas of a grid (single-grid workloads), or partitions the
members of an ensemble / the requests of a serving stream across the ranks.
The only collectives are scalar reductions of the timing and of the work done,
taken after the timed region: the job's time is the maximum over ranks and its
throughput the sum of all ranks' cell updates divided by that time.

The process group uses NCCL when the ranks own GPUs and gloo otherwise (the
CPU tests run two gloo ranks).
"""
import datetime
import os


def env():
    """(world, rank, local_rank) from the torch.distributed launcher's environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend=None, timeout_s=300):
    """Join the process group when WORLD_SIZE > 1; returns (world, rank, local_rank)."""
    world, rank, local = env()
    if world > 1:
        import torch
        import torch.distributed as dist
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        if not dist.is_initialized():
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return world, rank, local


def _device():
    import torch
    import torch.distributed as dist
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def _reduce(x, op):
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=op)
    return float(t.item())


def allmax(x):
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.MAX)


def allsum(x):
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.SUM)


def barrier():
    import torch.distributed as dist
    if dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def partition(items, rank, world):
    """Round-robin share of a list (ensemble members, serving requests) for one rank."""
    return [x for k, x in enumerate(items) if k % world == rank]


def job_throughput(local_units, local_ms):
    """Whole-job rate: units summed over ranks / the slowest rank's time (units per s)."""
    units = allsum(local_units)
    ms = allmax(local_ms)
    return units / (ms * 1e-3) if ms > 0 else 0.0, units, ms


def finalize():
    import torch.distributed as dist
    if dist.is_initialized():
        dist.destroy_process_group()
