"""Multi-process host path (fosite_b200.replicas) with two gloo ranks on the CPU.

The GPU runs use one process per GPU over NCCL; the plumbing they share with
this test is the rank/world handling, the round-robin partition of ensemble
members and serving requests, and the max-over-ranks timing reduction.
"""
import json
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    from fosite_b200 import replicas
    w, r, local = replicas.init(backend="gloo", timeout_s=60)
    res = {"world": w, "rank": r, "local": local}
    res["max"] = replicas.allmax(rank + 1.5)
    res["sum"] = replicas.allsum(rank + 1.0)
    res["part"] = replicas.partition(list(range(7)), r, w)
    rate, units, ms = replicas.job_throughput(100.0 * (rank + 1), 10.0 * (rank + 1))
    res["rate"], res["units"], res["ms"] = rate, units, ms
    replicas.barrier()
    replicas.finalize()
    with open(os.path.join(out_dir, "rank%d.json" % rank), "w") as f:
        json.dump(res, f)


def test_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = [json.load(open(tmp_path / ("rank%d.json" % r))) for r in range(2)]
    for r, x in enumerate(res):
        assert x["world"] == 2 and x["rank"] == r and x["local"] == r
        assert x["max"] == 2.5 and x["sum"] == 3.0
        assert x["units"] == 300.0 and x["ms"] == 20.0
        assert x["rate"] == pytest.approx(300.0 / 0.020)
    assert res[0]["part"] == [0, 2, 4, 6] and res[1]["part"] == [1, 3, 5]


def test_single_process_defaults(monkeypatch):
    from fosite_b200 import replicas
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    assert replicas.init() == (1, 0, 0)
    assert replicas.allmax(3.0) == 3.0 and replicas.allsum(2.0) == 2.0
    assert replicas.partition([1, 2, 3], 0, 1) == [1, 2, 3]
