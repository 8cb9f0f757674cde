"""Multi-process path of bench.py on CPU: replicas over gloo (world size 2).

bench.py shards designs by rank (independent seeds, no data-path collective) and takes the
max-over-ranks time with one all_reduce(MAX). This runs that host logic with the CPU oracle as the
per-rank work, on two gloo ranks."""
import os

import numpy as np
import pytest
import torch.multiprocessing as mp


def _rank(rank, world, port, out):
    import sys
    import time

    import torch
    import torch.distributed as dist

    sys.path.insert(0, os.path.join(os.path.dirname(__file__), ".."))
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    import pgj_oracle as O
    from __graft_entry__ import load_package

    pkg = load_package()
    seeds = bench.design_seeds(rank, 2)
    t0 = time.perf_counter()
    Cs = []
    for s in seeds:
        a = pkg.baseline_design(4, s, 1e-4)
        Cs.append(O.homogenize(a, *O.PAPER, 0.5)["C"])
    local_ms = (time.perf_counter() - t0) * 1e3 + 100.0 * rank
    t = torch.tensor([local_ms], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    out[rank] = dict(seeds=seeds, max_ms=float(t[0]), local_ms=local_ms, C0=Cs[0].tolist())
    dist.barrier()
    dist.destroy_process_group()


def test_replicas_shard_designs_and_take_max_time():
    world = 2
    port = 29500 + os.getpid() % 1000
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert set(res[0]["seeds"]).isdisjoint(res[1]["seeds"])
    assert res[0]["max_ms"] == res[1]["max_ms"] == pytest.approx(max(r["local_ms"] for r in res.values()))
    assert not np.allclose(res[0]["C0"], res[1]["C0"])
