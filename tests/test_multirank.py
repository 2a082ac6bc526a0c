"""Multi-rank host logic of bench.py on CPU (gloo, world size 2, 127.0.0.1):
the LPT split of the many-systems workload across ranks, and the max-over-
ranks timing reduction.  No GPU is touched."""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_lpt_partition_balances_and_covers():
    rng = np.random.default_rng(0)
    costs = list(np.exp(rng.uniform(np.log(1e3), np.log(1e5), 512)))
    for parts in (1, 2, 4, 8):
        owner = bench.lpt_partition(costs, parts)
        assert sorted(set(owner)) == list(range(parts))
        loads = np.zeros(parts)
        for c, o in zip(costs, owner):
            loads[o] += c
        assert loads.max() <= loads.mean() + max(costs)   # LPT bound
        assert loads.max() / loads.mean() < 1.02


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    cells, pos, qs = bench.batch_systems(64, seed=11)
    owner = bench.lpt_partition([len(q) for q in qs], world)
    mine = [i for i in range(len(qs)) if owner[i] == rank]
    # gather every rank's systems and its (fake) step time; reduce the max
    got = [None] * world
    dist.all_gather_object(got, mine)
    t = torch.tensor([0.1 * (rank + 1)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    out[rank] = (sorted(i for g in got for i in g), float(t.item()),
                 sum(len(qs[i]) for i in mine), sum(len(q) for q in qs))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_split_systems_and_reduce_max():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    all_ids, tmax, _, total = res[0]
    assert all_ids == list(range(64))          # every system on exactly one rank
    assert tmax == 0.2 and res[1][1] == 0.2    # max over ranks on every rank
    assert res[0][2] + res[1][2] == total
    assert abs(res[0][2] - res[1][2]) / total < 0.05
