"""Specimens sharded across ranks (rfdem.shard): the balancing rule, and on two gloo
ranks the one end-of-run reduction that assembles every specimen's scalars, with a
stand-in runner in place of the GPU engine."""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "rockfit-dem_b200"))


def test_assign_balances_whole_specimens():
    from rfdem.shard import assign
    rng = np.random.default_rng(7)
    costs = np.exp(rng.uniform(np.log(5000), np.log(80000), 64)).astype(int)
    for world in (1, 2, 3, 8):
        parts = assign(costs, world)
        assert len(parts) == world
        flat = sorted(q for p in parts for q in p)
        assert flat == list(range(64))                       # every specimen exactly once
        loads = [sum(costs[q] for q in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)         # greedy longest-first bound
        assert parts == assign(costs, world)                 # deterministic
    assert assign([3, 1, 2], 5)[3:] == [[], []]              # more ranks than specimens


class _Spec:
    def __init__(self, n):
        self.N = n


def _fake_runner(tasks, params, Rs, radii):
    # a specimen's "result" is a function of its own data only
    return [[float(p), float(t.N), 0.5 * p, 0.0, 0.0, 1.0, float(p) * 2] for t, p in zip(tasks, params)]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, os.path.join(ROOT, "rockfit-dem_b200"))
    from rfdem.shard import run_sharded
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    sizes = [1000 + 137 * q for q in range(11)]
    tasks = [_Spec(n) for n in sizes]
    params = list(range(100, 111))
    table = run_sharded(tasks, params, [None] * 11, [None] * 11, steps=10, dist=dist, runner=_fake_runner)
    out[rank] = table.tolist()
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_gather_every_specimen():
    from rfdem.shard import run_sharded
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    sizes = [1000 + 137 * q for q in range(11)]
    want = np.array(_fake_runner([_Spec(n) for n in sizes], list(range(100, 111)), None, None))
    for r in range(world):
        assert np.array_equal(np.array(res[r]), want)
    # the same table without a process group
    alone = run_sharded([_Spec(n) for n in sizes], list(range(100, 111)), [None] * 11, [None] * 11, steps=10,
                        runner=_fake_runner)
    assert np.array_equal(alone, want)
