"""The multi-rank bench path on CPU: two gloo ranks, each with its own seeded specimen
(weak scaling by specimens), and the max / sum reductions bench.py uses for the
elapsed time and the particle count."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "rockfit-dem_b200"))
    import bench
    import rfdem
    r, ws, dist = bench.dist_init()
    assert (r, ws) == (rank, world) and dist.get_backend() == "gloo"
    # each rank builds its own specimen from its own seed (a small lattice disc here)
    t, R = rfdem.make_test(rfdem.RF_TEST_BRAZIL, 8.0 + 2.0 * rank, 3.0, seed=bench.rank_seed(rank))
    n = float(t.N)
    elapsed = 1.0 + rank                       # a stand-in for each rank's timed region
    tot = bench.sum_over_ranks(n, dist)
    mx = bench.max_over_ranks(elapsed, dist)
    out[rank] = (n, tot, mx, bench.rank_seed(rank))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_weak_scaling():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    n0, n1 = res[0][0], res[1][0]
    assert n0 != n1                                  # different specimens per rank
    for r in range(world):
        assert res[r][1] == n0 + n1                  # sum of particles over ranks
        assert res[r][2] == 2.0                      # max of the elapsed times
    assert res[0][3] != res[1][3]
