"""Multi-rank host logic on CPU (gloo, world size 2): scene sharding covers every
scene once and balances the load; the timing reduction returns the max and
the particle count the sum over ranks."""
import os

import pytest

from morphompm_b200.shard import lpt_assign


def test_lpt_assign_covers_and_balances():
    from morphompm_b200 import scenes
    scn = scenes.config4(n_scenes=64)
    costs = [s["x"].shape[0] * 200 for s in scn]
    for world in (1, 2, 3, 8):
        parts = lpt_assign(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(scn)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from morphompm_b200.shard import lpt_assign, max_over_ranks, sum_over_ranks
    from morphompm_b200 import scenes
    scn = scenes.config4(n_scenes=16, seed=4 + 1000 * rank)     # each rank: its own batch (weak scaling)
    n = sum(s["x"].shape[0] for s in scn)
    mine = lpt_assign([1.0, 5.0, 3.0, 2.0, 4.0], world)[rank]
    t = max_over_ranks(10.0 + rank)
    tot = sum_over_ranks(n)
    q.put((rank, n, mine, t, tot))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gloo():
    import multiprocessing as mp
    import socket
    ctx = mp.get_context("spawn")
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][1] != res[1][1]                       # different batches per rank
    assert sorted(res[0][2] + res[1][2]) == [0, 1, 2, 3, 4]
    assert res[0][3] == res[1][3] == 11.0               # max over ranks
    assert res[0][4] == res[1][4] == res[0][1] + res[1][1]   # particles of all ranks
