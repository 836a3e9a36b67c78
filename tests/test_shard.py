"""Multi-rank host logic on CPU (gloo, world size 2): scene sharding covers every
scene once and balances the load; one fixed batch, LPT-sharded over two ranks
that each evaluate their scenes, gathers per-scene losses and gradients that
are bitwise those of one process running the whole batch, and so is the
fixed-order reduction of a parameter shared by all scenes; the timing
reduction returns the max and the particle count the sum over ranks.

The oracle stands in for the device path here (no GPU on the CPU runner): the
scenes are independent units, so what is checked is the sharding, gathering
and reduction logic around them."""
import os

import numpy as np
import pytest

from morphompm_b200.shard import lpt_assign

STEPS = 2


def _small_batch():
    from morphompm_b200 import scenes
    return scenes.config4(n_scenes=10, n_lo=64, n_hi=512)


def _scene_result(s):
    """Loss (sum det F) and d loss / d g of one scene, oracle FP64."""
    from oracle import mpm_oracle as O
    sp = s["dx"] / 2
    sc = O.Scene(shape=s["shape"], dx=s["dx"], dt=s["dt"], damping=s["damping"], pmass=s["density"] * sp ** 3,
                 vol0=sp ** 3, wall=s["wall"])
    gr = O.Growth(A=s["growth_A"])
    st, caches = O.rollout(O.State.rest(s["x"]), O.Model.elastic(s["model"], s["E"], s["nu"]), sc, STEPS,
                           advect=True, growth=gr)
    n = s["x"].shape[0]
    z3, z33 = np.zeros((n, 3)), np.zeros((n, 3, 3))
    dA = O.rollout_vjp(caches, z3, z3, z33, O.seed_detF(st.F), z33, advect=True, growth=gr)[5]
    return [O.loss_detF(st.F), dA]


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
    from morphompm_b200.shard import lpt_assign, max_over_ranks, sum_over_ranks, gather_scenes, fixed_order_sum
    scn = _small_batch()                       # the same fixed batch on every rank
    costs = [s["x"].shape[0] * STEPS for s in scn]
    mine = lpt_assign(costs, world)[rank]
    local = [_scene_result(scn[i]) for i in mine]
    full = gather_scenes(local, mine, len(scn))
    shared = fixed_order_sum(full[:, 1])
    n_mine = sum(scn[i]["x"].shape[0] for i in mine)
    t = max_over_ranks(10.0 + rank)
    tot = sum_over_ranks(n_mine)
    q.put((rank, mine, full, shared, t, n_mine, tot))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gloo_sharded_batch():
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
    res = sorted((q.get(timeout=300) for _ in procs), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    scn = _small_batch()
    assert sorted(res[0][1] + res[1][1]) == list(range(len(scn)))     # every scene once
    assert res[0][1] and res[1][1]
    single = np.array([_scene_result(s) for s in scn])               # one process, the whole batch
    from morphompm_b200.shard import fixed_order_sum
    for r in res:
        assert np.array_equal(r[2], single)                          # gathered, in scene order, bitwise
        assert r[3] == fixed_order_sum(single[:, 1])                 # shared-parameter reduction, bitwise
    assert res[0][4] == res[1][4] == 11.0                            # max over ranks
    assert res[0][6] == res[1][6] == sum(s["x"].shape[0] for s in scn)   # particles of all ranks

