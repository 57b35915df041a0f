"""Multi-rank host logic on CPU: two gloo ranks shard ensembles and all-reduce
their FP64 moments; the result equals the single-process sum."""
import os
import socket

import numpy as np
import pytest

from bec_b200 import distributed as D
from bec_b200.configs import uneven_batch


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_shard_covers_every_group_once_and_balances():
    groups = uneven_batch(n_traj=97, seed=3)
    for world in (1, 2, 3, 8):
        owned = [D.shard(groups, r, world) for r in range(world)]
        flat = sorted(i for o in owned for i in o)
        assert flat == list(range(len(groups)))
        loads = [sum(D.cost(groups[i]) for i in o) for o in owned]
        assert max(loads) - min(loads) <= max(D.cost(g) for g in groups)


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        groups = uneven_batch(n_traj=10, seed=5)
        mine = D.shard(groups, rank, world)
        rng = np.random.default_rng(0)
        allm = rng.standard_normal((3, len(groups), 5))
        allm[:, :, 0] = np.arange(3)[:, None] * 0.01
        red = D.allreduce_moments(allm[:, mine, :], mine, len(groups))
        mx = D.max_over_ranks(float(rank + 1))
        q.put((rank, red, mx, allm))
    finally:
        dist.destroy_process_group()


def test_two_rank_allreduce_matches_single_process():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, red, mx, allm in res:
        np.testing.assert_allclose(red[:, :, 1:], allm[:, :, 1:], rtol=0, atol=0)
        np.testing.assert_allclose(red[:, :, 0], allm[:, :, 0])
        assert mx == 2.0
