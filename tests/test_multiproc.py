"""Multi-rank host logic on CPU: two gloo ranks shard ensembles and all-reduce
their FP64 moments; the result equals the single-process sum. The sharded run is
the one bench.py makes with --gpus N (D.shard of one global batch, then
D.allreduce_moments), here with the CPU oracle standing in for each rank's GPU."""
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


def _oracle_worker(rank, world, port, q):
    import torch.distributed as dist
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        groups = _oracle_batch()
        mine = D.shard(groups, rank, world)
        local = np.stack([_oracle_samples(O, groups[i]) for i in mine], axis=1)
        q.put((rank, mine, D.allreduce_moments(local, mine, len(groups))))
    finally:
        dist.destroy_process_group()


def _oracle_batch():
    return uneven_batch(n_traj=5, seed=7, grids=((8, 8, 64), (16, 16, 32)))


def _oracle_samples(O, p):
    """pi/2, then 6 steps with moments after steps 3 and 6 (Thomas-Fermi start, noise and losses on)."""
    d = O.derive(p)
    x = -d.xmax + d.dx * np.arange(d.nvx)
    y = -d.ymax + d.dy * np.arange(d.nvy)
    z = -d.zmax + d.dz * np.arange(d.nvz)
    V = (x[None, None, :] ** 2 + y[None, :, None] ** 2 + z[:, None, None] ** 2 / d.lambda_ ** 2) / 2
    gs = np.sqrt(np.maximum(d.mu - V, 0.0) / d.g11).reshape(-1).astype(np.complex128)
    e = O.OracleEnsemble(p)
    e.init(gs)
    e.start_evolution(1)
    out = []
    for _ in range(2):
        e.evolve(3, 1)
        out.append(e.moments())
    return np.array(out)


def test_two_ranks_shard_an_oracle_ensemble_like_the_bench():
    import multiprocessing as mp
    from oracle import oracle as O
    groups = _oracle_batch()
    single = np.stack([_oracle_samples(O, p) for p in groups], axis=1)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_oracle_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    owned = sorted(i for _, mine, _ in res for i in mine)
    assert owned == list(range(len(groups)))
    assert all(len(mine) > 0 for _, mine, _ in res)
    for _, _, red in res:
        np.testing.assert_array_equal(red[:, :, 1:], single[:, :, 1:])
        np.testing.assert_allclose(red[:, :, 0], single[:, :, 0])
