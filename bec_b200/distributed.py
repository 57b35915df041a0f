"""Multi-GPU plumbing: trajectories shard across ranks with no data-path exchange.

Every trajectory is independent (the reference keeps ensembles in one buffer
on one GPU, programs/bec_wigner_3d.cuda/defines.h:160-168), so ranks only
exchange the per-sample FP64 moments of each ensemble once, a few KB, after
the run. One process per GPU; torch.distributed carries the all-reduce (NCCL
on GPUs, gloo on CPU).
"""
import numpy as np


def cost(p):
    """Work estimate of an ensemble: cells x trajectories."""
    return p.nvx * p.nvy * p.nvz * p.ne


def shard(groups, rank, world):
    """Longest-processing-time assignment of ensembles to ranks (balanced by cells).

    Returns the indices of `groups` owned by `rank`, in ascending order; every
    index is owned by exactly one rank, and the assignment depends only on the
    inputs (all ranks compute the same map)."""
    order = sorted(range(len(groups)), key=lambda i: (-cost(groups[i]), i))
    load = [0] * world
    owner = [0] * len(groups)
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += cost(groups[i])
    return [i for i in range(len(groups)) if owner[i] == rank]


def allreduce_moments(local_moments, local_index, n_groups, device=None):
    """Sums per-ensemble moments across ranks.

    local_moments: [n_samples, n_local, 5] (t, na, nb, s_re, s_im) of the ensembles in
    local_index. Returns [n_samples, n_groups, 5] on every rank; t is taken as the max."""
    import torch
    import torch.distributed as dist
    m = np.asarray(local_moments, dtype=np.float64)
    ns = m.shape[0]
    full = np.zeros((ns, n_groups, 5))
    full[:, local_index, :] = m
    t = torch.tensor(full[:, :, 1:], dtype=torch.float64, device=device)
    tt = torch.tensor(full[:, :, 0], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    out = np.zeros((ns, n_groups, 5))
    out[:, :, 1:] = t.cpu().numpy()
    out[:, :, 0] = tt.cpu().numpy()
    return out


def max_over_ranks(x, device=None):
    """Maximum of a scalar over ranks (device-timed step time)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
