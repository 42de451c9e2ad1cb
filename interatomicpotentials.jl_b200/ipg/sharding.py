"""Multi-GPU evaluation of many configurations: one process per GPU, configurations sharded
across ranks, no data-path collective except the all-reduce (sum) of the force-matching loss
and its beta gradient (K * nspecies doubles + 1).

Configurations are independent units of work, so each rank evaluates its own shard with the
batched library calls (``SNAP.batch_loss_grad`` / ``SNAP.batch_energy_forces``) on its own GPU.
Shards are balanced by the estimated cost of a configuration, atoms x neighbors per atom
(the SNAP work is per atom plus per neighbor), with a deterministic longest-first greedy
assignment so that every rank computes the same partition without communication.
"""
from __future__ import annotations

import numpy as np


def config_costs(systems, rcut):
    """Estimated work per configuration: N_c * (1 + expected neighbors within rcut)."""
    out = []
    for s in systems:
        n = len(s)
        L = s.L
        vol = float(np.prod(np.where(np.isfinite(L), L, np.ptp(s.positions, axis=0) + 2 * rcut)))
        nbr = (n / max(vol, 1e-30)) * 4.0 / 3.0 * np.pi * rcut ** 3
        out.append(n * (1.0 + min(nbr, n - 1)))
    return np.asarray(out, dtype=np.float64)


def shard(costs, world):
    """Longest-first greedy partition of configuration indices into `world` shards.
    Ties break by index, so the result depends only on (costs, world)."""
    costs = np.asarray(costs, dtype=np.float64)
    order = sorted(range(len(costs)), key=lambda c: (-costs[c], c))
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for c in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(c)
        load[r] += costs[c]
    return [sorted(p) for p in parts]


def _all_reduce_sum(vec, group=None):
    """Sum of a float64 vector over the process group (NCCL tensors live on the rank's GPU)."""
    import torch
    import torch.distributed as dist
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor(np.asarray(vec, dtype=np.float64), device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


def loss_grad(evaluate, systems, beta, F_ref, rcut, group=None):
    """Force-matching loss and dL/dbeta over all configurations, sharded across the ranks of
    `group` (torch.distributed must be initialised).

    evaluate(shard_systems, beta, shard_F_ref) -> (loss, gbeta) runs one rank's shard, e.g.
    ``snap.batch_loss_grad``; F_ref is the flattened (n_total, 3) reference of all configurations.
    Every rank returns the same (loss, gbeta)."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    parts = shard(config_costs(systems, rcut), world)
    off = np.concatenate([[0], np.cumsum([len(s) for s in systems])])
    F_ref = np.asarray(F_ref, dtype=np.float64).reshape(-1, 3)
    mine = parts[rank]
    gshape = np.shape(beta)
    if mine:
        sub = [systems[c] for c in mine]
        Fr = np.concatenate([F_ref[off[c]:off[c + 1]] for c in mine])
        loss, g = evaluate(sub, beta, Fr)
        g = np.asarray(g, dtype=np.float64)
        gshape = g.shape
    else:  # an empty shard still joins the collective
        loss, g = 0.0, np.zeros(gshape)
    flat = np.concatenate([[float(loss)], np.asarray(g, dtype=np.float64).ravel()])
    tot = _all_reduce_sum(flat, group)
    return tot[0], tot[1:].reshape(gshape)


def energy_forces(evaluate, systems, beta, beta0, rcut, group=None):
    """Per-configuration energies and forces of all configurations, each rank evaluating its
    shard; results are gathered to every rank with one all-reduce of the scattered arrays.

    evaluate(shard_systems, beta, beta0) -> (E (nshard,), F (n_shard, 3), W (nshard, 6))."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    parts = shard(config_costs(systems, rcut), world)
    off = np.concatenate([[0], np.cumsum([len(s) for s in systems])])
    nc, n = len(systems), int(off[-1])
    E, F, W = np.zeros(nc), np.zeros((n, 3)), np.zeros((nc, 6))
    mine = parts[rank]
    if mine:
        e, f, w = evaluate([systems[c] for c in mine], beta, beta0)
        p = 0
        for k, c in enumerate(mine):
            m = off[c + 1] - off[c]
            E[c], W[c] = e[k], w[k]
            F[off[c]:off[c + 1]] = f[p:p + m]
            p += m
    tot = _all_reduce_sum(np.concatenate([E, F.ravel(), W.ravel()]), group)
    return tot[:nc], tot[nc:nc + 3 * n].reshape(n, 3), tot[nc + 3 * n:].reshape(nc, 6)
