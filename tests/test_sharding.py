"""Sharded batch evaluation across ranks (ipg/sharding.py), world size 2 over gloo on CPU.

The GPU evaluator is replaced by a CPU stand-in with the same call shape: a model whose
forces are linear in beta, F = D(x) beta, so the loss gradient has a closed form and the
sharded, all-reduced result must equal the single-process one to rounding."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from ipg import sharding
from ipg import workloads as W


def _model(systems, beta, F_ref):
    """loss = sum |D beta - F_ref|^2 with a per-configuration descriptor D from positions."""
    loss, g = 0.0, np.zeros_like(beta)
    p = 0
    for s in systems:
        n = len(s)
        D = np.stack([np.sin((k + 1) * s.positions) for k in range(beta.size)], axis=-1)  # (n, 3, K)
        F = D @ beta
        r = F - F_ref[p:p + n]
        loss += float(np.sum(r * r))
        g += 2.0 * np.einsum("nck,nc->k", D, r)
        p += n
    return loss, g


def _ef(systems, beta, beta0):
    E = np.array([beta0 + float(np.sum(np.cos(s.positions)) * beta.sum()) for s in systems])
    F = np.concatenate([np.sin(s.positions) * beta[0] for s in systems])
    Wv = np.stack([np.full(6, len(s) * beta[1]) for s in systems])
    return E, F, Wv


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        systems = W.batch512(nconf=11, nmin=32, nmax=200)
        rng = np.random.default_rng(3)
        beta = rng.normal(size=4)
        F_ref = rng.normal(size=(sum(len(s) for s in systems), 3))
        loss, g = sharding.loss_grad(_model, systems, beta, F_ref, rcut=5.0)
        E, F, Wv = sharding.energy_forces(_ef, systems, beta, 0.25, rcut=5.0)
        q.put((rank, loss, g, E, F, Wv))
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_shard_is_balanced_and_deterministic():
    costs = np.random.default_rng(0).uniform(1, 100, 97)
    for world in (1, 2, 4, 8):
        parts = sharding.shard(costs, world)
        assert sorted(c for p in parts for c in p) == list(range(97))
        loads = [costs[p].sum() for p in parts]
        assert max(loads) - min(loads) <= costs.max()  # greedy longest-first bound
        assert parts == sharding.shard(costs, world)


def test_two_ranks_gloo_match_single_process():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    systems = W.batch512(nconf=11, nmin=32, nmax=200)
    rng = np.random.default_rng(3)
    beta = rng.normal(size=4)
    F_ref = rng.normal(size=(sum(len(s) for s in systems), 3))
    loss1, g1 = _model(systems, beta, F_ref)
    E1, F1, W1 = _ef(systems, beta, 0.25)
    for rank, loss, g, E, F, Wv in out:
        assert abs(loss - loss1) <= 1e-12 * loss1
        assert np.allclose(g, g1, rtol=1e-12, atol=0)
        assert np.array_equal(E, E1) and np.array_equal(F, F1) and np.array_equal(Wv, W1)
