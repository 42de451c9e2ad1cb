"""Batched SNAP (many configurations per launch) and the force-matching loss gradient."""
import numpy as np
import pytest

import oracle
import ipg
from ipg import workloads as W
from conftest import TOL, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def batch():
    systems = W.batch512(nconf=24, nmin=32, nmax=400)
    prm = W.snap_j8_params()
    snap = ipg.SNAP(1, prm["twojmax"], prm["species"], prm["rcutfac"], prm["rmin0"], prm["rfac0"], prm["radii"],
                    prm["weight"], switch_flag=True)
    orc = oracle.Snap(prm["twojmax"], prm["radii"], prm["weight"], prm["rcutfac"], prm["rmin0"], prm["rfac0"],
                      switch=True)
    beta = np.random.default_rng(5).normal(0, 1e-2, (2, len(snap)))
    return systems, snap, orc, beta


@pytest.mark.parametrize("mode", ["adjoint", "plain"])
def test_batch_matches_single_and_oracle(batch, mode):
    systems, snap, orc, beta = batch
    E, F, Wv = snap.batch_energy_forces(systems, beta, 0.1, mode=mode)
    off = np.concatenate([[0], np.cumsum([len(s) for s in systems])])
    for c, s in enumerate(systems):
        eo, fo, wo = orc.energy_forces(s.positions, snap.species_ids(s), s.L, beta, 0.1)
        assert abs(E[c] - eo) <= TOL * abs(eo)
        assert rel_err(F[off[c]:off[c + 1]], fo) <= TOL
        assert rel_err(Wv[c], wo) <= TOL
        if c < 3:
            e1, f1, w1 = snap.energy_forces(s, beta, 0.1, mode=mode)
            assert abs(E[c] - e1) <= 1e-13 * abs(e1)
            assert rel_err(F[off[c]:off[c + 1]], f1) <= 1e-13


def test_loss_gradient(batch):
    systems, snap, orc, beta = batch
    rng = np.random.default_rng(6)
    beta_ref = beta + rng.normal(0, 1e-3, beta.shape)
    _, Fref, _ = snap.batch_energy_forces(systems, beta_ref, 0.0)
    Fref = Fref + rng.normal(0, 0.01, Fref.shape)
    loss, g = snap.batch_loss_grad(systems, beta, Fref)
    _, F, _ = snap.batch_energy_forces(systems, beta, 0.0)
    assert abs(loss - np.sum((F - Fref) ** 2)) <= 1e-12 * loss
    # oracle: dL/dbeta = sum_k 2 (F_k - Fref_k) . dF_k/dbeta, per configuration
    off = np.concatenate([[0], np.cumsum([len(s) for s in systems])])
    go = np.zeros_like(g)
    for c, s in enumerate(systems):
        gF = 2.0 * (F[off[c]:off[c + 1]] - Fref[off[c]:off[c + 1]])
        gb, _ = orc.vjp_beta(s.positions, snap.species_ids(s), s.L, 0.0, gF)
        go += gb
    assert rel_err(g, go) <= TOL
    # L is quadratic in beta: central differences are exact up to rounding
    h = 1e-4
    for (s_, k) in [(0, 0), (1, 7), (0, 54)]:
        bp = beta.copy(); bp[s_, k] += h
        bm = beta.copy(); bm[s_, k] -= h
        lp = snap.batch_loss_grad(systems, bp, Fref)[0]
        lm = snap.batch_loss_grad(systems, bm, Fref)[0]
        assert abs((lp - lm) / (2 * h) - g[s_, k]) <= 1e-6 * np.abs(g).max()


def _moved(systems, rng, sigma=0.05):
    return [ipg.System(s.positions + rng.normal(0, sigma, s.positions.shape), s.symbols, s.box, s.periodic)
            for s in systems]


def test_graph_replay(batch):
    """ipg_snap_batch_energy_forces_dev with graph=1: capture on the first call, one graph launch
    on later calls (new positions and beta read from the buffers), bitwise equal to eager runs."""
    import torch
    systems, snap, orc, beta = batch
    db = ipg.DeviceBatch(snap, systems)
    E0, F0, W0 = snap.batch_energy_forces(systems, beta, 0.1)
    for call in range(3):
        l0 = snap.ctx.launch_count()
        E, F, W = db.evaluate(beta, 0.1, graph=True)
        torch.cuda.synchronize()
        if call > 0:  # a replay launches only k_ycoef through the library, the rest is the graph
            assert snap.ctx.launch_count() - l0 <= 2
        assert np.array_equal(E.cpu().numpy(), E0)
        assert np.array_equal(F.cpu().numpy(), F0)
        assert np.array_equal(W.cpu().numpy(), W0)
    # new positions and beta through the same graph
    rng = np.random.default_rng(7)
    moved = _moved(systems, rng)
    db.set_positions(np.concatenate([s.positions for s in moved]))
    beta2 = 1.3 * beta
    l0 = snap.ctx.launch_count()
    E, F, W = db.evaluate(beta2, -0.2, graph=True)
    torch.cuda.synchronize()
    assert snap.ctx.launch_count() - l0 <= 2
    E1, F1, W1 = snap.batch_energy_forces(moved, beta2, -0.2)
    assert np.array_equal(E.cpu().numpy(), E1)
    assert np.array_equal(F.cpu().numpy(), F1)
    assert np.array_equal(W.cpu().numpy(), W1)
    # plain mode gets its own graph
    Ep, Fp, _ = db.evaluate(beta2, -0.2, mode="plain", graph=True)
    Ep, Fp, _ = db.evaluate(beta2, -0.2, mode="plain", graph=True)
    assert rel_err(Fp.cpu().numpy(), F1) <= TOL


def test_graph_capacity_overflow_reruns(batch):
    """A replay whose pair count outgrows the captured capacity re-runs eagerly (correct
    results) and recaptures."""
    import torch
    systems, snap, orc, beta = batch
    db = ipg.DeviceBatch(snap, systems)
    db.evaluate(beta, 0.0, graph=True)
    db.evaluate(beta, 0.0, graph=True)
    # squeeze the largest configuration: many more neighbors than the 25% headroom
    big = int(np.argmax([len(s) for s in systems]))
    dense = list(systems)
    s = systems[big]
    c = s.positions.mean(axis=0)
    dense[big] = ipg.System(c + 0.45 * (s.positions - c), s.symbols, s.box, s.periodic)
    db.set_positions(np.concatenate([x.positions for x in dense]))
    E, F, W = db.evaluate(beta, 0.0, graph=True)
    torch.cuda.synchronize()
    E1, F1, W1 = snap.batch_energy_forces(dense, beta, 0.0)
    assert np.array_equal(E.cpu().numpy(), E1)
    assert np.array_equal(F.cpu().numpy(), F1)
    l0 = snap.ctx.launch_count()
    E, F, W = db.evaluate(beta, 0.0, graph=True)  # the recaptured graph
    torch.cuda.synchronize()
    assert snap.ctx.launch_count() - l0 <= 2
    assert np.array_equal(F.cpu().numpy(), F1)


def test_graph_open_boundaries_run_eagerly():
    import torch
    prm = W.snap_j8_params()
    snap = ipg.SNAP(1, prm["twojmax"], prm["species"], prm["rcutfac"], prm["rmin0"], prm["rfac0"], prm["radii"],
                    prm["weight"], switch_flag=True)
    systems = W.batch512(nconf=4, nmin=32, nmax=120)
    systems = [ipg.System(s.positions, s.symbols, s.box, (True, False, True)) for s in systems]
    beta = np.random.default_rng(8).normal(0, 1e-2, (2, len(snap)))
    db = ipg.DeviceBatch(snap, systems)
    E0, F0, _ = snap.batch_energy_forces(systems, beta, 0.0)
    for _ in range(2):
        E, F, _ = db.evaluate(beta, 0.0, graph=True)
        torch.cuda.synchronize()
        assert np.array_equal(F.cpu().numpy(), F0)


def test_fitting_matrices(batch):
    """ipg_snap_batch_descriptors: energy, force and virial rows of every configuration equal
    the single-configuration descriptors and reproduce E, F and W of the batched evaluation."""
    systems, snap, orc, beta = batch
    sub = systems[:6]
    Ae, Af, Aw = snap.fitting_matrices(sub)
    K, nsp = len(snap), len(snap.species)
    off = np.concatenate([[0], np.cumsum([len(s) for s in sub])])
    for c, s in enumerate(sub):
        B, dB, Wd = ipg.compute_all_descriptors(s, snap)  # B (n, K), dB (n, 3, K*nsp), W (6, K*nsp)
        sp = snap.species_ids(s)
        ae = np.concatenate([B[sp == q].sum(axis=0) for q in range(nsp)])
        assert rel_err(Ae[c], ae) <= 1e-13
        assert rel_err(Af[3 * off[c]:3 * off[c + 1]], dB.reshape(-1, K * nsp)) <= 1e-13
        assert rel_err(Aw[c], Wd) <= 1e-13
    E, F, Wv = snap.batch_energy_forces(sub, beta, 0.25, mode="plain")
    b = beta.reshape(-1)
    assert rel_err(Ae @ b + 0.25, E) <= 1e-12
    assert rel_err(Af @ b, F.reshape(-1)) <= 1e-12


def test_train_step_graph(batch):
    """ipg_snap_batch_loss_grad_dev: E, F, the loss and dL/dbeta of one force-matching step;
    with graph=1 the first call captures the whole step and later calls replay it with one graph
    launch (new positions and beta read from the buffers), bitwise equal to eager steps and
    equal to the host-pointer loss gradient and to the oracle."""
    import torch
    systems, snap, orc, beta = batch
    rng = np.random.default_rng(9)
    _, F0, _ = snap.batch_energy_forces(systems, beta + rng.normal(0, 1e-3, beta.shape), 0.0)
    Fref_h = F0 + rng.normal(0, 0.01, F0.shape)
    db = ipg.DeviceBatch(snap, systems)
    Fref = torch.tensor(Fref_h, device=db.pos.device)
    loss_e, g_e = db.train_step(beta, Fref, 0.2, graph=False)
    loss_e, g_e = loss_e.item(), g_e.cpu().numpy().copy()
    E_e, F_e = db.E.cpu().numpy().copy(), db.F.cpu().numpy().copy()
    loss_h, g_h = snap.batch_loss_grad(systems, beta, Fref_h, 0.2)
    assert abs(loss_e - loss_h) <= 1e-13 * loss_h and rel_err(g_e, g_h) <= 1e-13
    off = np.concatenate([[0], np.cumsum([len(s) for s in systems])])
    go = np.zeros_like(g_e)
    for c, s in enumerate(systems):
        eo, fo, _ = orc.energy_forces(s.positions, snap.species_ids(s), s.L, beta, 0.2)
        assert abs(E_e[c] - eo) <= TOL * abs(eo)
        gF = 2.0 * (fo - Fref_h[off[c]:off[c + 1]])
        go += orc.vjp_beta(s.positions, snap.species_ids(s), s.L, 0.0, gF)[0]
    assert rel_err(g_e, go) <= TOL
    for call in range(3):
        l0 = snap.ctx.launch_count()
        loss, g = db.train_step(beta, Fref, 0.2, graph=True)
        torch.cuda.synchronize()
        if call > 0:  # k_ycoef through the library, the rest is one graph launch
            assert snap.ctx.launch_count() - l0 <= 2
        assert loss.item() == loss_e and np.array_equal(g.cpu().numpy(), g_e)
        assert np.array_equal(db.E.cpu().numpy(), E_e) and np.array_equal(db.F.cpu().numpy(), F_e)
    moved = _moved(systems, np.random.default_rng(10))
    db.set_positions(np.concatenate([s.positions for s in moved]))
    beta2 = 0.9 * beta
    loss, g = db.train_step(beta2, Fref, 0.0, graph=True)
    torch.cuda.synchronize()
    loss_h2, g_h2 = snap.batch_loss_grad(moved, beta2, Fref_h, 0.0)
    assert abs(loss.item() - loss_h2) <= 1e-13 * loss_h2 and rel_err(g.cpu().numpy(), g_h2) <= 1e-13
