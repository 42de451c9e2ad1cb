"""Parity at the full benchmark sizes, against the oracle (the reference algorithm restated in
C++, OpenMP over the host cores).

  * SNAP twojmax 8, two species, BCC 30^3 = 54,000 atoms: energy, forces and virial of the
    adjoint and the plain dB/dr paths against the oracle's plain path
    (compute_all_descriptors, src/BasisSystems/SNAP/snap.jl:226-285, contracted with beta as
    in src/BasisPotentials/linear_potential.jl:20-49); the beta pullback against the oracle's;
    central finite differences (h = 1e-5 A) of the energy against the forces, and of
    gE E + gF . F against the position pullback, on 64 random atoms x 3 components.
  * 512 configurations of 32..2000 atoms (crystals and small-box liquids): every
    configuration's energy, forces and virial against the oracle, both paths, and the
    force-matching loss gradient of the whole batch against the oracle's beta pullback.
  * The fitting matrices (per-configuration sums of B, the dB rows, the W rows) and the
    Verlet-skin reuse path directly against the oracle.
Tolerance: 1e-10 relative (max|delta| / max|ref| per array; scalars relative), FP64.
"""
import numpy as np
import pytest

import ipg
import oracle
from ipg import workloads as W
from conftest import TOL, rel_err

pytestmark = pytest.mark.gpu


def _pair(prm):
    snap = ipg.SNAP(1, prm["twojmax"], prm["species"], prm["rcutfac"], prm["rmin0"], prm["rfac0"], prm["radii"],
                    prm["weight"], switch_flag=True)
    orc = oracle.Snap(prm["twojmax"], prm["radii"], prm["weight"], prm["rcutfac"], prm["rmin0"], prm["rfac0"],
                      switch=True)
    return snap, orc


@pytest.fixture(scope="module")
def j8_full():
    system, prm, beta = W.snap_j8()
    snap, orc = _pair(prm)
    sp = snap.species_ids(system)
    eo, fo, wo = orc.energy_forces(system.positions, sp, system.L, beta, 0.3)
    return system, snap, orc, beta, sp, (eo, fo, wo)


@pytest.mark.parametrize("mode", ["adjoint", "plain"])
def test_snap_j8_54000_atoms_vs_oracle(j8_full, mode):
    system, snap, orc, beta, sp, (eo, fo, wo) = j8_full
    assert len(system) == 54000
    e, f, w = snap.energy_forces(system, beta, 0.3, mode=mode)
    assert abs(e - eo) <= TOL * abs(eo), (e, eo)
    assert rel_err(f, fo) <= TOL
    assert rel_err(w, wo) <= TOL


def test_snap_j8_54000_atoms_vjp_beta_vs_oracle(j8_full):
    system, snap, orc, beta, sp, _ = j8_full
    gF = np.random.default_rng(11).normal(size=(len(system), 3))
    gb, gb0 = snap.vjp_beta(system, 0.6, gF)
    gbo, gbo0 = orc.vjp_beta(system.positions, sp, system.L, 0.6, gF)
    assert rel_err(gb, gbo) <= TOL
    assert gb0 == gbo0 == 0.6


def _local_energy_difference(snap, system, beta, pa, pm):
    """sum_i beta[s_i] . (B_i(pa) - B_i(pm)): the descriptors of atoms away from the moved atom
    are identical in both evaluations, so their differences vanish exactly and the sum keeps the
    full precision of the per-atom energies (a difference of two totals of 54,000 atoms loses
    about five digits to cancellation)."""
    sp = snap.species_ids(system)
    Bp = ipg.compute_local_descriptors(ipg.System(pa, system.symbols, system.box, system.periodic), snap)
    Bm = ipg.compute_local_descriptors(ipg.System(pm, system.symbols, system.box, system.periodic), snap)
    d = Bp - Bm
    rows = np.nonzero(np.any(d != 0.0, axis=1))[0]
    return float(np.sum(np.einsum("ik,ik->i", d[rows], beta[sp[rows]])))


def test_snap_j8_54000_atoms_finite_differences(j8_full):
    """-dE/dx by central differences (h = 1e-5 A) on 64 random atoms x 3 components equals the
    adjoint forces to 1e-7 of max|F| (truncation error h^2 F''' / 6 is far below)."""
    system, snap, orc, beta, sp, (eo, fo, wo) = j8_full
    _, f, _ = snap.energy_forces(system, beta, 0.3, mode="adjoint")
    h = 1e-5
    rng = np.random.default_rng(64)
    worst = 0.0
    for a in rng.choice(len(system), 64, replace=False):
        for c in range(3):
            pp = system.positions.copy()
            pp[a, c] += h
            pm = system.positions.copy()
            pm[a, c] -= h
            fd = -_local_energy_difference(snap, system, beta, pp, pm) / (2 * h)
            worst = max(worst, abs(fd - f[a, c]))
    assert worst <= 1e-7 * np.abs(f).max(), worst / np.abs(f).max()


def test_snap_j8_54000_atoms_position_pullback_fd(j8_full):
    """gpos of the rrule pullback (ipg_snap_vjp) against central differences (h = 1e-5 A) of
    gE E + gF . F on 64 random atoms x 3 components; the force part is summed from
    per-atom differences, as the energy part."""
    system, snap, orc, beta, sp, _ = j8_full
    rng = np.random.default_rng(65)
    n = len(system)
    gE = 0.4
    gF = rng.normal(size=(n, 3))
    _, _, gpos = snap.vjp(system, beta, gE, gF)
    h = 1e-5
    scale = np.abs(gpos).max()
    worst = 0.0
    for a in rng.choice(n, 64, replace=False):
        for c in range(3):
            pp = system.positions.copy()
            pp[a, c] += h
            pm = system.positions.copy()
            pm[a, c] -= h
            sp_, sm_ = (ipg.System(x, system.symbols, system.box, system.periodic) for x in (pp, pm))
            _, Fp, _ = snap.energy_forces(sp_, beta, 0.0)
            _, Fm, _ = snap.energy_forces(sm_, beta, 0.0)
            dF = Fp - Fm
            rows = np.nonzero(np.any(dF != 0.0, axis=1))[0]
            dLF = float(np.sum(dF[rows] * gF[rows]))
            dLE = _local_energy_difference(snap, system, beta, pp, pm)
            fd = (gE * dLE + dLF) / (2 * h)
            worst = max(worst, abs(fd - gpos[a, c]))
    assert worst <= 1e-7 * scale, worst / scale


@pytest.fixture(scope="module")
def batch_full():
    systems = W.batch512()
    prm = W.snap_j8_params()
    snap, orc = _pair(prm)
    beta = np.random.default_rng(55).normal(0, 1e-2, (2, len(snap)))
    ref = [orc.energy_forces(s.positions, snap.species_ids(s), s.L, beta, 0.1) for s in systems]
    return systems, snap, orc, beta, ref


@pytest.mark.parametrize("mode", ["adjoint", "plain"])
def test_batch512_every_configuration_vs_oracle(batch_full, mode):
    systems, snap, orc, beta, ref = batch_full
    assert len(systems) == 512
    E, F, Wv = snap.batch_energy_forces(systems, beta, 0.1, mode=mode)
    off = np.concatenate([[0], np.cumsum([len(s) for s in systems])])
    for c, (eo, fo, wo) in enumerate(ref):
        assert abs(E[c] - eo) <= TOL * abs(eo), (c, E[c], eo)
        assert rel_err(F[off[c]:off[c + 1]], fo) <= TOL, c
        assert rel_err(Wv[c], wo) <= TOL, c


def test_batch512_graph_replay_vs_oracle(batch_full):
    """The CUDA-graph replay of the whole 512-configuration batch against the oracle."""
    import torch
    systems, snap, orc, beta, ref = batch_full
    db = ipg.DeviceBatch(snap, systems)
    for _ in range(3):  # eager, capture, replay
        E, F, Wv = db.evaluate(beta, 0.1, graph=True)
    torch.cuda.synchronize()
    E, F, Wv = E.cpu().numpy(), F.cpu().numpy(), Wv.cpu().numpy()
    off = np.concatenate([[0], np.cumsum([len(s) for s in systems])])
    for c, (eo, fo, wo) in enumerate(ref):
        assert abs(E[c] - eo) <= TOL * abs(eo), c
        assert rel_err(F[off[c]:off[c + 1]], fo) <= TOL, c
        assert rel_err(Wv[c], wo) <= TOL, c


def test_batch512_loss_gradient_vs_oracle(batch_full):
    """L = sum |F - F_ref|^2 over all 512 configurations and dL/dbeta against the oracle's
    beta pullback with gF = 2 (F - F_ref), summed over configurations."""
    systems, snap, orc, beta, ref = batch_full
    rng = np.random.default_rng(56)
    Fo = np.concatenate([r[1] for r in ref])
    Fref = Fo + rng.normal(0, 0.01, Fo.shape)
    loss, g = snap.batch_loss_grad(systems, beta, Fref, 0.1)
    assert abs(loss - np.sum((Fo - Fref) ** 2)) <= TOL * loss
    off = np.concatenate([[0], np.cumsum([len(s) for s in systems])])
    go = np.zeros_like(g)
    for c, s in enumerate(systems):
        gF = 2.0 * (Fo[off[c]:off[c + 1]] - Fref[off[c]:off[c + 1]])
        go += orc.vjp_beta(s.positions, snap.species_ids(s), s.L, 0.0, gF)[0]
    assert rel_err(g, go) <= TOL


def test_fitting_matrices_vs_oracle(batch_full):
    """ipg_snap_batch_descriptors against the oracle's compute_all_descriptors: energy rows are
    per-species sums of B, force rows dB_a[x][:], virial rows W (snap.jl:267-281)."""
    systems, snap, orc, beta, ref = batch_full
    sub = systems[:40]
    Ae, Af, Aw = snap.fitting_matrices(sub)
    K, nsp = len(snap), len(snap.species)
    off = np.concatenate([[0], np.cumsum([len(s) for s in sub])])
    for c, s in enumerate(sub):
        sp = snap.species_ids(s)
        Bo, dBo, Wo = orc.descriptors(s.positions, sp, s.L)  # (n,K), (n,K*nsp,3), (K*nsp,6)
        ae = np.concatenate([Bo[sp == q].sum(axis=0) for q in range(nsp)])
        assert rel_err(Ae[c], ae) <= TOL, c
        af = dBo.transpose(0, 2, 1).reshape(-1, K * nsp)
        assert rel_err(Af[3 * off[c]:3 * off[c + 1]], af) <= TOL, c
        assert rel_err(Aw[c], Wo.T) <= TOL, c


def test_verlet_skin_steps_vs_oracle():
    """An MD-like sequence through the Verlet-skin path (reuse, then a rebuild after a large
    move), every step against the oracle."""
    system, prm, beta = W.snap_j8(cells=8)
    snap, orc = _pair(prm)
    snap.set_skin(0.4)
    rng = np.random.default_rng(31)
    sp = snap.species_ids(system)
    pos = system.positions.copy()
    for step in range(5):
        pos = pos + rng.normal(0, 0.02, pos.shape)
        if step == 3:
            pos = pos + rng.normal(0, 0.3, pos.shape)
        s = ipg.System(pos, system.symbols, system.box, system.periodic)
        for mode in ("adjoint", "plain"):
            e, f, w = snap.energy_forces(s, beta, 0.0, mode=mode)
            eo, fo, wo = orc.energy_forces(pos, sp, system.L, beta, 0.0)
            assert abs(e - eo) <= TOL * abs(eo), (step, mode)
            assert rel_err(f, fo) <= TOL and rel_err(w, wo) <= TOL, (step, mode)
    builds, reuses = snap.skin_stats()
    assert builds >= 2 and reuses >= 5
