"""Pullbacks of the SNAP energy and forces (ipg_snap_vjp and the torch autograd binding that
mirrors the Julia rrule): beta and position gradients, checked against the beta VJP that the
oracle pins, the exact -gE F energy term, central finite differences (h = 1e-5 A) of the
oracle's gE E + gF . F, and the symmetry of the exact Hessian-vector products."""
import numpy as np
import pytest

import oracle
import ipg
from ipg import workloads as W
from conftest import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    # 128 atoms, twojmax 8, two species; the 12.8 A box exceeds twice the 5 A cutoff, so every
    # neighbor has one image and E is smooth (a smaller box switches images as atoms move)
    system, prm, beta = W.snap_j8(cells=4)
    snap = ipg.SNAP(1, prm["twojmax"], prm["species"], prm["rcutfac"], prm["rmin0"], prm["rfac0"], prm["radii"],
                    prm["weight"], switch_flag=True)
    orc = oracle.Snap(prm["twojmax"], prm["radii"], prm["weight"], prm["rcutfac"], prm["rmin0"], prm["rfac0"],
                      switch=True)
    return system, snap, orc, beta


def _moved(s, d):
    return ipg.System(s.positions + d, s.symbols, s.box, s.periodic)


def test_vjp_beta_part_and_energy_term(case):
    system, snap, orc, beta = case
    rng = np.random.default_rng(11)
    gF = rng.normal(size=(len(system), 3))
    gb, gb0, _ = snap.vjp(system, beta, 0.7, gF)
    gb_ref, gb0_ref = snap.vjp_beta(system, 0.7, gF)
    assert rel_err(gb, gb_ref) <= 1e-14 and gb0 == 0.7
    go, _ = orc.vjp_beta(system.positions, snap.species_ids(system), system.L, 0.7, gF)
    assert rel_err(gb, go) <= 1e-10
    _, _, gp = snap.vjp(system, beta, 0.7, None)
    _, F, _ = snap.energy_forces(system, beta)
    assert rel_err(gp, -0.7 * F) <= 1e-14


def test_vjp_positions_finite_differences(case):
    """gpos . w == d/de [gE E + gF . F](x + e w) by central differences of the GPU's own E, F."""
    system, snap, orc, beta = case
    rng = np.random.default_rng(12)
    n = len(system)
    gE, gF = 0.3, rng.normal(size=(n, 3))
    _, _, gp = snap.vjp(system, beta, gE, gF)

    def L(s):
        E, F, _ = snap.energy_forces(s, beta)
        return gE * E + np.sum(gF * F)

    for seed in (1, 2):
        w = np.random.default_rng(seed).normal(size=(n, 3))
        eps = 1e-5
        fd = (L(_moved(system, eps * w)) - L(_moved(system, -eps * w))) / (2 * eps)
        assert abs(np.sum(gp * w) - fd) <= 1e-7 * max(abs(fd), 1e-12)


def _oracle_pullback_fd(orc, system, sp, beta, gE, gF, atoms, h=1e-5):
    """Central differences of the oracle's gE E + gF . F along single coordinates; the force
    part is summed from per-atom differences (exactly zero away from the moved atom)."""
    out = []
    for a, c in atoms:
        vals = []
        for sgn in (1.0, -1.0):
            pos = system.positions.copy()
            pos[a, c] += sgn * h
            E, F, _, Ei = orc.energy_forces(pos, sp, system.L, beta, 0.0, per_atom=True)
            vals.append((Ei, F))
        dE = np.sum(vals[0][0] - vals[1][0])
        dF = np.sum(gF * (vals[0][1] - vals[1][1]))
        out.append((gE * dE + dF) / (2 * h))
    return np.array(out)


@pytest.mark.parametrize("J", [4, 6, 8])
def test_position_pullback_vs_oracle_differences(J):
    """gpos of the exact second-order adjoint against central differences (h = 1e-5 A) of the
    oracle's energy and forces, 1e-7 of max|gpos|, on random coordinates of a two-species
    cluster in a periodic box."""
    rng = np.random.default_rng(40 + J)
    n = 60
    pos = rng.uniform(0, 9.0, (n, 3))
    sym = list(np.where(rng.random(n) < 0.6, "A", "B"))
    s = ipg.System(pos, sym, [9.0] * 3)
    prm = dict(twojmax=J, species=["A", "B"], rcutfac=2.0, rmin0=0.0, rfac0=0.98, radii=[1.0, 0.8],
               weight=[1.0, 0.7])
    snap = ipg.SNAP(1, J, prm["species"], prm["rcutfac"], prm["rmin0"], prm["rfac0"], prm["radii"], prm["weight"],
                    switch_flag=True)
    orc = oracle.Snap(J, prm["radii"], prm["weight"], prm["rcutfac"], prm["rmin0"], prm["rfac0"], switch=True)
    beta = rng.normal(0, 1e-2, (2, len(snap)))
    gE, gF = 0.4, rng.normal(size=(n, 3))
    _, _, gp = snap.vjp(s, beta, gE, gF)
    atoms = [(int(a), int(c)) for a, c in zip(rng.choice(n, 16, replace=False), rng.integers(0, 3, 16))]
    fd = _oracle_pullback_fd(orc, s, snap.species_ids(s), beta, gE, gF, atoms)
    got = np.array([gp[a, c] for a, c in atoms])
    assert np.abs(got - fd).max() <= 1e-7 * np.abs(gp).max(), np.abs(got - fd).max() / np.abs(gp).max()


def test_hessian_vector_symmetry(case):
    """a . (H b) == b . (H a) to rounding: gpos with gE = 0 is -H gF, taken exactly."""
    system, snap, orc, beta = case
    rng = np.random.default_rng(13)
    a, b = rng.normal(size=(2, len(system), 3))
    _, _, ha = snap.vjp(system, beta, 0.0, a)
    _, _, hb = snap.vjp(system, beta, 0.0, b)
    assert abs(np.sum(a * hb) - np.sum(b * ha)) <= 1e-12 * abs(np.sum(a * hb))


def test_hessian_vector_linear(case):
    """H (2a - 3b) == 2 H a - 3 H b to rounding (the tangent pass is linear in gF)."""
    system, snap, orc, beta = case
    rng = np.random.default_rng(15)
    a, b = rng.normal(size=(2, len(system), 3))
    _, _, ha = snap.vjp(system, beta, 0.0, a)
    _, _, hb = snap.vjp(system, beta, 0.0, b)
    _, _, hc = snap.vjp(system, beta, 0.0, 2 * a - 3 * b)
    assert rel_err(hc, 2 * ha - 3 * hb) <= 1e-12


def test_torch_autograd(case):
    torch = pytest.importorskip("torch")
    from ipg.autograd import snap_energy_forces, snap_loss
    system, snap, orc, beta = case
    pos = torch.tensor(system.positions, requires_grad=True)
    b = torch.tensor(beta, requires_grad=True)
    E, F = snap_energy_forces(snap, system, pos, b, 0.3)
    E.backward()
    assert rel_err(pos.grad.numpy(), -F.detach().numpy()) <= 1e-14
    gb, _ = snap.vjp_beta(system, 1.0, None)
    assert rel_err(b.grad.numpy(), gb) <= 1e-14
    # force-matching loss through the force output: beta gradient is exact (F is linear in beta)
    pos.grad = None
    b.grad = None
    E, F = snap_energy_forces(snap, system, pos, b, 0.3)
    loss = (F ** 2).sum()
    loss.backward()
    gb2, _ = snap.vjp_beta(system, 0.0, 2 * F.detach().numpy())
    assert rel_err(b.grad.numpy(), gb2) <= 1e-14
    _, _, gp2 = snap.vjp(system, beta, 0.0, 2 * F.detach().numpy())
    assert rel_err(pos.grad.numpy(), gp2) <= 1e-14
    # batch loss binding
    systems = [system, _moved(system, 0.01)]
    Fref = np.concatenate([snap.energy_forces(s, 1.1 * beta)[1] for s in systems])
    bl = torch.tensor(beta, requires_grad=True)
    lval = snap_loss(snap, systems, bl, Fref)
    lval.backward()
    l_ref, g_ref = snap.batch_loss_grad(systems, beta, Fref)
    assert abs(lval.item() - l_ref) <= 1e-14 * l_ref
    assert rel_err(bl.grad.numpy(), g_ref) <= 1e-14


@pytest.mark.parametrize("J", [2, 5, 8])
def test_chain_hvp_matches_forward_mode_kernel(J, monkeypatch):
    """The register-chain Hessian-vector product (Udot by k_snap_vsum, Ydot by polarization of
    the quadratic Y, the second-order pair chains) equals the per-atom forward-mode kernel
    (IPG_GENERIC_HVP=1) to rounding, at twojmax 2, 5 and 8."""
    rng = np.random.default_rng(70 + J)
    n = 90
    pos = rng.uniform(0, 10.0, (n, 3))
    sym = list(np.where(rng.random(n) < 0.5, "A", "B"))
    s = ipg.System(pos, sym, [10.0] * 3)
    args = (1, J, ["A", "B"], 2.2, 0.0, 0.97, [1.0, 0.8], [1.0, 0.6])
    fast = ipg.SNAP(*args, switch_flag=True)
    monkeypatch.setenv("IPG_GENERIC_HVP", "1")
    slow = ipg.SNAP(*args, switch_flag=True)
    beta = rng.normal(0, 1e-2, (2, len(fast)))
    gF = rng.normal(size=(n, 3))
    _, _, g1 = fast.vjp(s, beta, 0.25, gF)
    _, _, g2 = slow.vjp(s, beta, 0.25, gF)
    assert rel_err(g1, g2) <= 1e-12, rel_err(g1, g2)
