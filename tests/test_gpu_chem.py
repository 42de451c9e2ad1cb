"""Explicit multi-element SNAP (chem_flag, with bnorm) and quadratic SNAP on the GPU against the
oracle's restatement (src/BasisSystems/SNAP/utilities/compute_{ui,z,b}.jl with their element
loops; the quadratic products of LAMMPS_SNAP/snap.jl:45-47), FP64, 1e-10 relative.  The oracle's
own chem and quadratic paths are pinned by known answers in tests/test_oracle_golden.py (sums
over element triples reproduce the single-element descriptors; finite differences)."""
import numpy as np
import pytest

import ipg
import oracle
from ipg import workloads as W
from conftest import TOL, rel_err

pytestmark = pytest.mark.gpu


def _pair(J, radii, weight, rcutfac, chem=True, quadratic=False, bzero=False, wselfall=False, literal=False,
          rmin0=0.0, rfac0=0.99363):
    snap = ipg.SNAP(1, J, ["A", "B"][:len(radii)], rcutfac, rmin0, rfac0, radii, weight, chem_flag=chem,
                    bnorm_flag=chem, bzero_flag=bzero, switch_flag=True, wselfall_flag=wselfall,
                    quadratic_flag=quadratic, literal_chem_z=literal)
    orc = oracle.Snap(J, radii, weight, rcutfac, rmin0, rfac0, bzero=bzero, bnorm=chem, switch=True, chem=chem,
                      wselfall=wselfall, literal_chem_z=literal, quadratic=quadratic)
    assert len(snap) == orc.K
    return snap, orc


def _check(s, snap, orc, beta, beta0=0.2, modes=("plain", "adjoint")):
    sp = snap.species_ids(s)
    B, dB, Wd = ipg.compute_all_descriptors(s, snap)
    Bo, dBo, Wo = orc.descriptors(s.positions, sp, s.L)
    assert rel_err(B, Bo) <= TOL
    assert rel_err(dB, dBo.transpose(0, 2, 1)) <= TOL
    assert rel_err(Wd, Wo.T) <= TOL
    eo, fo, wo = orc.energy_forces(s.positions, sp, s.L, beta, beta0)
    for mode in modes:
        e, f, w = snap.energy_forces(s, beta, beta0, mode=mode)
        assert abs(e - eo) <= TOL * abs(eo), mode
        assert rel_err(f, fo) <= TOL, mode
        assert rel_err(w, wo) <= TOL, mode
    gF = np.random.default_rng(3).normal(size=(len(s), 3))
    gb, _ = snap.vjp_beta(s, 0.4, gF)
    gbo, _ = orc.vjp_beta(s.positions, sp, s.L, 0.4, gF)
    assert rel_err(gb, gbo) <= TOL


def test_chem_j8_two_species_bcc():
    """twojmax 8, two species (the 54,000-atom workload's parameters) on BCC 4^3 = 128 atoms:
    K = 55 * 2^3 = 440 components per species block."""
    s, prm, _ = W.snap_j8(cells=4)
    snap, orc = _pair(8, prm["radii"], prm["weight"], prm["rcutfac"])
    assert len(snap) == 440
    beta = np.random.default_rng(1).normal(0, 1e-2, (2, len(snap)))
    _check(s, snap, orc, beta)


@pytest.mark.parametrize("flags", [dict(bzero=True), dict(bzero=True, wselfall=True), dict(literal=True)])
def test_chem_flag_variants(flags):
    rng = np.random.default_rng(5)
    pos = rng.uniform(0, 9.0, (50, 3))
    s = ipg.System(pos, list(np.where(rng.random(50) < 0.6, "A", "B")), [9.0] * 3)
    snap, orc = _pair(6, [1.0, 0.8], [1.0, 0.7], 2.0, **flags)
    beta = rng.normal(0, 1e-2, (2, len(snap)))
    _check(s, snap, orc, beta)


@pytest.mark.parametrize("chem", [False, True])
def test_quadratic_snap(chem):
    rng = np.random.default_rng(6)
    pos = rng.uniform(0, 8.0, (40, 3))
    s = ipg.System(pos, list(np.where(rng.random(40) < 0.5, "A", "B")), [8.0] * 3)
    snap, orc = _pair(4, [1.0, 0.8], [1.0, 0.7], 2.0, chem=chem, quadratic=True)
    K = 14 * (8 if chem else 1)
    assert len(snap) == K + K * (K + 1) // 2
    beta = rng.normal(0, 1e-2, (2, len(snap)))
    _check(s, snap, orc, beta)


def test_chem_batch_and_fitting_rows():
    systems = W.batch512(nconf=6, nmin=32, nmax=160)
    prm = W.snap_j8_params()
    snap, orc = _pair(6, prm["radii"], prm["weight"], prm["rcutfac"])
    beta = np.random.default_rng(7).normal(0, 1e-2, (2, len(snap)))
    E, F, Wv = snap.batch_energy_forces(systems, beta, 0.1)
    off = np.concatenate([[0], np.cumsum([len(x) for x in systems])])
    Ae, Af, Aw = snap.fitting_matrices(systems)
    K, nsp = len(snap), 2
    for c, s in enumerate(systems):
        sp = snap.species_ids(s)
        eo, fo, wo = orc.energy_forces(s.positions, sp, s.L, beta, 0.1)
        assert abs(E[c] - eo) <= TOL * abs(eo)
        assert rel_err(F[off[c]:off[c + 1]], fo) <= TOL and rel_err(Wv[c], wo) <= TOL
        Bo, dBo, Wo = orc.descriptors(s.positions, sp, s.L)
        ae = np.concatenate([Bo[sp == q].sum(axis=0) for q in range(nsp)])
        assert rel_err(Ae[c], ae) <= TOL
        assert rel_err(Af[3 * off[c]:3 * off[c + 1]], dBo.transpose(0, 2, 1).reshape(-1, K * nsp)) <= TOL
        assert rel_err(Aw[c], Wo.T) <= TOL


def test_chem_position_pullback_unsupported():
    s, prm, _ = W.snap_j8(cells=3)
    snap, _ = _pair(4, prm["radii"], prm["weight"], prm["rcutfac"])
    beta = np.zeros((2, len(snap)))
    with pytest.raises(ipg.IPGError) as e:
        snap.vjp(s, beta, 0.0, np.ones((len(s), 3)))
    assert e.value.status == -8
