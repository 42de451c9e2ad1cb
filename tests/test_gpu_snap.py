"""GPU SNAP vs the oracle (restatement of src/BasisSystems/SNAP/**), FP64, 1e-10 relative.

SNAP has no stored reference outputs (its tests compare against live LAMMPS and are
disabled, test/runtests.jl:46-50), so besides oracle parity the tests pin known
answers: the isolated-atom bispectrum, rotation/permutation invariance, sum of forces,
finite differences of the energy, and adjoint == plain.
"""
import numpy as np
import pytest
from scipy.spatial.transform import Rotation

import oracle
import ipg
from ipg import workloads as W
from conftest import TOL, rel_err

pytestmark = pytest.mark.gpu


def make(prm, **kw):
    """GPU SNAP and oracle SNAP with the same parameters."""
    p = dict(prm)
    p.update(kw)
    snap = ipg.SNAP(1, p["twojmax"], p["species"], p["rcutfac"], p["rmin0"], p["rfac0"], p["radii"], p["weight"],
                    bzero_flag=p.get("bzero_flag", False), switch_flag=p.get("switch_flag", False),
                    literal_sqrt_radius=p.get("literal", False))
    orc = oracle.Snap(p["twojmax"], p["radii"], p["weight"], p["rcutfac"], p["rmin0"], p["rfac0"],
                      bzero=p.get("bzero_flag", False), bnorm=False, switch=p.get("switch_flag", False),
                      literal_sqrt=p.get("literal", False))
    return snap, orc


def fixture_system(golden, tag):
    return ipg.System(golden[f"snap_{tag}_pos"], list(golden[f"snap_{tag}_symbols"]), golden[f"snap_{tag}_box"],
                      (False, False, False))


def fixture_params(golden, tag):
    return dict(twojmax=int(golden[f"snap_{tag}_twojmax"]), species=list(golden[f"snap_{tag}_species"]),
                rcutfac=float(golden[f"snap_{tag}_rcutfac"]), rmin0=0.0, rfac0=float(golden[f"snap_{tag}_rfac0"]),
                radii=list(golden[f"snap_{tag}_radii"]), weight=list(golden[f"snap_{tag}_weight"]))


def check_descriptors(s, snap, orc):
    B, dB, Wd = ipg.compute_all_descriptors(s, snap)
    Bo, dBo, Wo = orc.descriptors(s.positions, snap.species_ids(s), s.L)
    assert rel_err(B, Bo) <= TOL
    assert rel_err(dB, dBo.transpose(0, 2, 1)) <= TOL
    assert rel_err(Wd, Wo.T) <= TOL
    assert rel_err(ipg.compute_local_descriptors(s, snap), Bo) <= TOL
    assert rel_err(ipg.compute_force_descriptors(s, snap), dBo.transpose(0, 2, 1)) <= TOL
    return B, dB, Wd


@pytest.mark.parametrize("tag", ["single", "multi"])
@pytest.mark.parametrize("literal", [False, True])
def test_reference_fixture_3atoms(golden, tag, literal):
    """test/SNAP/snap_test_{single,multi}_element.jl inputs (all pairs inside sqrt(cutmax))."""
    s = fixture_system(golden, tag)
    prm = fixture_params(golden, tag)
    snap, orc = make(prm, literal=literal)
    check_descriptors(s, snap, orc)


@pytest.mark.parametrize("flags", [dict(), dict(bzero_flag=True), dict(switch_flag=True)])
def test_fixture_flags(golden, flags):
    s = fixture_system(golden, "multi")
    snap, orc = make(fixture_params(golden, "multi"), **flags)
    check_descriptors(s, snap, orc)


def test_isolated_atom_closed_form():
    """Utot = wself*I gives B(j1,j2,j) = j+1 (and 0 with bzero)."""
    for J in (2, 4, 6, 8):
        snap = ipg.SNAP(1, J, ["X"], 1.0, 0.0, 0.99363, [0.5], [1.0])
        s = ipg.System([[0.0, 0.0, 0.0]], ["X"], [10.0] * 3, (False, False, False))
        B = ipg.compute_local_descriptors(s, snap)[0]
        orc = oracle.Snap(J, [0.5], [1.0], 1.0, 0.0, 0.99363)
        jj = orc.index_tables()["idxb"][:, 2]
        np.testing.assert_allclose(B, (jj + 1).astype(float), rtol=1e-13, atol=0)
        snap0 = ipg.SNAP(1, J, ["X"], 1.0, 0.0, 0.99363, [0.5], [1.0], bzero_flag=True)
        assert np.all(np.abs(ipg.compute_local_descriptors(s, snap0)) <= 1e-12)


@pytest.mark.parametrize("J", [2, 3, 5, 6, 8, 10])
def test_random_cluster_all_J(J):
    rng = np.random.default_rng(J)
    pos = rng.uniform(0, 6, (24, 3))
    s = ipg.System(pos, list(np.where(rng.random(24) < 0.5, "A", "B")), [6.0] * 3, (True, True, False))
    snap, orc = make(dict(twojmax=J, species=["A", "B"], rcutfac=2.0, rmin0=0.2, rfac0=0.97, radii=[1.0, 0.8],
                          weight=[1.0, 0.7], switch_flag=True))
    check_descriptors(s, snap, orc)


def test_snap_j6_config_plain_parity():
    """Config 3 (twojmax 6, BCC 16^3 = 8192 atoms): E and F through the plain dB/dr path."""
    s, prm, beta = W.snap_j6()
    snap, orc = make(prm)
    e, f, w = snap.energy_forces(s, beta, 0.0, mode="plain")
    eo, fo, wo = orc.energy_forces(s.positions, snap.species_ids(s), s.L, beta, 0.0, mode="plain")
    assert abs(e - eo) <= TOL * abs(eo)
    assert rel_err(f, fo) <= TOL
    assert rel_err(w, wo) <= TOL
    ea, fa, wa = snap.energy_forces(s, beta, 0.0, mode="adjoint")
    assert abs(ea - eo) <= TOL * abs(eo)
    assert rel_err(fa, fo) <= TOL
    assert rel_err(wa, wo) <= TOL


@pytest.mark.parametrize("mode", ["plain", "adjoint"])
def test_snap_j8_two_species_parity(mode):
    """Config 4 at reduced size (BCC 8^3 = 1024 atoms), per-species beta blocks."""
    s, prm, beta = W.snap_j8(cells=8)
    snap, orc = make(prm)
    e, f, w = snap.energy_forces(s, beta, 0.25, mode=mode)
    eo, fo, wo = orc.energy_forces(s.positions, snap.species_ids(s), s.L, beta, 0.25, mode="plain")
    assert abs(e - eo) <= TOL * abs(eo)
    assert rel_err(f, fo) <= TOL
    assert rel_err(w, wo) <= TOL
    assert np.abs(f.sum(0)).max() <= 1e-12 * np.abs(f).max()


def test_snap_j8_full_size_adjoint_equals_plain():
    """Config 4 at full size (54,000 atoms): adjoint and plain forces agree, sum F = 0."""
    s, prm, beta = W.snap_j8()
    snap, _ = make(prm)
    e1, f1, w1 = snap.energy_forces(s, beta, 0.0, mode="plain")
    e2, f2, w2 = snap.energy_forces(s, beta, 0.0, mode="adjoint")
    assert abs(e1 - e2) <= TOL * abs(e1)
    assert rel_err(f2, f1) <= TOL
    assert rel_err(w2, w1) <= TOL
    assert np.abs(f2.sum(0)).max() <= 1e-11 * np.abs(f2).max()


def test_fd_forces_j8():
    """Central differences (h = 1e-5 A) of E against F on a subset of atoms."""
    s, prm, beta = W.snap_j8(cells=4)
    snap, _ = make(prm)
    _, f, _ = snap.energy_forces(s, beta, mode="adjoint")
    rng = np.random.default_rng(0)
    h = 1e-5
    for a in rng.choice(len(s), 8, replace=False):
        for c in range(3):
            pp = s.positions.copy(); pp[a, c] += h
            pm = s.positions.copy(); pm[a, c] -= h
            ep = snap.energy_forces(ipg.System(pp, s.symbols, s.box), beta)[0]
            em = snap.energy_forces(ipg.System(pm, s.symbols, s.box), beta)[0]
            assert abs(-(ep - em) / (2 * h) - f[a, c]) <= 1e-7 * np.abs(f).max()


def test_rotation_and_permutation_invariance():
    rng = np.random.default_rng(3)
    pos = rng.normal(0, 1.5, (30, 3))
    sym = list(np.where(rng.random(30) < 0.5, "A", "B"))
    snap, _ = make(dict(twojmax=8, species=["A", "B"], rcutfac=3.0, rmin0=0.0, rfac0=0.99363, radii=[1.0, 0.9],
                        weight=[1.0, 0.6], switch_flag=True))
    s = ipg.System(pos, sym, [100.0] * 3, (False, False, False))
    B = ipg.compute_local_descriptors(s, snap)
    R = Rotation.random(random_state=4).as_matrix()
    B2 = ipg.compute_local_descriptors(ipg.System(pos @ R.T, sym, [100.0] * 3, (False, False, False)), snap)
    assert rel_err(B2, B) <= 1e-12
    perm = rng.permutation(30)
    B3 = ipg.compute_local_descriptors(ipg.System(pos[perm], [sym[k] for k in perm], [100.0] * 3,
                                                  (False, False, False)), snap)
    assert rel_err(B3, B[perm]) <= 1e-13


def test_vjp_beta_matches_oracle():
    s, prm, beta = W.snap_j8(cells=3)
    snap, orc = make(prm)
    rng = np.random.default_rng(1)
    gF = rng.normal(size=(len(s), 3))
    gb, gb0 = snap.vjp_beta(s, 0.7, gF)
    gbo, gbo0 = orc.vjp_beta(s.positions, snap.species_ids(s), s.L, 0.7, gF)
    assert rel_err(gb, gbo) <= TOL
    assert gb0 == 0.7


def test_deterministic_bitwise():
    s, prm, beta = W.snap_j8(cells=5)
    snap, _ = make(prm)
    r1 = snap.energy_forces(s, beta, mode="adjoint")
    r2 = snap.energy_forces(s, beta, mode="adjoint")
    assert r1[0] == r2[0] and np.array_equal(r1[1], r2[1])


def test_species_out_of_range_rejected():
    snap = ipg.SNAP(1, 4, ["A"], 1.0, 0.0, 0.99, [1.0], [1.0])
    s = ipg.System([[0, 0, 0], [1, 0, 0]], ["A", "A"], [5.0] * 3)
    lib = ipg._lib.lib()
    import ctypes as C
    sp = np.array([0, 3], np.int32)
    B = np.zeros((2, len(snap)))
    st = lib.ipg_snap_descriptors(snap.handle, 2, s.positions.ctypes.data_as(C.c_void_p),
                                  sp.ctypes.data_as(C.c_void_p), s.L.ctypes.data_as(C.c_void_p),
                                  B.ctypes.data_as(C.c_void_p), None, None, 1)
    assert st == -7


def test_chem_flag_requires_bnorm():
    """snap.jl:10-13: chem_flag and bnorm_flag must be the same."""
    with pytest.raises(ValueError):
        ipg.SNAP(1, 4, ["A"], 1.0, 0.0, 0.99, [1.0], [1.0], chem_flag=True, bnorm_flag=False)
    import ctypes as C
    p = ipg._lib.SnapParams()
    p.twojmax, p.nspecies, p.rcutfac, p.rfac0 = 4, 1, 1.0, 0.99
    p.radii[0], p.weight[0] = 1.0, 1.0
    p.chem_flag, p.bnorm_flag = 1, 0
    h = C.c_void_p()
    assert ipg._lib.lib().ipg_snap_create(ipg.default_context().handle, C.byref(p), C.byref(h)) == -1


def test_lbasis_potential_api():
    """LBasisPotential with the reference's single K-vector beta (linear_potential.jl:20-35)."""
    s, prm, _ = W.snap_j6(cells=4)
    snap, orc = make(prm)
    beta = np.random.default_rng(2).normal(0, 1e-2, len(snap))
    lbp = ipg.LBasisPotential(beta, [0.5], snap)
    e = ipg.potential_energy(s, lbp)
    B = ipg.compute_local_descriptors(s, snap)
    assert abs(e - (0.5 + B.sum(0) @ beta)) <= 1e-12 * abs(e)
    ef = ipg.energy_and_force(s, lbp)
    dB = ipg.compute_force_descriptors(s, snap)
    assert rel_err(ef.f, dB @ beta) <= TOL
    assert abs(ef.e - e) <= 1e-12 * abs(e)
    Wd = ipg.compute_virial_descriptors(s, snap)
    assert rel_err(ipg.virial_stress(s, lbp), Wd @ beta) <= TOL


@pytest.mark.parametrize("J", [4, 7, 8, 9, 10, 11])
def test_adjoint_paths_agree(J, monkeypatch):
    """twojmax <= 10 runs the register-chain kernel, larger twojmax (or IPG_GENERIC_ADJOINT=1)
    the in-block per-neighbor loop; both must equal the plain dB/dr path and the oracle."""
    rng = np.random.default_rng(100 + J)
    pos = rng.uniform(0, 7, (40, 3))
    s = ipg.System(pos, list(np.where(rng.random(40) < 0.6, "A", "B")), [7.0] * 3)
    prm = dict(twojmax=J, species=["A", "B"], rcutfac=2.2, rmin0=0.1, rfac0=0.98, radii=[1.0, 0.8],
               weight=[1.0, 0.7], switch_flag=True)
    snap, orc = make(prm)
    beta = rng.normal(0, 1e-2, (2, len(snap)))
    eo, fo, wo = orc.energy_forces(s.positions, snap.species_ids(s), s.L, beta, 0.0)
    for generic in ("0", "1"):
        monkeypatch.setenv("IPG_GENERIC_ADJOINT", generic)
        snap2, _ = make(prm)
        e, f, w = snap2.energy_forces(s, beta, 0.0, mode="adjoint")
        assert abs(e - eo) <= TOL * abs(eo)
        assert rel_err(f, fo) <= TOL, generic
        assert rel_err(w, wo) <= TOL


@pytest.mark.parametrize("J", [4, 7, 8, 11])
def test_vjp_paths_agree(J, monkeypatch):
    """The beta pullback: twojmax <= 8 runs the register-chain path (Z by the row-blocked kernel,
    V per neighbor chain, contraction per atom tile), in chunks of atoms when IPG_VJP_CHUNK is
    set; larger twojmax or IPG_GENERIC_ADJOINT=1 the per-atom block kernel.  All equal the
    oracle, with and without the energy term gE B."""
    rng = np.random.default_rng(200 + J)
    pos = rng.uniform(0, 7, (100, 3))
    s = ipg.System(pos, list(np.where(rng.random(100) < 0.6, "A", "B")), [7.0] * 3)
    prm = dict(twojmax=J, species=["A", "B"], rcutfac=2.2, rmin0=0.1, rfac0=0.98, radii=[1.0, 0.8],
               weight=[1.0, 0.7], switch_flag=True, bzero_flag=J % 2 == 0)
    gF = rng.normal(size=(100, 3))
    _, orc = make(prm)
    for gE in (0.0, 0.7):
        go, _ = orc.vjp_beta(s.positions, np.array([0 if x == "A" else 1 for x in s.symbols], np.int32), s.L, gE,
                             gF)
        for generic, chunk in (("0", "0"), ("0", "40"), ("1", "0")):
            monkeypatch.setenv("IPG_GENERIC_ADJOINT", generic)
            monkeypatch.setenv("IPG_VJP_CHUNK", chunk)
            snap, _ = make(prm)
            gb, _ = snap.vjp_beta(s, gE, gF)
            assert rel_err(gb, go) <= TOL, (gE, generic, chunk)


@pytest.mark.parametrize("J", [5, 8, 11])
def test_descriptor_paths_agree(J, monkeypatch):
    """Local descriptors: Z from the row-blocked kernel and B per atom tile for twojmax <= 8
    (whole, or in chunks of 40 atoms), the per-atom block kernel otherwise."""
    rng = np.random.default_rng(300 + J)
    pos = rng.uniform(0, 7, (100, 3))
    s = ipg.System(pos, list(np.where(rng.random(100) < 0.6, "A", "B")), [7.0] * 3)
    prm = dict(twojmax=J, species=["A", "B"], rcutfac=2.2, rmin0=0.1, rfac0=0.98, radii=[1.0, 0.8],
               weight=[1.0, 0.7], switch_flag=True, bzero_flag=J % 2 == 0)
    _, orc = make(prm)
    sp = np.array([0 if x == "A" else 1 for x in s.symbols], np.int32)
    Bo, _, _ = orc.descriptors(s.positions, sp, s.L)
    for generic, chunk in (("0", "0"), ("0", "40"), ("1", "0")):
        monkeypatch.setenv("IPG_GENERIC_ADJOINT", generic)
        monkeypatch.setenv("IPG_VJP_CHUNK", chunk)
        snap, _ = make(prm)
        assert rel_err(ipg.compute_local_descriptors(s, snap), Bo) <= TOL, (generic, chunk)


@pytest.mark.parametrize("J", [3, 6, 8, 9])
def test_plain_paths_agree(J, monkeypatch):
    """The plain dB/dr path: for twojmax <= 8 the fused kernel (dU rows from the register chains
    contracted with the owner's Z; Z whole or in chunks of 40 atoms), otherwise (or with
    IPG_GENERIC_PLAIN=1) the per-atom block kernel; B, dB, W, E and F all equal the oracle."""
    rng = np.random.default_rng(400 + J)
    pos = rng.uniform(0, 7, (100, 3))
    s = ipg.System(pos, list(np.where(rng.random(100) < 0.6, "A", "B")), [7.0] * 3)
    prm = dict(twojmax=J, species=["A", "B"], rcutfac=2.2, rmin0=0.1, rfac0=0.98, radii=[1.0, 0.8],
               weight=[1.0, 0.7], switch_flag=True, bzero_flag=J % 2 == 0)
    _, orc = make(prm)
    sp = np.array([0 if x == "A" else 1 for x in s.symbols], np.int32)
    Bo, dBo, Wo = orc.descriptors(s.positions, sp, s.L)
    beta = rng.normal(0, 1e-2, (2, Bo.shape[1]))
    eo, fo, wo = orc.energy_forces(s.positions, sp, s.L, beta, 0.0)
    for generic, zchunk in (("0", "0"), ("0", "40"), ("1", "0")):
        monkeypatch.setenv("IPG_GENERIC_PLAIN", generic)
        monkeypatch.setenv("IPG_VJP_CHUNK", zchunk)
        snap, _ = make(prm)
        B, dB, Wd = ipg.compute_all_descriptors(s, snap)
        assert rel_err(B, Bo) <= TOL, (generic, zchunk)
        assert rel_err(dB, dBo.transpose(0, 2, 1)) <= TOL and rel_err(Wd, Wo.T) <= TOL, (generic, zchunk)
        e, f, w = snap.energy_forces(s, beta, 0.0, mode="plain")
        assert abs(e - eo) <= TOL * abs(eo) and rel_err(f, fo) <= TOL and rel_err(w, wo) <= TOL, (generic, zchunk)


def test_neighbor_switches_bitwise(monkeypatch):
    """The neighbor build walked once into padded slots or twice (IPG_WALK_SINGLE), and the list
    transpose on the side stream or in order (IPG_SIDE_STREAM), give bit-identical forces; so do
    repeated calls on one handle (the first call walks twice, later ones once)."""
    s, prm, beta = W.snap_j8(cells=5)
    ref = None
    for single, side in (("0", "0"), ("1", "1"), ("1", "0"), ("0", "1")):
        monkeypatch.setenv("IPG_WALK_SINGLE", single)
        monkeypatch.setenv("IPG_SIDE_STREAM", side)
        ctx = ipg.Context(0)
        snap = ipg.SNAP(len(s), prm["twojmax"], prm["species"], prm["rcutfac"], prm["rmin0"], prm["rfac0"],
                        prm["radii"], prm["weight"], switch_flag=True, ctx=ctx)
        for _ in range(3):
            e, f, w = snap.energy_forces(s, beta, mode="adjoint")
            if ref is None:
                ref = (e, f, w)
            assert e == ref[0] and np.array_equal(f, ref[1]) and np.array_equal(w, ref[2]), (single, side)


def test_twojmax_beyond_shared_memory_is_unsupported():
    """twojmax 12 needs more than 227 KB of shared memory per block: a clean error."""
    s = ipg.System(np.random.default_rng(0).uniform(0, 5, (10, 3)), ["A"] * 10, [5.0] * 3)
    snap = ipg.SNAP(1, 12, ["A"], 2.0, 0.0, 0.99, [1.0], [1.0])
    with pytest.raises(ipg.IPGError) as e:
        ipg.compute_local_descriptors(s, snap)
    assert e.value.status == -8


def test_autotune_choice_and_cache(tmp_path):
    """The autotuner times the candidate kernel configurations, keeps the fastest, writes the
    cache, and applies a cached choice without timing; every choice gives the same forces."""
    system, prm, beta = W.snap_j8(cells=8)
    snap, orc = make(prm, switch_flag=True)
    E0, F0, _ = snap.energy_forces(system, beta)
    cache = tmp_path / "tune.jsonl"
    rep = snap.autotune(system, beta, cache)
    assert rep["cached"] == 0 and rep["tried"] >= 6 and rep["ms"] > 0
    assert rep["utot_warps"] in (1, 2, 4) and rep["walk_warps"] in (1, 2, 4)
    E1, F1, _ = snap.energy_forces(system, beta)
    assert abs(E1 - E0) <= 1e-12 * abs(E0) and rel_err(F1, F0) <= 1e-12
    snap2, _ = make(prm, switch_flag=True)
    rep2 = snap2.autotune(system, beta, cache)
    assert rep2["cached"] == 1 and rep2["tried"] == 0
    for k in ("y_entries", "pair_split", "utot_split", "utot_warps", "walk_warps"):
        assert rep2[k] == rep[k]
    E2, F2, _ = snap2.energy_forces(system, beta)
    assert abs(E2 - E0) <= 1e-12 * abs(E0) and rel_err(F2, F0) <= 1e-12


def test_verlet_skin_reuse():
    """An MD-like sequence of small moves: with a skin the list is reused (and rebuilt after
    a large move), and every step equals a fresh evaluation to rounding."""
    system, prm, beta = W.snap_j8(cells=6)
    fresh, orc = make(prm, switch_flag=True)
    md, _ = make(prm, switch_flag=True)
    md.set_skin(0.4)
    rng = np.random.default_rng(21)
    pos = system.positions.copy()
    for step in range(6):
        pos = pos + rng.normal(0, 0.02, pos.shape)  # well inside skin/2 per step at first
        if step == 4:
            pos = pos + rng.normal(0, 0.3, pos.shape)  # some atom moves more than skin/2
        s = ipg.System(pos, system.symbols, system.box, system.periodic)
        E0, F0, W0 = fresh.energy_forces(s, beta)
        E1, F1, W1 = md.energy_forces(s, beta)
        assert abs(E1 - E0) <= 1e-12 * abs(E0)
        assert rel_err(F1, F0) <= 1e-12 and rel_err(W1, W0) <= 1e-12
    builds, reuses = md.skin_stats()
    assert builds >= 2 and reuses >= 3 and builds + reuses == 6
    # the skin list also serves the plain path and the descriptors
    E2, F2, _ = md.energy_forces(s, beta, mode="plain")
    assert rel_err(F2, F0) <= 1e-12


@pytest.mark.parametrize("case", ["single", "isolated_and_pair", "sparse"])
def test_register_chain_paths_edge_cases(case):
    """Atoms without neighbors (a lone atom, an isolated atom beside a close pair, a sparse gas)
    through every register-chain path: local descriptors, adjoint and plain energy and forces,
    and the beta pullback, against the oracle."""
    rng = np.random.default_rng(500)
    if case == "single":
        pos = np.array([[1.0, 2.0, 3.0]])
    elif case == "isolated_and_pair":
        pos = np.array([[1.0, 1.0, 1.0], [9.0, 9.0, 9.0], [9.0, 9.0, 10.1]])
    else:
        pos = rng.uniform(0, 30, (40, 3))
    n = len(pos)
    sym = ["A" if k % 3 else "B" for k in range(n)]
    s = ipg.System(pos, sym, [30.0] * 3)
    prm = dict(twojmax=8, species=["A", "B"], rcutfac=2.2, rmin0=0.0, rfac0=0.99363, radii=[1.0, 0.8],
               weight=[1.0, 0.7], switch_flag=True)
    snap, orc = make(prm)
    sp = np.array([0 if x == "A" else 1 for x in sym], np.int32)
    Bo, _, _ = orc.descriptors(s.positions, sp, s.L)
    assert rel_err(ipg.compute_local_descriptors(s, snap), Bo) <= TOL
    beta = rng.normal(0, 1e-2, (2, Bo.shape[1]))
    eo, fo, _ = orc.energy_forces(s.positions, sp, s.L, beta, 0.0)
    for mode in ("adjoint", "plain"):
        e, f, _ = snap.energy_forces(s, beta, 0.0, mode=mode)
        assert abs(e - eo) <= TOL * max(abs(eo), 1e-300), mode
        assert np.abs(f - fo).max() <= TOL * max(np.abs(fo).max(), 1.0), mode
    gF = rng.normal(size=(n, 3))
    gb, _ = snap.vjp_beta(s, 0.4, gF)
    go, _ = orc.vjp_beta(s.positions, sp, s.L, 0.4, gF)
    assert rel_err(gb, go) <= TOL


def test_verlet_skin_reuse_checks_inputs():
    """With a skin set, a device-pointer call that would reuse the list still reports a
    non-finite position (IPG_ERR_NONFINITE) and an out-of-range species id (IPG_ERR_SPECIES),
    as a fresh build does, and a call that keeps the positions but changes species rebuilds
    the list (its enlarged cutoffs depend on the species pair) and equals a fresh evaluation."""
    import ctypes as C
    import torch
    system, prm, beta = W.snap_j8(cells=5)
    fresh, _ = make(prm, switch_flag=True)
    md, _ = make(prm, switch_flag=True)
    md.set_skin(0.4)
    n = len(system)
    bb = md.beta_blocks(beta)
    L = system.L
    vp = C.c_void_p
    E = torch.zeros(1, dtype=torch.float64, device="cuda")
    F = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    Wv = torch.zeros(6, dtype=torch.float64, device="cuda")

    def dev_call(pos, sp):
        p = torch.tensor(pos, dtype=torch.float64, device="cuda")
        q = torch.tensor(sp, dtype=torch.int32, device="cuda")
        st = ipg._lib.lib().ipg_snap_energy_forces_dev(md.handle, n, vp(p.data_ptr()), vp(q.data_ptr()),
                                                       L.ctypes.data_as(vp), bb.ctypes.data_as(vp), 0.0, 1,
                                                       vp(E.data_ptr()), vp(F.data_ptr()), vp(Wv.data_ptr()))
        torch.cuda.synchronize()
        return st, E.item(), F.cpu().numpy()

    md.ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    try:
        sp0 = md.species_ids(system)
        assert dev_call(system.positions, sp0)[0] == 0
        assert dev_call(system.positions, sp0)[0] == 0
        assert md.skin_stats() == (1, 1)
        bad = system.positions.copy()
        bad[7, 1] = np.nan
        assert dev_call(bad, sp0)[0] == -6
        E0, F0, _ = fresh.energy_forces(system, beta)
        st, E1, F1 = dev_call(system.positions, sp0)
        assert st == 0 and abs(E1 - E0) <= 1e-12 * abs(E0) and rel_err(F1, F0) <= 1e-12
        # same positions, species swapped on a tenth of the atoms
        sym = list(system.symbols)
        for k in range(0, len(sym), 10):
            sym[k] = "B" if sym[k] == "A" else "A"
        s2 = ipg.System(system.positions, sym, system.box, system.periodic)
        sp2 = md.species_ids(s2)
        b0 = md.skin_stats()[0]
        E0, F0, _ = fresh.energy_forces(s2, beta)
        st, E1, F1 = dev_call(system.positions, sp2)
        assert st == 0 and md.skin_stats()[0] == b0 + 1
        assert abs(E1 - E0) <= 1e-12 * abs(E0) and rel_err(F1, F0) <= 1e-12
        assert dev_call(system.positions, sp2)[0] == 0  # reuse again
        sp3 = sp2.copy()
        sp3[3] = 5
        assert dev_call(system.positions, sp3)[0] == -7
    finally:
        md.ctx.set_stream(None)


@pytest.mark.parametrize("env", [dict(IPG_YR_WARPS="8"), dict(IPG_YR_WARPS="10"), dict(IPG_YR_WARPS="16")])
def test_y_kernel_variants_agree(env, monkeypatch):
    """The adjoint Y kernel with 8, 10 or 16 warps per block (the default has twelve) gives the
    forces of the default kernel to rounding and the oracle's to 1e-10."""
    s, prm, beta = W.snap_j8(cells=6)
    ref, orc = make(prm, switch_flag=True)
    e0, f0, w0 = ref.energy_forces(s, beta, 0.1)
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    snap, _ = make(prm, switch_flag=True)
    e, f, w = snap.energy_forces(s, beta, 0.1)
    assert abs(e - e0) <= 1e-13 * abs(e0) and rel_err(f, f0) <= 1e-13 and rel_err(w, w0) <= 1e-13
    eo, fo, _ = orc.energy_forces(s.positions, snap.species_ids(s), s.L, beta, 0.1)
    assert abs(e - eo) <= TOL * abs(eo) and rel_err(f, fo) <= TOL


@pytest.mark.parametrize("J", [2, 5, 6, 8, 10])
@pytest.mark.parametrize("density", ["dense", "dilute"])
def test_pair_generator_identity_vs_tangent_chains(J, density, monkeypatch):
    """The adjoint pair kernel contracts U alone with the Lie-generator-shifted copies of Y
    (dU/dr = U times a generator of SU(2)); IPG_PAIR_TANGENT=1 runs the forward tangent chains
    instead.  Both give the same forces to rounding and the oracle's to 1e-10.  "dilute" gives
    atoms a few neighbors or none, so a block of pairs spans more atoms than it stages at once
    (its owners are staged group by group)."""
    rng = np.random.default_rng(700 + J)
    n, box = (60, 7.5) if density == "dense" else (90, 30.0)
    pos = rng.uniform(0, box, (n, 3))
    s = ipg.System(pos, list(np.where(rng.random(n) < 0.5, "A", "B")), [box] * 3)
    prm = dict(twojmax=J, species=["A", "B"], rcutfac=2.4, rmin0=0.05, rfac0=0.97, radii=[1.0, 0.85],
               weight=[1.0, 0.6], switch_flag=True)
    snap, orc = make(prm)
    beta = rng.normal(0, 1e-2, (2, len(snap)))
    e0, f0, w0 = snap.energy_forces(s, beta, 0.0, mode="adjoint")
    monkeypatch.setenv("IPG_PAIR_TANGENT", "1")
    snap_t, _ = make(prm)
    e1, f1, w1 = snap_t.energy_forces(s, beta, 0.0, mode="adjoint")
    assert e1 == e0  # the energy does not go through the pair kernel
    assert rel_err(f0, f1) <= 1e-12 and rel_err(w0, w1) <= 1e-12
    eo, fo, wo = orc.energy_forces(s.positions, snap.species_ids(s), s.L, beta, 0.0)
    assert abs(e0 - eo) <= TOL * abs(eo)
    assert rel_err(f0, fo) <= TOL and rel_err(w0, wo) <= TOL
    # the beta pullback's V = sum_j g_ij . dU_ij/dr (and the Utot tangent of the position
    # pullback) go through the same identity
    gF = rng.normal(size=(n, 3))
    gb0, g00 = snap.vjp_beta(s, 0.3, gF)
    gb1, g01 = snap_t.vjp_beta(s, 0.3, gF)
    assert rel_err(gb0, gb1) <= 1e-12 and g00 == g01
    ob, _ = orc.vjp_beta(s.positions, snap.species_ids(s), s.L, 0.3, gF)
    assert rel_err(gb0, ob) <= TOL
    if J <= 8:  # the position pullback covers twojmax <= 8 (its shared memory beyond)
        pb0, _, gp0 = snap.vjp(s, beta, 0.3, gF)
        pb1, _, gp1 = snap_t.vjp(s, beta, 0.3, gF)
        assert rel_err(pb0, pb1) <= 1e-12 and rel_err(gp0, gp1) <= 1e-12
