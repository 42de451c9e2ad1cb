"""The oracle pinned against the reference's golden vectors (CPU only).

The oracle (oracle/ipg_oracle.cpp, a restatement of the reference's Julia loops) is the
checker for every GPU parity test, so it is checked first: against the numbers the
reference's own tests assert, against an independent NumPy restatement, and against
known answers of the SNAP bispectrum.
"""
import numpy as np
import pytest
from scipy.spatial.transform import Rotation

import oracle
from ipg import units
from ipg import workloads as W


def test_nnlist_golden(golden):
    """test/unit/nnlist.jl: pairs (1,2), (1,3) and their displacements."""
    L = np.where(golden["nnlist_periodic"], golden["nnlist_box"], np.inf)
    off, j, r = oracle.nlist_half(golden["nnlist_pos"], L, float(golden["nnlist_rcut"]))
    assert np.diff(off).tolist() == golden["nnlist_true_j_count"].tolist()
    assert j.tolist() == golden["nnlist_true_j_flat"].tolist()
    np.testing.assert_allclose(r, golden["nnlist_true_r"], rtol=0, atol=1e-14)
    js, rs = oracle.np_nlist_half(golden["nnlist_pos"], L, float(golden["nnlist_rcut"]))
    assert sum(js, []) == j.tolist()


def test_mock_potential_golden(golden):
    """test/unit/types/empirical_potential.jl: E = 0.5, F = +-0.125, virial exactly."""
    syms = list(golden["mock_symbols"])
    idx = {s: k for k, s in enumerate(dict.fromkeys(syms))}
    sp = np.array([idx[s] for s in syms], np.int32)
    mask = sum(1 << idx[s] for s in golden["mock_species"])
    E, F, Wv = oracle.pair_eval(golden["mock_pos"], sp, golden["mock_box"],
                                [dict(kind="MOCK_R2", rcut=float(golden["mock_rcut"]), mask=mask,
                                      params=[float(golden["mock_seed"])])])
    assert E == float(golden["mock_e"])
    assert np.array_equal(F, golden["mock_f"])
    assert np.array_equal(Wv, golden["mock_virial"])


@pytest.mark.parametrize("n", [150, 1000])
def test_lj_clusters_golden(golden, n):
    """test/integration/lj_clusters/lj_{150,1000}.jl."""
    A, eV = units.angstrom, units.eV
    pos = golden[f"lj{n}_pos"] * A
    eps, sig = float(golden[f"lj{n}_eps_eV"]) * eV, float(golden[f"lj{n}_sigma_A"]) * A
    E, F, Wv = oracle.pair_eval(pos, np.zeros(n, np.int32), np.full(3, np.inf),
                                [dict(kind="LJ", rcut=float(golden[f"lj{n}_rcut_A"]) * A, params=[eps, sig])])
    e_atol = float(golden[f"lj{n}_E_atol_eV"]) * eV
    f_atol = float(golden[f"lj{n}_F_atol_eVA"]) * eV / A
    assert abs(E - float(golden[f"lj{n}_E_eV"]) * eV) <= e_atol
    assert np.all(np.abs(F.sum(0)) <= f_atol)
    if n == 150:
        assert np.all(np.abs(F) <= f_atol)
        assert abs(Wv[:3].sum()) <= e_atol
    En, Fn = oracle.np_lj_allpairs(pos, eps, sig)
    assert abs(E - En) <= 1e-12 * abs(En)


def test_half_list_vs_numpy_periodic():
    rng = np.random.default_rng(0)
    pos = rng.uniform(-5, 25, (150, 3))
    L = np.array([12.0, np.inf, 9.0])
    off, j, r = oracle.nlist_half(pos, L, 4.0)
    js, rs = oracle.np_nlist_half(pos, L, 4.0)
    assert j.tolist() == sum(js, [])
    np.testing.assert_array_equal(r, np.array(sum(rs, [])).reshape(-1, 3))


def test_snap_table_sizes():
    """Sizes of the prebuilt tables (prebuilt_arrays.jl:76-216) for twojmax 4, 6, 8."""
    for J, sizes in ((4, (55, 185, 14, 305)), (6, (140, 779, 30, 1321)), (8, (285, 2386, 55, 4098))):
        s = oracle.Snap(J, [1.0], [1.0], 1.0)
        assert (s.idxu_max, s.idxz_max, s.idxb_max, s.idxcg_max) == sizes


def test_cg_orthonormality():
    """sum over (m1, m2) of CG(j1 m1 j2 m2 | j m)^2 = 1 for each (j1, j2, j, m) block."""
    J = 8
    s = oracle.Snap(J, [1.0], [1.0], 1.0)
    cg = s.cglist()
    t = s.index_tables()
    for j1 in range(J + 1):
        for j2 in range(j1 + 1):
            for j in range(j1 - j2, min(J, j1 + j2) + 1, 2):
                blk = cg[t["idxcg_block"][j1, j2, j]:][: (j1 + 1) * (j2 + 1)].reshape(j1 + 1, j2 + 1)
                for m in range(j + 1):
                    tot = sum(blk[m1, m2] ** 2 for m1 in range(j1 + 1) for m2 in range(j2 + 1)
                              if (2 * m1 - j1 + 2 * m2 - j2 + j) // 2 == m and (2 * m1 - j1 + 2 * m2 - j2 + j) % 2 == 0)
                    assert abs(tot - 1.0) < 1e-12


def test_snap_known_answers():
    s = oracle.Snap(8, [0.5, 0.45], [1.0, 0.5], 5.0, 0.0, 0.99363, switch=True)
    t = s.index_tables()
    B, _, _ = s.descriptors(np.zeros((1, 3)), [0], np.full(3, np.inf))
    # isolated atom: Utot = wself*I gives B(j1,j2,j) = j+1 (up to rounding of the CG sums)
    np.testing.assert_allclose(B[0], (t["idxb"][:, 2] + 1).astype(float), rtol=1e-13, atol=0)
    rng = np.random.default_rng(2)
    pos = rng.normal(0, 1.6, (20, 3))
    sp = (rng.random(20) < 0.4).astype(np.int32)
    B, dB, _ = s.descriptors(pos, sp, np.full(3, np.inf))
    R = Rotation.random(random_state=7).as_matrix()
    B2, _, _ = s.descriptors(pos @ R.T, sp, np.full(3, np.inf))
    assert np.abs(B2 - B).max() <= 1e-12 * np.abs(B).max()
    beta = rng.normal(0, 1e-2, (2, s.K))
    e, f, w = s.energy_forces(pos, sp, np.full(3, np.inf), beta, 0.3)
    ea, fa, wa = s.energy_forces(pos, sp, np.full(3, np.inf), beta, 0.3, mode="adjoint")
    assert abs(e - ea) <= 1e-13 * abs(e)
    assert np.abs(f - fa).max() <= 1e-13 * np.abs(f).max()
    assert np.abs(f.sum(0)).max() <= 1e-13 * np.abs(f).max()
    h = 1e-5
    for a, c in [(0, 0), (5, 1), (13, 2)]:
        pp = pos.copy(); pp[a, c] += h
        pm = pos.copy(); pm[a, c] -= h
        fd = -(s.energy_forces(pp, sp, np.full(3, np.inf), beta)[0] - s.energy_forces(pm, sp, np.full(3, np.inf), beta)[0]) / (2 * h)
        assert abs(fd - f[a, c]) <= 1e-7 * np.abs(f).max()


def test_snap_literal_radius_finds_no_neighbors():
    """utl.jl:81 taken literally searches within sqrt(cutmax): nothing on the configs."""
    s, prm, _ = W.snap_j8(cells=3)
    sp = np.array([prm["species"].index(x) for x in s.symbols], np.int32)
    off, j, r = oracle.nlist_snap(s.positions, s.L, sp, prm["radii"], prm["rcutfac"], literal_sqrt=True)
    assert len(j) == 0
    off, j, r = oracle.nlist_snap(s.positions, s.L, sp, prm["radii"], prm["rcutfac"], literal_sqrt=False)
    assert 20 < np.diff(off).mean() < 30


# ---- chem_flag and quadratic SNAP (oracle known answers; no reference values exist) ------
def _cluster(seed, n=24, nsp=2):
    rng = np.random.default_rng(seed)
    pos = rng.normal(0, 1.6, (n, 3))
    sp = rng.integers(0, nsp, n).astype(np.int32)
    return pos, sp


@pytest.mark.parametrize("bzero", [False, True])
def test_chem_components_sum_to_single_element_descriptors(bzero):
    """With chem_flag the element-resolved Utot of an atom sum to the single-element Utot (wself
    once, on the centre's element), Z is bilinear and B trilinear in them, so B and dB summed
    over all element triples equal the single-element B and dB with the same bnorm (and the
    bzero shift, taken once on the centre's triple)."""
    J = 6
    pos, sp = _cluster(31)
    L = np.full(3, np.inf)
    kw = dict(rmin0=0.0, rfac0=0.99363, switch=True, bzero=bzero, bnorm=True)
    one = oracle.Snap(J, [0.5, 0.45], [1.0, 0.6], 2.2, **kw)
    chem = oracle.Snap(J, [0.5, 0.45], [1.0, 0.6], 2.2, chem=True, **kw)
    K = one.K
    assert chem.K == 8 * K
    B1, dB1, W1 = one.descriptors(pos, sp, L)
    Bc, dBc, Wc = chem.descriptors(pos, sp, L)
    Bsum = Bc.reshape(len(pos), 8, K).sum(axis=1)
    assert np.abs(Bsum - B1).max() <= 1e-12 * np.abs(B1).max()
    # dB [n][K*nsp][3]: the species blocks keep their order, the triples sum inside each block
    dsum = dBc.reshape(len(pos), 2, 8, K, 3).sum(axis=2).reshape(len(pos), 2 * K, 3)
    assert np.abs(dsum - dB1).max() <= 1e-12 * np.abs(dB1).max()
    wsum = Wc.reshape(2, 8, K, 6).sum(axis=1).reshape(2 * K, 6)
    assert np.abs(wsum - W1).max() <= 1e-12 * np.abs(W1).max()


def test_chem_single_species_equals_plain_bnorm():
    """One species: the chem_flag descriptors are the single-element ones."""
    pos, _ = _cluster(32)
    sp = np.zeros(len(pos), np.int32)
    L = np.full(3, np.inf)
    a = oracle.Snap(8, [0.5], [1.0], 2.0, switch=True, bnorm=True)
    b = oracle.Snap(8, [0.5], [1.0], 2.0, switch=True, bnorm=True, chem=True)
    Ba, dBa, _ = a.descriptors(pos, sp, L)
    Bb, dBb, _ = b.descriptors(pos, sp, L)
    assert np.array_equal(Ba, Bb) and np.array_equal(dBa, dBb)


def test_chem_literal_z_index():
    """compute_z.jl:19-20,44-47 taken literally: every element pair sums into the first Z block
    (the running sum divided by j+1 after each pair with bnorm) and the other blocks stay zero,
    so B of every triple whose element pair is not the first vanishes."""
    pos, sp = _cluster(33)
    L = np.full(3, np.inf)
    s = oracle.Snap(4, [0.5, 0.45], [1.0, 0.6], 2.2, switch=True, bnorm=True, chem=True, literal_chem_z=True)
    K = s.idxb_max
    B, _, _ = s.descriptors(pos, sp, L)
    B = B.reshape(len(pos), 4, 2, K)  # (elem1 elem2), elem3, component
    assert np.all(B[:, 1:] == 0.0)
    assert np.abs(B[:, 0]).max() > 0.0


def test_chem_forces_are_energy_gradient():
    pos, sp = _cluster(34, n=16)
    L = np.full(3, np.inf)
    s = oracle.Snap(6, [0.5, 0.45], [1.0, 0.6], 2.2, switch=True, bnorm=True, chem=True, bzero=True)
    beta = np.random.default_rng(3).normal(0, 1e-2, (2, s.K))
    e, f, _ = s.energy_forces(pos, sp, L, beta, 0.1)
    h = 1e-5
    for a, c in [(0, 0), (7, 2), (11, 1)]:
        pp = pos.copy(); pp[a, c] += h
        pm = pos.copy(); pm[a, c] -= h
        fd = -(s.energy_forces(pp, sp, L, beta)[0] - s.energy_forces(pm, sp, L, beta)[0]) / (2 * h)
        assert abs(fd - f[a, c]) <= 1e-7 * np.abs(f).max()


@pytest.mark.parametrize("chem", [False, True])
def test_quadratic_descriptors_and_forces(chem):
    """Quadratic SNAP: B is followed by 0.5 B_k^2 and B_k B_l (l > k); E = beta . B_ext, and the
    forces (through the per-atom effective linear coefficients) are -dE/dx."""
    pos, sp = _cluster(35, n=14)
    L = np.full(3, np.inf)
    kw = dict(switch=True, bnorm=chem, chem=chem)
    lin = oracle.Snap(4, [0.5, 0.45], [1.0, 0.6], 2.2, **kw)
    q = oracle.Snap(4, [0.5, 0.45], [1.0, 0.6], 2.2, quadratic=True, **kw)
    K = lin.K
    assert q.K == K + K * (K + 1) // 2
    Bl, dBl, _ = lin.descriptors(pos, sp, L)
    Bq, dBq, _ = q.descriptors(pos, sp, L)
    assert np.array_equal(Bq[:, :K], Bl)
    iu = np.triu_indices(K)
    outer = Bl[:, :, None] * Bl[:, None, :]
    outer[:, np.arange(K), np.arange(K)] *= 0.5
    assert np.abs(Bq[:, K:] - outer[:, iu[0], iu[1]]).max() <= 1e-14 * np.abs(Bq).max()
    beta = np.random.default_rng(4).normal(0, 1e-2, (2, q.K))
    e, f, _ = q.energy_forces(pos, sp, L, beta, 0.0)
    assert abs(e - np.einsum("ik,ik->", Bq, beta[sp])) <= 1e-12 * abs(e)
    # compute_all_descriptors' dB is -d(sum B)/dx per centre-species block, so F = dB . beta
    fd_b = np.einsum("ikc,k->ic", dBq[:, :q.K], beta[0]) + np.einsum("ikc,k->ic", dBq[:, q.K:], beta[1])
    assert np.abs(f - fd_b).max() <= 1e-12 * np.abs(f).max()
    h = 1e-5
    for a, c in [(0, 0), (9, 2)]:
        pp = pos.copy(); pp[a, c] += h
        pm = pos.copy(); pm[a, c] -= h
        fd = -(q.energy_forces(pp, sp, L, beta)[0] - q.energy_forces(pm, sp, L, beta)[0]) / (2 * h)
        assert abs(fd - f[a, c]) <= 1e-7 * np.abs(f).max()
