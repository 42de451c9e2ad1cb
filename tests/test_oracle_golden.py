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
