"""GPU pair potentials vs the reference's golden values and the oracle (FP64, 1e-10 rel)."""
import numpy as np
import pytest

import oracle
import ipg
from ipg import units
from ipg import workloads as W
from conftest import TOL, rel_err

pytestmark = pytest.mark.gpu


def oracle_terms(system, pot):
    idx = {s: k for k, s in enumerate(system.unique_symbols())}
    out = []
    for c, p in ipg.empirical.empirical_terms(pot):
        t = p.term(idx, c)
        out.append(dict(kind=t.kind, coeff=c, rcut=p.rcutoff, mask=int(t.species_mask), params=list(t.params)))
    return out


def oracle_eval(system, pot):
    idx = {s: k for k, s in enumerate(system.unique_symbols())}
    sp = np.array([idx[s] for s in system.symbols], np.int32)
    return oracle.pair_eval(system.positions, sp, system.L, oracle_terms(system, pot))


def test_mock_potential_exact(golden):
    """test/unit/types/empirical_potential.jl with test/mocks.jl: exact values."""
    s = ipg.periodic_system(golden["mock_pos"], list(golden["mock_symbols"]), golden["mock_box"])
    p = ipg.MockR2(float(golden["mock_seed"]), float(golden["mock_rcut"]), tuple(golden["mock_species"]))
    ef = ipg.energy_and_force(s, p)
    assert ef.e == float(golden["mock_e"])
    assert np.array_equal(ef.f, golden["mock_f"])
    assert np.array_equal(ipg.virial_stress(s, p), golden["mock_virial"])


@pytest.mark.parametrize("n", [150, 1000])
def test_lj_cluster_golden(golden, n):
    """test/integration/lj_clusters/lj_{150,1000}.jl: open boundaries, rcut 100 A."""
    A, eV = units.angstrom, units.eV
    pos = golden[f"lj{n}_pos"] * A
    s = ipg.System(pos, ["Ar"] * n, [8.0 * A] * 3, (False, False, False))
    p = ipg.LennardJones(float(golden[f"lj{n}_eps_eV"]) * eV, float(golden[f"lj{n}_sigma_A"]) * A,
                         float(golden[f"lj{n}_rcut_A"]) * A, ["Ar"])
    e, f = ipg.energy_and_force(s, p)
    e_atol = float(golden[f"lj{n}_E_atol_eV"]) * eV
    f_atol = float(golden[f"lj{n}_F_atol_eVA"]) * eV / A
    assert abs(e - float(golden[f"lj{n}_E_eV"]) * eV) <= e_atol
    assert np.all(np.abs(f.sum(0)) <= f_atol)
    if n == 150:
        assert np.all(np.abs(f) <= f_atol)
        assert abs(ipg.virial(s, p)) <= e_atol
    eo, fo, wo = oracle_eval(s, p)
    assert abs(e - eo) <= TOL * abs(eo)


def check_vs_oracle(s, p):
    e, f = ipg.energy_and_force(s, p)
    w = ipg.virial_stress(s, p)
    eo, fo, wo = oracle_eval(s, p)
    assert abs(e - eo) <= TOL * max(abs(eo), 1e-300), (e, eo)
    assert rel_err(f, fo) <= TOL
    assert rel_err(w, wo) <= TOL


def test_lj1000_config():
    s, p = W.lj1000()
    check_vs_oracle(s, p)


def test_lc_config_small():
    s, p = W.lc32000(cells=10)
    check_vs_oracle(s, p)


@pytest.mark.parametrize("zbl_e", [W.EULER_E, 1.0])
def test_lc_config_full(zbl_e):
    s, p = W.lc32000(zbl_e=zbl_e)
    check_vs_oracle(s, p)


@pytest.mark.parametrize("kind", ["LJ", "BM", "COUL", "MORSE", "ZBL"])
def test_each_kind_mixed_boundaries(kind):
    rng = np.random.default_rng(7)
    pos = rng.uniform(0, 20, (400, 3))
    sym = list(np.where(rng.random(400) < 0.6, "Ar", "Xe"))
    s = ipg.System(pos, sym, [20.0, 20.0, 20.0], (True, False, True))
    rc = 6.0
    p = {"LJ": ipg.LennardJones(0.01, 3.0, rc, ["Ar", "Xe"]),
         "BM": ipg.BornMayer(2.0, 0.5, 1.0, 0.8, 0.7, rc, ["Ar"]),
         "COUL": ipg.Coulomb(1.0, -1.0, rc, ["Xe"]),
         "MORSE": ipg.Morse(0.1, 1.2, 3.0, rc, ["Ar", "Xe"]),
         "ZBL": ipg.ZBL(18, 54, W.EULER_E, rc, ["Ar", "Xe"])}[kind]
    check_vs_oracle(s, p)


def test_species_filter_and_coefficients():
    """A term over (Ar, Xe) hits Ar-Ar, Xe-Xe and Ar-Xe (empirical_potential.jl:26-43)."""
    rng = np.random.default_rng(8)
    pos = rng.uniform(0, 15, (300, 3))
    sym = list(np.where(rng.random(300) < 0.5, "Ar", "Xe"))
    s = ipg.System(pos, sym, [15.0] * 3)
    a = ipg.LennardJones(0.01, 3.0, 5.0, ["Ar"])
    b = ipg.LennardJones(0.02, 3.5, 6.0, ["Ar", "Xe"])
    c = ipg.Morse(0.1, 1.0, 3.0, 4.0, ["He"])  # species absent from the system: no pairs
    p = 2.0 * a - b / 4.0 + c
    check_vs_oracle(s, p)
    e_sum = 2.0 * ipg.potential_energy(s, a) - 0.25 * ipg.potential_energy(s, b) + ipg.potential_energy(s, c)
    assert abs(ipg.potential_energy(s, p) - e_sum) <= 1e-12 * abs(e_sum)


def test_deterministic():
    s, p = W.lc32000(cells=8)
    e1, f1 = ipg.energy_and_force(s, p)
    e2, f2 = ipg.energy_and_force(s, p)
    assert e1 == e2 and np.array_equal(f1, f2)


def test_fd_lj():
    """LJ force is the gradient of its energy (central differences)."""
    s, p = W.lj1000()
    pos0 = s.positions.copy()
    _, f = ipg.energy_and_force(s, p)
    h = 1e-5
    for a, c in [(0, 0), (17, 1), (500, 2)]:
        pp = pos0.copy(); pp[a, c] += h
        pm = pos0.copy(); pm[a, c] -= h
        ep = ipg.potential_energy(ipg.System(pp, s.symbols, s.box), p)
        em = ipg.potential_energy(ipg.System(pm, s.symbols, s.box), p)
        assert abs(-(ep - em) / (2 * h) - f[a, c]) <= 1e-6 * np.abs(f).max()


def test_dev_entry_point_with_torch():
    torch = pytest.importorskip("torch")
    s, p = W.lj1000()
    ctx = ipg.default_context()
    pos = torch.tensor(s.positions, device="cuda")
    sp = torch.zeros(len(s), dtype=torch.int32, device="cuda")
    E = torch.zeros(1, dtype=torch.float64, device="cuda")
    F = torch.zeros((len(s), 3), dtype=torch.float64, device="cuda")
    Wv = torch.zeros(6, dtype=torch.float64, device="cuda")
    import ctypes as C
    terms = (ipg._lib.PairTerm * 1)()
    terms[0] = p.term({"Ar": 0})
    L = s.L
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    try:
        ctx.check(ipg._lib.lib().ipg_pair_eval_dev(ctx.handle, len(s), C.c_void_p(pos.data_ptr()),
                                                   C.c_void_p(sp.data_ptr()), L.ctypes.data_as(C.c_void_p),
                                                   C.cast(terms, C.c_void_p), 1, C.c_void_p(E.data_ptr()),
                                                   C.c_void_p(F.data_ptr()), C.c_void_p(Wv.data_ptr()), 7))
    finally:
        ctx.set_stream(None)
    e, f = ipg.energy_and_force(s, p)
    assert abs(E.item() - e) <= 1e-13 * abs(e)
    assert rel_err(F.cpu().numpy(), f) <= 1e-13


@pytest.mark.parametrize("case", ["dense_cells", "mixed_boundaries", "two_cells_periodic", "open_cluster",
                                  "empty_cells"])
@pytest.mark.parametrize("full", ["0", "1"])
def test_half_and_full_stencil_paths(case, full, monkeypatch):
    """The half-stencil tiles (each pair once; every periodic axis with >= 3 cells) and the
    full-stencil walk (IPG_PAIR_FULL=1, and the fallback for fewer cells) against the oracle:
    cells of more than 32 atoms (several tiles per cell pair), open and periodic axes mixed,
    2 cells on a periodic axis, one open cell, and a sparse gas with empty cells."""
    monkeypatch.setenv("IPG_PAIR_FULL", full)
    ctx = ipg.Context(0)
    rng = np.random.default_rng(77)
    if case == "dense_cells":  # ~74 atoms per cell
        s = ipg.System(rng.uniform(0, 12, (2000, 3)), list(np.where(rng.random(2000) < 0.5, "Ar", "Xe")), [12.0] * 3)
        p = ipg.LennardJones(0.01, 1.0, 4.0, ["Ar"]) + ipg.Morse(0.1, 1.0, 1.5, 3.5, ["Ar", "Xe"])
    elif case == "mixed_boundaries":
        s = ipg.System(rng.uniform(0, 30, (900, 3)), list(np.where(rng.random(900) < 0.5, "Ar", "Xe")),
                       [30.0, 30.0, 30.0], (True, False, True))
        p = ipg.LennardJones(0.01, 3.0, 6.0, ["Ar", "Xe"]) + ipg.ZBL(18, 54, W.EULER_E, 5.0, ["Ar", "Xe"])
    elif case == "two_cells_periodic":
        s = ipg.System(rng.uniform(0, 10, (300, 3)), ["Ar"] * 300, [10.0, 30.0, 30.0])
        p = ipg.LennardJones(0.01, 2.0, 4.5, ["Ar"])
    elif case == "open_cluster":
        s = ipg.System(rng.normal(0, 3, (200, 3)), ["Ar"] * 200, [10.0] * 3, (False, False, False))
        p = ipg.BornMayer(2.0, 0.5, 1.0, 0.8, 0.7, 50.0, ["Ar"])
    else:
        s = ipg.System(rng.uniform(0, 200, (300, 3)), ["Ar"] * 300, [200.0] * 3)
        p = ipg.LennardJones(0.01, 3.0, 12.0, ["Ar"])
    e, f, w = ipg.empirical.pair_eval(s, ipg.empirical.empirical_terms(p), ctx=ctx)
    eo, fo, wo = oracle_eval(s, p)
    assert abs(e - eo) <= TOL * max(abs(eo), 1e-300), (e, eo)
    assert rel_err(f, fo) <= TOL
    assert rel_err(w, wo) <= TOL


def test_dev_graph_replay():
    """IPG_PAIR_GRAPH: the first call captures, later calls with the same buffers replay one
    graph (no library launches) and give the eager results bit for bit, also after the
    positions change in place; another box length captures anew."""
    torch = pytest.importorskip("torch")
    import ctypes as C
    s, p = W.lc32000(cells=8)
    ctx = ipg.Context(0)
    idx = {sym: k for k, sym in enumerate(s.unique_symbols())}
    terms = ipg.empirical.empirical_terms(p)
    arr = (ipg._lib.PairTerm * len(terms))()
    for q, (c, pp) in enumerate(terms):
        arr[q] = pp.term(idx, c)
    n = len(s)
    pos = torch.tensor(s.positions, device="cuda")
    sp = torch.tensor(np.array([idx[x] for x in s.symbols], np.int32), device="cuda")
    out = [torch.zeros(k, dtype=torch.float64, device="cuda") for k in (1, 3 * n, 6)]
    vp = C.c_void_p

    def call(L, flags):
        ctx.check(ipg._lib.lib().ipg_pair_eval_dev(ctx.handle, n, vp(pos.data_ptr()), vp(sp.data_ptr()),
                                                   L.ctypes.data_as(vp), C.cast(arr, vp), len(terms),
                                                   vp(out[0].data_ptr()), vp(out[1].data_ptr()),
                                                   vp(out[2].data_ptr()), flags))
        torch.cuda.synchronize()
        return [t.cpu().numpy().copy() for t in out]

    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    try:
        L = s.L.copy()
        ref = call(L, 7)
        call(L, 7 | 8)  # eager + capture
        for step in range(3):
            l0 = ctx.launch_count()
            got = call(L, 7 | 8)
            assert ctx.launch_count() == l0  # one graph launch, no library kernel launches
            for a, b in zip(got, ref):
                assert np.array_equal(a, b)
            pos.add_(torch.tensor(np.random.default_rng(step).normal(0, 0.02, (n, 3)), device="cuda"))
            ref = call(L, 7)
        L2 = L * 1.01
        r2 = call(L2, 7)
        call(L2, 7 | 8)
        l0 = ctx.launch_count()
        assert all(np.array_equal(a, b) for a, b in zip(call(L2, 7 | 8), r2)) and ctx.launch_count() == l0
    finally:
        ctx.set_stream(None)
