"""ipg_pair_eval_noalloc: the pair evaluation for callers that cannot allocate.

Callers such as an MD engine that owns all device memory, or a host that holds only a
stream and device buffers, cannot let the library call cudaMalloc (or create a context,
which allocates).  ipg_pair_eval_noalloc keeps its scratch in a fixed device array; this
test calls it through the C ABI on device buffers that the test allocates beforehand and
checks it against ipg_pair_eval_dev, on two calls in a row (the second reuses the shared
scratch left by the first), and against the oracle.  It lives in its own file, collected last.
"""
import ctypes as C

import numpy as np
import pytest

import ipg
import oracle
from ipg import workloads as W
from ipg._lib import IPG_OK, PairTerm, lib
from conftest import TOL, rel_err

pytestmark = pytest.mark.gpu


def _device_case(torch, system, pot):
    idx = {s: k for k, s in enumerate(system.unique_symbols())}
    terms = ipg.empirical.empirical_terms(pot)
    arr = (PairTerm * len(terms))()
    for q, (c, p) in enumerate(terms):
        arr[q] = p.term(idx, c)
    pos = torch.tensor(system.positions, device="cuda")
    sp = torch.tensor(np.array([idx[s] for s in system.symbols], np.int32), device="cuda")
    return arr, len(terms), pos, sp


def _oracle(system, pot):
    idx = {x: k for k, x in enumerate(system.unique_symbols())}
    terms = []
    for c, p in ipg.empirical.empirical_terms(pot):
        t = p.term(idx, c)
        terms.append(dict(kind=t.kind, coeff=c, rcut=p.rcutoff, mask=int(t.species_mask), params=list(t.params)))
    return oracle.pair_eval(system.positions, np.array([idx[x] for x in system.symbols], np.int32), system.L, terms)


@pytest.mark.parametrize("case", ["lj1000", "lc_small", "open", "sparse", "outlier"])
def test_noalloc_matches_dev_entry_point(case):
    """Against ipg_pair_eval_dev and the oracle.  "sparse" (500 atoms in a 1000-bohr periodic
    box, cutoff 6) and "outlier" (an open cluster with one atom far away) need more cells than
    the fixed array holds, so the grid is coarsened before the walk."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(3)
    if case == "lj1000":
        s, p = W.lj1000()
    elif case == "lc_small":
        s, p = W.lc32000(cells=8)
    elif case == "open":
        s = ipg.System(rng.uniform(0, 25, (500, 3)), ["Ar"] * 500, [25.0] * 3, (True, False, True))
        p = ipg.LennardJones(0.01, 3.0, 6.0, ["Ar"]) + ipg.Morse(0.1, 1.0, 3.0, 5.0, ["Ar"])
    elif case == "sparse":
        s = ipg.System(rng.uniform(0, 1000, (500, 3)), ["Ar"] * 500, [1000.0] * 3)
        p = ipg.LennardJones(0.01, 3.0, 6.0, ["Ar"])
    else:
        pos = rng.uniform(0, 30, (800, 3))
        pos[17] = [5000.0, -4000.0, 9000.0]
        s = ipg.System(pos, ["Ar"] * 800, [np.inf] * 3, (False, False, False))
        p = ipg.LennardJones(0.01, 3.0, 6.0, ["Ar"])
    arr, nt, pos, sp = _device_case(torch, s, p)
    n = len(s)
    L = s.L
    vp = C.c_void_p
    # reference results from the existing device entry point
    ctx = ipg.default_context()
    E0 = torch.zeros(1, dtype=torch.float64, device="cuda")
    F0 = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    W0 = torch.zeros(6, dtype=torch.float64, device="cuda")
    ctx.check(lib().ipg_pair_eval_dev(ctx.handle, n, vp(pos.data_ptr()), vp(sp.data_ptr()), L.ctypes.data_as(vp),
                                      C.cast(arr, vp), nt, vp(E0.data_ptr()), vp(F0.data_ptr()), vp(W0.data_ptr()), 7))
    e0, f0, w0 = E0.item(), F0.cpu().numpy(), W0.cpu().numpy()
    stream = torch.cuda.current_stream()
    for call in range(2):  # two calls in a row share the scratch array
        E = torch.full((1,), np.nan, dtype=torch.float64, device="cuda")
        F = torch.full((n, 3), np.nan, dtype=torch.float64, device="cuda")
        Wv = torch.full((6,), np.nan, dtype=torch.float64, device="cuda")
        st = lib().ipg_pair_eval_noalloc(vp(stream.cuda_stream), n, vp(pos.data_ptr()), vp(sp.data_ptr()),
                                         L.ctypes.data_as(vp), C.cast(arr, vp), nt, vp(E.data_ptr()),
                                         vp(F.data_ptr()), vp(Wv.data_ptr()), 7)
        assert st == IPG_OK
        torch.cuda.synchronize()
        assert abs(E.item() - e0) <= TOL * abs(e0), call
        assert rel_err(F.cpu().numpy(), f0) <= TOL, call
        assert rel_err(Wv.cpu().numpy(), w0) <= TOL, call
    eo, fo, wo = _oracle(s, p)
    assert abs(E.item() - eo) <= TOL * abs(eo)
    assert rel_err(F.cpu().numpy(), fo) <= TOL
    assert rel_err(Wv.cpu().numpy(), wo) <= TOL


def test_noalloc_empty_system():
    """n = 0: E and the virial are zero, nothing else is touched."""
    torch = pytest.importorskip("torch")
    vp = C.c_void_p
    arr = (PairTerm * 1)()
    arr[0] = ipg.LennardJones(0.01, 3.0, 6.0, ["Ar"]).term({"Ar": 0})
    L = np.array([10.0, 10.0, 10.0])
    E = torch.full((1,), np.nan, dtype=torch.float64, device="cuda")
    Wv = torch.full((6,), np.nan, dtype=torch.float64, device="cuda")
    st = lib().ipg_pair_eval_noalloc(None, 0, None, None, L.ctypes.data_as(vp), C.cast(arr, vp), 1,
                                     vp(E.data_ptr()), None, vp(Wv.data_ptr()), 5)
    assert st == IPG_OK
    torch.cuda.synchronize()
    assert E.item() == 0.0 and np.all(Wv.cpu().numpy() == 0.0)


def test_noalloc_rejects_too_many_atoms():
    torch = pytest.importorskip("torch")
    vp = C.c_void_p
    n = 65537
    pos = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    sp = torch.zeros(n, dtype=torch.int32, device="cuda")
    arr = (PairTerm * 1)()
    arr[0] = ipg.LennardJones(0.01, 3.0, 6.0, ["Ar"]).term({"Ar": 0})
    L = np.array([100.0, 100.0, 100.0])
    E = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = lib().ipg_pair_eval_noalloc(None, n, vp(pos.data_ptr()), vp(sp.data_ptr()), L.ctypes.data_as(vp),
                                     C.cast(arr, vp), 1, vp(E.data_ptr()), None, None, 1)
    assert st == -4  # IPG_ERR_CAPACITY
