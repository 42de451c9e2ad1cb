"""GPU neighbor lists vs the oracle and the reference's golden list (test/unit/nnlist.jl).

Pair sets must be identical (bit-exact indices) and displacements bit-identical: the
kernels use the reference's minimum-image arithmetic without contraction.
"""
import numpy as np
import pytest

import oracle
import ipg
from ipg import workloads as W

pytestmark = pytest.mark.gpu


def as_pairs(off, j):
    i = np.repeat(np.arange(len(off) - 1), np.diff(off))
    return np.stack([i, j], 1)


def test_golden_nnlist(golden):
    s = ipg.System(golden["nnlist_pos"], ["Ar"] * 3, golden["nnlist_box"], golden["nnlist_periodic"])
    nl = ipg.neighborlist(s, float(golden["nnlist_rcut"]))
    assert len(nl) == len(s)
    cnt = [len(x) for x in nl.j]
    assert cnt == golden["nnlist_true_j_count"].tolist()
    assert np.concatenate(nl.j).tolist() == golden["nnlist_true_j_flat"].tolist()
    np.testing.assert_allclose(np.concatenate(nl.r), golden["nnlist_true_r"], rtol=0, atol=1e-14)


@pytest.mark.parametrize("case", ["lj1000", "lc_small", "open_mixed", "tiny_box", "empty", "single"])
def test_half_list_matches_oracle(case):
    rng = np.random.default_rng(11)
    if case == "lj1000":
        s, p = W.lj1000()
        rc = p.rcutoff
    elif case == "lc_small":
        s, p = W.lc32000(cells=8)
        rc = p.get_rcutoff()
    elif case == "open_mixed":  # atoms outside the box on periodic axes, one open axis
        pos = rng.uniform(-30, 60, (700, 3))
        s = ipg.System(pos, ["Ar"] * len(pos), [25.0, 30.0, 40.0], (True, False, True))
        rc = 6.0
    elif case == "tiny_box":  # fewer than three cells per axis, rcut > L/2
        pos = rng.uniform(0, 7, (60, 3))
        s = ipg.System(pos, ["Ar"] * len(pos), [7.0, 7.0, 7.0], (True, True, True))
        rc = 5.0
    elif case == "empty":
        s = ipg.System(np.zeros((0, 3)), [], [5.0, 5.0, 5.0])
        rc = 2.0
    else:
        s = ipg.System(np.zeros((1, 3)), ["Ar"], [5.0, 5.0, 5.0])
        rc = 2.0
    nl = ipg.neighborlist(s, rc)
    off, j, r = oracle.nlist_half(s.positions, s.L, rc)
    assert np.array_equal(nl.offsets, off)
    assert np.array_equal(nl._j, j)
    assert np.array_equal(nl._r, r)  # bitwise


@pytest.mark.parametrize("literal", [False, True])
def test_snap_full_list_matches_oracle(literal):
    s, prm, _ = W.snap_j8(cells=6)
    snap = ipg.SNAP(len(s), prm["twojmax"], prm["species"], prm["rcutfac"], prm["rmin0"], prm["rfac0"],
                    prm["radii"], prm["weight"], switch_flag=True, literal_sqrt_radius=literal)
    nl = ipg.neighborlist_snap(s, snap)
    off, j, r = oracle.nlist_snap(s.positions, s.L, snap.species_ids(s), prm["radii"], prm["rcutfac"], literal)
    assert np.array_equal(nl.offsets, off)
    assert np.array_equal(nl._j, j)
    assert np.array_equal(nl._r, r)
    if literal:  # sqrt(cutmax) = sqrt(5) A < nearest neighbor (utl.jl:81 taken literally)
        assert len(j) == 0
    else:
        assert np.diff(off).mean() > 20


def test_nonfinite_positions_rejected():
    pos = np.zeros((4, 3))
    pos[2, 1] = np.nan
    s = ipg.System(pos, ["Ar"] * 4, [5.0, 5.0, 5.0])
    with pytest.raises(ipg.IPGError) as e:
        ipg.neighborlist(s, 1.0)
    assert e.value.status == -6


def test_neighbor_count_matches_built_list():
    from ipg import workloads as W
    s1, p1 = W.lj1000()
    s2, p2 = W.lc32000(cells=6)
    for s, rc in ((s1, p1.get_rcutoff()), (s2, p2.get_rcutoff())):
        assert ipg.api.neighbor_count(s, rc) == len(ipg.neighborlist(s, rc)._j)


def test_single_walk_padded_slots_and_overflow():
    """After a first build (two walks: count, then emit) a list of the same name is built in one
    walk into padded per-atom slots sized from the previous maximum, then compacted; a denser
    system than the slots allow falls back to the emit walk.  Every build equals the oracle."""
    ctx = ipg.Context(0)
    rng = np.random.default_rng(5)
    dense = ipg.System(rng.uniform(0, 20, (1500, 3)), ["Ar"] * 1500, [20.0] * 3)
    sparse = ipg.System(rng.uniform(0, 40, (900, 3)), ["Ar"] * 900, [40.0] * 3)
    rc = 4.0
    for s in (dense, dense, sparse, dense, dense, sparse):
        nl = ipg.neighborlist(s, rc, ctx=ctx)
        off, j, r = oracle.nlist_half(s.positions, s.L, rc)
        assert np.array_equal(nl.offsets, off)
        assert np.array_equal(nl._j, j)
        assert np.array_equal(nl._r, r)
