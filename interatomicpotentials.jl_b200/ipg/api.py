"""The InteratomicPotentials.jl API (src/api.jl:5-10) over the GPU library.

    energy_and_force(s, p) -> (e, f)      potential_energy(s, p) -> e
    force(s, p) -> f (n, 3)               virial_stress(s, p) -> (6,)   virial(s, p)
    neighborlist(s, rcut) -> NeighborList

Pair potentials return hartree and hartree/bohr (atomic units, src/unit_convention.jl);
SNAP potentials return values in the units implied by beta and the system's length unit.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import NLIST_HALF, WANT_E, WANT_F, WANT_W, lib
from .context import default_context
from .empirical import (EmpiricalPotential, EnergyAndForce, LinearCombinationPotential, empirical_terms,
                        pair_eval)
from .snap import LBasisPotential


def _is_empirical(p):
    if isinstance(p, EmpiricalPotential):
        return True
    if isinstance(p, LinearCombinationPotential):
        return all(isinstance(q, EmpiricalPotential) for _, q in p.flat_terms())
    return False


def _combo(f, s, p):
    """linear_combination_potential.jl:34 for mixed (non-empirical) combinations."""
    return sum(c * f(s, q) for c, q in p.flat_terms())


def energy_and_force(s, p):
    if _is_empirical(p):
        e, f, _ = pair_eval(s, empirical_terms(p), WANT_E | WANT_F)
        return EnergyAndForce(e, f)
    if isinstance(p, LBasisPotential):
        e, f, _ = p.basis.energy_forces(s, _beta(p), p.beta0[0], p.mode)
        return EnergyAndForce(e, f)
    if isinstance(p, LinearCombinationPotential):  # linear_combination_potential.jl:27-32
        efs = [(c, energy_and_force(s, q)) for c, q in p.flat_terms()]
        return EnergyAndForce(sum(c * ef.e for c, ef in efs), sum(c * ef.f for c, ef in efs))
    raise TypeError(f"no energy_and_force for {type(p).__name__}")


def potential_energy(s, p):
    if isinstance(p, LBasisPotential):  # basis_potentials.jl:14-21 (energy only)
        return _energy_only(s, p)[0]
    if _is_empirical(p):
        return pair_eval(s, empirical_terms(p), WANT_E)[0]
    if isinstance(p, LinearCombinationPotential):
        return _combo(potential_energy, s, p)
    return energy_and_force(s, p).e


def force(s, p):
    return energy_and_force(s, p).f


def virial_stress(s, p):
    """[xx, yy, zz, zy, zx, yx] (empirical_potential.jl:60-67); W.beta for SNAP."""
    if _is_empirical(p):
        return pair_eval(s, empirical_terms(p), WANT_W)[2]
    if isinstance(p, LBasisPotential):
        _, _, w = p.basis.energy_forces(s, _beta(p), p.beta0[0], p.mode)
        return w
    if isinstance(p, LinearCombinationPotential):
        return _combo(virial_stress, s, p)
    raise TypeError(f"no virial_stress for {type(p).__name__}")


def virial(s, p):
    """Trace of the virial stress (abstract_potential.jl:10).  For basis potentials the
    reference sums all six components (basis_potentials.jl:52-57); that is kept."""
    if isinstance(p, LBasisPotential):
        return float(np.sum(virial_stress(s, p)))
    if isinstance(p, LinearCombinationPotential) and not _is_empirical(p):
        return _combo(virial, s, p)
    return float(np.sum(virial_stress(s, p)[:3]))


def _beta(p):
    return p.basis.beta_blocks(p.beta)


def _energy_only(s, p):
    from .snap import compute_local_descriptors
    B = compute_local_descriptors(s, p.basis)
    sp = p.basis.species_ids(s)
    beta = _beta(p)
    e = p.beta0[0] + float(np.einsum("ik,ik->", B, beta[sp]))
    return e, None, None


class NeighborList:
    """src/nnlist.jl:5-14: j[n] (0-based neighbor ids > n) and r[n] (displacements)."""

    def __init__(self, offsets, j, r):
        self.offsets, self._j, self._r = offsets, j, r
        n = len(offsets) - 1
        self.j = [j[offsets[a]:offsets[a + 1]] for a in range(n)]
        self.r = [r[offsets[a]:offsets[a + 1]] for a in range(n)]

    def __len__(self):
        return len(self.j)


def neighborlist(s, rcutoff, ctx=None):
    """Half list within rcutoff (PeriodicEuclidean), r = x_n - x_m (src/nnlist.jl:23-46)."""
    return _nlist(s, np.array([float(rcutoff)]), None, 1, NLIST_HALF, ctx)


def neighborlist_snap(s, snap, ctx=None):
    """Full SNAP list (utl.jl:38-101), r = x_nb - x_n."""
    nsp = len(snap.species)
    cutsq = np.zeros((nsp, nsp))
    for a in range(nsp):
        for b in range(nsp):
            cutsq[a, b] = ((snap.radii[a] + snap.radii[b]) * snap.rcutfac) ** 2
    from ._lib import NLIST_FULL, NLIST_LITERAL_SQRT
    mode = NLIST_FULL | (NLIST_LITERAL_SQRT if snap.literal_sqrt_radius else 0)
    return _nlist(s, cutsq.ravel(), snap.species_ids(s), nsp, mode, ctx)


def neighbor_count(s, rcut, ctx=None):
    """Number of half pairs within rcut (the size of neighborlist(s, rcut)) without building it."""
    ctx = ctx or default_context()
    vp = lambda a: a.ctypes.data_as(C.c_void_p)
    cut = np.array([float(rcut)])
    out = C.c_int64()
    ctx.check(lib().ipg_neighbor_count(ctx.handle, len(s), vp(s.positions), vp(s.L), None, 1, vp(cut), 0,
                                       C.byref(out)))
    return out.value


def _nlist(s, cut, species, nsp, mode, ctx):
    ctx = ctx or default_context()
    vp = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)
    h = C.c_void_p()
    n = len(s)
    ctx.check(lib().ipg_neighbor_build(ctx.handle, n, vp(s.positions), vp(s.L), vp(species), nsp, vp(cut), mode,
                                       C.byref(h)))
    try:
        np_ = C.c_int64()
        ctx.check(lib().ipg_nlist_size(h, C.byref(np_)))
        off = np.zeros(n + 1, np.int64)
        j = np.zeros(max(1, np_.value), np.int32)
        r = np.zeros((max(1, np_.value), 3))
        ctx.check(lib().ipg_nlist_export(h, vp(off), vp(j), vp(r)))
    finally:
        lib().ipg_nlist_free(h)
    return NeighborList(off, j[:np_.value], r[:np_.value])
