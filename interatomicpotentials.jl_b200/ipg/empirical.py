"""Empirical pair potentials and their linear combinations, evaluated on the GPU.

Mirrors src/empirical/*.jl and src/mixed/linear_combination_potential.jl: the same
types, parameter names, cutoffs and species filters.  Every evaluation of an
EmpiricalPotential or of a LinearCombinationPotential of them is ONE call of
``ipg_pair_eval`` (all terms fused, one neighbor walk at the largest cutoff).
Parameters are in atomic units (see ipg.units), as after ``austrip`` in the reference
constructors.
"""
from __future__ import annotations

import ctypes as C
from collections import namedtuple

import numpy as np

from ._lib import MAX_PAIR_TERMS, PAIR_KIND, WANT_E, WANT_F, WANT_W, PairTerm, lib
from .context import default_context

EnergyAndForce = namedtuple("EnergyAndForce", ["e", "f"])
ALL_SPECIES = (1 << 64) - 1


class AbstractPotential:
    """Root of the potential hierarchy (src/types.jl)."""

    def get_rcutoff(self):
        return np.inf  # src/types/abstract_potential.jl:4

    def get_species(self):
        return None  # `missing`

    # algebra of src/mixed/linear_combination_potential.jl:14-22
    def __add__(self, other):
        return LinearCombinationPotential.of(self) + LinearCombinationPotential.of(other)

    def __sub__(self, other):
        return self + (-1.0) * other

    def __neg__(self):
        return (-1.0) * self

    def __pos__(self):
        return 1.0 * self

    def __rmul__(self, a):
        return LinearCombinationPotential.of(self).scaled(float(a))

    def __truediv__(self, a):
        return (1.0 / a) * self


class EmpiricalPotential(AbstractPotential):
    kind = None

    def __init__(self, rcutoff, species):
        self.rcutoff = float(rcutoff)
        self.species = tuple(species) if species is not None else None

    def get_rcutoff(self):
        return self.rcutoff

    def get_species(self):
        return self.species

    def params(self):
        raise NotImplementedError

    def get_parameters(self):
        return {}

    def term(self, symbols_index, coeff=1.0):
        t = PairTerm()
        t.kind = PAIR_KIND[self.kind]
        t.coeff = coeff
        t.rcut = self.rcutoff
        if self.species is None:
            t.species_mask = ALL_SPECIES
        else:
            m = 0
            for s in self.species:
                if s in symbols_index:
                    m |= 1 << symbols_index[s]
            t.species_mask = m
        p = self.params()
        for k, v in enumerate(p):
            t.params[k] = float(v)
        return t


class LennardJones(EmpiricalPotential):
    """src/empirical/lj.jl:18-36: V = 4e((s/R)^12 - (s/R)^6)."""
    kind = "LJ"

    def __init__(self, epsilon, sigma, rcutoff, species):
        super().__init__(rcutoff, species)
        self.epsilon, self.sigma = float(epsilon), float(sigma)

    def params(self):
        return [self.epsilon, self.sigma]

    def get_parameters(self):
        return {"epsilon": self.epsilon, "sigma": self.sigma}


class BornMayer(EmpiricalPotential):
    """src/empirical/bm.jl:18-39: V = A exp((s-R)/rho) + (C/R)^6 - (D/R)^8 (force literal)."""
    kind = "BM"

    def __init__(self, A, rho, sigma, C, D, rcutoff, species):
        super().__init__(rcutoff, species)
        self.A, self.rho, self.sigma, self.C, self.D = map(float, (A, rho, sigma, C, D))

    def params(self):
        return [self.A, self.rho, self.sigma, self.C, self.D]

    def get_parameters(self):
        return {"A": self.A, "rho": self.rho, "sigma": self.sigma, "C": self.C, "D": self.D}


class Coulomb(EmpiricalPotential):
    """src/empirical/coulomb.jl:19-37: V = k_e q1 q2 / R."""
    kind = "COUL"

    def __init__(self, q1, q2, rcutoff, species):
        super().__init__(rcutoff, species)
        self.q1, self.q2 = float(q1), float(q2)

    def params(self):
        return [self.q1, self.q2]


class Morse(EmpiricalPotential):
    """src/empirical/morse.jl:18-39: V = D (1 - exp(-alpha (R - s)))^2 (force literal)."""
    kind = "MORSE"

    def __init__(self, D, alpha, sigma, rcutoff, species):
        super().__init__(rcutoff, species)
        self.D, self.alpha, self.sigma = float(D), float(alpha), float(sigma)

    def params(self):
        return [self.D, self.alpha, self.sigma]

    def get_parameters(self):
        return {"D": self.D, "alpha": self.alpha, "sigma": self.sigma}


class ZBL(EmpiricalPotential):
    """src/empirical/zbl.jl:9-36 (screening with base `e`, force literal)."""
    kind = "ZBL"

    def __init__(self, Z1, Z2, e, rcutoff, species):
        super().__init__(rcutoff, species)
        self.Z1, self.Z2, self.e = int(Z1), int(Z2), float(e)

    def params(self):
        return [float(self.Z1), float(self.Z2), self.e]


class MockR2(EmpiricalPotential):
    """The reference's MockEmpiricalPotential (test/mocks.jl:22-34): E = seed R^2, f = seed R^2 r."""
    kind = "MOCK_R2"

    def __init__(self, seed, rcutoff, species):
        super().__init__(rcutoff, species)
        self.seed = float(seed)

    def params(self):
        return [self.seed]


class LinearCombinationPotential(AbstractPotential):
    """src/mixed/linear_combination_potential.jl:7-39."""

    def __init__(self, potentials, coefficients):
        self.potentials = list(potentials)
        self.coefficients = [float(c) for c in coefficients]

    @staticmethod
    def of(p):
        if isinstance(p, LinearCombinationPotential):
            return p
        return LinearCombinationPotential([p], [1.0])

    def __add__(self, other):
        o = LinearCombinationPotential.of(other)
        return LinearCombinationPotential(self.potentials + o.potentials, self.coefficients + o.coefficients)

    def scaled(self, a):
        return LinearCombinationPotential(self.potentials, [a * c for c in self.coefficients])

    def __rmul__(self, a):
        return self.scaled(float(a))

    def __eq__(self, other):
        return (isinstance(other, LinearCombinationPotential) and self.potentials == other.potentials
                and self.coefficients == other.coefficients)

    def get_rcutoff(self):
        return max(p.get_rcutoff() for p in self.potentials)  # :24

    def get_species(self):
        return None  # :25 (missing)

    def flat_terms(self):
        """(coefficient, EmpiricalPotential) pairs, nested combinations expanded."""
        out = []
        for p, c in zip(self.potentials, self.coefficients):
            if isinstance(p, LinearCombinationPotential):
                out += [(c * cc, pp) for cc, pp in p.flat_terms()]
            else:
                out.append((c, p))
        return out


def _symbol_index(system):
    return {s: k for k, s in enumerate(system.unique_symbols())}


def pair_eval(system, terms, flags=WANT_E | WANT_F | WANT_W, ctx=None):
    """One fused ipg_pair_eval over [(coeff, EmpiricalPotential)] -> (E, F, W6)."""
    if len(terms) > MAX_PAIR_TERMS:
        raise ValueError(f"at most {MAX_PAIR_TERMS} pair terms per call")
    ctx = ctx or default_context()
    idx = _symbol_index(system)
    if len(idx) > 64:
        raise ValueError("at most 64 distinct species")
    sp = system.species_index(list(idx))
    arr = (PairTerm * max(1, len(terms)))()
    for k, (c, p) in enumerate(terms):
        arr[k] = p.term(idx, c)
    n = len(system)
    pos = system.positions
    L = system.L
    E = np.zeros(1)
    F = np.zeros((n, 3))
    W = np.zeros(6)
    vp = lambda a: a.ctypes.data_as(C.c_void_p)
    ctx.check(lib().ipg_pair_eval(ctx.handle, n, vp(pos), vp(sp), vp(L), C.cast(arr, C.c_void_p), len(terms),
                                  vp(E), vp(F), vp(W), flags))
    return E[0], F, W


def empirical_terms(p):
    if isinstance(p, EmpiricalPotential):
        return [(1.0, p)]
    if isinstance(p, LinearCombinationPotential):
        return p.flat_terms()
    raise TypeError(type(p))
