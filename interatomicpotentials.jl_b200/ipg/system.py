"""A minimal AtomsBase-like system: positions, atomic symbols, orthorhombic box, periodicity.

Only what the hot path reads from an ``AbstractSystem`` is kept: ``position``,
``atomic_symbol``, the box diagonal ``bounding_box(s)[i][i]`` and ``periodicity``
(src/nnlist.jl:25-29, src/BasisSystems/SNAP/utilities/utl.jl:60-64).
"""
from __future__ import annotations

import numpy as np


class System:
    def __init__(self, positions, symbols, box, periodic=(True, True, True)):
        """positions: (n, 3); symbols: n atomic symbols (str) or ints; box: 3 lengths or a
        3x3 matrix of which only the diagonal is used; periodic: 3 booleans."""
        self.positions = np.ascontiguousarray(np.asarray(positions, dtype=np.float64).reshape(-1, 3))
        self.symbols = tuple(symbols)  # immutable, so that the per-species index below can be cached
        if len(self.symbols) != len(self.positions):
            raise ValueError("one symbol per atom is required")
        b = np.asarray(box, dtype=np.float64)
        self.box = np.diag(b).copy() if b.ndim == 2 else b.reshape(3).copy()
        self.periodic = tuple(bool(p) for p in periodic)

    def __len__(self):
        return len(self.positions)

    @property
    def L(self):
        """Box diagonal with +inf on open axes (src/nnlist.jl:29)."""
        return np.array([self.box[a] if self.periodic[a] else np.inf for a in range(3)], dtype=np.float64)

    def atomic_symbol(self):
        return list(self.symbols)

    def unique_symbols(self):
        """The distinct symbols in order of first appearance."""
        u = getattr(self, "_unique", None)
        if u is None:
            u = self._unique = list(dict.fromkeys(self.symbols))
        return list(u)

    def species_index(self, species):
        """int32 index of each atom's symbol in `species` (KeyError for a symbol not in it),
        computed once per species list."""
        key = tuple(species)
        cache = self.__dict__.setdefault("_species_index", {})
        arr = cache.get(key)
        if arr is None:
            lut = {s: k for k, s in enumerate(key)}
            arr = np.fromiter((lut[s] for s in self.symbols), dtype=np.int32, count=len(self.symbols))
            arr.flags.writeable = False
            cache[key] = arr
        return arr


def periodic_system(positions, symbols, box):
    return System(positions, symbols, box, (True, True, True))
