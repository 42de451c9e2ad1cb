"""ipg — B200-native (sm_100a, FP64) force-field evaluation with the API of
InteratomicPotentials.jl: pair potentials and their linear combinations, SNAP
descriptors, and the linear SNAP potential with plain and adjoint force paths.

All numerics run in libipg.so (CUDA); this package is the host-side mirror of the
reference's Julia API and has no CPU fallback.
"""
from ._lib import IPGError
from .api import (NeighborList, energy_and_force, force, neighborlist, neighborlist_snap, potential_energy,
                  virial, virial_stress)
from .context import Context, default_context
from .empirical import (ZBL, AbstractPotential, BornMayer, Coulomb, EmpiricalPotential, LennardJones,
                        LinearCombinationPotential, MockR2, Morse)
from .snap import (SNAP, DeviceBatch, LBasisPotential, compute_all_descriptors, compute_force_descriptors,
                   compute_local_descriptors, compute_virial_descriptors, get_num_snap_coeffs)
from .system import System, periodic_system
from . import units

__all__ = [
    "IPGError", "Context", "default_context", "System", "periodic_system", "units",
    "AbstractPotential", "EmpiricalPotential", "LennardJones", "BornMayer", "Coulomb", "Morse", "ZBL", "MockR2",
    "LinearCombinationPotential", "SNAP", "DeviceBatch", "LBasisPotential", "get_num_snap_coeffs",
    "compute_local_descriptors", "compute_force_descriptors", "compute_virial_descriptors",
    "compute_all_descriptors", "energy_and_force", "potential_energy", "force", "virial", "virial_stress",
    "neighborlist", "neighborlist_snap", "NeighborList",
]
