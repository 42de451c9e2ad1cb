"""Atomic-unit conventions of the reference (src/unit_convention.jl:6-10, src/constants.jl).

Numbers handed to the pair potentials are in atomic units (hartree, bohr), which is
what the reference works in after ``austrip``.  Multiply by these factors to convert:

    LennardJones(1.0 * eV, 1.0 * angstrom, 100.0 * angstrom, ["Ar"])

Values follow CODATA 2018, the constants UnitfulAtomic.jl is built on.
"""
BOHR_IN_ANGSTROM = 0.529177210903
HARTREE_IN_EV = 27.211386245988

hartree = 1.0
bohr = 1.0
eV = 1.0 / HARTREE_IN_EV          # hartree per eV
angstrom = 1.0 / BOHR_IN_ANGSTROM  # bohr per angstrom

k_e = 1.0                    # Coulomb constant in atomic units (src/constants.jl:7)
epsilon_0 = 1.0 / (4.0 * 3.141592653589793)  # src/constants.jl:13
