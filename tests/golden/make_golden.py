"""Generates tests/golden/reference_fixtures.npz from the reference's own test files.

    python tests/golden/make_golden.py /path/to/InteratomicPotentials.jl

The reference (cesmix-mit/InteratomicPotentials.jl) is Julia and cannot run here, so
its golden vectors are read from its test sources as text:
  test/unit/nnlist.jl                      3-atom half list with mixed boundaries
  test/unit/types/empirical_potential.jl   MockEmpiricalPotential E / F / virial
  test/integration/lj_clusters/{150,1000}.xyz and lj_{150,1000}.jl  LJ cluster energies
  test/SNAP/snap_test_{single,multi}_element.jl   3-atom SNAP inputs and parameters
Every number is parsed from those files; nothing is typed in by hand.
"""
import os
import re
import sys

import numpy as np

if len(sys.argv) != 2:
    sys.exit("usage: make_golden.py /path/to/InteratomicPotentials.jl")
REF = sys.argv[1]
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_fixtures.npz")

NUM = r"-?\d+(?:\.\d*)?(?:[eE][-+]?\d+)?"


def read(rel):
    with open(os.path.join(REF, rel)) as f:
        return f.read()


def vectors(text):
    return [[float(x) for x in re.findall(NUM, m)] for m in re.findall(r"\[([^\[\]]*)\]", text)]


def main():
    out = {}

    # ---- test/unit/nnlist.jl
    t = read("test/unit/nnlist.jl")
    atoms = re.findall(r"Atom\(:(\w+), \(@SVector \[([^\]]+)\]\)", t)
    out["nnlist_pos"] = np.array([[float(x) for x in a[1].split(",")] for a in atoms])
    box = re.search(r"box = \[(.*)\]u\"bohr\"", t).group(1)
    out["nnlist_box"] = np.array(vectors(box)).diagonal().copy()
    bcs = re.search(r"boundary_conditions = \[(.*)\]", t).group(1)
    out["nnlist_periodic"] = np.array([b.strip().startswith("Periodic") for b in bcs.split(",")])
    out["nnlist_rcut"] = np.array(float(re.search(r"rcutoff = (" + NUM + ")", t).group(1)))
    tj = re.search(r"true_j = \[(.*?)\n    \]", t, re.S).group(1)
    js = [[int(x) for x in re.findall(r"\d+", m)] for m in re.findall(r"Int\[([^\]]*)\]", tj)]
    out["nnlist_true_j_flat"] = np.array([j for row in js for j in row], dtype=np.int64) - 1  # 0-based
    out["nnlist_true_j_count"] = np.array([len(r) for r in js], dtype=np.int64)
    tr = re.search(r"true_r = \[(.*?)\n    \]", t, re.S).group(1)
    rows = re.findall(r"Vector\{Float64\}\[(.*?)\](?=,\n|\n)", tr)
    r_flat = []
    for row in rows:
        r_flat += vectors(row)
    out["nnlist_true_r"] = np.array(r_flat).reshape(-1, 3)

    # ---- test/unit/types/empirical_potential.jl (MockEmpiricalPotential, test/mocks.jl)
    t = read("test/unit/types/empirical_potential.jl")
    atoms = re.findall(r":(\w+) => \(@SVector \[([^\]]+)\]\)", t)
    out["mock_symbols"] = np.array([a[0] for a in atoms])
    out["mock_pos"] = np.array([[float(x) for x in a[1].split(",")] for a in atoms])
    out["mock_box"] = np.array(vectors(re.search(r"box = \[(.*)\]u\"bohr\"", t).group(1))).diagonal().copy()
    m = re.search(r"MockEmpiricalPotential\((" + NUM + "), (" + NUM + r"), \(:(\w+),\)\)", t)
    out["mock_seed"], out["mock_rcut"] = np.array(float(m.group(1))), np.array(float(m.group(2)))
    out["mock_species"] = np.array([m.group(3)])
    out["mock_e"] = np.array(float(re.search(r"\.e == (" + NUM + ")u", t).group(1)))
    fblock = re.search(r"\.f == \[(.*?)\n    \]", t, re.S).group(1)
    out["mock_f"] = np.array([[float(x) for x in v.split(",")] for v in re.findall(r"@SVector\[([^\]]+)\]", fblock)])
    vs = re.search(r"virial_stress\(system, p\) == \(@SVector\[([^\]]+)\]\)", t).group(1)
    out["mock_virial"] = np.array([float(x) for x in vs.split(",")])

    # ---- LJ clusters
    for n in (150, 1000):
        out[f"lj{n}_pos"] = np.loadtxt(os.path.join(REF, f"test/integration/lj_clusters/{n}.xyz"))
        t = read(f"test/integration/lj_clusters/lj_{n}.jl")
        out[f"lj{n}_E_eV"] = np.array(float(re.search(r"es ≈ auconvert\((" + NUM + r") \* 1u\"eV\"\)", t).group(1)))
        out[f"lj{n}_eps_eV"] = np.array(float(re.search(r"ϵ = (" + NUM + r")u\"eV\"", t).group(1)))
        out[f"lj{n}_sigma_A"] = np.array(float(re.search(r"σ = (" + NUM + r")u\"[^\"]+\"", t).group(1)))
        out[f"lj{n}_rcut_A"] = np.array(float(re.search(r"rcutoff = (" + NUM + r")u\"[^\"]+\"", t).group(1)))
        out[f"lj{n}_E_atol_eV"] = np.array(float(re.search(r"e_a_tol = auconvert\((" + NUM + r") \*", t).group(1)))
        out[f"lj{n}_F_atol_eVA"] = np.array(float(re.search(r"f_a_tol = auconvert\((" + NUM + r") \*", t).group(1)))

    # ---- SNAP 3-atom fixtures
    for tag in ("single", "multi"):
        t = read(f"test/SNAP/snap_test_{tag}_element.jl")
        g = lambda name: float(re.search(name + r" = (" + NUM + ")", t).group(1))
        out[f"snap_{tag}_twojmax"] = np.array(int(g("twojmax")))
        out[f"snap_{tag}_rcutfac"] = np.array(g("rcutfac"))
        out[f"snap_{tag}_rfac0"] = np.array(g("rcut0"))
        out[f"snap_{tag}_radii"] = np.array([float(x) for x in re.findall(NUM, re.search(r"radii = \[(.*)\]", t).group(1))])
        out[f"snap_{tag}_weight"] = np.array([float(x) for x in re.findall(NUM, re.search(r"weight = \[(.*)\]", t).group(1))])
        out[f"snap_{tag}_pos"] = np.array([[float(x) for x in re.findall(NUM, re.search(f"position{k} = @SVector \\[(.*)\\]", t).group(1))]
                                           for k in (1, 2, 3)])
        syms = re.findall(r"Atom\(:(\w+), position\d", t)
        out[f"snap_{tag}_symbols"] = np.array(syms)
        sp = re.search(r"SNAP\(num_atoms, twojmax, \[([^\]]*)\]", t).group(1)
        out[f"snap_{tag}_species"] = np.array(re.findall(r":(\w+)", sp))
        out[f"snap_{tag}_box"] = np.array(vectors(re.search(r"box = \[(.*)\]\n", t).group(1))).diagonal().copy()

    np.savez(OUT, **out)
    for k in sorted(out):
        print(k, np.asarray(out[k]).tolist() if np.asarray(out[k]).size <= 12 else np.asarray(out[k]).shape)


if __name__ == "__main__":
    main()
