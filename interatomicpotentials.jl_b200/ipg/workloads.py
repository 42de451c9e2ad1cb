"""Seeded synthetic workloads for the five benchmark configurations.

No dataset is involved: every configuration is generated here from a seed, with the
lattice, box, jitter, species mix and potential parameters stated for it.

  lj1000    LennardJones (eps 0.0104 eV, sigma 3.4 A, rcut 8.5 A), Ar FCC a=5.26 A,
            5x5x10 cells (N=1000), periodic, jitter N(0, 0.05 A), seed 1.
  lc32000   LJ(Ar) + LJ(Xe) + LJ(Ar,Xe) + ZBL(18, 54, e) + BornMayer(A=1000 eV, rho=0.3 A),
            rcut 10 A, FCC a=5.5 A 20^3 cells (N=32000), Ar/Xe 50/50 and jitter
            N(0, 0.08 A) from seed 2.  LJ(Xe): eps 0.020 eV, sigma 4.1 A; LJ(Ar,Xe) by
            Lorentz-Berthelot; ZBL base e = 2.718281828459045 (Euler's number).
  snap_j6   SNAP twojmax 6, BCC a=3.3 A 16^3 cells (N=8192), jitter N(0, 0.1 A) seed 3,
            rcutfac 4.7, radius 0.5, rfac0 0.99363, rmin0 0, switch on, beta ~ N(0, 1e-2).
  snap_j8   SNAP twojmax 8, two species (weights 1.0/0.5, radii 0.5/0.45, rcutfac 5.0),
            BCC a=3.2 A 30^3 cells (N=54000), species 70/30 and jitter N(0, 0.12 A)
            from seed 4, switch on, per-species beta ~ N(0, 1e-2).
  batch512  512 configurations (seed 5) of 32..2000 atoms: jittered BCC/FCC crystals with
            a in [3.1, 3.4] A (N snapped to 2k^3 / 4k^3) or random liquids at 0.06 / A^3
            with a 1.8 A minimum separation; two species 70/30; snap_j8 parameters;
            F_ref = F(beta_ref) + N(0, 0.01) noise (computed by the caller).

Pair workloads are returned in atomic units (bohr, hartree); SNAP workloads in
angstrom, like the reference's austrip / ustrip conventions.
"""
from __future__ import annotations

import math

import numpy as np

from . import units
from .system import System

EULER_E = 2.718281828459045


def lattice(kind, a, nx, ny, nz):
    basis = {"fcc": [(0, 0, 0), (0.5, 0.5, 0), (0.5, 0, 0.5), (0, 0.5, 0.5)],
             "bcc": [(0, 0, 0), (0.5, 0.5, 0.5)]}[kind]
    g = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"), -1).reshape(-1, 3)
    pts = np.concatenate([g + np.asarray(b) for b in basis])
    order = np.lexsort((pts[:, 2], pts[:, 1], pts[:, 0]))
    return pts[order] * a, np.array([nx * a, ny * a, nz * a], dtype=np.float64)


# ----------------------------------------------------------------------------------
def lj1000(scale=1):
    """LJ FCC Ar; scale multiplies the cell counts along each axis (scale=1 -> N=1000)."""
    rng = np.random.default_rng(1)
    pos, box = lattice("fcc", 5.26, 5 * scale, 5 * scale, 10 * scale)
    pos = pos + rng.normal(0.0, 0.05, pos.shape)
    A = units.angstrom
    sys_ = System(pos * A, ["Ar"] * len(pos), box * A, (True, True, True))
    from .empirical import LennardJones
    pot = LennardJones(0.0104 * units.eV, 3.4 * A, 8.5 * A, ["Ar"])
    return sys_, pot


def lc_potential(zbl_e=EULER_E):
    from .empirical import ZBL, BornMayer, LennardJones
    A, eV = units.angstrom, units.eV
    rc = 10.0 * A
    e_ar, s_ar, e_xe, s_xe = 0.0104, 3.4, 0.020, 4.1
    lj_ar = LennardJones(e_ar * eV, s_ar * A, rc, ["Ar"])
    lj_xe = LennardJones(e_xe * eV, s_xe * A, rc, ["Xe"])
    lj_arxe = LennardJones(math.sqrt(e_ar * e_xe) * eV, 0.5 * (s_ar + s_xe) * A, rc, ["Ar", "Xe"])
    zbl = ZBL(18, 54, zbl_e, rc, ["Ar", "Xe"])
    bm = BornMayer(1000.0 * eV, 0.3 * A, 0.0, 0.0, 0.0, rc, ["Ar", "Xe"])
    return lj_ar + lj_xe + lj_arxe + zbl + bm


def lc32000(cells=20, zbl_e=EULER_E):
    """LC over FCC a=5.5 A; cells=20 -> N=32000 (cells=101 -> 4.12 M atoms)."""
    rng = np.random.default_rng(2)
    pos, box = lattice("fcc", 5.5, cells, cells, cells)
    sym = np.where(rng.random(len(pos)) < 0.5, "Ar", "Xe")
    pos = pos + rng.normal(0.0, 0.08, pos.shape)
    A = units.angstrom
    return System(pos * A, list(sym), box * A, (True, True, True)), lc_potential(zbl_e)


# ----------------------------------------------------------------------------------
def snap_j6_params():
    return dict(twojmax=6, species=["W"], rcutfac=4.7, rmin0=0.0, rfac0=0.99363, radii=[0.5], weight=[1.0],
                switch_flag=True)


def snap_j8_params():
    return dict(twojmax=8, species=["A", "B"], rcutfac=5.0, rmin0=0.0, rfac0=0.99363, radii=[0.5, 0.45],
                weight=[1.0, 0.5], switch_flag=True)


def snap_j6(cells=16):
    rng = np.random.default_rng(3)
    pos, box = lattice("bcc", 3.3, cells, cells, cells)
    pos = pos + rng.normal(0.0, 0.1, pos.shape)
    beta = rng.normal(0.0, 1e-2, 30)
    return System(pos, ["W"] * len(pos), box, (True, True, True)), snap_j6_params(), beta


def snap_j8(cells=30):
    rng = np.random.default_rng(4)
    pos, box = lattice("bcc", 3.2, cells, cells, cells)
    sym = np.where(rng.random(len(pos)) < 0.7, "A", "B")
    pos = pos + rng.normal(0.0, 0.12, pos.shape)
    beta = rng.normal(0.0, 1e-2, (2, 55))
    return System(pos, list(sym), box, (True, True, True)), snap_j8_params(), beta


def _liquid(rng, n, density=0.06, dmin=1.8):
    """Random sequential addition in a periodic cube: candidates are proposed in chunks
    and accepted in proposal order when no accepted atom lies within dmin."""
    from scipy.spatial import cKDTree

    L = (n / density) ** (1.0 / 3.0)
    acc = np.empty((0, 3))
    while len(acc) < n:
        cand = rng.random((max(64, 2 * (n - len(acc))), 3)) * L
        if len(acc):
            d, _ = cKDTree(acc, boxsize=L).query(cand, k=1)
            cand = cand[d >= dmin]
        if len(cand) == 0:
            continue
        conflicts = {}
        for a, b in cKDTree(cand, boxsize=L).query_pairs(dmin):
            conflicts.setdefault(max(a, b), []).append(min(a, b))
        keep = np.zeros(len(cand), bool)
        for q in range(len(cand)):
            keep[q] = not any(keep[p] for p in conflicts.get(q, ()))
        acc = np.concatenate([acc, cand[keep]])[:n]
    return acc, np.array([L, L, L])


def batch512(nconf=512, nmin=32, nmax=2000):
    """List of Systems (angstrom) for the batched configuration."""
    rng = np.random.default_rng(5)
    out = []
    for c in range(nconf):
        target = int(rng.integers(nmin, nmax + 1))
        kind = rng.choice(["bcc", "fcc", "liquid"])
        if kind == "liquid":
            pos, box = _liquid(rng, target)
        else:
            a = float(rng.uniform(3.1, 3.4))
            per = 2 if kind == "bcc" else 4
            k = max(2, int(round((target / per) ** (1.0 / 3.0))))
            pos, box = lattice(kind, a, k, k, k)
            pos = pos + rng.normal(0.0, 0.05, pos.shape)
        sym = np.where(rng.random(len(pos)) < 0.7, "A", "B")
        out.append(System(pos, list(sym), box, (True, True, True)))
    return out
