"""Algorithmic FP64 operation counts of the SNAP kernels (for the roofline).

Counts follow the loop structure of the kernels in csrc/ipg_snap.cu exactly, one flop
per add / multiply (an FMA counts as two).  Transcendental geometry per pair (sqrt,
sincos, tan, a few divisions) is not counted, so the figures are a lower bound.

  per_atom(J)  : Z contraction + B + E (+ Y for the adjoint path)
  per_pair(J)  : Utot recursion + derivative recursion + contraction with Y (adjoint)
                 or dB/dr (plain)
"""
from __future__ import annotations


def _levels(J):
    for j in range(J + 1):
        for mb in range(j // 2 + 1):
            for ma in range(j + 1):
                yield j, mb, ma


def _terms(j, ma):
    return (ma > 0) + (ma < j)


def _tables(J):
    """idxz entries (j1, j2, j, na, nb) and idxb triples, in the reference's order."""
    zs, bs = [], []
    for j1 in range(J + 1):
        for j2 in range(j1 + 1):
            for j in range(j1 - j2, min(J, j1 + j2) + 1, 2):
                if j >= j1:
                    bs.append((j1, j2, j))
                for mb in range(j // 2 + 1):
                    for ma in range(j + 1):
                        ma1min = max(0, (2 * ma - j - j2 + j1) // 2)
                        na = min(j1, (2 * ma - j + j2 + j1) // 2) - ma1min + 1
                        mb1min = max(0, (2 * mb - j - j2 + j1) // 2)
                        nb = min(j1, (2 * mb - j + j2 + j1) // 2) - mb1min + 1
                        zs.append((j1, j2, j, na, nb))
    return zs, bs


def _nfull(l):
    return ((l + 1) // 2) * (l + 1) + (0 if l % 2 else l // 2)


def u_pair(J):
    """Phase 1: one neighbor's contribution to Utot (recursion + accumulate)."""
    f = 2  # level 0 accumulate
    for j, mb, ma in _levels(J):
        if j == 0:
            continue
        t = _terms(j, ma)
        f += 8 * t + (2 if t == 2 else 0) + 4
    return f


def du_pair(J):
    """Phase 5 recursion: U and the three components of dU/dr of one neighbor."""
    f = 0
    for j, mb, ma in _levels(J):
        if j == 0:
            continue
        t = _terms(j, ma)
        f += 8 * t + (2 if t == 2 else 0)           # U
        f += 3 * (16 * t + (2 if t == 2 else 0))    # dU/dx, dU/dy, dU/dz
    return f


def adjoint_contract_pair(J):
    """Phase 5 adjoint: dE/dr = 2 sum w Re(conj(dU) Y) with the switching product rule."""
    n = 0
    for j in range(J + 1):
        n += _nfull(j) + (0 if j % 2 else 1)
    return 39 * n


def plain_db_pair(J):
    """Phase 5 plain: product rule for every half-plane entry + the 3 dB/dr sums."""
    nhalf = sum(1 for _ in _levels(J))
    f = 24 * nhalf
    _, bs = _tables(J)
    for (j1, j2, j) in bs:
        for l in (j, j1, j2):
            f += 3 * (4 * _nfull(l) + (5 if l % 2 == 0 else 0) + 2)
        f += 3 * 2
    return f


def z_atom(J):
    zs, _ = _tables(J)
    return sum(nb * (10 * na + 4) for (_, _, _, na, nb) in zs)


def b_atom(J):
    _, bs = _tables(J)
    return sum(4 * _nfull(j) + (5 if j % 2 == 0 else 0) + 2 for (_, _, j) in bs) + 2 * len(bs)


def y_atom(J):
    zs, _ = _tables(J)
    return 4 * len(zs)


def u_half(J):
    """Half-plane entries (mb <= j/2) of all levels."""
    return sum(1 for _ in _levels(J))


def _n_contract(J):
    """Half-plane entries carrying a non-zero weight (the middle row of an even level stops at j/2)."""
    return sum(1 for j, mb, ma in _levels(J) if not (2 * mb == j and ma > mb))


def yatoms_atom(J):
    """k_snap_yatoms, one atom: every Z entry, its share of Y, the weight and the Euler energy term."""
    return z_atom(J) + y_atom(J) + 6 * u_half(J)


def utot_pair(J):
    """k_snap_utot, one directed pair: the U recursion of every half-plane row and the sfac-weighted
    accumulation (the staircase recomputation of the chain kernels is overhead, not counted)."""
    return u_pair(J)


def chain_adjoint_pair(J):
    """k_snap_pair_adj_all, one directed pair: U and dU/dr of the half plane, the S0/S_k contraction with
    the weighted Y (4 flops for S0 and 4 for each S_k per weighted entry), and the final 2(dsfac u S0 + sfac S)."""
    return du_pair(J) + 16 * _n_contract(J) + 12


def lie_pair(J):
    """k_snap_pair_lie, one directed pair: the U recursion of the half plane (no tangents), its
    contraction with the staged Yw, Y2, Y3 (S0: 4 flops, T1: 5, T2 and T3: 4 each per contracted
    entry; T1 vanishes where j = 2 ma; the middle row of an even level runs to ma = mb + 1), the
    generator coefficients (30 flops per direction) and F_k (8 flops per direction)."""
    f = 0
    for j, mb, ma in _levels(J):
        if j == 0:
            continue
        t = _terms(j, ma)
        f += 8 * t + (2 if t == 2 else 0)
    for j, mb, ma in _levels(J):
        lim = min(mb + 1, j) if 2 * mb == j else j
        if ma <= lim:
            f += 12 + (5 if j != 2 * ma else 0)
    return f + 3 * (30 + 8)


def adjoint_kernels(J, natoms, npairs, pair_kernel="lie"):
    """Flops per launch of each kernel of the adjoint step, keyed like the library's timing names.
    pair_kernel: "lie" (k_snap_pair_lie, the default) or "tangent" (k_snap_pair_adj_all)."""
    pair = lie_pair(J) if pair_kernel == "lie" else chain_adjoint_pair(J)
    return {"snap_atom": natoms * yatoms_atom(J), "snap_utot": npairs * utot_pair(J),
            "snap_pair": npairs * pair}


def snap_atom_kernel(J, natoms, npairs, mode):
    """Flops of one launch of the fused per-atom SNAP kernel."""
    atom = z_atom(J) + b_atom(J)
    pair = u_pair(J) + du_pair(J)
    if mode == "adjoint":
        atom += y_atom(J)
        pair += adjoint_contract_pair(J)
    else:
        pair += plain_db_pair(J)
    return natoms * atom + npairs * pair
