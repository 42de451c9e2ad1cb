"""The su(2) generator identity behind the adjoint pair kernels, checked on the CPU.

The Wigner matrices U^j(r) of compute_uarray (src/BasisSystems/SNAP/utilities/compute_ui.jl:
50-129) are the spin-j/2 representation of the unit quaternion (a, b) of r, so
    dU^j/dr_k = U^j (al_k D1 + Re(be_k) D2 + Im(be_k) D3),
with D1 = diag(i (j - 2 ma)), D2[m][m+1] = s_m = -D2[m+1][m], D3[m][m+1] = D3[m+1][m] = i s_m,
s_m = sqrt((m + 1)(j - m)), al_k = Im(a conj(da_k) + conj(b) db_k), be_k = conj(b) da_k -
a conj(db_k).  The GPU kernels k_snap_pair_lie, k_snap_vlie and k_snap_pair_hvp_lie rest on
it; their results are compared with the tangent-chain kernels and the oracle on the GPU.
Here a NumPy restatement of the recursion is pinned to the oracle's Utot, and the identity,
and the contraction with the generator-shifted copies of Y that k_snap_pair_lie stages, are
checked against central differences.
"""
import numpy as np
import pytest

import oracle

J = 8
RMIN0, RFAC0, RCUT = 0.0, 0.99363, 5.0


def rootpq(p, q):
    return np.sqrt(p / q)


def umat(a, b):
    """U^j[mb][ma] for j = 0..J: rows mb <= j/2 by the recursion, the others by inversion
    symmetry U[mb][ma] = (-1)^(ma+mb) conj(U[j-mb][j-ma]) (compute_ui.jl:50-129)."""
    U = [np.array([[1.0 + 0j]])]
    for j in range(1, J + 1):
        M = np.zeros((j + 1, j + 1), complex)
        P = U[j - 1]
        for mb in range(j // 2 + 1):
            for ma in range(j + 1):
                v = 0j
                if ma < j:
                    v += rootpq(j - ma, j - mb) * np.conj(a) * P[mb, ma]
                if ma > 0:
                    v -= rootpq(ma, j - mb) * np.conj(b) * P[mb, ma - 1]
                M[mb, ma] = v
        for mb in range(j // 2 + 1, j + 1):
            for ma in range(j + 1):
                M[mb, ma] = (-1) ** (ma + mb) * np.conj(M[j - mb, j - ma])
        U.append(M)
    return U


def ab(r):
    """The Cayley-Klein parameters of compute_ui.jl (theta0 from the pair cutoff)."""
    x, y, z = r
    rr = np.sqrt(x * x + y * y + z * z)
    th = (rr - RMIN0) * RFAC0 * np.pi / (RCUT - RMIN0)
    z0 = rr / np.tan(th)
    r0inv = 1.0 / np.sqrt(rr * rr + z0 * z0)
    return r0inv * (z0 - 1j * z), r0inv * (y - 1j * x)


def generators(j):
    s = np.array([np.sqrt((m + 1) * (j - m)) for m in range(j)])
    D1 = np.diag([1j * (j - 2 * m) for m in range(j + 1)])
    D2 = np.zeros((j + 1, j + 1), complex)
    D3 = np.zeros((j + 1, j + 1), complex)
    for m in range(j):
        D2[m, m + 1], D2[m + 1, m] = s[m], -s[m]
        D3[m, m + 1] = D3[m + 1, m] = 1j * s[m]
    return D1, D2, D3


def coeffs(r, k, h=1e-6):
    """a, b, their r_k derivatives (central differences) and (al_k, Re be_k, Im be_k)."""
    e = np.zeros(3)
    e[k] = h
    a, b = ab(r)
    ap, bp = ab(r + e)
    am, bm = ab(r - e)
    da, db = (ap - am) / (2 * h), (bp - bm) / (2 * h)
    al = (a * np.conj(da) + np.conj(b) * db).imag
    be = np.conj(b) * da - a * np.conj(db)
    return al, be.real, be.imag


def directions(rng, n):
    out = []
    for _ in range(n):
        r = rng.normal(size=3)
        out.append(r * rng.uniform(1.0, 4.5) / np.linalg.norm(r))
    return out


def test_recursion_restatement_matches_oracle_utot():
    """Two atoms in an open box: Utot of atom 0 = wself I + w U(x_1 - x_0) (no switching)."""
    orc = oracle.Snap(J, [0.5], [0.7], RCUT, RMIN0, RFAC0, switch=False)
    for r in directions(np.random.default_rng(3), 4):
        pos = np.array([[0.0, 0.0, 0.0], r])
        _, _, _, ut = orc.descriptors(pos, np.zeros(2, np.int32), np.full(3, np.inf), want_utot=True)
        a, b = ab(r)
        U = umat(a, b)
        blk = 0
        for j in range(J + 1):
            ref = (ut[0, blk:blk + (j + 1) ** 2].reshape(j + 1, j + 1) - np.eye(j + 1)) / 0.7
            np.testing.assert_allclose(U[j], ref, rtol=0, atol=1e-13)
            blk += (j + 1) ** 2


def test_derivative_is_u_times_generator():
    """dU/dr_k (central differences of the recursion) = U (al D1 + Re be D2 + Im be D3)."""
    gens = [generators(j) for j in range(J + 1)]
    h = 1e-6
    for r in directions(np.random.default_rng(5), 6):
        U = umat(*ab(r))
        for k in range(3):
            e = np.zeros(3)
            e[k] = h
            Up, Um = umat(*ab(r + e)), umat(*ab(r - e))
            al, br, bi = coeffs(r, k)
            for j in range(J + 1):
                D1, D2, D3 = gens[j]
                dU = (Up[j] - Um[j]) / (2 * h)
                np.testing.assert_allclose(U[j] @ (al * D1 + br * D2 + bi * D3), dU, rtol=0, atol=1e-8)


@pytest.mark.parametrize("seed", [0, 1])
def test_contraction_with_shifted_y_copies(seed):
    """S_k = sum over the weighted half plane of Re(conj(dU_k) Y) equals al T1 + Re(be) T2 +
    Im(be) T3 with the copies the pair kernel stages: Y2[m] = s_m Y[m+1] - s_{m-1} Y[m-1],
    Y3[m] = -i (s_m Y[m+1] + s_{m-1} Y[m-1]) and T1 = sum (j - 2m) Im(conj(U) Y)."""
    rng = np.random.default_rng(seed)
    # a weighted Y on the half plane: rows mb <= j/2, zero beyond ma = mb in the middle row
    Y = []
    for j in range(J + 1):
        M = np.zeros((j + 1, j + 1), complex)
        for mb in range(j // 2 + 1):
            last = mb if 2 * mb == j else j
            M[mb, : last + 1] = rng.normal(size=last + 1) + 1j * rng.normal(size=last + 1)
        Y.append(M)
    h = 1e-6
    for r in directions(rng, 3):
        U = umat(*ab(r))
        for k in range(3):
            e = np.zeros(3)
            e[k] = h
            Up, Um = umat(*ab(r + e)), umat(*ab(r - e))
            Sk = sum(np.sum(np.conj((Up[j] - Um[j]) / (2 * h)) * Y[j]).real for j in range(J + 1))
            T = np.zeros(3)
            for j in range(J + 1):
                s = [np.sqrt((m + 1) * (j - m)) if m < j else 0.0 for m in range(j + 1)]
                for mb in range(j // 2 + 1):
                    y = Y[j][mb]
                    for m in range(j + 1):
                        A = s[m] * y[m + 1] if m < j else 0.0
                        B = s[m - 1] * y[m - 1] if m >= 1 else 0.0
                        u = U[j][mb, m]
                        T[0] += (j - 2 * m) * (np.conj(u) * y[m]).imag
                        T[1] += (np.conj(u) * (A - B)).real
                        T[2] += (np.conj(u) * (-1j * (A + B))).real
            al, br, bi = coeffs(r, k)
            assert abs(al * T[0] + br * T[1] + bi * T[2] - Sk) <= 1e-7 * max(1.0, abs(Sk))
