"""CPU oracle for the force-field hot path — TEST INFRASTRUCTURE ONLY.

This module is the checker for the CUDA library.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import it; the product
path (``libipg.so`` and the ``ipg`` package) never does.

Two independent restatements of the reference (cesmix-mit/InteratomicPotentials.jl
v0.3.2) live here:

* ``liboracle`` — the C++ restatement in ``ipg_oracle.cpp`` (built by ``make -C oracle``),
  OpenMP over atoms; it also serves as the timed CPU baseline.
* ``np_*`` functions — NumPy / pure-Python restatements for small cases, used to
  cross-check the C++ oracle against the reference's golden vectors
  (test/unit/nnlist.jl, test/unit/types/empirical_potential.jl,
  test/integration/lj_clusters/*.jl).
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "build", "libipg_oracle.so")

KIND = {"LJ": 1, "BM": 2, "COUL": 3, "MORSE": 4, "ZBL": 5, "MOCK_R2": 6}

_lib = None


def build():
    """Compile the C++ oracle (g++ with OpenMP) into oracle/build/."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = C.CDLL(LIB_PATH)
        d, i32, i64, vp = C.c_double, C.c_int32, C.c_int64, C.c_void_p
        P = C.POINTER
        _lib.orc_nlist_half.restype = i64
        _lib.orc_nlist_half.argtypes = [i64, vp, vp, d, vp, vp, vp, i64]
        _lib.orc_nlist_snap.restype = i64
        _lib.orc_nlist_snap.argtypes = [i64, vp, vp, vp, i32, vp, d, i32, vp, vp, vp, i64]
        _lib.orc_pair_eval.restype = C.c_int
        _lib.orc_pair_eval.argtypes = [i64, vp, vp, vp, i32, vp, vp, vp, vp, vp, vp, vp, vp]
        _lib.orc_snap_create.restype = vp
        _lib.orc_snap_create.argtypes = [i32, i32, d, d, d, vp, vp, i32, i32, i32, i32, i32, i32, i32, i32]
        _lib.orc_snap_ncoef.restype = i32
        _lib.orc_snap_ncoef.argtypes = [vp]
        _lib.orc_snap_destroy.restype = None
        _lib.orc_snap_destroy.argtypes = [vp]
        _lib.orc_snap_sizes.restype = None
        _lib.orc_snap_sizes.argtypes = [vp, vp]
        _lib.orc_snap_cglist.restype = None
        _lib.orc_snap_cglist.argtypes = [vp, vp]
        _lib.orc_snap_index_tables.restype = None
        _lib.orc_snap_index_tables.argtypes = [vp, vp, vp, vp, vp, vp]
        _lib.orc_snap_descriptors.restype = C.c_int
        _lib.orc_snap_descriptors.argtypes = [vp, i64, vp, vp, vp, vp, vp, vp, vp]
        _lib.orc_snap_energy_forces.restype = C.c_int
        _lib.orc_snap_energy_forces.argtypes = [vp, i64, vp, vp, vp, vp, d, i32, i64, i64, vp, vp, vp, vp, i32]
        _lib.orc_snap_vjp_beta.restype = C.c_int
        _lib.orc_snap_vjp_beta.argtypes = [vp, i64, vp, vp, vp, d, vp, vp, vp]
        del P
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


# ----------------------------------------------------------------------------------
# Neighbor lists
def nlist_half(pos, L, rcut):
    """Half list of src/nnlist.jl:23-46 -> (offsets, j, r) with r = x_n - x_m."""
    pos, L = _f64(pos), _f64(L)
    n = pos.shape[0]
    np_ = lib().orc_nlist_half(n, _p(pos), _p(L), float(rcut), None, None, None, 0)
    if np_ < 0:
        raise ValueError(f"oracle status {np_}")
    off = np.zeros(n + 1, np.int64)
    j = np.zeros(max(np_, 1), np.int32)
    r = np.zeros((max(np_, 1), 3))
    lib().orc_nlist_half(n, _p(pos), _p(L), float(rcut), _p(off), _p(j), _p(r), np_)
    return off, j[:np_], r[:np_]


def nlist_snap(pos, L, species, radii, rcutfac, literal_sqrt=False):
    """Full SNAP list of src/BasisSystems/SNAP/utilities/utl.jl:38-101, r = x_nb - x_n."""
    pos, L, species, radii = _f64(pos), _f64(L), _i32(species), _f64(radii)
    n = pos.shape[0]
    args = (n, _p(pos), _p(L), _p(species), len(radii), _p(radii), float(rcutfac), int(literal_sqrt))
    np_ = lib().orc_nlist_snap(*args, None, None, None, 0)
    if np_ < 0:
        raise ValueError(f"oracle status {np_}")
    off = np.zeros(n + 1, np.int64)
    j = np.zeros(max(np_, 1), np.int32)
    r = np.zeros((max(np_, 1), 3))
    lib().orc_nlist_snap(*args, _p(off), _p(j), _p(r), np_)
    return off, j[:np_], r[:np_]


# ----------------------------------------------------------------------------------
# Pair potentials
def pair_eval(pos, species, L, terms):
    """terms: list of dicts {kind, coeff, rcut, mask, params[<=8]} -> (E, F[n,3], W[6])."""
    pos, species, L = _f64(pos), _i32(species), _f64(L)
    n = pos.shape[0]
    nt = len(terms)
    kinds = np.array([KIND[t["kind"]] if isinstance(t["kind"], str) else t["kind"] for t in terms], np.int32)
    coeffs = np.array([t.get("coeff", 1.0) for t in terms], np.float64)
    rcuts = np.array([t["rcut"] for t in terms], np.float64)
    masks = np.array([t.get("mask", (1 << 64) - 1) for t in terms], np.uint64)
    params = np.zeros((nt, 8))
    for k, t in enumerate(terms):
        params[k, : len(t["params"])] = t["params"]
    E = np.zeros(1)
    F = np.zeros((n, 3))
    W = np.zeros(6)
    st = lib().orc_pair_eval(n, _p(pos), _p(species), _p(L), nt, _p(kinds), _p(coeffs), _p(rcuts), _p(masks),
                             _p(params), _p(E), _p(F), _p(W))
    if st:
        raise ValueError(f"oracle status {st}")
    return E[0], F, W


# ----------------------------------------------------------------------------------
# SNAP
class Snap:
    """Oracle SNAP basis (prebuilt tables of prebuilt_arrays.jl:48-321)."""

    def __init__(self, twojmax, radii, weight, rcutfac, rmin0=0.0, rfac0=0.99363, bzero=False, bnorm=False,
                 switch=False, literal_sqrt=False, chem=False, wselfall=False, literal_chem_z=False,
                 quadratic=False):
        self.radii = _f64(radii)
        self.weight = _f64(weight)
        self.nsp = len(self.radii)
        self.twojmax = twojmax
        self.rcutfac = float(rcutfac)
        self.literal_sqrt = bool(literal_sqrt)
        self.h = lib().orc_snap_create(twojmax, self.nsp, rcutfac, rmin0, rfac0, _p(self.radii), _p(self.weight),
                                       int(bzero), int(bnorm), int(switch), int(literal_sqrt), int(chem),
                                       int(wselfall), int(literal_chem_z), int(quadratic))
        if not self.h:
            raise ValueError("oracle rejected SNAP parameters")
        sz = np.zeros(4, np.int32)
        lib().orc_snap_sizes(self.h, _p(sz))
        self.idxu_max, self.idxz_max, self.idxb_max, self.idxcg_max = (int(x) for x in sz)
        self.K = int(lib().orc_snap_ncoef(self.h))  # components per species block

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_snap_destroy(self.h)
            self.h = None

    def cglist(self):
        out = np.zeros(self.idxcg_max)
        lib().orc_snap_cglist(self.h, _p(out))
        return out

    def index_tables(self):
        jd = self.twojmax + 1
        idxz = np.zeros((self.idxz_max, 10), np.int32)
        idxb = np.zeros((self.idxb_max, 3), np.int32)
        cgb = np.zeros(jd ** 3, np.int32)
        zb = np.zeros(jd ** 3, np.int32)
        ub = np.zeros(jd, np.int32)
        lib().orc_snap_index_tables(self.h, _p(idxz), _p(idxb), _p(cgb), _p(zb), _p(ub))
        return dict(idxz=idxz, idxb=idxb, idxcg_block=cgb.reshape(jd, jd, jd), idxz_block=zb.reshape(jd, jd, jd),
                    idxu_block=ub)

    def descriptors(self, pos, species, L, want_utot=False):
        """compute_all_descriptors (snap.jl:251-310) -> B[n,K], dB[n,K*nsp,3], W[K*nsp,6]."""
        pos, species, L = _f64(pos), _i32(species), _f64(L)
        n = pos.shape[0]
        Kn = self.K * self.nsp
        B = np.zeros((n, self.K))
        dB = np.zeros((n, Kn, 3))
        W = np.zeros((Kn, 6))
        ut = np.zeros((n, self.idxu_max, 2)) if want_utot else None
        st = lib().orc_snap_descriptors(self.h, n, _p(pos), _p(species), _p(L), _p(B), _p(dB), _p(W), _p(ut))
        if st:
            raise ValueError(f"oracle status {st}")
        if want_utot:
            return B, dB, W, ut[..., 0] + 1j * ut[..., 1]
        return B, dB, W

    def energy_forces(self, pos, species, L, beta, beta0=0.0, mode="plain", i0=0, i1=None, nthreads=0,
                      per_atom=False):
        """E, F[n,3], W6 for E = beta0 + sum_i beta[s_i].B_i (mode 'plain' or 'adjoint')."""
        pos, species, L = _f64(pos), _i32(species), _f64(L)
        beta = _f64(beta).reshape(self.nsp, self.K)
        n = pos.shape[0]
        i1 = n if i1 is None else i1
        E = np.zeros(1)
        F = np.zeros((n, 3))
        W = np.zeros(6)
        Ei = np.zeros(n) if per_atom else None
        st = lib().orc_snap_energy_forces(self.h, n, _p(pos), _p(species), _p(L), _p(beta), float(beta0),
                                          1 if mode == "adjoint" else 0, int(i0), int(i1), _p(E), _p(F), _p(W),
                                          _p(Ei), int(nthreads))
        if st:
            raise ValueError(f"oracle status {st}")
        if per_atom:
            return E[0], F, W, Ei
        return E[0], F, W

    def vjp_beta(self, pos, species, L, gE, gF):
        pos, species, L = _f64(pos), _i32(species), _f64(L)
        n = pos.shape[0]
        gF = None if gF is None else _f64(gF).reshape(n, 3)
        gb = np.zeros((self.nsp, self.K))
        gb0 = np.zeros(1)
        st = lib().orc_snap_vjp_beta(self.h, n, _p(pos), _p(species), _p(L), float(gE), _p(gF), _p(gb), _p(gb0))
        if st:
            raise ValueError(f"oracle status {st}")
        return gb, gb0[0]


# ----------------------------------------------------------------------------------
# NumPy restatements for small cases (independent of the C++ code above).
def np_jl_mod(x, y):
    r = np.fmod(x, y)
    return np.where((r != 0) & ((r > 0) != (y > 0)), r + y, r)


def np_disp(L, x, y):
    """src/nnlist.jl:18-21."""
    out = x - y
    per = np.isfinite(L)
    d = np_jl_mod(x - y, np.where(per, L, 1.0))
    d = np.where(2 * d < L, d, d - L)
    return np.where(per, d, out)


def np_nlist_half(pos, L, rcut):
    """All-pairs half list, src/nnlist.jl:23-46."""
    pos = np.asarray(pos, float)
    L = np.asarray(L, float)
    n = len(pos)
    js, rs = [], []
    for a in range(n):
        ja, ra = [], []
        for m in range(a + 1, n):
            s1 = np.abs(pos[a] - pos[m])
            s2 = np.where(np.isfinite(L), np_jl_mod(s1, np.where(np.isfinite(L), L, 1.0)), s1)
            s3 = np.where(np.isfinite(L), np.minimum(s2, L - s2), s1)
            if math.sqrt(float(s3[0] ** 2 + s3[1] ** 2 + s3[2] ** 2)) <= rcut:
                ja.append(m)
                ra.append(np_disp(L, pos[a], pos[m]))
        js.append(ja)
        rs.append(ra)
    return js, rs


def np_lj_allpairs(pos, eps, sigma):
    """Open-boundary, no-cutoff LJ energy and forces (all pairs), lj.jl:35-36."""
    pos = np.asarray(pos, float)
    d = pos[:, None, :] - pos[None, :, :]
    R2 = np.einsum("ijk,ijk->ij", d, d)
    iu = np.triu_indices(len(pos), 1)
    s2 = sigma * sigma / R2[iu]
    s6 = s2 ** 3
    E = np.sum(4 * eps * (s6 * s6 - s6))
    g = np.zeros_like(R2)
    g[iu] = 24 * eps * (2 * s6 * s6 - s6) / R2[iu]
    g = g + g.T
    F = np.einsum("ij,ijk->ik", g, d)
    return E, F
