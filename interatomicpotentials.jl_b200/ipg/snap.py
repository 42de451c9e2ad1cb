"""SNAP basis, its descriptors and the linear SNAP potential, evaluated on the GPU.

Mirrors src/BasisSystems/SNAP/snap.jl (SNAP{S,T} and compute_*_descriptors) and
src/BasisPotentials/{basis_potentials,linear_potential}.jl (LBasisPotential).  Positions
are in the system's own length unit, as the reference's ``ustrip`` leaves them.

Array layouts (NumPy, row-major):
  compute_local_descriptors -> B  (n, K)
  compute_force_descriptors -> dB (n, 3, K*nspecies)   (each atom's 3 x K*nspecies matrix)
  compute_all_descriptors   -> (B, dB, W) with W (6, K*nspecies), rows [xx,yy,zz,yz,xz,xy]
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import (DESC_B, DESC_DB, DESC_W, MAX_SNAP_SPECIES, SNAP_ADJOINT, SNAP_PLAIN, SnapParams, lib)
from .context import default_context


def _vp(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def get_num_snap_coeffs(twojmax, n_elems, chem_flag, quadratic_flag=False):
    """src/BasisSystems/SNAP/utilities/utl.jl:8-25 (quadratic_flag: plus K(K+1)/2 products)."""
    J = twojmax
    if J % 2 == 0:
        m = J // 2 + 1
        nc = m * (m + 1) * (2 * m + 1) // 6
    else:
        m = (J + 1) // 2
        nc = m * (m + 1) * (m + 2) // 3
    k = nc * n_elems ** 3 if chem_flag else nc
    return k + k * (k + 1) // 2 if quadratic_flag else k


class SNAP:
    """SNAP{S,T} (src/BasisSystems/SNAP/types/types.jl:8-25).

    Keyword flags follow the reference constructors (snap.jl:6-97); chem_flag must equal
    bnorm_flag (snap.jl:10-13).  chem_flag resolves the descriptors by element triple
    (K = idxb_max * nspecies^3); literal_chem_z reproduces compute_z.jl's Z index with it.
    quadratic_flag appends the products 0.5 B_k^2 and B_k B_l (l > k) to the K linear
    components (the quadratic option of LAMMPS_SNAP/snap.jl:45-47).
    literal_sqrt_radius=True reproduces the sqrt(cutmax) neighbor search radius of
    utl.jl:81 literally; the default searches within cutmax.
    """

    def __init__(self, n_atoms, twojmax, species, rcutfac, rmin0, rfac0, radii, weight, chem_flag=False,
                 bzero_flag=False, bnorm_flag=False, switch_flag=False, wselfall_flag=False,
                 literal_sqrt_radius=False, quadratic_flag=False, literal_chem_z=False, ctx=None):
        if chem_flag != bnorm_flag:
            raise ValueError("chem_flag and bnorm_flag should be the same")
        self.n_atoms = n_atoms
        self.twojmax = int(twojmax)
        self.species = list(species)
        self.rcutfac, self.rmin0, self.rfac0 = float(rcutfac), float(rmin0), float(rfac0)
        self.radii = [float(r) for r in radii]
        self.weight = [float(w) for w in weight]
        self.chem_flag, self.bzero_flag, self.bnorm_flag = bool(chem_flag), bool(bzero_flag), bool(bnorm_flag)
        self.switch_flag, self.wselfall_flag = bool(switch_flag), bool(wselfall_flag)
        self.literal_sqrt_radius = bool(literal_sqrt_radius)
        if len(self.species) > MAX_SNAP_SPECIES:
            raise ValueError(f"at most {MAX_SNAP_SPECIES} species")
        self.ctx = ctx or default_context()
        p = SnapParams()
        p.twojmax = self.twojmax
        p.nspecies = len(self.species)
        p.rcutfac, p.rmin0, p.rfac0 = self.rcutfac, self.rmin0, self.rfac0
        for k in range(len(self.species)):
            p.radii[k] = self.radii[k]
            p.weight[k] = self.weight[k]
        p.chem_flag, p.bzero_flag, p.bnorm_flag = int(chem_flag), int(bzero_flag), int(bnorm_flag)
        p.switch_flag, p.wselfall_flag = int(switch_flag), int(wselfall_flag)
        p.literal_sqrt_radius = int(literal_sqrt_radius)
        p.quadratic_flag = int(quadratic_flag)
        p.literal_chem_z = int(literal_chem_z)
        self.quadratic_flag = bool(quadratic_flag)
        h = C.c_void_p()
        self.ctx.check(lib().ipg_snap_create(self.ctx.handle, C.byref(p), C.byref(h)))
        self._h = h
        self.ctx._register(self)
        K = C.c_int32()
        self.ctx.check(lib().ipg_snap_ncoeff(h, C.byref(K)))
        self.K = K.value

    @property
    def handle(self):
        return self._h

    def __len__(self):  # length(snap), snap.jl:4
        return self.K

    def get_species(self):
        return self.species

    def get_rcutoff(self):
        return max(2.0 * r * self.rcutfac for r in self.radii)

    def species_ids(self, system):
        """0-based species ids of the system's atoms, by their position in snap.species."""
        try:
            return system.species_index(self.species)
        except KeyError as e:
            raise ValueError(f"system has a species not in snap.species: {e}") from None

    def close(self):
        if getattr(self, "_h", None):
            if getattr(self.ctx, "_h", None):  # a closed context has closed its SNAP handles
                lib().ipg_snap_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- descriptors ------------------------------------------------------------------
    def _descriptors(self, system, what):
        n = len(system)
        nsp = len(self.species)
        sp = self.species_ids(system)
        B = np.zeros((n, self.K)) if what & DESC_B else None
        dB = np.zeros((n, self.K * nsp, 3)) if what & DESC_DB else None
        W = np.zeros((self.K * nsp, 6)) if what & DESC_W else None
        self.ctx.check(lib().ipg_snap_descriptors(self._h, n, _vp(system.positions), _vp(sp), _vp(system.L), _vp(B),
                                                  _vp(dB), _vp(W), what))
        return B, (None if dB is None else np.ascontiguousarray(dB.transpose(0, 2, 1))), \
            (None if W is None else np.ascontiguousarray(W.T))

    def energy_forces(self, system, beta, beta0=0.0, mode="adjoint"):
        """E, F (n, 3), W6 for E = beta0 + sum_i beta[s_i] . B_i; beta is (K,) or (nsp, K)."""
        n = len(system)
        beta = self.beta_blocks(beta)
        sp = self.species_ids(system)
        E = np.zeros(1)
        F = np.zeros((n, 3))
        W = np.zeros(6)
        m = SNAP_ADJOINT if mode == "adjoint" else SNAP_PLAIN
        self.ctx.check(lib().ipg_snap_energy_forces(self._h, n, _vp(system.positions), _vp(sp), _vp(system.L),
                                                    _vp(beta), float(beta0), m, _vp(E), _vp(F), _vp(W)))
        return E[0], F, W

    def beta_blocks(self, beta):
        b = np.asarray(beta, dtype=np.float64)
        nsp = len(self.species)
        if b.ndim == 1:
            if b.size != self.K:
                raise ValueError(f"beta must have {self.K} entries (or shape ({nsp}, {self.K}))")
            b = np.tile(b, (nsp, 1))
        if b.shape != (nsp, self.K):
            raise ValueError(f"beta must have shape ({nsp}, {self.K})")
        return np.ascontiguousarray(b)

    def vjp_beta(self, system, gE, gF=None):
        """(d(gE*E + gF.F)/dbeta (nsp, K), d/dbeta0)."""
        n = len(system)
        sp = self.species_ids(system)
        gb = np.zeros((len(self.species), self.K))
        gb0 = np.zeros(1)
        gF = None if gF is None else np.ascontiguousarray(gF, dtype=np.float64).reshape(n, 3)
        self.ctx.check(lib().ipg_snap_vjp_beta(self._h, n, _vp(system.positions), _vp(sp), _vp(system.L),
                                               float(gE), _vp(gF), _vp(gb), _vp(gb0)))
        return gb, gb0[0]

    def vjp(self, system, beta, gE=0.0, gF=None):
        """Pullback of (E, F) (include/ipg.h: ipg_snap_vjp): returns (gbeta (nsp, K), gbeta0,
        gpos (n, 3)) with gpos = d(gE E + gF . F)/dpos = -gE F - H gF."""
        n = len(system)
        sp = self.species_ids(system)
        beta = self.beta_blocks(beta)
        gb = np.zeros((len(self.species), self.K))
        gb0 = np.zeros(1)
        gp = np.zeros((n, 3))
        gF = None if gF is None else np.ascontiguousarray(gF, dtype=np.float64).reshape(n, 3)
        self.ctx.check(lib().ipg_snap_vjp(self._h, n, _vp(system.positions), _vp(sp), _vp(system.L), _vp(beta),
                                          float(gE), _vp(gF), _vp(gb), _vp(gb0), _vp(gp)))
        return gb, gb0[0], gp

    def autotune(self, system, beta, cache_path=None):
        """Picks the fastest kernel configuration for workloads like `system`
        (include/ipg.h: ipg_snap_autotune); returns the choice as a dict."""
        import json
        sp = self.species_ids(system)
        beta = self.beta_blocks(beta)
        buf = C.create_string_buffer(1024)
        path = None if cache_path is None else str(cache_path).encode()
        self.ctx.check(lib().ipg_snap_autotune(self._h, len(system), _vp(system.positions), _vp(sp), _vp(system.L),
                                               _vp(beta), path, buf, len(buf)))
        return json.loads(buf.value.decode())

    # ---- batches ----------------------------------------------------------------------
    def _flatten(self, systems):
        off = np.zeros(len(systems) + 1, np.int64)
        off[1:] = np.cumsum([len(s) for s in systems])
        pos = np.ascontiguousarray(np.concatenate([s.positions for s in systems]).reshape(-1, 3))
        sp = np.ascontiguousarray(np.concatenate([self.species_ids(s) for s in systems]), dtype=np.int32)
        L = np.ascontiguousarray(np.stack([s.L for s in systems]))
        return off, pos, sp, L

    def batch_energy_forces(self, systems, beta, beta0=0.0, mode="adjoint"):
        """Per-configuration E (nconf,), forces (n_total, 3), W6 (nconf, 6)."""
        off, pos, sp, L = self._flatten(systems)
        beta = self.beta_blocks(beta)
        nc = len(systems)
        E = np.zeros(nc)
        F = np.zeros((int(off[-1]), 3))
        W = np.zeros((nc, 6))
        m = SNAP_ADJOINT if mode == "adjoint" else SNAP_PLAIN
        self.ctx.check(lib().ipg_snap_batch_energy_forces(self._h, nc, _vp(off), _vp(pos), _vp(sp), _vp(L),
                                                          _vp(beta), float(beta0), m, _vp(E), _vp(F), _vp(W)))
        return E, F, W

    def set_skin(self, skin):
        """Reuse the neighbor list across calls while atoms move less than skin/2
        (include/ipg.h: ipg_snap_set_skin); 0 builds every call."""
        self.ctx.check(lib().ipg_snap_set_skin(self._h, float(skin)))

    def skin_stats(self):
        """(list builds, list reuses) since the handle was created."""
        b, r = C.c_int64(), C.c_int64()
        self.ctx.check(lib().ipg_snap_skin_stats(self._h, C.byref(b), C.byref(r)))
        return b.value, r.value

    def fitting_matrices(self, systems):
        """The fitting system of many configurations (include/ipg.h: ipg_snap_batch_descriptors):
        energy rows Ae (nconf, K*nsp), force rows Af (3 n_total, K*nsp), virial rows Aw
        (nconf, 6, K*nsp); column s*K + k belongs to species block s."""
        off, pos, sp, L = self._flatten(systems)
        nc, KN = len(systems), self.K * len(self.species)
        Ae = np.zeros((nc, KN))
        Af = np.zeros((3 * int(off[-1]), KN))
        Aw = np.zeros((nc, 6, KN))
        self.ctx.check(lib().ipg_snap_batch_descriptors(self._h, nc, _vp(off), _vp(pos), _vp(sp), _vp(L), _vp(Ae),
                                                        _vp(Af), _vp(Aw)))
        return Ae, Af, Aw

    def batch_loss_grad(self, systems, beta, F_ref, beta0=0.0):
        """L = sum |F - F_ref|^2 over the batch and dL/dbeta (nsp, K)."""
        off, pos, sp, L = self._flatten(systems)
        beta = self.beta_blocks(beta)
        Fr = np.ascontiguousarray(F_ref, dtype=np.float64).reshape(-1, 3)
        loss = np.zeros(1)
        gb = np.zeros((len(self.species), self.K))
        self.ctx.check(lib().ipg_snap_batch_loss_grad(self._h, len(systems), _vp(off), _vp(pos), _vp(sp), _vp(L),
                                                      _vp(beta), float(beta0), _vp(Fr), _vp(loss), _vp(gb)))
        return loss[0], gb


class DeviceBatch:
    """A fixed set of configurations resident on the GPU as torch tensors, evaluated with
    ``ipg_snap_batch_energy_forces_dev``.  With ``graph=True`` the first evaluation is captured
    into a CUDA graph (neighbor build included) and later ones replay it with one launch;
    positions change in place through :meth:`set_positions`, beta per call.  The library runs on
    torch's current stream of the snap's device."""

    def __init__(self, snap, systems):
        import torch
        off, pos, sp, L = snap._flatten(systems)
        self.snap, self.off, self.L = snap, off, L
        self.nconfig = len(systems)
        dev = torch.device("cuda", snap.ctx.device)
        self.pos = torch.tensor(pos, dtype=torch.float64, device=dev)
        self.species = torch.tensor(sp, dtype=torch.int32, device=dev)
        self.E = torch.zeros(self.nconfig, dtype=torch.float64, device=dev)
        self.F = torch.zeros((int(off[-1]), 3), dtype=torch.float64, device=dev)
        self.W = torch.zeros((self.nconfig, 6), dtype=torch.float64, device=dev)
        snap.ctx.set_stream(torch.cuda.current_stream(dev).cuda_stream)

    def set_positions(self, pos):
        import torch
        self.pos.copy_(torch.as_tensor(pos, dtype=torch.float64).reshape(-1, 3))

    def train_step(self, beta, F_ref, beta0=0.0, graph=True):
        """One force-matching training step (``ipg_snap_batch_loss_grad_dev``): fills E, F, W
        and returns the device tensors (loss (1,), dL/dbeta (nsp, K)); with ``graph=True`` the
        whole step is one CUDA-graph launch after the first call.  F_ref: a device tensor
        (n_total, 3) that must stay the same buffer across graph replays."""
        import torch
        beta = self.snap.beta_blocks(beta)
        if not hasattr(self, "loss"):
            dev = self.pos.device
            self.loss = torch.zeros(1, dtype=torch.float64, device=dev)
            self.gbeta = torch.zeros((len(self.snap.species), self.snap.K), dtype=torch.float64, device=dev)
        ptr = lambda t: C.c_void_p(t.data_ptr())
        self.snap.ctx.check(lib().ipg_snap_batch_loss_grad_dev(
            self.snap._h, self.nconfig, _vp(self.off), ptr(self.pos), ptr(self.species), _vp(self.L), _vp(beta),
            float(beta0), ptr(F_ref), int(bool(graph)), ptr(self.E), ptr(self.F), ptr(self.W), ptr(self.loss),
            ptr(self.gbeta)))
        return self.loss, self.gbeta

    def evaluate(self, beta, beta0=0.0, mode="adjoint", graph=True):
        """Fills (and returns) the device tensors E (nconf,), F (n_total, 3), W (nconf, 6)."""
        beta = self.snap.beta_blocks(beta)
        m = SNAP_ADJOINT if mode == "adjoint" else SNAP_PLAIN
        ptr = lambda t: C.c_void_p(t.data_ptr())
        self.snap.ctx.check(lib().ipg_snap_batch_energy_forces_dev(
            self.snap._h, self.nconfig, _vp(self.off), ptr(self.pos), ptr(self.species), _vp(self.L), _vp(beta),
            float(beta0), m, int(bool(graph)), ptr(self.E), ptr(self.F), ptr(self.W)))
        return self.E, self.F, self.W


def compute_local_descriptors(system, snap):
    """snap.jl:103-124 -> B (n, K)."""
    return snap._descriptors(system, DESC_B)[0]


def compute_force_descriptors(system, snap):
    """snap.jl:126-167 (with compute_all_descriptors' U-row indexing) -> dB (n, 3, K*nsp)."""
    return snap._descriptors(system, DESC_DB)[1]


def compute_virial_descriptors(system, snap):
    """The W of compute_all_descriptors (snap.jl:267-285) -> (6, K*nsp)."""
    return snap._descriptors(system, DESC_W)[2]


def compute_all_descriptors(system, snap):
    """snap.jl:226-285 -> (B (n, K), dB (n, 3, K*nsp), W (6, K*nsp))."""
    return snap._descriptors(system, DESC_B | DESC_DB | DESC_W)


class LBasisPotential:
    """src/BasisPotentials/linear_potential.jl:6-16: E = beta0 + (sum_i B_i) . beta.

    beta may be the reference's (K,) vector (applied to every centre species) or an
    (nspecies, K) array of per-species blocks.  `mode` selects the force path:
    "adjoint" (Y / dE/dr) or "plain" (materialised dB/dr).
    """

    def __init__(self, beta, beta0, basis, mode="adjoint"):
        self.beta = np.asarray(beta, dtype=np.float64)
        self.beta0 = np.atleast_1d(np.asarray(beta0, dtype=np.float64))
        self.basis = basis
        self.mode = mode

    def get_rcutoff(self):
        return self.basis.get_rcutoff()

    def get_species(self):
        return self.basis.get_species()

    def get_parameters(self):
        return (self.beta0, self.beta)
