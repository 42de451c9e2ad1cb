"""PyTorch autograd bindings: the torch counterpart of the ChainRulesCore.rrule methods the
Julia shim defines for the same library calls.

``snap_energy_forces(snap, system, positions, beta, beta0)`` returns (E, F) as tensors that
carry gradients to ``positions`` (n, 3) and ``beta`` (nsp, K): the pullback is
``ipg_snap_vjp`` (include/ipg.h), i.e. dE/dbeta = sum_i B_i, dE/dpos = -F, and the force
cotangent through dF/dbeta (exact, linear in beta) and -H gF (exact: the directional
derivative of the adjoint force computation along gF, a second-order adjoint).  ``snap_loss`` is the force-matching loss
L = sum |F - F_ref|^2 over a batch with its exact beta gradient (``ipg_snap_batch_loss_grad``).
"""
from __future__ import annotations

import numpy as np

from .system import System


def _torch():
    import torch
    return torch


class _SnapEF:
    """Holder for the autograd.Function subclass (built lazily so that torch stays optional)."""
    fn = None


def _make_fn():
    torch = _torch()

    class SnapEnergyForces(torch.autograd.Function):
        @staticmethod
        def forward(ctx, positions, beta, beta0, snap, system):
            pos = positions.detach().cpu().numpy().astype(np.float64).reshape(-1, 3)
            b = beta.detach().cpu().numpy().astype(np.float64)
            sysx = System(pos, system.symbols, system.box, system.periodic)
            E, F, _ = snap.energy_forces(sysx, b, float(beta0), mode="adjoint")
            ctx.snap, ctx.system, ctx.beta = snap, sysx, b
            ctx.beta_shape = tuple(beta.shape)
            ctx.device, ctx.dtype = positions.device, positions.dtype
            return (torch.tensor(E, dtype=positions.dtype, device=positions.device),
                    torch.tensor(F, dtype=positions.dtype, device=positions.device))

        @staticmethod
        def backward(ctx, gE, gF):
            gE_ = 0.0 if gE is None else float(gE.detach().cpu())
            gF_ = None if gF is None else gF.detach().cpu().numpy().astype(np.float64).reshape(-1, 3)
            if gF_ is not None and not np.any(gF_):
                gF_ = None
            gb, gb0, gp = ctx.snap.vjp(ctx.system, ctx.beta, gE_, gF_)
            if len(ctx.beta_shape) == 1:  # a single K-vector shared by every species block
                gb = gb.sum(axis=0)
            t = lambda a: torch.tensor(a, dtype=ctx.dtype, device=ctx.device)
            return t(gp), t(gb).reshape(ctx.beta_shape), t(gb0), None, None

    return SnapEnergyForces


def snap_energy_forces(snap, system, positions, beta, beta0=0.0):
    """(E, F) of LBasisPotential(beta, beta0, snap) at `positions` (a tensor that may require
    grad); beta is a (K,) or (nsp, K) tensor."""
    torch = _torch()
    if _SnapEF.fn is None:
        _SnapEF.fn = _make_fn()
    b0 = beta0 if torch.is_tensor(beta0) else torch.tensor(float(beta0), dtype=torch.float64)
    return _SnapEF.fn.apply(positions, beta, b0, snap, system)


def snap_loss(snap, systems, beta, F_ref):
    """Force-matching loss sum |F - F_ref|^2 over a batch; differentiable in beta (nsp, K)."""
    torch = _torch()

    class SnapLoss(torch.autograd.Function):
        @staticmethod
        def forward(ctx, b):
            loss, g = snap.batch_loss_grad(systems, b.detach().cpu().numpy().astype(np.float64),
                                           np.asarray(F_ref, dtype=np.float64))
            ctx.g = torch.tensor(g, dtype=b.dtype, device=b.device).reshape(b.shape if b.dim() == 2 else g.shape)
            ctx.single = b.dim() == 1
            return torch.tensor(loss, dtype=b.dtype, device=b.device)

        @staticmethod
        def backward(ctx, gl):
            g = ctx.g.sum(dim=0) if ctx.single else ctx.g
            return gl * g

    return SnapLoss.apply(beta)
