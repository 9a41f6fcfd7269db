"""torch.autograd wrapper over the C ABI for sensitivities of the solve.

``SnapSolve.apply(t_xs, qi, snap, dprob, epsi)`` returns the converged scalar
flux [G, C] of the steady-state solve with total cross section ``t_xs``
[G, C] and fixed source ``qi`` [G, C]; its backward runs
``snap_adjoint_solve`` (the hand-written adjoint sweep) with the incoming
gradient as the response, so for J = (w * flux).sum() it returns dJ/dt_xs and
dJ/dqi per cell and group.  The scattering tables stay fixed (their
sensitivity is ``Snap.adjoint_solve``'s grad_sxs).
"""
from __future__ import annotations

import torch


class SnapSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, t_xs, qi, snap, dprob, epsi=None):
        flux, rec = snap.solve_with_txs(dprob, t_xs.detach(), qi.detach(), epsi=epsi)
        ctx.snap, ctx.dprob, ctx.epsi, ctx.rec = snap, dprob, epsi, rec
        ctx.save_for_backward(t_xs.detach(), qi.detach(), flux)
        return flux[..., 0].clone()

    @staticmethod
    def backward(ctx, grad_phi):
        t_xs, qi, flux = ctx.saved_tensors
        dprob = dict(ctx.dprob, qi=qi.contiguous())
        g = ctx.snap.adjoint_solve(dprob, t_xs, flux, grad_phi.contiguous().double(),
                                   epsi=ctx.epsi)
        return g["grad_sigt"], g["grad_qi"], None, None, None
