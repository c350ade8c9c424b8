"""Gradient of the KDK step through torch.autograd (libqj's adjoint sweep).

The reference states that the solver is differentiable (README.md:7) but no
script calls jax.grad; this provides the gradient path for the step with the
particles as a fixed source (quantum-stars.py:295-330 with the star density
rho_s held fixed, quantum-tidal.py:186-207 with a static V_ext):
``kdk_evolve(theta, sqrt_rho, plan, dt, nsteps, K)`` maps the initial phase
field theta and amplitude sqrt(rho) to psi_T and backpropagates with libqj's
checkpointed adjoint (ckpt every K steps, recompute in between).
"""

from __future__ import annotations

import torch

from ._lib import check, lib
from .core import _ptr, _stream


def _nseg(nsteps, K):
    return (nsteps + K - 1) // K


class KDKEvolve(torch.autograd.Function):
    """psi_T = KDK^nsteps(sqrt_rho * exp(i theta))."""

    @staticmethod
    def forward(ctx, theta, sqrt_rho, plan, dt, nsteps, K, self_interaction=False, v_ext=None,
                rho_s=None):
        psi = (sqrt_rho.to(plan.rdtype) * torch.exp(1j * theta.to(plan.rdtype))).to(plan.cdtype)
        psi = psi.contiguous()
        plan._field(psi, "psi", complex_=True)
        for t, name in ((v_ext, "v_ext"), (rho_s, "rho_s")):
            if t is not None:
                plan._field(t, name)
        ckpt = torch.empty((_nseg(nsteps, K),) + plan.grid.shape, dtype=plan.cdtype,
                           device=psi.device)
        check(lib().qj_kdk_forward_ckpt(plan._h, _ptr(psi), int(nsteps), int(K), _ptr(ckpt),
                                        float(dt), int(bool(self_interaction)), _ptr(v_ext),
                                        _ptr(rho_s), _stream()))
        ctx.save_for_backward(theta, sqrt_rho, ckpt)
        ctx.plan, ctx.dt, ctx.nsteps, ctx.K = plan, dt, nsteps, K
        ctx.si, ctx.v_ext, ctx.rho_s = self_interaction, v_ext, rho_s
        return psi

    @staticmethod
    def backward(ctx, grad_psi):
        theta, sqrt_rho, ckpt = ctx.saved_tensors
        plan = ctx.plan
        g = grad_psi.to(plan.cdtype).contiguous().clone()
        check(lib().qj_kdk_adjoint(plan._h, _ptr(ckpt), _ptr(g), int(ctx.nsteps), int(ctx.K),
                                   float(ctx.dt), int(bool(ctx.si)), _ptr(ctx.v_ext),
                                   _ptr(ctx.rho_s), _stream()))
        # psi_0 = s exp(i theta): dL/dtheta = Re(conj(g) i psi_0), dL/ds = Re(conj(g) e^{i theta})
        e = torch.exp(1j * theta.to(plan.rdtype)).to(plan.cdtype)
        psi0 = sqrt_rho.to(plan.rdtype) * e
        g_theta = -(torch.conj(g) * psi0).imag
        g_s = (torch.conj(g) * e).real
        return (g_theta.to(theta.dtype), g_s.to(sqrt_rho.dtype), None, None, None, None, None,
                None, None)


def kdk_evolve(theta, sqrt_rho, plan, dt, nsteps, K=20, self_interaction=False, v_ext=None,
               rho_s=None):
    """psi_T after nsteps KDK steps from psi_0 = sqrt_rho exp(i theta); rho_s is
    an optional fixed density (e.g. the stars' CIC density) added to |psi|^2."""
    return KDKEvolve.apply(theta, sqrt_rho, plan, dt, nsteps, K, self_interaction, v_ext, rho_s)
