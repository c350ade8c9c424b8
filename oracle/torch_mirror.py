"""Torch float64 (CPU) mirror of the KDK step, for gradients.

TEST INFRASTRUCTURE ONLY (like oracle.py).  The reference's gradient would
be jax.grad of its step (quantum-stars.py:295-330, or quantum-tidal.py:186-207);
JAX is absent, so this mirror restates the same step op for op in torch
float64 and lets torch.autograd differentiate it.  kdk is the step with the
stars' density as a fixed source (or none); kdk_stars (below) moves the
stars and differentiates through their deposit, interpolation and leapfrog:

    rho = |psi|^2 (+ rho_s, a fixed star density, :298-299)
    V = Re ifftn(-fftn(4 pi G (rho - rho_bar)) / (k^2 + [k^2 == 0]))
                        (+ b rho) (+ V_ext)                       (:189-193)
    psi <- exp(-1j m_per_hbar dt / 2 V) psi                        (:301)
    psi <- ifftn(exp(dt (-1j k^2 / m_per_hbar / 2)) fftn(psi))     (:307-309)
    psi <- kick again                                              (:318)
"""

from __future__ import annotations

import math

import numpy as np
import torch


def kgrid(shape, L):
    ks = [torch.as_tensor(np.fft.ifftshift(2.0 * np.pi / l * np.arange(-n / 2, n / 2)))
          for n, l in zip(shape, L)]
    kx, ky, kz = torch.meshgrid(*ks, indexing="ij")
    return kx**2 + ky**2 + kz**2


def potential(rho, k_sq, G, rho_bar, b_coeff=0.0, v_ext=None):
    Vh = -torch.fft.fftn(4.0 * math.pi * G * (rho - rho_bar)) / (k_sq + (k_sq == 0))
    V = torch.real(torch.fft.ifftn(Vh))
    if b_coeff:
        V = V + b_coeff * rho
    if v_ext is not None:
        V = V + v_ext
    return V


def kdk(psi, k_sq, G, rho_bar, m_per_hbar, dt, nsteps, b_coeff=0.0, v_ext=None, rho_s=None):
    prop = torch.exp(dt * (-1j * k_sq / m_per_hbar / 2.0))
    src = 0.0 if rho_s is None else rho_s
    for _ in range(nsteps):
        V = potential(torch.abs(psi) ** 2 + src, k_sq, G, rho_bar, b_coeff, v_ext)
        psi = torch.exp(-1j * m_per_hbar * dt / 2.0 * V) * psi
        psi = torch.fft.ifftn(prop * torch.fft.fftn(psi))
        V = potential(torch.abs(psi) ** 2 + src, k_sq, G, rho_bar, b_coeff, v_ext)
        psi = torch.exp(-1j * m_per_hbar * dt / 2.0 * V) * psi
    return psi


def loss_and_grad(theta, sqrt_rho, rho_tgt, k_sq, G, rho_bar, m_per_hbar, dt, nsteps,
                  b_coeff=0.0, v_ext=None, rho_s=None):
    """L = mean((|psi_T|^2 - rho_tgt)^2) and dL/dtheta (float64 numpy)."""
    th = torch.as_tensor(theta, dtype=torch.float64).requires_grad_(True)
    s = torch.as_tensor(sqrt_rho, dtype=torch.float64)
    psi = s * torch.exp(1j * th)
    psiT = kdk(psi, k_sq, G, rho_bar, m_per_hbar, dt, nsteps, b_coeff,
               None if v_ext is None else torch.as_tensor(v_ext),
               None if rho_s is None else torch.as_tensor(rho_s))
    L = torch.mean((torch.abs(psiT) ** 2 - torch.as_tensor(rho_tgt)) ** 2)
    L.backward()
    return float(L.detach()), th.grad.numpy()


# ---------------------------------------------------------------------------
# The step with moving stars, differentiable through them (quantum-stars.py
# :200-288 and :295-330): CIC weights are linear in the positions (the cell
# index is a floor, with zero derivative), the deposit and the interpolation
# are sums over the eight corners in the reference's order, and the leapfrog
# and the periodic wrap (jnp.mod, derivative 1) are plain arithmetic.  This is
# what jax.grad of the reference's compute_step differentiates.
# ---------------------------------------------------------------------------

_CORNERS = ((0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0), (1, 0, 1), (0, 1, 1), (1, 1, 1))


def _kvecs(shape, L):
    return [torch.as_tensor(np.fft.ifftshift(2.0 * np.pi / l * np.arange(-n / 2, n / 2)))
            for n, l in zip(shape, L)]


def cic_corners(pos, shape, L):
    """[(flat cell index, weight)] of the eight corners (quantum-stars.py:200-209)."""
    dxs = torch.tensor([L[a] / shape[a] for a in range(3)], dtype=torch.float64)
    i = torch.floor((pos - 0.5 * dxs) / dxs).detach()
    ip1 = i + 1.0
    w_i = ((ip1 + 0.5) * dxs - pos) / dxs
    w_ip1 = (pos - (i + 0.5) * dxs) / dxs
    n = torch.tensor(shape)
    i = torch.remainder(i, n).long()
    ip1 = torch.remainder(ip1, n).long()
    out = []
    for cx, cy, cz in _CORNERS:
        ix = ip1[:, 0] if cx else i[:, 0]
        iy = ip1[:, 1] if cy else i[:, 1]
        iz = ip1[:, 2] if cz else i[:, 2]
        w = ((w_ip1[:, 0] if cx else w_i[:, 0]) * (w_ip1[:, 1] if cy else w_i[:, 1])
             * (w_ip1[:, 2] if cz else w_i[:, 2]))
        out.append(((ix * shape[1] + iy) * shape[2] + iz, w))
    return out


def bin_stars(pos, m_s, shape, L):
    """CIC density of the stars (quantum-stars.py:212-247)."""
    vol = L[0] * L[1] * L[2] / (shape[0] * shape[1] * shape[2])
    rho = torch.zeros(shape[0] * shape[1] * shape[2], dtype=torch.float64)
    for flat, w in cic_corners(pos, shape, L):
        rho = rho.index_add(0, flat, w * (m_s / vol))
    return rho.reshape(shape)


def star_acceleration(pos, rho, ks, k_sq, G, rho_bar, shape, L):
    """The grid accelerations interpolated to the stars (quantum-stars.py:250-288)."""
    Vh = -torch.fft.fftn(4.0 * math.pi * G * (rho - rho_bar)) / (k_sq + (k_sq == 0))
    kg = torch.meshgrid(*ks, indexing="ij")
    a = [-torch.real(torch.fft.ifftn(1j * kd * Vh)).reshape(-1) for kd in kg]
    acc = torch.zeros_like(pos)
    for flat, w in cic_corners(pos, shape, L):
        acc = acc + w[:, None] * torch.stack([ad[flat] for ad in a], dim=1)
    return acc


def kdk_stars(psi, pos, vel, shape, L, G, rho_bar, m_per_hbar, m_s, dt, nsteps, moving=True):
    """nsteps of compute_step (quantum-stars.py:295-330) -> (psi, pos, vel).
    moving=False holds the stars' density at its initial value in every kick
    and leaves the stars where they are (the fixed-source model)."""
    k_sq = kgrid(shape, L)
    ks = _kvecs(shape, L)
    prop = torch.exp(dt * (-1j * k_sq / m_per_hbar / 2.0))
    box = torch.tensor(L, dtype=torch.float64)
    rho_fixed = None if moving else bin_stars(pos, m_s, shape, L).detach()
    for _ in range(nsteps):
        for first in (True, False):
            rho_s = bin_stars(pos, m_s, shape, L) if moving else rho_fixed
            rho_tot = torch.abs(psi) ** 2 + rho_s
            psi = torch.exp(-1j * m_per_hbar * dt / 2.0 * potential(rho_tot, k_sq, G, rho_bar)) * psi
            if moving:
                vel = vel + star_acceleration(pos, rho_tot, ks, k_sq, G, rho_bar, shape, L) * dt / 2.0
            if first:
                psi = torch.fft.ifftn(prop * torch.fft.fftn(psi))
                if moving:
                    pos = torch.remainder(pos + vel * dt, box)
    return psi, pos, vel


def loss_and_grad_stars(theta, sqrt_rho, pos, vel, rho_tgt, shape, L, G, rho_bar, m_per_hbar, m_s,
                        dt, nsteps, moving=True):
    """L = mean((|psi_T|^2 - rho_tgt)^2) of the step with stars and dL/dtheta
    (float64 numpy), differentiated through the stars when moving."""
    th = torch.as_tensor(theta, dtype=torch.float64).requires_grad_(True)
    psi = torch.as_tensor(sqrt_rho, dtype=torch.float64) * torch.exp(1j * th)
    psiT, _, _ = kdk_stars(psi, torch.as_tensor(pos, dtype=torch.float64),
                           torch.as_tensor(vel, dtype=torch.float64), shape, L, G, rho_bar,
                           m_per_hbar, m_s, dt, nsteps, moving)
    loss = torch.mean((torch.abs(psiT) ** 2 - torch.as_tensor(rho_tgt)) ** 2)
    loss.backward()
    return float(loss.detach()), th.grad.numpy()
