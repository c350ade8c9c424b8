"""Torch float64 (CPU) mirror of the psi-only KDK step, for gradients.

TEST INFRASTRUCTURE ONLY (like oracle.py).  The reference's gradient would
be jax.grad of its step (quantum-stars.py:295-330 without stars, or
quantum-tidal.py:186-207); JAX is absent, so this mirror restates the same
step op for op in torch float64 and lets torch.autograd differentiate it:

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
