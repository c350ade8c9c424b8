"""The torch float64 mirror (the gradient oracle) reproduces the float64
oracle's psi-only step, which is pinned to the reference's own functions."""

import numpy as np
import torch

from oracle import oracle as O
from oracle import torch_mirror as TM


def test_mirror_matches_oracle_forward():
    psi, pos, vel, g, p = O.stars_ic(16, 0, seed=0, shape=(16, 32, 16), L=(1.0, 2.0, 1.0))
    p.b_coeff = -0.1
    dt = O.default_dt(g, p)
    k = TM.kgrid(g.shape, (g.Lx, g.Ly, g.Lz))
    a = TM.kdk(torch.as_tensor(psi), k, p.G, p.rho_bar, p.m_per_hbar, dt, 3, p.b_coeff).numpy()
    b = O.stars_run(psi, pos, vel, 3, g, p, dt, self_interaction=True)[0]
    assert O.rel_l2(a, b) < 1e-13


def test_mirror_gradient_matches_finite_difference():
    psi, _, _, g, p = O.stars_ic(8, 0, seed=2, shape=(16, 16, 16))
    dt = O.default_dt(g, p)
    k = TM.kgrid(g.shape, (1.0, 1.0, 1.0))
    s = np.abs(psi)
    th = 0.3 * O.delta_field(16, 5)
    tgt = np.abs(psi) ** 2 * 1.01
    L0, gr = TM.loss_and_grad(th, s, tgt, k, p.G, p.rho_bar, p.m_per_hbar, dt, 2)
    d = np.random.default_rng(0).standard_normal(th.shape)
    eps = 1e-5
    Lp, _ = TM.loss_and_grad(th + eps * d, s, tgt, k, p.G, p.rho_bar, p.m_per_hbar, dt, 2)
    Lm, _ = TM.loss_and_grad(th - eps * d, s, tgt, k, p.G, p.rho_bar, p.m_per_hbar, dt, 2)
    assert (Lp - Lm) / (2 * eps) == __import__("pytest").approx(float(np.sum(gr * d)), rel=1e-6)


def test_mirror_with_fixed_star_density_matches_oracle_functions():
    """With the stars held fixed, their CIC density rho_s enters every kick's
    potential (quantum-stars.py:298-301, :315-318); the mirror's step with
    rho_s equals the oracle's get_potential / kick / drift composed the same
    way."""
    psi, pos, vel, g, p = O.stars_ic(16, 40, seed=3, shape=(16, 32, 16), L=(1.0, 2.0, 1.0))
    p.b_coeff = -0.1
    dt = O.default_dt(g, p)
    rho_s = O.bin_stars(pos, g, np.full(len(pos), p.m_s))
    k = TM.kgrid(g.shape, (g.Lx, g.Ly, g.Lz))
    a = TM.kdk(torch.as_tensor(psi), k, p.G, p.rho_bar, p.m_per_hbar, dt, 2, p.b_coeff,
               rho_s=torch.as_tensor(rho_s)).numpy()
    kk = O.kgrid(g)
    b = psi
    for _ in range(2):
        b = O.kick(b, O.get_potential(np.abs(b) ** 2 + rho_s, g, p, kk, True), p, dt)
        b = O.drift(b, g, p, dt, kk)
        b = O.kick(b, O.get_potential(np.abs(b) ** 2 + rho_s, g, p, kk, True), p, dt)
    assert O.rel_l2(a, b) < 1e-13
