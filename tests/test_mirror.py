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


def test_mirror_with_moving_stars_matches_oracle_forward():
    """The mirror's step with moving stars (CIC deposit, interpolation,
    leapfrog) equals the oracle's compute_step (quantum-stars.py:295-330)."""
    psi, pos, vel, g, p = O.stars_ic(16, 40, seed=3, shape=(16, 32, 16), L=(1.0, 2.0, 1.0))
    vel = np.random.default_rng(4).standard_normal(pos.shape)  # stars that cross cells
    dt = O.default_dt(g, p)
    L = (g.Lx, g.Ly, g.Lz)
    a = TM.kdk_stars(torch.as_tensor(psi), torch.as_tensor(pos), torch.as_tensor(vel), g.shape, L,
                     p.G, p.rho_bar, p.m_per_hbar, p.m_s, dt, 3)
    b = O.stars_run(psi, pos, vel, 3, g, p, dt)
    for x, y in zip(a, b[:3]):
        assert O.rel_l2(x.numpy(), y) < 1e-12


def test_mirror_moving_stars_gradient_matches_finite_difference():
    """dL/dtheta through the moving stars against central differences."""
    psi, pos, vel, g, p = O.stars_ic(16, 24, seed=6)
    vel = 3.0 * np.random.default_rng(7).standard_normal(pos.shape)
    dt = O.default_dt(g, p)
    L = (g.Lx, g.Ly, g.Lz)
    s = np.abs(psi)
    th = 0.3 * O.delta_field(16, 5)
    tgt = np.abs(psi) ** 2 * 1.01
    args = (pos, vel, tgt, g.shape, L, p.G, p.rho_bar, p.m_per_hbar, p.m_s, dt, 4)
    _, gr = TM.loss_and_grad_stars(th, s, *args)
    d = np.random.default_rng(0).standard_normal(th.shape)
    eps = 1e-5
    Lp, _ = TM.loss_and_grad_stars(th + eps * d, s, *args)
    Lm, _ = TM.loss_and_grad_stars(th - eps * d, s, *args)
    assert (Lp - Lm) / (2 * eps) == __import__("pytest").approx(float(np.sum(gr * d)), rel=1e-6)


def test_star_motion_term_of_the_gradient_is_negligible_for_the_ic_family():
    """The libqj adjoint differentiates the step with the stars' density as a
    fixed source.  For the IC family (stars at rest, 10 % of the mass), over
    200 steps at 32^3 (T = 0.033, 16 times the 128^3, 200-step horizon), the
    gradient through the moving stars (the whole step, as jax.grad would
    take it) equals the fixed-source gradient to rel-L2 3e-9: the stars move
    3e-5 of the box."""
    n, n_s, steps = 32, 64, 200
    psi, pos, vel, g, p = O.stars_ic(n, n_s, seed=0)
    dt = O.default_dt(g, p)
    L = (g.Lx, g.Ly, g.Lz)
    psi2, pos2, vel2, *_ = O.stars_ic(n, n_s, seed=1)
    with torch.no_grad():
        tgt = (torch.abs(TM.kdk_stars(torch.as_tensor(psi2), torch.as_tensor(pos2),
                                      torch.as_tensor(vel2), g.shape, L, p.G, p.rho_bar,
                                      p.m_per_hbar, p.m_s, dt, steps)[0]) ** 2).numpy()
    s = np.abs(psi)
    th = 0.5 * O.delta_field(n, 21)
    args = (pos, vel, tgt, g.shape, L, p.G, p.rho_bar, p.m_per_hbar, p.m_s, dt, steps)
    L_mov, g_mov = TM.loss_and_grad_stars(th, s, *args, moving=True)
    L_fix, g_fix = TM.loss_and_grad_stars(th, s, *args, moving=False)
    # the fixed-source mirror is the one the adjoint tests pin libqj to
    rho_s = O.bin_stars(pos, g, np.full(n_s, p.m_s))
    L_tm, g_tm = TM.loss_and_grad(th, s, tgt, TM.kgrid(g.shape, L), p.G, p.rho_bar, p.m_per_hbar,
                                  dt, steps, rho_s=rho_s)
    assert O.rel_l2(g_fix, g_tm) < 1e-12
    assert L_fix == __import__("pytest").approx(L_mov, rel=1e-8)
    assert O.rel_l2(g_fix, g_mov) < 1e-6
