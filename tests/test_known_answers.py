"""Known answers that do not depend on the float64 restatement.

Each case has a closed-form or symmetry answer, checked first on the oracle
(CPU) and then on the CUDA path in both precisions (marked gpu):

1. a plane wave e^{ik.x} with G = 0 drifts to e^{ik.x - i k^2 t / (2 m/hbar)};
2. a Gaussian packet spreads as the free-particle closed form;
3. Poisson of one Fourier mode plus a uniform offset c gives
   V = -4 pi G A cos(k.x) / k^2 - 4 pi G c (the k = 0 mode is divided by 1,
   quantum-stars.py:191-192);
4. rho = rho_bar and constant psi: V = 0 and psi does not change;
5. CIC weights sum to one on each axis and the deposited mass is sum(m);
6. the step is unitary: sum |psi|^2 is conserved to round-off;
7. the MUSCL-Hancock gas update is symmetric under a mirror (x -> -x,
   vx -> -vx) and under swapping two axes (with their velocities).

Tolerances: float64 paths 1e-10 or tighter; float32 paths as stated per test
(rel-L2 against the closed form, which carries the float32 rounding of every
step).
"""

import math

import numpy as np
import pytest

from oracle import oracle as O

TWO_PI = 2.0 * math.pi


def grid(n, L=1.0):
    return O.Grid(n, n, n, L, L, L)


def plane_wave(g, modes):
    X, Y, Z = O.cell_centres(g)
    k = [TWO_PI * m / g.Lx for m in modes]
    return np.exp(1j * (k[0] * X + k[1] * Y + k[2] * Z)), sum(kk * kk for kk in k)


def gaussian_packet(g, sigma, t, m, c=(0.5, 0.5, 0.5)):
    """Free-particle packet, hbar = 1, mass m: the product over axes of
    (2 pi s^2)^(-1/4) (1 + i t / (2 m s^2))^(-1/2) exp(-x^2 / (4 s^2 (1 + i t / (2 m s^2))))."""
    a = 1.0 + 1j * t / (2.0 * m * sigma * sigma)
    out = np.ones(g.shape, dtype=np.complex128)
    for X, cc in zip(O.cell_centres(g), c):
        out = out * (2 * math.pi * sigma * sigma) ** -0.25 * a ** -0.5 * \
            np.exp(-((X - cc) ** 2) / (4.0 * sigma * sigma * a))
    return out


def single_mode(g, p, A, modes, offset):
    X, Y, Z = O.cell_centres(g)
    k = [TWO_PI * m / g.Lx for m in modes]
    ph = k[0] * X + k[1] * Y + k[2] * Z
    rho = p.rho_bar + A * np.cos(ph) + offset
    V = -4.0 * math.pi * p.G * A * np.cos(ph) / sum(kk * kk for kk in k) \
        - 4.0 * math.pi * p.G * offset
    return rho, V


def mirror_x(f, flip=False):
    out = np.ascontiguousarray(f[::-1, :, :])
    return -out if flip else out


def swap_xy(f):
    return np.ascontiguousarray(np.transpose(f, (1, 0, 2)))


# ---------------------------------------------------------------------------
# oracle (CPU)
# ---------------------------------------------------------------------------


def test_oracle_plane_wave_drift():
    g = grid(16)
    p = O.Phys(m_per_hbar=1.7)
    psi0, k2 = plane_wave(g, (1, 2, -3))
    dt = 0.01
    got = O.drift(psi0, g, p, dt)
    want = psi0 * np.exp(-1j * k2 * dt / (2.0 * p.m_per_hbar))
    assert O.rel_l2(got, want) < 1e-12


def test_oracle_gaussian_packet_spreads_as_closed_form():
    # sigma = 0.04 on 64^3: the spectrum at the Nyquist k and the periodic
    # images at the box edge (after spreading to 1.12 sigma) are below 1e-13
    g = grid(64)
    p = O.Phys(m_per_hbar=1.0)
    sigma, t = 0.04, 0.0016
    psi = gaussian_packet(g, sigma, 0.0, p.m_per_hbar)
    for _ in range(4):
        psi = O.drift(psi, g, p, t / 4)
    assert O.rel_l2(psi, gaussian_packet(g, sigma, t, p.m_per_hbar)) < 1e-10


def test_oracle_poisson_single_mode_and_k0_offset():
    g = grid(16)
    p = O.Phys(G=0.7, rho_bar=1.3)
    rho, V = single_mode(g, p, 0.25, (2, -1, 3), 0.05)
    got = O.get_potential(rho, g, p)
    assert np.abs(got - V).max() < 1e-12 * np.abs(V).max()


def test_oracle_uniform_state_is_stationary():
    g = grid(16)
    p = O.Phys(rho_bar=1.2)
    assert np.abs(O.get_potential(np.full(g.shape, p.rho_bar), g, p)).max() == 0.0
    psi = np.full(g.shape, math.sqrt(p.rho_bar), dtype=np.complex128)
    out = O.stars_run(psi, np.zeros((0, 3)), np.zeros((0, 3)), 3, g, p, O.default_dt(g, p))[0]
    assert np.abs(out - psi).max() < 1e-13


def test_oracle_cic_partition_of_unity_and_mass():
    g = grid(16)
    rng = np.random.default_rng(4)
    pos = rng.uniform(0.0, 1.0, (200, 3))
    _, _, w_i, w_ip1 = O.get_cic_indices_and_weights(pos, g)
    assert np.abs(w_i + w_ip1 - 1.0).max() < 1e-12
    masses = rng.uniform(0.5, 2.0, 200)
    rho = O.bin_stars(pos, g, masses)
    assert rho.sum() * g.vol == pytest.approx(masses.sum(), rel=1e-13)


def test_oracle_step_is_unitary():
    psi, pos, vel, g, p = O.stars_ic(16, 8, seed=2)
    n0 = np.sum(np.abs(psi) ** 2)
    out = O.stars_run(psi, pos, vel, 5, g, p, O.default_dt(g, p))[0]
    assert np.sum(np.abs(out) ** 2) == pytest.approx(n0, rel=1e-12)


def _gas_state(n, seed=5):
    rho = 0.3 * (1.0 + 0.2 * O.delta_field(n, seed))
    rng = np.random.default_rng(seed)
    v = [0.1 * rng.standard_normal((n, n, n)) for _ in range(3)]
    return rho, v


def test_oracle_hydro_mirror_and_axis_swap_symmetry():
    n = 16
    dx = 1.0 / n
    dt = 0.2 * dx
    rho, (vx, vy, vz) = _gas_state(n)
    base = O.solve_hydro(rho, vx, vy, vz, dt, dx, 1.0)
    mir = O.solve_hydro(mirror_x(rho), mirror_x(vx, True), mirror_x(vy), mirror_x(vz),
                        dt, dx, 1.0)
    for a, b, flip in zip(base, mir, (False, True, False, False)):
        assert np.abs(mirror_x(a, flip) - b).max() < 1e-13 * max(np.abs(a).max(), 1.0)
    sw = O.solve_hydro(swap_xy(rho), swap_xy(vy), swap_xy(vx), swap_xy(vz), dt, dx, 1.0)
    for a, b in zip((base[0], base[2], base[1], base[3]), sw):
        assert np.abs(swap_xy(a) - b).max() < 1e-13 * max(np.abs(a).max(), 1.0)


# ---------------------------------------------------------------------------
# CUDA path (plain float64 and fused float32)
# ---------------------------------------------------------------------------


def _qj():
    import qj

    return qj


def _plan(g, p, precision, n_s=1):
    qj = _qj()
    return qj.Plan(qj.Grid(g.nx, g.ny, g.nz, g.Lx, g.Ly, g.Lz),
                   qj.Phys(m_per_hbar=p.m_per_hbar, G=p.G, rho_bar=p.rho_bar, b_coeff=p.b_coeff,
                           cs=p.cs, c_light=p.c_light), precision, n_s)


def _precisions():
    qj = _qj()
    # (precision, complex dtype, real dtype, tolerance of a rel-L2 against a closed form)
    import torch

    return ((qj.PLAIN_F64, torch.complex128, torch.float64, 1e-10),
            (qj.FUSED_F32, torch.complex64, torch.float32, 2e-5))


def _evolve(g, p, psi, dt, nsteps, precision, ct, pos=None, vel=None, m_s=0.0):
    import torch

    plan = _plan(g, p, precision, max(1, 0 if pos is None else len(pos)))
    rt = torch.float64 if ct == torch.complex128 else torch.float32
    ps = torch.as_tensor(psi, dtype=ct, device="cuda").contiguous()
    po = ve = None
    if pos is not None:
        po = torch.as_tensor(pos, dtype=rt, device="cuda").contiguous()
        ve = torch.as_tensor(vel, dtype=rt, device="cuda").contiguous()
    diag = torch.tensor([0.0, 0.0, dt], dtype=torch.float64, device="cuda")
    plan.kdk_step(ps, po, ve, diag, dt, nsteps, m_s)
    plan.status()
    out = ps.cpu().numpy().astype(np.complex128)
    plan.close()
    return out


@pytest.mark.gpu
def test_plane_wave_free_evolution():
    g = grid(32)
    p = O.Phys(m_per_hbar=1.7, G=0.0, rho_bar=1.0)
    psi0, k2 = plane_wave(g, (1, 2, -3))
    dt, nsteps = 2.0e-4, 12
    want = psi0 * np.exp(-1j * k2 * dt * nsteps / (2.0 * p.m_per_hbar))
    for prec, ct, _, tol in _precisions():
        assert O.rel_l2(_evolve(g, p, psi0, dt, nsteps, prec, ct), want) < tol


@pytest.mark.gpu
def test_gaussian_packet_spreading():
    g = grid(64)
    p = O.Phys(m_per_hbar=1.0, G=0.0, rho_bar=1.0)
    sigma, dt, nsteps = 0.04, 8.0e-5, 20
    psi0 = gaussian_packet(g, sigma, 0.0, p.m_per_hbar)
    want = gaussian_packet(g, sigma, dt * nsteps, p.m_per_hbar)
    for prec, ct, _, tol in _precisions():
        assert O.rel_l2(_evolve(g, p, psi0, dt, nsteps, prec, ct), want) < tol


@pytest.mark.gpu
def test_poisson_single_mode_and_k0_offset():
    import torch

    g = grid(32)
    p = O.Phys(G=0.7, rho_bar=1.3)
    rho, V = single_mode(g, p, 0.25, (2, -1, 3), 0.05)
    for prec, _, rt, _ in _precisions():
        plan = _plan(g, p, prec)
        got = plan.get_potential(torch.as_tensor(rho, dtype=rt, device="cuda").contiguous())
        plan.status()
        err = np.abs(got.cpu().numpy() - V).max() / np.abs(V).max()
        plan.close()
        assert err < (1e-12 if rt == torch.float64 else 2e-6)


@pytest.mark.gpu
def test_uniform_state_is_stationary():
    g = grid(32)
    p = O.Phys(rho_bar=1.2)
    psi = np.full(g.shape, math.sqrt(p.rho_bar), dtype=np.complex128)
    dt = O.default_dt(g, p)
    for prec, ct, _, _ in _precisions():
        out = _evolve(g, p, psi, dt, 5, prec, ct)
        assert np.abs(out - psi).max() < (1e-13 if ct.itemsize == 16 else 1e-6)


@pytest.mark.gpu
def test_cic_partition_of_unity_and_mass():
    import torch

    g = grid(32)
    p = O.Phys()
    rng = np.random.default_rng(4)
    pos = rng.uniform(0.0, 1.0, (300, 3))
    masses = rng.uniform(0.5, 2.0, 300)
    for prec, _, rt, _ in _precisions():
        plan = _plan(g, p, prec, 300)
        rho = plan.bin_stars(torch.as_tensor(pos, dtype=rt, device="cuda").contiguous(),
                             masses=torch.as_tensor(masses, dtype=rt, device="cuda"))
        plan.status()
        total = rho.double().sum().item() * g.vol
        plan.close()
        assert total == pytest.approx(masses.sum(), rel=1e-12 if rt == torch.float64 else 2e-6)


@pytest.mark.gpu
def test_step_is_unitary():
    psi, pos, vel, g, p = O.stars_ic(32, 64, seed=2)
    n0 = np.sum(np.abs(psi) ** 2)
    dt = O.default_dt(g, p)
    for prec, ct, _, _ in _precisions():
        out = _evolve(g, p, psi, dt, 20, prec, ct, pos, vel, p.m_s)
        tol = 1e-12 if ct.itemsize == 16 else 2e-6
        assert np.sum(np.abs(out) ** 2) == pytest.approx(n0, rel=tol)


def _gas_step(g, p, precision, psi, rho, v, dt, nsteps):
    import torch

    qj = _qj()
    dbl = precision == qj.PLAIN_F64
    ct = torch.complex128 if dbl else torch.complex64
    rt = torch.float64 if dbl else torch.float32
    plan = _plan(g, p, precision, 1)

    def c(a, t):
        return torch.as_tensor(np.ascontiguousarray(a), dtype=t, device="cuda")

    # a black hole of zero mass at the box centre: no accretion, no density
    T = [c(psi, ct), c(rho, rt), c(v[0], rt), c(v[1], rt), c(v[2], rt), c(np.zeros(1), rt),
         c(np.full((1, 3), 0.5), rt), c(np.zeros((1, 3)), rt)]
    plan.kdk_gas_bh(*T, dt, nsteps, 0.0, dm_accretion=False)
    plan.status()
    out = [x.cpu().numpy().astype(np.float64 if x.dtype != ct else np.complex128) for x in T[:5]]
    plan.close()
    return out


@pytest.mark.gpu
def test_gas_step_mirror_and_axis_swap_symmetry():
    qj = _qj()
    n = 32
    g = grid(n)
    rho_dm = 1.0 + 0.1 * O.delta_field(n, 7)
    psi = np.sqrt(rho_dm).astype(np.complex128)
    rho, v = _gas_state(n)
    p = O.Phys(m_per_hbar=1.0, G=1.0 / (4.0 * math.pi), rho_bar=float(rho_dm.mean()), cs=1.0,
               c_light=0.3)
    dt = min(g.dx ** 2 / 6.0, 0.3 * g.dx / 1.5)
    # rel-L2 bars: psi and gas density at tol, the (small) velocities at 10 tol
    scale = (1, 1, 10, 10, 10)
    for prec, tol in ((qj.PLAIN_F64, 1e-11), (qj.FUSED_F32, 1e-5)):
        base = _gas_step(g, p, prec, psi, rho, v, dt, 3)
        mir = _gas_step(g, p, prec, mirror_x(psi), mirror_x(rho),
                        [mirror_x(v[0], True), mirror_x(v[1]), mirror_x(v[2])], dt, 3)
        for a, b, flip, sc in zip(base, mir, (False, False, True, False, False), scale):
            assert O.rel_l2(mirror_x(a, flip), b) < tol * sc
        sw = _gas_step(g, p, prec, swap_xy(psi), swap_xy(rho), [swap_xy(v[1]), swap_xy(v[0]),
                                                                 swap_xy(v[2])], dt, 3)
        for a, b, sc in zip((base[0], base[1], base[3], base[2], base[4]), sw, scale):
            assert O.rel_l2(swap_xy(a), b) < tol * sc
