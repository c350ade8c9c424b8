"""CPU oracle for the quantum-jax kick-drift-kick Schroedinger-Poisson step.

TEST INFRASTRUCTURE ONLY.  This module is the float64 NumPy/SciPy restatement
of the reference's step functions, op for op, used as the correctness checker,
plus the stars step in the reference's own complex64 / float32 precision
(``stars_compute_step_f32``), the CPU baseline's timed step.
Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
may import it; the product path (``qj``) never does and has no CPU fallback.

Parity pin: ``tests/golden/make_golden.py`` executes the reference scripts'
own functions (quantum-stars.py, quantum-gas-bh.py, quantum-tidal.py,
quantum-cosmo.py, quantum-fluid-accretion-test.py) on a float64 NumPy stand-in
for ``jax.numpy`` (JAX itself is not installable here) and stores their outputs
under ``tests/golden``.  ``tests/test_oracle_golden.py`` checks this module
against those fixtures.  The pin covers the algorithm (k-grid, k=0 handling,
Nyquist sign, CIC weights and order, limiter, fluxes, accretion formulas), not
XLA's float32 rounding, which cannot be run here.

Every function cites the reference lines it restates.  Arrays are C-order
``[nx][ny][nz]`` (z fastest), as built by ``meshgrid(..., indexing="ij")``.
"""

from __future__ import annotations

import dataclasses
import math
import os

import numpy as np

try:  # scipy's pocketfft is threaded; numpy's is the fallback
    import scipy.fft as _sfft

    def _fftn(a, workers):
        return _sfft.fftn(a, workers=workers)

    def _ifftn(a, workers):
        return _sfft.ifftn(a, workers=workers)

except ImportError:  # pragma: no cover
    def _fftn(a, workers):
        return np.fft.fftn(a)

    def _ifftn(a, workers):
        return np.fft.ifftn(a)


WORKERS = int(os.environ.get("QJ_ORACLE_WORKERS", "1"))


# ---------------------------------------------------------------------------
# Configuration (the reference keeps these as module globals,
# quantum-stars.py:61-157, quantum-gas-bh.py:46-133)
# ---------------------------------------------------------------------------


@dataclasses.dataclass
class Grid:
    nx: int
    ny: int
    nz: int
    Lx: float
    Ly: float
    Lz: float

    @property
    def shape(self):
        return (self.nx, self.ny, self.nz)

    @property
    def dx(self):
        return self.Lx / self.nx

    @property
    def dy(self):
        return self.Ly / self.ny

    @property
    def dz(self):
        return self.Lz / self.nz

    @property
    def vol(self):
        return self.dx * self.dy * self.dz

    @property
    def ncell(self):
        return self.nx * self.ny * self.nz


@dataclasses.dataclass
class Phys:
    m_per_hbar: float = 1.0
    G: float = 1.0 / (4.0 * math.pi)
    rho_bar: float = 1.0
    b_coeff: float = 0.0  # self-interaction, quantum-stars.py:117-125
    m_s: float = 0.0  # star particle mass, quantum-stars.py:115
    cs: float = 1.0  # gas sound speed, quantum-gas-bh.py:74
    c_light: float = 299792.458  # quantum-gas-bh.py:86


# ---------------------------------------------------------------------------
# R1: Fourier grid, quantum-stars.py:142-149
# ---------------------------------------------------------------------------


def k_lin(n: int, L: float) -> np.ndarray:
    """ifftshift(2 pi / L * arange(-n/2, n/2)): index n/2 holds -pi n / L."""
    return np.fft.ifftshift(2.0 * np.pi / L * np.arange(-n / 2, n / 2))


def kgrid(g: Grid):
    kx, ky, kz = np.meshgrid(
        k_lin(g.nx, g.Lx), k_lin(g.ny, g.Ly), k_lin(g.nz, g.Lz), indexing="ij"
    )
    k_sq = kx**2 + ky**2 + kz**2
    return kx, ky, kz, k_sq


def cell_centres(g: Grid):
    """quantum-stars.py:136-139."""
    x = np.linspace(0.5 * g.dx, g.Lx - 0.5 * g.dx, g.nx)
    y = np.linspace(0.5 * g.dy, g.Ly - 0.5 * g.dy, g.ny)
    z = np.linspace(0.5 * g.dz, g.Lz - 0.5 * g.dz, g.nz)
    return np.meshgrid(x, y, z, indexing="ij")


# ---------------------------------------------------------------------------
# R2: Poisson, quantum-stars.py:189-193
# ---------------------------------------------------------------------------


def get_potential(rho, g: Grid, p: Phys, k=None, self_interaction=False):
    """V = Re ifftn(-fftn(4 pi G (rho - rho_bar)) / (k^2 + [k^2 == 0]))."""
    k_sq = (k if k is not None else kgrid(g))[3]
    V_hat = -_fftn(4.0 * np.pi * p.G * (rho - p.rho_bar), WORKERS) / (
        k_sq + (k_sq == 0)
    )
    V = np.real(_ifftn(V_hat, WORKERS))
    return V + p.b_coeff * rho if self_interaction else V


# ---------------------------------------------------------------------------
# R3/R4: cloud-in-cell, quantum-stars.py:200-247
# ---------------------------------------------------------------------------

# The 8 corner visits in the fixed order of quantum-stars.py:220-243 and
# :264-287: 0 selects i, 1 selects ip1, per axis.
CORNERS = (
    (0, 0, 0),
    (1, 0, 0),
    (0, 1, 0),
    (0, 0, 1),
    (1, 1, 0),
    (1, 0, 1),
    (0, 1, 1),
    (1, 1, 1),
)


def get_cic_indices_and_weights(pos, g: Grid):
    """quantum-stars.py:200-209 (float64)."""
    dxs = np.array([g.dx, g.dy, g.dz])
    i = np.floor((pos - 0.5 * dxs) / dxs)
    ip1 = i + 1.0
    weight_i = ((ip1 + 0.5) * dxs - pos) / dxs
    weight_ip1 = (pos - (i + 0.5) * dxs) / dxs
    n = np.array([g.nx, g.ny, g.nz])
    i = np.mod(i, n).astype(np.int64)
    ip1 = np.mod(ip1, n).astype(np.int64)
    return i, ip1, weight_i, weight_ip1


def bin_stars(pos, g: Grid, masses):
    """quantum-stars.py:212-247 / quantum-gas-bh.py:414-449.

    ``masses`` is the per-particle mass (m_s for every star, m_bh[s] for black
    holes).  Deposits in star order, corners in the fixed order: the products
    w_x w_y w_z fac are formed left to right and added by ``np.add.at``
    (unbuffered, in index order) star-major, corner-minor, so each cell sums
    its contributions in the reference's sequential order."""
    i, ip1, w_i, w_ip1 = get_cic_indices_and_weights(pos, g)
    vol = g.dx * g.dy * g.dz
    idx = (i, ip1)
    w = (w_i, w_ip1)
    fac = np.asarray(masses, dtype=np.float64) / vol
    vals = np.stack([w[c[0]][:, 0] * w[c[1]][:, 1] * w[c[2]][:, 2] * fac for c in CORNERS],
                    axis=1)
    cells = np.stack([np.ravel_multi_index((idx[c[0]][:, 0], idx[c[1]][:, 1], idx[c[2]][:, 2]),
                                           g.shape) for c in CORNERS], axis=1)
    rho = np.zeros(g.ncell)
    np.add.at(rho, cells.ravel(), vals.ravel())
    return rho.reshape(g.shape)


def grid_accelerations(rho, g: Grid, p: Phys, k=None):
    """Grid part of quantum-stars.py:254-260: a_d = -Re ifftn(i k_d V_hat)."""
    kx, ky, kz, k_sq = k if k is not None else kgrid(g)
    V_hat = -_fftn(4.0 * np.pi * p.G * (rho - p.rho_bar), WORKERS) / (
        k_sq + (k_sq == 0)
    )
    ax = -np.real(_ifftn(1.0j * kx * V_hat, WORKERS))
    ay = -np.real(_ifftn(1.0j * ky * V_hat, WORKERS))
    az = -np.real(_ifftn(1.0j * kz * V_hat, WORKERS))
    return ax, ay, az


def interpolate_cic(a_grid, pos, g: Grid):
    """quantum-stars.py:262-287: 8-point gather in fixed corner order."""
    i, ip1, w_i, w_ip1 = get_cic_indices_and_weights(pos, g)
    idx = (i, ip1)
    w = (w_i, w_ip1)
    acc = np.zeros((pos.shape[0], a_grid.shape[-1]))
    for c in CORNERS:
        acc += (w[c[0]][:, 0] * w[c[1]][:, 1] * w[c[2]][:, 2])[:, None] * a_grid[
            idx[c[0]][:, 0], idx[c[1]][:, 1], idx[c[2]][:, 2]
        ]
    return acc


def get_acceleration(pos, rho, g: Grid, p: Phys, k=None):
    """quantum-stars.py:250-288 -> (acc [n,3], a_max)."""
    ax, ay, az = grid_accelerations(rho, g, p, k)
    a_grid = np.stack((ax, ay, az), axis=-1)
    a_max = np.max(np.abs(a_grid))
    return interpolate_cic(a_grid, pos, g), a_max


def ref_mod(x, y):
    """jnp.mod / np.mod: result carries the sign of the divisor."""
    return np.mod(x, y)


# ---------------------------------------------------------------------------
# R6-R9: the stars KDK step, quantum-stars.py:295-330
# ---------------------------------------------------------------------------


def kick(psi, V, p: Phys, dt):
    """quantum-stars.py:301 / :318."""
    return np.exp(-1.0j * p.m_per_hbar * dt / 2.0 * V) * psi


def drift(psi, g: Grid, p: Phys, dt, k=None, kin_fac=1.0):
    """quantum-stars.py:307-309 (kin_fac: quantum-cosmo.py:185)."""
    k_sq = (k if k is not None else kgrid(g))[3]
    psi_hat = _fftn(psi, WORKERS)
    psi_hat = np.exp(dt * kin_fac * (-1.0j * k_sq / p.m_per_hbar / 2.0)) * psi_hat
    return _ifftn(psi_hat, WORKERS)


def stars_compute_step(
    psi, pos, vel, t, a_max, dt_s, g: Grid, p: Phys, dt, k=None,
    self_interaction=False,
):
    """quantum-stars.py:295-330, float64."""
    if k is None:
        k = kgrid(g)
    L = np.array([g.Lx, g.Ly, g.Lz])
    masses = np.full(pos.shape[0], p.m_s)
    # (1/2) kick
    rho_s = bin_stars(pos, g, masses)
    rho_tot = np.abs(psi) ** 2 + rho_s
    V = get_potential(rho_tot, g, p, k, self_interaction)
    psi = kick(psi, V, p, dt)
    acc, a_max1 = get_acceleration(pos, rho_tot, g, p, k)
    vel = vel + acc * dt / 2.0
    # drift
    psi = drift(psi, g, p, dt, k)
    pos = pos + vel * dt
    pos = ref_mod(pos, L)
    # (1/2) kick
    rho_s = bin_stars(pos, g, masses)
    rho_tot = np.abs(psi) ** 2 + rho_s
    V = get_potential(rho_tot, g, p, k, self_interaction)
    psi = kick(psi, V, p, dt)
    acc, a_max2 = get_acceleration(pos, rho_tot, g, p, k)
    vel = vel + acc * dt / 2.0
    t = t + dt
    a_max = max(a_max, a_max1, a_max2)
    with np.errstate(divide="ignore"):
        dt_s = np.min(np.abs(g.dx / vel)) if vel.size else np.inf
    return psi, pos, vel, t, a_max, dt_s


def stars_run(psi, pos, vel, nsteps, g, p, dt, t=0.0, a_max=0.0, dt_s=None,
              self_interaction=False):
    k = kgrid(g)
    if dt_s is None:
        dt_s = dt
    for _ in range(nsteps):
        psi, pos, vel, t, a_max, dt_s = stars_compute_step(
            psi, pos, vel, t, a_max, dt_s, g, p, dt, k, self_interaction
        )
    return psi, pos, vel, t, a_max, dt_s


def timestep_constants(g: Grid, p: Phys, t_end, dt_fac=1.0):
    """quantum-stars.py:151-157: dt_kin, nt (multiple of 100), nt_sub, dt."""
    dt_kin = dt_fac * p.m_per_hbar / 6.0 * (g.dx * g.dy * g.dz) ** (2.0 / 3.0)
    nt = int(math.ceil(math.ceil(t_end / dt_kin) / 100.0) * 100)
    nt_sub = int(round(nt / 100.0))
    return dt_kin, nt, nt_sub, t_end / nt


# ---------------------------------------------------------------------------
# R11: tidal and cosmological variants
# ---------------------------------------------------------------------------


def external_potential(g: Grid, G, M_halo):
    """quantum-tidal.py:175-179 (point mass at the box centre, softened)."""
    X, Y, Z = cell_centres(g)
    r = np.sqrt((X - 0.5 * g.Lx) ** 2 + (Y - 0.5 * g.Ly) ** 2 + (Z - 0.5 * g.Lz) ** 2)
    return -G * M_halo / (r + 0.5 * g.dx)


def tidal_compute_step(psi, t, g: Grid, p: Phys, dt, V_ext, k=None):
    """quantum-tidal.py:186-207."""
    if k is None:
        k = kgrid(g)
    V = get_potential(np.abs(psi) ** 2, g, p, k) + V_ext
    psi = kick(psi, V, p, dt)
    psi = drift(psi, g, p, dt, k)
    V = get_potential(np.abs(psi) ** 2, g, p, k) + V_ext
    psi = kick(psi, V, p, dt)
    return psi, t + dt


def cosmo_compute_dt(a, da, H0, omega_matter, omega_lambda):
    """quantum-cosmo.py:149-162 (1000-point midpoint quadrature)."""
    n_quad = 1000
    h = 1.0 / n_quad
    lin = np.linspace(0.5 * h, 1.0 - 0.5 * h, n_quad)
    a_tmp = a * lin
    adot = H0 * np.sqrt((omega_matter / a_tmp) + (omega_lambda * a_tmp**2))
    t = np.mean(1.0 / adot) * (a - 0.0)
    a_tmp = (a + da) * lin
    adot = H0 * np.sqrt((omega_matter / a_tmp) + (omega_lambda * a_tmp**2))
    return np.mean(1.0 / adot) * ((a + da) - 0.0) - t


def cosmo_factors(a, da, H0, omega_matter, omega_lambda):
    """quantum-cosmo.py:173-176 -> (dt, kin_fac, pot_fac)."""
    kin_fac = 0.5 * (a**-2 + (a + da) ** -2)
    pot_fac = 0.5 * (a**-1 + (a + da) ** -1)
    return cosmo_compute_dt(a, da, H0, omega_matter, omega_lambda), kin_fac, pot_fac


def cosmo_compute_step(psi, a, da, g: Grid, p: Phys, H0, om, ol, k=None):
    """quantum-cosmo.py:169-196."""
    if k is None:
        k = kgrid(g)
    dt, kin_fac, pot_fac = cosmo_factors(a, da, H0, om, ol)
    V = get_potential(np.abs(psi) ** 2, g, p, k)
    psi = np.exp(-1.0j * p.m_per_hbar * dt * pot_fac / 2.0 * V) * psi
    psi = drift(psi, g, p, dt, k, kin_fac)
    V = get_potential(np.abs(psi) ** 2, g, p, k)
    psi = np.exp(-1.0j * p.m_per_hbar * dt * pot_fac / 2.0 * V) * psi
    return psi, a + da


# ---------------------------------------------------------------------------
# R12/R13: isothermal MUSCL hydro, quantum-gas-bh.py:170-395
# (cubic grid with spacing dx, as in the reference)
# ---------------------------------------------------------------------------


def get_conserved(rho, vx, vy, vz, vol):
    """quantum-gas-bh.py:170-176."""
    return rho * vol, rho * vx * vol, rho * vy * vol, rho * vz * vol


def get_primitive(Mass, Momx, Momy, Momz, vol):
    """quantum-gas-bh.py:179-185."""
    return Mass / vol, Momx / Mass, Momy / Mass, Momz / Mass


def get_gradient(f, dx):
    """quantum-gas-bh.py:188-193 (central differences)."""
    return (
        (np.roll(f, -1, axis=0) - np.roll(f, 1, axis=0)) / (2.0 * dx),
        (np.roll(f, -1, axis=1) - np.roll(f, 1, axis=1)) / (2.0 * dx),
        (np.roll(f, -1, axis=2) - np.roll(f, 1, axis=2)) / (2.0 * dx),
    )


def extrap_to_face(f, f_dx, f_dy, f_dz, dx):
    """quantum-gas-bh.py:196-209."""
    f_XL = f + 0.5 * f_dx * dx
    f_XR = np.roll(f - 0.5 * f_dx * dx, -1, axis=0)
    f_YL = f + 0.5 * f_dy * dx
    f_YR = np.roll(f - 0.5 * f_dy * dx, -1, axis=1)
    f_ZL = f + 0.5 * f_dz * dx
    f_ZR = np.roll(f - 0.5 * f_dz * dx, -1, axis=2)
    return f_XL, f_XR, f_YL, f_YR, f_ZL, f_ZR


def apply_fluxes(F, fX, fY, fZ, dx, dt):
    """quantum-gas-bh.py:212-223."""
    fac = dt * dx * dx
    F = F + -fac * fX
    F = F + fac * np.roll(fX, 1, axis=0)
    F = F + -fac * fY
    F = F + fac * np.roll(fY, 1, axis=1)
    F = F + -fac * fZ
    F = F + fac * np.roll(fZ, 1, axis=2)
    return F


def get_flux(rho_L, vx_L, vy_L, vz_L, rho_R, vx_R, vy_R, vz_R, cs):
    """quantum-gas-bh.py:226-252: Rusanov flux evaluated on the averaged state."""
    rho_star = 0.5 * (rho_L + rho_R)
    momx_star = 0.5 * (rho_L * vx_L + rho_R * vx_R)
    momy_star = 0.5 * (rho_L * vy_L + rho_R * vy_R)
    momz_star = 0.5 * (rho_L * vz_L + rho_R * vz_R)
    P_star = rho_star * cs * cs
    flux_Mass = momx_star
    flux_Momx = momx_star**2 / rho_star + P_star
    flux_Momy = momx_star * momy_star / rho_star
    flux_Momz = momx_star * momz_star / rho_star
    C = np.maximum(cs + np.abs(vx_L), cs + np.abs(vx_R))
    flux_Mass = flux_Mass - C * 0.5 * (rho_R - rho_L)
    flux_Momx = flux_Momx - C * 0.5 * (rho_R * vx_R - rho_L * vx_L)
    flux_Momy = flux_Momy - C * 0.5 * (rho_R * vy_R - rho_L * vy_L)
    flux_Momz = flux_Momz - C * 0.5 * (rho_R * vz_R - rho_L * vz_L)
    return flux_Mass, flux_Momx, flux_Momy, flux_Momz


def _adjust_denominator(denom, eps=1.0e-12):
    """quantum-gas-bh.py:353-357."""
    return np.where(denom > 0, denom + eps, np.where(denom < 0, denom - eps, eps))


def slope_limiter(f, dx, f_dx, f_dy, f_dz):
    """quantum-gas-bh.py:340-395: two clamp01 ratios applied multiplicatively."""
    out = []
    for axis, fd in enumerate((f_dx, f_dy, f_dz)):
        denom = _adjust_denominator(fd)
        num = (f - np.roll(f, 1, axis=axis)) / dx
        fd = np.maximum(0.0, np.minimum(1.0, num / denom)) * fd
        num = -(f - np.roll(f, -1, axis=axis)) / dx
        fd = np.maximum(0.0, np.minimum(1.0, num / denom)) * fd
        out.append(fd)
    return tuple(out)


def solve_hydro(rho, vx, vy, vz, dt, dx, cs):
    """quantum-gas-bh.py:269-337."""
    vol = dx * dx * dx
    rho_dx, rho_dy, rho_dz = get_gradient(rho, dx)
    vx_dx, vx_dy, vx_dz = get_gradient(vx, dx)
    vy_dx, vy_dy, vy_dz = get_gradient(vy, dx)
    vz_dx, vz_dy, vz_dz = get_gradient(vz, dx)
    rho_dx, rho_dy, rho_dz = slope_limiter(rho, dx, rho_dx, rho_dy, rho_dz)
    vx_dx, vx_dy, vx_dz = slope_limiter(vx, dx, vx_dx, vx_dy, vx_dz)
    vy_dx, vy_dy, vy_dz = slope_limiter(vy, dx, vy_dx, vy_dy, vy_dz)
    vz_dx, vz_dy, vz_dz = slope_limiter(vz, dx, vz_dx, vz_dy, vz_dz)
    rho_prime = rho - 0.5 * dt * (
        vx * rho_dx + rho * vx_dx + vy * rho_dy + rho * vy_dy + vz * rho_dz
        + rho * vz_dz
    )
    vx_prime = vx - 0.5 * dt * (
        vx * vx_dx + vy * vx_dy + vz * vx_dz + (1.0 / rho) * rho_dx * cs * cs
    )
    vy_prime = vy - 0.5 * dt * (
        vx * vy_dx + vy * vy_dy + vz * vy_dz + (1.0 / rho) * rho_dy * cs * cs
    )
    vz_prime = vz - 0.5 * dt * (
        vx * vz_dx + vy * vz_dy + vz * vz_dz + (1.0 / rho) * rho_dz * cs * cs
    )
    r_XL, r_XR, r_YL, r_YR, r_ZL, r_ZR = extrap_to_face(rho_prime, rho_dx, rho_dy, rho_dz, dx)
    x_XL, x_XR, x_YL, x_YR, x_ZL, x_ZR = extrap_to_face(vx_prime, vx_dx, vx_dy, vx_dz, dx)
    y_XL, y_XR, y_YL, y_YR, y_ZL, y_ZR = extrap_to_face(vy_prime, vy_dx, vy_dy, vy_dz, dx)
    z_XL, z_XR, z_YL, z_YR, z_ZL, z_ZR = extrap_to_face(vz_prime, vz_dx, vz_dy, vz_dz, dx)
    fM_X, fPx_X, fPy_X, fPz_X = get_flux(r_XL, x_XL, y_XL, z_XL, r_XR, x_XR, y_XR, z_XR, cs)
    fM_Y, fPy_Y, fPz_Y, fPx_Y = get_flux(r_YL, y_YL, z_YL, x_YL, r_YR, y_YR, z_YR, x_YR, cs)
    fM_Z, fPz_Z, fPx_Z, fPy_Z = get_flux(r_ZL, z_ZL, x_ZL, y_ZL, r_ZR, z_ZR, x_ZR, y_ZR, cs)
    Mass, Momx, Momy, Momz = get_conserved(rho, vx, vy, vz, vol)
    Mass = apply_fluxes(Mass, fM_X, fM_Y, fM_Z, dx, dt)
    Momx = apply_fluxes(Momx, fPx_X, fPx_Y, fPx_Z, dx, dt)
    Momy = apply_fluxes(Momy, fPy_X, fPy_Y, fPy_Z, dx, dt)
    Momz = apply_fluxes(Momz, fPz_X, fPz_Y, fPz_Z, dx, dt)
    return get_primitive(Mass, Momx, Momy, Momz, vol)


def apply_grav_accel(rho, vx, vy, vz, dt, g: Grid, p: Phys, k=None):
    """quantum-gas-bh.py:255-266."""
    ax, ay, az = grid_accelerations(rho, g, p, k)
    return vx + ax * dt, vy + ay * dt, vz + az * dt


# ---------------------------------------------------------------------------
# R14: black-hole dark-matter accretion, quantum-gas-bh.py:497-530
# ---------------------------------------------------------------------------


def do_accretion(psi, pos, vel, m_bh, g: Grid, p: Phys, dt, sigma_v):
    """quantum-gas-bh.py:497-530 (sigma_v = cs there, sigma in quantum-bh.py:319)."""
    dxs = np.array([g.dx, g.dy, g.dz])
    i = np.floor((pos - 0.5 * dxs) / dxs)
    i = np.mod(i, np.array(g.shape)).astype(np.int64)
    s = 0
    psi = psi.copy()
    psi_at_bh = psi[i[s, 0], i[s, 1], i[s, 2]]
    psi_amp = np.abs(psi_at_bh)
    psi_theta = np.angle(psi_at_bh)
    v = np.sqrt(sigma_v**2 + vel[0, 0] ** 2 + vel[0, 1] ** 2 + vel[0, 2] ** 2)
    xi = 2.0 * np.pi * p.G * m_bh[0] * p.m_per_hbar / v
    dM_dt = (
        32.0 * np.pi**2 * (p.G * m_bh[0]) ** 3 * p.m_per_hbar * psi_amp**2
        / (p.c_light**3 * v * (1.0 - np.exp(-xi)))
    )
    new_psi_amp = np.abs(psi_amp) - np.sqrt(dM_dt * dt / g.vol)
    psi[i[s, 0], i[s, 1], i[s, 2]] = new_psi_amp * np.exp(1.0j * psi_theta)
    m_bh = m_bh + dM_dt * dt
    return psi, m_bh


# ---------------------------------------------------------------------------
# R15: isothermal Bondi gas sink, quantum-fluid-accretion-test.py:404-494
# ---------------------------------------------------------------------------

LAMBDA_ISO = math.exp(1.5) / 4.0


def bondi_sink(rho, M_bh, x_bh, dx, Lx, cs, G, dt, r_acc_mult=4.0,
               lam=LAMBDA_ISO, fmax=0.25):
    """quantum-fluid-accretion-test.py:454-494 (v_rel = 0)."""
    nx = rho.shape[0]
    r_B = G * M_bh / (cs * cs)
    r_acc = r_acc_mult * dx
    rK = np.clip(r_B, 0.25 * dx, 0.5 * r_acc)
    xs = (np.arange(nx) + 0.5) * dx

    def pdelta(x0):
        d = np.abs(xs - x0)
        return np.minimum(d, Lx - d)

    dX, dY, dZ = np.meshgrid(pdelta(x_bh[0]), pdelta(x_bh[1]), pdelta(x_bh[2]), indexing="ij")
    R2 = dX * dX + dY * dY + dZ * dZ
    mask = R2 <= r_acc * r_acc
    W = np.exp(-0.5 * R2 / (rK * rK)) * mask
    sumW = np.sum(W) + 1e-30
    rho_inf = np.sum(W * rho) / sumW
    dMdt = 4.0 * np.pi * lam * (G * M_bh) ** 2 * rho_inf / (cs**3)
    dM = dMdt * dt
    WRho = W * rho
    sumWRho = np.sum(WRho) + 1e-30
    phi = WRho / sumWRho
    M_avail = np.sum(rho * mask) * (dx**3)
    dM_cap = min(dM, fmax * M_avail)
    rho_new = np.maximum(0.0, rho - (dM_cap / (dx**3)) * phi)
    return rho_new, M_bh + dM_cap, dMdt, rho_inf, r_B, dM_cap


def bondi_sink_ambient(rho, M_bh, x_bh, dx, Lx, cs, G, dt, r_acc_mult=2.5,
                       lam=LAMBDA_ISO, fmax=None, ann_lo=1.1, ann_hi=1.8,
                       v=None, v_bh=(0.0, 0.0, 0.0)):
    """Fixed-grid sink with the ambient density sampled in a shell just outside
    r_acc, quantum-fluid-accretion.py:440-510.  v = (vx, vy, vz) gas
    velocities enable the BHL denominator (cs^2 + v_rel^2)^1.5.
    Returns (rho_new, dMdt_target, rho_inf, rB, dM_cap, r_acc, M_avail, dM_uncl)."""
    nx = rho.shape[0]
    xs = (np.arange(nx) + 0.5) * dx

    def pdelta(x0):
        d = np.abs(xs - x0)
        return np.minimum(d, Lx - d)

    dX, dY, dZ = np.meshgrid(pdelta(x_bh[0]), pdelta(x_bh[1]), pdelta(x_bh[2]), indexing="ij")
    R = np.sqrt(dX * dX + dY * dY + dZ * dZ)
    rB = G * M_bh / (cs * cs + 1e-30)
    r_acc = r_acc_mult * dx
    rK = min(0.5 * r_acc, max(0.5 * dx, rB))
    mask = R <= r_acc
    W = np.exp(-0.5 * (R / (rK + 1e-30)) ** 2) * mask
    r_lo = max(ann_lo * r_acc, r_acc + 0.25 * dx)
    r_hi = max(ann_hi * r_acc, r_lo + 0.5 * dx)
    shell = (R >= r_lo) & (R <= r_hi)
    n_sh = np.sum(shell) + 1e-30
    rho_inf = np.sum(rho * shell) / n_sh
    if v is not None:
        v_inf = [np.sum(c * shell) / n_sh for c in v]
        v_rel2 = sum((b - c) ** 2 for b, c in zip(v_bh, v_inf))
        denom = (cs**2 + v_rel2) ** 1.5
    else:
        denom = cs**3
    dMdt = 4.0 * np.pi * lam * (G * M_bh) ** 2 * rho_inf / (denom + 1e-30)
    dM_uncl = dMdt * dt
    WRho = W * rho
    phi = WRho / (np.sum(WRho) + 1e-30)
    M_avail = np.sum(rho * mask) * dx**3
    dM_cap = min(dM_uncl, M_avail) if fmax is None else min(dM_uncl, fmax * M_avail)
    rho_new = np.maximum(0.0, rho - (dM_cap / dx**3) * phi)
    return rho_new, dMdt, rho_inf, rB, dM_cap, r_acc, M_avail, dM_uncl


def hydro_cfl_dt(vx, vy, vz, cs, dx, cfl, dt):
    """dt_eff = min(dt, cfl dx / max(c + |v|)), quantum-fluid-accretion.py:697-701
    with the constant sound speed of cs2_local (:248-250)."""
    cmax = np.max(cs + np.sqrt(vx * vx + vy * vy + vz * vz))
    return min(dt, cfl * dx / (cmax + 1e-30))


# ---------------------------------------------------------------------------
# quantum-fluid-accretion.py: the kick-drift-kick step with a moving, softened,
# accreting black hole seeded at the dark-matter peak (:695-870)
# ---------------------------------------------------------------------------


@dataclasses.dataclass
class FaccParams:
    """The toggles and constants of quantum-fluid-accretion.py:41-100, 670-690."""

    cs: float = 60.0
    hydro_cfl: float = 0.15
    bh_on: bool = True
    bh_grav: bool = True
    bh_move: bool = True
    bh_accretion: bool = True
    bh_init_m: float = 1.0e7
    bh_inject_t: float = 13.0
    ramp_on: bool = True
    ramp_center: float = 13.0
    ramp_w: float = 1.0
    r_acc_mult: float = 2.5
    lam: float = LAMBDA_ISO
    fmax: float | None = None
    ann_lo: float = 1.1
    ann_hi: float = 1.8
    k_cut_frac: float = 0.6
    inject_smooth_on: bool = True
    inject_smooth_kpc: float = 0.0
    rho_gas: float = 1.0e6  # reported as rho_inf while the sink is inactive


def facc_seed_mass(t, placed, q: FaccParams):
    """seed_mass_from_time, :682-690."""
    pl = 1.0 if placed > 0.5 else 0.0
    if q.ramp_on:
        s = 0.5 * (1.0 + math.tanh((t - q.ramp_center) / (q.ramp_w + 1e-30)))
        s = s * (1.0 if t >= q.bh_inject_t else 0.0)
    else:
        s = 1.0 if t >= q.bh_inject_t else 0.0
    return q.bh_init_m * s * pl


def facc_potential(rho_src, rho_bg, g: Grid, G, k_sq):
    """get_potential_bg, :182-185 -> (V_hat, V)."""
    V_hat = -np.fft.fftn(4.0 * np.pi * G * (rho_src - rho_bg)) / (k_sq + (k_sq == 0))
    return V_hat, np.real(np.fft.ifftn(V_hat))


def facc_accel(V_hat, k):
    """accel_from_Vhat, :187-191."""
    kx, ky, kz = k[0], k[1], k[2]
    return tuple(-np.real(np.fft.ifftn(1.0j * kd * V_hat)) for kd in (kx, ky, kz))


def facc_cic(x_bh, dx, n):
    """CIC cells and weights of a point, :388-417 / 419-437 (corner order of both)."""
    xi = np.asarray(x_bh) / dx - 0.5
    i0 = np.floor(xi).astype(int)
    f = xi - i0
    w = np.array([(1 - f[0]) * (1 - f[1]) * (1 - f[2]), f[0] * (1 - f[1]) * (1 - f[2]),
                  (1 - f[0]) * f[1] * (1 - f[2]), (1 - f[0]) * (1 - f[1]) * f[2],
                  f[0] * f[1] * (1 - f[2]), f[0] * (1 - f[1]) * f[2],
                  (1 - f[0]) * f[1] * f[2], f[0] * f[1] * f[2]])
    off = ((0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0), (1, 0, 1), (0, 1, 1), (1, 1, 1))
    cells = [tuple(int((i0[d] + o[d]) % n) for d in range(3)) for o in off]
    return cells, w


def facc_bh_density(M, x_bh, dx, n):
    rho = np.zeros((n, n, n))
    cells, w = facc_cic(x_bh, dx, n)
    for c, wk in zip(cells, w):
        rho[c] += wk * M / dx**3
    return rho


def facc_sample(field, x_bh, dx, n):
    cells, w = facc_cic(x_bh, dx, n)
    return float(np.sum(w * np.array([field[c] for c in cells])))


def facc_hydro(rho, vx, vy, vz, dt, dx, cs):
    """solve_hydro of quantum-fluid-accretion.py:273-317 (limited pressure
    gradient, constant c^2 from cs2_local, eps-guarded divisions)."""
    vol = dx**3
    eps = 1e-30
    c2 = np.full_like(rho, cs * cs)
    P = rho * c2
    grads = [get_gradient(f, dx) for f in (rho, vx, vy, vz, P)]
    lim = [slope_limiter(f, dx, *gd) for f, gd in zip((rho, vx, vy, vz, P), grads)]
    (rdx, rdy, rdz), (uxx, uxy, uxz), (uyx, uyy, uyz), (uzx, uzy, uzz), (Px, Py, Pz) = lim
    rho_p = rho - 0.5 * dt * (vx * rdx + rho * uxx + vy * rdy + rho * uyy + vz * rdz + rho * uzz)
    vx_p = vx - 0.5 * dt * (vx * uxx + vy * uxy + vz * uxz + Px / (rho + eps))
    vy_p = vy - 0.5 * dt * (vx * uyx + vy * uyy + vz * uyz + Py / (rho + eps))
    vz_p = vz - 0.5 * dt * (vx * uzx + vy * uzy + vz * uzz + Pz / (rho + eps))
    R_ = extrap_to_face(rho_p, rdx, rdy, rdz, dx)
    X_ = extrap_to_face(vx_p, uxx, uxy, uxz, dx)
    Y_ = extrap_to_face(vy_p, uyx, uyy, uyz, dx)
    Z_ = extrap_to_face(vz_p, uzx, uzy, uzz, dx)

    def flux(rL, uL, aL, bL, rR, uR, aR, bR, c2L, c2R):
        rs = 0.5 * (rL + rR)
        mu = 0.5 * (rL * uL + rR * uR)
        ma = 0.5 * (rL * aL + rR * aR)
        mb = 0.5 * (rL * bL + rR * bR)
        Ps = rs * 0.5 * (c2L + c2R)
        fM, fU = mu, mu**2 / (rs + eps) + Ps
        fA, fB = mu * ma / (rs + eps), mu * mb / (rs + eps)
        C = np.maximum(np.sqrt(c2L) + np.abs(uL), np.sqrt(c2R) + np.abs(uR))
        return (fM - C * 0.5 * (rR - rL), fU - C * 0.5 * (rR * uR - rL * uL),
                fA - C * 0.5 * (rR * aR - rL * aL), fB - C * 0.5 * (rR * bR - rL * bL))

    c2R = [np.roll(c2, -1, axis=a) for a in range(3)]
    FX = flux(R_[0], X_[0], Y_[0], Z_[0], R_[1], X_[1], Y_[1], Z_[1], c2, c2R[0])
    FYr = flux(R_[2], Y_[2], Z_[2], X_[2], R_[3], Y_[3], Z_[3], X_[3], c2, c2R[1])
    FZr = flux(R_[4], Z_[4], X_[4], Y_[4], R_[5], Z_[5], X_[5], Y_[5], c2, c2R[2])
    FY = (FYr[0], FYr[3], FYr[1], FYr[2])  # (M, My, Mz, Mx) -> (M, Mx, My, Mz)
    FZ = (FZr[0], FZr[2], FZr[3], FZr[1])  # (M, Mz, Mx, My) -> (M, Mx, My, Mz)
    U = get_conserved(rho, vx, vy, vz, vol)
    U = [apply_fluxes(U[i], FX[i], FY[i], FZ[i], dx, dt) for i in range(4)]
    Mass = U[0]
    return Mass / vol, U[1] / (Mass + eps), U[2] / (Mass + eps), U[3] / (Mass + eps)


def facc_compute_step(psi, rho, vx, vy, vz, t, M_acc, x_bh, v_bh, placed, g: Grid, p: Phys,
                      q: FaccParams, dt, k=None):
    """compute_step of quantum-fluid-accretion.py:695-870, float64.  Returns
    (psi, rho, vx, vy, vz, t, M_bh_eff_out, M_acc, x_bh, v_bh, placed, diag) with
    diag = (dMdt, rho_inf, r_B, dMdt_real, cap_ratio, r_acc_eff)."""
    k = k if k is not None else kgrid(g)
    k_sq = k[3]
    n, dx, L, G, mph, cs = g.nx, g.dx, g.Lx, p.G, p.m_per_hbar, q.cs
    x_bh = np.array(x_bh, dtype=float)
    v_bh = np.array(v_bh, dtype=float)
    dt_eff = hydro_cfl_dt(vx, vy, vz, cs, dx, q.hydro_cfl, dt)
    M_eff = facc_seed_mass(t, placed, q) + M_acc
    r_soft = q.r_acc_mult * dx
    rho_bg = np.mean(np.abs(psi) ** 2) + np.mean(rho)
    k_cut = q.k_cut_frac * (np.pi / dx)
    LP = np.exp(-((k_sq / (k_cut**2 + 1e-30)) ** 4))
    active = 1.0 if placed > 0.5 else 0.0

    def bh_kick(psi_, v_bh_):
        Vh, _ = facc_potential(np.abs(psi_) ** 2 + rho, rho_bg, g, G, k_sq)
        a = facc_accel(Vh * LP, k)
        return v_bh_ + np.array([facc_sample(ad, x_bh, dx, n) for ad in a]) * (dt_eff / 2.0) * active

    if q.bh_on and q.bh_move:
        v_bh = bh_kick(psi, v_bh)
    rho_src = np.abs(psi) ** 2 + rho

    def soft_bh(M, r):
        if not (q.bh_on and q.bh_grav):
            return 0.0
        hat = np.fft.fftn(facc_bh_density(M, x_bh, dx, n)) * np.exp(-0.5 * r * r * k_sq)
        on = 1.0 if (placed > 0.5 and M > 0.0) else 0.0
        return np.real(np.fft.ifftn(hat)) * on

    Vh, V = facc_potential(rho_src + soft_bh(M_eff, r_soft), rho_bg, g, G, k_sq)
    psi = np.exp(-1.0j * mph * dt_eff / 2.0 * V) * psi
    ax, ay, az = facc_accel(Vh, k)
    vx, vy, vz = vx + ax * (dt_eff / 2.0), vy + ay * (dt_eff / 2.0), vz + az * (dt_eff / 2.0)
    psi = np.fft.ifftn(np.exp(dt_eff * (-1.0j * k_sq / mph / 2.0)) * np.fft.fftn(psi))
    rho, vx, vy, vz = facc_hydro(rho, vx, vy, vz, dt_eff, dx, cs)
    if q.bh_on and q.bh_move:
        x_bh = np.mod(x_bh + dt_eff * v_bh * active, L)
    active_acc = 1.0 if (placed > 0.5 and M_eff > 0.0) else 0.0
    dMdt = dMdt_real = cap_ratio = r_B = 0.0
    rho_inf = q.rho_gas
    r_acc_eff = max(q.r_acc_mult * dx, 2.0 * (G * M_eff / (cs**2 + 1e-30)))
    if q.bh_on and q.bh_accretion:
        r = bondi_sink_ambient(rho, M_eff, x_bh, dx, L, cs, G, dt_eff, r_acc_mult=q.r_acc_mult,
                               lam=q.lam, fmax=q.fmax, ann_lo=q.ann_lo, ann_hi=q.ann_hi,
                               v=(vx, vy, vz), v_bh=tuple(v_bh))
        rho_try, dMdt_try, rho_inf_try, r_B_try, dM_cap, r_acc_used, _, dM_uncl = r
        rho = rho * (1.0 - active_acc) + rho_try * active_acc
        dMdt = dMdt_try * active_acc
        rho_inf = rho_inf_try * active_acc + (1.0 - active_acc) * q.rho_gas
        r_B = r_B_try * active_acc
        M_acc = M_acc + dM_cap * active_acc
        dMdt_real = dM_cap / (dt_eff + 1e-30) if active_acc > 0.5 else 0.0
        cap_ratio = dM_cap / (dM_uncl + 1e-30) if (dM_uncl > 0.0 and active_acc > 0.5) else 0.0
        r_acc_eff = r_acc_used * active_acc + (1.0 - active_acc) * r_acc_eff
    M_mid = facc_seed_mass(t, placed, q) + M_acc
    Vh2, V2 = facc_potential(np.abs(psi) ** 2 + rho + soft_bh(M_mid, r_acc_eff), rho_bg, g, G,
                             k_sq)
    psi = np.exp(-1.0j * mph * dt_eff / 2.0 * V2) * psi
    ax, ay, az = facc_accel(Vh2, k)
    vx, vy, vz = vx + ax * (dt_eff / 2.0), vy + ay * (dt_eff / 2.0), vz + az * (dt_eff / 2.0)
    if q.bh_on and q.bh_move:
        v_bh = bh_kick(psi, v_bh)
    t = t + dt_eff
    if placed < 0.5 and t >= q.bh_inject_t:
        rho3 = np.abs(psi) ** 2
        if q.inject_smooth_on:
            s2 = max(q.inject_smooth_kpc, 1.5 * dx) ** 2
            rho3 = np.real(np.fft.ifftn(np.fft.fftn(rho3) * np.exp(-0.5 * s2 * k_sq)))
        i0, j0, k0 = np.unravel_index(np.argmax(rho3), rho3.shape)
        x_bh = np.array([(i0 + 0.5) * dx, (j0 + 0.5) * dx, (k0 + 0.5) * dx])
        v_bh = np.zeros(3)
        placed = 1.0
    M_out = facc_seed_mass(t, placed, q) + M_acc
    return (psi, rho, vx, vy, vz, t, M_out, M_acc, x_bh, v_bh, placed,
            (dMdt, rho_inf, r_B, dMdt_real, cap_ratio, r_acc_eff))


# ---------------------------------------------------------------------------
# R16: the gas + black-hole step, quantum-gas-bh.py:537-578
# ---------------------------------------------------------------------------


def gasbh_compute_step(psi, rho, vx, vy, vz, m_bh, pos, vel, t, g: Grid, p: Phys,
                       dt, k=None, bondi_r_acc_mult=None, dm_accretion=True):
    """quantum-gas-bh.py:537-578.

    With ``bondi_r_acc_mult`` set, the isothermal Bondi gas sink of
    quantum-fluid-accretion-test.py:534-536 is applied after the hydro and
    black-hole drift, before the second half kick."""
    if k is None:
        k = kgrid(g)
    L = np.array([g.Lx, g.Ly, g.Lz])
    gas = rho is not None  # rho None: quantum-bh.py:346-381 (no gas)
    # (1/2) kick
    rho_bh = bin_stars(pos, g, m_bh)
    rho_tot = np.abs(psi) ** 2 + rho_bh + (rho if gas else 0.0)
    V = get_potential(rho_tot, g, p, k)
    psi = kick(psi, V, p, dt)
    if gas:
        vx, vy, vz = apply_grav_accel(rho_tot, vx, vy, vz, dt / 2.0, g, p, k)
    acc, _ = get_acceleration(pos, rho_tot, g, p, k)
    vel = vel + acc * dt / 2.0
    # drift
    psi = drift(psi, g, p, dt, k)
    if gas:
        rho, vx, vy, vz = solve_hydro(rho, vx, vy, vz, dt, g.dx, p.cs)
    pos = pos + vel * dt
    pos = ref_mod(pos, L)
    if bondi_r_acc_mult is not None and gas:
        rho, M_new, *_ = bondi_sink(rho, m_bh[0], pos[0], g.dx, g.Lx, p.cs, p.G, dt,
                                    r_acc_mult=bondi_r_acc_mult)
        m_bh = np.array([M_new] + list(m_bh[1:]))
    # (1/2) kick
    rho_bh = bin_stars(pos, g, m_bh)
    rho_tot = np.abs(psi) ** 2 + rho_bh + (rho if gas else 0.0)
    V = get_potential(rho_tot, g, p, k)
    psi = kick(psi, V, p, dt)
    if gas:
        vx, vy, vz = apply_grav_accel(rho_tot, vx, vy, vz, dt / 2.0, g, p, k)
    acc, _ = get_acceleration(pos, rho_tot, g, p, k)
    vel = vel + acc * dt / 2.0
    # accretion
    if dm_accretion:
        psi, m_bh = do_accretion(psi, pos, vel, m_bh, g, p, dt, p.cs)
    return psi, rho, vx, vy, vz, m_bh, pos, vel, t + dt


# ---------------------------------------------------------------------------
# float32 star deposit in the reference's exact operation order
# ---------------------------------------------------------------------------


def cic_weights_f32(pos32, g: Grid):
    """quantum-stars.py:200-209 evaluated in float32 like the x64-off reference.

    dxs is float32(dx); every operation rounds to float32 in the written order
    (no fused multiply-add)."""
    f = np.float32
    pos32 = np.asarray(pos32, dtype=np.float32)
    dxs = np.array([g.dx, g.dy, g.dz], dtype=np.float32)
    half = f(0.5)
    i = np.floor((pos32 - half * dxs) / dxs)
    ip1 = i + f(1.0)
    w_i = ((ip1 + half) * dxs - pos32) / dxs
    w_ip1 = (pos32 - (i + half) * dxs) / dxs
    n = np.array(g.shape, dtype=np.float32)
    ii = np.mod(i, n).astype(np.int64)
    ip = np.mod(ip1, n).astype(np.int64)
    return ii, ip, w_i.astype(np.float32), w_ip1.astype(np.float32)


def bin_stars_f32(pos32, g: Grid, m_s):
    """Sequential float32 deposit, stars in order, corners in the order of
    quantum-stars.py:220-243; each cell accumulates from 0 in that order.
    fac = float32(m_s / (dx dy dz)) as the weak-typed Python scalar becomes."""
    ii, ip, w_i, w_ip1 = cic_weights_f32(pos32, g)
    fac = np.float32(m_s / (g.dx * g.dy * g.dz))
    rho = np.zeros(g.shape, dtype=np.float32)
    idx = (ii, ip)
    w = (w_i, w_ip1)
    for s in range(ii.shape[0]):
        for c in CORNERS:
            v = np.float32(np.float32(np.float32(w[c[0]][s, 0] * w[c[1]][s, 1])
                                      * w[c[2]][s, 2]) * fac)
            cell = (idx[c[0]][s, 0], idx[c[1]][s, 1], idx[c[2]][s, 2])
            rho[cell] = np.float32(rho[cell] + v)
    return rho


def bin_stars_f32_vec(pos32, g: Grid, m_s):
    """``bin_stars_f32`` vectorised, bit for bit: the same float32 products,
    added by ``np.add.at`` (unbuffered, in index order) in star-major,
    corner-minor order -- the sequential order of quantum-stars.py:220-246."""
    ii, ip, w_i, w_ip1 = cic_weights_f32(pos32, g)
    fac = np.float32(m_s / (g.dx * g.dy * g.dz))
    idx = (ii, ip)
    w = (w_i, w_ip1)
    vals = np.stack([((w[c[0]][:, 0] * w[c[1]][:, 1]) * w[c[2]][:, 2]) * fac for c in CORNERS],
                    axis=1)
    cells = np.stack([np.ravel_multi_index((idx[c[0]][:, 0], idx[c[1]][:, 1], idx[c[2]][:, 2]),
                                           g.shape) for c in CORNERS], axis=1)
    rho = np.zeros(g.ncell, dtype=np.float32)
    np.add.at(rho, cells.ravel(), vals.ravel())
    return rho.reshape(g.shape)


def kgrid_f32(g: Grid):
    """R1 in float32, as the x64-off reference builds it (quantum-stars.py:142-149)."""
    return tuple(a.astype(np.float32) for a in kgrid(g))


def stars_compute_step_f32(psi, pos, vel, t, a_max, dt_s, g: Grid, p: Phys, dt, k32):
    """quantum-stars.py:295-330 in the reference's own precision: complex64
    psi, float32 fields and particles (x64 is off, quantum-stars.py:70).

    The CPU baseline's timed step.  The deposit and the gather are vectorised
    (the deposit bit for bit as ``bin_stars_f32``); the kinetic factor is
    evaluated every step, as the reference does (:307-309)."""
    f = np.float32
    kx, ky, kz, k_sq = k32
    L = np.array([g.Lx, g.Ly, g.Lz], dtype=np.float32)
    four_pi_G = f(4.0 * np.pi * p.G)
    div = k_sq + (k_sq == 0)

    def potential_and_accel(psi, pos):
        rho = np.abs(psi) ** 2 + bin_stars_f32_vec(pos, g, p.m_s)
        V_hat = -_fftn(four_pi_G * (rho - f(p.rho_bar)), WORKERS) / div
        V = np.real(_ifftn(V_hat, WORKERS))
        a_grid = np.stack([-np.real(_ifftn(1j * kd * V_hat, WORKERS)) for kd in (kx, ky, kz)],
                          axis=-1)
        ii, ip, w_i, w_ip1 = cic_weights_f32(pos, g)
        idx = (ii, ip)
        w = (w_i, w_ip1)
        acc = np.zeros((pos.shape[0], 3), dtype=np.float32)
        for c in CORNERS:
            acc += ((w[c[0]][:, 0] * w[c[1]][:, 1]) * w[c[2]][:, 2])[:, None] * a_grid[
                idx[c[0]][:, 0], idx[c[1]][:, 1], idx[c[2]][:, 2]]
        return V, acc, np.max(np.abs(a_grid))

    V, acc, a1 = potential_and_accel(psi, pos)
    psi = np.exp(-1j * f(p.m_per_hbar * dt / 2.0) * V) * psi
    vel = vel + acc * f(dt / 2.0)
    psi = _ifftn(np.exp(f(dt) * (-1j * k_sq / f(p.m_per_hbar) / f(2.0))) * _fftn(psi, WORKERS),
                 WORKERS)
    pos = np.mod(pos + vel * f(dt), L)
    V, acc, a2 = potential_and_accel(psi, pos)
    psi = np.exp(-1j * f(p.m_per_hbar * dt / 2.0) * V) * psi
    vel = vel + acc * f(dt / 2.0)
    with np.errstate(divide="ignore"):
        dt_s = np.min(np.abs(f(g.dx) / vel)) if vel.size else np.inf
    return psi, pos, vel, t + dt, max(a_max, a1, a2), dt_s


# ---------------------------------------------------------------------------
# Seeded initial conditions (the benchmark IC family)
# ---------------------------------------------------------------------------


def delta_field(n, seed, shape=None):
    """Unit-variance Gaussian random field with P(k) ~ k^-3 for
    0 < |k| <= k_Nyq/2 (zero elsewhere, k=0 included), float64."""
    shape = shape or (n, n, n)
    rng = np.random.default_rng(seed)
    w = rng.standard_normal(shape)
    kk = np.meshgrid(*[np.fft.fftfreq(m) * m for m in shape], indexing="ij")
    kmag = np.sqrt(sum(k**2 for k in kk))
    knyq = min(shape) / 2.0
    amp = np.zeros(shape)
    sel = (kmag > 0) & (kmag <= knyq / 2.0)
    amp[sel] = kmag[sel] ** -1.5
    d = np.real(np.fft.ifftn(np.fft.fftn(w) * amp))
    d -= d.mean()
    d /= d.std()
    return d


def stars_ic(n, n_s, seed=0, shape=None, L=(1.0, 1.0, 1.0), star_frac=0.1):
    """psi = sqrt(1 + 0.1 delta), theta = 0; n_s uniform stars at rest with
    total mass star_frac of the dark-matter box mass.  Returns
    (psi complex128, pos, vel, Grid, Phys)."""
    shape = shape or (n, n, n)
    g = Grid(*shape, *L)
    rho_dm = 1.0 + 0.1 * delta_field(n, seed, shape)
    psi = np.sqrt(rho_dm).astype(np.complex128)
    rng = np.random.default_rng(seed + 1)
    pos = rng.uniform(0.0, 1.0, (n_s, 3)) * np.array(L)
    vel = np.zeros((n_s, 3))
    M_dm = rho_dm.sum() * g.vol
    M_s = star_frac * M_dm
    Lvol = L[0] * L[1] * L[2]
    p = Phys(m_per_hbar=1.0, G=1.0 / (4.0 * np.pi),
             rho_bar=rho_dm.mean() + M_s / Lvol,
             m_s=(M_s / n_s) if n_s else 0.0)
    return psi, pos, vel, g, p


def default_dt(g: Grid, p: Phys):
    """dt = dx^2/6 for m/hbar = 1 (quantum-stars.py:153 with a cubic cell)."""
    return p.m_per_hbar / 6.0 * (g.dx * g.dy * g.dz) ** (2.0 / 3.0)


def rel_l2(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))
