"""The reference scripts' set-up, initial conditions, state I/O and outer loop,
on top of the libqj step, so a quantum-stars run goes end to end here.

- ``StarsSetup.reference(res)``: the module constants of quantum-stars.py:61-157
  (grid, units, star mass, time step, ``nt_sub``).
- Initial conditions: ``stars_blob_ic`` (quantum-stars.py:373-423),
  ``random_phase_psi`` (quantum-fluid.py:511-522 with sorted phases,
  quantum-bh.py:455-462 without), ``soliton_psi`` (quantum-bh.py:438-450,
  quantum-gas-bh.py's soliton).  They run on the host in float64 with NumPy,
  like the reference, and use its seed (``np.random.seed(17)``).
- ``save_state`` / ``load_state``: the state dict as ``.npz`` (the keys of
  quantum-stars.py:425-432), in place of the reference's orbax checkpoints.
- ``run_stars``: the main loop of quantum-stars.py:440-459 -- ``outer``
  iterations of ``nt_sub`` steps, a checkpoint after each and the reference's
  a-posteriori time-step checks -- without the plots.
"""

from __future__ import annotations

import dataclasses
import math
import os

import numpy as np
import torch

from .core import FUSED_F32, PLAIN_F64, Grid, Phys, StarsStep

# physical constants of the reference scripts (kpc, km/s, Msun)
G_KPC = 4.30241002e-6
HBAR = 1.71818134e-87
EV_TO_MSUN = 8.96215334e-67
EV_TO_INTERNAL = 8.05478173e-56
C_KMS = 299792.458


def m_per_hbar_of(m_22: float) -> float:
    """Axion mass over hbar, quantum-stars.py:95-96."""
    return m_22 * 1.0e-22 * EV_TO_MSUN / HBAR


@dataclasses.dataclass
class StarsSetup:
    """Module constants of quantum-stars.py for a resolution factor."""

    nx: int
    ny: int
    nz: int
    Lx: float
    Ly: float
    Lz: float
    rho_bar: float
    t_end: float
    m_per_hbar: float
    G: float
    n_s: int
    m_s: float
    frac_dm: float
    b_coeff: float
    dt: float
    nt: int
    nt_sub: int

    @classmethod
    def reference(cls, res: int = 1, self_interaction: bool = False) -> "StarsSetup":
        """quantum-stars.py:61-157 with ``--res res``."""
        nx, ny, nz = 128 * res, 64 * res, 16 * res
        Lx, Ly, Lz = 128.0, 64.0, 16.0
        rho_bar, t_end, m_22, frac_s = 1.0e4, 10.0, 1.0, 0.1
        M_s = frac_s * rho_bar * Lx * Ly * Lz
        n_s = 400 * res
        mph = m_per_hbar_of(m_22)
        b_coeff = 0.0
        if self_interaction:  # quantum-stars.py:118-125
            f_internal = 1.5 * 1.0e24 * EV_TO_INTERNAL
            m = m_22 * 1.0e-22 * EV_TO_MSUN
            a_s = HBAR * C_KMS**3 * m / (32.0 * math.pi * f_internal**2)
            b_coeff = -4.0 * math.pi * a_s / mph**2 / HBAR
        dx, dy, dz = Lx / nx, Ly / ny, Lz / nz
        # quantum-stars.py:151-157: dt_kin, nt a multiple of 100, nt_sub = nt / 100
        dt_kin = mph / 6.0 * (dx * dy * dz) ** (2.0 / 3.0)
        nt = int(math.ceil(math.ceil(t_end / dt_kin) / 100.0) * 100)
        nt_sub = int(round(nt / 100.0))
        return cls(nx, ny, nz, Lx, Ly, Lz, rho_bar, t_end, mph, G_KPC, n_s, M_s / n_s,
                   1.0 - frac_s, b_coeff, t_end / nt, nt, nt_sub)

    def grid(self) -> Grid:
        return Grid(self.nx, self.ny, self.nz, self.Lx, self.Ly, self.Lz)

    def phys(self) -> Phys:
        return Phys(m_per_hbar=self.m_per_hbar, G=self.G, rho_bar=self.rho_bar,
                    b_coeff=self.b_coeff)

    def cell_centres(self):
        """x_lin = linspace(dx/2, L - dx/2, n) per axis, meshgrid 'ij'."""
        lin = [np.linspace(0.5 * L / n, L - 0.5 * L / n, n)
               for n, L in ((self.nx, self.Lx), (self.ny, self.Ly), (self.nz, self.Lz))]
        return np.meshgrid(*lin, indexing="ij")


# (weight, x / Lx, y / Ly) of the Gaussian dark-matter blobs, quantum-stars.py:377-421
STARS_BLOBS = ((2.0, 0.5, 0.4), (1.5, 0.6, 0.5), (1.0, 0.4, 0.6), (1.0, 0.6, 0.4),
               (1.0, 0.6, 0.6), (1.0, 0.6, 0.4), (1.0, 0.5, 0.4), (1.0, 0.5, 0.4))


def stars_blob_ic(s: StarsSetup, amp: float = 100.0, sigma: float = 4.0, rho0: float = 10.0):
    """quantum-stars.py:373-423: a uniform background plus Gaussian blobs in
    (x, y), normalised to <|psi|^2> = frac_dm rho_bar; stars uniform in the
    box with velocities uniform in [-1, 1), from np.random.seed(17).
    Returns (psi complex128, pos float64 [n_s,3], vel float64 [n_s,3])."""
    X, Y, _ = s.cell_centres()
    rho = np.full(X.shape, rho0)
    norm = sigma**3 * math.sqrt(2.0 * math.pi) ** 2
    for w, fx, fy in STARS_BLOBS:
        rho = rho + w * amp * np.exp(-((X - fx * s.Lx) ** 2 + (Y - fy * s.Ly) ** 2)
                                     / 2.0 / sigma**2) / norm
    rho = rho * (s.frac_dm * s.rho_bar / np.mean(rho))
    psi = np.sqrt(rho) + 0.0j
    np.random.seed(17)
    pos = np.random.uniform(0.0, 1.0, (s.n_s, 3)) * np.array([s.Lx, s.Ly, s.Lz])
    vel = np.random.uniform(-1.0, 1.0, (s.n_s, 3))
    return psi, pos, vel


def random_phase_psi(k_sq, sigma: float, m_per_hbar: float, mean_rho: float,
                     sort_by_k: bool):
    """Random-phase field with a Gaussian power spectrum (Eq. 27 of
    arXiv:1801.03507), normalised to <|psi|^2> = mean_rho.  sort_by_k: phases
    drawn in order of increasing k^2 (stable), quantum-fluid.py:511-522;
    otherwise in array order, quantum-bh.py:455-462.  np.random.seed(17)."""
    np.random.seed(17)
    if sort_by_k:
        sid = np.argsort(k_sq.flatten(), stable=True)
        flat = np.zeros(k_sq.size, dtype=complex)
        flat[sid] = np.exp(1.0j * 2.0 * np.pi * np.random.rand(k_sq.size))
        psi = flat.reshape(k_sq.shape)
    else:
        psi = np.exp(1.0j * 2.0 * np.pi * np.random.rand(*k_sq.shape))
    psi = psi * np.sqrt(np.exp(-k_sq / (2.0 * sigma**2 * m_per_hbar**2)))
    psi = np.fft.ifftn(psi)
    return psi * np.sqrt(mean_rho / np.mean(np.abs(psi) ** 2))


def soliton_psi(X, Y, Z, L: float, m_22: float, r_soliton: float):
    """Soliton profile centred in the box, quantum-bh.py:438-450:
    rho = 1.9e7 m22^-2 r_sol^-4 / (1 + 0.091 (r / r_sol)^2)^8."""
    r = np.sqrt((X - 0.5 * L) ** 2 + (Y - 0.5 * L) ** 2 + (Z - 0.5 * L) ** 2)
    rho = 1.9e7 * m_22**-2 * r_soliton**-4 / (1.0 + 0.091 * (r / r_soliton) ** 2) ** 8
    return np.sqrt(rho) + 0.0j


def k_squared(shape, L):
    """k^2 on the reference's grid (ifftshift of 2 pi / L arange(-n/2, n/2))."""
    ks = [np.fft.ifftshift(2.0 * np.pi / Ld * np.arange(-n / 2, n / 2))
          for n, Ld in zip(shape, L)]
    KX, KY, KZ = np.meshgrid(*ks, indexing="ij")
    return KX**2 + KY**2 + KZ**2


def _host(x):
    if isinstance(x, torch.Tensor):
        return x.detach().cpu().numpy()
    return np.asarray(x)


def save_state(path: str, state: dict) -> None:
    """Write a state dict (tensors or arrays, scalars) as an .npz file."""
    np.savez(path, **{k: _host(v) for k, v in state.items()})


def load_state(path: str, device=None, precision=FUSED_F32) -> dict:
    """Read a state dict written by save_state.  With a device, arrays become
    tensors of the precision's types (complex64/float32 or complex128/float64)
    and 0-d entries become Python floats."""
    out = {}
    with np.load(path) as z:
        for k in z.files:
            a = z[k]
            if a.ndim == 0 or device is None:
                out[k] = float(a) if a.ndim == 0 else a
                continue
            if np.iscomplexobj(a):
                dt = torch.complex64 if precision == FUSED_F32 else torch.complex128
            else:
                dt = torch.float32 if precision == FUSED_F32 else torch.float64
            out[k] = torch.as_tensor(a, dtype=dt, device=device).contiguous()
    return out


def run_stars(s: StarsSetup, outer: int = 100, checkpoint_dir: str | None = None,
              precision=FUSED_F32, device="cuda", state: dict | None = None,
              self_interaction: bool = False):
    """The main loop of quantum-stars.py:440-459 on the libqj step: ``outer``
    iterations of ``nt_sub`` steps, an .npz checkpoint after each
    (``checkpoint_dir/state_{i:03d}.npz``) and the reference's a-posteriori
    checks dt < 2 pi / (m/hbar) / dx / a_max and dt < dt_s.  Starts from the
    blob initial condition unless a state is given.  Returns the final state."""
    cdt = torch.complex64 if precision == FUSED_F32 else torch.complex128
    rdt = torch.float32 if precision == FUSED_F32 else torch.float64
    if state is None:
        psi, pos, vel = stars_blob_ic(s)
        state = {"t": 0.0,
                 "psi": torch.as_tensor(psi, dtype=cdt, device=device).contiguous(),
                 "pos": torch.as_tensor(pos, dtype=rdt, device=device).contiguous(),
                 "vel": torch.as_tensor(vel, dtype=rdt, device=device).contiguous(),
                 "a_max": 0.0, "dt_s": s.dt}
    step = StarsStep(s.grid(), s.phys(), s.m_s, s.dt, s.n_s,
                     self_interaction=self_interaction, precision=precision)
    dx = s.Lx / s.nx
    try:
        for i in range(outer):
            (state["psi"], state["pos"], state["vel"], t, a_max, dt_s) = step.compute_step(
                state["psi"], state["pos"], state["vel"], state["t"], state["a_max"],
                state["dt_s"], nsteps=s.nt_sub)
            state["t"], state["a_max"], state["dt_s"] = float(t), float(a_max), float(dt_s)
            if checkpoint_dir is not None:
                os.makedirs(checkpoint_dir, exist_ok=True)
                save_state(os.path.join(checkpoint_dir, f"state_{i:03d}.npz"), state)
            # a posteriori timestep checks, quantum-stars.py:448-449
            if state["a_max"] > 0.0:
                assert s.dt < 2.0 * math.pi / s.m_per_hbar / dx / state["a_max"]
            assert s.dt < state["dt_s"]
    finally:
        step.plan.close()
    return state
