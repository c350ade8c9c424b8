"""Generate the golden vectors that pin the oracle to the reference.

The reference (pmocz/quantum-jax) is a set of JAX scripts; JAX 0.5.3 is not
installable here (no network).  This script executes the reference scripts'
OWN functions, unmodified, with ``jax.numpy`` replaced by a float64 NumPy
stand-in (``jnp.X`` -> ``numpy.X``; ``x.at[i].add/set`` -> copy-and-update;
``jax.lax.fori_loop`` -> a Python loop; ``jax.jit`` -> identity) and orbax /
matplotlib / h5py / IPython replaced by inert stubs (nothing is written to
disk).  The scripts' physics, constants, k-grids, CIC weights, limiter, fluxes
and step orchestration are therefore the reference's own code; only the array
backend differs (float64 NumPy instead of XLA, i.e. the reference run with
x64 enabled).

Inputs are seeded synthetic fields in each script's own units and grid (the
``--res 1`` configuration).  Outputs are stored as checksums (sum, sum of
squares, a seeded random projection) plus a strided subsample for grids and
in full for particle arrays, in ``tests/golden/*.npz``.

Run from the repository root, in a container where the reference is mounted:

    python tests/golden/make_golden.py [reference_dir]

The GPU box does not have the reference; the tests only read the .npz files.
"""

from __future__ import annotations

import argparse as _argparse
import importlib.util
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))

from oracle import oracle as O  # noqa: E402


# ---------------------------------------------------------------------------
# float64 NumPy stand-in for jax / jax.numpy
# ---------------------------------------------------------------------------


class AtArray(np.ndarray):
    """ndarray with JAX's functional ``.at[idx].add/set`` update syntax."""

    @property
    def at(self):
        return _At(self)


class _At:
    def __init__(self, arr):
        self.arr = arr

    def __getitem__(self, idx):
        return _AtIdx(self.arr, idx)


class _AtIdx:
    def __init__(self, arr, idx):
        self.arr, self.idx = arr, idx

    def add(self, v):
        out = np.array(self.arr, copy=True).view(AtArray)
        out[self.idx] += v
        return out

    def set(self, v):
        out = np.array(self.arr, copy=True).view(AtArray)
        out[self.idx] = v
        return out


def _as_at(x):
    if isinstance(x, np.ndarray) and not isinstance(x, AtArray):
        return x.view(AtArray)
    if isinstance(x, tuple):
        return tuple(_as_at(y) for y in x)
    if isinstance(x, list):
        return [_as_at(y) for y in x]
    return x


def _wrap(fn):
    def w(*a, **k):
        return _as_at(fn(*a, **k))

    return w


def _proxy_module(name, target):
    mod = types.ModuleType(name)

    def __getattr__(attr):
        obj = getattr(target, attr)
        if callable(obj) and not isinstance(obj, type):
            return _wrap(obj)
        return obj

    mod.__getattr__ = __getattr__
    return mod


class _Inert:
    """Stand-in object: every attribute / call returns another inert object."""

    def __getattr__(self, name):
        return _Inert()

    def __call__(self, *a, **k):
        return _Inert()

    def __getitem__(self, key):
        return _Inert()

    def __setitem__(self, key, value):
        pass


def _install_stubs():
    jnp = _proxy_module("jax.numpy", np)
    jnp.fft = _proxy_module("jax.numpy.fft", np.fft)
    jax = types.ModuleType("jax")
    jax.numpy = jnp
    lax = types.ModuleType("jax.lax")

    def fori_loop(lo, hi, body, init_val):
        v = init_val
        for i in range(int(lo), int(hi)):
            v = body(i, v)
        return v

    def lax_slice(x, start, limit):
        return x[tuple(slice(s, e) for s, e in zip(start, limit))]

    lax.fori_loop = fori_loop
    lax.slice = lax_slice
    jax.lax = lax
    jax.jit = lambda f=None, **k: (f if f is not None else (lambda g: g))
    jax.block_until_ready = lambda x: x
    jax.config = types.SimpleNamespace(update=lambda *a, **k: None)
    sys.modules["jax"] = jax
    sys.modules["jax.numpy"] = jnp
    sys.modules["jax.lax"] = lax
    for name in (
        "orbax", "orbax.checkpoint", "matplotlib", "matplotlib.pyplot",
        "matplotlib.animation", "matplotlib.patches", "h5py", "IPython",
        "IPython.display", "imageio_ffmpeg", "imageio", "imageio.v2", "imageio.v3",
        "cmasher", "matplotlib.patheffects",
    ):
        m = types.ModuleType(name)
        m.__getattr__ = lambda attr: _Inert()
        sys.modules[name] = m


def load_reference(ref_dir, script, argv=()):
    """Execute ``script`` from the reference with the stand-ins installed."""
    _install_stubs()
    path = os.path.join(ref_dir, script)
    old = sys.argv
    sys.argv = [path, *argv]
    try:
        spec = importlib.util.spec_from_file_location(
            "ref_" + script.replace("-", "_").replace(".py", ""), path
        )
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
    finally:
        sys.argv = old
    return mod


# ---------------------------------------------------------------------------
# checksums
# ---------------------------------------------------------------------------


def summarize(prefix, a, out):
    a = np.asarray(a)
    out[prefix + ".shape"] = np.array(a.shape)
    out[prefix + ".sum"] = np.array(np.sum(a))
    out[prefix + ".sumsq"] = np.array(np.sum(np.abs(a) ** 2))
    w = np.random.default_rng(12345).standard_normal(a.shape)
    out[prefix + ".proj"] = np.array(np.sum(w * a))
    if a.ndim == 3:
        s = 1
        while a[::s, ::s, ::s].size > 4096:
            s += 1
        out[prefix + ".stride"] = np.array(s)
        out[prefix + ".sub"] = a[::s, ::s, ::s].copy()
    else:
        out[prefix + ".full"] = a.copy()


def plain(a):
    return np.asarray(a).view(np.ndarray)


# ---------------------------------------------------------------------------
# per-script golden cases
# ---------------------------------------------------------------------------


def gen_stars(ref_dir):
    ref = load_reference(ref_dir, "quantum-stars.py", ["--res", "1"])
    g = O.Grid(ref.nx, ref.ny, ref.nz, ref.Lx, ref.Ly, ref.Lz)
    rho_dm = ref.frac_dm * ref.rho_bar * (1.0 + 0.1 * O.delta_field(0, 0, g.shape))
    psi = np.sqrt(rho_dm).astype(np.complex128)
    rng = np.random.default_rng(1)
    pos = rng.uniform(0.0, 1.0, (ref.n_s, 3)) * np.array([g.Lx, g.Ly, g.Lz])
    vel = np.random.default_rng(2).uniform(-1.0, 1.0, (ref.n_s, 3))
    out = {}
    out["const.G"] = np.array(ref.G)
    out["const.m_per_hbar"] = np.array(ref.m_per_hbar)
    out["const.rho_bar"] = np.array(ref.rho_bar)
    out["const.m_s"] = np.array(ref.m_s)
    out["const.dt"] = np.array(ref.dt)
    out["const.nt"] = np.array(ref.nt)
    out["const.nt_sub"] = np.array(ref.nt_sub)
    out["const.grid"] = np.array([g.nx, g.ny, g.nz, g.Lx, g.Ly, g.Lz])
    out["input.rho_dm0"] = np.array(ref.frac_dm * ref.rho_bar)
    out["input.n_s"] = np.array(ref.n_s)
    rho_s = ref.bin_stars(_as_at(pos))
    rho_tot = np.abs(psi) ** 2 + plain(rho_s)
    summarize("bin_stars", plain(rho_s), out)
    summarize("get_potential", plain(ref.get_potential(_as_at(rho_tot))), out)
    acc, a_max = ref.get_acceleration(_as_at(pos), _as_at(rho_tot))
    summarize("get_acceleration.acc", plain(acc), out)
    out["get_acceleration.a_max"] = np.array(float(a_max))
    k = ref.kx, ref.ky, ref.kz, ref.k_sq
    summarize("k_sq", plain(k[3]), out)
    state = {"psi": _as_at(psi), "pos": _as_at(pos), "vel": _as_at(vel),
             "t": 0.0, "a_max": 0.0, "dt_s": ref.dt}
    for i in range(2):
        state = ref.update(i, state)
    for key in ("psi", "pos", "vel"):
        summarize("step2." + key, plain(state[key]), out)
    for key in ("t", "a_max", "dt_s"):
        out["step2." + key] = np.array(float(state[key]))
    # self-interaction variant: b_coeff and V + b rho (quantum-stars.py:117-125, 193)
    ref_si = load_reference(ref_dir, "quantum-stars.py", ["--res", "1", "--self_interaction"])
    out["si.b_coeff"] = np.array(float(ref_si.b_coeff))
    summarize("si.get_potential", plain(ref_si.get_potential(_as_at(rho_tot))), out)
    np.savez_compressed(os.path.join(HERE, "stars_res1.npz"), **out)


def gen_gasbh(ref_dir):
    ref = load_reference(ref_dir, "quantum-gas-bh.py", ["--res", "1"])
    n, L = ref.nx, ref.Lx
    g = O.Grid(n, n, n, L, L, L)
    rho0 = ref.M_soliton / L**3
    psi = np.sqrt(rho0 * (1.0 + 0.1 * O.delta_field(n, 3))).astype(np.complex128)
    rho = 0.1 * rho0 * (1.0 + 0.05 * O.delta_field(n, 4))
    rng = np.random.default_rng(5)
    vx, vy, vz = (0.1 * ref.cs * rng.standard_normal(g.shape) for _ in range(3))
    m_bh = ref.M_bh * np.ones(1)
    pos = np.array([[0.6 * L, 0.5 * L, 0.5 * L]])
    vel = np.array([[0.0, 40.0, 0.0]])
    ref.rho_bar = float(np.mean(np.abs(psi) ** 2))
    out = {}
    out["const.G"] = np.array(ref.G)
    out["const.m_per_hbar"] = np.array(ref.m_per_hbar)
    out["const.cs"] = np.array(ref.cs)
    out["const.c"] = np.array(ref.c)
    out["const.dt"] = np.array(ref.dt)
    out["const.rho_bar"] = np.array(ref.rho_bar)
    out["const.grid"] = np.array([n, n, n, L, L, L])
    out["input.rho0"] = np.array(rho0)
    out["input.M_bh"] = np.array(ref.M_bh)
    h = ref.solve_hydro(_as_at(rho), _as_at(vx), _as_at(vy), _as_at(vz), ref.dt)
    for name, a in zip(("rho", "vx", "vy", "vz"), h):
        summarize("solve_hydro." + name, plain(a), out)
    m_big = np.array([1.0e11])
    p2, m2 = ref.do_accretion(_as_at(psi), _as_at(pos), _as_at(vel), _as_at(m_big))
    summarize("do_accretion.psi", plain(p2), out)
    out["do_accretion.m_bh"] = plain(m2).copy()
    state = {"psi": _as_at(psi), "rho": _as_at(rho), "vx": _as_at(vx), "vy": _as_at(vy),
             "vz": _as_at(vz), "m_bh": _as_at(m_bh), "pos": _as_at(pos),
             "vel": _as_at(vel), "t": 0.0}
    for i in range(2):
        state = ref.update(i, state)
    for key in ("psi", "rho", "vx", "vy", "vz", "m_bh", "pos", "vel"):
        summarize("step2." + key, plain(state[key]), out)
    out["step2.t"] = np.array(float(state["t"]))
    np.savez_compressed(os.path.join(HERE, "gasbh_res1.npz"), **out)


def gen_tidal(ref_dir):
    ref = load_reference(ref_dir, "quantum-tidal.py", ["--res", "1"])
    n, L = ref.nx, ref.Lx
    rho0 = ref.M_soliton / L**3
    psi = np.sqrt(rho0 * (1.0 + 0.1 * O.delta_field(n, 6))).astype(np.complex128)
    psi = psi * np.exp(1.0j * ref.k_soliton * plain(ref.X))
    ref.rho_bar = float(np.mean(np.abs(psi) ** 2) + ref.M_halo / L**3)
    out = {}
    out["const.G"] = np.array(ref.G)
    out["const.m_per_hbar"] = np.array(ref.m_per_hbar)
    out["const.M_halo"] = np.array(ref.M_halo)
    out["const.dt"] = np.array(ref.dt)
    out["const.rho_bar"] = np.array(ref.rho_bar)
    out["const.grid"] = np.array([n, n, n, L, L, L])
    out["input.rho0"] = np.array(rho0)
    out["input.k_soliton"] = np.array(ref.k_soliton)
    summarize("external_potential", plain(ref.external_potential()), out)
    state = {"psi": _as_at(psi), "t": 0.0}
    for i in range(2):
        state = ref.update(i, state)
    summarize("step2.psi", plain(state["psi"]), out)
    out["step2.t"] = np.array(float(state["t"]))
    np.savez_compressed(os.path.join(HERE, "tidal_res1.npz"), **out)


def gen_cosmo(ref_dir):
    ref = load_reference(ref_dir, "quantum-cosmo.py", ["--res", "1"])
    out = {}
    out["const.G"] = np.array(ref.G)
    out["const.m_per_hbar"] = np.array(ref.m_per_hbar)
    out["const.rho_bar"] = np.array(ref.rho_bar)
    out["const.H0"] = np.array(ref.H0)
    out["const.omega_matter"] = np.array(ref.omega_matter)
    out["const.omega_lambda"] = np.array(ref.omega_lambda)
    out["const.a_start"] = np.array(ref.a_start)
    out["const.da"] = np.array(ref.da)
    a0 = ref.a_start
    out["compute_dt.a_start"] = np.array(float(ref.compute_dt(a0, ref.da)))
    out["compute_dt.a_half"] = np.array(float(ref.compute_dt(0.5, ref.da)))
    # The script's own 256^3 k-grid is replaced by the same construction on a
    # 32^3 grid of the same box, so the step runs at fixture size.
    n, L = 32, ref.Lx
    kl = 2.0 * np.pi / L * np.arange(-n / 2, n / 2)
    kx, ky, kz = np.meshgrid(kl, kl, kl, indexing="ij")
    kx, ky, kz = (np.fft.ifftshift(a) for a in (kx, ky, kz))
    ref.k_sq = _as_at(kx**2 + ky**2 + kz**2)
    psi = np.sqrt(ref.rho_bar * (1.0 + 0.1 * O.delta_field(n, 7))).astype(np.complex128)
    state = {"psi": _as_at(psi), "a": a0}
    for i in range(2):
        state = ref.update(i, state)
    summarize("step2.psi", plain(state["psi"]), out)
    out["step2.a"] = np.array(float(state["a"]))
    out["const.grid"] = np.array([n, n, n, L, L, L])
    np.savez_compressed(os.path.join(HERE, "cosmo_n32.npz"), **out)


def gen_bondi(ref_dir):
    ref = load_reference(ref_dir, "quantum-fluid-accretion-test.py", ["--res", "1"])
    n, L = ref.nx, ref.Lx
    rho = ref.rho_gas * (1.0 + 0.05 * O.delta_field(n, 8))
    x_bh = np.array([0.5 * L, 0.52 * L, 0.47 * L])
    out = {}
    out["const.grid"] = np.array([n, n, n, L, L, L])
    out["const.cs"] = np.array(ref.cs)
    out["const.G"] = np.array(ref.G)
    out["const.dt"] = np.array(ref.dt)
    out["input.rho_gas"] = np.array(ref.rho_gas)
    for tag, M in (("m1e8", 1.0e8), ("m1e10", 1.0e10)):
        r = ref.bh_bondi_step_no_vrel(
            rho=_as_at(rho), M_bh=M, x_bh=_as_at(x_bh), dx=ref.dx, Lx=L,
            cs=ref.cs, G=ref.G, dt=ref.dt,
        )
        summarize(f"bondi.{tag}.rho", plain(r[0]), out)
        out[f"bondi.{tag}.scalars"] = np.array([float(v) for v in r[1:]])
    np.savez_compressed(os.path.join(HERE, "bondi_res1.npz"), **out)


def gen_bondi_ambient(ref_dir):
    """bh_bondi_step_ambient (quantum-fluid-accretion.py:440-510), with and
    without the BHL velocity term, and the hydro CFL step (:697-701) with the
    script's own cs2_local and HYDRO_CFL."""
    ref = load_reference(ref_dir, "quantum-fluid-accretion.py", [])
    n, L, dx = ref.nx, ref.Lx, ref.dx
    rho = ref.rho_gas * (1.0 + 0.05 * O.delta_field(n, 9))
    rng = np.random.default_rng(10)
    vx, vy, vz = (5.0 * rng.standard_normal((n, n, n)) for _ in range(3))
    x_bh = np.array([0.5 * L, 0.52 * L, 0.47 * L])
    v_bh = (12.0, -7.0, 3.0)
    out = {}
    out["const.grid"] = np.array([n, n, n, L, L, L])
    out["const.cs"] = np.array(ref.cs_const)
    out["const.G"] = np.array(ref.G)
    out["const.dt"] = np.array(ref.dt)
    out["const.r_acc_mult"] = np.array(ref.R_ACC_MULT)
    out["const.ann"] = np.array([ref.ann_lo, ref.ann_hi])
    out["input.rho_gas"] = np.array(ref.rho_gas)
    for tag, M, bhl in (("m1e8", 1.0e8, False), ("m1e10_bhl", 1.0e10, True)):
        kw = dict(vx=_as_at(vx), vy=_as_at(vy), vz=_as_at(vz), vxbh=v_bh[0], vybh=v_bh[1],
                  vzbh=v_bh[2]) if bhl else {}
        r = ref.bh_bondi_step_ambient(rho=_as_at(rho), M_bh_eff=M, x_bh=_as_at(x_bh), dx=dx,
                                      Lx=L, cs_iso=ref.cs_const, G=ref.G, dt=ref.dt, **kw)
        summarize(f"amb.{tag}.rho", plain(r[0]), out)
        out[f"amb.{tag}.scalars"] = np.array([float(v) for v in r[1:]])
    c_eff = np.sqrt(plain(ref.cs2_local(_as_at(rho))))
    vmag = np.sqrt(vx * vx + vy * vy + vz * vz)
    out["cfl.dt_eff"] = np.array(min(ref.dt, ref.HYDRO_CFL * dx / (np.max(c_eff + vmag) + 1e-30)))
    out["cfl.dt_big"] = np.array(min(1.0, ref.HYDRO_CFL * dx / (np.max(c_eff + vmag) + 1e-30)))
    out["const.hydro_cfl"] = np.array(ref.HYDRO_CFL)
    np.savez_compressed(os.path.join(HERE, "bondi_ambient.npz"), **out)


def facc_params_of(ref):
    """The step's toggles and constants as read from the loaded script."""
    return np.array([ref.cs_const, ref.HYDRO_CFL, ref.BH_INIT_M, ref.BH_INJECT_T,
                     ref.BH_RAMP_CENTER, ref.BH_RAMP_W, ref.R_ACC_MULT, ref.LAMBDA_ISO,
                     ref.ann_lo, ref.ann_hi, ref.K_CUT_FRAC, ref.INJECT_SMOOTH_KPC, ref.rho_gas,
                     float(ref.BH_ON), float(ref.BH_GRAV), float(ref.BH_MOVE),
                     float(ref.BH_ACCRETION), float(ref.BH_RAMP_ON), float(ref.INJECT_SMOOTH_ON)])


def facc_inputs(ref):
    n = ref.nx
    rho_dm = ref.rho_bar * ref.frac_dm * (1.0 + 0.1 * O.delta_field(n, 11))
    psi = np.sqrt(rho_dm) * np.exp(1.0j * 0.3 * O.delta_field(n, 12))
    rho = ref.rho_gas * (1.0 + 0.05 * O.delta_field(n, 13))
    rng = np.random.default_rng(14)
    v = [10.0 * rng.standard_normal((n, n, n)) for _ in range(3)]
    return psi, rho, v


def gen_facc(ref_dir):
    """compute_step of quantum-fluid-accretion.py (:695-870), two steps from two
    seeded states: one crossing the injection time (the black hole is placed
    at the smoothed dark-matter peak), one with a placed, ramped, moving black
    hole (softened gravity, low-pass force, ambient Bondi sink)."""
    ref = load_reference(ref_dir, "quantum-fluid-accretion.py", [])
    L = ref.Lx
    psi0, rho0, v0 = facc_inputs(ref)
    out = {"const.params": facc_params_of(ref), "const.grid": np.array([ref.nx, L, ref.dx]),
           "const.G": np.array(ref.G), "const.m_per_hbar": np.array(ref.m_per_hbar),
           "const.dt": np.array(ref.dt), "const.rho_bar": np.array(ref.rho_bar)}
    cases = {
        "inject": (ref.BH_INJECT_T - 0.5 * ref.dt, 0.0, [0.5 * L] * 3, [0.0, 0.0, 0.0], 0.0),
        "massive": (ref.BH_RAMP_CENTER, 2.0e6, [0.43 * L, 0.55 * L, 0.61 * L], [20.0, -10.0, 5.0],
                    1.0),
    }
    for tag, (t, M_acc, x_bh, v_bh, placed) in cases.items():
        st = [_as_at(psi0), _as_at(rho0), _as_at(v0[0]), _as_at(v0[1]), _as_at(v0[2]), t, M_acc,
              _as_at(np.array(x_bh)), v_bh[0], v_bh[1], v_bh[2], placed]
        for step in (1, 2):
            r = ref.compute_step(*st)
            (psi, rho, vx, vy, vz, t, M_out, M_acc, x_b, vbx, vby, vbz, dMdt, rho_inf, r_B,
             placed, dMdt_real, cap_ratio, r_acc_eff) = r[:19]
            pre = f"{tag}.s{step}."
            summarize(pre + "psi", plain(psi), out)
            summarize(pre + "rho", plain(rho), out)
            summarize(pre + "vx", plain(vx), out)
            out[pre + "scalars"] = np.array([float(x) for x in (
                t, M_out, M_acc, *plain(x_b), float(vbx), float(vby), float(vbz), float(placed),
                dMdt, rho_inf, r_B, dMdt_real, cap_ratio, r_acc_eff)])
            st = [psi, rho, vx, vy, vz, t, M_acc, x_b, vbx, vby, vbz, placed]
    np.savez_compressed(os.path.join(HERE, "facc_steps.npz"), **out)


def gen_bh(ref_dir):
    ref = load_reference(ref_dir, "quantum-bh.py", ["--res", "1"])
    n, L = ref.nx, ref.Lx
    psi = np.sqrt(ref.rho_bar * (1.0 + 0.1 * O.delta_field(n, 9))).astype(np.complex128)
    psi = psi * np.exp(0.3j * O.delta_field(n, 10))
    pos = np.array([[0.5 * L, 0.5 * L, 0.5 * L]])
    vel = np.array([[10.0, -5.0, 3.0]])
    m_bh = ref.M_bh * np.ones(1)
    out = {}
    out["const.grid"] = np.array([n, n, n, L, L, L])
    out["const.sigma"] = np.array(ref.sigma)
    out["const.G"] = np.array(ref.G)
    out["const.m_per_hbar"] = np.array(ref.m_per_hbar)
    out["const.c"] = np.array(ref.c)
    out["const.dt"] = np.array(ref.dt)
    out["const.rho_bar"] = np.array(ref.rho_bar)
    out["input.M_bh"] = np.array(ref.M_bh)
    p2, m2 = ref.do_accretion(_as_at(psi), _as_at(pos), _as_at(vel), _as_at(m_bh))
    summarize("do_accretion.psi", plain(p2), out)
    out["do_accretion.m_bh"] = plain(m2).copy()
    np.savez_compressed(os.path.join(HERE, "bh_res1.npz"), **out)


def run_ic_block(mod):
    """Execute the initial-condition block of the script's own main() (the
    lines from "# Initial Conditions" up to "# Construct initial simulation
    state") in the module's namespace; returns that namespace."""
    import inspect
    import textwrap

    lines = textwrap.dedent(inspect.getsource(mod.main)).splitlines()[1:]
    i0 = next(i for i, ln in enumerate(lines) if "# Initial Conditions" in ln)
    i1 = next(i for i, ln in enumerate(lines) if "# Construct initial simulation state" in ln)
    ns = dict(vars(mod))
    exec(textwrap.dedent("\n".join(lines[i0:i1])), ns)
    return ns


def gen_ics(ref_dir):
    """Initial conditions of quantum-stars (Gaussian blobs, seeded stars),
    quantum-fluid (sorted random phases), quantum-bh (random phases and the
    soliton), from the scripts' own main() code."""
    out = {}
    ref = load_reference(ref_dir, "quantum-stars.py", ["--res", "1"])
    ns = run_ic_block(ref)
    summarize("stars.psi", plain(ns["psi"]), out)
    out["stars.pos"] = plain(ns["pos"]).copy()
    out["stars.vel"] = plain(ns["vel"]).copy()
    ref = load_reference(ref_dir, "quantum-fluid.py", ["--res", "1"])
    ns = run_ic_block(ref)
    summarize("fluid.psi", plain(ns["psi"]), out)
    out["fluid.const"] = np.array([ref.nx, ref.Lx, ref.sigma, ref.m_per_hbar, ref.frac_dm,
                                   ref.rho_bar, ref.rho_gas])
    ref = load_reference(ref_dir, "quantum-bh.py", ["--res", "1"])
    ns = run_ic_block(ref)
    summarize("bh.psi", plain(ns["psi"]), out)
    out["bh.const"] = np.array([ref.nx, ref.Lx, ref.sigma, ref.m_per_hbar, ref.rho_bar])
    ref = load_reference(ref_dir, "quantum-bh.py", ["--res", "1", "--soliton"])
    ns = run_ic_block(ref)
    summarize("soliton.psi", plain(ns["psi"]), out)
    out["soliton.const"] = np.array([ref.nx, ref.Lx, ref.m_22, ref.r_soliton])
    np.savez_compressed(os.path.join(HERE, "ic_res1.npz"), **out)


def main():
    ap = _argparse.ArgumentParser()
    ap.add_argument("ref_dir", nargs="?", default=os.environ.get("QJ_REFERENCE_DIR"),
                    help="checkout of the reference scripts (or $QJ_REFERENCE_DIR)")
    ap.add_argument("--only", default=None, help="generate one case, e.g. gen_ics")
    a = ap.parse_args()
    if not a.ref_dir:
        ap.error("give the reference checkout as ref_dir or in $QJ_REFERENCE_DIR")
    fns = (gen_stars, gen_gasbh, gen_tidal, gen_cosmo, gen_bondi, gen_bh, gen_ics, gen_bondi_ambient, gen_facc)
    for fn in fns:
        if a.only and fn.__name__ != a.only:
            continue
        print(fn.__name__, flush=True)
        fn(a.ref_dir)


if __name__ == "__main__":
    main()
