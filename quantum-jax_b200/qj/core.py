"""Torch front end of libqj: plans and the reference's step functions.

The reference scripts keep the grid and physical constants in module globals
(quantum-stars.py:61-157); here they live in a :class:`Plan`.  Every method
mirrors one reference function with the same argument meaning and returns
the same quantities; tensors are CUDA tensors and every call is asynchronous
on torch's current stream.
"""

from __future__ import annotations

import ctypes
import dataclasses
import math

import torch

from . import _lib
from ._lib import QJ_FUSED_F32, QJ_PLAIN_F64, check, lib

FUSED_F32 = QJ_FUSED_F32
PLAIN_F64 = QJ_PLAIN_F64


@dataclasses.dataclass
class Grid:
    """Box [0,Lx]x[0,Ly]x[0,Lz] with nx x ny x nz cells (quantum-stars.py:73-80)."""

    nx: int
    ny: int
    nz: int
    Lx: float = 1.0
    Ly: float = 1.0
    Lz: float = 1.0

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
    def ncell(self):
        return self.nx * self.ny * self.nz


@dataclasses.dataclass
class Phys:
    """Constants the reference reads as globals (quantum-stars.py:83-125)."""

    m_per_hbar: float = 1.0
    G: float = 1.0 / (4.0 * math.pi)
    rho_bar: float = 1.0
    b_coeff: float = 0.0
    cs: float = 1.0
    c_light: float = 299792.458


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def read_tuning_cache(path):
    """The autotuner's cache as a dict; a missing or unreadable file (e.g.
    one cut short by a crash) reads as empty, so tuning is redone."""
    import json
    import os

    if not os.path.exists(path):
        return {}
    try:
        with open(path) as f:
            cache = json.load(f)
    except (OSError, ValueError):
        return {}
    return cache if isinstance(cache, dict) else {}


def write_tuning_cache(path, cache):
    """Replace the cache file atomically (write a temporary file in the same
    folder, then rename): processes tuning at the same time never leave a
    half-written file; the last writer's entries win."""
    import json
    import os
    import tempfile

    folder = os.path.dirname(os.path.abspath(path))
    os.makedirs(folder, exist_ok=True)
    fd, tmp = tempfile.mkstemp(prefix=".tuning.", suffix=".json", dir=folder)
    try:
        with os.fdopen(fd, "w") as f:
            json.dump(cache, f, indent=1)
        os.replace(tmp, path)
    except BaseException:
        if os.path.exists(tmp):
            os.unlink(tmp)
        raise


class Plan:
    """A libqj plan: grid, constants, tables and device workspace.

    precision: ``FUSED_F32`` (complex64 psi, float32 fields and particles) or
    ``PLAIN_F64`` (complex128 / float64, unfused reference-order kernels).
    """

    def __init__(self, grid: Grid, phys: Phys, precision=FUSED_F32, max_particles=4096, nbox=1):
        self.grid = grid
        self.phys = phys
        self.precision = precision
        self.max_particles = int(max_particles)
        self.nbox = int(nbox)
        self.rdtype = torch.float32 if precision == FUSED_F32 else torch.float64
        self.cdtype = torch.complex64 if precision == FUSED_F32 else torch.complex128
        self._h = ctypes.c_void_p()
        g = _lib.QjGrid(grid.nx, grid.ny, grid.nz, grid.Lx, grid.Ly, grid.Lz)
        check(lib().qj_plan_create_batched(ctypes.byref(self._h), ctypes.byref(g),
                                           ctypes.byref(self._phys_struct()), int(precision),
                                           self.max_particles, self.nbox))

    def _phys_struct(self):
        p = self.phys
        return _lib.QjPhys(p.m_per_hbar, p.G, p.rho_bar, p.b_coeff, p.cs, p.c_light)

    def set_phys(self, phys: Phys):
        self.phys = phys
        check(lib().qj_plan_set_phys(self._h, ctypes.byref(self._phys_struct())))

    def close(self):
        if self._h:
            torch.cuda.synchronize()
            lib().qj_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def workspace_bytes(self):
        return int(lib().qj_plan_workspace_bytes(self._h))

    # ----- launch tuning -----
    @property
    def tuning(self):
        """The plan's launch tuning (QJ_TUNE_N ints, see include/qj.h)."""
        buf = (ctypes.c_int32 * _lib.QJ_TUNE_N)()
        check(lib().qj_plan_get_tuning(self._h, buf, _lib.QJ_TUNE_N))
        return list(buf)

    @tuning.setter
    def tuning(self, values):
        buf = (ctypes.c_int32 * _lib.QJ_TUNE_N)(*[int(v) for v in values])
        check(lib().qj_plan_set_tuning(self._h, buf, _lib.QJ_TUNE_N))

    def autotune(self, psi, pos, vel, m_s, dt, probe_steps=10, cache_file=None, shapes=True):
        """Pick the fused passes' launch tuning by timing qj_kdk_step on a
        copy of (psi, pos, vel); the arrays are only read.  shapes=True also
        picks the FFT radix plan and pencil tile of the 128- and 256-long
        axes (which change the rounding, within the single-precision bars);
        shapes=False keeps them and tunes only what is bit-identical (CTAs per
        SM, reserved slots).  Results are cached in a JSON file
        (QJ_TUNING_CACHE, default ~/.cache/qj/tuning.json) keyed by device,
        grid, boxes, stars, precision and the shapes flag; a cached entry is
        applied without timing.  Returns the tuning list."""
        import os

        n_s = 0 if pos is None else int(pos.shape[-2])
        key = "|".join(str(x) for x in (
            torch.cuda.get_device_name(psi.device), self.grid.nx, self.grid.ny, self.grid.nz,
            self.nbox, n_s, self.precision, "shapes" if shapes else "ctas"))
        path = cache_file or os.environ.get(
            "QJ_TUNING_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "qj", "tuning.json"))
        cache = read_tuning_cache(path)
        if key in cache and len(cache[key]) == _lib.QJ_TUNE_N:
            self.tuning = cache[key]
            return self.tuning
        ncell = self.grid.nx * self.grid.ny * self.grid.nz
        if (not psi.is_cuda or psi.dtype != self.cdtype or not psi.is_contiguous()
                or psi.numel() != self.nbox * ncell):
            raise ValueError(f"psi must be a contiguous CUDA {self.cdtype} tensor of "
                             f"{self.nbox} box(es) of {ncell} cells")
        for t, name in ((pos, "pos"), (vel, "vel")):
            if n_s and (not t.is_cuda or t.dtype != self.rdtype or not t.is_contiguous()
                        or t.numel() != self.nbox * n_s * 3):
                raise ValueError(f"{name} must be a contiguous CUDA {self.rdtype} tensor "
                                 f"[nbox, n_s, 3] (or [n_s, 3] for one box)")
        check(lib().qj_autotune_kdk(self._h, _ptr(psi), _ptr(pos) if n_s else None,
                                    _ptr(vel) if n_s else None, n_s, float(m_s), float(dt),
                                    int(probe_steps), _lib.QJ_AUTOTUNE_SHAPES if shapes else 0,
                                    _stream()))
        tuning = self.tuning
        cache = read_tuning_cache(path)  # entries other processes added meanwhile
        cache[key] = tuning
        write_tuning_cache(path, cache)
        return tuning

    def status(self):
        """Wait for the device; raise if a fused pass of this plan gave up a
        bounded wait for a tile copy since the last call."""
        check(lib().qj_plan_status(self._h))

    def selftest_wait(self, limit_ms=20.0):
        """Make one bounded device wait give up (nothing completes it) so that
        the next status() reports the timeout; exercises the failure path
        without a fault."""
        check(lib().qj_plan_selftest_wait(self._h, int(limit_ms * 1e6), _stream()))

    # ----- argument checks -----
    def _field(self, t, name, complex_=False):
        dt = self.cdtype if complex_ else self.rdtype
        if not isinstance(t, torch.Tensor) or not t.is_cuda:
            raise TypeError(f"{name} must be a CUDA tensor")
        if t.dtype != dt:
            raise TypeError(f"{name} must be {dt}, got {t.dtype}")
        if tuple(t.shape) != self.grid.shape or not t.is_contiguous():
            raise ValueError(f"{name} must be a contiguous {self.grid.shape} tensor")
        return t

    def _particles(self, t, name, n=None):
        if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != self.rdtype:
            raise TypeError(f"{name} must be a CUDA {self.rdtype} tensor")
        if t.dim() != 2 or t.shape[1] != 3 or not t.is_contiguous():
            raise ValueError(f"{name} must be a contiguous [n, 3] tensor")
        if n is not None and t.shape[0] != n:
            raise ValueError(f"{name} must have {n} rows")
        return t

    # ----- reference functions -----
    def get_potential(self, rho, self_interaction=False):
        """quantum-stars.py:189-193."""
        self._field(rho, "rho")
        V = torch.empty_like(rho)
        check(lib().qj_get_potential(self._h, _ptr(rho), _ptr(V), int(bool(self_interaction)),
                                     _stream()))
        return V

    def bin_stars(self, pos, m_s=None, masses=None):
        """quantum-stars.py:212-247 (m_s per star) / quantum-gas-bh.py:414-449
        (``masses`` per particle)."""
        self._particles(pos, "pos")
        n = pos.shape[0]
        if masses is not None:
            if masses.dtype != self.rdtype or masses.shape != (n,) or not masses.is_cuda:
                raise ValueError("masses must be a CUDA [n] tensor of the plan's real type")
        elif m_s is None:
            raise ValueError("give m_s or masses")
        rho = torch.empty(self.grid.shape, dtype=self.rdtype, device=pos.device)
        check(lib().qj_bin_stars(self._h, _ptr(pos), n, float(m_s or 0.0), _ptr(masses),
                                 _ptr(rho), _stream()))
        return rho

    def get_acceleration(self, pos, rho):
        """quantum-stars.py:250-288 -> (acc [n, 3], a_max 0-d float64 tensor)."""
        self._particles(pos, "pos")
        self._field(rho, "rho")
        acc = torch.empty_like(pos)
        a_max = torch.empty((), dtype=torch.float64, device=pos.device)
        check(lib().qj_get_acceleration(self._h, _ptr(pos), pos.shape[0], _ptr(rho), _ptr(acc),
                                        _ptr(a_max), _stream()))
        return acc, a_max

    def fftn(self, x, inverse=False):
        """jnp.fft.fftn / ifftn with the plan's pencil kernels."""
        self._field(x, "x", complex_=True)
        out = torch.empty_like(x)
        check(lib().qj_fft3d(self._h, _ptr(x), _ptr(out), 1 if inverse else -1, _stream()))
        return out

    def kdk_gas_bh(self, psi, rho, vx, vy, vz, m_bh, pos, vel, dt, nsteps=1, t=0.0,
                   sigma_v=None, dm_accretion=True, bondi_r_acc_mult=None):
        """nsteps x compute_step(psi, rho, vx, vy, vz, m_bh, pos, vel, t) of
        quantum-gas-bh.py:537-578, in place; returns t.  rho=None: no gas
        (quantum-bh.py).  bondi_r_acc_mult: optional isothermal Bondi gas sink
        (quantum-fluid-accretion-test.py:454-494)."""
        self._field(psi, "psi", complex_=True)
        gas = rho is not None
        if gas:
            for name, f in (("rho", rho), ("vx", vx), ("vy", vy), ("vz", vz)):
                self._field(f, name)
        n_bh = 0
        if pos is not None:
            self._particles(pos, "pos")
            n_bh = pos.shape[0]
            self._particles(vel, "vel", n_bh)
            if m_bh.dtype != self.rdtype or m_bh.shape != (n_bh,) or not m_bh.is_cuda:
                raise ValueError("m_bh must be a CUDA [n_bh] tensor of the plan's real type")
        t_io = ctypes.c_double(float(t))
        sv = self.phys.cs if sigma_v is None else float(sigma_v)
        check(lib().qj_kdk_gas_bh_step(
            self._h, _ptr(psi), _ptr(rho) if gas else None, _ptr(vx) if gas else None,
            _ptr(vy) if gas else None, _ptr(vz) if gas else None,
            _ptr(m_bh) if n_bh else None, _ptr(pos) if n_bh else None,
            _ptr(vel) if n_bh else None, n_bh, float(dt), int(nsteps), sv,
            int(bool(dm_accretion)), float(bondi_r_acc_mult or 0.0), ctypes.byref(t_io),
            _stream()))
        return t_io.value

    def bondi_ambient(self, rho, M_bh, x_bh, dt, v=None, v_bh=(0.0, 0.0, 0.0),
                      r_acc_mult=2.5, lam=math.exp(1.5) / 4.0, fmax=None, ann_lo=1.1,
                      ann_hi=1.8):
        """bh_bondi_step_ambient (quantum-fluid-accretion.py:440-510): rho is
        updated in place; returns (dMdt_target, rho_inf, rB, dM_cap, r_acc,
        M_avail, dM_uncl).  v = (vx, vy, vz) adds the BHL term with v_bh."""
        self._field(rho, "rho")
        if v is not None:
            for c, name in zip(v, ("vx", "vy", "vz")):
                self._field(c, name)
        out = torch.zeros(7, dtype=torch.float64, device=rho.device)
        xb = (ctypes.c_double * 3)(*[float(c) for c in x_bh])
        vb = (ctypes.c_double * 3)(*[float(c) for c in v_bh])
        check(lib().qj_bondi_ambient(
            self._h, _ptr(rho), _ptr(v[0]) if v is not None else None,
            _ptr(v[1]) if v is not None else None, _ptr(v[2]) if v is not None else None,
            xb, vb, float(M_bh), float(dt), float(r_acc_mult), float(lam),
            float(fmax) if fmax is not None else 0.0, float(ann_lo), float(ann_hi), _ptr(out),
            _stream()))
        return tuple(float(x) for x in out.cpu())

    def fluid_accretion_step(self, psi, rho, vx, vy, vz, state: dict, params: dict, dt,
                             nsteps=1):
        """nsteps x compute_step of quantum-fluid-accretion.py (:695-870) on a
        PLAIN_F64 plan, fields in place.  state: t, M_acc, x_bh (3), v_bh (3),
        placed -- updated; params: the script's toggles and constants (fields
        of QjFaccParams; booleans as 0/1).  Returns the last step's
        diagnostics (dMdt, rho_inf, r_B, dMdt_real, cap_ratio, r_acc_eff,
        M_bh_eff_out, dt_eff)."""
        self._field(psi, "psi", complex_=True)
        for f, name in ((rho, "rho"), (vx, "vx"), (vy, "vy"), (vz, "vz")):
            self._field(f, name)
        st = _lib.QjFaccState(float(state["t"]), float(state["M_acc"]),
                              (ctypes.c_double * 3)(*[float(x) for x in state["x_bh"]]),
                              (ctypes.c_double * 3)(*[float(x) for x in state["v_bh"]]),
                              float(state["placed"]))
        pr = _lib.QjFaccParams()
        for name, typ in _lib.QjFaccParams._fields_:
            setattr(pr, name, typ(params[name]).value if name in params else 0)
        dg = _lib.QjFaccDiag()
        check(lib().qj_fluid_accretion_step(self._h, _ptr(psi), _ptr(rho), _ptr(vx), _ptr(vy),
                                            _ptr(vz), ctypes.byref(st), ctypes.byref(pr),
                                            float(dt), int(nsteps), ctypes.byref(dg), _stream()))
        state.update(t=st.t, M_acc=st.M_acc, x_bh=list(st.x_bh), v_bh=list(st.v_bh),
                     placed=st.placed)
        return {name: getattr(dg, name) for name, _ in _lib.QjFaccDiag._fields_}

    def hydro_cfl_dt(self, vx, vy, vz, cs, cfl, dt):
        """min(dt, cfl dx / max(cs + |v|)), quantum-fluid-accretion.py:697-701."""
        for c, name in ((vx, "vx"), (vy, "vy"), (vz, "vz")):
            self._field(c, name)
        out = torch.zeros(1, dtype=torch.float64, device=vx.device)
        check(lib().qj_hydro_cfl_dt(self._h, _ptr(vx), _ptr(vy), _ptr(vz), float(cs), float(cfl),
                                    float(dt), _ptr(out), _stream()))
        return float(out.cpu())

    def kdk_cosmo(self, psi, a, da, H0, omega_m, omega_l, nsteps=1):
        """nsteps x compute_step(psi, a) of quantum-cosmo.py:169-196, in place;
        returns the new scale factor a."""
        self._field(psi, "psi", complex_=True)
        a_io = ctypes.c_double(float(a))
        check(lib().qj_kdk_cosmo(self._h, _ptr(psi), ctypes.byref(a_io), float(da), float(H0),
                                 float(omega_m), float(omega_l), int(nsteps), _stream()))
        return a_io.value

    def kdk_step(self, psi, pos, vel, diag, dt, nsteps=1, m_s=0.0, self_interaction=False,
                 v_ext=None):
        """nsteps x compute_step (quantum-stars.py:295-330), in place.

        diag: CUDA float64 tensor [3] = (t, a_max, dt_s), updated in place.
        A batched plan takes psi [nbox, nx, ny, nz], pos / vel [nbox, n_s, 3]
        and diag [nbox, 3]."""
        n_s = 0
        if self.nbox == 1:
            self._field(psi, "psi", complex_=True)
            if pos is not None:
                self._particles(pos, "pos")
                n_s = pos.shape[0]
                self._particles(vel, "vel", n_s)
        else:
            shape = (self.nbox,) + self.grid.shape
            if (not psi.is_cuda or psi.dtype != self.cdtype or tuple(psi.shape) != shape
                    or not psi.is_contiguous()):
                raise ValueError(f"psi must be a contiguous CUDA {self.cdtype} {shape} tensor")
            if pos is not None:
                for name, t in (("pos", pos), ("vel", vel)):
                    if (not t.is_cuda or t.dtype != self.rdtype or t.dim() != 3
                            or t.shape[0] != self.nbox or t.shape[2] != 3
                            or not t.is_contiguous()):
                        raise ValueError(f"{name} must be a contiguous [nbox, n_s, 3] tensor")
                n_s = pos.shape[1]
                if tuple(vel.shape) != tuple(pos.shape):
                    raise ValueError("vel must match pos")
        if diag.dtype != torch.float64 or diag.numel() != 3 * self.nbox or not diag.is_cuda:
            raise ValueError("diag must be a CUDA float64 tensor of 3 * nbox elements")
        if v_ext is not None:
            self._field(v_ext, "v_ext")
        check(lib().qj_kdk_step(self._h, _ptr(psi), _ptr(pos) if n_s else None,
                                _ptr(vel) if n_s else None, n_s, float(m_s), float(dt),
                                int(nsteps), int(bool(self_interaction)), _ptr(v_ext),
                                _ptr(diag), _stream()))
        return psi, pos, vel, diag


class Ensemble:
    """Independent boxes of uneven size stepped together: one batched plan per
    size, each on its own stream, with the step body captured once in a CUDA
    graph and replayed (qj_ensemble_step).  ``merge=True`` runs each fused
    pass as one persistent launch for all plans instead, when they are cubes
    of distinct sizes among 64, 96 and 128 (``merged`` tells); same bits,
    measured slower than the streams."""

    def __init__(self, plans, merge=False):
        self.plans = list(plans)
        self._h = ctypes.c_void_p()
        arr = (ctypes.c_void_p * len(self.plans))(*[p._h.value for p in self.plans])
        check(lib().qj_ensemble_create(ctypes.byref(self._h), arr, len(self.plans)))
        self.merge = merge

    @property
    def merge(self):
        return self._merge

    @merge.setter
    def merge(self, on):
        check(lib().qj_ensemble_set_merge(self._h, int(bool(on))))
        self._merge = bool(on)

    @property
    def merged(self):
        """True when a step runs one launch per fused pass for all plans."""
        rc = lib().qj_ensemble_merged(self._h)
        if rc < 0:
            check(rc)
        return rc == 1

    def step(self, psi, pos, vel, diag, dt, m_s, nsteps, chunk=10, graph=True):
        """psi / pos / vel / diag: per-plan tensors as for a batched
        Plan.kdk_step; dt, m_s: per-plan floats."""
        n = len(self.plans)
        P = ctypes.c_void_p * n
        n_s = [0 if p is None else int(p.shape[1] if p.dim() == 3 else p.shape[0]) for p in pos]
        check(lib().qj_ensemble_step(
            self._h, P(*[t.data_ptr() for t in psi]),
            P(*[0 if t is None else t.data_ptr() for t in pos]),
            P(*[0 if t is None else t.data_ptr() for t in vel]),
            (ctypes.c_int * n)(*n_s), (ctypes.c_double * n)(*[float(x) for x in m_s]),
            (ctypes.c_double * n)(*[float(x) for x in dt]),
            P(*[t.data_ptr() for t in diag]), int(nsteps), int(chunk), int(bool(graph)),
            _stream()))

    def close(self):
        if self._h:
            torch.cuda.synchronize()
            lib().qj_ensemble_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class StarsStep:
    """The quantum-stars.py step as a drop-in: ``compute_step`` and ``update``
    with the same signatures and state dict keys (quantum-stars.py:295-351).

    The constants the script holds as globals (grid, m_per_hbar, G, rho_bar,
    m_s, dt, b_coeff with --self_interaction) are given once here."""

    def __init__(self, grid: Grid, phys: Phys, m_s: float, dt: float, n_s: int,
                 self_interaction=False, precision=FUSED_F32, v_ext=None):
        self.plan = Plan(grid, phys, precision, max_particles=max(n_s, 1))
        self.m_s = float(m_s)
        self.dt = float(dt)
        self.self_interaction = self_interaction
        self.v_ext = v_ext

    def compute_step(self, psi, pos, vel, t, a_max, dt_s, nsteps=1):
        """Returns (psi, pos, vel, t, a_max, dt_s); tensors are updated in place."""
        dev = psi.device
        diag = torch.tensor([float(t), float(a_max), float(dt_s)], dtype=torch.float64,
                            device=dev)
        self.plan.kdk_step(psi, pos, vel, diag, self.dt, nsteps, self.m_s,
                           self.self_interaction, self.v_ext)
        return psi, pos, vel, diag[0], diag[1], diag[2]

    def update(self, _, state):
        """quantum-stars.py:333-351: one step on the state dict."""
        (state["psi"], state["pos"], state["vel"], state["t"], state["a_max"],
         state["dt_s"]) = self.compute_step(state["psi"], state["pos"], state["vel"],
                                            state["t"], state["a_max"], state["dt_s"])
        return state


class HostPipeline:
    """Host-resident states stepped on the device with the copies overlapped.

    The reference hands its state back to the host every nt_sub steps
    (quantum-stars.py:452-459).  For a sequence of states that live in host
    memory (an ensemble fed from the host, or snapshots written out), each
    call of ``run`` takes state i from pinned host memory, runs ``nsteps``
    KDK steps on it and writes the result to pinned host memory.  The device
    holds ``depth`` state buffers: while state i steps on the caller's current
    stream, state i + 1 is copied in on one copy stream and state i - 1
    copied out on another, so a call costs about the larger of the steps and
    one copy instead of their sum.  Results are the same bits as
    ``Plan.kdk_step`` on each state alone.

    inputs / outputs: sequences of (psi, pos, vel, diag) pinned CPU tensors
    (diag float64 [3] = t, a_max, dt_s; pos / vel None without stars).  The
    outputs are complete when the caller's current stream is (``run``
    returns once everything is enqueued)."""

    def __init__(self, plan: Plan, dt, nsteps, m_s=0.0, n_s=0, depth=3, self_interaction=False,
                 v_ext=None, device=None):
        if depth < 2:
            raise ValueError("depth must be at least 2")
        self.plan, self.dt, self.nsteps, self.m_s = plan, float(dt), int(nsteps), float(m_s)
        self.si, self.v_ext = self_interaction, v_ext
        dev = torch.device(device) if device is not None else torch.device("cuda")
        shape = plan.grid.shape
        self.bufs = []
        for _ in range(depth):
            ps = torch.empty(shape, dtype=plan.cdtype, device=dev)
            po = torch.empty((n_s, 3), dtype=plan.rdtype, device=dev) if n_s else None
            ve = torch.empty((n_s, 3), dtype=plan.rdtype, device=dev) if n_s else None
            dg = torch.empty(3, dtype=torch.float64, device=dev)
            self.bufs.append((ps, po, ve, dg))
        self.h2d = torch.cuda.Stream(device=dev)
        self.d2h = torch.cuda.Stream(device=dev)
        self.free = [None] * depth  # event: buffer b's last copy-out is done

    def run(self, inputs, outputs):
        cur = torch.cuda.current_stream()
        depth = len(self.bufs)
        for i, (hin, hout) in enumerate(zip(inputs, outputs)):
            b = i % depth
            buf = self.bufs[b]
            with torch.cuda.stream(self.h2d):
                if self.free[b] is not None:
                    self.h2d.wait_event(self.free[b])
                for d, h in zip(buf, hin):
                    if d is not None:
                        d.copy_(h, non_blocking=True)
                ev_in = torch.cuda.Event()
                ev_in.record(self.h2d)
            cur.wait_event(ev_in)
            ps, po, ve, dg = buf
            self.plan.kdk_step(ps, po, ve, dg, self.dt, self.nsteps, self.m_s, self.si,
                               self.v_ext)
            ev_done = torch.cuda.Event()
            ev_done.record(cur)
            with torch.cuda.stream(self.d2h):
                self.d2h.wait_event(ev_done)
                for h, d in zip(hout, buf):
                    if d is not None:
                        h.copy_(d, non_blocking=True)
                ev_free = torch.cuda.Event()
                ev_free.record(self.d2h)
                self.free[b] = ev_free
        cur.wait_stream(self.d2h)
        return outputs
