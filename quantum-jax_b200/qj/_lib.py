"""ctypes binding of libqj.so (the C ABI declared in include/qj.h).

The library is built in-tree (``python quantum-jax_b200/build.py``) and loaded
from this directory.  There is no fallback: if the library is missing or
fails to load, every entry point raises.
"""

from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqj.so")

QJ_OK = 0
QJ_ERR_ARG = 1
QJ_ERR_CUDA = 2
QJ_ERR_NONFINITE = 3
QJ_ERR_TIMEOUT = 4
QJ_ERR_ALLOC = 5
QJ_PLAIN_F64 = 0
QJ_FUSED_F32 = 1
QJ_TUNE_N = 12
QJ_TUNE_RADIX = 10
QJ_TUNE_TILE = 11
QJ_AUTOTUNE_SHAPES = 1

# Every symbol include/qj.h declares, with (restype, argtypes).
c_void_p, c_int, c_double, c_int64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int64


class QjGrid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
                ("Lx", c_double), ("Ly", c_double), ("Lz", c_double)]


class QjPhys(ctypes.Structure):
    _fields_ = [("m_per_hbar", c_double), ("G", c_double), ("rho_bar", c_double),
                ("b_coeff", c_double), ("cs", c_double), ("c_light", c_double)]


SIGNATURES = {
    "qj_plan_create": (c_int, [ctypes.POINTER(c_void_p), ctypes.POINTER(QjGrid),
                               ctypes.POINTER(QjPhys), c_int, c_int]),
    "qj_plan_destroy": (c_int, [c_void_p]),
    "qj_plan_create_batched": (c_int, [ctypes.POINTER(c_void_p), ctypes.POINTER(QjGrid),
                                       ctypes.POINTER(QjPhys), c_int, c_int, c_int]),
    "qj_ensemble_create": (c_int, [ctypes.POINTER(c_void_p), ctypes.POINTER(c_void_p), c_int]),
    "qj_ensemble_destroy": (c_int, [c_void_p]),
    "qj_ensemble_set_merge": (c_int, [c_void_p, c_int]),
    "qj_ensemble_merged": (c_int, [c_void_p]),
    "qj_ensemble_step": (c_int, [c_void_p, ctypes.POINTER(c_void_p), ctypes.POINTER(c_void_p),
                                 ctypes.POINTER(c_void_p), ctypes.POINTER(c_int),
                                 ctypes.POINTER(c_double), ctypes.POINTER(c_double),
                                 ctypes.POINTER(c_void_p), c_int, c_int, c_int, c_void_p]),
    "qj_plan_set_phys": (c_int, [c_void_p, ctypes.POINTER(QjPhys)]),
    "qj_last_error": (ctypes.c_char_p, []),
    "qj_get_potential": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
    "qj_bin_stars": (c_int, [c_void_p, c_void_p, c_int, c_double, c_void_p, c_void_p, c_void_p]),
    "qj_get_acceleration": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p,
                                    c_void_p]),
    "qj_kdk_step": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_double, c_double,
                            c_int, c_int, c_void_p, c_void_p, c_void_p]),
    "qj_fft3d": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
    "qj_kdk_gas_bh_step": (c_int, [c_void_p] + [c_void_p] * 8 + [c_int, c_double, c_int, c_double,
                                                                 c_int, c_double,
                                                                 ctypes.POINTER(c_double), c_void_p]),
    "qj_kdk_forward_ckpt": (c_int, [c_void_p, c_void_p, c_int, c_int, c_void_p, c_double, c_int,
                                    c_void_p, c_void_p, c_void_p]),
    "qj_kdk_adjoint": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_double, c_int,
                               c_void_p, c_void_p, c_void_p]),
    "qj_kdk_cosmo": (c_int, [c_void_p, c_void_p, ctypes.POINTER(c_double), c_double, c_double,
                             c_double, c_double, c_int, c_void_p]),
    "qj_get_potential_f32_noalloc": (c_int, [ctypes.POINTER(QjGrid), ctypes.POINTER(QjPhys),
                                             c_void_p, c_void_p, c_int, c_void_p]),
    "qj_plan_workspace_bytes": (c_int64, [c_void_p]),
    "qj_plan_status": (c_int, [c_void_p]),
    "qj_plan_selftest_wait": (c_int, [c_void_p, c_int64, c_void_p]),
    "qj_plan_get_tuning": (c_int, [c_void_p, c_void_p, c_int]),
    "qj_fluid_accretion_step": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                        c_void_p, c_void_p, c_void_p, c_double, c_int, c_void_p,
                                        c_void_p]),
    "qj_bondi_ambient": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                 c_void_p, c_double, c_double, c_double, c_double, c_double,
                                 c_double, c_double, c_void_p, c_void_p]),
    "qj_hydro_cfl_dt": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_double, c_double,
                                c_double, c_void_p, c_void_p]),
    "qj_plan_set_tuning": (c_int, [c_void_p, c_void_p, c_int]),
    "qj_autotune_kdk": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_double,
                                c_double, c_int, c_int, c_void_p]),
    "qj_selftest_sincos": (c_int, [c_void_p, c_void_p, c_int, c_void_p]),
    "qj_xla_kdk_step_f32": (None, [c_void_p, ctypes.POINTER(c_void_p), ctypes.c_char_p,
                                   ctypes.c_size_t, c_void_p]),
    "qj_xla_get_potential_f32": (None, [c_void_p, ctypes.POINTER(c_void_p), ctypes.c_char_p,
                                        ctypes.c_size_t, c_void_p]),
    "qj_xla_set_status_fn": (None, [c_void_p]),
    "qj_xla_last_status": (c_int, []),
    "qj_xla_release_plans": (c_int, []),
    "qj_launch_count": (c_int64, []),
    "qj_profile_enable": (c_int, [c_int]),
    "qj_profile_read": (c_int, [ctypes.POINTER(c_double), ctypes.POINTER(c_int64), c_int]),
}


QJ_XLA_DESC_VERSION = 1


class QjXlaKdkDesc(ctypes.Structure):
    """qj_xla_kdk_desc: the backend_config of a qj_xla_kdk_step_f32 custom call."""
    _fields_ = [("version", ctypes.c_int32), ("nsteps", ctypes.c_int32), ("n_s", ctypes.c_int32),
                ("self_interaction", ctypes.c_int32), ("has_v_ext", ctypes.c_int32),
                ("reserved", ctypes.c_int32), ("grid", QjGrid), ("phys", QjPhys),
                ("m_s", c_double), ("dt", c_double)]


class QjXlaPoissonDesc(ctypes.Structure):
    """qj_xla_poisson_desc: the backend_config of a qj_xla_get_potential_f32 call."""
    _fields_ = [("version", ctypes.c_int32), ("self_interaction", ctypes.c_int32),
                ("grid", QjGrid), ("phys", QjPhys)]


class QjFaccState(ctypes.Structure):
    _fields_ = [("t", c_double), ("M_acc", c_double), ("x_bh", c_double * 3),
                ("v_bh", c_double * 3), ("placed", c_double)]


class QjFaccParams(ctypes.Structure):
    _fields_ = [("cs", c_double), ("hydro_cfl", c_double), ("bh_on", c_int), ("bh_grav", c_int),
                ("bh_move", c_int), ("bh_accretion", c_int), ("bh_init_m", c_double),
                ("bh_inject_t", c_double), ("ramp_on", c_int), ("ramp_center", c_double),
                ("ramp_w", c_double), ("r_acc_mult", c_double), ("lam", c_double),
                ("fmax", c_double), ("ann_lo", c_double), ("ann_hi", c_double),
                ("k_cut_frac", c_double), ("inject_smooth_on", c_int),
                ("inject_smooth_kpc", c_double), ("rho_gas", c_double)]


class QjFaccDiag(ctypes.Structure):
    _fields_ = [(k, c_double) for k in ("dMdt", "rho_inf", "r_B", "dMdt_real", "cap_ratio",
                                        "r_acc_eff", "M_bh_eff_out", "dt_eff")]


class QjError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"libqj error {code}: {msg}")
        self.code = code


_lib = None


def lib():
    """Load libqj.so once; raise if it is absent (no CPU fallback exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python quantum-jax_b200/build.py`"
            )
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc):
    if rc != QJ_OK:
        msg = lib().qj_last_error()
        raise QjError(rc, msg.decode() if msg else "")
    return rc
