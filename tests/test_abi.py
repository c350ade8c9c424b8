"""The C ABI library loads without a GPU, exports every declared symbol, and
turns bad arguments into status codes before any CUDA call."""

import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if h.endswith(".h"):
            src = open(os.path.join(ROOT, "include", h)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names += re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(qj_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    import qj

    lib = qj.lib()
    names = declared_functions()
    assert "qj_kdk_step" in names and "qj_get_potential" in names
    for n in names:
        assert hasattr(lib, n), n
        assert n in qj._lib.SIGNATURES, f"{n} has no ctypes signature"


def test_error_path_without_gpu_is_a_status_not_a_crash():
    import ctypes

    import qj

    lib = qj.lib()
    rc = lib.qj_kdk_step(None, None, None, None, 0, 0.0, 1.0, 1, 0, None, None, None)
    assert rc == qj._lib.QJ_ERR_ARG
    assert b"bad argument" in lib.qj_last_error()
    h = ctypes.c_void_p()
    g = qj._lib.QjGrid(48, 32, 32, 1.0, 1.0, 1.0)
    ph = qj._lib.QjPhys(1.0, 1.0, 1.0, 0.0, 1.0, 1.0)
    assert lib.qj_plan_create(ctypes.byref(h), ctypes.byref(g), ctypes.byref(ph), 1, 8) == 1
    assert b"unsupported" in lib.qj_last_error()


# Entry points whose zero / null call is defined to succeed: destroying
# nothing, the error text, the launch counter, the profiler switches, and the
# workspace size of no plan (0).
_OK_ON_NULL = {"qj_plan_destroy", "qj_ensemble_destroy", "qj_last_error", "qj_launch_count",
               "qj_profile_enable", "qj_profile_read", "qj_plan_workspace_bytes",
               "qj_xla_set_status_fn", "qj_xla_last_status", "qj_xla_release_plans"}
# XLA custom-call targets return nothing; their status is qj_xla_last_status().
_VOID_TARGETS = {"qj_xla_kdk_step_f32", "qj_xla_get_potential_f32"}


def _zero_args(argtypes):
    import ctypes

    vals = []
    for a in argtypes:
        if a in (ctypes.c_int, ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64, ctypes.c_size_t):
            vals.append(0)
        elif a in (ctypes.c_double, ctypes.c_float):
            vals.append(0.0)
        else:
            vals.append(None)
    return vals


def test_every_entry_point_rejects_null_arguments_without_a_gpu():
    """Null plans, tensors and sizes come back as QJ_ERR_ARG with a message,
    checked before any CUDA call (no exception, no exit, no crash across the
    ABI)."""
    import qj

    lib = qj.lib()
    for name, (_, argtypes) in sorted(qj._lib.SIGNATURES.items()):
        if name in _OK_ON_NULL:
            continue
        rc = getattr(lib, name)(*_zero_args(argtypes))
        if name in _VOID_TARGETS:
            rc = lib.qj_xla_last_status()
        assert rc == qj._lib.QJ_ERR_ARG, name
        assert lib.qj_last_error(), name
    n = qj._lib.QJ_TUNE_N
    assert lib.qj_plan_get_tuning(None, None, n) == qj._lib.QJ_ERR_ARG
    assert lib.qj_plan_set_tuning(None, None, n) == qj._lib.QJ_ERR_ARG
    assert lib.qj_plan_destroy(None) == 0


@pytest.mark.parametrize("dims,prec,max_particles,nbox,text", [
    ((32, 32, 24), 1, 8, 1, "length 24 unsupported"),
    ((17, 32, 32), 1, 8, 1, "length 17 unsupported"),
    ((32, 32, 32), 7, 8, 1, "precision must be"),
    ((32, 32, 32), 1, -1, 1, "max_particles must be"),
    ((32, 32, 32), 0, 8, 2, "batches need QJ_FUSED_F32"),
    ((32, 32, 32), 1, 8, 0, "nbox must be"),
])
def test_plan_create_rejects_bad_configurations(dims, prec, max_particles, nbox, text):
    import ctypes

    import qj

    lib = qj.lib()
    h = ctypes.c_void_p()
    g = qj._lib.QjGrid(*dims, 1.0, 1.0, 1.0)
    ph = qj._lib.QjPhys(1.0, 1.0, 1.0, 0.0, 1.0, 1.0)
    rc = lib.qj_plan_create_batched(ctypes.byref(h), ctypes.byref(g), ctypes.byref(ph), prec,
                                    max_particles, nbox)
    assert rc == qj._lib.QJ_ERR_ARG and h.value is None
    assert text.encode() in lib.qj_last_error()


def test_valid_plan_without_a_device_is_a_cuda_status():
    import ctypes

    import qj
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    lib = qj.lib()
    h = ctypes.c_void_p()
    g = qj._lib.QjGrid(32, 32, 32, 1.0, 1.0, 1.0)
    ph = qj._lib.QjPhys(1.0, 1.0, 1.0, 0.0, 1.0, 1.0)
    rc = lib.qj_plan_create(ctypes.byref(h), ctypes.byref(g), ctypes.byref(ph), 1, 8)
    assert rc == qj._lib.QJ_ERR_CUDA and h.value is None
    assert b"CUDA error" in lib.qj_last_error()


def test_xla_descriptors_match_the_c_layout():
    """The packed backend_config of each XLA target has the size the library
    expects: a descriptor of the right length with a bad field is rejected as
    a bad descriptor (not a wrong length), one byte short as a wrong length;
    no CUDA call is reached."""
    import ctypes

    import qj
    from qj import jax_ffi

    lib = qj.lib()
    g, ph = qj.Grid(32, 32, 32), qj.Phys()
    bufs = (ctypes.c_void_p * 8)()
    good = jax_ffi.pack_kdk(g, ph, n_s=-1, m_s=0.0, dt=1.0, nsteps=1)
    assert len(good) == ctypes.sizeof(qj._lib.QjXlaKdkDesc) == 128
    lib.qj_xla_kdk_step_f32(None, bufs, good, len(good), None)
    assert lib.qj_xla_last_status() == qj._lib.QJ_ERR_ARG
    assert b"bad descriptor" in lib.qj_last_error()
    lib.qj_xla_kdk_step_f32(None, bufs, good, len(good) - 1, None)
    assert b"descriptor of 127 bytes, expected 128" in lib.qj_last_error()
    pot = jax_ffi.pack_poisson(g, ph)
    assert len(pot) == ctypes.sizeof(qj._lib.QjXlaPoissonDesc)
    lib.qj_xla_get_potential_f32(None, bufs, pot, len(pot), None)
    assert lib.qj_xla_last_status() == qj._lib.QJ_ERR_ARG
    assert b"null buffer" in lib.qj_last_error()


def test_xla_failure_reaches_the_status_function():
    """A failing target hands its message to the status function the binding
    installs (jaxlib's XlaCustomCallStatusSetFailure in a JAX process)."""
    import ctypes

    import qj

    lib = qj.lib()
    seen = []
    FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t)
    cb = FN(lambda status, msg, n: seen.append((status, msg[:n])))
    lib.qj_xla_set_status_fn(ctypes.cast(cb, ctypes.c_void_p))
    try:
        lib.qj_xla_kdk_step_f32(None, None, b"x", 1, ctypes.c_void_p(0x1234))
    finally:
        lib.qj_xla_set_status_fn(None)
    assert seen and seen[0][0] == 0x1234 and b"descriptor of 1 bytes" in seen[0][1]
