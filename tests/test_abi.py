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
               "qj_profile_enable", "qj_profile_read", "qj_plan_workspace_bytes"}


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
