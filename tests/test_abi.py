"""The C ABI library loads without a GPU and exports every declared symbol."""

import os
import re

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
