"""qj_get_potential_f32_noalloc: the allocation-free Poisson solve.

Callers such as an XLA FFI handler cannot let the library call cudaMalloc
(XLA holds most of the device memory and cudaMalloc / cudaFree would
synchronise its stream schedule); this entry point keeps its scratch in a
fixed device array instead.  It is checked through the C ABI against the
plan-based qj_get_potential (single precision, same tolerance as the other
float32 Poisson tests), on two calls in a row with different inputs, since
the scratch array is shared and keeps the previous call's contents, and on
its own against the float64 oracle.

The file name makes pytest collect it last.
"""

import ctypes

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-5  # rel-L2, as for the float32 get_potential parity test


def rel(a, b):
    return float(torch.linalg.vector_norm((a - b).double()) / torch.linalg.vector_norm(b.double()))


@pytest.mark.parametrize("shape,L", [((32, 64, 16), (2.0, 4.0, 1.0)), ((64, 64, 64), (1.0, 1.0, 1.0))])
def test_noalloc_matches_plan_two_calls(shape, L):
    import qj
    from qj import _lib

    lib = qj.lib()
    phys = qj.Phys(m_per_hbar=1.0, G=1.0 / (4 * np.pi), rho_bar=1.05, b_coeff=-0.03)
    plan = qj.Plan(qj.Grid(*shape, *L), phys, qj.FUSED_F32, 1)
    g = _lib.QjGrid(*shape, *L)
    ph = plan._phys_struct()
    rng = np.random.default_rng(0)
    for call in range(2):
        rho = torch.as_tensor(1.0 + 0.2 * rng.standard_normal(shape), dtype=torch.float32,
                              device="cuda")
        for si in (0, 1):
            V = torch.full(shape, float("nan"), dtype=torch.float32, device="cuda")
            stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
            rc = lib.qj_get_potential_f32_noalloc(ctypes.byref(g), ctypes.byref(ph),
                                                  ctypes.c_void_p(rho.data_ptr()),
                                                  ctypes.c_void_p(V.data_ptr()), si, stream)
            assert rc == 0, lib.qj_last_error()
            ref = plan.get_potential(rho, self_interaction=bool(si))
            torch.cuda.synchronize()
            assert torch.isfinite(V).all()
            assert rel(V, ref) < TOL, (call, si)
            # and on its own against the float64 oracle of quantum-stars.py:189-193
            og = O.Grid(*shape, *L)
            op = O.Phys(m_per_hbar=1.0, G=phys.G, rho_bar=phys.rho_bar, b_coeff=phys.b_coeff)
            want = O.get_potential(rho.double().cpu().numpy(), og, op, self_interaction=bool(si))
            assert O.rel_l2(V.double().cpu().numpy(), want) < TOL, (call, si)
    plan.close()


def test_noalloc_rejects_sizes_beyond_the_limit():
    import qj
    from qj import _lib

    lib = qj.lib()
    g = _lib.QjGrid(128, 64, 64, 1.0, 1.0, 1.0)
    ph = _lib.QjPhys(1.0, 1.0, 1.0, 0.0, 1.0, 1.0)
    x = torch.zeros(16, dtype=torch.float32, device="cuda")
    rc = lib.qj_get_potential_f32_noalloc(ctypes.byref(g), ctypes.byref(ph),
                                          ctypes.c_void_p(x.data_ptr()),
                                          ctypes.c_void_p(x.data_ptr()), 0, None)
    assert rc == _lib.QJ_ERR_ARG
    assert b"16, 32 or 64" in lib.qj_last_error()
