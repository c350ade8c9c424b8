"""The XLA custom-call targets, called as XLA calls them: an array of device
pointers (operands, then results), a packed descriptor as the opaque string,
XLA's stream.  Results must be bit-identical to the entry points the targets
wrap (qj_kdk_step on a fused float32 plan; qj_get_potential_f32_noalloc on
small grids, qj_get_potential on larger ones), whether XLA aliases each result
with its operand or hands separate result buffers."""

import ctypes

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def ptrs(*ts):
    return (ctypes.c_void_p * len(ts))(*[t.data_ptr() for t in ts])


def stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def bits(t):
    return (torch.view_as_real(t) if t.is_complex() else t).cpu().numpy().view(np.uint8)


@pytest.mark.parametrize("aliased", [True, False])
@pytest.mark.parametrize("n_s,si", [(64, False), (0, True)])
def test_xla_kdk_target_matches_kdk_step(aliased, n_s, si):
    import qj
    from qj import jax_ffi

    lib = qj.lib()
    psi, pos, vel, g, p = O.stars_ic(32, n_s, seed=2, shape=(32, 64, 16), L=(1.0, 2.0, 0.5))
    p.b_coeff = -0.1
    dt = O.default_dt(g, p)
    grid = qj.Grid(g.nx, g.ny, g.nz, g.Lx, g.Ly, g.Lz)
    phys = qj.Phys(m_per_hbar=1.0, G=p.G, rho_bar=p.rho_bar, b_coeff=p.b_coeff)
    dev = "cuda"

    def fresh():
        return (torch.as_tensor(psi, dtype=torch.complex64, device=dev),
                torch.as_tensor(pos.reshape(-1, 3), dtype=torch.float32, device=dev),
                torch.as_tensor(vel.reshape(-1, 3), dtype=torch.float32, device=dev),
                torch.tensor([0.0, 0.0, dt], dtype=torch.float64, device=dev))

    ref = fresh()
    plan = qj.Plan(grid, phys, qj.FUSED_F32, max(n_s, 1))
    plan.kdk_step(ref[0], ref[1] if n_s else None, ref[2] if n_s else None, ref[3], dt, 7, p.m_s,
                  si)
    plan.status()
    plan.close()

    ins = fresh()
    outs = ins if aliased else tuple(torch.full_like(t, float("nan")) for t in ins)
    opaque = jax_ffi.pack_kdk(grid, phys, n_s, p.m_s, dt, 7, self_interaction=si)
    for _ in range(2):  # the second call reuses the cached plan
        if not aliased:
            outs = tuple(torch.full_like(t, float("nan")) for t in ins)
        src = fresh()
        lib.qj_xla_kdk_step_f32(stream(), ptrs(*src, *outs) if not aliased else ptrs(*src, *src),
                                opaque, len(opaque), None)
        assert lib.qj_xla_last_status() == 0, lib.qj_last_error()
        got = src if aliased else outs
        torch.cuda.synchronize()
        for a, b in zip(got, ref):
            assert np.array_equal(bits(a), bits(b))
        if not aliased:  # operands are left as they were
            for a, b in zip(src, fresh()):
                assert np.array_equal(bits(a), bits(b))
    assert lib.qj_xla_release_plans() == 0


@pytest.mark.parametrize("shape", [(32, 64, 16), (128, 64, 32)])
def test_xla_poisson_target_matches_entry_points(shape):
    import qj
    from qj import _lib, jax_ffi

    lib = qj.lib()
    grid = qj.Grid(*shape, 2.0, 1.0, 1.0)
    phys = qj.Phys(m_per_hbar=1.0, G=1.0 / (4 * np.pi), rho_bar=1.02, b_coeff=0.05)
    rho = torch.as_tensor(1.0 + 0.1 * np.random.default_rng(1).standard_normal(shape),
                          dtype=torch.float32, device="cuda")
    for si in (False, True):
        V = torch.full_like(rho, float("nan"))
        opaque = jax_ffi.pack_poisson(grid, phys, si)
        lib.qj_xla_get_potential_f32(stream(), ptrs(rho, V), opaque, len(opaque), None)
        assert lib.qj_xla_last_status() == 0, lib.qj_last_error()
        if max(shape) <= 64:
            ref = torch.full_like(rho, float("nan"))
            g = _lib.QjGrid(*shape, 2.0, 1.0, 1.0)
            ph = _lib.QjPhys(phys.m_per_hbar, phys.G, phys.rho_bar, phys.b_coeff, phys.cs,
                             phys.c_light)
            assert lib.qj_get_potential_f32_noalloc(ctypes.byref(g), ctypes.byref(ph),
                                                    ctypes.c_void_p(rho.data_ptr()),
                                                    ctypes.c_void_p(ref.data_ptr()), int(si),
                                                    stream()) == 0
        else:
            plan = qj.Plan(grid, phys, qj.FUSED_F32, 1)
            ref = plan.get_potential(rho, self_interaction=si)
            torch.cuda.synchronize()
            plan.close()
        torch.cuda.synchronize()
        assert np.array_equal(bits(V), bits(ref))
        og = O.Grid(*shape, 2.0, 1.0, 1.0)
        op = O.Phys(m_per_hbar=1.0, G=phys.G, rho_bar=phys.rho_bar, b_coeff=phys.b_coeff)
        want = O.get_potential(rho.double().cpu().numpy(), og, op, self_interaction=si)
        assert O.rel_l2(V.double().cpu().numpy(), want) < 1e-5
    assert lib.qj_xla_release_plans() == 0
