"""Failure detection without a GPU fault.

The fused passes wait for their tile copies with a bounded wait that gives up,
sets the plan's error word and lets the kernel return, instead of hanging the
GPU.  Here a wait that nothing completes (an mbarrier armed for bytes that no
copy brings) runs out after a short limit; qj_plan_status must report
QJ_ERR_TIMEOUT once, clear it, and leave the plan usable: the next step matches
a step on a fresh plan bit for bit.
"""

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _plan(qj, g, p, n_s):
    return qj.Plan(qj.Grid(g.nx, g.ny, g.nz, g.Lx, g.Ly, g.Lz),
                   qj.Phys(m_per_hbar=p.m_per_hbar, G=p.G, rho_bar=p.rho_bar, b_coeff=p.b_coeff),
                   qj.FUSED_F32, n_s)


def _step(plan, psi, pos, vel, dt, m_s, nsteps=3):
    ps = torch.as_tensor(psi, dtype=torch.complex64, device="cuda").contiguous()
    po = torch.as_tensor(pos, dtype=torch.float32, device="cuda").contiguous()
    ve = torch.as_tensor(vel, dtype=torch.float32, device="cuda").contiguous()
    diag = torch.tensor([0.0, 0.0, dt], dtype=torch.float64, device="cuda")
    plan.kdk_step(ps, po, ve, diag, dt, nsteps, m_s)
    return ps.cpu().numpy(), po.cpu().numpy()


def test_bounded_wait_gives_up_reports_and_recovers():
    import qj
    from qj._lib import QJ_ERR_TIMEOUT, QjError

    psi, pos, vel, g, p = O.stars_ic(32, 16, seed=5)
    dt = O.default_dt(g, p)
    plan = _plan(qj, g, p, len(pos))
    plan.status()  # nothing pending on a new plan

    plan.selftest_wait(20.0)  # 20 ms limit
    with pytest.raises(QjError) as ei:
        plan.status()
    assert ei.value.code == QJ_ERR_TIMEOUT
    plan.status()  # reported once, then cleared

    # the plan still works: the same step as on a fresh plan, bit for bit
    psi_a, pos_a = _step(plan, psi, pos, vel, dt, p.m_s)
    plan.status()
    plan.close()
    fresh = _plan(qj, g, p, len(pos))
    psi_b, pos_b = _step(fresh, psi, pos, vel, dt, p.m_s)
    fresh.status()
    fresh.close()
    assert np.array_equal(psi_a, psi_b)
    assert np.array_equal(pos_a, pos_b)


def test_selftest_limit_is_checked():
    import qj
    from qj._lib import QJ_ERR_ARG, QjError

    psi, pos, vel, g, p = O.stars_ic(16, 0, seed=0)
    plan = _plan(qj, g, p, 1)
    for bad in (0.0, 5000.0):  # below 1 ms, above 2 s
        with pytest.raises(QjError) as ei:
            plan.selftest_wait(bad)
        assert ei.value.code == QJ_ERR_ARG
    plan.status()
    plan.close()
