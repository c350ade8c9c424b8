"""Launch tuning of the fused passes (CTAs per SM, reserved slots, hydro block)
and the autotuner: every setting gives bit-identical results; the autotuner's
choice is cached and reused."""

import os

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def stars_state(n=64, n_s=64, seed=3):
    import qj

    psi, pos, vel, g, p = O.stars_ic(n, n_s, seed=seed)
    vel = 0.2 * np.random.default_rng(seed).standard_normal(pos.shape)
    plan = qj.Plan(qj.Grid(n, n, n), qj.Phys(m_per_hbar=1.0, G=p.G, rho_bar=p.rho_bar),
                   qj.FUSED_F32, n_s)

    def fresh():
        return (torch.as_tensor(psi, dtype=torch.complex64, device="cuda").contiguous(),
                torch.as_tensor(pos, dtype=torch.float32, device="cuda").contiguous(),
                torch.as_tensor(vel, dtype=torch.float32, device="cuda").contiguous(),
                torch.tensor([0.0, 0.0, O.default_dt(g, p)], dtype=torch.float64, device="cuda"))
    return plan, fresh, O.default_dt(g, p), p.m_s


def run(plan, fresh, dt, m_s, steps=5):
    s = fresh()
    plan.kdk_step(*s, dt, steps, m_s)
    plan.status()
    return [x.cpu() for x in s]


def test_tuning_is_bit_identical_and_cached(tmp_path):
    plan, fresh, dt, m_s = stars_state()
    ref = run(plan, fresh, dt, m_s)
    cache = str(tmp_path / "tuning.json")
    s = fresh()
    tuned = plan.autotune(s[0], s[1], s[2], m_s, dt, probe_steps=3, cache_file=cache)
    assert len(tuned) == 10 and os.path.exists(cache)
    assert all(0 <= k <= 32 for k in tuned[:8]) and -1 <= tuned[8] <= 64
    # the autotuner only read the state
    for x, y in zip(s, fresh()):
        assert torch.equal(x, y)
    for got in (run(plan, fresh, dt, m_s),):
        for x, y in zip(got, ref):
            assert torch.equal(x, y)
    plan.tuning = [1] * 8 + [0, 0]
    for x, y in zip(run(plan, fresh, dt, m_s), ref):
        assert torch.equal(x, y)
    # a second plan with the same key takes the cached choice without timing
    plan2, fresh2, _, _ = stars_state()
    s2 = fresh2()
    assert plan2.autotune(s2[0], s2[1], s2[2], m_s, dt, cache_file=cache) == tuned
    with pytest.raises(Exception):
        plan.tuning = [99] * 10
    plan.close()
    plan2.close()


def test_hydro_block_tuning_bit_identical():
    import qj

    n = 32
    g = O.Grid(n, n, n, 1.0, 1.0, 1.0)
    rho_dm = 1.0 + 0.1 * O.delta_field(n, 0)
    rho_g = 0.2 * (1.0 + 0.05 * O.delta_field(n, 1))
    phys = qj.Phys(m_per_hbar=1.0, G=1.0 / (4.0 * np.pi), rho_bar=float(rho_dm.mean()), cs=1.0)
    outs = []
    for block in (0, 64, 128):
        plan = qj.Plan(qj.Grid(n, n, n), phys, qj.FUSED_F32, 1)
        t = plan.tuning
        t[9] = block
        plan.tuning = t
        st = [torch.as_tensor(np.sqrt(rho_dm), dtype=torch.complex64, device="cuda").contiguous(),
              torch.as_tensor(rho_g, dtype=torch.float32, device="cuda").contiguous()]
        st += [torch.zeros((n, n, n), dtype=torch.float32, device="cuda") for _ in range(3)]
        plan.kdk_gas_bh(*st, None, None, None, O.default_dt(g, O.Phys()), 4, 0.0)
        outs.append([x.cpu() for x in st])
        plan.close()
    for o in outs[1:]:
        for x, y in zip(o, outs[0]):
            assert torch.equal(x, y)
