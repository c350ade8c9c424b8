"""qj.HostPipeline: states in pinned host memory stepped with overlapped
copies give the same bits as qj_kdk_step on each state alone."""

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("depth", [2, 3])
def test_pipeline_bit_identical_to_single_calls(depth):
    import qj

    n, n_s, steps = 32, 64, 3
    states = []
    for seed in range(5):
        psi, pos, vel, g, p = O.stars_ic(n, n_s, seed=seed)
        vel = 0.2 * np.random.default_rng(seed).standard_normal(pos.shape)
        states.append((psi, pos, vel))
    dt = O.default_dt(g, p)
    grid = qj.Grid(n, n, n)
    phys = qj.Phys(m_per_hbar=1.0, G=p.G, rho_bar=p.rho_bar)
    plan = qj.Plan(grid, phys, qj.FUSED_F32, n_s)

    def host(psi, pos, vel):
        return (torch.as_tensor(psi, dtype=torch.complex64).pin_memory(),
                torch.as_tensor(pos, dtype=torch.float32).pin_memory(),
                torch.as_tensor(vel, dtype=torch.float32).pin_memory(),
                torch.tensor([0.0, 0.0, dt], dtype=torch.float64).pin_memory())

    ins = [host(*s) for s in states]
    outs = [tuple(torch.full_like(t, float("nan")).pin_memory() for t in h) for h in ins]
    pipe = qj.HostPipeline(plan, dt, steps, m_s=p.m_s, n_s=n_s, depth=depth)
    pipe.run(ins, outs)
    torch.cuda.current_stream().synchronize()
    plan.status()
    for h, o in zip(ins, outs):
        d = [t.cuda() for t in h]
        plan.kdk_step(d[0], d[1], d[2], d[3], dt, steps, p.m_s)
        ref = [t.cpu() for t in d]
        for x, y in zip(o, ref):
            xr = torch.view_as_real(x) if x.is_complex() else x
            yr = torch.view_as_real(y) if y.is_complex() else y
            assert torch.equal(xr, yr)
    plan.close()
