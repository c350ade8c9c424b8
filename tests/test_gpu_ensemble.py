"""Batched plans and ensembles of uneven boxes (IC ensemble, one seed per box).

A batched plan must give, box by box, the same bits as single-box plans; the
graph-captured ensemble the same bits as eager stepping; and each box must
match the float64 oracle within the single-precision bar (rel-L2 <= 1e-5).
"""

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def boxes(n, seeds, n_s):
    out = []
    for s in seeds:
        psi, pos, vel, g, p = O.stars_ic(n, n_s, seed=s)
        vel = 0.2 * np.random.default_rng(s + 7).standard_normal(pos.shape)
        out.append((psi, pos, vel, g, p))
    return out


def tensors(bx):
    psi = torch.as_tensor(np.stack([b[0] for b in bx]), dtype=torch.complex64, device="cuda")
    pos = torch.as_tensor(np.stack([b[1] for b in bx]), dtype=torch.float32, device="cuda")
    vel = torch.as_tensor(np.stack([b[2] for b in bx]), dtype=torch.float32, device="cuda")
    dt = O.default_dt(bx[0][3], bx[0][4])
    diag = torch.tensor([[0.0, 0.0, dt]] * len(bx), dtype=torch.float64, device="cuda")
    return psi.contiguous(), pos.contiguous(), vel.contiguous(), diag, dt


def plan_for(bx, nbox):
    import qj

    g, p = bx[0][3], bx[0][4]
    return qj.Plan(qj.Grid(g.nx, g.ny, g.nz), qj.Phys(m_per_hbar=1.0, G=p.G, rho_bar=p.rho_bar),
                   qj.FUSED_F32, bx[0][1].shape[0], nbox=nbox)


def test_batched_equals_single_box_plans():
    bx = boxes(32, [100, 101, 102], 64)
    psi, pos, vel, diag, dt = tensors(bx)
    m_s = bx[0][4].m_s
    plan = plan_for(bx, 3)
    plan.kdk_step(psi, pos, vel, diag, dt, 5, m_s)
    torch.cuda.synchronize()
    single = plan_for(bx, 1)
    for b in range(3):
        ps = torch.as_tensor(bx[b][0], dtype=torch.complex64, device="cuda")
        po = torch.as_tensor(bx[b][1], dtype=torch.float32, device="cuda")
        ve = torch.as_tensor(bx[b][2], dtype=torch.float32, device="cuda")
        d = torch.tensor([0.0, 0.0, dt], dtype=torch.float64, device="cuda")
        single.kdk_step(ps, po, ve, d, dt, 5, m_s)
        torch.cuda.synchronize()
        assert torch.equal(ps, psi[b]) and torch.equal(po, pos[b]) and torch.equal(ve, vel[b])
        assert torch.equal(d, diag[b])
    plan.close()
    single.close()


def test_ensemble_graph_matches_eager_and_oracle():
    import qj

    groups = [boxes(32, [100, 101, 102, 103], 32), boxes(64, [104, 105], 32),
              boxes(96, [106], 32)]
    state_a = [tensors(bx) for bx in groups]
    state_b = [tuple(t.clone() if isinstance(t, torch.Tensor) else t for t in s) for s in state_a]
    plans = [plan_for(bx, len(bx)) for bx in groups]
    ens = qj.Ensemble(plans)
    dts = [s[4] for s in state_a]
    m_s = [bx[0][4].m_s for bx in groups]
    nsteps = 6
    ens.step([s[0] for s in state_a], [s[1] for s in state_a], [s[2] for s in state_a],
             [s[3] for s in state_a], dts, m_s, nsteps, chunk=2, graph=True)
    ens.step([s[0] for s in state_b], [s[1] for s in state_b], [s[2] for s in state_b],
             [s[3] for s in state_b], dts, m_s, nsteps, chunk=2, graph=False)
    torch.cuda.synchronize()
    for sa, sb in zip(state_a, state_b):
        for x, y in zip(sa[:4], sb[:4]):
            assert torch.equal(x, y)
    # one box of each size against the float64 oracle
    for bx, s in zip(groups, state_a):
        psi0, pos0, vel0, g, p = bx[-1]
        ref = O.stars_run(psi0, pos0, vel0, nsteps, g, p, s[4])
        assert O.rel_l2(s[0][-1].cpu().numpy(), ref[0]) < 1e-5
        assert O.rel_l2(s[1][-1].cpu().numpy(), ref[1]) < 1e-5
    ens.close()
    for pl in plans:
        pl.close()


def test_single_launch_per_pass_equals_per_plan_streams():
    """Plans of 64^3, 96^3 and 128^3 share one launch per fused pass; that
    gives the same bits as stepping each plan on its own stream, eager and
    graph-captured, with stars on some plans and none on another."""
    import qj

    groups = [boxes(64, [140, 141, 142], 64), boxes(96, [143, 144], 32), boxes(128, [145], 0)]
    plans = [plan_for(bx, len(bx)) for bx in groups]
    results = []
    for merge, graph in ((True, True), (True, False), (False, True)):
        state = [tensors(bx) for bx in groups]
        ens = qj.Ensemble(plans, merge=merge)
        assert ens.merged == merge
        m_s = [bx[0][4].m_s for bx in groups]
        pos = [s[1] if bx[0][1].shape[0] else None for s, bx in zip(state, groups)]
        vel = [s[2] if bx[0][1].shape[0] else None for s, bx in zip(state, groups)]
        ens.step([s[0] for s in state], pos, vel, [s[3] for s in state], [s[4] for s in state],
                 m_s, 7, chunk=3, graph=graph)
        torch.cuda.synchronize()
        for pl in plans:
            pl.status()
        results.append(state)
        ens.close()
    for other in results[1:]:
        for sa, sb in zip(results[0], other):
            for x, y in zip(sa[:4], sb[:4]):
                assert torch.equal(x, y)
    # and a plan with a shape variant in its tuning keeps the per-plan streams
    t = plans[2].tuning
    t[11] = 1 << 2
    plans[2].tuning = t
    ens = qj.Ensemble(plans, merge=True)
    assert not ens.merged
    ens.close()
    for pl in plans:
        pl.close()


def test_ensemble_every_box_of_the_32_box_mix():
    """The 32-box mix (16 x 64^3, 8 x 96^3, 8 x 128^3, 256 stars each), 10
    graph-captured steps as one launch per fused pass for all sizes: every box
    against the plain float64 path (itself matched to the oracle), and the
    first 128^3 box against the float64 oracle directly."""
    import qj

    groups = [boxes(64, range(100, 116), 256), boxes(96, range(116, 124), 256),
              boxes(128, range(124, 132), 256)]
    state = [tensors(bx) for bx in groups]
    plans = [plan_for(bx, len(bx)) for bx in groups]
    ens = qj.Ensemble(plans, merge=True)
    assert ens.merged
    nsteps = 10
    m_s = [bx[0][4].m_s for bx in groups]
    ens.step([s[0] for s in state], [s[1] for s in state], [s[2] for s in state],
             [s[3] for s in state], [s[4] for s in state], m_s, nsteps, chunk=5, graph=True)
    torch.cuda.synchronize()
    for bx, s, ms in zip(groups, state, m_s):
        g, p = bx[0][3], bx[0][4]
        pl64 = qj.Plan(qj.Grid(g.nx, g.ny, g.nz),
                       qj.Phys(m_per_hbar=1.0, G=p.G, rho_bar=p.rho_bar), qj.PLAIN_F64, 256)
        for b, (psi0, pos0, vel0, _, _) in enumerate(bx):
            ps = torch.as_tensor(psi0, dtype=torch.complex128, device="cuda")
            po = torch.as_tensor(pos0, dtype=torch.float64, device="cuda")
            ve = torch.as_tensor(vel0, dtype=torch.float64, device="cuda")
            d = torch.tensor([0.0, 0.0, s[4]], dtype=torch.float64, device="cuda")
            pl64.kdk_step(ps, po, ve, d, s[4], nsteps, ms)
            torch.cuda.synchronize()
            got = s[0][b].to(torch.complex128)
            err = float(torch.linalg.vector_norm(got - ps) / torch.linalg.vector_norm(ps))
            assert err < 1e-5, (g.nx, b, err)
            assert O.rel_l2(s[1][b].double().cpu().numpy(), po.cpu().numpy()) < 1e-5
        pl64.close()
    psi0, pos0, vel0, g, p = groups[2][0]
    ref = O.stars_run(psi0, pos0, vel0, nsteps, g, p, state[2][4])
    assert O.rel_l2(state[2][0][0].cpu().numpy(), ref[0]) < 1e-5
    assert O.rel_l2(state[2][1][0].cpu().numpy(), ref[1]) < 1e-5
    ens.close()
    for pl in plans:
        pl.close()


@pytest.mark.parametrize("dbl", [False, True])
def test_fft_radix3_length_96(dbl):
    import qj

    for shape in [(96, 96, 96), (96, 32, 96), (32, 96, 16)]:
        plan = qj.Plan(qj.Grid(*shape), qj.Phys(), qj.PLAIN_F64 if dbl else qj.FUSED_F32, 1)
        rng = np.random.default_rng(1)
        x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
        ct = torch.complex128 if dbl else torch.complex64
        y = plan.fftn(torch.as_tensor(x, dtype=ct, device="cuda")).cpu().numpy()
        assert O.rel_l2(y, np.fft.fftn(x)) < (1e-13 if dbl else 2e-6)
        plan.close()
