"""GPU parity of the gas + black-hole step (quantum-gas-bh.py:537-578) against
the float64 oracle: plain float64 path rel-L2 <= 1e-10, fused float32 path
rel-L2 <= 1e-5 for psi and the gas density (1e-4 for the small gas velocities).
"""

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def gas_ic(n=32, seed=0, vamp=0.05):
    g = O.Grid(n, n, n, 1.0, 1.0, 1.0)
    rho_dm = 1.0 + 0.1 * O.delta_field(n, seed)
    psi = np.sqrt(rho_dm).astype(np.complex128)
    rho = 0.2 * (1.0 + 0.05 * O.delta_field(n, seed + 1))
    rng = np.random.default_rng(seed + 2)
    vx, vy, vz = (vamp * rng.standard_normal(g.shape) for _ in range(3))
    M = 0.01 * (rho_dm.sum() + rho.sum()) * g.vol
    m_bh = np.array([M])
    pos = np.array([[0.5, 0.5, 0.5]]) + 0.013
    vel = np.array([[0.02, -0.01, 0.03]])
    p = O.Phys(m_per_hbar=1.0, G=1.0 / (4.0 * np.pi), rho_bar=rho_dm.mean(), cs=1.0, c_light=0.3)
    return g, p, psi, rho, vx, vy, vz, m_bh, pos, vel


def run(precision, g, p, state, dt, nsteps, bondi=None, gas=True, dm_acc=True):
    import qj

    dbl = precision == qj.PLAIN_F64
    ct = torch.complex128 if dbl else torch.complex64
    rt = torch.float64 if dbl else torch.float32
    plan = qj.Plan(qj.Grid(g.nx, g.ny, g.nz, g.Lx, g.Ly, g.Lz),
                   qj.Phys(m_per_hbar=p.m_per_hbar, G=p.G, rho_bar=p.rho_bar, cs=p.cs,
                           c_light=p.c_light), precision, 4)
    psi, rho, vx, vy, vz, m_bh, pos, vel = state

    def c(a, t):
        return torch.as_tensor(np.ascontiguousarray(a), dtype=t, device="cuda")

    T = [c(psi, ct)] + ([c(a, rt) for a in (rho, vx, vy, vz)] if gas else [None] * 4) + \
        [c(m_bh, rt), c(pos, rt), c(vel, rt)]
    t = plan.kdk_gas_bh(*T, dt, nsteps, 0.0, dm_accretion=dm_acc, bondi_r_acc_mult=bondi)
    torch.cuda.synchronize()
    out = [x.cpu().numpy() if x is not None else None for x in T]
    plan.close()
    return out, t


def oracle(g, p, state, dt, nsteps, bondi=None, gas=True, dm_acc=True):
    psi, rho, vx, vy, vz, m_bh, pos, vel = state
    k = O.kgrid(g)
    if not gas:
        rho = vx = vy = vz = None
    t = 0.0
    for _ in range(nsteps):
        psi, rho, vx, vy, vz, m_bh, pos, vel, t = O.gasbh_compute_step(
            psi, rho, vx, vy, vz, m_bh, pos, vel, t, g, p, dt, k, bondi_r_acc_mult=bondi,
            dm_accretion=dm_acc)
    return [psi, rho, vx, vy, vz, m_bh, pos, vel], t


@pytest.mark.parametrize("bondi", [None, 2.0])
def test_gas_bh_plain_f64(bondi):
    import qj

    g, p, *state = gas_ic()
    dt = O.default_dt(g, p)
    got, t = run(qj.PLAIN_F64, g, p, state, dt, 3, bondi)
    ref, tr = oracle(g, p, state, dt, 3, bondi)
    for i, name in enumerate(["psi", "rho", "vx", "vy", "vz", "m_bh", "pos", "vel"]):
        assert O.rel_l2(got[i], ref[i]) < 1e-10, name
    assert t == pytest.approx(tr, rel=1e-14)


@pytest.mark.parametrize("bondi", [None, 2.0])
def test_gas_bh_fused_f32(bondi):
    import qj

    g, p, *state = gas_ic()
    dt = O.default_dt(g, p)
    got, _ = run(qj.FUSED_F32, g, p, state, dt, 3, bondi)
    ref, _ = oracle(g, p, state, dt, 3, bondi)
    assert O.rel_l2(got[0], ref[0]) < 1e-5
    assert O.rel_l2(got[1], ref[1]) < 1e-5
    for i in (2, 3, 4):
        assert O.rel_l2(got[i], ref[i]) < 1e-4
    assert O.rel_l2(got[5], ref[5]) < 1e-5
    assert O.rel_l2(got[6], ref[6]) < 1e-6
    assert O.rel_l2(got[7], ref[7]) < 1e-4


def test_bh_without_gas_both_precisions():
    """quantum-bh.py:346-381: dark matter + black hole, no gas."""
    import qj

    g, p, *state = gas_ic(seed=5)
    dt = O.default_dt(g, p)
    ref, _ = oracle(g, p, state, dt, 3, gas=False)
    got, _ = run(qj.PLAIN_F64, g, p, state, dt, 3, gas=False)
    assert O.rel_l2(got[0], ref[0]) < 1e-10
    assert O.rel_l2(got[5], ref[5]) < 1e-10
    got, _ = run(qj.FUSED_F32, g, p, state, dt, 3, gas=False)
    assert O.rel_l2(got[0], ref[0]) < 1e-5
    assert O.rel_l2(got[5], ref[5]) < 1e-5


def test_hydro_uniform_state_is_fixed_point_and_mass_conserved():
    """Known answers: a uniform gas at rest stays uniform; flux form conserves
    gas mass to round-off (no black hole, no dark-matter gravity)."""
    import qj

    n = 32
    g = O.Grid(n, n, n, 1.0, 1.0, 1.0)
    p = O.Phys(m_per_hbar=1.0, G=0.0, rho_bar=1.0, cs=1.0)
    psi = np.ones(g.shape, dtype=np.complex128)
    rho = np.full(g.shape, 0.3)
    z = np.zeros(g.shape)
    dt = O.default_dt(g, p)
    for prec, tol in ((qj.PLAIN_F64, 1e-15), (qj.FUSED_F32, 1e-7)):
        got, _ = run(prec, g, p, [psi, rho, z, z, z, np.zeros(1), np.zeros((1, 3)),
                                  np.zeros((1, 3))], dt, 2, dm_acc=False)
        assert np.abs(got[1] - 0.3).max() < tol * 10
        assert np.abs(got[2]).max() < tol
    rho2 = 0.3 * (1.0 + 0.2 * O.delta_field(n, 3))
    v = 0.1 * np.random.default_rng(0).standard_normal(g.shape)
    got, _ = run(qj.PLAIN_F64, g, p, [psi, rho2, v, -v, 0.5 * v, np.zeros(1), np.zeros((1, 3)),
                                      np.zeros((1, 3))], dt, 3, dm_acc=False)
    assert got[1].sum() == pytest.approx(rho2.sum(), rel=1e-13)


def ambient_case(n=64, L=10.0, seed=9):
    rho = 1.0e6 * (1.0 + 0.05 * O.delta_field(n, seed))
    rng = np.random.default_rng(10)
    v = tuple(5.0 * rng.standard_normal((n, n, n)) for _ in range(3))
    return rho, v, np.array([0.5 * L, 0.52 * L, 0.47 * L]), (12.0, -7.0, 3.0)


@pytest.mark.parametrize("dbl", [True, False])
@pytest.mark.parametrize("M,bhl", [(1.0e8, False), (1.0e10, True)])
def test_bondi_ambient_vs_oracle(dbl, M, bhl):
    """bh_bondi_step_ambient (quantum-fluid-accretion.py:440-510) on the GPU
    against the oracle (itself pinned to the reference's own function)."""
    import qj

    n, L, G, cs, dt = 64, 10.0, 4.30241002e-6, 60.0, 3.7e-5
    rho, v, x_bh, v_bh = ambient_case(n, L)
    ref = O.bondi_sink_ambient(rho, M, x_bh, L / n, L, cs, G, dt, v=v if bhl else None, v_bh=v_bh)
    prec = qj.PLAIN_F64 if dbl else qj.FUSED_F32
    rt = torch.float64 if dbl else torch.float32
    plan = qj.Plan(qj.Grid(n, n, n, L, L, L), qj.Phys(G=G, cs=cs), prec, 1)
    r = torch.as_tensor(rho, dtype=rt, device="cuda").contiguous()
    vt = tuple(torch.as_tensor(c, dtype=rt, device="cuda").contiguous() for c in v)
    out = plan.bondi_ambient(r, M, x_bh, dt, v=vt if bhl else None, v_bh=v_bh)
    tol = 1e-12 if dbl else 1e-6
    assert O.rel_l2(r.cpu().numpy(), ref[0]) < tol
    np.testing.assert_allclose(out, np.array(ref[1:], dtype=float), rtol=1e-11 if dbl else 1e-5)
    plan.close()


@pytest.mark.parametrize("dbl", [True, False])
def test_hydro_cfl_vs_oracle(dbl):
    import qj

    n, L = 32, 10.0
    _, v, _, _ = ambient_case(n, L)
    rt = torch.float64 if dbl else torch.float32
    plan = qj.Plan(qj.Grid(n, n, n, L, L, L), qj.Phys(cs=60.0),
                   qj.PLAIN_F64 if dbl else qj.FUSED_F32, 1)
    vt = [torch.as_tensor(c, dtype=rt, device="cuda").contiguous() for c in v]
    for dt in (3.7e-5, 1.0):
        got = plan.hydro_cfl_dt(*vt, 60.0, 0.15, dt)
        vv = [c.cpu().numpy().astype(np.float64) for c in vt]
        assert got == pytest.approx(O.hydro_cfl_dt(*vv, 60.0, L / n, 0.15, dt), rel=1e-14)
    plan.close()
