"""GPU parity: libqj (through the C ABI) against the float64 oracle.

Tolerances: plain float64 path rel-L2 <= 1e-11 (FFT round-off); fused float32
path rel-L2(psi) <= 1e-5 against the float64 oracle (the stated target for the
single-precision step); CIC deposits bit-exact.
"""

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def qj_mod():
    import qj

    return qj


def make_plan(g, p, precision, max_particles=4096):
    qj = qj_mod()
    return qj.Plan(qj.Grid(g.nx, g.ny, g.nz, g.Lx, g.Ly, g.Lz),
                   qj.Phys(m_per_hbar=p.m_per_hbar, G=p.G, rho_bar=p.rho_bar,
                           b_coeff=p.b_coeff, cs=p.cs, c_light=p.c_light),
                   precision, max_particles)


def cuda(a, dtype):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


SHAPES = [(16, 16, 16), (32, 64, 16), (64, 64, 64), (128, 64, 16), (256, 32, 32), (32, 16, 512)]


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("dbl", [False, True])
def test_fft3d(shape, dbl):
    qj = qj_mod()
    g = O.Grid(*shape, 1.0, 1.0, 1.0)
    plan = make_plan(g, O.Phys(), qj.PLAIN_F64 if dbl else qj.FUSED_F32, 1)
    rng = np.random.default_rng(0)
    x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    ct = torch.complex128 if dbl else torch.complex64
    xt = cuda(x, ct)
    y = plan.fftn(xt).cpu().numpy()
    ref = np.fft.fftn(x)
    tol = 1e-13 if dbl else 2e-6
    assert O.rel_l2(y, ref) < tol
    z = plan.fftn(cuda(ref, ct), inverse=True).cpu().numpy()
    assert O.rel_l2(z, x) < tol


@pytest.mark.parametrize("dbl", [False, True])
def test_get_potential(dbl):
    qj = qj_mod()
    psi, pos, vel, g, p = O.stars_ic(32, 64, seed=3, shape=(32, 64, 16), L=(2.0, 4.0, 1.0))
    p.b_coeff = -0.05
    plan = make_plan(g, p, qj.PLAIN_F64 if dbl else qj.FUSED_F32)
    rho = np.abs(psi) ** 2 + O.bin_stars(pos, g, np.full(len(pos), p.m_s))
    rt = torch.float64 if dbl else torch.float32
    for si in (False, True):
        V = plan.get_potential(cuda(rho, rt), self_interaction=si).cpu().numpy()
        ref = O.get_potential(rho, g, p, self_interaction=si)
        assert O.rel_l2(V, ref) < (1e-12 if dbl else 1e-5)


def test_bin_stars_bit_exact_f32():
    qj = qj_mod()
    psi, pos, vel, g, p = O.stars_ic(32, 300, seed=5)
    # clump: 40 stars in one cell, some exactly on faces and at the box edge
    pos[:40] = 0.5 + 1e-3 * np.random.default_rng(1).random((40, 3))
    pos[40] = [0.0, 0.5, 1.0]
    pos[41] = [g.dx, 2 * g.dy, 0.5 * g.dz]
    pos32 = pos.astype(np.float32)
    plan = make_plan(g, p, qj.FUSED_F32)
    got = plan.bin_stars(cuda(pos32, torch.float32), m_s=p.m_s).cpu().numpy()
    ref = O.bin_stars_f32(pos32, g, p.m_s)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    # deterministic across repeats
    again = plan.bin_stars(cuda(pos32, torch.float32), m_s=p.m_s).cpu().numpy()
    assert np.array_equal(got.view(np.uint32), again.view(np.uint32))


def test_bin_stars_f64_and_masses():
    qj = qj_mod()
    psi, pos, vel, g, p = O.stars_ic(16, 50, seed=7, shape=(16, 32, 16), L=(1.0, 2.0, 1.0))
    plan = make_plan(g, p, qj.PLAIN_F64)
    got = plan.bin_stars(cuda(pos, torch.float64), m_s=p.m_s).cpu().numpy()
    ref = O.bin_stars(pos, g, np.full(len(pos), p.m_s))
    np.testing.assert_allclose(got, ref, rtol=1e-14, atol=0)
    masses = np.random.default_rng(2).random(len(pos))
    got = plan.bin_stars(cuda(pos, torch.float64), masses=cuda(masses, torch.float64)).cpu().numpy()
    np.testing.assert_allclose(got, O.bin_stars(pos, g, masses), rtol=1e-13, atol=1e-300)


@pytest.mark.parametrize("dbl", [False, True])
def test_get_acceleration(dbl):
    qj = qj_mod()
    psi, pos, vel, g, p = O.stars_ic(32, 128, seed=11)
    plan = make_plan(g, p, qj.PLAIN_F64 if dbl else qj.FUSED_F32)
    rho = np.abs(psi) ** 2 + O.bin_stars(pos, g, np.full(len(pos), p.m_s))
    rt = torch.float64 if dbl else torch.float32
    acc, amax = plan.get_acceleration(cuda(pos, rt), cuda(rho, rt))
    ref, ref_max = O.get_acceleration(pos, rho, g, p)
    tol = 1e-12 if dbl else 1e-5
    assert O.rel_l2(acc.cpu().numpy(), ref) < tol
    assert abs(float(amax) - ref_max) <= tol * ref_max


def run_qj(g, p, psi, pos, vel, dt, nsteps, precision, chunks=1, si=False, v_ext=None):
    qj = qj_mod()
    plan = make_plan(g, p, precision, max(1, len(pos)))
    ct = torch.complex128 if precision == qj.PLAIN_F64 else torch.complex64
    rt = torch.float64 if precision == qj.PLAIN_F64 else torch.float32
    ps = cuda(psi, ct)
    po = cuda(pos, rt) if len(pos) else None
    ve = cuda(vel, rt) if len(pos) else None
    diag = torch.tensor([0.0, 0.0, dt], dtype=torch.float64, device="cuda")
    vx = cuda(v_ext, rt) if v_ext is not None else None
    for c in range(chunks):
        plan.kdk_step(ps, po, ve, diag, dt, nsteps // chunks, p.m_s, si, vx)
    plan.status()  # no fused pass gave up a bounded tile wait
    out = (ps.cpu().numpy(), po.cpu().numpy() if po is not None else pos,
           ve.cpu().numpy() if ve is not None else vel, diag.cpu().numpy())
    plan.close()
    return out


def oracle_run(g, p, psi, pos, vel, dt, nsteps, si=False, v_ext=None):
    k = O.kgrid(g)
    t, a_max, dt_s = 0.0, 0.0, dt
    for _ in range(nsteps):
        if v_ext is not None:
            psi, t = O.tidal_compute_step(psi, t, g, p, dt, v_ext, k)
            continue
        psi, pos, vel, t, a_max, dt_s = O.stars_compute_step(
            psi, pos, vel, t, a_max, dt_s, g, p, dt, k, self_interaction=si)
    return psi, pos, vel, (t, a_max, dt_s)


CASES = [
    ("cube32", 32, (32, 32, 32), (1.0, 1.0, 1.0), 64),
    ("noncubic", 0, (64, 32, 16), (2.0, 1.0, 0.5), 100),
]


@pytest.mark.parametrize("name,n,shape,L,n_s", CASES)
def test_kdk_plain_f64(name, n, shape, L, n_s):
    qj = qj_mod()
    psi, pos, vel, g, p = O.stars_ic(n, n_s, seed=1, shape=shape, L=L)
    vel = 0.3 * np.random.default_rng(9).standard_normal(pos.shape)
    dt = O.default_dt(g, p)
    nsteps = 4
    got = run_qj(g, p, psi, pos, vel, dt, nsteps, qj.PLAIN_F64)
    ref = oracle_run(g, p, psi, pos, vel, dt, nsteps)
    assert O.rel_l2(got[0], ref[0]) < 1e-11
    assert O.rel_l2(got[1], ref[1]) < 1e-12
    assert O.rel_l2(got[2], ref[2]) < 1e-10
    assert got[3][0] == pytest.approx(ref[3][0], rel=1e-13)
    assert got[3][1] == pytest.approx(ref[3][1], rel=1e-10)
    assert got[3][2] == pytest.approx(ref[3][2], rel=1e-10)


@pytest.mark.parametrize("name,n,shape,L,n_s", CASES)
def test_kdk_fused_f32(name, n, shape, L, n_s):
    qj = qj_mod()
    psi, pos, vel, g, p = O.stars_ic(n, n_s, seed=2, shape=shape, L=L)
    vel = 0.3 * np.random.default_rng(9).standard_normal(pos.shape)
    dt = O.default_dt(g, p)
    nsteps = 10
    got = run_qj(g, p, psi, pos, vel, dt, nsteps, qj.FUSED_F32)
    ref = oracle_run(g, p, psi, pos, vel, dt, nsteps)
    assert O.rel_l2(got[0], ref[0]) < 1e-5
    assert O.rel_l2(np.abs(got[0]) ** 2, np.abs(ref[0]) ** 2) < 1e-5
    assert O.rel_l2(got[1], ref[1]) < 1e-5
    assert O.rel_l2(got[2], ref[2]) < 1e-3
    assert got[3][1] == pytest.approx(ref[3][1], rel=1e-4)
    assert got[3][2] == pytest.approx(ref[3][2], rel=1e-4)


def test_fused_f32_64cube_400_stars_100_steps():
    """The small stars configuration at its own size: 64^3, 400 stars at rest,
    seed 0, 100 steps of dt = dx^2/6; fused float32 against the float64 oracle."""
    qj = qj_mod()
    psi, pos, vel, g, p = O.stars_ic(64, 400, seed=0)
    dt = O.default_dt(g, p)
    got = run_qj(g, p, psi, pos, vel, dt, 100, qj.FUSED_F32)
    ref = oracle_run(g, p, psi, pos, vel, dt, 100)
    assert O.rel_l2(got[0], ref[0]) < 1e-5
    assert O.rel_l2(np.abs(got[0]) ** 2, np.abs(ref[0]) ** 2) < 1e-5
    assert O.rel_l2(got[1], ref[1]) < 1e-5
    assert O.rel_l2(got[2], ref[2]) < 1e-3
    m0 = np.sum(np.abs(psi) ** 2)
    assert abs(np.sum(np.abs(got[0].astype(np.complex128)) ** 2) / m0 - 1.0) < 1e-6
    assert got[3][1] == pytest.approx(ref[3][1], rel=1e-4)


def test_fused_deterministic_and_chunking():
    qj = qj_mod()
    psi, pos, vel, g, p = O.stars_ic(32, 200, seed=4)
    vel = 0.3 * np.random.default_rng(1).standard_normal(pos.shape)
    dt = O.default_dt(g, p)
    a = run_qj(g, p, psi, pos, vel, dt, 6, qj.FUSED_F32)
    b = run_qj(g, p, psi, pos, vel, dt, 6, qj.FUSED_F32)
    for x, y in zip(a, b):
        assert np.array_equal(np.asarray(x), np.asarray(y))
    c = run_qj(g, p, psi, pos, vel, dt, 6, qj.FUSED_F32, chunks=3)
    assert O.rel_l2(c[0], a[0]) < 1e-6
    assert O.rel_l2(c[1], a[1]) < 1e-6


def test_fused_no_stars_self_interaction_vext():
    qj = qj_mod()
    psi, pos, vel, g, p = O.stars_ic(32, 0, seed=6)
    p.b_coeff = -0.2
    dt = O.default_dt(g, p)
    got = run_qj(g, p, psi, pos, vel, dt, 5, qj.FUSED_F32, si=True)
    ref = oracle_run(g, p, psi, pos, vel, dt, 5, si=True)
    assert O.rel_l2(got[0], ref[0]) < 1e-5
    assert np.isinf(got[3][2])
    V_ext = O.external_potential(g, p.G, 0.5)
    got = run_qj(g, p, psi, pos, vel, dt, 5, qj.FUSED_F32, v_ext=V_ext)
    ref = oracle_run(g, p, psi, pos, vel, dt, 5, v_ext=V_ext)
    assert O.rel_l2(got[0], ref[0]) < 1e-5
    got = run_qj(g, p, psi, pos, vel, dt, 5, qj.PLAIN_F64, v_ext=V_ext)
    assert O.rel_l2(got[0], ref[0]) < 1e-11


def test_bad_arguments_raise():
    qj = qj_mod()
    with pytest.raises(qj.QjError):
        qj.Plan(qj.Grid(48, 32, 32), qj.Phys())
    with pytest.raises(qj.QjError):
        qj.Plan(qj.Grid(32, 32, 8), qj.Phys())
    plan = qj.Plan(qj.Grid(16, 16, 16), qj.Phys(), qj.FUSED_F32, 4)
    pos = torch.zeros((5, 3), dtype=torch.float32, device="cuda")
    with pytest.raises(qj.QjError):
        plan.bin_stars(pos, m_s=1.0)


@pytest.mark.parametrize("dbl", [False, True])
def test_cosmo_step(dbl):
    """quantum-cosmo.py:169-196 with the script's constants (h = 1, m22 = 2.5,
    omega_m = 0.27, omega_l = 0.73) on a 32^3 box of the script's size."""
    qj = qj_mod()
    G = 4.30241002e-6
    H0 = 0.1
    om, ol = 0.27, 0.73
    rho_crit = 3.0 * H0**2 / (8.0 * np.pi * G)
    m_per_hbar = 2.5e-22 * 8.96215334e-67 / 1.71818134e-87
    g = O.Grid(32, 32, 32, 1000.0, 1000.0, 1000.0)
    p = O.Phys(m_per_hbar=m_per_hbar, G=G, rho_bar=om * rho_crit)
    psi = np.sqrt(p.rho_bar * (1.0 + 0.1 * O.delta_field(32, 7))).astype(np.complex128)
    a0, da = 1.0 / 128.0, 1.0e-4
    ref, a = psi, a0
    for _ in range(6):
        ref, a = O.cosmo_compute_step(ref, a, da, g, p, H0, om, ol)
    plan = make_plan(g, p, qj.PLAIN_F64 if dbl else qj.FUSED_F32, 1)
    ps = cuda(psi, torch.complex128 if dbl else torch.complex64)
    a1 = plan.kdk_cosmo(ps, a0, da, H0, om, ol, 4)
    a2 = plan.kdk_cosmo(ps, a1, da, H0, om, ol, 2)
    torch.cuda.synchronize()
    assert a2 == pytest.approx(a, rel=1e-14)
    assert O.rel_l2(ps.cpu().numpy(), ref) < (1e-11 if dbl else 1e-5)


def test_fused_large_kick_phase():
    """Kick phases of O(20) rad exercise the float64 quadrant reduction of
    the kick's sin / cos (every quadrant is visited)."""
    qj = qj_mod()
    psi, pos, vel, g, p = O.stars_ic(32, 0, seed=8)
    dt = O.default_dt(g, p)
    V0 = O.get_potential(np.abs(psi) ** 2, g, p)
    theta = p.m_per_hbar * dt / 2.0 * np.abs(V0).max()
    p.G *= 20.0 / theta
    got = run_qj(g, p, psi, pos, vel, dt, 2, qj.FUSED_F32)
    ref = oracle_run(g, p, psi, pos, vel, dt, 2)
    assert O.rel_l2(got[0], ref[0]) < 1e-4
    got = run_qj(g, p, psi, pos, vel, dt, 2, qj.PLAIN_F64)
    assert O.rel_l2(got[0], ref[0]) < 1e-10
