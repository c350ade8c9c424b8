"""The oracle against golden vectors produced by the reference's own functions.

``tests/golden/make_golden.py`` executed the reference scripts (float64 NumPy
array backend standing in for the absent JAX) on the seeded inputs rebuilt
here; each test recomputes the same quantities with ``oracle.oracle`` and
compares checksums, strided subsamples and particle arrays.
"""

import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")
RTOL = 1e-9


def load(name):
    return dict(np.load(os.path.join(GOLD, name)))


def check(f, prefix, a, rtol=RTOL):
    a = np.asarray(a)
    assert tuple(f[prefix + ".shape"]) == a.shape, prefix
    scale = np.sqrt(float(f[prefix + ".sumsq"])) + 1e-300
    w = np.random.default_rng(12345).standard_normal(a.shape)
    assert abs(np.sum(a) - f[prefix + ".sum"]) <= rtol * scale * np.sqrt(a.size), prefix
    assert abs(np.sum(np.abs(a) ** 2) - f[prefix + ".sumsq"]) <= rtol * float(f[prefix + ".sumsq"]) + 1e-300, prefix
    assert abs(np.sum(w * a) - f[prefix + ".proj"]) <= rtol * scale * np.sqrt(a.size), prefix
    if a.ndim == 3:
        s = int(f[prefix + ".stride"])
        ref = f[prefix + ".sub"]
        np.testing.assert_allclose(a[::s, ::s, ::s], ref, rtol=0, atol=rtol * np.abs(ref).max() + 1e-300)
    else:
        ref = f[prefix + ".full"]
        np.testing.assert_allclose(a, ref, rtol=0, atol=rtol * (np.abs(ref).max() + 1e-300))


def grid_from(f):
    nx, ny, nz, Lx, Ly, Lz = f["const.grid"]
    return O.Grid(int(nx), int(ny), int(nz), float(Lx), float(Ly), float(Lz))


def test_stars_golden():
    f = load("stars_res1.npz")
    g = grid_from(f)
    p = O.Phys(m_per_hbar=float(f["const.m_per_hbar"]), G=float(f["const.G"]),
               rho_bar=float(f["const.rho_bar"]), m_s=float(f["const.m_s"]))
    dt = float(f["const.dt"])
    # timestep constants (quantum-stars.py:151-157), t_end = 10
    _, nt, nt_sub, dt_o = O.timestep_constants(g, p, 10.0)
    assert nt == int(f["const.nt"]) and nt_sub == int(f["const.nt_sub"])
    assert dt_o == pytest.approx(dt, rel=1e-15)
    n_s = int(f["input.n_s"])
    rho_dm = float(f["input.rho_dm0"]) * (1.0 + 0.1 * O.delta_field(0, 0, g.shape))
    psi = np.sqrt(rho_dm).astype(np.complex128)
    pos = np.random.default_rng(1).uniform(0.0, 1.0, (n_s, 3)) * np.array([g.Lx, g.Ly, g.Lz])
    vel = np.random.default_rng(2).uniform(-1.0, 1.0, (n_s, 3))
    k = O.kgrid(g)
    check(f, "k_sq", k[3])
    rho_s = O.bin_stars(pos, g, np.full(n_s, p.m_s))
    check(f, "bin_stars", rho_s)
    rho_tot = np.abs(psi) ** 2 + rho_s
    check(f, "get_potential", O.get_potential(rho_tot, g, p, k))
    acc, a_max = O.get_acceleration(pos, rho_tot, g, p, k)
    check(f, "get_acceleration.acc", acc)
    assert a_max == pytest.approx(float(f["get_acceleration.a_max"]), rel=RTOL)
    out = O.stars_run(psi, pos, vel, 2, g, p, dt)
    for key, val in zip(("psi", "pos", "vel"), out[:3]):
        check(f, "step2." + key, val)
    for key, val in zip(("t", "a_max", "dt_s"), out[3:]):
        assert val == pytest.approx(float(f["step2." + key]), rel=RTOL), key
    # self-interaction: V + b_coeff rho
    p_si = O.Phys(**{**p.__dict__, "b_coeff": float(f["si.b_coeff"])})
    check(f, "si.get_potential", O.get_potential(rho_tot, g, p_si, k, self_interaction=True))


def test_gasbh_golden():
    f = load("gasbh_res1.npz")
    g = grid_from(f)
    n, L = g.nx, g.Lx
    p = O.Phys(m_per_hbar=float(f["const.m_per_hbar"]), G=float(f["const.G"]),
               rho_bar=float(f["const.rho_bar"]), cs=float(f["const.cs"]),
               c_light=float(f["const.c"]))
    dt = float(f["const.dt"])
    rho0 = float(f["input.rho0"])
    psi = np.sqrt(rho0 * (1.0 + 0.1 * O.delta_field(n, 3))).astype(np.complex128)
    rho = 0.1 * rho0 * (1.0 + 0.05 * O.delta_field(n, 4))
    rng = np.random.default_rng(5)
    vx, vy, vz = (0.1 * p.cs * rng.standard_normal(g.shape) for _ in range(3))
    pos = np.array([[0.6 * L, 0.5 * L, 0.5 * L]])
    vel = np.array([[0.0, 40.0, 0.0]])
    assert p.rho_bar == pytest.approx(float(np.mean(np.abs(psi) ** 2)), rel=1e-14)
    h = O.solve_hydro(rho, vx, vy, vz, dt, g.dx, p.cs)
    for name, a in zip(("rho", "vx", "vy", "vz"), h):
        check(f, "solve_hydro." + name, a)
    p2, m2 = O.do_accretion(psi, pos, vel, np.array([1.0e11]), g, p, dt, p.cs)
    check(f, "do_accretion.psi", p2)
    np.testing.assert_allclose(m2, f["do_accretion.m_bh.full"] if "do_accretion.m_bh.full" in f
                               else f["do_accretion.m_bh"], rtol=RTOL)
    m_bh = float(f["input.M_bh"]) * np.ones(1)
    state = (psi, rho, vx, vy, vz, m_bh, pos, vel, 0.0)
    k = O.kgrid(g)
    for _ in range(2):
        state = O.gasbh_compute_step(*state, g, p, dt, k)
    for key, val in zip(("psi", "rho", "vx", "vy", "vz", "m_bh", "pos", "vel"), state[:8]):
        check(f, "step2." + key, val)
    assert state[8] == pytest.approx(float(f["step2.t"]), rel=1e-15)


def test_tidal_golden():
    f = load("tidal_res1.npz")
    g = grid_from(f)
    n = g.nx
    p = O.Phys(m_per_hbar=float(f["const.m_per_hbar"]), G=float(f["const.G"]),
               rho_bar=float(f["const.rho_bar"]))
    dt = float(f["const.dt"])
    X, _, _ = O.cell_centres(g)
    psi = np.sqrt(float(f["input.rho0"]) * (1.0 + 0.1 * O.delta_field(n, 6))).astype(np.complex128)
    psi = psi * np.exp(1.0j * float(f["input.k_soliton"]) * X)
    V_ext = O.external_potential(g, p.G, float(f["const.M_halo"]))
    check(f, "external_potential", V_ext)
    k = O.kgrid(g)
    t = 0.0
    for _ in range(2):
        psi, t = O.tidal_compute_step(psi, t, g, p, dt, V_ext, k)
    check(f, "step2.psi", psi)


def test_cosmo_golden():
    f = load("cosmo_n32.npz")
    g = grid_from(f)
    H0, om, ol = float(f["const.H0"]), float(f["const.omega_matter"]), float(f["const.omega_lambda"])
    da, a0 = float(f["const.da"]), float(f["const.a_start"])
    assert O.cosmo_compute_dt(a0, da, H0, om, ol) == pytest.approx(float(f["compute_dt.a_start"]), rel=1e-12)
    assert O.cosmo_compute_dt(0.5, da, H0, om, ol) == pytest.approx(float(f["compute_dt.a_half"]), rel=1e-12)
    p = O.Phys(m_per_hbar=float(f["const.m_per_hbar"]), G=float(f["const.G"]),
               rho_bar=float(f["const.rho_bar"]))
    psi = np.sqrt(p.rho_bar * (1.0 + 0.1 * O.delta_field(g.nx, 7))).astype(np.complex128)
    a = a0
    for _ in range(2):
        psi, a = O.cosmo_compute_step(psi, a, da, g, p, H0, om, ol)
    check(f, "step2.psi", psi)
    assert a == pytest.approx(float(f["step2.a"]), rel=1e-15)


def test_bondi_golden():
    f = load("bondi_res1.npz")
    g = grid_from(f)
    rho = float(f["input.rho_gas"]) * (1.0 + 0.05 * O.delta_field(g.nx, 8))
    x_bh = np.array([0.5 * g.Lx, 0.52 * g.Lx, 0.47 * g.Lx])
    for tag, M in (("m1e8", 1.0e8), ("m1e10", 1.0e10)):
        r = O.bondi_sink(rho, M, x_bh, g.dx, g.Lx, float(f["const.cs"]), float(f["const.G"]),
                         float(f["const.dt"]))
        check(f, f"bondi.{tag}.rho", r[0])
        np.testing.assert_allclose(np.array(r[1:], dtype=float), f[f"bondi.{tag}.scalars"], rtol=RTOL)


def ambient_inputs(f):
    g = grid_from(f)
    n = g.nx
    rho = float(f["input.rho_gas"]) * (1.0 + 0.05 * O.delta_field(n, 9))
    rng = np.random.default_rng(10)
    v = tuple(5.0 * rng.standard_normal((n, n, n)) for _ in range(3))
    return g, rho, v, np.array([0.5 * g.Lx, 0.52 * g.Lx, 0.47 * g.Lx]), (12.0, -7.0, 3.0)


def test_bondi_ambient_golden():
    f = load("bondi_ambient.npz")
    g, rho, v, x_bh, v_bh = ambient_inputs(f)
    lo, hi = (float(x) for x in f["const.ann"])
    for tag, M, bhl in (("m1e8", 1.0e8, False), ("m1e10_bhl", 1.0e10, True)):
        r = O.bondi_sink_ambient(rho, M, x_bh, g.dx, g.Lx, float(f["const.cs"]),
                                 float(f["const.G"]), float(f["const.dt"]),
                                 r_acc_mult=float(f["const.r_acc_mult"]), ann_lo=lo, ann_hi=hi,
                                 v=v if bhl else None, v_bh=v_bh)
        check(f, f"amb.{tag}.rho", r[0])
        np.testing.assert_allclose(np.array(r[1:], dtype=float), f[f"amb.{tag}.scalars"], rtol=RTOL)


def test_hydro_cfl_golden():
    f = load("bondi_ambient.npz")
    g, rho, v, _, _ = ambient_inputs(f)
    cfl, cs = float(f["const.hydro_cfl"]), float(f["const.cs"])
    assert O.hydro_cfl_dt(*v, cs, g.dx, cfl, float(f["const.dt"])) == pytest.approx(
        float(f["cfl.dt_eff"]), rel=1e-14)
    assert O.hydro_cfl_dt(*v, cs, g.dx, cfl, 1.0) == pytest.approx(float(f["cfl.dt_big"]), rel=1e-14)


def test_bh_golden():
    f = load("bh_res1.npz")
    g = grid_from(f)
    p = O.Phys(m_per_hbar=float(f["const.m_per_hbar"]), G=float(f["const.G"]),
               c_light=float(f["const.c"]))
    n, L = g.nx, g.Lx
    psi = np.sqrt(float(f["const.rho_bar"]) * (1.0 + 0.1 * O.delta_field(n, 9))).astype(np.complex128)
    psi = psi * np.exp(0.3j * O.delta_field(n, 10))
    pos = np.array([[0.5 * L, 0.5 * L, 0.5 * L]])
    vel = np.array([[10.0, -5.0, 3.0]])
    p2, m2 = O.do_accretion(psi, pos, vel, float(f["input.M_bh"]) * np.ones(1), g, p,
                            float(f["const.dt"]), float(f["const.sigma"]))
    check(f, "do_accretion.psi", p2)
    np.testing.assert_allclose(m2, f["do_accretion.m_bh"], rtol=RTOL)


def facc_setup(f):
    prm = f["const.params"]
    n, L, dx = int(f["const.grid"][0]), float(f["const.grid"][1]), float(f["const.grid"][2])
    g = O.Grid(n, n, n, L, L, L)
    p = O.Phys(m_per_hbar=float(f["const.m_per_hbar"]), G=float(f["const.G"]),
               rho_bar=float(f["const.rho_bar"]))
    q = O.FaccParams(cs=prm[0], hydro_cfl=prm[1], bh_init_m=prm[2], bh_inject_t=prm[3],
                     ramp_center=prm[4], ramp_w=prm[5], r_acc_mult=prm[6], lam=prm[7],
                     ann_lo=prm[8], ann_hi=prm[9], k_cut_frac=prm[10], inject_smooth_kpc=prm[11],
                     rho_gas=prm[12], bh_on=bool(prm[13]), bh_grav=bool(prm[14]),
                     bh_move=bool(prm[15]), bh_accretion=bool(prm[16]), ramp_on=bool(prm[17]),
                     inject_smooth_on=bool(prm[18]))
    return g, p, q


def facc_inputs(n, rho_bar, rho_gas, frac_dm=0.9):
    rho_dm = rho_bar * frac_dm * (1.0 + 0.1 * O.delta_field(n, 11))
    psi = np.sqrt(rho_dm) * np.exp(1.0j * 0.3 * O.delta_field(n, 12))
    rho = rho_gas * (1.0 + 0.05 * O.delta_field(n, 13))
    rng = np.random.default_rng(14)
    v = [10.0 * rng.standard_normal((n, n, n)) for _ in range(3)]
    return psi, rho, v


FACC_CASES = {"inject": ("bh_inject_t", 0.0, (0.5, 0.5, 0.5), (0.0, 0.0, 0.0), 0.0),
              "massive": ("ramp_center", 2.0e6, (0.43, 0.55, 0.61), (20.0, -10.0, 5.0), 1.0)}


@pytest.mark.parametrize("tag", ["inject", "massive"])
def test_fluid_accretion_step_golden(tag):
    f = load("facc_steps.npz")
    g, p, q = facc_setup(f)
    dt = float(f["const.dt"])
    psi, rho, v = facc_inputs(g.nx, p.rho_bar, q.rho_gas)
    t_key, M_acc, xf, v_bh, placed = FACC_CASES[tag]
    t = getattr(q, t_key) - (0.5 * dt if tag == "inject" else 0.0)
    x_bh = np.array(xf) * g.Lx
    k = O.kgrid(g)
    vx, vy, vz = v
    for step in (1, 2):
        psi, rho, vx, vy, vz, t, M_out, M_acc, x_bh, v_bh, placed, diag = O.facc_compute_step(
            psi, rho, vx, vy, vz, t, M_acc, x_bh, v_bh, placed, g, p, q, dt, k)
        pre = f"{tag}.s{step}."
        check(f, pre + "psi", psi)
        check(f, pre + "rho", rho)
        check(f, pre + "vx", vx)
        got = np.array([t, M_out, M_acc, *x_bh, *v_bh, placed, *diag])
        np.testing.assert_allclose(got, f[pre + "scalars"], rtol=1e-9, atol=1e-12)
