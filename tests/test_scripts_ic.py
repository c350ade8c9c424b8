"""Reference set-up constants, initial conditions and state I/O (host side,
no GPU): checked against golden vectors produced by the reference scripts' own
main() code (tests/golden/make_golden.py, gen_ics and gen_stars)."""

import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def golden(name):
    return np.load(os.path.join(HERE, "golden", name))


def check_summary(z, prefix, a, rel=1e-12):
    a = np.asarray(a)
    assert tuple(z[prefix + ".shape"]) == a.shape
    assert np.sum(a) == pytest.approx(complex(z[prefix + ".sum"]), rel=rel, abs=1e-300)
    assert np.sum(np.abs(a) ** 2) == pytest.approx(float(z[prefix + ".sumsq"]), rel=rel)
    w = np.random.default_rng(12345).standard_normal(a.shape)
    assert np.sum(w * a) == pytest.approx(complex(z[prefix + ".proj"]), rel=1e-9)
    s = int(z[prefix + ".stride"])
    sub = a[::s, ::s, ::s]
    assert np.max(np.abs(sub - z[prefix + ".sub"])) <= rel * np.max(np.abs(sub))


def test_stars_setup_matches_reference_constants():
    from qj.scripts import StarsSetup

    z = golden("stars_res1.npz")
    s = StarsSetup.reference(1)
    assert [s.nx, s.ny, s.nz, s.Lx, s.Ly, s.Lz] == list(z["const.grid"])
    assert s.G == pytest.approx(float(z["const.G"]), rel=1e-15)
    assert s.m_per_hbar == pytest.approx(float(z["const.m_per_hbar"]), rel=1e-13)
    assert s.rho_bar == float(z["const.rho_bar"])
    assert s.m_s == pytest.approx(float(z["const.m_s"]), rel=1e-14)
    assert s.nt == int(z["const.nt"]) and s.nt_sub == int(z["const.nt_sub"])
    assert s.dt == pytest.approx(float(z["const.dt"]), rel=1e-14)
    assert StarsSetup.reference(1, self_interaction=True).b_coeff == pytest.approx(
        float(z["si.b_coeff"]), rel=1e-12)


def test_stars_blob_ic():
    from qj.scripts import StarsSetup, stars_blob_ic

    z = golden("ic_res1.npz")
    psi, pos, vel = stars_blob_ic(StarsSetup.reference(1))
    check_summary(z, "stars.psi", psi)
    np.testing.assert_array_equal(pos, z["stars.pos"])
    np.testing.assert_array_equal(vel, z["stars.vel"])


@pytest.mark.parametrize("case,sort", [("fluid", True), ("bh", False)])
def test_random_phase_ic(case, sort):
    from qj.scripts import k_squared, random_phase_psi

    z = golden("ic_res1.npz")
    c = z[case + ".const"]
    n, L, sigma, mph = int(c[0]), float(c[1]), float(c[2]), float(c[3])
    mean_rho = float(c[4] * c[5]) if case == "fluid" else float(c[4])
    psi = random_phase_psi(k_squared((n, n, n), (L, L, L)), sigma, mph, mean_rho, sort)
    check_summary(z, case + ".psi", psi, rel=1e-10)


def test_soliton_ic():
    from qj.scripts import soliton_psi

    z = golden("ic_res1.npz")
    n, L, m22, r_sol = z["soliton.const"]
    n = int(n)
    lin = np.linspace(0.5 * L / n, L - 0.5 * L / n, n)
    X, Y, Z = np.meshgrid(lin, lin, lin, indexing="ij")
    check_summary(z, "soliton.psi", soliton_psi(X, Y, Z, float(L), float(m22), float(r_sol)))


def test_state_roundtrip(tmp_path):
    import torch

    from qj.scripts import load_state, save_state

    st = {"t": 1.25, "psi": torch.randn(4, 4, 4, dtype=torch.complex64),
          "pos": torch.rand(3, 3), "vel": np.zeros((3, 3)), "a_max": 2.0, "dt_s": 0.5}
    p = str(tmp_path / "s.npz")
    save_state(p, st)
    back = load_state(p)
    assert back["t"] == 1.25 and back["a_max"] == 2.0 and back["dt_s"] == 0.5
    np.testing.assert_array_equal(back["psi"], st["psi"].numpy())
    np.testing.assert_array_equal(back["pos"], st["pos"].numpy())
    on_cpu = load_state(p, device="cpu")
    assert on_cpu["psi"].dtype == torch.complex64 and on_cpu["pos"].dtype == torch.float32
