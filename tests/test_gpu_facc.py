"""The quantum-fluid-accretion step (moving, softened, accreting black hole
seeded at the dark-matter peak; that script's hydro; per-step CFL dt) on the
GPU float64 path, against the reference's own compute_step outputs
(tests/golden/facc_steps.npz, two steps from two seeded states at 128^3)."""

import os

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def golden():
    return np.load(os.path.join(HERE, "golden", "facc_steps.npz"))


def check(f, prefix, a, rtol=1e-9):
    a = np.asarray(a)
    assert np.sum(a) == pytest.approx(complex(f[prefix + ".sum"]), rel=rtol, abs=1e-300)
    assert np.sum(np.abs(a) ** 2) == pytest.approx(float(f[prefix + ".sumsq"]), rel=rtol)
    s = int(f[prefix + ".stride"])
    sub = a[::s, ::s, ::s]
    assert np.max(np.abs(sub - f[prefix + ".sub"])) <= rtol * np.max(np.abs(sub))


@pytest.mark.parametrize("tag", ["inject", "massive"])
def test_fluid_accretion_step_vs_reference(tag):
    import qj

    f = golden()
    prm = f["const.params"]
    n, L = int(f["const.grid"][0]), float(f["const.grid"][1])
    dt = float(f["const.dt"])
    names = ["cs", "hydro_cfl", "bh_init_m", "bh_inject_t", "ramp_center", "ramp_w",
             "r_acc_mult", "lam", "ann_lo", "ann_hi", "k_cut_frac", "inject_smooth_kpc", "rho_gas",
             "bh_on", "bh_grav", "bh_move", "bh_accretion", "ramp_on", "inject_smooth_on"]
    params = {k: (int(v) if k.startswith(("bh_on", "bh_grav", "bh_move", "bh_acc", "ramp_on",
                                          "inject_smooth_on")) else float(v))
              for k, v in zip(names, prm)}
    params["fmax"] = 0.0  # None in the reference: no cap beyond the sink's mass
    rho_bar = float(f["const.rho_bar"])
    rho_dm = rho_bar * 0.9 * (1.0 + 0.1 * O.delta_field(n, 11))
    psi0 = np.sqrt(rho_dm) * np.exp(1.0j * 0.3 * O.delta_field(n, 12))
    rho0 = params["rho_gas"] * (1.0 + 0.05 * O.delta_field(n, 13))
    rng = np.random.default_rng(14)
    v0 = [10.0 * rng.standard_normal((n, n, n)) for _ in range(3)]
    if tag == "inject":
        state = dict(t=params["bh_inject_t"] - 0.5 * dt, M_acc=0.0, x_bh=[0.5 * L] * 3,
                     v_bh=[0.0, 0.0, 0.0], placed=0.0)
    else:
        state = dict(t=params["ramp_center"], M_acc=2.0e6, x_bh=[0.43 * L, 0.55 * L, 0.61 * L],
                     v_bh=[20.0, -10.0, 5.0], placed=1.0)
    plan = qj.Plan(qj.Grid(n, n, n, L, L, L),
                   qj.Phys(m_per_hbar=float(f["const.m_per_hbar"]), G=float(f["const.G"]),
                           rho_bar=rho_bar, cs=params["cs"]), qj.PLAIN_F64, 1)
    T = [torch.as_tensor(a, dtype=torch.complex128 if np.iscomplexobj(a) else torch.float64,
                         device="cuda").contiguous() for a in (psi0, rho0, *v0)]
    for step in (1, 2):
        d = plan.fluid_accretion_step(*T, state, params, dt, 1)
        pre = f"{tag}.s{step}."
        check(f, pre + "psi", T[0].cpu().numpy())
        check(f, pre + "rho", T[1].cpu().numpy())
        check(f, pre + "vx", T[2].cpu().numpy())
        got = np.array([state["t"], d["M_bh_eff_out"], state["M_acc"], *state["x_bh"],
                        *state["v_bh"], state["placed"], d["dMdt"], d["rho_inf"], d["r_B"],
                        d["dMdt_real"], d["cap_ratio"], d["r_acc_eff"]])
        np.testing.assert_allclose(got, f[pre + "scalars"], rtol=1e-9, atol=1e-12)
    plan.close()
