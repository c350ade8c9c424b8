"""End-to-end quantum-stars run on the libqj step (the reference's --res 1
set-up, blob initial condition, outer loop with .npz checkpoints and the
a-posteriori time-step checks) against the float64 oracle."""

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_run_stars_matches_oracle(tmp_path):
    from qj.scripts import StarsSetup, load_state, run_stars, stars_blob_ic

    s = StarsSetup.reference(1)
    outer = 2
    st = run_stars(s, outer=outer, checkpoint_dir=str(tmp_path))
    psi0, pos0, vel0 = stars_blob_ic(s)
    g = O.Grid(s.nx, s.ny, s.nz, s.Lx, s.Ly, s.Lz)
    p = O.Phys(m_per_hbar=s.m_per_hbar, G=s.G, rho_bar=s.rho_bar, m_s=s.m_s)
    ref = O.stars_run(psi0, pos0, vel0, outer * s.nt_sub, g, p, s.dt)
    assert O.rel_l2(st["psi"].cpu().numpy(), ref[0]) < 1e-5
    assert O.rel_l2(st["pos"].cpu().numpy(), ref[1]) < 1e-5
    assert st["t"] == pytest.approx(ref[3], rel=1e-12)
    last = load_state(str(tmp_path / f"state_{outer - 1:03d}.npz"))
    np.testing.assert_array_equal(last["psi"], st["psi"].cpu().numpy())
