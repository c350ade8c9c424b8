"""The oracle's vectorised deposits and its complex64 / float32 stars step
(the CPU baseline's timed step, in the reference's own precision): both
deposits are bit-identical to the sequential star-by-star loop, the float32
step keeps complex64 / float32 throughout, and it follows the float64
restatement to float32 rounding."""

import numpy as np

from oracle import oracle as O


def test_vectorised_f32_deposit_is_bit_identical():
    psi, pos, vel, g, p = O.stars_ic(32, 64, seed=3)
    pos32 = pos.astype(np.float32)
    # a clump in one cell and stars on cell faces exercise repeated cells
    pos32[:8] = np.float32(0.5)
    pos32[8:12, 0] = np.float32(g.dx * 3)
    a = O.bin_stars_f32(pos32, g, p.m_s)
    b = O.bin_stars_f32_vec(pos32, g, p.m_s)
    assert a.dtype == b.dtype == np.float32
    assert np.array_equal(a, b)


def test_f32_step_follows_the_f64_restatement():
    psi, pos, vel, g, p = O.stars_ic(32, 16, seed=3)
    dt = O.default_dt(g, p)
    k, k32 = O.kgrid(g), O.kgrid_f32(g)
    s64 = (psi, pos, vel, 0.0, 0.0, dt)
    s32 = (psi.astype(np.complex64), pos.astype(np.float32), vel.astype(np.float32), 0.0, 0.0,
           dt)
    for _ in range(3):
        s64 = O.stars_compute_step(*s64, g, p, dt, k)
        s32 = O.stars_compute_step_f32(*s32, g, p, dt, k32)
    assert [x.dtype for x in s32[:3]] == [np.complex64, np.float32, np.float32]
    assert O.rel_l2(s32[0], s64[0]) < 1e-5
    assert O.rel_l2(s32[1], s64[1]) < 1e-5
    assert O.rel_l2(s32[2], s64[2]) < 1e-4
    assert abs(s32[4] - s64[4]) < 1e-5 * s64[4]


def _bin_stars_loop(pos, g, masses):
    """The sequential deposit written as the reference's loop (star by star,
    corners in the fixed order), kept here to pin the vectorised oracle."""
    rho = np.zeros(g.shape)
    i, ip1, w_i, w_ip1 = O.get_cic_indices_and_weights(pos, g)
    vol = g.dx * g.dy * g.dz
    idx, w = (i, ip1), (w_i, w_ip1)
    for s in range(pos.shape[0]):
        fac = masses[s] / vol
        for c in O.CORNERS:
            rho[idx[c[0]][s, 0], idx[c[1]][s, 1], idx[c[2]][s, 2]] += (
                w[c[0]][s, 0] * w[c[1]][s, 1] * w[c[2]][s, 2] * fac)
    return rho


def test_vectorised_f64_deposit_is_bit_identical_to_the_loop():
    psi, pos, vel, g, p = O.stars_ic(16, 300, seed=8)
    pos[:10] = 0.5  # a clump: repeated cells
    pos[10:14, 1] = 1.0  # on the upper face (wraps to cell 0)
    masses = np.random.default_rng(2).uniform(0.5, 2.0, len(pos))
    assert np.array_equal(O.bin_stars(pos, g, masses), _bin_stars_loop(pos, g, masses))
