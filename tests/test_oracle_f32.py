"""The oracle's complex64 / float32 stars step (the CPU baseline's timed step,
in the reference's own precision): its vectorised deposit is bit-identical to
the sequential float32 deposit, it keeps complex64 / float32 throughout, and
it follows the float64 restatement to float32 rounding."""

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
