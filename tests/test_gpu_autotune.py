"""Launch tuning of the fused passes and the autotuner.

CTAs per SM, reserved slots and the hydro block give bit-identical results.
The radix plan and pencil tile variants (per-pass bit masks) change the
rounding: each variant, alone or mixed per pass, stays within the
single-precision bar of the float64 path, is deterministic, and is
bit-identical under CTA tuning.  The autotuner's choice is cached and reused.
"""

import os

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def stars_state(n=64, n_s=64, seed=3):
    import qj

    psi, pos, vel, g, p = O.stars_ic(n, n_s, seed=seed)
    vel = 0.2 * np.random.default_rng(seed).standard_normal(pos.shape)
    plan = qj.Plan(qj.Grid(n, n, n), qj.Phys(m_per_hbar=1.0, G=p.G, rho_bar=p.rho_bar),
                   qj.FUSED_F32, n_s)

    def fresh():
        return (torch.as_tensor(psi, dtype=torch.complex64, device="cuda").contiguous(),
                torch.as_tensor(pos, dtype=torch.float32, device="cuda").contiguous(),
                torch.as_tensor(vel, dtype=torch.float32, device="cuda").contiguous(),
                torch.tensor([0.0, 0.0, O.default_dt(g, p)], dtype=torch.float64, device="cuda"))
    return plan, fresh, O.default_dt(g, p), p.m_s


def run(plan, fresh, dt, m_s, steps=5):
    s = fresh()
    plan.kdk_step(*s, dt, steps, m_s)
    plan.status()
    return [x.cpu() for x in s]


def test_tuning_is_bit_identical_and_cached(tmp_path):
    plan, fresh, dt, m_s = stars_state()
    ref = run(plan, fresh, dt, m_s)
    cache = str(tmp_path / "tuning.json")
    s = fresh()
    tuned = plan.autotune(s[0], s[1], s[2], m_s, dt, probe_steps=3, cache_file=cache,
                          shapes=False)
    assert len(tuned) == 12 and os.path.exists(cache)
    assert all(0 <= k <= 32 for k in tuned[:8]) and -1 <= tuned[8] <= 64
    assert tuned[10] == tuned[11] == 0
    # the autotuner only read the state
    for x, y in zip(s, fresh()):
        assert torch.equal(x, y)
    for got in (run(plan, fresh, dt, m_s),):
        for x, y in zip(got, ref):
            assert torch.equal(x, y)
    plan.tuning = [1] * 8 + [0, 0, 0, 0]
    for x, y in zip(run(plan, fresh, dt, m_s), ref):
        assert torch.equal(x, y)
    # a second plan with the same key takes the cached choice without timing
    plan2, fresh2, _, _ = stars_state()
    s2 = fresh2()
    assert plan2.autotune(s2[0], s2[1], s2[2], m_s, dt, cache_file=cache, shapes=False) == tuned
    with pytest.raises(Exception):
        plan.tuning = [99] * 12
    with pytest.raises(Exception):
        plan.tuning = [0] * 10 + [0x80, 0]  # bit 7 (the deposit) has no variants
    plan.close()
    plan2.close()


def test_hydro_block_tuning_bit_identical():
    import qj

    n = 32
    g = O.Grid(n, n, n, 1.0, 1.0, 1.0)
    rho_dm = 1.0 + 0.1 * O.delta_field(n, 0)
    rho_g = 0.2 * (1.0 + 0.05 * O.delta_field(n, 1))
    phys = qj.Phys(m_per_hbar=1.0, G=1.0 / (4.0 * np.pi), rho_bar=float(rho_dm.mean()), cs=1.0)
    outs = []
    for block in (0, 64, 128):
        plan = qj.Plan(qj.Grid(n, n, n), phys, qj.FUSED_F32, 1)
        t = plan.tuning
        t[9] = block
        plan.tuning = t
        st = [torch.as_tensor(np.sqrt(rho_dm), dtype=torch.complex64, device="cuda").contiguous(),
              torch.as_tensor(rho_g, dtype=torch.float32, device="cuda").contiguous()]
        st += [torch.zeros((n, n, n), dtype=torch.float32, device="cuda") for _ in range(3)]
        plan.kdk_gas_bh(*st, None, None, None, O.default_dt(g, O.Phys()), 4, 0.0)
        outs.append([x.cpu() for x in st])
        plan.close()
    for o in outs[1:]:
        for x, y in zip(o, outs[0]):
            assert torch.equal(x, y)


def variant_state(shape, n_s=256, seed=5):
    """A seeded state on a grid whose axes are (or are not) of the lengths
    with shape variants, the fused plan, and the plain float64 plan."""
    import qj

    L = tuple(n / shape[2] for n in shape)  # cubic cells
    psi, pos, vel, g, p = O.stars_ic(shape[0], n_s, seed=seed, shape=shape, L=L)
    vel = 0.2 * np.random.default_rng(seed).standard_normal(pos.shape)
    phys = qj.Phys(m_per_hbar=1.0, G=p.G, rho_bar=p.rho_bar)
    grid = qj.Grid(*shape, *L)
    dt = O.default_dt(g, p)

    def fresh(dbl=False):
        ct, rt = (torch.complex128, torch.float64) if dbl else (torch.complex64, torch.float32)
        return (torch.as_tensor(psi, dtype=ct, device="cuda").contiguous(),
                torch.as_tensor(pos, dtype=rt, device="cuda").contiguous(),
                torch.as_tensor(vel, dtype=rt, device="cuda").contiguous(),
                torch.tensor([0.0, 0.0, dt], dtype=torch.float64, device="cuda"))
    return (qj.Plan(grid, phys, qj.FUSED_F32, n_s), qj.Plan(grid, phys, qj.PLAIN_F64, n_s),
            fresh, dt, p.m_s)


def rel(a, b):
    return float(torch.linalg.vector_norm((a.to(b.dtype) - b).flatten()) /
                 torch.linalg.vector_norm(b.flatten()))


ALL = 0x7f7f  # every pass with variants, both orientations
KICK = (1 << 4) | (1 << 12)  # the kick along x or y, and along z
KICK_Z = 1 << 12


@pytest.mark.parametrize("shape", [(128, 128, 128), (256, 128, 64)])
def test_shape_variants_within_bar_and_deterministic(shape):
    """Every (radix, tile) combination on every pass, the kick alone in radix
    plan 1, and a per-orientation mix, against the plain float64 path after 20
    steps (psi, star positions <= 1e-5).  (256, 128, 64) mixes a 256 axis, a 128 axis and an
    axis without variants (64: its passes keep the default shape; the 8-wide
    z tiles also cover its half spectrum)."""
    fused, plain, fresh, dt, m_s = variant_state(shape)
    steps = 20
    ref = fresh(True)
    plain.kdk_step(*ref, dt, steps, m_s)
    base = None
    for radix, tile in [(0, 0), (ALL, 0), (0, ALL), (ALL, ALL), (KICK, 0), (KICK_Z, KICK)]:
        t = fused.tuning
        t[:8] = [0] * 8
        t[10], t[11] = radix, tile
        fused.tuning = t
        runs = []
        for _ in range(2):
            s = fresh()
            fused.kdk_step(*s, dt, steps, m_s)
            fused.status()
            runs.append(s)
        for x, y in zip(runs[0], runs[1]):
            assert torch.equal(x, y), (radix, tile)
        s = runs[0]
        assert rel(s[0], ref[0]) < 1e-5, (radix, tile, rel(s[0], ref[0]))
        assert rel(s[1], ref[1]) < 1e-5, (radix, tile, rel(s[1], ref[1]))
        if base is None:
            base = s
        elif radix == 0 and tile == 0:
            assert all(torch.equal(x, y) for x, y in zip(s, base))
        # CTA tuning inside the variant is bit-identical
        t[:8] = [1] * 8
        fused.tuning = t
        s2 = fresh()
        fused.kdk_step(*s2, dt, steps, m_s)
        fused.status()
        for x, y in zip(s2, s):
            assert torch.equal(x, y), (radix, tile)
    fused.close()
    plain.close()


def test_autotune_picks_shapes_within_bar(tmp_path):
    fused, plain, fresh, dt, m_s = variant_state((128, 128, 128))
    s = fresh()
    tuned = fused.autotune(s[0], s[1], s[2], m_s, dt, probe_steps=3,
                           cache_file=str(tmp_path / "tuning.json"))
    assert len(tuned) == 12 and tuned[10] & ~ALL == 0 and tuned[11] & ~ALL == 0
    for x, y in zip(s, fresh()):  # the autotuner only read the state
        assert torch.equal(x, y)
    got, ref = fresh(), fresh(True)
    fused.kdk_step(*got, dt, 10, m_s)
    fused.status()
    plain.kdk_step(*ref, dt, 10, m_s)
    assert rel(got[0], ref[0]) < 1e-5 and rel(got[1], ref[1]) < 1e-5
    fused.close()
    plain.close()
