"""The adjoint (torch.autograd.Function over qj_kdk_forward_ckpt / qj_kdk_adjoint)
against the torch float64 autograd mirror of the step and against central finite
differences.  Loss L = mean((|psi_T|^2 - rho_target)^2) w.r.t. the initial phase
theta; rho_target comes from a forward run of a second seed.  The stars enter
as a fixed source density rho_s (their CIC density, held fixed).

Bars: plain float64 gradient rel-L2 <= 1e-9 vs the mirror; fused float32
gradient cosine >= 0.9999 vs the mirror; finite differences (16 seeded
directions, eps = 1e-3) cosine >= 0.9999 with the adjoint directional
derivatives.
"""

import numpy as np
import pytest
import torch

from oracle import oracle as O
from oracle import torch_mirror as TM

pytestmark = pytest.mark.gpu

N, NSTEPS, K = 32, 10, 4


def setup(si=False, shape=None, L=(1.0, 1.0, 1.0)):
    psi, _, _, g, p = O.stars_ic(N, 0, seed=0, shape=shape, L=L)
    if si:
        p.b_coeff = -0.1
    sqrt_rho = np.abs(psi)
    theta = 0.5 * O.delta_field(N, 21, shape)
    dt = O.default_dt(g, p)
    k_sq = TM.kgrid(g.shape, (g.Lx, g.Ly, g.Lz))
    # target from a forward run of a second seed
    psi2, *_ = O.stars_ic(N, 0, seed=1, shape=shape, L=L)
    tgt = TM.kdk(torch.as_tensor(psi2), k_sq, p.G, p.rho_bar, p.m_per_hbar, dt, NSTEPS, p.b_coeff)
    rho_tgt = (torch.abs(tgt) ** 2).numpy()
    return g, p, sqrt_rho, theta, dt, k_sq, rho_tgt


def qj_grad(precision, g, p, sqrt_rho, theta, dt, rho_tgt, si=False, rho_s=None, nsteps=NSTEPS,
            K=K):
    import qj
    from qj.autograd import kdk_evolve

    plan = qj.Plan(qj.Grid(g.nx, g.ny, g.nz, g.Lx, g.Ly, g.Lz),
                   qj.Phys(m_per_hbar=p.m_per_hbar, G=p.G, rho_bar=p.rho_bar, b_coeff=p.b_coeff),
                   precision, 1)
    rt = plan.rdtype
    th = torch.as_tensor(theta, dtype=rt, device="cuda").requires_grad_(True)
    s = torch.as_tensor(sqrt_rho, dtype=rt, device="cuda")
    tg = torch.as_tensor(rho_tgt, dtype=rt, device="cuda")
    src = None if rho_s is None else torch.as_tensor(rho_s, dtype=rt, device="cuda")
    psiT = kdk_evolve(th, s, plan, dt, nsteps, K, self_interaction=si, rho_s=src)
    L = torch.mean((torch.abs(psiT) ** 2 - tg) ** 2)
    L.backward()
    plan.status()
    return plan, float(L.detach()), th.grad.double().cpu().numpy()


def cos(a, b):
    return float(np.dot(a.ravel(), b.ravel()) / (np.linalg.norm(a) * np.linalg.norm(b)))


@pytest.mark.parametrize("si", [False, True])
def test_adjoint_vs_torch_f64_mirror(si):
    import qj

    g, p, s, th, dt, k_sq, tgt = setup(si)
    L_ref, g_ref = TM.loss_and_grad(th, s, tgt, k_sq, p.G, p.rho_bar, p.m_per_hbar, dt, NSTEPS,
                                    p.b_coeff)
    plan, L64, g64 = qj_grad(qj.PLAIN_F64, g, p, s, th, dt, tgt, si)
    plan.close()
    assert L64 == pytest.approx(L_ref, rel=1e-10)
    assert O.rel_l2(g64, g_ref) < 1e-9
    plan, L32, g32 = qj_grad(qj.FUSED_F32, g, p, s, th, dt, tgt, si)
    plan.close()
    assert L32 == pytest.approx(L_ref, rel=1e-4)
    assert cos(g32, g_ref) >= 0.9999
    assert O.rel_l2(g32, g_ref) < 1e-2


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_adjoint_vs_finite_differences(prec):
    """Directions d have unit variance per cell, so eps = 1e-3 perturbs each
    phase by about 1e-3 rad."""
    import qj
    from qj.autograd import kdk_evolve

    precision = qj.FUSED_F32 if prec == "f32" else qj.PLAIN_F64
    g, p, s, th, dt, k_sq, tgt = setup()
    plan, L0, grad = qj_grad(precision, g, p, s, th, dt, tgt)
    rt = plan.rdtype
    sd = torch.as_tensor(s, dtype=rt, device="cuda")
    tg = torch.as_tensor(tgt, dtype=torch.float64, device="cuda")

    def loss(theta):
        with torch.no_grad():
            psiT = kdk_evolve(torch.as_tensor(theta, dtype=rt, device="cuda"), sd, plan, dt,
                              NSTEPS, K)
            return float(torch.mean((torch.abs(psiT).double() ** 2 - tg) ** 2))

    rng = np.random.default_rng(77)
    eps = 1e-3
    fd, ad = [], []
    for _ in range(16):
        d = rng.standard_normal(th.shape)
        fd.append((loss(th + eps * d) - loss(th - eps * d)) / (2 * eps))
        ad.append(float(np.sum(grad * d)))
    fd, ad = np.array(fd), np.array(ad)
    plan.close()
    assert cos(fd, ad) >= 0.9999
    assert np.abs(fd - ad).max() <= (1e-2 if prec == "f32" else 1e-4) * np.abs(ad).max()


def test_adjoint_noncubic_f32():
    """A non-cubic box with unequal sides: the single-precision reverse sweep
    runs its drift adjoint as three fused passes of different lengths."""
    import qj

    g, p, s, th, dt, k_sq, tgt = setup(shape=(32, 16, 64), L=(2.0, 1.0, 4.0))
    L_ref, g_ref = TM.loss_and_grad(th, s, tgt, k_sq, p.G, p.rho_bar, p.m_per_hbar, dt, NSTEPS,
                                    p.b_coeff)
    plan, L32, g32 = qj_grad(qj.FUSED_F32, g, p, s, th, dt, tgt)
    plan.close()
    assert L32 == pytest.approx(L_ref, rel=1e-4)
    assert cos(g32, g_ref) >= 0.9999
    assert O.rel_l2(g32, g_ref) < 1e-2


@pytest.mark.parametrize("si", [False, True])
def test_adjoint_with_fixed_star_density(si):
    """The star density as a fixed source in every kick's potential: both
    precisions against the mirror with the same source."""
    import qj

    g, p, s, th, dt, k_sq, _ = setup(si)
    _, pos, _, _, ps = O.stars_ic(N, 64, seed=5)
    rho_s = O.bin_stars(pos, g, np.full(len(pos), ps.m_s))
    psi2, *_ = O.stars_ic(N, 0, seed=1)
    tgt = (torch.abs(TM.kdk(torch.as_tensor(psi2), k_sq, p.G, p.rho_bar, p.m_per_hbar, dt, NSTEPS,
                            p.b_coeff, rho_s=torch.as_tensor(rho_s))) ** 2).numpy()
    L_ref, g_ref = TM.loss_and_grad(th, s, tgt, k_sq, p.G, p.rho_bar, p.m_per_hbar, dt, NSTEPS,
                                    p.b_coeff, rho_s=rho_s)
    plan, L64, g64 = qj_grad(qj.PLAIN_F64, g, p, s, th, dt, tgt, si, rho_s=rho_s)
    plan.close()
    assert L64 == pytest.approx(L_ref, rel=1e-10)
    assert O.rel_l2(g64, g_ref) < 1e-9
    plan, L32, g32 = qj_grad(qj.FUSED_F32, g, p, s, th, dt, tgt, si, rho_s=rho_s)
    plan.close()
    assert L32 == pytest.approx(L_ref, rel=1e-4)
    assert cos(g32, g_ref) >= 0.9999


def test_adjoint_config3_128cube_200_steps():
    """The adjoint configuration at its own size: 128^3, 200 KDK steps, psi
    checkpointed every 20 steps, the IC family with 4096 stars as a fixed
    source density, target |psi_T|^2 of a forward run from a second seed, loss
    mean((|psi_T|^2 - rho_target)^2) w.r.t. the initial phase theta (float32
    128^3).  The single-precision adjoint gradient against the float64 one
    (cosine >= 0.9999); central finite differences of the float64 forward
    along 16 seeded directions (eps = 1e-3) against the directional
    derivatives of both (cosine >= 0.9999)."""
    import qj
    from qj.autograd import kdk_evolve

    n, steps, kc = 128, 200, 20
    psi, pos, _, g, p = O.stars_ic(n, 4096, seed=0)
    rho_s = O.bin_stars(pos, g, np.full(len(pos), p.m_s))
    s = np.abs(psi)
    th = 0.5 * O.delta_field(n, 21)
    dt = O.default_dt(g, p)
    phys = qj.Phys(m_per_hbar=p.m_per_hbar, G=p.G, rho_bar=p.rho_bar)
    plan64 = qj.Plan(qj.Grid(n, n, n), phys, qj.PLAIN_F64, 1)
    src64 = torch.as_tensor(rho_s, dtype=torch.float64, device="cuda")
    psi2, *_ = O.stars_ic(n, 0, seed=1)
    t2 = torch.as_tensor(psi2, dtype=torch.complex128, device="cuda")
    with torch.no_grad():
        tgt = torch.abs(kdk_evolve(torch.angle(t2), torch.abs(t2), plan64, dt, steps, kc,
                                   rho_s=src64)) ** 2
    tgt = tgt.cpu().numpy()
    plan64.close()
    plan, L64, g64 = qj_grad(qj.PLAIN_F64, g, p, s, th, dt, tgt, rho_s=rho_s, nsteps=steps, K=kc)
    plan32, L32, g32 = qj_grad(qj.FUSED_F32, g, p, s, th, dt, tgt, rho_s=rho_s, nsteps=steps,
                               K=kc)
    plan32.close()
    print(f"config 3: L64 {L64:.6e} L32 {L32:.6e} cos(g32, g64) {cos(g32, g64):.7f}")
    assert L32 == pytest.approx(L64, rel=1e-4)
    assert cos(g32, g64) >= 0.9999
    sd = torch.as_tensor(s, dtype=torch.float64, device="cuda")
    tg = torch.as_tensor(tgt, dtype=torch.float64, device="cuda")

    def loss(theta):
        with torch.no_grad():
            psiT = kdk_evolve(torch.as_tensor(theta, dtype=torch.float64, device="cuda"), sd, plan,
                              dt, steps, kc, rho_s=src64)
            return float(torch.mean((torch.abs(psiT) ** 2 - tg) ** 2))

    rng = np.random.default_rng(77)
    eps = 1e-3
    fd, a64, a32 = [], [], []
    for _ in range(16):
        d = rng.standard_normal(th.shape)
        fd.append((loss(th + eps * d) - loss(th - eps * d)) / (2 * eps))
        a64.append(float(np.sum(g64 * d)))
        a32.append(float(np.sum(g32 * d)))
    plan.close()
    fd, a64, a32 = np.array(fd), np.array(a64), np.array(a32)
    print(f"config 3: cos(fd, a64) {cos(fd, a64):.7f} cos(fd, a32) {cos(fd, a32):.7f}")
    assert cos(fd, a64) >= 0.9999
    assert cos(fd, a32) >= 0.9999


def test_adjoint_config3_against_the_step_with_moving_stars():
    """The adjoint holds the stars' density fixed; the whole step also moves
    the stars.  At the adjoint configuration's size (128^3, 200 steps, K = 20,
    the IC family's 4096 stars), its gradient against central differences
    (eps = 1e-3, 8 seeded directions) of the loss of the full float64 step,
    qj_kdk_step with the stars moving: cosine >= 0.9999."""
    import qj

    n, steps, kc = 128, 200, 20
    psi, pos, vel, g, p = O.stars_ic(n, 4096, seed=0)
    rho_s = O.bin_stars(pos, g, np.full(len(pos), p.m_s))
    s = np.abs(psi)
    th = 0.5 * O.delta_field(n, 21)
    dt = O.default_dt(g, p)
    phys = qj.Phys(m_per_hbar=p.m_per_hbar, G=p.G, rho_bar=p.rho_bar)
    step = qj.Plan(qj.Grid(n, n, n), phys, qj.PLAIN_F64, len(pos))
    dev = torch.device("cuda")

    def run(psi0, pos0, vel0):
        ps = torch.as_tensor(psi0, dtype=torch.complex128, device=dev).contiguous()
        po = torch.as_tensor(pos0, dtype=torch.float64, device=dev).contiguous()
        ve = torch.as_tensor(vel0, dtype=torch.float64, device=dev).contiguous()
        dg = torch.tensor([0.0, 0.0, dt], dtype=torch.float64, device=dev)
        step.kdk_step(ps, po, ve, dg, dt, steps, p.m_s)
        return ps, po

    psi2, pos2, vel2, *_ = O.stars_ic(n, 4096, seed=1)
    tgt = (torch.abs(run(psi2, pos2, vel2)[0]) ** 2).cpu().numpy()
    tg = torch.as_tensor(tgt, dtype=torch.float64, device=dev)

    def loss(theta):
        psiT, _ = run(s * np.exp(1j * theta), pos, vel)
        return float(torch.mean((torch.abs(psiT) ** 2 - tg) ** 2))

    _, posT = run(s * np.exp(1j * th), pos, vel)
    moved = float(np.max(np.abs(posT.cpu().numpy() - pos)))
    plan, _, g64 = qj_grad(qj.PLAIN_F64, g, p, s, th, dt, tgt, rho_s=rho_s, nsteps=steps, K=kc)
    plan.close()
    plan, _, g32 = qj_grad(qj.FUSED_F32, g, p, s, th, dt, tgt, rho_s=rho_s, nsteps=steps, K=kc)
    plan.close()
    rng = np.random.default_rng(78)
    eps = 1e-3
    fd, a64, a32 = [], [], []
    for _ in range(8):
        d = rng.standard_normal(th.shape)
        fd.append((loss(th + eps * d) - loss(th - eps * d)) / (2 * eps))
        a64.append(float(np.sum(g64 * d)))
        a32.append(float(np.sum(g32 * d)))
    step.close()
    fd, a64, a32 = np.array(fd), np.array(a64), np.array(a32)
    print(f"moving stars (largest move {moved:.2e}): cos(fd, a64) {cos(fd, a64):.7f} "
          f"cos(fd, a32) {cos(fd, a32):.7f}")
    assert cos(fd, a64) >= 0.9999
    assert cos(fd, a32) >= 0.9999
