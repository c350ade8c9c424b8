#!/usr/bin/env python
"""Benchmark: kick-drift-kick cell-steps/s of the quantum-jax stars step.

Workload (one B200): periodic box L=1, 256^3 complex64 psi = sqrt(1 + 0.1 delta)
(delta: seeded Gaussian field, P(k) ~ k^-3 cut at k_Nyq/2, unit variance),
4096 equal-mass stars (10 % of the dark-matter mass) uniform at rest,
hbar/m = 1, 4 pi G = 1, dt = dx^2/6.  Synthetic seeded data (no dataset).

A step is one KDK step (quantum-stars.py:295-330); K steps run as one
qj_kdk_step call (the fori_loop of quantum-stars.py:454).  psi is 128 MiB,
larger than L2 (126 MB), so no explicit flush is needed between steps.

Printed (one JSON line on rank 0): value = fused float32 cell-steps/s over all
ranks (device time, CUDA events, max over ranks); the plain float64 GPU path's
rate; psi / rho rel-L2 of the fused path against the float64 path after
1000 steps (--err-steps, outside the timed region); e2e through the public API with host buffers; the roofline of the
dominant pass; the CPU baseline (the float64 NumPy oracle on the host cores);
SM clocks sampled during the timed region.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl qj|reference]
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "quantum-jax_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "KDK cell-steps/s at 256^3 (fused FP32; plain FP64 and psi rel-L2 reported)"
UNIT = "cell-steps/s"
# Algorithmic HBM bytes per cell of each fused pass (complex64 fields: each
# input read once, each output written once).
PASS_NAMES = ["density", "fft_y", "poisson", "ifft2_y", "kick_drift", "drift_y",
              "drift_density", "deposit_sort", "particles"]
# Only half of the real density's spectrum R is kept: the density passes write
# half of R (density 8 + 4, drift + density 16 + 4), forward y reads and writes
# half of R (8), Poisson reads half of R and writes half of A~ and B~ (4 + 8),
# inverse y reads those halves and writes S1 and S2 whole (8 + 16).
PASS_BYTES = {0: 12, 1: 8, 2: 12, 3: 24, 4: 32, 5: 16, 6: 20}
STEP_BYTES = 112  # per cell per steady-state step: passes 1..6 once each


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="qj", choices=["qj", "reference"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--stars", type=int, default=4096)
    ap.add_argument("--err-steps", type=int, default=1000,
                    help="steps of the fused-vs-float64 error check, run outside the timed "
                         "region (1000: the accuracy target's run length)")
    ap.add_argument("--ref-budget-s", type=float, default=150.0,
                    help="reference arm: most seconds of timed CPU steps (fewer steps are "
                         "timed, and reported as such, when --steps would take longer)")
    ap.add_argument("--plain-steps", type=int, default=10)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-gas", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--tune-dir", default=os.path.join(os.environ.get("TMPDIR", "/tmp"), "qj_tune"),
                    help="where the autotuner's JSON cache lives")
    ap.add_argument("--gas-n", type=int, default=128)
    ap.add_argument("--gas-steps", type=int, default=500)
    ap.add_argument("--ens-steps", type=int, default=100)
    ap.add_argument("--ens-chunk", type=int, default=10)
    ap.add_argument("--adj-n", type=int, default=128)
    ap.add_argument("--adj-steps", type=int, default=200)
    ap.add_argument("--adj-ckpt", type=int, default=20)
    ap.add_argument("--e2e-sub", type=int, default=10,
                    help="steps per public-API call in the e2e leg (the reference's nt_sub)")
    ap.add_argument("--e2e-calls", type=int, default=16,
                    help="public-API calls timed in the e2e leg")
    return ap.parse_args()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic():
    """dram bytes per launch of each pass from the committed ncu summary."""
    out = {}
    path = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch["):
                    k, v = line.split("=", 1)
                    out[k[len("traffic_bytes_per_launch["):-1]] = float(v)
    except OSError:
        pass
    return out


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_ic(n, n_s):
    from oracle import oracle as O

    psi, pos, vel, g, p = O.stars_ic(n, n_s, seed=0)
    return psi, pos, vel, g, p, O.default_dt(g, p)


def gas_bh_leg(a, dev, stream, barrier):
    """Gas + black-hole step at gas_n^3: psi = sqrt(1 + 0.1 delta), isothermal gas
    rho = 0.2 (1 + 0.05 delta'), v = 0, c_s = 1; one black hole at the box centre
    with 1 % of the box mass, Bondi sink radius 2 cells; dt = min(dx^2/6,
    0.3 dx / (c_s + |v|max)).  The speed of light keeps the reference's c / c_s
    (299792.458 / 20).  Fused float32 against the plain float64 path after the
    same steps; the total mass counts psi, gas and the black hole."""
    import numpy as np
    import torch

    import qj
    from oracle import oracle as O

    n, steps = a.gas_n, a.gas_steps
    dx = 1.0 / n
    rho_dm = 1.0 + 0.1 * O.delta_field(n, 0)
    rho_g = 0.2 * (1.0 + 0.05 * O.delta_field(n, 1))
    vol = dx ** 3
    m_bh0 = 0.01 * (rho_dm.sum() + rho_g.sum()) * vol
    dt = min(dx * dx / 6.0, 0.3 * dx / (1.0 + 0.0))
    phys = qj.Phys(m_per_hbar=1.0, G=1.0 / (4.0 * np.pi), rho_bar=float(rho_dm.mean()), cs=1.0,
                   c_light=299792.458 / 20.0)
    out, ms = {}, {}
    for prec, name in ((qj.FUSED_F32, "fused"), (qj.PLAIN_F64, "plain")):
        ct = torch.complex64 if prec == qj.FUSED_F32 else torch.complex128
        rt = torch.float32 if prec == qj.FUSED_F32 else torch.float64
        plan = qj.Plan(qj.Grid(n, n, n), phys, prec, 1)

        def state():
            return [torch.as_tensor(np.sqrt(rho_dm), dtype=ct, device=dev).contiguous(),
                    torch.as_tensor(rho_g, dtype=rt, device=dev).contiguous(),
                    torch.zeros((n, n, n), dtype=rt, device=dev),
                    torch.zeros((n, n, n), dtype=rt, device=dev),
                    torch.zeros((n, n, n), dtype=rt, device=dev),
                    torch.tensor([m_bh0], dtype=rt, device=dev),
                    torch.tensor([[0.5, 0.5, 0.5]], dtype=rt, device=dev),
                    torch.zeros((1, 3), dtype=rt, device=dev)]

        w = state()
        plan.kdk_gas_bh(*w, dt, 3, 0.0, bondi_r_acc_mult=2.0)  # warm-up
        st = state()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        e0.record(stream)
        plan.kdk_gas_bh(*st, dt, steps, 0.0, bondi_r_acc_mult=2.0)
        e1.record(stream)
        barrier()
        ms[name] = e0.elapsed_time(e1)
        plan.status()
        out[name] = [x.to(torch.complex128 if x.is_complex() else torch.float64) for x in st]
        plan.close()
        del w, st

    def rel(x, y):
        return float(torch.linalg.vector_norm(x - y) / torch.linalg.vector_norm(y))

    f, p = out["fused"], out["plain"]
    mass0 = (rho_dm.sum() + rho_g.sum()) * vol + m_bh0

    def mass(s):
        return float(((s[0].abs() ** 2).sum() + s[1].sum()) * vol + s[5].sum())

    cells = n ** 3
    return {"workload": f"gas + black hole {n}^3 (psi complex64, gas rho + 3 velocities "
                        f"float32), Bondi sink radius 2 cells", "steps": steps, "dt": dt,
            "fused_cell_steps_per_s": cells * steps / (ms["fused"] * 1e-3),
            "plain_f64_cell_steps_per_s": cells * steps / (ms["plain"] * 1e-3),
            "fused_over_plain": ms["plain"] / ms["fused"],
            "psi_rel_l2_vs_f64": rel(f[0], p[0]),
            "rho_dm_rel_l2_vs_f64": rel(f[0].abs() ** 2, p[0].abs() ** 2),
            "gas_rho_rel_l2_vs_f64": rel(f[1], p[1]),
            "gas_v_rel_l2_vs_f64": rel(torch.stack(f[2:5]), torch.stack(p[2:5])),
            "m_bh_rel_vs_f64": float(abs(f[5] - p[5]).max() / abs(p[5]).max()),
            "mass_drift_fused": mass(f) / mass0 - 1.0,
            "mass_drift_f64": mass(p) / mass0 - 1.0,
            "l2_resident": "yes (fields of 8-16 MiB): not HBM-bound"}


def cpu_baseline(n, n_s, steps=2):
    """The oracle's stars step on the host cores (scipy.fft workers = all).

    The baseline value is the complex64 / float32 restatement, the
    reference's own precision (x64 off); the float64 restatement is timed on
    the same sample and reported beside it."""
    import numpy as np

    from oracle import oracle as O

    O.WORKERS = os.cpu_count() or 1
    psi, pos, vel, g, p, dt = make_ic(n, n_s)

    def timed(step, state, k):
        state = step(*state, g, p, dt, k)  # warm-up
        t0 = time.perf_counter()
        for _ in range(steps):
            state = step(*state, g, p, dt, k)
        el = time.perf_counter() - t0
        assert np.isfinite(state[0]).all()
        return el / steps

    s32 = timed(O.stars_compute_step_f32, (psi.astype(np.complex64), pos.astype(np.float32),
                                           vel.astype(np.float32), 0.0, 0.0, dt), O.kgrid_f32(g))
    s64 = timed(O.stars_compute_step, (psi, pos, vel, 0.0, 0.0, dt), O.kgrid(g))
    return {"value": g.ncell / s32, "unit": UNIT, "cores": O.WORKERS, "kind": "port",
            "sample": f"{steps} timed steps (after 1 warm-up) of the {n}^3, {n_s}-star "
                      f"workload; complex64/float32 NumPy/SciPy restatement of "
                      f"quantum-stars.py:295-330, the reference's own precision (x64 off); "
                      f"reference JAX is not installable",
            "s_per_step": s32,
            "float64": {"value": g.ncell / s64, "s_per_step": s64,
                        "sample": "the float64 restatement (the oracle), same steps"}}


def bench_config(n, n_s, dt, world):
    """The `config` of both arms' JSON lines (the same workload)."""
    return {"workload": f"stars KDK {n}^3 complex64, {n_s} stars, one box per GPU (replicas)",
            "grid": [n, n, n], "n_stars": n_s, "dt": dt,
            "l2_flush": (f"inputs larger than L2 (psi {n ** 3 * 8 >> 20} MiB)" if n ** 3 * 8 > 126e6
                         else f"none: psi ({n ** 3 * 8 >> 20} MiB) fits in L2"),
            "parallelism": f"replicas x{world}"}


def run_reference(a, rank, world):
    """The reference arm: the complex64 / float32 restatement of the stars step
    (quantum-stars.py:295-330) on the host cores, rank 0 only.  It runs
    --warmup untimed steps, then times --steps steps of the same 256^3
    workload; when --steps would take longer than --ref-budget-s (estimated
    from the warm-up), it times as many as fit and reports that number in
    `steps` (with `steps_requested`)."""
    if rank != 0:
        return
    import numpy as np

    from oracle import oracle as O

    O.WORKERS = os.cpu_count() or 1
    psi, pos, vel, g, p, dt = make_ic(a.n, a.stars)
    k = O.kgrid_f32(g)
    state = (psi.astype(np.complex64), pos.astype(np.float32), vel.astype(np.float32), 0.0, 0.0, dt)
    t0 = time.perf_counter()
    state = O.stars_compute_step_f32(*state, g, p, dt, k)
    t_step = time.perf_counter() - t0
    warm = 1
    while warm < a.warmup and (warm + 1) * t_step < 60.0:
        state = O.stars_compute_step_f32(*state, g, p, dt, k)
        warm += 1
    steps = max(1, min(a.steps, int(a.ref_budget_s / max(t_step, 1e-9))))
    t0 = time.perf_counter()
    for _ in range(steps):
        state = O.stars_compute_step_f32(*state, g, p, dt, k)
    el = time.perf_counter() - t0
    assert np.isfinite(state[0]).all()
    value = g.ncell * steps / el
    sample = (f"{steps} timed steps (after {warm} warm-up) of the {a.n}^3, {a.stars}-star "
              f"workload; complex64/float32 NumPy/SciPy restatement of "
              f"quantum-stars.py:295-330, the reference's own precision (x64 off); reference "
              f"JAX is not installable")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": world, "steps": steps, "steps_requested": a.steps, "warmup": warm,
            "ms_per_step": el / steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c64/f32 (x64 off, as the reference)",
            "data": "synthetic (seeded Gaussian random field, uniform stars)",
            "config": bench_config(a.n, a.stars, dt, world),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": O.WORKERS, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    a = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        run_reference(a, rank, world)
        return

    import numpy as np
    import torch

    import qj
    from oracle import oracle as O

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    from qj import dist as qdist

    dist = qdist.init("nccl", device=dev)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        return qdist.max_over_ranks(x, dist, dev)

    n, n_s = a.n, a.stars
    psi0, pos0, vel0, g, p, dt = make_ic(n, n_s)
    C = g.ncell
    grid = qj.Grid(n, n, n)
    phys = qj.Phys(m_per_hbar=1.0, G=p.G, rho_bar=p.rho_bar)

    def fresh(precision):
        ct = torch.complex64 if precision == qj.FUSED_F32 else torch.complex128
        rt = torch.float32 if precision == qj.FUSED_F32 else torch.float64
        ps = torch.as_tensor(psi0, dtype=ct, device=dev)
        po = torch.as_tensor(pos0, dtype=rt, device=dev)
        ve = torch.as_tensor(vel0, dtype=rt, device=dev)
        diag = torch.tensor([0.0, 0.0, dt], dtype=torch.float64, device=dev)
        return ps, po, ve, diag

    lib = qj.lib()
    stream = torch.cuda.current_stream()

    # ---------------- fused float32: device-timed ----------------
    fused = qj.Plan(grid, phys, qj.FUSED_F32, n_s)
    ps, po, ve, diag = fresh(qj.FUSED_F32)
    # launch tuning (per pass: radix plan, pencil tile, CTAs per SM; reserved
    # slots), timed on a copy of the state before the warm-up; the accuracy
    # leg below runs the same tuned plan
    tuning = fused.tuning
    if not a.no_autotune:
        tuning = fused.autotune(ps, po, ve, p.m_s, dt, probe_steps=20,
                                cache_file=os.path.join(a.tune_dir, "tuning.json"))
    fused.kdk_step(ps, po, ve, diag, dt, a.warmup, p.m_s)
    barrier()
    clocks = Clocks(local)
    clocks.start()
    time.sleep(0.3)
    l0 = lib.qj_launch_count()
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    fused.kdk_step(ps, po, ve, diag, dt, a.steps, p.m_s)
    e1.record(stream)
    barrier()
    launches = int(lib.qj_launch_count() - l0)
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    ms_max = max_over_ranks(ms)
    value = world * C * a.steps / (ms_max * 1e-3)
    # the per-pass split: CUDA events around every pass on the launching
    # stream, in a separate run (events between the passes would also stand
    # between a pass and its programmatic dependent in the timed run)
    import ctypes

    prof_steps = min(a.steps, 200)
    lib.qj_profile_enable(1)
    fused.kdk_step(ps, po, ve, diag, dt, prof_steps, p.m_s)
    torch.cuda.synchronize()
    pms = (ctypes.c_double * 9)()
    pcnt = (ctypes.c_int64 * 9)()
    lib.qj_profile_read(pms, pcnt, 9)
    lib.qj_profile_enable(0)

    # roofline of the dominant pass
    hbm, hbm_kind = peaks()
    per_pass = {}
    for b in range(9):
        if pcnt[b]:
            per_pass[PASS_NAMES[b]] = {"launches": int(pcnt[b]), "total_ms": pms[b],
                                       "avg_us": 1e3 * pms[b] / pcnt[b]}
    dom = max((b for b in PASS_BYTES if pcnt[b]), key=lambda b: pms[b])
    avg_s = pms[dom] / pcnt[dom] * 1e-3
    achieved = PASS_BYTES[dom] * C / avg_s / 1e9
    tr = ncu_traffic().get(PASS_NAMES[dom])
    roofline = {"bound": "hbm", "kernel": PASS_NAMES[dom], "achieved": achieved, "peak": hbm,
                "peak_kind": hbm_kind, "unit": "GB/s", "frac": achieved / hbm,
                "traffic": tr, "alg_bytes_per_launch": PASS_BYTES[dom] * C}
    step_bw = STEP_BYTES * C * a.steps / (ms * 1e-3) / 1e9
    step_roof = {"alg_bytes_per_cell_step": STEP_BYTES, "achieved_gbs": step_bw,
                 "frac": step_bw / hbm}

    # ---------------- plain float64 rate ----------------
    plain = qj.Plan(grid, phys, qj.PLAIN_F64, n_s)
    qs, qo, qv, qd = fresh(qj.PLAIN_F64)
    plain.kdk_step(qs, qo, qv, qd, dt, 1, p.m_s)
    barrier()
    e0.record(stream)
    plain.kdk_step(qs, qo, qv, qd, dt, a.plain_steps, p.m_s)
    e1.record(stream)
    barrier()
    pl_ms = max_over_ranks(e0.elapsed_time(e1))
    plain_value = world * C * a.plain_steps / (pl_ms * 1e-3)

    # ---------------- accuracy: fused vs float64 after the same steps --------
    err_steps = a.err_steps
    ps, po, ve, diag = fresh(qj.FUSED_F32)
    qs, qo, qv, qd = fresh(qj.PLAIN_F64)
    mass0 = float((qs.abs() ** 2).sum())
    fused.kdk_step(ps, po, ve, diag, dt, err_steps, p.m_s)
    plain.kdk_step(qs, qo, qv, qd, dt, err_steps, p.m_s)
    torch.cuda.synchronize()
    psi_err = float(torch.linalg.vector_norm(ps.to(torch.complex128) - qs) /
                    torch.linalg.vector_norm(qs))
    rf, rp = ps.abs().double() ** 2, qs.abs() ** 2
    rho_err = float(torch.linalg.vector_norm(rf - rp) / torch.linalg.vector_norm(rp))
    mass_drift = float(rf.sum()) / mass0 - 1.0
    pos_err = float(torch.linalg.vector_norm(po.double() - qo) / torch.linalg.vector_norm(qo))
    del qs, qo, qv, qd
    plain.close()

    # ---------------- e2e through the public API with host buffers ----------
    # qj.HostPipeline: each call takes a state from pinned host memory, runs
    # e2e_sub KDK steps (the reference's host-sync interval nt_sub) and writes
    # the state and diagnostics back to pinned host memory; the copies of the
    # neighbouring calls overlap the steps (copy streams, three device buffers)
    e2e = None
    if not a.no_e2e:
        sub = a.e2e_sub
        h_in = (torch.as_tensor(psi0, dtype=torch.complex64).pin_memory(),
                torch.as_tensor(pos0, dtype=torch.float32).pin_memory(),
                torch.as_tensor(vel0, dtype=torch.float32).pin_memory(),
                torch.tensor([0.0, 0.0, dt], dtype=torch.float64).pin_memory())
        h_out = [tuple(torch.empty_like(t).pin_memory() for t in h_in) for _ in range(3)]
        plan_e = qj.Plan(grid, phys, qj.FUSED_F32, n_s)
        plan_e.tuning = tuning  # the device-timed plan's launch tuning
        pipe = qj.HostPipeline(plan_e, dt, sub, m_s=p.m_s, n_s=n_s, device=dev)
        calls = a.e2e_calls
        pipe.run([h_in] * 3, h_out)  # warm-up
        barrier()
        e0.record(stream)
        pipe.run([h_in] * calls, [h_out[i % 3] for i in range(calls)])
        e1.record(stream)
        barrier()
        e_ms = max_over_ranks(e0.elapsed_time(e1))
        h2d = sum(t.numel() * t.element_size() for t in h_in)
        d2h = h2d
        e2e = {"value": world * C * sub * calls / (e_ms * 1e-3), "unit": UNIT,
               "h2d_bytes_per_step": h2d / sub, "d2h_bytes_per_step": d2h / sub,
               "calls": calls, "ms_per_call": e_ms / calls,
               "unit_of_call": f"one qj.HostPipeline call = host->device psi/pos/vel/diag, {sub} "
                               f"KDK steps, device->host psi/pos/vel/diag (the reference's "
                               f"host-sync interval nt_sub); neighbouring calls' copies overlap "
                               f"the steps"}
        plan_e.close()

    # ---------------- adjoint / forward time (128^3, 200 steps, ckpt 20) -------
    adjoint = None
    if not a.no_adjoint:
        from qj.autograd import kdk_evolve

        na, steps_a, K = a.adj_n, a.adj_steps, a.adj_ckpt
        # the IC family with its 4096 stars as a fixed source density
        psi_a, pos_a, _, ga, pa = O.stars_ic(na, 4096, seed=0)
        rho_sa = torch.as_tensor(O.bin_stars(pos_a, ga, np.full(len(pos_a), pa.m_s)),
                                 dtype=torch.float32, device=dev)
        dta = O.default_dt(ga, pa)
        plan_a = qj.Plan(qj.Grid(na, na, na), qj.Phys(m_per_hbar=1.0, G=pa.G, rho_bar=pa.rho_bar),
                         qj.FUSED_F32, 1)
        s = torch.as_tensor(np.abs(psi_a), dtype=torch.float32, device=dev)
        th = torch.as_tensor(0.5 * O.delta_field(na, 21), dtype=torch.float32,
                             device=dev).requires_grad_(True)
        psi2, *_ = O.stars_ic(na, 0, seed=1)
        with torch.no_grad():  # target: a forward run from a second seed
            s2 = torch.as_tensor(np.abs(psi2), dtype=torch.float32, device=dev)
            tgt = torch.abs(kdk_evolve(torch.zeros_like(s2), s2, plan_a, dta, steps_a, K,
                                       rho_s=rho_sa)) ** 2

        def fwd():
            return kdk_evolve(th, s, plan_a, dta, steps_a, K, rho_s=rho_sa)

        def run_bwd(psiT):
            L = torch.mean((torch.abs(psiT) ** 2 - tgt) ** 2)
            L.backward()

        run_bwd(fwd())  # warm-up
        barrier()
        psi_plain = torch.polar(s, th.detach()).to(torch.complex64)
        diag_a = torch.tensor([0.0, 0.0, dta], dtype=torch.float64, device=dev)
        e0.record(stream)
        plan_a.kdk_step(psi_plain, None, None, diag_a, dta, steps_a)
        e1.record(stream)
        barrier()
        f_ms = e0.elapsed_time(e1)
        e0.record(stream)
        psiT = fwd()
        e1.record(stream)
        barrier()
        fc_ms = e0.elapsed_time(e1)
        th.grad = None
        e0.record(stream)
        run_bwd(psiT)
        e1.record(stream)
        barrier()
        b_ms = e0.elapsed_time(e1)
        adjoint = {"grid": [na] * 3, "steps": steps_a, "checkpoint_every": K,
                   "star_source": "4096 stars' CIC density, held fixed",
                   "forward_ms": fc_ms, "forward_psi_only_ms": f_ms,
                   "backward_ms": b_ms, "adjoint_over_forward": b_ms / fc_ms,
                   "note": "forward = the checkpointed forward with the star source "
                           "(kdk_evolve); backward = chunk recompute from checkpoints + reverse "
                           "sweep (two Poisson solves per kick); forward_psi_only = qj_kdk_step "
                           "without the source"}
        plan_a.close()

    # ---------------- ensemble: 16x64^3 + 8x96^3 + 8x128^3, 256 stars each -----
    ensemble = None
    if not a.no_ensemble:
        all_groups = [(64, 16), (96, 8), (128, 8)]
        # the 32 boxes (seeds 100..131) split across ranks by cost; one batched
        # plan per size class a rank holds (no collective between ranks)
        boxes = [(n_e, 100 + i) for i, n_e in enumerate(
            [n_e for n_e, nb in all_groups for _ in range(nb)])]
        mine = qdist.partition_boxes([qdist.box_cost(b[0] ** 3) for b in boxes], world)[rank]
        groups = []
        for n_e, _ in all_groups:
            seeds = [boxes[i][1] for i in mine if boxes[i][0] == n_e]
            if seeds:
                groups.append((n_e, len(seeds), seeds))
        ens_steps = a.ens_steps
        plans, state, singles = [], [], []
        for n_e, nb, seeds in groups:
            ics = [O.stars_ic(n_e, 256, seed=sd) for sd in seeds]
            g_e, p_e = ics[0][3], ics[0][4]
            dt_e = O.default_dt(g_e, p_e)
            pl = qj.Plan(qj.Grid(n_e, n_e, n_e),
                         qj.Phys(m_per_hbar=1.0, G=p_e.G, rho_bar=p_e.rho_bar), qj.FUSED_F32, 256,
                         nbox=nb)
            psi_e = torch.as_tensor(np.stack([i[0] for i in ics]), dtype=torch.complex64,
                                    device=dev).contiguous()
            pos_e = torch.as_tensor(np.stack([i[1] for i in ics]), dtype=torch.float32,
                                    device=dev).contiguous()
            vel_e = torch.zeros_like(pos_e)
            diag_e = torch.tensor([[0.0, 0.0, dt_e]] * nb, dtype=torch.float64, device=dev)
            plans.append(pl)
            state.append([psi_e, pos_e, vel_e, diag_e, dt_e, p_e.m_s])
            singles.append(qj.Plan(qj.Grid(n_e, n_e, n_e),
                                   qj.Phys(m_per_hbar=1.0, G=p_e.G, rho_bar=p_e.rho_bar),
                                   qj.FUSED_F32, 256))
        if not a.no_autotune:
            # each batched plan, and each single-box plan of the one-by-one
            # comparison, on its own state (the first box for the latter); the
            # batched plans keep the default radix plan and tile, which the
            # ensemble's one launch per pass requires
            for pl, sg, stt in zip(plans, singles, state):
                pl.autotune(stt[0], stt[1], stt[2], stt[5], stt[4], probe_steps=5,
                            cache_file=os.path.join(a.tune_dir, "tuning.json"), shapes=False)
                sg.autotune(stt[0][0].contiguous(), stt[1][0].contiguous(),
                            stt[2][0].contiguous(), stt[5], stt[4], probe_steps=5,
                            cache_file=os.path.join(a.tune_dir, "tuning.json"))
        ens = qj.Ensemble(plans)
        merged = ens.merged
        init = [[t.clone() if isinstance(t, torch.Tensor) else t for t in s] for s in state]

        def ens_run(m):
            ens.step([s[0] for s in state], [s[1] for s in state], [s[2] for s in state],
                     [s[3] for s in state], [s[4] for s in state], [s[5] for s in state], m,
                     chunk=a.ens_chunk, graph=True)

        ens_run(a.ens_chunk)  # capture + warm-up
        barrier()
        e0.record(stream)
        ens_run(ens_steps)
        e1.record(stream)
        barrier()
        ens_ms = max_over_ranks(e0.elapsed_time(e1))
        # the same steps as one launch per fused pass for all sizes (same
        # bits), on a copy of the state, for comparison
        ens_m = qj.Ensemble(plans, merge=True)
        merged_ms = None
        if ens_m.merged:
            sm = [[t.clone() if isinstance(t, torch.Tensor) else t for t in x] for x in init]

            def ens_m_run(m):
                ens_m.step([x[0] for x in sm], [x[1] for x in sm], [x[2] for x in sm],
                           [x[3] for x in sm], [x[4] for x in sm], [x[5] for x in sm], m,
                           chunk=a.ens_chunk, graph=True)

            ens_m_run(a.ens_chunk)
            barrier()
            e0.record(stream)
            ens_m_run(ens_steps)
            e1.record(stream)
            barrier()
            merged_ms = max_over_ranks(e0.elapsed_time(e1))
        ens_m.close()
        cells = sum(n_e**3 * nb for n_e, nb in all_groups)  # all ranks' boxes
        # one by one: each box alone through a single-box plan, same steps
        views, first = [], []
        for gi, (n_e, nb, _) in enumerate(groups):
            first.append(len(views))
            for b in range(nb):
                s = init[gi]
                views.append((singles[gi], s[0][b].clone(), s[1][b].clone(), s[2][b].clone(),
                              s[3][b].clone(), s[4], s[5]))
        for i in first:  # warm-up each size
            v = views[i]
            v[0].kdk_step(v[1], v[2], v[3], v[4], v[5], 2, v[6])
        barrier()
        e0.record(stream)
        for v in views:
            v[0].kdk_step(v[1], v[2], v[3], v[4], v[5], ens_steps, v[6])
        e1.record(stream)
        barrier()
        seq_ms = max_over_ranks(e0.elapsed_time(e1))
        # every box against the float64 path (outside the timed region), then
        # the end-of-run gather of the per-box diagnostics from all ranks
        records = []
        for gi, (n_e, nb, seeds) in enumerate(groups):
            pl64 = qj.Plan(qj.Grid(n_e, n_e, n_e),
                           qj.Phys(m_per_hbar=1.0, G=plans[gi].phys.G, rho_bar=plans[gi].phys.rho_bar),
                           qj.PLAIN_F64, 256)
            s0 = init[gi]
            for b in range(nb):
                ps64 = s0[0][b].to(torch.complex128).contiguous()
                po64 = s0[1][b].double().contiguous()
                ve64 = s0[2][b].double().contiguous()
                d64 = torch.tensor([0.0, 0.0, s0[4]], dtype=torch.float64, device=dev)
                m0 = float((ps64.abs() ** 2).sum())
                pl64.kdk_step(ps64, po64, ve64, d64, s0[4], a.ens_chunk + ens_steps, s0[5])
                got = state[gi][0][b].to(torch.complex128)
                records.append({
                    "box": seeds[b] - 100, "n": n_e, "seed": seeds[b], "rank": rank,
                    "psi_rel_l2_vs_f64": float(torch.linalg.vector_norm(got - ps64) /
                                               torch.linalg.vector_norm(ps64)),
                    "mass_drift": float((got.abs() ** 2).sum()) / m0 - 1.0})
            pl64.close()
        per_box = qdist.gather_box_records(records, dist)
        worst = {}
        for r in per_box:
            k = f"{r['n']}^3"
            worst[k] = max(worst.get(k, 0.0), r["psi_rel_l2_vs_f64"])
        ensemble = {"boxes": "16x64^3 + 8x96^3 + 8x128^3, 256 stars each",
                    "launches": ("one persistent launch per fused pass for all sizes"
                                 if merged else "one stream per size class"),
                    "sharding": f"{world} rank(s), greedy by C log C; this rank: "
                                + ", ".join(f"{nb}x{n_e}^3" for n_e, nb, _ in groups),
                    "tuning": {f"{n_e}^3": pl.tuning for (n_e, _, _), pl in zip(groups, plans)},
                    "cells": cells, "steps": ens_steps, "graph_chunk": a.ens_chunk,
                    "ensemble_cell_steps_per_s": cells * ens_steps / (ens_ms * 1e-3),
                    "one_launch_per_pass_cell_steps_per_s": (
                        cells * ens_steps / (merged_ms * 1e-3) if merged_ms else None),
                    "one_by_one_cell_steps_per_s": cells * ens_steps / (seq_ms * 1e-3),
                    "speedup": seq_ms / ens_ms,
                    "psi_rel_l2_vs_f64_max": worst,
                    "mass_drift_max_abs": max(abs(r["mass_drift"]) for r in per_box),
                    "boxes_checked": len(per_box),
                    "per_box": [{k: (float(f"{v:.3e}") if isinstance(v, float) else v)
                                 for k, v in r.items() if k != "seed"} for r in per_box],
                    "error_steps": a.ens_chunk + ens_steps}
        ens.close()
        for pl in plans + singles:
            pl.close()

    # ---------------- gas + black hole, 128^3 (quantum-gas-bh.py:537-578) ------
    gas_bh = None
    if not a.no_gas:
        gas_bh = gas_bh_leg(a, dev, stream, barrier)

    cb = None
    if rank == 0 and world == 1 and not a.no_cpu:
        cb = cpu_baseline(n, n_s, 5)
        cb = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample", "float64")}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_max / a.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "c64/f32 (phases, k=0 mode, mean density in f64)",
                "data": "synthetic (seeded Gaussian random field, uniform stars)",
                "config": bench_config(n, n_s, dt, world),
                "plain_f64": {"value": plain_value, "ms_per_step": pl_ms / a.plain_steps,
                              "steps": a.plain_steps},
                "fused_over_plain": value / plain_value,
                "accuracy": {"steps": err_steps, "psi_rel_l2_vs_f64": psi_err,
                             "rho_rel_l2_vs_f64": rho_err, "mass_drift": mass_drift,
                             "pos_rel_l2_vs_f64": pos_err,
                             "f64_path": "plain float64 GPU path (matches the oracle to 1e-11)"},
                "roofline": roofline, "step_roofline": step_roof, "passes": per_pass,
                "passes_note": f"CUDA events around each pass, a separate {prof_steps}-step run",
                "tuning": tuning,
                "gpu_launches": launches, "clocks": clk, "e2e": e2e, "cpu_baseline": cb,
                "adjoint": adjoint, "ensemble": ensemble, "gas_bh": gas_bh}
        print(json.dumps(line), flush=True)
    fused.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
