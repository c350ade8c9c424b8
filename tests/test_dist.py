"""Multi-process host logic on CPU (gloo, world size 2): the max-over-ranks
timing, the box partition every rank computes identically, the end-of-run
gather of per-box diagnostics, the reference arm's rank-0-only output, and a
rank that leaves: the other rank's next collective ends with an error within
the short process-group timeout instead of waiting for good."""

import os
import socket
import subprocess
import sys
import time

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_partition_boxes_covers_each_box_once_and_balances():
    from qj import dist

    costs = [dist.box_cost(n**3) for n in [64] * 16 + [96] * 8 + [128] * 8]
    for world in (1, 2, 3, 4, 8):
        parts = dist.partition_boxes(costs, world)
        assert sorted(i for p in parts for i in p) == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs) + 1e-9
        assert parts == dist.partition_boxes(costs, world)  # deterministic


def _worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, os.path.join(ROOT, "quantum-jax_b200"))
    from qj import dist as qd

    d = qd.init("gloo", timeout_s=60)
    m = qd.max_over_ranks(1.5 + rank, d)
    costs = [qd.box_cost(n**3) for n in [64] * 16 + [96] * 8 + [128] * 8]
    mine = qd.partition_boxes(costs, world)[rank]
    allp = [None] * world
    d.all_gather_object(allp, mine)
    recs = qd.gather_box_records([{"box": i, "rank": rank, "err": 1e-7 * i} for i in mine], d)
    dup = None
    try:  # a box claimed by both ranks is refused on both
        qd.gather_box_records([{"box": 0, "rank": rank}], d)
    except ValueError as e:
        dup = str(e)
    d.barrier()
    d.destroy_process_group()
    out.put((rank, m, allp, recs, dup))


@pytest.mark.timeout(120)
def test_two_gloo_ranks_agree():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=100) for _ in procs)
    for p in procs:
        p.join(30)
        assert p.exitcode == 0
    (r0, m0, a0, g0, d0), (r1, m1, a1, g1, d1) = res
    assert m0 == m1 == 2.5
    assert a0 == a1 and sorted(a0[0] + a0[1]) == list(range(32))
    # the per-box diagnostics gather: every box once, in box order, on both ranks
    assert g0 == g1 and [r["box"] for r in g0] == list(range(32))
    assert all(r["rank"] == (0 if r["box"] in a0[0] else 1) for r in g0)
    assert d0 and d1 and "more than one rank" in d0


def test_reference_arm_prints_only_on_rank_zero():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "0"],
                       capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""


def _leaving_worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, os.path.join(ROOT, "quantum-jax_b200"))
    from qj import dist as qd

    d = qd.init("gloo", timeout_s=5)
    if rank == 1:
        os._exit(3)  # leaves between steps, before the timing collective
    t0 = time.time()
    try:
        qd.max_over_ranks(1.0, d)
        res = "returned"
    except Exception as e:  # the error a surviving rank sees
        res = type(e).__name__
    out.put((rank, res, time.time() - t0))
    out.close()
    out.join_thread()
    os._exit(0)


@pytest.mark.timeout(120)
def test_rank_that_leaves_ends_the_others_collective_with_an_error():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_leaving_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    rank, res, waited = q.get(timeout=100)
    for p in procs:
        p.join(30)
    assert rank == 0 and res != "returned"
    assert waited < 60
    assert [p.exitcode for p in procs] == [0, 3]
