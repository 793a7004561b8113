"""Multi-rank plumbing (rsgpu.ranks) with world_size 2 over gloo on the CPU:
the max-over-ranks reduction the benchmark times with, the stripe partition,
and failure detection on the host (a rank that dies before a collective makes
the other fail with an error inside the group's timeout instead of hanging)."""
import multiprocessing as mp
import os
import socket
import sys
import time

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "rustfs-erasure-codec_b200"))

from rsgpu import ranks as R  # noqa: E402


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank, world, port):
    return {"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
            "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)}


def _worker_reduce(rank, world, port, q):
    os.environ.update(_env(rank, world, port))
    sys.path.insert(0, os.path.join(ROOT, "rustfs-erasure-codec_b200"))
    from rsgpu import ranks

    rk = ranks.from_env()
    g = ranks.Group(rk, "gloo", timeout_s=30.0, device="cpu")
    try:
        g.barrier()
        mx = g.max(1.5 + rk.rank)           # per-rank step time
        sm = g.sum(10.0 * (rk.rank + 1))
        first, count = ranks.stripe_share(4097, rk.rank, rk.world)
        q.put((rk.rank, mx, sm, first, count, g.distributed))
    finally:
        g.close()


def _worker_dies(rank, world, port, q):
    os.environ.update(_env(rank, world, port))
    sys.path.insert(0, os.path.join(ROOT, "rustfs-erasure-codec_b200"))
    from rsgpu import ranks

    rk = ranks.from_env()
    g = ranks.Group(rk, "gloo", timeout_s=5.0, device="cpu")
    if rk.rank == 1:
        os._exit(3)  # dies between steps: joined the group, never reaches the collective
    t0 = time.time()
    try:
        g.max(1.0)
        q.put((rk.rank, "no error", time.time() - t0))
    except Exception as e:  # the survivor learns of the failure from the collective
        q.put((rk.rank, type(e).__name__, time.time() - t0))


def _run(target, world=2, timeout=120):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=target, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout)
    alive = [p for p in procs if p.is_alive()]
    for p in alive:
        p.kill()
    assert not alive, "a rank hung"
    out = []
    while not q.empty():
        out.append(q.get())
    return procs, out


def test_max_and_sum_over_two_gloo_ranks():
    procs, out = _run(_worker_reduce)
    assert all(p.exitcode == 0 for p in procs)
    assert len(out) == 2
    shares = []
    for rank, mx, sm, first, count, distributed in out:
        assert distributed
        assert mx == 2.5           # the slowest rank's time, on every rank
        assert sm == 30.0
        shares.append((first, count))
    shares.sort()
    assert shares == [(0, 2049), (2049, 2048)]


def test_dead_rank_fails_the_survivor_within_the_timeout():
    procs, out = _run(_worker_dies)
    assert procs[1].exitcode == 3
    assert len(out) == 1
    rank, what, waited = out[0]
    assert rank == 0 and what != "no error"
    assert waited < 60


def test_single_rank_needs_no_group():
    rk = R.from_env({})
    assert (rk.rank, rk.world, rk.local) == (0, 1, 0)
    g = R.Group(rk, "gloo", device="cpu")
    assert not g.distributed
    assert g.max(3.25) == 3.25 and g.sum(2.0) == 2.0
    g.barrier()
    g.close()


@pytest.mark.parametrize("n,world", [(0, 2), (1, 2), (10, 3), (4096, 8), (7, 8)])
def test_stripe_share_covers_every_stripe_once(n, world):
    seen = []
    for r in range(world):
        first, count = R.stripe_share(n, r, world)
        seen += list(range(first, first + count))
    assert seen == list(range(n))


def test_bad_rank_environment_is_rejected():
    with pytest.raises(ValueError):
        R.from_env({"RANK": "2", "WORLD_SIZE": "2"})


def test_reference_arm_other_ranks_exit_without_work(capsys):
    sys.path.insert(0, ROOT)
    import bench

    class A:
        steps, warmup = 1, 0

    assert bench.run_reference(A(), 1, 2) == 0
    assert capsys.readouterr().out == ""
