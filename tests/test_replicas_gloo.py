"""CPU: the multi-GPU host path of bench.py with two gloo ranks.

The path shards as replicas (independent systems, no exchange step), so the
only collective is the timing reduction: every rank gets the slowest rank's
time, and the whole-job value counts every rank's work.  The reference arm
runs on rank 0 alone; the other ranks exit 0 without work.
"""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import bench
    r, w, lr = bench.rank_info()
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t = bench.max_over_ranks(1.0 + rank, dist, "cpu")  # rank 1 is the slow one
        value = bench.whole_job_ns_per_day(w, 1000, t)
        out.put((rank, r, w, lr, t, value))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    import torch.multiprocessing as mp
    import bench
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, r, w, lr, t, value in res:
        assert (r, w, lr) == (rank, 2, rank)
        assert t == 2.0  # max over ranks, on every rank
        assert value == pytest.approx(2 * 1000 * 1e-6 / 2.0 * 86400.0)
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5


def test_reference_arm_exits_without_work_on_other_ranks(monkeypatch):
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("LOCAL_RANK", "1")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--gpus", "2"])

    def no_work(*a, **k):
        raise AssertionError("rank 1 must not run the reference")
    monkeypatch.setattr(bench, "run_reference", no_work)
    assert bench.main() == 0


def _gpus_worker(rank, world, port, gpus, out):
    """A gloo rank that asks bench.py's GPU count for `gpus` GPUs."""
    import datetime
    import torch.distributed as dist
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        r, w, _ = bench.rank_info()
        try:
            n = bench.check_world(gpus, w)
        except SystemExit as exc:
            n = "refused: " + str(exc)
        # the whole-job value counts the ranks that ran, each its own replica
        value = bench.whole_job_ns_per_day(n, 1000, 1.0) if isinstance(n, int) else None
        out.put((rank, n, value))
    finally:
        dist.destroy_process_group()


def test_gpus_count_is_the_ranks_that_ran():
    """--gpus 2 under two ranks counts two replicas; --gpus 4 under two
    ranks is refused on every rank (no value inflated by replicas that were
    never started)."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    for gpus, want in ((2, 2), (4, None)):
        q = ctx.Queue()
        port = _free_port()
        procs = [ctx.Process(target=_gpus_worker, args=(r, 2, port, gpus, q)) for r in range(2)]
        for p in procs:
            p.start()
        res = sorted(q.get(timeout=120) for _ in procs)
        for p in procs:
            p.join(timeout=60)
            assert p.exitcode == 0
        for rank, n, value in res:
            if want is None:
                assert isinstance(n, str) and n.startswith("refused") and "--nproc-per-node 4" in n
            else:
                assert n == want
                assert value == pytest.approx(2 * 1000 * 1e-6 / 1.0 * 86400.0)


def test_gpus_without_launcher_is_refused(monkeypatch):
    """One process asked for eight GPUs: refused before any work."""
    import bench
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    monkeypatch.setattr(sys, "argv", ["bench.py", "--gpus", "8", "--impl", "reference"])
    with pytest.raises(SystemExit) as exc:
        bench.main()
    assert "needs 8 ranks" in str(exc.value)
    assert bench.check_world(1, 1) == 1


def test_warmup_plan_covers_whole_periods():
    """The headline run's warm-up ends on a list-period boundary and has
    run every step-block shape the timed region replays."""
    import bench
    B = bench.BLOCK
    for w, k in ((5, 20), (3, 7), (100, 2000), (0, 25), (12, 13)):
        plan = bench.warmup_plan(w, k)
        assert sum(plan) >= max(3, w)
        assert sum(plan) % B == 0
        if k % B:
            assert k % B in plan
        assert all(1 <= b <= B for b in plan)
