"""The multi-rank host logic of bench.py on CPU: two gloo ranks take the same
collective steps in the same order, the reported time is the slowest rank's,
the whole-job rate counts every rank's units, each rank gets its own replica
seed, and the reference arm runs on rank 0 only."""
import contextlib
import io
import os
import socket
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    import bench

    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        w, r, lr = bench.rank_env()
        dist.barrier()
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, dist, "cpu")   # device-timed region
        el = bench.max_over_ranks(2.0 - 0.5 * rank, dist, "cpu")    # e2e wall clock
        dist.barrier()
        out.put((rank, w, r, lr, ms, el, bench.replica_seed(122335456, r),
                 bench.whole_job_rate(1000, w, ms / 1e3)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_time_the_slowest_and_count_all_units():
    import torch.multiprocessing as mp

    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[0] for r in res] == [0, 1]
    for rank, w, r, lr, ms, el, seed, rate in res:
        assert (w, r, lr) == (2, rank, rank)
        assert ms == 15.0 and el == 2.0
        assert rate == pytest.approx(1000 * 2 / 0.015)
    assert res[0][6] != res[1][6]


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    import bench

    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    called = []
    monkeypatch.setattr(bench, "reference_build_run", lambda *a, **k: called.append(1))
    monkeypatch.setattr(bench, "cpu_port_rate", lambda *a, **k: called.append(1))
    args = type("A", (), dict(scounts="2,3", steps=2, warmup=1, N=256, gpus=2))()
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        assert bench.run_reference(args) == 0
    assert buf.getvalue() == "" and not called


def test_single_process_defaults(monkeypatch):
    import bench

    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    assert bench.rank_env() == (1, 0, 0)
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
    assert bench.replica_seed(7, 0) == 7


def test_reference_arm_line_on_rank_zero(monkeypatch):
    """Rank 0 prints one reference line on the arm's metric and config, its
    measured ms_per_step unscaled, with cpu_baseline and a zero-copy e2e."""
    import json

    import bench

    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    monkeypatch.setattr(bench, "reference_available", lambda: True)
    monkeypatch.setattr(bench, "reference_build_run", lambda N, sc, w, k, R: (1.0e6, 16.7e3, 16.7 * k))
    args = type("A", (), dict(scounts="2,3", steps=3, warmup=1, N=256, gpus=1))()
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        assert bench.run_reference(args) == 0
    line = json.loads(buf.getvalue())
    assert line["impl"] == "reference" and line["metric"] == "Model G site-updates/s"
    assert line["ms_per_step"] == 16.7e3 and line["steps"] == 3 and line["config"]["N"] == 256
    assert line["cpu_baseline"]["kind"] == "reference" and line["e2e"]["h2d_bytes_per_step"] == 0

