"""The multi-rank host logic of bench.py on CPU: two gloo ranks (the path runs
as independent replicas, so the only exchange is the max-over-ranks timing),
and the reference arm's non-zero ranks exiting without work."""
import os
import socket
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch

    sys.path.insert(0, REPO)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = [3.0, 5.0][rank]
        worst = bench.max_over_ranks(ms, world, "cpu")
        torch.distributed.barrier()
        out.put((rank, worst, bench.replica_value(282_048, world, worst)))
    finally:
        torch.distributed.destroy_process_group()


def test_max_over_ranks_gloo():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # both ranks see the slower rank's time, and the whole-job value counts both replicas
    assert [g[1] for g in got] == [5.0, 5.0]
    assert got[0][2] == pytest.approx(2 * 282_048 / 5e-3 / 1e6)


def test_replica_value_single_rank():
    sys.path.insert(0, REPO)
    import bench

    assert bench.max_over_ranks(2.5, 1, "cpu") == 2.5
    assert bench.replica_value(1_000_000, 1, 10.0) == pytest.approx(100.0)


def test_reference_arm_nonzero_rank_exits_without_work():
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
