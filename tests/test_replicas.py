"""The multi-GPU path of bench.py is independent replicas: the process group carries only the
barriers and the max-over-ranks timing reduction.  Exercised here with world size 2 on the
gloo backend (CPU), as bench.py would run it under torchrun."""
import os
import socket
import sys
from pathlib import Path

import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, str(ROOT))
    import bench

    r, w, local = bench.dist_env()
    bench.init_replicas(w, local, backend="gloo")
    bench.replica_barrier(w)
    # rank-dependent timings: the job time is the slowest rank's
    got = bench.max_over_ranks([10.0 + r, 3.0 - r, 7.5], w, "cpu")
    bench.close_replicas(w)
    out.put((r, got))


def test_world_size_two_takes_the_max_over_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert results[0] == results[1] == [11.0, 3.0, 7.5]


def test_single_process_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.max_over_ranks([1.0, 2.0], 1, "cpu") == [1.0, 2.0]
    bench.replica_barrier(1)
    bench.close_replicas(1)


def test_reference_arm_prints_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, str(ROOT))
    import bench

    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    args = type("A", (), {"gpus": 2, "steps": 1, "warmup": 0, "segment": 1})()
    bench.run_reference(args)
    assert capsys.readouterr().out == ""
