"""Host logic of bench.py's multi-GPU arm (replicas: one process per GPU, no
data-path exchange), on CPU with the gloo backend and world size 2: each
rank gets its own seeded image, timings reduce to the maximum over ranks, the
whole-job rate counts every rank's patches over that maximum, and the CPU
reference arm prints on rank 0 only."""

import os
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        r, w, local = bench.dist_env()
        ms = 10.0 + 5.0 * rank  # rank 1 is the slower one
        mx = bench.reduce_max(ms, dist)
        rate = bench.aggregate_rate(1000, w, mx)
        from ksvd_loader import load
        wl = load().synth.WORKLOADS["img512_p12s3_k256"]
        img = bench.replica_workload(wl, r).images()[1]
        q.put((r, w, local, mx, rate, float(img[:8, :8].sum())))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 2000)
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, w0, l0, mx0, rate0, s0), (r1, w1, l1, mx1, rate1, s1) = res
    assert (r0, r1) == (0, 1) and w0 == w1 == 2 and (l0, l1) == (0, 1)
    assert mx0 == mx1 == 15.0                         # max over ranks
    assert rate0 == rate1 == pytest.approx(2 * 1000 / 0.015)
    assert s0 != s1                                   # replicas denoise different images


def test_reference_arm_runs_on_rank0_only(monkeypatch, capsys):
    sys.path.insert(0, str(ROOT))
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class A:
        steps, warmup, gpus = 1, 3, 2
    assert bench.run_reference(A, None) == 0
    assert capsys.readouterr().out == ""


def test_single_process_helpers():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.reduce_max(3.5, None) == 3.5
    assert bench.aggregate_rate(461041, 1, 10.0) == pytest.approx(46104100.0)
    assert np.isfinite(bench.aggregate_rate(1, 8, 1e-3))
