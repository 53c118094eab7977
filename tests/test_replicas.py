"""The multi-GPU form of the benchmark is replicas only: every rank runs the
whole workload on its own GPU, and the job reports the aggregate rate over
the slowest replica's time (bench.py replicas_max / replicas_rate).  The
host-side logic runs here as two gloo ranks on the CPU."""
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, times, q):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=timedelta(seconds=60))
    try:
        t = bench.replicas_max(times[rank], ws, device="cpu")
        q.put((rank, t, bench.replicas_rate(1000.0, ws, t)))
    finally:
        dist.destroy_process_group()


def test_replicas_take_the_slowest_rank_and_aggregate_the_units():
    ws, times = 2, [0.25, 0.40]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, ws, port, times, q)) for r in range(ws)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(ws))
    for _, t, rate in out:
        assert t == 0.40  # every rank sees the slowest replica's time
        assert rate == pytest.approx(1000.0 * ws / 0.40)


def test_single_rank_needs_no_process_group():
    assert bench.replicas_max(1.5, 1) == 1.5
    assert bench.replicas_rate(10.0, 1, 2.0) == 5.0


def test_reference_arm_runs_on_rank_zero_only():
    """Under torchrun the reference arm (the CPU implementation) runs on rank
    0 alone; the other ranks exit 0 without work or output."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "1"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_a_failing_extra_is_reported_not_raised():
    out = bench.guarded(lambda: 1 / 0)
    assert out == {"error": "ZeroDivisionError: division by zero"}
    assert bench.guarded(lambda a, b=0: a + b, 2, b=3) == 5
