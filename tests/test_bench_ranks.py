"""The multi-rank plumbing of bench.py on CPU: world size 2 over gloo (the GPU runs use
the same code over NCCL, one process per GPU)."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def _worker(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        step_ms = 10.0 + 5.0 * rank          # rank 1 is the slowest
        slowest = bench.max_over_ranks(step_ms, dist, "cpu")
        out.put((rank, slowest, bench.whole_job_rate(4_194_304, world, slowest)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_rate_world_size_2():
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    results = sorted(out.get(timeout=10) for _ in range(2))
    assert [r[1] for r in results] == [15.0, 15.0]           # every rank sees the max
    assert results[0][2] == pytest.approx(2 * 4_194_304 / 15e-3 / 1e6)


def test_reference_arm_prints_only_on_rank_0():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "1"],
                       capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""
