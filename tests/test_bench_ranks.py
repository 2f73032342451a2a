"""CPU tests of the bench's multi-rank plumbing (replicas, no data-path
collective): two gloo ranks agree on the slowest rank's time and the whole-job
rate, and the rank environment is read as torchrun sets it."""
import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank_main(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ws, r, local = bench.dist_env()
        ms = 10.0 + 5.0 * rank          # rank 1 is the slower replica
        slow = bench.max_over_ranks(ms, dist)
        rate = bench.job_rate(ws, 64 ** 3, 55, slow * 1e-3)
        out.put((rank, ws, r, local, slow, rate))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_report_the_slowest_replica():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29000 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ws, r, local, slow, rate in res:
        assert (ws, r, local) == (2, rank, rank)
        assert slow == 15.0
        assert rate == pytest.approx(2 * 64 ** 3 * 55 / 15e-3)


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(12.5) == 12.5
    assert bench.job_rate(1, 100, 4, 2.0) == 200.0


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    """Under torchrun the reference arm's other ranks exit 0 without work."""
    sys.path.insert(0, ROOT)
    import argparse

    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    args = argparse.Namespace(gpus=2, steps=2, warmup=1)
    assert bench.run_reference_arm(args) == 0
    assert capsys.readouterr().out == ""


def test_reference_arm_maps_no_package_library():
    """The reference arm builds its initial condition from hit_ic.py alone and
    runs the reference's C++ (or the oracle port): its process never maps
    libmc3d.so, and it imports nothing of the package."""
    import subprocess
    code = ("import sys; sys.path.insert(0, %r); import bench; r = bench.cpu_reference_rate(16, 5, 0); "
            "maps = open('/proc/self/maps').read(); "
            "print('libmc3d' in maps, 'mpi_3dcompact_b200' in sys.modules, r[2], r[0] > 0)" % ROOT)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr
    mapped, imported, kind, positive = out.stdout.split()
    assert mapped == "False" and imported == "False" and positive == "True", out.stdout
    assert kind in ("reference", "port")
