"""Replica scaling plumbing of bench.py on the CPU: two gloo ranks (the
GPU run uses NCCL with the same code), barrier + max over ranks of the timed
region, the whole-job rate, and the reference arm running on rank 0 only."""
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench
    d = bench.Dist(backend="gloo", timeout_s=60)
    d.barrier()
    m = d.max(10.0 + rank)          # each rank's "timed region" in ms
    out[rank] = (m, bench.whole_job_rate(3, d.world, m))
    d.barrier()
    d.close()


def test_two_gloo_ranks_take_the_max_time():
    world, port = 2, _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank_main, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
    assert out[0][0] == out[1][0] == 11.0
    assert out[0][1] == pytest.approx(3 * 2 / 0.011)


def test_single_process_rate():
    import bench
    assert bench.whole_job_rate(2, 1, 1000.0) == pytest.approx(2.0)


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""
