"""The multi-process path of bench.py on the CPU (gloo, world size 2).

The plain microenvironment does not shard: `bench.py --gpus N` runs N independent replicas, one
per rank, with no collective on the data path.  What the ranks share is the timing: the job's time
is the slowest rank's, and the throughput counts every rank's units.  These tests run that logic,
and the reference arm's multi-rank launch, as real processes on the CPU.
"""

import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, results):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = [12.5, 20.0][rank]  # rank 1 is the slower replica
        slowest = bench.reduce_max_over_ranks(ms, world, "cpu")
        rate = bench.whole_job_rate(world, 1000, 10, slowest)
        dist.barrier()
        results[rank] = (slowest, rate)
    finally:
        dist.destroy_process_group()


def test_replica_timing_takes_the_slowest_rank():
    import torch.multiprocessing as mp

    world = 2
    with mp.get_context("spawn").Manager() as manager:
        results = manager.dict()
        mp.start_processes(_rank_main, args=(world, _free_port(), results), nprocs=world, join=True,
                           start_method="spawn")
        got = dict(results)
    assert got[0] == got[1]  # every rank agrees
    slowest, rate = got[0]
    assert slowest == 20.0
    assert rate == pytest.approx(2 * 1000 * 10 / 0.020)


def test_whole_job_rate_single_rank():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.reduce_max_over_ranks(3.0, 1, "cpu") == 3.0
    assert bench.whole_job_rate(1, 500, 4, 2.0) == pytest.approx(500 * 4 / 0.002)


@pytest.mark.slow
def test_reference_arm_under_torchrun_prints_one_line():
    """`bench.py --impl reference` launched like the multi-GPU runs: rank 0 alone measures and
    prints; the other rank exits 0 without work."""
    import oracle

    oracle.build()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py", "--impl", "reference",
           "--gpus", "2", "--workload", "plain-50", "--steps", "2", "--warmup", "1"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["value"] > 0 and line["cpu_baseline"]["kind"] == "port"
    assert line["cpu_baseline"]["cpu_model"] is None or isinstance(line["cpu_baseline"]["cpu_model"], str)
    assert line["e2e"]["h2d_bytes_per_step"] == 0


@pytest.mark.slow
@pytest.mark.parametrize("workload", ["batch-256", "surrogate-128"])
def test_reference_arm_of_the_other_workloads(workload):
    """The reference arm on the batched and surrogate workloads: the batch times the CPU port over
    as many instances as fit its budget; the reference has no surrogate, which the line says."""
    import oracle

    oracle.build()
    cmd = [sys.executable, "bench.py", "--impl", "reference", "--workload", workload, "--reference-budget-s", "2"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    if workload == "surrogate-128":
        assert "unavailable" in line
    else:
        assert line["value"] > 0 and line["cpu_baseline"]["kind"] == "port"
        assert line["e2e"]["d2h_bytes_per_step"] == 0
