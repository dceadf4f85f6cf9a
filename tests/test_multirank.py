"""The multi-rank path of bench.py on the CPU (gloo, two ranks): the job's
time is the slowest rank's, whole-job throughput counts every rank's cells,
and the reference arm runs on rank 0 alone.  Shots are independent (replicas,
no data-path collective), so this reduction is the only exchange."""
import os
import socket
import sys
import tempfile

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    ms = 10.0 + 5.0 * rank                  # rank 1 is the slow one
    job_ms = bench.max_over_ranks(ms, dist, "cpu")
    value = bench.job_gcells(1_000_000, 100, world, job_ms)

    class Args:
        workload, steps, warmup = "a3d", 2, 3
    ref = bench.run_reference_arm(Args(), rank, world) if rank == 1 else "skipped"
    dist.barrier()
    dist.destroy_process_group()
    with open(os.path.join(out_dir, f"r{rank}"), "w") as f:
        f.write(f"{job_ms} {value} {ref is None}\n")


@pytest.mark.timeout(120)
def test_two_rank_reduction_and_rank0_only_reference():
    world = 2
    out = tempfile.mkdtemp()
    mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, join=True,
                       start_method="spawn")
    rows = [open(os.path.join(out, f"r{r}")).read().split() for r in range(world)]
    for r, (job_ms, value, ref_none) in enumerate(rows):
        assert float(job_ms) == 15.0                          # max over ranks
        assert abs(float(value) - 2 * 1e6 * 100 / 15e-3 / 1e9) < 1e-9
    assert rows[1][2] == "True"                               # rank 1 runs no reference
