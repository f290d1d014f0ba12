"""The multi-GPU form is replicas only: every rank proves on its own GPU and the
one collective is the MAX of the timed region.  Two gloo ranks on CPU run the
same aggregation bench.py uses under torchrun, and the reference arm's rank
rule (rank 0 alone runs it)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, times, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    v = bench.replica_ms_per_proof(times[rank], proofs=4, world=world, dist=dist)
    assert bench._dist() == (world, rank, rank)
    out[rank] = v
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_report_the_slowest_rank_over_all_proofs():
    world, port = 2, _free_port()
    times = [40.0, 100.0]   # ms for 4 proofs on each rank
    out = mp.get_context("spawn").Manager().dict()
    mp.start_processes(_rank, args=(world, port, times, out), nprocs=world, start_method="spawn")
    # 8 proofs in 100 ms (the slower rank) = 12.5 ms per proof, seen by every rank
    assert dict(out) == {0: 12.5, 1: 12.5}


def test_single_process_needs_no_collective():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.replica_ms_per_proof(90.0, proofs=3, world=1) == 30.0


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")
    args = type("A", (), {"gpus": 2, "steps": 1, "warmup": 0})()
    bench.run_reference(args)          # rank 1 returns without work or output
    assert capsys.readouterr().out == ""
