"""The multi-GPU path of bench.py, on the CPU with two gloo ranks.

A circuit does not shard, so `bench.py --gpus N` runs one replica per rank
(weak scaling); the only collective is the max over ranks of the timed
region, and the reference arm runs on rank 0 alone."""
import os
import socket
import sys

import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench

    dev_ms, wall = bench.aggregate_ranks(dist, "cpu", 100.0 + 50.0 * rank, 1.0 + rank)
    out[rank] = (dev_ms, wall)
    dist.barrier()
    dist.destroy_process_group()


def test_timing_is_the_max_over_two_gloo_ranks():
    world = 2
    with mp.Manager() as man:
        out = man.dict()
        mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
        got = dict(out)
    assert got == {0: (150.0, 2.0), 1: (150.0, 2.0)}


def test_single_rank_keeps_its_own_times():
    import bench

    assert bench.aggregate_ranks(None, "cpu", 12.5, 0.5) == (12.5, 0.5)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    import bench

    monkeypatch.setenv("RANK", "1")
    args = bench.argparse.Namespace(workload="config0", reference_budget=0.1, warmup=0, steps=1, gpus=2)
    bench.run_reference(args)
    assert capsys.readouterr().out == ""
