"""The multi-rank host logic of bench.py on CPU: two gloo ranks, as torchrun starts them, agree
on the slowest rank's time and the job's total work (the two reductions every N > 1 line uses),
read their rank from the environment, and the reference arm runs on rank 0 only."""
import os
import socket

import pytest

import bench


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    r, w, lr = bench.dist_env()
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        slowest = bench.max_over_ranks(1.5 + rank, w, device="cpu")
        total = bench.sum_over_ranks(1000 * (rank + 1), w, device="cpu")
        out.put((r, w, lr, slowest, total))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_like_the_bench():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get() for _ in range(2))
    assert [g[:3] for g in got] == [(0, 2, 0), (1, 2, 1)]
    assert all(g[3] == 2.5 and g[4] == 3000.0 for g in got)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("LOCAL_RANK", "1")
    import argparse
    ns = argparse.Namespace(seed=0, warmup=1, steps=1, gpus=2)
    assert bench.run_reference_pusch(ns) == 0
    assert capsys.readouterr().out == ""


def test_single_rank_reductions_are_identity():
    assert bench.max_over_ranks(3.25, 1) == 3.25 and bench.sum_over_ranks(7, 1) == 7.0
