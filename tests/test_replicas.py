"""The bench's multi-GPU mode is replicas: every rank re-depths its own frames, with no collective on the data
path; the job's time is the slowest rank's, taken with one all-reduce MAX. These tests run that plumbing as
two gloo ranks on the CPU (the rendezvous on 127.0.0.1)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, init_method=f"tcp://127.0.0.1:{port}")
    try:
        w, r, local = bench.dist_setup()
        slowest = bench.max_over_ranks(10.0 + 5.0 * r, w, "cpu")  # rank 1 is the slow one
        q.put((r, w, local, slowest, bench.replica_seed0(r)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_time_the_slowest_and_render_disjoint_frames():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=5) for _ in range(world))
    assert [g[0] for g in got] == [0, 1] and all(g[1] == 2 and g[2] == g[0] for g in got)
    assert all(g[3] == 15.0 for g in got)              # every rank reports the job's slowest time
    seeds = [g[4] for g in got]
    assert len(set(seeds)) == 2                       # replicas render different scenes
    assert abs(seeds[1] - seeds[0]) >= 16             # ... with no overlap for the default 16 frames per step


def test_single_process_needs_no_process_group():
    import bench
    assert bench.max_over_ranks(3.5, 1, "cpu") == 3.5


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    import argparse

    import bench
    args = argparse.Namespace(gpus=2, steps=1, warmup=0, reference_budget=1.0)
    assert bench.run_reference(args, 2, 1) == 0       # rank 1: no work, no output
    assert capsys.readouterr().out == ""
