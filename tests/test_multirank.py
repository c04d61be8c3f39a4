"""Replicas across ranks (the stepper does not shard): the bench's job time is
the slowest rank's and its rate counts every rank's steps.  Two gloo ranks
on the CPU, rendezvous on 127.0.0.1."""

import os
import socket
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        ms = 10.0 + 5.0 * rank                      # rank 1 is the slow replica
        m = bench.max_over_ranks(ms, True, "cpu")
        out[rank] = (m, bench.job_rate(20, world, m))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_replicas_time_is_slowest_rank():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0] == res[1]
    m, rate = res[0]
    assert m == 15.0
    assert rate == pytest.approx(2 * 20 / 0.015)


def test_single_process_passes_value_through():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, False, "cpu") == 3.5
    assert bench.job_rate(10, 1, 500.0) == pytest.approx(20.0)


def test_batched_instances_split_over_ranks():
    """The batched form's instances split over ranks: every instance on
    exactly one rank, node counts balanced to within the largest instance."""
    sys.path.insert(0, ROOT)
    import bench
    devs, _, _ = bench.batched_workload()
    sizes = [d.params.n_interior for d in devs]
    for world in (2, 4, 8):
        shards = [bench.batched_shard(sizes, r, world) for r in range(world)]
        assert sorted(i for s in shards for i in s) == list(range(len(sizes)))
        loads = [sum(sizes[i] for i in s) for s in shards]
        assert max(loads) - min(loads) <= max(sizes)
