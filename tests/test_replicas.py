"""Multi-process path of bench.py (replicas: one independent case per GPU, no
data-path collective) on CPU with the gloo backend, world size 2: every rank
gets the slowest rank's time and the whole-job rate world*steps/max_ms; the
reference arm runs on rank 0 only."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist

    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms, rate = bench.replica_rate(10.0 * (rank + 1), 20, world, "cpu")
        ref = bench.run_reference(type("A", (), {"steps": 1, "warmup": 0})(), rank, world) \
            if rank == 1 else None
        out[rank] = (ms, rate, ref)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_replica_rate_takes_the_slowest_rank():
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        for r in range(2):
            ms, rate, _ = out[r]
            assert ms == pytest.approx(20.0)
            assert rate == pytest.approx(2 * 20 / 0.020)
        assert out[1][2] is None  # the reference arm: rank 0 only


def test_replica_rate_single_process():
    import bench
    ms, rate = bench.replica_rate(5.0, 10, 1)
    assert ms == 5.0 and rate == pytest.approx(2000.0)


def _ensemble_rank(rank, world, port, out):
    import torch.distributed as dist

    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        n = 7
        mine = bench.shard_cases(n, rank, world)
        # per-case scalars that identify the case and the rank that ran it
        local = {i: (float(i * i), float(rank)) for i in mine}
        out[rank] = (mine, bench.gather_case_scalars(local, n, 2, world, "cpu"))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_ensemble_cases_are_sharded_and_gathered():
    """The ensemble's multi-GPU path (whole cases per rank, one gather of the
    per-case scalars) on two gloo ranks: the shards partition the cases and
    every rank ends with all cases' scalars in case order."""
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_ensemble_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        shards = [out[r][0] for r in range(2)]
        assert sorted(shards[0] + shards[1]) == list(range(7))
        assert not set(shards[0]) & set(shards[1])
        for r in range(2):
            got = out[r][1]
            assert [v[0] for v in got] == [float(i * i) for i in range(7)]
            assert [v[1] for v in got] == [float(i % 2) for i in range(7)]


def test_ensemble_gather_single_process():
    import bench
    assert bench.shard_cases(5, 0, 1) == [0, 1, 2, 3, 4]
    got = bench.gather_case_scalars({0: (1.0,), 2: (3.0,)}, 3, 1, 1)
    assert got == [(1.0,), (0.0,), (3.0,)]
