"""Sharding of an ensemble over ranks (no GPU): the greedy size-balanced
partition, and the report-cadence gather of per-instance diagnostics over a
world_size-2 gloo group, in the style of the reference's emulated
communicator tests (parallel/comm.py:17-78)."""

import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from slchannel_b200.ensemble import ensemble_specs, gather_diagnostics, partition_instances


def test_partition_covers_and_balances():
    specs = ensemble_specs(48, seed=4)
    cost = [s["nx"] * s["ny"] * s["nz"] for s in specs]
    for world in (1, 2, 3, 4, 8):
        parts = partition_instances(specs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(48))
        loads = [sum(cost[i] for i in p) for p in parts]
        # LPT bound: max load <= mean + largest item
        assert max(loads) <= sum(cost) / world + max(cost)
        assert parts == partition_instances(specs, world)


def test_partition_rejects_empty_world():
    with pytest.raises(ValueError):
        partition_instances(ensemble_specs(4), 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        specs = ensemble_specs(12, seed=7)
        mine = partition_instances(specs, world)[rank]
        local = [float(specs[i]["Re"]) for i in mine]  # stand-in per-instance diagnostic
        merged = gather_diagnostics(local, mine, world)
        q.put((rank, mine, merged))
    finally:
        dist.destroy_process_group()


def test_gather_diagnostics_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    specs = ensemble_specs(12, seed=7)
    expect = {i: float(s["Re"]) for i, s in enumerate(specs)}
    mines = {r: m for r, m, _ in res}
    assert sorted(mines[0] + mines[1]) == list(range(12))
    assert not set(mines[0]) & set(mines[1])
    for _, _, merged in res:
        assert merged == expect


class _FakeShard:
    """Stands in for EnsembleShard on the CPU: stepping counts steps (and
    sleeps a rank-dependent time, so the max-over-ranks reduction shows)."""

    def __init__(self, indices, rank):
        self.indices, self.rank, self.steps = list(indices), rank, 0

    def step(self):
        import time

        time.sleep(0.002 * (1 + self.rank))
        self.steps += 1

    def diagnostics(self):
        return [(i, self.steps) for i in self.indices]


class _Wall:
    def start(self):
        import time

        self.t = time.perf_counter()

    def stop(self):
        import time

        return time.perf_counter() - self.t


def _driver_worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from slchannel_b200.ensemble import drive_sharded

        specs = ensemble_specs(12, seed=7)
        wall = _Wall()
        mine, reports, secs = drive_sharded(specs, rank, world, 10, 4,
                                            lambda idx: _FakeShard(idx, rank), lambda: wall,
                                            warmup=2)
        q.put((rank, mine, reports, secs))
    finally:
        dist.destroy_process_group()


def test_sharded_driver_two_ranks():
    """drive_sharded over a world_size-2 gloo group: each rank steps only its
    partition (warm-up untimed), the reports arrive at the cadence (steps 4,
    8 and the last, 10) holding every instance of both ranks with its step
    count, and the returned time is the maximum over the ranks."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_driver_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    specs = ensemble_specs(12, seed=7)
    parts = partition_instances(specs, 2)
    by_rank = {r: (m, rep, s) for r, m, rep, s in res}
    for r in (0, 1):
        assert by_rank[r][0] == parts[r]
    secs = {s for _, _, s in by_rank.values()}
    assert len(secs) == 1  # both ranks hold the same maximum
    assert secs.pop() >= 10 * 0.004  # at least the slower rank's 10 timed steps
    for _, rep, _ in by_rank.values():
        assert sorted(rep) == [4, 8, 10]
        for step, merged in rep.items():
            assert sorted(merged) == list(range(12))
            assert all(v == (i, 2 + step) for i, v in merged.items())
