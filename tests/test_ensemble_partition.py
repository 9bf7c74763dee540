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
