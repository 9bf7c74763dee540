"""The sharded ensemble driver (drive_sharded + EnsembleShard) with real GPU
ensembles: two gloo ranks as processes on one GPU, each stepping only its
partition of a 10-channel ensemble (no collective on the step path, so the
ranks' kernels never wait on one another), the per-instance bulk velocity and
forcing and kinetic energy gathered every 2 steps.  Every instance's
reported values match a
one-rank run of the whole ensemble: an instance's arithmetic does not depend
on which other instances share its launches, except through cuFFT's choice of
kernels for a different batch of same-sized transforms (last-bit
differences), so the bulk velocity is held to 1e-13, the forcing to 1e-9
(it is the bulk correction over dt) and the kinetic energy to 1e-12
relative."""

import os
import socket

import pytest
import torch
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu
N_INST, STEPS, EVERY = 10, 4, 2


def _specs():
    from slchannel_b200.ensemble import ensemble_specs

    return ensemble_specs(N_INST, seed=11, sizes=(32, 48), cfl=1.5)


class _Wall:
    def start(self):
        import time

        self.t = time.perf_counter()

    def stop(self):
        import time

        torch.cuda.synchronize()
        return time.perf_counter() - self.t


def _run(rank, world, port, q):
    import torch.distributed as dist

    from slchannel_b200.ensemble import EnsembleShard, drive_sharded

    torch.cuda.set_device(0)
    if world > 1:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        specs = _specs()
        held = {}

        def make(idx):
            held["s"] = EnsembleShard(specs, idx, order=6, precision="fp64", autotune=False)
            return held["s"]

        wall = _Wall()
        mine, reports, secs = drive_sharded(specs, rank, world, STEPS, EVERY, make, lambda: wall,
                                            warmup=1)
        held["s"].close()
        q.put((rank, mine, reports, secs))
    finally:
        if world > 1:
            dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharded_ensemble_matches_one_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    one = ctx.Process(target=_run, args=(0, 1, 0, q))
    one.start()
    _, mine1, rep1, _ = q.get(timeout=600)
    one.join(timeout=120)
    assert one.exitcode == 0 and mine1 == list(range(N_INST))
    port = _free_port()
    procs = [ctx.Process(target=_run, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=600) for _ in procs]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    parts = {r: m for r, m, _, _ in res}
    assert sorted(parts[0] + parts[1]) == list(range(N_INST)) and parts[0] and parts[1]
    for _, _, rep2, secs in res:
        assert sorted(rep2) == sorted(rep1) == [2, 4] and secs > 0
        for step in rep1:
            assert sorted(rep2[step]) == list(range(N_INST))
            for i, (ub, fo, ke) in rep1[step].items():
                ub2, fo2, ke2 = rep2[step][i]
                assert abs(ub2 - ub) < 1e-13 and abs(fo2 - fo) < 1e-9, (step, i)
                assert abs(ke2 - ke) < 1e-12 * ke, (step, i)
    for ub, _, ke in rep1[STEPS].values():
        assert abs(ub - 1.0) < 1e-12 and ke > 0
