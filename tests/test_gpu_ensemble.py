"""The ensemble form (many channels, one launch per substep, CUDA graph)
against the same channels stepped one by one with the single-channel solver.

Per instance the ensemble kernels do the single-channel step's arithmetic,
and the FFTs of instances sharing (nx, ny) are batched into one cuFFT call;
the instance trajectories must agree with the loop to 1e-13 relative (the
run records the exact maximum), bulk velocities and clamp counts included,
whatever the tile shapes, with and without the graph."""

import math

import pytest
import torch

from slchannel_b200.ensemble import ChannelEnsemble, ensemble_specs, loop_step, make_flow

pytestmark = pytest.mark.gpu

SPECS = [
    {"nx": 32, "ny": 48, "nz": 32, "gamma": 1.7, "Re": 2300.0},
    {"nx": 48, "ny": 32, "nz": 64, "gamma": 2.1, "Re": 4100.0},
    {"nx": 32, "ny": 48, "nz": 48, "gamma": 1.9, "Re": 3000.0},   # shares (nx, ny) with #0
    {"nx": 64, "ny": 32, "nz": 96, "gamma": 2.2, "Re": 4900.0},
    {"nx": 32, "ny": 32, "nz": 33, "gamma": 1.6, "Re": 2000.0},   # odd nz
]


def _specs():
    out = []
    for i, s in enumerate(SPECS):
        d = dict(s, Lx=2 * math.pi, Ly=math.pi, Lz=2.0, seed=100 + i, cfl=3.0, urms=0.1)
        out.append(d)
    return out


def _bootstrapped(specs, precision="fp64"):
    flows, dts = [], []
    for s in specs:
        f, dt = make_flow(s, order=6, precision=precision)
        f.step_sl_bdf2(dt)  # BDF1 bootstrap
        flows.append(f)
        dts.append(dt)
    return flows, dts


def _rel(a, b):
    return ((a - b).abs().max() / b.abs().max()).item()


@pytest.mark.parametrize("use_graph,precision", [(True, "fp64"), (False, "fp64"), (True, "mixed")])
def test_ensemble_matches_single_channel_loop(use_graph, precision):
    specs = _specs()
    ref, dts = _bootstrapped(specs, precision)
    mine, dts2 = _bootstrapped(specs, precision)
    assert dts == dts2
    ens = ChannelEnsemble(mine, dts, use_graph=use_graph, autotune=False)
    worst = 0.0
    for step in range(4):  # phases 0, 1, 2, 0: every captured graph and its reuse
        loop_step(ref, dts)
        ens.step()
        torch.cuda.synchronize()
        for i, f in enumerate(ref):
            for c, a, b in zip("uvw", ens.velocity(i), (f.u, f.v, f.w)):
                e = _rel(a, b)
                worst = max(worst, e)
                assert e <= 1e-13, (step, i, c, e)
            ub, fc = ens.bulk(i)
            assert abs(float(ub) - 1.0) < 1e-12
            assert abs(float(fc) - float(f.forcing)) <= 1e-12 * max(1.0, abs(float(f.forcing)))
            assert int(ens.nclamp[i]) == int(f.sl.n_clamped_last)
            assert _rel(ens.p[i], f.p) <= 1e-12
    print(f"ensemble vs loop ({precision}): max relative difference {worst:.3e}")


@pytest.mark.parametrize("trajs", [(4, 4, 4, 4, 4), (2, 4, 2, 4, 2)])
def test_ensemble_mixed_tricubic_trajectories(trajs):
    """The mixed form with tricubic trajectory sampling: every instance at
    traj_interp_order 4 (one instantiation), and a mixture of 2 and 4 (read
    per instance), against the loop over the same single-channel solvers."""
    specs = [dict(s, traj_order=t) for s, t in zip(_specs(), trajs)]
    ref, dts = _bootstrapped(specs, "mixed")
    mine, _ = _bootstrapped(specs, "mixed")
    ens = ChannelEnsemble(mine, dts, use_graph=True, autotune=False)
    worst = 0.0
    for step in range(3):
        loop_step(ref, dts)
        ens.step()
        torch.cuda.synchronize()
        for i, f in enumerate(ref):
            for c, a, b in zip("uvw", ens.velocity(i), (f.u, f.v, f.w)):
                worst = max(worst, _rel(a, b))
    print(f"tricubic mixed ensemble vs loop {trajs}: max relative difference {worst:.3e}")
    assert worst <= 1e-13


def test_ensemble_refuses_incremental_pressure():
    spec = _specs()[0]
    f, dt = make_flow(spec, order=6)
    f.sl_bdf2_pressure = "inc"
    f.step_sl_bdf2(dt)
    with pytest.raises(ValueError, match="noninc"):
        ChannelEnsemble([f], [dt], use_graph=False, autotune=False)


def test_ensemble_tiles_do_not_change_results():
    specs = _specs()
    a_flows, dts = _bootstrapped(specs)
    b_flows, _ = _bootstrapped(specs)
    a = ChannelEnsemble(a_flows, dts, autotune=False)
    b = ChannelEnsemble(b_flows, dts, autotune=False)
    b.set_tiles([32, 128, 64, 128, 32])
    assert b.tiles == [32, 128, 64, 128, 32]
    for _ in range(3):
        a.step()
        b.step()
    torch.cuda.synchronize()
    for i in range(len(specs)):
        for x, y in zip(a.velocity(i), b.velocity(i)):
            assert torch.equal(x, y)


def test_autotuner_picks_a_candidate_per_shape():
    specs = _specs()
    flows, dts = _bootstrapped(specs)
    ens = ChannelEnsemble(flows, dts, autotune=True, autotune_reps=2)
    assert set(ens.tiles) <= {32, 64, 128}
    for shape, (tk, ms) in ens.tune_ms.items():
        assert tk in (32, 64, 128)
        assert all(t > 0 for t in ms)
        assert tk == (32, 64, 128)[min(range(3), key=lambda c: ms[c])]
    ens.run(2)
    torch.cuda.synchronize()
    for i in range(len(specs)):
        assert torch.isfinite(ens.velocity(i)[0]).all()


def test_ensemble_specs_recipe():
    specs = ensemble_specs(48, seed=4)
    assert len(specs) == 48
    for s in specs:
        assert s["nx"] in (32, 48, 64, 96, 128) and s["nz"] in (32, 48, 64, 96, 128)
        assert 1.6 <= s["gamma"] <= 2.2 and 2000.0 <= s["Re"] <= 5000.0
    assert specs == ensemble_specs(48, seed=4)


def test_ensemble_rejects_mixed_precisions():
    specs = _specs()[:2]
    f0, d0 = make_flow(specs[0], order=6)
    f1, d1 = make_flow(specs[1], order=6, precision="mixed")
    f0.step_sl_bdf2(d0)
    f1.step_sl_bdf2(d1)
    with pytest.raises(ValueError):
        ChannelEnsemble([f0, f1], [d0, d1])


def test_ensemble_rejects_mixed_orders():
    specs = _specs()[:2]
    f0, d0 = make_flow(specs[0], order=6)
    f1, d1 = make_flow(specs[1], order=4)
    f0.step_sl_bdf2(d0)
    f1.step_sl_bdf2(d1)
    with pytest.raises(ValueError):
        ChannelEnsemble([f0, f1], [d0, d1])
