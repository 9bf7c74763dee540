"""SLChannelFlow.run_steps as the reference's run loop drives the step
(solver.py:1330-1436): the adaptive dt of time.dt_update_interval and
CFL_target (compute_cfl_dt, solver.py:652-674) -- checked against the
formula evaluated on the state before each adapting step -- and the BDF1
re-bootstrap that a dt change triggers (solver.py:834-844)."""

import math

import pytest
import torch

from slchannel_b200.solver import SLChannelFlow
from slchannel_b200.utils import compute_cfl_fused

pytestmark = pytest.mark.gpu


def _config(interval, cfl, dt=0.01, dt_max=0.05):
    return {"grid": {"nx": 16, "ny": 12, "nz": 20},
            "domain": {"Lx": 2 * math.pi, "Ly": math.pi, "Lz": 2.0},
            "flow": {"Re": 2800.0, "Re_tau": 180.0, "U_bulk": 1.0, "gamma": 2.0},
            "initialization": {"type": "vortices", "perturbation_intensity": 0.1, "n_vortices": 2},
            "time": {"dt": dt, "dt_update_interval": interval, "CFL_target": cfl,
                     "dt_max": dt_max, "dt_min": 1e-4},
            "compute": {"device": "cuda"},
            "sl": {"interp_order": 6}}


def _formula(flow):
    dti = compute_cfl_fused(flow.u, flow.v, flow.w, flow.nx, flow.ny, flow.nz, flow.dx, flow.dy,
                            flow.dz_f, flow.dz_c)
    dt = flow.cfl_target / (dti if dti >= 1e-10 else 1.0)
    dt = min(dt, flow.diff_stability_C / (flow.nu * (1.0 / flow.dx**2 + 1.0 / flow.dy**2)))
    return min(max(dt, flow.dt_min), flow.dt_max)


def test_adaptive_dt_follows_the_reference_loop():
    flow = SLChannelFlow(config=_config(interval=2, cfl=0.5))
    seen = []
    for step in range(1, 7):
        if step % 2 == 0:
            want = _formula(flow)
            expect = want if abs(want - flow.dt) / flow.dt > 0.05 else flow.dt
        else:
            expect = flow.dt
        flow.run_steps(1)
        assert flow.current_step == step
        assert flow._dt_prev_step == pytest.approx(expect, rel=1e-15)
        assert flow.dt == pytest.approx(expect, rel=1e-15)
        seen.append(flow.dt)
    assert seen[1] != 0.01  # the first adaptation changed dt
    assert flow.time == pytest.approx(sum(seen), rel=1e-14)
    assert torch.isfinite(flow.u).all()


def test_fixed_dt_argument_and_no_adaptation():
    flow = SLChannelFlow(config=_config(interval=0, cfl=None))
    flow.run_steps(3)
    assert flow.dt == 0.01 and flow._dt_prev_step == 0.01 and flow.current_step == 3
    flow2 = SLChannelFlow(config=_config(interval=1, cfl=0.5))
    flow2.run_steps(2, dt=0.02)  # an explicit dt is used as given
    assert flow2._dt_prev_step == 0.02 and flow2.dt == 0.01
