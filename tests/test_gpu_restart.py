"""Restart continuity (the reference's tests/test_restart_sl.py restated):
10 steps, checkpoint with save_flow_fields, restart from the file with a new
SLChannelFlow (BDF1 re-bootstrap, forcing restored from the file), 10 more
steps: within 1e-4 of 20 uninterrupted steps (not bit-exact by design), and
the step / time counters continue from the checkpoint."""

import os

import pytest

from slchannel_b200.solver import SLChannelFlow
from slchannel_b200.utils import save_flow_fields

pytestmark = pytest.mark.gpu
DT = 0.01


def _cfg(tmp, field_file=None):
    init = {"type": "vortices", "perturbation_intensity": 0.08}
    if field_file:
        init["field_file"] = field_file
    return {"grid": {"nx": 16, "ny": 16, "nz": 32},
            "domain": {"Lx": 6.283185307179586, "Ly": 3.141592653589793, "Lz": 2.0},
            "flow": {"Re": 1000.0, "Re_tau": 180.0, "U_bulk": 1.0, "gamma": 1.5},
            "initialization": init, "time": {"dt": DT},
            "compute": {"device": "cuda"}, "output": {"results_folder": str(tmp)},
            "sl": {"interp_order": 4, "n_traj_iters": 2}}


def test_restart_matches_uninterrupted(tmp_path):
    ref = SLChannelFlow(config=_cfg(tmp_path))
    ref.run_steps(20, DT)
    s1 = SLChannelFlow(config=_cfg(tmp_path))
    s1.run_steps(10, DT)
    save_flow_fields(s1.u, s1.v, s1.w, s1.p, s1.z_c, s1.z_f, s1.Lx, s1.Ly, 10, 10 * DT, 0.05,
                     s1.forcing, str(tmp_path), "fields_ckpt.npz")
    s2 = SLChannelFlow(config=_cfg(tmp_path, os.path.join(tmp_path, "fields_ckpt.npz")))
    assert s2.initial_step == 10 and abs(s2.initial_time - 10 * DT) < 1e-12
    assert abs(s2.forcing - float(s1.forcing)) < 1e-15
    s2.run_steps(10, DT)
    umax = ref.u.abs().max().item()
    rel = max((a - b).abs().max().item() for a, b in [(ref.u, s2.u), (ref.v, s2.v), (ref.w, s2.w)]) / umax
    print(f"restart vs uninterrupted: rel {rel:.2e}")
    assert rel < 1e-4
    assert s2.current_step == 20
