"""SLChannelFlow's statistics keys on the GPU (solver.py:510-550 and the
run loop's sampling, solver.py:1424-1436, 1593-1599), against the reference's
own statistics state (tests/golden/stats_state.npz and stats_final.npz, made
by make_stats_golden.py: the reference's TurbulenceStats on three seeded
snapshots of an 8 x 6 x 12 channel with one extra spectra plane, z+ = 30).

- a config with n_stats > 0 builds turbulence_stats; restart_state_file loads
  the reference's state bit for bit, and save_state writes it back unchanged;
- the same three snapshots accumulated on the GPU reproduce the reference's
  state to 1e-12 relative, and continuing from the restored state doubles it;
- run_steps samples every n_stats steps once time >= t_stats, and
  finalize_statistics writes the state and statistics files."""

import os
import sys

import numpy as np
import pytest
import torch

from slchannel_b200.solver import SLChannelFlow
from slchannel_b200.turbstats import PROFILES, SPECTRA, TurbulenceStats

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from make_stats_golden import (EXTRA_PLANES, GAMMA, LX, LY, LZ, N_SNAPSHOTS, NU, NX, NY,  # noqa: E402
                               NZ, RE_TAU)

pytestmark = pytest.mark.gpu
STATE = os.path.join(HERE, "golden", "stats_state.npz")
FINAL = os.path.join(HERE, "golden", "stats_final.npz")
KINDS = ("uu", "vv", "ww", "uw")
TOL = 1e-12


def _config(results, restart=None, n_stats=1, t_stats=0.0):
    stats = {"n_stats": n_stats, "t_stats": t_stats, "spectra_z_planes": list(EXTRA_PLANES),
             "state_file": "state.npz", "output_file": "stats.npz"}
    if restart is not None:
        stats["restart_state_file"] = restart
    return {"grid": {"nx": NX, "ny": NY, "nz": NZ},
            "domain": {"Lx": LX, "Ly": LY, "Lz": LZ},
            "flow": {"Re": 1.0 / NU, "Re_tau": RE_TAU, "U_bulk": 1.0, "gamma": GAMMA},
            "initialization": {"type": "parabolic"}, "time": {"dt": 0.01},
            "compute": {"device": "cuda"}, "output": {"results_folder": str(results)},
            "sl": {"interp_order": 4}, "statistics": stats}


def _snapshots():
    """The generator's three seeded snapshots (make_stats_golden.py)."""
    r = np.random.default_rng(77)
    out = []
    for _ in range(N_SNAPSHOTS):
        u = 1.0 + 0.1 * r.normal(size=(NX + 1, NY + 2, NZ + 2))
        v = 0.1 * r.normal(size=(NX + 2, NY + 1, NZ + 2))
        w = 0.1 * r.normal(size=(NX + 2, NY + 2, NZ + 1))
        out.append(tuple(torch.from_numpy(a).cuda() for a in (u, v, w)))
    return out


def _sums(ts):
    d = {name: getattr(ts, name).detach().cpu().numpy() for name in PROFILES + SPECTRA}
    for pl in ts.extra_planes:
        for k in KINDS:
            d[f"E_{k}_2d_z{pl['zp']:.0f}_sum"] = pl["sums"][k].detach().cpu().numpy()
    return d


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_restart_state_loads_and_saves_the_reference_state(tmp_path):
    flow = SLChannelFlow(config=_config(tmp_path, restart=STATE))
    ts = flow.turbulence_stats
    assert isinstance(ts, TurbulenceStats)
    assert ts.n_samples == N_SNAPSHOTS and ts.n_samples_extra == N_SNAPSHOTS
    ref = np.load(STATE)
    for key, val in _sums(ts).items():
        np.testing.assert_array_equal(val, ref[key], err_msg=key)
    out = tmp_path / "roundtrip.npz"
    ts.save_state(str(out))
    got = np.load(out)
    assert got.files == ref.files
    for key in ref.files:
        np.testing.assert_array_equal(got[key], ref[key], err_msg=key)


def test_accumulation_matches_the_reference_and_continues_a_restart(tmp_path):
    ref = np.load(STATE)
    fresh = SLChannelFlow(config=_config(tmp_path))
    assert fresh.turbulence_stats.n_samples == 0
    snaps = _snapshots()
    for u, v, w in snaps:
        fresh.turbulence_stats.accumulate_statistics(u, v, w, 0.05)
    for key, val in _sums(fresh.turbulence_stats).items():
        assert _rel(val, ref[key]) < TOL, key
    fin, fin_ref = fresh.turbulence_stats.finalize_statistics(), np.load(FINAL)
    for key in ("U_mean", "uu_mean", "vv_mean", "ww_mean", "uw_mean", "E_uu_2d", "E_uw_2d",
                "u_tau"):
        assert _rel(np.asarray(fin[key]), fin_ref[key]) < 1e-11, key
    # continuing the reference's accumulation from its restart state
    cont = SLChannelFlow(config=_config(tmp_path, restart=STATE))
    for u, v, w in snaps:
        cont.turbulence_stats.accumulate_statistics(u, v, w, 0.05)
    assert cont.turbulence_stats.n_samples == 2 * N_SNAPSHOTS
    for key, val in _sums(cont.turbulence_stats).items():
        assert _rel(val, 2.0 * ref[key]) < TOL, key


def test_run_steps_samples_every_n_stats_after_t_stats(tmp_path):
    # dt 0.01, t_stats 0.015: steps 2 and 4 of four are sampled
    flow = SLChannelFlow(config=_config(tmp_path, n_stats=2, t_stats=0.015))
    probe = TurbulenceStats(NX, NY, NZ, LX, LY, LZ, flow.z_c, flow.z_f, flow.dz_c, flow.dz_f,
                            flow.dx, flow.dy, flow.nu, RE_TAU, device=flow.device,
                            spectra_z_planes=list(EXTRA_PLANES))
    for step in range(1, 5):
        flow.run_steps(1)
        if step % 2 == 0:
            probe.accumulate_statistics(flow.u, flow.v, flow.w, None)
    assert flow.turbulence_stats.n_samples == 2
    want = _sums(probe)
    for key, val in _sums(flow.turbulence_stats).items():
        np.testing.assert_array_equal(val, want[key], err_msg=key)
    assert flow.finalize_statistics()
    state = np.load(tmp_path / "state.npz")
    assert int(state["n_samples"]) == 2
    stats = TurbulenceStats.load_statistics(str(tmp_path / "stats.npz"))
    assert int(stats["n_samples"]) == 2
    np.testing.assert_array_equal(stats["U_mean"], probe.finalize_statistics()["U_mean"])


def test_statistics_off_builds_nothing(tmp_path):
    cfg = _config(tmp_path)
    cfg["statistics"]["enabled"] = False
    flow = SLChannelFlow(config=cfg)
    assert flow.turbulence_stats is None
    flow.run_steps(2)
    assert not flow.finalize_statistics()
