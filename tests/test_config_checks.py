"""SLChannelFlow's YAML checks (solver.py:172-282), on CPU: a bad key raises
the reference's ValueError, with its message, before any device work; a valid
config asking for the CPU device refuses with RuntimeError (no CPU path)."""

import copy

import pytest

from slchannel_b200.solver import SLChannelFlow

BASE = {
    "grid": {"nx": 16, "ny": 16, "nz": 16},
    "domain": {"Lx": 6.283185307179586, "Ly": 3.141592653589793, "Lz": 2.0,
               "stretching_type": "symmetric"},
    "flow": {"Re": 2800.0, "Re_tau": 180.0, "U_bulk": 1.0, "gamma": 2.0},
    "boundary_conditions": {"top_wall": {"type": "dirichlet"}},
    "time": {"dt": 0.01},
    "sl": {"interp_order": 6, "traj_interp_order": 2, "n_traj_iters": 2,
           "interp_dtype": "fp64", "bdf2_pressure": "noninc", "bdf2_xy_rhs": "extrap"},
    "compute": {"device": "cpu"},
}


def _with(path, value):
    cfg = copy.deepcopy(BASE)
    d = cfg
    for k in path[:-1]:
        d = d.setdefault(k, {})
    d[path[-1]] = value
    return cfg


@pytest.mark.parametrize("path, value, msg", [
    (("domain", "stretching_type"), "top",
     r"Invalid stretching type: top\. slChannel supports 'symmetric' or 'bottom'"),
    (("boundary_conditions", "top_wall", "type"), "robin", r"Invalid top wall BC type: robin"),
    (("advection", "scheme"), "spectral", r"advection\.scheme must be 'sl' or 'eulerian', got spectral"),
    (("sl", "interp_order"), 8, r"sl\.interp_order must be 4 \(tricubic\) or 6 \(triquintic\), got 8"),
    (("sl", "bdf2_pressure"), "rotational", r"sl\.bdf2_pressure must be 'noninc' or 'inc', got rotational"),
    (("sl", "bdf2_xy_rhs"), "implicit", r"sl\.bdf2_xy_rhs must be 'extrap' or 'lagged', got implicit"),
    (("sl", "time_scheme"), "bdf1", r"sl\.time_scheme was removed in the bdf2-only cleanup"),
    (("sl", "traj_extrapolation"), True, r"sl\.traj_extrapolation was removed"),
    (("sl", "field_interp"), "cubic", r"sl\.field_interp was removed"),
    (("solver", "type"), "multigrid", r"solver\.type must be 'fft', got 'multigrid'"),
])
def test_bad_config_keys_raise_the_reference_message(path, value, msg):
    with pytest.raises(ValueError, match=msg):
        SLChannelFlow(config=_with(path, value), allocate_fields=False)


def test_missing_re_tau_raises_key_error():
    # solver.py:210 reads config['flow']['Re_tau'] without a default; it sets
    # the statistics' nominal u_tau and spectra planes, so it stays required
    cfg = copy.deepcopy(BASE)
    del cfg["flow"]["Re_tau"]
    with pytest.raises(KeyError, match="Re_tau"):
        SLChannelFlow(config=cfg, allocate_fields=False)


def test_adaptive_dt_needs_cfl_target():
    # solver.py:222 reads time.CFL_target; here it is required only when
    # time.dt_update_interval asks for the adaptive dt (solver.py:652-674)
    cfg = copy.deepcopy(BASE)
    cfg["time"]["dt_update_interval"] = 10
    with pytest.raises(KeyError, match="CFL_target"):
        SLChannelFlow(config=cfg, allocate_fields=False)
    cfg["time"]["CFL_target"] = 3.0
    with pytest.raises(RuntimeError, match="no CPU path"):
        SLChannelFlow(config=cfg, allocate_fields=False)


def test_valid_config_on_the_cpu_device_refuses_without_fallback():
    with pytest.raises(RuntimeError, match="no CPU path"):
        SLChannelFlow(config=copy.deepcopy(BASE), allocate_fields=False)


@pytest.mark.parametrize("path, value", [
    (("domain", "stretching_type"), "bottom"),
    (("boundary_conditions", "top_wall", "type"), "neumann"),
    (("advection", "scheme"), "eulerian"),
    (("sl", "interp_order"), 4),
    (("sl", "bdf2_pressure"), "inc"),
    (("sl", "bdf2_xy_rhs"), "lagged"),
])
def test_every_accepted_value_passes_the_checks(path, value):
    # accepted by the checks, then refused only for the CPU device
    with pytest.raises(RuntimeError, match="no CPU path"):
        SLChannelFlow(config=_with(path, value), allocate_fields=False)


@pytest.mark.parametrize("stats, n_stats, t_stats", [
    (None, 0, 10.0),
    ({"n_stats": 5}, 5, 10.0),
    ({"n_stats": 5, "t_stats": 2.5}, 5, 2.5),
    ({"n_stats": 5, "enabled": False}, 0, 10.0),
    ({"enabled": True}, 0, 10.0),
])
def test_statistics_keys(stats, n_stats, t_stats):
    # solver.py:510-514: `enabled` is an off switch and n_stats 0 disables;
    # the keys are read before the device, so they can be inspected here
    cfg = copy.deepcopy(BASE)
    if stats is not None:
        cfg["statistics"] = stats
    flow = SLChannelFlow.__new__(SLChannelFlow)
    with pytest.raises(RuntimeError, match="no CPU path"):
        flow.__init__(config=cfg, allocate_fields=False)
    assert flow.n_stats == n_stats and flow.t_stats == t_stats
