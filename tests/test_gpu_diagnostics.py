"""On-device diagnostics and statistics against the reference's own
functions on seeded fields (tests/golden/diagnostics.npz, made by
make_diag_golden.py): max|div|, u_tau (no-slip and free-slip tops), the CFL
inverse of compute_cfl_fused, the bulk velocity, and TurbulenceStats over two
snapshots (profiles, time-mean moments, spectra at the z+ = 15 and z+ = 30
planes, finalize_statistics).  Tolerance 1e-12 relative to each quantity's
scale (the reductions run in another order than torch's)."""

import math
import os
import sys

import numpy as np
import pytest
import torch

from slchannel_b200.solver import SLChannelFlow
from slchannel_b200.turbstats import TurbulenceStats
from slchannel_b200.utils import compute_cfl_fused, compute_u_tau

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_diag_golden as G  # noqa: E402

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope="module")
def setup():
    g = np.load(os.path.join(HERE, "golden", "diagnostics.npz"))
    c = G.CASE
    cfg = {"grid": {"nx": c["nx"], "ny": c["ny"], "nz": c["nz"]},
           "domain": {"Lx": c["Lx"], "Ly": c["Ly"], "Lz": c["Lz"]},
           "flow": {"Re": 1.0 / c["nu"], "Re_tau": 180.0, "U_bulk": 1.0, "gamma": c["gamma"]},
           "initialization": {"type": "parabolic"}, "compute": {"device": "cuda"},
           "sl": {"interp_order": 4}}
    flow = SLChannelFlow(config=cfg)
    assert np.abs(flow.z_f.cpu().numpy() - g["z_f"]).max() < 1e-15
    snaps = []
    for seed in c["seeds"]:
        flow.set_state(*(torch.from_numpy(a) for a in G.snapshot(g["z_f"], g["z_c"], seed)))
        flow.apply_bc_uvw()
        snaps.append(tuple(t.clone() for t in (flow.u, flow.v, flow.w)))
    return g, flow, snaps


def test_diagnostics_match_reference(setup):
    g, flow, snaps = setup
    flow.set_state(*snaps[0])
    d = flow.diagnostics().cpu().numpy()
    assert _rel(d[0], g["max_div"]) < TOL
    assert _rel(d[1], g["u_tau_dirichlet"]) < TOL
    assert _rel(d[2], g["cfl_dti"]) < TOL
    assert _rel(d[3], g["u_bulk"]) < TOL
    u, v, w = snaps[0]
    assert _rel(float(compute_u_tau(u, flow.z_c, flow.nu, "dirichlet")), g["u_tau_dirichlet"]) < TOL
    assert _rel(float(compute_u_tau(u, flow.z_c, flow.nu, "neumann")), g["u_tau_neumann"]) < TOL
    cfl = compute_cfl_fused(u, v, w, flow.nx, flow.ny, flow.nz, flow.dx, flow.dy, flow.dz_f, flow.dz_c)
    assert _rel(cfl, g["cfl_dti"]) < TOL
    again = flow.diagnostics()
    assert torch.equal(again, flow.diagnostics())  # fixed-order reductions


def test_turbulence_stats_match_reference(setup):
    g, flow, snaps = setup
    c = G.CASE
    st = TurbulenceStats(flow.nx, flow.ny, flow.nz, flow.Lx, flow.Ly, flow.Lz, flow.z_c, flow.z_f,
                         flow.dz_c, flow.dz_f, flow.dx, flow.dy, flow.nu, c["Re_tau"],
                         z_plus_target=c["zplus"], device=flow.device, spectra_z_planes=list(c["extra"]))
    assert (st.k_bot, st.k_top) == (int(g["k_bot"]), int(g["k_top"]))
    for u, v, w in snaps:
        st.accumulate_statistics(u, v, w, 0.05)
    for k in ("U_sum", "uu_sum", "vv_sum", "ww_sum", "uw_sum", "Vm_sum", "Wm_sum", "Um2_sum",
              "Vm2_sum", "Wm2_sum", "UmWm_sum", "E_uu_2d_sum", "E_vv_2d_sum", "E_ww_2d_sum",
              "E_uw_2d_sum"):
        assert _rel(getattr(st, k).cpu().numpy(), g[k]) < TOL, k
    for pl in st.extra_planes:
        for k, t in pl["sums"].items():
            assert _rel(t.cpu().numpy(), g[f"extra_{pl['zp']:.0f}_{k}"]) < TOL, k
    fin = st.finalize_statistics()
    for k in ("U_mean", "uu_mean", "vv_mean", "ww_mean", "uw_mean", "E_uu_2d", "E_uw_2d", "u_tau"):
        assert _rel(fin[k], g[f"fin_{k}"]) < 1e-11, k
