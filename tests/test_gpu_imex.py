"""The Eulerian IMEX scheme on the GPU (slc_imex_rhs, slc_step_imex through
SLChannelFlow.step_imex) against the reference's own right-hand side and
four steps (tests/golden/imex_*.npz, make_imex_golden.py): no-slip symmetric
and free-slip bottom-stretched channels."""

import numpy as np
import pytest
import torch
from helpers import rel_err

from slchannel_b200 import _native as N
from slchannel_b200.solver import SLChannelFlow

pytestmark = pytest.mark.gpu


def _load(name):
    import os

    return np.load(os.path.join(os.path.dirname(__file__), "golden", f"imex_{name}.npz"))


@pytest.mark.parametrize("name", ["sym", "bottom_neumann"])
def test_imex_matches_reference(name):
    s = _load(name)
    nx, ny, nz, Lx, Ly, Lz, gamma, Re, dt = s["params"]
    cfg = {"grid": {"nx": int(nx), "ny": int(ny), "nz": int(nz)},
           "domain": {"Lx": float(Lx), "Ly": float(Ly), "Lz": float(Lz),
                      "stretching_type": str(s["stretching"])},
           "flow": {"Re": float(Re), "Re_tau": 180.0, "U_bulk": 1.0, "gamma": float(gamma)},
           "boundary_conditions": {"top_wall": {"type": str(s["top"])}},
           "advection": {"scheme": "eulerian"}, "time": {"dt": float(dt)},
           "compute": {"device": "cuda"}}
    flow = SLChannelFlow(config=cfg)
    assert np.abs(flow.z_f.cpu().numpy() - s["z_f"]).max() < 1e-15
    flow.set_state(*(torch.from_numpy(s[f"init_{c}"]) for c in "uvwp"))
    outs = [torch.zeros_like(t) for t in (flow.u, flow.v, flow.w)]
    flow._grid.call("slc_imex_rhs", N.ptr(flow.u), N.ptr(flow.v), N.ptr(flow.w),
                    *[N.ptr(t) for t in outs], N.stream_of(flow.u))
    for c, t in zip("uvw", outs):
        assert rel_err(t.cpu().numpy(), s[f"rhs_{c}"]) < 1e-13, c
    for step in range(1, 5):
        ub, forcing = flow.step_imex(float(dt))
        for c in "uvw":
            assert rel_err(getattr(flow, c).cpu().numpy(), s[f"s{step}_{c}"]) < 1e-12, (step, c)
        assert rel_err(flow.p.cpu().numpy(), s[f"s{step}_p"]) < 1e-11
        assert abs(float(ub) - float(s[f"s{step}_ubulk"])) < 1e-13
        assert abs(float(forcing) - float(s[f"s{step}_forcing"])) < 1e-10
