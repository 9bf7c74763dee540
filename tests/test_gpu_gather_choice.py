"""The FP64 order-6 step's choice between its TMA-staged and its L1 gather.

The step gathers from staged boxes while at least 90 % of the blocks staged
both feet, reading the counters of an earlier call back without
synchronising, and otherwise through L1, trying the staged gather again
every 50 calls.  Where the feet spread wider than a box (large dt on a
coarse grid) the staged counters stop growing after the first call, and come
back for one probe call later; the two gathers give the same results, so the
step's output does not depend on the choice (checked against the L1 entry
point on the same state)."""

import ctypes
import math

import pytest
import torch

from slchannel_b200 import _native as N
from slchannel_b200.fields import synthetic_channel_field
from slchannel_b200.solver import SLChannelFlow
from slchannel_b200.utils import compute_bulk_velocity

pytestmark = pytest.mark.gpu


def _flow(n3, dt, urms):
    nx, ny, nz = n3
    cfg = {"grid": {"nx": nx, "ny": ny, "nz": nz},
           "domain": {"Lx": 2 * math.pi, "Ly": math.pi, "Lz": 2.0},
           "flow": {"Re": 2800.0, "Re_tau": 180.0, "U_bulk": 1.0, "gamma": 2.0},
           "initialization": {"type": "parabolic"}, "time": {"dt": dt},
           "compute": {"device": "cuda"},
           "sl": {"interp_order": 6, "n_traj_iters": 2, "interp_dtype": "fp64"}}
    f = SLChannelFlow(config=cfg)
    u, v, w = synthetic_channel_field(nx, ny, nz, 2 * math.pi, math.pi, 2.0, f.z_f.cpu().numpy(),
                                      f.z_c.cpu().numpy(), urms=urms, seed=3)
    f.set_state(*(torch.from_numpy(a) for a in (u, v, w)))
    f.apply_bc_uvw()
    f.u *= 1.0 / float(compute_bulk_velocity(f.u, f.cell_vol_ratio, f.total_volume))
    f._save_and_project_initial()
    f.step_sl_bdf2(dt)  # bootstrap
    return f


def _stats(f):
    s = (ctypes.c_int64 * 4)()
    N.check(N.lib().slc_gather_stats(f._grid.handle, s, 0), f._grid.handle)
    return list(s)


def test_step_leaves_the_staged_gather_where_feet_spread():
    dt = 0.6
    f = _flow((24, 16, 48), dt, 0.35)
    s0 = _stats(f)
    blocks = []
    for _ in range(55):
        f.step_sl_bdf2(dt)
        torch.cuda.synchronize()
        blocks.append(_stats(f)[1] - s0[1])
    first = blocks[0]
    st = _stats(f)
    assert first > 0 and st[0] == 0, (blocks[:3], st)
    # after the first call the step gathers through L1 ...
    assert blocks[1] == first and blocks[10] == first, blocks[:12]
    # ... and probes the staged gather once more within the next 50 calls
    assert blocks[-1] > first, blocks


def test_step_output_equals_the_l1_gather_either_way():
    dt = 0.6
    f = _flow((24, 16, 48), dt, 0.35)
    for _ in range(3):
        f.step_sl_bdf2(dt)
    cur, prev = (f.u, f.v, f.w), (f.u_nm1, f.v_nm1, f.w_nm1)
    out = []
    for name in ("slc_trace_gather_bdf2", "slc_trace_gather_bdf2_staged"):
        o = [torch.zeros_like(t) for t in cur]
        ncl = torch.zeros((), dtype=torch.int64, device=f.device)
        f._grid.call(name, *[N.ptr(t) for t in cur], *[N.ptr(t) for t in prev], float(dt),
                     *[N.ptr(t) for t in o], N.ptr(ncl), N.stream_of(f.u))
        out.append(o)
    torch.cuda.synchronize()
    for a, b in zip(*out):
        assert torch.equal(a, b)
