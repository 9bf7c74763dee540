"""The mixed form's TMA-staged trace+gather (slc_trace_gather_bdf2_staged on a
mixed-precision handle: FP32 fluctuation boxes staged in shared memory)
against its L1 gather (slc_trace_gather_bdf2): equal clamp counts and equal
outputs with every box staged, with blocks falling back to L1 (wide feet),
at both orders and both trajectory orders; and the mixed step (which gathers
from staged boxes) against the FP64 step.

The staged and the L1 kernels share the per-point arithmetic in separately
compiled kernels, so ptxas could fuse the FP32 trajectory's multiplies and
adds into FMAs differently; the bound allows for the FP32 trace's round-off
(1e-6 relative), although the outputs measured equal bit for bit, clamp
counts included."""

import ctypes
import math

import pytest
import torch

from slchannel_b200 import _native as N
from slchannel_b200.fields import synthetic_channel_field
from slchannel_b200.solver import SLChannelFlow
from slchannel_b200.utils import compute_bulk_velocity

pytestmark = pytest.mark.gpu


def _flow(n3, dt, urms, order=6, traj=2, precision="mixed"):
    nx, ny, nz = n3
    cfg = {"grid": {"nx": nx, "ny": ny, "nz": nz},
           "domain": {"Lx": 2 * math.pi, "Ly": math.pi, "Lz": 2.0},
           "flow": {"Re": 2800.0, "Re_tau": 180.0, "U_bulk": 1.0, "gamma": 2.0},
           "initialization": {"type": "parabolic"}, "time": {"dt": dt},
           "compute": {"device": "cuda"},
           "sl": {"interp_order": order, "n_traj_iters": 2, "interp_dtype": precision,
                  "traj_interp_order": traj}}
    f = SLChannelFlow(config=cfg)
    u, v, w = synthetic_channel_field(nx, ny, nz, 2 * math.pi, math.pi, 2.0, f.z_f.cpu().numpy(),
                                      f.z_c.cpu().numpy(), urms=urms, seed=5)
    f.set_state(*(torch.from_numpy(a) for a in (u, v, w)))
    f.apply_bc_uvw()
    f.u *= 1.0 / float(compute_bulk_velocity(f.u, f.cell_vol_ratio, f.total_volume))
    f._save_and_project_initial()
    for _ in range(2):
        f.step_sl_bdf2(dt)
    return f


def _both(f, dt):
    cur, prev = (f.u, f.v, f.w), (f.u_nm1, f.v_nm1, f.w_nm1)
    stats = (ctypes.c_int64 * 4)()
    N.lib().slc_gather_stats(f._grid.handle, stats, 1)
    res = []
    for name in ("slc_trace_gather_bdf2", "slc_trace_gather_bdf2_staged"):
        out = [torch.zeros_like(t) for t in cur]
        ncl = torch.zeros((), dtype=torch.int64, device=f.device)
        f._grid.call(name, *[N.ptr(t) for t in cur], *[N.ptr(t) for t in prev], float(dt),
                     *[N.ptr(t) for t in out], N.ptr(ncl), N.stream_of(f.u))
        res.append((out, int(ncl)))
    torch.cuda.synchronize()
    N.lib().slc_gather_stats(f._grid.handle, stats, 1)
    return res, list(stats)


def _close(a, b, tol):
    for c, x, y in zip("uvw", a, b):
        e = float((x - y).abs().max() / y.abs().max())
        print(f"{c}: staged vs L1 max relative difference {e:.3e}")
        assert e <= tol, (c, e)


@pytest.mark.parametrize("order,traj", [(6, 2), (4, 2), (6, 4)])
def test_mixed_staged_equals_l1_all_staged(order, traj):
    f = _flow((40, 24, 64), 0.01, 0.1, order, traj)
    ((a, na), (b, nb)), stats = _both(f, 0.01)
    _close(a, b, 1e-6)
    assert na == nb
    assert stats[0] == 0 and stats[1] > 0 and stats[2] == stats[1] and stats[3] == stats[1], stats


@pytest.mark.parametrize("dt", [0.15, 0.3])
def test_mixed_staged_equals_l1_wide_feet(dt):
    f = _flow((24, 16, 64), dt, 0.35)
    ((a, na), (b, nb)), stats = _both(f, dt)
    _close(a, b, 1e-6)
    assert na == nb
    # both paths taken: some boxes staged, some blocks through L1
    print("time-outs, blocks, near boxes staged, far boxes staged:", stats)
    assert stats[0] == 0 and 0 < stats[2] + stats[3] < 2 * stats[1], stats


def test_mixed_step_uses_staged_boxes_and_tracks_fp64():
    n3, dt = (48, 32, 64), 0.01
    fm = _flow(n3, dt, 0.1, precision="mixed")
    fd = _flow(n3, dt, 0.1, precision="fp64")
    stats = (ctypes.c_int64 * 4)()
    N.lib().slc_gather_stats(fm._grid.handle, stats, 1)
    for _ in range(3):
        fm.step_sl_bdf2(dt)
        fd.step_sl_bdf2(dt)
    torch.cuda.synchronize()
    N.lib().slc_gather_stats(fm._grid.handle, stats, 0)
    assert stats[0] == 0 and stats[1] > 0 and stats[2] > 0, list(stats)
    for x, y in zip((fm.u, fm.v, fm.w), (fd.u, fd.v, fd.w)):
        e = float((x - y).abs().max() / y.abs().max())
        assert e < 1e-5, e
