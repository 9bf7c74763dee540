"""slc_step_bdf2_host (state in pinned host memory, pipelined copies) against
the device-resident step: four chained steps with the host buffers rotated
as a caller would, bit-identical V, p and (u_bulk, forcing).  Grids with
nx >= 96 take the slab-streamed path; a fast jet in one slab makes the slabs
released after it stand down and be recomputed at the end."""

import math

import pytest
import torch

from slchannel_b200 import _native as N
from slchannel_b200.fields import synthetic_channel_field
from slchannel_b200.host import HostStateStepper, pinned_like
from slchannel_b200.solver import SLChannelFlow
from slchannel_b200.utils import compute_bulk_velocity

pytestmark = pytest.mark.gpu


def _flow(nx, ny, nz, dt, precision="fp64"):
    cfg = {"grid": {"nx": nx, "ny": ny, "nz": nz},
           "domain": {"Lx": 2 * math.pi, "Ly": math.pi, "Lz": 2.0},
           "flow": {"Re": 2800.0, "Re_tau": 180.0, "U_bulk": 1.0, "gamma": 2.0},
           "initialization": {"type": "parabolic"}, "time": {"dt": dt},
           "compute": {"device": "cuda"},
           "sl": {"interp_order": 6, "n_traj_iters": 2, "interp_dtype": precision}}
    f = SLChannelFlow(config=cfg)
    u, v, w = synthetic_channel_field(nx, ny, nz, 2 * math.pi, math.pi, 2.0, f.z_f.cpu().numpy(),
                                      f.z_c.cpu().numpy(), urms=0.1, seed=9)
    f.set_state(*(torch.from_numpy(a) for a in (u, v, w)))
    f.apply_bc_uvw()
    f.u *= 1.0 / float(compute_bulk_velocity(f.u, f.cell_vol_ratio, f.total_volume))
    f._save_and_project_initial()
    f.step_sl_bdf2(dt)  # bootstrap
    return f


@pytest.mark.parametrize("n3,precision", [((40, 32, 48), "fp64"), ((24, 16, 20), "fp64"),
                                         ((24, 16, 20), "mixed")])
def test_host_state_steps_match_device_steps(n3, precision):
    dt = 0.02
    f = _flow(*n3, dt, precision)
    hs = HostStateStepper(f)
    H = [tuple(pinned_like(t) for t in (f.u, f.v, f.w)) for _ in range(3)]
    for h, d in zip(H[0], (f.u_nm1, f.v_nm1, f.w_nm1)):
        h.copy_(d)
    for h, d in zip(H[1], (f.u, f.v, f.w)):
        h.copy_(d)
    hp = pinned_like(f.p)
    hb = torch.zeros(2, dtype=torch.float64).pin_memory()
    prev, cur, nxt = H
    for step in range(4):
        hs.step(cur, prev, nxt, hp, hb, dt)
        ub, fc = f.step_sl_bdf2(dt)
        torch.cuda.current_stream().synchronize()
        for a, b in zip(nxt, (f.u, f.v, f.w)):
            assert torch.equal(a, b.cpu()), step
        assert torch.equal(hp, f.p.cpu())
        assert float(hb[0]) == float(ub) and float(hb[1]) == float(fc)
        prev, cur, nxt = cur, nxt, prev


def _run_pair(f, dt, steps):
    hs = HostStateStepper(f)
    H = [tuple(pinned_like(t) for t in (f.u, f.v, f.w)) for _ in range(3)]
    for h, d in zip(H[0], (f.u_nm1, f.v_nm1, f.w_nm1)):
        h.copy_(d)
    for h, d in zip(H[1], (f.u, f.v, f.w)):
        h.copy_(d)
    hp = pinned_like(f.p)
    hb = torch.zeros(2, dtype=torch.float64).pin_memory()
    prev, cur, nxt = H
    stats = []
    for step in range(steps):
        hs.step(cur, prev, nxt, hp, hb, dt)
        ub, fc = f.step_sl_bdf2(dt)
        torch.cuda.current_stream().synchronize()
        stats.append(hs.stats())
        for a, b in zip(nxt, (f.u, f.v, f.w)):
            assert torch.equal(a, b.cpu()), step
        assert torch.equal(hp, f.p.cpu()), step
        assert float(hb[0]) == float(ub) and float(hb[1]) == float(fc)
        prev, cur, nxt = cur, nxt, prev
    return stats


def test_streamed_host_steps_match_device_steps():
    # 96 x nodes: at least three slabs, feet far inside the neighbour slabs
    dt = 0.02
    f = _flow(96, 40, 48, dt)
    st = _run_pair(f, dt, 4)
    assert [s["streamed_calls"] for s in st] == [1, 2, 3, 4]
    assert all(s["whole_calls"] == 0 and s["slabs"] >= 3 and s["deferred_slabs"] == 0 for s in st)


def test_streamed_host_step_defers_slabs_the_feet_leave():
    # slabs of W x nodes arrive in the order S-1, 0, 1, ..., S-2, and slab s
    # is released once slab s+1 is there.  A jet of +40 in u over x nodes
    # 70..89 carries feet ~30 nodes, beyond the W - 8 a released slab allows:
    # the slabs released before the jet's first slab arrives run streamed,
    # every later one is recomputed after the last slab; the results stay
    # those of the device step
    dt = 0.02
    f = _flow(128, 24, 40, dt)
    for t in (f.u, f.u_nm1):
        t[70:90] += 40.0
    # ghosts consistent again in both levels, as a step leaves them (the
    # device step's next V^{n-1} is its V^n with the boundary conditions
    # applied, the host caller's is the buffer it passed)
    for tri in ((f.u, f.v, f.w), (f.u_nm1, f.v_nm1, f.w_nm1)):
        f._grid.call("slc_apply_bc", *[N.ptr(t) for t in tri], N.stream_of(f.u))
    st = _run_pair(f, dt, 2)
    S = st[0]["slabs"]
    assert S >= 3
    jet_slab = 70 * S // 128  # slab of x node 70 (bounds floor(s * 128 / S))
    released_before_jet = jet_slab - 1
    assert released_before_jet >= 1
    assert st[0]["deferred_slabs"] == S - released_before_jet, st


def test_host_state_step_refuses_incremental_pressure():
    f = _flow(16, 12, 20, 0.01)
    f.sl_bdf2_pressure = "inc"
    with pytest.raises(ValueError, match="noninc"):
        HostStateStepper(f)
