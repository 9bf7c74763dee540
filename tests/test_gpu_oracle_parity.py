"""GPU SL-BDF2 step vs the CPU oracle on the benchmark's seeded field recipe
(Poiseuille + curl of a seeded vector potential, tanh gamma = 2, Re_b 2800),
and size-independent properties at the benchmark's full 256^3 size.

Per-step parity (resync=True: every step starts both sides from the
oracle's state): 1e-12 relative (to each field's max) on u, v, w, pressure
1e-11, clamp counts exact.  Free-running trajectories (resync=False) drift
apart only by round-off amplified by the flow: held to 1e-12 at trajectory
CFL <= 1 and to 1e-10 in the wall-clamping, far-foot-CFL ~7 case."""

import math

import numpy as np
import pytest
import torch
from helpers import rel_err

from oracle.slbdf2 import OracleChannel
from slchannel_b200.fields import synthetic_channel_field
from slchannel_b200.solver import SLChannelFlow
from slchannel_b200.utils import compute_bulk_velocity, compute_divergence, generate_grid

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")


def config(nx, ny, nz, Lx, Ly, order, Re=2800.0, gamma=2.0, dt=0.01, top="dirichlet",
           stretching="symmetric"):
    return {
        "grid": {"nx": nx, "ny": ny, "nz": nz},
        "domain": {"Lx": Lx, "Ly": Ly, "Lz": 2.0, "stretching_type": stretching},
        "flow": {"Re": Re, "Re_tau": 180.0, "U_bulk": 1.0, "gamma": gamma},
        "boundary_conditions": {"top_wall": {"type": top}},
        "initialization": {"type": "parabolic"},
        "time": {"dt": dt},
        "compute": {"device": "cuda"},
        "sl": {"interp_order": order, "n_traj_iters": 2, "interp_dtype": "fp64"},
    }


def projected_field(nx, ny, nz, Lx, Ly, gamma, urms, seed, order, Re):
    """Seeded field, bulk-rescaled and projected by the ORACLE, so both sides
    start from bit-identical arrays."""
    Lz = 2.0
    z_f, z_c, dz_f, dz_c = (t.numpy() for t in generate_grid(gamma, nz, Lz))
    u, v, w = synthetic_channel_field(nx, ny, nz, Lx, Ly, Lz, z_f, z_c, urms=urms, seed=seed)
    ch = OracleChannel(nx, ny, nz, Lx, Ly, Lz, gamma, 1.0 / Re, u, v, w, order=order,
                       z_f=z_f, z_c=z_c)
    ub = ch.bulk_velocity()
    ch.u *= 1.0 / ub
    ch.project_initial()
    return ch


def run_parity(nx, ny, nz, Lx, Ly, order, steps, dt, urms=0.1, seed=1, Re=2800.0,
               resync=True, tol=1e-12):
    ch = projected_field(nx, ny, nz, Lx, Ly, 2.0, urms, seed, order, Re)
    flow = SLChannelFlow(config=config(nx, ny, nz, Lx, Ly, order, Re=Re, dt=dt))
    flow.set_state(*(torch.from_numpy(a) for a in (ch.u, ch.v, ch.w, ch.p)))
    worst = 0.0
    for step in range(steps):
        ub_o, f_o = ch.step_bdf2(dt)
        ub, f = flow.step_sl_bdf2(dt)
        for c in "uvw":
            e = rel_err(getattr(flow, c).cpu().numpy(), getattr(ch, c))
            worst = max(worst, e)
            assert e < tol, (step, c, e)
        assert rel_err(flow.p.cpu().numpy(), ch.p) < 10 * tol, step
        assert abs(float(ub) - ub_o) < 1e-13
        if resync or step == 0:
            assert int(flow.sl.n_clamped_last) == ch.n_clamped_last
        if resync:
            for name in ("u", "v", "w", "u_nm1", "v_nm1", "w_nm1", "p"):
                getattr(flow, name).copy_(torch.from_numpy(getattr(ch, name)))
    return worst


@pytest.mark.parametrize("order", [6, 4])
def test_parity_ragged_grid(order):
    # odd, non-power-of-two sizes and nx != ny: exercises every wrap and tile edge
    run_parity(30, 18, 22, 2 * math.pi, math.pi, order, steps=6, dt=0.05, urms=0.15)
    run_parity(30, 18, 22, 2 * math.pi, math.pi, order, steps=6, dt=0.05, urms=0.15,
               resync=False)


@pytest.mark.parametrize("order", [6, 4])
def test_parity_staged_gather_ragged(order):
    """A ragged 30 x 18 x 48 grid: partial x, y and z tiles and feet across
    the periodic seams, both orders."""
    run_parity(30, 18, 48, 2 * math.pi, math.pi, order, steps=4, dt=0.05, urms=0.15)


def test_parity_staged_gather_wide_feet():
    """Large dt: feet several cells from their arrival points, wall clamps
    on both walls."""
    run_parity(24, 16, 40, 2 * math.pi, math.pi, 6, steps=3, dt=0.6, urms=0.35)


def test_parity_config1_64cubed_20_steps():
    """Config 1: 64^3 in 2pi x pi x 2, gamma 2, Re_b 2800 on the channel
    height (nu = 1/1400), order 6, dt 0.01, 20 steps (BDF1 bootstrap + 19
    BDF2), free-running, against the oracle every step."""
    run_parity(64, 64, 64, 2 * math.pi, math.pi, 6, steps=20, dt=0.01, urms=0.1, resync=False,
               Re=1400.0)


def test_parity_large_dt_clamps():
    """A far foot that crosses the walls: dt large enough for clamping."""
    run_parity(24, 16, 20, 2 * math.pi, math.pi, 6, steps=4, dt=0.6, urms=0.35)
    run_parity(24, 16, 20, 2 * math.pi, math.pi, 6, steps=4, dt=0.6, urms=0.35, resync=False,
               tol=1e-10)


def test_full_size_properties_256():
    """256^3 (4pi x 2pi x 2, Re_b 2792.8, dt 0.01, order 6) -- the benchmark
    size: every step divergence-free to 1e-11, bulk velocity 1, finite, and a
    rerun from the same state is bit-identical (deterministic reductions,
    no floating-point atomics)."""
    n = 256
    Lx, Ly = 4 * math.pi, 2 * math.pi
    cfg = config(n, n, n, Lx, Ly, 6, Re=2792.8, dt=0.01)
    flow = SLChannelFlow(config=cfg)
    z_f, z_c = flow.z_f.cpu().numpy(), flow.z_c.cpu().numpy()
    u, v, w = synthetic_channel_field(n, n, n, Lx, Ly, 2.0, z_f, z_c, urms=0.1, seed=0)
    flow.set_state(*(torch.from_numpy(a) for a in (u, v, w)))
    ub0 = float(compute_bulk_velocity(flow.u, flow.cell_vol_ratio, flow.total_volume))
    flow.u *= 1.0 / ub0
    flow._save_and_project_initial()
    snap = None
    for step in range(3):
        if step == 1:
            snap = [t.clone() for t in (flow.u, flow.v, flow.w, flow.u_nm1, flow.v_nm1, flow.w_nm1)]
        ub, _ = flow.step_sl_bdf2(0.01)
        div = compute_divergence(flow.u, flow.v, flow.w, n, n, n, flow.dx, flow.dy, flow.dz_f)
        assert div.abs().max().item() < 1e-11
        assert abs(float(ub) - 1.0) < 1e-12
        assert torch.isfinite(flow.u).all()
    first = [t.clone() for t in (flow.u, flow.v, flow.w)]
    # replay steps 2..3 from the snapshot: bit-identical
    flow.u, flow.v, flow.w, flow.u_nm1, flow.v_nm1, flow.w_nm1 = snap
    for _ in range(2):
        flow.step_sl_bdf2(0.01)
    for a, b in zip(first, (flow.u, flow.v, flow.w)):
        assert torch.equal(a, b)
