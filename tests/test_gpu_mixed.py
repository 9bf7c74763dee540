"""The mixed-precision form (FP32 fluctuation about an FP64 plane mean in the
trace and gather; everything else FP64) against the FP64 oracle.

* test_mixed_advect_vs_fp64: the reference's own bar for its FP32 path
  (tests/test_semilag_triton.py: relative max error < 5e-6 against the FP64
  eager advect, orders 4 and 6, no clamps).
* test_mixed_step_error: every SL-BDF2 step, started from the oracle's
  state, within 1e-5 relative velocity error of the FP64 oracle, divergence
  below 1e-11 and the bulk velocity at 1.
* test_mixed_step_error_traj4: the same with tricubic trajectory sampling
  (traj_interp_order 4) against the oracle stepping with tricubic
  trajectories.
* test_mixed_step_error_bottom_free_slip: the per-step bar with bottom-only
  tanh stretching and a free-slip top (the FP32 locate's other branch and the
  Neumann closure).
* test_mixed_inc_pressure: the incremental-pressure form (bdf2_pressure inc),
  trilinear and tricubic trajectories, free-running 3 steps beside the FP64
  oracle within 1e-5.
* test_mixed_statistics_drift: free-running 40 steps beside the FP64 GPU
  form; plane-averaged U, u'_rms, v'_rms, w'_rms and uw drift stated and
  bounded."""

import math

import numpy as np
import pytest
import torch
from helpers import make_field, rel_err

from oracle.slbdf2 import OracleAdvector, OracleChannel
from slchannel_b200.fields import synthetic_channel_field
from slchannel_b200.semilag import SLAdvector
from slchannel_b200.solver import SLChannelFlow
from slchannel_b200.utils import compute_divergence, generate_grid

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")


@pytest.mark.parametrize("order", [4, 6])
def test_mixed_advect_vs_fp64(order):
    NX = NY = 32
    NZ, LX, LZ, G = 48, 2 * math.pi, 2.0, 1.5
    dx = LX / NX
    z_f, z_c, _, _ = generate_grid(G, NZ, LZ)
    zf, zc = z_f.numpy(), z_c.numpy()
    adv = SLAdvector(NX, NY, NZ, dx, dx, LX, LX, LZ, z_f, z_c, G, order=order,
                     interp_dtype="fp32_accum64", device=DEV)
    ora = OracleAdvector(NX, NY, NZ, dx, dx, LX, LX, LZ, zf, zc, G, order=order)

    def f(X, Y, Z):
        return np.sin(2 * math.pi * X / LX) * np.cos(2 * math.pi * Y / LX) * (1.0 + 0.3 * Z)

    u = make_field("u", f, NX, NY, NZ, dx, dx, zf, zc)
    v = make_field("v", f, NX, NY, NZ, dx, dx, zf, zc)
    w = make_field("w", lambda X, Y, Z: 0 * X + 0 * Y + 0 * Z, NX, NY, NZ, dx, dx, zf, zc)
    T = lambda a: torch.from_numpy(a).to(DEV)  # noqa: E731
    outs = adv.advect(T(u), T(v), T(w), T(u), T(v), T(w), 0.05)
    refs = ora.advect(u, v, w, u, v, w, 0.05)
    for c, a, b in zip("uvw", outs, refs):
        scale = np.abs(b).max() or 1.0
        err = np.abs(a.cpu().numpy() - b).max() / scale
        assert err < 5e-6, (c, err)
    assert int(adv.n_clamped_last) == 0


@pytest.mark.parametrize("order", [4, 6])
def test_mixed_advect_extra_rhs_vs_fp64(order):
    """advect(..., extra_rhs=[two triples]) in the mixed form: the advected
    triple and each extra triple within the reference's FP32 bar (5e-6) of
    the FP64 oracle advecting that triple along the same trajectory velocity,
    and the extras arrival-shaped."""
    NX = NY = 32
    NZ, LX, LZ, G = 48, 2 * math.pi, 2.0, 1.5
    dx = LX / NX
    z_f, z_c, _, _ = generate_grid(G, NZ, LZ)
    zf, zc = z_f.numpy(), z_c.numpy()
    adv = SLAdvector(NX, NY, NZ, dx, dx, LX, LX, LZ, z_f, z_c, G, order=order,
                     interp_dtype="fp32_accum64", device=DEV)
    ora = OracleAdvector(NX, NY, NZ, dx, dx, LX, LX, LZ, zf, zc, G, order=order)

    def f(a, b):
        return lambda X, Y, Z: np.sin(2 * math.pi * a * X / LX) * np.cos(2 * math.pi * b * Y / LX) * (1.0 + 0.3 * Z)

    u = make_field("u", f(1, 1), NX, NY, NZ, dx, dx, zf, zc)
    v = make_field("v", f(1, 2), NX, NY, NZ, dx, dx, zf, zc)
    w = make_field("w", lambda X, Y, Z: 0 * X + 0 * Y + 0 * Z, NX, NY, NZ, dx, dx, zf, zc)
    extra = [tuple(make_field(c, f(2, a), NX, NY, NZ, dx, dx, zf, zc) for c in "uvw") for a in (1, 3)]
    T = lambda a: torch.from_numpy(a).to(DEV)  # noqa: E731
    us, vs, ws, ex = adv.advect(T(u), T(v), T(w), T(u), T(v), T(w), 0.05,
                                extra_rhs=[tuple(T(a) for a in e) for e in extra])
    for c, a, b in zip("uvw", (us, vs, ws), ora.advect(u, v, w, u, v, w, 0.05)):
        assert np.abs(a.cpu().numpy() - b).max() / (np.abs(b).max() or 1.0) < 5e-6, c
    for e, got in zip(extra, ex):
        refs = ora.advect(*e, u, v, w, 0.05)
        for c, a, b in zip("uvw", got, refs):
            b = b[1:NX + 1, 1:NY + 1, 1:(NZ if c == "w" else NZ + 1)]
            assert tuple(a.shape) == b.shape
            assert np.abs(a.cpu().numpy() - b).max() / (np.abs(b).max() or 1.0) < 5e-6, c


def _config(n, Lx, Ly, order, precision, Re=2800.0, dt=0.01):
    return {
        "grid": {"nx": n, "ny": n, "nz": n},
        "domain": {"Lx": Lx, "Ly": Ly, "Lz": 2.0},
        "flow": {"Re": Re, "Re_tau": 180.0, "U_bulk": 1.0, "gamma": 2.0},
        "initialization": {"type": "parabolic"},
        "time": {"dt": dt},
        "compute": {"device": "cuda"},
        "sl": {"interp_order": order, "n_traj_iters": 2, "interp_dtype": precision},
    }


def _projected(n, Lx, Ly, order, urms, seed, Re=2800.0):
    z_f, z_c, _, _ = (t.numpy() for t in generate_grid(2.0, n, 2.0))
    u, v, w = synthetic_channel_field(n, n, n, Lx, Ly, 2.0, z_f, z_c, urms=urms, seed=seed)
    ch = OracleChannel(n, n, n, Lx, Ly, 2.0, 2.0, 1.0 / Re, u, v, w, order=order, z_f=z_f, z_c=z_c)
    ch.u *= 1.0 / ch.bulk_velocity()
    ch.project_initial()
    return ch


@pytest.mark.parametrize("order", [6, 4])
def test_mixed_step_error(order):
    n, Lx, Ly, dt = 48, 2 * math.pi, math.pi, 0.02
    ch = _projected(n, Lx, Ly, order, 0.12, 7)
    flow = SLChannelFlow(config=_config(n, Lx, Ly, order, "mixed", dt=dt))
    flow.set_state(*(torch.from_numpy(a) for a in (ch.u, ch.v, ch.w, ch.p)))
    for step in range(5):
        ch.step_bdf2(dt)
        ub, _ = flow.step_sl_bdf2(dt)
        for c in "uvw":
            e = rel_err(getattr(flow, c).cpu().numpy(), getattr(ch, c))
            assert e < 1e-5, (step, c, e)
        div = compute_divergence(flow.u, flow.v, flow.w, n, n, n, flow.dx, flow.dy, flow.dz_f)
        assert div.abs().max().item() < 1e-11
        assert abs(float(ub) - 1.0) < 1e-12
        for name in ("u", "v", "w", "u_nm1", "v_nm1", "w_nm1", "p"):
            getattr(flow, name).copy_(torch.from_numpy(getattr(ch, name)))


@pytest.mark.parametrize("order", [6, 4])
def test_mixed_step_error_traj4(order):
    n, Lx, Ly, dt, Re = 48, 2 * math.pi, math.pi, 0.02, 2800.0
    ch0 = _projected(n, Lx, Ly, order, 0.12, 7)
    ch = OracleChannel(n, n, n, Lx, Ly, 2.0, 2.0, 1.0 / Re, ch0.u, ch0.v, ch0.w, ch0.p,
                       order=order, traj_order=4, z_f=ch0.z_f, z_c=ch0.z_c)
    cfg = _config(n, Lx, Ly, order, "mixed", dt=dt)
    cfg["sl"]["traj_interp_order"] = 4
    flow = SLChannelFlow(config=cfg)
    flow.set_state(*(torch.from_numpy(a) for a in (ch.u, ch.v, ch.w, ch.p)))
    for step in range(4):
        ch.step_bdf2(dt)
        ub, _ = flow.step_sl_bdf2(dt)
        for c in "uvw":
            e = rel_err(getattr(flow, c).cpu().numpy(), getattr(ch, c))
            assert e < 1e-5, (step, c, e)
        div = compute_divergence(flow.u, flow.v, flow.w, n, n, n, flow.dx, flow.dy, flow.dz_f)
        assert div.abs().max().item() < 1e-11
        assert abs(float(ub) - 1.0) < 1e-12
        for name in ("u", "v", "w", "u_nm1", "v_nm1", "w_nm1", "p"):
            getattr(flow, name).copy_(torch.from_numpy(getattr(ch, name)))


@pytest.mark.parametrize("order", [6, 4])
def test_mixed_step_error_bottom_free_slip(order):
    n, Lx, Ly, dt, Re = 40, 2 * math.pi, math.pi, 0.02, 2800.0
    z_f, z_c, _, _ = (t.numpy() for t in generate_grid(2.0, n, 2.0, stretching_type="bottom"))
    u, v, w = synthetic_channel_field(n, n, n, Lx, Ly, 2.0, z_f, z_c, urms=0.12, seed=13)
    ch = OracleChannel(n, n, n, Lx, Ly, 2.0, 2.0, 1.0 / Re, u, v, w, order=order, z_f=z_f,
                       z_c=z_c, stretching_type="bottom", top_wall_bc_type="neumann")
    ch.apply_bc()
    ch.u *= 1.0 / ch.bulk_velocity()
    ch.project_initial()
    cfg = _config(n, Lx, Ly, order, "mixed", dt=dt)
    cfg["domain"]["stretching_type"] = "bottom"
    cfg["boundary_conditions"] = {"top_wall": {"type": "neumann"}}
    flow = SLChannelFlow(config=cfg)
    flow.set_state(*(torch.from_numpy(a) for a in (ch.u, ch.v, ch.w, ch.p)))
    for step in range(4):
        ch.step_bdf2(dt)
        ub, _ = flow.step_sl_bdf2(dt)
        for c in "uvw":
            e = rel_err(getattr(flow, c).cpu().numpy(), getattr(ch, c))
            assert e < 1e-5, (step, c, e)
        assert abs(float(ub) - 1.0) < 1e-12
        for name in ("u", "v", "w", "u_nm1", "v_nm1", "w_nm1", "p"):
            getattr(flow, name).copy_(torch.from_numpy(getattr(ch, name)))


@pytest.mark.parametrize("traj", [2, 4])
def test_mixed_inc_pressure(traj):
    n, Lx, Ly, dt, Re = 40, 2 * math.pi, math.pi, 0.02, 2800.0
    ch0 = _projected(n, Lx, Ly, 6, 0.12, 11)
    ch = OracleChannel(n, n, n, Lx, Ly, 2.0, 2.0, 1.0 / Re, ch0.u, ch0.v, ch0.w, ch0.p, order=6,
                       traj_order=traj, z_f=ch0.z_f, z_c=ch0.z_c, bdf2_pressure="inc")
    cfg = _config(n, Lx, Ly, 6, "mixed", dt=dt)
    cfg["sl"]["traj_interp_order"] = traj
    cfg["sl"]["bdf2_pressure"] = "inc"
    flow = SLChannelFlow(config=cfg)
    flow.set_state(*(torch.from_numpy(a) for a in (ch.u, ch.v, ch.w, ch.p)))
    for step in range(3):
        ch.step_bdf2(dt)
        ub, _ = flow.step_sl_bdf2(dt)
        for c in "uvw":
            e = rel_err(getattr(flow, c).cpu().numpy(), getattr(ch, c))
            assert e < 1e-5, (step, c, e)
        assert abs(float(ub) - 1.0) < 1e-12
    div = compute_divergence(flow.u, flow.v, flow.w, n, n, n, flow.dx, flow.dy, flow.dz_f)
    assert div.abs().max().item() < 1e-11


def plane_stats(flow):
    n = flow.nx
    u = flow.u[1 : n + 1, 1 : n + 1, 1 : n + 1]
    v = flow.v[1 : n + 1, 1 : n + 1, 1 : n + 1]
    w = 0.5 * (flow.w[1 : n + 1, 1 : n + 1, 0:n] + flow.w[1 : n + 1, 1 : n + 1, 1 : n + 1])
    U = u.mean(dim=(0, 1))
    up, vp, wp = u - U, v - v.mean(dim=(0, 1)), w - w.mean(dim=(0, 1))
    return {"U": U, "urms": up.pow(2).mean((0, 1)).sqrt(), "vrms": vp.pow(2).mean((0, 1)).sqrt(),
            "wrms": wp.pow(2).mean((0, 1)).sqrt(), "uw": (up * wp).mean((0, 1))}


def test_mixed_statistics_drift():
    n, Lx, Ly, dt, order = 48, 2 * math.pi, math.pi, 0.02, 6
    ch = _projected(n, Lx, Ly, order, 0.12, 11)
    flows = {}
    for prec in ("fp64", "mixed"):
        fl = SLChannelFlow(config=_config(n, Lx, Ly, order, prec, dt=dt))
        fl.set_state(*(torch.from_numpy(a) for a in (ch.u, ch.v, ch.w, ch.p)))
        for _ in range(40):
            fl.step_sl_bdf2(dt)
        flows[prec] = fl
    s64, s32 = plane_stats(flows["fp64"]), plane_stats(flows["mixed"])
    for k in s64:
        scale = s64[k].abs().max().item() or 1.0
        drift = (s32[k] - s64[k]).abs().max().item() / scale
        assert drift < 1e-5, (k, drift)
    for c in "uvw":
        e = rel_err(getattr(flows["mixed"], c).cpu().numpy(), getattr(flows["fp64"], c).cpu().numpy())
        assert e < 1e-4, (c, e)
