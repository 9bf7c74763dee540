"""Parity at the benchmark's headline size (config 2): 256^3 in 4pi x 2pi x 2,
tanh gamma 2, Re_b 2792.8 (nu = 1/2792.8), dt 0.01, from the benchmark's
seeded field (u'_rms 0.1, seed 0), triquintic and tricubic.

The BDF1 bootstrap and four BDF2 steps run on the GPU and in the oracle,
every step started from the oracle's state (resync) and compared at 1e-12
relative (pressure 1e-11), bulk velocity to 1e-13, clamp counts exact
(solver.py:813-1018).  Step 5 is then taken apart substep by substep, each
GPU substep fed the oracle's own input for it:
  ubar (near foot, dt) and ubarbar (far foot, 2 dt) through SLAdvector.advect
  with U* = 2 V^n - V^{n-1};  u_hat from the fused trace+gather+BDF2 kernel
  (slc_trace_gather_bdf2);  the z-solve (slc_zsolve);  phi and the projected
  velocity (slc_project);  the bulk shift and forcing (slc_bulk_shift);
all at 1e-12 relative (phi 1e-11).  The oracle takes about 10 s per 256^3
step on 16 host threads, so each order costs about a minute."""

import math

import numpy as np
import pytest
import torch
from helpers import interior, rel_err

from oracle.slbdf2 import OracleChannel, max_threads
from slchannel_b200 import _native as N
from slchannel_b200.fields import synthetic_channel_field
from slchannel_b200.solver import SLChannelFlow
from slchannel_b200.utils import generate_grid

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")
NG = 256
LX, LY, LZ, GAMMA, RE, DT = 4 * math.pi, 2 * math.pi, 2.0, 2.0, 2792.8, 0.01


def _config(order):
    return {
        "grid": {"nx": NG, "ny": NG, "nz": NG},
        "domain": {"Lx": LX, "Ly": LY, "Lz": LZ, "stretching_type": "symmetric"},
        "flow": {"Re": RE, "Re_tau": 180.0, "U_bulk": 1.0, "gamma": GAMMA},
        "boundary_conditions": {"top_wall": {"type": "dirichlet"}},
        "initialization": {"type": "parabolic"},
        "time": {"dt": DT},
        "compute": {"device": "cuda"},
        "sl": {"interp_order": order, "n_traj_iters": 2, "interp_dtype": "fp64"},
    }


def T(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def C(t):
    return t.detach().cpu().numpy()


def _assert_fields(got, want, tol, what, comps="uvw"):
    for c, g, w in zip(comps, got, want):
        e = rel_err(interior(c, C(g), NG, NG, NG), interior(c, w, NG, NG, NG))
        assert e < tol, (what, c, e)


@pytest.mark.parametrize("order", [6, 4])
def test_config2_parity_256(order):
    z_f, z_c, _, _ = (t.numpy() for t in generate_grid(GAMMA, NG, LZ))
    u, v, w = synthetic_channel_field(NG, NG, NG, LX, LY, LZ, z_f, z_c, urms=0.1, seed=0)
    ch = OracleChannel(NG, NG, NG, LX, LY, LZ, GAMMA, 1.0 / RE, u, v, w, order=order,
                       z_f=z_f, z_c=z_c)
    del u, v, w
    ch.u *= 1.0 / ch.bulk_velocity()
    ch.project_initial()
    flow = SLChannelFlow(config=_config(order))
    flow.set_state(*(T(a) for a in (ch.u, ch.v, ch.w, ch.p)))
    assert max_threads() >= 1

    # steps 1-4: BDF1 bootstrap + three BDF2 steps, resynced every step
    for step in range(1, 5):
        ub_o, f_o = ch.step_bdf2(DT)
        ub, f = flow.step_sl_bdf2(DT)
        _assert_fields((flow.u, flow.v, flow.w), (ch.u, ch.v, ch.w), 1e-12, f"step {step}")
        assert rel_err(C(flow.p), ch.p) < 1e-11, step
        assert abs(float(ub) - ub_o) < 1e-13 and abs(float(f) - f_o) < 1e-9, step
        assert int(flow.sl.n_clamped_last) == ch.n_clamped_last, step
        for name in ("u", "v", "w", "u_nm1", "v_nm1", "w_nm1", "p"):
            getattr(flow, name).copy_(T(getattr(ch, name)))

    # step 5, substep by substep, from the oracle's step-4 state
    cur = tuple(a.copy() for a in (ch.u, ch.v, ch.w))
    prev = tuple(a.copy() for a in (ch.u_nm1, ch.v_nm1, ch.w_nm1))
    ub_o, f_o, cap = ch.step_bdf2(DT, capture=True)
    g = flow.sl.native
    st = N.stream_of(flow.u)
    dcur, dprev = [T(a) for a in cur], [T(a) for a in prev]
    mid = [2.0 * a - b for a, b in zip(dcur, dprev)]
    # the two feet (SLAdvector.advect, one foot each)
    _assert_fields(flow.sl.advect(*dcur, *mid, DT), cap["ubar"], 1e-12, "ubar")
    _assert_fields(flow.sl.advect(*dprev, *mid, 2.0 * DT), cap["ubarbar"], 1e-12, "ubarbar")
    assert int(flow.sl.n_clamped_last) >= 0
    del mid
    # u_hat: the fused trace + gather + BDF2 epilogue
    out = [torch.zeros_like(t) for t in dcur]
    ncl = torch.zeros((), dtype=torch.int64, device=DEV)
    g.call("slc_trace_gather_bdf2", *[N.ptr(t) for t in dcur], *[N.ptr(t) for t in dprev], DT,
           *[N.ptr(t) for t in out], N.ptr(ncl), st)
    _assert_fields(out, cap["uhat"], 1e-12, "uhat")
    assert int(ncl) == ch.n_clamped_last
    del out, dcur, dprev
    # the theta = 1 z-solve of the oracle's u_hat
    dte = (2.0 / 3.0) * DT
    zin = [T(a) for a in cap["uhat"]]
    g.call("slc_zsolve", *[N.ptr(t) for t in zin], dte, st)
    _assert_fields(zin, cap["zsolve"], 1e-12, "zsolve")
    del zin
    # phi and the projection of the oracle's z-solve output
    pin = [T(a) for a in cap["zsolve"]]
    p = torch.zeros(NG + 2, NG + 2, NG + 2, dtype=torch.float64, device=DEV)
    g.call("slc_project", *[N.ptr(t) for t in pin], N.ptr(p), dte, dte, st)
    assert rel_err(C(p), cap["phi"]) < 1e-11
    _assert_fields(pin, cap["proj"], 1e-12, "projection")
    # the bulk shift of the oracle's projected velocity
    bin_ = [T(a) for a in cap["proj"]]
    res = torch.empty(2, dtype=torch.float64, device=DEV)
    g.call("slc_bulk_shift", *[N.ptr(t) for t in bin_], 1.0, DT, N.ptr(res), st)
    _assert_fields(bin_, (ch.u, ch.v, ch.w), 1e-12, "bulk shift")
    assert abs(float(res[0]) - ub_o) < 1e-13 and abs(float(res[1]) - f_o) < 1e-9
