"""The hand-written adjoint of the SL-BDF2 step (slc_adjoint_step behind
SLRollout, a torch.autograd.Function with step checkpointing):

* against torch autograd through the reference's eager FP64 path on a 48^3
  channel (tests/golden/adjoint_48.npz, made by make_adjoint_golden.py):
  the loss and four directional derivatives;
* against central finite differences (h = 1e-6) in seeded smooth
  directions, over 1, 2 and 5 steps, orders 4 and 6, no-slip and free-slip
  top walls, symmetric and bottom stretching;
* determinism: reruns and different checkpoint intervals give bit-identical
  gradients (no floating-point atomics in the transposed gathers)."""

import math
import os
import sys

import numpy as np
import pytest
import torch

from slchannel_b200 import adjoint as A
from slchannel_b200.solver import SLChannelFlow
from slchannel_b200.utils import compute_bulk_velocity

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_adjoint_golden as G  # noqa: E402

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "adjoint_48.npz")


def _flow(nx, ny, nz, Lx, Ly, Re, dt, order, gamma=2.0, top="dirichlet", stretching="symmetric"):
    cfg = {
        "grid": {"nx": nx, "ny": ny, "nz": nz},
        "domain": {"Lx": Lx, "Ly": Ly, "Lz": 2.0, "stretching_type": stretching},
        "flow": {"Re": Re, "Re_tau": 180.0, "U_bulk": 1.0, "gamma": gamma},
        "boundary_conditions": {"top_wall": {"type": top}},
        "initialization": {"type": "parabolic"},
        "time": {"dt": dt},
        "compute": {"device": "cuda"},
        "sl": {"interp_order": order, "n_traj_iters": 2, "interp_dtype": "fp64"},
    }
    return SLChannelFlow(config=cfg)


def _projected(flow, fields):
    flow.set_state(*(torch.from_numpy(a) for a in fields))
    flow.apply_bc_uvw()
    ub = float(compute_bulk_velocity(flow.u, flow.cell_vol_ratio, flow.total_volume))
    flow.u *= 1.0 / ub
    flow._save_and_project_initial()
    return tuple(t.clone() for t in (flow.u, flow.v, flow.w))


def _as_ghost(flow, interior):
    out = [torch.zeros_like(t) for t in (flow.u, flow.v, flow.w)]
    nx, ny, nz = flow.nx, flow.ny, flow.nz
    for c, d in enumerate(interior):
        kz = nz - 1 if c == 2 else nz
        out[c][1:nx + 1, 1:ny + 1, 1:kz + 1] = torch.as_tensor(d, device=flow.device)
    return out


def test_adjoint_matches_reference_autograd_48():
    g = np.load(GOLDEN)
    c = G.CASE
    flow = _flow(c["nx"], c["ny"], c["nz"], c["Lx"], c["Ly"], c["Re"], c["dt"], c["order"], c["gamma"])
    z_f, z_c = flow.z_f.cpu().numpy(), flow.z_c.cpu().numpy()
    assert np.abs(z_f - g["z_f"]).max() < 1e-14
    V0 = _projected(flow, G.initial_field(c, z_f, z_c))
    mask = [torch.from_numpy(m).to(flow.device) for m in G.mask_fields(c, z_f, z_c)]
    J, grad = A.gradient(flow, V0, c["dt"], c["n_steps"], mask, checkpoint_every=2)
    assert abs(J - float(g["J"])) <= 1e-11 * abs(float(g["J"]))
    dd = [A.dot(grad, _as_ghost(flow, G.direction_fields(c, z_f, z_c, s))) for s in c["direction_seeds"]]
    ref = g["dirderiv"]
    scale = np.abs(ref).max()
    err = np.abs(np.array(dd) - ref).max() / scale
    print(f"adjoint vs reference autograd (48^3, 3 steps): {dd} vs {ref.tolist()}, rel {err:.2e}")
    assert err < 1e-8


CASES = [
    # (order, top, stretching, n_steps)
    (6, "dirichlet", "symmetric", 1),
    (6, "dirichlet", "symmetric", 2),
    (6, "dirichlet", "symmetric", 5),
    (4, "neumann", "bottom", 3),
]


@pytest.mark.parametrize("order,top,stretching,n_steps", CASES)
def test_adjoint_vs_central_fd(order, top, stretching, n_steps):
    nx, ny, nz, dt = 24, 16, 20, 0.1
    flow = _flow(nx, ny, nz, 2 * math.pi, math.pi, 800.0, dt, order, 1.8, top, stretching)
    c = dict(G.CASE, nx=nx, ny=ny, nz=nz, field_seed=17, mask_seed=18)
    z_f, z_c = flow.z_f.cpu().numpy(), flow.z_c.cpu().numpy()
    V0 = _projected(flow, G.initial_field(c, z_f, z_c))
    mask = [torch.from_numpy(m).to(flow.device) for m in G.mask_fields(c, z_f, z_c)]
    J, grad = A.gradient(flow, V0, dt, n_steps, mask, checkpoint_every=2)
    worst = 0.0
    for seed in (1, 2, 3):
        d = _as_ghost(flow, G.direction_fields(c, z_f, z_c, seed))
        fd = A.central_fd(flow, V0, d, 1e-6, dt, n_steps, mask)
        ad = A.dot(grad, d)
        # central FD with h = 1e-6 on J ~ 2e3 carries ~1e-7 absolute roundoff
        e = abs(fd - ad) / max(abs(fd), 0.1)
        worst = max(worst, e)
        assert e < 1e-5, (seed, fd, ad, e)
    print(f"adjoint vs FD order {order} {top} {stretching} {n_steps} steps: worst rel {worst:.2e}")


def test_adjoint_is_deterministic_and_checkpoint_invariant():
    nx, ny, nz, dt = 20, 16, 24, 0.08
    flow = _flow(nx, ny, nz, 2 * math.pi, math.pi, 1500.0, dt, 6)
    c = dict(G.CASE, nx=nx, ny=ny, nz=nz, field_seed=23, mask_seed=24)
    z_f, z_c = flow.z_f.cpu().numpy(), flow.z_c.cpu().numpy()
    V0 = _projected(flow, G.initial_field(c, z_f, z_c))
    mask = [torch.from_numpy(m).to(flow.device) for m in G.mask_fields(c, z_f, z_c)]
    runs = [A.gradient(flow, V0, dt, 7, mask, checkpoint_every=k)[1] for k in (3, 3, 1, 7, 0)]
    for r in runs[1:]:
        for a, b in zip(runs[0], r):
            assert torch.equal(a, b)
    # ghosts of the returned gradient are zero (folded into the interiors)
    gu = runs[0][0]
    assert float(gu[0].abs().max()) == 0.0 and float(gu[:, 0].abs().max()) == 0.0


@pytest.mark.parametrize("attr,value", [("sl_bdf2_pressure", "inc"), ("sl_traj_order", 4)])
def test_adjoint_refuses_unsupported_forms(attr, value):
    dt = 0.01
    f = _flow(16, 12, 20, 2 * math.pi, math.pi, 2800.0, dt, 6)
    setattr(f, attr, value)
    V0 = tuple(t.clone() for t in (f.u, f.v, f.w))
    with pytest.raises(ValueError, match="noninc"):
        A.loss_of(f, V0, dt, 1, A.smooth_mask(f, seed=1))
