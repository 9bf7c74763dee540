"""The reference's own test suite for the SL path, restated against the GPU
drop-in with the reference's thresholds:

    tests/test_zmap_inverse.py       -> test_zmap_inverse
    tests/test_interp_convergence.py -> test_interp_convergence
    tests/test_departure_points.py   -> test_departure_points
    tests/test_sl_shear.py           -> test_sl_shear
    tests/test_sl_solid_body.py      -> test_sl_solid_body
    tests/test_sl_wall_clamp.py      -> test_sl_wall_clamp
    tests/test_sl_divergence.py      -> test_sl_divergence
    tests/test_stokes_decay.py       -> test_stokes_decay
"""

import math

import numpy as np
import pytest
import torch
from helpers import make_field

from slchannel_b200.semilag import SLAdvector
from slchannel_b200.solver import SLChannelFlow
from slchannel_b200.utils import compute_divergence, generate_grid

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")


def T(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(DEV)


def grid_np(gamma, nz, Lz, stretching="symmetric"):
    z_f, z_c, dz_f, dz_c = generate_grid(gamma, nz, Lz, stretching_type=stretching)
    return z_f, z_c, z_f.numpy(), z_c.numpy()


def fmap(kf, gamma, nz, Lz, st):
    g = torch.tensor(gamma, dtype=torch.float64)
    if st == "symmetric":
        return 0.5 * Lz * (1 + torch.tanh(g * (2.0 * kf / nz - 1.0)) / torch.tanh(g))
    return Lz * (1.0 - torch.tanh(g * (1.0 - kf / nz)) / torch.tanh(g))


def test_zmap_inverse():
    Lz = 2.0
    for st in ("symmetric", "bottom"):
        for gamma in (0.8, 1.8, 2.6):
            for nz in (64, 180):
                z_f, z_c, _, _ = grid_np(gamma, nz, Lz, st)
                adv = SLAdvector(4, 4, nz, 0.5, 0.5, 2.0, 2.0, Lz, z_f, z_c, gamma,
                                 stretching_type=st, device=DEV)
                kf = adv._face_coord(z_f.to(DEV)).cpu()
                err_f = (kf - torch.arange(nz + 1, dtype=torch.float64)).abs().max().item()
                torch.manual_seed(0)
                kr = torch.rand(5000, dtype=torch.float64) * nz
                err_r = (adv._face_coord(fmap(kr, gamma, nz, Lz, st).to(DEV)).cpu() - kr).abs().max().item()
                assert err_f < 1e-8 and err_r < 1e-8, (st, gamma, nz, err_f, err_r)


def test_interp_convergence():
    Lx, Ly, Lz, G = 2 * math.pi, 2 * math.pi, 2.0, 1.8

    def f(x, y, z):
        return (np.sin(2 * math.pi * x / Lx + 0.3) * np.cos(4 * math.pi * y / Ly - 1.1)
                * np.sin(1.5 * math.pi * z / Lz + 0.4))

    def err(n, order):
        z_f, z_c, zf, zc = grid_np(G, n, Lz)
        adv = SLAdvector(n, n, n, Lx / n, Ly / n, Lx, Ly, Lz, z_f, z_c, G, order=order, device=DEV)
        xg = (np.arange(n) * Lx / n)[:, None, None]
        yg = ((np.arange(n) + 0.5) * Ly / n)[None, :, None]
        buf = f(xg, yg, zc[None, None, :]) * np.ones((n, n, n + 2))
        rng = np.random.default_rng(1234)
        xq, yq = rng.uniform(0, Lx, 20000), rng.uniform(0, Ly, 20000)
        zq = adv.z_lo + rng.uniform(0, 1, 20000) * (adv.z_hi - adv.z_lo)
        iw = adv._build_iw(adv.spec["u"], T(xq), T(yq), T(zq), order)
        vals = adv._apply_iw(T(buf), iw).cpu().numpy()
        return np.abs(vals - f(xq, yq, zq)).max()

    for order, min_ratio in ((4, 10.0), (6, 40.0)):
        e = [err(n, order) for n in (32, 64, 128)]
        assert e[0] / e[1] > min_ratio and e[1] / e[2] > min_ratio, (order, e)


def test_departure_points():
    Lx, Ly, Lz, NX, NY, NZ, G = 2 * math.pi, 2 * math.pi, 2.0, 16, 16, 32, 1.5
    dx, dy = Lx / NX, Ly / NY
    z_f, z_c, zf, zc = grid_np(G, NZ, Lz)

    def mk(n_iters=2):
        return SLAdvector(NX, NY, NZ, dx, dy, Lx, Ly, Lz, z_f, z_c, G, n_traj_iters=n_iters, device=DEV)

    def fill(adv, fu, fv, fw):
        for c, fn in zip("uvw", (fu, fv, fw)):
            adv._fill(adv.mbuf[c], c, T(make_field(c, fn, NX, NY, NZ, dx, dy, zf, zc)))

    def arr(adv, comp):
        xa, ya, za, shape = adv.arrival[comp]
        return [t.expand(shape).cpu().numpy() for t in (xa, ya, za)]

    adv = mk()
    U0, V0, W0 = 0.7, -0.3, 0.02
    fill(adv, lambda X, Y, Z: U0 + 0 * X, lambda X, Y, Z: V0 + 0 * X, lambda X, Y, Z: W0 + 0 * X)
    dt = 0.05
    for comp in "uvw":
        xa, ya, za = arr(adv, comp)
        xd, yd, zd = (t.cpu().numpy() for t in adv.departure_coords(comp, dt))
        e = max(np.abs(xd - (xa - dt * U0)).max(), np.abs(yd - (ya - dt * V0)).max(),
                np.abs(zd - (za - dt * W0)).max())
        assert e < 1e-13, (comp, e)
    S = 0.8
    fill(adv, lambda X, Y, Z: S * Z, lambda X, Y, Z: 0 * X, lambda X, Y, Z: 0 * X)
    xa, ya, za = arr(adv, "u")
    xd, yd, zd = (t.cpu().numpy() for t in adv.departure_coords("u", dt))
    e = max(np.abs(xd - (xa - dt * S * za)).max(), np.abs(yd - ya).max(), np.abs(zd - za).max())
    assert e < 1e-13
    x0, z0, om = math.pi, 1.0, 0.3
    errs = []
    for dtv in (0.2, 0.1, 0.05):
        adv = mk(8)
        fill(adv, lambda X, Y, Z: -om * (Z - z0), lambda X, Y, Z: 0 * X, lambda X, Y, Z: om * (X - x0))
        xa, ya, za = arr(adv, "u")
        xd, yd, zd = (t.cpu().numpy() for t in adv.departure_coords("u", dtv))
        th = om * dtv
        xe = x0 + math.cos(th) * (xa - x0) + math.sin(th) * (za - z0)
        ze = z0 - math.sin(th) * (xa - x0) + math.cos(th) * (za - z0)
        mask = (np.abs(za - z0) < 0.7) & (xa > 1.0) & (xa < Lx - 1.0)
        errs.append(np.maximum(np.abs(xd - xe), np.abs(zd - ze))[mask].max())
    assert errs[0] / errs[1] > 6.0 and errs[1] / errs[2] > 6.0, errs


def _advect_fields(adv, n, fields_fn, mids, dt, zf, zc, dx, dy, nz):
    f = {c: T(make_field(c, fields_fn, n, n, nz, dx, dy, zf, zc)) for c in "uvw"}
    return adv.advect(f["u"], f["v"], f["w"], *mids, dt)


def test_sl_shear():
    Lx, Ly, Lz, G, S, DT = 2 * math.pi, 2 * math.pi, 2.0, 1.5, 0.8, 0.1

    def err(nx, order):
        nz = 32
        dx, dy = Lx / nx, Ly / nx
        z_f, z_c, zf, zc = grid_np(G, nz, Lz)
        adv = SLAdvector(nx, nx, nz, dx, dy, Lx, Ly, Lz, z_f, z_c, G, order=order, device=DEV)
        mids = (T(make_field("u", lambda X, Y, Z: S * Z + 0 * X, nx, nx, nz, dx, dy, zf, zc)),
                torch.zeros(nx + 2, nx + 1, nz + 2, device=DEV),
                torch.zeros(nx + 2, nx + 2, nz + 1, device=DEV))
        outs = _advect_fields(adv, nx, lambda X, Y, Z: np.sin(2 * math.pi * X / Lx) + 0 * Y + 0 * Z,
                              mids, DT, zf, zc, dx, dy, nz)
        e = 0.0
        for comp, out in zip("uvw", outs):
            xa, ya, za, shape = adv.arrival[comp]
            exact = np.sin(2 * math.pi * (xa - S * za * DT).cpu().numpy() / Lx) * np.ones(shape)
            o = out.cpu().numpy()
            got = o[1 : nx + 1, 1 : nx + 1, 1:nz] if comp == "w" else o[1 : nx + 1, 1 : nx + 1, 1 : nz + 1]
            e = max(e, np.abs(got - exact).max())
        return e

    ec = err(64, 4)
    assert ec < 1e-5
    e1, e2 = err(32, 4), err(64, 4)
    assert e1 / e2 > 10.0
    assert err(64, 6) < ec / 10


def test_sl_solid_body():
    Lx, Ly, Lz, G, U0, V0, DT = 2 * math.pi, 2 * math.pi, 2.0, 1.5, 0.9, -0.4, 0.08

    def err(n, fn, dt):
        dx, dy = Lx / n, Ly / n
        z_f, z_c, zf, zc = grid_np(G, n, Lz)
        adv = SLAdvector(n, n, n, dx, dy, Lx, Ly, Lz, z_f, z_c, G, device=DEV)
        mids = (T(make_field("u", lambda X, Y, Z: U0 + 0 * X, n, n, n, dx, dy, zf, zc)),
                T(make_field("v", lambda X, Y, Z: V0 + 0 * X, n, n, n, dx, dy, zf, zc)),
                torch.zeros(n + 2, n + 2, n + 1, device=DEV))
        outs = _advect_fields(adv, n, fn, mids, dt, zf, zc, dx, dy, n)
        e = 0.0
        for comp, out in zip("uvw", outs):
            xa, ya, za, shape = adv.arrival[comp]
            xa, ya, za = (t.cpu().numpy() for t in (xa, ya, za))
            exact = fn(xa - dt * U0, ya - dt * V0, za) * np.ones(shape)
            o = out.cpu().numpy()
            got = o[1 : n + 1, 1 : n + 1, 1:n] if comp == "w" else o[1 : n + 1, 1 : n + 1, 1 : n + 1]
            e = max(e, np.abs(got - exact).max())
        return e, int(adv.n_clamped_last)

    e, ncl = err(16, lambda X, Y, Z: 1.0 + 0.5 * Z - 0.3 * Z**2 + 0.1 * Z**3 + 0 * X, DT)
    assert e < 1e-12 and ncl == 0, (e, ncl)

    def f(X, Y, Z):
        return np.sin(2 * math.pi * X / Lx) * np.cos(2 * math.pi * Y / Ly) * np.sin(1.2 * math.pi * Z / Lz + 0.2)

    e1, _ = err(24, f, DT)
    e2, _ = err(48, f, DT / 2)
    assert e1 / e2 > 12.0, (e1, e2)


def test_sl_wall_clamp():
    Lx, Ly, Lz, NX, NZ, G = 2 * math.pi, 2 * math.pi, 2.0, 16, 48, 2.0
    dx = Lx / NX
    z_f, z_c, zf, zc = grid_np(G, NZ, Lz)

    def f(X, Y, Z):
        return np.cos(2 * math.pi * X / Lx) * np.sin(math.pi * Z / Lz) + 0 * Y

    for w0 in (-0.5, 0.5):
        adv = SLAdvector(NX, NX, NZ, dx, dx, Lx, Ly, Lz, z_f, z_c, G, device=DEV)
        mids = (torch.zeros(NX + 1, NX + 2, NZ + 2, device=DEV),
                torch.zeros(NX + 2, NX + 1, NZ + 2, device=DEV),
                torch.full((NX + 2, NX + 2, NZ + 1), w0, device=DEV))
        outs = _advect_fields(adv, NX, f, mids, 0.5, zf, zc, dx, dx, NZ)
        finite = all(torch.isfinite(t).all().item() for t in outs)
        bound = max(t.abs().max().item() for t in outs)
        assert finite and int(adv.n_clamped_last) > 0 and bound < 1.5


def make_config(*, nx=16, ny=16, nz=32, Re=1000.0, gamma=1.5, dt=0.01, init_type="vortices",
                pert=0.05, order=4, Lx=2 * math.pi, Ly=2 * math.pi):
    return {
        "grid": {"nx": nx, "ny": ny, "nz": nz},
        "domain": {"Lx": Lx, "Ly": Ly, "Lz": 2.0},
        "flow": {"Re": Re, "Re_tau": 180.0, "U_bulk": 1.0, "gamma": gamma},
        "initialization": {"type": init_type, "perturbation_intensity": pert, "n_vortices": 2},
        "solver": {"type": "fft"},
        "time": {"dt": dt, "n_steps": 10**9, "CFL_target": 3.0, "dt_update_interval": 0},
        "compute": {"device": "cuda"},
        "advection": {"scheme": "sl"},
        "sl": {"interp_order": order, "n_traj_iters": 2, "interp_dtype": "fp64"},
        "statistics": {"n_stats": 0},
    }


@pytest.mark.parametrize("order", [4, 6])
def test_sl_divergence(order):
    flow = SLChannelFlow(config=make_config(Re=1000.0, gamma=1.5, pert=0.08, dt=0.02, order=order))
    max_div = 0.0
    for _ in range(25):
        flow.step_sl_bdf2(0.02)
        div = compute_divergence(flow.u, flow.v, flow.w, flow.nx, flow.ny, flow.nz, flow.dx,
                                 flow.dy, flow.dz_f)
        max_div = max(max_div, div.abs().max().item())
    finite = all(torch.isfinite(t).all().item() for t in (flow.u, flow.v, flow.w, flow.p))
    frac = int(flow.sl.n_clamped_last) / (3 * flow.nx * flow.ny * flow.nz)
    assert finite and max_div < 1e-10 and frac < 0.01, (max_div, frac)


def test_stokes_decay():
    flow = SLChannelFlow(config=make_config(nx=8, ny=8, nz=96, Re=100.0, gamma=1.3,
                                            init_type="parabolic", pert=0.0, dt=0.02))
    flow.u[:] = torch.sin(math.pi * flow.z_c).view(1, 1, -1)
    flow.v[:] = 0.0
    flow.w[:] = 0.0
    flow.p[:] = 0.0
    flow.apply_bc_uvw()
    flow.forcing = 0.0
    flow._apply_bulk_forcing = lambda dt: (0.0, 0.0)
    dt, Tend = 0.02, 1.0
    for _ in range(round(Tend / dt)):
        flow.step_sl_bdf2(dt)
    decay = math.exp(-flow.nu * math.pi**2 * Tend)
    exact = decay * torch.sin(math.pi * flow.z_c[1:-1]).cpu()
    got = flow.u[4, 4, 1:-1].cpu()
    rel = ((got - exact).abs().max() / exact.abs().max()).item()
    assert rel < 0.01, rel
    assert flow.v.abs().max().item() < 1e-12 and flow.w.abs().max().item() < 1e-12
