"""Golden values for the adjoint: torch autograd through the REFERENCE's eager
float64 CPU path (gmcavallazzi/SLchannel v1.0.1), on a 48^3 channel.

    python tests/golden/make_adjoint_golden.py /path/to/SLchannel

Case: 48 x 48 x 48 in 2pi x pi x 2, tanh gamma 2, Re_b 2800, dt 0.01,
order 6, three steps (the BDF1 bootstrap and two BDF2 steps, each with the
exact bulk shift).  The initial field is the seeded `initial_field` below,
refreshed, rescaled to bulk velocity 1 and projected with the reference's own
Poisson solver.  The loss is J = 1/2 sum over interior points of m_c V_c^2 at
the final step, with the seeded smooth mask `mask_fields` in (0, 1).

Stored: J, and the directional derivatives <dJ/dV^0, d_i> for the seeded
unit directions `direction_fields(seed_i)`; dJ/dV^0 is the gradient with
respect to the projected initial velocity's interior values.  The helpers are
plain numpy, so the GPU test rebuilds the same inputs from the same seeds.
"""

import math
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

CASE = dict(nx=48, ny=48, nz=48, Lx=2 * math.pi, Ly=math.pi, Lz=2.0, gamma=2.0, Re=2800.0,
            dt=0.01, order=6, n_steps=3, field_seed=5, mask_seed=6, direction_seeds=(101, 102, 103, 104))


def _modes(rng, X, Y, Z, Lx, Ly, Lz, n, zdamp):
    f = np.zeros(np.broadcast_shapes(X.shape, Y.shape, Z.shape))
    for _ in range(n):
        m, k = rng.integers(0, 3, size=2)
        l = rng.integers(0, 3)
        a = rng.normal()
        ph = rng.uniform(0, 2 * math.pi, 2)
        zz = np.cos(math.pi * l * Z / Lz)
        if zdamp:
            zz = zz * 4.0 * (Z / Lz) * (1.0 - Z / Lz)
        f = f + a * np.cos(2 * math.pi * m * X / Lx + ph[0]) * np.cos(2 * math.pi * k * Y / Ly + ph[1]) * zz
    return f


def ghost_positions(comp, nx, ny, dx, dy, z_f, z_c):
    if comp == 0:
        return ((np.arange(nx + 1) * dx)[:, None, None], ((np.arange(ny + 2) - 0.5) * dy)[None, :, None],
                z_c[None, None, :])
    if comp == 1:
        return (((np.arange(nx + 2) - 0.5) * dx)[:, None, None], (np.arange(ny + 1) * dy)[None, :, None],
                z_c[None, None, :])
    return (((np.arange(nx + 2) - 0.5) * dx)[:, None, None], ((np.arange(ny + 2) - 0.5) * dy)[None, :, None],
            z_f[None, None, :])


def interior_positions(comp, nx, ny, nz, dx, dy, z_f, z_c):
    x = (np.arange(nx) + (1.0 if comp == 0 else 0.5)) * dx
    y = (np.arange(ny) + (1.0 if comp == 1 else 0.5)) * dy
    z = z_f[1:nz] if comp == 2 else z_c[1:nz + 1]
    return np.meshgrid(x, y, z, indexing="ij")


def initial_field(c, z_f, z_c):
    """Ghost-shaped (u, v, w): Poiseuille profile plus seeded smooth
    wall-damped modes (ghost values are refreshed by the caller)."""
    nx, ny = c["nx"], c["ny"]
    dx, dy = c["Lx"] / nx, c["Ly"] / ny
    rng = np.random.default_rng(c["field_seed"])
    out = []
    for comp in range(3):
        X, Y, Z = ghost_positions(comp, nx, ny, dx, dy, z_f, z_c)
        f = 0.15 * _modes(rng, X, Y, Z, c["Lx"], c["Ly"], c["Lz"], 6, True)
        if comp == 0:
            f = f + 1.5 * Z * (2.0 - Z) / c["Lz"]
        out.append(np.ascontiguousarray(f * np.ones(np.broadcast_shapes(X.shape, Y.shape, Z.shape))))
    return out


def mask_fields(c, z_f, z_c):
    """Interior-shaped weights in (0, 1): a logistic of seeded smooth modes."""
    nx, ny, nz = c["nx"], c["ny"], c["nz"]
    dx, dy = c["Lx"] / nx, c["Ly"] / ny
    rng = np.random.default_rng(c["mask_seed"])
    out = []
    for comp in range(3):
        X, Y, Z = interior_positions(comp, nx, ny, nz, dx, dy, z_f, z_c)
        s = _modes(rng, X, Y, Z, c["Lx"], c["Ly"], c["Lz"], 6, False)
        out.append(1.0 / (1.0 + np.exp(-s)))
    return out


def direction_fields(c, z_f, z_c, seed):
    """Interior-shaped smooth seeded perturbation, unit 2-norm over all three."""
    nx, ny, nz = c["nx"], c["ny"], c["nz"]
    dx, dy = c["Lx"] / nx, c["Ly"] / ny
    rng = np.random.default_rng(seed)
    out = []
    for comp in range(3):
        X, Y, Z = interior_positions(comp, nx, ny, nz, dx, dy, z_f, z_c)
        out.append(_modes(rng, X, Y, Z, c["Lx"], c["Ly"], c["Lz"], 8, False))
    norm = math.sqrt(sum(float((d * d).sum()) for d in out))
    return [d / norm for d in out]


def main(ref_root):
    from make_golden import _stub_matplotlib

    _stub_matplotlib()
    sys.path.insert(0, ref_root)
    import torch
    import yaml

    torch.set_default_dtype(torch.float64)
    import slchannel.solver as ref_solver

    c = CASE
    with tempfile.TemporaryDirectory() as tmp:
        cfg = {
            "grid": {"nx": c["nx"], "ny": c["ny"], "nz": c["nz"]},
            "domain": {"Lx": float(c["Lx"]), "Ly": float(c["Ly"]), "Lz": c["Lz"],
                       "stretching_type": "symmetric"},
            "flow": {"Re": c["Re"], "Re_tau": 180.0, "U_bulk": 1.0, "gamma": c["gamma"]},
            "boundary_conditions": {"top_wall": {"type": "dirichlet"}},
            "initialization": {"type": "parabolic", "perturbation_intensity": 0.0},
            "solver": {"type": "fft"},
            "time": {"dt": c["dt"], "n_steps": c["n_steps"], "t_max": 1e9, "CFL_target": 3.0,
                     "dt_update_interval": 0, "dt_max": 1.0, "dt_min": 1e-4},
            "compute": {"device": "cpu"},
            "output": {"results_folder": os.path.join(tmp, "results"), "n_out": 10**8, "n_save": 10**8},
            "advection": {"scheme": "sl"},
            "sl": {"interp_order": c["order"], "n_traj_iters": 2, "interp_dtype": "fp64"},
            "statistics": {"n_stats": 0},
        }
        path = os.path.join(tmp, "cfg.yaml")
        with open(path, "w") as fh:
            yaml.safe_dump(cfg, fh)
        s = ref_solver.SLChannelFlow(config_file=path)
        z_f, z_c = s.z_f.numpy().copy(), s.z_c.numpy().copy()
        nx, ny, nz = c["nx"], c["ny"], c["nz"]
        u, v, w = (torch.from_numpy(a).clone() for a in initial_field(c, z_f, z_c))
        s.u, s.v, s.w = u, v, w
        s.apply_bc_uvw()
        ub = ref_solver.compute_bulk_velocity(s.u, s.cell_vol_ratio, s.total_volume)
        s.u = s.u * (1.0 / ub)
        s.apply_bc_uvw()
        div = ref_solver.compute_divergence(s.u, s.v, s.w, nx, ny, nz, s.dx, s.dy, s.dz_f)
        s.p = ref_solver.solve_poisson_fft(div, s.fft_data).clone()
        s.u, s.v, s.w = ref_solver.project_velocity(s.u, s.v, s.w, s.p, nx, ny, nz, s.dx, s.dy,
                                                    s.dz_c, s.dz_f, 1.0)
        s.apply_bc_uvw()
        # the independent variable: interior values of the projected V^0
        leaves = [t.detach().clone().requires_grad_(True) for t in (s.u, s.v, s.w)]
        s.u, s.v, s.w = (t.clone() for t in leaves)
        s.u_nm1 = s.v_nm1 = s.w_nm1 = None
        for _ in range(c["n_steps"]):
            s.step_sl_bdf2(c["dt"])
        mask = [torch.from_numpy(m) for m in mask_fields(c, z_f, z_c)]
        fin = (s.u[1:nx + 1, 1:ny + 1, 1:nz + 1], s.v[1:nx + 1, 1:ny + 1, 1:nz + 1],
               s.w[1:nx + 1, 1:ny + 1, 1:nz])
        J = sum(0.5 * (m * f * f).sum() for m, f in zip(mask, fin))
        J.backward()
        g = [t.grad.numpy() for t in leaves]
        gi = (g[0][1:nx + 1, 1:ny + 1, 1:nz + 1], g[1][1:nx + 1, 1:ny + 1, 1:nz + 1],
              g[2][1:nx + 1, 1:ny + 1, 1:nz])
        dd = []
        for sd in c["direction_seeds"]:
            d = direction_fields(c, z_f, z_c, sd)
            dd.append(sum(float((a * b).sum()) for a, b in zip(gi, d)))
        res = {
            "J": np.array(float(J.detach())),
            "dirderiv": np.array(dd),
            "grad_norm": np.array([float(np.sqrt((x * x).sum())) for x in gi]),
            "ghost_grad_abs": np.array([float(np.abs(x).sum() - np.abs(y).sum()) for x, y in zip(g, gi)]),
            "z_f": z_f, "z_c": z_c,
        }
    np.savez_compressed(os.path.join(HERE, "adjoint_48.npz"), **res)
    print({k: (v if v.size < 8 else v.shape) for k, v in res.items()})


if __name__ == "__main__":
    sys.path.insert(0, HERE)
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SLCHANNEL_REF", "."))
