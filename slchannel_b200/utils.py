"""Grid construction and the step diagnostics (reference: slchannel/utils.py).

``generate_grid`` is init-time host code (the reference's formulas, float64);
``compute_divergence`` and ``compute_bulk_velocity`` run as CUDA kernels of
libslc_b200.so and return device tensors.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _native as N


def generate_grid(gamma, nz, Lz, device="cpu", stretching_type="symmetric"):
    """utils.py:21-61 -- tanh-stretched faces z_f (nz+1), centres z_c with the
    two mirrored ghost centres (nz+2), dz_f (nz) and dz_c (nz+1), float64.

    Evaluated on the host (init only) and moved to `device`."""
    k = torch.linspace(0, nz, nz + 1, dtype=torch.float64)
    g = torch.tensor(gamma, dtype=torch.float64)
    if stretching_type == "bottom":
        xi = k / nz
        z_f = Lz * (1.0 - torch.tanh(gamma * (1.0 - xi)) / torch.tanh(g))
    else:
        xi = (2 * k / nz) - 1
        z_f = 0.5 * Lz * (1 + torch.tanh(gamma * xi) / torch.tanh(g))
    z_c_inn = 0.5 * (z_f[:-1] + z_f[1:])
    z_c = torch.cat([-z_c_inn[:1], z_c_inn, (2 * z_f[-1] - z_c_inn[-1]).reshape(1)])
    dz_f = z_f[1:] - z_f[:-1]
    dz_c = z_c[1:] - z_c[:-1]
    return tuple(t.to(device) for t in (z_f, z_c, dz_f, dz_c))


def field_shapes(nx, ny, nz):
    return {"u": (nx + 1, ny + 2, nz + 2), "v": (nx + 2, ny + 1, nz + 2),
            "w": (nx + 2, ny + 2, nz + 1), "p": (nx + 2, ny + 2, nz + 2)}


def compute_divergence(u, v, w, nx, ny, nz, dx, dy, dz_f):
    """utils.py:166-180 -- divergence of the staggered field, (nx, ny, nz)."""
    sh = field_shapes(nx, ny, nz)
    N.require(u, sh["u"], "u")
    N.require(v, sh["v"], "v")
    N.require(w, sh["w"], "w")
    dz = dz_f.to(device=u.device, dtype=torch.float64).contiguous()
    if dz.numel() < nz:
        raise ValueError("dz_f must have nz entries")
    div = torch.empty((nx, ny, nz), dtype=torch.float64, device=u.device)
    rc = N.lib().slc_divergence_raw(nx, ny, nz, float(dx), float(dy), N.ptr(dz), N.ptr(u),
                                    N.ptr(v), N.ptr(w), N.ptr(div), N.stream_of(u))
    N.check(rc)
    return div


def compute_bulk_velocity(u, cell_vol_ratio, total_volume):
    """utils.py:147-163 -- sum(u_int * cell_vol) / V as a 0-D device tensor.

    `cell_vol_ratio` is the solver's (nx, ny, nz) cell-volume tensor
    dx*dy*dz_f expanded over x and y (solver.py:303-306); its per-level
    column is what the kernel reads."""
    nx, ny, nz = cell_vol_ratio.shape
    N.require(u, (nx + 1, ny + 2, nz + 2), "u")
    vol_k = cell_vol_ratio[0, 0, :].to(device=u.device, dtype=torch.float64).contiguous()
    if cell_vol_ratio.stride()[:2] != (0, 0) and not torch.equal(
            cell_vol_ratio.to(vol_k.device), vol_k.view(1, 1, nz).expand(nx, ny, nz)):
        raise ValueError("cell_vol_ratio must be constant over x and y (dx*dy*dz_f)")
    scratch = torch.empty(N.lib().slc_bulk_scratch_doubles(), dtype=torch.float64, device=u.device)
    out = torch.empty((), dtype=torch.float64, device=u.device)
    rc = N.lib().slc_bulk_velocity_raw(nx, ny, nz, N.ptr(u), N.ptr(vol_k),
                                       1.0 / float(total_volume), N.ptr(scratch), N.ptr(out),
                                       N.stream_of(u))
    N.check(rc)
    return out


def save_flow_fields(u, v, w, p, z_c, z_f, Lx, Ly, step, time, u_tau, forcing, results_folder,
                     filename="fields.npz"):
    """utils.py:183-214: the reference's checkpoint, one .npz with the
    ghost-shaped u, v, w, p, the z tables, Lx, Ly, step, time, u_tau and
    forcing (tensors are copied to the host; scalars stored as 0-d arrays)."""
    import os

    def host(x):
        return x.detach().cpu().numpy() if torch.is_tensor(x) else x

    def scalar(x):
        return x.item() if torch.is_tensor(x) else x

    np.savez(os.path.join(results_folder, filename), u=host(u), v=host(v), w=host(w), p=host(p),
             z_c=host(z_c), z_f=host(z_f), Lx=Lx, Ly=Ly, step=step, time=time,
             u_tau=scalar(u_tau), forcing=scalar(forcing))


def load_flow_fields(filepath, device="cpu"):
    """utils.py:216-258: the checkpoint as a dict of tensors (u, v, w, p,
    z_c, z_f on `device`) and floats / ints (Lx, Ly, step, time, u_tau,
    forcing).  Raises FileNotFoundError for a missing file."""
    import os

    if not os.path.exists(filepath):
        raise FileNotFoundError(f"Field file not found: {filepath}")
    data = np.load(filepath)
    t = lambda k: torch.tensor(data[k], device=device)  # noqa: E731
    return {"u": t("u"), "v": t("v"), "w": t("w"), "p": t("p"), "z_c": t("z_c"), "z_f": t("z_f"),
            "Lx": float(data["Lx"]), "Ly": float(data["Ly"]), "step": int(data["step"]),
            "time": float(data["time"]), "u_tau": float(data["u_tau"]),
            "forcing": float(data["forcing"])}


def _diag_raw(u, v, w, nx, ny, nz, dx, dy, dz_f, dz_c, z_c, nu, top_wall_bc_type, Lx, Ly, Lz):
    dev = u.device
    out = torch.empty(4, dtype=torch.float64, device=dev)
    scratch = torch.empty(N.lib().slc_diagnostics_scratch_doubles(), dtype=torch.float64, device=dev)
    f = lambda t: t.to(device=dev, dtype=torch.float64).contiguous()  # noqa: E731
    dzf, dzc, zc = f(dz_f), f(dz_c), f(z_c)
    rc = N.lib().slc_diagnostics_raw(int(nx), int(ny), int(nz), float(dx), float(dy), N.ptr(dzf),
                                     N.ptr(dzc), N.ptr(zc), float(nu),
                                     1 if top_wall_bc_type == "neumann" else 0, float(Lx), float(Ly),
                                     float(Lz), N.ptr(u), N.ptr(v), N.ptr(w), N.ptr(out),
                                     N.ptr(scratch), N.stream_of(u))
    N.check(rc, None)
    return out


def compute_u_tau(u, z_c, nu, top_wall_bc_type="dirichlet"):
    """utils.py:116-144 -- friction velocity from the wall-adjacent plane
    means of u (one-sided difference to the wall), on the device; a 0-D
    tensor.  Bottom wall only for a free-slip top."""
    N.require(u, tuple(u.shape), "u")
    nx, ny, nz = u.shape[0] - 1, u.shape[1] - 2, u.shape[2] - 2
    v = torch.zeros(nx + 2, ny + 1, nz + 2, dtype=torch.float64, device=u.device)
    w = torch.zeros(nx + 2, ny + 2, nz + 1, dtype=torch.float64, device=u.device)
    ones = torch.ones(nz + 1, dtype=torch.float64, device=u.device)
    return _diag_raw(u, v, w, nx, ny, nz, 1.0, 1.0, ones[:nz], ones, z_c, nu, top_wall_bc_type,
                     1.0, 1.0, 1.0)[1]


def compute_cfl_fused(u, v, w, nx, ny, nz, dx, dy, dz_f, dz_c):
    """operators.py:839-940 -- max over cells and directions of the CFL
    inverse (|u|/dx + |v|/dy + |w|/dz with the staggered averages), one fused
    reduction on the device; returns a float (one synchronisation, as the
    reference's .item())."""
    zc = torch.ones(nz + 2, dtype=torch.float64, device=u.device)
    return float(_diag_raw(u, v, w, nx, ny, nz, dx, dy, dz_f, dz_c, zc, 1.0, "dirichlet",
                           1.0, 1.0, 1.0)[2])
