"""Initial fields for SLChannelFlow (reference: slchannel/initflow.py).

Init-time host code, so that a reference YAML config builds the same starting
field: the 'parabolic', 'vortices' and 'uniform' types of initialize_flow
(initflow.py:123-223) and the npz restart reader (initflow.py:225-286).
The synthetic turbulence-like field used by the benchmarks is in
``slchannel_b200.fields``.
"""

from __future__ import annotations

import numpy as np
import torch


def initialize_flow(nx, ny, nz, z_c, Ly, Lz, U_bulk=1.0, init_type="parabolic",
                    perturbation_intensity=0.0, n_vortices=4, device="cpu",
                    top_wall_bc_type="dirichlet"):
    """initflow.py:123-223: ghost-shaped u, v, w, p (float64) on `device`."""
    f = dict(dtype=torch.float64, device=device)
    u = torch.zeros(nx + 1, ny + 2, nz + 2, **f)
    v = torch.zeros(nx + 2, ny + 1, nz + 2, **f)
    w = torch.zeros(nx + 2, ny + 2, nz + 1, **f)
    p = torch.zeros(nx + 2, ny + 2, nz + 2, **f)
    z_c = z_c.to(**f)
    if init_type in ("parabolic", "vortices"):
        if top_wall_bc_type == "neumann":
            z_norm = z_c / Lz
            prof = 1.5 * U_bulk * z_norm * (2 - z_norm)
        else:
            z_norm = 2 * z_c / Lz - 1
            prof = 1.5 * U_bulk * (1 - z_norm**2)
        u[:, :, :] = prof[None, None, :]
    if init_type == "uniform":
        u[:, :, :] = U_bulk
    elif init_type == "vortices":
        A = perturbation_intensity * U_bulk
        ky = n_vortices * torch.pi / Ly
        y_v = torch.linspace(0, Ly, ny + 1, **f)
        y_c = 0.5 * (y_v[:-1] + y_v[1:])
        zci = z_c[1 : nz + 1]
        yy_v, zz_v = torch.meshgrid(y_v, zci, indexing="ij")
        v_pert = (-A * torch.sin(ky * yy_v) * 2 * torch.sin(torch.pi * zz_v / Lz)
                  * torch.cos(torch.pi * zz_v / Lz) * (torch.pi / Lz))
        v[1 : nx + 1, :, 1 : nz + 1] += v_pert[None, :, :]
        z_f_local = torch.cat([torch.zeros(1, **f), 0.5 * (zci[:-1] + zci[1:]),
                               torch.full((1,), float(Lz), **f)])
        yy_w, zz_w = torch.meshgrid(y_c, z_f_local, indexing="ij")
        w_pert = A * torch.cos(ky * yy_w) * ky * torch.sin(torch.pi * zz_w / Lz) ** 2
        w[1 : nx + 1, 1 : ny + 1, :] += w_pert[None, :, :]
    if perturbation_intensity > 0.0 and init_type != "vortices":
        s = perturbation_intensity * U_bulk
        u[1:-1, 1:-1, 2:-2] += (torch.rand_like(u[1:-1, 1:-1, 2:-2]) - 0.5) * 2 * s
        v[1:-1, 1:-1, 2:-2] += (torch.rand_like(v[1:-1, 1:-1, 2:-2]) - 0.5) * 2 * s
        w[1:-1, 1:-1, 2:-2] += (torch.rand_like(w[1:-1, 1:-1, 2:-2]) - 0.5) * 2 * s
    u[:, :, 0] = -u[:, :, 1]
    u[:, :, -1] = -u[:, :, -2]
    v[:, :, 0] = -v[:, :, 1]
    v[:, :, -1] = -v[:, :, -2]
    w[:, :, 0] = 0.0
    w[:, :, -1] = 0.0
    return u, v, w, p


def initialize_flow_from_file(field_file, device="cpu", reset_time=False):
    """initflow.py:225-286: (u, v, w, p, step, time) from a fields .npz
    written by save_flow_fields; the wall ghosts are re-applied as the
    reference does (u, v odd at both walls, w = 0 on both walls)."""
    from .utils import load_flow_fields

    fields = load_flow_fields(field_file, device=device)
    u, v, w, p = fields["u"], fields["v"], fields["w"], fields["p"]
    step = 0 if reset_time else int(fields["step"])
    time = 0.0 if reset_time else float(fields["time"])
    u[:, :, 0] = -u[:, :, 1]
    u[:, :, -1] = -u[:, :, -2]
    v[:, :, 0] = -v[:, :, 1]
    v[:, :, -1] = -v[:, :, -2]
    w[:, :, 0] = 0.0
    w[:, :, -1] = 0.0
    return u, v, w, p, step, time
