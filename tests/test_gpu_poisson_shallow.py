"""slc_project (divergence -> rfft2 -> two-ended tridiagonal sweep per
spectral column -> irfft2 -> gradient correction) against the oracle's
projection (projection.py:133-272) on shallow grids, where the sweeps' meeting
row nz/2 sits next to a wall row: nz = 3, 4, 5, 7, with odd ny, from random
BC-consistent fields (large divergence).  Velocity and pressure to 1e-11
relative, divergence after projection at round-off."""

import math

import numpy as np
import pytest
import torch
from helpers import rel_err

from oracle.slbdf2 import OracleChannel, compute_divergence
from slchannel_b200 import _native as N
from slchannel_b200.utils import generate_grid

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nx,ny,nz", [(8, 6, 3), (6, 7, 4), (10, 7, 5), (9, 12, 7)])
def test_projection_shallow(nx, ny, nz):
    Lx, Ly, Lz, gamma = 2 * math.pi, math.pi, 2.0, 1.5
    z_f, z_c, dz_f, dz_c = (t.numpy() for t in generate_grid(gamma, nz, Lz))
    rng = np.random.default_rng(100 + nz)
    u = rng.standard_normal((nx + 1, ny + 2, nz + 2))
    v = rng.standard_normal((nx + 2, ny + 1, nz + 2))
    w = rng.standard_normal((nx + 2, ny + 2, nz + 1))
    ch = OracleChannel(nx, ny, nz, Lx, Ly, Lz, gamma, 1e-3, u, v, w, order=4, z_f=z_f, z_c=z_c)
    ch.apply_bc()
    dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (ch.u, ch.v, ch.w)]
    dp = torch.zeros((nx + 2, ny + 2, nz + 2), dtype=torch.float64, device="cuda")
    div0 = np.abs(ch.divergence()).max()
    ch.project_initial()

    g = N.Grid(nx, ny, nz, Lx, Ly, Lz, gamma, z_f, z_c, order=4, device="cuda")
    g.call("slc_project", *[N.ptr(t) for t in dev], N.ptr(dp), 1.0, 1.0, N.stream_of(dp))
    torch.cuda.synchronize()
    for name, a, b in zip("uvw", dev, (ch.u, ch.v, ch.w)):
        assert rel_err(a.cpu().numpy(), b) < 1e-11, name
    assert rel_err(dp.cpu().numpy(), ch.p) < 1e-11
    uu, vv, ww = (t.cpu().numpy() for t in dev)
    div = compute_divergence(uu, vv, ww, nx, ny, nz, Lx / nx, Ly / ny, dz_f)
    assert np.abs(div).max() < 1e-12 * max(div0, 1.0)
    g.close()
