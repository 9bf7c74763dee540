"""The synthetic initial-field generator (host code): seeded, BC-consistent,
scaled to the requested fluctuation rms, Poiseuille mean.  CPU only."""

import numpy as np

from oracle.slbdf2 import apply_bc_all, compute_divergence, generate_grid
from slchannel_b200.fields import synthetic_channel_field


def test_field_generator_properties():
    nx, ny, nz, Lx, Ly, Lz = 24, 16, 20, 2 * np.pi, np.pi, 2.0
    z_f, z_c, dz_f, _ = generate_grid(2.0, nz, Lz)
    u, v, w = synthetic_channel_field(nx, ny, nz, Lx, Ly, Lz, z_f, z_c, urms=0.1, seed=3)
    u2, v2, w2 = synthetic_channel_field(nx, ny, nz, Lx, Ly, Lz, z_f, z_c, urms=0.1, seed=3)
    assert np.array_equal(u, u2) and np.array_equal(w, w2)
    # BC-consistent: re-applying the reference BCs changes nothing
    uc, vc, wc = u.copy(), v.copy(), w.copy()
    apply_bc_all(uc, vc, wc)
    assert np.abs(uc - u).max() < 1e-15 and np.abs(vc - v).max() < 1e-15 and np.abs(wc - w).max() < 1e-15
    U = 1.5 * (1 - (2 * z_c[1:-1] / Lz - 1) ** 2)
    up = u[1 : nx + 1, 1 : ny + 1, 1 : nz + 1] - U
    rms = np.sqrt((np.mean(up**2) + np.mean(v[1:nx+1, 1:ny+1, 1:nz+1] ** 2)
                   + np.mean(w[1:nx+1, 1:ny+1, 1:nz] ** 2)) / 3)
    assert abs(rms - 0.1) < 0.02
    # the curl of a smooth potential is nearly divergence-free already
    div = compute_divergence(u, v, w, nx, ny, nz, Lx / nx, Ly / ny, dz_f)
    assert np.abs(div).max() < 0.5
