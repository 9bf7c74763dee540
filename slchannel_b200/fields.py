"""Seeded synthetic channel fields (host, numpy, init only).

The benchmark configurations start from: the Poiseuille profile
U(z) = 1.5 (1 - (2z/Lz - 1)^2) (= 1.5 z (2 - z) for Lz = 2), plus the curl of a
seeded random vector potential psi whose Fourier content is limited to
|k| <= kmax in integer mode numbers (m along x, n along y, l along z with
m^2 + n^2 + l^2 <= kmax^2), damped at the walls by (z (Lz - z))^2, scaled so
that the fluctuation's rms over the three components equals `urms`.  The
caller then rescales the bulk velocity and projects the field
divergence-free (SLChannelFlow.set_state + projection), as the reference does
for its own initial fields (solver.py:396-402, 593-613).

The x, y dependence is built as a half spectrum and synthesised with one
inverse real FFT per component, evaluated at each component's staggered
positions (half-cell phase shifts), so a 256^3 field takes seconds.
"""

from __future__ import annotations

import numpy as np


def _profiles(rng, kmax, Lz, mn):
    """Seeded z-profile coefficients for one (m, n) pair and the three psi
    components: list of (l, a_cos, a_sin) per component."""
    m, n = mn
    out = []
    lmax2 = kmax * kmax - m * m - n * n
    for _ in range(3):
        terms = []
        l = 0
        while l * l <= lmax2:
            k = np.sqrt(m * m + n * n + l * l)
            amp = 1.0 / (1.0 + k)
            a, b = rng.normal(size=2) * amp
            terms.append((l, a, b))
            l += 1
        out.append(terms)
    return out


def _eval_profile(terms, z, Lz):
    """S(z) = sum a cos(pi l z / Lz) + b sin(pi l z / Lz) and dS/dz."""
    S = np.zeros_like(z)
    dS = np.zeros_like(z)
    for l, a, b in terms:
        kz = np.pi * l / Lz
        c, s = np.cos(kz * z), np.sin(kz * z)
        S += a * c + b * s
        dS += kz * (-a * s + b * c)
    return S, dS


def synthetic_channel_field(nx, ny, nz, Lx, Ly, Lz, z_f, z_c, *, urms=0.1, kmax=8, seed=0,
                            U_bulk=1.0):
    """Ghost-shaped float64 (u, v, w) arrays: Poiseuille profile plus the
    curl of a seeded random vector potential, BCs applied (periodic x, y;
    u, v odd and w zero at the walls).  Not yet divergence-free on the
    discrete grid: project before stepping."""
    z_f = np.asarray(z_f, dtype=np.float64)
    z_c = np.asarray(z_c, dtype=np.float64)
    rng = np.random.default_rng(seed)
    nky = ny // 2 + 1
    kxv = 2 * np.pi * np.fft.fftfreq(nx, d=1.0 / nx) / Lx  # 2 pi m / Lx
    kyv = 2 * np.pi * np.arange(nky) / Ly
    pairs = [(m, n) for m in range(-kmax, kmax + 1) for n in range(0, kmax + 1)
             if m * m + n * n <= kmax * kmax and abs(m) < (nx + 1) // 2 and n < nky - (ny % 2 == 0)]
    prof = {mn: _profiles(rng, kmax, Lz, mn) for mn in pairs}
    phase = {mn: np.exp(2j * np.pi * rng.uniform(size=3)) for mn in pairs}

    def damp(z):
        D = (z * (Lz - z)) ** 2
        dD = 2 * z * (Lz - z) * (Lz - 2 * z)
        return D, dD

    dx, dy = Lx / nx, Ly / ny
    z_cent = z_c[1 : nz + 1]
    z_face = z_f[1:nz]

    def component(which, zpts, sx, sy):
        """Spectrum of one velocity component at z points, then synthesis."""
        D, dD = damp(zpts)
        spec = np.zeros((nx, nky, len(zpts)), dtype=np.complex128)
        for (m, n) in pairs:
            ikx = 1j * kxv[m % nx]
            iky = 1j * kyv[n]
            ps = []
            for c in range(3):
                S, dS = _eval_profile(prof[(m, n)][c], zpts, Lz)
                ps.append((phase[(m, n)][c] * D * S, phase[(m, n)][c] * (dD * S + D * dS)))
            (px, dpx), (py, dpy), (pz, dpz) = ps
            if which == "u":  # d psi_z/dy - d psi_y/dz
                val = iky * pz - dpy
            elif which == "v":  # d psi_x/dz - d psi_z/dx
                val = dpx - ikx * pz
            else:  # d psi_y/dx - d psi_x/dy
                val = ikx * py - iky * px
            shift = np.exp(1j * (kxv[m % nx] * sx + kyv[n] * sy))
            spec[m % nx, n, :] += val * shift
        return np.fft.irfft2(spec, s=(nx, ny), axes=(0, 1)) * (nx * ny)

    up = component("u", z_cent, 0.0, 0.5 * dy)  # u node (i, j): x = i dx, y = (j+1/2) dy
    vp = component("v", z_cent, 0.5 * dx, 0.0)
    wp = component("w", z_face, 0.5 * dx, 0.5 * dy)
    ms = (np.mean(up**2) + np.mean(vp**2) + np.mean(wp**2)) / 3.0
    scale = urms / np.sqrt(ms) if ms > 0 else 0.0
    up *= scale
    vp *= scale
    wp *= scale

    U = 1.5 * U_bulk * (1.0 - (2.0 * z_cent / Lz - 1.0) ** 2)
    u = np.zeros((nx + 1, ny + 2, nz + 2))
    v = np.zeros((nx + 2, ny + 1, nz + 2))
    w = np.zeros((nx + 2, ny + 2, nz + 1))
    # node (i, j) of u sits at ghost-array (i, j+1); of v at (i+1, j); of w at (i+1, j+1)
    u[0:nx, 1 : ny + 1, 1 : nz + 1] = up + U[None, None, :]
    v[1 : nx + 1, 0:ny, 1 : nz + 1] = vp
    w[1 : nx + 1, 1 : ny + 1, 1:nz] = wp
    apply_bc_numpy(u, v, w)
    return u, v, w


def apply_bc_numpy(u, v, w, top_wall_bc_type="dirichlet"):
    """Ghost cells of (u, v, w), in place (the rules of solver.py:70-107,
    written for the node rows this generator fills: u row 0, v column 0)."""
    nx = u.shape[0] - 1
    ny = v.shape[1] - 1
    # u: rows 0..nx-1 filled -> row nx is the periodic image of row 0
    u[nx] = u[0]
    u[:, 0] = u[:, ny]
    u[:, ny + 1] = u[:, 1]
    u[:, :, 0] = -u[:, :, 1]
    u[:, :, -1] = u[:, :, -2] if top_wall_bc_type == "neumann" else -u[:, :, -2]
    # v: columns 0..ny-1 filled -> column ny is the image of column 0
    v[:, ny] = v[:, 0]
    v[0] = v[nx]
    v[nx + 1] = v[1]
    v[:, :, 0] = -v[:, :, 1]
    v[:, :, -1] = v[:, :, -2] if top_wall_bc_type == "neumann" else -v[:, :, -2]
    w[0] = w[nx]
    w[nx + 1] = w[1]
    w[:, 0] = w[:, ny]
    w[:, ny + 1] = w[:, 1]
    w[:, :, 0] = 0.0
    w[:, :, -1] = 0.0
