"""TEST INFRASTRUCTURE ONLY -- numpy restatement of slChannel's SL-BDF2 step.

Follows gmcavallazzi/SLchannel v1.0.1 (paths relative to that project):

* grid                     slchannel/utils.py:21-61
* node buffers / advector  slchannel/semilag.py:102-127, 133-381, 387-394, 584-671
  (the per-point trace and gather are in ``sl_oracle.c``)
* boundary conditions      slchannel/solver.py:70-107
* explicit xy-diffusion    slchannel/operators.py:293-367
* implicit z-diffusion     slchannel/operators.py:382-630 with tridiag.py:36-61 (PCR)
* divergence, bulk         slchannel/utils.py:147-180
* FFT Poisson + projection slchannel/projection.py:24-272
* BDF1 bootstrap, BDF2     slchannel/solver.py:694-1018

Arrays are numpy float64 in the reference's ghost-shaped layouts:
u (nx+1, ny+2, nz+2), v (nx+2, ny+1, nz+2), w (nx+2, ny+2, nz+1),
p (nx+2, ny+2, nz+2), z contiguous.
"""

from __future__ import annotations

import ctypes
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libslc_oracle.so")
_MAX_ORDER = 6


# ---------------------------------------------------------------------------
# C library (sl_oracle.c)
# ---------------------------------------------------------------------------


class _Spec(ctypes.Structure):
    _fields_ = [
        ("NX", ctypes.c_int64),
        ("NY", ctypes.c_int64),
        ("NZ", ctypes.c_int64),
        ("shift_x", ctypes.c_double),
        ("shift_y", ctypes.c_double),
        ("centers", ctypes.c_int32),
        ("pad_", ctypes.c_int32),
        ("znodes", ctypes.c_void_p),
        ("dinv", ctypes.c_void_p * (_MAX_ORDER + 1)),
    ]


class _Grid(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int64),
        ("ny", ctypes.c_int64),
        ("nz", ctypes.c_int64),
        ("dx", ctypes.c_double),
        ("dy", ctypes.c_double),
        ("Lz", ctypes.c_double),
        ("gamma", ctypes.c_double),
        ("tanh_g", ctypes.c_double),
        ("z_lo", ctypes.c_double),
        ("z_hi", ctypes.c_double),
        ("symmetric", ctypes.c_int32),
        ("n_traj_iters", ctypes.c_int32),
        ("traj_order", ctypes.c_int32),
        ("order", ctypes.c_int32),
        ("udenom", (ctypes.c_double * _MAX_ORDER) * (_MAX_ORDER + 1)),
        ("z_c", ctypes.c_void_p),
        ("z_f", ctypes.c_void_p),
        ("spec", _Spec * 3),
    ]


_lib = None


def build_library(force=False):
    """Compile sl_oracle.c with oracle/Makefile (gcc, seconds)."""
    if force or not os.path.exists(_LIB_PATH):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def _load():
    global _lib
    if _lib is not None:
        return _lib
    build_library()
    lib = ctypes.CDLL(_LIB_PATH)
    P = ctypes.c_void_p
    i64 = ctypes.c_int64
    lib.orc_set_threads.argtypes = [ctypes.c_int]
    lib.orc_max_threads.restype = ctypes.c_int
    lib.orc_face_coord.argtypes = [P, P, i64, P]
    lib.orc_interp.argtypes = [P, ctypes.c_int, ctypes.c_int, P, P, P, P, i64, ctypes.c_int, P]
    lib.orc_interp.restype = i64
    lib.orc_departure.argtypes = [P, ctypes.c_int, P, P, P, ctypes.c_double, P, P, P]
    lib.orc_advect_comp.argtypes = [P, ctypes.c_int, P, P, P, P, ctypes.c_double, P]
    lib.orc_advect_comp.restype = i64
    lib.orc_advect_comp_range.argtypes = [
        P, ctypes.c_int, P, P, P, P, ctypes.c_double, i64, i64, P,
    ]
    lib.orc_advect_comp_range.restype = i64
    lib.orc_n_arrival.argtypes = [P, ctypes.c_int]
    lib.orc_n_arrival.restype = i64
    lib.orc_pcr_batch.argtypes = [P, P, P, P, i64, ctypes.c_int]
    lib.orc_pcr_batch.restype = ctypes.c_int
    _lib = lib
    return lib


def set_threads(n):
    """Number of POSIX threads the C oracle uses (0 = all online CPUs)."""
    _load().orc_set_threads(int(n))


def max_threads():
    return int(_load().orc_max_threads())


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


# ---------------------------------------------------------------------------
# Grid (utils.py:21-61)
# ---------------------------------------------------------------------------


def generate_grid(gamma, nz, Lz, stretching_type="symmetric"):
    """utils.py:21-61 -- tanh-stretched faces z_f (nz+1), centres z_c with the
    two mirrored ghosts (nz+2), dz_f (nz), dz_c (nz+1)."""
    k = np.arange(nz + 1, dtype=np.float64)
    if stretching_type == "bottom":
        xi = k / nz
        z_f = Lz * (1.0 - np.tanh(gamma * (1.0 - xi)) / np.tanh(np.float64(gamma)))
    else:
        xi = (2 * k / nz) - 1
        z_f = 0.5 * Lz * (1 + np.tanh(gamma * xi) / np.tanh(np.float64(gamma)))
    z_c_inn = 0.5 * (z_f[:-1] + z_f[1:])
    z_c = np.concatenate([[-z_c_inn[0]], z_c_inn, [2 * z_f[-1] - z_c_inn[-1]]])
    dz_f = z_f[1:] - z_f[:-1]
    dz_c = z_c[1:] - z_c[:-1]
    return z_f, z_c, dz_f, dz_c


def z_denominator_table(znodes, order):
    """semilag.py:102-114 -- denom_inv[b, m] = 1 / prod_{l != m}(z[b+m] - z[b+l])."""
    znodes = np.asarray(znodes, dtype=np.float64)
    nb = len(znodes) - order + 1
    zn = np.stack([znodes[m : m + nb] for m in range(order)], axis=1)  # (nb, order)
    diff = zn[:, :, None] - zn[:, None, :] + np.eye(order)[None]
    prod = diff[:, :, 0].copy()
    for l in range(1, order):
        prod = prod * diff[:, :, l]
    return np.ascontiguousarray(1.0 / prod)


def uniform_inv_denominators(order):
    """semilag.py:117-127."""
    offs = [m - (order // 2 - 1) for m in range(order)]
    inv = []
    for m in range(order):
        d = 1.0
        for l in range(order):
            if l != m:
                d *= offs[m] - offs[l]
        inv.append(1.0 / d)
    return inv


# ---------------------------------------------------------------------------
# Advector (semilag.py)
# ---------------------------------------------------------------------------


class OracleAdvector:
    """semilag.py:133-381 SLAdvector, float64 eager path.  The per-point work
    (trace, stencil, gather) runs in sl_oracle.c."""

    def __init__(self, nx, ny, nz, dx, dy, Lx, Ly, Lz, z_f, z_c, gamma,
                 stretching_type="symmetric", order=4, traj_order=2, n_traj_iters=2):
        if order not in (4, 6):
            raise ValueError(f"sl.interp_order must be 4 (tricubic) or 6 (triquintic), got {order}")
        if traj_order not in (2, 4):
            raise ValueError(f"sl.traj_interp_order must be 2 or 4, got {traj_order}")
        if stretching_type not in ("symmetric", "bottom"):
            raise ValueError(f"unsupported stretching '{stretching_type}'")
        if nz + 1 < order:
            raise ValueError(f"nz={nz} too small for interpolation order {order}")
        self.nx, self.ny, self.nz = nx, ny, nz
        self.dx, self.dy = dx, dy
        self.Lx, self.Ly, self.Lz = Lx, Ly, Lz
        self.gamma = float(gamma)
        self.stretching_type = stretching_type
        self.order, self.traj_order, self.n_traj_iters = order, traj_order, n_traj_iters
        self.z_f = np.ascontiguousarray(z_f, dtype=np.float64)
        self.z_c = np.ascontiguousarray(z_c, dtype=np.float64)
        self.tanh_g = math.tanh(self.gamma)
        eps_z = 1e-12 * Lz  # semilag.py:244-247
        self.z_lo = float(self.z_f[0] + eps_z)
        self.z_hi = float(self.z_f[-1] - eps_z)
        # semilag.py:282-286: u, v on centres (ghosts incl.), w on faces
        self._specs = {
            "u": (0.0, -0.5, self.z_c, 1),
            "v": (-0.5, 0.0, self.z_c, 1),
            "w": (-0.5, -0.5, self.z_f, 0),
        }
        orders = sorted({2, traj_order, order})
        self._keep = []
        g = _Grid()
        g.nx, g.ny, g.nz = nx, ny, nz
        g.dx, g.dy, g.Lz = dx, dy, Lz
        g.gamma, g.tanh_g, g.z_lo, g.z_hi = self.gamma, self.tanh_g, self.z_lo, self.z_hi
        g.symmetric = 1 if stretching_type == "symmetric" else 0
        g.n_traj_iters, g.traj_order, g.order = n_traj_iters, traj_order, order
        for o in orders:
            for m, val in enumerate(uniform_inv_denominators(o)):
                g.udenom[o][m] = val
        g.z_c = self.z_c.ctypes.data
        g.z_f = self.z_f.ctypes.data
        self.denoms = {}
        for ic, c in enumerate("uvw"):
            sx, sy, zn, centers = self._specs[c]
            s = g.spec[ic]
            s.NX, s.NY, s.NZ = nx, ny, len(zn)
            s.shift_x, s.shift_y, s.centers = sx, sy, centers
            s.znodes = zn.ctypes.data
            self.denoms[c] = {}
            for o in orders:
                t = z_denominator_table(zn, o)
                self._keep.append(t)
                self.denoms[c][o] = t
                s.dinv[o] = t.ctypes.data
        self._g = g
        self._gp = ctypes.byref(g)
        self.n_clamped_last = 0

    # semilag.py:387-394
    def fill(self, comp, field):
        nx, ny = self.nx, self.ny
        if comp == "u":
            return np.ascontiguousarray(field[0:nx, 1 : ny + 1, :])
        if comp == "v":
            return np.ascontiguousarray(field[1 : nx + 1, 0:ny, :])
        return np.ascontiguousarray(field[1 : nx + 1, 1 : ny + 1, :])

    def arrival_shape(self, comp):
        return (self.nx, self.ny, self.nz - 1 if comp == "w" else self.nz)

    def arrival_coords(self, comp):
        """semilag.py:292-307, broadcast to the full arrival shape."""
        nx, ny, nz, dx, dy = self.nx, self.ny, self.nz, self.dx, self.dy
        ar = np.arange(1, nx + 1, dtype=np.float64)
        aj = np.arange(1, ny + 1, dtype=np.float64)
        if comp == "u":
            x, y, z = ar * dx, (aj - 0.5) * dy, self.z_c[1 : nz + 1]
        elif comp == "v":
            x, y, z = (ar - 0.5) * dx, aj * dy, self.z_c[1 : nz + 1]
        else:
            x, y, z = (ar - 0.5) * dx, (aj - 0.5) * dy, self.z_f[1:nz]
        X, Y, Z = np.broadcast_arrays(x[:, None, None], y[None, :, None], z[None, None, :])
        return X.copy(), Y.copy(), Z.copy()

    def face_coord(self, z):
        """semilag.py:400-411."""
        z = np.ascontiguousarray(z, dtype=np.float64).ravel()
        out = np.empty_like(z)
        _load().orc_face_coord(self._gp, _ptr(z), z.size, _ptr(out))
        return out

    def interp(self, comp, order, buf, x, y, z, count_clamp=False):
        """semilag.py:460-510 _build_iw + _apply_iw at arbitrary points.
        Returns (values, n_clamped)."""
        buf = np.ascontiguousarray(buf, dtype=np.float64)
        x, y, z = (np.ascontiguousarray(a, dtype=np.float64).ravel() for a in (x, y, z))
        out = np.empty_like(x)
        ncl = _load().orc_interp(self._gp, "uvw".index(comp), order, _ptr(buf), _ptr(x),
                                 _ptr(y), _ptr(z), x.size, int(count_clamp), _ptr(out))
        return out, int(ncl)

    def departure_from_bufs(self, comp, mbufs, dt):
        """semilag.py:534-552 with the trajectory node buffers given."""
        mb = [np.ascontiguousarray(mbufs[c], dtype=np.float64) for c in "uvw"]
        shape = self.arrival_shape(comp)
        xd, yd, zd = (np.empty(shape) for _ in range(3))
        _load().orc_departure(self._gp, "uvw".index(comp), _ptr(mb[0]), _ptr(mb[1]),
                              _ptr(mb[2]), float(dt), _ptr(xd), _ptr(yd), _ptr(zd))
        return xd, yd, zd

    def departure_coords(self, comp, u_mid, v_mid, w_mid, dt):
        mbufs = {c: self.fill(c, f) for c, f in zip("uvw", (u_mid, v_mid, w_mid))}
        return self.departure_from_bufs(comp, mbufs, dt)

    def advect_comp(self, comp, fbuf, mbufs, dt, p0=0, p1=None):
        """semilag.py:560-571 for arrival points [p0, p1) of `comp` (flat,
        z fastest).  Returns (values, n_clamped)."""
        lib = _load()
        ic = "uvw".index(comp)
        n = lib.orc_n_arrival(self._gp, ic)
        p1 = n if p1 is None else p1
        out = np.empty(p1 - p0)
        ncl = lib.orc_advect_comp_range(self._gp, ic, _ptr(fbuf), _ptr(mbufs["u"]),
                                        _ptr(mbufs["v"]), _ptr(mbufs["w"]), float(dt),
                                        int(p0), int(p1), _ptr(out))
        return out, int(ncl)

    def advect(self, u, v, w, u_mid, v_mid, w_mid, dt):
        """semilag.py:584-671.  Returns fresh ghost-shaped (ustar, vstar,
        wstar) with the interiors filled and zero ghosts; the clamp count of
        the call is left in n_clamped_last."""
        nx, ny, nz = self.nx, self.ny, self.nz
        mbufs = {c: self.fill(c, f) for c, f in zip("uvw", (u_mid, v_mid, w_mid))}
        outs = {
            "u": np.zeros((nx + 1, ny + 2, nz + 2)),
            "v": np.zeros((nx + 2, ny + 1, nz + 2)),
            "w": np.zeros((nx + 2, ny + 2, nz + 1)),
        }
        ncl = 0
        for comp, f in zip("uvw", (u, v, w)):
            vals, c = self.advect_comp(comp, self.fill(comp, f), mbufs, dt)
            ncl += c
            shape = self.arrival_shape(comp)
            if comp == "w":
                outs["w"][1 : nx + 1, 1 : ny + 1, 1:nz] = vals.reshape(shape)
            else:
                outs[comp][1 : nx + 1, 1 : ny + 1, 1 : nz + 1] = vals.reshape(shape)
        self.n_clamped_last = ncl
        return outs["u"], outs["v"], outs["w"]


# ---------------------------------------------------------------------------
# Boundary conditions and operators
# ---------------------------------------------------------------------------


def apply_bc_all(u, v, w, top_wall_bc_type="dirichlet"):
    """solver.py:70-107, in place."""
    u[0, :, :] = u[-1, :, :]
    u[:, 0, :] = u[:, -2, :]
    u[:, -1, :] = u[:, 1, :]
    u[:, :, 0] = -u[:, :, 1]
    u[:, :, -1] = u[:, :, -2] if top_wall_bc_type == "neumann" else -u[:, :, -2]
    v[0, :, :] = v[-2, :, :]
    v[-1, :, :] = v[1, :, :]
    v[:, 0, :] = v[:, -1, :]
    v[:, :, 0] = -v[:, :, 1]
    v[:, :, -1] = v[:, :, -2] if top_wall_bc_type == "neumann" else -v[:, :, -2]
    w[0, :, :] = w[-2, :, :]
    w[-1, :, :] = w[1, :, :]
    w[:, 0, :] = w[:, -2, :]
    w[:, -1, :] = w[:, 1, :]
    w[:, :, 0] = 0.0
    w[:, :, -1] = 0.0


def diffusion_xy(comp, f, nx, ny, nz, dx, dy, nu):
    """operators.py:293-367 (diffusion_xy_u / _v / _w): nu*(dxx + dyy) on the
    interior, zero ghosts."""
    out = np.zeros_like(f)
    if comp == "u":
        ext = np.concatenate([f, f[1:2]], axis=0)
        d2x = (ext[2 : nx + 2, 1 : ny + 1, 1 : nz + 1] - 2 * ext[1 : nx + 1, 1 : ny + 1, 1 : nz + 1]
               + ext[0:nx, 1 : ny + 1, 1 : nz + 1]) / dx**2
        d2y = (f[1 : nx + 1, 2 : ny + 2, 1 : nz + 1] - 2 * f[1 : nx + 1, 1 : ny + 1, 1 : nz + 1]
               + f[1 : nx + 1, 0:ny, 1 : nz + 1]) / dy**2
        out[1 : nx + 1, 1 : ny + 1, 1 : nz + 1] = nu * (d2x + d2y)
    elif comp == "v":
        d2x = (f[2 : nx + 2, 1 : ny + 1, 1 : nz + 1] - 2 * f[1 : nx + 1, 1 : ny + 1, 1 : nz + 1]
               + f[0:nx, 1 : ny + 1, 1 : nz + 1]) / dx**2
        ext = np.concatenate([f, f[:, 1:2]], axis=1)
        d2y = (ext[1 : nx + 1, 2 : ny + 2, 1 : nz + 1] - 2 * ext[1 : nx + 1, 1 : ny + 1, 1 : nz + 1]
               + ext[1 : nx + 1, 0:ny, 1 : nz + 1]) / dy**2
        out[1 : nx + 1, 1 : ny + 1, 1 : nz + 1] = nu * (d2x + d2y)
    else:
        d2x = (f[2 : nx + 2, 1 : ny + 1, 1:nz] - 2 * f[1 : nx + 1, 1 : ny + 1, 1:nz]
               + f[0:nx, 1 : ny + 1, 1:nz]) / (dx**2)
        d2y = (f[1 : nx + 1, 2 : ny + 2, 1:nz] - 2 * f[1 : nx + 1, 1 : ny + 1, 1:nz]
               + f[1 : nx + 1, 0:ny, 1:nz]) / (dy**2)
        out[1 : nx + 1, 1 : ny + 1, 1:nz] = nu * (d2x + d2y)
    return out


def _shift(x, s, down, fill):
    """tridiag.py:23-33."""
    n = x.shape[-1]
    y = np.full_like(x, fill)
    if s < n:
        if down:
            y[..., s:] = x[..., : n - s]
        else:
            y[..., : n - s] = x[..., s:]
    return y


def pcr_solve(a, b, c, d):
    """tridiag.py:36-61 -- parallel cyclic reduction, 1-D diagonals shared by
    the batch, RHS (batch, n).  A (batch, n) float64 right-hand side goes to
    the C restatement (the same operations in the same order on all host
    threads, bit-identical to pcr_solve_numpy); anything else to numpy."""
    if d.ndim == 2 and d.dtype == np.float64 and a.ndim == b.ndim == c.ndim == 1:
        n = d.shape[-1]
        out = np.array(d, dtype=np.float64, order="C", copy=True)
        da, db, dc = (np.ascontiguousarray(x, dtype=np.float64) for x in (a, b, c))
        if da.shape[0] == db.shape[0] == dc.shape[0] == n:
            rc = _load().orc_pcr_batch(_ptr(da), _ptr(db), _ptr(dc), _ptr(out), out.shape[0], n)
            if rc != 0:
                raise RuntimeError(f"orc_pcr_batch failed ({rc})")
            return out
    return pcr_solve_numpy(a, b, c, d)


def pcr_solve_numpy(a, b, c, d):
    """tridiag.py:36-61 in numpy, any batch shape."""
    n = d.shape[-1]
    a, b, c, d = a.copy(), b.copy(), c.copy(), d.copy()
    s = 1
    while s < n:
        a_dn = _shift(a, s, True, 0.0)
        b_dn = _shift(b, s, True, 1.0)
        c_dn = _shift(c, s, True, 0.0)
        a_up = _shift(a, s, False, 0.0)
        b_up = _shift(b, s, False, 1.0)
        c_up = _shift(c, s, False, 0.0)
        d_dn = _shift(d, s, True, 0.0)
        d_up = _shift(d, s, False, 0.0)
        alpha = -a / b_dn
        gamma = -c / b_up
        b = b + alpha * c_dn + gamma * a_up
        d = d + alpha * d_dn + gamma * d_up
        a = alpha * a_dn
        c = gamma * c_up
        s *= 2
    return d / b


def zsolve_coefficients(comp, dt, nz, dz_c, dz_f, nu, theta=1.0, top_wall_bc_type="dirichlet"):
    """operators.py:382-630 -- the three diagonals of (I - theta dt nu Dzz),
    with the wall closures, for component `comp`."""
    alpha = theta * dt * nu
    if comp in ("u", "v"):
        dz_left, dz_right, dz_cell = dz_c[0:nz], dz_c[1 : nz + 1], dz_f[0:nz]
        lower = -alpha / (dz_left * dz_cell)
        center = 1.0 + alpha * (1.0 / dz_left + 1.0 / dz_right) / dz_cell
        upper = -alpha / (dz_right * dz_cell)
        a, b, c = lower.copy(), center.copy(), upper.copy()
        a[0] = 0.0
        b[0] = center[0] - lower[0]
        if top_wall_bc_type == "neumann":
            b[nz - 1] = center[nz - 1] + upper[nz - 1]
        else:
            b[nz - 1] = center[nz - 1] - upper[nz - 1]
        c[nz - 1] = 0.0
    else:
        ni = nz - 1
        dz_left, dz_right, dz_cv = dz_f[0:ni], dz_f[1:nz], dz_c[1:nz]
        lower = -alpha / (dz_left * dz_cv)
        center = 1.0 + alpha * (1.0 / dz_left + 1.0 / dz_right) / dz_cv
        upper = -alpha / (dz_right * dz_cv)
        a, b, c = lower.copy(), center.copy(), upper.copy()
        a[0] = 0.0
        c[ni - 1] = 0.0
    return a, b, c


def cn_explicit(comp, f, dt, nx, ny, nz, dz_c, dz_f, nu, theta, top_wall_bc_type="dirichlet"):
    """operators.py:443-461, 610-622 -- (1 - theta) dt nu d2f/dz2 on the
    interior unknowns, with the reference's wall closures (for w, its stencil
    on faces m - 1, m, m + 1 for unknown m)."""
    beta = (1.0 - theta) * dt * nu
    if comp in ("u", "v"):
        dl, dr, dc = dz_c[0:nz], dz_c[1 : nz + 1], dz_f[0:nz]
        F = f[1 : nx + 1, 1 : ny + 1, :]
        d2 = ((F[:, :, 2 : nz + 2] - F[:, :, 1 : nz + 1]) / dr - (F[:, :, 1 : nz + 1] - F[:, :, 0:nz]) / dl) / dc
        d2[:, :, 0] = ((F[:, :, 2] - F[:, :, 1]) / dr[0] - 2.0 * F[:, :, 1] / dl[0]) / dc[0]
        if top_wall_bc_type == "neumann":
            d2[:, :, nz - 1] = (-(F[:, :, nz] - F[:, :, nz - 1]) / dl[nz - 1]) / dc[nz - 1]
        else:
            d2[:, :, nz - 1] = (-2.0 * F[:, :, nz] / dr[nz - 1]
                                - (F[:, :, nz] - F[:, :, nz - 1]) / dl[nz - 1]) / dc[nz - 1]
    else:
        ni = nz - 1
        dl, dr, dcv = dz_f[0:ni], dz_f[1:nz], dz_c[1:nz]
        W = f[1 : nx + 1, 1 : ny + 1, :]
        d2 = np.empty((nx, ny, ni))
        d2[:, :, 1 : ni - 1] = ((W[:, :, 2:ni] - W[:, :, 1 : ni - 1]) / dr[1 : ni - 1]
                                - (W[:, :, 1 : ni - 1] - W[:, :, 0 : ni - 2]) / dl[1 : ni - 1]) / dcv[1 : ni - 1]
        d2[:, :, 0] = ((W[:, :, 1] - W[:, :, 0]) / dr[0] - W[:, :, 0] / dl[0]) / dcv[0]
        d2[:, :, ni - 1] = (-W[:, :, ni - 1] / dr[ni - 1]
                            - (W[:, :, ni - 1] - W[:, :, ni - 2]) / dl[ni - 1]) / dcv[ni - 1]
    return beta * d2


def solve_implicit_diffusion(comp, f, dt, nx, ny, nz, dz_c, dz_f, nu, theta=1.0,
                             top_wall_bc_type="dirichlet"):
    """operators.py:382-630: returns a new array whose interior solves
    (I - theta dt nu Dzz) f_new = f + (1 - theta) dt nu Dzz f."""
    a, b, c = zsolve_coefficients(comp, dt, nz, dz_c, dz_f, nu, theta, top_wall_bc_type)
    out = f.copy()
    if comp in ("u", "v"):
        d = f[1 : nx + 1, 1 : ny + 1, 1 : nz + 1].copy()
        if theta < 1.0:
            d += cn_explicit(comp, f, dt, nx, ny, nz, dz_c, dz_f, nu, theta, top_wall_bc_type)
        out[1 : nx + 1, 1 : ny + 1, 1 : nz + 1] = pcr_solve(a, b, c, d.reshape(nx * ny, nz)).reshape(nx, ny, nz)
    else:
        d = f[1 : nx + 1, 1 : ny + 1, 1:nz].copy()
        if theta < 1.0:
            d += cn_explicit(comp, f, dt, nx, ny, nz, dz_c, dz_f, nu, theta)
        out[1 : nx + 1, 1 : ny + 1, 1:nz] = pcr_solve(a, b, c, d.reshape(nx * ny, nz - 1)).reshape(nx, ny, nz - 1)
    return out


def momentum_rhs_imex(u, v, w, nx, ny, nz, dx, dy, dz_c, dz_f, nu):
    """operators.py:638-832 -- explicit x,y diffusion minus flux-form
    advection of u, v, w on the interiors (ghosts zero)."""
    ru, rv, rw = np.zeros_like(u), np.zeros_like(v), np.zeros_like(w)
    dxi, dyi = 1.0 / dx, 1.0 / dy
    nudx2, nudy2 = nu * (1.0 / (dx * dx)), nu * (1.0 / (dy * dy))
    dzfi = (1.0 / dz_f)[None, None, :]
    X = slice(1, nx + 1)
    Y = slice(1, ny + 1)
    Z = slice(1, nz + 1)
    ue = np.concatenate([u, u[1:2]], axis=0)
    ui = 0.5 * (ue[1 : nx + 1, Y, Z] + ue[2 : nx + 2, Y, Z])
    uu_r = ui * ui
    ui = 0.5 * (ue[0:nx, Y, Z] + ue[1 : nx + 1, Y, Z])
    duudx = (uu_r - ui * ui) * dxi
    vi = 0.5 * (v[X, Y, Z] + v[2 : nx + 2, Y, Z])
    uy = 0.5 * (ue[X, Y, Z] + ue[X, 2 : ny + 2, Z])
    vu_t = vi * uy
    vi = 0.5 * (v[X, 0:ny, Z] + v[2 : nx + 2, 0:ny, Z])
    uy = 0.5 * (ue[X, 0:ny, Z] + ue[X, Y, Z])
    dvudy = (vu_t - vi * uy) * dyi
    wi = 0.5 * (w[X, Y, 1 : nz + 1] + w[2 : nx + 2, Y, 1 : nz + 1])
    uz = 0.5 * (ue[X, Y, Z] + ue[X, Y, 2 : nz + 2])
    wu_t = wi * uz
    wi = 0.5 * (w[X, Y, 0:nz] + w[2 : nx + 2, Y, 0:nz])
    uz = 0.5 * (ue[X, Y, 0:nz] + ue[X, Y, Z])
    dwudz = (wu_t - wi * uz) * dzfi
    adv = duudx + dvudy + dwudz
    d2x = (ue[2 : nx + 2, Y, Z] - 2.0 * ue[X, Y, Z] + ue[0:nx, Y, Z]) * nudx2
    d2y = (u[X, 2 : ny + 2, Z] - 2.0 * u[X, Y, Z] + u[X, 0:ny, Z]) * nudy2
    ru[X, Y, Z] = (d2x + d2y) - adv
    ve = np.concatenate([v, v[:, 1:2]], axis=1)
    ui = 0.5 * (u[X, Y, Z] + u[X, 2 : ny + 2, Z])
    vx = 0.5 * (ve[X, Y, Z] + ve[2 : nx + 2, Y, Z])
    uv_r = ui * vx
    ui = 0.5 * (u[0:nx, Y, Z] + u[0:nx, 2 : ny + 2, Z])
    vx = 0.5 * (ve[0:nx, Y, Z] + ve[X, Y, Z])
    duvdx = (uv_r - ui * vx) * dxi
    vi = 0.5 * (ve[X, Y, Z] + ve[X, 2 : ny + 2, Z])
    vv_t = vi * vi
    vi = 0.5 * (ve[X, 0:ny, Z] + ve[X, Y, Z])
    dvvdy = (vv_t - vi * vi) * dyi
    wi = 0.5 * (w[X, Y, 1 : nz + 1] + w[X, 2 : ny + 2, 1 : nz + 1])
    vz = 0.5 * (ve[X, Y, Z] + ve[X, Y, 2 : nz + 2])
    wv_t = wi * vz
    wi = 0.5 * (w[X, Y, 0:nz] + w[X, 2 : ny + 2, 0:nz])
    vz = 0.5 * (ve[X, Y, 0:nz] + ve[X, Y, Z])
    dwvdz = (wv_t - wi * vz) * dzfi
    adv = duvdx + dvvdy + dwvdz
    d2x = (v[2 : nx + 2, Y, Z] - 2.0 * v[X, Y, Z] + v[0:nx, Y, Z]) * nudx2
    d2y = (ve[X, 2 : ny + 2, Z] - 2.0 * ve[X, Y, Z] + ve[X, 0:ny, Z]) * nudy2
    rv[X, Y, Z] = (d2x + d2y) - adv
    W = slice(1, nz)
    ui = 0.5 * (u[X, Y, 1:nz] + u[X, Y, 2 : nz + 1])
    wx = 0.5 * (w[X, Y, W] + w[2 : nx + 2, Y, W])
    uw_r = ui * wx
    ui = 0.5 * (u[0:nx, Y, 1:nz] + u[0:nx, Y, 2 : nz + 1])
    wx = 0.5 * (w[0:nx, Y, W] + w[X, Y, W])
    duwdx = (uw_r - ui * wx) * dxi
    vi = 0.5 * (v[X, Y, 1:nz] + v[X, Y, 2 : nz + 1])
    wy = 0.5 * (w[X, Y, W] + w[X, 2 : ny + 2, W])
    vw_t = vi * wy
    vi = 0.5 * (v[X, 0:ny, 1:nz] + v[X, 0:ny, 2 : nz + 1])
    wy = 0.5 * (w[X, 0:ny, W] + w[X, Y, W])
    dvwdy = (vw_t - vi * wy) * dyi
    wi = 0.5 * (w[X, Y, 1:nz] + w[X, Y, 2 : nz + 1])
    ww_t = wi * wi
    wi = 0.5 * (w[X, Y, 0 : nz - 1] + w[X, Y, 1:nz])
    dwwdz = (ww_t - wi * wi) / dz_c[1:nz][None, None, :]
    adv = duwdx + dvwdy + dwwdz
    d2x = (w[2 : nx + 2, Y, W] - 2.0 * w[X, Y, W] + w[0:nx, Y, W]) * nudx2
    d2y = (w[X, 2 : ny + 2, W] - 2.0 * w[X, Y, W] + w[X, 0:ny, W]) * nudy2
    rw[X, Y, W] = (d2x + d2y) - adv
    return ru, rv, rw


def compute_divergence(u, v, w, nx, ny, nz, dx, dy, dz_f):
    """utils.py:166-180."""
    du = (u[1 : nx + 1, 1 : ny + 1, 1 : nz + 1] - u[0:nx, 1 : ny + 1, 1 : nz + 1]) / dx
    dv = (v[1 : nx + 1, 1 : ny + 1, 1 : nz + 1] - v[1 : nx + 1, 0:ny, 1 : nz + 1]) / dy
    dw = (w[1 : nx + 1, 1 : ny + 1, 1 : nz + 1] - w[1 : nx + 1, 1 : ny + 1, 0:nz]) / dz_f[0:nz]
    return du + dv + dw


def compute_bulk_velocity(u, nx, ny, nz, dx, dy, dz_f, total_volume):
    """utils.py:147-163 with cell_vol = dx*dy*dz_f (solver.py:303-306)."""
    vol = (dx * dy * dz_f[None, None, :])
    return float(np.sum(u[1 : nx + 1, 1 : ny + 1, 1 : nz + 1] * vol) / total_volume)


def initialize_fft_solver(nx, ny, nz, dx, dy, dz_c, dz_f):
    """projection.py:24-131 (Neumann pressure rows at both walls, the
    (0,0) mode pinned by an identity first row)."""
    kx = np.fft.fftfreq(nx, d=dx / (2 * math.pi))
    ky = np.fft.rfftfreq(ny, d=dy / (2 * math.pi))
    kx_mod = (2.0 / dx) * np.sin(kx * dx / 2.0)
    ky_mod = (2.0 / dy) * np.sin(ky * dy / 2.0)
    nkx, nky = len(kx), len(ky)
    kxg, kyg = np.meshgrid(kx_mod, ky_mod, indexing="ij")
    k2 = kxg**2 + kyg**2
    dz_left, dz_right = dz_c[:-1], dz_c[1:]
    coeff_left = 1.0 / (dz_left * dz_f)
    coeff_right = 1.0 / (dz_right * dz_f)
    tri_a = np.zeros((nkx, nky, nz))
    tri_a[:, :, 1:] = coeff_left[1:]
    tri_c = np.zeros((nkx, nky, nz))
    tri_c[:, :, :-1] = coeff_right[:-1]
    coeff_sum = coeff_left + coeff_right
    tri_b = -(coeff_sum[None, None, :] + k2[:, :, None])
    tri_b[:, :, 0] += coeff_left[0]
    tri_b[:, :, -1] += coeff_right[-1]
    tri_b[0, 0, 0] = 1.0
    tri_c[0, 0, 0] = 0.0
    return {"k2": k2, "tri_a": tri_a, "tri_b": tri_b, "tri_c": tri_c, "nx": nx, "ny": ny, "nz": nz}


def thomas(a, b, c, d):
    """projection.py:199-247 -- batched Thomas sweep, (batch, n) arrays."""
    batch, n = d.shape
    cp = np.zeros((batch, n))
    dp = np.zeros((batch, n), dtype=d.dtype)
    x = np.zeros((batch, n), dtype=d.dtype)
    cp[:, 0] = c[:, 0] / b[:, 0]
    dp[:, 0] = d[:, 0] / b[:, 0]
    for i in range(1, n):
        denom = b[:, i] - a[:, i] * cp[:, i - 1]
        if i < n - 1:
            cp[:, i] = c[:, i] / denom
        dp[:, i] = (d[:, i] - a[:, i] * dp[:, i - 1]) / denom
    x[:, n - 1] = dp[:, n - 1]
    for i in range(n - 2, -1, -1):
        x[:, i] = dp[:, i] - cp[:, i] * x[:, i + 1]
    return x


def solve_poisson_fft(div, fft):
    """projection.py:133-197 -- returns the ghost-shaped pressure (nx+2,
    ny+2, nz+2) with periodic x,y ghosts and Neumann z ghosts."""
    nx, ny, nz = fft["nx"], fft["ny"], fft["nz"]
    dh = np.fft.rfft2(div, axes=(0, 1))
    nkx, nky = dh.shape[0], dh.shape[1]
    ph = thomas(fft["tri_a"].reshape(-1, nz), fft["tri_b"].reshape(-1, nz),
                fft["tri_c"].reshape(-1, nz), dh.reshape(-1, nz)).reshape(nkx, nky, nz)
    pin = np.fft.irfft2(ph, s=(nx, ny), axes=(0, 1))
    p = np.zeros((nx + 2, ny + 2, nz + 2))
    p[1 : nx + 1, 1 : ny + 1, 1 : nz + 1] = pin
    p[0] = p[nx]
    p[nx + 1] = p[1]
    p[:, 0] = p[:, ny]
    p[:, ny + 1] = p[:, 1]
    p[:, :, 0] = p[:, :, 1]
    p[:, :, nz + 1] = p[:, :, nz]
    return p


def project_velocity(u, v, w, p, nx, ny, nz, dx, dy, dz_c, dz_f, dt):
    """projection.py:250-272, in place."""
    dpx = (p[2 : nx + 2, 1 : ny + 1, 1 : nz + 1] - p[1 : nx + 1, 1 : ny + 1, 1 : nz + 1]) / dx
    u[1 : nx + 1, 1 : ny + 1, 1 : nz + 1] -= dt * dpx
    dpy = (p[1 : nx + 1, 2 : ny + 2, 1 : nz + 1] - p[1 : nx + 1, 1 : ny + 1, 1 : nz + 1]) / dy
    v[1 : nx + 1, 1 : ny + 1, 1 : nz + 1] -= dt * dpy
    dpz = (p[1 : nx + 1, 1 : ny + 1, 2 : nz + 1] - p[1 : nx + 1, 1 : ny + 1, 1:nz]) / dz_c[1:nz]
    w[1 : nx + 1, 1 : ny + 1, 1:nz] -= dt * dpz


# ---------------------------------------------------------------------------
# The step (solver.py:694-1018)
# ---------------------------------------------------------------------------


class OracleChannel:
    """State and step of SLChannelFlow's SL-BDF2 scheme (noninc or inc
    pressure, theta = 1 z-solve, exact bulk shift), on numpy arrays."""

    def __init__(self, nx, ny, nz, Lx, Ly, Lz, gamma, nu, u, v, w, p=None, *,
                 stretching_type="symmetric", order=6, traj_order=2, n_traj_iters=2,
                 top_wall_bc_type="dirichlet", U_bulk=1.0, xy_rhs="extrap",
                 z_f=None, z_c=None, bulk_forcing=True, bdf2_pressure="noninc"):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.Lx, self.Ly, self.Lz = Lx, Ly, Lz
        self.dx, self.dy = Lx / nx, Ly / ny
        self.nu, self.U_bulk, self.gamma = nu, U_bulk, gamma
        self.top = top_wall_bc_type
        self.xy_rhs = xy_rhs
        self.bulk_forcing = bulk_forcing
        if z_f is None:
            z_f, z_c, dz_f, dz_c = generate_grid(gamma, nz, Lz, stretching_type)
        else:
            z_f, z_c = np.asarray(z_f, np.float64), np.asarray(z_c, np.float64)
            dz_f, dz_c = z_f[1:] - z_f[:-1], z_c[1:] - z_c[:-1]
        self.z_f, self.z_c, self.dz_f, self.dz_c = z_f, z_c, dz_f, dz_c
        self.total_volume = Lx * Ly * Lz
        self.fft = initialize_fft_solver(nx, ny, nz, self.dx, self.dy, dz_c, dz_f)
        self.sl = OracleAdvector(nx, ny, nz, self.dx, self.dy, Lx, Ly, Lz, z_f, z_c, gamma,
                                 stretching_type, order, traj_order, n_traj_iters)
        self.u, self.v, self.w = (np.array(a, dtype=np.float64) for a in (u, v, w))
        self.p = np.zeros((nx + 2, ny + 2, nz + 2)) if p is None else np.array(p, np.float64)
        self.u_nm1 = self.v_nm1 = self.w_nm1 = None
        self.R_nm1 = None
        self.dt_prev = None
        self.n_clamped_last = 0
        self.forcing = 0.0
        self.pressure = bdf2_pressure
        self.P_curr = self.P_prev = None  # full pressure levels of the inc branch

    def apply_bc(self):
        apply_bc_all(self.u, self.v, self.w, self.top)

    def explicit_xy_rhs(self):
        """solver.py:680-688."""
        a = (self.nx, self.ny, self.nz, self.dx, self.dy, self.nu)
        return (diffusion_xy("u", self.u, *a), diffusion_xy("v", self.v, *a),
                diffusion_xy("w", self.w, *a))

    def divergence(self):
        return compute_divergence(self.u, self.v, self.w, self.nx, self.ny, self.nz,
                                  self.dx, self.dy, self.dz_f)

    def bulk_velocity(self):
        return compute_bulk_velocity(self.u, self.nx, self.ny, self.nz, self.dx, self.dy,
                                     self.dz_f, self.total_volume)

    def project_initial(self):
        """solver.py:593-613 -- project the initial field with dt = 1."""
        div = self.divergence()
        self.p = solve_poisson_fft(div, self.fft)
        project_velocity(self.u, self.v, self.w, self.p, self.nx, self.ny, self.nz,
                         self.dx, self.dy, self.dz_c, self.dz_f, 1.0)
        self.apply_bc()

    def _zsolve_all(self, dt_eff):
        nx, ny, nz = self.nx, self.ny, self.nz
        self.u = solve_implicit_diffusion("u", self.u, dt_eff, nx, ny, nz, self.dz_c, self.dz_f,
                                          self.nu, 1.0, self.top)
        self.v = solve_implicit_diffusion("v", self.v, dt_eff, nx, ny, nz, self.dz_c, self.dz_f,
                                          self.nu, 1.0, self.top)
        self.w = solve_implicit_diffusion("w", self.w, dt_eff, nx, ny, nz, self.dz_c, self.dz_f,
                                          self.nu, 1.0)
        self.apply_bc()

    def _project(self, dt_div, dt_proj, cap):
        div = self.divergence()
        phi = solve_poisson_fft(div / dt_div, self.fft)
        if cap is not None:
            cap["phi"] = phi.copy()
        project_velocity(self.u, self.v, self.w, phi, self.nx, self.ny, self.nz, self.dx,
                         self.dy, self.dz_c, self.dz_f, dt_proj)
        self.p = phi
        self.apply_bc()
        return phi

    def _bulk_shift(self, dt):
        """solver.py:694-723 -- exact uniform shift of u to the target bulk."""
        if not self.bulk_forcing:
            return 0.0, 0.0
        nx, ny, nz = self.nx, self.ny, self.nz
        ub_star = self.bulk_velocity()
        corr = self.U_bulk - ub_star
        self.u[1 : nx + 1, 1 : ny + 1, 1 : nz + 1] += corr
        self.apply_bc()
        self.forcing = corr / dt
        return self.bulk_velocity(), self.forcing

    def _interior_add(self, outs, rhs, coef):
        nx, ny, nz = self.nx, self.ny, self.nz
        outs[0][1 : nx + 1, 1 : ny + 1, 1 : nz + 1] += coef * rhs[0][1 : nx + 1, 1 : ny + 1, 1 : nz + 1]
        outs[1][1 : nx + 1, 1 : ny + 1, 1 : nz + 1] += coef * rhs[1][1 : nx + 1, 1 : ny + 1, 1 : nz + 1]
        outs[2][1 : nx + 1, 1 : ny + 1, 1:nz] += coef * rhs[2][1 : nx + 1, 1 : ny + 1, 1:nz]

    def step_bdf1_bootstrap(self, dt, capture=False):
        """solver.py:729-811."""
        cap = {} if capture else None
        rhs = self.explicit_xy_rhs()
        self.u_nm1, self.v_nm1, self.w_nm1 = self.u.copy(), self.v.copy(), self.w.copy()
        self.R_nm1 = tuple(r.copy() for r in rhs)
        outs = list(self.sl.advect(self.u, self.v, self.w, self.u, self.v, self.w, dt))
        self.n_clamped_last = self.sl.n_clamped_last
        if cap is not None:
            cap["ubar"] = tuple(o.copy() for o in outs)
        self._interior_add(outs, rhs, dt)
        self.u, self.v, self.w = outs
        self.apply_bc()
        if cap is not None:
            cap["uhat"] = (self.u.copy(), self.v.copy(), self.w.copy())
        self._zsolve_all(dt)
        if cap is not None:
            cap["zsolve"] = (self.u.copy(), self.v.copy(), self.w.copy())
        phi = self._project(dt, dt, cap)
        if self.pressure == "inc":  # solver.py:802-807
            self.P_curr = phi.copy()
            self.P_prev = None
        if cap is not None:
            cap["proj"] = (self.u.copy(), self.v.copy(), self.w.copy())
        self.dt_prev = dt
        ub, f = self._bulk_shift(dt)
        return (ub, f, cap) if capture else (ub, f)

    def step_imex(self, dt, theta=0.5):
        """solver.py:1055-1135 -- AB2 explicit advection + x,y diffusion,
        Crank-Nicolson z-diffusion, projection at dt, exact bulk shift."""
        nx, ny, nz = self.nx, self.ny, self.nz
        self.apply_bc()
        rhs = momentum_rhs_imex(self.u, self.v, self.w, nx, ny, nz, self.dx, self.dy, self.dz_c,
                                self.dz_f, self.nu)
        prev = getattr(self, "rhs_prev", None)
        if prev is None:
            self.u += dt * rhs[0]
            self.v += dt * rhs[1]
            self.w += dt * rhs[2]
        else:
            self.u += dt * (1.5 * rhs[0] - 0.5 * prev[0])
            self.v += dt * (1.5 * rhs[1] - 0.5 * prev[1])
            self.w += dt * (1.5 * rhs[2] - 0.5 * prev[2])
        self.rhs_prev = rhs
        self.apply_bc()
        self.u = solve_implicit_diffusion("u", self.u, dt, nx, ny, nz, self.dz_c, self.dz_f, self.nu,
                                          theta, self.top)
        self.v = solve_implicit_diffusion("v", self.v, dt, nx, ny, nz, self.dz_c, self.dz_f, self.nu,
                                          theta, self.top)
        self.w = solve_implicit_diffusion("w", self.w, dt, nx, ny, nz, self.dz_c, self.dz_f, self.nu,
                                          theta)
        self.apply_bc()
        self._project(dt, dt, None)
        return self._bulk_shift(dt)

    def step_bdf2(self, dt, capture=False):
        """solver.py:813-1018 (noninc or inc pressure)."""
        nx, ny, nz = self.nx, self.ny, self.nz
        self.apply_bc()
        if self.u_nm1 is None or self.dt_prev is None or abs(dt - self.dt_prev) > 1e-12 * dt:
            return self.step_bdf1_bootstrap(dt, capture)
        cap = {} if capture else None
        rhs = self.explicit_xy_rhs()
        if self.xy_rhs == "extrap":
            Rh = tuple(2.0 * r - rn for r, rn in zip(rhs, self.R_nm1))
        else:
            Rh = rhs
        self.R_nm1 = tuple(r.copy() for r in rhs)
        mid = (2.0 * self.u - self.u_nm1, 2.0 * self.v - self.v_nm1, 2.0 * self.w - self.w_nm1)
        far = self.sl.advect(self.u_nm1, self.v_nm1, self.w_nm1, *mid, 2.0 * dt)
        nc_far = self.sl.n_clamped_last
        near = list(self.sl.advect(self.u, self.v, self.w, *mid, dt))
        self.n_clamped_last = self.sl.n_clamped_last + nc_far
        if cap is not None:
            cap["ubarbar"] = tuple(f.copy() for f in far)
            cap["ubar"] = tuple(f.copy() for f in near)
        dt_eff = (2.0 / 3.0) * dt
        outs = [n * (4.0 / 3.0) + f * (-1.0 / 3.0) for n, f in zip(near, far)]
        self._interior_add(outs, Rh, dt_eff)
        p_ext = None
        if self.pressure == "inc" and self.P_curr is not None:  # solver.py:905-941
            p_ext = self.P_curr if self.P_prev is None else 2.0 * self.P_curr - self.P_prev
            gp = [np.zeros_like(o) for o in outs]
            project_velocity(gp[0], gp[1], gp[2], p_ext, nx, ny, nz, self.dx, self.dy,
                             self.dz_c, self.dz_f, 1.0)
            for o, g in zip(outs, gp):
                o += dt_eff * g
        self.u_nm1, self.v_nm1, self.w_nm1 = self.u.copy(), self.v.copy(), self.w.copy()
        self.u, self.v, self.w = outs
        self.apply_bc()
        if cap is not None:
            cap["uhat"] = (self.u.copy(), self.v.copy(), self.w.copy())
        self._zsolve_all(dt_eff)
        if cap is not None:
            cap["zsolve"] = (self.u.copy(), self.v.copy(), self.w.copy())
        phi = self._project(dt_eff, dt_eff, cap)
        if self.pressure == "inc":  # solver.py:1001-1012
            if self.P_curr is None:
                self.P_curr = phi.copy()
            elif self.P_prev is None:
                self.P_prev = self.P_curr.copy()
                self.P_curr = self.P_curr + phi
            else:
                self.P_prev = self.P_curr.copy()
                self.P_curr = p_ext + phi
            self.p = self.P_curr
        if cap is not None:
            cap["proj"] = (self.u.copy(), self.v.copy(), self.w.copy())
        self.dt_prev = dt
        ub, f = self._bulk_shift(dt)
        return (ub, f, cap) if capture else (ub, f)
