"""SLAdvector: drop-in for slchannel.semilag.SLAdvector on a B200.

Same constructor, attributes and ``advect`` contract as the reference
(slchannel/semilag.py:133-671); the per-point work -- characteristic trace,
stencil location through the analytic inverse tanh map, Lagrange weights and
the order^3 gather -- runs in the sm_100a kernels of libslc_b200.so.  There is
no CPU or eager fallback: a CPU device raises.
"""

from __future__ import annotations

from dataclasses import dataclass

import torch

from . import _native as N


@dataclass
class _GridSpec:
    """Node grid of one velocity component (semilag.py:87-99)."""

    name: str
    shift_x: float
    shift_y: float
    NX: int
    NY: int
    NZ: int
    znodes: torch.Tensor
    ztype: str
    denom_inv: dict


@dataclass
class PointStencil:
    """Result of ``_build_iw``: the interpolation points of one component
    grid at one order.  The weights themselves are never materialised; the
    kernel rebuilds them in registers (semilag.py:67-84 holds them as
    (N, order) tensors instead)."""

    comp: str
    x: torch.Tensor
    y: torch.Tensor
    z: torch.Tensor
    order: int
    count_clamp: bool
    n_clamped: torch.Tensor


def _z_denominator_table(znodes: torch.Tensor, order: int) -> torch.Tensor:
    """semilag.py:102-114 (host, init only)."""
    zn = znodes.detach().cpu().to(torch.float64).unfold(0, order, 1)
    diff = zn.unsqueeze(2) - zn.unsqueeze(1)
    diff = diff + torch.eye(order, dtype=diff.dtype).unsqueeze(0)
    return 1.0 / diff.prod(dim=2)


class SLAdvector:
    """Semi-Lagrangian advection of the three staggered velocity components
    (slchannel/semilag.py:130-671) on the GPU."""

    _COMPS = {"u": 0, "v": 1, "w": 2}

    def __init__(self, nx, ny, nz, dx, dy, Lx, Ly, Lz, z_f, z_c, gamma,
                 stretching_type="symmetric", order=4, traj_order=2, n_traj_iters=2,
                 top_wall_bc_type="dirichlet", interp_dtype="fp64",
                 device=torch.device("cpu"), *, nu=0.0, xy_rhs="extrap"):
        # argument checks and messages as semilag.py:204-219
        if order not in (4, 6):
            raise ValueError(f"sl.interp_order must be 4 (tricubic) or 6 (triquintic), got {order}")
        if traj_order not in (2, 4):
            raise ValueError(
                f"sl.traj_interp_order must be 2 (trilinear) or 4 (tricubic), got {traj_order}")
        if stretching_type not in ("symmetric", "bottom"):
            raise ValueError(
                f"SLAdvector supports 'symmetric'/'bottom' stretching, got '{stretching_type}'")
        if interp_dtype not in ("fp64", "fp32_accum64", "mixed"):
            raise ValueError(
                f"sl.interp_dtype must be 'fp64', 'fp32_accum64' or 'mixed', got {interp_dtype}")
        if nz + 1 < order:
            raise ValueError(f"nz={nz} too small for interpolation order {order}")
        device = torch.device(device)
        if device.type != "cuda":
            raise RuntimeError("slchannel_b200 runs on a CUDA device (sm_100a); there is no CPU path")
        if device.index is None:
            device = torch.device("cuda", torch.cuda.current_device())

        self.nx, self.ny, self.nz = nx, ny, nz
        self.dx, self.dy = dx, dy
        self.Lx, self.Ly, self.Lz = Lx, Ly, Lz
        self.gamma = float(gamma)
        self.stretching_type = stretching_type
        self.order = order
        self.traj_order = traj_order
        self.n_traj_iters = n_traj_iters
        self.top_wall_bc_type = top_wall_bc_type
        self.interp_dtype = interp_dtype
        self.device = device

        self.z_f = z_f.to(device=device, dtype=torch.float64)
        self.z_c = z_c.to(device=device, dtype=torch.float64)
        self._tanh_g = float(torch.tanh(torch.tensor(self.gamma, dtype=torch.float64)))
        zf_host = z_f.detach().to("cpu", torch.float64)
        eps_z = 1e-12 * Lz
        self.z_lo = float(zf_host[0] + eps_z)
        self.z_hi = float(zf_host[-1] - eps_z)

        precision = N.PREC_FP64 if interp_dtype == "fp64" else N.PREC_MIXED
        self._grid = N.Grid(nx, ny, nz, Lx, Ly, Lz, gamma, zf_host, z_c, stretching_type=stretching_type,
                            order=order, traj_order=traj_order, n_traj_iters=n_traj_iters,
                            top_wall_bc_type=top_wall_bc_type, precision=precision, nu=nu,
                            device=device, xy_rhs=xy_rhs)

        def make_spec(name, sx, sy, znodes, ztype):
            denoms = {o: _z_denominator_table(znodes, o).to(device)
                      for o in sorted({2, traj_order, order})}
            return _GridSpec(name, sx, sy, nx, ny, len(znodes), znodes.to(device, torch.float64),
                             ztype, denoms)

        self.spec = {
            "u": make_spec("u", 0.0, -0.5, z_c, "centers"),
            "v": make_spec("v", -0.5, 0.0, z_c, "centers"),
            "w": make_spec("w", -0.5, -0.5, z_f, "faces"),
        }

        f64 = dict(dtype=torch.float64, device=device)
        ar = torch.arange(1, nx + 1, **f64)
        aj = torch.arange(1, ny + 1, **f64)
        x_face = (ar * dx).view(nx, 1, 1)
        x_cent = ((ar - 0.5) * dx).view(nx, 1, 1)
        y_face = (aj * dy).view(1, ny, 1)
        y_cent = ((aj - 0.5) * dy).view(1, ny, 1)
        z_cent = self.z_c[1 : nz + 1].view(1, 1, nz)
        z_facei = self.z_f[1:nz].view(1, 1, nz - 1)
        self.arrival = {
            "u": (x_face, y_cent, z_cent, (nx, ny, nz)),
            "v": (x_cent, y_face, z_cent, (nx, ny, nz)),
            "w": (x_cent, y_cent, z_facei, (nx, ny, nz - 1)),
        }

        def alloc(spec):
            return torch.empty(spec.NX, spec.NY, spec.NZ, **f64)

        self.fbuf = {c: alloc(self.spec[c]) for c in "uvw"}
        self._mbuf = {c: alloc(self.spec[c]) for c in "uvw"}
        self._mbuf_src = None
        self.ustar = torch.zeros(nx + 1, ny + 2, nz + 2, **f64)
        self.vstar = torch.zeros(nx + 2, ny + 1, nz + 2, **f64)
        self.wstar = torch.zeros(nx + 2, ny + 2, nz + 1, **f64)
        self.n_clamped_last = torch.zeros((), dtype=torch.int64, device=device)
        self.last_iw = {}
        self._scratch_count = torch.zeros((), dtype=torch.int64, device=device)

    # ------------------------------------------------------------------
    @property
    def native(self):
        """The native grid handle (libslc_b200.so)."""
        return self._grid

    def _stream(self):
        return N.stream_of(self.ustar)

    def _check_fields(self, u, v, w, what):
        nx, ny, nz = self.nx, self.ny, self.nz
        N.require(u, (nx + 1, ny + 2, nz + 2), f"{what} u")
        N.require(v, (nx + 2, ny + 1, nz + 2), f"{what} v")
        N.require(w, (nx + 2, ny + 2, nz + 1), f"{what} w")

    @property
    def mbuf(self):
        """The trajectory-velocity node buffers (semilag.py:367).  The
        reference's advect leaves them holding its last trajectory velocity;
        the kernels here read the ghost-shaped arrays directly, so that copy
        is made only when the buffers are read (departure_coords, _sample, or
        a caller's _fill, which then overwrites it) -- from the trajectory
        tensors of the last advect as they are at that moment."""
        if self._mbuf_src is not None:
            src, self._mbuf_src = self._mbuf_src, None
            for c, f in zip("uvw", src):
                self._fill(self._mbuf[c], c, f)
        return self._mbuf

    # semilag.py:387-394 (plain copies of views)
    def _fill(self, buf, comp, field):
        nx, ny = self.nx, self.ny
        if comp == "u":
            buf.copy_(field[0:nx, 1 : ny + 1, :])
        elif comp == "v":
            buf.copy_(field[1 : nx + 1, 0:ny, :])
        else:
            buf.copy_(field[1 : nx + 1, 1 : ny + 1, :])

    # semilag.py:400-411
    def _face_coord(self, z):
        zz = z.to(device=self.device, dtype=torch.float64).contiguous()
        out = torch.empty_like(zz)
        self._grid.call("slc_face_coord", N.ptr(zz), zz.numel(), N.ptr(out), self._stream())
        return out

    # semilag.py:460-469
    def _build_iw(self, spec, x, y, z, order, count_clamp=False):
        f = dict(device=self.device, dtype=torch.float64)
        x = x.to(**f).reshape(-1).contiguous()
        y = y.to(**f).reshape(-1).contiguous()
        z = z.to(**f).reshape(-1).contiguous()
        if count_clamp:
            n_clamped = ((z < self.z_lo) | (z > self.z_hi)).sum()
        else:
            n_clamped = torch.zeros((), dtype=torch.int64, device=self.device)
        return PointStencil(spec.name, x, y, z, order, count_clamp, n_clamped)

    # semilag.py:502-510
    def _apply_iw(self, buf, iw):
        spec = self.spec[iw.comp]
        buf = N.require(buf.to(self.device).contiguous(), (spec.NX, spec.NY, spec.NZ), "node buffer")
        out = torch.empty(iw.x.numel(), dtype=torch.float64, device=self.device)
        self._scratch_count.zero_()
        self._grid.call("slc_interp_points", self._COMPS[iw.comp], iw.order, N.ptr(buf),
                        N.ptr(iw.x), N.ptr(iw.y), N.ptr(iw.z), iw.x.numel(),
                        1 if iw.count_clamp else 0, N.ptr(out), N.ptr(self._scratch_count),
                        self._stream())
        return out

    # semilag.py:512-528
    def _sample(self, comp, x, y, z):
        shape = x.shape
        iw = self._build_iw(self.spec[comp], x, y, z, self.traj_order, count_clamp=True)
        return self._apply_iw(self.mbuf[comp], iw).reshape(shape)

    # semilag.py:534-552
    def departure_coords(self, comp, dt_t):
        shape = self.arrival[comp][3]
        xd, yd, zd = (torch.empty(shape, dtype=torch.float64, device=self.device) for _ in range(3))
        self._grid.call("slc_departure", self._COMPS[comp], N.ptr(self.mbuf["u"]),
                        N.ptr(self.mbuf["v"]), N.ptr(self.mbuf["w"]), float(dt_t), N.ptr(xd),
                        N.ptr(yd), N.ptr(zd), self._stream())
        return xd, yd, zd

    # semilag.py:573-578
    def compute_departure(self, comp, dt_t):
        xd, yd, zd = self.departure_coords(comp, dt_t)
        return self._build_iw(self.spec[comp], xd, yd, zd, self.order, count_clamp=True)

    # semilag.py:584-671
    def advect(self, u, v, w, u_mid, v_mid, w_mid, dt_t, extra_rhs=None):
        """Semi-Lagrangian advection of (u, v, w) along the trajectory velocity
        (u_mid, v_mid, w_mid) over dt_t.  Returns the advector's persistent
        ghost-shaped buffers (ustar, vstar, wstar), interiors filled, ghosts
        not refreshed, w walls 0; overwritten by the next call.  With
        extra_rhs (a list of field triples), each triple is interpolated at
        the same departure points -- traced once, in one launch per component
        for up to seven extra triples -- and returned as a fourth element: a
        list of new interior-shaped (arrival-shaped) triples."""
        self._check_fields(u, v, w, "advected")
        self._check_fields(u_mid, v_mid, w_mid, "trajectory")
        dt = float(dt_t)
        # the reference leaves the trajectory node buffers filled; here they
        # are filled only if someone reads them (see the mbuf property)
        self._mbuf_src = (u_mid, v_mid, w_mid)
        s = self._stream()
        counter = torch.zeros((), dtype=torch.int64, device=self.device)
        if extra_rhs is None:
            self._grid.call("slc_advect", N.ptr(u), N.ptr(v), N.ptr(w), N.ptr(u_mid),
                            N.ptr(v_mid), N.ptr(w_mid), dt, N.ptr(self.ustar), N.ptr(self.vstar),
                            N.ptr(self.wstar), N.ptr(counter), s)
            self.n_clamped_last = counter
            return self.ustar, self.vstar, self.wstar
        extra_rhs = list(extra_rhs)
        for triple in extra_rhs:
            if len(triple) != 3:
                raise ValueError("extra_rhs entries must be (Ru, Rv, Rw) triples")
            self._check_fields(*triple, "extra_rhs")
        f = dict(dtype=torch.float64, device=self.device)
        extras = [tuple(torch.empty(self.arrival[c][3], **f) for c in "uvw") for _ in extra_rhs]
        pin, kin = N.ptr_array([t for triple in extra_rhs for t in triple])
        pout, kout = N.ptr_array([t for triple in extras for t in triple])
        self._grid.call("slc_advect_extra", N.ptr(u), N.ptr(v), N.ptr(w), N.ptr(u_mid),
                        N.ptr(v_mid), N.ptr(w_mid), dt, N.ptr(self.ustar), N.ptr(self.vstar),
                        N.ptr(self.wstar), len(extra_rhs), pin, pout, N.ptr(counter), s)
        self.n_clamped_last = counter
        return self.ustar, self.vstar, self.wstar, extras
