"""SLChannelFlow: drop-in for slchannel.solver.SLChannelFlow's SL-BDF2 step.

Reads the reference's YAML surface (slchannel/solver.py:168-282,
docs/CONFIG.md), builds the grid and the initial field, and advances it with
``step_sl_bdf2`` (solver.py:813-1018) -- Boukir BDF2 along characteristics,
theta = 1 wall-normal diffusion, FFT pressure projection and the exact
bulk-flux shift -- executed by libslc_b200.so on one GPU.  The fields
``u, v, w, p`` and the history ``u_nm1, v_nm1, w_nm1`` are ghost-shaped
float64 CUDA tensors, exactly as in the reference; between steps they are
BC-consistent.

The time loop / output shell of the reference (run_simulation,
solver.py:1140-1637) and the Eulerian comparison scheme are not part of this
package.
"""

from __future__ import annotations

import os

import numpy as np
import torch
import yaml

from . import _native as N
from .initflow import initialize_flow, initialize_flow_from_file
from .semilag import SLAdvector
from .turbstats import TurbulenceStats
from .utils import (compute_bulk_velocity, compute_cfl_fused, compute_divergence, compute_u_tau,
                    generate_grid)


class SLChannelFlow:
    """Channel-flow DNS driver with the SL-BDF2 step on a B200."""

    def __init__(self, config_file="config.yaml", allocate_fields=True, *, config=None):
        if config is None:
            with open(config_file, "r") as f:
                config = yaml.safe_load(f)
        self.config = config

        # The config is checked before the device, so a bad key raises the
        # reference's ValueError on any machine (the reference, without a GPU,
        # falls back to its CPU device and then checks, solver.py:172-282).
        self.nx = config["grid"]["nx"]
        self.ny = config["grid"]["ny"]
        self.nz = config["grid"]["nz"]
        self.Lx = config["domain"]["Lx"]
        self.Ly = config["domain"]["Ly"]
        self.Lz = config["domain"]["Lz"]
        self.stretching_type = config["domain"].get("stretching_type", "symmetric")
        if self.stretching_type not in ["symmetric", "bottom"]:
            raise ValueError(
                f"Invalid stretching type: {self.stretching_type}. "
                "slChannel supports 'symmetric' or 'bottom'")
        self.nu = 1.0 / config["flow"]["Re"]
        self.Re_tau = config["flow"]["Re_tau"]  # required, as in solver.py:210 (KeyError)
        self.U_bulk = config["flow"]["U_bulk"]
        self.gamma = config["flow"]["gamma"]
        bc_config = config.get("boundary_conditions", {})
        self.top_wall_bc_type = bc_config.get("top_wall", {}).get("type", "dirichlet")
        if self.top_wall_bc_type not in ["dirichlet", "neumann"]:
            raise ValueError(f"Invalid top wall BC type: {self.top_wall_bc_type}")
        t = config.get("time", {})
        self.dt = t.get("dt", 0.01)
        self.n_steps = t.get("n_steps", 0)
        self.t_max = t.get("t_max", 1000.0)
        self.dt_update_interval = t.get("dt_update_interval", 0)
        # adaptive dt (solver.py:222-239, 652-674); the reference requires
        # CFL_target, here only when dt_update_interval asks for adaptation
        self.cfl_target = t.get("CFL_target", None)
        self.dt_max = t.get("dt_max", 0.01)
        self.dt_min = t.get("dt_min", 0.0001)
        self.diff_stability_C = t.get("diff_stability_C", 0.2)
        if self.dt_update_interval > 0 and self.cfl_target is None:
            raise KeyError("CFL_target")

        self.advection_scheme = config.get("advection", {}).get("scheme", "sl")
        if self.advection_scheme not in ["sl", "eulerian"]:
            raise ValueError(
                f"advection.scheme must be 'sl' or 'eulerian', got {self.advection_scheme}")
        sl_cfg = config.get("sl", {})
        self.sl_order = sl_cfg.get("interp_order", 4)
        if self.sl_order not in (4, 6):
            raise ValueError(
                f"sl.interp_order must be 4 (tricubic) or 6 (triquintic), got {self.sl_order}")
        self.sl_traj_order = sl_cfg.get("traj_interp_order", 2)
        self.sl_traj_iters = sl_cfg.get("n_traj_iters", 2)
        self.sl_interp_dtype = sl_cfg.get("interp_dtype", "fp64")
        self.sl_bdf2_pressure = sl_cfg.get("bdf2_pressure", "noninc")
        self.sl_bdf2_xy_rhs = sl_cfg.get("bdf2_xy_rhs", "extrap")
        for removed in ("time_scheme", "traj_extrapolation", "field_interp"):
            if removed in sl_cfg:
                raise ValueError(
                    f"sl.{removed} was removed in the bdf2-only cleanup: the SL scheme is always "
                    f"Boukir BDF2 characteristics now (drop the key from the config)")
        if self.sl_bdf2_pressure not in ["noninc", "inc"]:
            raise ValueError(
                f"sl.bdf2_pressure must be 'noninc' or 'inc', got {self.sl_bdf2_pressure}")
        if self.sl_bdf2_xy_rhs not in ["extrap", "lagged"]:
            raise ValueError(
                f"sl.bdf2_xy_rhs must be 'extrap' or 'lagged', got {self.sl_bdf2_xy_rhs}")
        solver_type = config.get("solver", {}).get("type", "fft")
        if solver_type != "fft":
            raise ValueError(f"solver.type must be 'fft', got {solver_type!r}.")
        self._stats_cfg = config.get("statistics", {}) or {}
        self.n_stats = (self._stats_cfg.get("n_stats", 0)
                        if self._stats_cfg.get("enabled", True) else 0)
        self.t_stats = self._stats_cfg.get("t_stats", 10.0)

        dev_cfg = config.get("compute", {}).get("device", "auto")
        if dev_cfg == "cpu":
            raise RuntimeError("slchannel_b200 runs on a CUDA device (sm_100a); there is no CPU path")
        if not torch.cuda.is_available():
            raise RuntimeError("CUDA requested but not available")
        self.device = torch.device("cuda", torch.cuda.current_device())

        out_cfg = config.get("output", {})
        self.results_folder = out_cfg.get("results_folder", "results")
        self.allocate_fields = allocate_fields

        torch.set_default_dtype(torch.float64)
        self.z_f, self.z_c, self.dz_f, self.dz_c = generate_grid(
            self.gamma, self.nz, self.Lz, device=self.device, stretching_type=self.stretching_type)
        self.dx = self.Lx / self.nx
        self.dy = self.Ly / self.ny
        self.cell_vol = (self.dx * self.dy * self.dz_f.view(1, 1, -1)).expand(self.nx, self.ny, self.nz)
        self.cell_vol_ratio = self.cell_vol
        self.total_volume = self.Lx * self.Ly * self.Lz

        self.sl = SLAdvector(
            self.nx, self.ny, self.nz, self.dx, self.dy, self.Lx, self.Ly, self.Lz,
            self.z_f, self.z_c, self.gamma, stretching_type=self.stretching_type,
            order=self.sl_order, traj_order=self.sl_traj_order, n_traj_iters=self.sl_traj_iters,
            top_wall_bc_type=self.top_wall_bc_type, interp_dtype=self.sl_interp_dtype,
            device=self.device, nu=self.nu, xy_rhs=self.sl_bdf2_xy_rhs)
        self._grid = self.sl.native

        init_cfg = config.get("initialization", {})
        field_file = init_cfg.get("field_file", None)
        self.forcing = 0.0
        self.initial_step, self.time = 0, 0.0
        if not allocate_fields:
            self.u = self.v = self.w = self.p = None
        elif field_file is not None and init_cfg.get("type", "parabolic") != "interpolate":
            self.u, self.v, self.w, self.p, self.initial_step, self.time = initialize_flow_from_file(
                field_file, device=self.device, reset_time=init_cfg.get("reset_time", False))
            # the bulk-forcing state saved with the fields (solver.py:338-350)
            try:
                self.forcing = float(np.load(field_file)["forcing"])
            except Exception:
                self.forcing = 0.0
        else:
            self.u, self.v, self.w, self.p = initialize_flow(
                self.nx, self.ny, self.nz, self.z_c, self.Ly, self.Lz, U_bulk=self.U_bulk,
                init_type=init_cfg.get("type", "parabolic"),
                perturbation_intensity=init_cfg.get("perturbation_intensity", 0.0),
                n_vortices=init_cfg.get("n_vortices", 4), device=self.device,
                top_wall_bc_type=self.top_wall_bc_type)
            ub = float(compute_bulk_velocity(self.u, self.cell_vol_ratio, self.total_volume))
            if abs(ub) > 1e-9:
                self.u *= self.U_bulk / ub
        self.initial_time = self.time
        self.current_step = self.initial_step

        self.u_nm1 = self.v_nm1 = self.w_nm1 = None
        self._next = None
        self._dt_prev_step = None
        # Eulerian IMEX: the explicit right-hand sides of the last two steps
        self._rhs_cur = self._rhs_prev = None
        self._rhs_have_prev = False
        # incremental pressure (sl.bdf2_pressure: inc): p^{n-1} and whether it holds one
        self._p_prev = None
        self._p_have_prev = False
        if allocate_fields:
            self._save_and_project_initial()

        # Statistics (solver.py:510-550): `enabled` is an off switch and
        # n_stats 0 also disables; restart_state_file continues an
        # accumulation saved by save_state (this implementation's or the
        # reference's).  run_steps samples every n_stats steps after t_stats.
        self.turbulence_stats = None
        if self.n_stats > 0:
            self.stats_output_path = os.path.join(
                self.results_folder, self._stats_cfg.get("output_file", "turbulence_stats.npz"))
            self.stats_state_path = os.path.join(
                self.results_folder,
                self._stats_cfg.get("state_file", "turbulence_stats_state.npz"))
            self.turbulence_stats = TurbulenceStats(
                self.nx, self.ny, self.nz, self.Lx, self.Ly, self.Lz, self.z_c, self.z_f,
                self.dz_c, self.dz_f, self.dx, self.dy, self.nu, self.Re_tau,
                z_plus_target=self._stats_cfg.get("z_plus_target", 15.0), device=self.device,
                top_wall_bc_type=self.top_wall_bc_type,
                spectra_z_planes=self._stats_cfg.get("spectra_z_planes", None))
            restart = self._stats_cfg.get("restart_state_file", None)
            if restart is not None:
                self.turbulence_stats.load_state(restart)

    # ------------------------------------------------------------------
    def _stream(self):
        return N.stream_of(self.u)

    def _check_state(self):
        nx, ny, nz = self.nx, self.ny, self.nz
        N.require(self.u, (nx + 1, ny + 2, nz + 2), "u")
        N.require(self.v, (nx + 2, ny + 1, nz + 2), "v")
        N.require(self.w, (nx + 2, ny + 2, nz + 1), "w")
        N.require(self.p, (nx + 2, ny + 2, nz + 2), "p")

    def apply_bc_uvw(self):
        """solver.py:646-647 -> apply_bc_all (solver.py:70-107), on the GPU."""
        self._grid.call("slc_apply_bc", N.ptr(self.u), N.ptr(self.v), N.ptr(self.w), self._stream())

    def _project(self, dt_div, dt_proj):
        self._grid.call("slc_project", N.ptr(self.u), N.ptr(self.v), N.ptr(self.w), N.ptr(self.p),
                        float(dt_div), float(dt_proj), self._stream())

    def _save_and_project_initial(self):
        """solver.py:593-625 -- project the initial field (dt = 1)."""
        self._check_state()
        self.apply_bc_uvw()
        self._project(1.0, 1.0)

    def set_state(self, u, v, w, p=None):
        """Replace the velocity (and pressure) with caller-given ghost-shaped
        arrays and drop the BDF2 history (the next step re-bootstraps, as a
        restart does in the reference)."""
        f = dict(device=self.device, dtype=torch.float64)
        self.u = torch.as_tensor(u).to(**f).contiguous().clone()
        self.v = torch.as_tensor(v).to(**f).contiguous().clone()
        self.w = torch.as_tensor(w).to(**f).contiguous().clone()
        if p is not None:
            self.p = torch.as_tensor(p).to(**f).contiguous().clone()
        self.u_nm1 = self.v_nm1 = self.w_nm1 = None
        self._next = None
        self._dt_prev_step = None
        self._p_have_prev = False
        self._check_state()

    def diagnostics(self):
        """(max |div|, u_tau, CFL inverse, u_bulk) of the current state as a
        4-element device tensor, from one fused on-device reduction (no host
        synchronisation; utils.py:116-180, operators.py:839-940)."""
        out = torch.empty(4, dtype=torch.float64, device=self.device)
        self._grid.call("slc_diagnostics", N.ptr(self.u), N.ptr(self.v), N.ptr(self.w), N.ptr(out),
                        self._stream())
        return out

    def compute_divergence(self):
        return compute_divergence(self.u, self.v, self.w, self.nx, self.ny, self.nz, self.dx,
                                  self.dy, self.dz_f)

    # ------------------------------------------------------------------
    # SL-BDF2
    # ------------------------------------------------------------------
    def _apply_bulk_forcing(self, dt):
        """solver.py:694-723 -- exact uniform shift of u to the target bulk
        velocity; returns (u_bulk after the shift, forcing = shift / dt) as
        0-D device tensors."""
        out = torch.empty(2, dtype=torch.float64, device=self.device)
        self._grid.call("slc_bulk_shift", N.ptr(self.u), N.ptr(self.v), N.ptr(self.w),
                        float(self.U_bulk), float(dt), N.ptr(out), self._stream())
        self.forcing = out[1]
        return out[0], out[1]

    def _bdf2_forcing_update(self, dt):
        return self._apply_bulk_forcing(dt)

    def _alloc_next(self):
        return (torch.zeros_like(self.u), torch.zeros_like(self.v), torch.zeros_like(self.w))

    def _step_sl_bdf1_bootstrap(self, dt, dt_t=None):
        """solver.py:729-811 -- one BDF1 characteristics step; seeds the
        history (V^{n-1} <- V^n)."""
        self._check_state()
        nxt = self._next if self._next is not None else self._alloc_next()
        cur = (self.u, self.v, self.w)
        pc, kc = N.ptr_array(cur)
        pn, kn = N.ptr_array(nxt)
        self._grid.call("slc_step_bdf1", pc, pn, N.ptr(self.p), float(dt),
                        N.ptr(self.sl.n_clamped_last), self._stream())
        old = (self.u_nm1, self.v_nm1, self.w_nm1)
        self.u_nm1, self.v_nm1, self.w_nm1 = cur
        self.u, self.v, self.w = nxt
        self._next = old if old[0] is not None else None
        self._dt_prev_step = dt
        self._p_have_prev = False  # the bootstrap's p is its phi (solver.py:802-807)
        return self._bdf2_forcing_update(dt)

    def step_sl_bdf2(self, dt):
        """solver.py:813-1018 -- one SL-BDF2 step (BDF1 bootstrap on the
        first step, after set_state and whenever dt changes).  Returns
        (u_bulk, forcing) as 0-D device tensors."""
        dt = float(dt)
        if (self.u_nm1 is None or self._dt_prev_step is None
                or abs(dt - self._dt_prev_step) > 1e-12 * dt):
            if self._dt_prev_step is not None and self.u_nm1 is not None:
                print(f"[bdf2] dt changed ({self._dt_prev_step:.6g} -> {dt:.6g}): BDF1 re-bootstrap",
                      flush=True)
            return self._step_sl_bdf1_bootstrap(dt)
        self._check_state()
        if self._next is None:
            self._next = self._alloc_next()
        cur = (self.u, self.v, self.w)
        prev = (self.u_nm1, self.v_nm1, self.w_nm1)
        nxt = self._next
        pc, kc = N.ptr_array(cur)
        pp, kp = N.ptr_array(prev)
        pn, kn = N.ptr_array(nxt)
        if self.sl_bdf2_pressure == "inc":
            if self._p_prev is None:
                self._p_prev = torch.zeros_like(self.p)
            self._grid.call("slc_step_bdf2_inc", pc, pp, pn, N.ptr(self.p), N.ptr(self._p_prev),
                            1 if self._p_have_prev else 0, dt, N.ptr(self.sl.n_clamped_last),
                            self._stream())
            self._p_have_prev = True
        else:
            self._grid.call("slc_step_bdf2", pc, pp, pn, N.ptr(self.p), dt,
                            N.ptr(self.sl.n_clamped_last), self._stream())
        self.u_nm1, self.v_nm1, self.w_nm1 = cur
        self.u, self.v, self.w = nxt
        self._next = prev
        self._dt_prev_step = dt
        return self._bdf2_forcing_update(dt)

    def step_imex(self, dt):
        """solver.py:1055-1135 -- the Eulerian IMEX step: AB2 explicit
        advection + x,y diffusion, Crank-Nicolson z-diffusion, projection,
        exact bulk shift.  Returns (u_bulk, forcing)."""
        self._check_state()
        if self._rhs_cur is None:
            self._rhs_cur = tuple(torch.zeros_like(t) for t in (self.u, self.v, self.w))
            self._rhs_prev = tuple(torch.zeros_like(t) for t in (self.u, self.v, self.w))
        pv, k1 = N.ptr_array((self.u, self.v, self.w))
        pc, k2 = N.ptr_array(self._rhs_cur)
        pp, k3 = N.ptr_array(self._rhs_prev)
        self._grid.call("slc_step_imex", pv, N.ptr(self.p), pc, pp,
                        1 if self._rhs_have_prev else 0, float(dt), 0.5, self._stream())
        self._rhs_cur, self._rhs_prev = self._rhs_prev, self._rhs_cur
        self._rhs_have_prev = True
        return self._apply_bulk_forcing(dt)

    def compute_cfl_dt(self):
        """solver.py:652-674 -- the adaptive dt: CFL_target over the fused CFL
        inverse (a trajectory CFL for the SL scheme, capped by the explicit
        x,y-diffusion bound), clamped to [dt_min, dt_max]."""
        dti = compute_cfl_fused(self.u, self.v, self.w, self.nx, self.ny, self.nz, self.dx,
                                self.dy, self.dz_f, self.dz_c)
        if dti < 1e-10:
            dti = 1.0
        dt_new = self.cfl_target / dti
        if self.advection_scheme == "sl":
            dt_diff = self.diff_stability_C / (self.nu * (1.0 / self.dx**2 + 1.0 / self.dy**2))
            dt_new = min(dt_new, dt_diff)
        return min(max(dt_new, self.dt_min), self.dt_max)

    def run_steps(self, n, dt=None):
        """Advance n steps of the configured scheme; returns the last
        (u_bulk, forcing).  With dt given, every step uses it.  Otherwise the
        steps use time.dt, adapted as the reference's run loop does
        (solver.py:1347-1353): with dt_update_interval > 0, before every step
        whose number is a multiple of it, compute_cfl_dt() replaces time.dt
        when it differs by more than 5 % (the SL step then re-bootstraps with
        one BDF1 step).  With statistics on (n_stats > 0) a snapshot is
        accumulated after every step whose number is a multiple of n_stats
        once time >= t_stats (solver.py:1424-1436); the samples stay on the
        device until finalize_statistics() writes them."""
        fixed = dt
        res = None
        step = self.step_imex if self.advection_scheme == "eulerian" else self.step_sl_bdf2
        for _ in range(int(n)):
            nxt = self.current_step + 1
            if fixed is None and self.dt_update_interval > 0 and nxt % self.dt_update_interval == 0:
                dt_new = self.compute_cfl_dt()
                if abs(dt_new - self.dt) / self.dt > 0.05:
                    self.dt = dt_new
            dt = self.dt if fixed is None else fixed
            res = step(dt)
            self.time += dt
            self.current_step += 1
            if (self.turbulence_stats is not None and self.time >= self.t_stats
                    and self.current_step % self.n_stats == 0):
                u_tau = compute_u_tau(self.u, self.z_c, self.nu,
                                      top_wall_bc_type=self.top_wall_bc_type)
                self.turbulence_stats.accumulate_statistics(self.u, self.v, self.w, u_tau)
        return res

    def finalize_statistics(self):
        """Write the statistics restart state and the finalized statistics
        to the configured files (statistics.state_file / output_file under
        output.results_folder), as the reference does at the end of a run
        (solver.py:1593-1599).  Returns False when nothing was sampled."""
        ts = self.turbulence_stats
        if ts is None or ts.n_samples == 0:
            return False
        os.makedirs(self.results_folder, exist_ok=True)
        ts.save_state(self.stats_state_path)
        ts.save_statistics(self.stats_output_path)
        return True


def load_config(path):
    with open(path) as f:
        return yaml.safe_load(f)


__all__ = ["SLChannelFlow", "load_config"]
