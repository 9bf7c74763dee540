"""Turbulence statistics of the channel state, accumulated on the device
(reference: slchannel/turbstats.py, TurbulenceStats).

Each ``accumulate_statistics`` call adds one snapshot through the C ABI's
``slc_stats_accumulate``:
* the plane-mean profile U and the second moments u'u', v'v', w'w', u'w'
  about the instantaneous plane means, formed as the reference forms them
  (u'u' and v'v' at the components' own nodes, w'w' at the faces then
  averaged to centres, u'w' from cell-centred values);
* the plane-mean moments V, W, U^2, V^2, W^2 and U W for the time-mean
  correction in ``finalize_statistics``;
* the folded 2-D spectra E_uu, E_vv, E_ww, E_uw at the z+ target planes
  from both walls (w negated at the top wall), and at any extra planes.

Nothing is synchronised per snapshot; ``finalize_statistics`` reads the
accumulators once.
"""

from __future__ import annotations

import os
import warnings

import numpy as np
import torch

from . import _native as N

PROFILES = ("U_sum", "uu_sum", "vv_sum", "ww_sum", "uw_sum", "Vm_sum", "Wm_sum", "Um2_sum",
            "Vm2_sum", "Wm2_sum", "UmWm_sum")
SPECTRA = ("E_uu_2d_sum", "E_vv_2d_sum", "E_ww_2d_sum", "E_uw_2d_sum")


class TurbulenceStats:
    def __init__(self, nx, ny, nz, Lx, Ly, Lz, z_c, z_f, dz_c, dz_f, dx, dy, nu, Re_tau_target,
                 z_plus_target=15.0, device="cuda", top_wall_bc_type="dirichlet",
                 spectra_z_planes=None, grid=None):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.Lx, self.Ly, self.Lz = Lx, Ly, Lz
        self.z_c, self.z_f, self.dz_c, self.dz_f = z_c, z_f, dz_c, dz_f
        self.dx, self.dy, self.nu = dx, dy, nu
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise RuntimeError("slchannel_b200 runs on a CUDA device (sm_100a); there is no CPU path")
        self.top_wall_bc_type = top_wall_bc_type
        delta = Lz / 2.0
        self.u_tau_target = Re_tau_target * nu / delta
        z_target = z_plus_target * nu / self.u_tau_target
        zci = torch.as_tensor(z_c, dtype=torch.float64).cpu()[1:nz + 1]
        self.k_bot = int(torch.argmin(torch.abs(zci - z_target)).item()) + 1
        self.k_top = int(torch.argmin(torch.abs(zci - (Lz - z_target))).item()) + 1
        self.n_samples = 0
        f = dict(dtype=torch.float64, device=self.device)
        self._prof = torch.zeros(len(PROFILES), nz, **f)
        for q, name in enumerate(PROFILES):
            setattr(self, name, self._prof[q])
        nkx, nky = nx // 2, ny // 2
        self._spec = torch.zeros(4, nkx, nky, **f)
        self.E_uu_2d_sum, self.E_vv_2d_sum, self.E_ww_2d_sum, self.E_uw_2d_sum = self._spec
        self.kx = 2 * np.pi * np.fft.rfftfreq(nx, d=dx)[1:]
        self.ky = 2 * np.pi * np.fft.rfftfreq(ny, d=dy)[1:]
        self.spectra_z_planes = [float(zp) for zp in (spectra_z_planes or [])]
        self.n_samples_extra = 0
        self.extra_planes = []
        for zp in self.spectra_z_planes:
            z_t = zp * nu / self.u_tau_target
            kb = int(torch.argmin(torch.abs(zci - z_t)).item()) + 1
            kt = int(torch.argmin(torch.abs(zci - (Lz - z_t))).item()) + 1
            spec = torch.zeros(4, nkx, nky, **f)
            self.extra_planes.append({"zp": zp, "k_bot": kb, "k_top": kt, "spec": spec,
                                      "sums": dict(zip(("uu", "vv", "ww", "uw"), spec))})
        if grid is None:
            zf = torch.as_tensor(z_f, dtype=torch.float64)
            zc = torch.as_tensor(z_c, dtype=torch.float64)
            # the statistics kernels use only the grid sizes and workspaces;
            # gamma does not enter them
            grid = N.Grid(nx, ny, nz, Lx, Ly, Lz, 1.0, zf, zc, order=4, nu=nu,
                          top_wall_bc_type=top_wall_bc_type, device=self.device)
        self._grid = grid

    def accumulate_statistics(self, u, v, w, u_tau_current=None):
        """turbstats.py:156-360 -- add one snapshot (asynchronous)."""
        s = N.stream_of(u)
        self._grid.call("slc_stats_accumulate", N.ptr(u), N.ptr(v), N.ptr(w), N.ptr(self._prof),
                        N.ptr(self._spec), self.k_bot, self.k_top, s)
        for pl in self.extra_planes:
            self._grid.call("slc_stats_accumulate", N.ptr(u), N.ptr(v), N.ptr(w), None,
                            N.ptr(pl["spec"]), pl["k_bot"], pl["k_top"], s)
        if self.extra_planes:
            self.n_samples_extra += 1
        self.n_samples += 1

    def finalize_statistics(self):
        """turbstats.py:362-462 -- averages with the time-mean correction."""
        if self.n_samples == 0:
            raise RuntimeError("No samples accumulated - cannot finalize statistics")
        n = self.n_samples
        U = self.U_sum / n
        Vm, Wm = self.Vm_sum / n, self.Wm_sum / n
        uu = self.uu_sum / n + self.Um2_sum / n - U**2
        vv = self.vv_sum / n + self.Vm2_sum / n - Vm**2
        ww = self.ww_sum / n + self.Wm2_sum / n - Wm**2
        uw = self.uw_sum / n + self.UmWm_sum / n - U * Wm
        dz_utau = float(self.z_c[1])
        if self.top_wall_bc_type == "neumann":
            dUdz = float(U[0] / dz_utau)
        else:
            dUdz = float(0.5 * (U[0] + U[-1]) / dz_utau)
        c = lambda t: np.asarray(t.detach().cpu().numpy())  # noqa: E731
        stats = {
            "n_samples": n, "z_c": c(torch.as_tensor(self.z_c)[1:self.nz + 1]),
            "U_mean": c(U), "uu_mean": c(uu), "vv_mean": c(vv), "ww_mean": c(ww), "uw_mean": c(uw),
            "kx": self.kx[: self.nx // 2], "ky": self.ky[: self.ny // 2],
            "E_uu_2d": c(self.E_uu_2d_sum / n), "E_vv_2d": c(self.E_vv_2d_sum / n),
            "E_ww_2d": c(self.E_ww_2d_sum / n), "E_uw_2d": c(self.E_uw_2d_sum / n),
            "z_plus_target": self.k_bot,
            "Re_tau_target": self.u_tau_target * (self.Lz / 2) / self.nu,
            "nu": self.nu, "Re": 1.0 / self.nu, "u_tau": float(np.sqrt(self.nu * dUdz)),
        }
        if self.extra_planes and self.n_samples_extra > 0:
            stats["n_samples_extra"] = self.n_samples_extra
            stats["spectra_z_planes"] = np.asarray(self.spectra_z_planes)
            for pl in self.extra_planes:
                stats[f"z_index_z{pl['zp']:.0f}"] = pl["k_bot"]
                for k in ("uu", "vv", "ww", "uw"):
                    stats[f"E_{k}_2d_z{pl['zp']:.0f}"] = c(pl["sums"][k] / self.n_samples_extra)
        return stats

    def save_statistics(self, filepath):
        """turbstats.py:464-473 -- the finalized statistics as a compressed .npz."""
        np.savez_compressed(filepath, **self.finalize_statistics())

    @staticmethod
    def load_statistics(filepath):
        """turbstats.py:475-490 -- a saved statistics file as a dict of arrays."""
        if not os.path.exists(filepath):
            raise FileNotFoundError(f"Statistics file not found: {filepath}")
        data = np.load(filepath)
        return {key: data[key] for key in data.files}

    def save_state(self, filepath):
        """turbstats.py:492-534 -- the running sums and sample counts in the
        reference's key layout, so a run can continue the accumulation of
        either implementation after a restart."""
        c = lambda t: np.asarray(t.detach().cpu().numpy())  # noqa: E731
        state = {"n_samples": self.n_samples}
        for name in PROFILES + SPECTRA:
            state[name] = c(getattr(self, name))
        state.update(nx=self.nx, ny=self.ny, nz=self.nz)
        if self.extra_planes:
            state["n_samples_extra"] = self.n_samples_extra
            state["spectra_z_planes"] = np.asarray(self.spectra_z_planes)
            for pl in self.extra_planes:
                for k in ("uu", "vv", "ww", "uw"):
                    state[f"E_{k}_2d_z{pl['zp']:.0f}_sum"] = c(pl["sums"][k])
        np.savez_compressed(filepath, **state)

    def load_state(self, filepath):
        """turbstats.py:536-609 -- restore the running sums written by
        save_state (this implementation's or the reference's).  The values are
        copied into the existing device accumulators, which the statistics
        kernel updates in place.  Extra spectra planes are restored only when
        the file holds the same plane set; otherwise they start at this
        restart.  A file without the plane-mean moments (written before the
        reference added them) leaves those at zero and warns: the normal
        stresses of its samples are biased low by the time variance of the
        plane mean, which cannot be recovered."""
        if not os.path.exists(filepath):
            raise FileNotFoundError(f"Statistics state file not found: {filepath}")
        data = np.load(filepath)
        if data["nx"] != self.nx or data["ny"] != self.ny or data["nz"] != self.nz:
            raise ValueError(
                f"Grid dimension mismatch! State file has (nx={data['nx']}, ny={data['ny']}, "
                f"nz={data['nz']}) but current simulation has (nx={self.nx}, ny={self.ny}, "
                f"nz={self.nz})")

        def put(dst, key):
            src = torch.as_tensor(np.asarray(data[key]), dtype=torch.float64)
            if tuple(src.shape) != tuple(dst.shape):
                raise ValueError(f"{key}: shape {tuple(src.shape)} in the state file, "
                                 f"{tuple(dst.shape)} expected")
            dst.copy_(src)

        self.n_samples = int(data["n_samples"])
        for name in ("U_sum", "uu_sum", "vv_sum", "ww_sum", "uw_sum") + SPECTRA:
            put(getattr(self, name), name)
        saved_planes = (list(np.asarray(data["spectra_z_planes"]).ravel())
                        if "spectra_z_planes" in data.files else [])
        if self.extra_planes and saved_planes == self.spectra_z_planes:
            self.n_samples_extra = int(data["n_samples_extra"])
            for pl in self.extra_planes:
                for k in ("uu", "vv", "ww", "uw"):
                    put(pl["sums"][k], f"E_{k}_2d_z{pl['zp']:.0f}_sum")
        if "Um2_sum" in data.files:
            for name in ("Vm_sum", "Wm_sum", "Um2_sum", "Vm2_sum", "Wm2_sum", "UmWm_sum"):
                put(getattr(self, name), name)
        else:
            warnings.warn("statistics state predates the plane-mean moments: normal stresses "
                          "of its samples are biased low by the time variance of the plane mean",
                          RuntimeWarning, stacklevel=2)
