"""Golden values for the on-device diagnostics and statistics, from the
REFERENCE (gmcavallazzi/SLchannel v1.0.1): compute_divergence,
compute_u_tau, compute_cfl_fused, compute_bulk_velocity and TurbulenceStats
(two snapshots, profiles, spectra at the z+ = 15 planes and at an extra
z+ = 30 pair, finalize_statistics) on a seeded 16 x 12 x 20 channel.

    python tests/golden/make_diag_golden.py /path/to/SLchannel

The input fields are `snapshot(seed)` below: plain numpy, with the
reference's ghost refresh applied, rebuilt identically by the GPU test.
"""

import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CASE = dict(nx=16, ny=12, nz=20, Lx=2 * math.pi, Ly=math.pi, Lz=2.0, gamma=1.8, nu=1.0 / 800.0,
            Re_tau=180.0, zplus=15.0, extra=(30.0,), seeds=(31, 32))


def snapshot(z_f, z_c, seed):
    """Ghost-shaped (u, v, w): Poiseuille + seeded smooth modes + seeded
    noise (not divergence-free); ghosts refreshed by the caller."""
    from make_adjoint_golden import initial_field

    c = dict(nx=CASE["nx"], ny=CASE["ny"], nz=CASE["nz"], Lx=CASE["Lx"], Ly=CASE["Ly"], Lz=CASE["Lz"],
             field_seed=seed)
    u, v, w = initial_field(c, z_f, z_c)
    r = np.random.default_rng(seed + 1000)
    return [a + 0.02 * r.normal(size=a.shape) for a in (u, v, w)]


def main(ref_root):
    from make_golden import _stub_matplotlib

    _stub_matplotlib()
    sys.path.insert(0, ref_root)
    import torch

    torch.set_default_dtype(torch.float64)
    import slchannel.solver as ref_solver
    from slchannel.operators import compute_cfl_fused
    from slchannel.turbstats import TurbulenceStats
    from slchannel.utils import compute_bulk_velocity, compute_divergence, compute_u_tau, generate_grid

    c = CASE
    nx, ny, nz = c["nx"], c["ny"], c["nz"]
    dx, dy = c["Lx"] / nx, c["Ly"] / ny
    z_f, z_c, dz_f, dz_c = generate_grid(c["gamma"], nz, c["Lz"])
    res = {"z_f": z_f.numpy(), "z_c": z_c.numpy()}
    stats = TurbulenceStats(nx, ny, nz, c["Lx"], c["Ly"], c["Lz"], z_c, z_f, dz_c, dz_f, dx, dy, c["nu"],
                            c["Re_tau"], z_plus_target=c["zplus"], device="cpu",
                            spectra_z_planes=list(c["extra"]))
    for n, seed in enumerate(c["seeds"]):
        u, v, w = (torch.from_numpy(a) for a in snapshot(z_f.numpy(), z_c.numpy(), seed))
        ref_solver.apply_bc_all(u, v, w, "dirichlet")
        if n == 0:
            div = compute_divergence(u, v, w, nx, ny, nz, dx, dy, dz_f)
            res["max_div"] = np.array(float(div.abs().max()))
            res["u_tau_dirichlet"] = np.array(float(compute_u_tau(u, z_c, c["nu"], "dirichlet")))
            res["u_tau_neumann"] = np.array(float(compute_u_tau(u, z_c, c["nu"], "neumann")))
            res["cfl_dti"] = np.array(float(compute_cfl_fused(u, v, w, nx, ny, nz, dx, dy, dz_f, dz_c)))
            cvr = (dx * dy * dz_f.view(1, 1, -1)).expand(nx, ny, nz)
            res["u_bulk"] = np.array(float(compute_bulk_velocity(u, cvr, c["Lx"] * c["Ly"] * c["Lz"])))
        stats.accumulate_statistics(u, v, w, 0.05)
    for k in ("U_sum", "uu_sum", "vv_sum", "ww_sum", "uw_sum", "Vm_sum", "Wm_sum", "Um2_sum", "Vm2_sum",
              "Wm2_sum", "UmWm_sum", "E_uu_2d_sum", "E_vv_2d_sum", "E_ww_2d_sum", "E_uw_2d_sum"):
        res[k] = getattr(stats, k).numpy()
    res["k_bot"], res["k_top"] = np.array(stats.k_bot), np.array(stats.k_top)
    for pl in stats.extra_planes:
        for k, t in pl["sums"].items():
            res[f"extra_{pl['zp']:.0f}_{k}"] = t.numpy()
    fin = stats.finalize_statistics()
    for k in ("U_mean", "uu_mean", "vv_mean", "ww_mean", "uw_mean", "E_uu_2d", "E_uw_2d", "u_tau"):
        res[f"fin_{k}"] = np.asarray(fin[k])
    np.savez_compressed(os.path.join(HERE, "diagnostics.npz"), **res)
    print({k: (v if np.asarray(v).size < 3 else np.asarray(v).shape) for k, v in res.items()})


if __name__ == "__main__":
    sys.path.insert(0, HERE)
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SLCHANNEL_REF", "."))
