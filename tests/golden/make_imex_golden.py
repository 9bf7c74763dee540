"""Golden vectors of the reference's Eulerian IMEX scheme (gmcavallazzi/
SLchannel v1.0.1: compute_momentum_rhs_fused_imex, operators.py:638-832;
SLChannelFlow.step_imex, solver.py:1055-1135): the explicit right-hand side
of a seeded state and four IMEX steps, on an 8 x 6 x 12 channel, for a
symmetric grid with no-slip walls and a bottom-stretched grid with a
free-slip top.

    python tests/golden/make_imex_golden.py /path/to/SLchannel
"""

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = [dict(name="sym", st="symmetric", top="dirichlet"),
         dict(name="bottom_neumann", st="bottom", top="neumann")]
NX, NY, NZ, LX, LY, LZ, GAMMA, RE, DT, NSTEPS = 8, 6, 12, 2 * np.pi, np.pi, 2.0, 2.0, 200.0, 0.02, 4


def main(ref_root):
    from make_golden import _stub_matplotlib, positions, smooth_field

    _stub_matplotlib()
    sys.path.insert(0, ref_root)
    import torch
    import yaml

    torch.set_default_dtype(torch.float64)
    import slchannel.solver as ref_solver
    from slchannel.operators import compute_momentum_rhs_fused_imex

    N = lambda t: t.detach().cpu().numpy().copy()  # noqa: E731
    for case in CASES:
        with tempfile.TemporaryDirectory() as tmp:
            cfg = {
                "grid": {"nx": NX, "ny": NY, "nz": NZ},
                "domain": {"Lx": float(LX), "Ly": float(LY), "Lz": LZ, "stretching_type": case["st"]},
                "flow": {"Re": RE, "Re_tau": 180.0, "U_bulk": 1.0, "gamma": GAMMA},
                "boundary_conditions": {"top_wall": {"type": case["top"]}},
                "initialization": {"type": "parabolic", "perturbation_intensity": 0.0},
                "solver": {"type": "fft"},
                "time": {"dt": DT, "n_steps": NSTEPS, "t_max": 1e9, "CFL_target": 0.3,
                         "dt_update_interval": 0, "dt_max": 1.0, "dt_min": 1e-4},
                "compute": {"device": "cpu"},
                "output": {"results_folder": os.path.join(tmp, "results"), "n_out": 10**8, "n_save": 10**8},
                "advection": {"scheme": "eulerian"},
                "statistics": {"n_stats": 0},
            }
            path = os.path.join(tmp, "cfg.yaml")
            with open(path, "w") as fh:
                yaml.safe_dump(cfg, fh)
            s = ref_solver.SLChannelFlow(config_file=path)
            zf, zc = N(s.z_f), N(s.z_c)
            r = np.random.default_rng(77)
            init = {}
            for ci, comp in enumerate("uvw"):
                X, Y, Z = positions(comp, NX, NY, s.dx, s.dy, zf, zc)
                f = smooth_field(r, X, Y, Z, LX, LY, LZ, 0.35)
                if comp == "u":
                    f = f + 1.5 * Z * (2 - Z) / LZ
                init[comp] = f * np.ones(np.broadcast_shapes(X.shape, Y.shape, Z.shape))
            s.u, s.v, s.w = (torch.from_numpy(init[c]).clone() for c in "uvw")
            s.apply_bc_uvw()
            div = ref_solver.compute_divergence(s.u, s.v, s.w, NX, NY, NZ, s.dx, s.dy, s.dz_f)
            s.p = ref_solver.solve_poisson_fft(div, s.fft_data).clone()
            s.u, s.v, s.w = ref_solver.project_velocity(s.u, s.v, s.w, s.p, NX, NY, NZ, s.dx, s.dy, s.dz_c,
                                                        s.dz_f, 1.0)
            s.apply_bc_uvw()
            res = {"params": np.array([NX, NY, NZ, LX, LY, LZ, GAMMA, RE, DT]),
                   "stretching": np.array(case["st"]), "top": np.array(case["top"]),
                   "z_f": zf, "z_c": zc, "init_u": N(s.u), "init_v": N(s.v), "init_w": N(s.w),
                   "init_p": N(s.p)}
            ru, rv, rw = compute_momentum_rhs_fused_imex(s.u, s.v, s.w, NX, NY, NZ, s.dx, s.dy, s.dz_c,
                                                         s.dz_f, s.nu)
            res["rhs_u"], res["rhs_v"], res["rhs_w"] = N(ru), N(rv), N(rw)
            for step in range(1, NSTEPS + 1):
                ub, forcing = s.step_imex(DT)
                res[f"s{step}_u"], res[f"s{step}_v"], res[f"s{step}_w"] = N(s.u), N(s.v), N(s.w)
                res[f"s{step}_p"] = N(s.p)
                res[f"s{step}_ubulk"] = np.array(float(ub))
                res[f"s{step}_forcing"] = np.array(float(forcing))
            np.savez_compressed(os.path.join(HERE, f"imex_{case['name']}.npz"), **res)
    print("imex goldens written")


if __name__ == "__main__":
    sys.path.insert(0, HERE)
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SLCHANNEL_REF", "."))
