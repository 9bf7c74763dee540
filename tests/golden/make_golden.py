"""Generate the golden vectors in tests/golden/ by running the REFERENCE itself
(gmcavallazzi/SLchannel v1.0.1, its float64 eager CPU path).

Run in a container that has the reference source tree (read-only is fine):

    python tests/golden/make_golden.py /path/to/SLchannel

The reference imports matplotlib at module level (slchannel/utils.py:19) only
for plots; a stub module with no-op plotting functions stands in for it.

Every case uses seeded inputs built here with numpy, so the fixtures can be
regenerated bit-for-bit.  Outputs are small .npz files (a few hundred KB in
all) that the CPU tests compare the oracle against, and that the GPU tests
compare the CUDA path against.
"""

import os
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _stub_matplotlib():
    mpl = types.ModuleType("matplotlib")
    plt = types.ModuleType("matplotlib.pyplot")

    def _noop(*a, **k):
        return None

    for name in ("figure", "plot", "xlabel", "ylabel", "title", "legend", "grid",
                 "savefig", "close", "semilogx", "subplots", "tight_layout"):
        setattr(plt, name, _noop)
    mpl.pyplot = plt
    mpl.use = _noop
    sys.modules["matplotlib"] = mpl
    sys.modules["matplotlib.pyplot"] = plt


def smooth_field(rng, X, Y, Z, Lx, Ly, Lz, amp, nmodes=4, wall_damp=True):
    """Seeded sum of low Fourier modes in x, y times a low polynomial in z."""
    f = np.zeros(np.broadcast_shapes(X.shape, Y.shape, Z.shape))
    for _ in range(nmodes):
        kx = rng.integers(0, 3)
        ky = rng.integers(0, 3)
        ph = rng.uniform(0, 2 * np.pi, 2)
        a = rng.normal()
        zz = Z / Lz
        zpoly = 1.0 + rng.normal() * zz + rng.normal() * zz**2
        if wall_damp:
            zpoly = zpoly * (zz * (1 - zz)) * 4.0
        f = f + a * np.cos(2 * np.pi * kx * X / Lx + ph[0]) * np.cos(2 * np.pi * ky * Y / Ly + ph[1]) * zpoly
    return amp * f


def positions(comp, nx, ny, dx, dy, z_f, z_c):
    """Physical positions of every entry of a ghost-shaped array."""
    if comp == "u":
        X = (np.arange(0, nx + 1) * dx)[:, None, None]
        Y = ((np.arange(0, ny + 2) - 0.5) * dy)[None, :, None]
        Z = z_c[None, None, :]
    elif comp == "v":
        X = ((np.arange(0, nx + 2) - 0.5) * dx)[:, None, None]
        Y = (np.arange(0, ny + 1) * dy)[None, :, None]
        Z = z_c[None, None, :]
    else:
        X = ((np.arange(0, nx + 2) - 0.5) * dx)[:, None, None]
        Y = ((np.arange(0, ny + 2) - 0.5) * dy)[None, :, None]
        Z = z_f[None, None, :]
    return X, Y, Z


def main(ref_root):
    _stub_matplotlib()
    sys.path.insert(0, ref_root)
    import torch

    torch.set_default_dtype(torch.float64)
    torch.set_num_threads(1)
    import yaml

    import slchannel.solver as ref_solver
    from slchannel.semilag import SLAdvector
    from slchannel.utils import generate_grid

    T = lambda a: torch.from_numpy(np.ascontiguousarray(a))  # noqa: E731
    N = lambda t: t.detach().cpu().numpy().copy()  # noqa: E731

    # ------------------------------------------------------------------ zmap
    zmap = {}
    rng = np.random.default_rng(11)
    for st in ("symmetric", "bottom"):
        for gamma in (0.8, 1.8, 2.6):
            for nz in (64, 180):
                z_f, z_c, _, _ = generate_grid(gamma, nz, 2.0, stretching_type=st)
                adv = SLAdvector(4, 4, nz, 0.5, 0.5, 2.0, 2.0, 2.0, z_f, z_c, gamma,
                                 stretching_type=st)
                z = np.concatenate([N(z_f), rng.uniform(0.0, 2.0, 200)])
                key = f"{st}_{gamma}_{nz}"
                zmap[f"z_{key}"] = z
                zmap[f"kf_{key}"] = N(adv._face_coord(T(z)))
                zmap[f"zf_{key}"] = N(z_f)
                zmap[f"zc_{key}"] = N(z_c)
    np.savez_compressed(os.path.join(HERE, "zmap.npz"), **zmap)

    # ------------------------------------------------ interp / departure / advect
    nx, ny, nz = 10, 8, 14
    Lx, Ly, Lz = 2 * np.pi, np.pi, 2.0
    gamma = 1.8
    dx, dy = Lx / nx, Ly / ny
    z_f, z_c, _, _ = generate_grid(gamma, nz, Lz, stretching_type="symmetric")
    zf, zc = N(z_f), N(z_c)
    out = {"grid": np.array([nx, ny, nz, Lx, Ly, Lz, gamma]), "z_f": zf, "z_c": zc}
    rng = np.random.default_rng(12)
    npts = 300
    for order in (4, 6):
        adv = SLAdvector(nx, ny, nz, dx, dy, Lx, Ly, Lz, z_f, z_c, gamma, order=order)
        for comp in "uvw":
            spec = adv.spec[comp]
            buf = rng.normal(size=(spec.NX, spec.NY, spec.NZ))
            x = rng.uniform(-Lx, 2 * Lx, npts)
            y = rng.uniform(-Ly, 2 * Ly, npts)
            z = rng.uniform(-0.05, Lz + 0.05, npts)  # some outside: clamped + counted
            # a few points on nodes, on walls and on periodic seams
            x[:4] = [0.0, dx, Lx, -dx]
            y[:4] = [0.0, dy * 0.5, Ly, Ly + 0.5 * dy]
            z[:4] = [zf[0], zc[1], zf[-1], zc[nz // 2]]
            iw = adv._build_iw(spec, T(x), T(y), T(z), order, count_clamp=True)
            vals = adv._apply_iw(T(buf), iw)
            key = f"o{order}_{comp}"
            out[f"interp_buf_{key}"] = buf
            out[f"interp_x_{key}"] = x
            out[f"interp_y_{key}"] = y
            out[f"interp_z_{key}"] = z
            out[f"interp_out_{key}"] = N(vals)
            out[f"interp_ncl_{key}"] = np.array(int(iw.n_clamped))

    # trajectory velocity (ghost-shaped, BC-consistent) and fields
    def fields(seed, amp_u, amp_w, mean=True):
        r = np.random.default_rng(seed)
        res = {}
        for comp in "uvw":
            X, Y, Z = positions(comp, nx, ny, dx, dy, zf, zc)
            f = smooth_field(r, X, Y, Z, Lx, Ly, Lz, amp_w if comp == "w" else amp_u)
            if comp == "u" and mean:
                f = f + 1.5 * Z * (2 - Z)
            res[comp] = np.ascontiguousarray(f * np.ones(np.broadcast_shapes(X.shape, Y.shape, Z.shape)))
        u, v, w = (T(res[c]).clone() for c in "uvw")
        ref_solver.apply_bc_all(u, v, w, "dirichlet")
        return N(u), N(v), N(w)

    mu, mv, mw = fields(21, 0.4, 0.3)
    fu, fv, fw = fields(22, 1.0, 1.0, mean=False)
    out.update(mid_u=mu, mid_v=mv, mid_w=mw, f_u=fu, f_v=fv, f_w=fw)
    for order in (4, 6):
        adv = SLAdvector(nx, ny, nz, dx, dy, Lx, Ly, Lz, z_f, z_c, gamma, order=order)
        for dt in (0.3, 0.9):
            for comp in ("uvw" if order == 4 else ""):  # feet do not depend on order
                adv._fill(adv.mbuf["u"], "u", T(mu))
                adv._fill(adv.mbuf["v"], "v", T(mv))
                adv._fill(adv.mbuf["w"], "w", T(mw))
                xd, yd, zd = adv.departure_coords(comp, torch.tensor(dt))
                key = f"dt{dt}_{comp}"
                out[f"dep_x_{key}"] = N(xd)
                out[f"dep_y_{key}"] = N(yd)
                out[f"dep_z_{key}"] = N(zd)
            us, vs, ws = adv.advect(T(fu), T(fv), T(fw), T(mu), T(mv), T(mw), torch.tensor(dt))
            key = f"o{order}_dt{dt}"
            out[f"adv_u_{key}"] = N(us)[1 : nx + 1, 1 : ny + 1, 1 : nz + 1]
            out[f"adv_v_{key}"] = N(vs)[1 : nx + 1, 1 : ny + 1, 1 : nz + 1]
            out[f"adv_w_{key}"] = N(ws)[1 : nx + 1, 1 : ny + 1, 1:nz]
            out[f"adv_ncl_{key}"] = np.array(int(adv.n_clamped_last))
    # wall clamps: uniform vertical trajectory velocity, walls included
    # (as tests/test_sl_wall_clamp.py builds it)
    for w0 in (-0.5, 0.5):
        cu = np.full((nx + 1, ny + 2, nz + 2), 0.3)
        cv = np.zeros((nx + 2, ny + 1, nz + 2))
        cw = np.full((nx + 2, ny + 2, nz + 1), w0)
        out[f"clamp_mid_u_{w0}"], out[f"clamp_mid_v_{w0}"], out[f"clamp_mid_w_{w0}"] = cu, cv, cw
        for order in (4, 6):
            adv = SLAdvector(nx, ny, nz, dx, dy, Lx, Ly, Lz, z_f, z_c, gamma, order=order)
            us, vs, ws = adv.advect(T(fu), T(fv), T(fw), T(cu), T(cv), T(cw), torch.tensor(0.5))
            key = f"o{order}_w{w0}"
            out[f"clamp_u_{key}"] = N(us)[1 : nx + 1, 1 : ny + 1, 1 : nz + 1]
            out[f"clamp_v_{key}"] = N(vs)[1 : nx + 1, 1 : ny + 1, 1 : nz + 1]
            out[f"clamp_w_{key}"] = N(ws)[1 : nx + 1, 1 : ny + 1, 1:nz]
            out[f"clamp_ncl_{key}"] = np.array(int(adv.n_clamped_last))
    np.savez_compressed(os.path.join(HERE, "advect.npz"), **out)

    # ------------------------------------------------------------ full steps
    cases = [
        dict(name="o6_sym", order=6, st="symmetric", top="dirichlet", capture=(1, 3)),
        dict(name="o4_sym", order=4, st="symmetric", top="dirichlet", capture=(3,)),
        dict(name="o4_bottom_neumann", order=4, st="bottom", top="neumann", capture=()),
        # the incremental pressure branch (solver.py:905-941, 1001-1012) and the
        # order-4 trajectory sampling (semilag.py:206-209, 512-528)
        dict(name="o6_inc", order=6, st="symmetric", top="dirichlet", capture=(3,), pressure="inc"),
        dict(name="o6_traj4", order=6, st="symmetric", top="dirichlet", capture=(3,), traj=4),
        dict(name="o4_inc_traj4_bottom_neumann", order=4, st="bottom", top="neumann", capture=(),
             pressure="inc", traj=4),
    ]
    snx, sny, snz = 8, 6, 12
    sLx, sLy, sLz = 2 * np.pi, np.pi, 2.0
    sgamma, Re, dt, nsteps = 2.0, 200.0, 0.3, 4
    for case in cases:
        with tempfile.TemporaryDirectory() as tmp:
            cfg = {
                "grid": {"nx": snx, "ny": sny, "nz": snz},
                "domain": {"Lx": float(sLx), "Ly": float(sLy), "Lz": sLz,
                           "stretching_type": case["st"]},
                "flow": {"Re": Re, "Re_tau": 180.0, "U_bulk": 1.0, "gamma": sgamma},
                "boundary_conditions": {"top_wall": {"type": case["top"]}},
                "initialization": {"type": "parabolic", "perturbation_intensity": 0.0},
                "solver": {"type": "fft"},
                "time": {"dt": dt, "n_steps": nsteps, "t_max": 1e9, "CFL_target": 3.0,
                         "dt_update_interval": 0, "dt_max": 1.0, "dt_min": 1e-4},
                "compute": {"device": "cpu"},
                "output": {"results_folder": os.path.join(tmp, "results"),
                           "n_out": 10**8, "n_save": 10**8},
                "advection": {"scheme": "sl"},
                "sl": {"interp_order": case["order"], "n_traj_iters": 2,
                       "interp_dtype": "fp64", "traj_interp_order": case.get("traj", 2),
                       "bdf2_pressure": case.get("pressure", "noninc")},
                "statistics": {"n_stats": 0},
            }
            path = os.path.join(tmp, "cfg.yaml")
            with open(path, "w") as fh:
                yaml.safe_dump(cfg, fh)
            s = ref_solver.SLChannelFlow(config_file=path)
            sdx, sdy = s.dx, s.dy
            szf, szc = N(s.z_f), N(s.z_c)
            r = np.random.default_rng(31)
            init = {}
            for comp in "uvw":
                if comp == "u":
                    X = (np.arange(0, snx + 1) * sdx)[:, None, None]
                    Y = ((np.arange(0, sny + 2) - 0.5) * sdy)[None, :, None]
                    Z = szc[None, None, :]
                elif comp == "v":
                    X = ((np.arange(0, snx + 2) - 0.5) * sdx)[:, None, None]
                    Y = (np.arange(0, sny + 1) * sdy)[None, :, None]
                    Z = szc[None, None, :]
                else:
                    X = ((np.arange(0, snx + 2) - 0.5) * sdx)[:, None, None]
                    Y = ((np.arange(0, sny + 2) - 0.5) * sdy)[None, :, None]
                    Z = szf[None, None, :]
                f = smooth_field(r, X, Y, Z, sLx, sLy, sLz, 0.35)
                if comp == "u":
                    f = f + 1.5 * Z * (2 - Z) / sLz
                init[comp] = f * np.ones(np.broadcast_shapes(X.shape, Y.shape, Z.shape))
            s.u, s.v, s.w = (T(init[c]).clone() for c in "uvw")
            s.apply_bc_uvw()
            # project with the reference's own Poisson (solver.py:593-613)
            div = ref_solver.compute_divergence(s.u, s.v, s.w, snx, sny, snz, sdx, sdy, s.dz_f)
            s.p = ref_solver.solve_poisson_fft(div, s.fft_data).clone()
            s.u, s.v, s.w = ref_solver.project_velocity(s.u, s.v, s.w, s.p, snx, sny, snz, sdx,
                                                        sdy, s.dz_c, s.dz_f, 1.0)
            s.apply_bc_uvw()
            res = {
                "params": np.array([snx, sny, snz, sLx, sLy, sLz, sgamma, Re, dt, case["order"]]),
                "stretching": np.array(case["st"]),
                "top": np.array(case["top"]),
                "pressure": np.array(case.get("pressure", "noninc")),
                "traj_order": np.array(case.get("traj", 2)),
                "z_f": szf, "z_c": szc,
                "init_u": N(s.u), "init_v": N(s.v), "init_w": N(s.w), "init_p": N(s.p),
            }

            # substep capture hooks (record, then delegate to the reference)
            rec = {}
            orig_adv = s.sl.advect

            def adv_hook(*a, **k):
                o = orig_adv(*a, **k)
                # interiors only: advect() leaves its ghosts stale (semilag.py:594-596)
                rec.setdefault("advect", []).append((
                    N(o[0])[1 : snx + 1, 1 : sny + 1, 1 : snz + 1],
                    N(o[1])[1 : snx + 1, 1 : sny + 1, 1 : snz + 1],
                    N(o[2])[1 : snx + 1, 1 : sny + 1, 1:snz],
                ))
                return o

            s.sl.advect = adv_hook
            zfns = {}
            for c in "uvw":
                name = f"solve_implicit_diffusion_{c}"
                orig = getattr(ref_solver, name)
                zfns[name] = orig

                def zhook(*a, _orig=orig, _c=c, **k):
                    rec.setdefault("zin", {})[_c] = N(a[0])
                    o = _orig(*a, **k)
                    rec.setdefault("zout", {})[_c] = N(o)
                    return o

                setattr(ref_solver, name, zhook)
            orig_poisson = s._solve_poisson

            def phook(rhs):
                o = orig_poisson(rhs)
                rec["phi"] = N(o)
                return o

            s._solve_poisson = phook
            orig_proj = ref_solver.project_velocity

            def prhook(*a, **k):
                o = orig_proj(*a, **k)
                rec["proj"] = tuple(N(t) for t in o)
                return o

            ref_solver.project_velocity = prhook
            try:
                for step in range(1, nsteps + 1):
                    rec.clear()
                    ub, forcing = s.step_sl_bdf2(dt)
                    res[f"s{step}_u"], res[f"s{step}_v"], res[f"s{step}_w"] = N(s.u), N(s.v), N(s.w)
                    res[f"s{step}_p"] = N(s.p)
                    res[f"s{step}_ubulk"] = np.array(float(ub))
                    res[f"s{step}_forcing"] = np.array(float(forcing))
                    res[f"s{step}_nclamp"] = np.array(int(s.sl.n_clamped_last))
                    if step in case["capture"]:
                        advs = rec["advect"]
                        if step == 1:
                            res[f"s{step}_ubar"] = np.concatenate([a.ravel() for a in advs[0]])
                        else:
                            res[f"s{step}_ubarbar"] = np.concatenate([a.ravel() for a in advs[0]])
                            res[f"s{step}_ubar"] = np.concatenate([a.ravel() for a in advs[1]])
                        for c in "uvw":
                            res[f"s{step}_uhat_{c}"] = rec["zin"][c]
                            res[f"s{step}_zsolve_{c}"] = rec["zout"][c]
                        res[f"s{step}_phi"] = rec["phi"]
                        for c, a in zip("uvw", rec["proj"]):
                            res[f"s{step}_proj_{c}"] = a
            finally:
                for name, fn in zfns.items():
                    setattr(ref_solver, name, fn)
                ref_solver.project_velocity = orig_proj
            np.savez_compressed(os.path.join(HERE, f"step_{case['name']}.npz"), **res)
    print("golden vectors written to", HERE)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SLCHANNEL_REF", "."))
