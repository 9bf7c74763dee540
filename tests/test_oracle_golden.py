"""Pin the oracle to the reference: every golden vector in tests/golden/ (made
by running the reference itself, see make_golden.py) is reproduced by the CPU
restatement in oracle/.  CPU only.

Tolerances: the trace/gather restatement keeps the reference's operation order,
so it is held to 1e-13 relative (it is bit-identical in practice); full steps
go through FFTs and a PCR solve whose rounding is library-dependent and are
held to 1e-12 relative (pressure, a small field, to 1e-11 of its max)."""

import numpy as np
import pytest
from helpers import interior, load_golden, rel_err

from oracle.slbdf2 import OracleAdvector, OracleChannel, generate_grid


@pytest.fixture(scope="module")
def adv_golden():
    return load_golden("advect.npz")


def _grid(d):
    nx, ny, nz, Lx, Ly, Lz, gamma = d["grid"]
    nx, ny, nz = int(nx), int(ny), int(nz)
    return nx, ny, nz, Lx, Ly, Lz, gamma


def test_grid_restatement(adv_golden):
    nx, ny, nz, Lx, Ly, Lz, gamma = _grid(adv_golden)
    z_f, z_c, _, _ = generate_grid(gamma, nz, Lz)
    assert np.abs(z_f - adv_golden["z_f"]).max() < 1e-15
    assert np.abs(z_c - adv_golden["z_c"]).max() < 1e-15


def test_zmap_golden():
    z = load_golden("zmap.npz")
    keys = [k[2:] for k in z.files if k.startswith("z_")]
    assert len(keys) == 12
    for key in keys:
        st, g, n = key.split("_")
        adv = OracleAdvector(4, 4, int(n), 0.5, 0.5, 2.0, 2.0, 2.0, z["zf_" + key], z["zc_" + key],
                             float(g), stretching_type=st)
        err = np.abs(adv.face_coord(z["z_" + key]) - z["kf_" + key]).max()
        assert err < 1e-12, (key, err)


@pytest.mark.parametrize("order", [4, 6])
def test_interp_golden(adv_golden, order):
    d = adv_golden
    nx, ny, nz, Lx, Ly, Lz, gamma = _grid(d)
    adv = OracleAdvector(nx, ny, nz, Lx / nx, Ly / ny, Lx, Ly, Lz, d["z_f"], d["z_c"], gamma,
                         order=order)
    for comp in "uvw":
        k = f"o{order}_{comp}"
        out, ncl = adv.interp(comp, order, d["interp_buf_" + k], d["interp_x_" + k],
                              d["interp_y_" + k], d["interp_z_" + k], count_clamp=True)
        assert rel_err(out, d["interp_out_" + k]) < 1e-13
        assert ncl == int(d["interp_ncl_" + k])


def test_departure_golden(adv_golden):
    d = adv_golden
    nx, ny, nz, Lx, Ly, Lz, gamma = _grid(d)
    adv = OracleAdvector(nx, ny, nz, Lx / nx, Ly / ny, Lx, Ly, Lz, d["z_f"], d["z_c"], gamma)
    mid = (d["mid_u"], d["mid_v"], d["mid_w"])
    for dt in (0.3, 0.9):
        for comp in "uvw":
            feet = adv.departure_coords(comp, *mid, dt)
            for a, nm in zip(feet, "xyz"):
                assert np.abs(a - d[f"dep_{nm}_dt{dt}_{comp}"]).max() < 1e-13


@pytest.mark.parametrize("order", [4, 6])
def test_advect_golden(adv_golden, order):
    d = adv_golden
    nx, ny, nz, Lx, Ly, Lz, gamma = _grid(d)
    adv = OracleAdvector(nx, ny, nz, Lx / nx, Ly / ny, Lx, Ly, Lz, d["z_f"], d["z_c"], gamma,
                         order=order)
    f = (d["f_u"], d["f_v"], d["f_w"])
    for dt in (0.3, 0.9):
        outs = adv.advect(*f, d["mid_u"], d["mid_v"], d["mid_w"], dt)
        for c, o in zip("uvw", outs):
            assert rel_err(interior(c, o, nx, ny, nz), d[f"adv_{c}_o{order}_dt{dt}"]) < 1e-13
        assert adv.n_clamped_last == int(d[f"adv_ncl_o{order}_dt{dt}"])
    for w0 in (-0.5, 0.5):
        mid = (d[f"clamp_mid_u_{w0}"], d[f"clamp_mid_v_{w0}"], d[f"clamp_mid_w_{w0}"])
        outs = adv.advect(*f, *mid, 0.5)
        for c, o in zip("uvw", outs):
            assert rel_err(interior(c, o, nx, ny, nz), d[f"clamp_{c}_o{order}_w{w0}"]) < 1e-13
        assert adv.n_clamped_last == int(d[f"clamp_ncl_o{order}_w{w0}"]) > 0


@pytest.mark.parametrize("order", [4, 6])
def test_advect_extra_rhs_golden(order):
    """advect(..., extra_rhs=[two triples]) of the reference: each extra triple
    is the advection of that triple along the same trajectory velocity (the
    same departure points), so the oracle's advect reproduces it."""
    d = load_golden("advect_extra.npz")
    nx, ny, nz, Lx, Ly, Lz, gamma = _grid(d)
    adv = OracleAdvector(nx, ny, nz, Lx / nx, Ly / ny, Lx, Ly, Lz, d["z_f"], d["z_c"], gamma,
                         order=order)
    f = tuple(d[f"f_{c}"] for c in "uvw")
    extra = [tuple(d[f"e{t}_{c}"] for c in "uvw") for t in range(2)]
    for name, pre, dt in (("dt0.3", "mid", 0.3), ("dt0.9", "mid", 0.9), ("clamp", "clamp_mid", 0.5)):
        mid = tuple(d[f"{pre}_{c}"] for c in "uvw")
        key = f"o{order}_{name}"
        outs = adv.advect(*f, *mid, dt)
        for c, o in zip("uvw", outs):
            assert rel_err(interior(c, o, nx, ny, nz), d[f"adv_{c}_{key}"]) < 1e-13
        assert adv.n_clamped_last == int(d[f"ncl_{key}"])
        for t, triple in enumerate(extra):
            outs = adv.advect(*triple, *mid, dt)
            for c, o in zip("uvw", outs):
                assert rel_err(interior(c, o, nx, ny, nz), d[f"extra{t}_{c}_{key}"]) < 1e-13, (t, c)


def oracle_from_step_golden(s):
    nx, ny, nz, Lx, Ly, Lz, gamma, Re, dt, order = s["params"]
    nx, ny, nz, order = int(nx), int(ny), int(nz), int(order)
    pressure = str(s["pressure"]) if "pressure" in s.files else "noninc"
    traj = int(s["traj_order"]) if "traj_order" in s.files else 2
    ch = OracleChannel(nx, ny, nz, Lx, Ly, Lz, gamma, 1.0 / Re, s["init_u"], s["init_v"],
                       s["init_w"], s["init_p"], stretching_type=str(s["stretching"]),
                       order=order, top_wall_bc_type=str(s["top"]), z_f=s["z_f"], z_c=s["z_c"],
                       traj_order=traj, bdf2_pressure=pressure)
    return ch, float(dt)


@pytest.mark.parametrize("name", ["o6_sym", "o4_sym", "o4_bottom_neumann", "o6_inc", "o6_traj4",
                                  "o4_inc_traj4_bottom_neumann"])
def test_step_golden(name):
    s = load_golden(f"step_{name}.npz")
    ch, dt = oracle_from_step_golden(s)
    nx, ny, nz = ch.nx, ch.ny, ch.nz
    for step in range(1, 5):
        ub, forcing, cap = ch.step_bdf2(dt, capture=True)
        for c in "uvw":
            assert rel_err(getattr(ch, c), s[f"s{step}_{c}"]) < 1e-12, (step, c)
        assert rel_err(ch.p, s[f"s{step}_p"]) < 1e-11
        assert abs(ub - float(s[f"s{step}_ubulk"])) < 1e-13
        assert abs(forcing - float(s[f"s{step}_forcing"])) < 1e-11
        assert ch.n_clamped_last == int(s[f"s{step}_nclamp"])
        if f"s{step}_phi" in s.files:
            assert rel_err(cap["phi"], s[f"s{step}_phi"]) < 1e-11
            ubar = np.concatenate([interior(c, a, nx, ny, nz).ravel()
                                   for c, a in zip("uvw", cap["ubar"])])
            assert rel_err(ubar, s[f"s{step}_ubar"]) < 1e-13
            if step > 1:
                ubb = np.concatenate([interior(c, a, nx, ny, nz).ravel()
                                      for c, a in zip("uvw", cap["ubarbar"])])
                assert rel_err(ubb, s[f"s{step}_ubarbar"]) < 1e-13
            for i, c in enumerate("uvw"):
                assert rel_err(cap["uhat"][i], s[f"s{step}_uhat_{c}"]) < 1e-12
                assert rel_err(interior(c, cap["zsolve"][i], nx, ny, nz),
                               interior(c, s[f"s{step}_zsolve_{c}"], nx, ny, nz)) < 1e-12
                assert rel_err(interior(c, cap["proj"][i], nx, ny, nz),
                               interior(c, s[f"s{step}_proj_{c}"], nx, ny, nz)) < 1e-12


@pytest.mark.parametrize("name", ["sym", "bottom_neumann"])
def test_imex_golden(name):
    """The oracle's Eulerian IMEX right-hand side and step against the
    reference's (tests/golden/make_imex_golden.py)."""
    from oracle.slbdf2 import momentum_rhs_imex

    s = load_golden(f"imex_{name}.npz")
    nx, ny, nz, Lx, Ly, Lz, gamma, Re, dt = s["params"]
    nx, ny, nz = int(nx), int(ny), int(nz)
    ch = OracleChannel(nx, ny, nz, Lx, Ly, Lz, gamma, 1.0 / Re, s["init_u"], s["init_v"], s["init_w"],
                       s["init_p"], stretching_type=str(s["stretching"]), top_wall_bc_type=str(s["top"]),
                       z_f=s["z_f"], z_c=s["z_c"])
    rhs = momentum_rhs_imex(ch.u, ch.v, ch.w, nx, ny, nz, ch.dx, ch.dy, ch.dz_c, ch.dz_f, ch.nu)
    for c, r in zip("uvw", rhs):
        assert rel_err(r, s[f"rhs_{c}"]) < 1e-13, c
    for step in range(1, 5):
        ub, forcing = ch.step_imex(float(dt))
        for c in "uvw":
            assert rel_err(getattr(ch, c), s[f"s{step}_{c}"]) < 1e-12, (step, c)
        assert rel_err(ch.p, s[f"s{step}_p"]) < 1e-11
        assert abs(ub - float(s[f"s{step}_ubulk"])) < 1e-13
        assert abs(forcing - float(s[f"s{step}_forcing"])) < 1e-10


def test_pcr_c_restatement_is_bit_identical_to_numpy():
    """The oracle's threaded C PCR (tridiag.py:36-61) gives exactly what the
    numpy restatement gives, for power-of-two and other sizes."""
    from oracle.slbdf2 import pcr_solve, pcr_solve_numpy

    rng = np.random.default_rng(3)
    for n in (2, 5, 16, 63, 258):
        a, c = 0.3 * rng.normal(size=n), 0.3 * rng.normal(size=n)
        b = 2.0 + rng.random(n)
        a[0] = c[-1] = 0.0
        d = rng.normal(size=(4500, n))
        assert np.array_equal(pcr_solve(a, b, c, d), pcr_solve_numpy(a, b, c, d)), n
