"""GPU path vs the reference's own outputs (tests/golden/*.npz, produced by
running gmcavallazzi/SLchannel's float64 eager path; see make_golden.py).

Everything goes through the public drop-in (SLAdvector, SLChannelFlow) or the
C ABI.  Tolerances (north star: FP64 kernels agree to 1e-12 relative per
substep): interpolation, feet and advection 1e-12 relative to the field's
max; full steps and every substep 1e-12 relative (pressure 1e-11, a small
field); clamp counts exact."""

import numpy as np
import pytest
import torch
from helpers import interior, load_golden, rel_err

from slchannel_b200 import _native as N
from slchannel_b200.semilag import SLAdvector
from slchannel_b200.solver import SLChannelFlow

pytestmark = pytest.mark.gpu

DEV = torch.device("cuda")


def T(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(DEV)


def C(t):
    return t.detach().cpu().numpy()


@pytest.fixture(scope="module")
def adv_golden():
    return load_golden("advect.npz")


def _grid(d):
    nx, ny, nz, Lx, Ly, Lz, gamma = d["grid"]
    return int(nx), int(ny), int(nz), Lx, Ly, Lz, gamma


def _adv(d, order):
    nx, ny, nz, Lx, Ly, Lz, gamma = _grid(d)
    return SLAdvector(nx, ny, nz, Lx / nx, Ly / ny, Lx, Ly, Lz, torch.from_numpy(d["z_f"]),
                      torch.from_numpy(d["z_c"]), gamma, order=order, device=DEV)


def test_zmap_golden():
    z = load_golden("zmap.npz")
    for key in [k[2:] for k in z.files if k.startswith("z_")]:
        st, g, n = key.split("_")
        adv = SLAdvector(4, 4, int(n), 0.5, 0.5, 2.0, 2.0, 2.0, torch.from_numpy(z["zf_" + key]),
                         torch.from_numpy(z["zc_" + key]), float(g), stretching_type=st, device=DEV)
        kf = C(adv._face_coord(T(z["z_" + key])))
        assert np.abs(kf - z["kf_" + key]).max() < 1e-11, key


@pytest.mark.parametrize("order", [4, 6])
def test_interp_golden(adv_golden, order):
    d = adv_golden
    adv = _adv(d, order)
    for comp in "uvw":
        k = f"o{order}_{comp}"
        iw = adv._build_iw(adv.spec[comp], T(d["interp_x_" + k]), T(d["interp_y_" + k]),
                           T(d["interp_z_" + k]), order, count_clamp=True)
        out = C(adv._apply_iw(T(d["interp_buf_" + k]), iw))
        assert rel_err(out, d["interp_out_" + k]) < 1e-12, comp
        assert int(iw.n_clamped) == int(d["interp_ncl_" + k])
        assert int(adv._scratch_count) == int(d["interp_ncl_" + k])  # the kernel's own count


def test_departure_golden(adv_golden):
    d = adv_golden
    adv = _adv(d, 4)
    adv._fill(adv.mbuf["u"], "u", T(d["mid_u"]))
    adv._fill(adv.mbuf["v"], "v", T(d["mid_v"]))
    adv._fill(adv.mbuf["w"], "w", T(d["mid_w"]))
    for dt in (0.3, 0.9):
        for comp in "uvw":
            feet = adv.departure_coords(comp, dt)
            for a, nm in zip(feet, "xyz"):
                assert np.abs(C(a) - d[f"dep_{nm}_dt{dt}_{comp}"]).max() < 1e-12, (dt, comp, nm)


@pytest.mark.parametrize("order", [4, 6])
def test_advect_golden(adv_golden, order):
    d = adv_golden
    nx, ny, nz = _grid(d)[:3]
    adv = _adv(d, order)
    f = [T(d[k]) for k in ("f_u", "f_v", "f_w")]
    mid = [T(d[k]) for k in ("mid_u", "mid_v", "mid_w")]
    for dt in (0.3, 0.9):
        outs = adv.advect(*f, *mid, torch.tensor(dt))
        for c, o in zip("uvw", outs):
            assert rel_err(interior(c, C(o), nx, ny, nz), d[f"adv_{c}_o{order}_dt{dt}"]) < 1e-12
        assert int(adv.n_clamped_last) == int(d[f"adv_ncl_o{order}_dt{dt}"])
    for w0 in (-0.5, 0.5):
        mid = [T(d[f"clamp_mid_{c}_{w0}"]) for c in "uvw"]
        outs = adv.advect(*f, *mid, 0.5)
        for c, o in zip("uvw", outs):
            assert rel_err(interior(c, C(o), nx, ny, nz), d[f"clamp_{c}_o{order}_w{w0}"]) < 1e-12
        assert int(adv.n_clamped_last) == int(d[f"clamp_ncl_o{order}_w{w0}"]) > 0


@pytest.mark.parametrize("order", [4, 6])
def test_advect_extra_rhs_golden(order):
    """advect(..., extra_rhs=[two triples]) against the reference's own
    (tests/golden/advect_extra.npz): the advected triple and each extra triple
    (interior-shaped, interpolated at the same feet) at 1e-12 relative, the
    clamp count exact (880 clamped feet in the wall case); inputs unchanged;
    a second call returns new extra tensors."""
    d = load_golden("advect_extra.npz")
    nx, ny, nz = _grid(d)[:3]
    adv = _adv(d, order)
    f = [T(d[f"f_{c}"]) for c in "uvw"]
    extra = [tuple(T(d[f"e{t}_{c}"]) for c in "uvw") for t in range(2)]
    keep = [t.clone() for triple in extra for t in triple]
    first = None
    for name, pre, dt in (("dt0.3", "mid", 0.3), ("dt0.9", "mid", 0.9), ("clamp", "clamp_mid", 0.5)):
        mid = [T(d[f"{pre}_{c}"]) for c in "uvw"]
        key = f"o{order}_{name}"
        us, vs, ws, ex = adv.advect(*f, *mid, torch.tensor(dt), extra_rhs=extra)
        for c, o in zip("uvw", (us, vs, ws)):
            assert rel_err(interior(c, C(o), nx, ny, nz), d[f"adv_{c}_{key}"]) < 1e-12, (name, c)
        assert int(adv.n_clamped_last) == int(d[f"ncl_{key}"])
        assert len(ex) == 2
        for t, triple in enumerate(ex):
            for c, o in zip("uvw", triple):
                want = d[f"extra{t}_{c}_{key}"]
                assert tuple(o.shape) == want.shape and o.is_contiguous()
                assert rel_err(C(o), want) < 1e-12, (name, t, c)
        if first is None:
            first = ex
        else:
            assert first[0][0].data_ptr() != ex[0][0].data_ptr()
    for a, b in zip(keep, [t for triple in extra for t in triple]):
        assert torch.equal(a, b)
    # without extra_rhs the result and the count are the same as with it
    mid = [T(d[f"clamp_mid_{c}"]) for c in "uvw"]
    outs = adv.advect(*f, *mid, 0.5)
    assert len(outs) == 3
    assert rel_err(interior("u", C(outs[0]), nx, ny, nz), d[f"adv_u_o{order}_clamp"]) < 1e-12
    assert int(adv.n_clamped_last) == int(d[f"ncl_o{order}_clamp"])


def test_advect_extra_rhs_many_triples():
    """Ten extra triples (two trace groups in the FP64 form): each matches a
    plain advect of that triple exactly."""
    d = load_golden("advect_extra.npz")
    nx, ny, nz = _grid(d)[:3]
    adv = _adv(d, 6)
    f = [T(d[f"f_{c}"]) for c in "uvw"]
    mid = [T(d[f"mid_{c}"]) for c in "uvw"]
    extra = [tuple(T(d[f"e{t % 2}_{c}"]) * (1.0 + 0.25 * t) for c in "uvw") for t in range(10)]
    *_, ex = adv.advect(*f, *mid, 0.3, extra_rhs=extra)
    for t, triple in enumerate(extra):
        ref = [C(o).copy() for o in adv.advect(*triple, *mid, 0.3)]
        for c, o, r in zip("uvw", ex[t], ref):
            assert np.array_equal(C(o), interior(c, r, nx, ny, nz)), (t, c)


def config_from_step_golden(s):
    nx, ny, nz, Lx, Ly, Lz, gamma, Re, dt, order = s["params"]
    return {
        "grid": {"nx": int(nx), "ny": int(ny), "nz": int(nz)},
        "domain": {"Lx": float(Lx), "Ly": float(Ly), "Lz": float(Lz),
                   "stretching_type": str(s["stretching"])},
        "flow": {"Re": float(Re), "Re_tau": 180.0, "U_bulk": 1.0, "gamma": float(gamma)},
        "boundary_conditions": {"top_wall": {"type": str(s["top"])}},
        "initialization": {"type": "parabolic"},
        "time": {"dt": float(dt)},
        "compute": {"device": "cuda"},
        "sl": {"interp_order": int(order), "n_traj_iters": 2, "interp_dtype": "fp64",
               "traj_interp_order": int(s["traj_order"]) if "traj_order" in s.files else 2,
               "bdf2_pressure": str(s["pressure"]) if "pressure" in s.files else "noninc"},
    }, float(dt)


CASES = ["o6_sym", "o4_sym", "o4_bottom_neumann", "o6_inc", "o6_traj4", "o4_inc_traj4_bottom_neumann"]


@pytest.mark.parametrize("name", CASES)
def test_steps_golden(name):
    s = load_golden(f"step_{name}.npz")
    cfg, dt = config_from_step_golden(s)
    flow = SLChannelFlow(config=cfg)
    assert np.abs(C(flow.z_f) - s["z_f"]).max() < 1e-15
    flow.set_state(T(s["init_u"]), T(s["init_v"]), T(s["init_w"]), T(s["init_p"]))
    for step in range(1, 5):
        ub, forcing = flow.step_sl_bdf2(dt)
        for c in "uvw":
            assert rel_err(C(getattr(flow, c)), s[f"s{step}_{c}"]) < 1e-12, (step, c)
        assert rel_err(C(flow.p), s[f"s{step}_p"]) < 1e-11, step
        assert abs(float(ub) - float(s[f"s{step}_ubulk"])) < 1e-13
        assert abs(float(forcing) - float(s[f"s{step}_forcing"])) < 1e-11
        assert int(flow.sl.n_clamped_last) == int(s[f"s{step}_nclamp"])


@pytest.mark.parametrize("name", ["o6_sym", "o4_sym"])
def test_bdf2_substeps_golden(name):
    """Each substep kernel of BDF2 step 3, fed the reference's own step-2 and
    step-1 states: fused trace+gather+BDF2 epilogue, z-solve, projection."""
    s = load_golden(f"step_{name}.npz")
    cfg, dt = config_from_step_golden(s)
    flow = SLChannelFlow(config=cfg)
    nx, ny, nz = flow.nx, flow.ny, flow.nz
    g = flow.sl.native
    cur = [T(s[f"s2_{c}"]) for c in "uvw"]
    prev = [T(s[f"s1_{c}"]) for c in "uvw"]
    out = [torch.zeros_like(t) for t in cur]
    ncl = torch.zeros((), dtype=torch.int64, device=DEV)
    st = N.stream_of(cur[0])
    g.call("slc_trace_gather_bdf2", *[N.ptr(t) for t in cur], *[N.ptr(t) for t in prev], dt,
           *[N.ptr(t) for t in out], N.ptr(ncl), st)
    for c, o in zip("uvw", out):
        assert rel_err(interior(c, C(o), nx, ny, nz),
                       interior(c, s[f"s3_uhat_{c}"], nx, ny, nz)) < 1e-12, c
    # z-solve on the reference's own u_hat
    zin = [T(s[f"s3_uhat_{c}"]) for c in "uvw"]
    g.call("slc_zsolve", *[N.ptr(t) for t in zin], (2.0 / 3.0) * dt, st)
    for c, o in zip("uvw", zin):
        assert rel_err(interior(c, C(o), nx, ny, nz),
                       interior(c, s[f"s3_zsolve_{c}"], nx, ny, nz)) < 1e-12, c
    # projection of the reference's own z-solve output (ghosts from apply_bc)
    pin = [T(s[f"s3_zsolve_{c}"]) for c in "uvw"]
    g.call("slc_apply_bc", *[N.ptr(t) for t in pin], st)
    p = torch.zeros(nx + 2, ny + 2, nz + 2, dtype=torch.float64, device=DEV)
    dte = (2.0 / 3.0) * dt
    g.call("slc_project", *[N.ptr(t) for t in pin], N.ptr(p), dte, dte, st)
    assert rel_err(C(p), s["s3_phi"]) < 1e-11
    for c, o in zip("uvw", pin):
        assert rel_err(interior(c, C(o), nx, ny, nz),
                       interior(c, s[f"s3_proj_{c}"], nx, ny, nz)) < 1e-12, c


def test_bdf1_bootstrap_substep_golden():
    s = load_golden("step_o6_sym.npz")
    cfg, dt = config_from_step_golden(s)
    flow = SLChannelFlow(config=cfg)
    nx, ny, nz = flow.nx, flow.ny, flow.nz
    f = [T(s[f"init_{c}"]) for c in "uvw"]
    outs = flow.sl.advect(*f, *f, dt)
    ubar = np.concatenate([interior(c, C(o), nx, ny, nz).ravel() for c, o in zip("uvw", outs)])
    assert rel_err(ubar, s["s1_ubar"]) < 1e-12
