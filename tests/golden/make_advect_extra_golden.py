"""Golden vectors for SLAdvector.advect(..., extra_rhs=...): the REFERENCE's
float64 eager advect (gmcavallazzi/SLchannel v1.0.1, slchannel/semilag.py:
584-671) with two extra field triples interpolated at the same departure
points, on the 10 x 8 x 14 grid of advect.npz (gamma 1.8), orders 4 and 6,
two time steps, plus a wall-clamping trajectory velocity.  Writes
advect_extra.npz.

    python tests/golden/make_advect_extra_golden.py /path/to/SLchannel
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NX, NY, NZ = 10, 8, 14
LX, LY, LZ, GAMMA = 2 * np.pi, np.pi, 2.0, 1.8


def main(ref_root):
    sys.path.insert(0, HERE)
    from make_golden import _stub_matplotlib, positions, smooth_field

    _stub_matplotlib()
    sys.path.insert(0, ref_root)
    import torch

    torch.set_default_dtype(torch.float64)
    torch.set_num_threads(1)
    import slchannel.solver as ref_solver
    from slchannel.semilag import SLAdvector
    from slchannel.utils import generate_grid

    T = lambda a: torch.from_numpy(np.ascontiguousarray(a))  # noqa: E731
    N = lambda t: t.detach().cpu().numpy().copy()  # noqa: E731
    dx, dy = LX / NX, LY / NY
    z_f, z_c, _, _ = generate_grid(GAMMA, NZ, LZ, stretching_type="symmetric")
    zf, zc = N(z_f), N(z_c)

    def fields(seed, amp_u, amp_w, mean):
        r = np.random.default_rng(seed)
        res = {}
        for comp in "uvw":
            X, Y, Z = positions(comp, NX, NY, dx, dy, zf, zc)
            f = smooth_field(r, X, Y, Z, LX, LY, LZ, amp_w if comp == "w" else amp_u)
            if comp == "u" and mean:
                f = f + 1.5 * Z * (2 - Z)
            res[comp] = np.ascontiguousarray(f * np.ones(np.broadcast_shapes(X.shape, Y.shape, Z.shape)))
        u, v, w = (T(res[c]).clone() for c in "uvw")
        ref_solver.apply_bc_all(u, v, w, "dirichlet")
        return N(u), N(v), N(w)

    out = {"grid": np.array([NX, NY, NZ, LX, LY, LZ, GAMMA]), "z_f": zf, "z_c": zc}
    mid = fields(21, 0.4, 0.3, True)
    f = fields(22, 1.0, 1.0, False)
    extra = [fields(23, 0.7, 0.5, False), fields(24, 2.0, 1.5, True)]
    for c, a in zip("uvw", mid):
        out[f"mid_{c}"] = a
    for c, a in zip("uvw", f):
        out[f"f_{c}"] = a
    for t, triple in enumerate(extra):
        for c, a in zip("uvw", triple):
            out[f"e{t}_{c}"] = a
    clamp_mid = (np.full((NX + 1, NY + 2, NZ + 2), 0.3), np.zeros((NX + 2, NY + 1, NZ + 2)),
                 np.full((NX + 2, NY + 2, NZ + 1), 0.5))
    for c, a in zip("uvw", clamp_mid):
        out[f"clamp_mid_{c}"] = a
    cases = [("dt0.3", mid, 0.3), ("dt0.9", mid, 0.9), ("clamp", clamp_mid, 0.5)]
    for order in (4, 6):
        adv = SLAdvector(NX, NY, NZ, dx, dy, LX, LY, LZ, z_f, z_c, GAMMA, order=order)
        for name, m, dt in cases:
            res = adv.advect(*(T(a) for a in f), *(T(a) for a in m), torch.tensor(dt),
                             extra_rhs=[tuple(T(a) for a in triple) for triple in extra])
            us, vs, ws, ex = res
            key = f"o{order}_{name}"
            out[f"adv_u_{key}"] = N(us)[1 : NX + 1, 1 : NY + 1, 1 : NZ + 1]
            out[f"adv_v_{key}"] = N(vs)[1 : NX + 1, 1 : NY + 1, 1 : NZ + 1]
            out[f"adv_w_{key}"] = N(ws)[1 : NX + 1, 1 : NY + 1, 1:NZ]
            out[f"ncl_{key}"] = np.array(int(adv.n_clamped_last))
            for t, triple in enumerate(ex):
                for c, a in zip("uvw", triple):
                    out[f"extra{t}_{c}_{key}"] = N(a)
    np.savez_compressed(os.path.join(HERE, "advect_extra.npz"), **out)
    print("wrote", os.path.join(HERE, "advect_extra.npz"))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SLCHANNEL_REF", "."))
