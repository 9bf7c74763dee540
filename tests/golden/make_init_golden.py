"""Golden initial fields: the REFERENCE's initialize_flow (gmcavallazzi/SLchannel
v1.0.1, slchannel/initflow.py:123-223) for every deterministic configuration
on a 6 x 8 x 10 channel (gamma 1.7, Lz 2, Ly pi): types 'parabolic',
'uniform' and 'vortices' (n_vortices 2 and 4, intensity 0.05) with the
Dirichlet and the Neumann (free-slip) top wall, in float64 as the solver runs
it (the reference's SLChannelFlow sets float64 as torch's default dtype).
The random perturbation of the other types is not deterministic across
implementations and is left out.

    python tests/golden/make_init_golden.py /path/to/SLchannel
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NX, NY, NZ = 6, 8, 10
GAMMA, LY, LZ, U_BULK = 1.7, float(np.pi), 2.0, 1.0


def cases():
    """(key, init_type, perturbation_intensity, n_vortices, top_wall_bc_type)."""
    out = []
    for top in ("dirichlet", "neumann"):
        out.append((f"parabolic_{top}", "parabolic", 0.0, 4, top))
        out.append((f"uniform_{top}", "uniform", 0.0, 4, top))
        for nv in (2, 4):
            out.append((f"vortices{nv}_{top}", "vortices", 0.05, nv, top))
    return out


def main(ref_root):
    from make_golden import _stub_matplotlib

    _stub_matplotlib()
    sys.path.insert(0, ref_root)
    import torch

    torch.set_default_dtype(torch.float64)
    from slchannel.initflow import initialize_flow
    from slchannel.utils import generate_grid

    out = {}
    for st in ("symmetric", "bottom"):
        _, z_c, _, _ = generate_grid(GAMMA, NZ, LZ, stretching_type=st)
        out[f"z_c_{st}"] = z_c.numpy()
        for key, kind, amp, nv, top in cases():
            u, v, w, p = initialize_flow(NX, NY, NZ, z_c, LY, LZ, U_bulk=U_BULK, init_type=kind,
                                         perturbation_intensity=amp, n_vortices=nv,
                                         top_wall_bc_type=top)
            for name, t in (("u", u), ("v", v), ("w", w), ("p", p)):
                out[f"{name}_{key}_{st}"] = t.numpy()
    np.savez_compressed(os.path.join(HERE, "init.npz"), **out)


if __name__ == "__main__":
    sys.path.insert(0, HERE)
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SLCHANNEL_REF", "."))
