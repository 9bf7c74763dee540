"""Golden statistics restart state: the REFERENCE's TurbulenceStats
(gmcavallazzi/SLchannel v1.0.1, slchannel/turbstats.py) on CPU, three seeded
snapshots of an 8 x 6 x 12 channel accumulated with one extra spectra plane
(z+ = 30), then written by its save_state (turbstats.py:492-534) to
stats_state.npz and by its save_statistics (:464-473) to stats_final.npz.

    python tests/golden/make_stats_golden.py /path/to/SLchannel
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NX, NY, NZ = 8, 6, 12
LX, LY, LZ, GAMMA, NU, RE_TAU = 2 * np.pi, np.pi, 2.0, 1.8, 1.0 / 180.0, 180.0
EXTRA_PLANES = [30.0]
N_SNAPSHOTS = 3


def main(ref_root):
    from make_golden import _stub_matplotlib

    _stub_matplotlib()
    sys.path.insert(0, ref_root)
    import torch

    torch.set_default_dtype(torch.float64)
    from slchannel.turbstats import TurbulenceStats
    from slchannel.utils import generate_grid

    z_f, z_c, dz_f, dz_c = generate_grid(GAMMA, NZ, LZ)
    ts = TurbulenceStats(NX, NY, NZ, LX, LY, LZ, z_c, z_f, dz_c, dz_f, LX / NX, LY / NY, NU,
                         RE_TAU, device="cpu", spectra_z_planes=EXTRA_PLANES)
    r = np.random.default_rng(77)
    for _ in range(N_SNAPSHOTS):
        u = torch.from_numpy(1.0 + 0.1 * r.normal(size=(NX + 1, NY + 2, NZ + 2)))
        v = torch.from_numpy(0.1 * r.normal(size=(NX + 2, NY + 1, NZ + 2)))
        w = torch.from_numpy(0.1 * r.normal(size=(NX + 2, NY + 2, NZ + 1)))
        ts.accumulate_statistics(u, v, w, 0.05)
    ts.save_state(os.path.join(HERE, "stats_state.npz"))
    ts.save_statistics(os.path.join(HERE, "stats_final.npz"))


if __name__ == "__main__":
    sys.path.insert(0, HERE)
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SLCHANNEL_REF", "."))
