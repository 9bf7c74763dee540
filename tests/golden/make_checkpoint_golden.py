"""Golden checkpoint: the REFERENCE's save_flow_fields (gmcavallazzi/SLchannel
v1.0.1, slchannel/utils.py:183-214) writing seeded ghost-shaped fields of an
8 x 6 x 12 channel, so the tests can check that slchannel_b200 reads that
file and writes the same format.

    python tests/golden/make_checkpoint_golden.py /path/to/SLchannel
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NX, NY, NZ = 8, 6, 12


def checkpoint_inputs():
    """Seeded arrays and scalars (plain numpy, shared with the tests)."""
    r = np.random.default_rng(44)
    return {
        "u": r.normal(size=(NX + 1, NY + 2, NZ + 2)), "v": r.normal(size=(NX + 2, NY + 1, NZ + 2)),
        "w": r.normal(size=(NX + 2, NY + 2, NZ + 1)), "p": r.normal(size=(NX + 2, NY + 2, NZ + 2)),
        "z_c": np.sort(r.uniform(0, 2, NZ + 2)), "z_f": np.sort(r.uniform(0, 2, NZ + 1)),
        "Lx": 2 * np.pi, "Ly": np.pi, "step": 1234, "time": 12.34, "u_tau": 0.0571,
        "forcing": 0.0033,
    }


def main(ref_root):
    from make_golden import _stub_matplotlib

    _stub_matplotlib()
    sys.path.insert(0, ref_root)
    import torch

    from slchannel.utils import save_flow_fields

    a = checkpoint_inputs()
    T = torch.from_numpy
    save_flow_fields(T(a["u"]), T(a["v"]), T(a["w"]), T(a["p"]), T(a["z_c"]), T(a["z_f"]), a["Lx"],
                     a["Ly"], a["step"], a["time"], torch.tensor(a["u_tau"]), a["forcing"], HERE,
                     "fields_ckpt.npz")


if __name__ == "__main__":
    sys.path.insert(0, HERE)
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SLCHANNEL_REF", "."))
