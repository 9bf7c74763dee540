"""The drop-in's initial fields (slchannel_b200.initflow.initialize_flow), on
CPU, against the reference's own initialize_flow (initflow.py:123-223) run by
tests/golden/make_init_golden.py: every deterministic type ('parabolic',
'uniform', 'vortices' with 2 and 4 vortices) with either top wall, on both
stretchings.  The same float64 operations in the same order, so the fields
are bit-identical."""

import os
import sys

import numpy as np
import pytest
import torch

from slchannel_b200.initflow import initialize_flow

HERE = os.path.dirname(__file__)
sys.path.insert(0, os.path.join(HERE, "golden"))
from make_init_golden import GAMMA, LY, LZ, NX, NY, NZ, U_BULK, cases  # noqa: E402

GOLD = np.load(os.path.join(HERE, "golden", "init.npz"))


@pytest.mark.parametrize("st", ["symmetric", "bottom"])
@pytest.mark.parametrize("key, kind, amp, nv, top", cases(), ids=lambda v: v if isinstance(v, str) else None)
def test_initial_fields_match_the_reference(st, key, kind, amp, nv, top):
    z_c = torch.from_numpy(GOLD[f"z_c_{st}"])
    u, v, w, p = initialize_flow(NX, NY, NZ, z_c, LY, LZ, U_bulk=U_BULK, init_type=kind,
                                 perturbation_intensity=amp, n_vortices=nv, device="cpu",
                                 top_wall_bc_type=top)
    for name, t in (("u", u), ("v", v), ("w", w), ("p", p)):
        ref = GOLD[f"{name}_{key}_{st}"]
        assert t.dtype == torch.float64 and tuple(t.shape) == ref.shape, name
        np.testing.assert_array_equal(t.numpy(), ref, err_msg=f"{name} {key} {st}")


def test_golden_grid_is_the_drop_in_grid():
    from slchannel_b200.utils import generate_grid

    for st in ("symmetric", "bottom"):
        _, z_c, _, _ = generate_grid(GAMMA, NZ, LZ, stretching_type=st)
        np.testing.assert_array_equal(z_c.numpy(), GOLD[f"z_c_{st}"])
