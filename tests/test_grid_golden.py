"""The drop-in's host-side grid set-up, on CPU, against the reference's own
outputs: generate_grid (utils.py:21-61) against the z_f / z_c the reference
wrote into tests/golden (zmap.npz: two stretchings x gamma 0.8, 1.8, 2.6 x
nz 64, 180; step_*.npz: the step goldens' grids), and the Lagrange
inverse-denominator tables (semilag.py:102-114) against a direct evaluation
of 1 / prod_{l != m} (z_m - z_l).  The grids are bit-identical to the
reference's."""

import glob
import os

import numpy as np
import pytest

from slchannel_b200.semilag import _z_denominator_table
from slchannel_b200.utils import generate_grid

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _zmap_cases():
    z = np.load(os.path.join(GOLDEN, "zmap.npz"))
    keys = sorted(k[3:] for k in z.files if k.startswith("zf_"))
    return [(k, z["zf_" + k], z["zc_" + k]) for k in keys]


@pytest.mark.parametrize("key, zf_ref, zc_ref", _zmap_cases(), ids=lambda v: v if isinstance(v, str) else "")
def test_generate_grid_matches_the_reference(key, zf_ref, zc_ref):
    st, gamma, nz = key.split("_")
    z_f, z_c, dz_f, dz_c = (t.numpy() for t in generate_grid(float(gamma), int(nz), 2.0,
                                                              stretching_type=st))
    # the same float64 operations in the same order: bit-identical
    np.testing.assert_array_equal(z_f, zf_ref)
    np.testing.assert_array_equal(z_c, zc_ref)
    np.testing.assert_array_equal(dz_f, zf_ref[1:] - zf_ref[:-1])
    np.testing.assert_array_equal(dz_c, zc_ref[1:] - zc_ref[:-1])
    assert z_f[0] == 0.0 and abs(z_f[-1] - 2.0) < 1e-15
    assert len(z_c) == int(nz) + 2 and np.all(np.diff(z_c) > 0)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "step_*.npz"))),
                         ids=os.path.basename)
def test_step_golden_grids_match(path):
    g = np.load(path)
    nx, ny, nz, Lx, Ly, Lz, gamma = g["params"][:7]
    z_f, z_c, _, _ = (t.numpy() for t in generate_grid(float(gamma), int(nz), float(Lz),
                                                        stretching_type=str(g["stretching"])))
    np.testing.assert_array_equal(z_f, g["z_f"])
    np.testing.assert_array_equal(z_c, g["z_c"])


@pytest.mark.parametrize("order", [2, 4, 6])
@pytest.mark.parametrize("st", ["symmetric", "bottom"])
def test_denominator_tables(order, st):
    z_f, z_c, _, _ = generate_grid(1.8, 64, 2.0, stretching_type=st)
    for zn in (z_f, z_c):
        tab = _z_denominator_table(zn, order).numpy()
        z = zn.numpy()
        rows = len(z) - order + 1
        assert tab.shape == (rows, order)
        want = np.empty((rows, order))
        for b in range(rows):
            s = z[b:b + order]
            for m in range(order):
                want[b, m] = 1.0 / np.prod([s[m] - s[l] for l in range(order) if l != m])
        np.testing.assert_allclose(tab, want, rtol=1e-13, atol=0)
        # Lagrange weights from the table reproduce polynomials of degree < order
        # at a point inside each stencil
        for b in range(0, rows, 7):
            s = z[b:b + order]
            x = 0.5 * (s[order // 2 - 1] + s[order // 2])
            w = np.array([np.prod([x - s[l] for l in range(order) if l != m]) * tab[b, m]
                          for m in range(order)])
            for p in range(order):
                np.testing.assert_allclose(w @ s ** p, x ** p, rtol=1e-10, atol=1e-12)
