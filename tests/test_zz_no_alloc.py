"""slc_zsolve_noalloc -- the z-solve for callers that cannot allocate device
memory (their own memory manager owns the GPU, or their time loop cannot
afford cudaMalloc's implicit synchronisation) -- must give the same result as
the handle-based slc_zsolve, on two calls in a row through the C ABI.

The second call uses another dt and other fields, so a stale table from the
first call would show.  This file is collected last on purpose; it passes
alone in a fresh process and after the rest of the suite."""

import math

import pytest
import torch

from slchannel_b200 import _native as N
from slchannel_b200.utils import generate_grid

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative to each field's max, as the other FP64 parity tests


def _fields(nx, ny, nz, seed):
    g = torch.Generator().manual_seed(seed)
    shapes = [(nx + 1, ny + 2, nz + 2), (nx + 2, ny + 1, nz + 2), (nx + 2, ny + 2, nz + 1)]
    out = [torch.rand(s, generator=g, dtype=torch.float64) - 0.5 for s in shapes]
    out[2][:, :, 0] = 0.0
    out[2][:, :, -1] = 0.0
    return [t.cuda() for t in out]


@pytest.mark.parametrize("top", ["dirichlet", "neumann"])
def test_zsolve_noalloc_matches_handle_path(top):
    nx, ny, nz, Re, gamma = 20, 14, 40, 2800.0, 2.0
    nu = 1.0 / Re
    z_f, z_c, dz_f, dz_c = generate_grid(gamma, nz, 2.0)
    grid = N.Grid(nx, ny, nz, 2 * math.pi, math.pi, 2.0, gamma, z_f, z_c, order=6, nu=nu,
                  top_wall_bc_type=top, device=torch.device("cuda", torch.cuda.current_device()))
    dzc, dzf = dz_c.cuda().contiguous(), dz_f.cuda().contiguous()
    lib = N.lib()
    for call, (dt, seed) in enumerate(((0.01 * 2 / 3, 1), (0.05, 2))):
        ref = _fields(nx, ny, nz, seed)
        got = [t.clone() for t in ref]
        stream = N.stream_of(ref[0])
        grid.call("slc_zsolve", *[N.ptr(t) for t in ref], dt, stream)
        rc = lib.slc_zsolve_noalloc(nx, ny, nz, nu, 1 if top == "neumann" else 0, N.ptr(dzc),
                                    N.ptr(dzf), dt, *[N.ptr(t) for t in got], stream)
        assert rc == N.SLC_OK, lib.slc_last_error(None)
        torch.cuda.synchronize()
        for c, a, b in zip("uvw", got, ref):
            err = ((a - b).abs().max() / b.abs().max()).item()
            assert err < TOL, (call, c, err)


def test_zsolve_noalloc_rejects_oversized_grid():
    lib = N.lib()
    t = torch.zeros(4, dtype=torch.float64, device="cuda")
    p = N.ptr(t)
    rc = lib.slc_zsolve_noalloc(4, 4, 1025, 1e-3, 0, p, p, 0.01, p, p, p, None)
    assert rc == N.SLC_E_INVALID
    assert b"1024" in lib.slc_last_error(None)
