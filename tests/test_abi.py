"""The C-ABI library builds, loads and exports every symbol include/slc_b200.h
declares; argument errors come back as status codes and messages (checked on
the host, before any device work).  CPU only: no kernel is launched."""

import ctypes
import os
import re

import numpy as np
import pytest

from slchannel_b200 import _native as N

HEADER = os.path.join(os.path.dirname(__file__), "..", "include", "slc_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"SLC_API\s+[\w\s\*]+?\b(slc_\w+)\s*\(", text)))


def test_header_declares_the_abi():
    names = declared_symbols()
    assert "slc_step_bdf2" in names and "slc_grid_create" in names
    assert set(names) == set(N.SIGNATURES), set(names) ^ set(N.SIGNATURES)


def test_library_exports_every_declared_symbol():
    lib = N.lib()
    assert os.path.exists(N.library_path())
    for name in declared_symbols():
        assert hasattr(lib, name), name
    assert lib.slc_version().decode().startswith("slc_b200")


def _desc(**over):
    d = N.GridDesc()
    nx, ny, nz = over.pop("nx", 8), over.pop("ny", 6), over.pop("nz", 12)
    d.nx, d.ny, d.nz = nx, ny, nz
    d.Lx, d.Ly, d.Lz, d.gamma = 2 * np.pi, np.pi, 2.0, 2.0
    d.stretching, d.order, d.traj_order, d.n_traj_iters = 0, 6, 2, 2
    d.top_wall_neumann, d.precision, d.nu, d.device, d.xy_rhs_lagged = 0, 0, 1e-3, 0, 0
    zf = np.linspace(0.0, 2.0, nz + 1)
    zc = np.concatenate([[-0.5 * zf[1]], 0.5 * (zf[1:] + zf[:-1]), [2 * zf[-1] - 0.5 * (zf[-1] + zf[-2])]])
    keep = (zf, zc)
    d.z_f = zf.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    d.z_c = zc.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    for k, v in over.items():
        setattr(d, k, v)
    return d, keep


@pytest.mark.parametrize(
    "field,value,msg",
    [("order", 5, "interp_order"), ("traj_order", 3, "traj_interp_order"),
     ("n_traj_iters", 0, "n_traj_iters"), ("stretching", 3, "stretching"),
     ("precision", 7, "precision"), ("nz", 1, "nz")],
)
def test_grid_create_rejects_bad_arguments(field, value, msg):
    lib = N.lib()
    d, keep = _desc(**{field: value})
    h = ctypes.c_void_p()
    rc = lib.slc_grid_create(ctypes.byref(d), ctypes.byref(h))
    assert rc == N.SLC_E_INVALID
    assert not h.value
    assert msg in lib.slc_last_error(None).decode()


def test_order_too_large_for_grid():
    lib = N.lib()
    d, keep = _desc(nz=4, order=6)
    h = ctypes.c_void_p()
    assert lib.slc_grid_create(ctypes.byref(d), ctypes.byref(h)) == N.SLC_E_INVALID
    assert "too small" in lib.slc_last_error(None).decode()


def test_null_handle_is_an_error_not_a_crash():
    lib = N.lib()
    assert lib.slc_apply_bc(None, None, None, None, None) == N.SLC_E_INVALID
    assert lib.slc_step_bdf2(None, None, None, None, None, 0.1, None, None) == N.SLC_E_INVALID
    assert lib.slc_divergence_raw(0, 1, 1, 1.0, 1.0, None, None, None, None, None, None) == N.SLC_E_INVALID
    assert lib.slc_bulk_scratch_doubles() > 0


def test_python_layer_refuses_cpu_tensors():
    import torch

    with pytest.raises(ValueError):
        N.require(torch.zeros(3, dtype=torch.float64), (3,), "x")
    with pytest.raises(RuntimeError):
        from slchannel_b200.semilag import SLAdvector

        z_f = torch.linspace(0, 2, 13)
        z_c = torch.cat([-z_f[1:2] / 2, 0.5 * (z_f[1:] + z_f[:-1]), z_f[-1:] + (z_f[-1:] - z_f[-2:-1]) / 2])
        SLAdvector(8, 6, 12, 0.5, 0.5, 4.0, 3.0, 2.0, z_f, z_c, 2.0, order=6, device="cpu")
