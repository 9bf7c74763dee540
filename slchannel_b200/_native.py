"""ctypes binding of libslc_b200.so (the C ABI in include/slc_b200.h).

PyTorch tensors are only carriers here: their device pointers, the current
CUDA stream and plain sizes are what cross the boundary.  There is no CPU or
torch fallback: if the library cannot be built or loaded, or a tensor is not a
float64 CUDA tensor of the expected shape, a call raises.
"""

from __future__ import annotations

import ctypes
import os
import threading

import torch

from . import build as _build

SLC_OK = 0
SLC_E_INVALID = 1
PREC_FP64 = 0
PREC_MIXED = 1

_lock = threading.Lock()
_lib = None


class GridDesc(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32),
        ("ny", ctypes.c_int32),
        ("nz", ctypes.c_int32),
        ("Lx", ctypes.c_double),
        ("Ly", ctypes.c_double),
        ("Lz", ctypes.c_double),
        ("gamma", ctypes.c_double),
        ("stretching", ctypes.c_int32),
        ("order", ctypes.c_int32),
        ("traj_order", ctypes.c_int32),
        ("n_traj_iters", ctypes.c_int32),
        ("top_wall_neumann", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("nu", ctypes.c_double),
        ("z_f", ctypes.POINTER(ctypes.c_double)),
        ("z_c", ctypes.POINTER(ctypes.c_double)),
        ("device", ctypes.c_int32),
        ("xy_rhs_lagged", ctypes.c_int32),
    ]


# Every symbol include/slc_b200.h declares, with its argument types.
_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
_L = ctypes.c_int64
SIGNATURES = {
    "slc_version": ([], ctypes.c_char_p),
    "slc_grid_create": ([ctypes.POINTER(GridDesc), ctypes.POINTER(_P)], _I),
    "slc_grid_destroy": ([_P], _I),
    "slc_last_error": ([_P], ctypes.c_char_p),
    "slc_apply_bc": ([_P, _P, _P, _P, _P], _I),
    "slc_face_coord": ([_P, _P, _L, _P, _P], _I),
    "slc_interp_points": ([_P, _I, _I, _P, _P, _P, _P, _L, _I, _P, _P, _P], _I),
    "slc_departure": ([_P, _I, _P, _P, _P, _D, _P, _P, _P, _P], _I),
    "slc_advect": ([_P, _P, _P, _P, _P, _P, _P, _D, _P, _P, _P, _P, _P], _I),
    "slc_advect_extra": ([_P, _P, _P, _P, _P, _P, _P, _D, _P, _P, _P, _I, ctypes.POINTER(_P),
                          ctypes.POINTER(_P), _P, _P], _I),
    "slc_trace_gather_bdf2": ([_P, _P, _P, _P, _P, _P, _P, _D, _P, _P, _P, _P, _P], _I),
    "slc_step_bdf2_host": ([_P, ctypes.POINTER(_P), ctypes.POINTER(_P), ctypes.POINTER(_P), _P, _P, _D,
                            _D, _P], _I),
    "slc_trace_gather_bdf2_staged": ([_P, _P, _P, _P, _P, _P, _P, _D, _P, _P, _P, _P, _P], _I),
    "slc_zsolve": ([_P, _P, _P, _P, _D, _P], _I),
    "slc_divergence": ([_P, _P, _P, _P, _P, _P], _I),
    "slc_divergence_raw": ([_I, _I, _I, _D, _D, _P, _P, _P, _P, _P, _P], _I),
    "slc_project": ([_P, _P, _P, _P, _P, _D, _D, _P], _I),
    "slc_bulk_velocity": ([_P, _P, _P, _P], _I),
    "slc_bulk_scratch_doubles": ([], _I),
    "slc_bulk_velocity_raw": ([_I, _I, _I, _P, _P, _D, _P, _P, _P], _I),
    "slc_bulk_shift": ([_P, _P, _P, _P, _D, _D, _P, _P], _I),
    "slc_step_bdf1": ([_P, ctypes.POINTER(_P), ctypes.POINTER(_P), _P, _D, _P, _P], _I),
    "slc_step_bdf2": ([_P, ctypes.POINTER(_P), ctypes.POINTER(_P), ctypes.POINTER(_P), _P, _D,
                       _P, _P], _I),
    "slc_step_bdf2_inc": ([_P, ctypes.POINTER(_P), ctypes.POINTER(_P), ctypes.POINTER(_P), _P, _P, _I,
                           _D, _P, _P], _I),
    "slc_imex_rhs": ([_P, _P, _P, _P, _P, _P, _P, _P], _I),
    "slc_step_imex": ([_P, ctypes.POINTER(_P), _P, ctypes.POINTER(_P), ctypes.POINTER(_P), _I, _D, _D, _P], _I),
    "slc_timing": ([_P, _I], _I),
    "slc_timing_read": ([_P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_L)], _I),
    "slc_kernel_launches": ([], _L),
    "slc_gather_stats": ([_P, ctypes.POINTER(_L), _I], _I),
    "slc_host_step_stats": ([_P, ctypes.POINTER(_L)], _I),
    "slc_gather_probe": ([_I, _I, ctypes.POINTER(_D), _P], _I),
    "slc_diagnostics": ([_P, _P, _P, _P, _P, _P], _I),
    "slc_diagnostics_scratch_doubles": ([], _I),
    "slc_diagnostics_raw": ([_I, _I, _I, _D, _D, _P, _P, _P, _D, _I, _D, _D, _D, _P, _P, _P, _P, _P, _P], _I),
    "slc_stats_accumulate": ([_P, _P, _P, _P, _P, _P, _I, _I, _P], _I),
    "slc_zsolve_noalloc": ([_I, _I, _I, _D, _I, _P, _P, _D, _P, _P, _P, _P], _I),
    "slc_fma_peak": ([_I, _P, _P], _I),
    "slc_adjoint_bc": ([_P, _P, _P, _P, _P], _I),
    "slc_adjoint_step": ([_P, _I, ctypes.POINTER(_P), ctypes.POINTER(_P), ctypes.POINTER(_P),
                          ctypes.POINTER(_P), ctypes.POINTER(_P), _D, _P], _I),
    "slc_ensemble_create": ([ctypes.POINTER(GridDesc), _I, ctypes.POINTER(_P)], _I),
    "slc_ensemble_destroy": ([_P], _I),
    "slc_ensemble_size": ([_P], _I),
    "slc_ensemble_grid": ([_P, _I], _P),
    "slc_ensemble_last_error": ([_P], ctypes.c_char_p),
    "slc_ensemble_bind": ([_P, ctypes.POINTER(_P), ctypes.POINTER(_P), ctypes.POINTER(_D),
                           ctypes.POINTER(_D), _P, _P], _I),
    "slc_ensemble_set_tiles": ([_P, ctypes.POINTER(_I)], _I),
    "slc_ensemble_get_tiles": ([_P, ctypes.POINTER(_I)], _I),
    "slc_ensemble_autotune": ([_P, _I, _I, ctypes.POINTER(_I), ctypes.POINTER(_D), _P], _I),
    "slc_ensemble_step_bdf2": ([_P, _I, _I, _P], _I),
}

PHASES = ("bc", "mid", "sl", "zsolve", "project", "bulk")


def lib():
    """Load (building in-tree first if needed) libslc_b200.so."""
    global _lib
    with _lock:
        if _lib is None:
            path = _build.build()  # no-op when the library is current
            handle = ctypes.CDLL(path)
            for name, (args, res) in SIGNATURES.items():
                fn = getattr(handle, name)
                fn.argtypes = args
                fn.restype = res
            _lib = handle
    return _lib


def library_path():
    return _build.LIB


def check(rc, handle=None):
    if rc == SLC_OK:
        return
    msg = lib().slc_last_error(handle)
    msg = msg.decode() if msg else f"slc error {rc}"
    if rc == SLC_E_INVALID:
        raise ValueError(msg)
    raise RuntimeError(msg)


def stream_of(t: torch.Tensor):
    return ctypes.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


def ptr(t):
    """Device pointer of a CUDA tensor (None -> NULL)."""
    if t is None:
        return None
    if not isinstance(t, torch.Tensor) or t.device.type != "cuda":
        raise ValueError("slchannel_b200 expects CUDA tensors (no CPU path)")
    return ctypes.c_void_p(t.data_ptr())


def require(t, shape, name, dtype=torch.float64):
    if not isinstance(t, torch.Tensor):
        raise ValueError(f"{name} must be a torch tensor")
    if t.device.type != "cuda":
        raise ValueError(f"{name} must live on a CUDA device (slchannel_b200 has no CPU path)")
    if t.dtype != dtype:
        raise ValueError(f"{name} must be {dtype}, got {t.dtype}")
    if tuple(t.shape) != tuple(shape):
        raise ValueError(f"{name} has shape {tuple(t.shape)}, expected {tuple(shape)}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    return t


class Grid:
    """Owner of one native slc_grid handle."""

    def __init__(self, nx, ny, nz, Lx, Ly, Lz, gamma, z_f, z_c, *, stretching_type="symmetric",
                 order=4, traj_order=2, n_traj_iters=2, top_wall_bc_type="dirichlet",
                 precision=PREC_FP64, nu=0.0, device=None, xy_rhs="extrap"):
        L = lib()
        zf = torch.as_tensor(z_f, dtype=torch.float64).detach().cpu().contiguous()
        zc = torch.as_tensor(z_c, dtype=torch.float64).detach().cpu().contiguous()
        if zf.numel() != nz + 1 or zc.numel() != nz + 2:
            raise ValueError("z_f must have nz+1 and z_c nz+2 entries")
        dev = torch.device(device) if device is not None else torch.device("cuda")
        if dev.type != "cuda":
            raise ValueError("slchannel_b200 runs on CUDA devices only")
        d = GridDesc()
        d.nx, d.ny, d.nz = int(nx), int(ny), int(nz)
        d.Lx, d.Ly, d.Lz = float(Lx), float(Ly), float(Lz)
        d.gamma = float(gamma)
        d.stretching = 0 if stretching_type == "symmetric" else 1
        d.order, d.traj_order, d.n_traj_iters = int(order), int(traj_order), int(n_traj_iters)
        d.top_wall_neumann = 1 if top_wall_bc_type == "neumann" else 0
        d.precision = int(precision)
        d.nu = float(nu)
        d.z_f = ctypes.cast(zf.data_ptr(), ctypes.POINTER(ctypes.c_double))
        d.z_c = ctypes.cast(zc.data_ptr(), ctypes.POINTER(ctypes.c_double))
        d.device = dev.index if dev.index is not None else torch.cuda.current_device()
        d.xy_rhs_lagged = 1 if xy_rhs == "lagged" else 0
        h = ctypes.c_void_p()
        rc = L.slc_grid_create(ctypes.byref(d), ctypes.byref(h))
        check(rc, None)
        self._h = h
        self.desc = d
        self.device = torch.device("cuda", d.device)
        self.nx, self.ny, self.nz = d.nx, d.ny, d.nz

    @property
    def handle(self):
        return self._h

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib is not None:
            _lib.slc_grid_destroy(h)
        self._h = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass

    # -- thin wrappers; shapes are checked by the callers ---------------------
    def call(self, name, *args):
        rc = getattr(lib(), name)(self._h, *args)
        check(rc, self._h)

    def timing(self, enable=True):
        check(lib().slc_timing(self._h, 1 if enable else 0), self._h)

    def timing_read(self):
        """{phase: (total_ms, n_intervals)} since the last read; synchronises."""
        ms = (ctypes.c_double * len(PHASES))()
        cnt = (ctypes.c_int64 * len(PHASES))()
        check(lib().slc_timing_read(self._h, ms, cnt), self._h)
        return {p: (ms[i], cnt[i]) for i, p in enumerate(PHASES)}


def kernel_launches():
    return int(lib().slc_kernel_launches())


def fma_peak_gflops(fp64=True, stream=None):
    """Measured FMA-pipe throughput (GFLOP/s) of the current device, FP64 or
    FP32, from the library's register-resident FMA-chain kernel."""
    out = ctypes.c_double(0.0)
    s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    check(lib().slc_fma_peak(1 if fp64 else 0, ctypes.byref(out), ctypes.c_void_p(s)), None)
    return out.value


def gather_probe(n=128, reps=10, stream=None):
    """The scalar and the tensor-core formulations of the order-6 FP32
    gather on a synthetic n^3 problem (slc_gather_probe): per-launch ms of
    each, their largest relative difference, fallback groups per launch."""
    out = (ctypes.c_double * 4)()
    s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    check(lib().slc_gather_probe(int(n), int(reps), out, ctypes.c_void_p(s)), None)
    return {"scalar_ms": out[0], "tensor_ms": out[1], "max_rel_diff": out[2],
            "fallback_groups_per_launch": out[3]}


def ptr_array(tensors):
    """A C array of the tensors' device pointers (any length) and the ctypes
    object that keeps it alive."""
    tensors = list(tensors)
    arr = (ctypes.c_void_p * max(len(tensors), 1))(*[t.data_ptr() for t in tensors])
    return ctypes.cast(arr, ctypes.POINTER(ctypes.c_void_p)), arr
