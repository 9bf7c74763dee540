"""SLAdvector's argument checks (semilag.py:204-219), on CPU: the same
ValueError messages as the reference, in the same order of precedence, raised
before any device work.  A valid argument set on a CPU device raises
RuntimeError instead: there is no CPU path."""

import pytest
import torch

from slchannel_b200.semilag import SLAdvector


def _grid(nz=12):
    z_f = torch.linspace(0, 2, nz + 1, dtype=torch.float64)
    z_c = torch.cat([-z_f[1:2] / 2, 0.5 * (z_f[1:] + z_f[:-1]),
                     z_f[-1:] + (z_f[-1:] - z_f[-2:-1]) / 2])
    return z_f, z_c


def _make(nz=12, **kw):
    z_f, z_c = _grid(nz)
    args = dict(order=6, device="cpu")
    args.update(kw)
    return SLAdvector(8, 6, nz, 0.5, 0.5, 4.0, 3.0, 2.0, z_f, z_c, 2.0, **args)


@pytest.mark.parametrize("kw, nz, msg", [
    (dict(order=5), 12, r"sl\.interp_order must be 4 \(tricubic\) or 6 \(triquintic\), got 5"),
    (dict(order=2), 12, r"sl\.interp_order must be 4 \(tricubic\) or 6 \(triquintic\), got 2"),
    (dict(traj_order=3), 12, r"sl\.traj_interp_order must be 2 \(trilinear\) or 4 \(tricubic\), got 3"),
    (dict(stretching_type="top"), 12, r"SLAdvector supports 'symmetric'/'bottom' stretching, got 'top'"),
    (dict(interp_dtype="fp16"), 12, r"sl\.interp_dtype must be .*got fp16"),
    (dict(order=6), 4, r"nz=4 too small for interpolation order 6"),
    (dict(order=4), 2, r"nz=2 too small for interpolation order 4"),
])
def test_bad_arguments_raise_the_reference_message(kw, nz, msg):
    with pytest.raises(ValueError, match=msg):
        _make(nz=nz, **kw)


def test_checks_run_in_the_reference_order():
    # order is checked before traj_order, traj_order before stretching, and so on
    with pytest.raises(ValueError, match="interp_order"):
        _make(order=3, traj_order=3, stretching_type="x", interp_dtype="x", nz=1)
    with pytest.raises(ValueError, match="traj_interp_order"):
        _make(traj_order=3, stretching_type="x", interp_dtype="x", nz=1)
    with pytest.raises(ValueError, match="stretching"):
        _make(stretching_type="x", interp_dtype="x", nz=1)
    with pytest.raises(ValueError, match="interp_dtype"):
        _make(interp_dtype="x", nz=1)


@pytest.mark.parametrize("kw", [dict(order=6), dict(order=4, traj_order=4),
                                dict(stretching_type="bottom"), dict(interp_dtype="fp32_accum64"),
                                dict(interp_dtype="mixed")])
def test_valid_arguments_on_cpu_refuse_without_fallback(kw):
    with pytest.raises(RuntimeError, match="no CPU path"):
        _make(**kw)


def test_smallest_grid_the_stencil_allows_passes_the_checks():
    # nz + 1 == order is accepted by the checks (it then needs a CUDA device)
    with pytest.raises(RuntimeError, match="no CPU path"):
        _make(nz=5, order=6)
