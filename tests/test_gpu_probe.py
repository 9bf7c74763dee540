"""slc_fma_peak: the FMA-chain probe that gives the trace+gather kernels'
FP64 / FP32 arithmetic roofline returns a plausible rate for this GPU."""

import pytest

from slchannel_b200 import _native as N

pytestmark = pytest.mark.gpu


def test_fma_peak_plausible():
    f64 = N.fma_peak_gflops(True)
    f32 = N.fma_peak_gflops(False)
    assert 1e3 < f64 < 2e5  # GFLOP/s
    assert 1e3 < f32 < 4e5
    assert f32 >= 0.5 * f64


def test_gather_probe_formulations_agree():
    """slc_gather_probe: the tensor-core (FP16x3 mma.sync) gather agrees with
    the one-thread-per-point FP32 gather to FP32-level accuracy, and both
    report a time."""
    r = N.gather_probe(64, 2)
    assert r["scalar_ms"] > 0 and r["tensor_ms"] > 0
    assert r["max_rel_diff"] < 1e-5
    assert r["fallback_groups_per_launch"] >= 0


def test_gather_probe_rejects_bad_sizes():
    with pytest.raises(ValueError, match="n must be"):
        N.gather_probe(100, 1)
