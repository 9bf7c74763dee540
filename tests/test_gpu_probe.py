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
