"""mlgpu_probe_fp64_rate, the measured denominator of the tracers' compute
roofline: plausible FP64 rates for a B200 (nominal 37 TFLOP/s with FMAs),
and adds/multiplies at about half the FMA FLOP rate (one operation per
cycle and lane either way)."""
import ctypes as C

import pytest

pytestmark = pytest.mark.gpu


def test_fp64_rate_probe():
    import torch
    assert torch.cuda.is_available()
    from merlict_development_kit_b200 import _native
    L = _native.lib()
    fma, addmul = C.c_double(0.0), C.c_double(0.0)
    _native.check(L.mlgpu_probe_fp64_rate(1, C.byref(fma), None))
    _native.check(L.mlgpu_probe_fp64_rate(0, C.byref(addmul), None))
    assert 5e12 < fma.value < 60e12, fma.value
    assert 2e12 < addmul.value < 40e12, addmul.value
    assert 1.5 < fma.value / addmul.value < 2.5
    with pytest.raises(ValueError):
        _native.check(L.mlgpu_probe_fp64_rate(1, None, None))
