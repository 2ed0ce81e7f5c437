"""The FMA-rate microbenchmark behind the FP64 roofline of bench.py: a
plausible B200 rate in both precisions (B200: 148 SMs at up to 1.965 GHz;
FP64 at most 64 and FP32 at most 128 FMA lanes per SM and clock)."""
import pytest

from exocubed_b200 import _native as nat

pytestmark = pytest.mark.gpu


def test_fma_peaks_are_plausible():
    f64 = nat.fma_peak(True, repeats=2)
    f32 = nat.fma_peak(False, repeats=2)
    ceiling64 = 148 * 64 * 2 * 2.0e9
    assert 0.2 * ceiling64 < f64 < 1.05 * ceiling64, f64
    assert f64 < f32 < 1.05 * 2 * ceiling64, (f64, f32)


def test_fma_peak_rejects_bad_arguments():
    import ctypes
    out = ctypes.c_double()
    assert nat.lib().exo_measure_fma_peak(1, 0, ctypes.byref(out)) == nat.EXO_ERR_ARG
    assert nat.lib().exo_measure_fma_peak(1, 1, None) == nat.EXO_ERR_ARG
