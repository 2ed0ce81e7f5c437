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


def test_bounded_wait_gives_up_and_the_device_stays_usable():
    """Failure detection without a fault: a wait on an mbarrier phase that
    nothing completes (the bounded wait the back-substitution kernel uses for
    its bulk copies) gives up after about 0.1 s and the kernel ends; the
    device then runs a step as usual."""
    import ctypes

    from exocubed_b200 import workloads as W
    from exocubed_b200.atmosphere import CubedSphereAtmosphere
    gave_up, ms = ctypes.c_int(-1), ctypes.c_double()
    nat.check(nat.lib().exo_check_bounded_wait(ctypes.byref(gave_up), ctypes.byref(ms)))
    assert gave_up.value == 1
    assert 90.0 <= ms.value < 2000.0, ms.value
    cfg = W.dry_atmosphere_config(N=8, L=8)
    with CubedSphereAtmosphere(cfg) as a:
        a.set_primitive(W.dry_atmosphere_state(cfg, seed=1))
        a.step(2)
        assert a.invalid() == 0


@pytest.mark.parametrize("precision", [nat.EXO_PREC_FP64, nat.EXO_PREC_MIXED])
def test_reciprocal_of_the_implicit_blocks(precision):
    """1/x as the implicit solve's FP64 blocks take it: the FP64 build's IEEE
    division equals numpy's bit for bit; the mixed build's reciprocal refined
    by Newton's method stays within two ulps of it, for finite x of either
    sign whose reciprocal is a normal number."""
    import numpy as np
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(7)
    x = np.concatenate([np.sign(rng.uniform(-1, 1, 20000)) * 10.0 ** rng.uniform(-300, 300, 20000),
                        rng.uniform(0.5, 2.0, 20000), np.array([1.0, -1.0, 3.0, 0.1, 7e-301])])
    xd = torch.from_numpy(x).cuda()
    out = torch.empty_like(xd)
    nat.check(nat.lib().exo_reciprocal(precision, x.size, xd.data_ptr(), out.data_ptr(), None))
    torch.cuda.synchronize()
    got, want = out.cpu().numpy(), 1.0 / x
    if precision == nat.EXO_PREC_FP64:
        assert np.array_equal(got, want)
    else:
        ulps = np.abs(got - want) / np.spacing(np.abs(want))
        assert ulps.max() <= 2.0, ulps.max()


def test_reciprocal_rejects_bad_arguments():
    assert nat.lib().exo_reciprocal(1, -1, None, None, None) == nat.EXO_ERR_ARG
    assert nat.lib().exo_reciprocal(7, 0, 1, 1, None) == nat.EXO_ERR_ARG
