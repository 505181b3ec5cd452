"""ecg_measure_fp64_peak: the FP64 FMA throughput the bench divides the
explicit step's FP64 flop rate by (no counterpart in the reference)."""
import pytest

from amrex_euler_allmach_explicit_imex_b200 import api

pytestmark = pytest.mark.gpu


def test_fp64_peak_is_plausible(gpu):
    # B200 datasheet: 37-40 TFLOP/s FP64; allow clocks well below boost
    t = api.measure_fp64_peak(0)
    assert 5.0 < t < 100.0, t


def test_fp64_peak_rejects_bad_device(gpu):
    with pytest.raises(api.EcgError):
        api.measure_fp64_peak(1 << 20)
