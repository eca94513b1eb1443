"""Tensor-pipe peak probes (lt_measure_peak): each tcgen05 form passes its own accumulator check
(A = 1 / 3 per CTA, B = 1 / 2 per half of N) and the measured rates are physically plausible for
a B200 (148 SMs, FP64 128 FLOP/clk/SM, INT8 16384 op/clk/SM, clocks up to about 2 GHz)."""
from __future__ import annotations

import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,lo,hi", [(0, 20e12, 45e12), (1, 2.0e15, 6.0e15), (2, 2.0e15, 6.0e15),
                                        (3, 2.0e15, 6.0e15)])
def test_peak_probe(cuda, kind, lo, hi):
    import libthom_b200 as lt

    v = lt.measure_peak(kind)
    assert lo < v < hi, v
    lt.device_status()


def test_sustained_rate_not_above_burst(cuda):
    """LT_PEAK_SUSTAINED times the same loop after 0.5 s at the power limit: never meaningfully
    faster than one launch, and within the physical range."""
    import libthom_b200 as lt

    burst = max(lt.measure_peak(lt.LT_PEAK_INT8_MMA_PAIR) for _ in range(2))
    sustained = lt.measure_peak(lt.LT_PEAK_INT8_MMA_PAIR | lt.LT_PEAK_SUSTAINED)
    assert 2.0e15 < sustained <= 1.05 * burst, (sustained, burst)
