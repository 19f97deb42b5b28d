"""The FP32 FMA throughput probe that gives the trace's roofline its denominator."""
from __future__ import annotations

import pytest

import kerrtrace_b200 as kt

pytestmark = pytest.mark.gpu


def test_fma_peak_is_near_the_nominal_fp32_rate(cuda):
    props = cuda.cuda.get_device_properties(0)
    tf, ms = kt.fma_peak(0, 16384)
    # SMs x 128 FP32 lanes x 2 flops at the highest SM clock of a B200 (1965 MHz)
    nominal_max = props.multi_processor_count * 128 * 2 * 1.965e9 / 1e12
    print("measured", tf, "TFLOP/s in", ms, "ms; nominal at 1965 MHz", nominal_max)
    assert 0.5 * nominal_max < tf < 1.05 * nominal_max
