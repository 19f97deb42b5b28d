"""Algorithmic operation counts of the geodesic integration (the roofline numerator).

Counted by hand from the restated source (csrc/kt_device.cuh hamilton_rhs, csrc/kt_ray.cuh
ray_advance / step_tolerance): an FMA counts 2 flops, every other add / mul / min / max /
divide / reciprocal-square-root counts 1, sign and absolute-value bit operations 0.  The
work unit counts (RHS evaluations, DP5(4) attempts, committed steps) come from the counting
trace of the same scene (kt_trace_counted), so the total is the work the plain method needs
for that frame, independent of how it is scheduled.

  RHS_FLOPS      one Hamiltonian right-hand side (kerr_math.cuh:82-156)           160
  ATTEMPT_FLOPS  stage inputs of k2..k7, the 5th-order update, the embedded error
                 norm and the step-size update of one attempt (kerr_trace.cuh:85-121) 371
  STEP_FLOPS     tolerance at the step start and radius after the commit
                 (kerr_trace.cuh:67-73, 135)                                        41
"""
RHS_FLOPS = 160
ATTEMPT_FLOPS = 371
STEP_FLOPS = 41


def trace_flops(stats) -> int:
    return int(stats.rhs_evals) * RHS_FLOPS + int(stats.attempts) * ATTEMPT_FLOPS + int(stats.steps) * STEP_FLOPS


# FP32 lanes per SM on sm_100 (4 SM sub-partitions x 32 FP32 lanes)
FP32_LANES_PER_SM = 128
