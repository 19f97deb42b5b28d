"""Host-side helpers of bench.py on CPU: the whole-job throughput and the histogram quantiles
that the 4096^2 precision ablation reports."""
from __future__ import annotations

import numpy as np
import torch

import bench


def test_job_throughput_counts_every_rank():
    # 2 ranks x 1000 rays in 2 ms (the slowest rank) = 1 Mrays/s
    assert abs(bench.job_mrays_s(1000, 2, 2.0) - 1.0) < 1e-12


def test_histogram_quantiles_are_within_one_bin():
    rng = np.random.default_rng(0)
    x = torch.tensor(10.0 ** rng.uniform(-9.0, -2.0, size=200_000))
    hist = torch.zeros(1300, dtype=torch.float64)
    bench._log_hist(x, hist)
    assert float(hist.sum()) == x.numel()
    for q in (0.5, 0.99, 0.999):
        exact = float(np.quantile(x.numpy(), q))
        got = bench._hist_quantile(hist, q)
        assert exact <= got <= exact * 10 ** 0.02 * 1.0001, (q, exact, got)
    # zeros land in the first bin
    hz = torch.zeros(1300, dtype=torch.float64)
    bench._log_hist(torch.zeros(10, dtype=torch.float64), hz)
    assert float(hz[0]) == 10
    assert bench._hist_quantile(torch.zeros(1300, dtype=torch.float64), 0.5) is None


def test_both_arms_describe_the_same_workload(kt, orc):
    """bench.py's own arm builds its scene through the library's host entry points, the
    reference arm through the oracle's restatement (so that it loads no product library); both
    must print the same config.workload and see the same scene and camera bits."""
    from kerrtrace_b200 import workloads
    for size in (None, "480x270"):
        c_lib, cam_lib = bench.rank_camera(workloads, "c2", 0, 1, size)
        c_ref, cam_ref = bench.rank_camera(workloads, "c2", 0, 1, size, host=orc.Host())
        assert bench.workload_label("c2", c_lib) == bench.workload_label("c2", c_ref)
        assert bytes(c_lib) == bytes(c_ref) and bytes(cam_lib) == bytes(cam_ref)
