"""Batched renders on the GPU: one launch over many scenes and cameras must render each job
exactly as its own kt_trace does, directly and through the captured CUDA graph."""
from __future__ import annotations

import numpy as np
import pytest

import kerrtrace_b200 as kt
from kerrtrace_b200 import workloads
from tests.helpers import run_ours

pytestmark = pytest.mark.gpu


def _alloc(torch, jobs):
    bufs = []
    for cfg, cam in jobs:
        n = cfg.width * cfg.height
        bufs.append((torch.full((n, 4), -1.0, device="cuda"), torch.zeros(2, dtype=torch.int32, device="cuda")))
    return bufs


@pytest.mark.parametrize("mode,prec", [(kt.MODE_REF, kt.PREC_FP32), (kt.MODE_SPEC, kt.PREC_MIXED),
                                       (kt.MODE_SPEC, kt.PREC_FP64)])
def test_batch_matches_per_job_traces(cuda, mode, prec):
    jobs = workloads.c4_jobs(scale=16)[::8]   # 8 jobs of different sizes, spins, cameras, disks
    for c, _ in jobs:
        c.mode, c.precision = mode, prec
    bufs = _alloc(cuda, jobs)
    b = kt.Batch([(c, cam, h.data_ptr(), e.data_ptr()) for (c, cam), (h, e) in zip(jobs, bufs)])
    assert b.rays() == sum(c.width * c.height for c, _ in jobs)
    expected = [run_ours(cuda, c, cam, kt.SCHED_PLAIN)[0] for c, cam in jobs]

    def check():
        cuda.cuda.synchronize()
        for (h, _), exp in zip(bufs, expected):
            assert np.array_equal(h.cpu().numpy().view(np.uint32), exp.view(np.uint32))

    b.trace()
    check()
    for h, _ in bufs:
        h.fill_(-1.0)
    b.trace_graph()
    b.trace_graph()
    check()
    b.set_block(8, 8)
    for h, _ in bufs:
        h.fill_(-1.0)
    b.trace_graph()
    check()
    for h, _ in bufs:
        h.fill_(-1.0)
    b.trace_sequential()
    check()
    # the persistent launch (32-pixel units of one job per warp, one counter over all jobs)
    for bps in (4, 6):
        b.set_tuning(kt.SCHED_WAVEFRONT, blocks_per_sm=bps)
        assert b.tuning().schedule == kt.SCHED_WAVEFRONT
        for h, _ in bufs:
            h.fill_(-1.0)
        b.trace()
        check()
        for h, _ in bufs:
            h.fill_(-1.0)
        b.trace_graph()
        b.trace_graph()
        check()
    # the batch tuner: every candidate identical, the installed one reproduces the images
    rows = b.autotune(reps=1)
    assert len(rows) == (9 if prec == kt.PREC_FP32 else 7) and all(ok for _, _, ok in rows)
    for h, _ in bufs:
        h.fill_(-1.0)
    b.trace_graph()
    check()
    b.set_block(8, 8)
    # a new camera for job 2 is picked up by the next graph launch
    cfg2, _ = jobs[2]
    cam2 = kt.orbit_camera(77.0, 33.0, 25.0)
    b.set_camera(2, cam2)
    b.trace_graph()
    cuda.cuda.synchronize()
    exp2 = run_ours(cuda, cfg2, cam2, kt.SCHED_PLAIN)[0]
    assert np.array_equal(bufs[2][0].cpu().numpy().view(np.uint32), exp2.view(np.uint32))
    b.close()


def test_batch_limits(cuda):
    cfg, cam = workloads.scene("t2")
    h = cuda.zeros((cfg.width * cfg.height, 4), device="cuda")
    e = cuda.zeros(2, dtype=cuda.int32, device="cuda")
    with pytest.raises(kt.KtError):
        kt.Batch([])
    with pytest.raises(kt.KtError):
        kt.Batch([(cfg, cam, h.data_ptr(), e.data_ptr())] * (kt.BATCH_MAX_JOBS + 1))
    c2 = cfg.copy()
    c2.mode = kt.MODE_SPEC
    with pytest.raises(kt.KtError):
        kt.Batch([(cfg, cam, h.data_ptr(), e.data_ptr()), (c2, cam, h.data_ptr(), e.data_ptr())])


@pytest.mark.parametrize("schedule", [kt.SCHED_PLAIN, kt.SCHED_WAVEFRONT])
def test_batch_jobs_match_the_reference_kernel(cuda, schedule):
    """Jobs of one batch, compared one by one with the reference's own trace_kernel
    (oracle/_ref).  The reference bakes some scene values into #defines, so the jobs keep the
    1080p scene's (temperature scale, horizon epsilon, tolerance, step budget) and vary what it
    takes at run time: spin, camera, frame size, disk outer radius and LUT range.  Plain and
    persistent batched launches."""
    from tests.helpers import run_ref
    base, _ = workloads.scene("c2")
    rng = np.random.default_rng(5)
    jobs = []
    for w, h in ((96, 64), (160, 90), (64, 128), (200, 120)):
        c = workloads.scaled(base, w, h)
        c.spin = float(rng.uniform(-0.95, 0.95))
        c.disk_outer_radius = float(rng.uniform(12.0, 40.0))
        c.lut_max_temp = float(rng.uniform(1e5, 3e5))
        cam = kt.orbit_camera(float(rng.uniform(40.0, 150.0)), float(rng.uniform(10.0, 85.0)), 25.0)
        jobs.append((c, cam))
    bufs = _alloc(cuda, jobs)
    b = kt.Batch([(c, cam, h.data_ptr(), e.data_ptr()) for (c, cam), (h, e) in zip(jobs, bufs)])
    if schedule == kt.SCHED_WAVEFRONT:
        b.set_tuning(kt.SCHED_WAVEFRONT, blocks_per_sm=5)
    else:
        b.set_block(8, 16)
    b.trace()
    cuda.cuda.synchronize()
    for (c, cam), (h, e) in zip(jobs, bufs):
        ref, err_r = run_ref(cuda, "c2", c, cam)
        ours = h.cpu().numpy()
        assert np.all(ours[:, 3] == 1.0)
        assert np.array_equal(ours.view(np.uint32), ref.view(np.uint32)), (c.width, c.height, c.spin)
        assert np.array_equal(e.cpu().numpy().view(np.uint32), err_r)
    b.close()


def test_persistent_batch_of_64_ragged_jobs(cuda):
    """The largest batch (64 jobs) of ragged frames, one pixel, single rows and columns and odd
    sizes, whose 32-pixel units end inside a row or straddle none: every job equals its own
    kt_trace bit for bit under the persistent launch (4 and 6 resident blocks per SM) and its
    graph replay, and every pixel is written."""
    base, _ = workloads.scene("t1")
    sizes = [(1, 1), (1, 17), (23, 1), (37, 23), (31, 1), (33, 2), (5, 7), (64, 3)] * 8
    rng = np.random.default_rng(9)
    jobs = []
    for w, h in sizes:
        c = workloads.scaled(base, w, h)
        c.spin = float(rng.uniform(-0.9, 0.9))
        c.disk_temperature_scale = base.disk_temperature_scale
        jobs.append((c, kt.orbit_camera(float(rng.uniform(20.0, 60.0)), float(rng.uniform(20.0, 85.0)), 40.0)))
    assert len(jobs) == kt.BATCH_MAX_JOBS
    bufs = _alloc(cuda, jobs)
    b = kt.Batch([(c, cam, h.data_ptr(), e.data_ptr()) for (c, cam), (h, e) in zip(jobs, bufs)])
    expected = [run_ours(cuda, c, cam, kt.SCHED_PLAIN)[0] for c, cam in jobs]
    for bps, graph in ((4, False), (6, True)):
        for h, _ in bufs:
            h.fill_(-1.0)
        b.set_tuning(kt.SCHED_WAVEFRONT, blocks_per_sm=bps)
        (b.trace_graph if graph else b.trace)()
        cuda.cuda.synchronize()
        for (h, _), exp in zip(bufs, expected):
            got = h.cpu().numpy()
            assert np.all(got[:, 3] == 1.0)
            assert np.array_equal(got.view(np.uint32), exp.view(np.uint32))
    b.close()
