"""The CudaRenderer mirror (src/renderer/mod.rs) on the GPU: two-frame ring, ready/finish order,
LUT-overflow reporting, and frame contents equal to the kernel-level pipeline."""
from __future__ import annotations

import time

import numpy as np
import pytest

import kerrtrace_b200 as kt
from kerrtrace_b200 import workloads

pytestmark = pytest.mark.gpu


def _wait_ready(r, timeout=60.0):
    t0 = time.time()
    while time.time() - t0 < timeout:
        f = r.ready_frame()
        if f is not None:
            return f
        time.sleep(0.001)
    raise TimeoutError("frame not ready")


def test_ring_and_order(cuda):
    cfg, cam = workloads.scene("t1")
    r = kt.Renderer(cfg)
    args = (list(cam.cam_pos), list(cam.fwd), list(cam.rgt), list(cam.up), cam.fov_scale)
    assert r.submit_render(*args)
    assert r.submit_render(*args)
    assert not r.submit_render(*args)          # both frames in flight (mod.rs:127-129)
    with pytest.raises(kt.KtError) as e:
        r.finish_frame(1)                      # out of order (mod.rs:253-256)
    assert e.value.status == kt.KT_ERR_QUEUE_ORDER
    i0, img0 = _wait_ready(r)
    img0 = img0.copy()
    r.finish_frame(i0)
    i1, img1 = _wait_ready(r)
    assert i1 != i0 and np.array_equal(img0, img1)
    r.finish_frame(i1)
    assert r.ready_frame() is None
    with pytest.raises(kt.KtError):
        r.finish_frame(0)
    # the frame equals trace + fused post through the kernel-level entry points
    ctx = kt.Context(cfg)
    n = cfg.width * cfg.height
    hdr = cuda.zeros((n, 4), device="cuda")
    err = cuda.zeros(2, dtype=cuda.int32, device="cuda")
    img = cuda.zeros(n, dtype=cuda.int32, device="cuda")
    ctx.trace(cam, hdr.data_ptr(), err.data_ptr(), 0, kt.SCHED_PLAIN)
    ctx.post_fused(hdr.data_ptr(), img.data_ptr())
    cuda.cuda.synchronize()
    assert np.array_equal(img.cpu().numpy().view(np.uint32), img0)
    assert np.all(img0 >> 24 == 0) and img0.max() > 0
    r.close()


def test_overflow_is_reported_by_ready_frame(cuda):
    cfg, cam = workloads.scene("t1")
    cfg.lut_max_temp = 1500.0
    r = kt.Renderer(cfg)
    assert r.submit_render(list(cam.cam_pos), list(cam.fwd), list(cam.rgt), list(cam.up), cam.fov_scale)
    r.wait()
    with pytest.raises(kt.LutOverflow) as e:
        r.ready_frame()
    assert e.value.temp > 1500.0
    r.close()


def test_both_schedules_render_the_same_frame(cuda):
    cfg, cam = workloads.scene("t2")
    frames = []
    for sched in (kt.SCHED_PLAIN, kt.SCHED_WAVEFRONT):
        r = kt.Renderer(cfg)
        r.set_schedule(sched)
        assert r.submit_render(list(cam.cam_pos), list(cam.fwd), list(cam.rgt), list(cam.up), cam.fov_scale)
        r.wait()
        idx, img = r.ready_frame()
        frames.append(img.copy())
        r.finish_frame(idx)
        r.close()
    assert np.array_equal(frames[0], frames[1])


def test_pipelined_frames_keep_their_own_camera(cuda):
    """Two frames in flight (the post passes and the copy of one overlapping the trace of the
    next, on their own streams): each frame handed back is the image of the camera it was
    submitted with."""
    cfg, _ = workloads.scene("t2")
    cams = [kt.orbit_camera(40.0, 50.0 + 6.0 * k, 30.0) for k in range(6)]
    ctx = kt.Context(cfg)
    n = cfg.width * cfg.height
    hdr = cuda.zeros((n, 4), device="cuda")
    err = cuda.zeros(2, dtype=cuda.int32, device="cuda")
    img = cuda.zeros(n, dtype=cuda.int32, device="cuda")
    expect = []
    for cam in cams:
        ctx.trace(cam, hdr.data_ptr(), err.data_ptr(), 0, kt.SCHED_PLAIN)
        ctx.post_fused(hdr.data_ptr(), img.data_ptr())
        cuda.cuda.synchronize()
        expect.append(img.cpu().numpy().view(np.uint32).copy())
    assert not np.array_equal(expect[0], expect[1])
    r = kt.Renderer(cfg)
    r.set_schedule(kt.SCHED_PLAIN)
    got, submitted, t0 = [], 0, time.time()
    while len(got) < len(cams) and time.time() - t0 < 60:
        if submitted < len(cams):
            c = cams[submitted]
            if r.submit_render(list(c.cam_pos), list(c.fwd), list(c.rgt), list(c.up), c.fov_scale):
                submitted += 1
                continue
        f = r.ready_frame()
        if f is not None:
            got.append(f[1].copy())
            r.finish_frame(f[0])
    r.close()
    assert len(got) == len(cams)
    for k in range(len(cams)):
        assert np.array_equal(got[k], expect[k]), k
