"""Progressive sampling and the headless render loop on the GPU: the reference's per-pixel
sample loop split over launches gives, after N samples, the spp = N image bit for bit; the
re-render policy submits only changed views and the first frame written as PNG is the frame."""
from __future__ import annotations

import struct
import time
import zlib

import numpy as np
import pytest

import kerrtrace_b200 as kt
from kerrtrace_b200 import workloads

pytestmark = pytest.mark.gpu


def _trace(torch, cfg, cam):
    ctx = kt.Context(cfg)
    n = cfg.width * cfg.height
    hdr = torch.zeros((n, 4), device="cuda")
    err = torch.zeros(2, dtype=torch.int32, device="cuda")
    ctx.trace(cam, hdr.data_ptr(), err.data_ptr(), 0, kt.SCHED_PLAIN)
    torch.cuda.synchronize()
    ctx.close()
    return hdr


@pytest.mark.parametrize("mode", [kt.MODE_REF, kt.MODE_SPEC])
def test_progressive_samples_equal_the_spp_render(cuda, mode):
    cfg, cam = workloads.scene("t1")
    cfg.mode = mode
    n = cfg.width * cfg.height
    expect = {}
    for spp in (2, 3, 4):
        c = cfg.copy()
        c.spp = spp
        expect[spp] = _trace(cuda, c, cam)
    ctx = kt.Context(cfg)
    acc = cuda.full((n, 4), float("nan"), device="cuda")   # never read at first_sample 0
    hdr = cuda.zeros((n, 4), device="cuda")
    err = cuda.zeros(2, dtype=cuda.int32, device="cuda")
    done = 0
    for first, count in ((0, 2), (2, 1), (3, 1)):
        ctx.trace_progressive(cam, first, count, acc.data_ptr(), hdr.data_ptr(), err.data_ptr())
        cuda.cuda.synchronize()
        done = first + count
        assert cuda.equal(hdr.view(cuda.int32), expect[done].view(cuda.int32)), (mode, done)
        assert bool((acc[:, 3] == done).all())
    assert int(err[0]) == 0
    ctx.close()


def test_view_sequence_submits_changed_views_and_writes_the_first_frame(cuda, tmp_path):
    cfg, _ = workloads.scene("t2")
    ctx = kt.Context(cfg)
    n = cfg.width * cfg.height
    # a camera that orbits, then rests for a few ticks (the policy renders nothing), then turns
    views = [kt.make_view([30.0 * np.sin(np.radians(3 * k)), 8.0, 30.0 * np.cos(np.radians(3 * k))],
                          180.0 - 3 * k, -15.0, 40.0) for k in range(5)]
    views += [views[-1]] * 4
    views += [kt.make_view(list(views[-1].cam_pos), views[-1].yaw_deg + 2.0, -15.0, 40.0)]
    state = kt.ViewState(views[0])
    r = kt.Renderer(cfg)
    r.set_schedule(kt.SCHED_PLAIN)
    submitted, frames, t0 = [], [], time.time()
    for k, v in enumerate(views):
        while state.should_render(v) and time.time() - t0 < 60:
            if r.submit_view(state, v):
                submitted.append(k)
                break
            f = r.ready_frame()
            if f is not None:
                frames.append(f[1].copy())
                r.finish_frame(f[0])
    while len(frames) < len(submitted) and time.time() - t0 < 60:
        f = r.ready_frame()
        if f is not None:
            frames.append(f[1].copy())
            r.finish_frame(f[0])
    r.close()
    assert submitted == [0, 1, 2, 3, 4, 9]
    # each frame is the kernel-level render of its view
    hdr = cuda.zeros((n, 4), device="cuda")
    err = cuda.zeros(2, dtype=cuda.int32, device="cuda")
    img = cuda.zeros(n, dtype=cuda.int32, device="cuda")
    for k, frame in zip(submitted, frames):
        v = views[k]
        cam = kt.make_camera(list(v.cam_pos), v.yaw_deg, v.pitch_deg, v.fov_deg)
        ctx.trace(cam, hdr.data_ptr(), err.data_ptr(), 0, kt.SCHED_PLAIN)
        ctx.post_fused(hdr.data_ptr(), img.data_ptr())
        cuda.cuda.synchronize()
        assert np.array_equal(img.cpu().numpy().view(np.uint32), frame), k
    ctx.close()
    path = tmp_path / "first_frame.png"
    assert kt.write_png(path, frames[0], cfg.width, cfg.height)
    data = path.read_bytes()
    (n_ihdr,) = struct.unpack(">I", data[8:12])
    idat_at = 8 + 12 + n_ihdr
    (n_idat,) = struct.unpack(">I", data[idat_at:idat_at + 4])
    raw = np.frombuffer(zlib.decompress(data[idat_at + 8:idat_at + 8 + n_idat]), np.uint8)
    rgba = raw.reshape(cfg.height, 1 + 4 * cfg.width)[:, 1:].reshape(-1, 4).astype(np.uint32)
    assert np.array_equal((rgba[:, 0] << 16) | (rgba[:, 1] << 8) | rgba[:, 2], frames[0])
