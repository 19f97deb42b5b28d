"""The lookup tables generated on the device against the host generators (which are bit-equal to
the reference's Rust generators, tests/test_abi.py): agreement to a few ulp of the table."""
from __future__ import annotations

import numpy as np
import pytest

import kerrtrace_b200 as kt
from kerrtrace_b200 import workloads

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["c1", "c2", "t1"])
def test_device_luts_match_host_luts(cuda, name):
    cfg, _ = workloads.scene(name)
    n = cfg.lut_size
    host_bb = kt.generate_blackbody_lut(n, cfg.lut_max_temp, cfg.wavelength_start, cfg.wavelength_end,
                                        cfg.wavelength_step)
    p = kt.build_kerr_params(cfg)
    host_disk = kt.generate_disk_lut(p, cfg.disk_outer_radius, n)
    bb = cuda.full((n, 4), float("nan"), device="cuda")
    disk = cuda.full((n,), float("nan"), device="cuda")
    kt.generate_blackbody_lut_device(n, cfg.lut_max_temp, cfg.wavelength_start, cfg.wavelength_end,
                                     cfg.wavelength_step, bb.data_ptr())
    kt.generate_disk_lut_device(p, cfg.disk_outer_radius, n, disk.data_ptr())
    cuda.cuda.synchronize()
    dev_bb, dev_disk = bb.cpu().numpy(), disk.cpu().numpy()
    assert np.all(np.isfinite(dev_bb)) and np.all(np.isfinite(dev_disk))
    assert np.all(dev_bb[0] == 0.0) and np.all(dev_bb[:, 3] == 0.0)
    # blackbody rows: relative to each row's largest channel (rows span 40 decades)
    scale = np.maximum(np.abs(host_bb[:, :3]).max(1, keepdims=True), 1e-37)
    rel_bb = (np.abs(dev_bb[:, :3].astype(np.float64) - host_bb[:, :3]) / scale).max()
    rel_disk = np.abs(dev_disk.astype(np.float64) - host_disk).max() / np.abs(host_disk).max()
    print(name, "blackbody", rel_bb, "disk", rel_disk)
    assert rel_bb < 2e-5, rel_bb
    # near the ISCO of a = 0.998 the flux factor subtracts nearly equal logarithms in f32: an ulp
    # of either libm grows to 1.7e-5 of the table maximum there
    assert rel_disk < 1e-4, rel_disk
    assert dev_disk[0] == 0.0 and host_disk[0] == 0.0


@pytest.mark.parametrize("name,size", [("c2", (320, 180)), ("t1", None), ("c1", (128, 128))])
def test_context_with_device_luts_renders_within_parity(cuda, name, size):
    """A context whose LUTs were generated on the device (kt_context_create_device_luts) renders
    the frame of a host-table context to the parity tolerance, and its post gives the same image
    to one code value."""
    from tests.helpers import compare_hdr, run_ours
    cfg, cam = workloads.scene(name)
    if size:
        cfg = workloads.scaled(cfg, *size)
    a, ea, _, ca = run_ours(cuda, cfg, cam, kt.SCHED_PLAIN)
    cd = kt.Context(cfg, luts="device")
    b, eb, _, _ = run_ours(cuda, cfg, cam, kt.SCHED_PLAIN, ctx=cd)
    r = compare_hdr(b, a, cfg.width, cfg.height)
    print(name, r)
    assert np.all(b[:, 3] == 1.0)
    assert r["class_mismatch_inner"] == 0, r
    assert r["over_tol_inner"] <= max(2, 2e-4 * r["n"]), r
    assert r["over_tol_all"] <= max(2, 0.005 * r["n"]), r
    assert np.array_equal(ea, eb)
    n = cfg.width * cfg.height
    img = {}
    for key, ctx, h in (("host", ca, a), ("device", cd, b)):
        hd = cuda.tensor(h, device="cuda")
        im = cuda.zeros(n, dtype=cuda.int32, device="cuda")
        ctx.post_fused(hd.data_ptr(), im.data_ptr())
        cuda.cuda.synchronize()
        img[key] = im.cpu().numpy().view(np.uint32)
    d = np.max(np.abs(np.stack([(img["host"] >> s) & 255 for s in (16, 8, 0)]).astype(int) -
                      np.stack([(img["device"] >> s) & 255 for s in (16, 8, 0)]).astype(int)), axis=0)
    assert np.mean(d > 1) <= 1e-3, np.bincount(d)
    ca.close()
    cd.close()
