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
