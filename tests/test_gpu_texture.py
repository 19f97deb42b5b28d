"""Pins the oracle's model of hardware linear texture filtering (used for the reference's LUT
lookups, src/renderer/texture.rs:176-202) against the texture unit itself, sampled through the
reference harness.  The model: x = u*N - 0.5, i = floor(x), weight = frac(x) in 1.8 fixed point."""
from __future__ import annotations

import numpy as np
import pytest

from kerrtrace_b200 import workloads

pytestmark = pytest.mark.gpu


def emulate(lut, u, mode):
    n = lut.shape[0]
    x = u.astype(np.float64) * n - 0.5
    i0 = np.floor(x)
    w = x - i0
    if mode == "round":
        w = np.rint(w * 256) / 256
    elif mode == "trunc":
        w = np.floor(w * 256) / 256
    i0 = i0.astype(np.int64)
    a = lut[np.clip(i0, 0, n - 1)].astype(np.float64)
    b = lut[np.clip(i0 + 1, 0, n - 1)].astype(np.float64)
    w = w.reshape((-1,) + (1,) * (lut.ndim - 1))
    return (1 - w) * a + w * b


def test_texture_model(cuda, orc):
    cfg, _ = workloads.scene("t1")
    p, bb, disk = orc.reference_inputs(cfg)
    ref = orc.RefKernel("t1")
    ref.setup(p, bb, disk)
    rng = np.random.default_rng(3)
    u = np.concatenate([rng.random(20000), np.linspace(-0.01, 1.01, 4001)]).astype(np.float32)
    us = cuda.from_numpy(u).cuda()
    out = cuda.zeros(len(u), device="cuda")
    ref.tex_probe("disk", us.data_ptr(), out.data_ptr(), len(u))
    hw = out.cpu().numpy().astype(np.float64)
    errs = {m: np.max(np.abs(emulate(disk, u, m) - hw)) for m in ("exact", "round", "trunc")}
    print(errs)
    scale = float(np.abs(disk).max())
    # the 1/256 weight model is the closest of the three; it is what the oracle uses (tex_mode 1)
    assert errs["round"] == min(errs.values()), errs
    assert errs["round"] <= 1e-3 * scale, errs
    out4 = cuda.zeros((len(u), 4), device="cuda")
    ref.tex_probe("bb", us.data_ptr(), out4.data_ptr(), len(u))
    hw4 = out4.cpu().numpy().astype(np.float64)
    e4 = np.max(np.abs(emulate(bb, u, "round") - hw4) / np.maximum(np.abs(hw4), 1e-3 * np.abs(bb).max()))
    assert e4 <= 1e-2, e4
    ref.close()
