"""Generates the golden fixtures in tests/golden/ from the reference itself.

Runs on a CUDA machine: the reference's own cuda/kernel.cu, compiled from its source into
oracle/_ref/libktref_<scene>.so (oracle/build.py), traces each scene with the launch sequence of
src/renderer/mod.rs; the HDR buffer, the LUT error word and the post-processed 0x00RRGGBB
image are saved.  It also samples the reference's LUT textures (linear filter, normalised
coordinates, clamp) at chosen coordinates, to pin the oracle's model of hardware filtering.

    python tests/golden/make_golden.py <out_dir>
"""
from __future__ import annotations

import json
import math
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

# scene -> resolution of the fixture (the scene's #defines are unchanged)
FIXTURES = {"t1": None, "t2": None, "c1": (64, 64), "c2": (192, 108)}


def main(out: Path) -> None:
    import torch

    import oracle
    from kerrtrace_b200 import workloads

    host = oracle.Host()
    out.mkdir(parents=True, exist_ok=True)
    meta = {}
    for name, size in FIXTURES.items():
        cfg, cam = workloads.scene(name, host=host)
        if size:
            cfg = workloads.scaled(cfg, *size)
        # the reference host's inputs from the oracle's restatement (no product code on this path)
        p, bb, disk = oracle.reference_inputs(cfg)
        ref = oracle.RefKernel(name)
        ref.setup(p, bb, disk)
        n = cfg.width * cfg.height
        hdr = torch.zeros((n, 4), device="cuda")
        bloom = torch.zeros((n, 4), device="cuda")
        img = torch.zeros(n, dtype=torch.int32, device="cuda")
        err = torch.zeros(2, dtype=torch.int32, device="cuda")
        ref.trace(hdr.data_ptr(), cfg, cam, cfg.lut_max_temp, err.data_ptr(), p.disk_inner)
        radius = int(math.ceil(np.float32(cfg.bloom_radius))) if cfg.bloom_radius > 0 else 0
        sigma = float(np.float32(cfg.bloom_radius) / np.float32(3.0))
        active = int(bool(cfg.bloom_enabled) and radius > 0 and cfg.bloom_intensity > 0)
        if active:
            ref.bloom(hdr.data_ptr(), bloom.data_ptr(), cfg, radius, sigma, active)
        ref.post(hdr.data_ptr(), bloom.data_ptr(), img.data_ptr(), cfg, radius, sigma, cfg.bloom_intensity, active)
        torch.cuda.synchronize()
        np.savez_compressed(out / f"ref_{name}.npz", hdr=hdr.cpu().numpy()[:, :3],
                            err=err.cpu().numpy().view(np.uint32), image=img.cpu().numpy().view(np.uint32))
        meta[name] = {"width": int(cfg.width), "height": int(cfg.height), "config": cfg.as_dict(),
                      "camera": {"cam_pos": list(cam.cam_pos), "fwd": list(cam.fwd), "rgt": list(cam.rgt),
                                 "up": list(cam.up), "fov_scale": cam.fov_scale}}
        if name == "t1":
            rng = np.random.default_rng(3)
            u = np.concatenate([rng.random(4000), np.linspace(-0.01, 1.01, 2001)]).astype(np.float32)
            us = torch.from_numpy(u).cuda()
            o1 = torch.zeros(len(u), device="cuda")
            o4 = torch.zeros((len(u), 4), device="cuda")
            ref.tex_probe("disk", us.data_ptr(), o1.data_ptr(), len(u))
            ref.tex_probe("bb", us.data_ptr(), o4.data_ptr(), len(u))
            np.savez_compressed(out / "tex_probe_t1.npz", u=u, disk=o1.cpu().numpy(), bb=o4.cpu().numpy(),
                                disk_lut=disk, bb_lut=bb)
        ref.close()
    (out / "golden_meta.json").write_text(json.dumps(meta, indent=1, sort_keys=True))


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).resolve().parent)
