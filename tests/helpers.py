"""Helpers shared by the GPU parity tests: run the product, the reference kernel (oracle/_ref)
and the CPU oracle on the same scene, and compare images the way the parity bar states it."""
from __future__ import annotations

import numpy as np

import kerrtrace_b200 as kt


def run_ours(torch, cfg, cam, schedule=kt.SCHED_WAVEFRONT, counted=False, ctx=None):
    ctx = ctx or kt.Context(cfg)
    n = cfg.width * cfg.height
    hdr = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    err = torch.zeros(2, dtype=torch.int32, device="cuda")
    stats = None
    if counted:
        stats = ctx.trace_counted(cam, hdr.data_ptr(), err.data_ptr(), 0, schedule)
    else:
        ctx.trace(cam, hdr.data_ptr(), err.data_ptr(), 0, schedule)
    torch.cuda.synchronize()
    return hdr.cpu().numpy(), err.cpu().numpy().view(np.uint32), stats, ctx


def run_ref(torch, scene: str, cfg, cam):
    """The reference's trace_kernel on the same inputs (defines of `scene`, runtime cfg/cam).
    Its KerrParams and LUTs come from the oracle's restatement of the reference host, not from
    the product, so a bit-identical image also pins the product's host tables."""
    import oracle
    p, bb, disk = oracle.reference_inputs(cfg)
    ref = oracle.RefKernel(scene)
    ref.setup(p, bb, disk)
    n = cfg.width * cfg.height
    hdr = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    err = torch.zeros(2, dtype=torch.int32, device="cuda")
    ref.trace(hdr.data_ptr(), cfg, cam, cfg.lut_max_temp, err.data_ptr(), p.disk_inner)
    torch.cuda.synchronize()
    out = hdr.cpu().numpy(), err.cpu().numpy().view(np.uint32)
    ref.close()
    return out


def pixel_class(rgb: np.ndarray) -> np.ndarray:
    """0 black, 1 grey (sky grid only), 2 coloured (disk emission)."""
    r, g, b = rgb[..., 0], rgb[..., 1], rgb[..., 2]
    black = (r == 0) & (g == 0) & (b == 0)
    grey = (r == g) & (g == b) & ~black
    return np.where(black, 0, np.where(grey, 1, 2))


def edge_mask(cls: np.ndarray, w: int, h: int) -> np.ndarray:
    """Pixels whose 3x3 neighbourhood holds more than one class (silhouettes of the shadow,
    disk edges, sky lines)."""
    c = cls.reshape(h, w)
    pad = np.pad(c, 1, mode="edge")
    edge = np.zeros_like(c, dtype=bool)
    for dy in (-1, 0, 1):
        for dx in (-1, 0, 1):
            edge |= pad[1 + dy:1 + dy + h, 1 + dx:1 + dx + w] != c
    return edge.reshape(-1)


def compare_hdr(ours: np.ndarray, ref: np.ndarray, w: int, h: int, rtol: float = 1e-3):
    """Returns a dict: exact-equal fraction, class mismatches outside edges, the fraction of
    pixels beyond rtol (relative per channel, floor 1e-6 x image max) outside edges, edge count."""
    a, b = ours[:, :3].astype(np.float64), ref[:, :3].astype(np.float64)
    fin = np.isfinite(a).all(1) & np.isfinite(b).all(1)
    floor = 1e-6 * max(np.abs(b[fin]).max(initial=0.0), 1e-30)
    rel = np.where(fin[:, None], np.abs(a - b) / np.maximum(np.abs(b), floor), np.where(np.isnan(a) == np.isnan(b), 0, np.inf))
    rel_px = rel.max(1)
    ca, cb = pixel_class(ours[:, :3]), pixel_class(ref[:, :3])
    edge = edge_mask(cb, w, h) | edge_mask(ca, w, h)
    inner = ~edge
    return {
        "n": len(a),
        "bit_equal": float(np.mean(np.all(ours.view(np.uint32) == ref.view(np.uint32), axis=1))),
        "class_mismatch_inner": int(np.sum((ca != cb) & inner)),
        "over_tol_inner": int(np.sum((rel_px > rtol) & inner)),
        "over_tol_all": int(np.sum(rel_px > rtol)),
        "edge": int(edge.sum()),
        "max_rel_inner": float(rel_px[inner].max(initial=0.0)),
        "p99_rel": float(np.quantile(rel_px, 0.99)),
    }


def sky_flip(a: np.ndarray, b: np.ndarray, sky_unit: float) -> np.ndarray:
    """Pixels whose difference is a grey offset (equal in the three channels) of visible size:
    a sky-grid line seen by one trajectory and not the other."""
    d = a - b
    grey = (np.abs(d[:, 0] - d[:, 1]) <= 1e-3 * np.abs(d[:, 0]) + 1e-9) & \
           (np.abs(d[:, 1] - d[:, 2]) <= 1e-3 * np.abs(d[:, 1]) + 1e-9)
    return grey & (np.abs(d[:, 0]) > 1e-4 * sky_unit)


def oracle_parity(ours: np.ndarray, exp: np.ndarray, cfg) -> dict:
    """Comparison of two independent solutions of the same adaptive scheme (GPU vs CPU oracle):
    edges are class silhouettes and sky-grid line flips; very dim pixels (below 1e-4 of the image
    maximum, where 8-bit texture weights cross a steep Planck curve) are reported separately."""
    a = ours[:, :3].astype(np.float64)
    ref = exp[:, :3].astype(np.float64)
    floor = 1e-6 * max(np.abs(ref).max(), 1e-30)
    rel = (np.abs(a - ref) / np.maximum(np.abs(ref), floor)).max(1)
    cls_r, cls_o = pixel_class(ref), pixel_class(a)
    edge = edge_mask(cls_r, cfg.width, cfg.height) | edge_mask(cls_o, cfg.width, cfg.height)
    sky_unit = float(np.float32(cfg.sky_intensity) * np.float32(cfg.exposure_scale))
    edge |= sky_flip(a, ref, sky_unit)
    dim = np.abs(ref).max(1) < 1e-4 * np.abs(ref).max()
    inner = ~edge & ~dim
    return {"n": len(ref), "class_mismatch": int(np.sum((cls_r != cls_o) & ~edge)),
            "over_1e-3": int(np.sum((rel > 1e-3) & inner)), "close_1e-4": float(np.mean(rel[inner] <= 1e-4)),
            "p99": float(np.quantile(rel[inner], 0.99)), "max": float(rel[inner].max(initial=0.0)),
            "edge": int(edge.sum()), "dim": int(dim.sum())}
