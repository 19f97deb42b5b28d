"""Autotuner of the trace launch shape.

The per-ray work of a frame depends on the scene: its spread, and the share of rays that
freeze, shade the disk or escape.  The best launch shape therefore differs per scene. The
candidates are:

  plain      one thread per pixel; the hardware block scheduler balances blocks (block shape)
  wavefront  persistent blocks; lanes are refilled from a device work counter once `refill_min`
             lanes of a warp are idle (resident blocks per SM = register cap, refill threshold)

each in tile order and in long-rays-first order (a rank kernel moves the pixels whose rays are
predicted to wind near a photon orbit to the front, so they do not form the frame's tail).

Every candidate must reproduce the first candidate's image bit for bit (they all run the same
per-ray arithmetic).  The fastest one is installed in the context, and KT_SCHED_AUTO then runs it.
Timing uses CUDA events on the launch stream, median of `reps` launches after a warm-up launch.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import ORDER_LONG_FIRST, ORDER_TILES, SCHED_AUTO, SCHED_PLAIN, SCHED_WAVEFRONT, Context, KtCamera

PLAIN_BLOCKS = [(16, 16), (32, 8), (8, 8), (16, 8), (32, 4), (8, 16)]
PLAIN_BLOCKS_128 = [(16, 8), (8, 16), (32, 4)]
WAVE_BLOCKS_PER_SM = [3, 4, 5, 6]
WAVE_REFILL = [1, 4, 8, 16]


def candidates(precision: int = 0, mode: int = 0) -> list[dict]:
    out = []
    for order in (ORDER_TILES, ORDER_LONG_FIRST):
        out += [dict(schedule=SCHED_PLAIN, block_x=bx, block_y=by, blocks_per_sm=4, refill_min=1, order=order)
                for bx, by in PLAIN_BLOCKS]
        # 128-thread blocks with more resident per SM: 5 or 6 (FP32 and mixed), 3 or 4 (FP64)
        out += [dict(schedule=SCHED_PLAIN, block_x=bx, block_y=by, blocks_per_sm=b, refill_min=1, order=order)
                for bx, by in PLAIN_BLOCKS_128 for b in ((3, 4) if precision == 2 else (5, 6))]
        # only the FP32 reference-semantics kernel has the 3/5/6 blocks-per-SM variants
        bps = WAVE_BLOCKS_PER_SM if (precision == 0 and mode == 0) else [4]
        out += [dict(schedule=SCHED_WAVEFRONT, block_x=0, block_y=0, blocks_per_sm=b, refill_min=r, order=order)
                for b in bps for r in WAVE_REFILL]
    return out


@dataclass
class TuneResult:
    best: dict
    best_ms: float
    table: list  # (ms, candidate, bit-identical)

    def summary(self, top: int = 5) -> dict:
        rows = sorted(self.table, key=lambda t: t[0])[:top]
        return {"best": self.best, "best_ms": round(self.best_ms, 4),
                "top": [{"ms": round(ms, 4), **c, "identical": ok} for ms, c, ok in rows],
                "candidates": len(self.table)}


def autotune(ctx: Context, cam: KtCamera, reps: int = 3, cands: list[dict] | None = None,
             stream: int = 0) -> TuneResult:
    import torch

    cfg = ctx.cfg
    n = cfg.width * cfg.height
    hdr = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    err = torch.zeros(2, dtype=torch.int32, device="cuda")
    cands = cands if cands is not None else candidates(cfg.precision, cfg.mode)
    table = []
    base = None
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
    for cand in cands:
        ctx.set_tuning(**cand)
        err.zero_()
        ctx.trace(cam, hdr.data_ptr(), err.data_ptr(), stream, SCHED_AUTO)
        torch.cuda.synchronize()
        out = hdr.cpu().numpy().view(np.uint32)
        if base is None:
            base = out.copy()
        same = bool(np.array_equal(out, base))
        times = []
        for e0, e1 in ev:
            e0.record()
            ctx.trace(cam, hdr.data_ptr(), err.data_ptr(), stream, SCHED_AUTO)
            e1.record()
        torch.cuda.synchronize()
        times = sorted(a.elapsed_time(b) for a, b in ev)
        table.append((times[len(times) // 2], cand, same))
    ok = [t for t in table if t[2]]
    ms, best, _ = min(ok, key=lambda t: t[0])
    ctx.set_tuning(**best)
    return TuneResult(best=best, best_ms=ms, table=table)
