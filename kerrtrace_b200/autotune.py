"""Launch-shape autotuner of the trace: a thin caller of the library's kt_context_autotune.

The tuner itself is C++ (kerrtrace_b200/csrc/kt_tune.cpp), so that any host of the C ABI can
run it.  It times the trace of one view under each candidate launch shape (plain block shapes,
128-thread plain blocks with more resident blocks per SM, persistent wavefront blocks per SM x
refill thresholds, each in tile and long-rays-first order) with CUDA events, keeps only the
candidates whose image is bit for bit the first candidate's, and installs the fastest of those
in the context; KT_SCHED_AUTO then runs it.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

from . import TUNE_MAX_CANDIDATES, Context, KtCamera, KtTuneEntry, KtTuning, check, lib


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
    """Tunes `ctx` for the view `cam` on `stream`; `cands` (dicts of kt_tuning fields) replaces
    the built-in candidate list."""
    n_max = TUNE_MAX_CANDIDATES if cands is None else len(cands)
    table = (KtTuneEntry * n_max)()
    n = C.c_uint32(0)
    if cands is None:
        check(lib().kt_context_autotune(ctx.handle, C.c_void_p(stream), C.byref(cam), reps, None, 0, table,
                                        C.byref(n)))
    else:
        arr = (KtTuning * len(cands))(*[KtTuning(**c) for c in cands])
        check(lib().kt_context_autotune(ctx.handle, C.c_void_p(stream), C.byref(cam), reps, arr, len(cands), table,
                                        C.byref(n)))
    rows = [(float(table[i].ms), table[i].tuning.as_dict(), bool(table[i].identical)) for i in range(n.value)]
    best = ctx.tuning().as_dict()
    best_ms = min(ms for ms, c, ok in rows if ok and c == best)
    return TuneResult(best=best, best_ms=best_ms, table=rows)
