// kt_tune.cpp — launch-shape autotuner of the trace (kt_context_autotune), host C++ and CUDA
// events only, so that any host of the C ABI (a Rust CudaRenderer included) can tune.
//
// The per-ray work of a frame depends on the scene: its spread, and the share of rays that
// freeze, shade the disk or escape.  The best launch shape therefore differs per scene.  The
// candidates are
//   plain      one thread per pixel; the hardware block scheduler balances blocks (block
//              shape; 128-thread blocks may ask for more resident blocks per SM, which caps
//              registers per thread)
//   wavefront  persistent blocks of 128 threads; lanes are refilled from a device work counter
//              once `refill_min` lanes of a warp are idle (resident blocks per SM, refill)
// each in tile order and in long-rays-first order.  Every candidate must reproduce the first
// candidate's image bit for bit (they run the same per-ray arithmetic; a device kernel counts
// differing pixels).  Each is timed with CUDA events on the caller's stream, `reps` launches
// after one warm-up launch, and scored by the median; the fastest identical one is installed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <vector>

#include "../../include/kerrtrace.h"
#include "kt_context.h"
#include "kt_internal.h"

namespace {

kt_status tune_fail(cudaError_t e, const char* what) {
    char msg[256];
    snprintf(msg, sizeof msg, "autotune: %s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
    return ktd::set_error(KT_ERR_CUDA, msg);
}

kt_tuning make(int schedule, int bx, int by, int bps, int refill, int order, int keep_frozen) {
    kt_tuning t;
    t.schedule = schedule;
    t.block_x = bx;
    t.block_y = by;
    t.blocks_per_sm = bps;
    t.refill_min = refill;
    t.order = order;
    t.keep_frozen = keep_frozen;
    return t;
}

// The candidate list (kt_context_autotune with candidates == NULL).
std::vector<kt_tuning> default_candidates(int precision, int mode, int keep_frozen) {
    static const int kPlain[][2] = {{16, 16}, {32, 8}, {8, 8}, {16, 8}, {32, 4}, {8, 16}};
    static const int kPlain128[][2] = {{16, 8}, {8, 16}, {32, 4}};
    static const int kRefill[] = {1, 4, 8, 16};
    std::vector<kt_tuning> out;
    for (int order : {KT_ORDER_TILES, KT_ORDER_LONG_FIRST}) {
        for (const auto& b : kPlain) out.push_back(make(KT_SCHED_PLAIN, b[0], b[1], 4, 1, order, keep_frozen));
        // 128-thread blocks with more resident per SM: 5 or 6 (FP32, mixed), 3 or 4 (FP64)
        for (const auto& b : kPlain128)
            for (int bps : (precision == KT_PREC_FP64 ? std::vector<int>{3, 4} : std::vector<int>{5, 6}))
                out.push_back(make(KT_SCHED_PLAIN, b[0], b[1], bps, 1, order, keep_frozen));
        // only the FP32 reference-semantics wavefront kernel has the 3/5/6 blocks-per-SM variants
        const std::vector<int> bps = (precision == KT_PREC_FP32 && mode == KT_MODE_REF) ? std::vector<int>{3, 4, 5, 6}
                                                                                       : std::vector<int>{4};
        for (int b : bps)
            for (int r : kRefill) out.push_back(make(KT_SCHED_WAVEFRONT, 0, 0, b, r, order, keep_frozen));
    }
    return out;
}

// Device buffers of one tuning run, released on every path.
struct Scratch {
    float* hdr = nullptr;
    float* base = nullptr;
    uint32_t* err = nullptr;
    unsigned long long* diff = nullptr;
    std::vector<cudaEvent_t> ev;
    ~Scratch() {
        cudaFree(hdr);
        cudaFree(base);
        cudaFree(err);
        cudaFree(diff);
        for (cudaEvent_t e : ev)
            if (e) cudaEventDestroy(e);
    }
};

}  // namespace

extern "C" kt_status kt_context_autotune(kt_context* ctx, void* stream, const kt_camera* cam, uint32_t reps,
                                         const kt_tuning* candidates, uint32_t n_candidates, kt_tune_entry* table,
                                         uint32_t* n_entries) {
    using ktd::set_error;
    if (!ctx || !cam) return set_error(KT_ERR_INVALID_ARG, "kt_context_autotune: NULL argument");
    if (reps == 0 || reps > 64) return set_error(KT_ERR_INVALID_ARG, "kt_context_autotune: reps must be in 1..64");
    if (candidates && (n_candidates == 0 || n_candidates > KT_TUNE_MAX_CANDIDATES))
        return set_error(KT_ERR_INVALID_ARG, "kt_context_autotune: n_candidates must be in 1..KT_TUNE_MAX_CANDIDATES");
    kt_tuning saved;
    kt_status st = kt_context_get_tuning(ctx, &saved);
    if (st != KT_OK) return st;
    const std::vector<kt_tuning> cands =
        candidates ? std::vector<kt_tuning>(candidates, candidates + n_candidates)
                   : default_candidates(ctx->cfg.precision, ctx->cfg.mode, saved.keep_frozen);
    if (cands.size() > KT_TUNE_MAX_CANDIDATES)
        return set_error(KT_ERR_INVALID_ARG, "kt_context_autotune: candidate list longer than KT_TUNE_MAX_CANDIDATES");

    int prev_dev = 0;
    cudaGetDevice(&prev_dev);
    if (prev_dev != ctx->device) cudaSetDevice(ctx->device);
    struct Restore {
        int dev, prev;
        ~Restore() {
            if (dev != prev) cudaSetDevice(prev);
        }
    } restore{ctx->device, prev_dev};

    // any failure below puts the caller's tuning back
    struct KeepTuning {
        kt_context* ctx;
        kt_tuning saved;
        bool done = false;
        ~KeepTuning() {
            if (!done) kt_context_set_tuning(ctx, &saved);
        }
    } keep{ctx, saved};
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t px = (size_t)ctx->cfg.width * ctx->cfg.height;
    Scratch sc;
    sc.ev.assign(2 * reps, nullptr);
    cudaError_t e;
    if ((e = cudaMalloc(&sc.hdr, px * 4 * sizeof(float))) != cudaSuccess ||
        (e = cudaMalloc(&sc.base, px * 4 * sizeof(float))) != cudaSuccess ||
        (e = cudaMalloc(&sc.err, 2 * sizeof(uint32_t))) != cudaSuccess ||
        (e = cudaMalloc(&sc.diff, sizeof(unsigned long long))) != cudaSuccess)
        return tune_fail(e, "allocate scratch");
    for (cudaEvent_t& ev : sc.ev)
        if ((e = cudaEventCreate(&ev)) != cudaSuccess) return tune_fail(e, "create events");

    std::vector<kt_tune_entry> rows;
    rows.reserve(cands.size());
    for (size_t i = 0; i < cands.size(); ++i) {
        if ((st = kt_context_set_tuning(ctx, &cands[i])) != KT_OK) return st;
        if ((e = cudaMemsetAsync(sc.err, 0, 2 * sizeof(uint32_t), s)) != cudaSuccess) return tune_fail(e, "clear error word");
        if ((st = kt_trace(ctx, stream, cam, KT_SCHED_AUTO, sc.hdr, sc.err)) != KT_OK) return st;
        unsigned long long diff = 0;
        if (i == 0) {
            if ((e = cudaMemcpyAsync(sc.base, sc.hdr, px * 4 * sizeof(float), cudaMemcpyDeviceToDevice, s)) != cudaSuccess)
                return tune_fail(e, "keep the first image");
        } else {
            if ((e = ktd::launch_count_mismatch(sc.hdr, sc.base, px, sc.diff, s)) != cudaSuccess ||
                (e = cudaMemcpyAsync(&diff, sc.diff, sizeof diff, cudaMemcpyDeviceToHost, s)) != cudaSuccess)
                return tune_fail(e, "compare images");
        }
        for (uint32_t r = 0; r < reps; ++r) {
            if ((e = cudaEventRecord(sc.ev[2 * r], s)) != cudaSuccess) return tune_fail(e, "record event");
            if ((st = kt_trace(ctx, stream, cam, KT_SCHED_AUTO, sc.hdr, sc.err)) != KT_OK) return st;
            if ((e = cudaEventRecord(sc.ev[2 * r + 1], s)) != cudaSuccess) return tune_fail(e, "record event");
        }
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return tune_fail(e, "synchronise");
        std::vector<float> ms(reps);
        for (uint32_t r = 0; r < reps; ++r)
            if ((e = cudaEventElapsedTime(&ms[r], sc.ev[2 * r], sc.ev[2 * r + 1])) != cudaSuccess)
                return tune_fail(e, "read event time");
        std::sort(ms.begin(), ms.end());
        kt_tune_entry row;
        row.tuning = cands[i];
        row.ms = ms[reps / 2];
        row.identical = diff == 0 ? 1 : 0;
        rows.push_back(row);
    }
    size_t best = rows.size();
    for (size_t i = 0; i < rows.size(); ++i)
        if (rows[i].identical && (best == rows.size() || rows[i].ms < rows[best].ms)) best = i;
    // the first candidate is identical to itself, so best is always found
    if ((st = kt_context_set_tuning(ctx, &rows[best].tuning)) != KT_OK) return st;
    keep.done = true;
    if (table)
        for (size_t i = 0; i < rows.size(); ++i) table[i] = rows[i];
    if (n_entries) *n_entries = (uint32_t)rows.size();
    return KT_OK;
}
