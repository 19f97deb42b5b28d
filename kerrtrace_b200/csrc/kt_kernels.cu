// kt_kernels.cu — trace and post-process kernels for sm_100a.
//
// Built with -use_fast_math, the flag set the reference compiles kernel.cu with
// (config.yaml `cuda.use_fast_math: true`, src/renderer/init.rs:112-118), so that `/`, powf and
// expf lower to the same instructions as in the reference.
//
// Trace kernels (replace trace_kernel, cuda/kernel.cu:88-142):
//   trace_plain_kernel      one thread per pixel on a 2D grid of block_dim tiles; each thread
//                           runs its spp rays to completion through the attempt state machine.
//   trace_wavefront_kernel  persistent: one block per resident slot, each lane owns a pixel and
//                           pulls a new one from a device work counter (warp-aggregated atomics)
//                           as soon as its rays are done, so long rays never idle a whole warp.
// Post kernels (replace bloom_horizontal / post_process, cuda/kernel.cu:144-251):
//   bloom_h_kernel          horizontal normalised Gaussian, register-blocked over staged rows
//   post_v_kernel           vertical Gaussian streamed from the bloom buffer + composite, ACES,
//                           sRGB OETF, 0x00RRGGBB pack
//   post_vt_kernel          the same over the column-major bloom buffer of the fused post
//   tonemap_kernel          tone map alone (bloom inactive)
// kt_post_fused runs both passes over a bloom buffer that the context owns, stored column-major
// between them: bloom_h_kernel<true> writes it, post_vt_kernel stages its columns like rows.  The post kernels
// produce the reference's bits: same tap order, weights, division and tone-map expressions.
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "kt_internal.h"
#include "kt_ray.cuh"

namespace ktd {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kWavefrontBlock = 128;

// ---- work counters (counting kernels only) -----------------------------------------------
__device__ __forceinline__ void add_tally(unsigned long long* ctr, uint64_t rays, const Tally& t) {
    atomicAdd(ctr + 0, (unsigned long long)rays);
    atomicAdd(ctr + 1, (unsigned long long)t.steps);
    atomicAdd(ctr + 2, (unsigned long long)t.attempts);
    atomicAdd(ctr + 3, (unsigned long long)t.rhs);
    atomicAdd(ctr + 4, (unsigned long long)t.frozen);
    atomicAdd(ctr + 5, (unsigned long long)t.fp64);
}
__device__ __forceinline__ void tally_ray(Tally& acc, const Tally& ray) {
    acc.steps += ray.steps;
    acc.attempts += ray.attempts;
    acc.rhs += ray.rhs;
    acc.frozen += ray.frozen ? 1u : 0u;
    acc.fp64 += ray.fp64;
}
// First shaded disk hit of sample 0 of a pixel (counting kernels, when aux is given).
__device__ __forceinline__ void write_aux(float4* aux, size_t idx, const Tally& t) {
    if (aux) aux[idx] = make_float4(t.first_r, t.first_g, t.first_T, (float)t.hits);
}

// Runs one ray to completion (plain schedule).
template <class R, int MODE, bool COUNT>
__device__ __forceinline__ void run_ray(int px, int py, int smp, const Scene& sc, const Camera& cam,
                                        uint32_t* err, float acc[3], Tally& total, float4* aux) {
    float dir[3];
    pixel_ray<MODE>(px, py, smp, sc, cam, dir);
    RayRun<R> ry;
    Tally tl;
    tl.clear();
    if (start(ry, cam, dir, sc)) {
        while (!advance<MODE, COUNT>(ry, sc, err, tl)) {
        }
    }
    acc[0] += ry.col[0];
    acc[1] += ry.col[1];
    acc[2] += ry.col[2];
    if (COUNT) {
        tally_ray(total, tl);
        if (smp == 0) write_aux(aux, (size_t)py * sc.width + px, tl);
    }
}

// Work unit -> pixel.  Units run over 16-row bands, 16-column tiles inside a band, row-major
// inside a tile, so 32 consecutive units form a 16x2 patch (the footprint of one warp of the
// reference's 16x16 blocks).  Exact bijection onto [0, W) x [0, H), partial tiles included.
__device__ __forceinline__ void unit_to_pixel(unsigned u, int W, int H, int& px, int& py) {
    const unsigned band_px = (unsigned)W * 16u;
    const unsigned band = u / band_px;
    const unsigned rem = u - band * band_px;
    const int row0 = (int)band * 16;
    const int hb = min(16, H - row0);
    const unsigned tile_px = 16u * (unsigned)hb;
    const unsigned tile = rem / tile_px;
    const unsigned rem2 = rem - tile * tile_px;
    const int col0 = (int)tile * 16;
    const int wt = min(16, W - col0);
    py = row0 + (int)(rem2 / (unsigned)wt);
    px = col0 + (int)(rem2 % (unsigned)wt);
}

// ---- long-rays-first pixel order -----------------------------------------------------------
// A ray that passes close to a spherical photon orbit winds around the hole about ln(1/delta)
// times before it falls in or escapes, and takes several times the average step count.  Traced
// last, such rays leave single latency-bound warps running after the rest of the frame is done.
// The Kerr constants of motion of the initial state (E = -p_t, the angular momentum about the
// spin axis L = z p_x - x p_z, the Carter constant Q, with p_theta from the spheroidal
// coordinates of the Kerr-Schild point) fix the radial potential
//   R(r) = (E (r^2 + a^2) - a L)^2 - (r^2 - 2 M r + a^2) ((L - a E)^2 + Q),
// whose local minimum outside the horizon is close to 0 exactly for those rays.  The rank kernel
// marks pixels with |R(r_min)| < kHotThreshold E^2 r_min^4 (0.2% to 4% of a frame) and writes
// a permutation of the pixels: the marked ones first, then the rest in tile order.  The tracers
// read it when the tuning's order is 1.  Per-pixel results do not depend on the order.
constexpr float kHotThreshold = 0.1f;

__device__ __forceinline__ bool predicted_long(const Scene& sc, const Camera& cam, const float dir[3]) {
    RayRun<float> ry;
    ray_start<float>(ry, cam, dir, sc);
    const float a = sc.a, M = sc.M;
    const float x = ry.s[0], y = ry.s[1], z = ry.s[2];
    const float px = ry.s[3], py = ry.s[4], pz = ry.s[5];
    const float E = -ry.pt, E2 = E * E;
    const float L = z * px - x * pz;
    const float r = ks_radius<float>(x, y, z, sc.aa);
    const float ct = __fdividef(y, r);
    const float st2 = fmaxf(1.0f - ct * ct, 1e-12f);
    const float st = sqrtf(st2);
    const float pth = __fdividef(ct, st) * (x * px + z * pz) - r * st * py;
    const float Q = pth * pth + ct * ct * (__fdividef(L * L, st2) - a * a * E2);
    const float K = (L - a * E) * (L - a * E) + Q;
    const float B = a * (a * E - L);
    const float c2 = 2.0f * E * B - K;
    // Newton on R'(r) = 4 E^2 r^3 + 2 c2 r + 2 M K from the right of its largest root, where R'
    // is increasing and convex: the iterates decrease monotonically onto the root
    float rr = fmaxf(5.0f * M, sqrtf(__fdividef(fabsf(K), E2)));
#pragma unroll 1
    for (int it = 0; it < 16; ++it) {
        const float d1 = 4.0f * E2 * rr * rr * rr + 2.0f * c2 * rr + 2.0f * M * K;
        const float d2 = 12.0f * E2 * rr * rr + 2.0f * c2;
        if (!(d2 > 0.0f)) break;
        rr -= __fdividef(d1, d2);
    }
    const float r2 = rr * rr, r4 = r2 * r2;
    const float Rm = E2 * r4 + c2 * r2 + 2.0f * M * K * rr + B * B - a * a * K;
    return rr > sc.rh && fabsf(Rm) < kHotThreshold * E2 * r4;
}

// order[0], order[1]: marked / unmarked pixel counts; order[kOrderHeader + i]: pixel index
// py * width + px of work unit i.  Units are written in warp-sized runs (a 16x2 patch of the
// tile order, compacted): marked runs from the front, unmarked runs from the back.
__device__ __forceinline__ void ordered_pixel(unsigned u, unsigned n, const unsigned* order, unsigned n_hot,
                                              int W, int& px, int& py) {
    const unsigned* list = order + kOrderHeader;
    const unsigned idx = u < n_hot ? list[u] : list[n - 1u - (u - n_hot)];
    py = (int)(idx / (unsigned)W);
    px = (int)(idx - (unsigned)py * (unsigned)W);
}

template <int MODE>
__global__ void __launch_bounds__(256) rank_pixels_kernel(const Scene sc, const Camera cam,
                                                          unsigned* __restrict__ order) {
    const unsigned n = (unsigned)sc.width * (unsigned)sc.height;
    const unsigned u = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const bool valid = u < n;
    bool hot = false;
    unsigned idx = 0;
    if (valid) {
        int px, py;
        unit_to_pixel(u, sc.width, sc.height, px, py);
        idx = (unsigned)py * (unsigned)sc.width + (unsigned)px;
        float dir[3];
        pixel_ray<MODE>(px, py, 0, sc, cam, dir);
        hot = predicted_long(sc, cam, dir);
    }
    const unsigned hm = __ballot_sync(kFull, valid && hot);
    const unsigned cm = __ballot_sync(kFull, valid && !hot);
    unsigned hb = 0, cb = 0;
    if (lane == 0) {
        if (hm) hb = atomicAdd(order + 0, (unsigned)__popc(hm));
        if (cm) cb = atomicAdd(order + 1, (unsigned)__popc(cm));
    }
    hb = __shfl_sync(kFull, hb, 0);
    cb = __shfl_sync(kFull, cb, 0);
    const unsigned lt = (1u << lane) - 1u;
    unsigned* list = order + kOrderHeader;
    if (valid) {
        if (hot)
            list[hb + (unsigned)__popc(hm & lt)] = idx;
        else
            list[n - 1u - (cb + (unsigned)__popc(cm & lt))] = idx;
    }
}

// Resident 256-thread blocks per SM asked of the compiler for the plain kernel: two for the
// FP32 and mixed paths (at most 128 registers per thread, 16 warps per SM), one for FP64.
// Blocks of at most 128 threads can also ask for 5 or 6 resident blocks (at most 102 or 85
// registers: 20 or 24 warps per SM), a choice of the tuning (blocks_per_sm) for FP32 and mixed,
// and FP64 for 3 or 4 (at most 170 or 128 registers, with some spills: 12 or 16 warps per SM
// instead of 8).
template <class R> struct PlainMinBlocks { static constexpr int v = 2; };
template <> struct PlainMinBlocks<double> { static constexpr int v = 1; };

template <class R, int MODE, bool COUNT, int MAXT, int MINB = (MAXT == 256 ? PlainMinBlocks<R>::v : 1)>
__global__ void __launch_bounds__(MAXT, MINB)
    trace_plain_kernel(const __grid_constant__ Scene sc, const Camera cam,
                                                           float4* __restrict__ hdr,
                                                           uint32_t* __restrict__ err,
                                                           unsigned long long* __restrict__ ctr,
                                                           float4* __restrict__ aux,
                                                           const unsigned* __restrict__ order) {
    int px, py;
    if (order) {  // 1D launch over the ranked work units
        const unsigned n = (unsigned)sc.width * (unsigned)sc.height;
        const unsigned u = blockIdx.x * (blockDim.x * blockDim.y) + threadIdx.y * blockDim.x + threadIdx.x;
        if (u >= n) return;
        ordered_pixel(u, n, order, order[0], sc.width, px, py);
    } else {
        px = blockIdx.x * blockDim.x + threadIdx.x;
        py = blockIdx.y * blockDim.y + threadIdx.y;
        if (px >= sc.width || py >= sc.height) return;
    }
    float acc[3] = {0.0f, 0.0f, 0.0f};
    const int pix = py * sc.width + px;
    if (sc.accum && sc.sample_first > 0) {  // progressive: continue the running sum
        const float4 a = sc.accum[pix];
        acc[0] = a.x;
        acc[1] = a.y;
        acc[2] = a.z;
    }
    Tally total;
    total.clear();
    const int s_end = sc.sample_first + sc.spp;
    for (int smp = sc.sample_first; smp < s_end; ++smp) run_ray<R, MODE, COUNT>(px, py, smp, sc, cam, err, acc, total, aux);
    if (sc.accum) sc.accum[pix] = make_float4(acc[0], acc[1], acc[2], (float)s_end);
    const float fs = sc.final_scale;
    hdr[pix] = make_float4(acc[0] * fs, acc[1] * fs, acc[2] * fs, 1.0f);
    if (COUNT) add_tally(ctr, (uint64_t)sc.spp, total);
}

// Persistent wavefront tracer.  A lane whose pixel is done takes a new one from the work
// counter; lanes are refilled together once at least `refill_min` of the warp's lanes are idle
// (or when the warp has nothing else to do), which trades idle lanes against how often the
// divergent start-up code runs.
template <class R, int MODE, bool COUNT, int MINB>
__global__ void __launch_bounds__(kWavefrontBlock, MINB)
    trace_wavefront_kernel(const __grid_constant__ Scene sc, const Camera cam, float4* __restrict__ hdr,
                           uint32_t* __restrict__ err, unsigned* __restrict__ queue,
                           unsigned long long* __restrict__ ctr, float4* __restrict__ aux,
                           int refill_min, const unsigned* __restrict__ order) {
    const int lane = threadIdx.x & 31;
    const unsigned lane_lt = (1u << lane) - 1u;
    const unsigned n_units = (unsigned)sc.width * (unsigned)sc.height;
    const unsigned n_hot = order ? order[0] : 0u;
    RayRun<R> ry;
    int px = 0, py = 0, smp = 0;
    float acc[3] = {0.0f, 0.0f, 0.0f};
    bool active = false;
    bool open = true;
    Tally tl, total;
    tl.clear();
    total.clear();
    uint64_t rays = 0;

    while (true) {
        if (open) {
            const unsigned need = __ballot_sync(kFull, !active);
            const int idle = __popc(need);
            if (idle >= refill_min || (idle > 0 && idle == 32)) {
                const int leader = __ffs(need) - 1;
                const unsigned cnt = (unsigned)idle;
                unsigned base = 0;
                if (lane == leader) base = atomicAdd(queue, cnt);
                base = __shfl_sync(kFull, base, leader);
                if (base + cnt >= n_units) open = false;
                if (!active) {
                    const unsigned u = base + (unsigned)__popc(need & lane_lt);
                    if (u < n_units) {
                        if (order)
                            ordered_pixel(u, n_units, order, n_hot, sc.width, px, py);
                        else
                            unit_to_pixel(u, sc.width, sc.height, px, py);
                        acc[0] = acc[1] = acc[2] = 0.0f;
                        // first sample with work; samples whose loop would not run add zero
                        for (smp = 0; smp < sc.spp; ++smp) {
                            float dir[3];
                            pixel_ray<MODE>(px, py, smp, sc, cam, dir);
                            if (COUNT) tl.clear();
                            if (start(ry, cam, dir, sc)) break;
                        }
                        if (smp < sc.spp) {
                            active = true;
                        } else {
                            const float fs = sc.final_scale;
                            hdr[py * sc.width + px] =
                                make_float4(acc[0] * fs, acc[1] * fs, acc[2] * fs, 1.0f);
                            if (COUNT) rays += (uint64_t)sc.spp;
                        }
                    }
                }
            }
        }
        if (!__any_sync(kFull, active)) {
            if (!open) break;
            continue;
        }
        if (active && advance<MODE, COUNT>(ry, sc, err, tl)) {
            acc[0] += ry.col[0];
            acc[1] += ry.col[1];
            acc[2] += ry.col[2];
            if (COUNT) {
                tally_ray(total, tl);
                if (smp == 0) write_aux(aux, (size_t)py * sc.width + px, tl);
            }
            for (++smp; smp < sc.spp; ++smp) {
                float dir[3];
                pixel_ray<MODE>(px, py, smp, sc, cam, dir);
                if (COUNT) tl.clear();
                if (start(ry, cam, dir, sc)) break;
            }
            if (smp >= sc.spp) {
                const float fs = sc.final_scale;
                hdr[py * sc.width + px] = make_float4(acc[0] * fs, acc[1] * fs, acc[2] * fs, 1.0f);
                if (COUNT) rays += (uint64_t)sc.spp;
                active = false;
            }
        }
    }
    if (COUNT) add_tally(ctr, rays, total);
}

// ---- launch -------------------------------------------------------------------------------
// Resident blocks per SM requested from the compiler (which caps registers per thread at
// 65536 / (128 * MINB)): the default per arithmetic type, and the variants the autotuner may
// pick for the FP32 reference-semantics kernel.
template <class R> struct WaveDefaults { static constexpr int minb = 4; };
template <> struct WaveDefaults<double> { static constexpr int minb = 2; };
template <> struct WaveDefaults<Mixed> { static constexpr int minb = 4; };

template <class R, int MODE, bool COUNT>
static cudaError_t launch_plain(const Scene& sc, const Camera& cam, float4* hdr, uint32_t* err,
                                unsigned long long* ctr, float4* aux, int bx, int by, int minb,
                                const unsigned* order, cudaStream_t st) {
    const dim3 block(bx, by);
    const unsigned n = (unsigned)sc.width * (unsigned)sc.height, per = (unsigned)(bx * by);
    const dim3 grid = order ? dim3((n + per - 1) / per)
                            : dim3((sc.width + bx - 1) / bx, (sc.height + by - 1) / by);
    if constexpr (std::is_same<R, double>::value) {
        if (bx * by <= 128 && minb == 3) {
            trace_plain_kernel<R, MODE, COUNT, 128, 3><<<grid, block, 0, st>>>(sc, cam, hdr, err, ctr, aux, order);
            return cudaGetLastError();
        }
        if (bx * by <= 128 && minb == 4) {
            trace_plain_kernel<R, MODE, COUNT, 128, 4><<<grid, block, 0, st>>>(sc, cam, hdr, err, ctr, aux, order);
            return cudaGetLastError();
        }
    } else {
        if (bx * by <= 128 && minb == 5) {
            trace_plain_kernel<R, MODE, COUNT, 128, 5><<<grid, block, 0, st>>>(sc, cam, hdr, err, ctr, aux, order);
            return cudaGetLastError();
        }
        if (bx * by <= 128 && minb == 6) {
            trace_plain_kernel<R, MODE, COUNT, 128, 6><<<grid, block, 0, st>>>(sc, cam, hdr, err, ctr, aux, order);
            return cudaGetLastError();
        }
    }
    if (bx * by <= 256)
        trace_plain_kernel<R, MODE, COUNT, 256><<<grid, block, 0, st>>>(sc, cam, hdr, err, ctr, aux, order);
    else
        trace_plain_kernel<R, MODE, COUNT, 1024><<<grid, block, 0, st>>>(sc, cam, hdr, err, ctr, aux, order);
    return cudaGetLastError();
}

template <class R, int MODE, bool COUNT, int MINB>
static cudaError_t launch_wave_minb(const Scene& sc, const Camera& cam, float4* hdr, uint32_t* err,
                                    unsigned* queue, unsigned long long* ctr, float4* aux, int refill,
                                    const unsigned* order, cudaStream_t st) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trace_wavefront_kernel<R, MODE, COUNT, MINB>,
                                                      kWavefrontBlock, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    e = cudaMemsetAsync(queue, 0, sizeof(unsigned), st);
    if (e != cudaSuccess) return e;
    trace_wavefront_kernel<R, MODE, COUNT, MINB>
        <<<sms * per_sm, kWavefrontBlock, 0, st>>>(sc, cam, hdr, err, queue, ctr, aux, refill, order);
    return cudaGetLastError();
}

template <class R, int MODE, bool COUNT>
static cudaError_t launch_wave(const Scene& sc, const Camera& cam, float4* hdr, uint32_t* err,
                               unsigned* queue, unsigned long long* ctr, float4* aux, const Tuning& tn,
                               const unsigned* order, cudaStream_t st) {
    const int refill = tn.refill_min < 1 ? 1 : (tn.refill_min > 32 ? 32 : tn.refill_min);
    if constexpr (std::is_same<R, float>::value && MODE == 0 && !COUNT) {
        switch (tn.blocks_per_sm) {
            case 3: return launch_wave_minb<R, MODE, COUNT, 3>(sc, cam, hdr, err, queue, ctr, aux, refill, order, st);
            case 5: return launch_wave_minb<R, MODE, COUNT, 5>(sc, cam, hdr, err, queue, ctr, aux, refill, order, st);
            case 6: return launch_wave_minb<R, MODE, COUNT, 6>(sc, cam, hdr, err, queue, ctr, aux, refill, order, st);
            default: break;
        }
    }
    return launch_wave_minb<R, MODE, COUNT, WaveDefaults<R>::minb>(sc, cam, hdr, err, queue, ctr, aux, refill, order, st);
}

template <class R, int MODE>
static cudaError_t launch_typed(const Scene& sc, const Camera& cam, int schedule, float4* hdr,
                                uint32_t* err, unsigned* queue, unsigned long long* ctr, float4* aux,
                                const Tuning& tn, int bx, int by, unsigned* order, cudaStream_t st) {
    if (order) {
        const unsigned n = (unsigned)sc.width * (unsigned)sc.height;
        cudaError_t e = cudaMemsetAsync(order, 0, 2 * sizeof(unsigned), st);
        if (e != cudaSuccess) return e;
        rank_pixels_kernel<MODE><<<(n + 255) / 256, 256, 0, st>>>(sc, cam, order);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (schedule == 0)
        return ctr ? launch_plain<R, MODE, true>(sc, cam, hdr, err, ctr, aux, bx, by, tn.blocks_per_sm, order, st)
                   : launch_plain<R, MODE, false>(sc, cam, hdr, err, ctr, aux, bx, by, tn.blocks_per_sm, order, st);
    return ctr ? launch_wave<R, MODE, true>(sc, cam, hdr, err, queue, ctr, aux, tn, order, st)
               : launch_wave<R, MODE, false>(sc, cam, hdr, err, queue, ctr, aux, tn, order, st);
}

cudaError_t launch_trace(const Scene& sc, const Camera& cam, int schedule, float4* hdr,
                         uint32_t* err, unsigned* queue, unsigned long long* ctr, float4* aux,
                         const Tuning& tn, int bx, int by, unsigned* order, cudaStream_t st) {
    if (sc.width <= 0 || sc.height <= 0) return cudaSuccess;
    if (sc.precision == 2) return launch_typed<double, 1>(sc, cam, schedule, hdr, err, queue, ctr, aux, tn, bx, by, order, st);
    if (sc.precision == 1) return launch_typed<Mixed, 1>(sc, cam, schedule, hdr, err, queue, ctr, aux, tn, bx, by, order, st);
    if (sc.mode == 1) return launch_typed<float, 1>(sc, cam, schedule, hdr, err, queue, ctr, aux, tn, bx, by, order, st);
    return launch_typed<float, 0>(sc, cam, schedule, hdr, err, queue, ctr, aux, tn, bx, by, order, st);
}

// ---- batched renders -----------------------------------------------------------------------
template <class R, int MODE, int MAXT>
__global__ void __launch_bounds__(MAXT, MAXT == 256 ? PlainMinBlocks<R>::v : 1)
    trace_batch_kernel(const __grid_constant__ BatchTable bt) {
    const int b = blockIdx.x;
    int j = 0;
    while (j + 1 < bt.n && b >= bt.job[j + 1].tile_begin) ++j;
    const BatchJob& jb = bt.job[j];
    const Scene& sc = jb.sc;
    const int t = b - jb.tile_begin;
    const int ty = t / jb.tiles_x, tx = t - ty * jb.tiles_x;
    const int px = tx * (int)blockDim.x + (int)threadIdx.x;
    const int py = ty * (int)blockDim.y + (int)threadIdx.y;
    if (px >= sc.width || py >= sc.height) return;
    float acc[3] = {0.0f, 0.0f, 0.0f};
    Tally total;
    total.clear();
    for (int smp = 0; smp < sc.spp; ++smp) run_ray<R, MODE, false>(px, py, smp, sc, jb.cam, jb.err, acc, total, nullptr);
    const float fs = sc.final_scale;
    jb.hdr[py * sc.width + px] = make_float4(acc[0] * fs, acc[1] * fs, acc[2] * fs, 1.0f);
}

template <class R, int MODE>
static cudaError_t launch_batch_typed(const BatchTable& bt, int bx, int by, cudaStream_t st) {
    if (bx * by <= 256)
        trace_batch_kernel<R, MODE, 256><<<bt.total_tiles, dim3(bx, by), 0, st>>>(bt);
    else
        trace_batch_kernel<R, MODE, 1024><<<bt.total_tiles, dim3(bx, by), 0, st>>>(bt);
    return cudaGetLastError();
}

cudaError_t launch_batch(const BatchTable& bt, int bx, int by, cudaStream_t st) {
    if (bt.n <= 0 || bt.total_tiles <= 0) return cudaSuccess;
    const Scene& s0 = bt.job[0].sc;
    if (s0.precision == 2) return launch_batch_typed<double, 1>(bt, bx, by, st);
    if (s0.precision == 1) return launch_batch_typed<Mixed, 1>(bt, bx, by, st);
    if (s0.mode == 1) return launch_batch_typed<float, 1>(bt, bx, by, st);
    return launch_batch_typed<float, 0>(bt, bx, by, st);
}

// Persistent batched trace.  The pixels of every job are cut into units of 32 (the tile order of
// unit_to_pixel, so a unit is a 16x2 patch of one frame); job j owns units [unit_begin,
// unit_begin of j + 1).  A warp takes one unit at a time from a single device counter over all
// jobs, so the 32 rays of a warp always share one scene and its parameters stay uniform
// constant-bank loads, and an SM never waits for a whole block: each warp moves on as soon as
// its own unit is done.  Per-pixel arithmetic is the plain kernel's (run_ray).
template <class R, int MODE, int MINB>
__global__ void __launch_bounds__(kWavefrontBlock, MINB)
    trace_batch_persistent_kernel(const __grid_constant__ BatchTable bt, unsigned* __restrict__ counter) {
    const int lane = threadIdx.x & 31;
    while (true) {
        unsigned u = 0;
        if (lane == 0) u = atomicAdd(counter, 1u);
        u = __shfl_sync(kFull, u, 0);
        if (u >= bt.total_units) break;
        int lo = 0, hi = bt.n - 1;  // last job whose first unit is <= u
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (bt.job[mid].unit_begin <= u) lo = mid; else hi = mid - 1;
        }
        const BatchJob& jb = bt.job[lo];
        const Scene& sc = jb.sc;
        const unsigned pix = (u - jb.unit_begin) * 32u + (unsigned)lane;
        if (pix < (unsigned)sc.width * (unsigned)sc.height) {
            int px, py;
            unit_to_pixel(pix, sc.width, sc.height, px, py);
            float acc[3] = {0.0f, 0.0f, 0.0f};
            Tally total;
            total.clear();
            for (int smp = 0; smp < sc.spp; ++smp)
                run_ray<R, MODE, false>(px, py, smp, sc, jb.cam, jb.err, acc, total, nullptr);
            const float fs = sc.final_scale;
            jb.hdr[py * sc.width + px] = make_float4(acc[0] * fs, acc[1] * fs, acc[2] * fs, 1.0f);
        }
    }
}

template <class R, int MODE, int MINB>
static cudaError_t launch_batch_persistent_minb(const BatchTable& bt, unsigned* counter, cudaStream_t st) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trace_batch_persistent_kernel<R, MODE, MINB>,
                                                           kWavefrontBlock, 0)) != cudaSuccess)
        return e;
    if (per_sm < 1) per_sm = 1;
    if ((e = cudaMemsetAsync(counter, 0, sizeof(unsigned), st)) != cudaSuccess) return e;
    trace_batch_persistent_kernel<R, MODE, MINB><<<sms * per_sm, kWavefrontBlock, 0, st>>>(bt, counter);
    return cudaGetLastError();
}

cudaError_t launch_batch_persistent(const BatchTable& bt, int blocks_per_sm, unsigned* counter, cudaStream_t st) {
    if (bt.n <= 0 || bt.total_units == 0) return cudaSuccess;
    const Scene& s0 = bt.job[0].sc;
    if (s0.precision == 2) return launch_batch_persistent_minb<double, 1, 2>(bt, counter, st);
    if (s0.precision == 1) return launch_batch_persistent_minb<Mixed, 1, 4>(bt, counter, st);
    if (s0.mode == 1) return launch_batch_persistent_minb<float, 1, 4>(bt, counter, st);
    switch (blocks_per_sm) {
        case 5: return launch_batch_persistent_minb<float, 0, 5>(bt, counter, st);
        case 6: return launch_batch_persistent_minb<float, 0, 6>(bt, counter, st);
        default: return launch_batch_persistent_minb<float, 0, 4>(bt, counter, st);
    }
}

// ---- image comparison (the autotuner's bit-identity filter) ---------------------------------
__global__ void __launch_bounds__(256) count_mismatch_kernel(const uint4* __restrict__ a, const uint4* __restrict__ b,
                                                             size_t n, unsigned long long* __restrict__ out) {
    unsigned long long local = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const uint4 x = __ldg(a + i), y = __ldg(b + i);
        local += (x.x != y.x || x.y != y.y || x.z != y.z || x.w != y.w) ? 1u : 0u;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(kFull, local, o);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(out, local);
}

cudaError_t launch_count_mismatch(const void* a, const void* b, size_t n16, unsigned long long* out, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess || n16 == 0) return e;
    int dev = 0, sms = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    const size_t want = (n16 + 255) / 256;
    const unsigned blocks = (unsigned)(want < (size_t)sms * 8 ? want : (size_t)sms * 8);
    count_mismatch_kernel<<<blocks, 256, 0, st>>>(static_cast<const uint4*>(a), static_cast<const uint4*>(b), n16, out);
    return cudaGetLastError();
}

// =========================================================================================
// Post-processing
// =========================================================================================

// Gaussian tap weight (cuda/kernel.cu:48-53).
__device__ __forceinline__ float tap_weight(int i, float sigma) {
    const float t = (float)i;
    const float den = 2.0f * sigma * sigma;
    return __expf(-(t * t) / den);
}

// ACES filmic fit (cuda/kernel.cu:17-29) and sRGB OETF (cuda/kernel.cu:30-43).
__device__ __forceinline__ float aces1(float x) {
    const float a = 2.51f, b = 0.03f, c = 2.43f, d = 0.59f, e = 0.14f;
    return (x * (a * x + b)) / (x * (c * x + d) + e);
}
__device__ __forceinline__ float srgb1(float x) {
    if (x <= 0.0031308f) return 12.92f * x;
    return 1.055f * powf(x, 0.4166666666666667f) - 0.055f;
}
__device__ __forceinline__ uint32_t to_byte(float v) {
    return (uint32_t)(unsigned char)__float2int_rn(__saturatef(v) * 255.0f);
}
__device__ __forceinline__ uint32_t tone_pack(float r, float g, float b) {
    const float mr = srgb1(aces1(r)), mg = srgb1(aces1(g)), mb = srgb1(aces1(b));
    return (to_byte(mr) << 16) | (to_byte(mg) << 8) | to_byte(mb);
}

// Bloom source (stated physics: only the part of the luminance above the threshold blooms).
__device__ __forceinline__ float4 bloom_source(float4 c, const PostParams& pp) {
    if (pp.mode != 1) return c;
    const float L = 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z;
    const float k = L > pp.threshold ? (L - pp.threshold) / L : 0.0f;
    return make_float4(c.x * k, c.y * k, c.z * k, c.w);
}

// ---- separable Gaussian, register-blocked ------------------------------------------------
// Each thread makes kBJ consecutive outputs along the blur direction from one stream of
// kBJ + 2R source values: value k feeds output j with weight w[k - j] (tap i = k - j - R), so
// every output still accumulates its taps in increasing i, the order of the reference's loop
// (cuda/kernel.cu:156-166, 199-209), with the same contracted multiply-adds, and gets the same
// bits.  A source value is read once per kBJ outputs instead of once per output.  The weight
// sum of an output (its in-image weights, added in the same order) depends only on its position
// and is computed once per block.  Chunks whose taps all lie inside the image run the head /
// middle / tail loop; chunks at the border run the reference's per-output loop.
constexpr int kBJ = 8;

template <class Load>
__device__ __forceinline__ void blur_interior(const Load& load, const float* w, int R, float (&acc)[kBJ][3]) {
#pragma unroll
    for (int j = 0; j < kBJ; ++j) acc[j][0] = acc[j][1] = acc[j][2] = 0.0f;
    // head: value k (< kBJ - 1) feeds outputs 0..k
#pragma unroll
    for (int k = 0; k < kBJ - 1; ++k) {
        const float4 v = load(k);
#pragma unroll
        for (int j = 0; j <= k; ++j) {
            const float wi = w[k - j];
            acc[j][0] += v.x * wi;
            acc[j][1] += v.y * wi;
            acc[j][2] += v.z * wi;
        }
    }
    // middle: every output; wr[j] = w[k - j] slides with k (w has a zero at index 2R + 1)
    float wr[kBJ];
#pragma unroll
    for (int j = 0; j < kBJ; ++j) wr[j] = w[kBJ - 1 - j];
#pragma unroll 8
    for (int k = kBJ - 1; k <= 2 * R; ++k) {
        const float4 v = load(k);
#pragma unroll
        for (int j = 0; j < kBJ; ++j) {
            acc[j][0] += v.x * wr[j];
            acc[j][1] += v.y * wr[j];
            acc[j][2] += v.z * wr[j];
        }
#pragma unroll
        for (int j = kBJ - 1; j > 0; --j) wr[j] = wr[j - 1];
        wr[0] = w[k + 1];
    }
    // tail: value 2R + t feeds outputs t..kBJ-1
#pragma unroll
    for (int t = 1; t < kBJ; ++t) {
        const float4 v = load(2 * R + t);
#pragma unroll
        for (int j = t; j < kBJ; ++j) {
            const float wi = w[2 * R + t - j];
            acc[j][0] += v.x * wi;
            acc[j][1] += v.y * wi;
            acc[j][2] += v.z * wi;
        }
    }
}

// Border chunk: the reference's loop per output, out-of-image taps skipped.  pos0 = position of
// output 0 along the blur, n = image extent along it; load(k) is only called for in-image taps.
template <class Load>
__device__ __forceinline__ void blur_edge(const Load& load, const float* w, int R, int pos0, int n,
                                          float (&acc)[kBJ][3]) {
#pragma unroll
    for (int j = 0; j < kBJ; ++j) {
        float ax = 0.0f, ay = 0.0f, az = 0.0f;
        for (int i = -R; i <= R; ++i) {
            const int sp = pos0 + j + i;
            if (sp < 0 || sp >= n) continue;
            const float wi = w[i + R];
            const float4 c = load(j + i + R);
            ax += c.x * wi;
            ay += c.y * wi;
            az += c.z * wi;
        }
        acc[j][0] = ax;
        acc[j][1] = ay;
        acc[j][2] = az;
    }
}

// Sum of the in-image tap weights of the output at `pos` (n = extent), in tap order.
__device__ __forceinline__ float weight_sum(int pos, int n, const float* w, int R) {
    float ws = 0.0f;
    for (int i = -R; i <= R; ++i) {
        const int sp = pos + i;
        if (sp < 0 || sp >= n) continue;
        ws += w[i + R];
    }
    return ws;
}

__device__ __forceinline__ void load_weights(float* w, int R, float sigma, int tid, int nthreads) {
    for (int i = tid; i <= 2 * R + 1; i += nthreads) w[i] = i <= 2 * R ? tap_weight(i - R, sigma) : 0.0f;
}

// 16-byte asynchronous copy global -> shared (cp.async, L2 only); the bytes past src_bytes are
// zero-filled and nothing is read when src_bytes is 0.  Both addresses are 16-byte aligned.
__device__ __forceinline__ void copy16_async(float4* dst, const float4* src, int src_bytes) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void copy_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Horizontal pass (bloom_horizontal, cuda/kernel.cu:144-173): a block makes a 32-row x 64-column
// tile.  Lane = row, warp = a kBJ-column chunk, so every tap test is uniform across the warp.
// The 32 source rows (64 + 2R columns) are staged at an odd float4 row stride (conflict-free
// column reads): warp w copies rows w, w + kHWarps, ..., its lanes taking consecutive
// float4 of a row (coalesced, no index division), every copy in flight before the first is
// waited for.
constexpr int kHRows = 32, kHWarps = 8, kHCols = kHWarps * kBJ;

__host__ __device__ constexpr int bloom_h_stride(int R) { return (kHCols + 2 * R) | 1; }

// Stages kHRows lines of a line-major source (line l at src + l * pitch; n_lines lines of
// n_pos values) into `stage`: lines line0 .. line0 + kHRows - 1, positions p0 - R ..
// p0 + kHCols + R - 1, zero outside the source.  Returns after the block's copies have landed
// (a barrier follows).
__device__ __forceinline__ void stage_lines(float4* stage, int stride, int segw, const float4* __restrict__ src,
                                            size_t pitch, int n_lines, int n_pos, int line0, int p0, int R,
                                            int tid) {
    const int wr = tid >> 5, ln = tid & 31;
    for (int r = wr; r < kHRows; r += kHWarps) {
        const int gl = line0 + r;
        const bool line_in = gl < n_lines;
        const float4* src_line = src + (line_in ? (size_t)gl * pitch : 0);
        for (int c = ln; c < segw; c += 32) {
            const int gp = p0 - R + c;
            const bool in = line_in && gp >= 0 && gp < n_pos;
            copy16_async(stage + r * stride + c, src_line + (in ? gp : 0), in ? 16 : 0);
        }
    }
    copy_async_wait_all();
}

// TRANSPOSED writes the bloom buffer column-major (bloom[x * height + y]): the layout that the
// fused post's vertical pass (post_vt_kernel) stages like this pass stages its rows.  Lanes
// being rows, it stores straight from registers; the row-major output goes back through shared
// memory for coalesced stores.
template <bool TRANSPOSED>
__global__ void __launch_bounds__(kHRows * kHWarps) bloom_h_kernel(const PostParams pp,
                                                                    const float4* __restrict__ hdr,
                                                                    float4* __restrict__ bloom) {
    extern __shared__ float4 smem4[];
    const int R = pp.radius;
    const int segw = kHCols + 2 * R, stride = bloom_h_stride(R);
    float4* stage = smem4;                                             // kHRows x stride
    float* w = reinterpret_cast<float*>(stage + kHRows * stride);      // 2R + 2
    float* wsum = w + 2 * R + 2;                                       // kHCols
    const int x0 = blockIdx.x * kHCols, y0 = blockIdx.y * kHRows;
    const int tid = threadIdx.x;
    load_weights(w, R, pp.sigma, tid, blockDim.x);
    stage_lines(stage, stride, segw, hdr, (size_t)pp.width, pp.height, pp.width, y0, x0, R, tid);
    if (pp.mode == 1) {  // stated physics: the bloom source of each in-image value, in place
        const int wr = tid >> 5, ln = tid & 31;
        for (int r = wr; r < kHRows; r += kHWarps) {
            const int gy = y0 + r;
            for (int c = ln; c < segw; c += 32) {
                const int gx = x0 - R + c;
                if (gy < pp.height && gx >= 0 && gx < pp.width) stage[r * stride + c] = bloom_source(stage[r * stride + c], pp);
            }
        }
    }
    __syncthreads();
    if (tid < kHCols) wsum[tid] = weight_sum(x0 + tid, pp.width, w, R);
    const int lane = tid & 31, cb = (tid >> 5) * kBJ;
    const float4* row = stage + lane * stride + cb;
    auto load = [row](int k) { return row[k]; };
    float acc[kBJ][3];
    const int xs = x0 + cb;
    if (2 * R >= kBJ - 1 && xs - R >= 0 && xs + kBJ - 1 + R < pp.width)
        blur_interior(load, w, R, acc);
    else
        blur_edge(load, w, R, xs, pp.width, acc);
    __syncthreads();  // staged sources no longer read; wsum written
    if (TRANSPOSED) {  // lane = row: each output column's 32 rows are one coalesced store
        const int gy = y0 + lane;
        if (gy >= pp.height) return;
#pragma unroll
        for (int j = 0; j < kBJ; ++j) {
            const int gx = xs + j;
            if (gx >= pp.width) break;
            const float ws = wsum[cb + j];
            float ax = acc[j][0], ay = acc[j][1], az = acc[j][2];
            if (ws > 0.0f) {
                ax /= ws;
                ay /= ws;
                az /= ws;
            }
            bloom[(size_t)gx * pp.height + gy] = make_float4(ax, ay, az, 0.0f);
        }
        return;
    }
    constexpr int ostride = kHCols + 1;
#pragma unroll
    for (int j = 0; j < kBJ; ++j) {
        const float ws = wsum[cb + j];
        float ax = acc[j][0], ay = acc[j][1], az = acc[j][2];
        if (ws > 0.0f) {
            ax /= ws;
            ay /= ws;
            az /= ws;
        }
        stage[lane * ostride + cb + j] = make_float4(ax, ay, az, 0.0f);
    }
    __syncthreads();
    for (int j = tid; j < kHRows * kHCols; j += blockDim.x) {
        const int r = j / kHCols, c = j - r * kHCols;
        const int gy = y0 + r, gx = x0 + c;
        if (gy < pp.height && gx < pp.width) bloom[(size_t)gy * pp.width + gx] = stage[r * ostride + c];
    }
}

// Vertical pass + composite + ACES + sRGB + pack (post_process, cuda/kernel.cu:175-251): a block
// makes a 64-column x 32-row tile; warp w covers 32 columns ((w & 1) * 32) and kBJ rows
// ((w >> 1) * kBJ); each thread streams its column of the bloom buffer with coalesced loads.
constexpr int kVCols = 64, kVRows = 32, kVThreads = 256;

__global__ void __launch_bounds__(kVThreads) post_v_kernel(const PostParams pp,
                                                            const float4* __restrict__ hdr,
                                                            const float4* __restrict__ bloom,
                                                            uint32_t* __restrict__ image) {
    extern __shared__ float smemf[];
    const int R = pp.active ? pp.radius : 0;
    float* w = smemf;                 // 2R + 2
    float* wsum = w + 2 * R + 2;      // kVRows
    const int tid = threadIdx.x;
    const int x0 = blockIdx.x * kVCols, y0 = blockIdx.y * kVRows;
    if (pp.active) {
        load_weights(w, R, pp.sigma, tid, blockDim.x);
        __syncthreads();
        if (tid < kVRows) wsum[tid] = weight_sum(y0 + tid, pp.height, w, R);
        __syncthreads();
    }
    const int lane = tid & 31, warp = tid >> 5;
    const int x = x0 + (warp & 1) * 32 + lane;
    const int rb = (warp >> 1) * kBJ;
    const int yb = y0 + rb;
    if (x >= pp.width || yb >= pp.height) return;
    float acc[kBJ][3];
    if (pp.active) {
        const float4* col = bloom + x;
        const int W = pp.width;
        auto load = [col, yb, R, W](int k) { return __ldg(col + (size_t)(yb - R + k) * W); };
        if (2 * R >= kBJ - 1 && yb - R >= 0 && yb + kBJ - 1 + R < pp.height)
            blur_interior(load, w, R, acc);
        else
            blur_edge(load, w, R, yb, pp.height, acc);
    }
#pragma unroll
    for (int j = 0; j < kBJ; ++j) {
        const int y = yb + j;
        if (y >= pp.height) break;
        const size_t idx = (size_t)y * pp.width + x;
        const float4 base = __ldg(hdr + idx);
        float fr = base.x, fg = base.y, fb = base.z;
        if (pp.active) {
            const float ws = wsum[rb + j];
            float ax = acc[j][0], ay = acc[j][1], az = acc[j][2];
            if (ws > 0.0f) {
                ax /= ws;
                ay /= ws;
                az /= ws;
            }
            fr += ax * pp.intensity;
            fg += ay * pp.intensity;
            fb += az * pp.intensity;
        }
        image[idx] = tone_pack(fr, fg, fb);
    }
}

// Vertical pass of the fused post over the column-major bloom buffer that bloom_h_kernel<true>
// writes: a block makes a 32-column x 64-row tile.  Lane = column, warp = a kBJ-row chunk; the
// block stages its 32 columns (64 + 2R rows each) exactly as the horizontal pass stages rows,
// so every source value is read from L2 once per tile instead of once per kBJ outputs, then
// blurs, composites, tone-maps and packs with the arithmetic of post_v_kernel (same bits).
__global__ void __launch_bounds__(kHRows * kHWarps) post_vt_kernel(const PostParams pp,
                                                                    const float4* __restrict__ hdr,
                                                                    const float4* __restrict__ bloom_t,
                                                                    uint32_t* __restrict__ image) {
    extern __shared__ float4 smem4[];
    const int R = pp.radius;
    const int segw = kHCols + 2 * R, stride = bloom_h_stride(R);
    float4* stage = smem4;                                             // kHRows x stride
    float* w = reinterpret_cast<float*>(stage + kHRows * stride);      // 2R + 2
    float* wsum = w + 2 * R + 2;                                       // kHCols
    const int x0 = blockIdx.x * kHRows, y0 = blockIdx.y * kHCols;
    const int tid = threadIdx.x;
    load_weights(w, R, pp.sigma, tid, blockDim.x);
    stage_lines(stage, stride, segw, bloom_t, (size_t)pp.height, pp.width, pp.height, x0, y0, R, tid);
    __syncthreads();
    if (tid < kHCols) wsum[tid] = weight_sum(y0 + tid, pp.height, w, R);
    const int lane = tid & 31, cb = (tid >> 5) * kBJ;
    const float4* col = stage + lane * stride + cb;
    auto load = [col](int k) { return col[k]; };
    float acc[kBJ][3];
    const int ys = y0 + cb;
    if (2 * R >= kBJ - 1 && ys - R >= 0 && ys + kBJ - 1 + R < pp.height)
        blur_interior(load, w, R, acc);
    else
        blur_edge(load, w, R, ys, pp.height, acc);
    __syncthreads();  // wsum written
    const int x = x0 + lane;
    if (x >= pp.width) return;
    float4 base[kBJ];  // all of a thread's composite sources in flight before the first is used
#pragma unroll
    for (int j = 0; j < kBJ; ++j)
        base[j] = ys + j < pp.height ? __ldg(hdr + (size_t)(ys + j) * pp.width + x) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int j = 0; j < kBJ; ++j) {
        const int y = ys + j;
        if (y >= pp.height) break;
        const size_t idx = (size_t)y * pp.width + x;
        float fr = base[j].x, fg = base[j].y, fb = base[j].z;
        const float ws = wsum[cb + j];
        float ax = acc[j][0], ay = acc[j][1], az = acc[j][2];
        if (ws > 0.0f) {
            ax /= ws;
            ay /= ws;
            az /= ws;
        }
        fr += ax * pp.intensity;
        fg += ay * pp.intensity;
        fb += az * pp.intensity;
        image[idx] = tone_pack(fr, fg, fb);
    }
}

// Tone map only (bloom inactive): one thread per pixel.
__global__ void tonemap_kernel(const PostParams pp, const float4* __restrict__ hdr,
                               uint32_t* __restrict__ image) {
    const size_t n = (size_t)pp.width * pp.height;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const float4 c = __ldg(hdr + i);
        image[i] = tone_pack(c.x, c.y, c.z);
    }
}

static size_t bloom_h_smem(int R) {
    return (size_t)kHRows * bloom_h_stride(R) * sizeof(float4) + (size_t)(2 * R + 2 + kHCols) * sizeof(float);
}
static size_t post_v_smem(int R) { return (size_t)(2 * R + 2 + kVRows) * sizeof(float); }
constexpr size_t kSmemLimit = 200 * 1024;

static cudaError_t set_smem(const void* fn, size_t bytes) {
    if (bytes <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

cudaError_t launch_bloom_horizontal(const PostParams& pp, const float4* hdr, float4* bloom, cudaStream_t st) {
    if (pp.width <= 0 || pp.height <= 0) return cudaSuccess;
    const size_t sm = bloom_h_smem(pp.radius);
    if (sm > kSmemLimit) return cudaErrorInvalidValue;
    cudaError_t e = set_smem((const void*)bloom_h_kernel<false>, sm);
    if (e != cudaSuccess) return e;
    const dim3 grid((pp.width + kHCols - 1) / kHCols, (pp.height + kHRows - 1) / kHRows);
    bloom_h_kernel<false><<<grid, kHRows * kHWarps, sm, st>>>(pp, hdr, bloom);
    return cudaGetLastError();
}

cudaError_t launch_post_process(const PostParams& pp, const float4* hdr, const float4* bloom,
                                uint32_t* image, cudaStream_t st) {
    if (pp.width <= 0 || pp.height <= 0) return cudaSuccess;
    const size_t sm = pp.active ? post_v_smem(pp.radius) : 0;
    if (sm > kSmemLimit) return cudaErrorInvalidValue;
    cudaError_t e = set_smem((const void*)post_v_kernel, sm);
    if (e != cudaSuccess) return e;
    const dim3 grid((pp.width + kVCols - 1) / kVCols, (pp.height + kVRows - 1) / kVRows);
    post_v_kernel<<<grid, kVThreads, sm, st>>>(pp, hdr, bloom, image);
    return cudaGetLastError();
}

// FP32 FMA throughput probe (the denominator of the trace's roofline): eight independent
// dependent chains per thread hide the FMA latency; the chains are kept alive by a store that
// only a sum of exactly 12345.678 would trigger.
__global__ void __launch_bounds__(512) fma_probe_kernel(float b, float c, int iters, float* sink) {
    float v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = (float)threadIdx.x * 1e-3f + (float)i;
#pragma unroll 8
    for (int k = 0; k < iters; ++k) {
#pragma unroll
        for (int i = 0; i < 8; ++i) v[i] = fmaf(v[i], b, c);
    }
    float s = 0.0f;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += v[i];
    if (s == 12345.678f) sink[0] = s;
}

cudaError_t launch_fma_probe(int blocks, int iters, float* sink, cudaStream_t st) {
    fma_probe_kernel<<<blocks, 512, 0, st>>>(0.999999f, 1e-6f, iters, sink);
    return cudaGetLastError();
}

cudaError_t launch_post_fused(const PostParams& pp, const float4* hdr, uint32_t* image, float4* scratch,
                              cudaStream_t st) {
    if (pp.width <= 0 || pp.height <= 0) return cudaSuccess;
    if (!pp.active) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        tonemap_kernel<<<sms * 8, 256, 0, st>>>(pp, hdr, image);
        return cudaGetLastError();
    }
    if (!scratch) return cudaErrorInvalidValue;
    // both passes through the context's scratch, column-major in between (never seen by callers)
    const size_t sm = bloom_h_smem(pp.radius);
    if (sm > kSmemLimit) return cudaErrorInvalidValue;
    cudaError_t e = set_smem((const void*)bloom_h_kernel<true>, sm);
    if (e == cudaSuccess) e = set_smem((const void*)post_vt_kernel, sm);
    if (e != cudaSuccess) return e;
    const dim3 gh((pp.width + kHCols - 1) / kHCols, (pp.height + kHRows - 1) / kHRows);
    bloom_h_kernel<true><<<gh, kHRows * kHWarps, sm, st>>>(pp, hdr, scratch);
    const dim3 gv((pp.width + kHRows - 1) / kHRows, (pp.height + kHCols - 1) / kHCols);
    post_vt_kernel<<<gv, kHRows * kHWarps, sm, st>>>(pp, hdr, scratch, image);
    return cudaGetLastError();
}

}  // namespace ktd
