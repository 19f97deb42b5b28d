// kt_internal.h — launchers shared by the C-ABI layer (kt_host.cpp) and the kernels
// translation unit (kt_kernels.cu).  Not part of the public ABI.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "kt_types.h"

namespace ktd {

// Bloom / post-process constants of one context (src/renderer/init.rs:43-73, mod.rs:139-148).
struct PostParams {
    int width, height;
    int radius;       // ceil(bloom.radius)
    float sigma;      // bloom.radius / 3
    float intensity;
    int active;       // enabled && radius > 0 && intensity > 0
    int mode;         // stated-physics luminance threshold when 1
    float threshold;
};

// Tuning of the persistent tracer: resident blocks per SM (3..6 for the FP32 reference
// kernel; the default otherwise) and the number of idle lanes a warp waits for before it
// refills them (1..32).
struct Tuning {
    int schedule = 1;
    int block_x = 0, block_y = 0;
    int blocks_per_sm = 4;
    int refill_min = 1;
    int order = 0;  // 1: pixels ranked long-rays-first by the rank kernel before the trace
    int keep_frozen = 0;  // 1: NaN-frozen rays iterate to max_steps (Scene::keep_frozen)
};

// Pixel-order buffer: kOrderHeader header words (marked / unmarked counts), then one pixel
// index per work unit.
constexpr unsigned kOrderHeader = 16;

// Trace launch: schedule 0 = plain 2D grid (block bx x by), 1 = persistent wavefront.
// precision 0 = FP32, 1 = mixed, 2 = FP64.  queue: one device word, reset here on `stream`.
// ctr: optional 6 x u64 device counters (selects the counting kernels); aux: optional float4
// per pixel with the first shaded disk hit (r, g, T, hits) of sample 0 (counting kernels only).
// order: NULL for tile order, else a pixel-order buffer of kOrderHeader + width * height words
// that the rank kernel fills on `stream` before the trace.
cudaError_t launch_trace(const Scene& sc, const Camera& cam, int schedule, float4* hdr,
                         uint32_t* err, unsigned* queue, unsigned long long* ctr, float4* aux,
                         const Tuning& tn, int bx, int by, unsigned* order, cudaStream_t stream);

// Batched trace: one plain-schedule launch over the tiles of up to kBatchMaxJobs renders.  The
// table travels as a kernel parameter (__grid_constant__); each block finds its job from the
// tile prefix, so the job index and its scene constants are uniform across the block.
constexpr int kBatchMaxJobs = 64;
struct BatchJob {
    Scene sc;
    Camera cam;
    float4* hdr;
    uint32_t* err;
    int tiles_x;
    int tile_begin;
    unsigned unit_begin;  // persistent launch: first 32-pixel unit of this job
};
struct BatchTable {
    BatchJob job[kBatchMaxJobs];
    int n;
    int total_tiles;
    unsigned total_units;
};
cudaError_t launch_batch(const BatchTable& bt, int bx, int by, cudaStream_t stream);
// Persistent batched trace: warps take 32-pixel units, each inside one job, from the device
// counter `counter` (one word, reset here on `stream`); blocks of 128 threads, blocks_per_sm
// resident per SM (the FP32 reference-semantics kernel has 4, 5 and 6; the others their default).
cudaError_t launch_batch_persistent(const BatchTable& bt, int blocks_per_sm, unsigned* counter, cudaStream_t stream);
// Number of 16-byte words that differ between a and b (n16 words each) into *out (device).
cudaError_t launch_count_mismatch(const void* a, const void* b, size_t n16, unsigned long long* out,
                                  cudaStream_t stream);

cudaError_t launch_bloom_horizontal(const PostParams& pp, const float4* hdr, float4* bloom,
                                    cudaStream_t stream);
cudaError_t launch_post_process(const PostParams& pp, const float4* hdr, const float4* bloom,
                                uint32_t* image, cudaStream_t stream);
// Both post passes; scratch: a width x height float4 bloom buffer (unused when bloom is off).
cudaError_t launch_post_fused(const PostParams& pp, const float4* hdr, uint32_t* image, float4* scratch,
                              cudaStream_t stream);
// FP32 FMA throughput probe: `blocks` x 512 threads, each running 8 independent FMA chains of
// `iters` steps (16 * iters flops per thread).
cudaError_t launch_fma_probe(int blocks, int iters, float* sink, cudaStream_t st);
// Lookup tables on the device (kt_luts.cu): n_lambda wavelengths from wl_start in steps of
// wl_step; disk radii from r_in to r_out.
cudaError_t launch_blackbody_lut(uint32_t size, float max_temp, float wl_start, int n_lambda, float wl_step,
                                 float4* out, cudaStream_t st);
cudaError_t launch_disk_lut(uint32_t size, float a_norm, float inv_m, float r_in, float r_out, float* out,
                            cudaStream_t st);

}  // namespace ktd

// Host helpers shared with the allocation-free entry point (kt_noalloc.cu).
#include "../../include/kerrtrace.h"
namespace ktd {
kt_status scene_from_config(const kt_config* cfg, Scene* out);
kt_status set_error(kt_status s, const char* msg);
}  // namespace ktd
