// kt_noalloc.cu — trace entry point that allocates no device memory (kt_trace_noalloc).
//
// Some callers cannot allocate device memory at the point where they render: a host whose
// device memory all belongs to its own pool allocator (an engine, or a framework with a caching
// allocator that must account for every byte), or a per-frame path that must not call
// cudaMalloc / cudaFree because they synchronise the device and would stall the frames already
// in flight.  Such a caller cannot create a kt_context, which allocates its LUT textures and
// its work counter.  kt_trace_noalloc takes everything from the caller instead — scene
// configuration, cameras, the two LUTs as plain device arrays, the output buffers — and keeps
// its only scratch, one work counter per view, in the file-scope array below.
//
// The array is part of the library's device image: every GPU that loads the library holds its
// 256 bytes until the process exits.  Every call shares it and it keeps the last call's
// counters; each call clears the counters it uses on its own stream before the trace kernel
// runs.  Calls that overlap on the GPU (other streams, other host threads on the same device)
// race on the counters and must be serialised by the caller.
//
// The kernel is the persistent wavefront tracer with reference semantics; the LUTs are read
// from the plain arrays through a model of the texture unit's linear filter (mode 2 of the
// device code), so results agree with kt_trace to the parity tolerance, not bit for bit.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/kerrtrace.h"
#include "kt_internal.h"
#include "kt_ray.cuh"

namespace ktd {

// Scratch of kt_trace_noalloc: one work counter per view.  In host code this name is only a
// stand-in for the device symbol; its device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned int g_noalloc_queue[KT_NOALLOC_MAX_VIEWS];

struct NoallocViews {
    Camera cam[KT_NOALLOC_MAX_VIEWS];
    int n;
};

constexpr unsigned kFullMask = 0xffffffffu;
constexpr int kNoallocBlock = 128;

// Same per-unit mapping as the wavefront kernel: 16-row bands, 16-column tiles, row-major.
__device__ __forceinline__ void noalloc_unit_to_pixel(unsigned u, int W, int H, int& px, int& py) {
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

// Persistent wavefront trace over several views of one scene.  A warp takes pixels from the
// counter of its current view and moves to the next view when that counter is exhausted;
// every lane remembers the view of the pixel it holds.
__global__ void __launch_bounds__(kNoallocBlock, 4)
    trace_views_noalloc_kernel(const __grid_constant__ Scene sc, const __grid_constant__ NoallocViews views,
                               float4* __restrict__ hdr,
                               uint32_t* __restrict__ err, unsigned* __restrict__ queue) {
    constexpr int MODE = 2;
    const int lane = threadIdx.x & 31;
    const unsigned lane_lt = (1u << lane) - 1u;
    const unsigned n_units = (unsigned)sc.width * (unsigned)sc.height;
    RayRun<float> ry;
    Tally tl;
    tl.clear();
    int px = 0, py = 0, smp = 0, lview = 0, view = 0;
    float acc[3] = {0.0f, 0.0f, 0.0f};
    bool active = false;
    bool open = views.n > 0;

    while (true) {
        if (open) {
            const unsigned need = __ballot_sync(kFullMask, !active);
            if (need) {
                const int leader = __ffs(need) - 1;
                const unsigned cnt = (unsigned)__popc(need);
                unsigned base = 0;
                if (lane == leader) base = atomicAdd(queue + view, cnt);
                base = __shfl_sync(kFullMask, base, leader);
                const int v = view;
                if (base + cnt >= n_units) {
                    ++view;
                    if (view >= views.n) open = false;
                }
                if (!active) {
                    const unsigned u = base + (unsigned)__popc(need & lane_lt);
                    if (u < n_units) {
                        lview = v;
                        const Camera cam = views.cam[lview];
                        noalloc_unit_to_pixel(u, sc.width, sc.height, px, py);
                        acc[0] = acc[1] = acc[2] = 0.0f;
                        for (smp = 0; smp < sc.spp; ++smp) {
                            float dir[3];
                            pixel_ray<MODE>(px, py, smp, sc, cam, dir);
                            if (ray_start<float>(ry, cam, dir, sc)) break;
                        }
                        if (smp < sc.spp) {
                            active = true;
                        } else {
                            const float fs = sc.final_scale;
                            hdr[(size_t)lview * n_units + (size_t)py * sc.width + px] =
                                make_float4(acc[0] * fs, acc[1] * fs, acc[2] * fs, 1.0f);
                        }
                    }
                }
            }
        }
        // A warp with no ray in flight goes back for more pixels while views remain: a claim
        // can come back empty (its view was used up, or every claimed pixel had no ray work,
        // e.g. max_steps = 0), and `view` has then already moved on to the next view.
        if (!__any_sync(kFullMask, active)) {
            if (!open) break;
            continue;
        }
        if (active && ray_advance<float, MODE, false>(ry, sc, err + 2 * lview, tl)) {
            acc[0] += ry.col[0];
            acc[1] += ry.col[1];
            acc[2] += ry.col[2];
            const Camera cam = views.cam[lview];
            for (++smp; smp < sc.spp; ++smp) {
                float dir[3];
                pixel_ray<MODE>(px, py, smp, sc, cam, dir);
                if (ray_start<float>(ry, cam, dir, sc)) break;
            }
            if (smp >= sc.spp) {
                const float fs = sc.final_scale;
                hdr[(size_t)lview * n_units + (size_t)py * sc.width + px] =
                    make_float4(acc[0] * fs, acc[1] * fs, acc[2] * fs, 1.0f);
                active = false;
            }
        }
    }
}

// Device address of g_noalloc_queue, looked up once per device.
constexpr int kMaxDevices = 64;
static std::mutex g_noalloc_mutex;
static unsigned* g_noalloc_addr[kMaxDevices];

static kt_status noalloc_scratch(int device, unsigned** out) {
    if (device < 0 || device >= kMaxDevices) return set_error(KT_ERR_INVALID_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_queue);
        if (e != cudaSuccess) {
            char msg[256];
            snprintf(msg, sizeof msg, "cudaGetSymbolAddress of the work counters failed: %s", cudaGetErrorString(e));
            return set_error(KT_ERR_CUDA, msg);
        }
        g_noalloc_addr[device] = static_cast<unsigned*>(p);
    }
    *out = g_noalloc_addr[device];
    return KT_OK;
}

}  // namespace ktd

extern "C" kt_status kt_trace_noalloc(const kt_config* cfg, const kt_camera* cams, uint32_t n_views,
                                      const float* bb_lut, const float* disk_lut, void* stream,
                                      float* hdr_out, uint32_t* err_words) {
    using namespace ktd;
    if (!cfg || !cams || !bb_lut || !disk_lut || !hdr_out || !err_words)
        return set_error(KT_ERR_INVALID_ARG, "kt_trace_noalloc: NULL argument");
    if (n_views == 0 || n_views > KT_NOALLOC_MAX_VIEWS) {
        char msg[160];
        snprintf(msg, sizeof msg, "kt_trace_noalloc: %u views requested; its scratch holds work counters for 1..%d views",
                 n_views, KT_NOALLOC_MAX_VIEWS);
        return set_error(KT_ERR_INVALID_ARG, msg);
    }
    if (cfg->mode != KT_MODE_REF || cfg->precision != KT_PREC_FP32)
        return set_error(KT_ERR_UNSUPPORTED, "kt_trace_noalloc implements the reference semantics in FP32 only");
    if ((uint64_t)cfg->width * cfg->height * n_views >= (1ull << 32))
        return set_error(KT_ERR_INVALID_ARG, "kt_trace_noalloc: frame too large for the 32-bit work counters");
    Scene sc;
    kt_status st = scene_from_config(cfg, &sc);
    if (st != KT_OK) return st;
    sc.bb_lut = reinterpret_cast<const float4*>(bb_lut);
    sc.disk_lut = disk_lut;
    sc.bb_tex = 0;
    sc.disk_tex = 0;
    NoallocViews views;
    views.n = (int)n_views;
    for (uint32_t v = 0; v < n_views; ++v) {
        for (int i = 0; i < 3; ++i) {
            views.cam[v].pos[i] = cams[v].cam_pos[i];
            views.cam[v].fwd[i] = cams[v].fwd[i];
            views.cam[v].rgt[i] = cams[v].rgt[i];
            views.cam[v].up[i] = cams[v].up[i];
        }
        views.cam[v].fov_scale = cams[v].fov_scale;
    }
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_error(KT_ERR_CUDA, "cudaGetDevice failed");
    unsigned* queue = nullptr;
    if ((st = noalloc_scratch(dev, &queue)) != KT_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess ||
        (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trace_views_noalloc_kernel, kNoallocBlock, 0)) !=
            cudaSuccess ||
        (e = cudaMemsetAsync(queue, 0, n_views * sizeof(unsigned), s)) != cudaSuccess)
        return set_error(KT_ERR_CUDA, cudaGetErrorString(e));
    if (per_sm < 1) per_sm = 1;
    trace_views_noalloc_kernel<<<sms * per_sm, kNoallocBlock, 0, s>>>(sc, views, reinterpret_cast<float4*>(hdr_out),
                                                                     err_words, queue);
    if ((e = cudaGetLastError()) != cudaSuccess) return set_error(KT_ERR_CUDA, cudaGetErrorString(e));
    return KT_OK;
}
