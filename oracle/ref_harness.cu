// ref_harness.cu — launches the reference's own kernels.  TEST INFRASTRUCTURE ONLY.
//
// The reference's cuda/kernel.cu (with kerr_trace.cuh and kerr_math.cuh) is compiled unmodified
// from its source tree: this file is built with `-I <reference>/cuda -include <defines.h>` where
// defines.h is the `#define` header the reference's host would prepend
// (src/renderer/utils.rs:121-163), and `-use_fast_math` as config.yaml sets
// (src/renderer/init.rs:112-118).  The C functions below redo what the Rust host does around
// the kernels: upload c_params (init.rs:129-139), create the two LUT textures
// (texture.rs:86-202) and launch trace_kernel / bloom_horizontal / post_process with the
// arguments of submit_render (mod.rs:153-206).  The outputs are the GPU golden the tests and
// the reference arm of bench.py compare against; nothing here is shipped.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include "kernel.cu"

extern "C" {

int ktref_sizeof_params(void) { return (int)sizeof(KerrParams); }

int ktref_set_params(const void* params, size_t bytes) {
    if (bytes != sizeof(KerrParams)) return -1;
    return (int)cudaMemcpyToSymbol(c_params, params, sizeof(KerrParams));
}

// texture.rs:86-202: float channels, linear filter, normalised coordinates, clamp.  The
// blackbody LUT array has height 1 and the disk LUT array height 0, as in texture.rs:37-67.
static int make_tex(const float* host, int n, int ch, size_t height, cudaArray_t* arr, cudaTextureObject_t* tex) {
    cudaChannelFormatDesc d = ch == 4 ? cudaCreateChannelDesc(32, 32, 32, 32, cudaChannelFormatKindFloat)
                                      : cudaCreateChannelDesc(32, 0, 0, 0, cudaChannelFormatKindFloat);
    cudaError_t e = cudaMallocArray(arr, &d, (size_t)n, height, cudaArrayDefault);
    if (e != cudaSuccess) return (int)e;
    const size_t bytes = (size_t)n * ch * sizeof(float);
    e = cudaMemcpy2DToArray(*arr, 0, 0, host, bytes, bytes, 1, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return (int)e;
    cudaResourceDesc rd;
    memset(&rd, 0, sizeof rd);
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = *arr;
    cudaTextureDesc td;
    memset(&td, 0, sizeof td);
    td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeClamp;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 1;
    return (int)cudaCreateTextureObject(tex, &rd, &td, nullptr);
}

typedef struct ktref_textures {
    cudaArray_t bb_arr, disk_arr;
    unsigned long long bb_tex, disk_tex;
} ktref_textures;

int ktref_make_textures(const float* bb_rgba, const float* disk, int n, ktref_textures* out) {
    memset(out, 0, sizeof *out);
    cudaTextureObject_t t1 = 0, t2 = 0;
    int e = make_tex(bb_rgba, n, 4, 1, &out->bb_arr, &t1);
    if (e) return e;
    e = make_tex(disk, n, 1, 0, &out->disk_arr, &t2);
    if (e) return e;
    out->bb_tex = t1;
    out->disk_tex = t2;
    return 0;
}

int ktref_free_textures(ktref_textures* t) {
    cudaDestroyTextureObject((cudaTextureObject_t)t->bb_tex);
    cudaDestroyTextureObject((cudaTextureObject_t)t->disk_tex);
    cudaFreeArray(t->bb_arr);
    cudaFreeArray(t->disk_arr);
    memset(t, 0, sizeof *t);
    return 0;
}

// mod.rs:153-173
int ktref_trace(float* hdr, int width, int height, const float* cam12, unsigned long long lut_tex, int lut_size,
                float max_temp, unsigned int* err, unsigned long long disk_tex, float disk_inner, float disk_outer,
                float fov_scale, int bx, int by, void* stream) {
    dim3 block(bx, by), grid((width + bx - 1) / bx, (height + by - 1) / by);
    trace_kernel<<<grid, block, 0, (cudaStream_t)stream>>>(
        (float4*)hdr, width, height, cam12[0], cam12[1], cam12[2], cam12[3], cam12[4], cam12[5], cam12[6], cam12[7],
        cam12[8], cam12[9], cam12[10], cam12[11], (cudaTextureObject_t)lut_tex, lut_size, max_temp, err,
        (cudaTextureObject_t)disk_tex, disk_inner, disk_outer, fov_scale);
    return (int)cudaGetLastError();
}

// mod.rs:177-191
int ktref_bloom(const float* hdr, float* bloom, int width, int height, int radius, float sigma, int enabled, int bx,
                int by, void* stream) {
    dim3 block(bx, by), grid((width + bx - 1) / bx, (height + by - 1) / by);
    bloom_horizontal<<<grid, block, 0, (cudaStream_t)stream>>>((const float4*)hdr, (float4*)bloom, width, height,
                                                               radius, sigma, enabled);
    return (int)cudaGetLastError();
}

// mod.rs:192-206 with the shared-memory size of mod.rs:275-292
int ktref_post(const float* hdr, const float* bloom, unsigned int* image, int width, int height, int radius,
               float sigma, float intensity, int enabled, int bx, int by, void* stream) {
    dim3 block(bx, by), grid((width + bx - 1) / bx, (height + by - 1) / by);
    size_t smem = enabled ? (size_t)bx * (size_t)(by + 2 * radius) * 16 : 0;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(post_process, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return (int)e;
    }
    post_process<<<grid, block, smem, (cudaStream_t)stream>>>((const float4*)hdr, (const float4*)bloom, image, width,
                                                               height, radius, sigma, intensity, enabled);
    return (int)cudaGetLastError();
}

// Samples a texture made like texture.rs at normalised coordinates (to check the oracle's
// model of hardware linear filtering).
__global__ void tex_probe_kernel(unsigned long long tex, const float* us, float* out, int n, int ch) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (ch == 4) {
        const float4 v = tex1D<float4>((cudaTextureObject_t)tex, us[i]);
        out[4 * i] = v.x;
        out[4 * i + 1] = v.y;
        out[4 * i + 2] = v.z;
        out[4 * i + 3] = v.w;
    } else {
        out[i] = tex1D<float>((cudaTextureObject_t)tex, us[i]);
    }
}
int ktref_tex_probe(unsigned long long tex, const float* us_dev, float* out_dev, int n, int ch) {
    tex_probe_kernel<<<(n + 255) / 256, 256>>>(tex, us_dev, out_dev, n, ch);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return (int)e;
    return (int)cudaDeviceSynchronize();
}

}  // extern "C"
