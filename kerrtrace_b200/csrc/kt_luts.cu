// kt_luts.cu — the two lookup tables generated on the device.
//
// The same tables as the host generators (kt_generate_blackbody_lut, kt_generate_disk_lut in
// kt_host.cpp, which follow src/renderer/blackbody.rs:6-124 and src/renderer/utils.rs:11-52,
// 172-201), one thread per table row, written into device memory on the caller's stream.
// This file is compiled without fast math: expm1f, expf, logf, acosf, cosf, cbrtf and sqrtf are
// CUDA's accurate versions, so the tables agree with the host ones to a few ulp (they are not
// bit-equal: CUDA's and glibc's libm round differently in the last place).
#include <cuda_runtime.h>
#include <stdint.h>

#include "kt_internal.h"

namespace ktd {

namespace {

// One lobe of the piecewise-Gaussian fit to the CIE 1931 matching functions.
__device__ float cmf_lobe_d(float x, float alpha, float mu, float s1, float s2) {
    const float sigma = x < mu ? s1 : s2;
    const float t = (x - mu) / sigma;
    return alpha * expf(-0.5f * t * t);
}

// Row ti: the linear-sRGB colour of a blackbody at temperature ti / (size - 1) x max_temp,
// integrated over the wavelength grid wl_start, wl_start + wl_step, ... (f32 accumulation, as the
// host grid) with the Planck law and the XYZ -> linear-sRGB matrix.
__global__ void blackbody_lut_kernel(uint32_t size, float max_temp, float wl_start, int n_lambda, float wl_step,
                                     float4* __restrict__ out) {
    const uint32_t ti = blockIdx.x * blockDim.x + threadIdx.x;
    if (ti >= size) return;
    const float t = (float)((double)ti / (double)(size - 1) * (double)max_temp);
    if (t == 0.0f) {
        out[ti] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        return;
    }
    const float c2 = 1.4388e7f;
    float xsum = 0.0f, ysum = 0.0f, zsum = 0.0f;
    float l = wl_start;
    for (int i = 0; i < n_lambda; ++i) {
        float inten = 0.0f;
        if (t > 0.0f) {
            const float expo = c2 / (l * t);
            if (!(expo > 80.0f)) {
                const float l2 = l * l;
                const float l5 = l * (l2 * l2);
                inten = ((1.0f / l5) / expm1f(expo)) * 1e15f;
            }
        }
        const float xs = cmf_lobe_d(l, 1.056f, 599.8f, 37.9f, 31.0f) + cmf_lobe_d(l, 0.362f, 442.0f, 16.0f, 26.7f) +
                         cmf_lobe_d(l, -0.065f, 501.1f, 20.4f, 26.2f);
        const float ys = cmf_lobe_d(l, 0.821f, 568.8f, 46.9f, 40.5f) + cmf_lobe_d(l, 0.286f, 530.9f, 16.3f, 31.1f);
        const float zs = cmf_lobe_d(l, 1.217f, 437.0f, 11.8f, 36.0f) + cmf_lobe_d(l, 0.681f, 459.0f, 26.2f, 13.8f);
        xsum += inten * xs;
        ysum += inten * ys;
        zsum += inten * zs;
        l += wl_step;
    }
    xsum *= wl_step;
    ysum *= wl_step;
    zsum *= wl_step;
    out[ti] = make_float4(fmaf(3.240454f, xsum, fmaf(-1.5371385f, ysum, -0.4985314f * zsum)),
                          fmaf(-0.969266f, xsum, fmaf(1.8760108f, ysum, 0.041556f * zsum)),
                          fmaf(0.0556434f, xsum, fmaf(-0.2040259f, ysum, 1.0572252f * zsum)), 0.0f);
}

// Page-Thorne flux factor with the roots 2 cos(acos(-a)/3 - 2 pi k / 3) of x^3 - 3x + 2a = 0.
__device__ float nt_factor_d(float r, float a_norm, float r_isco, float inv_m) {
    if (r <= r_isco) return 0.0f;
    const float r_norm = r * inv_m;
    const float r_isco_norm = r_isco * inv_m;
    const float x = sqrtf(r_norm);
    const float x_ms = sqrtf(r_isco_norm);
    const float third = 1.0f / 3.0f;
    const float angle_base = acosf(-a_norm) * third;
    const float ang_step = 2.0943952f;
    const float roots[3] = {2.0f * cosf(angle_base), 2.0f * cosf(angle_base - ang_step),
                            2.0f * cosf(angle_base + ang_step)};
    float sum_log = 0.0f;
    for (int i = 0; i < 3; ++i) {
        const float xi = roots[i];
        const float den = xi * (xi - roots[(i + 1) % 3]) * (xi - roots[(i + 2) % 3]);
        if (den <= 0.0f) continue;
        const float coef = 3.0f * (xi - a_norm) * (xi - a_norm) / den;
        const float val = (x - xi) / (x_ms - xi);
        if (val > 0.0f) sum_log += coef * logf(val);
    }
    const float q = fmaf(1.5f * a_norm, -logf(x / x_ms), x - x_ms) - sum_log;
    const float geo = r_norm * fmaf(2.0f, a_norm, fmaf(r_norm, x, -(3.0f * x)));
    return fmaxf(q / geo, 0.0f);
}

// Row i: f^(1/4) of the flux factor at r_i = r_in + i / (size - 1) (r_out - r_in).
__global__ void disk_lut_kernel(uint32_t size, float a_norm, float inv_m, float r_in, float r_out,
                                float* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= size) return;
    const double ratio = (double)i / (double)(size - 1);
    const float r = (float)fma(ratio, (double)(r_out - r_in), (double)r_in);
    out[i] = sqrtf(sqrtf(nt_factor_d(r, a_norm, r_in, inv_m)));
}

}  // namespace

cudaError_t launch_blackbody_lut(uint32_t size, float max_temp, float wl_start, int n_lambda, float wl_step,
                                 float4* out, cudaStream_t st) {
    blackbody_lut_kernel<<<(size + 127) / 128, 128, 0, st>>>(size, max_temp, wl_start, n_lambda, wl_step, out);
    return cudaGetLastError();
}

cudaError_t launch_disk_lut(uint32_t size, float a_norm, float inv_m, float r_in, float r_out, float* out,
                            cudaStream_t st) {
    disk_lut_kernel<<<(size + 127) / 128, 128, 0, st>>>(size, a_norm, inv_m, r_in, r_out, out);
    return cudaGetLastError();
}

}  // namespace ktd
