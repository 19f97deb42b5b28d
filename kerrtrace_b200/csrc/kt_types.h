// kt_types.h — plain structs shared by host and device code (no device functions here).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ktd {

// ----------------------------------------------------------------------------------------
// Per-render constants.  The first block mirrors KerrParams (cuda/kerr_math.cuh:3-9); the
// second holds the values the reference bakes into #defines (src/renderer/utils.rs:121-163)
// — double-typed where the reference's unsuffixed literals make the expression double.
// ----------------------------------------------------------------------------------------
struct Scene {
    float a, M, aa, inv_M, a_norm, rh, disk_inner, disk_outer;
    float inv_w_2, inv_h_2, aspect;
    float noise_scale, noise_strength, noise_winding;
    int noise_enabled, noise_detail;

    int spp, max_steps, max_attempts, sky_div;
    float sky_spacing;   // 3.14159265f / (float)CONFIG_SKY_GRID_DIVISIONS, folded on the host
    float h0;            // (float)CONFIG_INTEGRATOR_INITIAL_STEP
    float base_tol;      // (float)CONFIG_INTEGRATOR_TOLERANCE
    float sky_thickness; // (float)CONFIG_SKY_LINE_THICKNESS
    // Exact float forms of the reference's mixed float/double comparisons:
    //   r < rh + HORIZON_EPS (double)   <=>  r < horizon_lt   (horizon_lt = smallest float >= the double sum)
    //   r > ESCAPE_RADIUS (double)      <=>  r > escape_gt    (escape_gt  = largest float <= the double)
    //   tau > TRANSMITTANCE_CUTOFF      <=>  tau > cutoff_gt
    float horizon_lt, escape_gt, cutoff_gt;
    float final_scale;   // (float)(EXPOSURE_SCALE * (1.0f / spp)), kernel.cu:136
    double temp_scale;   // CONFIG_DISK_TEMPERATURE_SCALE
    double wl_step;      // CONFIG_BLACKBODY_WAVELENGTH_STEP
    double sky_intensity;// CONFIG_SKY_INTENSITY
    // double forms of the same scene for the FP64 path
    double a_d, aa_d, M_d, horizon_d, escape_d, cutoff_d, h0_d, base_tol_d;

    cudaTextureObject_t bb_tex;    // float4, linear, normalised, clamp (texture.rs:176-202)
    cudaTextureObject_t disk_tex;  // float1, same sampler
    const float4* bb_lut;          // same LUTs as plain arrays (software interpolation)
    const float* disk_lut;
    int lut_size;
    float lut_max_temp;

    int mode;            // 0 = reference semantics, 1 = stated physics
    int precision;       // 0 = FP32, 1 = mixed, 2 = FP64
    unsigned noise_seed;
    float noise_phase;
    float zone_r;        // mixed precision: FP64 update below this Kerr-Schild radius
    int zone_err64;      // mixed precision: FP64 error norm in the zone (tolerance below 3e-7)
    // FP64 path: disk radii, and optionally a double disk LUT (the differentiable trace sets
    // them from double parameters; otherwise they are the float values and the float LUT)
    double disk_inner_d, disk_outer_d;
    const double* disk_lut_d;
    float spec_tol_floor;// stated physics: tolerance never drops below base_tol * this
    int width, height;
    // Samples: the kernel traces samples [sample_first, sample_first + spp) of each pixel.
    // pixel_centre: stated physics with one sample per pixel uses the pixel centre.  accum
    // (progressive sampling, plain schedule): the running sum of the raw sample colours per
    // pixel, read when sample_first > 0 and written back with the sample count in w.
    int sample_first;
    int pixel_centre;
    float4* accum;
    // 1: a ray whose state has become NaN keeps iterating to max_steps, as the reference's
    // does (cuda/kerr_trace.cuh:62,83-125); 0 (default): it is retired at that commit.  The
    // image is the same either way; the switch measures what retirement saves.
    int keep_frozen;
};

struct Camera {
    float pos[3], fwd[3], rgt[3], up[3];
    float fov_scale;
};

}  // namespace ktd
