// kt_context.h — the device context behind the opaque kt_context handle (private to the
// library's host translation units: kt_host.cpp, kt_tune.cpp).
#pragma once
#include <cuda_runtime.h>

#include "../../include/kerrtrace.h"
#include "kt_internal.h"

struct kt_context {
    int device = 0;
    kt_config cfg{};
    kt_kerr_params params{};
    ktd::Scene scene{};
    ktd::PostParams post{};
    cudaArray_t bb_array = nullptr, disk_array = nullptr;
    cudaTextureObject_t bb_tex = 0, disk_tex = 0;
    float4* bb_lut_dev = nullptr;
    float* disk_lut_dev = nullptr;
    unsigned* queue = nullptr;              // wavefront work counter (1 word)
    ktd::Tuning tuning;                     // persistent-tracer launch shape
    unsigned long long* counters = nullptr; // 6 x u64 for the counting launches
    unsigned* order = nullptr;              // pixel order (allocated when a tuning asks for it)
    float4* bloom_scratch = nullptr;        // kt_post_fused's bloom buffer (when bloom is active)
    int block_x = 16, block_y = 16;
};
