// kt_diff.h — records and launchers of the differentiable trace (host and device).
//
// The recording forward keeps, per ray, a doubly linked list of segment records drawn from one
// device pool: each holds the state at the segment start and up to kSegSteps accepted step
// sizes.  The records freeze the step sequence (replay at other parameters = the frozen-step
// model that central differences need) and serve as the adjoint's checkpoints (one state every
// kSegSteps accepted steps; the steps in between are recomputed).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "kt_types.h"

namespace ktd {

constexpr int kSegSteps = 32;

enum DiffTerm : int {
    kTermBudget = 0,      // max_steps or transmittance cutoff
    kTermHorizon = 1,
    kTermEscape = 2,
    kTermFrozen = 3,      // state became NaN (the NaN step is not recorded)
    kTermNotStarted = 4,  // the integration loop never ran
    kTermOverflow = 5,    // the segment pool ran out: the ray has no usable record
};

struct DiffRay {
    int first_seg, last_seg;  // -1 when the ray has no segment
    int n_steps;              // recorded accepted steps
    int n_hits;               // shaded disk crossings
    int term;                 // DiffTerm
    float sky;                // sky value at transmittance 1 when the ray escaped, else 0
};

template <class R>
struct alignas(16) DiffSeg {
    int prev, next;   // neighbours in the ray's list, -1 at the ends
    int n;            // steps in this segment (1..kSegSteps)
    int first_step;   // index of its first step along the ray
    unsigned hits;    // bit j: step j shaded a disk crossing
    int pad;
    R tau;            // transmittance at the segment start
    R s[6];           // state at the segment start
    R h[kSegSteps];   // accepted step sizes
};

// Type-erased record set (segs points to DiffSeg<float> or DiffSeg<double>).
struct DiffRecRaw {
    DiffRay* rays;
    void* segs;
    unsigned* seg_count;  // pool cursor
    unsigned cap;         // pool capacity (segments)
    unsigned* status;     // [0]: rays that overflowed the pool
};

// Derivatives of the scene inputs that depend on the parameters.
struct DiffLut {
    const double* lut_d;     // the disk LUT entries in double
    const double* dlut_da;   // d(disk LUT entry)/d(spin)
    const double* dlut_dro;  // d(disk LUT entry)/d(disk outer radius)
    double dr_in_da;         // d(ISCO)/d(spin)
    double dtemp_ds;         // d(disk temperature scale)/d(temperature-scale parameter)
};

// Camera in double (the FP64 differentiable trace builds its rays from it) and, as dcam, its
// derivative in the inclination.
struct CameraD {
    double pos[3], fwd[3], rgt[3], up[3];
    double fov_scale;
};

// Forward over all pixels of sc (stated physics, spp 1).  replay = 0: adaptive steps, records
// written; replay = 1: the recorded steps at the scene's (new) parameters, flags[p] = 1 where
// the ray's events (termination step or kind, shaded crossings) differ from the record.
// sc.precision selects float (0) or double (2) arithmetic.  hdr64: optional, 3 doubles per
// pixel (the colour before the float store).  float_records (replay with double arithmetic
// only): the records are DiffSeg<float>, replayed in double.
cudaError_t launch_diff_forward(const Scene& sc, const Camera& cam, const CameraD& camd, const DiffRecRaw& rec,
                                int replay, float4* hdr, double* hdr64, uint32_t* err, uint32_t* flags,
                                cudaStream_t stream, bool float_records = false);
// Scratch of the adjoint's work ordering: bucket and order (one word per pixel each), ctl
// (kDiffWorkCtl words).
constexpr int kDiffWorkCtl = 65;
struct DiffWork {
    int* bucket;
    unsigned* order;
    unsigned* ctl;
};

// Adjoint: grad[0..3] += d(sum_p dl_dhdr[p] . hdr[p]) / d(spin, inclination in degrees,
// temperature-scale parameter, disk outer radius).  dcamd = d(camera)/d(inclination in degrees).
// The float path starts its rays from cam (the renderer's camera), the double path from camd.
// float_records (double arithmetic only): the records are DiffSeg<float>, differentiated as the
// FP64 replay of their steps (segment starts replayed in double from the ray's start).
cudaError_t launch_diff_backward(const Scene& sc, const Camera& cam, const CameraD& camd, const CameraD& dcamd,
                                 const DiffRecRaw& rec, const DiffLut& dl, const float4* dl_dhdr, double* grad,
                                 const DiffWork& work, cudaStream_t stream, bool float_records = false);

}  // namespace ktd
