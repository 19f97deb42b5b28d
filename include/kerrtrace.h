/*
 * kerrtrace.h — C ABI of the B200-native KerrTrace geodesic hot path.
 *
 * The reference (DamoyY/KerrTrace) JIT-compiles cuda/kernel.cu with NVRTC, uploads
 * `__constant__ KerrParams c_params`, builds two LUT textures and launches three kernels per
 * frame from Rust (src/renderer/{init,mod,texture,utils,blackbody}.rs).  This header is the
 * drop-in for that layer: plain C types, caller-owned buffers, stream-ordered calls, status
 * codes instead of panics.  Each entry point names the reference item it replaces.
 *
 * Conventions
 *  - Every `stream` argument is a `cudaStream_t` passed as `void*` (NULL = legacy default
 *    stream, the one cudarc's `context.default_stream()` uses, src/renderer/mod.rs:80).
 *  - Device pointers are marked `dev`; host pointers `host`.  The caller owns every output
 *    buffer.  A context owns its LUT textures and the small scratch words of the wavefront
 *    tracer; calls on one context must be ordered on one stream at a time.
 *  - No call synchronises unless its comment says so.  Device-side failures (LUT overflow,
 *    non-finite input) are reported through the 2 x u32 error word exactly like the
 *    reference's `lut_error_flag` (cuda/kernel.cu:3-9): word[0] = 1 on the first failure,
 *    word[1] = the f32 bits of the offending temperature.
 *  - No exception or abort crosses this boundary.  On failure a call returns a status and
 *    `kt_last_error()` holds a message for the calling thread.
 */
#ifndef KERRTRACE_H
#define KERRTRACE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KT_ABI_VERSION 3

typedef enum kt_status {
    KT_OK = 0,
    KT_ERR_INVALID_ARG = 1,   /* bad config / pointer / size (reference: anyhow! in utils.rs, init.rs) */
    KT_ERR_CUDA = 2,          /* a CUDA runtime call failed (reference: cudarc DriverError) */
    KT_ERR_LUT_OVERFLOW = 3,  /* colour temperature above lut_max_temp (mod.rs:236-241) */
    KT_ERR_NOT_READY = 4,     /* frame not complete yet (mod.rs:226-228 returns Ok(None)) */
    KT_ERR_QUEUE_ORDER = 5,   /* finish_frame out of order (mod.rs:253-256) */
    KT_ERR_NO_DEVICE = 6,     /* no CUDA device / library built without one */
    KT_ERR_UNSUPPORTED = 7,   /* option not available in this build */
    KT_ERR_TIMEOUT = 8        /* a bounded device wait gave up */
} kt_status;

/* Integration semantics.  KT_MODE_REF reproduces the reference kernel exactly, including its
 * documented quirks (linear-guess crossing root, H-scaled tolerance that reaches zero near the
 * hole, always-jittered pixel samples).  KT_MODE_SPEC follows the stated physics instead:
 * Newton/bisection crossing root on the dense output, tolerance never below `tolerance`,
 * pixel-centre samples at spp = 1, seeded/phased FBM and a luminance bloom threshold. */
typedef enum kt_mode { KT_MODE_REF = 0, KT_MODE_SPEC = 1 } kt_mode;

/* Arithmetic of the geodesic integration.  FP32 is the reference's arithmetic.  MIXED keeps
 * FP32 for the bulk and uses FP64 for the state update / error norm inside 1.5 x the photon
 * orbit radius or near the horizon, the null-constraint renormalisation of p and the crossing
 * solve.  FP64 runs the whole integration in double. */
typedef enum kt_precision { KT_PREC_FP32 = 0, KT_PREC_MIXED = 1, KT_PREC_FP64 = 2 } kt_precision;

/* Scheduling of the trace kernel.  All schedules produce the same image bits. */
typedef enum kt_schedule {
    KT_SCHED_PLAIN = 0,     /* one thread per pixel on a 2D grid of block_dim tiles (kernel.cu:88) */
    KT_SCHED_WAVEFRONT = 1, /* persistent kernel, lanes refilled from a device work counter */
    KT_SCHED_AUTO = 2       /* whichever the context's kt_tuning selects (the autotuner's choice) */
} kt_schedule;

/* Order in which the tracers take pixels.  Per-pixel results are the same in both. */
typedef enum kt_order {
    KT_ORDER_TILES = 0,      /* 16x16 tiles in raster order (plain: the 2D grid) */
    KT_ORDER_LONG_FIRST = 1  /* a rank kernel first moves the pixels whose rays are predicted to
                                wind near a photon orbit (Kerr constants of motion) to the front,
                                so the longest rays start first instead of forming the tail */
} kt_order;

/* Launch shape used by KT_SCHED_AUTO (see kt_context_set_tuning). */
typedef struct kt_tuning {
    int32_t schedule;      /* KT_SCHED_PLAIN or KT_SCHED_WAVEFRONT */
    int32_t block_x;       /* plain: block shape, 0 = the config's block_dim */
    int32_t block_y;
    int32_t blocks_per_sm; /* wavefront: resident blocks of 128 threads per SM, 3..6; plain (blocks
                              of at most 128 threads): 5 or 6 (FP32, mixed) or 3 or 4 (FP64) asks
                              for that many resident blocks, anything else for the default shape */
    int32_t refill_min;    /* wavefront: idle lanes a warp collects before refilling them, 1..32 */
    int32_t order;         /* kt_order; KT_ORDER_LONG_FIRST allocates a 4-byte-per-pixel buffer */
    int32_t keep_frozen;   /* 0 (default): a ray whose state has become NaN (the reference's
                              tolerance reaches 0 near the hole, cuda/kerr_trace.cuh:66-73) is
                              retired at that step; 1: it iterates to max_steps like the
                              reference's (kerr_trace.cuh:62,83-125).  Same image bits either way;
                              1 only serves to time the reference's amount of work. */
} kt_tuning;

/*
 * Full configuration.  Field names follow the reference's config.yaml / serde structs
 * (src/main.rs:15-122); values that the reference bakes into `#define`s
 * (src/renderer/utils.rs:121-163) are runtime values here.  Use kt_config_default() for the
 * reference's config.yaml values.
 */
typedef struct kt_config {
    /* window (main.rs:28-32) */
    uint32_t width;
    uint32_t height;
    /* renderer (main.rs:50-54) */
    uint32_t block_dim[2];
    /* bloom (main.rs:56-60) */
    int32_t bloom_enabled;
    float bloom_intensity;
    float bloom_radius;
    /* blackbody (main.rs:68-74) */
    uint32_t lut_size;
    float lut_max_temp;
    float wavelength_start;
    float wavelength_end;
    float wavelength_step;
    /* cuda (main.rs:76-78).  Must be 1: the kernels are built with -use_fast_math. */
    int32_t use_fast_math;
    /* kernel (main.rs:88-122) */
    uint32_t spp;
    float exposure_scale;
    uint32_t sky_grid_divisions;
    float sky_line_thickness;
    float sky_intensity;
    float spin;
    float mass;
    float disk_outer_radius;
    float disk_temperature_scale;
    float initial_step;
    float tolerance;
    uint32_t max_steps;
    uint32_t max_attempts;
    float transmittance_cutoff;
    float horizon_epsilon;
    float escape_radius;
    /* disk_noise (main.rs:80-86) */
    int32_t noise_enabled;
    float noise_scale;
    float noise_strength;
    float noise_winding;
    uint32_t noise_detail;
    /* extensions (no reference counterpart; zero = reference behaviour) */
    int32_t mode;            /* kt_mode */
    int32_t precision;       /* kt_precision */
    uint32_t noise_seed;     /* KT_MODE_SPEC only: XORed into the FBM lattice hash */
    float noise_phase;       /* KT_MODE_SPEC only: added to the disk azimuth */
    float bloom_threshold;   /* KT_MODE_SPEC only: bloom source = max(L - threshold, 0)/L * hdr */
    float photon_zone_factor;/* KT_PREC_MIXED: FP64 zone radius = factor * photon orbit radius (0 = 1.5) */
} kt_config;

/* Mirror of the reference's `KerrParams` (cuda/kerr_math.cuh:3-9, src/renderer/init.rs:15-33). */
typedef struct kt_kerr_params {
    float a, m, aa, inv_m, a_norm, rh, disk_inner;
    float inv_w_2, inv_h_2, aspect_ratio;
    float disk_noise_scale, disk_noise_strength, disk_noise_winding;
    int32_t disk_noise_enabled, disk_noise_detail;
} kt_kerr_params;

/* Camera of one frame: the arguments of CudaRenderer::submit_render (mod.rs:119-126). */
typedef struct kt_camera {
    float cam_pos[3];
    float fwd[3];
    float rgt[3];
    float up[3];
    float fov_scale;  /* tan(fov / 2), src/app.rs:163 */
} kt_camera;

/* Per-launch statistics of a trace (optional; pass NULL to skip counting). */
typedef struct kt_trace_stats {
    uint64_t rays;
    uint64_t steps;        /* committed integration steps */
    uint64_t attempts;     /* DP5(4) attempts (accepted + rejected) */
    uint64_t rhs_evals;    /* Hamiltonian right-hand-side evaluations */
    uint64_t frozen_rays;  /* rays retired early because their state became NaN */
    uint64_t fp64_steps;   /* steps taken with the FP64 update (KT_PREC_MIXED) */
} kt_trace_stats;

typedef struct kt_context kt_context;
typedef struct kt_renderer kt_renderer;

/* ---- status ---------------------------------------------------------------------------- */
const char* kt_status_str(kt_status s);
/* Message of the last failure on the calling thread ("" if none). */
const char* kt_last_error(void);
int kt_abi_version(void);

/* ---- host precompute (CPU only, no device needed) ---------------------------------------- */
/* Defaults of the reference's config.yaml (config.yaml:1-67). */
kt_status kt_config_default(kt_config* cfg);
/* build_kerr_params (src/renderer/utils.rs:53-113): rh, prograde ISCO, 2/W, 2/H, W/H. */
kt_status kt_build_kerr_params(const kt_config* cfg, kt_kerr_params* out);
/* calc_isco (src/renderer/utils.rs:11-20), f32 arithmetic as the reference host. */
float kt_calc_isco(float a_norm, int prograde, float mass);
/* generate_blackbody_lut (src/renderer/blackbody.rs:56-124): `size` RGBA f32 rows on a linear
 * temperature grid [0, max_temp].  out_rgba holds size*4 floats. */
kt_status kt_generate_blackbody_lut(uint32_t size, float max_temp, float wavelength_start,
                                    float wavelength_end, float wavelength_step, float* out_rgba);
/* generate_disk_temperature_lut (src/renderer/utils.rs:172-201): f^(1/4) of the
 * Novikov-Thorne / Page-Thorne flux factor on `size` radii in [disk_inner, disk_outer]. */
kt_status kt_generate_disk_lut(const kt_kerr_params* params, float disk_outer, uint32_t size,
                               float* out);
/* The same two tables generated on the device, on `stream`, into device memory (dev_out:
 * float[4*size] / float[size]), one thread per row.  They use CUDA's accurate math functions and
 * agree with the host tables to a few ulp, not bit for bit (CUDA's and glibc's libm round
 * differently in the last place).  For hosts that build many per-scene tables (batches) or keep
 * everything on the device. */
kt_status kt_generate_blackbody_lut_device(uint32_t size, float max_temp, float wavelength_start,
                                           float wavelength_end, float wavelength_step, float* dev_out,
                                           void* stream);
kt_status kt_generate_disk_lut_device(const kt_kerr_params* params, float disk_outer, uint32_t size,
                                      float* dev_out, void* stream);
/* build_cuda_defines (src/renderer/utils.rs:121-163): the `#define` header text the reference
 * prepends to kernel.cu.  Writes a NUL-terminated string; *len gets its length. */
kt_status kt_build_defines(const kt_config* cfg, char* buf, size_t cap, size_t* len);
/* calculate_camera_basis (src/math.rs:3-14): forward from yaw/pitch in degrees, right =
 * forward x (0,1,0), up = right x forward, each normalised (glam f32 arithmetic). */
kt_status kt_camera_basis(float yaw_deg, float pitch_deg, float fwd[3], float rgt[3], float up[3]);
/* fov_scale = tan(fov.to_radians() / 2) (src/app.rs:163). */
float kt_fov_scale(float fov_deg);
/* validate_bloom_settings (src/renderer/init.rs:43-73). */
kt_status kt_validate_bloom(const kt_config* cfg, int32_t* enabled, float* intensity,
                            float* radius, int32_t* radius_int);

/* ---- device context: replaces build_textures + build_cuda_kernels (init.rs:74-140) -------- */
/* Builds KerrParams and both LUTs on the host, uploads the LUTs as 1D linear-filtered,
 * normalised, clamped textures (texture.rs:86-202) and keeps the scene parameters. */
kt_status kt_context_create(const kt_config* cfg, int device, kt_context** out);
/* Same, with caller-supplied LUTs (host arrays: bb_rgba lut_n*4 floats, disk lut_n floats). */
kt_status kt_context_create_with_luts(const kt_config* cfg, int device, const float* bb_rgba,
                                      const float* disk, uint32_t lut_n, kt_context** out);
/* Same as kt_context_create, with both LUTs generated on the device (kt_generate_*_lut_device)
 * and the textures filled from device memory: no host table is built or copied.  The device
 * tables agree with the host's (which are bit-equal to the reference's Rust generators) to a few
 * ulp, so images match kt_context_create's to the parity tolerance, not bit for bit.
 * Synchronises the device once. */
kt_status kt_context_create_device_luts(const kt_config* cfg, int device, kt_context** out);
void kt_context_destroy(kt_context* ctx);
/* Copies out the derived KerrParams the context uses. */
kt_status kt_context_params(const kt_context* ctx, kt_kerr_params* out);

/* ---- per-frame kernels: replace the three launches of submit_render (mod.rs:153-206) ------ */
/* trace_kernel (cuda/kernel.cu:88-142): writes W*H float4 (r,g,b,1) HDR, row-major.
 * hdr_out: dev float[4*W*H]; err_word: dev uint32[2] (not cleared here, like the reference,
 * which clears it with memset_zeros before the launch, mod.rs:150-152). */
kt_status kt_trace(kt_context* ctx, void* stream, const kt_camera* cam, int32_t schedule,
                   float* hdr_out, uint32_t* err_word);
/* Same as kt_trace, plus per-launch counters (synchronises the stream to read them).
 * aux_out (dev float[4*W*H], may be NULL) receives, per pixel, the first shaded disk hit of
 * sample 0: Kerr-Schild radius, redshift g, temperature T and the number of shaded hits
 * (NaN where the ray shaded nothing). */
kt_status kt_trace_counted(kt_context* ctx, void* stream, const kt_camera* cam,
                           int32_t schedule, float* hdr_out, uint32_t* err_word,
                           kt_trace_stats* stats, float* aux_out);
/* Progressive sampling: the reference's per-pixel sample loop (cuda/kernel.cu:104-139) split
 * over launches.  Traces samples [first_sample, first_sample + n_samples) of every pixel with
 * the reference's jitter keys (pixel index << 32 | sample index), continues the running sum of
 * the raw sample colours in accum (dev float[4*W*H]: rgb = sum, w = samples so far; read when
 * first_sample > 0, written every call) and writes hdr_out = sum x (float)(exposure x (1.0f /
 * samples so far)).  After samples 0..N-1, in any split, hdr_out is bit for bit the kt_trace
 * image of the same scene at spp = N.  Samples are always jittered (also in stated physics,
 * whose spp = 1 trace uses the pixel centre).  Plain schedule, stream-ordered. */
kt_status kt_trace_progressive(kt_context* ctx, void* stream, const kt_camera* cam, uint32_t first_sample,
                               uint32_t n_samples, float* accum, float* hdr_out, uint32_t* err_word);
/* Launch shape of the trace (the autotuner's knobs, kerrtrace_b200/autotune.py).  For the
 * persistent schedule: resident blocks of 128 threads per SM (3..6; the compiler caps registers
 * per thread accordingly; only the FP32 reference-semantics kernel has the 3/5/6 variants) and
 * the refill threshold.  For the plain schedule: the block shape (at most 1024 threads).
 * kt_trace(KT_SCHED_AUTO) runs tuning->schedule; the explicit schedules use the rest of the
 * tuning too, the pixel order included.  Default: wavefront, config block_dim, 4 blocks per
 * SM, refill 1, tile order.  Call it outside stream capture: the first long-first tuning of a
 * context allocates the order buffer. */
kt_status kt_context_set_tuning(kt_context* ctx, const kt_tuning* tuning);
kt_status kt_context_get_tuning(const kt_context* ctx, kt_tuning* tuning);

/* Launch-shape autotuner (no reference counterpart: the reference launches its trace on the
 * config's block_dim, src/renderer/mod.rs:132-136 and init.rs compute_launch_dims).  Times the
 * trace of `cam` under each candidate tuning with CUDA events on `stream` (one warm-up launch,
 * then `reps` launches, 1..64, scored by the median), keeps only candidates whose image is bit
 * for bit the first candidate's, and installs the fastest of those in the context
 * (kt_context_set_tuning); kt_trace(KT_SCHED_AUTO) then runs it.  candidates == NULL uses the
 * built-in list (plain block shapes, 128-thread plain blocks with more resident blocks per SM,
 * wavefront blocks per SM x refill thresholds, each in tile and long-rays-first order; at most
 * KT_TUNE_MAX_CANDIDATES, keep_frozen taken from the current tuning).  table (may be NULL)
 * receives one row per candidate, *n_entries their number.  Allocates scratch for one frame
 * and synchronises `stream`; call it at set-up, outside stream capture. */
#define KT_TUNE_MAX_CANDIDATES 64
typedef struct kt_tune_entry {
    kt_tuning tuning;
    float ms;          /* median trace time of the candidate */
    int32_t identical; /* 1 when its image equals the first candidate's bit for bit */
} kt_tune_entry;
kt_status kt_context_autotune(kt_context* ctx, void* stream, const kt_camera* cam, uint32_t reps,
                              const kt_tuning* candidates, uint32_t n_candidates, kt_tune_entry* table,
                              uint32_t* n_entries);
/* The post entry points read and write float4 pixels: hdr and bloom must be 16-byte aligned
 * (KT_ERR_INVALID_ARG otherwise), image_out 4-byte aligned.
 * bloom_horizontal (cuda/kernel.cu:144-173): dev float4 hdr -> dev float4 bloom. */
kt_status kt_bloom_horizontal(kt_context* ctx, void* stream, const float* hdr, float* bloom);
/* post_process (cuda/kernel.cu:175-251): vertical blur + composite + ACES + sRGB + pack to
 * 0x00RRGGBB.  bloom may be NULL when bloom is inactive. */
kt_status kt_post_process(kt_context* ctx, void* stream, const float* hdr, const float* bloom,
                          uint32_t* image_out);
/* Both post passes through the context's own bloom buffer (allocated with the context when
 * bloom is active): same output bits as kt_bloom_horizontal followed by kt_post_process.  Calls
 * on one context must not overlap in time (they share that buffer). */
kt_status kt_post_fused(kt_context* ctx, void* stream, const float* hdr, uint32_t* image_out);

/* ---- batched renders (many scenes / cameras in one launch) -------------------------------- */
/* Largest number of renders in one batch (the job table is a kernel parameter). */
#define KT_BATCH_MAX_JOBS 64
/* One render of a batch: its own scene (spin, disk, resolution, ...), camera and outputs.
 * All jobs of a batch share `mode` and `precision`. */
typedef struct kt_job {
    kt_config cfg;
    kt_camera cam;
    float* hdr_out;      /* dev float[4*W*H] */
    uint32_t* err_word;  /* dev uint32[2], not cleared by the trace calls */
} kt_job;
typedef struct kt_batch kt_batch;
/* Builds one context per job (its LUTs and textures) and the launch table. */
kt_status kt_batch_create(const kt_job* jobs, uint32_t n_jobs, int device, kt_batch** out);
/* Plain-schedule block shape of the batched launch (default 16x16; at most 1024 threads). */
kt_status kt_batch_set_block(kt_batch* b, int32_t block_x, int32_t block_y);
/* Launch shape of the batch.  schedule KT_SCHED_PLAIN: one thread per pixel on tiles of
 * block_x x block_y (as kt_batch_set_block).  KT_SCHED_WAVEFRONT: one persistent launch of
 * 128-thread blocks (blocks_per_sm resident per SM, 4..6; only the FP32 reference-semantics
 * kernel has 5 and 6) whose warps take 32-pixel units, each inside one job, from one device
 * counter over all jobs.  Both give every job the image of its own kt_trace, bit for bit. */
kt_status kt_batch_set_tuning(kt_batch* b, const kt_tuning* tuning);
kt_status kt_batch_get_tuning(const kt_batch* b, kt_tuning* tuning);
/* Times the batched launch under each candidate shape (six plain block shapes, the persistent
 * launch at each blocks_per_sm it has) with CUDA events on `stream` (one launch to compare the
 * images with the first candidate's, then `reps` timed launches, median), and installs the
 * fastest whose images of every job equal the first candidate's bit for bit.  table (may be
 * NULL; room for KT_TUNE_MAX_CANDIDATES rows) and *n_entries as kt_context_autotune.  Allocates
 * a copy of all job images and synchronises `stream`: call it at set-up, outside capture. */
kt_status kt_batch_autotune(kt_batch* b, void* stream, uint32_t reps, kt_tune_entry* table, uint32_t* n_entries);
/* New camera for job j (the next kt_batch_trace_graph re-captures its graph). */
kt_status kt_batch_set_camera(kt_batch* b, uint32_t j, const kt_camera* cam);
/* Traces every job in one kernel launch on `stream`. */
kt_status kt_batch_trace(kt_batch* b, void* stream);
/* The same launch replayed from a CUDA graph, captured on first use (and after a change). */
kt_status kt_batch_trace_graph(kt_batch* b, void* stream);
/* Baseline: one kt_trace launch per job, in job order, on `stream`. */
kt_status kt_batch_trace_sequential(kt_batch* b, void* stream, int32_t schedule);
uint64_t kt_batch_rays(const kt_batch* b);
void kt_batch_destroy(kt_batch* b);

/* ---- trace without any device allocation --------------------------------------------------- */
/* Largest n_views of one kt_trace_noalloc call: its scratch is one 32-bit work counter per view,
 * held in a 256-byte array inside the library's device image. */
#define KT_NOALLOC_MAX_VIEWS 64
/*
 * No counterpart in the reference.  For callers that cannot allocate device memory where they
 * render: hosts whose device memory all belongs to their own pool allocator, and per-frame
 * paths that must not call cudaMalloc/cudaFree because those synchronise the device and stall
 * the frames in flight.  Such a caller cannot create a kt_context (it allocates LUT textures and
 * a work counter), so this call takes everything from the caller and allocates nothing:
 *   cfg        scene configuration (reference semantics, FP32: mode KT_MODE_REF, precision FP32)
 *   cams       host array of n_views cameras (1 <= n_views <= KT_NOALLOC_MAX_VIEWS, else
 *              KT_ERR_INVALID_ARG with a message)
 *   bb_lut     dev float[lut_size*4], the blackbody LUT (kt_generate_blackbody_lut layout)
 *   disk_lut   dev float[lut_size], the disk temperature LUT (kt_generate_disk_lut)
 *   hdr_out    dev float[n_views*W*H*4], view v at offset v*W*H*4
 *   err_words  dev uint32[2*n_views], the LUT error word of each view (not cleared here)
 * It runs the wavefront tracer on the current device and stream, reading the LUTs through a
 * model of the texture unit's filter, so its images match kt_trace to the parity tolerance.
 * The first call on a device looks up the scratch array's device address
 * (cudaGetSymbolAddress) with that device current; make that first call before any stream
 * capture.  The address is kept for the life of the process: after a cudaDeviceReset of that
 * device (which unloads the library's device image) do not call this entry point on it again.  Every call shares the scratch: calls that overlap on the GPU race and must be
 * serialised by the caller.
 */
kt_status kt_trace_noalloc(const kt_config* cfg, const kt_camera* cams, uint32_t n_views,
                           const float* bb_lut, const float* disk_lut, void* stream,
                           float* hdr_out, uint32_t* err_words);

/* ---- CudaRenderer mirror (src/renderer/mod.rs:52-293) ------------------------------------ */
/* CudaRenderer::new (mod.rs:76-117): context + two frame buffers with pinned host images. */
kt_status kt_renderer_new(const kt_config* cfg, int device, kt_renderer** out);
/* CudaRenderer::submit_render (mod.rs:119-218).  *submitted = 0 when both frames are in
 * flight (the reference returns Ok(false)). */
kt_status kt_renderer_submit_render(kt_renderer* r, const float cam_pos[3], const float fwd[3],
                                    const float rgt[3], const float up[3], float fov_scale,
                                    int32_t* submitted);
/* CudaRenderer::ready_frame (mod.rs:220-250).  Returns KT_ERR_NOT_READY when no frame is
 * complete, KT_ERR_LUT_OVERFLOW (and *overflow_temp) when the frame's error word was set. */
kt_status kt_renderer_ready_frame(kt_renderer* r, uint32_t* index, const uint32_t** data,
                                  float* overflow_temp);
/* CudaRenderer::finish_frame (mod.rs:252-260). */
kt_status kt_renderer_finish_frame(kt_renderer* r, uint32_t index);
/* Blocks until every submitted frame is complete (no reference counterpart; used by hosts
 * that render headless). */
kt_status kt_renderer_wait(kt_renderer* r);
/* Selects the trace schedule used by submit_render (default KT_SCHED_AUTO). */
kt_status kt_renderer_set_schedule(kt_renderer* r, int32_t schedule);
/* Sets the launch shape of the renderer's context (kt_context_set_tuning). */
kt_status kt_renderer_set_tuning(kt_renderer* r, const kt_tuning* tuning);
/* Runs kt_context_autotune on the renderer's context and stream for the view `cam` (its
 * built-in candidates); submit_render then uses the installed shape.  Synchronises; call it
 * after kt_renderer_new and before the first frame (a Rust CudaRenderer::new, mod.rs:76-117,
 * would call it once with the config's initial camera). */
kt_status kt_renderer_autotune(kt_renderer* r, const kt_camera* cam, uint32_t reps);
/* The device HDR buffer of a frame (valid until the frame is resubmitted). */
kt_status kt_renderer_frame_hdr(kt_renderer* r, uint32_t index, const float** hdr_dev);
void kt_renderer_destroy(kt_renderer* r);

/* ---- measurement ---------------------------------------------------------------------------- */
/* FP32 FMA throughput of `device` in TFLOP/s (the denominator of the trace's roofline): a
 * kernel of 8 independent FMA chains of `iters` steps per thread, 512-thread blocks filling
 * every SM, best of 5 timed launches (CUDA events) after one warm-up.  Synchronises. */
kt_status kt_fma_peak(int device, uint32_t iters, double* tflops, float* ms);

/* ---- headless mirror of the interactive loop's render policy (src/app.rs) ------------------ */
/* A camera as the app holds it: position, yaw and pitch in degrees, vertical fov in degrees. */
typedef struct kt_view {
    float cam_pos[3];
    float yaw_deg, pitch_deg, fov_deg;
} kt_view;
/* The app's record of the last submitted view (prev_cam_pos/yaw/pitch, prev_fov, has_frame). */
typedef struct kt_view_state {
    kt_view prev;
    int32_t has_frame;
} kt_view_state;
/* App::new (src/app.rs:43-56): prev = the initial view, no frame yet. */
kt_status kt_view_state_init(kt_view_state* s, const kt_view* initial);
/* App::should_render (src/app.rs:184-198): 1 when there is no frame yet, the position moved
 * (f32 length of the difference > 0), yaw or pitch changed by more than 1e-4, or the fov by
 * more than 1e-4; else 0 (and -1 on a NULL argument). */
int32_t kt_should_render(const kt_view_state* s, const kt_view* v);
/* App::update_render_if_needed (src/app.rs:157-182): when kt_should_render, builds the camera
 * (kt_camera_basis, kt_fov_scale) and calls kt_renderer_submit_render; a submitted frame makes
 * v the new prev view.  *submitted = 1 when a frame was submitted. */
kt_status kt_renderer_submit_view(kt_renderer* r, kt_view_state* s, const kt_view* v, int32_t* submitted);
/* The first-frame writer (src/app.rs:219-236): 0x00RRGGBB pixels, rows top to bottom, as an
 * RGBA8 PNG with alpha 255 (stored deflate blocks).  Like the reference it does not replace an
 * existing file: *written = 0 then, 1 when the file was written. */
kt_status kt_write_png(const char* path, const uint32_t* pixels, uint32_t width, uint32_t height,
                       int32_t* written);

/* ---- differentiable trace (discrete adjoint) ------------------------------------------------
 * No counterpart in the reference (its renderer is forward only).  The image is the linear HDR
 * of a stated-physics trace (KT_MODE_SPEC, spp 1, disk noise off, FP32 or FP64) seen by an orbit
 * camera; its parameters theta are the spin, the observer inclination (degrees from the spin
 * axis), a multiplier of the view's base disk temperature scale and the disk outer radius.
 *
 *   kt_diff_forward   renders at theta and records, per ray, every accepted step size and the
 *                     state every 32 accepted steps (the adjoint's checkpoints);
 *   kt_diff_backward  vector-Jacobian product: grad_out[0..3] = d(sum_p dl_dhdr[p] . hdr[p]) /
 *                     d theta for the recorded frozen-step model (step sizes held fixed);
 *   kt_diff_replay    the recorded step sequence at another theta (the frozen-step model whose
 *                     central differences the adjoint matches); flags_out[p] = 1 where the
 *                     ray's events (termination, shaded crossings) differ from the record, so
 *                     that discontinuous pixels can be masked.
 * All three are stream-ordered; the records live in the kt_diff object, sized by
 * segment_capacity (segments of 32 steps; 0 = 4 per pixel).  A ray whose record does not fit
 * renders normally but carries no gradient; kt_diff_get_info reports how many.  The FP64 path
 * takes theta, the camera and the disk LUT in double and accumulates colour in double. */
typedef struct kt_diff kt_diff;
typedef struct kt_diff_params {
    double spin;
    double inclination_deg;
    double temperature_scale;  /* disk_temperature_scale = view.base_temperature_scale * this */
    double disk_outer_radius;
} kt_diff_params;
typedef struct kt_diff_view {
    float observer_r;              /* Kerr-Schild radius of the camera */
    float azimuth_deg;
    float fov_deg;                 /* vertical field of view */
    float base_temperature_scale;
} kt_diff_view;
typedef struct kt_diff_info {
    uint64_t segments_used, segments_capacity;
    uint64_t overflow_rays;  /* rays without a complete record (no gradient) */
    uint64_t record_bytes;   /* bytes of records written by the last forward */
    uint64_t device_bytes;   /* device memory the object holds */
} kt_diff_info;

/* cfg: the fixed scene (resolution, tolerance, LUTs, ...); its spin, disk outer radius and
 * temperature scale are replaced by theta at each call. */
kt_status kt_diff_create(const kt_config* cfg, const kt_diff_view* view, uint32_t segment_capacity, int device,
                         kt_diff** out);
kt_status kt_diff_forward(kt_diff* d, void* stream, const kt_diff_params* theta, float* hdr_out, uint32_t* err_word);
/* hdr64_out: optional (NULL), 3 doubles per pixel: the linear colour before the float store. */
kt_status kt_diff_replay(kt_diff* d, void* stream, const kt_diff_params* theta, float* hdr_out, double* hdr64_out,
                         uint32_t* flags_out, uint32_t* err_word);
/* The recorded step sequence at theta evaluated in double arithmetic (for an FP32 object, its
 * FP32 records replayed in FP64; for an FP64 object, kt_diff_replay).  Central differences of
 * hdr64_out measure the frozen-step model that the FP32 adjoint differentiates without the float
 * rounding of its images.  hdr64_out: 3 doubles per pixel; flags_out (may be NULL) as
 * kt_diff_replay; hdr_out: dev float[4*W*H]. */
kt_status kt_diff_replay_fp64(kt_diff* d, void* stream, const kt_diff_params* theta, double* hdr64_out,
                              uint32_t* flags_out, uint32_t* err_word, float* hdr_out);
/* dl_dhdr: device float4 per pixel (w ignored); grad_out: device, 4 doubles (overwritten). */
kt_status kt_diff_backward(kt_diff* d, void* stream, const float* dl_dhdr, double* grad_out);
/* The adjoint of the model kt_diff_replay_fp64 evaluates: for an FP32 object, its FP32 records
 * (step sizes, shaded crossings) replayed and differentiated in double from the double start of
 * each ray, so that the float rounding of the recorded trajectory does not enter the gradient
 * (the r_out derivative is the most sensitive to it); it costs about as much as the FP64 adjoint.
 * For an FP64 object it is kt_diff_backward.  Arguments as kt_diff_backward; it uploads the
 * double tables of the recorded theta into the buffers that kt_diff_replay_fp64 uses, so the two
 * are ordered on one stream. */
kt_status kt_diff_backward_fp64(kt_diff* d, void* stream, const float* dl_dhdr, double* grad_out);
kt_status kt_diff_get_info(kt_diff* d, kt_diff_info* info);  /* synchronises with the device */
/* The orbit camera of the diff trace and its derivative in the inclination (degrees). */
kt_status kt_diff_orbit_camera(float observer_r, float inclination_deg, float azimuth_deg, float fov_deg,
                               kt_camera* cam, kt_camera* dcam_dincl);
void kt_diff_destroy(kt_diff* d);

#ifdef __cplusplus
}
#endif
#endif /* KERRTRACE_H */
