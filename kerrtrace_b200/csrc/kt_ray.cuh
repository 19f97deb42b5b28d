// kt_ray.cuh — per-ray state machine of the geodesic tracer.
//
// The reference integrates one ray inside a single call (cuda/kerr_trace.cuh:4-240): an outer
// loop over steps, an inner loop over DP5(4) attempts.  Here the same computation is cut at
// attempt granularity: ray_advance() performs exactly one attempt and, when the attempt ends
// the step (accepted, or max_attempts reached), commits it and runs the horizon / disk-plane /
// escape tests.  A warp whose lanes hold rays at different attempt counts therefore keeps all
// lanes busy on the expensive part (six RHS evaluations), and a lane whose ray has ended can be
// refilled with a new ray without waiting for its neighbours.
//
// MODE: 0 reference semantics (LUTs through texture objects), 1 stated physics, 2 reference
// semantics with the LUTs read from plain device arrays through a model of the texture unit.
//
// Arithmetic follows the reference expression by expression; the only behavioural addition is
// retirement of rays whose state has become NaN (see ray_advance), which cannot change the
// output: once y is NaN every later crossing / horizon / escape comparison is false and the
// reference keeps iterating without touching the colour until max_steps.  Scene::keep_frozen
// turns retirement off, so that the reference's schedule of work can be timed as well.
#pragma once
#include "kt_device.cuh"

namespace ktd {

// scene constants in the integration type
template <class R> __device__ __forceinline__ R sc_a(const Scene& s);
template <class R> __device__ __forceinline__ R sc_aa(const Scene& s);
template <class R> __device__ __forceinline__ R sc_M(const Scene& s);
template <class R> __device__ __forceinline__ R sc_h0(const Scene& s);
template <class R> __device__ __forceinline__ R sc_tol(const Scene& s);
template <class R> __device__ __forceinline__ bool inside_horizon(R r, const Scene& s);
template <class R> __device__ __forceinline__ bool beyond_escape(R r, const Scene& s);
template <> __device__ __forceinline__ float sc_a<float>(const Scene& s) { return s.a; }
template <> __device__ __forceinline__ float sc_aa<float>(const Scene& s) { return s.aa; }
template <> __device__ __forceinline__ float sc_M<float>(const Scene& s) { return s.M; }
template <> __device__ __forceinline__ float sc_h0<float>(const Scene& s) { return s.h0; }
template <> __device__ __forceinline__ float sc_tol<float>(const Scene& s) { return s.base_tol; }
template <> __device__ __forceinline__ bool inside_horizon<float>(float r, const Scene& s) { return r < s.horizon_lt; }
template <> __device__ __forceinline__ bool beyond_escape<float>(float r, const Scene& s) { return r > s.escape_gt; }
template <> __device__ __forceinline__ double sc_a<double>(const Scene& s) { return s.a_d; }
template <> __device__ __forceinline__ double sc_aa<double>(const Scene& s) { return s.aa_d; }
template <> __device__ __forceinline__ double sc_M<double>(const Scene& s) { return s.M_d; }
template <> __device__ __forceinline__ double sc_h0<double>(const Scene& s) { return s.h0_d; }
template <> __device__ __forceinline__ double sc_tol<double>(const Scene& s) { return s.base_tol_d; }
template <> __device__ __forceinline__ bool inside_horizon<double>(double r, const Scene& s) { return r < s.horizon_d; }
template <> __device__ __forceinline__ bool beyond_escape<double>(double r, const Scene& s) { return r > s.escape_d; }
// transmittance above the cutoff (float: the exact float form of the reference's compare)
template <class R> __device__ __forceinline__ bool tau_alive(R tau, const Scene& s);
template <> __device__ __forceinline__ bool tau_alive<float>(float tau, const Scene& s) { return tau > s.cutoff_gt; }
template <> __device__ __forceinline__ bool tau_alive<double>(double tau, const Scene& s) { return tau > s.cutoff_d; }

template <class R>
struct RayRun {
    R s[6];      // x, y, z, p_x, p_y, p_z
    R k1[6];     // RHS at s (valid when have_k1)
    R pt, kt, h, tol;
    R col[3];    // colour and transmittance: float on the float paths, double on the FP64 path
    R tau;
    int step;    // committed steps (the reference's loop index i)
    int attempt; // attempts spent on the current step
    bool have_k1;
};

// Work counters of one ray (only maintained by the counting kernels).
// Work counters of one ray, and the first shaded disk hit (only maintained by the counting
// kernels).
struct Tally {
    uint32_t steps, attempts, rhs, frozen, fp64, hits;
    float first_r, first_g, first_T;
    __device__ __forceinline__ void clear() {
        steps = attempts = rhs = frozen = fp64 = hits = 0;
        first_r = first_g = first_T = __int_as_float(0x7fffffff);
    }
};

// Camera ray of sample `sample` of pixel (px, py) (cuda/kernel.cu:108-121): PCG jitter inside
// the pixel, vertical field of view, aspect on u.  Stated-physics mode with one sample uses the
// pixel centre.
template <int MODE>
__device__ __forceinline__ void pixel_ray(int px, int py, int sample, const Scene& sc,
                                          const Camera& cam, float dir[3]) {
    float jx, jy;
    if (MODE == 1 && sc.pixel_centre) {
        jx = 0.5f;
        jy = 0.5f;
    } else {
        const uint32_t pidx = (uint32_t)(py * sc.width + px);
        const uint64_t key = ((uint64_t)pidx << 32) | (uint64_t)(uint32_t)sample;
        jx = unit_float(key);
        jy = unit_float(key ^ 0xda3e39cb94b95bdbULL);
    }
    const float u = ((px + jx) * sc.inv_w_2 - 1.0f) * sc.aspect * cam.fov_scale;
    const float v = (1.0f - (py + jy) * sc.inv_h_2) * cam.fov_scale;
#pragma unroll
    for (int c = 0; c < 3; ++c) dir[c] = u * cam.rgt[c] + v * cam.up[c] + cam.fwd[c];
}

// Null initialisation (cuda/kerr_trace.cuh:14-47): p_t from the null condition with the
// "-sqrt" root, covariant spatial momentum p = n + 2 Hk l (k_t + l.n).  Returns false when
// the step loop would not run at all.
template <class R>
__device__ __forceinline__ bool ray_start(RayRun<R>& ry, const Camera& cam, const float dir[3],
                                          const Scene& sc) {
    using O = Ops<R>;
    const R a = sc_a<R>(sc), aa = sc_aa<R>(sc), M = sc_M<R>(sc);
    const R dx = (R)dir[0], dy = (R)dir[1], dz = (R)dir[2];
    const R inv_n = O::rsq(dx * dx + dy * dy + dz * dz);
    const R nx = dx * inv_n, ny = dy * inv_n, nz = dz * inv_n;
    const R x = (R)cam.pos[0], y = (R)cam.pos[1], z = (R)cam.pos[2];
    const R rho2 = O::fma(x, x, O::fma(y, y, z * z));
    const R u = rho2 - aa;
    const R s_term = O::sqrt_rn(O::fma(u, u, R(4) * aa * y * y));
    const R r2 = R(0.5) * (u + s_term);
    const R r = O::sqrt_rn(r2);
    const R den = r2 + aa;
    const R inv_den = O::fdiv(R(1), den);
    const R lx = (r * x - a * z) * inv_den;
    const R ly = O::fdiv(y, r);
    const R lz = (r * z + a * x) * inv_den;
    const R denH = O::fma(r2, r2, aa * y * y);
    const R Hk = M * r2 * r * O::fdiv(R(1), denH);
    const R ln = O::fma(lx, nx, O::fma(ly, ny, lz * nz));
    const R g_tt = R(-1) + R(2) * Hk;
    const R g_tn = R(2) * Hk * ln;
    const R g_nn = R(1) + R(2) * Hk * ln * ln;
    const R disc = g_tn * g_tn - g_tt * g_nn;
    const R kt = (-g_tn - O::sqrt_rn(disc)) / g_tt;
    const R pt = g_tt * kt + g_tn;
    const R w = kt + ln;
    ry.s[0] = x;
    ry.s[1] = y;
    ry.s[2] = z;
    ry.s[3] = nx + R(2) * Hk * lx * w;
    ry.s[4] = ny + R(2) * Hk * ly * w;
    ry.s[5] = nz + R(2) * Hk * lz * w;
    ry.pt = pt;
    ry.kt = kt;
    ry.h = sc_h0<R>(sc);
    ry.tol = R(0);
    ry.col[0] = ry.col[1] = ry.col[2] = 0.0f;
    ry.tau = 1.0f;
    ry.step = 0;
    ry.attempt = 0;
    ry.have_k1 = false;
    return 0 < sc.max_steps && 1.0f > sc.cutoff_gt;
}

// Tolerance of the step starting at s (cuda/kerr_trace.cuh:67-73): scaled by the Kerr-Schild
// potential from 5x far away down to 0 at Hk >= 0.3 (reference), or down to 1x (stated physics).
// rc is the Kerr-Schild radius of s; the step that ends at s has computed it already for its
// horizon and escape tests (the same ks_radius of the same state), so ray_advance passes that
// value on instead of evaluating it again at the next step's start.
template <class R, int MODE>
__device__ __forceinline__ R step_tolerance_at(R rc, const R* s, const Scene& sc) {
    using O = Ops<R>;
    const R aa = sc_aa<R>(sc), M = sc_M<R>(sc);
    const R rc2 = rc * rc;
    const R denH = O::fma(rc2, rc2, aa * s[1] * s[1]);
    const R Hk = M * rc * rc2 * O::fdiv(R(1), denH);
    R t = O::fdiv(Hk - lit<R>(0.05f, 0.05), lit<R>(0.3f, 0.3) - lit<R>(0.05f, 0.05));
    t = O::minr(O::maxr(t, R(0)), R(1));
    const R base = sc_tol<R>(sc);
    if (MODE != 1) return base * (R(5) - R(5) * t);
    return base * (R(5) - R(4) * t);
}
template <class R, int MODE>
__device__ __forceinline__ R step_tolerance(const R* s, const Scene& sc) {
    return step_tolerance_at<R, MODE>(ks_radius<R>(s[0], s[1], s[2], sc_aa<R>(sc)), s, sc);
}

// Blackbody colour for the FP64 path: software interpolation of the LUT in double.
__device__ __forceinline__ void blackbody_rgb_d(double T, const Scene& sc, uint32_t* err, double c[3]) {
    c[0] = c[1] = c[2] = 0.0;
    if (T > (double)sc.lut_max_temp) {
        if (atomicCAS(err, 0u, 1u) == 0u) err[1] = __float_as_uint((float)T);
        return;
    }
    const int n = sc.lut_size;
    const double pos = T / (double)sc.lut_max_temp * (double)(n - 1);
    const double fl = floor(pos);
    const double flc = fl < -1.0 ? -1.0 : (fl > (double)(n - 1) ? (double)(n - 1) : fl);
    int i0 = fl == fl ? (int)flc : 0;
    int i1 = i0 + 1;
    i0 = i0 < 0 ? 0 : i0;
    i1 = i1 > n - 1 ? n - 1 : i1;
    const double w = pos - fl;
    const float4 a = __ldg(sc.bb_lut + i0), b = __ldg(sc.bb_lut + i1);
    c[0] = (double)a.x + w * ((double)b.x - (double)a.x);
    c[1] = (double)a.y + w * ((double)b.y - (double)a.y);
    c[2] = (double)a.z + w * ((double)b.z - (double)a.z);
}

// Root of y(t) = 0 on the dense output (stated physics): safeguarded Newton with bisection
// fallback, starting from the secant guess.  This is what cuda/kerr_trace.cuh:147-168 intends.
template <class R>
__device__ __forceinline__ R crossing_root(R y0, R y1, R k1, R k3, R k4, R k5, R k6, R k7, R h,
                                           R t0) {
    using O = Ops<R>;
    R lo = R(0), hi = R(1), t = t0;
    const bool neg0 = y0 < R(0);
#pragma unroll 1
    for (int it = 0; it < 12; ++it) {
        const R yt = dense_eval<R>(y0, y1, k1, k3, k4, k5, k6, k7, h, t);
        if (yt == R(0)) break;
        if ((yt < R(0)) == neg0) lo = t; else hi = t;
        const R dyt = dense_slope<R>(y0, y1, k1, k3, k4, k5, k6, k7, h, t);
        R tn = dyt != R(0) ? t - yt / dyt : R(0.5) * (lo + hi);
        // a converged update (tn == t on the bracket end) is kept: the step is then 0 and the
        // loop ends; only steps leaving the bracket bisect
        if (!(tn >= lo && tn <= hi)) tn = R(0.5) * (lo + hi);
        const R step = O::absr(tn - t);
        t = tn;
        if (step <= lit<R>(1e-7f, 1e-15)) break;
    }
    return t;
}

// Shading of a disk-plane hit `hit` (the state on the dense output at the crossing)
// (cuda/kerr_trace.cuh:167-228): Novikov-Thorne disk test, redshift g, temperature from the disk
// LUT (with FBM modulation), blackbody colour and alpha compositing into col / tau.
template <class R, int MODE>
__device__ __forceinline__ void shade_hit(const R* hit, R pt, R kt, R* col, R& tau, const Scene& sc,
                                          uint32_t* err, Tally* tl) {
    using O = Ops<R>;
    const R a = sc_a<R>(sc), aa = sc_aa<R>(sc), M = sc_M<R>(sc);
    const R xh = hit[0], zh = hit[2], pxh = hit[3], pyh = hit[4], pzh = hit[5];
    R rh = ks_radius<R>(xh, R(0), zh, aa);
    const R r_in = sizeof(R) == 8 ? (R)sc.disk_inner_d : (R)sc.disk_inner;
    const R r_out = sizeof(R) == 8 ? (R)sc.disk_outer_d : (R)sc.disk_outer;
    if (!(rh >= r_in && rh <= r_out)) return;
    const R sqM = O::sqrt_rn(M), rs = O::sqrt_rn(rh);
    const R disc = R(1) - R(3) * M / rh + R(2) * a * sqM / (rh * rs);
    if (!(disc > R(0))) return;
    const R omega = -sqM / (rh * rs + a * sqM);
    const R r2h = rh * rh;
    const R inv = O::fdiv(R(1), r2h + aa);
    const R lx = (rh * xh - a * zh) * inv;
    const R ly = R(0);
    const R lz = (rh * zh + a * xh) * inv;
    const R ldotp = O::fma(lx, pxh, O::fma(ly, pyh, lz * pzh));
    const R ldotxi = lx * zh - lz * xh;
    const R denH = r2h * r2h;
    const R Hk = M * rh * r2h * O::fdiv(R(1), denH);
    const R L = (zh * pxh - xh * pzh) + R(2) * Hk * ldotxi * (ldotp + kt);
    const R energy = -pt;
    const R l_over_e = O::fdiv(L, energy);
    const R g = R(1) / (O::rsq(disc) * (R(1) - omega * l_over_e));
    const R span = r_out - r_in;
    const R u = span > R(0) ? (rh - r_in) / span : R(0);
    R sampled;
    if constexpr (sizeof(R) == 4) {
        if (MODE == 0) sampled = tex1D<float>(sc.disk_tex, u);
        else if (MODE == 2) sampled = lut_tex_model1(sc.disk_lut, sc.lut_size, u);
        else sampled = lut_lerp1<float>(sc.disk_lut, sc.lut_size, u);
    } else {
        sampled = sc.disk_lut_d ? lut_lerp1<double, double>(sc.disk_lut_d, sc.lut_size, u)
                                : lut_lerp1<double>(sc.disk_lut, sc.lut_size, u);
    }
    // CONFIG_DISK_TEMPERATURE_SCALE is a double literal in the reference: the product is double
    double Td = sc.temp_scale * (double)sampled * (double)g;
    R T = (R)Td;
    if (sc.noise_enabled && sc.noise_detail > 0 && sc.noise_strength != 0.0f) {
        R r_bl, sn_th, cs_th, phi;
        const R inv_M = sizeof(R) == 4 ? (R)sc.inv_M : R(1) / M;
        ks_to_bl<R>(xh, R(0), zh, a, aa, r_bl, sn_th, cs_th, phi);
        rh = r_bl;  // the reference's ks_bl_from_xyz writes back into r_hit
        const R r3 = rh * rh * rh;
        const R om = R(1) / (a + O::sqrt_rn(r3 * inv_M));
        R phase = phi + (R)sc.noise_winding * om;
        if (MODE == 1) phase += (R)sc.noise_phase;
        R sp, cp;
        O::sincosr(phase, &sp, &cp);
        const R nu = rh * cp * (R)sc.noise_scale;
        const R nv = rh * sp * (R)sc.noise_scale;
        const R nval = fbm2<R>(nu, nv, sc.noise_detail, MODE == 1 ? sc.noise_seed : 0u);
        const R modulator = R(1) + (R)sc.noise_strength * (nval - R(0.5));
        T *= modulator;
    }
    if (tl && tl->hits == 0) {
        tl->first_r = (float)rh;
        tl->first_g = (float)g;
        tl->first_T = (float)T;
    }
    if (O::isfiniter(T) && T > R(0)) {
        if (tl) tl->hits++;
        if constexpr (sizeof(R) == 4) {
            const float3 c = blackbody_rgb<MODE>(T, sc, err);
            const float luma = 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z;
            const float luma_s = (float)((double)luma / sc.wl_step);
            const float alpha = 1.0f - __expf(-luma_s * 0.5f);
            col[0] += c.x * alpha * tau;
            col[1] += c.y * alpha * tau;
            col[2] += c.z * alpha * tau;
            tau *= (1.0f - alpha);
        } else {
            double c[3];
            blackbody_rgb_d(T, sc, err, c);
            const double luma = 0.2126 * c[0] + 0.7152 * c[1] + 0.0722 * c[2];
            const double luma_s = luma / sc.wl_step;
            const double alpha = 1.0 - exp(-luma_s * 0.5);
            col[0] += c[0] * alpha * tau;
            col[1] += c[1] * alpha * tau;
            col[2] += c[2] * alpha * tau;
            tau *= 1.0 - alpha;
        }
    }
}

// Disk-plane crossing between prev and cur (cuda/kerr_trace.cuh:138-228): the hit point on the
// dense output (reference semantics: the linear guess, kerr_trace.cuh:150-166; stated physics:
// refined by the safeguarded Newton root), then shade_hit.
template <class R, int MODE>
__device__ __forceinline__ void shade_crossing(RayRun<R>& ry, const R* prev, const R* k1,
                                               const R* k3, const R* k4, const R* k5,
                                               const R* k6, const R* k7, R h, const Scene& sc,
                                               uint32_t* err, Tally* tl) {
    using O = Ops<R>;
    const R y0 = prev[1], y1 = ry.s[1];
    const R dy = y0 - y1;
    R t = dy != R(0) ? O::fdiv(y0, dy) : R(0.5);
    t = O::minr(O::maxr(t, R(0)), R(1));
    if (MODE == 1) t = crossing_root<R>(y0, y1, k1[1], k3[1], k4[1], k5[1], k6[1], k7[1], h, t);
    R hit[6];
#pragma unroll
    for (int c = 0; c < 6; ++c)
        hit[c] = dense_eval<R>(prev[c], ry.s[c], k1[c], k3[c], k4[c], k5[c], k6[c], k7[c], h, t);
    shade_hit<R, MODE>(hit, ry.pt, ry.kt, ry.col, ry.tau, sc, err, tl);
}

// One DP5(4) attempt; on the last attempt of a step, the commit and the per-step tests.
// Returns true when the ray has finished (its colour is final).
template <class R, int MODE, bool COUNT>
__device__ __forceinline__ bool ray_advance(RayRun<R>& ry, const Scene& sc, uint32_t* err,
                                            Tally& tl) {
    constexpr bool EXACT = MODE == 1;
    using O = Ops<R>;
    using C = DP<R>;
    const R a = sc_a<R>(sc), aa = sc_aa<R>(sc), M = sc_M<R>(sc);
    // the first step's tolerance; later steps get theirs from the commit of the step before
    if (ry.attempt == 0 && ry.step == 0) ry.tol = step_tolerance<R, MODE>(ry.s, sc);
    if (!ry.have_k1) {
        hamilton_rhs<R, EXACT>(ry.s, ry.pt, a, aa, M, ry.k1);
        ry.have_k1 = true;
        if (COUNT) tl.rhs++;
    }
    const R h = ry.h;
    const R* s = ry.s;
    const R* k1 = ry.k1;
    R y[6], k2[6], k3[6], k4[6], k5[6], k6[6], k7[6], nx[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) y[c] = s[c] + h * C::a21 * k1[c];
    hamilton_rhs<R, EXACT>(y, ry.pt, a, aa, M, k2);
#pragma unroll
    for (int c = 0; c < 6; ++c) y[c] = s[c] + h * (C::a31 * k1[c] + C::a32 * k2[c]);
    hamilton_rhs<R, EXACT>(y, ry.pt, a, aa, M, k3);
#pragma unroll
    for (int c = 0; c < 6; ++c) y[c] = s[c] + h * (C::a41 * k1[c] + C::a42 * k2[c] + C::a43 * k3[c]);
    hamilton_rhs<R, EXACT>(y, ry.pt, a, aa, M, k4);
#pragma unroll
    for (int c = 0; c < 6; ++c)
        y[c] = s[c] + h * (C::a51 * k1[c] + C::a52 * k2[c] + C::a53 * k3[c] + C::a54 * k4[c]);
    hamilton_rhs<R, EXACT>(y, ry.pt, a, aa, M, k5);
#pragma unroll
    for (int c = 0; c < 6; ++c)
        y[c] = s[c] + h * (C::a61 * k1[c] + C::a62 * k2[c] + C::a63 * k3[c] + C::a64 * k4[c] +
                           C::a65 * k5[c]);
    hamilton_rhs<R, EXACT>(y, ry.pt, a, aa, M, k6);
    // 5th-order solution; its stage-7 input is the same expression (a7j = b_j), so k7 is FSAL
#pragma unroll
    for (int c = 0; c < 6; ++c)
        nx[c] = s[c] + h * (C::b1 * k1[c] + C::b3 * k3[c] + C::b4 * k4[c] + C::b5 * k5[c] +
                            C::b6 * k6[c]);
    hamilton_rhs<R, EXACT>(nx, ry.pt, a, aa, M, k7);
    // max-norm of the embedded error, per-component scale tol * max(|y_i|, 1)
    R e[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        const R scale = ry.tol * O::maxr(O::absr(s[c]), R(1));
        e[c] = O::absr(h * (C::e1 * k1[c] + C::e3 * k3[c] + C::e4 * k4[c] + C::e5 * k5[c] +
                            C::e6 * k6[c] + C::e7 * k7[c])) / scale;
    }
    const R errv = O::maxr(O::maxr(O::maxr(e[0], e[1]), O::maxr(e[2], e[3])), O::maxr(e[4], e[5]));
    const bool ok = errv <= R(1);
    ry.h = h * lit<R>(0.9f, 0.9) * O::powr(errv, lit<R>(-0.2f, -0.2));
    ry.attempt++;
    if (COUNT) {
        tl.attempts++;
        tl.rhs += 6;
    }
    if (!ok && ry.attempt < sc.max_attempts) return false;  // retry; k1 stays valid at s

    // commit (also when every attempt was rejected: cuda/kerr_trace.cuh:123-134)
    R prev[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        prev[c] = ry.s[c];
        ry.s[c] = nx[c];
    }
    ry.attempt = 0;
    if (COUNT) tl.steps++;
    if (O::isnanr(ry.s[1])) {  // frozen: no later comparison can succeed (see file comment)
        if (COUNT) tl.frozen = 1;
        if (!sc.keep_frozen) return true;
    }
    const R r_now = ks_radius<R>(ry.s[0], ry.s[1], ry.s[2], aa);
    if (inside_horizon<R>(r_now, sc)) return true;
    if ((prev[1] < R(0) && ry.s[1] >= R(0)) || (prev[1] > R(0) && ry.s[1] <= R(0)))
        shade_crossing<R, MODE>(ry, prev, ry.k1, k3, k4, k5, k6, k7, h, sc, err, COUNT ? &tl : nullptr);
    if (ok) {
#pragma unroll
        for (int c = 0; c < 6; ++c) ry.k1[c] = k7[c];
        ry.have_k1 = true;
    } else {
        ry.have_k1 = false;
    }
    if (beyond_escape<R>(r_now, sc)) {
        R ke[6];
        hamilton_rhs<R, EXACT>(ry.s, ry.pt, a, aa, M, ke);
        if (COUNT) tl.rhs++;
        const R inv = O::rsq(ke[0] * ke[0] + ke[1] * ke[1] + ke[2] * ke[2]);
        const R sky = sky_value<R>(ke[0] * inv, ke[1] * inv, ke[2] * inv, ry.tau, sc);
        ry.col[0] += sky;
        ry.col[1] += sky;
        ry.col[2] += sky;
        return true;
    }
    ry.step++;
    const bool done = !(ry.step < sc.max_steps && tau_alive<R>(ry.tau, sc));
    if (!done) ry.tol = step_tolerance_at<R, MODE>(r_now, ry.s, sc);
    return done;
}

// =========================================================================================
// Mixed precision (stated physics only).  The state is a float pair: hi carries every FP32
// computation (right-hand sides, stages, tests), lo the rounding error of hi.  Outside the
// photon zone (Kerr-Schild radius of the step start >= sc.zone_r, 1.5 x the retrograde
// photon-orbit radius, which contains the horizon) the state update x + h sum b_i k_i is a
// compensated FP32 sum: Knuth's TwoSum of hi and the increment (plus the carried lo) gives the
// new hi and its exact rounding error, so the rounding of the update, which at tight
// tolerances is the floor of an FP32 trace that starts far out, does not accumulate.  Inside
// the zone the update runs in FP64 on hi + lo, every kRenormEvery-th accepted step renormalises
// p onto the null cone in FP64, and the result is split back into hi and lo.  The embedded error norm runs in FP64 when the tolerance is below
// 3e-7 (sc.zone_err64): the FP32 stage sum carries an absolute error of about
// 6e-9 h |k|, under 1% of the tolerance scale above that.  A crossing is located in FP32, its
// root refined by FP64 Newton steps on the hi + lo dense output, and the hit shaded in FP32.
// =========================================================================================
struct Mixed {};
constexpr int kRenormEvery = 8;

template <>
struct RayRun<Mixed> {
    float s[6];   // hi
    float lo[6];  // rounding error of hi (compensated update outside the zone, FP64 split inside)
    float k1[6];
    double pt, kt;
    float h, tol;
    float col[3];
    float tau;
    int step, attempt;
    bool have_k1, zone;
};

// FP64 reciprocal and reciprocal square root without the long-latency IEEE sequences: the FP32
// hardware approximation as the seed, then two Newton-Raphson steps (r <- r + r (1 - x r) and
// y <- y + y (1/2 - x y^2 / 2)); each step doubles the correct bits, 22 -> 44 -> beyond 53.
// Valid for |x| within the FP32 range, which holds for every quantity they are used on here.
__device__ __forceinline__ double rcp_nr(double x) {
    double r = (double)__fdividef(1.0f, (float)x);
    r = fma(r, fma(-x, r, 1.0), r);
    return fma(r, fma(-x, r, 1.0), r);
}
__device__ __forceinline__ double rsqrt_nr(double x) {
    double y = (double)rsqrtf((float)x);
    const double hx = 0.5 * x;
    y = fma(y, fma(-hx * y, y, 0.5), y);
    return fma(y, fma(-hx * y, y, 0.5), y);
}

// Rescales p onto the null cone: with H(p) = (|p|^2 - pt^2 - 2 Hk (l.p - pt)^2) / 2 and
// p -> lambda p, H is A lambda^2 + B lambda + C with A = |p|^2 - 2 Hk (l.p)^2,
// B = 4 Hk pt (l.p), C = -pt^2 (1 + 2 Hk).  One Newton step from lambda = 1,
// lambda = 1 - (A + B + C) / (2A + B), removes the drift of an accurate step (the residual is
// quadratic in it).  No change unless the correction is below 1e-3.
__device__ __forceinline__ void null_renormalise(double* s, double pt, const Scene& sc) {
    const double a = sc.a_d, aa = sc.aa_d, M = sc.M_d;
    const double x = s[0], y = s[1], z = s[2];
    const double rho2 = x * x + y * y + z * z;
    const double u = rho2 - aa;
    const double q = u * u + 4.0 * aa * y * y;
    const double r2 = 0.5 * (u + q * rsqrt_nr(q));
    const double inv_r = rsqrt_nr(r2);
    const double r = r2 * inv_r;
    const double inv_D = rcp_nr(r2 + aa);
    const double lx = (r * x - a * z) * inv_D, ly = y * inv_r, lz = (r * z + a * x) * inv_D;
    const double Hk = M * r2 * r * rcp_nr(r2 * r2 + aa * y * y);
    const double lp = lx * s[3] + ly * s[4] + lz * s[5];
    const double pp = s[3] * s[3] + s[4] * s[4] + s[5] * s[5];
    const double A = pp - 2.0 * Hk * lp * lp;
    const double B = 4.0 * Hk * pt * lp;
    const double Cq = -pt * pt * (1.0 + 2.0 * Hk);
    const double den = 2.0 * A + B;
    if (!(den != 0.0)) return;
    const double dl = -(A + B + Cq) * rcp_nr(den);
    if (!(fabs(dl) < 1e-3)) return;
    const double lam = 1.0 + dl;
    s[3] *= lam;
    s[4] *= lam;
    s[5] *= lam;
}

// The start is the FP32 start (the camera and direction are FP32 data; it runs once per ray in
// the refill path, where FP64 square roots and divisions would cost as much as the ray's steps).
__device__ __forceinline__ bool ray_start_mixed(RayRun<Mixed>& ry, const Camera& cam, const float dir[3],
                                                const Scene& sc) {
    RayRun<float> d;
    const bool run = ray_start<float>(d, cam, dir, sc);
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        ry.s[c] = d.s[c];
        ry.lo[c] = 0.0f;
    }
    ry.pt = (double)d.pt;
    ry.kt = (double)d.kt;
    ry.h = d.h;
    ry.tol = 0.0f;
    ry.col[0] = ry.col[1] = ry.col[2] = 0.0f;
    ry.tau = 1.0f;
    ry.step = 0;
    ry.attempt = 0;
    ry.have_k1 = false;
    ry.zone = false;
    return run;
}

// Disk crossing of a mixed-precision step.  Kept out of line: it runs on few steps and would
// otherwise raise the register count of the whole loop.  Everything it reads or writes is
// passed through small arrays that the caller fills only when it calls, so that the ray state
// of the stepping loop never has its address taken (which would move it to local memory).
// q rows: k1, k3, k4, k5, k6, k7, then hi and lo of the step start and of the step end; tc: the
// FP32 root; ct: colour and transmittance, updated.  Two FP64 Newton steps on the hi + lo dense
// output take the root to FP64 accuracy; the hit is then shaded in FP32.
static __device__ __noinline__ void shade_mixed(const float (*q)[6], float h, float tc, double ptd, double ktd,
                                                const Scene& sc, uint32_t* err, Tally* tl, float* ct) {
    const float (*ks)[6] = q;
    double y0[6], y1[6];
    for (int c = 0; c < 6; ++c) {
        y0[c] = (double)q[6][c] + (double)q[7][c];
        y1[c] = (double)q[8][c] + (double)q[9][c];
    }
    const double hd = (double)h;
    double t = (double)tc;
    for (int it = 0; it < 2; ++it) {
        const double yt = dense_eval<double>(y0[1], y1[1], ks[0][1], ks[1][1], ks[2][1], ks[3][1], ks[4][1],
                                             ks[5][1], hd, t);
        const double dyt = dense_slope<double>(y0[1], y1[1], ks[0][1], ks[1][1], ks[2][1], ks[3][1], ks[4][1],
                                               ks[5][1], hd, t);
        if (!(fabs(dyt) > 0.0)) break;
        t = fmin(fmax(t - yt / dyt, 0.0), 1.0);
    }
    float hit[6];
    for (int c = 0; c < 6; ++c)
        hit[c] = (float)dense_eval<double>(y0[c], y1[c], ks[0][c], ks[1][c], ks[2][c], ks[3][c], ks[4][c],
                                           ks[5][c], hd, t);
    shade_hit<float, 1>(hit, (float)ptd, (float)ktd, ct, ct[3], sc, err, tl);
}

template <int MODE, bool COUNT>
__device__ __forceinline__ bool ray_advance_mixed(RayRun<Mixed>& ry, const Scene& sc, uint32_t* err,
                                                  Tally& tl) {
    constexpr bool EXACT = true;
    using O = Ops<float>;
    using C = DP<float>;
    using CD = DP<double>;
    const float a = sc.a, aa = sc.aa, M = sc.M;
    const float pt = (float)ry.pt;
    if (ry.attempt == 0 && ry.step == 0) {  // later steps: set by the commit of the step before
        const float rc = ks_radius<float>(ry.s[0], ry.s[1], ry.s[2], aa);
        ry.tol = step_tolerance_at<float, 1>(rc, ry.s, sc);
        ry.zone = rc < sc.zone_r;
    }
    if (!ry.have_k1) {
        hamilton_rhs<float, EXACT>(ry.s, pt, a, aa, M, ry.k1);
        ry.have_k1 = true;
        if (COUNT) tl.rhs++;
    }
    const float h = ry.h;
    const float* s = ry.s;
    const float* k1 = ry.k1;
    float y[6], k2[6], k3[6], k4[6], k5[6], k6[6], k7[6], nx[6], inc[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) y[c] = s[c] + h * C::a21 * k1[c];
    hamilton_rhs<float, EXACT>(y, pt, a, aa, M, k2);
#pragma unroll
    for (int c = 0; c < 6; ++c) y[c] = s[c] + h * (C::a31 * k1[c] + C::a32 * k2[c]);
    hamilton_rhs<float, EXACT>(y, pt, a, aa, M, k3);
#pragma unroll
    for (int c = 0; c < 6; ++c) y[c] = s[c] + h * (C::a41 * k1[c] + C::a42 * k2[c] + C::a43 * k3[c]);
    hamilton_rhs<float, EXACT>(y, pt, a, aa, M, k4);
#pragma unroll
    for (int c = 0; c < 6; ++c)
        y[c] = s[c] + h * (C::a51 * k1[c] + C::a52 * k2[c] + C::a53 * k3[c] + C::a54 * k4[c]);
    hamilton_rhs<float, EXACT>(y, pt, a, aa, M, k5);
#pragma unroll
    for (int c = 0; c < 6; ++c)
        y[c] = s[c] + h * (C::a61 * k1[c] + C::a62 * k2[c] + C::a63 * k3[c] + C::a64 * k4[c] + C::a65 * k5[c]);
    hamilton_rhs<float, EXACT>(y, pt, a, aa, M, k6);
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        inc[c] = C::b1 * k1[c] + C::b3 * k3[c] + C::b4 * k4[c] + C::b5 * k5[c] + C::b6 * k6[c];
        nx[c] = s[c] + h * inc[c];
    }
    hamilton_rhs<float, EXACT>(nx, pt, a, aa, M, k7);
    float errv;
    if (COUNT && ry.zone) tl.fp64++;
    if (ry.zone && sc.zone_err64) {
        double em = 0.0;
        bool any = false;
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            const double e = (double)h * (CD::e1 * (double)k1[c] + CD::e3 * (double)k3[c] + CD::e4 * (double)k4[c] +
                                          CD::e5 * (double)k5[c] + CD::e6 * (double)k6[c] + CD::e7 * (double)k7[c]);
            // the FP64 part is the stage sum, where the terms cancel; the scaling is FP32
            const float scale = ry.tol * O::maxr(O::absr(s[c]), 1.0f);
            const double ec = fabs(e) * (double)__fdividef(1.0f, scale);
            if (ec == ec) {
                em = any ? fmax(em, ec) : ec;
                any = true;
            }
        }
        errv = any ? (float)em : __int_as_float(0x7fffffff);
    } else {
        float e[6];
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            const float scale = ry.tol * O::maxr(O::absr(s[c]), 1.0f);
            e[c] = O::absr(h * (C::e1 * k1[c] + C::e3 * k3[c] + C::e4 * k4[c] + C::e5 * k5[c] + C::e6 * k6[c] +
                                C::e7 * k7[c])) / scale;
        }
        errv = O::maxr(O::maxr(O::maxr(e[0], e[1]), O::maxr(e[2], e[3])), O::maxr(e[4], e[5]));
    }
    const bool ok = errv <= 1.0f;
    ry.h = h * 0.9f * O::powr(errv, -0.2f);
    ry.attempt++;
    if (COUNT) {
        tl.attempts++;
        tl.rhs += 6;
    }
    if (!ok && ry.attempt < sc.max_attempts) return false;

    float prev[6], prev_lo[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        prev[c] = ry.s[c];
        prev_lo[c] = ry.lo[c];
    }
    if (ry.zone) {
        double nd[6];
#pragma unroll
        for (int c = 0; c < 6; ++c) nd[c] = ((double)prev[c] + (double)prev_lo[c]) + (double)h * (double)inc[c];
        if (ok && ry.step % kRenormEvery == 0) null_renormalise(nd, ry.pt, sc);
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            ry.s[c] = (float)nd[c];
            ry.lo[c] = (float)(nd[c] - (double)ry.s[c]);
        }
    } else {
        // TwoSum(hi, d) with d = h inc + lo: sum + e == hi + d exactly (round-to-nearest
        // additions, written as intrinsics so that nothing contracts or reorders them)
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            const float d = fmaf(h, inc[c], prev_lo[c]);
            const float sum = __fadd_rn(prev[c], d);
            const float bv = __fsub_rn(sum, prev[c]);
            ry.lo[c] = __fadd_rn(__fsub_rn(prev[c], __fsub_rn(sum, bv)), __fsub_rn(d, bv));
            ry.s[c] = sum;
        }
    }
    ry.attempt = 0;
    if (COUNT) tl.steps++;
    if (O::isnanr(ry.s[1])) {
        if (COUNT) tl.frozen = 1;
        if (!sc.keep_frozen) return true;
    }
    const float r_now = ks_radius<float>(ry.s[0], ry.s[1], ry.s[2], aa);
    if (inside_horizon<float>(r_now, sc)) return true;
    bool near_disk = false;
    float tc = 0.5f;
    if ((prev[1] < 0.0f && ry.s[1] >= 0.0f) || (prev[1] > 0.0f && ry.s[1] <= 0.0f)) {
        // FP32 estimate of the hit radius first: the FP64 root and shading only run for
        // crossings that can land on the disk (1e-3 margin on both radii)
        const float dyc = prev[1] - ry.s[1];
        tc = dyc != 0.0f ? __fdividef(prev[1], dyc) : 0.5f;
        tc = fminf(fmaxf(tc, 0.0f), 1.0f);
        tc = crossing_root<float>(prev[1], ry.s[1], k1[1], k3[1], k4[1], k5[1], k6[1], k7[1], h, tc);
        const float xc = dense_eval<float>(prev[0], ry.s[0], k1[0], k3[0], k4[0], k5[0], k6[0], k7[0], h, tc);
        const float zc = dense_eval<float>(prev[2], ry.s[2], k1[2], k3[2], k4[2], k5[2], k6[2], k7[2], h, tc);
        const float rc = ks_radius<float>(xc, 0.0f, zc, aa);
        near_disk = rc >= sc.disk_inner * 0.999f && rc <= sc.disk_outer * 1.001f;
    }
    if (near_disk) {
        float q[10][6], ct[4];
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            q[0][c] = k1[c];
            q[1][c] = k3[c];
            q[2][c] = k4[c];
            q[3][c] = k5[c];
            q[4][c] = k6[c];
            q[5][c] = k7[c];
            q[6][c] = prev[c];
            q[7][c] = prev_lo[c];
            q[8][c] = ry.s[c];
            q[9][c] = ry.lo[c];
        }
        ct[0] = ry.col[0];
        ct[1] = ry.col[1];
        ct[2] = ry.col[2];
        ct[3] = ry.tau;
        if (COUNT) {
            Tally t2 = tl;
            shade_mixed(q, h, tc, ry.pt, ry.kt, sc, err, &t2, ct);
            tl = t2;
        } else {
            shade_mixed(q, h, tc, ry.pt, ry.kt, sc, err, nullptr, ct);
        }
        ry.col[0] = ct[0];
        ry.col[1] = ct[1];
        ry.col[2] = ct[2];
        ry.tau = ct[3];
    }
    if (ok) {
#pragma unroll
        for (int c = 0; c < 6; ++c) ry.k1[c] = k7[c];
        ry.have_k1 = true;
    } else {
        ry.have_k1 = false;
    }
    if (beyond_escape<float>(r_now, sc)) {
        float ke[6];
        hamilton_rhs<float, EXACT>(ry.s, pt, a, aa, M, ke);
        if (COUNT) tl.rhs++;
        const float inv = O::rsq(ke[0] * ke[0] + ke[1] * ke[1] + ke[2] * ke[2]);
        const float sky = sky_value<float>(ke[0] * inv, ke[1] * inv, ke[2] * inv, ry.tau, sc);
        ry.col[0] += sky;
        ry.col[1] += sky;
        ry.col[2] += sky;
        return true;
    }
    ry.step++;
    const bool done = !(ry.step < sc.max_steps && ry.tau > sc.cutoff_gt);
    if (!done) {
        ry.tol = step_tolerance_at<float, 1>(r_now, ry.s, sc);
        ry.zone = r_now < sc.zone_r;
    }
    return done;
}

// Uniform entry points used by the kernels for every arithmetic type.
template <class R>
__device__ __forceinline__ bool start(RayRun<R>& ry, const Camera& cam, const float dir[3], const Scene& sc) {
    return ray_start<R>(ry, cam, dir, sc);
}
__device__ __forceinline__ bool start(RayRun<Mixed>& ry, const Camera& cam, const float dir[3], const Scene& sc) {
    return ray_start_mixed(ry, cam, dir, sc);
}
template <int MODE, bool COUNT, class R>
__device__ __forceinline__ bool advance(RayRun<R>& ry, const Scene& sc, uint32_t* err, Tally& tl) {
    return ray_advance<R, MODE, COUNT>(ry, sc, err, tl);
}
template <int MODE, bool COUNT>
__device__ __forceinline__ bool advance(RayRun<Mixed>& ry, const Scene& sc, uint32_t* err, Tally& tl) {
    return ray_advance_mixed<MODE, COUNT>(ry, sc, err, tl);
}

}  // namespace ktd
