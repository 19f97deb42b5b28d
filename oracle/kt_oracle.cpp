// kt_oracle.cpp — CPU oracle of the KerrTrace hot path.  TEST INFRASTRUCTURE ONLY.
//
// This library is the checker: tests/, __graft_entry__.smoke() and the CPU-baseline leg of
// bench.py call it to produce the expected results.  The product (kerrtrace_b200) never links
// or calls it.
//
// It restates the reference's algorithm in plain C++, templated on the arithmetic type:
//   T = double : the f64 oracle
//   T = float  : an f32 emulation with correctly rounded operations in place of the GPU's
//                approximate intrinsics (rsqrtf, __fdividef, __powf, __expf, __sincosf)
// Sources followed (reference file:line):
//   ks_radius           cuda/kerr_math.cuh:50-59
//   bl_angles           cuda/kerr_math.cuh:60-81
//   hamilton_rhs        cuda/kerr_math.cuh:82-156
//   sky                 cuda/kerr_math.cuh:157-171
//   dense / dense_slope cuda/kerr_math.cuh:186-219
//   pcg32, noise, fbm   cuda/kerr_math.cuh:26-36, 172-179, 220-281
//   trace_ray           cuda/kerr_trace.cuh:4-240
//   lut fetch           cuda/kernel.cu:1-16 (+ texture sampling of src/renderer/texture.rs:176-202)
//   pixel loop          cuda/kernel.cu:88-142
//   bloom, tone map     cuda/kernel.cu:17-84, 144-251
//   params, ISCO, LUTs  src/renderer/utils.rs:11-113,172-201; src/renderer/blackbody.rs:6-124
//   define values       src/renderer/utils.rs:115-163 ({:.10} formatting -> double literal)
// Quirks of the reference reproduced in reference mode (mode 0): linear-guess crossing root
// (the Newton loop at kerr_trace.cuh:147-168 assigns a shadowing local), tolerance that is 0
// for Hk >= 0.3, rejected steps committed after max_attempts, jittered samples at spp = 1,
// unthresholded bloom.  Mode 1 ("stated physics") uses a safeguarded Newton root, a tolerance
// floor of 1x, pixel centres at spp = 1, seed/phase in the FBM and a bloom threshold.
//
// Texture sampling: hardware linear filtering uses a 1.8 fixed-point weight (CUDA C
// Programming Guide, texture fetching appendix).  tex_mode 0 uses the exact weight, 1 rounds
// the weight to 1/256, 2 truncates it.
#include <algorithm>
#include <charconv>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {

// Everything the oracle needs to trace one frame.  Derived quantities (ISCO, r_h, 2/W, ...)
// are computed by the oracle itself from these inputs.
typedef struct kto_scene {
    uint32_t width, height;
    float spin, mass;
    uint32_t spp, sky_grid_divisions, max_steps, max_attempts;
    float exposure_scale, sky_line_thickness, sky_intensity;
    float disk_outer_radius, disk_temperature_scale;
    float initial_step, tolerance, transmittance_cutoff, horizon_epsilon, escape_radius;
    float wavelength_step;
    int32_t noise_enabled;
    float noise_scale, noise_strength, noise_winding;
    uint32_t noise_detail;
    uint32_t lut_size;
    float lut_max_temp;
    const float* bb_lut;    // lut_size x 4
    const float* disk_lut;  // lut_size
    int32_t mode;           // 0 reference semantics, 1 stated physics
    int32_t tex_mode;       // 0 exact weight, 1 weight rounded to 1/256, 2 truncated
    int32_t retire_frozen;  // stop rays whose state is NaN (output-identical)
    uint32_t noise_seed;
    float noise_phase;
    float cam_pos[3], fwd[3], rgt[3], up[3];
    float fov_scale;
} kto_scene;

// Per-ray record (sample 0 of each traced pixel).
typedef struct kto_ray_info {
    int32_t term;       // 0 step budget / transmittance, 1 horizon, 2 escape, 3 frozen (NaN)
    int32_t hits;       // disk crossings that shaded
    int32_t crossings;  // y sign changes
    int32_t steps;
    int32_t attempts;
    int32_t rhs;
    double first_r;     // Kerr-Schild radius of the first shaded disk hit (NaN if none)
    double first_g;     // redshift factor g of that hit
    double first_T;     // temperature of that hit
} kto_ray_info;

}  // extern "C"

namespace {

template <class T> struct M;
template <> struct M<double> {
    static double rsq(double x) { return 1.0 / std::sqrt(x); }
    static double fdiv(double a, double b) { return a / b; }
    static double sqrt_(double x) { return std::sqrt(x); }
    static double fma_(double a, double b, double c) { return std::fma(a, b, c); }
    static double pow_(double a, double b) { return std::pow(a, b); }
    static double exp_(double a) { return std::exp(a); }
    static void sincos_(double a, double* s, double* c) { *s = std::sin(a); *c = std::cos(a); }
    static double atan2_(double y, double x) { return std::atan2(y, x); }
    static double asin_(double x) { return std::asin(x); }
    static double fmod_(double a, double b) { return std::fmod(a, b); }
    static constexpr double lit(float, double d) { return d; }
};
template <> struct M<float> {
    static float rsq(float x) { return 1.0f / std::sqrt(x); }
    static float fdiv(float a, float b) { return a / b; }
    static float sqrt_(float x) { return std::sqrt(x); }
    static float fma_(float a, float b, float c) { return std::fma(a, b, c); }
    static float pow_(float a, float b) { return std::pow(a, b); }
    static float exp_(float a) { return std::exp(a); }
    static void sincos_(float a, float* s, float* c) { *s = std::sin(a); *c = std::cos(a); }
    static float atan2_(float y, float x) { return std::atan2(y, x); }
    static float asin_(float x) { return std::asin(x); }
    static float fmod_(float a, float b) { return std::fmod(a, b); }
    static constexpr float lit(float f, double) { return f; }
};

// Dormand-Prince 5(4) (docs/dormand_prince_extended_tableau.md) and Hairer's dense output.
template <class T> struct Tab {
    static constexpr T a21 = T(1) / T(5);
    static constexpr T a31 = T(3) / T(40), a32 = T(9) / T(40);
    static constexpr T a41 = T(44) / T(45), a42 = T(-56) / T(15), a43 = T(32) / T(9);
    static constexpr T a51 = T(19372) / T(6561), a52 = T(-25360) / T(2187), a53 = T(64448) / T(6561), a54 = T(-212) / T(729);
    static constexpr T a61 = T(9017) / T(3168), a62 = T(-355) / T(33), a63 = T(46732) / T(5247), a64 = T(49) / T(176), a65 = T(-5103) / T(18656);
    static constexpr T b1 = T(35) / T(384), b3 = T(500) / T(1113), b4 = T(125) / T(192), b5 = T(-2187) / T(6784), b6 = T(11) / T(84);
    static constexpr T bh1 = T(5179) / T(57600), bh3 = T(7571) / T(16695), bh4 = T(393) / T(640), bh5 = T(-92097) / T(339200),
                       bh6 = T(187) / T(2100), bh7 = T(1) / T(40);
    static constexpr T d1 = T(-12715105075.0) / T(11282082432.0), d3 = T(87487479700.0) / T(32700410799.0),
                       d4 = T(-10690763975.0) / T(1880347072.0), d5 = T(701980252875.0) / T(199316789632.0),
                       d6 = T(-1453857185.0) / T(822651844.0), d7 = T(69997945.0) / T(29380423.0);
};

// ---- scalar pieces ---------------------------------------------------------------------
uint32_t pcg32(uint64_t state) {
    const uint64_t x = state * 6364136223846793005ULL + 1442695040888963407ULL;
    const uint32_t xs = (uint32_t)(((x >> 18u) ^ x) >> 27u);
    const uint32_t rot = (uint32_t)(x >> 59u);
    return (xs >> rot) | (xs << ((32u - rot) & 31u));
}
float rand01(uint64_t state) { return (float)pcg32(state) * 2.3283064365386963e-10f; }

template <class T> T ks_radius(T x, T y, T z, T aa) {
    using F = M<T>;
    const T rho2 = x * x + y * y + z * z;
    const T u = rho2 - aa;
    const T s = F::sqrt_(u * u + T(4) * aa * y * y);
    return F::sqrt_(T(0.5) * (u + s));
}

// dx/dl = p - 2 Hk (l.p - pt) l ;  dp/dl = grad(Hk) (l.p - pt)^2 + 2 Hk (l.p - pt) grad(l).p
// exact = false reproduces the reference's d(r^2)/dy = y (1 + (u + 4a^2)/(2s)) (kerr_math.cuh:97);
// exact = true uses the derivative of r^2 = (u + s)/2, y (1 + (u + 2a^2)/s).
template <class T> void hamilton_rhs(const T* st, T pt, T a, T aa, T Mm, T* d, bool exact) {
    using F = M<T>;
    const T x = st[0], y = st[1], z = st[2], px = st[3], py = st[4], pz = st[5];
    const T rho2 = x * x + y * y + z * z;
    const T u = rho2 - aa;
    const T s = F::sqrt_(u * u + T(4) * aa * y * y);
    const T r2 = T(0.5) * (u + s);
    const T r = F::sqrt_(r2);
    // r^4 - (rho^2 - a^2) r^2 - a^2 y^2 = 0  =>  d(r^2)/dx_i
    const T dr2x = x * (T(1) + u / s);
    const T dr2y = exact ? y * (T(1) + (u + T(2) * aa) / s) : y * (T(1) + (u + T(4) * aa) / (T(2) * s));
    const T dr2z = z * (T(1) + u / s);
    const T rx = dr2x / (T(2) * r), ry = dr2y / (T(2) * r), rz = dr2z / (T(2) * r);
    const T D = r2 + aa;
    const T Nx = r * x - a * z, Nz = r * z + a * x;
    const T lx = Nx / D, ly = y / r, lz = Nz / D;
    const T denH = r2 * r2 + aa * y * y;
    const T Hk = Mm * r2 * r / denH;
    const T lp = lx * px + ly * py + lz * pz - pt;
    d[0] = px - T(2) * Hk * lp * lx;
    d[1] = py - T(2) * Hk * lp * ly;
    d[2] = pz - T(2) * Hk * lp * lz;
    const T dD[3] = {T(2) * r * rx, T(2) * r * ry, T(2) * r * rz};
    const T dNx[3] = {rx * x + r, ry * x, rz * x - a};
    const T dNz[3] = {rx * z + a, ry * z, rz * z + r};
    const T dr[3] = {rx, ry, rz};
    const T dyi[3] = {T(0), T(1), T(0)};
    for (int i = 0; i < 3; ++i) {
        const T dlx = (dNx[i] * D - Nx * dD[i]) / (D * D);
        const T dlz = (dNz[i] * D - Nz * dD[i]) / (D * D);
        const T dly = (dyi[i] * r - y * dr[i]) / r2;
        const T ddenH = T(4) * r2 * r * dr[i] + (i == 1 ? T(2) * aa * y : T(0));
        const T dH = Mm * (T(3) * r2 * dr[i] * denH - r2 * r * ddenH) / (denH * denH);
        const T dlp = dlx * px + dly * py + dlz * pz;
        d[3 + i] = dH * lp * lp + T(2) * Hk * lp * dlp;
    }
}

template <class T> T dense(T y0, T y1, T k1, T k3, T k4, T k5, T k6, T k7, T h, T t) {
    using C = Tab<T>;
    const T q2 = y1 - y0, q3 = y0 + h * k1 - y1, q4 = T(2) * (y1 - y0) - h * (k1 + k7);
    const T q5 = h * (C::d1 * k1 + C::d3 * k3 + C::d4 * k4 + C::d5 * k5 + C::d6 * k6 + C::d7 * k7);
    return y0 + t * (q2 + q3) - t * t * (q3 - q4 - q5) - t * t * t * (q4 + T(2) * q5) + t * t * t * t * q5;
}
template <class T> T dense_slope(T y0, T y1, T k1, T k3, T k4, T k5, T k6, T k7, T h, T t) {
    using C = Tab<T>;
    const T q2 = y1 - y0, q3 = y0 + h * k1 - y1, q4 = T(2) * (y1 - y0) - h * (k1 + k7);
    const T q5 = h * (C::d1 * k1 + C::d3 * k3 + C::d4 * k4 + C::d5 * k5 + C::d6 * k6 + C::d7 * k7);
    return (q2 + q3) - T(2) * t * (q3 - q4 - q5) - T(3) * t * t * (q4 + T(2) * q5) + T(4) * t * t * t * q5;
}

// Root of y(t) = 0 on the dense output (stated physics): Newton from the secant guess t,
// safeguarded by the bracket [lo, hi] that the iterates keep; an update that leaves the bracket
// is replaced by bisection.  A converged update (tn == t, which may sit on the bracket end) is
// kept: the step is then 0 and the loop ends.
template <class T>
T crossing_root(T y0, T y1, T k1, T k3, T k4, T k5, T k6, T k7, T hs, T t) {
    T lo = 0, hi = 1;
    const bool neg0 = y0 < 0;
    for (int it = 0; it < 12; ++it) {
        const T yt = dense<T>(y0, y1, k1, k3, k4, k5, k6, k7, hs, t);
        if (yt == 0) break;
        if ((yt < 0) == neg0) lo = t; else hi = t;
        const T dyt = dense_slope<T>(y0, y1, k1, k3, k4, k5, k6, k7, hs, t);
        T tn = dyt != 0 ? t - yt / dyt : T(0.5) * (lo + hi);
        if (!(tn >= lo && tn <= hi)) tn = T(0.5) * (lo + hi);
        const T stp = std::fabs(tn - t);
        t = tn;
        if (stp <= M<T>::lit(1e-7f, 1e-15)) break;
    }
    return t;
}

template <class T> T fade(T t) { return t * t * t * (t * (t * T(6) - T(15)) + T(10)); }
template <class T> T lerp_(T a, T b, T t) { return a + t * (b - a); }
template <class T> void lattice_grad(int ix, int iy, uint32_t seed, T* gx, T* gy) {
    const uint64_t key = ((uint64_t)(uint32_t)ix << 32) | (uint64_t)(uint32_t)iy;
    const uint32_t h = pcg32(key ^ (uint64_t)seed);
    const float kAngle = 6.283185307f * 2.3283064365386963e-10f;
    const T ang = (T)((float)h) * (T)kAngle;
    M<T>::sincos_(ang, gy, gx);
}
template <class T> T gnoise(T u, T v, uint32_t seed) {
    const int ix0 = (int)std::floor(u), iy0 = (int)std::floor(v);
    const T fx = u - (T)ix0, fy = v - (T)iy0;
    T g[4][2];
    lattice_grad<T>(ix0, iy0, seed, &g[0][0], &g[0][1]);
    lattice_grad<T>(ix0 + 1, iy0, seed, &g[1][0], &g[1][1]);
    lattice_grad<T>(ix0, iy0 + 1, seed, &g[2][0], &g[2][1]);
    lattice_grad<T>(ix0 + 1, iy0 + 1, seed, &g[3][0], &g[3][1]);
    const T n00 = g[0][0] * fx + g[0][1] * fy;
    const T n10 = g[1][0] * (fx - 1) + g[1][1] * fy;
    const T n01 = g[2][0] * fx + g[2][1] * (fy - 1);
    const T n11 = g[3][0] * (fx - 1) + g[3][1] * (fy - 1);
    const T uf = fade(fx), vf = fade(fy);
    return lerp_(lerp_(n00, n10, uf), lerp_(n01, n11, uf), vf);
}
template <class T> T fbm(T u, T v, int octaves, uint32_t seed) {
    if (octaves <= 0) return T(0.5);
    T sum = 0, amp = 1, freq = 1, amp_sum = 0;
    for (int o = 0; o < octaves; ++o) {
        sum += gnoise<T>(u * freq, v * freq, seed) * amp;
        amp_sum += amp;
        amp *= T(0.5);
        freq *= T(2);
    }
    const T val = amp_sum > 0 ? sum / amp_sum : T(0);
    return val * T(0.5) + T(0.5);
}

// ---- host-side derivations (Rust f32 semantics) ----------------------------------------
bool f32_from_f64(double v, float* out) {
    if (!std::isfinite(v)) return false;
    char buf[64];
    auto res = std::to_chars(buf, buf + 63, v);
    *res.ptr = '\0';
    *out = std::strtof(buf, nullptr);
    return std::isfinite(*out);
}
double define_value(float v) {
    char buf[128];
    snprintf(buf, sizeof buf, "%.10f", (double)v);
    return std::strtod(buf, nullptr);
}
float isco(float a_norm, bool prograde, float mass) {
    const float aa = a_norm * a_norm;
    const float z1 = std::fma(std::cbrt(1.0f - aa), std::cbrt(1.0f + a_norm) + std::cbrt(1.0f - a_norm), 1.0f);
    const float z2 = std::sqrt(std::fma(3.0f, aa, z1 * z1));
    const float inside = (3.0f - z1) * std::fma(2.0f, z2, 3.0f + z1);
    const float root = std::sqrt(std::max(inside, 0.0f));
    return mass * (3.0f + z2 + (prograde ? -root : root));
}
float nt_factor(float r, float a, float r_isco, float inv_m) {
    if (r <= r_isco) return 0.0f;
    const float rn = r * inv_m, rin = r_isco * inv_m;
    const float x = std::sqrt(rn), xms = std::sqrt(rin);
    const float base = std::acos(-a) * (1.0f / 3.0f);
    const float step = 2.0943952f;
    const float xs[3] = {2.0f * std::cos(base), 2.0f * std::cos(base - step), 2.0f * std::cos(base + step)};
    float sl = 0.0f;
    for (int i = 0; i < 3; ++i) {
        const float xi = xs[i];
        const float den = xi * (xi - xs[(i + 1) % 3]) * (xi - xs[(i + 2) % 3]);
        if (den <= 0.0f) continue;
        const float coef = 3.0f * (xi - a) * (xi - a) / den;
        const float val = (x - xi) / (xms - xi);
        if (val > 0.0f) sl += coef * std::log(val);
    }
    const float q = std::fma(1.5f * a, -std::log(x / xms), x - xms) - sl;
    const float geo = rn * std::fma(2.0f, a, std::fma(rn, x, -(3.0f * x)));
    return std::max(q / geo, 0.0f);
}

struct Derived {
    // KerrParams
    float a, Mf, aa, inv_M, a_norm, rh, r_in, r_out, inv_w_2, inv_h_2, aspect;
    // define values
    double exposure, thick, sky_int, temp_scale, h0, tol, cutoff, hor_eps, escape, wl_step;
    float final_scale;
    float sky_spacing;
};

bool derive(const kto_scene& s, Derived* d) {
    if (s.width == 0 || s.height == 0 || s.mass == 0.0f) return false;
    d->a = s.spin;
    d->Mf = s.mass;
    d->inv_M = 1.0f / s.mass;
    d->aa = s.spin * s.spin;
    d->a_norm = s.spin * d->inv_M;
    d->rh = s.mass + std::sqrt(std::max(std::fma(s.mass, s.mass, -d->aa), 0.0f));
    d->r_in = isco(d->a_norm, true, s.mass);
    d->r_out = s.disk_outer_radius;
    if (!f32_from_f64((double)s.width / (double)s.height, &d->aspect)) return false;
    if (!f32_from_f64(2.0 / (double)s.width, &d->inv_w_2)) return false;
    if (!f32_from_f64(2.0 / (double)s.height, &d->inv_h_2)) return false;
    d->exposure = define_value(s.exposure_scale);
    d->thick = define_value(s.sky_line_thickness);
    d->sky_int = define_value(s.sky_intensity);
    d->temp_scale = define_value(s.disk_temperature_scale);
    d->h0 = define_value(s.initial_step);
    d->tol = define_value(s.tolerance);
    d->cutoff = define_value(s.transmittance_cutoff);
    d->hor_eps = define_value(s.horizon_epsilon);
    d->escape = define_value(s.escape_radius);
    d->wl_step = define_value(s.wavelength_step);
    d->final_scale = (float)(d->exposure * (double)(1.0f / (float)s.spp));
    d->sky_spacing = 3.14159265f / (float)s.sky_grid_divisions;
    return true;
}

// 1D linear, normalised, clamped fetch.
template <class T> T tex_weight(T frac, int tex_mode) {
    if (tex_mode == 1) return std::nearbyint(frac * T(256)) / T(256);
    if (tex_mode == 2) return std::floor(frac * T(256)) / T(256);
    return frac;
}
template <class T> void tex_fetch(const float* lut, int n, int ch, T u, int tex_mode, T* out) {
    const T x = u * T(n) - T(0.5);
    const T fl = std::floor(x);
    const T w = tex_weight<T>(x - fl, tex_mode);
    long i0 = (long)fl, i1 = i0 + 1;
    i0 = std::clamp<long>(i0, 0, n - 1);
    i1 = std::clamp<long>(i1, 0, n - 1);
    for (int c = 0; c < ch; ++c) {
        const T v0 = lut[i0 * ch + c], v1 = lut[i1 * ch + c];
        out[c] = (T(1) - w) * v0 + w * v1;
    }
}

struct RayResult {
    float col[3];
    kto_ray_info info;
};

template <class T>
RayResult trace_ray(const kto_scene& s, const Derived& dv, const float dirf[3], uint32_t* err) {
    using F = M<T>;
    using C = Tab<T>;
    RayResult out;
    out.col[0] = out.col[1] = out.col[2] = 0.0f;
    kto_ray_info& info = out.info;
    std::memset(&info, 0, sizeof info);
    info.first_r = info.first_g = info.first_T = std::numeric_limits<double>::quiet_NaN();
    const T a = (T)dv.a, aa = std::is_same<T, double>::value ? (T)dv.a * (T)dv.a : (T)dv.aa, Mm = (T)dv.Mf;
    // null initialisation (kerr_trace.cuh:14-46)
    const T dl = F::sqrt_((T)dirf[0] * dirf[0] + (T)dirf[1] * dirf[1] + (T)dirf[2] * dirf[2]);
    const T n[3] = {(T)dirf[0] / dl, (T)dirf[1] / dl, (T)dirf[2] / dl};
    T st[6] = {(T)s.cam_pos[0], (T)s.cam_pos[1], (T)s.cam_pos[2], 0, 0, 0};
    {
        const T x = st[0], y = st[1], z = st[2];
        const T r = ks_radius<T>(x, y, z, aa);
        const T r2 = r * r;
        const T D = r2 + aa;
        const T l[3] = {(r * x - a * z) / D, y / r, (r * z + a * x) / D};
        const T Hk = Mm * r2 * r / (r2 * r2 + aa * y * y);
        const T ln = l[0] * n[0] + l[1] * n[1] + l[2] * n[2];
        const T gtt = T(-1) + T(2) * Hk, gtn = T(2) * Hk * ln, gnn = T(1) + T(2) * Hk * ln * ln;
        const T kt = (-gtn - F::sqrt_(gtn * gtn - gtt * gnn)) / gtt;
        const T pt = gtt * kt + gtn;
        for (int c = 0; c < 3; ++c) st[3 + c] = n[c] + T(2) * Hk * l[c] * (kt + ln);
        st[0] = x;
        // stash in the loop below
        T h = (T)dv.h0;
        if (std::is_same<T, float>::value) h = (T)(float)dv.h0;
        const T base_tol = std::is_same<T, float>::value ? (T)(float)dv.tol : (T)dv.tol;
        float tau = 1.0f;
        float col[3] = {0, 0, 0};
        T k1[6];
        bool have_fsal = false;
        const double hor = (double)dv.rh + dv.hor_eps;
        for (uint32_t i = 0; i < s.max_steps && (double)tau > dv.cutoff; ++i) {
            // H-scaled tolerance (kerr_trace.cuh:67-73)
            const T rc = ks_radius<T>(st[0], st[1], st[2], aa);
            const T Hc = Mm * rc * rc * rc / (rc * rc * rc * rc + aa * st[1] * st[1]);
            T tt = (Hc - M<T>::lit(0.05f, 0.05)) / (M<T>::lit(0.3f, 0.3) - M<T>::lit(0.05f, 0.05));
            tt = std::min(std::max(tt, T(0)), T(1));
            const T tol = s.mode == 0 ? base_tol * (T(5) - T(5) * tt) : base_tol * (T(5) - T(4) * tt);
            T k[7][6], nx[6], y[6], hs = h, errv = 0;
            bool accepted = false;
            uint32_t att = 0;
            bool k1_ready = have_fsal;
            if (have_fsal) std::memcpy(k[0], k1, sizeof k1);
            while (!accepted && att < s.max_attempts) {
                hs = h;
                if (!k1_ready) {
                    hamilton_rhs<T>(st, pt, a, aa, Mm, k[0], s.mode == 1);
                    info.rhs++;
                    k1_ready = true;
                }
                static const T A[6][5] = {{C::a21, 0, 0, 0, 0},
                                          {C::a31, C::a32, 0, 0, 0},
                                          {C::a41, C::a42, C::a43, 0, 0},
                                          {C::a51, C::a52, C::a53, C::a54, 0},
                                          {C::a61, C::a62, C::a63, C::a64, C::a65},
                                          {C::b1, 0, C::b3, C::b4, C::b5}};
                for (int j = 1; j < 6; ++j) {
                    for (int c = 0; c < 6; ++c) {
                        T acc = 0;
                        for (int l = 0; l < j; ++l) acc += A[j - 1][l] * k[l][c];
                        y[c] = st[c] + hs * acc;
                    }
                    hamilton_rhs<T>(y, pt, a, aa, Mm, k[j], s.mode == 1);
                }
                for (int c = 0; c < 6; ++c)
                    nx[c] = st[c] + hs * (C::b1 * k[0][c] + C::b3 * k[2][c] + C::b4 * k[3][c] + C::b5 * k[4][c] + C::b6 * k[5][c]);
                hamilton_rhs<T>(nx, pt, a, aa, Mm, k[6], s.mode == 1);
                info.rhs += 6;
                errv = T(0);
                bool all_nan = true;
                T emax = -std::numeric_limits<T>::infinity();
                for (int c = 0; c < 6; ++c) {
                    const T e = hs * ((C::b1 - C::bh1) * k[0][c] + (C::b3 - C::bh3) * k[2][c] + (C::b4 - C::bh4) * k[3][c] +
                                      (C::b5 - C::bh5) * k[4][c] + (C::b6 - C::bh6) * k[5][c] - C::bh7 * k[6][c]);
                    const T ec = std::fabs(e) / (tol * std::max(std::fabs(st[c]), T(1)));
                    if (!std::isnan(ec)) {
                        all_nan = false;
                        emax = std::max(emax, ec);
                    }
                }
                errv = all_nan ? std::numeric_limits<T>::quiet_NaN() : emax;  // fmaxf semantics
                if (errv <= T(1)) accepted = true;
                h = hs * M<T>::lit(0.9f, 0.9) * F::pow_(errv, M<T>::lit(-0.2f, -0.2));
                att++;
                info.attempts++;
            }
            T prev[6];
            std::memcpy(prev, st, sizeof prev);
            std::memcpy(st, nx, sizeof st);
            info.steps++;
            if (accepted) {
                std::memcpy(k1, k[6], sizeof k1);
                have_fsal = true;
            } else {
                have_fsal = false;
            }
            if (s.retire_frozen && std::isnan(st[1])) {
                info.term = 3;
                break;
            }
            const T r_now = ks_radius<T>(st[0], st[1], st[2], aa);
            if ((double)r_now < hor) {
                info.term = 1;
                break;
            }
            if ((prev[1] < 0 && st[1] >= 0) || (prev[1] > 0 && st[1] <= 0)) {
                info.crossings++;
                const T* K1 = k[0];
                const T y0 = prev[1], y1 = st[1];
                T t = (y0 - y1) != T(0) ? y0 / (y0 - y1) : T(0.5);
                t = std::min(std::max(t, T(0)), T(1));
                if (s.mode == 1) t = crossing_root<T>(y0, y1, K1[1], k[2][1], k[3][1], k[4][1], k[5][1], k[6][1], hs, t);
                T hp[6];
                for (int c = 0; c < 6; ++c) hp[c] = dense<T>(prev[c], st[c], K1[c], k[2][c], k[3][c], k[4][c], k[5][c], k[6][c], hs, t);
                const T xh = hp[0], zh = hp[2];
                T rhit = ks_radius<T>(xh, T(0), zh, aa);
                if (rhit >= (T)dv.r_in && rhit <= (T)dv.r_out) {
                    const T sqM = F::sqrt_(Mm), rs = F::sqrt_(rhit);
                    const T disc = T(1) - T(3) * Mm / rhit + T(2) * a * sqM / (rhit * rs);
                    if (disc > 0) {
                        const T omega = -sqM / (rhit * rs + a * sqM);
                        const T D2 = rhit * rhit + aa;
                        const T lx = (rhit * xh - a * zh) / D2, lz = (rhit * zh + a * xh) / D2;
                        const T ldotp = lx * hp[3] + lz * hp[5];
                        const T ldotxi = lx * zh - lz * xh;
                        const T Hh = Mm / rhit;
                        const T L = (zh * hp[3] - xh * hp[5]) + T(2) * Hh * ldotxi * (ldotp + kt);
                        const T g = T(1) / ((T(1) / F::sqrt_(disc)) * (T(1) - omega * (L / (-pt))));
                        const T span = (T)dv.r_out - (T)dv.r_in;
                        const T u = span > 0 ? (rhit - (T)dv.r_in) / span : T(0);
                        T sampled;
                        tex_fetch<T>(s.disk_lut, (int)s.lut_size, 1, u, s.tex_mode, &sampled);
                        T Tm = (T)(dv.temp_scale * (double)sampled * (double)g);
                        if (s.noise_enabled && s.noise_detail > 0 && s.noise_strength != 0.0f) {
                            // Boyer-Lindquist azimuth of the hit (kerr_math.cuh:60-81); r_hit is replaced
                            const T rho2 = xh * xh + zh * zh;
                            const T uu = rho2 - aa;
                            const T r2b = T(0.5) * (uu + std::fabs(uu));
                            rhit = F::sqrt_(r2b);
                            const T phi = F::atan2_(rhit * xh - a * zh, rhit * zh + a * xh);
                            const T om = T(1) / (a + F::sqrt_(rhit * rhit * rhit / Mm));
                            T phase = phi + (T)s.noise_winding * om;
                            if (s.mode == 1) phase += (T)s.noise_phase;
                            T sp, cp;
                            F::sincos_(phase, &sp, &cp);
                            const T nu = rhit * cp * (T)s.noise_scale, nv = rhit * sp * (T)s.noise_scale;
                            const T nval = fbm<T>(nu, nv, (int)s.noise_detail, s.mode == 1 ? s.noise_seed : 0u);
                            Tm *= T(1) + (T)s.noise_strength * (nval - T(0.5));
                        }
                        if (info.hits == 0) {
                            info.first_r = (double)rhit;
                            info.first_g = (double)g;
                            info.first_T = (double)Tm;
                        }
                        if (std::isfinite(Tm) && Tm > 0) {
                            info.hits++;
                            T c3[4] = {0, 0, 0, 0};
                            if ((double)Tm > (double)s.lut_max_temp) {
                                if (err && err[0] == 0) {
                                    err[0] = 1;
                                    const float tf = (float)Tm;
                                    std::memcpy(&err[1], &tf, 4);
                                }
                            } else {
                                const T pos = Tm / (T)s.lut_max_temp * (T)(s.lut_size - 1);
                                const T uc = (pos + T(0.5)) / (T)s.lut_size;
                                tex_fetch<T>(s.bb_lut, (int)s.lut_size, 4, uc, s.tex_mode, c3);
                            }
                            const T luma = T(0.2126) * c3[0] + T(0.7152) * c3[1] + T(0.0722) * c3[2];
                            const T ls = (T)((double)luma / dv.wl_step);
                            const T alpha = T(1) - F::exp_(-ls * T(0.5));
                            for (int c = 0; c < 3; ++c) col[c] += (float)(c3[c] * alpha * (T)tau);
                            tau *= (float)(T(1) - alpha);
                        }
                    }
                }
            }
            if ((double)r_now > dv.escape) {
                T ke[6];
                hamilton_rhs<T>(st, pt, a, aa, Mm, ke, s.mode == 1);
                info.rhs++;
                const T nrm = F::sqrt_(ke[0] * ke[0] + ke[1] * ke[1] + ke[2] * ke[2]);
                const T ex = ke[0] / nrm, ey = ke[1] / nrm, ez = ke[2] / nrm;
                const T lon = F::atan2_(ez, ex), lat = F::asin_(ey);
                const T gs = (T)dv.sky_spacing, th = (T)(float)dv.thick;
                const T dlon = F::fmod_(std::fabs(lon), gs), dlat = F::fmod_(std::fabs(lat), gs);
                const bool grid = (dlon < th || dlon > gs - th) || (dlat < th || dlat > gs - th) || (std::fabs(lat) < th * T(3));
                const float sky = grid ? (float)(dv.sky_int * (double)tau) : 0.0f;
                for (int c = 0; c < 3; ++c) col[c] += sky;
                info.term = 2;
                break;
            }
        }
        for (int c = 0; c < 3; ++c) out.col[c] = col[c];
    }
    return out;
}

// ---- forward-mode derivatives of the stated-physics image ---------------------------------
// The reference gradient of the differentiable trace: the f64 stated-physics trace (mode 1,
// spp 1 at pixel centres, no noise, exact LUT weights) carried on D4 numbers, a value and its
// derivatives in theta = (spin, inclination in degrees, temperature scale, disk outer radius).
// Step sizes and every discrete decision (acceptance, crossings, disk membership, termination)
// are taken on the values, so the derivative is that of the frozen-step model.  The crossing
// root is differentiated by the implicit-function theorem.
struct D4 {
    double v, d[4];
    D4(double x = 0.0) : v(x), d{0.0, 0.0, 0.0, 0.0} {}
    static D4 seed(double x, int k) {
        D4 r(x);
        r.d[k] = 1.0;
        return r;
    }
};
D4 operator+(const D4& a, const D4& b) {
    D4 r(a.v + b.v);
    for (int i = 0; i < 4; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
D4 operator-(const D4& a, const D4& b) {
    D4 r(a.v - b.v);
    for (int i = 0; i < 4; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
D4 operator-(const D4& a) {
    D4 r(-a.v);
    for (int i = 0; i < 4; ++i) r.d[i] = -a.d[i];
    return r;
}
D4 operator*(const D4& a, const D4& b) {
    D4 r(a.v * b.v);
    for (int i = 0; i < 4; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
D4 operator/(const D4& a, const D4& b) {
    D4 r(a.v / b.v);
    for (int i = 0; i < 4; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) / b.v;
    return r;
}
D4& operator+=(D4& a, const D4& b) { return a = a + b; }
D4& operator*=(D4& a, const D4& b) { return a = a * b; }
D4 d4_chain(const D4& x, double f, double df) {
    D4 r(f);
    for (int i = 0; i < 4; ++i) r.d[i] = df * x.d[i];
    return r;
}
D4 d4_sqrt(const D4& x) { const double q = std::sqrt(x.v); return d4_chain(x, q, q > 0 ? 0.5 / q : 0.0); }
D4 d4_cbrt(const D4& x) { const double q = std::cbrt(x.v); return d4_chain(x, q, q != 0 ? 1.0 / (3.0 * q * q) : 0.0); }
D4 d4_exp(const D4& x) { const double q = std::exp(x.v); return d4_chain(x, q, q); }
D4 d4_log(const D4& x) { return d4_chain(x, std::log(x.v), 1.0 / x.v); }
D4 d4_sin(const D4& x) { return d4_chain(x, std::sin(x.v), std::cos(x.v)); }
D4 d4_cos(const D4& x) { return d4_chain(x, std::cos(x.v), -std::sin(x.v)); }
D4 d4_acos(const D4& x) { return d4_chain(x, std::acos(x.v), -1.0 / std::sqrt(1.0 - x.v * x.v)); }

template <> struct M<D4> {
    static D4 sqrt_(const D4& x) { return d4_sqrt(x); }
};

// ISCO and Page-Thorne flux factor (isco / nt_factor above) on D4
D4 isco_d4(const D4& an) {
    const D4 z1 = D4(1.0) + d4_cbrt(D4(1.0) - an * an) * (d4_cbrt(D4(1.0) + an) + d4_cbrt(D4(1.0) - an));
    const D4 z2 = d4_sqrt(D4(3.0) * an * an + z1 * z1);
    D4 inside = (D4(3.0) - z1) * (D4(3.0) + z1 + D4(2.0) * z2);
    if (inside.v < 0.0) inside = D4(0.0);
    return D4(3.0) + z2 - d4_sqrt(inside);
}
D4 nt_factor_d4(const D4& r, const D4& an, const D4& r_isco, double inv_m) {
    if (!(r.v > r_isco.v)) return D4(0.0);
    const D4 rn = r * inv_m, rin = r_isco * inv_m;
    const D4 x = d4_sqrt(rn), xms = d4_sqrt(rin);
    const D4 base = d4_acos(-an) * (1.0 / 3.0);
    const double step = 2.0943951023931957;
    const D4 roots[3] = {D4(2.0) * d4_cos(base), D4(2.0) * d4_cos(base - D4(step)), D4(2.0) * d4_cos(base + D4(step))};
    D4 sum(0.0);
    for (int i = 0; i < 3; ++i) {
        const D4 xi = roots[i];
        const D4 den = xi * (xi - roots[(i + 1) % 3]) * (xi - roots[(i + 2) % 3]);
        if (!(den.v > 0.0)) continue;
        const D4 coef = D4(3.0) * (xi - an) * (xi - an) / den;
        const D4 val = (x - xi) / (xms - xi);
        if (val.v > 0.0) sum += coef * d4_log(val);
    }
    const D4 q = x - xms - D4(1.5) * an * d4_log(x / xms) - sum;
    const D4 geo = rn * (rn * x - D4(3.0) * x + D4(2.0) * an);
    const D4 f = q / geo;
    return f.v > 0.0 ? f : D4(0.0);
}

D4 dense_d4(const D4& y0, const D4& y1, const D4& k1, const D4& k3, const D4& k4, const D4& k5, const D4& k6,
            const D4& k7, double h, const D4& t) {
    using C = Tab<double>;
    const D4 q2 = y1 - y0, q3 = y0 + h * k1 - y1, q4 = D4(2.0) * (y1 - y0) - h * (k1 + k7);
    const D4 q5 = h * (C::d1 * k1 + C::d3 * k3 + C::d4 * k4 + C::d5 * k5 + C::d6 * k6 + C::d7 * k7);
    const D4 t2 = t * t;
    return y0 + t * (q2 + q3) - t2 * (q3 - q4 - q5) - t2 * t * (q4 + D4(2.0) * q5) + t2 * t2 * q5;
}

// Inputs of the differentiable trace that depend on theta, shared by all pixels.
struct DiffSetup {
    D4 a, aa, r_in, r_out, ts;
    D4 pos[3], fwd[3], rgt[3], up[3];
    double fov, Mm;
    std::vector<D4> lut;
};

struct DiffRay {
    D4 col[3];
    int32_t term, hits, steps;
};

DiffRay trace_ray_diff(const kto_scene& s, const Derived& dv, const DiffSetup& ds, uint32_t px, uint32_t py) {
    using C = Tab<double>;
    DiffRay out;
    out.term = 0;
    out.hits = 0;
    out.steps = 0;
    for (int c = 0; c < 3; ++c) out.col[c] = D4(0.0);
    const D4 a = ds.a, aa = ds.aa;
    const double Mm = ds.Mm;
    const double W = (double)s.width, H = (double)s.height;
    const double u = ((px + 0.5) * (2.0 / W) - 1.0) * (W / H) * ds.fov;
    const double v = (1.0 - (py + 0.5) * (2.0 / H)) * ds.fov;
    D4 dir[3];
    for (int c = 0; c < 3; ++c) dir[c] = u * ds.rgt[c] + v * ds.up[c] + ds.fwd[c];
    // null initialisation (as trace_ray)
    const D4 dl = d4_sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
    const D4 n[3] = {dir[0] / dl, dir[1] / dl, dir[2] / dl};
    D4 st[6] = {ds.pos[0], ds.pos[1], ds.pos[2], D4(0.0), D4(0.0), D4(0.0)};
    const D4 x = st[0], y = st[1], z = st[2];
    const D4 r0 = ks_radius<D4>(x, y, z, aa);
    const D4 r2 = r0 * r0;
    const D4 Dd = r2 + aa;
    const D4 l[3] = {(r0 * x - a * z) / Dd, y / r0, (r0 * z + a * x) / Dd};
    const D4 Hk = D4(Mm) * r2 * r0 / (r2 * r2 + aa * y * y);
    const D4 ln = l[0] * n[0] + l[1] * n[1] + l[2] * n[2];
    const D4 gtt = D4(-1.0) + D4(2.0) * Hk, gtn = D4(2.0) * Hk * ln, gnn = D4(1.0) + D4(2.0) * Hk * ln * ln;
    const D4 kt = (-gtn - d4_sqrt(gtn * gtn - gtt * gnn)) / gtt;
    const D4 pt = gtt * kt + gtn;
    for (int c = 0; c < 3; ++c) st[3 + c] = n[c] + D4(2.0) * Hk * l[c] * (kt + ln);
    double h = dv.h0;
    D4 tau(1.0);
    D4 k1[6];
    bool have_fsal = false;
    const double hor = (double)dv.rh + dv.hor_eps;
    const int nl = (int)s.lut_size;
    for (uint32_t i = 0; i < s.max_steps && tau.v > dv.cutoff; ++i) {
        const double rc = ks_radius<double>(st[0].v, st[1].v, st[2].v, aa.v);
        const double Hc = Mm * rc * rc * rc / (rc * rc * rc * rc + aa.v * st[1].v * st[1].v);
        double tt = (Hc - 0.05) / (0.3 - 0.05);
        tt = std::min(std::max(tt, 0.0), 1.0);
        const double tol = dv.tol * (5.0 - 4.0 * tt);
        D4 k[7][6], nx[6], yy[6];
        double hs = h;
        bool accepted = false, k1_ready = have_fsal;
        uint32_t att = 0;
        if (have_fsal) for (int c = 0; c < 6; ++c) k[0][c] = k1[c];
        while (!accepted && att < s.max_attempts) {
            hs = h;
            if (!k1_ready) {
                hamilton_rhs<D4>(st, pt, a, aa, D4(Mm), k[0], true);
                k1_ready = true;
            }
            static const double A[6][5] = {{C::a21, 0, 0, 0, 0},
                                           {C::a31, C::a32, 0, 0, 0},
                                           {C::a41, C::a42, C::a43, 0, 0},
                                           {C::a51, C::a52, C::a53, C::a54, 0},
                                           {C::a61, C::a62, C::a63, C::a64, C::a65},
                                           {C::b1, 0, C::b3, C::b4, C::b5}};
            for (int j = 1; j < 6; ++j) {
                for (int c = 0; c < 6; ++c) {
                    D4 acc(0.0);
                    for (int q = 0; q < j; ++q) acc += A[j - 1][q] * k[q][c];
                    yy[c] = st[c] + hs * acc;
                }
                hamilton_rhs<D4>(yy, pt, a, aa, D4(Mm), k[j], true);
            }
            for (int c = 0; c < 6; ++c)
                nx[c] = st[c] + hs * (C::b1 * k[0][c] + C::b3 * k[2][c] + C::b4 * k[3][c] + C::b5 * k[4][c] + C::b6 * k[5][c]);
            hamilton_rhs<D4>(nx, pt, a, aa, D4(Mm), k[6], true);
            bool all_nan = true;
            double emax = -std::numeric_limits<double>::infinity();
            for (int c = 0; c < 6; ++c) {
                const double e = hs * ((C::b1 - C::bh1) * k[0][c].v + (C::b3 - C::bh3) * k[2][c].v +
                                       (C::b4 - C::bh4) * k[3][c].v + (C::b5 - C::bh5) * k[4][c].v +
                                       (C::b6 - C::bh6) * k[5][c].v - C::bh7 * k[6][c].v);
                const double ec = std::fabs(e) / (tol * std::max(std::fabs(st[c].v), 1.0));
                if (!std::isnan(ec)) {
                    all_nan = false;
                    emax = std::max(emax, ec);
                }
            }
            const double errv = all_nan ? std::numeric_limits<double>::quiet_NaN() : emax;
            if (errv <= 1.0) accepted = true;
            h = hs * 0.9 * std::pow(errv, -0.2);
            att++;
        }
        D4 prev[6];
        for (int c = 0; c < 6; ++c) {
            prev[c] = st[c];
            st[c] = nx[c];
        }
        out.steps++;
        if (accepted) {
            for (int c = 0; c < 6; ++c) k1[c] = k[6][c];
            have_fsal = true;
        } else {
            have_fsal = false;
        }
        if (std::isnan(st[1].v)) {
            out.term = 3;
            break;
        }
        const double r_now = ks_radius<double>(st[0].v, st[1].v, st[2].v, aa.v);
        if (r_now < hor) {
            out.term = 1;
            break;
        }
        if ((prev[1].v < 0 && st[1].v >= 0) || (prev[1].v > 0 && st[1].v <= 0)) {
            const double y0 = prev[1].v, y1 = st[1].v;
            double tv = (y0 - y1) != 0.0 ? y0 / (y0 - y1) : 0.5;
            tv = std::min(std::max(tv, 0.0), 1.0);
            tv = crossing_root<double>(y0, y1, k[0][1].v, k[2][1].v, k[3][1].v, k[4][1].v, k[5][1].v, k[6][1].v, hs, tv);
            // y(t*) = 0 on the dense output: dt* = -dy / y'(t*)
            const D4 yc = dense_d4(prev[1], st[1], k[0][1], k[2][1], k[3][1], k[4][1], k[5][1], k[6][1], hs, D4(tv));
            const double slope = dense_slope<double>(y0, y1, k[0][1].v, k[2][1].v, k[3][1].v, k[4][1].v, k[5][1].v,
                                                     k[6][1].v, hs, tv);
            D4 t(tv);
            if (slope != 0.0)
                for (int q = 0; q < 4; ++q) t.d[q] = -yc.d[q] / slope;
            D4 hp[6];
            for (int c = 0; c < 6; ++c)
                hp[c] = dense_d4(prev[c], st[c], k[0][c], k[2][c], k[3][c], k[4][c], k[5][c], k[6][c], hs, t);
            const D4 xh = hp[0], zh = hp[2];
            const D4 rhit = ks_radius<D4>(xh, D4(0.0), zh, aa);
            if (rhit.v >= ds.r_in.v && rhit.v <= ds.r_out.v) {
                const double sqM = std::sqrt(Mm);
                const D4 rs = d4_sqrt(rhit);
                const D4 disc = D4(1.0) - D4(3.0 * Mm) / rhit + D4(2.0 * sqM) * a / (rhit * rs);
                if (disc.v > 0) {
                    const D4 omega = -D4(sqM) / (rhit * rs + a * sqM);
                    const D4 D2 = rhit * rhit + aa;
                    const D4 lx = (rhit * xh - a * zh) / D2, lz = (rhit * zh + a * xh) / D2;
                    const D4 ldotp = lx * hp[3] + lz * hp[5];
                    const D4 ldotxi = lx * zh - lz * xh;
                    const D4 Hh = D4(Mm) / rhit;
                    const D4 L = (zh * hp[3] - xh * hp[5]) + D4(2.0) * Hh * ldotxi * (ldotp + kt);
                    const D4 g = D4(1.0) / ((D4(1.0) / d4_sqrt(disc)) * (D4(1.0) - omega * (L / (-pt))));
                    const D4 span = ds.r_out - ds.r_in;
                    const D4 uu = span.v > 0 ? (rhit - ds.r_in) / span : D4(0.0);
                    // texture-style coordinate of the LUT fetch, exact weight
                    const D4 xl = uu * (double)nl - 0.5;
                    const double fl = std::floor(xl.v);
                    int i0 = (int)std::min(std::max(fl, -1.0), (double)(nl - 1));
                    int i1 = i0 + 1;
                    i0 = std::max(i0, 0);
                    i1 = std::min(i1, nl - 1);
                    const D4 wl = xl - fl;
                    const D4 sampled = ds.lut[i0] + wl * (ds.lut[i1] - ds.lut[i0]);
                    const D4 Tm = ds.ts * sampled * g;
                    if (std::isfinite(Tm.v) && Tm.v > 0) {
                        out.hits++;
                        D4 c3[3] = {D4(0.0), D4(0.0), D4(0.0)};
                        if (Tm.v <= (double)s.lut_max_temp) {
                            const D4 pos = Tm / (double)s.lut_max_temp * (double)(nl - 1);
                            const double fb = std::floor(pos.v);
                            int j0 = (int)std::min(std::max(fb, -1.0), (double)(nl - 1));
                            int j1 = j0 + 1;
                            j0 = std::max(j0, 0);
                            j1 = std::min(j1, nl - 1);
                            const D4 wb = pos - fb;
                            for (int c = 0; c < 3; ++c) {
                                const double e0 = s.bb_lut[4 * j0 + c], e1 = s.bb_lut[4 * j1 + c];
                                c3[c] = D4(e0) + wb * (e1 - e0);
                            }
                        }
                        const D4 luma = 0.2126 * c3[0] + 0.7152 * c3[1] + 0.0722 * c3[2];
                        const D4 ls = luma / dv.wl_step;
                        const D4 alpha = D4(1.0) - d4_exp(-ls * 0.5);
                        for (int c = 0; c < 3; ++c) out.col[c] += c3[c] * alpha * tau;
                        tau *= D4(1.0) - alpha;
                    }
                }
            }
        }
        if (r_now > dv.escape) {
            double ke[6], stv[6];
            for (int c = 0; c < 6; ++c) stv[c] = st[c].v;
            hamilton_rhs<double>(stv, pt.v, a.v, aa.v, Mm, ke, true);
            const double nrm = std::sqrt(ke[0] * ke[0] + ke[1] * ke[1] + ke[2] * ke[2]);
            const double ex = ke[0] / nrm, ey = ke[1] / nrm, ez = ke[2] / nrm;
            const double lon = std::atan2(ez, ex), lat = std::asin(ey);
            const double gs = (double)dv.sky_spacing, th = (double)(float)dv.thick;
            const double dlon = std::fmod(std::fabs(lon), gs), dlat = std::fmod(std::fabs(lat), gs);
            const bool grid = (dlon < th || dlon > gs - th) || (dlat < th || dlat > gs - th) || (std::fabs(lat) < th * 3.0);
            if (grid)
                for (int c = 0; c < 3; ++c) out.col[c] += dv.sky_int * tau;
            out.term = 2;
            break;
        }
    }
    return out;
}

void pixel_dir(const kto_scene& s, const Derived& dv, uint32_t px, uint32_t py, uint32_t smp, float dir[3]) {
    float jx, jy;
    if (s.mode == 1 && s.spp == 1) {
        jx = jy = 0.5f;
    } else {
        const uint32_t pidx = py * s.width + px;
        const uint64_t key = ((uint64_t)pidx << 32) | (uint64_t)smp;
        jx = rand01(key);
        jy = rand01(key ^ 0xda3e39cb94b95bdbULL);
    }
    const float u = (((float)px + jx) * dv.inv_w_2 - 1.0f) * dv.aspect * s.fov_scale;
    const float v = (1.0f - ((float)py + jy) * dv.inv_h_2) * s.fov_scale;
    for (int c = 0; c < 3; ++c) dir[c] = u * s.rgt[c] + v * s.up[c] + s.fwd[c];
}

template <class T>
int render(const kto_scene* s, const int64_t* pixels, int64_t n, float* rgba, kto_ray_info* infos, uint32_t* err,
           int threads) {
    Derived dv;
    if (!s || !derive(*s, &dv)) return 1;
    if (s->max_attempts == 0) return 1;
    uint32_t err_local[2] = {0, 0};
    const int64_t total = pixels ? n : (int64_t)s->width * s->height;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#endif
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t k = 0; k < total; ++k) {
        const int64_t p = pixels ? pixels[k] : k;
        const uint32_t px = (uint32_t)(p % s->width), py = (uint32_t)(p / s->width);
        float acc[3] = {0, 0, 0};
        uint32_t e[2] = {0, 0};
        for (uint32_t smp = 0; smp < s->spp; ++smp) {
            float dir[3];
            pixel_dir(*s, dv, px, py, smp, dir);
            const RayResult rr = trace_ray<T>(*s, dv, dir, e);
            for (int c = 0; c < 3; ++c) acc[c] += rr.col[c];
            if (smp == 0 && infos) infos[k] = rr.info;
        }
        float* o = rgba + 4 * k;
        for (int c = 0; c < 3; ++c) o[c] = acc[c] * dv.final_scale;
        o[3] = 1.0f;
        if (e[0]) {
#pragma omp critical
            if (!err_local[0]) {
                err_local[0] = 1;
                err_local[1] = e[1];
            }
        }
    }
    if (err) {
        err[0] = err_local[0];
        err[1] = err_local[1];
    }
    return 0;
}

// ---- post (cuda/kernel.cu:17-84, 144-251) -----------------------------------------------
double aces(double x) { return (x * (2.51 * x + 0.03)) / (x * (2.43 * x + 0.59) + 0.14); }
double srgb(double x) { return x <= 0.0031308 ? 12.92 * x : 1.055 * std::pow(x, 1.0 / 2.4) - 0.055; }
uint32_t byte_of(double v) {
    const double c = std::isnan(v) ? 0.0 : std::min(std::max(v, 0.0), 1.0);
    return (uint32_t)std::nearbyint(c * 255.0);
}

}  // namespace

extern "C" {

int kto_abi_version(void) { return 1; }

// Trace W*H pixels (pixels == NULL) or the listed pixel indices; rgba gets 4 floats per traced
// pixel, infos one record per traced pixel (may be NULL).  precision 0 = f32 emulation, 2 = f64.
int kto_render(const kto_scene* s, int precision, const int64_t* pixels, int64_t n, float* rgba,
               kto_ray_info* infos, uint32_t* err, int threads) {
    if (precision == 2) return render<double>(s, pixels, n, rgba, infos, err, threads);
    if (precision == 0) return render<float>(s, pixels, n, rgba, infos, err, threads);
    return 2;
}

// Bloom + composite + ACES + sRGB + pack in double (bloom inactive when radius <= 0 or
// intensity <= 0).  mode 1 applies the luminance threshold to the bloom source.
int kto_post(const float* hdr, uint32_t w, uint32_t h, int radius, float sigma, float intensity, int mode,
             float threshold, uint32_t* image, float* bloom_out) {
    const size_t n = (size_t)w * h;
    const bool active = radius > 0 && intensity > 0.0f;
    std::vector<double> src(3 * n), hb(3 * n, 0.0), vb(3 * n, 0.0);
    for (size_t i = 0; i < n; ++i) {
        double k = 1.0;
        if (mode == 1) {
            const double L = 0.2126 * hdr[4 * i] + 0.7152 * hdr[4 * i + 1] + 0.0722 * hdr[4 * i + 2];
            k = L > threshold ? (L - threshold) / L : 0.0;
        }
        for (int c = 0; c < 3; ++c) src[3 * i + c] = hdr[4 * i + c] * k;
    }
    if (active) {
        std::vector<double> wt(2 * radius + 1);
        for (int i = -radius; i <= radius; ++i) wt[i + radius] = std::exp(-(double)i * i / (2.0 * (double)sigma * sigma));
#pragma omp parallel for
        for (int64_t y = 0; y < (int64_t)h; ++y)
            for (uint32_t x = 0; x < w; ++x) {
                double acc[3] = {0, 0, 0}, ws = 0;
                for (int i = -radius; i <= radius; ++i) {
                    const int64_t sx = (int64_t)x + i;
                    if (sx < 0 || sx >= (int64_t)w) continue;
                    for (int c = 0; c < 3; ++c) acc[c] += src[3 * (y * w + sx) + c] * wt[i + radius];
                    ws += wt[i + radius];
                }
                for (int c = 0; c < 3; ++c) hb[3 * (y * w + x) + c] = ws > 0 ? acc[c] / ws : acc[c];
            }
#pragma omp parallel for
        for (int64_t y = 0; y < (int64_t)h; ++y)
            for (uint32_t x = 0; x < w; ++x) {
                double acc[3] = {0, 0, 0}, ws = 0;
                for (int i = -radius; i <= radius; ++i) {
                    const int64_t sy = y + i;
                    if (sy < 0 || sy >= (int64_t)h) continue;
                    for (int c = 0; c < 3; ++c) acc[c] += hb[3 * (sy * w + x) + c] * wt[i + radius];
                    ws += wt[i + radius];
                }
                for (int c = 0; c < 3; ++c) vb[3 * (y * w + x) + c] = ws > 0 ? acc[c] / ws : acc[c];
            }
    }
    for (size_t i = 0; i < n; ++i) {
        uint32_t px = 0;
        for (int c = 0; c < 3; ++c) {
            const double v = (double)hdr[4 * i + c] + (active ? vb[3 * i + c] * intensity : 0.0);
            px |= byte_of(srgb(aces(v))) << (16 - 8 * c);
        }
        image[i] = px;
        if (bloom_out)
            for (int c = 0; c < 3; ++c) bloom_out[3 * i + c] = (float)hb[3 * i + c];
    }
    return 0;
}

// Host LUT generators and parameters, restated from the Rust host (f32).
int kto_blackbody_lut(uint32_t size, float max_temp, float wl_start, float wl_end, float wl_step, float* out) {
    if (size < 2 || !(wl_step > 0.0f) || !std::isfinite(wl_step)) return 1;
    std::vector<float> lam;
    for (float l = wl_start; !(l > wl_end); l += wl_step) {
        lam.push_back(l);
        if (lam.size() > (1u << 24)) return 1;
    }
    auto lobe = [](float x, float al, float mu, float s1, float s2) {
        const float t = (x - mu) / (x < mu ? s1 : s2);
        return al * std::exp(-0.5f * t * t);
    };
    std::vector<float> X(lam.size()), Y(lam.size()), Z(lam.size());
    for (size_t i = 0; i < lam.size(); ++i) {
        const float l = lam[i];
        X[i] = lobe(l, 1.056f, 599.8f, 37.9f, 31.0f) + lobe(l, 0.362f, 442.0f, 16.0f, 26.7f) + lobe(l, -0.065f, 501.1f, 20.4f, 26.2f);
        Y[i] = lobe(l, 0.821f, 568.8f, 46.9f, 40.5f) + lobe(l, 0.286f, 530.9f, 16.3f, 31.1f);
        Z[i] = lobe(l, 1.217f, 437.0f, 11.8f, 36.0f) + lobe(l, 0.681f, 459.0f, 26.2f, 13.8f);
    }
    for (uint32_t k = 0; k < size; ++k) {
        float T;
        if (!f32_from_f64((double)k / (double)(size - 1) * (double)max_temp, &T)) return 1;
        float* o = out + 4 * (size_t)k;
        o[0] = o[1] = o[2] = o[3] = 0.0f;
        if (T == 0.0f) continue;
        float sx = 0, sy = 0, sz = 0;
        for (size_t i = 0; i < lam.size(); ++i) {
            float I = 0.0f;
            if (T > 0.0f) {
                const float e = 1.4388e7f / (lam[i] * T);
                if (!(e > 80.0f)) {
                    const float l2 = lam[i] * lam[i];
                    I = (1.0f / (lam[i] * (l2 * l2))) / std::expm1(e) * 1e15f;
                }
            }
            sx += I * X[i];
            sy += I * Y[i];
            sz += I * Z[i];
        }
        sx *= wl_step;
        sy *= wl_step;
        sz *= wl_step;
        o[0] = std::fma(3.240454f, sx, std::fma(-1.5371385f, sy, -0.4985314f * sz));
        o[1] = std::fma(-0.969266f, sx, std::fma(1.8760108f, sy, 0.041556f * sz));
        o[2] = std::fma(0.0556434f, sx, std::fma(-0.2040259f, sy, 1.0572252f * sz));
    }
    return 0;
}

int kto_disk_lut(float spin, float mass, float disk_outer, uint32_t size, float* out) {
    if (size < 2 || mass == 0.0f) return 1;
    const float inv_m = 1.0f / mass, a_norm = spin * inv_m;
    const float r_in = isco(a_norm, true, mass);
    if (!(disk_outer > r_in)) return 1;
    for (uint32_t i = 0; i < size; ++i) {
        float r;
        if (!f32_from_f64(std::fma((double)i / (double)(size - 1), (double)(disk_outer - r_in), (double)r_in), &r)) return 1;
        out[i] = std::sqrt(std::sqrt(nt_factor(r, a_norm, r_in, inv_m)));
    }
    return 0;
}

// Derived KerrParams of a scene: a, M, aa, inv_M, a_norm, rh, r_in, inv_w_2, inv_h_2, aspect.
int kto_params(const kto_scene* s, float* out10) {
    Derived d;
    if (!s || !derive(*s, &d)) return 1;
    const float v[10] = {d.a, d.Mf, d.aa, d.inv_M, d.a_norm, d.rh, d.r_in, d.inv_w_2, d.inv_h_2, d.aspect};
    std::memcpy(out10, v, sizeof v);
    return 0;
}
float kto_isco(float a_norm, int prograde, float mass) { return isco(a_norm, prograde != 0, mass); }

// Camera basis of the app (src/math.rs:3-14) in f32 as glam computes it: Rust's
// f32::to_radians multiplies by the f32 constant PI / 180; Vec3::normalize scales by the
// reciprocal of sqrt(x*x + y*y + z*z); cross products are component-wise differences of
// products.  This file is built without FMA contraction, like Rust code.
namespace {
constexpr float kDegToRad = 3.14159265358979323846f / 180.0f;
void glam_normalize(float v[3]) {
    const float len = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    const float inv = 1.0f / len;
    for (int i = 0; i < 3; ++i) v[i] = v[i] * inv;
}
void glam_cross(const float a[3], const float b[3], float out[3]) {
    out[0] = a[1] * b[2] - b[1] * a[2];
    out[1] = a[2] * b[0] - b[2] * a[0];
    out[2] = a[0] * b[1] - b[0] * a[1];
}
}  // namespace
void kto_camera_basis(float yaw_deg, float pitch_deg, float* fwd, float* rgt, float* up) {
    const float yaw = yaw_deg * kDegToRad, pitch = pitch_deg * kDegToRad;
    float f[3] = {std::sin(yaw) * std::cos(pitch), std::sin(pitch), -std::cos(yaw) * std::cos(pitch)};
    glam_normalize(f);
    const float world_up[3] = {0.0f, 1.0f, 0.0f};
    glam_cross(f, world_up, rgt);
    glam_normalize(rgt);
    glam_cross(rgt, f, up);
    glam_normalize(up);
    for (int i = 0; i < 3; ++i) fwd[i] = f[i];
}
// fov_scale = (fov.to_radians() / 2.0).tan() (src/app.rs:163).
float kto_fov_scale(float fov_deg) { return std::tan(fov_deg * kDegToRad / 2.0f); }
float kto_nt_factor(float r, float a_norm, float r_isco, float inv_m) { return nt_factor(r, a_norm, r_isco, inv_m); }
double kto_define_value(float v) { return define_value(v); }
uint32_t kto_pcg32(uint64_t state) { return pcg32(state); }

// Scalar kernels in f64 for known-answer tests.
double kto_ks_radius(double x, double y, double z, double a) { return ks_radius<double>(x, y, z, a * a); }
void kto_rhs(const double* st, double pt, double a, double mass, double* d) { hamilton_rhs<double>(st, pt, a, a * a, mass, d, true); }
void kto_rhs_reference(const double* st, double pt, double a, double mass, double* d) {
    hamilton_rhs<double>(st, pt, a, a * a, mass, d, false);
}
double kto_dense(const double* q, double t) { return dense<double>(q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7], q[8], t); }
double kto_dense_slope(const double* q, double t) { return dense_slope<double>(q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7], q[8], t); }
// Differentiable trace (forward mode), stated physics, spp 1, no noise: colour (3 per pixel,
// final scale applied) and its derivatives in theta (3 x 4 per pixel, row = channel), plus
// (term, hits, steps) per pixel.  view = (observer r, azimuth deg, fov deg, base temperature
// scale); theta = (spin, inclination deg, temperature scale, disk outer radius).  The scene's
// spin, disk_outer_radius and disk_temperature_scale are replaced by theta.
int kto_diff_render(const kto_scene* sp, const double* view, const double* theta, const uint32_t* pixels,
                    int64_t n_pixels, double* color, double* dcolor, int32_t* info, int threads) {
    if (!sp || !view || !theta || !color || !dcolor) return -1;
    kto_scene s = *sp;
    if (s.mode != 1 || s.spp != 1 || s.noise_enabled) return -2;
    s.spin = (float)theta[0];
    s.disk_outer_radius = (float)theta[3];
    s.disk_temperature_scale = (float)(view[3] * theta[2]);
    Derived dv;
    if (!derive(s, &dv)) return -3;
    DiffSetup ds;
    const double inv_m = 1.0 / (double)s.mass;
    ds.Mm = (double)s.mass;
    ds.a = D4::seed(theta[0], 0);
    ds.aa = ds.a * ds.a;
    const D4 an = ds.a * inv_m;
    ds.r_in = isco_d4(an) * (double)s.mass;
    ds.r_out = D4::seed(theta[3], 3);
    D4 sc = D4::seed(theta[2], 2);
    ds.ts = sc * view[3];
    const int nl = (int)s.lut_size;
    ds.lut.resize(nl);
    for (int i = 0; i < nl; ++i) {
        const double ratio = (double)i / (double)(nl - 1);
        const D4 r = ds.r_in + ratio * (ds.r_out - ds.r_in);
        const D4 f = nt_factor_d4(r, an, ds.r_in, inv_m);
        ds.lut[i] = f.v > 0.0 ? d4_sqrt(d4_sqrt(f)) : D4(0.0);
    }
    const double d2r = 3.14159265358979323846 / 180.0;
    const D4 inc = D4::seed(theta[1], 1) * d2r;
    const double az = view[1] * d2r, r = view[0];
    ds.pos[0] = r * d4_sin(inc) * std::cos(az);
    ds.pos[1] = r * d4_cos(inc);
    ds.pos[2] = r * d4_sin(inc) * std::sin(az);
    for (int c = 0; c < 3; ++c) ds.fwd[c] = -ds.pos[c] / r;
    ds.rgt[0] = D4(std::sin(az));
    ds.rgt[1] = D4(0.0);
    ds.rgt[2] = D4(-std::cos(az));
    ds.up[0] = ds.rgt[1] * ds.fwd[2] - ds.rgt[2] * ds.fwd[1];
    ds.up[1] = ds.rgt[2] * ds.fwd[0] - ds.rgt[0] * ds.fwd[2];
    ds.up[2] = ds.rgt[0] * ds.fwd[1] - ds.rgt[1] * ds.fwd[0];
    ds.fov = std::tan(view[2] * d2r / 2.0);
    const double fs = (double)dv.final_scale;
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads > 0 ? threads : omp_get_max_threads())
    for (int64_t i = 0; i < n_pixels; ++i) {
        const uint32_t p = pixels ? pixels[i] : (uint32_t)i;
        const DiffRay rr = trace_ray_diff(s, dv, ds, p % s.width, p / s.width);
        for (int c = 0; c < 3; ++c) {
            color[3 * i + c] = rr.col[c].v * fs;
            for (int q = 0; q < 4; ++q) dcolor[12 * i + 4 * c + q] = rr.col[c].d[q] * fs;
        }
        if (info) {
            info[3 * i] = rr.term;
            info[3 * i + 1] = rr.hits;
            info[3 * i + 2] = rr.steps;
        }
    }
    return 0;
}

double kto_crossing_root(const double* q, double t0) {
    return crossing_root<double>(q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7], q[8], t0);
}
double kto_fbm(double u, double v, int octaves, uint32_t seed) { return fbm<double>(u, v, octaves, seed); }
double kto_aces(double x) { return aces(x); }
double kto_srgb(double x) { return srgb(x); }

// Null initialisation in f64 (kerr_trace.cuh:14-46): state (x, p) and p_t of a photon leaving
// `cam` along `dir` (normalised here).
void kto_null_init(const double* cam, const double* dir, double a, double mass, double* st, double* pt_out) {
    const double aa = a * a;
    const double dl = std::sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
    const double n[3] = {dir[0] / dl, dir[1] / dl, dir[2] / dl};
    const double x = cam[0], y = cam[1], z = cam[2];
    const double r = ks_radius<double>(x, y, z, aa), r2 = r * r, D = r2 + aa;
    const double l[3] = {(r * x - a * z) / D, y / r, (r * z + a * x) / D};
    const double Hk = mass * r2 * r / (r2 * r2 + aa * y * y);
    const double ln = l[0] * n[0] + l[1] * n[1] + l[2] * n[2];
    const double gtt = -1 + 2 * Hk, gtn = 2 * Hk * ln, gnn = 1 + 2 * Hk * ln * ln;
    const double kt = (-gtn - std::sqrt(gtn * gtn - gtt * gnn)) / gtt;
    *pt_out = gtt * kt + gtn;
    st[0] = x;
    st[1] = y;
    st[2] = z;
    for (int c = 0; c < 3; ++c) st[3 + c] = n[c] + 2 * Hk * l[c] * (kt + ln);
}

// One DP5(4) step of size h on the Hamiltonian flow (f64), returning the 5th-order state and
// the embedded error vector: used by the convergence-order known-answer test.
void kto_dp5_step(const double* st, double pt, double a, double mass, double h, double* out, double* err,
                  double* kout) {
    using C = Tab<double>;
    double k[7][6], y[6];
    const double aa = a * a;
    hamilton_rhs<double>(st, pt, a, aa, mass, k[0], true);
    static const double A[6][5] = {{C::a21, 0, 0, 0, 0},           {C::a31, C::a32, 0, 0, 0},
                                   {C::a41, C::a42, C::a43, 0, 0}, {C::a51, C::a52, C::a53, C::a54, 0},
                                   {C::a61, C::a62, C::a63, C::a64, C::a65}, {C::b1, 0, C::b3, C::b4, C::b5}};
    for (int j = 1; j < 7; ++j) {
        for (int c = 0; c < 6; ++c) {
            double acc = 0;
            for (int l = 0; l < j && l < 5; ++l) acc += A[j - 1][l] * k[l][c];
            if (j == 6) acc = C::b1 * k[0][c] + C::b3 * k[2][c] + C::b4 * k[3][c] + C::b5 * k[4][c] + C::b6 * k[5][c];
            y[c] = st[c] + h * acc;
        }
        hamilton_rhs<double>(y, pt, a, aa, mass, k[j], true);
    }
    if (kout)
        for (int j = 0; j < 7; ++j)
            for (int c = 0; c < 6; ++c) kout[6 * j + c] = k[j][c];
    for (int c = 0; c < 6; ++c) {
        out[c] = st[c] + h * (C::b1 * k[0][c] + C::b3 * k[2][c] + C::b4 * k[3][c] + C::b5 * k[4][c] + C::b6 * k[5][c]);
        err[c] = h * ((C::b1 - C::bh1) * k[0][c] + (C::b3 - C::bh3) * k[2][c] + (C::b4 - C::bh4) * k[3][c] +
                      (C::b5 - C::bh5) * k[4][c] + (C::b6 - C::bh6) * k[5][c] - C::bh7 * k[6][c]);
    }
}

}  // extern "C"
