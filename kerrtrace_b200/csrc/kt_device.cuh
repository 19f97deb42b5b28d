// kt_device.cuh — device-side geodesic core of the KerrTrace hot path (sm_100a).
//
// Restates, in this project's own structure, the per-ray algorithm of the reference:
//   cuda/kerr_math.cuh   (Kerr-Schild radius, Hamiltonian RHS, DP dense output, PCG, FBM, sky)
//   cuda/kerr_trace.cuh  (null initialisation, DP5(4) FSAL stepper, crossing, shading)
//   cuda/kernel.cu:1-16  (LUT fetch with overflow flag)
// The arithmetic of each formula is kept in the reference's order (same products, same
// fused multiply-adds, same fast-math intrinsics) so that the FP32 path reproduces the
// reference kernel's results; the scheduling around it (attempt-granular state machine,
// persistent refill, retirement of NaN-frozen rays) is this project's.
//
// Everything is templated on the integration type R (float for the reference arithmetic,
// double for the FP64 path); the mixed path uses float RHS with a double state update.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "kt_types.h"

namespace ktd {

// ----------------------------------------------------------------------------------------
// Arithmetic policies.  Ops<float> uses the intrinsics the reference calls (it is built with
// use_fast_math, config.yaml:39); Ops<double> their IEEE double counterparts.
// ----------------------------------------------------------------------------------------
template <class R> struct Ops;
template <> struct Ops<float> {
    static __device__ __forceinline__ float rsq(float x) { return rsqrtf(x); }
    static __device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }
    static __device__ __forceinline__ float sqrt_rn(float x) { return __fsqrt_rn(x); }
    static __device__ __forceinline__ float fma(float a, float b, float c) { return fmaf(a, b, c); }
    static __device__ __forceinline__ float powr(float a, float b) { return __powf(a, b); }
    static __device__ __forceinline__ float maxr(float a, float b) { return fmaxf(a, b); }
    static __device__ __forceinline__ float minr(float a, float b) { return fminf(a, b); }
    static __device__ __forceinline__ float absr(float a) { return fabsf(a); }
    static __device__ __forceinline__ float expr(float a) { return __expf(a); }
    static __device__ __forceinline__ float atan2r(float y, float x) { return atan2f(y, x); }
    static __device__ __forceinline__ void sincosr(float a, float* s, float* c) { __sincosf(a, s, c); }
    static __device__ __forceinline__ bool isnanr(float a) { return isnan(a); }
    static __device__ __forceinline__ bool isfiniter(float a) { return isfinite(a); }
};
template <> struct Ops<double> {
    static __device__ __forceinline__ double rsq(double x) { return rsqrt(x); }
    static __device__ __forceinline__ double fdiv(double a, double b) { return a / b; }
    static __device__ __forceinline__ double sqrt_rn(double x) { return sqrt(x); }
    static __device__ __forceinline__ double fma(double a, double b, double c) { return ::fma(a, b, c); }
    static __device__ __forceinline__ double powr(double a, double b) { return pow(a, b); }
    static __device__ __forceinline__ double maxr(double a, double b) { return fmax(a, b); }
    static __device__ __forceinline__ double minr(double a, double b) { return fmin(a, b); }
    static __device__ __forceinline__ double absr(double a) { return fabs(a); }
    static __device__ __forceinline__ double expr(double a) { return exp(a); }
    static __device__ __forceinline__ double atan2r(double y, double x) { return atan2(y, x); }
    static __device__ __forceinline__ void sincosr(double a, double* s, double* c) { sincos(a, s, c); }
    static __device__ __forceinline__ bool isnanr(double a) { return isnan(a); }
    static __device__ __forceinline__ bool isfiniter(double a) { return isfinite(a); }
};

// Literal of the integration type: the float spelling for float, the double one for double,
// so that no constant is rounded twice.
template <class R> __device__ __forceinline__ constexpr R lit(float f, double d);
template <> __device__ __forceinline__ constexpr float lit<float>(float f, double) { return f; }
template <> __device__ __forceinline__ constexpr double lit<double>(float, double d) { return d; }

// Dormand-Prince 5(4) tableau (docs/dormand_prince_extended_tableau.md:1-12), evaluated in R
// at compile time exactly as the reference's `static const float` initialisers
// (cuda/kerr_trace.cuh:52-59).
template <class R> struct DP {
    static constexpr R a21 = R(1) / R(5);
    static constexpr R a31 = R(3) / R(40), a32 = R(9) / R(40);
    static constexpr R a41 = R(44) / R(45), a42 = R(-56) / R(15), a43 = R(32) / R(9);
    static constexpr R a51 = R(19372) / R(6561), a52 = R(-25360) / R(2187),
                       a53 = R(64448) / R(6561), a54 = R(-212) / R(729);
    static constexpr R a61 = R(9017) / R(3168), a62 = R(-355) / R(33), a63 = R(46732) / R(5247),
                       a64 = R(49) / R(176), a65 = R(-5103) / R(18656);
    static constexpr R a71 = R(35) / R(384), a73 = R(500) / R(1113), a74 = R(125) / R(192),
                       a75 = R(-2187) / R(6784), a76 = R(11) / R(84);
    static constexpr R b1 = R(35) / R(384), b3 = R(500) / R(1113), b4 = R(125) / R(192),
                       b5 = R(-2187) / R(6784), b6 = R(11) / R(84);
    // embedded error weights b - b_hat
    static constexpr R e1 = R(35) / R(384) - R(5179) / R(57600);
    static constexpr R e3 = R(500) / R(1113) - R(7571) / R(16695);
    static constexpr R e4 = R(125) / R(192) - R(393) / R(640);
    static constexpr R e5 = R(-2187) / R(6784) + R(92097) / R(339200);
    static constexpr R e6 = R(11) / R(84) - R(187) / R(2100);
    static constexpr R e7 = R(-1) / R(40);
    // Hairer continuous-extension weights (cuda/kerr_math.cuh:188-193)
    static constexpr R d1 = R(-12715105075.0) / R(11282082432.0);
    static constexpr R d3 = R(87487479700.0) / R(32700410799.0);
    static constexpr R d4 = R(-10690763975.0) / R(1880347072.0);
    static constexpr R d5 = R(701980252875.0) / R(199316789632.0);
    static constexpr R d6 = R(-1453857185.0) / R(822651844.0);
    static constexpr R d7 = R(69997945.0) / R(29380423.0);
};

// ---- PCG hash (cuda/kerr_math.cuh:26-36) ------------------------------------------------
__device__ __forceinline__ uint32_t pcg_hash(uint64_t state) {
    const uint64_t x = state * 6364136223846793005ULL + 1442695040888963407ULL;
    const uint32_t xs = (uint32_t)(((x >> 18u) ^ x) >> 27u);
    const uint32_t rot = (uint32_t)(x >> 59u);
    return (xs >> rot) | (xs << ((32u - rot) & 31u));
}
__device__ __forceinline__ float unit_float(uint64_t state) {
    return (float)pcg_hash(state) * 2.3283064365386963e-10f;
}

// ---- Kerr-Schild radius with the spin along +y (cuda/kerr_math.cuh:50-59) ------------------
template <class R>
__device__ __forceinline__ R ks_radius(R x, R y, R z, R aa) {
    using O = Ops<R>;
    const R rho2 = O::fma(x, x, O::fma(y, y, z * z));
    const R u = rho2 - aa;
    const R s_sq = O::fma(u, u, R(4) * aa * y * y);
    const R inv_s = O::rsq(s_sq);
    const R s = s_sq * inv_s;
    const R r2 = R(0.5) * (u + s);
    return O::sqrt_rn(r2);
}

// ---- Hamiltonian right-hand side (cuda/kerr_math.cuh:82-156) -----------------------------
// y = (x, y, z, p_x, p_y, p_z); p_t = pt is conserved.  With the Kerr-Schild potential
// Hk = M r^3 / (r^4 + a^2 y^2) and null vector l, the RHS is
//   dx/dl = p - 2 Hk (l.p - pt) l,   dp/dl = dHk/dx (l.p - pt)^2 + 2 Hk (l.p - pt) d(l.p)/dx.
//
// EXACT selects the y-derivative of r^2.  The reference writes d(r^2)/dy = y (1 + (u + 4a^2)/(2s))
// (cuda/kerr_math.cuh:97); differentiating r^2 = (u + s)/2 with u = rho^2 - a^2 and
// s^2 = u^2 + 4 a^2 y^2 gives y (1 + (u + 2a^2)/s).  Reference mode keeps the reference's
// expression (the drop-in reproduces its images); stated-physics mode uses the exact one.
//
// Stated physics (EXACT) evaluates the same exact gradient in a shorter form.  With r_i = dr/dx_i,
// D = r^2 + a^2, N_x = r x - a z, N_z = r z + a x (l_x = N_x / D, l_z = N_z / D, l_y = y / r) and
// lp = l.p - pt, the momentum derivative of l.p is a multiple of grad r plus three direct terms,
//   d(l.p)/dx_i = r_i c + (r p_x + a p_z) / D [i = x], p_y / r [i = y], (r p_z - a p_x) / D [i = z],
//   c = (x p_x + z p_z) / D - 2 r (N_x p_x + N_z p_z) / D^2 - p_y y / r^2,
// and dHk/dx_i = r_i e - [i = y] f with e = M r^2 (3 a^2 y^2 - r^4) / denH^2 and
// f = 2 M a^2 y r^3 / denH^2 (denH = r^4 + a^2 y^2), so that
//   dp_i/dl = r_i (e lp^2 + 2 Hk lp c) - [i = y] f lp^2 + 2 Hk lp (direct term)_i,
// instead of the full 3 x 3 Jacobian of l that the reference form builds (about 40% fewer
// operations per evaluation).
template <class R, bool EXACT>
__device__ __forceinline__ void hamilton_rhs(const R* __restrict__ st, R pt, R a, R aa, R M,
                                             R* __restrict__ d) {
    using O = Ops<R>;
    const R x = st[0], y = st[1], z = st[2];
    const R px = st[3], py = st[4], pz = st[5];
    if constexpr (EXACT) {
        const R rho2 = O::fma(x, x, O::fma(y, y, z * z));
        const R u = rho2 - aa;
        const R aay2 = aa * y * y;
        const R s_sq = O::fma(u, u, R(4) * aay2);
        const R inv_s = O::rsq(s_sq);
        const R r2 = R(0.5) * O::fma(s_sq, inv_s, u);
        const R inv_r = O::rsq(r2);
        const R r = r2 * inv_r;
        const R half_inv_r = R(0.5) * inv_r;
        const R gxz = O::fma(u, inv_s, R(1)) * half_inv_r;     // r_x / x = r_z / z
        const R rx = x * gxz;
        const R rz = z * gxz;
        const R ry = y * (O::fma(u + R(2) * aa, inv_s, R(1)) * half_inv_r);
        const R den = r2 + aa;
        const R inv_den = O::fdiv(R(1), den);
        const R Nx = O::fma(r, x, -a * z);
        const R Nz = O::fma(r, z, a * x);
        const R lx = Nx * inv_den;
        const R ly = y * inv_r;
        const R lz = Nz * inv_den;
        const R r3 = r2 * r;
        const R denH = O::fma(r2, r2, aay2);
        const R inv_denH = O::fdiv(R(1), denH);
        const R Hk = M * r3 * inv_denH;
        const R lp = O::fma(lx, px, O::fma(ly, py, O::fma(lz, pz, -pt)));
        const R two_H_lp = R(2) * Hk * lp;
        d[0] = O::fma(-two_H_lp, lx, px);
        d[1] = O::fma(-two_H_lp, ly, py);
        d[2] = O::fma(-two_H_lp, lz, pz);
        const R A = O::fma(px, x, pz * z);
        const R B = O::fma(px, Nx, pz * Nz);
        const R c = O::fma(A - R(2) * r * B * inv_den, inv_den, -py * ly * inv_r);
        const R ih2 = inv_denH * inv_denH;
        const R e = M * r2 * O::fma(R(3), aay2, -r2 * r2) * ih2;
        const R f = R(2) * M * aa * y * r3 * ih2;
        const R lp2 = lp * lp;
        const R Q = O::fma(e, lp2, two_H_lp * c);
        const R tw = two_H_lp * inv_den;
        d[3] = O::fma(rx, Q, tw * O::fma(r, px, a * pz));
        d[4] = O::fma(ry, Q, O::fma(-f, lp2, two_H_lp * py * inv_r));
        d[5] = O::fma(rz, Q, tw * O::fma(r, pz, -a * px));
        return;
    }
    const R rho2 = O::fma(x, x, O::fma(y, y, z * z));
    const R u = rho2 - aa;
    const R s_sq = O::fma(u, u, R(4) * aa * y * y);
    const R inv_s = O::rsq(s_sq);
    const R r2 = R(0.5) * (u + s_sq * inv_s);
    const R inv_r = O::rsq(r2);
    const R r = r2 * inv_r;
    // gradient of r via r^2
    const R g2x = x * (R(1) + u * inv_s);
    const R g2y = EXACT ? y * (R(1) + (u + R(2) * aa) * inv_s)
                        : y * (R(1) + (u + R(4) * aa) * (R(0.5) * inv_s));
    const R g2z = z * (R(1) + u * inv_s);
    const R half_inv_r = R(0.5) * inv_r;
    const R rx = g2x * half_inv_r;
    const R ry = g2y * half_inv_r;
    const R rz = g2z * half_inv_r;
    // null vector l
    const R den = r2 + aa;
    const R inv_den = O::fdiv(R(1), den);
    const R inv_den2 = inv_den * inv_den;
    const R lx = (r * x - a * z) * inv_den;
    const R ly = y * inv_r;
    const R lz = (r * z + a * x) * inv_den;
    // potential
    const R r3 = r2 * r;
    const R denH = O::fma(r2, r2, aa * y * y);
    const R inv_denH = O::fdiv(R(1), denH);
    const R Hk = M * r3 * inv_denH;
    const R lp = O::fma(lx, px, O::fma(ly, py, O::fma(lz, pz, -pt)));
    const R two_H_lp = R(2) * Hk * lp;
    d[0] = px - two_H_lp * lx;
    d[1] = py - two_H_lp * ly;
    d[2] = pz - two_H_lp * lz;
    // derivatives of l_x = Nx / D and l_z = Nz / D, D = r^2 + a^2
    const R dDx = R(2) * r * rx;
    const R dDy = R(2) * r * ry;
    const R dDz = R(2) * r * rz;
    const R Nx = r * x - a * z;
    const R Nz = r * z + a * x;
    const R dNx_x = rx * x + r;
    const R dNx_y = ry * x;
    const R dNx_z = rz * x - a;
    const R dNz_x = rx * z + a;
    const R dNz_y = ry * z;
    const R dNz_z = rz * z + r;
    const R dlx_x = (dNx_x * den - Nx * dDx) * inv_den2;
    const R dlx_y = (dNx_y * den - Nx * dDy) * inv_den2;
    const R dlx_z = (dNx_z * den - Nx * dDz) * inv_den2;
    const R dlz_x = (dNz_x * den - Nz * dDx) * inv_den2;
    const R dlz_y = (dNz_y * den - Nz * dDy) * inv_den2;
    const R dlz_z = (dNz_z * den - Nz * dDz) * inv_den2;
    // derivatives of l_y = y / r
    const R inv_r2 = inv_r * inv_r;
    const R dly_x = -y * rx * inv_r2;
    const R dly_y = (r - y * ry) * inv_r2;
    const R dly_z = -y * rz * inv_r2;
    // derivatives of Hk
    const R dHd_x = R(4) * r3 * rx;
    const R dHd_y = O::fma(R(4) * r3, ry, R(2) * aa * y);
    const R dHd_z = R(4) * r3 * rz;
    const R inv_denH2 = inv_denH * inv_denH;
    const R fH = M * inv_denH2;
    const R dH_x = fH * (R(3) * r2 * rx * denH - r3 * dHd_x);
    const R dH_y = fH * (R(3) * r2 * ry * denH - r3 * dHd_y);
    const R dH_z = fH * (R(3) * r2 * rz * denH - r3 * dHd_z);
    const R dlp_x = dlx_x * px + dly_x * py + dlz_x * pz;
    const R dlp_y = dlx_y * px + dly_y * py + dlz_y * pz;
    const R dlp_z = dlx_z * px + dly_z * py + dlz_z * pz;
    const R lp2 = lp * lp;
    d[3] = dH_x * lp2 + two_H_lp * dlp_x;
    d[4] = dH_y * lp2 + two_H_lp * dlp_y;
    d[5] = dH_z * lp2 + two_H_lp * dlp_z;
}

// ---- DOPRI5 continuous extension in the step fraction t (cuda/kerr_math.cuh:186-219) -------
template <class R>
__device__ __forceinline__ R dense_eval(R y0, R y1, R k1, R k3, R k4, R k5, R k6, R k7, R h, R t) {
    using C = DP<R>;
    const R q1 = y0;
    const R q2 = y1 - y0;
    const R q3 = y0 + h * k1 - y1;
    const R q4 = R(2) * (y1 - y0) - h * (k1 + k7);
    const R q5 = h * (C::d1 * k1 + C::d3 * k3 + C::d4 * k4 + C::d5 * k5 + C::d6 * k6 + C::d7 * k7);
    const R t2 = t * t;
    const R t3 = t2 * t;
    const R t4 = t2 * t2;
    return q1 + t * (q2 + q3) - t2 * (q3 - q4 - q5) - t3 * (q4 + R(2) * q5) + t4 * q5;
}
template <class R>
__device__ __forceinline__ R dense_slope(R y0, R y1, R k1, R k3, R k4, R k5, R k6, R k7, R h, R t) {
    using C = DP<R>;
    const R q2 = y1 - y0;
    const R q3 = y0 + h * k1 - y1;
    const R q4 = R(2) * (y1 - y0) - h * (k1 + k7);
    const R q5 = h * (C::d1 * k1 + C::d3 * k3 + C::d4 * k4 + C::d5 * k5 + C::d6 * k6 + C::d7 * k7);
    const R t2 = t * t;
    const R t3 = t2 * t;
    return (q2 + q3) - R(2) * t * (q3 - q4 - q5) - R(3) * t2 * (q4 + R(2) * q5) + R(4) * t3 * q5;
}

// ---- gradient noise / FBM (cuda/kerr_math.cuh:172-179, 220-281) ----------------------------
// Float instantiation = the reference's arithmetic; double instantiation = the same lattice
// (same PCG hash, same float-rounded gradient angle) evaluated in double.
template <class R> __device__ __forceinline__ R smooth5(R t) { return t * t * t * (t * (t * R(6) - R(15)) + R(10)); }
template <class R> __device__ __forceinline__ R mixr(R a, R b, R t) { return Ops<R>::fma(t, b - a, a); }
template <class R>
__device__ __forceinline__ void lattice_gradient(int ix, int iy, unsigned seed, R& gx, R& gy) {
    const uint64_t key = (((uint64_t)(uint32_t)ix) << 32) | (uint64_t)(uint32_t)iy;
    const uint32_t hsh = pcg_hash(key ^ (uint64_t)seed);
    constexpr float kAngle = 6.283185307f * 2.3283064365386963e-10f;
    const R ang = (R)((float)hsh) * (R)kAngle;
    Ops<R>::sincosr(ang, &gy, &gx);
}
template <class R> __device__ __forceinline__ int floor_int(R v);
template <> __device__ __forceinline__ int floor_int<float>(float v) { return __float2int_rd(v); }
template <> __device__ __forceinline__ int floor_int<double>(double v) { return __double2int_rd(v); }
template <class R>
__device__ __forceinline__ R gradient_noise2(R u, R v, unsigned seed) {
    const int ix0 = floor_int<R>(u);
    const int iy0 = floor_int<R>(v);
    const int ix1 = ix0 + 1, iy1 = iy0 + 1;
    const R fx = u - (R)ix0;
    const R fy = v - (R)iy0;
    R g00x, g00y, g10x, g10y, g01x, g01y, g11x, g11y;
    lattice_gradient<R>(ix0, iy0, seed, g00x, g00y);
    lattice_gradient<R>(ix1, iy0, seed, g10x, g10y);
    lattice_gradient<R>(ix0, iy1, seed, g01x, g01y);
    lattice_gradient<R>(ix1, iy1, seed, g11x, g11y);
    const R n00 = g00x * fx + g00y * fy;
    const R n10 = g10x * (fx - R(1)) + g10y * fy;
    const R n01 = g01x * fx + g01y * (fy - R(1));
    const R n11 = g11x * (fx - R(1)) + g11y * (fy - R(1));
    const R uf = smooth5<R>(fx);
    const R vf = smooth5<R>(fy);
    const R m0 = mixr<R>(n00, n10, uf);
    const R m1 = mixr<R>(n01, n11, uf);
    return mixr<R>(m0, m1, vf);
}
template <class R>
__device__ __forceinline__ R fbm2(R u, R v, int octaves, unsigned seed) {
    if (octaves <= 0) return R(0.5);
    R sum = R(0), amp = R(1), freq = R(1), amp_sum = R(0);
    for (int o = 0; o < octaves; ++o) {
        sum += gradient_noise2<R>(u * freq, v * freq, seed) * amp;
        amp_sum += amp;
        amp *= R(0.5);
        freq *= R(2);
    }
    R val = amp_sum > R(0) ? (sum / amp_sum) : R(0);
    return val * R(0.5) + R(0.5);
}

// ---- procedural sky grid (cuda/kerr_math.cuh:157-171) -----------------------------------
__device__ __forceinline__ float asin_r(float x) { return asinf(x); }
__device__ __forceinline__ double asin_r(double x) { return asin(x); }
__device__ __forceinline__ float fmod_r(float a, float b) { return fmodf(a, b); }
__device__ __forceinline__ double fmod_r(double a, double b) { return fmod(a, b); }
template <class R>
__device__ __forceinline__ R sky_value(R dx, R dy, R dz, R tau, const Scene& sc) {
    const R lon = Ops<R>::atan2r(dz, dx);
    const R lat = asin_r(dy);
    const R spacing = (R)sc.sky_spacing;
    const R thick = (R)sc.sky_thickness;
    const R dlon = fmod_r(Ops<R>::absr(lon), spacing);
    const R dlat = fmod_r(Ops<R>::absr(lat), spacing);
    const bool on_line = (dlon < thick || dlon > (spacing - thick)) ||
                         (dlat < thick || dlat > (spacing - thick)) ||
                         (Ops<R>::absr(lat) < thick * R(3));
    return on_line ? (R)(sc.sky_intensity * (double)tau) : R(0);
}

// ---- LUT sampling ------------------------------------------------------------------------
// Software form of a 1D linear, normalised, clamped texture fetch (full-precision weight).
template <class R, class E = float>
__device__ __forceinline__ R lut_lerp1(const E* __restrict__ lut, int n, R u) {
    const R x = u * R(n) - R(0.5);
    const R fl = floor(x);
    const R w = x - fl;
    // clamp in floating point first so that NaN / huge coordinates cannot overflow the int
    const R flc = fl < R(-1) ? R(-1) : (fl > R(n - 1) ? R(n - 1) : fl);
    int i0 = fl == fl ? (int)flc : 0;
    int i1 = i0 + 1;
    i0 = i0 < 0 ? 0 : i0;
    i1 = i1 > n - 1 ? n - 1 : i1;
    const R v0 = (R)__ldg(lut + i0), v1 = (R)__ldg(lut + i1);
    return v0 + w * (v1 - v0);
}
template <class R>
__device__ __forceinline__ float4 lut_lerp4(const float4* __restrict__ lut, int n, R u) {
    const R x = u * R(n) - R(0.5);
    const R fl = floor(x);
    const R w = x - fl;
    // clamp in floating point first so that NaN / huge coordinates cannot overflow the int
    const R flc = fl < R(-1) ? R(-1) : (fl > R(n - 1) ? R(n - 1) : fl);
    int i0 = fl == fl ? (int)flc : 0;
    int i1 = i0 + 1;
    i0 = i0 < 0 ? 0 : i0;
    i1 = i1 > n - 1 ? n - 1 : i1;
    const float4 a = __ldg(lut + i0), b = __ldg(lut + i1);
    return make_float4((float)(a.x + w * (b.x - a.x)), (float)(a.y + w * (b.y - a.y)),
                       (float)(a.z + w * (b.z - a.z)), 0.0f);
}

// Software model of the texture unit's linear filter for plain device arrays (used where no
// texture object exists): the same coordinate, the weight rounded to 1/256 as the hardware's
// 1.8 fixed-point weight (checked against the texture unit to about 2e-5 of the LUT range).
__device__ __forceinline__ void tex_model_coord(int n, float u, int& i0, int& i1, float& w) {
    const float x = u * (float)n - 0.5f;
    const float fl = floorf(x);
    w = rintf((x - fl) * 256.0f) * (1.0f / 256.0f);
    const float flc = fminf(fmaxf(fl, -1.0f), (float)(n - 1));
    i0 = fl == fl ? (int)flc : 0;
    i1 = min(i0 + 1, n - 1);
    i0 = max(i0, 0);
}
__device__ __forceinline__ float lut_tex_model1(const float* __restrict__ lut, int n, float u) {
    int i0, i1;
    float w;
    tex_model_coord(n, u, i0, i1, w);
    return (1.0f - w) * __ldg(lut + i0) + w * __ldg(lut + i1);
}
__device__ __forceinline__ float4 lut_tex_model4(const float4* __restrict__ lut, int n, float u) {
    int i0, i1;
    float w;
    tex_model_coord(n, u, i0, i1, w);
    const float4 a = __ldg(lut + i0), b = __ldg(lut + i1);
    const float v = 1.0f - w;
    return make_float4(v * a.x + w * b.x, v * a.y + w * b.y, v * a.z + w * b.z, 0.0f);
}

// Blackbody colour of temperature T with the reference's overflow report
// (cuda/kernel.cu:1-16): above lut_max_temp the first thread to notice records T.
// MODE 0 samples the texture object, MODE 2 the plain array through the texture-unit model,
// MODE 1 the plain array with the exact weight.
template <int MODE>
__device__ __forceinline__ float3 blackbody_rgb(float T, const Scene& sc, uint32_t* err) {
    if (T > sc.lut_max_temp) {
        if (atomicCAS(err, 0u, 1u) == 0u) err[1] = __float_as_uint(T);
        return make_float3(0.0f, 0.0f, 0.0f);
    }
    const float tn = T / sc.lut_max_temp;
    const float pos = tn * (float)(sc.lut_size - 1);
    const float u = (pos + 0.5f) / (float)sc.lut_size;
    float4 c;
    if (MODE == 0) c = tex1D<float4>(sc.bb_tex, u);
    else if (MODE == 2) c = lut_tex_model4(sc.bb_lut, sc.lut_size, u);
    else c = lut_lerp4<float>(sc.bb_lut, sc.lut_size, u);
    return make_float3(c.x, c.y, c.z);
}

// ---- Boyer-Lindquist angles of a Kerr-Schild point (cuda/kerr_math.cuh:60-81) --------------
template <class R>
__device__ __forceinline__ void ks_to_bl(R x, R y, R z, R a, R aa, R& r, R& sin_th, R& cos_th,
                                         R& phi) {
    using O = Ops<R>;
    const R rho2 = O::fma(x, x, O::fma(y, y, z * z));
    const R u = rho2 - aa;
    const R s_sq = O::fma(u, u, R(4) * aa * y * y);
    const R inv_s = O::rsq(s_sq);
    const R s = s_sq * inv_s;
    const R r2 = R(0.5) * (u + s);
    const R inv_r = O::rsq(r2);
    r = r2 * inv_r;
    cos_th = y * inv_r;
    const R c2 = cos_th * cos_th;
    const R s2 = R(1) - c2;
    const R inv_sin = O::rsq(s2);
    sin_th = s2 * inv_sin;
    const R den = r2 + aa;
    const R inv = inv_sin * O::fdiv(R(1), den);
    const R cphi = (r * z + a * x) * inv;
    const R sphi = (r * x - a * z) * inv;
    phi = O::atan2r(sphi, cphi);
}

}  // namespace ktd
