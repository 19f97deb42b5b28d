// kt_diff.cu — differentiable trace (stated physics, spp 1, no disk noise).
//
// Three kernels share the ray code of the renderer (ray_advance<R, 1, true>), so the recorded
// forward image is bit for bit the stated-physics trace of the same scene (float path):
//
//   diff_forward_kernel<R, false>  adaptive trace; appends each accepted step size to the ray's
//                                  segment records (state + transmittance at every kSegSteps-th
//                                  step), writes the ray's event summary.
//   diff_forward_kernel<R, true>   frozen-step replay: the recorded step sizes, one attempt each
//                                  (max_attempts = 1 in the scene), at new parameters; flags the
//                                  rays whose events differ from the record.  Central
//                                  differences of the frozen-step model use it.
//   diff_backward_kernel<R>        discrete adjoint.  Per ray, from the last segment back: sweep
//                                  the segment forward from its checkpoint (states and stages of
//                                  each step, transmittance at the crossings the record marks as
//                                  shaded, kept in local memory), then reverse each step:
//     * crossing: the hit is the dense-output point at the root t* of y(t) = 0; its shading
//       (disk test, redshift, LUT temperature, blackbody, alpha) is differentiated with duals
//       in the hit state, p_t, k_t, spin, temperature scale and r_out; the transmittance chain
//       col += c a tau, tau' = tau (1 - a) is reversed; t* is differentiated by the
//       implicit-function theorem (dt* = -dy / y'(t*)) and the dense output's linear weights
//       carry the adjoint to the step's end points and stages;
//     * step: reverse of the explicit Runge-Kutta map with the step size frozen.  The
//       vector-Jacobian product of the right-hand side uses that f = J grad H is Hamiltonian:
//       J_f^T l = J^T J_f (J^T l), a forward (dual-number) JVP of hamilton_rhs in direction
//       J^T l = (-l_p, l_x); the same dual evaluation gives l . df/d(spin) and l . df/d(p_t).
//   At the start, the null initialisation is differentiated with duals in spin and
//   inclination (the camera's inclination tangent comes from the host).
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "kt_diff.h"
#include "kt_dual.cuh"
#include "kt_internal.h"
#include "kt_ray.cuh"

namespace ktd {

namespace {

constexpr unsigned kFullMask = 0xffffffffu;

template <class R>
__device__ __forceinline__ DiffSeg<R>* seg_at(const DiffRecRaw& rec, int i) {
    return reinterpret_cast<DiffSeg<R>*>(rec.segs) + i;
}

// Kind of ending of a ray whose advance() just returned true (same tests, same order as
// ray_advance): NaN state, inside the horizon, beyond the escape radius, else the budget.
template <class R>
__device__ __forceinline__ int classify_end(const RayRun<R>& ry, const Scene& sc) {
    if (Ops<R>::isnanr(ry.s[1])) return kTermFrozen;
    const R r_now = ks_radius<R>(ry.s[0], ry.s[1], ry.s[2], sc_aa<R>(sc));
    if (inside_horizon<R>(r_now, sc)) return kTermHorizon;
    if (beyond_escape<R>(r_now, sc)) return kTermEscape;
    return kTermBudget;
}

// Sky value at transmittance 1 in the escape direction of state s (ray_advance's escape branch).
template <class R>
__device__ __forceinline__ R escape_sky(const R* s, R pt, const Scene& sc) {
    using O = Ops<R>;
    R ke[6];
    hamilton_rhs<R, true>(s, pt, sc_a<R>(sc), sc_aa<R>(sc), sc_M<R>(sc), ke);
    const R inv = O::rsq(ke[0] * ke[0] + ke[1] * ke[1] + ke[2] * ke[2]);
    return sky_value<R>(ke[0] * inv, ke[1] * inv, ke[2] * inv, R(1), sc);
}

}  // namespace

// ---- adjoint helpers ---------------------------------------------------------------------------

// Weights of the dense output in (y0, y1, k1, k3, k4, k5, k6, k7): it is linear in them.
template <class R>
__device__ __forceinline__ void dense_weights(R t, R h, R w[8]) {
    using C = DP<R>;
    const R t2 = t * t, t3 = t2 * t, t4 = t2 * t2;
    const R q2 = t, q3 = t - t2, q4 = t2 - t3, q5 = t2 - R(2) * t3 + t4;
    w[0] = R(1) - q2 + q3 - R(2) * q4;
    w[1] = q2 - q3 + R(2) * q4;
    w[2] = h * (q3 - q4 + C::d1 * q5);
    w[3] = h * (C::d3 * q5);
    w[4] = h * (C::d4 * q5);
    w[5] = h * (C::d5 * q5);
    w[6] = h * (C::d6 * q5);
    w[7] = h * (-q4 + C::d7 * q5);
}

// l^T df/dY at Y (out), l . df/d(spin) (da) and l . df/d(p_t) (dpt), from one dual evaluation
// of the right-hand side in direction (J^T l, d spin, d p_t).
template <class R>
__device__ __forceinline__ void rhs_vjp(const R* Y, const R* l, R pt, R a, R aa, R M, R* out, R& da, R& dpt) {
    using D = Dual<R, 3>;
    D st[6], d[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) st[c] = D(Y[c]);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        st[c].d[0] = -l[c + 3];
        st[c + 3].d[0] = l[c];
    }
    D Da(a), Daa(aa), Dpt(pt), DM(M);
    Da.d[1] = R(1);
    Daa.d[1] = R(2) * a;
    Dpt.d[2] = R(1);
    hamilton_rhs<D, true>(st, Dpt, Da, Daa, DM, d);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        out[c] = -d[c + 3].d[0];
        out[c + 3] = d[c].d[0];
    }
    R sa = R(0), sp = R(0);
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        sa += l[c] * d[c].d[1];
        sp += l[c] * d[c].d[2];
    }
    da = sa;
    dpt = sp;
}

// Tangent slots of the shading duals.
enum : int { kSX = 0, kSPt = 6, kSKt = 7, kSA = 8, kSTs = 9, kSRo = 10, kSN = 11 };

// Value / tangent helpers shared by the plain and the dual evaluation of the shading.
template <class R> __device__ __forceinline__ R val(R x) { return x; }
template <class R, int N> __device__ __forceinline__ R val(const Dual<R, N>& x) { return x.v; }
template <class T, class R>
__device__ __forceinline__ T seeded(R x, int slot) {
    if constexpr (std::is_same<T, R>::value) return x;
    else return T::seed(x, slot);
}
// a scene input with its derivatives in the shading slots (plain value for T = R)
template <class T, class R>
__device__ __forceinline__ T with_tangent(R x, int slot, R dx) {
    T r(x);
    if constexpr (!std::is_same<T, R>::value) r.d[slot] = dx;
    return r;
}

// Disk shading of hit state X (shade_hit<R, 1> without noise), on plain values (T = R) or on
// duals in the hit state, p_t, k_t, spin, temperature scale and r_out (T = Dual<R, kSN>):
// returns false where the hit is not shaded; else the blackbody colour c and the opacity alpha.
template <class R, class T>
__device__ bool shade_eval(const R* X, R pt, R kt, const Scene& sc, const DiffLut& dl, T* c3, T& alpha) {
    using O = Ops<T>;
    const T xh = seeded<T>(X[0], kSX + 0), zh = seeded<T>(X[2], kSX + 2);
    const T pxh = seeded<T>(X[3], kSX + 3), pzh = seeded<T>(X[5], kSX + 5);
    const T Dpt = seeded<T>(pt, kSPt), Dkt = seeded<T>(kt, kSKt);
    const T a = seeded<T>(sc_a<R>(sc), kSA);
    const T aa = a * a;
    const R M = sc_M<R>(sc);
    const T r_in = with_tangent<T>(sizeof(R) == 8 ? (R)sc.disk_inner_d : (R)sc.disk_inner, kSA, (R)dl.dr_in_da);
    const T r_out = seeded<T>(sizeof(R) == 8 ? (R)sc.disk_outer_d : (R)sc.disk_outer, kSRo);
    const T rh = ks_radius<T>(xh, T(R(0)), zh, aa);
    if (!(val(rh) >= val(r_in) && val(rh) <= val(r_out))) return false;
    const R sqM = Ops<R>::sqrt_rn(M);
    const T rs = O::sqrt_rn(rh);
    const T disc = R(1) - R(3) * M / rh + R(2) * sqM * a / (rh * rs);
    if (!(val(disc) > R(0))) return false;
    const T omega = -sqM / (rh * rs + a * sqM);
    const T r2h = rh * rh;
    const T inv = R(1) / (r2h + aa);
    const T lx = (rh * xh - a * zh) * inv;
    const T lz = (rh * zh + a * xh) * inv;
    const T ldotp = O::fma(lx, pxh, lz * pzh);
    const T ldotxi = lx * zh - lz * xh;
    const T Hk = M * rh * r2h / (r2h * r2h);
    const T L = (zh * pxh - xh * pzh) + R(2) * Hk * ldotxi * (ldotp + Dkt);
    const T energy = -Dpt;
    const T l_over_e = L / energy;
    const T g = R(1) / (O::rsq(disc) * (R(1) - omega * l_over_e));
    const T span = r_out - r_in;
    const T u = val(span) > R(0) ? (rh - r_in) / span : T(R(0));
    // disk LUT, software linear fetch (lut_lerp1); the entries carry their spin / r_out tangents
    const int n = sc.lut_size;
    const T x = u * R(n) - R(0.5);
    const R fl = floor(val(x));
    const R flc = fl < R(-1) ? R(-1) : (fl > R(n - 1) ? R(n - 1) : fl);
    int i0 = fl == fl ? (int)flc : 0;
    int i1 = i0 + 1;
    i0 = i0 < 0 ? 0 : i0;
    i1 = i1 > n - 1 ? n - 1 : i1;
    const bool lut_d = sizeof(R) == 8 && sc.disk_lut_d;
    T v0 = with_tangent<T>(lut_d ? (R)__ldg(sc.disk_lut_d + i0) : (R)__ldg(sc.disk_lut + i0), kSA,
                           (R)__ldg(dl.dlut_da + i0));
    T v1 = with_tangent<T>(lut_d ? (R)__ldg(sc.disk_lut_d + i1) : (R)__ldg(sc.disk_lut + i1), kSA,
                           (R)__ldg(dl.dlut_da + i1));
    if constexpr (!std::is_same<T, R>::value) {
        v0.d[kSRo] = (R)__ldg(dl.dlut_dro + i0);
        v1.d[kSRo] = (R)__ldg(dl.dlut_dro + i1);
    }
    const T w = x - fl;
    T sampled = v0 + w * (v1 - v0);
    if constexpr (!std::is_same<T, R>::value && sizeof(R) == 4) {
        // Spin and r_out move the table's nodes and, at a fixed hit radius, the fetch coordinate;
        // the two nearly cancel (the table samples one function of r), so these two tangents are
        // summed in double from the double table: in float the remainder keeps few digits.
        const double span_d = (double)val(r_out) - (double)val(r_in);
        const double rh_d = (double)val(rh), wv = (double)val(w);
        const double dv = __ldg(dl.lut_d + i1) - __ldg(dl.lut_d + i0);
        const double du_drh = 1.0 / span_d;
        const double du_da = -dl.dr_in_da * ((double)val(r_out) - rh_d) / (span_d * span_d);
        const double du_dro = -(rh_d - (double)val(r_in)) / (span_d * span_d);
        const double ga = dv * (double)n * (du_drh * (double)rh.d[kSA] + du_da) +
                          (1.0 - wv) * __ldg(dl.dlut_da + i0) + wv * __ldg(dl.dlut_da + i1);
        const double gro = dv * (double)n * du_dro + (1.0 - wv) * __ldg(dl.dlut_dro + i0) + wv * __ldg(dl.dlut_dro + i1);
        sampled.d[kSA] = (R)ga;
        sampled.d[kSRo] = (R)gro;
    }
    const T ts = with_tangent<T>((R)sc.temp_scale, kSTs, (R)dl.dtemp_ds);
    const T T_ = ts * sampled * g;
    if (!(Ops<R>::isfiniter(val(T_)) && val(T_) > R(0))) return false;
    // blackbody LUT (blackbody_rgb<1> / blackbody_rgb_d): linear in T between two entries
    if (val(T_) > (R)sc.lut_max_temp) {
        c3[0] = c3[1] = c3[2] = T(R(0));
        alpha = T(R(0));
        return true;
    }
    const int nb = sc.lut_size;
    const T pos = T_ / (R)sc.lut_max_temp * R(nb - 1);
    const R fb = floor(val(pos));
    const R fbc = fb < R(-1) ? R(-1) : (fb > R(nb - 1) ? R(nb - 1) : fb);
    int j0 = fb == fb ? (int)fbc : 0;
    int j1 = j0 + 1;
    j0 = j0 < 0 ? 0 : j0;
    j1 = j1 > nb - 1 ? nb - 1 : j1;
    const float4 ca = __ldg(sc.bb_lut + j0), cb = __ldg(sc.bb_lut + j1);
    const T wb = pos - fb;
    c3[0] = (R)ca.x + wb * (R)(cb.x - ca.x);
    c3[1] = (R)ca.y + wb * (R)(cb.y - ca.y);
    c3[2] = (R)ca.z + wb * (R)(cb.z - ca.z);
    const T luma = R(0.2126) * c3[0] + R(0.7152) * c3[1] + R(0.0722) * c3[2];
    const T luma_s = luma / (R)sc.wl_step;
    alpha = R(1) - O::expr(luma_s * R(-0.5));
    return true;
}

// Null initialisation of ray_start on any number type (values, or duals for its derivatives):
// p_t from the null condition with the "-sqrt" root, p = n + 2 Hk l (k_t + l.n).
template <class T, class R>
__device__ __forceinline__ void start_state(const T* pos, const T* dirv, T a, R M, T* s, T& pt, T& kt) {
    using O = Ops<T>;
    const T aa = a * a;
    const T inv_n = O::rsq(dirv[0] * dirv[0] + dirv[1] * dirv[1] + dirv[2] * dirv[2]);
    const T nx = dirv[0] * inv_n, ny = dirv[1] * inv_n, nz = dirv[2] * inv_n;
    const T x = pos[0], y = pos[1], z = pos[2];
    const T rho2 = O::fma(x, x, O::fma(y, y, z * z));
    const T uu = rho2 - aa;
    const T s_term = O::sqrt_rn(O::fma(uu, uu, R(4) * aa * y * y));
    const T r2 = R(0.5) * (uu + s_term);
    const T r = O::sqrt_rn(r2);
    const T den = r2 + aa;
    const T inv_den = O::fdiv(T(R(1)), den);
    const T lx = (r * x - a * z) * inv_den;
    const T ly = O::fdiv(y, r);
    const T lz = (r * z + a * x) * inv_den;
    const T denH = O::fma(r2, r2, aa * y * y);
    const T Hk = M * r2 * r * O::fdiv(T(R(1)), denH);
    const T ln = O::fma(lx, nx, O::fma(ly, ny, lz * nz));
    const T g_tt = R(-1) + R(2) * Hk;
    const T g_tn = R(2) * Hk * ln;
    const T g_nn = R(1) + R(2) * Hk * ln * ln;
    const T disc = g_tn * g_tn - g_tt * g_nn;
    kt = (-g_tn - O::sqrt_rn(disc)) / g_tt;
    pt = g_tt * kt + g_tn;
    const T w = kt + ln;
    s[0] = x;
    s[1] = y;
    s[2] = z;
    s[3] = nx + R(2) * Hk * lx * w;
    s[4] = ny + R(2) * Hk * ly * w;
    s[5] = nz + R(2) * Hk * lz * w;
}

// Screen coordinates of a pixel centre (pixel_ray<1> at spp 1), in double.
__device__ __forceinline__ void pixel_uv(int px, int py, const Scene& sc, double fov, double& u, double& v) {
    const double W = (double)sc.width, H = (double)sc.height;
    u = ((px + 0.5) * (2.0 / W) - 1.0) * (W / H) * fov;
    v = (1.0 - (py + 0.5) * (2.0 / H)) * fov;
}

// Start of a pixel's ray.  Float: the renderer's start from the float camera (so the record is
// the renderer's image).  Double: the same initialisation from the double camera.
template <class R>
__device__ __forceinline__ bool ray_begin(int px, int py, const Scene& sc, const Camera& cam, const CameraD& camd,
                                          RayRun<R>& ry) {
    if constexpr (sizeof(R) == 4) {
        float dir[3];
        pixel_ray<1>(px, py, 0, sc, cam, dir);
        return start(ry, cam, dir, sc);
    } else {
        double u, v, dirv[3];
        pixel_uv(px, py, sc, camd.fov_scale, u, v);
#pragma unroll
        for (int c = 0; c < 3; ++c) dirv[c] = u * camd.rgt[c] + v * camd.up[c] + camd.fwd[c];
        start_state<double, double>(camd.pos, dirv, sc.a_d, sc.M_d, ry.s, ry.pt, ry.kt);
        ry.h = sc.h0_d;
        ry.tol = 0.0;
        ry.col[0] = ry.col[1] = ry.col[2] = 0.0;
        ry.tau = 1.0;
        ry.step = 0;
        ry.attempt = 0;
        ry.have_k1 = false;
        return 0 < sc.max_steps && 1.0f > sc.cutoff_gt;
    }
}

// Start state with derivatives in spin (slot 0) and inclination (slot 1).
template <class R>
__device__ __forceinline__ void start_dual(int px, int py, const Scene& sc, const Camera& cam, const CameraD& camd,
                                           const CameraD& dcamd, Dual<R, 2>* s, Dual<R, 2>& pt, Dual<R, 2>& kt) {
    using D = Dual<R, 2>;
    D dirv[3], pos[3];
    if constexpr (sizeof(R) == 4) {
        const float u = ((px + 0.5f) * sc.inv_w_2 - 1.0f) * sc.aspect * cam.fov_scale;
        const float v = (1.0f - (py + 0.5f) * sc.inv_h_2) * cam.fov_scale;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            dirv[c] = D((R)(u * cam.rgt[c] + v * cam.up[c] + cam.fwd[c]));
            dirv[c].d[1] = (R)(u * dcamd.rgt[c] + v * dcamd.up[c] + dcamd.fwd[c]);
            pos[c] = D((R)cam.pos[c]);
            pos[c].d[1] = (R)dcamd.pos[c];
        }
    } else {
        double u, v;
        pixel_uv(px, py, sc, camd.fov_scale, u, v);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            dirv[c] = D(u * camd.rgt[c] + v * camd.up[c] + camd.fwd[c]);
            dirv[c].d[1] = u * dcamd.rgt[c] + v * dcamd.up[c] + dcamd.fwd[c];
            pos[c] = D(camd.pos[c]);
            pos[c].d[1] = dcamd.pos[c];
        }
    }
    start_state<D, R>(pos, dirv, D::seed(sc_a<R>(sc), 0), sc_M<R>(sc), s, pt, kt);
}

// Stages of one DP5 step from s with step h (ray_advance's expressions): k[0..6] = k1..k7,
// nx = the 5th-order state.
template <class R>
// Stages k1..k6 into k, the 5th-order state into nx and k7 = f(nx) into k7.
__device__ __forceinline__ void dp5_stages(const R* s, R h, R pt, R a, R aa, R M, R (*k)[6], R* nx, R* k7,
                                           bool k1_given = false) {
    using C = DP<R>;
    R y[6];
    if (!k1_given) hamilton_rhs<R, true>(s, pt, a, aa, M, k[0]);
#pragma unroll
    for (int c = 0; c < 6; ++c) y[c] = s[c] + h * C::a21 * k[0][c];
    hamilton_rhs<R, true>(y, pt, a, aa, M, k[1]);
#pragma unroll
    for (int c = 0; c < 6; ++c) y[c] = s[c] + h * (C::a31 * k[0][c] + C::a32 * k[1][c]);
    hamilton_rhs<R, true>(y, pt, a, aa, M, k[2]);
#pragma unroll
    for (int c = 0; c < 6; ++c) y[c] = s[c] + h * (C::a41 * k[0][c] + C::a42 * k[1][c] + C::a43 * k[2][c]);
    hamilton_rhs<R, true>(y, pt, a, aa, M, k[3]);
#pragma unroll
    for (int c = 0; c < 6; ++c)
        y[c] = s[c] + h * (C::a51 * k[0][c] + C::a52 * k[1][c] + C::a53 * k[2][c] + C::a54 * k[3][c]);
    hamilton_rhs<R, true>(y, pt, a, aa, M, k[4]);
#pragma unroll
    for (int c = 0; c < 6; ++c)
        y[c] = s[c] + h * (C::a61 * k[0][c] + C::a62 * k[1][c] + C::a63 * k[2][c] + C::a64 * k[3][c] +
                           C::a65 * k[4][c]);
    hamilton_rhs<R, true>(y, pt, a, aa, M, k[5]);
#pragma unroll
    for (int c = 0; c < 6; ++c)
        nx[c] = s[c] + h * (C::b1 * k[0][c] + C::b3 * k[2][c] + C::b4 * k[3][c] + C::b5 * k[4][c] +
                            C::b6 * k[5][c]);
    hamilton_rhs<R, true>(nx, pt, a, aa, M, k7);
}

// Runge-Kutta matrix with row 7 = b (the stage-7 input is the 5th-order state).
template <class R>
__device__ __forceinline__ R rk_a(int m, int j) {
    using C = DP<R>;
    switch (m * 8 + j) {
        case 2 * 8 + 1: return C::a21;
        case 3 * 8 + 1: return C::a31;
        case 3 * 8 + 2: return C::a32;
        case 4 * 8 + 1: return C::a41;
        case 4 * 8 + 2: return C::a42;
        case 4 * 8 + 3: return C::a43;
        case 5 * 8 + 1: return C::a51;
        case 5 * 8 + 2: return C::a52;
        case 5 * 8 + 3: return C::a53;
        case 5 * 8 + 4: return C::a54;
        case 6 * 8 + 1: return C::a61;
        case 6 * 8 + 2: return C::a62;
        case 6 * 8 + 3: return C::a63;
        case 6 * 8 + 4: return C::a64;
        case 6 * 8 + 5: return C::a65;
        case 7 * 8 + 1: return C::b1;
        case 7 * 8 + 3: return C::b3;
        case 7 * 8 + 4: return C::b4;
        case 7 * 8 + 5: return C::b5;
        case 7 * 8 + 6: return C::b6;
        default: return R(0);
    }
}

// ---- forward: record / replay ----------------------------------------------------------------
// Four resident 128-thread blocks per SM: 128 registers at most (the FP64 kernel spills about
// 400 B there; 192 registers and two blocks otherwise).
// RR: arithmetic type of the records (R, or float records replayed in double arithmetic).
template <class R, bool REPLAY, class RR = R>
__global__ void __launch_bounds__(128, 4) diff_forward_kernel(const Scene sc, const Camera cam, const CameraD camd,
                                                          const DiffRecRaw rec, float4* __restrict__ hdr,
                                                          double* __restrict__ hdr64, uint32_t* __restrict__ err,
                                                          uint32_t* __restrict__ flags) {
    const unsigned n_px = (unsigned)sc.width * (unsigned)sc.height;
    const unsigned p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n_px) return;
    const int px = (int)(p % (unsigned)sc.width), py = (int)(p / (unsigned)sc.width);
    RayRun<R> ry;
    Tally tl;
    tl.clear();
    const bool started = ray_begin<R>(px, py, sc, cam, camd, ry);
    if (!REPLAY) {
        DiffRay out;
        out.first_seg = out.last_seg = -1;
        out.n_steps = 0;
        out.n_hits = 0;
        out.term = kTermNotStarted;
        out.sky = 0.0f;
        if (started) {
            int cur = -1, in_seg = 0;
            bool rec_ok = true;
            DiffSeg<R>* sg = nullptr;
            while (true) {
                if (ry.attempt == 0 && in_seg == 0 && rec_ok) {  // a step starts a new segment
                    const unsigned idx = atomicAdd(rec.seg_count, 1u);
                    if (idx >= rec.cap) {
                        rec_ok = false;
                        atomicAdd(rec.status, 1u);
                    } else {
                        sg = seg_at<R>(rec, (int)idx);
                        sg->prev = cur;
                        sg->next = -1;
                        sg->n = 0;
                        sg->hits = 0u;
                        sg->first_step = out.n_steps;
                        sg->tau = ry.tau;
#pragma unroll
                        for (int c = 0; c < 6; ++c) sg->s[c] = ry.s[c];
                        if (cur >= 0) seg_at<R>(rec, cur)->next = (int)idx;
                        else out.first_seg = (int)idx;
                        cur = (int)idx;
                    }
                }
                const R h_used = ry.h;
                const uint32_t hits0 = tl.hits;
                const bool done = advance<1, true>(ry, sc, err, tl);
                if (ry.attempt != 0) continue;  // rejected attempt: the step is retried
                if (Ops<R>::isnanr(ry.s[1])) {  // frozen: this step is not part of the record
                    out.term = kTermFrozen;
                    break;
                }
                if (rec_ok) {
                    sg->h[in_seg] = h_used;
                    if (tl.hits != hits0) sg->hits |= 1u << in_seg;
                    sg->n = ++in_seg;
                    out.last_seg = cur;
                    if (in_seg == kSegSteps) in_seg = 0;
                }
                ++out.n_steps;
                if (done) {
                    out.term = classify_end<R>(ry, sc);
                    if (out.term == kTermEscape) out.sky = (float)escape_sky<R>(ry.s, ry.pt, sc);
                    break;
                }
            }
            if (!rec_ok) out.term = kTermOverflow;
            // a segment opened by a step that froze holds no step: drop it from the list
            if (rec_ok && sg && sg->n == 0) {
                out.last_seg = sg->prev;
                if (sg->prev >= 0) seg_at<R>(rec, sg->prev)->next = -1;
                else out.first_seg = -1;
            }
        }
        out.n_hits = (int)tl.hits;
        rec.rays[p] = out;
    } else {
        const DiffRay rr = rec.rays[p];
        uint32_t flip = 0;
        int n_done = 0;
        int term = kTermNotStarted;
        if (started != (rr.term != kTermNotStarted)) flip = 1;
        if (started && rr.term != kTermNotStarted && rr.term != kTermOverflow) {
            bool done = false;
            for (int si = rr.first_seg; si >= 0 && !done; si = seg_at<RR>(rec, si)->next) {
                const DiffSeg<RR>* sg = seg_at<RR>(rec, si);
                for (int j = 0; j < sg->n && !done; ++j) {
                    ry.h = (R)sg->h[j];
                    done = advance<1, true>(ry, sc, err, tl);  // one attempt: always a commit
                    ++n_done;
                }
            }
            // a recorded ray that froze stops after its last recorded step (the NaN step adds
            // nothing to the image)
            if (done) term = classify_end<R>(ry, sc);
            else term = rr.term == kTermFrozen ? kTermFrozen : -1;
            if (term != rr.term || n_done != rr.n_steps || (int)tl.hits != rr.n_hits) flip = 1;
        } else if (rr.term == kTermOverflow) {
            flip = 1;
        }
        if (flags) flags[p] = flip;
    }
    const float fs = sc.final_scale;
    hdr[p] = make_float4((float)ry.col[0] * fs, (float)ry.col[1] * fs, (float)ry.col[2] * fs, 1.0f);
    if (hdr64) {
#pragma unroll
        for (int c = 0; c < 3; ++c) hdr64[3 * (size_t)p + c] = (double)ry.col[c] * (double)fs;
    }
}

// ---- adjoint work order ------------------------------------------------------------------------
// The backward's cost per ray is the number of steps up to its last shaded crossing, which
// ranges from a few to hundreds.  Rays are bucketed by that count (two buckets per power of 2,
// longest first) and the adjoint kernel takes them in bucket order, so that the rays of a warp
// have similar lengths; rays without a gradient path are left out.
constexpr int kWorkBuckets = 32;

template <class R>
__device__ __forceinline__ int backward_bucket(const DiffRecRaw& rec, const DiffRay& rr, float4 dlp) {
    const bool live = rr.term != kTermNotStarted && rr.term != kTermOverflow && rr.last_seg >= 0 && rr.n_hits > 0 &&
                      (dlp.x != 0.0f || dlp.y != 0.0f || dlp.z != 0.0f);
    if (!live) return -1;
    int si = rr.last_seg;
    while (si >= 0 && seg_at<R>(rec, si)->hits == 0u) si = seg_at<R>(rec, si)->prev;
    if (si < 0) return -1;
    const DiffSeg<R>* sg = seg_at<R>(rec, si);
    const unsigned w = (unsigned)sg->first_step + (unsigned)(32 - __clz((int)sg->hits));
    const int lg = (int)(2.0f * __log2f((float)w));
    return kWorkBuckets - 1 - (lg < 0 ? 0 : (lg > kWorkBuckets - 1 ? kWorkBuckets - 1 : lg));
}

// bucket of every pixel (-1: no work) and the bucket sizes; ctl[0..31] counts, ctl[32..63] cursors
template <class R>
__global__ void __launch_bounds__(256) diff_bucket_kernel(const Scene sc, const DiffRecRaw rec,
                                                         const float4* __restrict__ dl_dhdr, int* __restrict__ bucket,
                                                         unsigned* __restrict__ ctl) {
    __shared__ unsigned hist[kWorkBuckets];
    if (threadIdx.x < kWorkBuckets) hist[threadIdx.x] = 0u;
    __syncthreads();
    const unsigned n = (unsigned)sc.width * (unsigned)sc.height;
    const unsigned p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < n) {
        const int b = backward_bucket<R>(rec, rec.rays[p], dl_dhdr[p]);
        bucket[p] = b;
        if (b >= 0) atomicAdd(&hist[b], 1u);
    }
    __syncthreads();
    if (threadIdx.x < kWorkBuckets && hist[threadIdx.x]) atomicAdd(&ctl[threadIdx.x], hist[threadIdx.x]);
}

// exclusive scan of the bucket sizes into the cursors; ctl[64] = rays with work
__global__ void diff_bucket_scan_kernel(unsigned* __restrict__ ctl) {
    if (threadIdx.x != 0) return;
    unsigned acc = 0;
    for (int b = 0; b < kWorkBuckets; ++b) {
        ctl[kWorkBuckets + b] = acc;
        acc += ctl[b];
    }
    ctl[2 * kWorkBuckets] = acc;
}

__global__ void __launch_bounds__(256) diff_bucket_scatter_kernel(unsigned n, const int* __restrict__ bucket,
                                                                 unsigned* __restrict__ ctl,
                                                                 unsigned* __restrict__ order) {
    const unsigned p = blockIdx.x * blockDim.x + threadIdx.x;
    const int b = p < n ? bucket[p] : -1;
    const unsigned peers = __match_any_sync(kFullMask, b);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    unsigned base = 0;
    if (b >= 0 && lane == leader) base = atomicAdd(&ctl[kWorkBuckets + b], (unsigned)__popc(peers));
    base = __shfl_sync(peers, base, leader);
    if (b >= 0) order[base + (unsigned)__popc(peers & ((1u << lane) - 1u))] = p;
}

// ---- adjoint kernel ----------------------------------------------------------------------------
// Hit point of step (s -> nx) with stages k: the crossing root of shade_crossing<R, 1>; X the
// state there, dX its slope in the step fraction.
template <class R>
__device__ __forceinline__ R step_hit(const R* s, const R* nx, const R (*k)[6], const R* k7, R h, R* X, R* dX) {
    const R yv0 = s[1], yv1 = nx[1];
    const R dy = yv0 - yv1;
    R t = dy != R(0) ? Ops<R>::fdiv(yv0, dy) : R(0.5);
    t = Ops<R>::minr(Ops<R>::maxr(t, R(0)), R(1));
    t = crossing_root<R>(yv0, yv1, k[0][1], k[2][1], k[3][1], k[4][1], k[5][1], k7[1], h, t);
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        X[c] = dense_eval<R>(s[c], nx[c], k[0][c], k[2][c], k[3][c], k[4][c], k[5][c], k7[c], h, t);
        if (dX) dX[c] = dense_slope<R>(s[c], nx[c], k[0][c], k[2][c], k[3][c], k[4][c], k[5][c], k7[c], h, t);
    }
    return t;
}

// Float records differentiated in double (the model that kt_diff_replay_fp64 evaluates): the
// float checkpoints carry the float trajectory's rounding, so segment starts are replayed in
// double from the ray's double start instead.  sweep_segment advances the state s and the
// transmittance tau through every recorded step of one segment; k and k7 are scratch.
template <class R, class RR>
__device__ __forceinline__ void sweep_segment(const DiffSeg<RR>* sg, R pt, R kt, R a, R aa, R M, const Scene& sc,
                                              const DiffLut& dl, R (*k)[6], R* k7, R* s, R& tau) {
    for (int j = 0; j < sg->n; ++j) {
        R nx[6];
        dp5_stages<R>(s, (R)sg->h[j], pt, a, aa, M, k, nx, k7, false);
        if (sg->hits >> j & 1u) {
            R X[6], c3[3], al;
            step_hit<R>(s, nx, k, k7, (R)sg->h[j], X, nullptr);
            if (shade_eval<R, R>(X, pt, kt, sc, dl, c3, al)) tau *= R(1) - al;
        }
#pragma unroll
        for (int c = 0; c < 6; ++c) s[c] = nx[c];
    }
}
// The state and transmittance at the start of segment `target`, replayed from the ray's start.
template <class R, class RR>
__device__ __forceinline__ void replay_segment_start(const DiffRay& rr, const DiffRecRaw& rec, int target,
                                                     const RayRun<R>& ry0, R a, R aa, R M, const Scene& sc,
                                                     const DiffLut& dl, R (*k)[6], R* k7, R* s, R& tau) {
#pragma unroll
    for (int c = 0; c < 6; ++c) s[c] = ry0.s[c];
    tau = R(1);
    for (int si = rr.first_seg; si >= 0 && si != target; si = seg_at<RR>(rec, si)->next)
        sweep_segment<R, RR>(seg_at<RR>(rec, si), ry0.pt, ry0.kt, a, aa, M, sc, dl, k, k7, s, tau);
}

// Resident 128-thread blocks per SM asked of the compiler for the adjoint kernel: two, so that the
// reverse sweep's dual-number right-hand sides keep their values in registers (225 registers,
// no spills; four blocks per SM cap them at 128 with 452 B of spills and run 14% slower).
template <class R> struct BackMinBlocks { static constexpr int v = 2; };
template <> struct BackMinBlocks<double> { static constexpr int v = 2; };

// RR: the record type (float records of an FP32 object may be differentiated with R = double).
template <class R, class RR = R>
__global__ void __launch_bounds__(128, BackMinBlocks<R>::v) diff_backward_kernel(const Scene sc, const Camera cam, const CameraD camd,
                                                           const CameraD dcamd, const DiffRecRaw rec, const DiffLut dl,
                                                           const float4* __restrict__ dl_dhdr,
                                                           double* __restrict__ grad,
                                                           const unsigned* __restrict__ order,
                                                           const unsigned* __restrict__ n_work) {
    using C = DP<R>;
    const unsigned u = blockIdx.x * blockDim.x + threadIdx.x;
    double g[4] = {0.0, 0.0, 0.0, 0.0};
    if (u < *n_work) {
        const unsigned p = order[u];
        const DiffRay rr = rec.rays[p];
        const float4 dlp = dl_dhdr[p];
        const R fs = (R)sc.final_scale;
        const R lc[3] = {(R)dlp.x * fs, (R)dlp.y * fs, (R)dlp.z * fs};
        // only shaded crossings carry derivatives (the sky grid is piecewise constant)
        const bool live = rr.term != kTermNotStarted && rr.term != kTermOverflow && rr.last_seg >= 0 &&
                          rr.n_hits > 0 && (lc[0] != R(0) || lc[1] != R(0) || lc[2] != R(0));
        if (live) {
            const int px = (int)(p % (unsigned)sc.width), py = (int)(p / (unsigned)sc.width);
            RayRun<R> ry0;
            ray_begin<R>(px, py, sc, cam, camd, ry0);
            const R pt = ry0.pt, kt = ry0.kt;
            const R a = sc_a<R>(sc), aa = sc_aa<R>(sc), M = sc_M<R>(sc);
            R ls[6] = {R(0), R(0), R(0), R(0), R(0), R(0)};  // adjoint of the current state
            R lpt = R(0), lkt = R(0), ga = R(0), gts = R(0), gro = R(0);
            R ltau = rr.term == kTermEscape ? (lc[0] + lc[1] + lc[2]) * (R)rr.sky : R(0);
            R S[kSegSteps][6];          // state before each step of the segment
            R K[kSegSteps][6][6];       // its stages k1..k6 (a step's k7 is the next step's k1)
            R K7[6];                    // k7 of the segment's last step
            R TIN[kSegSteps];           // transmittance before a shaded crossing
            // the adjoint of the state is zero after the last shaded crossing: start there
            int si = rr.last_seg;
            while (si >= 0 && seg_at<RR>(rec, si)->hits == 0u) si = seg_at<RR>(rec, si)->prev;
            // float records in double: one replay from the ray's start gives the start states of
            // the segments up to si (the last kStoredStarts of them kept; earlier ones, on rays
            // longer than that, are replayed again when their turn comes)
            constexpr int kStoredStarts = std::is_same<R, RR>::value ? 1 : 8;
            R SS[kStoredStarts][6], ST[kStoredStarts];
            int SID[kStoredStarts];
            if constexpr (!std::is_same<R, RR>::value) {
#pragma unroll
                for (int q = 0; q < kStoredStarts; ++q) SID[q] = -1;
                R s[6];
#pragma unroll
                for (int c = 0; c < 6; ++c) s[c] = ry0.s[c];
                R tau = R(1);
                int ord = 0;
                for (int sj = rr.first_seg; sj >= 0; sj = seg_at<RR>(rec, sj)->next, ++ord) {
                    const int q = ord % kStoredStarts;
                    SID[q] = sj;
                    ST[q] = tau;
#pragma unroll
                    for (int c = 0; c < 6; ++c) SS[q][c] = s[c];
                    if (sj == si) break;
                    sweep_segment<R, RR>(seg_at<RR>(rec, sj), pt, kt, a, aa, M, sc, dl, K[0], K7, s, tau);
                }
            }
            bool first = true;
            while (si >= 0) {
                const DiffSeg<RR>* sg = seg_at<RR>(rec, si);
                const unsigned hits = sg->hits;
                const int n = first ? 32 - __clz((int)hits) : sg->n;
                first = false;
                // forward sweep: states, stages, transmittance at the shaded crossings
                {
                    R s[6];
                    R tau;
                    if constexpr (std::is_same<R, RR>::value) {
#pragma unroll
                        for (int c = 0; c < 6; ++c) s[c] = sg->s[c];
                        tau = sg->tau;
                    } else {
                        int q = -1;
#pragma unroll
                        for (int i = 0; i < kStoredStarts; ++i)
                            if (SID[i] == si) q = i;
                        if (q >= 0) {
#pragma unroll
                            for (int c = 0; c < 6; ++c) s[c] = SS[q][c];
                            tau = ST[q];
                        } else {
                            replay_segment_start<R, RR>(rr, rec, si, ry0, a, aa, M, sc, dl, K[0], K7, s, tau);
                        }
                    }
                    for (int j = 0; j < n; ++j) {
                        R nx[6];
#pragma unroll
                        for (int c = 0; c < 6; ++c) S[j][c] = s[c];
                        // FSAL: the previous step's k7 is f at this step's start, bit for bit
                        if (j > 0) {
#pragma unroll
                            for (int c = 0; c < 6; ++c) K[j][0][c] = K7[c];
                        }
                        dp5_stages<R>(s, sg->h[j], pt, a, aa, M, K[j], nx, K7, j > 0);
                        if (hits >> j & 1u) {
                            R X[6], c3[3], al;
                            step_hit<R>(s, nx, K[j], K7, sg->h[j], X, nullptr);
                            TIN[j] = tau;
                            if (shade_eval<R, R>(X, pt, kt, sc, dl, c3, al)) tau *= R(1) - al;
                        }
#pragma unroll
                        for (int c = 0; c < 6; ++c) s[c] = nx[c];
                    }
                }
                // reverse sweep
                for (int j = n - 1; j >= 0; --j) {
                    const R h = sg->h[j];
                    const R(*k)[6] = K[j];
                    const R* k7 = j + 1 < n ? K[j + 1][0] : K7;
                    const R* s0 = S[j];
                    R nx[6];
#pragma unroll
                    for (int c = 0; c < 6; ++c)
                        nx[c] = s0[c] + h * (C::b1 * k[0][c] + C::b3 * k[2][c] + C::b4 * k[3][c] + C::b5 * k[4][c] +
                                             C::b6 * k[5][c]);
                    R ly0[6] = {R(0), R(0), R(0), R(0), R(0), R(0)};
                    R ly1[6] = {R(0), R(0), R(0), R(0), R(0), R(0)};
                    R dk[7][6];  // adjoints of k1..k7 from the dense output (k2 stays 0)
#pragma unroll
                    for (int i = 0; i < 7; ++i)
#pragma unroll
                        for (int c = 0; c < 6; ++c) dk[i][c] = R(0);
                    if (hits >> j & 1u) {
                        R X[6], dX[6];
                        const R t = step_hit<R>(s0, nx, k, k7, h, X, dX);
                        Dual<R, kSN> cc[3], al;
                        if (shade_eval<R, Dual<R, kSN>>(X, pt, kt, sc, dl, cc, al)) {
                            const R tin = TIN[j];
                            // col += c alpha tau_in ; tau_out = tau_in (1 - alpha)
                            R q[kSN];
#pragma unroll
                            for (int i = 0; i < kSN; ++i) {
                                R v = R(0);
#pragma unroll
                                for (int ch = 0; ch < 3; ++ch) v += lc[ch] * (cc[ch].d[i] * al.v + cc[ch].v * al.d[i]);
                                q[i] = v * tin - ltau * tin * al.d[i];
                            }
                            ltau = (lc[0] * cc[0].v + lc[1] * cc[1].v + lc[2] * cc[2].v) * al.v +
                                   ltau * (R(1) - al.v);
                            lpt += q[kSPt];
                            lkt += q[kSKt];
                            ga += q[kSA];
                            gts += q[kSTs];
                            gro += q[kSRo];
                            // root: y(t*) = 0  =>  dt* = -(dD_1/din . din) / D_1'(t*)
                            R lt = R(0);
#pragma unroll
                            for (int c = 0; c < 6; ++c) lt += q[kSX + c] * dX[c];
                            const R mu = dX[1] != R(0) ? -lt / dX[1] : R(0);
                            R wd[8];
                            dense_weights<R>(t, h, wd);
#pragma unroll
                            for (int c = 0; c < 6; ++c) {
                                const R e = q[kSX + c] + (c == 1 ? mu : R(0));
                                ly0[c] += e * wd[0];
                                ly1[c] += e * wd[1];
                                dk[0][c] += e * wd[2];
                                dk[2][c] += e * wd[3];
                                dk[3][c] += e * wd[4];
                                dk[4][c] += e * wd[5];
                                dk[5][c] += e * wd[6];
                                dk[6][c] += e * wd[7];
                            }
                        }
                    }
                    // reverse of s' = s + h sum b_i k_i, k_i = f(Y_i), Y_i = s + h sum_j a_ij k_j
                    R lnext[6], lnew[6];
#pragma unroll
                    for (int c = 0; c < 6; ++c) {
                        lnext[c] = ls[c] + ly1[c];
                        lnew[c] = lnext[c] + ly0[c];
                    }
                    R acc[7][6];  // adjoint of k_i collected so far (i = 0..6 for k1..k7)
#pragma unroll
                    for (int i = 0; i < 7; ++i) {
                        const R b = i < 6 ? rk_a<R>(7, i + 1) : R(0);
#pragma unroll
                        for (int c = 0; c < 6; ++c) acc[i][c] = h * b * lnext[c] + dk[i][c];
                    }
#pragma unroll
                    for (int m = 6; m >= 0; --m) {  // stage m + 1
                        R Y[6];
#pragma unroll
                        for (int c = 0; c < 6; ++c) {
                            R sum = R(0);
#pragma unroll
                            for (int jj = 0; jj < m; ++jj) sum += rk_a<R>(m + 1, jj + 1) * k[jj][c];
                            Y[c] = m == 0 ? s0[c] : s0[c] + h * sum;
                        }
                        bool nz = false;
#pragma unroll
                        for (int c = 0; c < 6; ++c) nz = nz || acc[m][c] != R(0);
                        if (!nz) continue;
                        R lY[6], da, dpt;
                        rhs_vjp<R>(Y, acc[m], pt, a, aa, M, lY, da, dpt);
                        ga += da;
                        lpt += dpt;
#pragma unroll
                        for (int c = 0; c < 6; ++c) lnew[c] += lY[c];
#pragma unroll
                        for (int i = 0; i < m; ++i) {
                            const R coef = h * rk_a<R>(m + 1, i + 1);
#pragma unroll
                            for (int c = 0; c < 6; ++c) acc[i][c] += coef * lY[c];
                        }
                    }
#pragma unroll
                    for (int c = 0; c < 6; ++c) ls[c] = lnew[c];
                }
                si = sg->prev;
            }
            // initial state: s0, p_t, k_t as functions of spin and inclination
            Dual<R, 2> s0[6], dpt0, dkt0;
            start_dual<R>(px, py, sc, cam, camd, dcamd, s0, dpt0, dkt0);
            R gi = R(0);
#pragma unroll
            for (int c = 0; c < 6; ++c) {
                ga += ls[c] * s0[c].d[0];
                gi += ls[c] * s0[c].d[1];
            }
            ga += lpt * dpt0.d[0] + lkt * dkt0.d[0];
            gi += lpt * dpt0.d[1] + lkt * dkt0.d[1];
            g[0] = (double)ga;
            g[1] = (double)gi;
            g[2] = (double)gts;
            g[3] = (double)gro;
        }
    }
    // warp sums, one atomic per warp and parameter
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        double v = g[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFullMask, v, o);
        if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(grad + i, v);
    }
}

// ---- launchers ----------------------------------------------------------------------------------
cudaError_t launch_diff_forward(const Scene& sc, const Camera& cam, const CameraD& camd, const DiffRecRaw& rec,
                                int replay, float4* hdr, double* hdr64, uint32_t* err, uint32_t* flags,
                                cudaStream_t st, bool float_records) {
    const unsigned n = (unsigned)sc.width * (unsigned)sc.height;
    if (n == 0) return cudaSuccess;
    const dim3 grid((n + 127) / 128);
    if (sc.precision == 2 && float_records) {
        if (!replay) return cudaErrorInvalidValue;
        diff_forward_kernel<double, true, float><<<grid, 128, 0, st>>>(sc, cam, camd, rec, hdr, hdr64, err, flags);
    } else if (sc.precision == 2) {
        if (replay) diff_forward_kernel<double, true><<<grid, 128, 0, st>>>(sc, cam, camd, rec, hdr, hdr64, err, flags);
        else diff_forward_kernel<double, false><<<grid, 128, 0, st>>>(sc, cam, camd, rec, hdr, hdr64, err, flags);
    } else {
        if (replay) diff_forward_kernel<float, true><<<grid, 128, 0, st>>>(sc, cam, camd, rec, hdr, hdr64, err, flags);
        else diff_forward_kernel<float, false><<<grid, 128, 0, st>>>(sc, cam, camd, rec, hdr, hdr64, err, flags);
    }
    return cudaGetLastError();
}

cudaError_t launch_diff_backward(const Scene& sc, const Camera& cam, const CameraD& camd, const CameraD& dcamd,
                                 const DiffRecRaw& rec, const DiffLut& dl, const float4* dl_dhdr, double* grad,
                                 const DiffWork& wk, cudaStream_t st, bool float_records) {
    const unsigned n = (unsigned)sc.width * (unsigned)sc.height;
    if (n == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(wk.ctl, 0, (2 * kWorkBuckets + 1) * sizeof(unsigned), st);
    if (e != cudaSuccess) return e;
    const dim3 g256((n + 255) / 256), g128((n + 127) / 128);
    if (sc.precision == 2 && !float_records) diff_bucket_kernel<double><<<g256, 256, 0, st>>>(sc, rec, dl_dhdr, wk.bucket, wk.ctl);
    else diff_bucket_kernel<float><<<g256, 256, 0, st>>>(sc, rec, dl_dhdr, wk.bucket, wk.ctl);
    diff_bucket_scan_kernel<<<1, 32, 0, st>>>(wk.ctl);
    diff_bucket_scatter_kernel<<<g256, 256, 0, st>>>(n, wk.bucket, wk.ctl, wk.order);
    const unsigned* n_work = wk.ctl + 2 * kWorkBuckets;
    if (sc.precision == 2 && float_records)
        diff_backward_kernel<double, float><<<g128, 128, 0, st>>>(sc, cam, camd, dcamd, rec, dl, dl_dhdr, grad, wk.order,
                                                                  n_work);
    else if (sc.precision == 2)
        diff_backward_kernel<double><<<g128, 128, 0, st>>>(sc, cam, camd, dcamd, rec, dl, dl_dhdr, grad, wk.order, n_work);
    else
        diff_backward_kernel<float><<<g128, 128, 0, st>>>(sc, cam, camd, dcamd, rec, dl, dl_dhdr, grad, wk.order, n_work);
    return cudaGetLastError();
}

}  // namespace ktd
