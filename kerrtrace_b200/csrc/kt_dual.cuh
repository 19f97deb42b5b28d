// kt_dual.cuh — forward-mode dual numbers for the adjoint kernels.
//
// Dual<R, N> carries a value and N directional derivatives.  Evaluating a function on duals
// gives its Jacobian-vector products for N directions at once, exactly for the expression as
// written (same operations, same order), which is what a discrete adjoint has to differentiate.
// Ops<Dual<R, N>> provides the primitives the Hamiltonian right-hand side uses (fma, rsq, fdiv,
// sqrt_rn), so hamilton_rhs<Dual<...>, true> is the RHS together with its JVPs.
#pragma once
#include "kt_device.cuh"

namespace ktd {

template <class R, int N>
struct Dual {
    R v;
    R d[N];
    __device__ __forceinline__ Dual() {}
    __device__ __forceinline__ Dual(R x) : v(x) {
#pragma unroll
        for (int i = 0; i < N; ++i) d[i] = R(0);
    }
    // value with a unit derivative in direction k
    __device__ __forceinline__ static Dual seed(R x, int k) {
        Dual r(x);
        r.d[k] = R(1);
        return r;
    }
};

template <class R, int N>
__device__ __forceinline__ Dual<R, N> operator+(const Dual<R, N>& a, const Dual<R, N>& b) {
    Dual<R, N> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
template <class R, int N>
__device__ __forceinline__ Dual<R, N> operator-(const Dual<R, N>& a, const Dual<R, N>& b) {
    Dual<R, N> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
template <class R, int N>
__device__ __forceinline__ Dual<R, N> operator-(const Dual<R, N>& a) {
    Dual<R, N> r;
    r.v = -a.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
    return r;
}
template <class R, int N>
__device__ __forceinline__ Dual<R, N> operator*(const Dual<R, N>& a, const Dual<R, N>& b) {
    Dual<R, N> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
template <class R, int N>
__device__ __forceinline__ Dual<R, N> operator/(const Dual<R, N>& a, const Dual<R, N>& b) {
    Dual<R, N> r;
    const R inv = R(1) / b.v;
    r.v = a.v * inv;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * inv;
    return r;
}
// mixed operations with a plain value (constants of the expression)
template <class R, int N>
__device__ __forceinline__ Dual<R, N> operator+(const Dual<R, N>& a, R b) {
    Dual<R, N> r = a;
    r.v = a.v + b;
    return r;
}
template <class R, int N>
__device__ __forceinline__ Dual<R, N> operator+(R a, const Dual<R, N>& b) { return b + a; }
template <class R, int N>
__device__ __forceinline__ Dual<R, N> operator-(const Dual<R, N>& a, R b) {
    Dual<R, N> r = a;
    r.v = a.v - b;
    return r;
}
template <class R, int N>
__device__ __forceinline__ Dual<R, N> operator-(R a, const Dual<R, N>& b) {
    Dual<R, N> r = -b;
    r.v = a - b.v;
    return r;
}
template <class R, int N>
__device__ __forceinline__ Dual<R, N> operator*(const Dual<R, N>& a, R b) {
    Dual<R, N> r;
    r.v = a.v * b;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b;
    return r;
}
template <class R, int N>
__device__ __forceinline__ Dual<R, N> operator*(R a, const Dual<R, N>& b) { return b * a; }
template <class R, int N>
__device__ __forceinline__ Dual<R, N> operator/(const Dual<R, N>& a, R b) { return a * (R(1) / b); }
template <class R, int N>
__device__ __forceinline__ Dual<R, N> operator/(R a, const Dual<R, N>& b) { return Dual<R, N>(a) / b; }

template <class R, int N>
__device__ __forceinline__ bool operator<(const Dual<R, N>& a, const Dual<R, N>& b) { return a.v < b.v; }
template <class R, int N>
__device__ __forceinline__ bool operator>(const Dual<R, N>& a, const Dual<R, N>& b) { return a.v > b.v; }
template <class R, int N>
__device__ __forceinline__ bool operator<=(const Dual<R, N>& a, const Dual<R, N>& b) { return a.v <= b.v; }
template <class R, int N>
__device__ __forceinline__ bool operator>=(const Dual<R, N>& a, const Dual<R, N>& b) { return a.v >= b.v; }

template <class R, int N>
struct Ops<Dual<R, N>> {
    using D = Dual<R, N>;
    static __device__ __forceinline__ D fma(const D& a, const D& b, const D& c) {
        D r;
        r.v = Ops<R>::fma(a.v, b.v, c.v);
#pragma unroll
        for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i] + c.d[i];
        return r;
    }
    // d(x^-1/2) = -1/2 x^-3/2 dx
    static __device__ __forceinline__ D rsq(const D& x) {
        D r;
        r.v = Ops<R>::rsq(x.v);
        const R k = R(-0.5) * r.v * r.v * r.v;
#pragma unroll
        for (int i = 0; i < N; ++i) r.d[i] = k * x.d[i];
        return r;
    }
    static __device__ __forceinline__ D fdiv(const D& a, const D& b) {
        D r;
        r.v = Ops<R>::fdiv(a.v, b.v);
        const R inv = Ops<R>::fdiv(R(1), b.v);
#pragma unroll
        for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * inv;
        return r;
    }
    static __device__ __forceinline__ D sqrt_rn(const D& x) {
        D r;
        r.v = Ops<R>::sqrt_rn(x.v);
        const R k = r.v > R(0) ? R(0.5) / r.v : R(0);
#pragma unroll
        for (int i = 0; i < N; ++i) r.d[i] = k * x.d[i];
        return r;
    }
    static __device__ __forceinline__ D expr(const D& x) {
        D r;
        r.v = Ops<R>::expr(x.v);
#pragma unroll
        for (int i = 0; i < N; ++i) r.d[i] = r.v * x.d[i];
        return r;
    }
    static __device__ __forceinline__ D maxr(const D& a, const D& b) { return a.v >= b.v ? a : b; }
    static __device__ __forceinline__ D minr(const D& a, const D& b) { return a.v <= b.v ? a : b; }
    static __device__ __forceinline__ D absr(const D& a) { return a.v < R(0) ? -a : a; }
    static __device__ __forceinline__ bool isnanr(const D& a) { return Ops<R>::isnanr(a.v); }
    static __device__ __forceinline__ bool isfiniter(const D& a) { return Ops<R>::isfiniter(a.v); }
};

}  // namespace ktd
