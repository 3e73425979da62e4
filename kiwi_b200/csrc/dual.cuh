// Forward-mode derivatives for the adjoint: a value with N partial derivatives (Dual4: with respect to the
// particle's x0, y0, z0 and h; Dual3: x0, y0, z0), propagated through every arithmetic operation and libm
// call by the chain rule.  Instantiating the closed-form face walk (kiwi_math.cuh) with Dual4 gives the exact derivatives
// of the computed cell integral (branch by branch: region choices, the foot rule and the clamp are
// decided on values, as in the forward pass).
#pragma once

#include <math.h>

namespace kiwi_b200 {
// The type and its overloads live in their own namespace: argument-dependent lookup finds them for
// Dual4 arguments, while an unqualified sqrt(double) inside namespace kiwi_b200 still means ::sqrt.
namespace ad {

#ifdef __CUDACC__
#define KIWI_DD __host__ __device__ __forceinline__
#define KIWI_DC __host__ __device__
#else
#define KIWI_DD inline
#define KIWI_DC
#endif

template <int N>
struct DualN {
    double v;
    double d[N];

    KIWI_DC DualN() : v(0.0) {
#pragma unroll
        for (int k = 0; k < N; ++k) d[k] = 0.0;
    }
    KIWI_DC DualN(double x) : v(x) {
#pragma unroll
        for (int k = 0; k < N; ++k) d[k] = 0.0;
    }
    KIWI_DC static DualN seed(double x, int k) {
        DualN r(x);
        r.d[k] = 1.0;
        return r;
    }
};

// a * f'(x) chain helper: r.v = val, r.d = x.d * slope
template <int N>
KIWI_DD DualN<N> chain(const DualN<N>& x, double val, double slope) {
    DualN<N> r;
    r.v = val;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = x.d[k] * slope;
    return r;
}

template <int N>
KIWI_DD DualN<N> operator+(const DualN<N>& a, const DualN<N>& b) {
    DualN<N> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
}
template <int N>
KIWI_DD DualN<N> operator-(const DualN<N>& a, const DualN<N>& b) {
    DualN<N> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
}
template <int N>
KIWI_DD DualN<N> operator-(const DualN<N>& a) {
    DualN<N> r;
    r.v = -a.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = -a.d[k];
    return r;
}
template <int N>
KIWI_DD DualN<N> operator*(const DualN<N>& a, const DualN<N>& b) {
    DualN<N> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
template <int N>
KIWI_DD DualN<N> operator/(const DualN<N>& a, const DualN<N>& b) {
    DualN<N> r;
    r.v = a.v / b.v;
    const double inv = 1.0 / b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * inv;
    return r;
}
template <int N>
KIWI_DD DualN<N> operator+(const DualN<N>& a, double b) { return a + DualN<N>(b); }
template <int N>
KIWI_DD DualN<N> operator+(double a, const DualN<N>& b) { return DualN<N>(a) + b; }
template <int N>
KIWI_DD DualN<N> operator-(const DualN<N>& a, double b) { return a - DualN<N>(b); }
template <int N>
KIWI_DD DualN<N> operator-(double a, const DualN<N>& b) { return DualN<N>(a) - b; }
template <int N>
KIWI_DD DualN<N> operator*(const DualN<N>& a, double b) {
    DualN<N> r;
    r.v = a.v * b;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * b;
    return r;
}
template <int N>
KIWI_DD DualN<N> operator*(double a, const DualN<N>& b) { return b * a; }
template <int N>
KIWI_DD DualN<N> operator/(const DualN<N>& a, double b) {
    DualN<N> r;
    r.v = a.v / b;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] / b;
    return r;
}
template <int N>
KIWI_DD DualN<N> operator/(double a, const DualN<N>& b) { return DualN<N>(a) / b; }
template <int N>
KIWI_DD DualN<N>& operator+=(DualN<N>& a, const DualN<N>& b) { return a = a + b; }
template <int N>
KIWI_DD DualN<N>& operator-=(DualN<N>& a, const DualN<N>& b) { return a = a - b; }
template <int N>
KIWI_DD DualN<N>& operator*=(DualN<N>& a, const DualN<N>& b) { return a = a * b; }

#define KIWI_DUAL_CMP(op)                                                                              \
    template <int N>                                                                                   \
    KIWI_DD bool operator op(const DualN<N>& a, const DualN<N>& b) { return a.v op b.v; }             \
    template <int N>                                                                                   \
    KIWI_DD bool operator op(const DualN<N>& a, double b) { return a.v op b; }                         \
    template <int N>                                                                                   \
    KIWI_DD bool operator op(double a, const DualN<N>& b) { return a op b.v; }
KIWI_DUAL_CMP(<)
KIWI_DUAL_CMP(>)
KIWI_DUAL_CMP(<=)
KIWI_DUAL_CMP(>=)
KIWI_DUAL_CMP(==)
KIWI_DUAL_CMP(!=)
#undef KIWI_DUAL_CMP

template <int N>
KIWI_DD DualN<N> sqrt(const DualN<N>& x) {
    const double s = ::sqrt(x.v);
    return chain(x, s, 0.5 / s);
}
template <int N>
KIWI_DD DualN<N> fabs(const DualN<N>& x) { return x.v < 0.0 ? -x : x; }
template <int N>
KIWI_DD DualN<N> acos(const DualN<N>& x) { return chain(x, ::acos(x.v), -1.0 / ::sqrt(1.0 - x.v * x.v)); }
template <int N>
KIWI_DD DualN<N> atan(const DualN<N>& x) { return chain(x, ::atan(x.v), 1.0 / (1.0 + x.v * x.v)); }
template <int N>
KIWI_DD DualN<N> log(const DualN<N>& x) { return chain(x, ::log(x.v), 1.0 / x.v); }
template <int N>
KIWI_DD DualN<N> log1p(const DualN<N>& x) { return chain(x, ::log1p(x.v), 1.0 / (1.0 + x.v)); }
// max with a constant: the constant (no derivative) where it wins
template <int N>
KIWI_DD DualN<N> atanh(const DualN<N>& x) { return chain(x, ::atanh(x.v), 1.0 / (1.0 - x.v * x.v)); }
template <int N>
KIWI_DD DualN<N> fmax(const DualN<N>& x, double c) { return x.v >= c ? x : DualN<N>(c); }
template <int N>
KIWI_DD DualN<N> fmin(double c, const DualN<N>& x) { return x.v <= c ? x : DualN<N>(c); }
// a * b + c with the value fused (one rounding) and the derivative of a * b + c
template <int N>
KIWI_DD DualN<N> fma(const DualN<N>& a, const DualN<N>& b, const DualN<N>& c) {
    DualN<N> r;
    r.v = ::fma(a.v, b.v, c.v);
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k] + c.d[k];
    return r;
}
template <int N>
KIWI_DD DualN<N> sin(const DualN<N>& x) { return chain(x, ::sin(x.v), ::cos(x.v)); }
template <int N>
KIWI_DD DualN<N> cos(const DualN<N>& x) { return chain(x, ::cos(x.v), -::sin(x.v)); }
template <int N>
KIWI_DD void sincos(const DualN<N>& x, DualN<N>* s, DualN<N>* c) {
    double sv, cv;
    ::sincos(x.v, &sv, &cv);
    *s = chain(x, sv, cv);
    *c = chain(x, cv, -sv);
}
template <int N>
KIWI_DD DualN<N> atan2(const DualN<N>& y, const DualN<N>& x) {
    DualN<N> r;
    r.v = ::atan2(y.v, x.v);
    const double den = x.v * x.v + y.v * y.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = (x.v * y.d[k] - y.v * x.d[k]) / den;
    return r;
}
template <int N>
KIWI_DD double value(const DualN<N>& x) { return x.v; }
KIWI_DD double value(double x) { return x; }

#undef KIWI_DD
#undef KIWI_DC

using Dual4 = DualN<4>;
using Dual3 = DualN<3>;

}  // namespace ad
using ad::Dual3;
using ad::Dual4;
using ad::DualN;
}  // namespace kiwi_b200
