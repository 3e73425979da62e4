// Forward-mode derivatives for the adjoint: a value with its partial derivatives with respect to the
// particle's x0, y0, z0 and h, propagated through every arithmetic operation and libm call by the chain
// rule.  Instantiating the closed-form face walk (kiwi_math.cuh) with Dual4 gives the exact derivatives
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

struct Dual4 {
    double v;
    double d[4];

    KIWI_DC Dual4() : v(0.0), d{0.0, 0.0, 0.0, 0.0} {}
    KIWI_DC Dual4(double x) : v(x), d{0.0, 0.0, 0.0, 0.0} {}
    KIWI_DC static Dual4 seed(double x, int k) {
        Dual4 r(x);
        r.d[k] = 1.0;
        return r;
    }
};

// a * f'(x) chain helper: r.v = val, r.d = x.d * slope
KIWI_DD Dual4 chain(const Dual4& x, double val, double slope) {
    Dual4 r;
    r.v = val;
#pragma unroll
    for (int k = 0; k < 4; ++k) r.d[k] = x.d[k] * slope;
    return r;
}

KIWI_DD Dual4 operator+(const Dual4& a, const Dual4& b) {
    Dual4 r;
    r.v = a.v + b.v;
#pragma unroll
    for (int k = 0; k < 4; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
}
KIWI_DD Dual4 operator-(const Dual4& a, const Dual4& b) {
    Dual4 r;
    r.v = a.v - b.v;
#pragma unroll
    for (int k = 0; k < 4; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
}
KIWI_DD Dual4 operator-(const Dual4& a) {
    Dual4 r;
    r.v = -a.v;
#pragma unroll
    for (int k = 0; k < 4; ++k) r.d[k] = -a.d[k];
    return r;
}
KIWI_DD Dual4 operator*(const Dual4& a, const Dual4& b) {
    Dual4 r;
    r.v = a.v * b.v;
#pragma unroll
    for (int k = 0; k < 4; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
KIWI_DD Dual4 operator/(const Dual4& a, const Dual4& b) {
    Dual4 r;
    r.v = a.v / b.v;
    const double inv = 1.0 / b.v;
#pragma unroll
    for (int k = 0; k < 4; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * inv;
    return r;
}
KIWI_DD Dual4 operator+(const Dual4& a, double b) { return a + Dual4(b); }
KIWI_DD Dual4 operator+(double a, const Dual4& b) { return Dual4(a) + b; }
KIWI_DD Dual4 operator-(const Dual4& a, double b) { return a - Dual4(b); }
KIWI_DD Dual4 operator-(double a, const Dual4& b) { return Dual4(a) - b; }
KIWI_DD Dual4 operator*(const Dual4& a, double b) {
    Dual4 r;
    r.v = a.v * b;
#pragma unroll
    for (int k = 0; k < 4; ++k) r.d[k] = a.d[k] * b;
    return r;
}
KIWI_DD Dual4 operator*(double a, const Dual4& b) { return b * a; }
KIWI_DD Dual4 operator/(const Dual4& a, double b) {
    Dual4 r;
    r.v = a.v / b;
#pragma unroll
    for (int k = 0; k < 4; ++k) r.d[k] = a.d[k] / b;
    return r;
}
KIWI_DD Dual4 operator/(double a, const Dual4& b) { return Dual4(a) / b; }
KIWI_DD Dual4& operator+=(Dual4& a, const Dual4& b) { return a = a + b; }
KIWI_DD Dual4& operator-=(Dual4& a, const Dual4& b) { return a = a - b; }
KIWI_DD Dual4& operator*=(Dual4& a, const Dual4& b) { return a = a * b; }

#define KIWI_DUAL_CMP(op)                                                             \
    KIWI_DD bool operator op(const Dual4& a, const Dual4& b) { return a.v op b.v; }   \
    KIWI_DD bool operator op(const Dual4& a, double b) { return a.v op b; }           \
    KIWI_DD bool operator op(double a, const Dual4& b) { return a op b.v; }
KIWI_DUAL_CMP(<)
KIWI_DUAL_CMP(>)
KIWI_DUAL_CMP(<=)
KIWI_DUAL_CMP(>=)
KIWI_DUAL_CMP(==)
KIWI_DUAL_CMP(!=)
#undef KIWI_DUAL_CMP

KIWI_DD Dual4 sqrt(const Dual4& x) {
    const double s = ::sqrt(x.v);
    return chain(x, s, 0.5 / s);
}
KIWI_DD Dual4 fabs(const Dual4& x) { return x.v < 0.0 ? -x : x; }
KIWI_DD Dual4 acos(const Dual4& x) { return chain(x, ::acos(x.v), -1.0 / ::sqrt(1.0 - x.v * x.v)); }
KIWI_DD Dual4 atan(const Dual4& x) { return chain(x, ::atan(x.v), 1.0 / (1.0 + x.v * x.v)); }
KIWI_DD Dual4 log(const Dual4& x) { return chain(x, ::log(x.v), 1.0 / x.v); }
KIWI_DD Dual4 log1p(const Dual4& x) { return chain(x, ::log1p(x.v), 1.0 / (1.0 + x.v)); }
// max with a constant: the constant (no derivative) where it wins
KIWI_DD Dual4 fmax(const Dual4& x, double c) { return x.v >= c ? x : Dual4(c); }
KIWI_DD Dual4 sin(const Dual4& x) { return chain(x, ::sin(x.v), ::cos(x.v)); }
KIWI_DD Dual4 cos(const Dual4& x) { return chain(x, ::cos(x.v), -::sin(x.v)); }
KIWI_DD void sincos(const Dual4& x, Dual4* s, Dual4* c) {
    double sv, cv;
    ::sincos(x.v, &sv, &cv);
    *s = chain(x, sv, cv);
    *c = chain(x, cv, -sv);
}
KIWI_DD Dual4 atan2(const Dual4& y, const Dual4& x) {
    Dual4 r;
    r.v = ::atan2(y.v, x.v);
    const double den = x.v * x.v + y.v * y.v;
#pragma unroll
    for (int k = 0; k < 4; ++k) r.d[k] = (x.v * y.d[k] - y.v * x.d[k]) / den;
    return r;
}
KIWI_DD double value(const Dual4& x) { return x.v; }
KIWI_DD double value(double x) { return x; }

#undef KIWI_DD
#undef KIWI_DC

}  // namespace ad
using ad::Dual4;
}  // namespace kiwi_b200
