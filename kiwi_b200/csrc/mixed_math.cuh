// Cubic-spline (M4, support 2h) cell integral in the lattice form, written over the real type T for the
// FP32-mixed form (T = float) and for checking it (T = double).
//
// The cell integral is the same sum of vertex pyramids as the reference's face walk
// (src/kernel_integral.cpp:471-647 over the box faces of src/cartesian_grid.cpp:54-72), grouped by lattice
// corner: with the particle at the origin and a face lying in the plane at signed distance X, the face's
// pyramid is an inclusion-exclusion over its four corners (u, v) of the quadrant value
//   Q(r0, u, v) = sgn(u) sgn(v) [F(r0, |u|, |v|) + F(r0, |v|, |u|)],
// where F(r0, R, t) is the vertex tier (src/kernel_integral.cpp:356-400) of the right triangle with the
// edge line at in-plane distance R and the vertex at distance t along it.  The tier formulas are the
// reference's (wall B1..B3 :222-247, edge D2/D3 :253-350, I-series :278-294 and :372-386), rewritten in
// algebraically equal forms that avoid cancellation in low precision:
//   u = a sin(phi) / sqrt(a^2 + cos^2 phi)       (= sin(phi) sqrt(1 - mu^2), mu = cos(phi) / sqrt(a^2 + cos^2))
//   1 - u^2 = cos^2(phi) (1 + a^2) / (a^2 + cos^2)
//   I1 = atan(u / a) = atan(sin(phi) / sqrt(a^2 + cos^2 phi))
//   log((1 + u) / (1 - u)) = 2 log1p(u) - log(1 - u^2)
//   B_k / r0^3 and the r0^3/h^3 prefactors taken as powers of q = r0 / h.
// Every literal is converted to T, so T = float evaluates in FP32 throughout.
#pragma once

#include <math.h>

#ifdef __CUDACC__
#define KIWI_MX __host__ __device__ __forceinline__
#else
#define KIWI_MX inline
#endif

namespace kiwi_b200 {
namespace mixed {

template <class T>
KIWI_MX T mx_sqrt(T x) { return sqrt(x); }
template <class T>
KIWI_MX T mx_atan2(T y, T x) { return atan2(y, x); }
template <class T>
KIWI_MX T mx_atan(T x) { return atan(x); }
template <class T>
KIWI_MX T mx_log1p(T x) { return log1p(x); }
template <class T>
KIWI_MX T mx_log(T x) { return log(x); }
template <>
KIWI_MX float mx_sqrt<float>(float x) { return sqrtf(x); }
template <>
KIWI_MX float mx_atan2<float>(float y, float x) { return atan2f(y, x); }
template <>
KIWI_MX float mx_atan<float>(float x) { return atanf(x); }
template <>
KIWI_MX float mx_log1p<float>(float x) { return log1pf(x); }
template <>
KIWI_MX float mx_log<float>(float x) { return logf(x); }

// Wall tier of a plane at distance r0 > 0: q = r0/h and the B_k / r0^3 coefficients.
template <class T>
struct MxWall {
    T h, r0, q, q2, q3, iq3, b1, b2, b3;
};

template <class T>
KIWI_MX MxWall<T> mx_wall(T h, T r0) {
    MxWall<T> w;
    w.h = h;
    w.r0 = r0;
    w.q = r0 / h;
    w.q2 = w.q * w.q;
    w.q3 = w.q2 * w.q;
    const T iq = h / r0;
    const T iq2 = iq * iq;
    w.iq3 = iq2 * iq;
    w.b1 = w.b2 = T(0);
    if (r0 >= T(2) * h) {
        w.b3 = T(0.25) * w.iq3;
    } else if (r0 > h) {
        const T c = T(-4.0 / 3.0) + w.q - T(0.3) * w.q2 + T(1.0 / 30.0) * w.q3 - T(1.0 / 15.0) * w.iq3;
        w.b3 = T(0.25) * (c + T(1.6) * iq2);
        w.b2 = T(0.25) * c;
    } else {
        const T c = T(-2.0 / 3.0) + T(0.3) * w.q2 - T(0.1) * w.q3;
        w.b3 = T(0.25) * (c + T(1.4) * iq2);
        w.b2 = T(0.25) * (c - T(0.2) * iq2);
        w.b1 = T(0.25) * c;
    }
    return w;
}

template <class T>
struct MxSeries {
    T I0, I_2, I_4, I1, I_1, I_3, I_5;
};

// I-series at angle phi with sin/cos of phi and a = R0 / r0 > 0.
template <class T>
KIWI_MX MxSeries<T> mx_series(T phi, T sinp, T cosp, T a) {
    MxSeries<T> s;
    const T a2 = a * a;
    const T cos2 = cosp * cosp;
    const T den = a2 + cos2;
    const T rs = mx_sqrt(den);
    const T u = a * sinp / rs;
    const T omu2 = cos2 * (T(1) + a2) / den;  // 1 - u^2
    const T tanp = sinp / cosp;
    // log((1 + u) / (1 - u)) with 1 - u = (1 - u^2) / (1 + u): no cancellation as u -> 1
    const T logs = T(2) * mx_log1p(u) - mx_log(omu2);
    s.I0 = phi;
    s.I_2 = phi + a2 * tanp;
    s.I_4 = phi + T(2) * a2 * tanp + T(1.0 / 3.0) * a2 * a2 * tanp * (T(2) + T(1) / cos2);
    s.I1 = mx_atan(sinp / rs);
    s.I_1 = T(0.5) * a * logs + s.I1;
    const T opa2 = T(1) + a2;
    s.I_3 = s.I_1 + T(0.25) * a * opa2 * (T(2) * u / omu2 + logs);
    s.I_5 = s.I_3 + T(1.0 / 16.0) * a * opa2 * opa2 * ((T(10) * u - T(6) * u * u * u) / (omu2 * omu2) + T(3) * logs);
    return s;
}

// Edge tier: D2 (edge line within h) and D3 (within 2h) for the line at in-plane distance R0 > 0.
template <class T>
struct MxEdge {
    T D2, D3;
    T A2, A3;  // sums of the magnitudes of the terms of D2 and D3 (rounding-error scale)
};

template <class T>
KIWI_MX MxEdge<T> mx_edge(const MxWall<T>& w, T R0) {
    MxEdge<T> e;
    e.D2 = e.D3 = e.A2 = e.A3 = T(0);
    const T h = w.h, r0 = w.r0;
    const T ld2 = r0 * r0 + R0 * R0;
    if (ld2 > T(4) * h * h) return e;
    const T a = R0 / r0;
    if (ld2 <= h * h) {
        const T rr = mx_sqrt(h * h - r0 * r0);
        const T d = (rr - R0) * (rr + R0);  // >= 0 up to rounding (the line lies within h)
        const T sq = mx_sqrt(d > T(0) ? d : T(0));
        const MxSeries<T> s = mx_series(mx_atan2(sq, R0), sq / rr, R0 / rr, a);
        const T t0 = T(-1.0 / 6.0) * s.I_2, t1 = T(0.25) * w.q * s.I_3, t2 = T(-0.15) * w.q2 * s.I_4,
                t3 = T(1.0 / 30.0) * w.q3 * s.I_5, t4 = T(-1.0 / 60.0) * w.iq3 * s.I1, t5 = (w.b1 - w.b2) * s.I0;
        e.D2 = t0 + t1 + t2 + t3 + t4 + t5;
        e.A2 = fabs(t0) + fabs(t1) + fabs(t2) + fabs(t3) + fabs(t4) + fabs(t5);
    }
    const T rr = mx_sqrt(T(4) * h * h - r0 * r0);
    const T d = (rr - R0) * (rr + R0);  // >= 0 up to rounding (the line lies within 2h)
    const T sq = mx_sqrt(d > T(0) ? d : T(0));
    const MxSeries<T> s = mx_series(mx_atan2(sq, R0), sq / rr, R0 / rr, a);
    const T t0 = T(1.0 / 3.0) * s.I_2, t1 = T(-0.25) * w.q * s.I_3, t2 = T(3.0 / 40.0) * w.q2 * s.I_4,
            t3 = T(-1.0 / 120.0) * w.q3 * s.I_5, t4 = T(4.0 / 15.0) * w.iq3 * s.I1, t5 = (w.b2 - w.b3) * s.I0;
    e.D3 = t0 + t1 + t2 + t3 + t4 + t5 + e.D2;
    e.A3 = fabs(t0) + fabs(t1) + fabs(t2) + fabs(t3) + fabs(t4) + fabs(t5) + e.A2;
    return e;
}

// Vertex tier F(r0, R0, t): the right triangle from the foot of the perpendicular to the edge line (at
// in-plane distance R0 > 0) to the point at distance t > 0 along it.  *abs receives the sum of the
// magnitudes of its terms (with those of the edge constant it uses): the scale of its rounding error.
template <class T>
KIWI_MX T mx_vertex(const MxWall<T>& w, const MxEdge<T>& e, T R0, T t, T* abs) {
    const T r0 = w.r0;
    const T rr2 = R0 * R0 + t * t;
    const T rr = mx_sqrt(rr2);
    const T sinp = t / rr, cosp = R0 / rr;
    const T phi = mx_atan2(t, R0);
    const T a = R0 / r0;
    const T r2 = r0 * r0 + rr2;
    const T h2 = w.h * w.h;
    const T pre = w.q3 * T(1.0 / 3.14159265358979323846);
    if (!(r2 < T(4) * h2)) {
        const T a2 = a * a;
        const T I1 = mx_atan(sinp / mx_sqrt(a2 + cosp * cosp));
        const T t0 = T(-0.25) * w.iq3 * I1, t1 = w.b3 * phi;
        *abs = pre * (fabs(t0) + fabs(t1) + e.A3);
        return pre * (t0 + t1 + e.D3);
    }
    const MxSeries<T> s = mx_series(phi, sinp, cosp, a);
    if (r2 < h2) {
        const T t0 = T(1.0 / 6.0) * s.I_2, t1 = T(-3.0 / 40.0) * w.q2 * s.I_4, t2 = T(1.0 / 40.0) * w.q3 * s.I_5,
                t3 = w.b1 * s.I0;
        *abs = pre * (fabs(t0) + fabs(t1) + fabs(t2) + fabs(t3));
        return pre * (t0 + t1 + t2 + t3);
    }
    const T t0 = T(1.0 / 3.0) * s.I_2, t1 = T(-0.25) * w.q * s.I_3, t2 = T(0.075) * w.q2 * s.I_4,
            t3 = T(-1.0 / 120.0) * w.q3 * s.I_5, t4 = T(1.0 / 60.0) * w.iq3 * s.I1, t5 = w.b2 * s.I0;
    *abs = pre * (fabs(t0) + fabs(t1) + fabs(t2) + fabs(t3) + fabs(t4) + fabs(t5) + e.A2);
    return pre * (t0 + t1 + t2 + t3 + t4 + t5 + e.D2);
}

template <class T>
KIWI_MX T mx_sgn(T v) { return v > T(0) ? T(1) : (v < T(0) ? T(-1) : T(0)); }

// Quadrant value Q(r0, u, v) of the plane at distance r0 > 0 (its wall tier w) for the lattice corner
// at in-plane offsets (u, v) from the foot of the perpendicular.
template <class T>
KIWI_MX T mx_quadrant(const MxWall<T>& w, T u, T v, T* abs) {
    const T sg = mx_sgn(u) * mx_sgn(v);
    *abs = T(0);
    if (sg == T(0)) return T(0);
    const T au = fabs(u), av = fabs(v);
    const MxEdge<T> eu = mx_edge(w, au), ev = mx_edge(w, av);
    T a1, a2;
    const T f = mx_vertex(w, eu, au, av, &a1) + mx_vertex(w, ev, av, au, &a2);
    *abs = a1 + a2;
    return sg * f;
}

// Signed pyramid of the rectangle [u0, u1] x [v0, v1] in the plane at signed offset X from the particle.
template <class T>
KIWI_MX T mx_face(T h, T X, T u0, T u1, T v0, T v1, T* abs) {
    *abs = T(0);
    if (X == T(0)) return T(0);
    const MxWall<T> w = mx_wall(h, T(fabs(X)));
    T a0, a1, a2, a3;
    const T f = mx_quadrant(w, u1, v1, &a0) - mx_quadrant(w, u0, v1, &a1) - mx_quadrant(w, u1, v0, &a2) +
                mx_quadrant(w, u0, v0, &a3);
    *abs = a0 + a1 + a2 + a3;
    return f;
}

// Kernel mass of the box [x0, x1] x [y0, y1] x [z0, z1] (offsets from the particle) for smoothing length
// h: each face's pyramid counted + when the particle lies on the inner side of the face, - otherwise.
// *abs receives the sum of the term magnitudes (the scale of the rounding error of the result).
template <class T>
KIWI_MX T mx_cell(T h, T x0, T x1, T y0, T y1, T z0, T z1, T* abs) {
    T m = T(0), s = T(0), a;
    m += mx_sgn(x1) * mx_face(h, x1, y0, y1, z0, z1, &a);
    s += a;
    m -= mx_sgn(x0) * mx_face(h, x0, y0, y1, z0, z1, &a);
    s += a;
    m += mx_sgn(y1) * mx_face(h, y1, x0, x1, z0, z1, &a);
    s += a;
    m -= mx_sgn(y0) * mx_face(h, y0, x0, x1, z0, z1, &a);
    s += a;
    m += mx_sgn(z1) * mx_face(h, z1, x0, x1, y0, y1, &a);
    s += a;
    m -= mx_sgn(z0) * mx_face(h, z0, x0, x1, y0, y1, &a);
    s += a;
    *abs = s;
    return m;
}

}  // namespace mixed
}  // namespace kiwi_b200

#undef KIWI_MX
