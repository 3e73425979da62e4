// The closed-form maths of the lattice kernels (cubic spline and table-driven generic kernels), written over
// the real type T (double in the forward kernels, Dual4 in the adjoint) and compiled both for the device and,
// by the test-only check tests/host_math_check.cpp, for the host.  The kernels' bookkeeping (chunk lists,
// warp votes, lattice offsets) is in lattice.cuh.
#pragma once

#include <math.h>

#include "kiwi_math.cuh"

namespace kiwi_b200 {

constexpr int kLatPMax = 32;     // particles per chunk

// The edge and corner tiers are inlined into the lattice kernels by default (at 80 registers a call
// costs more in saved registers than the larger code does); define either as __noinline__ to keep it out
// of line.
#ifdef __CUDACC__
#ifndef KIWI_EDGE_INLINE
#define KIWI_EDGE_INLINE __forceinline__
#endif
#ifndef KIWI_CORNER_INLINE
#define KIWI_CORNER_INLINE __forceinline__
#endif
#define KIWI_LAT static __host__ __device__ __forceinline__
#define KIWI_LAT_EDGE static __host__ __device__ KIWI_EDGE_INLINE
#define KIWI_LAT_CORNER static __host__ __device__ KIWI_CORNER_INLINE
#define KIWI_LAT_NOINLINE static __host__ __device__ __noinline__
#else
#define KIWI_LAT static inline
#define KIWI_LAT_EDGE static inline
#define KIWI_LAT_CORNER static inline
#define KIWI_LAT_NOINLINE static inline
#endif

// The in-plane angles of the right triangle with legs a1, a2 (reciprocals ia1, ia2): pa = atan(a2 / a1) and
// pb = pi/2 - pa, the smaller one from one arctangent, the larger its complement.  The operand is selected
// and one arctangent evaluated, so that the threads of a warp do not split over two calls.
template <class T>
KIWI_LAT void leg_angles(T a1, T ia1, T a2, T ia2, T& pa, T& pb) {
    const bool lo = a2 <= a1;
    const T t = atan(lo ? a2 * ia1 : a1 * ia2);
    const T c = 0.5 * kPi - t;
    pa = lo ? t : c;
    pb = lo ? c : t;
}

// The wall constants of the cubic spline (src/kernel_integral.cpp:222-247) divided by r0^3, as
// polynomials in r0 / h and h / r0 (the reference forms B_k = r0^3 / 4 (...) and divides by r0^3 at each
// use).  Powers from one reciprocal of h and one of r0.  The functions below are written over the real
// type T: double for the forward kernels, Dual4 (dual.cuh) for the adjoint, whose value part is then the
// forward's bit for bit.
template <class T>
struct LatticeWall {
    T r0h, r0h2, r0h3, r0h_2, r0h_3;  // (r0/h)^k and (h/r0)^k
};
template <class T>
KIWI_LAT LatticeWall<T> lattice_wall(T ih, T h, T ir0, T r0) {
    LatticeWall<T> w;
    w.r0h = r0 * ih;
    w.r0h2 = w.r0h * w.r0h;
    w.r0h3 = w.r0h2 * w.r0h;
    const T hr0 = h * ir0;
    w.r0h_2 = hr0 * hr0;
    w.r0h_3 = w.r0h_2 * hr0;
    return w;
}
// B2 / r0^3 for h < r0 < 2h (its B1 is 0) and for r0 <= h; B1 / r0^3 for r0 <= h; B3 / r0^3 in each range.
template <class T>
KIWI_LAT T wall_b2_mid(const LatticeWall<T>& w) {
    return 0.25 * (-4. / 3. + w.r0h - 0.3 * w.r0h2 + 1. / 30. * w.r0h3 - 1. / 15. * w.r0h_3);
}
template <class T>
KIWI_LAT T wall_b2_in(const LatticeWall<T>& w) {
    return 0.25 * (-2. / 3. + 0.3 * w.r0h2 - 0.1 * w.r0h3 - 0.2 * w.r0h_2);
}
template <class T>
KIWI_LAT T wall_b1_in(const LatticeWall<T>& w) {
    return 0.25 * (-2. / 3. + 0.3 * w.r0h2 - 0.1 * w.r0h3);
}

// The edge tier of one (wall, edge line) pair: D2 (inner edges, line within h) and D3 (line within 2h),
// src/kernel_integral.cpp:253-350.  The tier evaluates the I-series at the angles phi_H where the distance
// to the particle along the edge line reaches H = h and 2h (the reference: acos(R_0 / sqrt(H^2 - r0^2)),
// its sincos, then the series).  Written in the edge's own lengths, with c2 = H^2 - r0^2 and
// t = sqrt(c2 - R_0^2) (the half-chord of the H-sphere on the line): phi_H = atan2(t, R_0),
// tan(phi_H) = t / R_0, 1 / cos^2(phi_H) = c2 / R_0^2, and the series variable u = sin(phi) sqrt(1 - mu^2)
// with mu = r0 / H is t / H, so 1 - u^2 = (r0^2 + R_0^2) / H^2 exactly and
// log(1 + u) - log(1 - u) = log1p(2 u (1 + u) / (1 - u^2)).  No cosine, sine or arccosine is needed, and
// the ratios come from the reciprocal of h and one of r0 R_0 (r0^2 + R_0^2).  The wall differences
// (B1 - B2) / r0^3 and (B2 - B3) / r0^3 are 0.05 (h/r0)^2 and -0.4 (h/r0)^2 within h; -B2 / r0^3 and
// -0.4 (h/r0)^2 between h and 2h.
// ih = 1 / h; r0, R_0 > 0 and r0^2 + R_0^2 <= 4 h^2 (the caller gives D2 = D3 = 0 otherwise).
template <class T>
struct LatticeEdgeT {
    T D2, D3;
};
using LatticeEdge = LatticeEdgeT<double>;
template <class T>
KIWI_LAT_EDGE LatticeEdgeT<T> lattice_edge(T h, T ih, T r0, T R_0) {
    const T ld2 = r0 * r0 + R_0 * R_0;
    const T inv = 1.0 / (r0 * R_0 * ld2);
    const T ir0 = R_0 * ld2 * inv, iR0 = r0 * ld2 * inv, ild2 = r0 * R_0 * inv;
    const LatticeWall<T> w = lattice_wall(ih, h, ir0, r0);
    const T a = R_0 * ir0, a2 = a * a;
    const T b12 = r0 > h ? -wall_b2_mid(w) : 0.05 * w.r0h_2;
    const T b23 = -0.4 * w.r0h_2;
    const T c3 = a * (1. + a2) / 4., c5 = a * (1. + a2) * (1. + a2) / 16.;
    T D2 = 0.0, D3 = 0.0;
#pragma unroll 1
    for (int pass = (ld2 <= h * h) ? 0 : 1; pass < 2; ++pass) {
        const T H = pass == 0 ? h : 2.0 * h, iH = pass == 0 ? ih : 0.5 * ih;
        const T c2 = H * H - r0 * r0;
        const T t = sqrt(fmax(c2 - R_0 * R_0, 0.0));
        const T phi = atan2(t, R_0);
        const T tanp = t * iR0, sec2 = c2 * iR0 * iR0;
        const T u = t * iH, iomu2 = H * H * ild2;
        const T logs = log1p(2.0 * u * (1.0 + u) * iomu2);
        const T I0 = phi;
        const T I_2 = phi + a2 * tanp;
        const T I_4 = phi + 2 * a2 * tanp + 1. / 3. * a2 * a2 * tanp * (2. + sec2);
        const T I1 = atan(u * r0 * iR0);
        const T I_1 = a / 2. * logs + I1;
        const T I_3 = I_1 + c3 * (2 * u * iomu2 + logs);
        const T I_5 = I_3 + c5 * ((10 * u - 6 * u * u * u) * iomu2 * iomu2 + 3. * logs);
        if (pass == 0)
            D2 = -1. / 6. * I_2 + 0.25 * w.r0h * I_3 - 0.15 * w.r0h2 * I_4 + 1. / 30. * w.r0h3 * I_5 -
                 1. / 60. * w.r0h_3 * I1 + b12 * I0;
        else
            D3 = 1. / 3. * I_2 - 0.25 * w.r0h * I_3 + 3. / 40. * w.r0h2 * I_4 - 1. / 120. * w.r0h3 * I_5 +
                 4. / 15. * w.r0h_3 * I1 + b23 * I0 + D2;
    }
    return {D2, D3};
}

// One vertex pyramid of the face walk (src/kernel_integral.cpp:356-400) from its right triangle's
// lengths: legs R_0 (projection -> edge line) and t (along the edge line) in a wall at distance r0,
// r the distance to the vertex.  The series is lattice_corner's for one pyramid: phi = atan2(t, R_0),
// tan(phi) = t / R_0, 1 / cos^2(phi) = (R_0^2 + t^2) / R_0^2, u = t / r, 1 - u^2 = (r0^2 + R_0^2) / r^2,
// u / a = t r0 / (R_0 r).  Beyond 2h the tier is K (-(h/r0)^3 / 4 I1 + B3 / r0^3 phi + D3) with
// K = (r0/h)^3 / pi, i.e. (-I1 + 4 x^3 b3 phi) / (4 pi) + K D3 with x = r0 / h and x^3 b3 a polynomial in
// x; for r0 >= 2h (B3 / r0^3 = (h/r0)^3 / 4) it is (phi - I1) / (4 pi) + K D3, the difference of the two
// arctangents taken as atan(t s^2 R_0 / ((r + r0) (R_0^2 r + t^2 r0))), s^2 = R_0^2 + t^2, which does not
// cancel.  The ratios come from one reciprocal of r0 r R_0 t and one of r0^2 + R_0^2.
// ih = 1 / h; r0, R_0, t > 0; (D2, D3) the edge tier of the triangle's edge line.
template <class T>
KIWI_LAT T lattice_pyramid(T h, T ih, T r0, T R_0, T t, T D2, T D3) {
    const T s2 = R_0 * R_0 + t * t;
    const T r2 = r0 * r0 + s2;
    const T r = sqrt(r2);
    const T phi = atan2(t, R_0);
    if (!(r2 < 4.0 * (h * h))) {
        const T x = r0 * ih, x2 = x * x, x3 = x2 * x;
        const T K = x3 * (1.0 / kPi);
        if (r0 >= 2.0 * h)
            return 0.25 / kPi * atan(t * s2 * R_0 / ((r + r0) * (R_0 * R_0 * r + t * t * r0))) + K * D3;
        const T x4 = x2 * x2, x5 = x4 * x, x6 = x3 * x3;
        const T p = r0 > h ? -4. / 3. * x3 + x4 - 0.3 * x5 + 1. / 30. * x6 - 1. / 15. + 8. / 5. * x
                                : -2. / 3. * x3 + 0.3 * x5 - 0.1 * x6 + 7. / 5. * x;
        return 0.25 / kPi * (p * phi - atan(t * r0 / (R_0 * r))) + K * D3;
    }
    const T inv = 1.0 / (r0 * r * (R_0 * t));
    const T ir0 = r * (R_0 * t) * inv, ir = r0 * (R_0 * t) * inv, iR0 = r0 * r * t * inv;
    const LatticeWall<T> w = lattice_wall(ih, h, ir0, r0);
    const T K = w.r0h3 * (1.0 / kPi);
    const T a = R_0 * ir0, a2k = a * a, u = t * ir;
    const T tanp = t * iR0, sec2 = s2 * iR0 * iR0;
    const T iomu2 = r2 / (r0 * r0 + R_0 * R_0);
    const T I0 = phi;
    const T I_2 = phi + a2k * tanp;
    const T I_4 = phi + 2 * a2k * tanp + 1. / 3. * a2k * a2k * tanp * (2. + sec2);
    const T logs = log1p(2.0 * u * (1.0 + u) * iomu2);
    const T I1 = atan(tanp * r0 * ir);
    const T I_1 = a / 2. * logs + I1;
    const T I_3 = I_1 + a * (1. + a2k) / 4. * (2 * u * iomu2 + logs);
    const T I_5 = I_3 + a * (1. + a2k) * (1. + a2k) / 16. * ((10 * u - 6 * u * u * u) * iomu2 * iomu2 + 3. * logs);
    if (r2 < h * h) return K * (1. / 6. * I_2 - 3. / 40. * w.r0h2 * I_4 + 1. / 40. * w.r0h3 * I_5 + wall_b1_in(w) * I0);
    return K * (0.25 * (4. / 3. * I_2 - w.r0h * I_3 + 0.3 * w.r0h2 * I_4 - 1. / 30. * w.r0h3 * I_5 + 1. / 15. * w.r0h_3 * I1) +
                (r0 > h ? wall_b2_mid(w) : wall_b2_in(w)) * I0 + D2);
}

// The pyramid pair of one corner value, F(r0, a1, a2) + F(r0, a2, a1): the two right triangles of the
// rectangle spanned by the particle's projection and the corner (legs a1 along the first edge line and a2
// along the second, and the reverse), in the wall at distance r0.  The vertex tier's series
// (src/kernel_integral.cpp:356-400) is written here in the triangle's own lengths, which the pair shares:
// with r the distance to the corner, the series variable u = sin(phi) sqrt(1 - mu^2) is a2 / r for the
// first pyramid and a1 / r for the second (so 1 - u^2 = (r0^2 + a1^2) / r^2, (r0^2 + a2^2) / r^2 exactly),
// tan(phi) = a2 / a1 (a1 / a2), 1 / cos^2(phi) = (a1^2 + a2^2) / a1^2 (/ a2^2), u / a = a2 r0 / (a1 r)
// (a1 r0 / (a2 r)), and the two angles sum to pi/2 (the smaller one is the arctangent of its tangent, the
// larger its complement, both to an ulp).  log(1 + u) - log(1 - u) = log1p(2 u (1 + u) / (1 - u^2)).  The
// ratios come from two reciprocals: of r0 r a1 a2 and of (r0^2 + a1^2)(r0^2 + a2^2).  Beyond 2h a tier
// needs I0 = phi and I1 only: the angles sum to pi/2 and I1a + I1b = atan(r0 r / (a1 a2)) (tan of the sum
// of the two arctangents), so the pair is one arctangent, and with the prefactor (r0/h)^3 / pi multiplied
// in, the wall term B3 / r0^3 x pi/2 is a polynomial in r0 / h: the pair needs no reciprocal of r0.  For
// r0 >= 2h (B3 / r0^3 = (h/r0)^3 / 4) it is atan(a1 a2 / (r0 r)) / (4 pi).  ih = 1 / h; r0, a1, a2 > 0 (the
// callers skip zero corners); (D2a, D3a) and (D2b, D3b) are the two edge tiers.
template <class T>
KIWI_LAT_CORNER T lattice_corner(T h, T ih, T r0, T a1, T a2, T D2a, T D3a, T D2b, T D3b) {
    const T s2 = a1 * a1 + a2 * a2;
    const T r2 = r0 * r0 + s2;
    const T r = sqrt(r2);
    if (!(r2 < 4.0 * (h * h))) {
        const T x = r0 * ih, x2 = x * x, x3 = x2 * x;
        const T K = x3 * (1.0 / kPi);
        if (r0 >= 2.0 * h) return 0.25 / kPi * atan(a1 * a2 / (r0 * r)) + K * (D3a + D3b);
        const T x4 = x2 * x2, x5 = x4 * x, x6 = x3 * x3;
        const T p = r0 > h ? -4. / 3. * x3 + x4 - 0.3 * x5 + 1. / 30. * x6 - 1. / 15. + 8. / 5. * x
                                : -2. / 3. * x3 + 0.3 * x5 - 0.1 * x6 + 7. / 5. * x;
        return -0.25 / kPi * atan(r0 * r / (a1 * a2)) + 0.125 * p + K * (D3a + D3b);
    }
    const T inv1 = 1.0 / (r0 * r * (a1 * a2));
    const T ir0 = r * (a1 * a2) * inv1, ir = r0 * (a1 * a2) * inv1;
    const T ia1 = r0 * r * a2 * inv1, ia2 = r0 * r * a1 * inv1;
    const LatticeWall<T> w = lattice_wall(ih, h, ir0, r0);
    const T K = w.r0h3 * (1.0 / kPi);
    T pa, pb;
    leg_angles(a1, ia1, a2, ia2, pa, pb);
    const bool inner = r2 < h * h;
    const T b1 = inner ? wall_b1_in(w) : 0.0;
    const T b2 = r0 > h ? wall_b2_mid(w) : wall_b2_in(w);
    const T q1 = r0 * r0 + a1 * a1, q2 = r0 * r0 + a2 * a2;
    const T inv2 = 1.0 / (q1 * q2);
    T sum = 0.0;
#pragma unroll 1
    for (int k = 0; k < 2; ++k) {
        const T leg = k ? a2 : a1, opp = k ? a1 : a2, ileg = k ? ia2 : ia1, phi = k ? pb : pa;
        const T a = leg * ir0, u = opp * ir;
        const T tanp = opp * ileg, sec2 = s2 * ileg * ileg;
        const T iomu2 = r2 * (k ? q1 : q2) * inv2;
        const T a2k = a * a;
        const T I0 = phi;
        const T I_2 = phi + a2k * tanp;
        const T I_4 = phi + 2 * a2k * tanp + 1. / 3. * a2k * a2k * tanp * (2. + sec2);
        const T logs = log1p(2.0 * u * (1.0 + u) * iomu2);
        // I_1, I_3, I_5 without their common I1 term (added below for the pair)
        const T I_1 = a / 2. * logs;
        const T I_3 = I_1 + a * (1. + a2k) / 4. * (2 * u * iomu2 + logs);
        const T I_5 = I_3 + a * (1. + a2k) * (1. + a2k) / 16. * ((10 * u - 6 * u * u * u) * iomu2 * iomu2 + 3. * logs);
        if (inner) sum += 1. / 6. * I_2 - 3. / 40. * w.r0h2 * I_4 + 1. / 40. * w.r0h3 * I_5 + b1 * I0;
        else
            sum += 0.25 * (4. / 3. * I_2 - w.r0h * I_3 + 0.3 * w.r0h2 * I_4 - 1. / 30. * w.r0h3 * I_5) + b2 * I0 +
                   (k ? D2b : D2a);
    }
    // I1 enters both pyramids with one coefficient (through I_1, I_3, I_5 and, between h and 2h, on its own):
    // the pair needs I1a + I1b = atan(r0 r / (a1 a2)) only.
    const T I1s = atan((r0 * r) * (r0 * r) * inv1);
    const T c1 = inner ? 1. / 40. * w.r0h3 : 0.25 * (-w.r0h - 1. / 30. * w.r0h3 + 1. / 15. * w.r0h_3);
    return K * (sum + c1 * I1s);
}

// ---- point-wise form: the three corner values of one lattice point and the two edge tiers of one pair
//
// A lattice point at offsets (ux, uy, uz) from the particle is a corner of three walls: the plane x = X
// (corner (y, z) in it, wall distance |ux|), y = Y and z = Z.  Its three corner values (lattice_corner)
// share the distance r, the product |ux uy uz| (r0 a1 a2 in every orientation) and, since the series
// variable u of a pyramid is opp / r with opp one of |ux|, |uy|, |uz|, only three distinct logarithm terms
// (log((1 + u) / (1 - u)) for u = |ux| / r, |uy| / r, |uz| / r) among their six pyramids.  So the point
// needs one square root, one reciprocal of r |ux uy uz| (giving 1/r, 1/|ux|, 1/|uy|, 1/|uz|), one of the
// product of the three pair sums S_xy S_xz S_yz (giving every 1 / (1 - u^2) = r^2 / S), three log1p and five
// arctangents (the three walls' I1 angles sum to pi, point_angles) -- where three separate corners need three
// roots, six reciprocals, six log1p and six arctangents.  Its octant value is the sum of the three: the kernel mass of the box spanned by the
// particle and the point (by the divergence theorem over that box, whose three faces through the particle
// carry no flux), so a cell's mass is the 8-term difference of its corners' octant values.

// The six edge tiers a lattice point reads: wall x with edge lines at |uy| (xy) and |uz| (xz), wall y with
// lines at |ux| (yx) and |uz| (yz), wall z with lines at |ux| (zx) and |uy| (zy).  lattice_point reads them
// through an accessor with D2(e) and D3(e), e one of these, so that each is loaded where it is used; this
// one holds them as values.
enum PointEdge { kEdgeXY = 0, kEdgeXZ, kEdgeYX, kEdgeYZ, kEdgeZX, kEdgeZY };
template <class T>
struct PointEdges {
    T d2[6], d3[6];
    KIWI_HD T D2(int e) const { return d2[e]; }
    KIWI_HD T D3(int e) const { return d3[e]; }
    // the in-plane angles of the wall whose legs lie along edge pair e's two axes (leg_angles)
    KIWI_HD void leg_angles(int e, T a1, T ia1, T a2, T ia2, T& pa, T& pb) const {
        kiwi_b200::leg_angles(a1, ia1, a2, ia2, pa, pb);
    }
};

// One vertex pyramid of the series inside 2h (lattice_corner's loop body): legs `leg` (towards the edge line
// of tier D2) and `opp`, wall w at r0; with a = leg / r0, u = opp / r, tan(phi) = opp / leg,
// 1 / cos^2(phi) = s2 / leg^2, iomu2 = 1 / (1 - u^2), logs = log((1 + u) / (1 - u)).  Without the I1 term.
template <class T>
KIWI_LAT T point_pyramid(const LatticeWall<T>& w, bool inner, T b1, T b2, T a, T u, T tanp,
                                                  T sec2, T iomu2, T logs, T phi, T D2) {
    const T a2k = a * a;
    const T I_2 = phi + a2k * tanp;
    const T I_4 = phi + 2 * a2k * tanp + 1. / 3. * a2k * a2k * tanp * (2. + sec2);
    const T I_1 = a / 2. * logs;
    const T I_3 = I_1 + a * (1. + a2k) / 4. * (2 * u * iomu2 + logs);
    const T I_5 = I_3 + a * (1. + a2k) * (1. + a2k) / 16. * ((10 * u - 6 * u * u * u) * iomu2 * iomu2 + 3. * logs);
    if (inner) return 1. / 6. * I_2 - 3. / 40. * w.r0h2 * I_4 + 1. / 40. * w.r0h3 * I_5 + b1 * phi;
    return 0.25 * (4. / 3. * I_2 - w.r0h * I_3 + 0.3 * w.r0h2 * I_4 - 1. / 30. * w.r0h3 * I_5) + b2 * phi + D2;
}

// One wall's corner value inside 2h (lattice_corner) from the point's shared quantities: wall distance r0
// and its reciprocal, in-plane legs a1 (edge tier E.D2(ea)) and a2 (E.D2(eb)) with reciprocals,
// s2 = a1^2 + a2^2, r and its reciprocal, the log terms of u = a2 / r (first pyramid) and u = a1 / r
// (second), their 1 / (1 - u^2), and the pair's I1 sum atan(r0 r / (a1 a2)) (point_angles).  The in-plane
// angles depend on a1 and a2 alone, so the Edges reader may hold them per edge pair: ec is the pair (the
// edge line along a2 at a1) whose angles they are.
template <class T, class Edges>
KIWI_LAT T point_wall(T h, T ih, bool inner, T r0, T ir0, T a1, T ia1, T a2, T ia2, T s2, T ir, T log_a2, T iom_a2,
                      T log_a1, T iom_a1, T I1s, const Edges& E, int ea, int eb, int ec) {
    const LatticeWall<T> w = lattice_wall(ih, h, ir0, r0);
    T pa, pb;
    E.leg_angles(ec, a1, ia1, a2, ia2, pa, pb);
    const T b1 = inner ? wall_b1_in(w) : 0.0;
    const T b2 = r0 > h ? wall_b2_mid(w) : wall_b2_in(w);
    T sum = point_pyramid(w, inner, b1, b2, a1 * ir0, a2 * ir, a2 * ia1, s2 * ia1 * ia1, iom_a2, log_a2, pa,
                          inner ? T(0.0) : E.D2(ea));
    sum += point_pyramid(w, inner, b1, b2, a2 * ir0, a1 * ir, a1 * ia2, s2 * ia2 * ia2, iom_a1, log_a1, pb,
                         inner ? T(0.0) : E.D2(eb));
    const T c1 = inner ? 1. / 40. * w.r0h3 : 0.25 * (-w.r0h - 1. / 30. * w.r0h3 + 1. / 15. * w.r0h_3);
    return w.r0h3 * (1.0 / kPi) * (sum + c1 * I1s);
}

// One wall's corner value beyond 2h (lattice_corner's first branch): x = r0 / h, the angle
// J = atan(r0 r / (a1 a2)) (point_angles), and the edge tiers E.D3(ea), E.D3(eb) of the wall's two edge lines.
// For r0 >= 2h the value is the rectangle's solid angle over 4 pi, atan(a1 a2 / (r0 r)) / (4 pi) =
// (pi/2 - J) / (4 pi): where that angle is small its relative precision is lost, not its absolute one, which
// is what the cell's alternating sum of octant values needs.
template <class T, class Edges>
KIWI_LAT T point_wall_far(T h, T ih, T r0, T J, const Edges& E, int ea, int eb) {
    const T x = r0 * ih, x2 = x * x, x3 = x2 * x;
    const T K = x3 * (1.0 / kPi);
    if (r0 >= 2.0 * h) return 0.25 / kPi * (0.5 * kPi - J) + K * (E.D3(ea) + E.D3(eb));
    const T x4 = x2 * x2, x5 = x4 * x, x6 = x3 * x3;
    const T p = r0 > h ? -4. / 3. * x3 + x4 - 0.3 * x5 + 1. / 30. * x6 - 1. / 15. + 8. / 5. * x
                       : -2. / 3. * x3 + 0.3 * x5 - 0.1 * x6 + 7. / 5. * x;
    return -0.25 / kPi * J + 0.125 * p + K * (E.D3(ea) + E.D3(eb));
}

// The three walls' angles J_c = atan(a_c r / (a_a a_b)) of a lattice point (a_a, a_b the other two offsets)
// sum to pi: tan J_x tan J_y = r^2 / az^2 > 1, so tan(J_x + J_y) = -tan J_z with J_x + J_y in (pi/2, pi).  Two
// come from arctangents, the largest (at least pi/3) as pi minus the others.
// The two arctangents take selected operands, so that the threads of a warp do not split over the three
// cases' calls.
template <class T>
KIWI_LAT void point_angles(T qx, T qy, T qz, T& Jx, T& Jy, T& Jz) {
    const bool mx = qx >= qy && qx >= qz, my = !mx && qy >= qz;  // the largest: x, y, else z
    const T ta = atan(mx ? qy : qx);                             // J_y if x is the largest, else J_x
    const T tb = atan(mx || my ? qz : qy);                       // J_z unless z is the largest, then J_y
    const T tc = kPi - ta - tb;
    Jx = mx ? tc : ta;
    Jy = mx ? ta : (my ? tc : tb);
    Jz = mx || my ? tb : tc;
}

// The sum of the three corner values of a lattice point at absolute offsets ax, ay, az > 0 from the
// particle (unsigned; the octant value is sgn(ux) sgn(uy) sgn(uz) times it).  Equal to
// lattice_corner(ax; ay, az) + lattice_corner(ay; ax, az) + lattice_corner(az; ax, ay) up to rounding.
template <class T, class Edges>
KIWI_LAT_CORNER T lattice_point(T h, T ih, T ax, T ay, T az, const Edges& E) {
    const T ax2 = ax * ax, ay2 = ay * ay, az2 = az * az;
    const T sxy = ax2 + ay2, sxz = ax2 + az2, syz = ay2 + az2;
    const T r2 = sxy + az2;
    const T r = sqrt(r2);
    const T axyz = ax * (ay * az);
    const T iP = 1.0 / (r * axyz);  // 1 / (r |ux uy uz|)
    // r0 r / (a1 a2) of the wall at a_c: a_c^2 r^2 iP; its inverse: (product of the other two)^2 iP
    T Jx, Jy, Jz;
    point_angles(ax2 * r2 * iP, ay2 * r2 * iP, az2 * r2 * iP, Jx, Jy, Jz);
    if (!(r2 < 4.0 * (h * h))) {
        return point_wall_far(h, ih, ax, Jx, E, kEdgeXY, kEdgeXZ) + point_wall_far(h, ih, ay, Jy, E, kEdgeYX, kEdgeYZ) +
               point_wall_far(h, ih, az, Jz, E, kEdgeZX, kEdgeZY);
    }
    const T ir = axyz * iP;
    const T iax = r * (ay * az) * iP, iay = r * (ax * az) * iP, iaz = r * (ax * ay) * iP;
    const T iQ = 1.0 / (sxy * sxz * syz);
    // 1 / (1 - u^2) = r^2 / (r^2 - a_c^2) for u = a_c / r
    const T iomx = r2 * (sxy * sxz) * iQ, iomy = r2 * (sxy * syz) * iQ, iomz = r2 * (sxz * syz) * iQ;
    const T ux = ax * ir, uy = ay * ir, uz = az * ir;
    const T Lx = log1p(2.0 * ux * (1.0 + ux) * iomx);
    const T Ly = log1p(2.0 * uy * (1.0 + uy) * iomy);
    const T Lz = log1p(2.0 * uz * (1.0 + uz) * iomz);
    const bool inner = r2 < h * h;
    T s = point_wall(h, ih, inner, ax, iax, ay, iay, az, iaz, syz, ir, Lz, iomz, Ly, iomy, Jx, E, kEdgeXY, kEdgeXZ,
                     kEdgeYZ);
    s += point_wall(h, ih, inner, ay, iay, ax, iax, az, iaz, sxz, ir, Lz, iomz, Lx, iomx, Jy, E, kEdgeYX, kEdgeYZ,
                    kEdgeXZ);
    s += point_wall(h, ih, inner, az, iaz, ax, iax, ay, iay, sxy, ir, Ly, iomy, Lx, iomx, Jz, E, kEdgeZX, kEdgeZY,
                    kEdgeXY);
    return s;
}

// The edge tiers of both orientations of one (p, q) pair (lattice_edge): e_pq is the tier of the edge line at
// in-plane distance q in the wall at distance p, e_qp the one at distance p in the wall at q.  They share
// r0^2 + R_0^2, the reciprocal of p q (p^2 + q^2), and per pass the half-chord t and the log term (u = t / H
// and 1 - u^2 = (p^2 + q^2) / H^2 are the same for both).  p, q > 0 and p^2 + q^2 <= 4 h^2.
template <class T>
KIWI_LAT_EDGE void lattice_edge_pair(T h, T ih, T p, T q, LatticeEdgeT<T>& e_pq,
                                                          LatticeEdgeT<T>& e_qp) {
    const T ld2 = p * p + q * q;
    const T inv = 1.0 / (p * q * ld2);
    const T ip = q * ld2 * inv, iq = p * ld2 * inv, ild2 = p * q * inv;
    const LatticeWall<T> wp = lattice_wall(ih, h, ip, p), wq = lattice_wall(ih, h, iq, q);
    const T ap = q * ip, ap2 = ap * ap;  // a = R_0 / r0 of e_pq
    const T aq = p * iq, aq2 = aq * aq;  // of e_qp
    const T b12p = p > h ? -wall_b2_mid(wp) : 0.05 * wp.r0h_2, b23p = -0.4 * wp.r0h_2;
    const T b12q = q > h ? -wall_b2_mid(wq) : 0.05 * wq.r0h_2, b23q = -0.4 * wq.r0h_2;
    const T c3p = ap * (1. + ap2) / 4., c5p = ap * (1. + ap2) * (1. + ap2) / 16.;
    const T c3q = aq * (1. + aq2) / 4., c5q = aq * (1. + aq2) * (1. + aq2) / 16.;
    T D2p = 0.0, D3p = 0.0, D2q = 0.0, D3q = 0.0;
#pragma unroll 1
    for (int pass = (ld2 <= h * h) ? 0 : 1; pass < 2; ++pass) {
        const T H = pass == 0 ? h : 2.0 * h, iH = pass == 0 ? ih : 0.5 * ih;
        const T t = sqrt(fmax(H * H - ld2, 0.0));
        const T u = t * iH, iomu2 = H * H * ild2;
        const T logs = log1p(2.0 * u * (1.0 + u) * iomu2);
        const T s35 = 2 * u * iomu2 + logs;
        const T s5 = (10 * u - 6 * u * u * u) * iomu2 * iomu2 + 3. * logs;
        // e_pq: R_0 = q, c2 = H^2 - p^2
        {
            const T phi = atan2(t, q);
            const T tanp = t * iq, sec2 = (H * H - p * p) * iq * iq;
            const T I_2 = phi + ap2 * tanp;
            const T I_4 = phi + 2 * ap2 * tanp + 1. / 3. * ap2 * ap2 * tanp * (2. + sec2);
            const T I1 = atan(u * p * iq);
            const T I_1 = ap / 2. * logs + I1;
            const T I_3 = I_1 + c3p * s35;
            const T I_5 = I_3 + c5p * s5;
            if (pass == 0)
                D2p = -1. / 6. * I_2 + 0.25 * wp.r0h * I_3 - 0.15 * wp.r0h2 * I_4 + 1. / 30. * wp.r0h3 * I_5 -
                      1. / 60. * wp.r0h_3 * I1 + b12p * phi;
            else
                D3p = 1. / 3. * I_2 - 0.25 * wp.r0h * I_3 + 3. / 40. * wp.r0h2 * I_4 - 1. / 120. * wp.r0h3 * I_5 +
                      4. / 15. * wp.r0h_3 * I1 + b23p * phi + D2p;
        }
        // e_qp: R_0 = p, c2 = H^2 - q^2
        {
            const T phi = atan2(t, p);
            const T tanp = t * ip, sec2 = (H * H - q * q) * ip * ip;
            const T I_2 = phi + aq2 * tanp;
            const T I_4 = phi + 2 * aq2 * tanp + 1. / 3. * aq2 * aq2 * tanp * (2. + sec2);
            const T I1 = atan(u * q * ip);
            const T I_1 = aq / 2. * logs + I1;
            const T I_3 = I_1 + c3q * s35;
            const T I_5 = I_3 + c5q * s5;
            if (pass == 0)
                D2q = -1. / 6. * I_2 + 0.25 * wq.r0h * I_3 - 0.15 * wq.r0h2 * I_4 + 1. / 30. * wq.r0h3 * I_5 -
                      1. / 60. * wq.r0h_3 * I1 + b12q * phi;
            else
                D3q = 1. / 3. * I_2 - 0.25 * wq.r0h * I_3 + 3. / 40. * wq.r0h2 * I_4 - 1. / 120. * wq.r0h3 * I_5 +
                      4. / 15. * wq.r0h_3 * I1 + b23q * phi + D2q;
        }
    }
    e_pq = {D2p, D3p};
    e_qp = {D2q, D3q};
}

// ---- generic kernels (table-driven tiers, src/kernel_integral_generic.cpp) in the lattice form
//
// The edge tier of a generic kernel is the list of the kernel's regions crossed along the edge line, with
// the angles where it leaves each region and the continuity offsets (generic_edge, :119-148).  Its lattice
// record packs that as 7 doubles: [0] = nseg + 8 x first region, [1..3] = phi_end of segments 0..2,
// [4..6] = offset of segments 1..3 (segment 0's is 0; the last segment ends at pi/2).
constexpr int kLatGenERec = 7;
constexpr int kLatGenECap = 640;  // edge records per chunk (a full 8^3 particle box needs 486)

// The value of a real number of any of the tiers' types (double, the FP32 type, a dual number), for the
// decisions taken on values: kernel regions and segment choices.
KIWI_LAT double lat_value(double x) { return x; }
template <class T>
KIWI_LAT double lat_value(const T& x) {
    return (double)x.v;
}

// G_k(phi) = bphi_k phi + sum_i coef_k,i I_i(phi) for a wall at q0 = r0 / H in region j of the kernel
// (generic_G, src/kernel_integral_generic.cpp:82-92), a = R0 / r0, with what the basis integrals are built
// from given: tn = tan(phi), sc = 1 / cos(phi), the series variable u = a sin(phi) / sqrt(a^2 + cos^2(phi))
// (= t / r for the vertex at distance r whose leg along the edge is t), iomu2 = 1 / (1 - u^2), I1 = atan(u / a)
// and K0 = atanh(u).  The wall coefficients A3 a_k,i q0^i are formed on the fly and each basis integral I_i
// (the recurrences of :19-66) is added as soon as it is formed, in ascending index order: every loop is
// unrolled over the table's fixed width and predicated on the region's lowest index, so the basis values,
// the sec-power integrals J_2l and the powers of q0 stay in registers.  q0^i is a compensated running
// product (hi + lo, the product's rounding error carried exactly by fma): the terms can cancel heavily, and a
// plain running product's rounding (up to ~i ulp) measurably raised the error of low-density cells; this is
// within an ulp, like pow, at a fraction of its cost; (1 - u^2)^-m in the K recurrence is formed the same way.
template <class T>
KIWI_LAT T lattice_generic_G_pt(const KiwiKernelTable* K, T q0, int j, int k, T a, T a2, T phi, T tn,
                                         T sc, T u, T iomu2, T I1, T K0) {
    const double* ak = K->a[k - 1];
    int imin = 1;
    for (int idx = KIWI_NI - 1; idx >= 0; --idx)
        if (ak[idx] != 0.0) {
            imin = 1 - idx;
            break;
        }
    const double A3 = K->A3_pi / kPi;
    T b = 0.0;
    if (k >= j)
        for (int p = KIWI_NB - 1; p >= 0; --p) b = b * q0 + K->B[j - 1][k - 1][p];
    T sum = (A3 * b) * phi;
    T ph = 1.0, pl = 0.0;  // q0^idx
    T wh = 1.0, wl = 0.0;  // (1 - u^2)^-m, compensated like q0^idx
    T Iodd = 0.0, Kc = 0.0, pow1a2 = 1.0, spow = 1.0;
    T J[(KIWI_NI + 1) / 2];  // J[l] = int_0^phi sec^(2l)
#pragma unroll
    for (int idx = 0; idx < KIWI_NI; ++idx) {
        if (1 - idx < imin) break;
        T Iv;
        if (idx == 0) {  // I_1 = atan(u / a)
            Iv = I1;
            Iodd = Iv;
            Kc = K0;
        } else if (idx == 1) {  // I_0 = phi
            Iv = phi;
        } else if ((idx & 1) == 0) {  // I_-(2m+1), m = idx / 2 - 1
            const int m = idx / 2 - 1;
            if (m > 0) {
                const T nw = wh * iomu2;
                wl = fma(wl, iomu2, fma(wh, iomu2, -nw));
                wh = nw;
                Kc = u * (wh + wl) * (1.0 / (2.0 * m)) + (2.0 * m - 1.0) / (2.0 * m) * Kc;
                pow1a2 *= (1.0 + a2);
            }
            Iodd += a * pow1a2 * Kc;
            Iv = Iodd;
        } else {  // I_-2kk = sum_l C(kk, l) a^2l J_2l, kk = (idx - 1) / 2
            const int kk = (idx - 1) / 2;
            if (kk == 1) {
                J[0] = phi;
                J[1] = tn;
            } else {
                spow *= sc * sc;
                J[kk] = spow * tn * (1.0 / (2 * kk - 1.0)) + (2 * kk - 2.0) / (2 * kk - 1.0) * J[kk - 1];
            }
            T s = J[0], apow = 1.0;
            double bc = 1.0;
#pragma unroll
            for (int l = 1; l <= kk; ++l) {
                bc = bc * (kk - l + 1) / l;
                apow *= a2;
                s += bc * apow * J[l];
            }
            Iv = s;
        }
        const double c = ak[idx];
        if (c != 0.0) sum += (A3 * c * (ph + pl)) * Iv;
        const T nh = ph * q0;
        pl = fma(pl, q0, fma(ph, q0, -nh));
        ph = nh;
    }
    return sum;
}

// G_k(phi) with sin(phi) and cos(phi) given: u / a = sin(phi) / sqrt(a^2 + cos^2(phi)) and
// 1 / (1 - u^2) = (a^2 + cos^2(phi)) / (cos^2(phi) (1 + a^2)): three reciprocals in all.
template <class T>
KIWI_LAT_NOINLINE T lattice_generic_G(const KiwiKernelTable* K, T q0, int j, int k, T a, T a2, T phi, T sinp,
                                      T cosp) {
    const T den = a2 + cosp * cosp, iden = 1.0 / den;
    const T ua = sinp * sqrt(iden), u = a * ua;
    const T iomu2 = den / (cosp * cosp * (1.0 + a2));
    const T sc = 1.0 / cosp, tn = sinp * sc;
    return lattice_generic_G_pt(K, q0, j, k, a, a2, phi, tn, sc, u, iomu2, atan(ua), atanh(u));
}

// The edge record of a generic kernel for the edge line at in-plane distance R0 in the wall at r0 (support
// radius H): the kernel regions crossed along the line and the angles where it leaves each
// (generic_edge, :119-148): w.set(nseg + 8 x first region), then per segment boundary s = 0..nseg-2 the
// angle phi_end(s) and the continuity offset of segment s + 1.
template <class T, class W>
KIWI_LAT void lattice_generic_edge_t(const KiwiKernelTable* K, double H, T r0, T R0, W& w) {
    if (r0 == 0.0 || R0 == 0.0) return;
    const T q0 = r0 / H, qR = R0 / H;
    const T a = R0 / r0, a2 = a * a;
    const int j = generic_region(K, lat_value(q0));
    const int k0 = generic_region(K, lat_value(sqrt(q0 * q0 + qR * qR)));
    const int nseg = K->nreg - k0 + 1;
    w.set_packed((double)(nseg + 8 * k0));
    T off = 0.0;
    for (int s = 0; s + 1 < nseg; ++s) {
        const int k = k0 + s;
        const double c = K->c[k - 1];
        const T pb = acos(fmin(1.0, qR / sqrt(c * c - q0 * q0)));
        const T sp = sin(pb), cp = cos(pb);
        off = off + lattice_generic_G(K, q0, j, k, a, a2, pb, sp, cp) - lattice_generic_G(K, q0, j, k + 1, a, a2, pb, sp, cp);
        if (s < 3) w.set_segment(s, pb, off);
    }
}

// The double record: [0] = nseg + 8 x first region, [1..3] = phi_end of segments 0..2, [4..6] = offset of
// segments 1..3.
// (The record is stored in doubles whatever type the tiers were evaluated in.)
struct GenEdgeWriter {
    double* rec;
    KIWI_HD void set_packed(double v) { rec[0] = v; }
    template <class T>
    KIWI_HD void set_segment(int s, T phi_end, T off) {
        rec[1 + s] = lat_value(phi_end);
        rec[4 + s] = lat_value(off);
    }
};

template <class T>
KIWI_LAT void lattice_generic_edge(const KiwiKernelTable* K, double H, T r0, T R0, double* rec) {
    for (int i = 0; i < kLatGenERec; ++i) rec[i] = 0.0;
    GenEdgeWriter w{rec};
    lattice_generic_edge_t(K, H, r0, R0, w);
}


// Vertex tier of a generic kernel for the right triangle with legs R0 (projection -> edge line) and t
// (along the edge) in a wall at distance r0 (generic_vertex, :150-156, at phi = atan2(t, R0)): the region
// segment holding phi, its offset, and G_k(phi).
// The two vertex tiers of a lattice corner (legs a1, a2 in the wall at r0; the edge records rec1 of the
// a1 line and rec2 of the a2 line: vertex 1 has R0 = a1, t = a2 and vertex 2 the reverse) share what the
// pair has in common: the distance sqrt(a1^2 + a2^2) and its reciprocal, 1 / r0, q0 = r0 / H and its
// kernel region, and the angle pair (the smaller one from atan2, the larger its complement, as in
// lattice_corner).  r0, a1, a2 > 0.  (lattice_generic_point evaluates a point's three walls together; it
// is the adjoint's form: in double it measured slower than three corners and less accurate in low-density
// cells of the generic fixtures.)
template <class T>
KIWI_LAT T lattice_generic_corner(const KiwiKernelTable* K, double H, T r0, T a1, T a2, const double* rec1,
                                  const double* rec2) {
    const T ir0 = 1.0 / r0, irr = 1.0 / sqrt(a1 * a1 + a2 * a2);
    const T q0 = r0 / H;
    const int j = generic_region(K, lat_value(q0));
    // the smaller angle from one atan2 with selected operands (no warp split over two calls), the larger
    // its complement
    const bool lo = a2 <= a1;
    const T tq = atan2(lo ? a2 : a1, lo ? a1 : a2), tc = 0.5 * kPi - tq;
    const T pa = lo ? tq : tc, pb = lo ? tc : tq;
    T sum = 0.0;
#pragma unroll 1
    for (int v = 0; v < 2; ++v) {
        const double* rec = v ? rec2 : rec1;
        const int packed = (int)rec[0];
        const int nseg = packed & 7, k0 = packed >> 3;
        if (nseg == 0) continue;
        const T R0 = v ? a2 : a1, t = v ? a1 : a2, phi = v ? pb : pa;
        const T a = R0 * ir0;
        int s = 0;
        while (s + 1 < nseg && phi > rec[1 + s]) ++s;
        const T G = lattice_generic_G(K, q0, j, k0 + s, a, a * a, phi, t * irr, R0 * irr);
        sum += (s > 0 ? T(rec[3 + s]) : T(0.0)) + G;
    }
    return sum;
}

// The three corner values of a lattice point for a generic kernel (support radius H), as
// lattice_generic_corner(ax; ay, az) + lattice_generic_corner(ay; ax, az) + lattice_generic_corner(az; ax, ay).
// The six vertex tiers share the point's distance r and one reciprocal of r |ux uy uz| (1/r and the 1/a_c),
// the series variable u = t / r with atanh(u) (three distinct, u_c = a_c / r) and 1 / (1 - u^2) =
// r^2 / (r^2 - a_c^2) from one reciprocal of S_xy S_xz S_yz, and I_1 = atan(u / a) = atan(a_a a_b / (a_c r)) =
// pi/2 - J_c for the leg a_c the vertex's edge line lies at (three distinct, their J_c summing to pi:
// point_angles).  ax, ay, az > 0.
// The six edge records of a lattice point: base + kLatGenERec x slot, in PointEdge order.  The slot is
// selected, not indexed, so that the lookup stays in registers.
struct GenEdgeRecs {
    const double* base;
    int slot[6];
    KIWI_HD const double* rec(int e) const {
        const int sl = e < 3 ? (e == 0 ? slot[0] : (e == 1 ? slot[1] : slot[2]))
                             : (e == 3 ? slot[3] : (e == 4 ? slot[4] : slot[5]));
        return base + kLatGenERec * sl;
    }
    KIWI_HD int packed(const double* r) const { return (int)r[0]; }
    KIWI_HD double phi_end(const double* r, int s) const { return r[1 + s]; }
    KIWI_HD double offset(const double* r, int s) const { return r[3 + s]; }  // segment s >= 1
};

// The three corner values of a lattice point for a generic kernel (support radius H), as
// lattice_generic_corner(ax; ay, az) + lattice_generic_corner(ay; ax, az) + lattice_generic_corner(az; ax, ay).
// The six vertex tiers share the point's distance r and one reciprocal of r |ux uy uz| (1/r and the 1/a_c),
// the series variable u = t / r with atanh(u) (three distinct, u_c = a_c / r) and 1 / (1 - u^2) =
// r^2 / (r^2 - a_c^2) from one reciprocal of S_xy S_xz S_yz, and I_1 = atan(u / a) = atan(a_a a_b / (a_c r)) =
// pi/2 - J_c for the leg a_c the vertex's edge line lies at (three distinct, their J_c summing to pi:
// point_angles).  R reads the six edge records (rec(e) in PointEdge order; packed, phi_end, offset).
// ax, ay, az > 0.
template <class T, class R>
KIWI_LAT T lattice_generic_point(const KiwiKernelTable* K, double H, T ax, T ay, T az, const R& recs) {
    const T ax2 = ax * ax, ay2 = ay * ay, az2 = az * az;
    const T sxy = ax2 + ay2, sxz = ax2 + az2, syz = ay2 + az2;
    const T r2 = sxy + az2;
    const T r = sqrt(r2);
    const T axyz = ax * (ay * az);
    const T iP = 1.0 / (r * axyz);
    const T ir = axyz * iP;
    const T iax = r * (ay * az) * iP, iay = r * (ax * az) * iP, iaz = r * (ax * ay) * iP;
    const T iQ = 1.0 / (sxy * sxz * syz);
    const T iomx = r2 * (sxy * sxz) * iQ, iomy = r2 * (sxy * syz) * iQ, iomz = r2 * (sxz * syz) * iQ;
    const T ux = ax * ir, uy = ay * ir, uz = az * ir;
    const T Kx = atanh(ux), Ky = atanh(uy), Kz = atanh(uz);
    T Ix, Iy, Iz;
    point_angles(ax2 * r2 * iP, ay2 * r2 * iP, az2 * r2 * iP, Ix, Iy, Iz);
    Ix = 0.5 * kPi - Ix;
    Iy = 0.5 * kPi - Iy;
    Iz = 0.5 * kPi - Iz;
    const double iH = 1.0 / H;
    T sum = 0.0;
    // per axis c: a_c, 1 / a_c, u_c, 1 / (1 - u_c^2), atanh(u_c), I_1 of the edge lines at a_c; selected, not
    // indexed, so that nothing leaves the registers in the walls' loop
#define KIWI_PICK(c, x, y, z) ((c) == 0 ? (x) : ((c) == 1 ? (y) : (z)))
#pragma unroll 1
    for (int w = 0; w < 3; ++w) {
        // the wall at a_w with legs a_c1, a_c2 (the other two axes in ascending order)
        const int c1 = w == 0 ? 1 : 0, c2 = w == 2 ? 1 : 2;
        const T r0 = KIWI_PICK(w, ax, ay, az), ir0 = KIWI_PICK(w, iax, iay, iaz);
        const T q0 = r0 * iH;
        const int j = generic_region(K, lat_value(q0));
        const T a1 = KIWI_PICK(c1, ax, ay, az), a2 = KIWI_PICK(c2, ax, ay, az);
        const T ia1 = KIWI_PICK(c1, iax, iay, iaz), ia2 = KIWI_PICK(c2, iax, iay, iaz);
        const T rho = sqrt(KIWI_PICK(w, syz, sxz, sxy));
        T pa, pb;
        leg_angles(a1, ia1, a2, ia2, pa, pb);
#pragma unroll 1
        for (int v = 0; v < 2; ++v) {
            const auto rc = recs.rec(2 * w + v);
            const int packed = recs.packed(rc);
            const int nseg = packed & 7, k0 = packed >> 3;
            if (nseg == 0) continue;
            // vertex 0: R0 = a_c1 (the edge line at a_c1, along c2), t = a_c2; vertex 1 the reverse
            const int cR = v ? c2 : c1, cT = v ? c1 : c2;
            const T R0 = v ? a2 : a1, t = v ? a1 : a2, iR0 = v ? ia2 : ia1, phi = v ? pb : pa;
            const T a = R0 * ir0;
            int s = 0;
            while (s + 1 < nseg && lat_value(phi) > recs.phi_end(rc, s)) ++s;
            const T G = lattice_generic_G_pt(K, q0, j, k0 + s, a, a * a, phi, t * iR0, rho * iR0,
                                             KIWI_PICK(cT, ux, uy, uz), KIWI_PICK(cT, iomx, iomy, iomz),
                                             KIWI_PICK(cR, Ix, Iy, Iz), KIWI_PICK(cT, Kx, Ky, Kz));
            sum += (s > 0 ? recs.offset(rc, s) : T(0.0)) + G;
        }
    }
#undef KIWI_PICK
    return sum;
}

}  // namespace kiwi_b200
