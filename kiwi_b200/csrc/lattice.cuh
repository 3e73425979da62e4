// Lattice-factorised cell integrals for box cells (cubic spline closed form).
//
// The reference evaluates each (particle, cell) pair as 6 faces x 4 edges x 2 vertex pyramids
// (src/kernel_integral.cpp:471-647, src/cartesian_grid.cpp:246-259).  For axis-aligned cells every one of
// those vertex pyramids is determined by three lattice distances: the wall distance r0 = |X_p - x0| of
// the face's plane, the in-plane distance R_0 = |Y_q - y0| from the particle's projection to the edge's
// line, and the offset t = |Z_r - z0| of the vertex along the edge.  So neighbouring cells share them,
// and a particle's whole box of cells needs only
//   - one edge tier (D2, D3: src/kernel_integral.cpp:253-350) per (plane, edge line): 6 (n+1)^2 for an
//     n^3 box, and
//   - one "corner" value per (plane, lattice point): S(p, q, r) = sgn(u) sgn(v) [I(r0, |u|, |v|) +
//     I(r0, |v|, |u|)], the cone mass of the rectangle spanned by the projection and the corner (two
//     right-triangle vertex pyramids, src/kernel_integral.cpp:356-400), u and v the corner's in-plane
//     offsets: 3 (n+1)^3;
// after which a cell is 24 signed lookups: its mass is sum over its 6 faces of (outward-normal side sign)
// x (inclusion-exclusion of S over the face's 4 corners).  This is algebraically the reference's sum --
// the same 48 vertex-pyramid terms with the same signs (a face's edge/foot-beyond rule of
// src/kernel_integral.cpp:613-631 is the 2-D inclusion-exclusion of a cumulative function) -- with
// every series written in its triangle's or edge's own lengths from a few reciprocals (lattice_edge,
// lattice_corner, lattice_pyramid) instead of acos(R_0/r12) followed by sincos and a division per ratio.
#pragma once

#include "cart_common.cuh"
#include "kiwi_math.cuh"

namespace kiwi_b200 {

constexpr int kLatPMax = 32;     // particles per chunk
constexpr int kLatECap = 1536;   // edge-tier entries per chunk (one full 8^3 particle box needs 486)
constexpr int kLatSCap = 4096;   // corner values per chunk (one full 8^3 particle box needs 2187)

// The edge and corner tiers are inlined into the lattice kernels by default (at 80 registers a call
// costs more in saved registers than the larger code does); define either as __noinline__ to keep it out
// of line.
#ifndef KIWI_EDGE_INLINE
#define KIWI_EDGE_INLINE __forceinline__
#endif
#ifndef KIWI_CORNER_INLINE
#define KIWI_CORNER_INLINE __forceinline__
#endif

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
static __device__ __forceinline__ LatticeWall<T> lattice_wall(T ih, T h, T ir0, T r0) {
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
static __device__ __forceinline__ T wall_b2_mid(const LatticeWall<T>& w) {
    return 0.25 * (-4. / 3. + w.r0h - 0.3 * w.r0h2 + 1. / 30. * w.r0h3 - 1. / 15. * w.r0h_3);
}
template <class T>
static __device__ __forceinline__ T wall_b2_in(const LatticeWall<T>& w) {
    return 0.25 * (-2. / 3. + 0.3 * w.r0h2 - 0.1 * w.r0h3 - 0.2 * w.r0h_2);
}
template <class T>
static __device__ __forceinline__ T wall_b1_in(const LatticeWall<T>& w) {
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
static __device__ KIWI_EDGE_INLINE LatticeEdgeT<T> lattice_edge(T h, T ih, T r0, T R_0) {
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
static __device__ __forceinline__ T lattice_pyramid(T h, T ih, T r0, T R_0, T t, T D2, T D3) {
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

// Face-walk evaluator of the plain FP64 Voronoi map (CubicEval's role): the edge tier in the edge's own
// lengths (lattice_edge) and each vertex pyramid from its triangle's lengths (lattice_pyramid); the face
// walk hands it the leg t along the edge instead of the angle (kLengths).
struct LenCubicEval {
    static constexpr bool kLengths = true;
    double h = 0.0, ih = 0.0, r0 = 0.0, R_0 = 0.0, D2 = 0.0, D3 = 0.0;
    __device__ void set_wall(double ar0) { r0 = ar0; }
    __device__ void set_edge(double R) {
        R_0 = R;
        D2 = D3 = 0.0;
        if (r0 != 0.0 && R != 0.0 && r0 * r0 + R * R <= 4.0 * (h * h)) {
            const LatticeEdge e = lattice_edge(h, ih, r0, R);
            D2 = e.D2;
            D3 = e.D3;
        }
    }
    __device__ double at_len(double t) const {
        return (r0 == 0.0 || R_0 == 0.0 || t == 0.0) ? 0.0 : lattice_pyramid(h, ih, r0, R_0, t, D2, D3);
    }
};

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
static __device__ KIWI_CORNER_INLINE T lattice_corner(T h, T ih, T r0, T a1, T a2, T D2a, T D3a, T D2b, T D3b) {
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
    if (a2 <= a1) {
        pa = atan(a2 * ia1);
        pb = 0.5 * kPi - pa;
    } else {
        pb = atan(a1 * ia2);
        pa = 0.5 * kPi - pb;
    }
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

// Position of the smallest j with s_off[j] <= it among the chunk's np particles (s_off ascending).
static __device__ __forceinline__ int chunk_search(const int* s_off, int np, int it) {
    int lo = 0, hi = np - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (s_off[mid] <= it) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// ---- generic kernels (table-driven tiers, src/kernel_integral_generic.cpp) in the lattice form
//
// The edge tier of a generic kernel is the list of the kernel's regions crossed along the edge line, with
// the angles where it leaves each region and the continuity offsets (generic_edge, :119-148).  Its lattice
// record packs that as 7 doubles: [0] = nseg + 8 x first region, [1..3] = phi_end of segments 0..2,
// [4..6] = offset of segments 1..3 (segment 0's is 0; the last segment ends at pi/2).
constexpr int kLatGenERec = 7;
constexpr int kLatGenECap = 640;  // edge records per chunk (a full 8^3 particle box needs 486)

// G_k(phi) = bphi_k phi + sum_i coef_k,i I_i(phi) for a wall at q0 = r0 / H in region j of the kernel
// (generic_G, src/kernel_integral_generic.cpp:82-92), a = R0 / r0, with sin(phi) and cos(phi) given.
// The wall coefficients A3 a_k,i q0^i are formed on the fly and each basis integral I_i (the recurrences
// of :19-66) is added as soon as it is formed, in ascending index order: every loop is unrolled over the
// table's fixed width and predicated on the region's lowest index, so the basis values, the sec-power
// integrals J_2l and the powers of q0 stay in registers.  q0^i is a compensated running product (hi + lo,
// the product's rounding error carried exactly by fma): the terms can cancel heavily, and a plain running
// product's rounding (up to ~i ulp) measurably raised the error of low-density cells; this is within an
// ulp, like pow, at a fraction of its cost; (1 - u^2)^-m in the K recurrence is formed the same way.
static __device__ __noinline__ double lattice_generic_G(const KiwiKernelTable* K, double q0, int j, int k, double a,
                                                        double a2, double phi, double sinp, double cosp) {
    const double* ak = K->a[k - 1];
    int imin = 1;
    for (int idx = KIWI_NI - 1; idx >= 0; --idx)
        if (ak[idx] != 0.0) {
            imin = 1 - idx;
            break;
        }
    const double A3 = K->A3_pi / kPi;
    double b = 0.0;
    if (k >= j)
        for (int p = KIWI_NB - 1; p >= 0; --p) b = b * q0 + K->B[j - 1][k - 1][p];
    double sum = (A3 * b) * phi;
    // u = a sin(phi) / sqrt(a^2 + cos^2(phi)), so u / a = sin(phi) / sqrt(...) and
    // 1 / (1 - u^2) = (a^2 + cos^2(phi)) / (cos^2(phi) (1 + a^2)): three reciprocals in all
    const double den = a2 + cosp * cosp, iden = 1.0 / den;
    const double ua = sinp * sqrt(iden), u = a * ua;
    const double iomu2 = den / (cosp * cosp * (1.0 + a2));
    const double sc = imin <= -2 ? 1.0 / cosp : 0.0, tn = sinp * sc;
    double ph = 1.0, pl = 0.0;  // q0^idx
    double wh = 1.0, wl = 0.0;  // (1 - u^2)^-m, compensated like q0^idx
    double Iodd = 0.0, Kc = 0.0, pow1a2 = 1.0, spow = 1.0;
    double J[(KIWI_NI + 1) / 2];  // J[l] = int_0^phi sec^(2l)
#pragma unroll
    for (int idx = 0; idx < KIWI_NI; ++idx) {
        if (1 - idx < imin) break;
        double Iv;
        if (idx == 0) {  // I_1 = atan(u / a)
            Iv = atan(ua);
            Iodd = Iv;
            Kc = atanh(u);
        } else if (idx == 1) {  // I_0 = phi
            Iv = phi;
        } else if ((idx & 1) == 0) {  // I_-(2m+1), m = idx / 2 - 1
            const int m = idx / 2 - 1;
            if (m > 0) {
                const double nw = wh * iomu2;
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
            double s = J[0], apow = 1.0, bc = 1.0;
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
        const double nh = ph * q0;
        pl = fma(pl, q0, fma(ph, q0, -nh));
        ph = nh;
    }
    return sum;
}

static __device__ __forceinline__ void lattice_generic_edge(const KiwiKernelTable* K, double H, double r0, double R0,
                                                           double* rec) {
    for (int i = 0; i < kLatGenERec; ++i) rec[i] = 0.0;
    if (r0 == 0.0 || R0 == 0.0) return;
    // the regions crossed along the edge line and the angles where it leaves them (generic_edge, :119-148)
    const double q0 = r0 / H, qR = R0 / H;
    const double a = R0 / r0, a2 = a * a;
    const int j = generic_region(K, q0);
    const int k0 = generic_region(K, sqrt(q0 * q0 + qR * qR));
    const int nseg = K->nreg - k0 + 1;
    rec[0] = (double)(nseg + 8 * k0);
    double off = 0.0;
    for (int s = 0; s + 1 < nseg; ++s) {
        const int k = k0 + s;
        const double c = K->c[k - 1];
        const double pb = acos(fmin(1.0, qR / sqrt(c * c - q0 * q0)));
        if (s < 3) rec[1 + s] = pb;
        const double sp = sin(pb), cp = cos(pb);
        off = off + lattice_generic_G(K, q0, j, k, a, a2, pb, sp, cp) - lattice_generic_G(K, q0, j, k + 1, a, a2, pb, sp, cp);
        if (s < 3) rec[4 + s] = off;
    }
}


// Vertex tier of a generic kernel for the right triangle with legs R0 (projection -> edge line) and t
// (along the edge) in a wall at distance r0 (generic_vertex, :150-156, at phi = atan2(t, R0)): the region
// segment holding phi, its offset, and G_k(phi).
// The two vertex tiers of a lattice corner (legs a1, a2 in the wall at r0; the edge records rec1 of the
// a1 line and rec2 of the a2 line: vertex 1 has R0 = a1, t = a2 and vertex 2 the reverse) share what the
// pair has in common: the distance sqrt(a1^2 + a2^2) and its reciprocal, 1 / r0, q0 = r0 / H and its
// kernel region, and the angle pair (the smaller one from atan2, the larger its complement, as in
// lattice_corner).  r0, a1, a2 > 0.
static __device__ __forceinline__ double lattice_generic_corner(const KiwiKernelTable* K, double H, double r0,
                                                               double a1, double a2, const double* rec1,
                                                               const double* rec2) {
    const double ir0 = 1.0 / r0, irr = 1.0 / sqrt(a1 * a1 + a2 * a2);
    const double q0 = r0 / H;
    const int j = generic_region(K, q0);
    double pa, pb;
    if (a2 <= a1) {
        pa = atan2(a2, a1);
        pb = 0.5 * kPi - pa;
    } else {
        pb = atan2(a1, a2);
        pa = 0.5 * kPi - pb;
    }
    double sum = 0.0;
#pragma unroll 1
    for (int v = 0; v < 2; ++v) {
        const double* rec = v ? rec2 : rec1;
        const int packed = (int)rec[0];
        const int nseg = packed & 7, k0 = packed >> 3;
        if (nseg == 0) continue;
        const double R0 = v ? a2 : a1, t = v ? a1 : a2, phi = v ? pb : pa;
        const double a = R0 * ir0;
        int s = 0;
        while (s + 1 < nseg && phi > rec[1 + s]) ++s;
        const double G = lattice_generic_G(K, q0, j, k0 + s, a, a * a, phi, t * irr, R0 * irr);
        sum += (s > 0 ? rec[3 + s] : 0.0) + G;
    }
    return sum;
}

// Bookkeeping shared by the lattice kernels (forward and adjoint).
// Half-width factor of the cells around a lattice point in the test for corners that no evaluated cell
// reads: the cells are padded by 1e-6 of a cell so that rounding never drops a corner a cell reads.
constexpr double kNeedPad = 1.0 + 1e-6;

// The chunk particle that owns item base + lane, for a warp whose 32 items start at base (a multiple of
// 32): off is this lane's particle's first item (lane < np; INT_MAX beyond).  Every particle owns at least
// one item, so the particles starting inside the window are distinct bits of one mask.  All 32 lanes call.
__device__ __forceinline__ int warp_owner(int base, int off, int lane) {
    const unsigned before = __ballot_sync(0xffffffffu, off <= base);
    const int d = off - base;
    const unsigned starts = __reduce_or_sync(0xffffffffu, (d > 0 && d < 32) ? 1u << d : 0u);
    return __popc(before) - 1 + __popc(starts & (0xffffffffu >> (31 - lane)));
}

// x / n for 0 <= x < 1400 and 1 <= n <= 81 as (x * magic(n)) >> 20 (exact over that range).
__host__ __device__ __forceinline__ uint32_t div_magic(int n) { return ((1u << 20) + (uint32_t)n - 1) / (uint32_t)n; }
__device__ __forceinline__ int div_by(int x, uint32_t m) { return (int)(((uint32_t)x * m) >> 20); }

// Offset of lattice plane P (global plane index) from the particle coordinate x0 along one axis.
__device__ __forceinline__ double lattice_offset(double mn, double d, int P, double x0) {
    return add_rn(mn, mul_rn((double)P, d)) - x0;
}

__device__ __forceinline__ double sgn(double v) { return (v > 0.0) ? 1.0 : ((v < 0.0) ? -1.0 : 0.0); }

}  // namespace kiwi_b200
