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
// the vertex angle taken from the right triangle directly (phi = atan2(t, R_0), sin and cos from t, R_0
// and their hypotenuse) instead of acos(R_0/r12) followed by sincos.
#pragma once

#include "cart_common.cuh"
#include "kiwi_math.cuh"

namespace kiwi_b200 {

constexpr int kLatPMax = 32;     // particles per chunk
constexpr int kLatECap = 1536;   // edge-tier entries per chunk (one full 8^3 particle box needs 486)
constexpr int kLatSCap = 4096;   // corner values per chunk (one full 8^3 particle box needs 2187)

// Vertex-pyramid mass of the right triangle with legs R_0 (projection -> edge line) and t (along the
// edge) in a wall at distance r0: the vertex tier of src/kernel_integral.cpp:356-400 at phi = atan2(t, R_0)
// (beyond 2h only I0 and I1 are needed, as in cubic_vertex).
// Written over the real type T: double here, Dual4 (dual.cuh) for the adjoint.
template <class T>
static __device__ __noinline__ T lattice_vertex_t(T h, T r0, T R_0, T t, T D2, T D3) {
    if (r0 == 0.0 || R_0 == 0.0 || t == 0.0) return T(0.0);
    const CubicWallT<T> w = cubic_wall_t<T>(h, r0);
    const T a = R_0 / r0;
    const T a2 = a * a;
    const T s2 = R_0 * R_0 + t * t;
    const T rr = sqrt(s2);
    const T phi = atan2(t, R_0);
    const T sinp = t / rr, cosp = R_0 / rr;
    const T r2 = r0 * r0 + s2;
    const T r03 = w.r03, r0h2 = w.r0h2, r0h3 = w.r0h3, r0h_3 = w.r0h_3;
    if (!(r2 < 4.0 * w.h2)) {
        const T I1 = phi_I1<T>(sinp, cosp, a, a2);
        return r0h3 / kPi * (-0.25 * r0h_3 * I1 + w.B3 / r03 * phi + D3);
    }
    const PhiSeriesT<T> s = phi_series_sc<T>(phi, sinp, cosp, a, a2);
    T full_int;
    if (r2 < w.h2) {
        full_int = r0h3 / kPi * (1. / 6. * s.I_2 - 3. / 40. * r0h2 * s.I_4 + 1. / 40. * r0h3 * s.I_5 + w.B1 / r03 * s.I0);
    } else if (r2 < 4.0 * w.h2) {
        full_int = r0h3 / kPi * (0.25 * (4. / 3. * s.I_2 - (r0 / h) * s.I_3 + 0.3 * r0h2 * s.I_4 - 1. / 30. * r0h3 * s.I_5 + 1. / 15. * r0h_3 * s.I1) + w.B2 / r03 * s.I0 + D2);
    } else {
        full_int = r0h3 / kPi * (-0.25 * r0h_3 * s.I1 + w.B3 / r03 * s.I0 + D3);
    }
    return full_int;
}
static __device__ __forceinline__ double lattice_vertex(double h, double r0, double R_0, double t, double D2, double D3) {
    return lattice_vertex_t<double>(h, r0, R_0, t, D2, D3);
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

static __device__ __forceinline__ void lattice_generic_edge(const KiwiKernelTable* K, double H, double r0, double R0,
                                                           double* rec) {
    for (int i = 0; i < kLatGenERec; ++i) rec[i] = 0.0;
    if (r0 == 0.0 || R0 == 0.0) return;
    GenericWall w;
    GenericEdge e;
    generic_wall(w, K, H, r0);
    generic_edge(e, w, R0);
    rec[0] = (double)(e.nseg + 8 * e.region[0]);
    for (int s = 0; s + 1 < e.nseg && s < 3; ++s) rec[1 + s] = e.phi_end[s];
    for (int s = 1; s < e.nseg && s < 4; ++s) rec[3 + s] = e.offset[s];
}

// Vertex tier of a generic kernel for the right triangle with legs R0 (projection -> edge line) and t
// (along the edge) in a wall at distance r0 (generic_vertex, :150-156, at phi = atan2(t, R0)): the region
// segment holding phi, its offset, and G_k(phi) = bphi_k phi + sum_i coef_k,i I_i(phi) with the wall
// coefficients A3 a_k,i (r0/H)^i formed on the fly.
static __device__ __noinline__ double lattice_generic_vertex(const KiwiKernelTable* K, double H, double r0, double R0,
                                                            double t, const double* rec) {
    const int packed = (int)rec[0];
    const int nseg = packed & 7, k0 = packed >> 3;
    if (nseg == 0 || t == 0.0) return 0.0;
    const double a = R0 / r0, a2 = a * a;
    const double rr = sqrt(R0 * R0 + t * t);
    const double phi = atan2(t, R0);
    const double sinp = t / rr, cosp = R0 / rr;
    int s = 0;
    while (s + 1 < nseg && phi > rec[1 + s]) ++s;
    const int k = k0 + s;
    const double q0 = r0 / H;
    const int j = generic_region(K, q0);
    int imin = 1;
    for (int idx = KIWI_NI - 1; idx >= 0; --idx)
        if (K->a[k - 1][idx] != 0.0) {
            imin = 1 - idx;
            break;
        }
    double I[KIWI_NI];
    generic_basis_sc(a, a2, phi, sinp, cosp, imin, I);
    const double A3 = K->A3_pi / kPi;
    double b = 0.0;
    if (k >= j)
        for (int p = KIWI_NB - 1; p >= 0; --p) b = b * q0 + K->B[j - 1][k - 1][p];
    double sum = (A3 * b) * phi;
    // q0^idx as a compensated running product (hi + lo, the product's rounding error carried exactly by
    // fma): the terms can cancel heavily, and a plain running product's rounding (up to ~idx ulp)
    // measurably raised the error of low-density cells; this is within an ulp, like pow, at a fraction
    // of its cost
    double ph = 1.0, pl = 0.0;
    for (int idx = 0; idx < KIWI_NI; ++idx) {
        const double c = K->a[k - 1][idx];
        if (c != 0.0) sum += (A3 * c * (ph + pl)) * I[idx];
        const double nh = ph * q0;
        pl = fma(pl, q0, fma(ph, q0, -nh));
        ph = nh;
    }
    return (s > 0 ? rec[3 + s] : 0.0) + sum;
}

// Offset of lattice plane P (global plane index) from the particle coordinate x0 along one axis.
__device__ __forceinline__ double lattice_offset(double mn, double d, int P, double x0) {
    return add_rn(mn, mul_rn((double)P, d)) - x0;
}

__device__ __forceinline__ double sgn(double v) { return (v > 0.0) ? 1.0 : ((v < 0.0) ? -1.0 : 0.0); }

}  // namespace kiwi_b200
