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
#include "lattice_math.cuh"

namespace kiwi_b200 {

constexpr int kLatECap = 1536;   // edge-tier entries per chunk (one full 8^3 particle box needs 486)
constexpr int kLatSCap = 4096;   // corner values per chunk (one full 8^3 particle box needs 2187)

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

// Position of the smallest j with s_off[j] <= it among the chunk's np particles (s_off ascending).
static __device__ __forceinline__ int chunk_search(const int* s_off, int np, int it) {
    int lo = 0, hi = np - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (s_off[mid] <= it) lo = mid; else hi = mid - 1;
    }
    return lo;
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
