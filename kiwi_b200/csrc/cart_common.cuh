// Cartesian-grid geometry shared by the binning step and every cell-integral kernel.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace kiwi_b200 {

// Cell tiles: one CTA of the gather kernels owns one TX x TY x TZ block of cells (z fastest, as the
// output layout (ix*ny + iy)*nz + iz).
constexpr int kTileX = 8, kTileY = 8, kTileZ = 8;
constexpr int kTileCells = kTileX * kTileY * kTileZ;

struct CartGeom {
    double x_min, y_min, z_min;
    double dpx, dpy, dpz;  // cell sizes, (max - min) / n as src/cartesian_grid.cpp:95-97
    double hpx, hpy, hpz;  // half sizes, 0.5 * d as src/cartesian_grid.cpp:160
    double cell_volume;    // dpx * dpy * dpz (src/cartesian_grid.cpp:161)
    int nx, ny, nz;
    int ntx, nty, ntz;     // tiles per axis
    double support_in_h;
};

struct CellBox {
    int x0, x1, y0, y1, z0, z1;  // inclusive cell index ranges, clamped to the grid
};

// Round-to-nearest multiply and add that are never contracted into an FMA, whatever the translation
// unit's --fmad setting: the bounding boxes and cell centres must come out exactly as the reference's
// x86-64 build computes them, in every arithmetic form.
__host__ __device__ __forceinline__ double mul_rn(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}
__host__ __device__ __forceinline__ double add_rn(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}

__host__ __device__ __forceinline__ int floor_to_int(double v) {
    // floor() then int conversion as src/cartesian_grid.cpp:220-225; the double is bounded first so
    // that the conversion stays defined for particles arbitrarily far outside the domain.
    v = floor(v);
    v = v < -2.0e9 ? -2.0e9 : (v > 2.0e9 ? 2.0e9 : v);
    return (int)v;
}

// The clamped bounding box of a particle's support in cell indices (src/cartesian_grid.cpp:211-237).
// Returns false if the particle contributes nothing (h <= 0, or its box misses the grid).
__host__ __device__ __forceinline__ bool particle_cell_box(const CartGeom& g, double x0, double y0, double z0,
                                                           double h, CellBox& b, bool* outside) {
    *outside = false;
    if (!(h > 0.0)) return false;
    const double radius = mul_rn(g.support_in_h, h);
    b.x0 = floor_to_int((x0 - radius - g.x_min) / g.dpx);
    b.x1 = floor_to_int((x0 + radius - g.x_min) / g.dpx);
    b.y0 = floor_to_int((y0 - radius - g.y_min) / g.dpy);
    b.y1 = floor_to_int((y0 + radius - g.y_min) / g.dpy);
    b.z0 = floor_to_int((z0 - radius - g.z_min) / g.dpz);
    b.z1 = floor_to_int((z0 + radius - g.z_min) / g.dpz);
    b.x0 = b.x0 > 0 ? b.x0 : 0;
    b.x1 = b.x1 < g.nx - 1 ? b.x1 : g.nx - 1;
    b.y0 = b.y0 > 0 ? b.y0 : 0;
    b.y1 = b.y1 < g.ny - 1 ? b.y1 : g.ny - 1;
    b.z0 = b.z0 > 0 ? b.z0 : 0;
    b.z1 = b.z1 < g.nz - 1 ? b.z1 : g.nz - 1;
    if (b.x0 > b.x1 || b.y0 > b.y1 || b.z0 > b.z1) {
        *outside = true;
        return false;
    }
    return true;
}

// Cell centre as src/cartesian_grid.cpp:240-244 computes it.
__host__ __device__ __forceinline__ double cell_centre(double mn, int i, double d) { return add_rn(mn, mul_rn(i + 0.5, d)); }

// Device counters of one call (int64, summed with integer atomics: order-independent).
struct DevStats {
    unsigned long long bbox_pairs, sphere_pairs, evaluated_pairs, skipped_outside, neg_clamped, neg_warned,
        fp64_fallback, tile_pairs, limit_hit;
    // work items of the lattice-factorised evaluation: edge tiers whose edge line lies outside 2h,
    // between h and 2h, within h of the particle; vertex pyramids evaluated
    unsigned long long edge_outer, edge_middle, edge_inner, vertex_pyramids;
    unsigned long long table_clamps;  // tabulated integral: lookup indices clamped into the table
};

}  // namespace kiwi_b200
