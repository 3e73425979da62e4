// Sites (Voronoi generators) on the device: which of them a Voro++ container over the domain keeps, in
// which of its blocks, and a uniform bin grid over the kept ones for nearest-site and neighbour searches.
//
// The container (built by the reference as pre_container -> guess_scaled_blocks -> setup,
// src/cartesian_map.cpp:66-80, src/point_set.cpp:268-283, src/mapping.cpp:228-240) keeps a site iff the
// pre_container accepts it (ax <= x <= bx on every axis, pre_container.cc:71-79) and its block index
// step_int((x - ax) * xsp) lies in [0, nx) (container.cc:174-192, xsp = 1 / ((bx - ax) / nx)): a site on an
// upper wall can fall out.  The block counts come from pre_container_base::guess_optimal
// (pre_container.cc:57-63: 5.6 sites per block for the domain-average density) scaled by the
// configuration's block_scale_factor (voro_grid.hpp), computed on the host with the same arithmetic.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>

#include "engine.hpp"
#include "prims.cuh"

namespace kiwi_b200 {

struct VoroBlocks {
    double ax, bx, ay, by, az, bz;
    double xsp, ysp, zsp;  // blocks per unit length
    int nx, ny, nz;
};

// The container's block grid for n_in sites inside the domain (inclusive bounds).
inline VoroBlocks voro_blocks(const double* b, int64_t n_in, double block_scale_factor) {
    VoroBlocks V;
    V.ax = b[0]; V.bx = b[1]; V.ay = b[2]; V.by = b[3]; V.az = b[4]; V.bz = b[5];
    const double dx = V.bx - V.ax, dy = V.by - V.ay, dz = V.bz - V.az;
    const double ilscale = std::pow((double)n_in / (5.6 * dx * dy * dz), 1 / 3.0);
    int nx = (int)(dx * ilscale + 1), ny = (int)(dy * ilscale + 1), nz = (int)(dz * ilscale + 1);
    if (block_scale_factor != 1.0) {
        nx = std::max(1, (int)std::round(nx * block_scale_factor));
        ny = std::max(1, (int)std::round(ny * block_scale_factor));
        nz = std::max(1, (int)std::round(nz * block_scale_factor));
    }
    V.nx = nx; V.ny = ny; V.nz = nz;
    V.xsp = 1 / (dx / nx);
    V.ysp = 1 / (dy / ny);
    V.zsp = 1 / (dz / nz);
    return V;
}

__host__ __device__ inline bool voro_inside(const VoroBlocks& V, double x, double y, double z) {
    return x >= V.ax && x <= V.bx && y >= V.ay && y <= V.by && z >= V.az && z <= V.bz;
}

__host__ __device__ inline int voro_step_int(double a) { return a < 0 ? (int)a - 1 : (int)a; }

// The container's block of a site, or -1 if the container does not keep it.
__host__ __device__ inline int64_t voro_block(const VoroBlocks& V, double x, double y, double z) {
    if (!voro_inside(V, x, y, z)) return -1;
    const int i = voro_step_int((x - V.ax) * V.xsp);
    if (i < 0 || i >= V.nx) return -1;
    const int j = voro_step_int((y - V.ay) * V.ysp);
    if (j < 0 || j >= V.ny) return -1;
    const int k = voro_step_int((z - V.az) * V.zsp);
    if (k < 0 || k >= V.nz) return -1;
    return i + (int64_t)V.nx * (j + (int64_t)V.ny * k);
}

// The block grid of the container for host site coordinates (3 per site): guess_optimal counts the sites
// the pre_container accepted.
inline VoroBlocks voro_blocks_for(const double* b, int64_t n, const double* xyz, double block_scale_factor) {
    VoroBlocks probe;
    probe.ax = b[0]; probe.bx = b[1]; probe.ay = b[2]; probe.by = b[3]; probe.az = b[4]; probe.bz = b[5];
    int64_t n_in = 0;
    for (int64_t i = 0; i < n; ++i) n_in += voro_inside(probe, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]) ? 1 : 0;
    return voro_blocks(b, n_in, block_scale_factor);
}

// A uniform grid of search bins over the domain (about one kept site per bin); a bin lists its sites in
// ascending site order.
struct SiteBins {
    double x0, y0, z0;     // domain minimum
    double wx, wy, wz;     // bin widths
    int nbx, nby, nbz;
    const int64_t* range;  // per bin [begin, end) in the sorted site arrays
    const double *sx, *sy, *sz;
    const int32_t* sidx;   // original site index
    double margin;         // safety margin of a search's stopping distance
};

__host__ __device__ inline int bin_of(double v, double v0, double w, int nb) {
    int b = (int)((v - v0) / w);
    return b < 0 ? 0 : (b >= nb ? nb - 1 : b);
}

// Search-bin key of each site the container keeps; the others get the key nbins, which sorts them past
// every bin.
static __global__ void k_site_keys(int64_t n, const double* __restrict__ xyz, VoroBlocks V, SiteBins B,
                                   uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
    uint32_t key = (uint32_t)B.nbx * B.nby * B.nbz;
    if (voro_block(V, x, y, z) >= 0) {
        const int bx = bin_of(x, B.x0, B.wx, B.nbx), by = bin_of(y, B.y0, B.wy, B.nby), bz = bin_of(z, B.z0, B.wz, B.nbz);
        key = (uint32_t)(((int64_t)bx * B.nby + by) * B.nbz + bz);
    }
    keys[i] = key;
    vals[i] = (uint32_t)i;
}

static __global__ void k_bin_ranges(const uint32_t* __restrict__ keys, int64_t n, uint32_t nbins,
                                    int64_t* __restrict__ range) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t k = keys[i];
    if (k >= nbins) return;
    if (i == 0 || keys[i - 1] != k) range[2 * (int64_t)k] = i;
    if (i == n - 1 || keys[i + 1] != k) range[2 * (int64_t)k + 1] = i + 1;
}

static __global__ void k_sorted_sites(int64_t n, const uint32_t* __restrict__ vals, const double* __restrict__ xyz,
                                      double* __restrict__ sx, double* __restrict__ sy, double* __restrict__ sz,
                                      int32_t* __restrict__ sidx) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t s = vals[i];
    sx[i] = xyz[3 * (int64_t)s];
    sy[i] = xyz[3 * (int64_t)s + 1];
    sz[i] = xyz[3 * (int64_t)s + 2];
    sidx[i] = (int32_t)s;
}

// The search-bin grid for about n_kept sites over the domain b.
inline void site_bins_shape(const double* b, int64_t n_kept, SiteBins& B) {
    const double ex = b[1] - b[0], ey = b[3] - b[2], ez = b[5] - b[4];
    const double w = std::cbrt(ex * ey * ez / std::max<double>((double)n_kept, 1.0));
    auto nb = [&](double e) { return (int)std::min<double>(std::max<double>(std::floor(e / w), 1.0), 1024.0); };
    B.nbx = nb(ex);
    B.nby = nb(ey);
    B.nbz = nb(ez);
    B.x0 = b[0];
    B.y0 = b[2];
    B.z0 = b[4];
    B.wx = ex / B.nbx;
    B.wy = ey / B.nby;
    B.wz = ez / B.nbz;
    B.margin = 1e-9 * std::max(B.wx, std::max(B.wy, B.wz));
}

// Bins the n sites at d_xyz (device, 3 per site) that the container V keeps: B's arrays point into the
// caller's scratch (sorted positions in d_sorted: 3 x max(n, 1) doubles; indices in d_sidx: n; ranges in
// d_range: 2 x nbins).  The kept sites come first in the sorted arrays, in bin order.
inline int build_site_bins(KiwiCtx* ctx, int64_t n, const double* d_xyz, const VoroBlocks& V, SiteBins& B,
                           double* d_sorted, int32_t* d_sidx, int64_t* d_range) {
    const int64_t nbins = (int64_t)B.nbx * B.nby * B.nbz;
    const int64_t ns = std::max<int64_t>(n, 1);
    uint32_t *k0, *v0, *k1, *v1;
    KIWI_TRY(scratch_t(ctx, S_KEYS0, (size_t)ns, &k0));
    KIWI_TRY(scratch_t(ctx, S_VALS0, (size_t)ns, &v0));
    KIWI_TRY(scratch_t(ctx, S_KEYS1, (size_t)ns, &k1));
    KIWI_TRY(scratch_t(ctx, S_VALS1, (size_t)ns, &v1));
    KIWI_CUDA(ctx, cudaMemsetAsync(d_range, 0, sizeof(int64_t) * 2 * nbins, ctx->stream));
    if (n > 0) {
        const unsigned g = (unsigned)((n + 255) / 256);
        k_site_keys<<<g, 256, 0, ctx->stream>>>(n, d_xyz, V, B, k0, v0);
        KIWI_LAUNCHED(ctx);
        int key_bits = 1;
        while ((1LL << key_bits) <= nbins) ++key_bits;
        bool second = false;
        KIWI_TRY(radix_sort_pairs(ctx, k0, v0, k1, v1, n, key_bits, &second));
        const uint32_t* sk = second ? k1 : k0;
        const uint32_t* sv = second ? v1 : v0;
        k_bin_ranges<<<g, 256, 0, ctx->stream>>>(sk, n, (uint32_t)nbins, d_range);
        KIWI_LAUNCHED(ctx);
        k_sorted_sites<<<g, 256, 0, ctx->stream>>>(n, sv, d_xyz, d_sorted, d_sorted + ns, d_sorted + 2 * ns, d_sidx);
        KIWI_LAUNCHED(ctx);
    }
    B.range = d_range;
    B.sx = d_sorted;
    B.sy = d_sorted + ns;
    B.sz = d_sorted + 2 * ns;
    B.sidx = d_sidx;
    return KIWI_OK;
}

}  // namespace kiwi_b200
