// The cartesian-map stage's point location (run_cartesian_map_stage, src/cartesian_map.cpp:84-200): each
// cell centre of a res^3 grid over the domain takes the mapping values of the Voronoi cell it lies in,
// i.e. of its nearest site (container::find_voronoi_cell, an exact nearest-site search), and that site's
// id.
//
// GPU form: the sites the reference's container keeps (sitebins.cuh) are binned into a uniform grid of
// about one site per bin (a stable radix sort by bin, so a bin lists its sites in ascending site order),
// and one thread per cell centre searches shells of bins around its own bin, nearest first, until no
// unsearched bin can hold a closer site.  Distances are (site - centre)^2 summed x, y, z, as the
// reference's search computes them.  Exact ties (equidistant sites) go to the smallest site index.  Built
// with --fmad=false, like the other FP64 units.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "engine.hpp"
#include "prims.cuh"
#include "sitebins.cuh"

using namespace kiwi_b200;

namespace {

__device__ __forceinline__ void scan_bin(const SiteBins& B, int64_t b, double x, double y, double z, double& best,
                                         int32_t& bi) {
    const int64_t e = B.range[2 * b + 1];
    for (int64_t k = B.range[2 * b]; k < e; ++k) {
        const double dx = B.sx[k] - x, dy = B.sy[k] - y, dz = B.sz[k] - z;
        const double d2 = dx * dx + dy * dy + dz * dz;
        const int32_t s = B.sidx[k];
        if (d2 < best || (d2 == best && s < bi)) {
            best = d2;
            bi = s;
        }
    }
}

// One thread per cell centre (iz fastest): nearest site by shells of bins, then the site's values.
__global__ void k_locate(int res, double xmin, double ymin, double zmin, double dpx, double dpy, double dpz,
                         SiteBins B, const int32_t* __restrict__ site_id, const double* __restrict__ cdens,
                         const double* __restrict__ cvx, const double* __restrict__ cvy, const double* __restrict__ cvz,
                         const uint8_t* __restrict__ mapped, double* __restrict__ dens, double* __restrict__ vx,
                         double* __restrict__ vy, double* __restrict__ vz, int32_t* __restrict__ cell_id,
                         unsigned long long* __restrict__ counts) {
    const int64_t n = (int64_t)res * res * res;
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long n_unres = 0, n_unmapped = 0;
    if (idx < n) {
        const int iz = (int)(idx % res), iy = (int)((idx / res) % res), ix = (int)(idx / ((int64_t)res * res));
        const double x = xmin + (ix + 0.5) * dpx, y = ymin + (iy + 0.5) * dpy, z = zmin + (iz + 0.5) * dpz;
        const int bx = bin_of(x, B.x0, B.wx, B.nbx), by = bin_of(y, B.y0, B.wy, B.nby), bz = bin_of(z, B.z0, B.wz, B.nbz);
        double best = INFINITY;
        int32_t bi = -1;
        const int rmax = max(max(B.nbx, B.nby), B.nbz);
        for (int r = 0; r <= rmax; ++r) {
            const int i0 = max(bx - r, 0), i1 = min(bx + r, B.nbx - 1);
            const int j0 = max(by - r, 0), j1 = min(by + r, B.nby - 1);
            const int k0 = max(bz - r, 0), k1 = min(bz + r, B.nbz - 1);
            for (int i = i0; i <= i1; ++i)
                for (int j = j0; j <= j1; ++j) {
                    const bool face = (i == bx - r || i == bx + r || j == by - r || j == by + r);
                    const int64_t row = ((int64_t)i * B.nby + j) * B.nbz;
                    if (face) {
                        for (int k = k0; k <= k1; ++k) scan_bin(B, row + k, x, y, z, best, bi);
                    } else {
                        if (bz - r >= 0) scan_bin(B, row + bz - r, x, y, z, best, bi);
                        if (r > 0 && bz + r < B.nbz) scan_bin(B, row + bz + r, x, y, z, best, bi);
                    }
                }
            // the searched cube [b - r, b + r] (clipped); every site outside it is at least dmin away
            if (i0 == 0 && j0 == 0 && k0 == 0 && i1 == B.nbx - 1 && j1 == B.nby - 1 && k1 == B.nbz - 1) break;
            double dmin = INFINITY;
            if (i0 > 0) dmin = fmin(dmin, x - (B.x0 + i0 * B.wx));
            if (i1 < B.nbx - 1) dmin = fmin(dmin, (B.x0 + (i1 + 1) * B.wx) - x);
            if (j0 > 0) dmin = fmin(dmin, y - (B.y0 + j0 * B.wy));
            if (j1 < B.nby - 1) dmin = fmin(dmin, (B.y0 + (j1 + 1) * B.wy) - y);
            if (k0 > 0) dmin = fmin(dmin, z - (B.z0 + k0 * B.wz));
            if (k1 < B.nbz - 1) dmin = fmin(dmin, (B.z0 + (k1 + 1) * B.wz) - z);
            // a margin of 1e-9 bin widths covers the rounding of the bin arithmetic (a site can land in
            // the neighbouring bin by ~1e-13 of a width); equal distances keep searching, for the tie rule
            dmin = fmax(dmin - B.margin, 0.0);
            if (bi >= 0 && best < dmin * dmin) break;
        }
        double d = 0.0, u = 0.0, v = 0.0, w = 0.0;
        int32_t id = 0;
        if (bi < 0) {
            n_unres = 1;
        } else {
            id = site_id ? site_id[bi] : bi;
            if (mapped && !mapped[bi]) {
                n_unmapped = 1;
            } else {
                d = cdens[bi];
                u = cvx[bi];
                v = cvy[bi];
                w = cvz[bi];
            }
        }
        dens[idx] = d;
        vx[idx] = u;
        vy[idx] = v;
        vz[idx] = w;
        cell_id[idx] = id;
    }
    for (int o = 16; o > 0; o >>= 1) {
        n_unres += __shfl_down_sync(0xffffffffu, n_unres, o);
        n_unmapped += __shfl_down_sync(0xffffffffu, n_unmapped, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (n_unres) atomicAdd(&counts[0], n_unres);
        if (n_unmapped) atomicAdd(&counts[1], n_unmapped);
    }
}

}  // namespace

extern "C" int kiwi_cartesian_map(KiwiCtx* ctx, int64_t n_sites, const double* site_xyz, const int32_t* site_id,
                                  const double* cell_density, const double* cell_vx, const double* cell_vy,
                                  const double* cell_vz, const uint8_t* mapped, const double* bounds6,
                                  int32_t resolution, double block_scale_factor, double* density, double* vx,
                                  double* vy, double* vz, int32_t* voronoi_cell_id, int64_t* counts2,
                                  KiwiStats* stats) {
    if (!ctx) return KIWI_ERR_ARG;
    KIWI_CUDA(ctx, cudaSetDevice(ctx->device));
    if (resolution <= 0) return set_err(ctx, KIWI_ERR_ARG, "cartesian_map.resolution must be > 0");
    if (!bounds6 || !(bounds6[0] < bounds6[1]) || !(bounds6[2] < bounds6[3]) || !(bounds6[4] < bounds6[5]))
        return set_err(ctx, KIWI_ERR_ARG, "domain bounds must satisfy min < max on every axis");
    if (n_sites < 0 || (n_sites > 0 && (!site_xyz || !cell_density || !cell_vx || !cell_vy || !cell_vz)))
        return set_err(ctx, KIWI_ERR_ARG, "bad site arrays");
    if (n_sites >= (1LL << 31)) return set_err(ctx, KIWI_ERR_ARG, "too many sites");
    if (block_scale_factor == 0.0) block_scale_factor = 3.0;  // GridBlocks' default
    if (!(block_scale_factor > 0.0)) return set_err(ctx, KIWI_ERR_ARG, "grid_blocks.block_scale_factor must be > 0");
    const int64_t nq = (int64_t)resolution * resolution * resolution;
    if (!density || !vx || !vy || !vz || !voronoi_cell_id) return set_err(ctx, KIWI_ERR_ARG, "null output");
    const int64_t launches0 = ctx->launches;
    const double xmin = bounds6[0], ymin = bounds6[2], zmin = bounds6[4];
    const double ex = bounds6[1] - xmin, ey = bounds6[3] - ymin, ez = bounds6[5] - zmin;
    const VoroBlocks V = voro_blocks_for(bounds6, n_sites, site_xyz, block_scale_factor);
    SiteBins B;
    site_bins_shape(bounds6, n_sites, B);
    const int64_t nbins = (int64_t)B.nbx * B.nby * B.nbz;

    // stage the sites and their values
    const int64_t ns = std::max<int64_t>(n_sites, 1);
    double* d = nullptr;    // xyz (3), values (4), sorted xyz (3)
    int32_t* di = nullptr;  // site ids, sorted index
    uint8_t* dm = nullptr;
    KIWI_TRY(scratch_t(ctx, S_PART, (size_t)(10 * ns), &d));
    KIWI_TRY(scratch_t(ctx, S_VOR_HOME, (size_t)(2 * ns), &di));
    KIWI_TRY(scratch_t(ctx, S_MISC2, (size_t)ns, &dm));
    int64_t* range = nullptr;
    KIWI_TRY(scratch_t(ctx, S_TILE_RANGE, (size_t)(2 * nbins), &range));
    double* dout = nullptr;
    int32_t* dcid = nullptr;
    unsigned long long* dcount = nullptr;
    KIWI_TRY(scratch_t(ctx, S_OUT, (size_t)(4 * nq), &dout));
    KIWI_TRY(scratch_t(ctx, S_COUNT, (size_t)nq, &dcid));
    KIWI_TRY(scratch_t(ctx, S_STATS, 2, &dcount));
    KIWI_CUDA(ctx, cudaEventRecord(ctx->ev[2], ctx->stream));
    const size_t b = sizeof(double) * (size_t)n_sites;
    if (n_sites > 0) {
        KIWI_CUDA(ctx, cudaMemcpyAsync(d, site_xyz, 3 * b, cudaMemcpyHostToDevice, ctx->stream));
        KIWI_CUDA(ctx, cudaMemcpyAsync(d + 3 * ns, cell_density, b, cudaMemcpyHostToDevice, ctx->stream));
        KIWI_CUDA(ctx, cudaMemcpyAsync(d + 4 * ns, cell_vx, b, cudaMemcpyHostToDevice, ctx->stream));
        KIWI_CUDA(ctx, cudaMemcpyAsync(d + 5 * ns, cell_vy, b, cudaMemcpyHostToDevice, ctx->stream));
        KIWI_CUDA(ctx, cudaMemcpyAsync(d + 6 * ns, cell_vz, b, cudaMemcpyHostToDevice, ctx->stream));
        if (site_id)
            KIWI_CUDA(ctx, cudaMemcpyAsync(di, site_id, sizeof(int32_t) * n_sites, cudaMemcpyHostToDevice, ctx->stream));
        if (mapped) KIWI_CUDA(ctx, cudaMemcpyAsync(dm, mapped, (size_t)n_sites, cudaMemcpyHostToDevice, ctx->stream));
    }
    KIWI_CUDA(ctx, cudaMemsetAsync(dcount, 0, 2 * sizeof(unsigned long long), ctx->stream));
    KIWI_CUDA(ctx, cudaEventRecord(ctx->ev[0], ctx->stream));
    KIWI_TRY(build_site_bins(ctx, n_sites, d, V, B, d + 7 * ns, di + ns, range));
    const double dpx = ex / resolution, dpy = ey / resolution, dpz = ez / resolution;
    k_locate<<<(unsigned)((nq + 255) / 256), 256, 0, ctx->stream>>>(
        resolution, xmin, ymin, zmin, dpx, dpy, dpz, B, site_id ? di : nullptr, d + 3 * ns, d + 4 * ns, d + 5 * ns,
        d + 6 * ns, mapped ? dm : nullptr, dout, dout + nq, dout + 2 * nq, dout + 3 * nq, dcid, dcount);
    KIWI_LAUNCHED(ctx);
    KIWI_CUDA(ctx, cudaEventRecord(ctx->ev[1], ctx->stream));
    const size_t bq = sizeof(double) * (size_t)nq;
    KIWI_CUDA(ctx, cudaMemcpyAsync(density, dout, bq, cudaMemcpyDeviceToHost, ctx->stream));
    KIWI_CUDA(ctx, cudaMemcpyAsync(vx, dout + nq, bq, cudaMemcpyDeviceToHost, ctx->stream));
    KIWI_CUDA(ctx, cudaMemcpyAsync(vy, dout + 2 * nq, bq, cudaMemcpyDeviceToHost, ctx->stream));
    KIWI_CUDA(ctx, cudaMemcpyAsync(vz, dout + 3 * nq, bq, cudaMemcpyDeviceToHost, ctx->stream));
    KIWI_CUDA(ctx, cudaMemcpyAsync(voronoi_cell_id, dcid, sizeof(int32_t) * nq, cudaMemcpyDeviceToHost, ctx->stream));
    unsigned long long hc[2] = {0, 0};
    KIWI_CUDA(ctx, cudaMemcpyAsync(hc, dcount, sizeof hc, cudaMemcpyDeviceToHost, ctx->stream));
    KIWI_CUDA(ctx, cudaEventRecord(ctx->ev[3], ctx->stream));
    KIWI_CUDA(ctx, cudaEventSynchronize(ctx->ev[3]));
    if (counts2) {
        counts2[0] = (int64_t)hc[0];
        counts2[1] = (int64_t)hc[1];
    }
    if (stats) {
        *stats = KiwiStats{};
        float ms = 0.f, tot = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
        cudaEventElapsedTime(&tot, ctx->ev[2], ctx->ev[3]);
        stats->gather_ms = ms;
        stats->total_ms = tot;
        stats->evaluated_pairs = nq;
        stats->skipped_outside = (int64_t)hc[0];
        stats->launches = ctx->launches - launches0;
    }
    return KIWI_OK;
}
