// Plain (all-FP64) form: the cell-integral gather over Cartesian cell tiles, the batched scalar
// integral API and the mean-velocity reduction.  Built with --fmad=false so that every product and sum
// rounds exactly as in the reference's x86-64 build (see kiwi_math.cuh).
#include <cuda_runtime.h>

#include <climits>

#include "engine.hpp"
#include "kiwi_math.cuh"
#include "lattice.cuh"
#include "tabulated.cuh"

namespace kiwi_b200 {

__constant__ KiwiKernelTable c_tables[KIWI_NUM_KERNELS];

int fp64_init_tables(KiwiCtx* ctx) {
    KIWI_CUDA(ctx, cudaMemcpyToSymbol(c_tables, kiwi_kernel_tables, sizeof(kiwi_kernel_tables)));
    KIWI_TRY(lattice_init_tables(ctx));
    return adjoint_init_tables(ctx);
}

}  // namespace kiwi_b200

#include "lattice_tile.cuh"

namespace kiwi_b200 {

namespace {

constexpr int kThreads = 256;
#ifndef KIWI_GATHER_MIN_BLOCKS
#define KIWI_GATHER_MIN_BLOCKS 2
#endif
constexpr int kMinBlocks = KIWI_GATHER_MIN_BLOCKS;  // resident CTAs per SM the register budget is sized for
constexpr int kPMax = 32;      // particles per chunk (one warp builds a chunk)
constexpr int kChunkCap = 2048; // (particle, cell) pairs per chunk; >= kTileCells so one particle always fits
static_assert(kChunkCap >= kTileCells, "a single particle's tile box must fit in one chunk");
constexpr int kCellsPerThread = kTileCells / kThreads;
static_assert(kTileCells % kThreads == 0, "tile cells must split evenly over the threads");

template <bool CUBIC>
__device__ __forceinline__ double pair_msum(int kernel, double x0, double y0, double z0, double h, double support,
                                            double cx, double cy, double cz, double hx, double hy, double hz) {
    if (CUBIC) {
        CubicEval ev;
        ev.h = h;
        return box_cell_msum(x0, y0, z0, support, cx, cy, cz, hx, hy, hz, ev);
    } else {
        GenericEval ev;
        ev.K = &c_tables[kernel];
        ev.H = support;
        return box_cell_msum(x0, y0, z0, support, cx, cy, cz, hx, hy, hz, ev);
    }
}

__device__ __forceinline__ void add_stat(unsigned long long* dst, unsigned long long v) {
    // warp-aggregate, then one atomic per warp
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(dst, v);
}

// One CTA = one tile of kTileX x kTileY x kTileZ cells.  The tile's particle list (ascending particle
// index) is walked in chunks of up to kPMax particles / kChunkCap pairs: all threads evaluate the
// chunk's (particle, cell) pairs into shared memory, then each thread adds, for the cells it owns, the
// chunk's values in particle order.  So every cell's sum runs over its particles in ascending order --
// the summation order of the reference's single-threaded loop -- with no atomics.
// Chunk pair k -> (chunk particle j, global cell ix, iy, iz): j is the last particle whose pair range
// starts at or before k; the cell runs z fastest within the particle's box inside the tile.
__device__ __forceinline__ void decode_pair(int k, int np, const int* s_start, const int (*s_lo)[3],
                                            const int (*s_dim)[3], int bx, int by, int bz, int& j, int& ix, int& iy,
                                            int& iz) {
    int lo = 0, hi = np - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (s_start[mid] <= k) lo = mid; else hi = mid - 1;
    }
    j = lo;
    const int q = k - s_start[j];
    const int dz = s_dim[j][2], dy = s_dim[j][1];
    const int qz = q % dz, qr = q / dz, qy = qr % dy, qx = qr / dy;
    ix = bx + s_lo[j][0] + qx;
    iy = by + s_lo[j][1] + qy;
    iz = bz + s_lo[j][2] + qz;
}

// The work of one CTA on one cell tile: t is the tile's index in its grid (its cell coordinates), t_range
// its entry in range[] (the same unless the tile lists of several grids are concatenated).  EV selects the
// pair integral: kEvGeneric, kEvCubic (closed form) or kEvTab (lookups in `tab`).  With RUNTIME_CUBIC the
// closed form is chosen by cubic_rt instead of EV (one instance serves both, so a kernel that needs both
// keeps one copy of the tile's shared memory).
constexpr int kEvGeneric = 0, kEvCubic = 1, kEvTab = 2;
template <int EV, bool CULL, bool RUNTIME_CUBIC = false>
__device__ __forceinline__ void gather_tile(const CartGeom& g, const DevParticles& P, int kernel,
                                            const uint32_t* __restrict__ list, const int64_t* __restrict__ range,
                                            int64_t t_range, int64_t t, const CartOutputs& out,
                                            DevStats* __restrict__ st, bool cubic_rt = false,
                                            const TabDev tab = TabDev{}) {
    static_assert(kChunkCap / kThreads <= 32, "per-thread keep mask is 32 bits");
    __shared__ double s_x[kPMax], s_y[kPMax], s_z[kPMax], s_h[kPMax], s_m[kPMax], s_vx[kPMax], s_vy[kPMax],
        s_vz[kPMax];
    __shared__ int s_lo[kPMax][3], s_dim[kPMax][3], s_start[kPMax];
    __shared__ int s_np, s_total;
    __shared__ int s_wsum[kThreads / 32];
    __shared__ unsigned short s_list[kChunkCap];
    __shared__ double s_R[kChunkCap];

    const int tz = (int)(t % g.ntz), ty = (int)((t / g.ntz) % g.nty), tx = (int)(t / ((int64_t)g.ntz * g.nty));
    const int bx = tx * kTileX, by = ty * kTileY, bz = tz * kTileZ;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    double acc[kCellsPerThread][4];
#pragma unroll
    for (int c = 0; c < kCellsPerThread; ++c) acc[c][0] = acc[c][1] = acc[c][2] = acc[c][3] = 0.0;

    unsigned long long n_bbox = 0, n_sphere = 0, n_eval = 0, n_neg = 0, n_warn = 0;
    unsigned n_clamp = 0;
    const int64_t beg = range[2 * t_range], end = range[2 * t_range + 1];
    const double sup_in_h = g.support_in_h;

    for (int64_t pos = beg; pos < end;) {
        if (warp == 0) {
            const int64_t idx = pos + lane;
            int size = 0, lo0 = 0, lo1 = 0, lo2 = 0, d0 = 0, d1 = 0, d2 = 0;
            double px = 0, py = 0, pz = 0, ph = 0, pm = 0, pvx = 0, pvy = 0, pvz = 0;
            if (idx < end) {
                const uint32_t p = list[idx];
                px = P.x[p]; py = P.y[p]; pz = P.z[p]; ph = P.h[p];
                pm = P.m[p]; pvx = P.vx[p]; pvy = P.vy[p]; pvz = P.vz[p];
                CellBox b;
                bool outside;
                particle_cell_box(g, px, py, pz, ph, b, &outside);
                const int x0 = max(b.x0, bx), x1 = min(b.x1, bx + kTileX - 1);
                const int y0 = max(b.y0, by), y1 = min(b.y1, by + kTileY - 1);
                const int z0 = max(b.z0, bz), z1 = min(b.z1, bz + kTileZ - 1);
                lo0 = x0 - bx; lo1 = y0 - by; lo2 = z0 - bz;
                d0 = x1 - x0 + 1; d1 = y1 - y0 + 1; d2 = z1 - z0 + 1;
                size = (d0 > 0 && d1 > 0 && d2 > 0) ? d0 * d1 * d2 : 0;
            }
            int incl = size;
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += v;
            }
            const bool take = (idx < end) && incl <= kChunkCap;
            const unsigned tm = __ballot_sync(0xffffffffu, take);
            const int np = __popc(tm);
            if (take) {
                s_x[lane] = px; s_y[lane] = py; s_z[lane] = pz; s_h[lane] = ph;
                s_m[lane] = pm; s_vx[lane] = pvx; s_vy[lane] = pvy; s_vz[lane] = pvz;
                s_lo[lane][0] = lo0; s_lo[lane][1] = lo1; s_lo[lane][2] = lo2;
                s_dim[lane][0] = d0; s_dim[lane][1] = d1; s_dim[lane][2] = d2;
                s_start[lane] = incl - size;
            }
            if (lane == np - 1) {
                s_np = np;
                s_total = incl;
            }
        }
        __syncthreads();
        const int np = s_np, total = s_total;

        // Pass 1: which of the chunk's box pairs are evaluated.  With culling, only cells whose closest
        // point lies within the support radius (the cells that can hold mass; the reference's other
        // bounding-box cells evaluate to rounding noise around zero); the rest get 0.
        unsigned keep = 0;
#pragma unroll
        for (int i = 0; i < kChunkCap / kThreads; ++i) {
            const int k = threadIdx.x + i * kThreads;
            if (k >= total) break;
            int j, ix, iy, iz;
            decode_pair(k, np, s_start, s_lo, s_dim, bx, by, bz, j, ix, iy, iz);
            const double radius = mul_rn(sup_in_h, s_h[j]);
            const double ex = fmax(fabs(s_x[j] - cell_centre(g.x_min, ix, g.dpx)) - g.hpx, 0.0);
            const double ey = fmax(fabs(s_y[j] - cell_centre(g.y_min, iy, g.dpy)) - g.hpy, 0.0);
            const double ez = fmax(fabs(s_z[j] - cell_centre(g.z_min, iz, g.dpz)) - g.hpz, 0.0);
            const bool in = ex * ex + ey * ey + ez * ez < radius * radius;
            ++n_bbox;
            n_sphere += in;
            if (!CULL || in) keep |= 1u << i;
            else s_R[k] = 0.0;
        }
        // compact the kept pairs into s_list (block-wide exclusive scan of the per-thread counts)
        const int nkeep = __popc(keep);
        int incl = nkeep;
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        if (lane == 31) s_wsum[warp] = incl;
        __syncthreads();
        int base = incl - nkeep;
        for (int w = 0; w < warp; ++w) base += s_wsum[w];
        int m_total = 0;
        for (int w = 0; w < kThreads / 32; ++w) m_total += s_wsum[w];
#pragma unroll
        for (int i = 0; i < kChunkCap / kThreads; ++i)
            if (keep & (1u << i)) s_list[base++] = (unsigned short)(threadIdx.x + i * kThreads);
        __syncthreads();

        // Pass 2: the cell integrals of the kept pairs.
        for (int li = threadIdx.x; li < m_total; li += kThreads) {
            const int k = s_list[li];
            int j, ix, iy, iz;
            decode_pair(k, np, s_start, s_lo, s_dim, bx, by, bz, j, ix, iy, iz);
            const double x0 = s_x[j], y0 = s_y[j], z0 = s_z[j], h = s_h[j];
            const double radius = mul_rn(sup_in_h, h);
            const double cx = cell_centre(g.x_min, ix, g.dpx);
            const double cy = cell_centre(g.y_min, iy, g.dpy);
            const double cz = cell_centre(g.z_min, iz, g.dpz);
            ++n_eval;
            double msum;
            if (EV == kEvTab) {
                TabEval ev{tab, h, 0.0, 0.0, &n_clamp};
                msum = box_cell_msum(x0, y0, z0, 2 * h, cx, cy, cz, g.hpx, g.hpy, g.hpz, ev);
            } else if (RUNTIME_CUBIC ? cubic_rt : EV == kEvCubic)
                msum = pair_msum<true>(kernel, x0, y0, z0, h, 2 * h, cx, cy, cz, g.hpx, g.hpy, g.hpz);
            else
                msum = pair_msum<false>(kernel, x0, y0, z0, h, radius, cx, cy, cz, g.hpx, g.hpy, g.hpz);
            if (msum < 0.0) {
                ++n_neg;
                if (msum <= -0.01) ++n_warn;
                msum = 0.0;
            }
            s_R[k] = msum;
        }
        __syncthreads();

#pragma unroll
        for (int c = 0; c < kCellsPerThread; ++c) {
            const int li = threadIdx.x + c * kThreads;
            const int lz = li % kTileZ, ly = (li / kTileZ) % kTileY, lx = li / (kTileZ * kTileY);
            for (int j = 0; j < np; ++j) {
                const int ox = lx - s_lo[j][0], oy = ly - s_lo[j][1], oz = lz - s_lo[j][2];
                if (ox < 0 || oy < 0 || oz < 0 || ox >= s_dim[j][0] || oy >= s_dim[j][1] || oz >= s_dim[j][2]) continue;
                const double msum = s_R[s_start[j] + (ox * s_dim[j][1] + oy) * s_dim[j][2] + oz];
                if (msum == 0.0) continue;
                const double mm = msum * s_m[j];
                acc[c][0] += mm;
                acc[c][1] += mm * s_vx[j];
                acc[c][2] += mm * s_vy[j];
                acc[c][3] += mm * s_vz[j];
            }
        }
        __syncthreads();
        pos += np;
    }

    const double mvx = out.meanv[0], mvy = out.meanv[1], mvz = out.meanv[2];
    const int64_t ncell = (int64_t)g.nx * g.ny * g.nz;
#pragma unroll
    for (int c = 0; c < kCellsPerThread; ++c) {
        const int li = threadIdx.x + c * kThreads;
        const int lz = li % kTileZ, ly = (li / kTileZ) % kTileY, lx = li / (kTileZ * kTileY);
        const int ix = bx + lx, iy = by + ly, iz = bz + lz;
        if (ix >= g.nx || iy >= g.ny || iz >= g.nz) continue;
        const int64_t i3 = ((int64_t)ix * g.ny + iy) * g.nz + iz;
        const double M = acc[c][0];
        if (out.density) out.density[i3] = M / g.cell_volume;
        const bool has = M > 0.0;
        if (out.vx) out.vx[i3] = has ? acc[c][1] / M : mvx;
        if (out.vy) out.vy[i3] = has ? acc[c][2] / M : mvy;
        if (out.vz) out.vz[i3] = has ? acc[c][3] / M : mvz;
        if (out.raw4) {
            out.raw4[i3] = M;
            out.raw4[ncell + i3] = acc[c][1];
            out.raw4[2 * ncell + i3] = acc[c][2];
            out.raw4[3 * ncell + i3] = acc[c][3];
        }
    }
    add_stat(&st->bbox_pairs, n_bbox);
    add_stat(&st->sphere_pairs, n_sphere);
    add_stat(&st->evaluated_pairs, n_eval);
    add_stat(&st->neg_clamped, n_neg);
    add_stat(&st->neg_warned, n_warn);
    if (EV == kEvTab) add_stat(&st->table_clamps, n_clamp);
}

template <bool CUBIC, bool CULL>
__global__ void __launch_bounds__(kThreads, kMinBlocks) k_cart_gather(CartGeom g, DevParticles P, int kernel,
                                                          const uint32_t* __restrict__ list,
                                                          const int64_t* __restrict__ range,
                                                          const int32_t* __restrict__ tile_map, CartOutputs out,
                                                          DevStats* __restrict__ st) {
    const int64_t t = tile_map ? (int64_t)tile_map[blockIdx.x] : (int64_t)blockIdx.x;
    gather_tile<CUBIC ? kEvCubic : kEvGeneric, CULL>(g, P, kernel, list, range, t, t, out, st);
}

// The per-cell gather with the tabulated integral, every cell of the particles' bounding boxes (outside the
// support the lookups do not cancel exactly, and the reference keeps what they leave).
__global__ void __launch_bounds__(kThreads, kMinBlocks) k_cart_gather_tab(CartGeom g, DevParticles P, const TabDev tab,
                                                                         const uint32_t* __restrict__ list,
                                                                         const int64_t* __restrict__ range,
                                                                         const int32_t* __restrict__ tile_map,
                                                                         CartOutputs out, DevStats* __restrict__ st) {
    const int64_t t = tile_map ? (int64_t)tile_map[blockIdx.x] : (int64_t)blockIdx.x;
    gather_tile<kEvTab, false>(g, P, 0, list, range, t, t, out, st, false, tab);
}

// ------------------------------------------------------------------ lattice form, tabulated integral

// Resident CTAs per SM the register budget of the tabulated lattice kernel is sized for (its 30 KB of
// shared memory fits more; four was slower).
#ifndef KIWI_LATTICE_TAB_MIN_BLOCKS
#define KIWI_LATTICE_TAB_MIN_BLOCKS 3
#endif
constexpr int kLatTabMinBlocks = KIWI_LATTICE_TAB_MIN_BLOCKS;

// The lattice form with the tabulated integral, every cell of the particles' bounding boxes (outside the
// support the lookups do not cancel exactly, and the reference keeps what they leave).  Built here, without
// FMA contraction, so that every lookup lands on the reference's table entries with its weights.
__global__ void __launch_bounds__(kLatThreads, kLatTabMinBlocks) k_cart_lattice_tab(CartGeom g, DevParticles P,
                                                                                 const TabDev tab,
                                                                                 const uint32_t* __restrict__ list,
                                                                                 const int64_t* __restrict__ range,
                                                                                 const int32_t* __restrict__ tile_map,
                                                                                 CartOutputs out,
                                                                                 DevStats* __restrict__ st) {
    const int64_t t = tile_map ? (int64_t)tile_map[blockIdx.x] : (int64_t)blockIdx.x;
    lattice_tile<false, false, true>(g, P, list, range, t, t, out, st, nullptr, tab);
}

// The tiles of a batch of grids whose items take the per-cell gather (the lattice families run in
// lattice.cu): each CTA takes the next of the family's tiles (order[w]) from the work counter and runs the
// same tile body as the single-grid kernel, so every cell's value and summation order are those of a
// single-grid call.
__global__ void __launch_bounds__(kThreads, 2) k_batch_gather_persistent(const BatchItemDev* __restrict__ items,
                                                                         const int32_t* __restrict__ item_of_tile,
                                                                         const int32_t* __restrict__ order,
                                                                         int64_t ntiles,
                                                                         const uint32_t* __restrict__ list,
                                                                         const int64_t* __restrict__ range,
                                                                         unsigned long long* __restrict__ next) {
    __shared__ long long s_w;
    for (;;) {
        if (threadIdx.x == 0) s_w = (long long)atomicAdd(next, 1ull);
        __syncthreads();
        const int64_t w = s_w;
        if (w >= ntiles) break;
        const int64_t tg = (int64_t)order[w];
        const BatchItemDev& it = items[item_of_tile[tg]];
        const int64_t tl = tg - it.tile_base;
        gather_tile<kEvGeneric, true, true>(it.g, it.P, it.kernel, list, range, tg, tl, it.out, it.st,
                                            it.mode == kBatchGatherCubic);
        __syncthreads();
    }
}

__global__ void k_full_integral(int kernel, int64_t n, const double* __restrict__ arg0, const double* __restrict__ phi,
                                const double* __restrict__ r0, const double* __restrict__ R0, double* __restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = (kernel < 0) ? cubic_full_integral(arg0[i], phi[i], r0[i], R0[i])
                          : generic_full_integral(&c_tables[kernel], arg0[i], phi[i], r0[i], R0[i]);
}

// The tier constants of n (r0, R_0) pairs as the reference's structs hold them: for the cubic spline
// (kernel < 0, arg0 = h) WallIntegralConstants and EdgeIntegralConstants (src/kernel_integral.cpp:222-350),
// for a generic kernel (arg0 = H) GenericWallConstants and GenericEdgeConstants
// (src/kernel_integral_generic.cpp:96-148), flattened field by field (flags and region numbers as doubles).
__global__ void k_tier_constants(int kernel, int64_t n, const double* __restrict__ arg0, const double* __restrict__ r0,
                                 const double* __restrict__ R0, double* __restrict__ wall, double* __restrict__ edge) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (kernel < 0) {
        const CubicWall w = cubic_wall_t(arg0[i], r0[i]);
        const CubicEdge e = cubic_edge_t(w, R0[i]);
        double* o = wall + KIWI_CUBIC_WALL_DOUBLES * i;
        const double wv[KIWI_CUBIC_WALL_DOUBLES] = {w.valid ? 1.0 : 0.0, w.r0, w.h, w.h2, w.r03, w.r0h2, w.r0h3,
                                                    w.r0h_2, w.r0h_3, w.B1, w.B2, w.B3};
        for (int k = 0; k < KIWI_CUBIC_WALL_DOUBLES; ++k) o[k] = wv[k];
        double* q = edge + KIWI_CUBIC_EDGE_DOUBLES * i;
        const double ev[KIWI_CUBIC_EDGE_DOUBLES] = {e.valid ? 1.0 : 0.0, e.R_0, e.a, e.a2, e.D2, e.D3};
        for (int k = 0; k < KIWI_CUBIC_EDGE_DOUBLES; ++k) q[k] = ev[k];
        return;
    }
    GenericWall w;
    generic_wall(w, &c_tables[kernel], arg0[i], r0[i]);
    GenericEdge e;
    generic_edge(e, w, R0[i]);
    double* o = wall + KIWI_GENERIC_WALL_DOUBLES * i;
    o[0] = w.valid ? 1.0 : 0.0;
    o[1] = w.H;
    o[2] = w.r0;
    o[3] = w.q0;
    o[4] = (double)w.j;
    for (int k = 0; k < KIWI_MAX_REGIONS; ++k)
        for (int idx = 0; idx < KIWI_NI; ++idx) o[5 + KIWI_NI * k + idx] = w.valid ? w.coef[k][idx] : 0.0;
    for (int k = 0; k < KIWI_MAX_REGIONS; ++k) o[5 + KIWI_NI * KIWI_MAX_REGIONS + k] = w.valid ? w.bphi[k] : 0.0;
    double* q = edge + KIWI_GENERIC_EDGE_DOUBLES * i;
    q[0] = e.valid ? 1.0 : 0.0;
    q[1] = e.R_0;
    q[2] = e.a;
    q[3] = e.a2;
    q[4] = (double)e.nseg;
    for (int s = 0; s < KIWI_MAX_REGIONS; ++s) {
        const bool on = s < e.nseg;
        q[5 + s] = on ? (double)e.region[s] : 0.0;
        q[5 + KIWI_MAX_REGIONS + s] = on ? e.phi_end[s] : 0.0;
        q[5 + 2 * KIWI_MAX_REGIONS + s] = on ? e.offset[s] : 0.0;
    }
}

__global__ void k_face_integral(bool cubic, int kernel, double support_in_h, const TabDev tab, bool tabulated,
                                int64_t n, const double* __restrict__ particle, const int64_t* __restrict__ vert_off,
                                const double* __restrict__ verts, double* __restrict__ out,
                                int32_t* __restrict__ out_vert) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double x0 = particle[4 * i], y0 = particle[4 * i + 1], z0 = particle[4 * i + 2], h = particle[4 * i + 3];
    FlatVerts V{verts + 3 * vert_off[i]};
    const int nv = (int)(vert_off[i + 1] - vert_off[i]);
    int ov = 0;
    double r;
    if (tabulated) {
        unsigned nc = 0;
        TabEval ev{tab, h, 0.0, 0.0, &nc};
        r = face_integral(x0, y0, z0, 2 * h, V, nv, &ov, ev);
    } else if (cubic) {
        CubicEval ev;
        ev.h = h;
        r = face_integral(x0, y0, z0, 2 * h, V, nv, &ov, ev);
    } else {
        GenericEval ev;
        ev.K = &c_tables[kernel];
        ev.H = mul_rn(support_in_h, h);
        r = face_integral(x0, y0, z0, ev.H, V, nv, &ov, ev);
    }
    out[i] = r;
    if (out_vert) out_vert[i] = ov;
}

// Mean particle velocity over all particles (src/cartesian_grid.cpp:205-207, 294-298), by one block
// in a fixed reduction order, so it is bitwise repeatable.
__global__ void k_mean_velocity(DevParticles P, double* __restrict__ meanv) {
    __shared__ double sh[3][1024];
    double s0 = 0, s1 = 0, s2 = 0;
    for (int64_t i = threadIdx.x; i < P.n; i += blockDim.x) {
        s0 += P.vx[i];
        s1 += P.vy[i];
        s2 += P.vz[i];
    }
    sh[0][threadIdx.x] = s0;
    sh[1][threadIdx.x] = s1;
    sh[2][threadIdx.x] = s2;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            sh[0][threadIdx.x] += sh[0][threadIdx.x + o];
            sh[1][threadIdx.x] += sh[1][threadIdx.x + o];
            sh[2][threadIdx.x] += sh[2][threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double n = (double)P.n;
        meanv[0] = P.n > 0 ? sh[0][0] / n : 0.0;
        meanv[1] = P.n > 0 ? sh[1][0] / n : 0.0;
        meanv[2] = P.n > 0 ? sh[2][0] / n : 0.0;
    }
}

// FP64 FMA throughput probe: 8 independent fma chains per thread.
__global__ void __launch_bounds__(256) k_dfma_peak(int iters, double seed, double* __restrict__ sink) {
    double a0 = seed + threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6,
           a7 = a0 + 7;
    const double m = 0.999999, c = 1e-7;
    for (int i = 0; i < iters; ++i) {
        a0 = fma(a0, m, c); a1 = fma(a1, m, c); a2 = fma(a2, m, c); a3 = fma(a3, m, c);
        a4 = fma(a4, m, c); a5 = fma(a5, m, c); a6 = fma(a6, m, c); a7 = fma(a7, m, c);
    }
    const double s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (s == 12345.678) sink[threadIdx.x] = s;  // keeps the chains live
}

}  // namespace

int fp64_measure_peak(KiwiCtx* ctx, double* tflops) {
    int sms = 0;
    KIWI_CUDA(ctx, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    double* sink = nullptr;
    KIWI_TRY(scratch_t(ctx, S_MISC0, 256, &sink));
    const int blocks = sms * 8, iters = 1 << 14;
    k_dfma_peak<<<blocks, 256, 0, ctx->stream>>>(256, 1.0, sink);  // warm-up
    KIWI_LAUNCHED(ctx);
    KIWI_CUDA(ctx, cudaEventRecord(ctx->ev[0], ctx->stream));
    k_dfma_peak<<<blocks, 256, 0, ctx->stream>>>(iters, 1.0, sink);
    KIWI_LAUNCHED(ctx);
    KIWI_CUDA(ctx, cudaEventRecord(ctx->ev[1], ctx->stream));
    KIWI_CUDA(ctx, cudaEventSynchronize(ctx->ev[1]));
    float ms = 0.f;
    KIWI_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]));
    *tflops = 2.0 * 8.0 * iters * (double)blocks * 256.0 / (ms * 1e-3) / 1e12;
    return KIWI_OK;
}

int fp64_cart_gather(KiwiCtx* ctx, const CartGeom& g, const DevParticles& P, const KernelChoice& k,
                     const TileLists& tl, const CartOutputs& out, DevStats* d_stats, bool full_box,
                     bool reference_order) {
    if (tl.ntiles <= 0) return KIWI_OK;
    if (tl.ntiles > 0x7fffffffLL) return set_err(ctx, KIWI_ERR_ARG, "too many cell tiles (%lld)", (long long)tl.ntiles);
    if (tl.map && tl.nmap <= 0) return KIWI_OK;
    const dim3 grid((unsigned)(tl.map ? tl.nmap : tl.ntiles));
    if (k.tabulated && !reference_order) {
        KIWI_CUDA(ctx, cudaFuncSetAttribute(k_cart_lattice_tab, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)kLatTabDynSmem));
        k_cart_lattice_tab<<<grid, kLatThreads, kLatTabDynSmem, ctx->stream>>>(g, P, k.tab, tl.list, tl.range, tl.map,
                                                                               out, d_stats);
    } else if (k.tabulated) {
        k_cart_gather_tab<<<grid, kThreads, 0, ctx->stream>>>(g, P, k.tab, tl.list, tl.range, tl.map, out, d_stats);
    } else if (!reference_order && (k.cubic || !full_box)) {
        return lattice_cart_gather(ctx, g, P, k, tl, out, d_stats, full_box);
    } else if (k.cubic && !full_box)
        k_cart_gather<true, true><<<grid, kThreads, 0, ctx->stream>>>(g, P, k.kernel, tl.list, tl.range, tl.map, out,
                                                                      d_stats);
    else if (k.cubic)
        k_cart_gather<true, false><<<grid, kThreads, 0, ctx->stream>>>(g, P, k.kernel, tl.list, tl.range, tl.map, out,
                                                                       d_stats);
    else if (!full_box)
        k_cart_gather<false, true><<<grid, kThreads, 0, ctx->stream>>>(g, P, k.kernel, tl.list, tl.range, tl.map, out,
                                                                       d_stats);
    else
        k_cart_gather<false, false><<<grid, kThreads, 0, ctx->stream>>>(g, P, k.kernel, tl.list, tl.range, tl.map, out,
                                                                        d_stats);
    KIWI_LAUNCHED(ctx);
    return KIWI_OK;
}

int fp64_batch_prepare(KiwiCtx* ctx) { return lattice_batch_prepare(ctx); }

int fp64_batch_gather(KiwiCtx* ctx, int family, const BatchItemDev* d_items, const int32_t* d_item_of_tile,
                      const int32_t* d_order, int64_t ntiles, const uint32_t* list, const int64_t* range,
                      unsigned long long* d_next, int blocks, bool mixed) {
    if (ntiles <= 0) return KIWI_OK;
    if (family != kBatchFamilyGather)
        return lattice_batch_gather(ctx, family, d_items, d_item_of_tile, d_order, ntiles, list, range, d_next, blocks,
                                    mixed);
    k_batch_gather_persistent<<<blocks, kThreads, 0, ctx->stream>>>(d_items, d_item_of_tile, d_order, ntiles, list,
                                                                   range, d_next);
    KIWI_LAUNCHED(ctx);
    return KIWI_OK;
}

int fp64_full_integral(KiwiCtx* ctx, int kernel, int64_t n, const double* arg0, const double* phi, const double* r0,
                       const double* R0, double* out) {
    if (n <= 0) return KIWI_OK;
    k_full_integral<<<(unsigned)((n + 127) / 128), 128, 0, ctx->stream>>>(kernel, n, arg0, phi, r0, R0, out);
    KIWI_LAUNCHED(ctx);
    return KIWI_OK;
}

int fp64_tier_constants(KiwiCtx* ctx, int kernel, int64_t n, const double* arg0, const double* r0, const double* R0,
                        double* wall, double* edge) {
    if (n <= 0) return KIWI_OK;
    k_tier_constants<<<(unsigned)((n + 127) / 128), 128, 0, ctx->stream>>>(kernel, n, arg0, r0, R0, wall, edge);
    KIWI_LAUNCHED(ctx);
    return KIWI_OK;
}

int fp64_face_integral(KiwiCtx* ctx, const KernelChoice& k, int64_t n, const double* particle,
                       const int64_t* vert_off, const double* verts, double* out, int32_t* out_vert) {
    if (n <= 0) return KIWI_OK;
    k_face_integral<<<(unsigned)((n + 127) / 128), 128, 0, ctx->stream>>>(
        k.cubic, k.kernel, k.support_in_h, k.tab, k.tabulated, n, particle, vert_off, verts, out, out_vert);
    KIWI_LAUNCHED(ctx);
    return KIWI_OK;
}

int fp64_mean_velocity(KiwiCtx* ctx, const DevParticles& P, double* d_meanv) {
    k_mean_velocity<<<1, 1024, 0, ctx->stream>>>(P, d_meanv);
    KIWI_LAUNCHED(ctx);
    return KIWI_OK;
}

}  // namespace kiwi_b200
