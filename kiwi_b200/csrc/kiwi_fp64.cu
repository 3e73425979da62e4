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
    return KIWI_OK;
}

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

// ------------------------------------------------------------------ lattice-factorised gather (cubic)

// Resident CTAs per SM the register budget is sized for: three for the cubic kernel (80 registers; its
// 70 KB of shared memory fits three times) and for the tabulated one (39 KB; four was slower), two for the
// generic one (78 KB of shared memory).
#ifndef KIWI_LATTICE_MIN_BLOCKS
#define KIWI_LATTICE_MIN_BLOCKS 3
#endif
#ifndef KIWI_LATTICE_GEN_MIN_BLOCKS
#define KIWI_LATTICE_GEN_MIN_BLOCKS 2
#endif
#ifndef KIWI_LATTICE_TAB_MIN_BLOCKS
#define KIWI_LATTICE_TAB_MIN_BLOCKS 3
#endif
constexpr int kLatMinBlocks = KIWI_LATTICE_MIN_BLOCKS;
constexpr int kLatGenMinBlocks = KIWI_LATTICE_GEN_MIN_BLOCKS;
constexpr int kLatTabMinBlocks = KIWI_LATTICE_TAB_MIN_BLOCKS;
constexpr int kLatPtCap = kLatSCap / 3;  // lattice points per chunk (three corner items each)
static_assert(kTileX <= 15 && kTileY <= 15 && kTileZ <= 15 && kLatPMax <= 32, "packed corner-list entries");
static_assert(kLatECap <= 2048, "packed edge-list entries");
constexpr size_t kLatDynSmem = sizeof(double) * (2 * kLatECap + kLatSCap);
constexpr size_t kLatGenDynSmem = sizeof(double) * (kLatGenERec * kLatGenECap + kLatSCap);
constexpr size_t kLatMaxDynSmem = kLatDynSmem > kLatGenDynSmem ? kLatDynSmem : kLatGenDynSmem;
constexpr size_t kLatTabDynSmem = sizeof(double) * kLatSCap;



// One CTA = one tile.  The tile's particle list (ascending particle index) is walked in chunks that fit
// the edge and corner tables in shared memory.  Per chunk: (A) the edge tiers of every (plane, edge
// line) of every particle's box, (B) the corner values of every (plane, lattice point), (C) each thread
// assembles the cells it owns from the corner values, particle by particle in list order, and adds them
// to its accumulators -- the same fixed per-cell summation order as k_cart_gather, no atomics.
// GENERIC: the table-driven tiers of kernel `kernel` (support radius support_in_h x h) instead of the
// cubic closed form; the edge tiers are then lattice_generic_edge records.  TAB: the tabulated cubic
// integral (lookups in `tab`): no edge tiers, a corner value is two lookups, and the corner items run in
// their natural order.
template <bool CULL, bool GENERIC = false, bool TAB = false>
__device__ __forceinline__ void lattice_tile(const CartGeom& g, const DevParticles& P,
                                             const uint32_t* __restrict__ list, const int64_t* __restrict__ range,
                                             int64_t t_range, int64_t t, const CartOutputs& out,
                                             DevStats* __restrict__ st, int kernel = 0, const TabDev tab = TabDev{}) {
    __shared__ double s_x[kLatPMax], s_y[kLatPMax], s_z[kLatPMax], s_h[kLatPMax], s_m[kLatPMax], s_vx[kLatPMax],
        s_vy[kLatPMax], s_vz[kLatPMax], s_ih[kLatPMax];
    __shared__ int s_lo[kLatPMax][3], s_dim[kLatPMax][3], s_eoff[kLatPMax], s_soff[kLatPMax];
    __shared__ uint32_t s_mag[kLatPMax][4];  // div_magic of n0, n1, n2 and n1 n2
    __shared__ TabWidths s_tw;               // TAB: the table's bin widths and their reciprocals
    if (TAB && threadIdx.x == 0) s_tw = tab_widths(tab);  // read after the chunk load's barrier
    __shared__ int s_np, s_etot, s_stot, s_nexp, s_ncheap, s_nheavy;
    __shared__ uint32_t s_blist[kLatPtCap];
    __shared__ uint16_t s_hlist[kLatECap];
    extern __shared__ double s_dyn[];
    double* s_D2 = s_dyn;
    double* s_D3 = s_dyn + kLatECap;
    double* s_S = s_dyn + (GENERIC ? kLatGenERec * kLatGenECap : (TAB ? 0 : 2 * kLatECap));
    double* s_E = s_dyn;  // generic edge records
    constexpr int kECap = GENERIC ? kLatGenECap : kLatECap;
    const KiwiKernelTable* K = &c_tables[kernel];

    const int tz = (int)(t % g.ntz), ty = (int)((t / g.ntz) % g.nty), tx = (int)(t / ((int64_t)g.ntz * g.nty));
    const int bx = tx * kTileX, by = ty * kTileY, bz = tz * kTileZ;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // the tile's lattice planes (every particle box is clipped to the tile, so its planes are these) and
    // cell centres, formed once as lattice_offset and cell_centre form them; read after the first barrier
    __shared__ double s_pl[3][kTileX + 1], s_cc[3][kTileX];
    static_assert(kTileX == kTileY && kTileX == kTileZ, "cubic tiles");
    if (threadIdx.x < 3 * (kTileX + 1)) {
        const int a = threadIdx.x / (kTileX + 1), l = threadIdx.x % (kTileX + 1);
        const double mn = a == 0 ? g.x_min : (a == 1 ? g.y_min : g.z_min), d = a == 0 ? g.dpx : (a == 1 ? g.dpy : g.dpz);
        const int b0 = a == 0 ? bx : (a == 1 ? by : bz);
        s_pl[a][l] = add_rn(mn, mul_rn((double)(b0 + l), d));
        if (l < kTileX) s_cc[a][l] = cell_centre(mn, b0 + l, d);
    }

    double acc[kCellsPerThread][4];
#pragma unroll
    for (int c = 0; c < kCellsPerThread; ++c) acc[c][0] = acc[c][1] = acc[c][2] = acc[c][3] = 0.0;
    // work counters: 32-bit per thread (a chunk adds at most 64 to any of them), flushed to the 64-bit
    // totals every 2^20 chunks and at the end
    unsigned n_bbox = 0, n_sphere = 0, n_eval = 0, n_neg = 0, n_warn = 0;
    unsigned n_eo = 0, n_em = 0, n_ei = 0, n_vp = 0, n_clamp = 0, n_chunks = 0;
    auto flush = [&]() {
        add_stat(&st->bbox_pairs, n_bbox);
        add_stat(&st->sphere_pairs, n_sphere);
        add_stat(&st->evaluated_pairs, n_eval);
        add_stat(&st->neg_clamped, n_neg);
        add_stat(&st->neg_warned, n_warn);
        add_stat(&st->edge_outer, n_eo);
        add_stat(&st->edge_middle, n_em);
        add_stat(&st->edge_inner, n_ei);
        add_stat(&st->vertex_pyramids, n_vp);
        if (TAB) add_stat(&st->table_clamps, n_clamp);
        n_bbox = n_sphere = n_eval = n_neg = n_warn = n_eo = n_em = n_ei = n_vp = n_clamp = 0;
    };
    const int64_t beg = range[2 * t_range], end = range[2 * t_range + 1];

    for (int64_t pos = beg; pos < end;) {
        if (warp == 0) {
            const int64_t idx = pos + lane;
            int ne = 0, ns = 0, lo0 = 0, lo1 = 0, lo2 = 0, d0 = 0, d1 = 0, d2 = 0;
            double px = 0, py = 0, pz = 0, ph = 0, pm = 0, pvx = 0, pvy = 0, pvz = 0;
            if (idx < end) {
                const uint32_t p = list[idx];
                px = P.x[p]; py = P.y[p]; pz = P.z[p]; ph = P.h[p];
                pm = P.m[p]; pvx = P.vx[p]; pvy = P.vy[p]; pvz = P.vz[p];
                CellBox b;
                bool outside;
                particle_cell_box(g, px, py, pz, ph, b, &outside);
                lo0 = max(b.x0, bx); lo1 = max(b.y0, by); lo2 = max(b.z0, bz);
                d0 = min(b.x1, bx + kTileX - 1) - lo0 + 1;
                d1 = min(b.y1, by + kTileY - 1) - lo1 + 1;
                d2 = min(b.z1, bz + kTileZ - 1) - lo2 + 1;
                const int n0 = d0 + 1, n1 = d1 + 1, n2 = d2 + 1;
                ne = TAB ? 0 : 2 * (n0 * n1 + n0 * n2 + n1 * n2);
                ns = 3 * n0 * n1 * n2;
            }
            int ie = ne, is = ns;
            for (int o = 1; o < 32; o <<= 1) {
                const int ve = __shfl_up_sync(0xffffffffu, ie, o), vs = __shfl_up_sync(0xffffffffu, is, o);
                if (lane >= o) {
                    ie += ve;
                    is += vs;
                }
            }
            const bool take = (idx < end) && ie <= kECap && is <= kLatSCap;
            const int np = __popc(__ballot_sync(0xffffffffu, take));
            if (take) {
                s_x[lane] = px; s_y[lane] = py; s_z[lane] = pz; s_h[lane] = ph; s_ih[lane] = 1.0 / ph;
                s_m[lane] = pm; s_vx[lane] = pvx; s_vy[lane] = pvy; s_vz[lane] = pvz;
                s_lo[lane][0] = lo0; s_lo[lane][1] = lo1; s_lo[lane][2] = lo2;
                s_dim[lane][0] = d0; s_dim[lane][1] = d1; s_dim[lane][2] = d2;
                s_eoff[lane] = ie - ne;
                s_soff[lane] = is - ns;
                s_mag[lane][0] = div_magic(d0 + 1);
                s_mag[lane][1] = div_magic(d1 + 1);
                s_mag[lane][2] = div_magic(d2 + 1);
                s_mag[lane][3] = div_magic((d1 + 1) * (d2 + 1));
            }
            if (lane == np - 1) {
                s_np = np;
                s_etot = ie;
                s_stot = is;
                s_nexp = s_ncheap = s_nheavy = 0;
            }
        }
        __syncthreads();
        const int np = s_np, etot = s_etot, stot = s_stot;

        // (A) edge tiers: block (a, b) holds r0 along axis a, R_0 along axis b.  Cubic: edges beyond 2h
        // (and zero ones) get D2 = D3 = 0 here; the others are appended to s_hlist (edge slot | particle
        // << 11) with r0, R_0 parked in their slots, and evaluated in (A2) by full warps.  Appends are
        // warp-aggregated; the list order does not affect the results.
        const int eoff_l = lane < np ? s_eoff[lane] : INT_MAX;
        for (int base = warp * 32; base < etot; base += kThreads) {
            const int it = base + lane;
            bool heavy = false;
            const int j = warp_owner(base, eoff_l, lane);
            const int eoff = __shfl_sync(0xffffffffu, eoff_l, j & 31);
            if (it < etot) {
                int e = it - eoff;
                const int n0 = s_dim[j][0] + 1, n1 = s_dim[j][1] + 1, n2 = s_dim[j][2] + 1;
                // blocks in order xy, xz, yx, yz, zx, zy (plane axis a = blk / 2, line axis from 0x102021)
                const int c1 = n0 * n1, c2 = c1 + n0 * n2, c3 = c2 + n1 * n0, c4 = c3 + n1 * n2, c5 = c4 + n2 * n0;
                const int blk = (e >= c1) + (e >= c2) + (e >= c3) + (e >= c4) + (e >= c5);
                e -= blk == 0 ? 0 : blk == 1 ? c1 : blk == 2 ? c2 : blk == 3 ? c3 : blk == 4 ? c4 : c5;
                const int a = blk >> 1, bax = (0x102021 >> (4 * blk)) & 15;
                const int nb = bax == 0 ? n0 : (bax == 1 ? n1 : n2);
                const int p = div_by(e, s_mag[j][bax]), q = e - p * nb;
                const double mna = a == 0 ? g.x_min : (a == 1 ? g.y_min : g.z_min);
                const double dda = a == 0 ? g.dpx : (a == 1 ? g.dpy : g.dpz);
                const double pca = a == 0 ? s_x[j] : (a == 1 ? s_y[j] : s_z[j]);
                const double mnb = bax == 0 ? g.x_min : (bax == 1 ? g.y_min : g.z_min);
                const double ddb = bax == 0 ? g.dpx : (bax == 1 ? g.dpy : g.dpz);
                const double pcb = bax == 0 ? s_x[j] : (bax == 1 ? s_y[j] : s_z[j]);
                const double r0 = fabs(lattice_offset(mna, dda, s_lo[j][a] + p, pca));
                const double R0 = fabs(lattice_offset(mnb, ddb, s_lo[j][bax] + q, pcb));
                if (GENERIC) {
                    lattice_generic_edge(K, mul_rn(g.support_in_h, s_h[j]), r0, R0, s_E + kLatGenERec * it);
                    ++n_ei;
                } else {
                    const double h2 = s_h[j] * s_h[j];
                    const double ld2 = r0 * r0 + R0 * R0;
                    heavy = r0 != 0.0 && R0 != 0.0 && ld2 <= 4.0 * h2;
                    if (heavy) {
                        if (ld2 > h2) ++n_em;
                        else ++n_ei;
                        s_D2[it] = r0;
                        s_D3[it] = R0;
                    } else {
                        ++n_eo;
                        s_D2[it] = 0.0;
                        s_D3[it] = 0.0;
                    }
                }
            }
            if (!GENERIC) {
                const unsigned m = __ballot_sync(0xffffffffu, heavy);
                int pos = 0;
                if (lane == 0 && m) pos = atomicAdd(&s_nheavy, __popc(m));
                pos = __shfl_sync(0xffffffffu, pos, 0);
                if (heavy) s_hlist[pos + __popc(m & ((1u << lane) - 1))] = (uint16_t)(it | j << 11);
            }
        }

        // (B0) list the corner items lattice point by lattice point (the three plane orientations of a
        // point share its offsets and its class), so that the cheap ones (corner beyond the support -- for
        // the cubic spline beyond 2h: only I0 and I1 -- or a zero corner) run in warps of their own (cubic
        // and generic kernels; the tabulated one runs the items in natural order): the others from the
        // front of s_blist, the
        // cheap ones from its end; a point's three items follow one another in (B).  Appends are
        // warp-aggregated; results do not depend on the order.
        // With CULL, a lattice point none of whose eight cells meets the support sphere is read by no
        // evaluated cell: its items are left out.  The test bounds the distance to the 2 x 2 x 2 cells
        // around the point, their half-widths padded by 1e-6 of a cell so that rounding never drops a point
        // an evaluated cell reads.  A list entry packs (particle, i, j, k): 5 + 3 x 4 bits.
        if (!TAB) {
            const int ptot = stot / 3;
            const int poff_l = lane < np ? s_soff[lane] / 3 : INT_MAX;
            for (int base = warp * 32; base < ptot; base += kThreads) {
                const int pt = base + lane;
                int cls = -1;  // -1 none, 0 general, 1 cheap
                uint32_t rec = 0;
                const int jp = warp_owner(base, poff_l, lane);
                const int poff = __shfl_sync(0xffffffffu, poff_l, jp & 31);
                if (pt < ptot) {
                    const int lp = pt - poff;
                    const int n2 = s_dim[jp][2] + 1, n12 = (s_dim[jp][1] + 1) * n2;
                    const int i = div_by(lp, s_mag[jp][3]), rem = lp - i * n12;
                    const int jj = div_by(rem, s_mag[jp][2]), k = rem - jj * n2;
                    const double ux = s_pl[0][s_lo[jp][0] - bx + i] - s_x[jp];
                    const double uy = s_pl[1][s_lo[jp][1] - by + jj] - s_y[jp];
                    const double uz = s_pl[2][s_lo[jp][2] - bz + k] - s_z[jp];
                    const double h = s_h[jp];
                    bool keep = true;
                    if (CULL) {
                        const double radius = mul_rn(g.support_in_h, h);
                        const double ex = fmax(fabs(ux) - kNeedPad * g.dpx, 0.0);
                        const double ey = fmax(fabs(uy) - kNeedPad * g.dpy, 0.0);
                        const double ez = fmax(fabs(uz) - kNeedPad * g.dpz, 0.0);
                        keep = ex * ex + ey * ey + ez * ez < radius * radius;
                    }
                    if (keep) {
                        // beyond the support (2h for the cubic spline)
                        const double H = GENERIC ? mul_rn(g.support_in_h, h) : 2.0 * h;
                        const bool zero = ux == 0.0 || uy == 0.0 || uz == 0.0;
                        cls = (zero || !(ux * ux + uy * uy + uz * uz < H * H)) ? 1 : 0;
                        rec = (uint32_t)jp | (uint32_t)i << 5 | (uint32_t)jj << 9 | (uint32_t)k << 13;
                    }
                }
                const unsigned me = __ballot_sync(0xffffffffu, cls == 0), mc = __ballot_sync(0xffffffffu, cls == 1);
                int pe = 0, pcb = 0;
                if (lane == 0) {
                    if (me) pe = atomicAdd(&s_nexp, __popc(me));
                    if (mc) pcb = atomicAdd(&s_ncheap, __popc(mc));
                }
                pe = __shfl_sync(0xffffffffu, pe, 0);
                pcb = __shfl_sync(0xffffffffu, pcb, 0);
                const unsigned below = (1u << lane) - 1;
                if (cls >= 0) s_blist[cls == 0 ? pe + __popc(me & below) : kLatPtCap - 1 - pcb - __popc(mc & below)] = rec;
            }
        }
        __syncthreads();

        // (A2) the listed edges (cubic)
        if (!GENERIC) {
            const int nheavy = s_nheavy;
            for (int li = threadIdx.x; li < nheavy; li += kThreads) {
                const int rec = s_hlist[li];
                const int it = rec & 2047, j = rec >> 11;
                const LatticeEdge ed = lattice_edge(s_h[j], s_ih[j], s_D2[it], s_D3[it]);
                s_D2[it] = ed.D2;
                s_D3[it] = ed.D3;
            }
            __syncthreads();
        }
        const int nexp = s_nexp, ncheap = s_ncheap;  // lattice points
        const int nblist = TAB ? stot : 3 * (nexp + ncheap);

        // (B) corner values S_a(i, j, k) for the three plane orientations a
        for (int li = threadIdx.x; li < nblist; li += kThreads) {
            int it, jp, axis, i, jj, k;
            if (TAB) {
                it = li;
                jp = chunk_search(s_soff, np, it);
                const int s = it - s_soff[jp];
                const int n1 = s_dim[jp][1] + 1, n2 = s_dim[jp][2] + 1;
                const int L = (s_dim[jp][0] + 1) * n1 * n2;
                axis = s / L;
                const int rem = s % L;
                i = rem / (n1 * n2);
                jj = (rem / n2) % n1;
                k = rem % n2;
            } else {
                const int pli = li / 3;
                axis = li - 3 * pli;
                const uint32_t rec = s_blist[pli < nexp ? pli : kLatPtCap - ncheap + (pli - nexp)];
                jp = (int)(rec & 31u);
                i = (int)((rec >> 5) & 15u);
                jj = (int)((rec >> 9) & 15u);
                k = (int)((rec >> 13) & 15u);
                const int n1 = s_dim[jp][1] + 1, n2 = s_dim[jp][2] + 1;
                it = s_soff[jp] + axis * ((s_dim[jp][0] + 1) * n1 * n2) + (i * n1 + jj) * n2 + k;
            }
            const int n0 = s_dim[jp][0] + 1, n1 = s_dim[jp][1] + 1, n2 = s_dim[jp][2] + 1;
            const double ux = s_pl[0][s_lo[jp][0] - bx + i] - s_x[jp];
            const double uy = s_pl[1][s_lo[jp][1] - by + jj] - s_y[jp];
            const double uz = s_pl[2][s_lo[jp][2] - bz + k] - s_z[jp];
            const int eb = s_eoff[jp];
            const int nxy = n0 * n1, nxz = n0 * n2, nyz = n1 * n2;
            double r0, u1, u2;
            int e1, e2;
            if (axis == 0) {  // plane x = X_i, corner (y, z)
                r0 = fabs(ux); u1 = uy; u2 = uz;
                e1 = eb + i * n1 + jj;                    // xy[i][jj]
                e2 = eb + nxy + i * n2 + k;               // xz[i][k]
            } else if (axis == 1) {  // plane y = Y_jj, corner (x, z)
                r0 = fabs(uy); u1 = ux; u2 = uz;
                e1 = eb + nxy + nxz + jj * n0 + i;        // yx[jj][i]
                e2 = eb + 2 * nxy + nxz + jj * n2 + k;    // yz[jj][k]
            } else {  // plane z = Z_k, corner (x, y)
                r0 = fabs(uz); u1 = ux; u2 = uy;
                e1 = eb + 2 * nxy + nxz + nyz + k * n0 + i;       // zx[k][i]
                e2 = eb + 2 * nxy + 2 * nxz + nyz + k * n1 + jj;  // zy[k][jj]
            }
            double f = 0.0;
            const double sg = sgn(u1) * sgn(u2);
            if (sg != 0.0 && r0 != 0.0) {
                const double a1 = fabs(u1), a2 = fabs(u2);
                if (TAB) {
                    // two right-triangle vertex pyramids; cos(phi) from the legs
                    f = tab_pair(tab, s_tw, s_ih[jp], r0, a1, a2, n_clamp);
                } else if (GENERIC) {
                    const double H = mul_rn(g.support_in_h, s_h[jp]);
                    f = lattice_generic_corner(K, H, r0, a1, a2, s_E + kLatGenERec * e1, s_E + kLatGenERec * e2);
                } else {
                    f = lattice_corner(s_h[jp], s_ih[jp], r0, a1, a2, s_D2[e1], s_D3[e1], s_D2[e2], s_D3[e2]);
                }
                n_vp += 2;
            }
            s_S[it] = sg * f;
        }
        __syncthreads();

        // (C) cells: 6 faces x inclusion-exclusion over 4 corners, in particle order
#pragma unroll
        for (int c = 0; c < kCellsPerThread; ++c) {
            const int li = threadIdx.x + c * kThreads;
            const int gz = bz + li % kTileZ, gy = by + (li / kTileZ) % kTileY, gx = bx + li / (kTileZ * kTileY);
            for (int j = 0; j < np; ++j) {
                const int i = gx - s_lo[j][0], jj = gy - s_lo[j][1], k = gz - s_lo[j][2];
                if (i < 0 || jj < 0 || k < 0 || i >= s_dim[j][0] || jj >= s_dim[j][1] || k >= s_dim[j][2]) continue;
                ++n_bbox;
                const double x0 = s_x[j], y0 = s_y[j], z0 = s_z[j];
                const double radius = mul_rn(g.support_in_h, s_h[j]);
                const double ex = fmax(fabs(x0 - s_cc[0][gx - bx]) - g.hpx, 0.0);
                const double ey = fmax(fabs(y0 - s_cc[1][gy - by]) - g.hpy, 0.0);
                const double ez = fmax(fabs(z0 - s_cc[2][gz - bz]) - g.hpz, 0.0);
                const bool in = ex * ex + ey * ey + ez * ez < radius * radius;
                n_sphere += in;
                if (CULL && !in) continue;
                ++n_eval;
                const int n1 = s_dim[j][1] + 1, n2 = s_dim[j][2] + 1;
                const int L = (s_dim[j][0] + 1) * n1 * n2;
                const double* Sx = s_S + s_soff[j];
                const double* Sy = Sx + L;
                const double* Sz = Sy + L;
                auto at = [&](const double* S, int a, int b, int cc) { return S[(a * n1 + b) * n2 + cc]; };
                const int lx = gx - bx, ly = gy - by, lz = gz - bz;
                const double sx1 = sgn(s_pl[0][lx + 1] - x0), sx0 = sgn(s_pl[0][lx] - x0);
                const double sy1 = sgn(s_pl[1][ly + 1] - y0), sy0 = sgn(s_pl[1][ly] - y0);
                const double sz1 = sgn(s_pl[2][lz + 1] - z0), sz0 = sgn(s_pl[2][lz] - z0);
                double msum = 0.0;
                msum += sx1 * (at(Sx, i + 1, jj + 1, k + 1) - at(Sx, i + 1, jj, k + 1) - at(Sx, i + 1, jj + 1, k) + at(Sx, i + 1, jj, k));
                msum -= sx0 * (at(Sx, i, jj + 1, k + 1) - at(Sx, i, jj, k + 1) - at(Sx, i, jj + 1, k) + at(Sx, i, jj, k));
                msum += sy1 * (at(Sy, i + 1, jj + 1, k + 1) - at(Sy, i, jj + 1, k + 1) - at(Sy, i + 1, jj + 1, k) + at(Sy, i, jj + 1, k));
                msum -= sy0 * (at(Sy, i + 1, jj, k + 1) - at(Sy, i, jj, k + 1) - at(Sy, i + 1, jj, k) + at(Sy, i, jj, k));
                msum += sz1 * (at(Sz, i + 1, jj + 1, k + 1) - at(Sz, i, jj + 1, k + 1) - at(Sz, i + 1, jj, k + 1) + at(Sz, i, jj, k + 1));
                msum -= sz0 * (at(Sz, i + 1, jj + 1, k) - at(Sz, i, jj + 1, k) - at(Sz, i + 1, jj, k) + at(Sz, i, jj, k));
                if (msum < 0.0) {
                    ++n_neg;
                    if (msum <= -0.01) ++n_warn;
                    msum = 0.0;
                }
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
        if (++n_chunks == (1u << 20)) {
            flush();
            n_chunks = 0;
        }
    }

    const double mvx = out.meanv[0], mvy = out.meanv[1], mvz = out.meanv[2];
    const int64_t ncell = (int64_t)g.nx * g.ny * g.nz;
#pragma unroll
    for (int c = 0; c < kCellsPerThread; ++c) {
        const int li = threadIdx.x + c * kThreads;
        const int ix = bx + li / (kTileZ * kTileY), iy = by + (li / kTileZ) % kTileY, iz = bz + li % kTileZ;
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
    flush();
}

template <bool CULL>
__global__ void __launch_bounds__(kThreads, kLatMinBlocks) k_cart_lattice(CartGeom g, DevParticles P,
                                                                          const uint32_t* __restrict__ list,
                                                                          const int64_t* __restrict__ range,
                                                                          const int32_t* __restrict__ tile_map,
                                                                          CartOutputs out, DevStats* __restrict__ st) {
    const int64_t t = tile_map ? (int64_t)tile_map[blockIdx.x] : (int64_t)blockIdx.x;
    lattice_tile<CULL>(g, P, list, range, t, t, out, st);
}

// The lattice form for the generic kernels (support cells only).
__global__ void __launch_bounds__(kThreads, kLatGenMinBlocks) k_cart_lattice_generic(CartGeom g, DevParticles P, int kernel,
                                                                                  const uint32_t* __restrict__ list,
                                                                                  const int64_t* __restrict__ range,
                                                                                  const int32_t* __restrict__ tile_map,
                                                                                  CartOutputs out,
                                                                                  DevStats* __restrict__ st) {
    const int64_t t = tile_map ? (int64_t)tile_map[blockIdx.x] : (int64_t)blockIdx.x;
    lattice_tile<true, true>(g, P, list, range, t, t, out, st, kernel);
}

// The lattice form with the tabulated integral, every cell of the particles' bounding boxes (outside the
// support the lookups do not cancel exactly, and the reference keeps what they leave).
__global__ void __launch_bounds__(kThreads, kLatTabMinBlocks) k_cart_lattice_tab(CartGeom g, DevParticles P, const TabDev tab,
                                                                              const uint32_t* __restrict__ list,
                                                                              const int64_t* __restrict__ range,
                                                                              const int32_t* __restrict__ tile_map,
                                                                              CartOutputs out,
                                                                              DevStats* __restrict__ st) {
    const int64_t t = tile_map ? (int64_t)tile_map[blockIdx.x] : (int64_t)blockIdx.x;
    lattice_tile<false, false, true>(g, P, list, range, t, t, out, st, 0, tab);
}

// The tiles of a batch of grids, one persistent launch per tile-body family (cubic lattice, generic
// lattice, per-cell gather): each CTA takes the next of the family's tiles (order[w]) from the work
// counter and runs the same tile body as the single-grid kernel, so every cell's value and summation
// order are those of a single-grid call.  One instance per family keeps each body's register budget.
template <int FAMILY>
__global__ void __launch_bounds__(kThreads, 2) k_batch_persistent(const BatchItemDev* __restrict__ items,
                                                                 const int32_t* __restrict__ item_of_tile,
                                                                 const int32_t* __restrict__ order, int64_t ntiles,
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
        if (FAMILY == kBatchFamilyLattice)
            lattice_tile<true>(it.g, it.P, list, range, tg, tl, it.out, it.st);
        else if (FAMILY == kBatchFamilyLatticeGeneric)
            lattice_tile<true, true>(it.g, it.P, list, range, tg, tl, it.out, it.st, it.kernel);
        else
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
        k_cart_lattice_tab<<<grid, kThreads, kLatTabDynSmem, ctx->stream>>>(g, P, k.tab, tl.list, tl.range, tl.map,
                                                                            out, d_stats);
    } else if (k.tabulated) {
        k_cart_gather_tab<<<grid, kThreads, 0, ctx->stream>>>(g, P, k.tab, tl.list, tl.range, tl.map, out, d_stats);
    } else if (k.cubic && !reference_order) {
        if (full_box) {
            KIWI_CUDA(ctx, cudaFuncSetAttribute(k_cart_lattice<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                (int)kLatDynSmem));
            KIWI_CUDA(ctx, cudaFuncSetAttribute(k_cart_lattice<false>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                                (int)cudaSharedmemCarveoutMaxShared));
            k_cart_lattice<false><<<grid, kThreads, kLatDynSmem, ctx->stream>>>(g, P, tl.list, tl.range, tl.map, out,
                                                                                d_stats);
        } else {
            KIWI_CUDA(ctx, cudaFuncSetAttribute(k_cart_lattice<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                (int)kLatDynSmem));
            KIWI_CUDA(ctx, cudaFuncSetAttribute(k_cart_lattice<true>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                                (int)cudaSharedmemCarveoutMaxShared));
            k_cart_lattice<true><<<grid, kThreads, kLatDynSmem, ctx->stream>>>(g, P, tl.list, tl.range, tl.map, out,
                                                                               d_stats);
        }
    } else if (!k.cubic && !reference_order && !full_box) {
        KIWI_CUDA(ctx, cudaFuncSetAttribute(k_cart_lattice_generic, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)kLatGenDynSmem));
        k_cart_lattice_generic<<<grid, kThreads, kLatGenDynSmem, ctx->stream>>>(g, P, k.kernel, tl.list, tl.range,
                                                                                tl.map, out, d_stats);
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

int fp64_batch_prepare(KiwiCtx* ctx) {
    KIWI_CUDA(ctx, cudaFuncSetAttribute(k_batch_persistent<kBatchFamilyLattice>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLatDynSmem));
    KIWI_CUDA(ctx, cudaFuncSetAttribute(k_batch_persistent<kBatchFamilyLatticeGeneric>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLatGenDynSmem));
    return KIWI_OK;
}

int fp64_batch_gather(KiwiCtx* ctx, int family, const BatchItemDev* d_items, const int32_t* d_item_of_tile,
                      const int32_t* d_order, int64_t ntiles, const uint32_t* list, const int64_t* range,
                      unsigned long long* d_next, int blocks) {
    if (ntiles <= 0) return KIWI_OK;
    if (family == kBatchFamilyLattice)
        k_batch_persistent<kBatchFamilyLattice><<<blocks, kThreads, kLatDynSmem, ctx->stream>>>(
            d_items, d_item_of_tile, d_order, ntiles, list, range, d_next);
    else if (family == kBatchFamilyLatticeGeneric)
        k_batch_persistent<kBatchFamilyLatticeGeneric><<<blocks, kThreads, kLatGenDynSmem, ctx->stream>>>(
            d_items, d_item_of_tile, d_order, ntiles, list, range, d_next);
    else
        k_batch_persistent<kBatchFamilyGather><<<blocks, kThreads, 0, ctx->stream>>>(d_items, d_item_of_tile, d_order,
                                                                                     ntiles, list, range, d_next);
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
