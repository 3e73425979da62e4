// Particle binning into cell tiles (the first step of every Cartesian call): per-particle tile counts,
// emission of (tile, particle) entries in particle order, and per-tile ranges of the sorted entries.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "engine.hpp"

namespace kiwi_b200 {

struct TileBox {
    int x0, x1, y0, y1, z0, z1;  // inclusive tile ranges
};

// Per particle: the number of cell tiles its clamped support box touches (0 if none).
static __global__ void k_tile_counts(CartGeom g, DevParticles P, uint32_t* __restrict__ counts, TileBox* __restrict__ boxes,
                              DevStats* __restrict__ st) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long outside_count = 0;
    if (i < P.n) {
        CellBox b;
        bool outside = false;
        uint32_t c = 0;
        TileBox tb{0, -1, 0, -1, 0, -1};
        if (particle_cell_box(g, P.x[i], P.y[i], P.z[i], P.h[i], b, &outside)) {
            tb.x0 = b.x0 / kTileX; tb.x1 = b.x1 / kTileX;
            tb.y0 = b.y0 / kTileY; tb.y1 = b.y1 / kTileY;
            tb.z0 = b.z0 / kTileZ; tb.z1 = b.z1 / kTileZ;
            c = (uint32_t)((tb.x1 - tb.x0 + 1) * (tb.y1 - tb.y0 + 1) * (tb.z1 - tb.z0 + 1));
        }
        if (outside) outside_count = 1;
        counts[i] = c;
        boxes[i] = tb;
    }
    for (int o = 16; o > 0; o >>= 1) outside_count += __shfl_down_sync(0xffffffffu, outside_count, o);
    if ((threadIdx.x & 31) == 0 && outside_count) atomicAdd(&st->skipped_outside, outside_count);
}

// One thread per (particle, tile) entry k in [k0, k0 + count): key = key_base + tile id, value = particle
// index (or, with value_is_entry, the entry index k itself), written in particle order (offs: the
// exclusive scan of the counts of these n particles, whose first entry is k0 -- entries of several grids
// can share one key space and one sort).
static __global__ void k_tile_emit(CartGeom g, int64_t n, const int64_t* __restrict__ offs, const TileBox* __restrict__ boxes,
                            int64_t k0, int64_t count, uint32_t key_base, uint32_t* __restrict__ keys,
                            uint32_t* __restrict__ vals, bool value_is_entry = false) {
    const int64_t kk = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (kk >= count) return;
    const int64_t k = k0 + kk;
    // particle = last p with offs[p] <= k
    int64_t lo = 0, hi = n - 1;
    while (lo < hi) {
        const int64_t mid = (lo + hi + 1) >> 1;
        if (offs[mid] <= k) lo = mid; else hi = mid - 1;
    }
    const TileBox tb = boxes[lo];
    const int64_t q = k - offs[lo];
    const int dz = tb.z1 - tb.z0 + 1, dy = tb.y1 - tb.y0 + 1;
    const int tz = tb.z0 + (int)(q % dz), ty = tb.y0 + (int)((q / dz) % dy), tx = tb.x0 + (int)(q / ((int64_t)dz * dy));
    keys[k] = key_base + (uint32_t)(((int64_t)tx * g.nty + ty) * g.ntz + tz);
    vals[k] = value_is_entry ? (uint32_t)k : (uint32_t)lo;
}

// range[2t], range[2t+1] = [begin, end) of tile t in the sorted key array (zero-length if absent).
static __global__ void k_tile_ranges(const uint32_t* __restrict__ keys, int64_t total, int64_t* __restrict__ range) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const uint32_t k = keys[i];
    if (i == 0 || keys[i - 1] != k) range[2 * (int64_t)k] = i;
    if (i == total - 1 || keys[i + 1] != k) range[2 * (int64_t)k + 1] = i + 1;
}


// Per tile: its (tile, particle) entry count, the weight by which the tiles are split between parts.
static __global__ void k_tile_entry_counts(const int64_t* __restrict__ range, int64_t ntiles, uint32_t* __restrict__ w) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntiles) return;
    const int64_t e = range[2 * t + 1] - range[2 * t];
    w[t] = (uint32_t)(e < 0xffffffffLL ? e : 0xffffffffLL);
}

// 1 if tile t belongs to part `part` of n: part floor(prefix(t) n / W), prefix(t) the entries of the tiles
// before t and W the total (capped at n - 1), so the parts are contiguous runs of the tile order with
// near-equal entry counts; with W = 0 the tiles are split evenly by number.
static __global__ void k_tile_part_flags(const int64_t* __restrict__ prefix, const int64_t* __restrict__ total,
                                         int64_t ntiles, int part, int n, uint32_t* __restrict__ flags) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntiles) return;
    const int64_t W = *total;
    int64_t owner = W > 0 ? (prefix[t] * n) / W : (t * n) / ntiles;
    if (owner > n - 1) owner = n - 1;
    flags[t] = owner == part ? 1u : 0u;
}

// map[offs[t]] = t for the flagged tiles (offs: the exclusive scan of the flags).
static __global__ void k_compact_map(const uint32_t* __restrict__ flags, const int64_t* __restrict__ offs, int64_t n,
                                     int32_t* __restrict__ map) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n && flags[t]) map[offs[t]] = (int32_t)t;
}

}  // namespace kiwi_b200
