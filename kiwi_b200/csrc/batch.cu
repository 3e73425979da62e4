// Batches of independent sph-to-grid problems (many snapshots, each on its own grid, with any kernel) in
// one persistent launch per tile-body family, replayed as a CUDA graph.
//
// kiwi_batch_create bins every item's particles into its own grid's cell tiles with one shared key space
// (item i's tiles follow item i-1's), so a single scan and a single stable sort build every tile list at
// once; it groups the tiles by the tile body their item needs (cubic lattice, generic lattice, per-cell
// gather), orders each group longest-first (by (tile, particle) entry count, ties by tile index) and
// records one CUDA graph: counter resets and per-item mean velocities, then one k_batch_persistent launch
// per group, whose CTAs pull tiles from a work counter and run the same tile bodies as the single-grid
// kernels.  Every cell
// is therefore summed in the same particle order with the same arithmetic as a single-grid call of the
// same form: the batch's outputs equal the per-item outputs bit for bit.  kiwi_batch_run replays the graph.
// kiwi_batch_tune times the launch shapes (tile order x resident CTAs per SM) and keeps the fastest.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "../../include/kiwi_b200.h"
#include "binning.cuh"
#include "engine.hpp"
#include "prims.cuh"

using namespace kiwi_b200;

struct KiwiBatch {
    KiwiCtx* ctx = nullptr;
    int n_items = 0;
    int precision = 0;
    int64_t n_particles = 0, n_tiles = 0, n_entries = 0;
    std::vector<int64_t> tile_base, item_entries, item_skipped;
    std::vector<void*> allocs;
    BatchItemDev* d_items = nullptr;
    int32_t* d_item_of_tile = nullptr;
    // per tile-body family: its tiles in natural (item, tile) order and longest-first, and its counter
    int32_t* d_natural[kBatchFamilies] = {};
    int32_t* d_lpt[kBatchFamilies] = {};
    int64_t fam_tiles[kBatchFamilies] = {};
    // both lattice families' tiles together (natural order and longest-first), for the merged launch
    int32_t* d_natural_m = nullptr;
    int32_t* d_lpt_m = nullptr;
    int64_t merged_tiles = 0;
    bool merge = false;
    const uint32_t* d_list = nullptr;
    int64_t* d_range = nullptr;
    unsigned long long* d_next = nullptr;  // kBatchFamilies counters
    DevStats* d_stats = nullptr;  // per item
    double* d_meanv = nullptr;    // 4 per item
    std::vector<BatchItemDev> items;
    bool lpt = true;
    int ctas_per_sm = 2;
    int sms = 148;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace {

__global__ void k_fill_i32(int32_t* __restrict__ dst, int64_t n, int32_t v) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = v;
}

__global__ void k_gather_i64(const int64_t* __restrict__ src, const int64_t* __restrict__ idx, int n,
                             int64_t* __restrict__ dst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[idx[i]];
}

// Longest-first sort keys for the tiles tiles[0 .. n): ~entries (ascending key = descending entry count),
// value = tile index.
__global__ void k_tile_weights(const int64_t* __restrict__ range, const int32_t* __restrict__ tiles, int64_t n,
                               uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= n) return;
    const int64_t t = tiles[w];
    const int64_t e = range[2 * t + 1] - range[2 * t];
    keys[w] = 0xffffffffu - (uint32_t)(e < 0xffffffffLL ? e : 0xffffffffLL);
    vals[w] = (uint32_t)t;
}

template <class T>
int balloc(KiwiBatch* b, size_t count, T** out) {
    void* p = nullptr;
    const size_t bytes = (count > 0 ? count : 1) * sizeof(T);
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        return set_err(b->ctx, KIWI_ERR_ALLOC, "batch: cudaMalloc of %zu bytes failed", bytes);
    }
    b->allocs.push_back(p);
    *out = static_cast<T*>(p);
    return KIWI_OK;
}

void batch_free(KiwiBatch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    for (void* p : b->allocs) cudaFree(p);
    b->allocs.clear();
}

// The replayed work: reset the counters, the mean velocities, one persistent launch per family present.
int batch_enqueue(KiwiBatch* b) {
    KiwiCtx* ctx = b->ctx;
    const bool mixed = (b->precision & KIWI_FORM_MASK) == KIWI_FP32_MIXED;
    KIWI_CUDA(ctx, cudaMemsetAsync(b->d_next, 0, sizeof(unsigned long long) * kBatchFamilies, ctx->stream));
    KIWI_CUDA(ctx, cudaMemsetAsync(b->d_stats, 0, sizeof(DevStats) * b->n_items, ctx->stream));
    for (int i = 0; i < b->n_items; ++i) KIWI_TRY(fp64_mean_velocity(ctx, b->items[i].P, b->d_meanv + 4 * i));
    for (int f = 0; f < kBatchFamilies; ++f) {
        if (b->merge && f == kBatchFamilyLatticeGeneric) continue;
        if (b->merge && f == kBatchFamilyLattice) {
            KIWI_TRY(fp64_batch_gather(ctx, kBatchFamilyLatticeMerged, b->d_items, b->d_item_of_tile,
                                       b->lpt ? b->d_lpt_m : b->d_natural_m, b->merged_tiles, b->d_list, b->d_range,
                                       b->d_next + f, b->sms * b->ctas_per_sm, mixed));
            continue;
        }
        KIWI_TRY(fp64_batch_gather(ctx, f, b->d_items, b->d_item_of_tile, b->lpt ? b->d_lpt[f] : b->d_natural[f],
                                   b->fam_tiles[f], b->d_list, b->d_range, b->d_next + f, b->sms * b->ctas_per_sm,
                                   mixed));
    }
    return KIWI_OK;
}

int batch_record(KiwiBatch* b) {
    KiwiCtx* ctx = b->ctx;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    KIWI_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = batch_enqueue(b);
    cudaGraph_t g = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(ctx->stream, &g);
    if (rc != KIWI_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (ec != cudaSuccess) return set_err(ctx, KIWI_ERR_CUDA, "batch: graph capture failed: %s", cudaGetErrorString(ec));
    b->graph = g;
    KIWI_CUDA(ctx, cudaGraphInstantiate(&b->exec, g, 0));
    return KIWI_OK;
}

int batch_build(KiwiBatch* b, const KiwiBatchItem* in) {
    KiwiCtx* ctx = b->ctx;
    const int n = b->n_items;
    b->items.resize(n);
    b->tile_base.resize(n + 1);
    std::vector<int64_t> pbase(n + 1);
    b->tile_base[0] = 0;
    pbase[0] = 0;
    for (int i = 0; i < n; ++i) {
        const KiwiBatchItem& it = in[i];
        int rc = KIWI_OK;
        if (!particles_ok(ctx, &it.particles, &rc)) return rc;
        KernelChoice kc;
        KIWI_TRY(resolve_kernel(ctx, &it.kernel, &kc));
        if (kc.tabulated) return set_err(ctx, KIWI_ERR_UNSUPPORTED, "batch: the tabulated integral is not available");
        BatchItemDev& d = b->items[i];
        KIWI_TRY(make_geom(ctx, &it.grid, kc.support_in_h, &d.g));
        d.P = DevParticles{it.particles.n, it.particles.x, it.particles.y, it.particles.z, it.particles.vx,
                           it.particles.vy, it.particles.vz, it.particles.m, it.particles.h};
        d.out = CartOutputs{it.density, it.vx, it.vy, it.vz, it.raw4, nullptr};
        d.kernel = kc.kernel;
        const int form = b->precision & KIWI_FORM_MASK;
        if (form == KIWI_FP64 || form == KIWI_FP32_MIXED) d.mode = kc.cubic ? kBatchLattice : kBatchLatticeGeneric;
        else d.mode = kc.cubic ? kBatchGatherCubic : kBatchGatherGeneric;
        d.tile_base = b->tile_base[i];
        b->tile_base[i + 1] = b->tile_base[i] + (int64_t)d.g.ntx * d.g.nty * d.g.ntz;
        pbase[i + 1] = pbase[i] + it.particles.n;
    }
    b->n_tiles = b->tile_base[n];
    b->n_particles = pbase[n];
    if (b->n_tiles >= (1LL << 31)) return set_err(ctx, KIWI_ERR_ARG, "batch: too many cell tiles (%lld)", (long long)b->n_tiles);
    if (b->n_particles >= (1LL << 32))
        return set_err(ctx, KIWI_ERR_ARG, "batch: too many particles (%lld)", (long long)b->n_particles);

    KIWI_TRY(balloc(b, (size_t)n, &b->d_stats));
    KIWI_TRY(balloc(b, (size_t)4 * n, &b->d_meanv));
    KIWI_TRY(balloc(b, kBatchFamilies, &b->d_next));
    KIWI_TRY(balloc(b, (size_t)n, &b->d_items));
    KIWI_TRY(balloc(b, (size_t)b->n_tiles, &b->d_item_of_tile));
    KIWI_TRY(balloc(b, (size_t)2 * b->n_tiles, &b->d_range));
    // each family's tiles in natural order (the tile ranges of its items, in item order)
    std::vector<int32_t> nat[kBatchFamilies];
    for (int i = 0; i < n; ++i) {
        std::vector<int32_t>& v = nat[batch_family(b->items[i].mode)];
        for (int64_t t = b->tile_base[i]; t < b->tile_base[i + 1]; ++t) v.push_back((int32_t)t);
    }
    for (int f = 0; f < kBatchFamilies; ++f) {
        b->fam_tiles[f] = (int64_t)nat[f].size();
        KIWI_TRY(balloc(b, nat[f].size(), &b->d_natural[f]));
        KIWI_TRY(balloc(b, nat[f].size(), &b->d_lpt[f]));
        if (!nat[f].empty())
            KIWI_CUDA(ctx, cudaMemcpyAsync(b->d_natural[f], nat[f].data(), sizeof(int32_t) * nat[f].size(),
                                           cudaMemcpyHostToDevice, ctx->stream));
    }
    std::vector<int32_t> nat_m;  // both lattice families, in item order
    for (int i = 0; i < n; ++i)
        if (batch_family(b->items[i].mode) != kBatchFamilyGather)
            for (int64_t t = b->tile_base[i]; t < b->tile_base[i + 1]; ++t) nat_m.push_back((int32_t)t);
    b->merged_tiles = (int64_t)nat_m.size();
    KIWI_TRY(balloc(b, nat_m.size(), &b->d_natural_m));
    KIWI_TRY(balloc(b, nat_m.size(), &b->d_lpt_m));
    if (!nat_m.empty())
        KIWI_CUDA(ctx, cudaMemcpyAsync(b->d_natural_m, nat_m.data(), sizeof(int32_t) * nat_m.size(),
                                       cudaMemcpyHostToDevice, ctx->stream));
    KIWI_CUDA(ctx, cudaMemsetAsync(b->d_stats, 0, sizeof(DevStats) * n, ctx->stream));
    for (int i = 0; i < n; ++i) {
        b->items[i].st = b->d_stats + i;
        b->items[i].out.meanv = b->d_meanv + 4 * i;
    }

    // (1) per-particle tile counts, every item into one array
    const int64_t N = b->n_particles;
    uint32_t* counts = nullptr;
    TileBox* boxes = nullptr;
    int64_t* offs = nullptr;
    KIWI_TRY(scratch_t(ctx, S_COUNT, (size_t)std::max<int64_t>(N, 1), &counts));
    KIWI_TRY(scratch_t(ctx, S_BOX, (size_t)std::max<int64_t>(N, 1), &boxes));
    KIWI_TRY(scratch_t(ctx, S_OFFS, (size_t)std::max<int64_t>(N, 1) + 1, &offs));
    int64_t* d_total = offs + std::max<int64_t>(N, 1);
    for (int i = 0; i < n; ++i) {
        const BatchItemDev& d = b->items[i];
        if (d.P.n > 0) {
            k_tile_counts<<<(unsigned)((d.P.n + 255) / 256), 256, 0, ctx->stream>>>(d.g, d.P, counts + pbase[i],
                                                                                    boxes + pbase[i], d.st);
            KIWI_LAUNCHED(ctx);
        }
    }
    KIWI_TRY(exclusive_scan<uint32_t>(ctx, counts, N, offs, d_total));
    // the scan at every item boundary (the first entry of each item, and the total)
    std::vector<int64_t> kfirst(n + 1, 0);
    {
        int64_t *d_idx = nullptr, *d_val = nullptr;
        KIWI_TRY(scratch_t(ctx, S_MISC0, (size_t)n + 1, &d_idx));
        KIWI_TRY(scratch_t(ctx, S_MISC1, (size_t)n + 1, &d_val));
        std::vector<int64_t> idx(n + 1);
        for (int i = 0; i <= n; ++i) idx[i] = std::min<int64_t>(pbase[i], std::max<int64_t>(N, 1));
        KIWI_CUDA(ctx, cudaMemcpyAsync(d_idx, idx.data(), sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice, ctx->stream));
        k_gather_i64<<<(n + 1 + 127) / 128, 128, 0, ctx->stream>>>(offs, d_idx, n + 1, d_val);
        KIWI_LAUNCHED(ctx);
        KIWI_CUDA(ctx, cudaMemcpyAsync(kfirst.data(), d_val, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToHost, ctx->stream));
        int64_t total = 0;
        KIWI_CUDA(ctx, cudaMemcpyAsync(&total, d_total, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
        KIWI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        kfirst[n] = total;
        for (int i = 0; i < n; ++i)
            if (pbase[i] >= N) kfirst[i] = total;  // empty trailing items
    }
    const int64_t total = kfirst[n];
    b->n_entries = total;
    if (total >= (1LL << 32)) return set_err(ctx, KIWI_ERR_LIMIT, "batch: too many (tile, particle) entries: %lld", (long long)total);
    b->item_entries.resize(n);
    for (int i = 0; i < n; ++i) b->item_entries[i] = kfirst[i + 1] - kfirst[i];

    // (2) entries of every item in one key space, one stable sort, per-tile ranges
    uint32_t *k0, *v0, *k1, *v1, *list = nullptr;
    const size_t cap = (size_t)std::max<int64_t>(std::max<int64_t>(total, b->n_tiles), 1);
    KIWI_TRY(scratch_t(ctx, S_KEYS0, cap, &k0));
    KIWI_TRY(scratch_t(ctx, S_VALS0, cap, &v0));
    KIWI_TRY(scratch_t(ctx, S_KEYS1, cap, &k1));
    KIWI_TRY(scratch_t(ctx, S_VALS1, cap, &v1));
    KIWI_TRY(balloc(b, (size_t)std::max<int64_t>(total, 1), &list));
    for (int i = 0; i < n; ++i) {
        const int64_t cnt = b->item_entries[i];
        if (cnt <= 0) continue;
        const BatchItemDev& d = b->items[i];
        k_tile_emit<<<(unsigned)((cnt + 255) / 256), 256, 0, ctx->stream>>>(d.g, d.P.n, offs + pbase[i], boxes + pbase[i],
                                                                          kfirst[i], cnt, (uint32_t)d.tile_base, k0, v0);
        KIWI_LAUNCHED(ctx);
    }
    KIWI_CUDA(ctx, cudaMemsetAsync(b->d_range, 0, sizeof(int64_t) * 2 * b->n_tiles, ctx->stream));
    if (total > 0) {
        int key_bits = 1;
        while ((1LL << key_bits) < b->n_tiles) ++key_bits;
        bool second = false;
        KIWI_TRY(radix_sort_pairs(ctx, k0, v0, k1, v1, total, key_bits, &second));
        k_tile_ranges<<<(unsigned)((total + 255) / 256), 256, 0, ctx->stream>>>(second ? k1 : k0, total, b->d_range);
        KIWI_LAUNCHED(ctx);
        KIWI_CUDA(ctx, cudaMemcpyAsync(list, second ? v1 : v0, sizeof(uint32_t) * total, cudaMemcpyDeviceToDevice,
                                       ctx->stream));
    }
    b->d_list = list;

    // (3) which item owns each tile; the longest-first tile order
    for (int i = 0; i < n; ++i) {
        const int64_t nt = b->tile_base[i + 1] - b->tile_base[i];
        k_fill_i32<<<(unsigned)((nt + 255) / 256), 256, 0, ctx->stream>>>(b->d_item_of_tile + b->tile_base[i], nt, i);
        KIWI_LAUNCHED(ctx);
    }
    for (int f = 0; f <= kBatchFamilies; ++f) {
        const int64_t nf = f < kBatchFamilies ? b->fam_tiles[f] : b->merged_tiles;
        if (nf <= 0) continue;
        const int32_t* nat_f = f < kBatchFamilies ? b->d_natural[f] : b->d_natural_m;
        int32_t* lpt_f = f < kBatchFamilies ? b->d_lpt[f] : b->d_lpt_m;
        k_tile_weights<<<(unsigned)((nf + 255) / 256), 256, 0, ctx->stream>>>(b->d_range, nat_f, nf, k0, v0);
        KIWI_LAUNCHED(ctx);
        bool second = false;
        KIWI_TRY(radix_sort_pairs(ctx, k0, v0, k1, v1, nf, 32, &second));
        KIWI_CUDA(ctx, cudaMemcpyAsync(lpt_f, second ? v1 : v0, sizeof(int32_t) * nf, cudaMemcpyDeviceToDevice,
                                       ctx->stream));
    }
    KIWI_CUDA(ctx, cudaMemcpyAsync(b->d_items, b->items.data(), sizeof(BatchItemDev) * n, cudaMemcpyHostToDevice,
                                   ctx->stream));
    DevStats* hs = nullptr;
    std::vector<DevStats> h(n);
    hs = h.data();
    KIWI_CUDA(ctx, cudaMemcpyAsync(hs, b->d_stats, sizeof(DevStats) * n, cudaMemcpyDeviceToHost, ctx->stream));
    KIWI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    b->item_skipped.resize(n);
    for (int i = 0; i < n; ++i) b->item_skipped[i] = (int64_t)h[i].skipped_outside;

    KIWI_TRY(fp64_batch_prepare(ctx));
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, ctx->device);
    return batch_record(b);
}

int batch_time_once(KiwiBatch* b, float* ms) {
    KiwiCtx* ctx = b->ctx;
    KIWI_CUDA(ctx, cudaEventRecord(ctx->ev[2], ctx->stream));
    KIWI_CUDA(ctx, cudaGraphLaunch(b->exec, ctx->stream));
    KIWI_CUDA(ctx, cudaEventRecord(ctx->ev[3], ctx->stream));
    KIWI_CUDA(ctx, cudaEventSynchronize(ctx->ev[3]));
    KIWI_CUDA(ctx, cudaEventElapsedTime(ms, ctx->ev[2], ctx->ev[3]));
    return KIWI_OK;
}

}  // namespace

extern "C" {

int kiwi_batch_create(KiwiCtx* ctx, const KiwiBatchItem* items, int n_items, int precision, KiwiBatch** out) {
    if (!ctx || !out) return KIWI_ERR_ARG;
    *out = nullptr;
    KIWI_CUDA(ctx, cudaSetDevice(ctx->device));
    if (n_items <= 0 || !items) return set_err(ctx, KIWI_ERR_ARG, "batch: no items");
    const int form = precision & KIWI_FORM_MASK;
    if (precision & ~KIWI_FORM_MASK)
        return set_err(ctx, KIWI_ERR_ARG, "batch: flags (KIWI_FULL_BOX, KIWI_FP32_GUARANTEE) are not supported");
    if (form != KIWI_FP64 && form != KIWI_FP64_REFERENCE_ORDER && form != KIWI_FP32_MIXED)
        return set_err(ctx, KIWI_ERR_UNSUPPORTED, "batch: precision %d is not available", precision);
    KiwiBatch* b = new KiwiBatch();
    b->ctx = ctx;
    b->n_items = n_items;
    b->precision = precision;
    const int rc = batch_build(b, items);
    if (rc != KIWI_OK) {
        batch_free(b);
        delete b;
        return rc;
    }
    *out = b;
    return KIWI_OK;
}

int kiwi_batch_run(KiwiBatch* b, KiwiStats* item_stats, KiwiStats* total) {
    if (!b) return KIWI_ERR_ARG;
    KiwiCtx* ctx = b->ctx;
    KIWI_CUDA(ctx, cudaSetDevice(ctx->device));
    const int64_t launches0 = ctx->launches;
    float ms = 0.f;
    KIWI_TRY(batch_time_once(b, &ms));
    std::vector<DevStats> h(b->n_items);
    KIWI_CUDA(ctx, cudaMemcpy(h.data(), b->d_stats, sizeof(DevStats) * b->n_items, cudaMemcpyDeviceToHost));
    int64_t kernels = b->n_items;  // mean velocities, then one gather launch per family present
    for (int f = 0; f < kBatchFamilies; ++f) kernels += b->fam_tiles[f] > 0 ? 1 : 0;
    (void)launches0;
    KiwiStats sum{};
    for (int i = 0; i < b->n_items; ++i) {
        KiwiStats s{};
        s.bbox_pairs = (int64_t)h[i].bbox_pairs;
        s.sphere_pairs = (int64_t)h[i].sphere_pairs;
        s.evaluated_pairs = (int64_t)h[i].evaluated_pairs;
        s.skipped_outside = b->item_skipped[i];
        s.neg_clamped = (int64_t)h[i].neg_clamped;
        s.neg_warned = (int64_t)h[i].neg_warned;
        s.tile_pairs = b->item_entries[i];
        s.launches = kernels;
        s.gather_ms = ms;
        s.total_ms = ms;
        s.edge_tiers_outer = (int64_t)h[i].edge_outer;
        s.edge_tiers_middle = (int64_t)h[i].edge_middle;
        s.edge_tiers_inner = (int64_t)h[i].edge_inner;
        s.vertex_pyramids = (int64_t)h[i].vertex_pyramids;
        if (item_stats) item_stats[i] = s;
        sum.bbox_pairs += s.bbox_pairs;
        sum.sphere_pairs += s.sphere_pairs;
        sum.evaluated_pairs += s.evaluated_pairs;
        sum.skipped_outside += s.skipped_outside;
        sum.neg_clamped += s.neg_clamped;
        sum.neg_warned += s.neg_warned;
        sum.tile_pairs += s.tile_pairs;
        sum.edge_tiers_outer += s.edge_tiers_outer;
        sum.edge_tiers_middle += s.edge_tiers_middle;
        sum.edge_tiers_inner += s.edge_tiers_inner;
        sum.vertex_pyramids += s.vertex_pyramids;
    }
    sum.launches = kernels;
    sum.gather_ms = ms;
    sum.total_ms = ms;
    if (total) *total = sum;
    return KIWI_OK;
}

int kiwi_batch_tune(KiwiBatch* b, int* chosen) {
    if (!b) return KIWI_ERR_ARG;
    KiwiCtx* ctx = b->ctx;
    KIWI_CUDA(ctx, cudaSetDevice(ctx->device));
    float best = 1e30f;
    bool best_lpt = b->lpt, best_merge = b->merge;
    int best_ctas = b->ctas_per_sm;
    const bool both = b->fam_tiles[kBatchFamilyLattice] > 0 && b->fam_tiles[kBatchFamilyLatticeGeneric] > 0;
    for (int merge = both ? 1 : 0; merge >= 0; --merge) {
        for (int lpt = 1; lpt >= 0; --lpt) {
            for (int ctas = 1; ctas <= 2; ++ctas) {
                b->merge = merge != 0;
                b->lpt = lpt != 0;
                b->ctas_per_sm = ctas;
                KIWI_TRY(batch_record(b));
                float ms = 0.f;
                KIWI_TRY(batch_time_once(b, &ms));
                if (ms < best) {
                    best = ms;
                    best_lpt = b->lpt;
                    best_ctas = ctas;
                    best_merge = b->merge;
                }
            }
        }
    }
    b->lpt = best_lpt;
    b->ctas_per_sm = best_ctas;
    b->merge = best_merge;
    KIWI_TRY(batch_record(b));
    if (chosen) *chosen = (best_merge ? 0x10000 : 0) | (best_lpt ? 0x100 : 0) | best_ctas;
    return KIWI_OK;
}

void kiwi_batch_destroy(KiwiBatch* b) {
    if (!b) return;
    cudaSetDevice(b->ctx->device);
    batch_free(b);
    delete b;
}

}  // extern "C"
