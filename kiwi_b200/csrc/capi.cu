// The C ABI (include/kiwi_b200.h): context management, the batched scalar integral API, and the
// sph-to-grid pipeline -- particle binning into cell tiles, then the cell-integral gather.
#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstring>
#include <string>
#include <new>
#include <vector>

#include "../../include/kiwi_b200.h"
#include "engine.hpp"
#include "kernel_tables.h"
#include "binning.cuh"
#include "prims.cuh"

using namespace kiwi_b200;

namespace {

// Heaviest-first order of a grid's tiles (build parameter; 1 in the default build).
#ifndef KIWI_TILE_LPT
#define KIWI_TILE_LPT 1
#endif
constexpr bool kTileLpt = KIWI_TILE_LPT != 0;

// sort keys of the heaviest-first tile order: descending (tile, particle) entry count, value the tile
__global__ void k_tile_order_keys(const int64_t* __restrict__ range, int64_t ntiles, uint32_t* __restrict__ keys,
                                  uint32_t* __restrict__ vals) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntiles) return;
    const int64_t e = range[2 * t + 1] - range[2 * t];
    keys[t] = 0xffffffffu - (uint32_t)(e < 0xffffffffLL ? e : 0xffffffffLL);
    vals[t] = (uint32_t)t;
}

}  // namespace

namespace kiwi_b200 {

int resolve_kernel(KiwiCtx* ctx, const KiwiKernelSel* sel, KernelChoice* out) {
    const int k = sel ? sel->kernel : 0;
    if (k < 0 || k >= KIWI_NUM_KERNELS) return set_err(ctx, KIWI_ERR_ARG, "unknown kernel index %d", k);
    double sup = sel ? sel->support_in_h : 0.0;
    if (sup < 0.0) return set_err(ctx, KIWI_ERR_ARG, "kernel.support_radius_in_h must be > 0 (or 0 for the default)");
    if (sup == 0.0) sup = kiwi_kernel_tables[k].radkern;
    const bool generic_path = sel && sel->generic_path;
    // Config::use_generic_kernel_path (src/config.cpp:275-277)
    const bool generic = generic_path || k != 0 || sup != 2.0;
    const bool tab = sel && sel->tabulated;
    if (generic && tab)
        return set_err(ctx, KIWI_ERR_ARG,
                       "use_tabulated_integral is only available for the cubic spline kernel with its default support "
                       "radius (and kernel.generic_path unset)");
    out->cubic = !generic;
    out->tabulated = tab;
    out->kernel = k;
    out->support_in_h = sup;
    return KIWI_OK;
}

int make_geom(KiwiCtx* ctx, const KiwiCartGrid* grid, double support_in_h, CartGeom* g) {
    if (!grid) return set_err(ctx, KIWI_ERR_ARG, "grid is null");
    const double* b = grid->bounds;
    if (!(b[0] < b[1])) return set_err(ctx, KIWI_ERR_ARG, "domain.x_min must be < domain.x_max");
    if (!(b[2] < b[3])) return set_err(ctx, KIWI_ERR_ARG, "domain.y_min must be < domain.y_max");
    if (!(b[4] < b[5])) return set_err(ctx, KIWI_ERR_ARG, "domain.z_min must be < domain.z_max");
    if (grid->nx <= 0 || grid->ny <= 0 || grid->nz <= 0)
        return set_err(ctx, KIWI_ERR_ARG, "cartesian_grid resolution (resolved nx/ny/nz) must be > 0");
    g->x_min = b[0];
    g->y_min = b[2];
    g->z_min = b[4];
    g->nx = grid->nx;
    g->ny = grid->ny;
    g->nz = grid->nz;
    g->dpx = (b[1] - b[0]) / grid->nx;
    g->dpy = (b[3] - b[2]) / grid->ny;
    g->dpz = (b[5] - b[4]) / grid->nz;
    g->hpx = 0.5 * g->dpx;
    g->hpy = 0.5 * g->dpy;
    g->hpz = 0.5 * g->dpz;
    g->cell_volume = g->dpx * g->dpy * g->dpz;
    g->ntx = (g->nx + kTileX - 1) / kTileX;
    g->nty = (g->ny + kTileY - 1) / kTileY;
    g->ntz = (g->nz + kTileZ - 1) / kTileZ;
    g->support_in_h = support_in_h;
    const int64_t nt = (int64_t)g->ntx * g->nty * g->ntz;
    if (nt >= (1LL << 31)) return set_err(ctx, KIWI_ERR_ARG, "grid too large (%lld tiles)", (long long)nt);
    return KIWI_OK;
}

int check_ctx(KiwiCtx* ctx) {
    if (!ctx) return KIWI_ERR_ARG;
    KIWI_CUDA(ctx, cudaSetDevice(ctx->device));
    return KIWI_OK;
}

// The full device pipeline of one sph-to-grid call: mean velocity, binning, gather.
int sph_to_grid_dev(KiwiCtx* ctx, const DevParticles& P, const CartGeom& g, const KernelChoice& kc_in, int precision,
                    const CartOutputs& out_in, KiwiStats* stats, int part, int n_parts) {
    if (n_parts < 1 || n_parts > 65536 || part < 0 || part >= n_parts)
        return set_err(ctx, KIWI_ERR_ARG, "part %d of %d parts is out of range (1 <= parts <= 65536)", part, n_parts);
    if (n_parts > 1 && (precision & KIWI_FP32_GUARANTEE))
        return set_err(ctx, KIWI_ERR_ARG, "KIWI_FP32_GUARANTEE needs the whole grid (n_parts = 1)");
    KernelChoice kc = kc_in;
    if (kc.tabulated) {
        if (ctx->arena)
            return set_err(ctx, KIWI_ERR_UNSUPPORTED,
                           "the tabulated integral needs a context holding its table (not the allocation-free call)");
        if ((precision & KIWI_FORM_MASK) == KIWI_FP32_MIXED)
            return set_err(ctx, KIWI_ERR_UNSUPPORTED, "the FP32-mixed form is available for the analytic integral only");
        KIWI_TRY(table_ensure(ctx, &kc.tab));
    }
    const int64_t launches0 = ctx->launches;
    DevStats* d_stats = nullptr;
    double* d_meanv = nullptr;
    KIWI_TRY(scratch_t(ctx, S_STATS, 1, &d_stats));
    KIWI_TRY(scratch_t(ctx, S_MEANV, 4, &d_meanv));
    KIWI_CUDA(ctx, cudaMemsetAsync(d_stats, 0, sizeof(DevStats), ctx->stream));
    CartOutputs out = out_in;
    out.meanv = d_meanv;
    KIWI_TRY(fp64_mean_velocity(ctx, P, d_meanv));

    const int64_t n = P.n;
    const int64_t ntiles = (int64_t)g.ntx * g.nty * g.ntz;
    uint32_t* counts = nullptr;
    TileBox* boxes = nullptr;
    int64_t* offs = nullptr;
    int64_t* range = nullptr;
    KIWI_TRY(scratch_t(ctx, S_COUNT, (size_t)std::max<int64_t>(n, 1), &counts));
    KIWI_TRY(scratch_t(ctx, S_BOX, (size_t)std::max<int64_t>(n, 1), &boxes));
    KIWI_TRY(scratch_t(ctx, S_OFFS, (size_t)std::max<int64_t>(n, 1) + 1, &offs));
    KIWI_TRY(scratch_t(ctx, S_TILE_RANGE, (size_t)(2 * ntiles), &range));
    int64_t* d_total = offs + std::max<int64_t>(n, 1);
    KIWI_CUDA(ctx, cudaMemsetAsync(range, 0, sizeof(int64_t) * 2 * ntiles, ctx->stream));
    if (n > 0) {
        k_tile_counts<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(g, P, counts, boxes, d_stats);
        KIWI_LAUNCHED(ctx);
    }
    KIWI_TRY(exclusive_scan<uint32_t>(ctx, counts, n, offs, d_total));
    int64_t total = 0;
    KIWI_CUDA(ctx, cudaMemcpyAsync(&total, d_total, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
    KIWI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (total >= (1LL << 32)) return set_err(ctx, KIWI_ERR_LIMIT, "too many (tile, particle) entries: %lld", (long long)total);

    uint32_t *k0, *v0, *k1, *v1;
    KIWI_TRY(scratch_t(ctx, S_KEYS0, (size_t)std::max<int64_t>(total, 1), &k0));
    KIWI_TRY(scratch_t(ctx, S_VALS0, (size_t)std::max<int64_t>(total, 1), &v0));
    KIWI_TRY(scratch_t(ctx, S_KEYS1, (size_t)std::max<int64_t>(total, 1), &k1));
    KIWI_TRY(scratch_t(ctx, S_VALS1, (size_t)std::max<int64_t>(total, 1), &v1));
    const uint32_t* sorted_vals = v0;
    if (total > 0) {
        k_tile_emit<<<(unsigned)((total + 255) / 256), 256, 0, ctx->stream>>>(g, n, offs, boxes, 0, total, 0u, k0, v0);
        KIWI_LAUNCHED(ctx);
        int key_bits = 1;
        while ((1LL << key_bits) < ntiles) ++key_bits;
        bool second = false;
        KIWI_TRY(radix_sort_pairs(ctx, k0, v0, k1, v1, total, key_bits, &second));
        const uint32_t* sk = second ? k1 : k0;
        sorted_vals = second ? v1 : v0;
        k_tile_ranges<<<(unsigned)((total + 255) / 256), 256, 0, ctx->stream>>>(sk, total, range);
        KIWI_LAUNCHED(ctx);
    }
    TileLists tl{sorted_vals, range, ntiles};
    if (n_parts > 1) {
        // this part's tiles: a contiguous run of the tile order holding ~1/n_parts of the entries
        uint32_t *w = nullptr, *flags = nullptr;
        int64_t* prefix = nullptr;
        int32_t* map = nullptr;
        KIWI_TRY(scratch_t(ctx, S_PART_W, (size_t)ntiles, &w));
        KIWI_TRY(scratch_t(ctx, S_PART_PREFIX, (size_t)ntiles + 1, &prefix));
        KIWI_TRY(scratch_t(ctx, S_PART_FLAGS, (size_t)ntiles, &flags));
        KIWI_TRY(scratch_t(ctx, S_TILE_MAP, (size_t)ntiles, &map));
        const unsigned nb = (unsigned)((ntiles + 255) / 256);
        k_tile_entry_counts<<<nb, 256, 0, ctx->stream>>>(range, ntiles, w);
        KIWI_LAUNCHED(ctx);
        KIWI_TRY(exclusive_scan<uint32_t>(ctx, w, ntiles, prefix, prefix + ntiles));
        k_tile_part_flags<<<nb, 256, 0, ctx->stream>>>(prefix, prefix + ntiles, ntiles, part, n_parts, flags);
        KIWI_LAUNCHED(ctx);
        int64_t* moffs = nullptr;
        KIWI_TRY(scratch_t(ctx, S_PART_OFFS, (size_t)ntiles + 1, &moffs));
        KIWI_TRY(exclusive_scan<uint32_t>(ctx, flags, ntiles, moffs, moffs + ntiles));
        k_compact_map<<<nb, 256, 0, ctx->stream>>>(flags, moffs, ntiles, map);
        KIWI_LAUNCHED(ctx);
        int64_t nmap = 0;
        KIWI_CUDA(ctx, cudaMemcpyAsync(&nmap, moffs + ntiles, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
        KIWI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        tl.map = map;
        tl.nmap = nmap;
    } else if (kTileLpt && !ctx->arena && ntiles > 1 && total > 0) {
        // the whole grid, heaviest tiles first (by (tile, particle) entry count; ties in tile order), so that
        // the dense tiles of a clustered field do not start last and leave the SMs a tail
        uint32_t *lk0, *lv0, *lk1, *lv1;
        KIWI_TRY(scratch_t(ctx, S_LPT_K0, (size_t)ntiles, &lk0));
        KIWI_TRY(scratch_t(ctx, S_LPT_V0, (size_t)ntiles, &lv0));
        KIWI_TRY(scratch_t(ctx, S_LPT_K1, (size_t)ntiles, &lk1));
        KIWI_TRY(scratch_t(ctx, S_LPT_V1, (size_t)ntiles, &lv1));
        k_tile_order_keys<<<(unsigned)((ntiles + 255) / 256), 256, 0, ctx->stream>>>(range, ntiles, lk0, lv0);
        KIWI_LAUNCHED(ctx);
        bool second = false;
        KIWI_TRY(radix_sort_pairs(ctx, lk0, lv0, lk1, lv1, ntiles, 32, &second));
        tl.map = reinterpret_cast<const int32_t*>(second ? lv1 : lv0);
        tl.nmap = ntiles;
    }

    KIWI_CUDA(ctx, cudaEventRecord(ctx->ev[0], ctx->stream));
    const int form = precision & KIWI_FORM_MASK;
    const bool full_box = (precision & KIWI_FULL_BOX) != 0;
    int64_t fp64_tiles = 0;
    if ((precision & KIWI_FP32_GUARANTEE) && form != KIWI_FP32_MIXED)
        return set_err(ctx, KIWI_ERR_ARG, "KIWI_FP32_GUARANTEE applies to the FP32-mixed form only");
    if (form == KIWI_FP64 || form == KIWI_FP64_REFERENCE_ORDER) {
        KIWI_TRY(fp64_cart_gather(ctx, g, P, kc, tl, out, d_stats, full_box, form == KIWI_FP64_REFERENCE_ORDER));
    } else if (form == KIWI_FP32_MIXED) {
        if (full_box) return set_err(ctx, KIWI_ERR_ARG, "KIWI_FULL_BOX is available with the FP64 forms only");
        const bool guarantee = (precision & KIWI_FP32_GUARANTEE) != 0;
        if (guarantee && !kc.cubic)
            return set_err(ctx, KIWI_ERR_UNSUPPORTED,
                           "KIWI_FP32_GUARANTEE is available for the cubic spline kernel with support 2h");
        const int64_t ncell = (int64_t)g.nx * g.ny * g.nz;
        double *cerr = nullptr, *cmass = nullptr;
        if (guarantee) {
            KIWI_TRY(scratch_t(ctx, S_CELL_ERR, (size_t)ncell, &cerr));
            KIWI_TRY(scratch_t(ctx, S_CELL_MASS, (size_t)ncell, &cmass));
        }
        if (guarantee)
            KIWI_TRY(mixed_cart_gather(ctx, g, P, tl, out, cerr, cmass, d_stats));
        else
            KIWI_TRY(lattice_mixed_gather(ctx, g, P, kc, tl, out, d_stats));
        if (guarantee) {
            int32_t* map = nullptr;
            int64_t* d_nmap = nullptr;
            DevStats* d_st2 = nullptr;
            KIWI_TRY(scratch_t(ctx, S_TILE_MAP, (size_t)ntiles, &map));
            KIWI_TRY(scratch_t(ctx, S_NMAP, 1, &d_nmap));
            KIWI_TRY(scratch_t(ctx, S_STATS2, 1, &d_st2));
            KIWI_TRY(mixed_flag_tiles(ctx, g, cerr, cmass, 1e-6, 1e-6, map, d_nmap));
            KIWI_CUDA(ctx, cudaMemcpyAsync(&fp64_tiles, d_nmap, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
            KIWI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            KIWI_CUDA(ctx, cudaMemsetAsync(d_st2, 0, sizeof(DevStats), ctx->stream));
            TileLists tl2 = tl;
            tl2.map = map;
            tl2.nmap = fp64_tiles;
            KIWI_TRY(fp64_cart_gather(ctx, g, P, kc, tl2, out, d_st2, false, false));
        }
    } else {
        return set_err(ctx, KIWI_ERR_UNSUPPORTED, "precision %d is not available in this library", precision);
    }
    KIWI_CUDA(ctx, cudaEventRecord(ctx->ev[1], ctx->stream));

    DevStats hs;
    KIWI_CUDA(ctx, cudaMemcpyAsync(&hs, d_stats, sizeof hs, cudaMemcpyDeviceToHost, ctx->stream));
    KIWI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (stats) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
        stats->bbox_pairs = (int64_t)hs.bbox_pairs;
        stats->sphere_pairs = (int64_t)hs.sphere_pairs;
        stats->evaluated_pairs = (int64_t)hs.evaluated_pairs;
        stats->skipped_outside = (int64_t)hs.skipped_outside;
        stats->neg_clamped = (int64_t)hs.neg_clamped;
        stats->neg_warned = (int64_t)hs.neg_warned;
        stats->fp64_fallback = (int64_t)hs.fp64_fallback;
        stats->tile_pairs = total;
        stats->gather_ms = ms;
        stats->launches = ctx->launches - launches0;
        stats->edge_tiers_outer = (int64_t)hs.edge_outer;
        stats->edge_tiers_middle = (int64_t)hs.edge_middle;
        stats->edge_tiers_inner = (int64_t)hs.edge_inner;
        stats->vertex_pyramids = (int64_t)hs.vertex_pyramids;
        stats->fp64_tiles = fp64_tiles;
        stats->table_clamps = (int64_t)hs.table_clamps;
    }
    return KIWI_OK;
}

bool particles_ok(KiwiCtx* ctx, const KiwiParticles* p, int* rc) {
    if (!p) {
        *rc = set_err(ctx, KIWI_ERR_ARG, "particles is null");
        return false;
    }
    if (p->n < 0 || p->n >= (1LL << 32)) {
        *rc = set_err(ctx, KIWI_ERR_ARG, "particle count %lld out of range", (long long)p->n);
        return false;
    }
    if (p->n > 0 && (!p->x || !p->y || !p->z || !p->vx || !p->vy || !p->vz || !p->m || !p->h)) {
        *rc = set_err(ctx, KIWI_ERR_ARG, "a particle array is null");
        return false;
    }
    return true;
}

}  // namespace kiwi_b200

extern "C" {

const char* kiwi_version(void) { return "kiwi_b200 0.1.0 (sm_100a)"; }

int kiwi_ctx_create(int device, KiwiCtx** out) {
    if (!out) return KIWI_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return KIWI_ERR_NODEV;
    }
    if (device < 0 || device >= ndev) return KIWI_ERR_NODEV;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major < 10) return KIWI_ERR_NODEV;
    KiwiCtx* ctx = new KiwiCtx();
    ctx->device = device;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return KIWI_ERR_CUDA;
    }
    for (auto& ev : ctx->ev) cudaEventCreate(&ev);
    if (fp64_init_tables(ctx) != KIWI_OK || voronoi_init_tables(ctx) != KIWI_OK) {
        kiwi_ctx_destroy(ctx);
        return KIWI_ERR_CUDA;
    }
    *out = ctx;
    return KIWI_OK;
}

void kiwi_ctx_destroy(KiwiCtx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    table_free(ctx);
    for (int i = 0; i < KiwiCtx::kSlots; ++i)
        if (ctx->slot_ptr[i]) cudaFree(ctx->slot_ptr[i]);
    for (auto& ev : ctx->ev)
        if (ev) cudaEventDestroy(ev);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char* kiwi_last_error(const KiwiCtx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

void* kiwi_ctx_stream(KiwiCtx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int kiwi_ctx_synchronize(KiwiCtx* ctx) {
    KIWI_TRY(check_ctx(ctx));
    KIWI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return KIWI_OK;
}

int kiwi_ctx_set_voronoi_face_tables(KiwiCtx* ctx, int enable) {
    KIWI_TRY(check_ctx(ctx));
    ctx->face_tables = enable != 0;
    return KIWI_OK;
}

int kiwi_measure_fp64_peak(KiwiCtx* ctx, double* tflops) {
    KIWI_TRY(check_ctx(ctx));
    if (!tflops) return set_err(ctx, KIWI_ERR_ARG, "tflops is null");
    return fp64_measure_peak(ctx, tflops);
}

int kiwi_measure_fp32_peak(KiwiCtx* ctx, double* tflops) {
    KIWI_TRY(check_ctx(ctx));
    if (!tflops) return set_err(ctx, KIWI_ERR_ARG, "tflops is null");
    return fp32_measure_peak(ctx, tflops);
}

int kiwi_kernel_index(const char* name) {
    if (!name) return -1;
    std::string n(name);
    std::transform(n.begin(), n.end(), n.begin(), [](unsigned char c) { return (char)std::tolower(c); });
    std::replace(n.begin(), n.end(), '-', '_');
    std::replace(n.begin(), n.end(), ' ', '_');
    // the aliases accepted by get_kernel (src/kernel_spec_data.cpp:175-187)
    static const char* const names[KIWI_NUM_KERNELS][3] = {
        {"cubic", "cubic_spline", "m4"},          {"quartic", "quartic_spline", "m5"},
        {"quintic", "quintic_spline", "m6"},      {"wendland_c2", "wendlandc2", "wc2"},
        {"wendland_c4", "wendlandc4", "wc4"},     {"wendland_c6", "wendlandc6", "wc6"}};
    for (int k = 0; k < KIWI_NUM_KERNELS; ++k)
        for (int a = 0; a < 3; ++a)
            if (n == names[k][a]) return k;
    return -1;
}

int kiwi_kernel_info(int kernel, double* out7) {
    if (kernel < 0 || kernel >= KIWI_NUM_KERNELS || !out7) return KIWI_ERR_ARG;
    const KiwiKernelTable& K = kiwi_kernel_tables[kernel];
    out7[0] = K.nreg;
    out7[1] = K.A2_pi;
    out7[2] = K.A3_pi;
    out7[3] = K.radkern;
    out7[4] = K.hfact;
    out7[5] = K.c[0];
    out7[6] = K.c[1];
    return KIWI_OK;
}

int kiwi_full_integral_batch(KiwiCtx* ctx, int kernel, int64_t n, const double* arg0, const double* phi,
                             const double* r0, const double* R_0, double* out) {
    KIWI_TRY(check_ctx(ctx));
    if (kernel >= KIWI_NUM_KERNELS) return set_err(ctx, KIWI_ERR_ARG, "unknown kernel index %d", kernel);
    if (n < 0 || (n > 0 && (!arg0 || !phi || !r0 || !R_0 || !out))) return set_err(ctx, KIWI_ERR_ARG, "bad arrays");
    if (n == 0) return KIWI_OK;
    double* d = nullptr;
    KIWI_TRY(scratch_t(ctx, S_MISC0, (size_t)(5 * n), &d));
    const size_t b = sizeof(double) * n;
    KIWI_CUDA(ctx, cudaMemcpyAsync(d, arg0, b, cudaMemcpyHostToDevice, ctx->stream));
    KIWI_CUDA(ctx, cudaMemcpyAsync(d + n, phi, b, cudaMemcpyHostToDevice, ctx->stream));
    KIWI_CUDA(ctx, cudaMemcpyAsync(d + 2 * n, r0, b, cudaMemcpyHostToDevice, ctx->stream));
    KIWI_CUDA(ctx, cudaMemcpyAsync(d + 3 * n, R_0, b, cudaMemcpyHostToDevice, ctx->stream));
    KIWI_TRY(fp64_full_integral(ctx, kernel < 0 ? -1 : kernel, n, d, d + n, d + 2 * n, d + 3 * n, d + 4 * n));
    KIWI_CUDA(ctx, cudaMemcpyAsync(out, d + 4 * n, b, cudaMemcpyDeviceToHost, ctx->stream));
    KIWI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return KIWI_OK;
}

int kiwi_tier_constants_batch(KiwiCtx* ctx, int kernel, int64_t n, const double* arg0, const double* r0,
                              const double* R_0, double* wall_out, double* edge_out) {
    KIWI_TRY(check_ctx(ctx));
    if (kernel >= KIWI_NUM_KERNELS) return set_err(ctx, KIWI_ERR_ARG, "unknown kernel index %d", kernel);
    if (n < 0 || (n > 0 && (!arg0 || !r0 || !R_0 || !wall_out || !edge_out)))
        return set_err(ctx, KIWI_ERR_ARG, "bad arrays");
    if (n == 0) return KIWI_OK;
    const int nw = kernel < 0 ? KIWI_CUBIC_WALL_DOUBLES : KIWI_GENERIC_WALL_DOUBLES;
    const int ne = kernel < 0 ? KIWI_CUBIC_EDGE_DOUBLES : KIWI_GENERIC_EDGE_DOUBLES;
    double* d = nullptr;
    KIWI_TRY(scratch_t(ctx, S_MISC0, (size_t)((3 + nw + ne) * n), &d));
    const size_t b = sizeof(double) * n;
    KIWI_CUDA(ctx, cudaMemcpyAsync(d, arg0, b, cudaMemcpyHostToDevice, ctx->stream));
    KIWI_CUDA(ctx, cudaMemcpyAsync(d + n, r0, b, cudaMemcpyHostToDevice, ctx->stream));
    KIWI_CUDA(ctx, cudaMemcpyAsync(d + 2 * n, R_0, b, cudaMemcpyHostToDevice, ctx->stream));
    double* dw = d + 3 * n;
    double* de = dw + (size_t)nw * n;
    KIWI_TRY(fp64_tier_constants(ctx, kernel < 0 ? -1 : kernel, n, d, d + n, d + 2 * n, dw, de));
    KIWI_CUDA(ctx, cudaMemcpyAsync(wall_out, dw, b * nw, cudaMemcpyDeviceToHost, ctx->stream));
    KIWI_CUDA(ctx, cudaMemcpyAsync(edge_out, de, b * ne, cudaMemcpyDeviceToHost, ctx->stream));
    KIWI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return KIWI_OK;
}

int kiwi_face_integral_batch(KiwiCtx* ctx, const KiwiKernelSel* kernel, int64_t n_faces, const double* particle,
                             const int64_t* vert_off, const double* verts, double* out, int32_t* out_vert) {
    KIWI_TRY(check_ctx(ctx));
    KernelChoice kc;
    KIWI_TRY(resolve_kernel(ctx, kernel, &kc));
    if (n_faces < 0 || (n_faces > 0 && (!particle || !vert_off || !verts || !out)))
        return set_err(ctx, KIWI_ERR_ARG, "bad arrays");
    if (n_faces == 0) return KIWI_OK;
    if (kc.tabulated) KIWI_TRY(table_ensure(ctx, &kc.tab));
    const int64_t nv = vert_off[n_faces];
    if (nv < 0 || vert_off[0] != 0) return set_err(ctx, KIWI_ERR_ARG, "vert_off must start at 0 and be non-decreasing");
    for (int64_t i = 0; i < n_faces; ++i)
        if (vert_off[i + 1] < vert_off[i]) return set_err(ctx, KIWI_ERR_ARG, "vert_off must be non-decreasing");
    double *dp = nullptr, *dv = nullptr, *dout = nullptr;
    int64_t* doff = nullptr;
    int32_t* dov = nullptr;
    KIWI_TRY(scratch_t(ctx, S_MISC0, (size_t)(4 * n_faces), &dp));
    KIWI_TRY(scratch_t(ctx, S_MISC1, (size_t)std::max<int64_t>(3 * nv, 1), &dv));
    KIWI_TRY(scratch_t(ctx, S_MISC2, (size_t)(n_faces + 1), &doff));
    KIWI_TRY(scratch_t(ctx, S_OUT, (size_t)n_faces, &dout));
    KIWI_TRY(scratch_t(ctx, S_COUNT, (size_t)n_faces, &dov));
    KIWI_CUDA(ctx, cudaMemcpyAsync(dp, particle, sizeof(double) * 4 * n_faces, cudaMemcpyHostToDevice, ctx->stream));
    if (nv > 0)
        KIWI_CUDA(ctx, cudaMemcpyAsync(dv, verts, sizeof(double) * 3 * nv, cudaMemcpyHostToDevice, ctx->stream));
    KIWI_CUDA(ctx, cudaMemcpyAsync(doff, vert_off, sizeof(int64_t) * (n_faces + 1), cudaMemcpyHostToDevice, ctx->stream));
    KIWI_TRY(fp64_face_integral(ctx, kc, n_faces, dp, doff, dv, dout, dov));
    KIWI_CUDA(ctx, cudaMemcpyAsync(out, dout, sizeof(double) * n_faces, cudaMemcpyDeviceToHost, ctx->stream));
    if (out_vert)
        KIWI_CUDA(ctx, cudaMemcpyAsync(out_vert, dov, sizeof(int32_t) * n_faces, cudaMemcpyDeviceToHost, ctx->stream));
    KIWI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return KIWI_OK;
}

int kiwi_sph_to_grid_device(KiwiCtx* ctx, const KiwiParticles* particles, const KiwiCartGrid* grid,
                            const KiwiKernelSel* kernel, int precision, double* density, double* vx, double* vy,
                            double* vz, double* raw4, KiwiStats* stats) {
    KIWI_TRY(check_ctx(ctx));
    int rc = KIWI_OK;
    if (!particles_ok(ctx, particles, &rc)) return rc;
    KernelChoice kc;
    KIWI_TRY(resolve_kernel(ctx, kernel, &kc));
    CartGeom g;
    KIWI_TRY(make_geom(ctx, grid, kc.support_in_h, &g));
    DevParticles P{particles->n, particles->x, particles->y, particles->z, particles->vx,
                   particles->vy, particles->vz, particles->m, particles->h};
    CartOutputs out{density, vx, vy, vz, raw4, nullptr};
    KIWI_CUDA(ctx, cudaEventRecord(ctx->ev[2], ctx->stream));
    KIWI_TRY(sph_to_grid_dev(ctx, P, g, kc, precision, out, stats));
    KIWI_CUDA(ctx, cudaEventRecord(ctx->ev[3], ctx->stream));
    KIWI_CUDA(ctx, cudaEventSynchronize(ctx->ev[3]));
    if (stats) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]);
        stats->total_ms = ms;
    }
    return KIWI_OK;
}

int kiwi_sph_to_grid_device_part(KiwiCtx* ctx, const KiwiParticles* particles, const KiwiCartGrid* grid,
                                 const KiwiKernelSel* kernel, int precision, int part, int n_parts, double* density,
                                 double* vx, double* vy, double* vz, double* raw4, KiwiStats* stats) {
    KIWI_TRY(check_ctx(ctx));
    int rc = KIWI_OK;
    if (!particles_ok(ctx, particles, &rc)) return rc;
    KernelChoice kc;
    KIWI_TRY(resolve_kernel(ctx, kernel, &kc));
    CartGeom g;
    KIWI_TRY(make_geom(ctx, grid, kc.support_in_h, &g));
    DevParticles P{particles->n, particles->x, particles->y, particles->z, particles->vx,
                   particles->vy, particles->vz, particles->m, particles->h};
    CartOutputs out{density, vx, vy, vz, raw4, nullptr};
    KIWI_CUDA(ctx, cudaEventRecord(ctx->ev[2], ctx->stream));
    KIWI_TRY(sph_to_grid_dev(ctx, P, g, kc, precision, out, stats, part, n_parts));
    KIWI_CUDA(ctx, cudaEventRecord(ctx->ev[3], ctx->stream));
    KIWI_CUDA(ctx, cudaEventSynchronize(ctx->ev[3]));
    if (stats) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]);
        stats->total_ms = ms;
    }
    return KIWI_OK;
}

// Host only: the split of kiwi_sph_to_grid_device_part restated over host arrays -- the same clamped
// support boxes (particle_cell_box), the (tile, particle) entries per tile from a 3-D difference array
// over the particles' tile boxes, and the same integer ownership rule as k_tile_part_flags -- so that a
// rank knows the x rows its part writes before any GPU work.
int kiwi_part_rows(KiwiCtx* ctx, const KiwiParticles* particles, const KiwiCartGrid* grid,
                   const KiwiKernelSel* kernel, int part, int n_parts, int* ix0, int* ix1) {
    try {
        if (!particles || !ix0 || !ix1) return set_err(ctx, KIWI_ERR_ARG, "particles, ix0 and ix1 must not be null");
        if (particles->n < 0 || (particles->n > 0 && (!particles->x || !particles->y || !particles->z || !particles->h)))
            return set_err(ctx, KIWI_ERR_ARG, "particles need n >= 0 and host arrays x, y, z, h");
        if (n_parts < 1 || n_parts > 65536 || part < 0 || part >= n_parts)
            return set_err(ctx, KIWI_ERR_ARG, "part %d of %d parts is out of range (1 <= n_parts <= 65536)", part,
                           n_parts);
        KernelChoice kc;
        KIWI_TRY(resolve_kernel(ctx, kernel, &kc));
        CartGeom g;
        KIWI_TRY(make_geom(ctx, grid, kc.support_in_h, &g));
        const int64_t ntx = g.ntx, nty = g.nty, ntz = g.ntz, nt = ntx * nty * ntz;
        std::vector<int64_t> d((size_t)((ntx + 1) * (nty + 1) * (ntz + 1)), 0);
        auto at = [&](int64_t x, int64_t y, int64_t z) -> int64_t& { return d[(size_t)((x * (nty + 1) + y) * (ntz + 1) + z)]; };
        for (int64_t i = 0; i < particles->n; ++i) {
            CellBox b;
            bool outside = false;
            if (!particle_cell_box(g, particles->x[i], particles->y[i], particles->z[i], particles->h[i], b, &outside))
                continue;
            const int64_t x0 = b.x0 / kTileX, x1 = b.x1 / kTileX + 1, y0 = b.y0 / kTileY, y1 = b.y1 / kTileY + 1,
                          z0 = b.z0 / kTileZ, z1 = b.z1 / kTileZ + 1;
            at(x0, y0, z0) += 1;
            at(x1, y0, z0) -= 1;
            at(x0, y1, z0) -= 1;
            at(x0, y0, z1) -= 1;
            at(x1, y1, z0) += 1;
            at(x1, y0, z1) += 1;
            at(x0, y1, z1) += 1;
            at(x1, y1, z1) -= 1;
        }
        for (int64_t x = 0; x <= ntx; ++x)  // prefix sums along z, y, x give each tile's entry count
            for (int64_t y = 0; y <= nty; ++y)
                for (int64_t z = 1; z <= ntz; ++z) at(x, y, z) += at(x, y, z - 1);
        for (int64_t x = 0; x <= ntx; ++x)
            for (int64_t y = 1; y <= nty; ++y)
                for (int64_t z = 0; z <= ntz; ++z) at(x, y, z) += at(x, y - 1, z);
        for (int64_t x = 1; x <= ntx; ++x)
            for (int64_t y = 0; y <= nty; ++y)
                for (int64_t z = 0; z <= ntz; ++z) at(x, y, z) += at(x - 1, y, z);
        std::vector<int64_t> w((size_t)nt);
        int64_t W = 0;
        for (int64_t t = 0; t < nt; ++t) {
            const int64_t tx = t / (nty * ntz), ty = (t / ntz) % nty, tz = t % ntz;
            w[(size_t)t] = std::min<int64_t>(at(tx, ty, tz), 0xFFFFFFFFLL);  // the device counts tiles in 32 bits
            W += w[(size_t)t];
        }
        int64_t first = -1, last = -1, prefix = 0;
        for (int64_t t = 0; t < nt; ++t) {
            int64_t owner = W > 0 ? (prefix * n_parts) / W : (t * n_parts) / nt;
            if (owner > n_parts - 1) owner = n_parts - 1;
            if (owner == part) {
                if (first < 0) first = t;
                last = t;
            }
            prefix += w[(size_t)t];
        }
        if (first < 0) {
            *ix0 = *ix1 = 0;
        } else {
            *ix0 = (int)(first / (nty * ntz)) * kTileX;
            *ix1 = std::min<int>(g.nx, (int)(last / (nty * ntz) + 1) * kTileX);
        }
        return KIWI_OK;
    } catch (const std::bad_alloc&) {
        return set_err(ctx, KIWI_ERR_ALLOC, "host memory allocation failed");
    }
}

int kiwi_snapshot_work(KiwiCtx* ctx, const KiwiParticles* particles, const KiwiCartGrid* grid,
                       const KiwiKernelSel* kernel, int64_t* bbox_pairs) {
    if (!particles || !bbox_pairs || particles->n < 0 ||
        (particles->n > 0 && (!particles->x || !particles->y || !particles->z || !particles->h)))
        return set_err(ctx, KIWI_ERR_ARG, "particles (host x, y, z, h) and bbox_pairs are needed");
    KernelChoice kc;
    KIWI_TRY(resolve_kernel(ctx, kernel, &kc));
    CartGeom g;
    KIWI_TRY(make_geom(ctx, grid, kc.support_in_h, &g));
    int64_t total = 0;
    for (int64_t i = 0; i < particles->n; ++i) {
        CellBox b;
        bool outside = false;
        if (!particle_cell_box(g, particles->x[i], particles->y[i], particles->z[i], particles->h[i], b, &outside))
            continue;
        total += (int64_t)(b.x1 - b.x0 + 1) * (b.y1 - b.y0 + 1) * (b.z1 - b.z0 + 1);
    }
    *bbox_pairs = total;
    return KIWI_OK;
}

namespace {
// A cell's vertex rows [vert_off[face_off[c]], vert_off[face_off[c + 1]]) (its faces, and their vertices,
// are back to back), checked against the geometry's sizes.
int voronoi_host_rows(KiwiCtx* ctx, const KiwiVoronoiCells* cells, std::vector<int64_t>* start,
                      std::vector<int64_t>* end) {
    if (!cells || cells->n_cells < 0 || (cells->n_cells > 0 && (!cells->face_off || !cells->vert_off || !cells->vxyz)))
        return set_err(ctx, KIWI_ERR_ARG, "cells need n_cells >= 0 and host arrays face_off, vert_off, vxyz");
    const int64_t nc = cells->n_cells;
    start->resize((size_t)nc);
    end->resize((size_t)nc);
    int64_t prev = 0;
    for (int64_t c = 0; c < nc; ++c) {
        const int64_t f0 = cells->face_off[c], f1 = cells->face_off[c + 1];
        if (f0 < 0 || f1 < f0) return set_err(ctx, KIWI_ERR_ARG, "face_off must start at 0 and not decrease");
        const int64_t a = cells->vert_off[f0], b = cells->vert_off[f1];
        if (a < prev || b < a) return set_err(ctx, KIWI_ERR_ARG, "vert_off must not decrease");
        (*start)[(size_t)c] = a;
        (*end)[(size_t)c] = b;
        prev = b;
    }
    return KIWI_OK;
}
}  // namespace

int kiwi_voronoi_cell_owners(KiwiCtx* ctx, const KiwiVoronoiCells* cells, int n_parts, int axis, int32_t* owner) {
    try {
        if (n_parts < 1 || axis < 0 || axis > 2 || (!owner && cells && cells->n_cells > 0))
            return set_err(ctx, KIWI_ERR_ARG, "n_parts must be >= 1, axis 0, 1 or 2, owner non-null");
        std::vector<int64_t> start, end;
        KIWI_TRY(voronoi_host_rows(ctx, cells, &start, &end));
        const int64_t nc = cells->n_cells;
        std::vector<double> mid((size_t)nc, 0.0);
        for (int64_t c = 0; c < nc; ++c) {
            if (end[(size_t)c] <= start[(size_t)c]) continue;
            double lo = cells->vxyz[3 * start[(size_t)c] + axis], hi = lo;
            for (int64_t r = start[(size_t)c] + 1; r < end[(size_t)c]; ++r) {
                const double v = cells->vxyz[3 * r + axis];
                lo = std::min(lo, v);
                hi = std::max(hi, v);
            }
            mid[(size_t)c] = (lo + hi) * 0.5;
        }
        std::vector<int64_t> order((size_t)nc);
        for (int64_t c = 0; c < nc; ++c) order[(size_t)c] = c;
        std::stable_sort(order.begin(), order.end(),
                         [&](int64_t a, int64_t b) { return mid[(size_t)a] < mid[(size_t)b]; });
        for (int64_t k = 0; k < nc; ++k) owner[(size_t)order[(size_t)k]] = (int32_t)((k * n_parts) / nc);
        return KIWI_OK;
    } catch (const std::bad_alloc&) {
        return set_err(ctx, KIWI_ERR_ALLOC, "host memory allocation failed");
    }
}

int kiwi_voronoi_part_particles(KiwiCtx* ctx, const KiwiParticles* particles, const int32_t* home_cell,
                                const KiwiVoronoiCells* cells, const KiwiKernelSel* kernel, const int32_t* owner,
                                int part, uint8_t* select, int64_t* n_selected) {
    try {
        if (!particles || !n_selected || particles->n < 0 ||
            (particles->n > 0 && (!particles->x || !particles->y || !particles->z || !particles->h || !home_cell ||
                                  !select)))
            return set_err(ctx, KIWI_ERR_ARG, "particles (host x, y, z, h), home_cell, select and n_selected are needed");
        std::vector<int64_t> start, end;
        KIWI_TRY(voronoi_host_rows(ctx, cells, &start, &end));
        if (cells->n_cells > 0 && !owner) return set_err(ctx, KIWI_ERR_ARG, "owner is null");
        KernelChoice kc;
        KIWI_TRY(resolve_kernel(ctx, kernel, &kc));
        const int64_t nc = cells->n_cells;
        double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
        bool any = false;
        for (int64_t c = 0; c < nc; ++c) {
            if (owner[(size_t)c] != part) continue;
            for (int64_t r = start[(size_t)c]; r < end[(size_t)c]; ++r)
                for (int a = 0; a < 3; ++a) {
                    const double v = cells->vxyz[3 * r + a];
                    lo[a] = any ? std::min(lo[a], v) : v;
                    hi[a] = any ? std::max(hi[a], v) : v;
                    if (a == 2) any = true;
                }
        }
        const double rscale = 1.001 * kc.support_in_h;
        int64_t count = 0;
        for (int64_t i = 0; i < particles->n; ++i) {
            const int32_t hc = home_cell[i];
            bool s = hc >= 0 && hc < nc && owner[hc] == part;
            if (!s && any) {
                const double c3[3] = {particles->x[i], particles->y[i], particles->z[i]};
                double d2 = 0.0;
                for (int a = 0; a < 3; ++a) {
                    const double t = std::max(std::max(lo[a] - c3[a], c3[a] - hi[a]), 0.0);
                    d2 += t * t;
                }
                const double r = rscale * particles->h[i];
                s = d2 <= r * r;
            }
            select[i] = s ? 1 : 0;
            count += s;
        }
        *n_selected = count;
        return KIWI_OK;
    } catch (const std::bad_alloc&) {
        return set_err(ctx, KIWI_ERR_ALLOC, "host memory allocation failed");
    }
}

int kiwi_sph_to_grid_adjoint_device(KiwiCtx* ctx, const KiwiParticles* particles, const KiwiCartGrid* grid,
                                    const KiwiKernelSel* kernel, const double* d_raw4, double* d_x, double* d_y,
                                    double* d_z, double* d_h, double* d_m, double* d_vx, double* d_vy, double* d_vz,
                                    KiwiStats* stats) {
    KIWI_TRY(check_ctx(ctx));
    int rc = KIWI_OK;
    if (!particles_ok(ctx, particles, &rc)) return rc;
    KernelChoice kc;
    KIWI_TRY(resolve_kernel(ctx, kernel, &kc));
    CartGeom g;
    KIWI_TRY(make_geom(ctx, grid, kc.support_in_h, &g));
    if (!d_raw4 && particles->n > 0) return set_err(ctx, KIWI_ERR_ARG, "adjoint: the cotangent array raw4 is null");
    if (stats) *stats = KiwiStats{};
    DevParticles P{particles->n, particles->x, particles->y, particles->z, particles->vx,
                   particles->vy, particles->vz, particles->m, particles->h};
    AdjointOutputs out{d_x, d_y, d_z, d_h, d_m, d_vx, d_vy, d_vz};
    const int64_t launches0 = ctx->launches;
    KIWI_CUDA(ctx, cudaEventRecord(ctx->ev[2], ctx->stream));
    KIWI_TRY(cart_adjoint_dev(ctx, P, g, kc, d_raw4, out, stats));
    KIWI_CUDA(ctx, cudaEventRecord(ctx->ev[3], ctx->stream));
    KIWI_CUDA(ctx, cudaEventSynchronize(ctx->ev[3]));
    if (stats) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]);
        stats->total_ms = ms;
        stats->gather_ms = ms;
        stats->launches = ctx->launches - launches0;
    }
    return KIWI_OK;
}

int kiwi_sph_to_grid(KiwiCtx* ctx, const KiwiParticles* particles, const KiwiCartGrid* grid,
                     const KiwiKernelSel* kernel, int precision, double* density, double* vx, double* vy, double* vz,
                     double* raw4, KiwiStats* stats) {
    KIWI_TRY(check_ctx(ctx));
    int rc = KIWI_OK;
    if (!particles_ok(ctx, particles, &rc)) return rc;
    KernelChoice kc;
    KIWI_TRY(resolve_kernel(ctx, kernel, &kc));
    CartGeom g;
    KIWI_TRY(make_geom(ctx, grid, kc.support_in_h, &g));
    const int64_t n = particles->n;
    const int64_t ncell = (int64_t)g.nx * g.ny * g.nz;
    double* dpart = nullptr;
    double* dout = nullptr;
    KIWI_TRY(scratch_t(ctx, S_PART, (size_t)std::max<int64_t>(8 * n, 1), &dpart));
    KIWI_TRY(scratch_t(ctx, S_OUT, (size_t)(raw4 ? 8 : 4) * ncell, &dout));
    KIWI_CUDA(ctx, cudaEventRecord(ctx->ev[2], ctx->stream));
    const double* src[8] = {particles->x, particles->y, particles->z, particles->vx,
                            particles->vy, particles->vz, particles->m, particles->h};
    for (int a = 0; a < 8 && n > 0; ++a)
        KIWI_CUDA(ctx, cudaMemcpyAsync(dpart + a * n, src[a], sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
    DevParticles P{n, dpart, dpart + n, dpart + 2 * n, dpart + 3 * n, dpart + 4 * n, dpart + 5 * n, dpart + 6 * n,
                   dpart + 7 * n};
    CartOutputs out{dout, dout + ncell, dout + 2 * ncell, dout + 3 * ncell, raw4 ? dout + 4 * ncell : nullptr, nullptr};
    KIWI_TRY(sph_to_grid_dev(ctx, P, g, kc, precision, out, stats));
    double* dst[4] = {density, vx, vy, vz};
    for (int a = 0; a < 4; ++a)
        if (dst[a])
            KIWI_CUDA(ctx, cudaMemcpyAsync(dst[a], dout + a * ncell, sizeof(double) * ncell, cudaMemcpyDeviceToHost,
                                           ctx->stream));
    if (raw4)
        KIWI_CUDA(ctx, cudaMemcpyAsync(raw4, dout + 4 * ncell, sizeof(double) * 4 * ncell, cudaMemcpyDeviceToHost,
                                       ctx->stream));
    KIWI_CUDA(ctx, cudaEventRecord(ctx->ev[3], ctx->stream));
    KIWI_CUDA(ctx, cudaEventSynchronize(ctx->ev[3]));
    if (stats) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]);
        stats->total_ms = ms;
    }
    return KIWI_OK;
}

}  // extern "C"

namespace {

// Host outputs of the inverse-mapping check (kiwi_inverse_map_voronoi).
struct InverseHost {
    const double* cell_mass;
    double* m_recovered;
    double* coverage;
    double* totals3;
};

// kiwi_map_voronoi on host arrays: stage, map (and with inv, the inverse check), copy back.
int map_voronoi_host(KiwiCtx* ctx, const KiwiParticles* particles, const int32_t* home_cell,
                     const KiwiVoronoiCells* cells, const KiwiKernelSel* kernel, int precision, double* density,
                     double* vx, double* vy, double* vz, double* raw4, KiwiStats* stats, const InverseHost* inv) {
    KIWI_TRY(check_ctx(ctx));
    int rc = KIWI_OK;
    if (!particles_ok(ctx, particles, &rc)) return rc;
    KernelChoice kc;
    KIWI_TRY(resolve_kernel(ctx, kernel, &kc));
    if ((precision & KIWI_FORM_MASK) != KIWI_FP64 && (precision & KIWI_FORM_MASK) != KIWI_FP64_REFERENCE_ORDER)
        return set_err(ctx, KIWI_ERR_UNSUPPORTED, "the Voronoi map is available in the FP64 form only");
    if (kc.tabulated) KIWI_TRY(table_ensure(ctx, &kc.tab));
    if (!cells || cells->n_cells < 0 || (cells->n_cells > 0 && (!cells->face_off || !cells->vert_off ||
                                                                 !cells->vxyz || !cells->face_nbr || !cells->volume)))
        return set_err(ctx, KIWI_ERR_ARG, "cell geometry is incomplete");
    if (particles->n > 0 && !home_cell) return set_err(ctx, KIWI_ERR_ARG, "home_cell is null");
    if (cells->n_cells >= (1LL << 31)) return set_err(ctx, KIWI_ERR_ARG, "too many cells");
    const int64_t n = particles->n, nc = cells->n_cells;
    const int64_t nf = nc > 0 ? cells->face_off[nc] : 0;
    const int64_t nv = nf > 0 ? cells->vert_off[nf] : 0;
    if (nc > 0 && (cells->face_off[0] != 0 || nf < 0 || nv < 0 || (nf > 0 && cells->vert_off[0] != 0)))
        return set_err(ctx, KIWI_ERR_ARG, "face_off / vert_off must start at 0");
    for (int64_t c = 0; c < nc; ++c)
        if (cells->face_off[c + 1] < cells->face_off[c]) return set_err(ctx, KIWI_ERR_ARG, "face_off must not decrease");
    for (int64_t f = 0; f < nf; ++f) {
        if (cells->vert_off[f + 1] < cells->vert_off[f]) return set_err(ctx, KIWI_ERR_ARG, "vert_off must not decrease");
        if (cells->face_nbr[f] >= nc) return set_err(ctx, KIWI_ERR_ARG, "face_nbr out of range");
    }
    for (int64_t i = 0; i < n; ++i)
        if (home_cell[i] >= nc) return set_err(ctx, KIWI_ERR_ARG, "home_cell out of range");
    // stage particles, home cells and geometry
    double* dpart = nullptr;
    int32_t* dhome = nullptr;
    unsigned char* dgeo = nullptr;
    double* dout = nullptr;
    const size_t b_fo = sizeof(int64_t) * (nc + 1), b_vo = sizeof(int64_t) * (nf + 1), b_v = sizeof(double) * 3 * nv;
    const size_t b_nb = sizeof(int32_t) * nf, b_vol = sizeof(double) * nc;
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t geo_bytes = al(b_fo) + al(b_vo) + al(b_v) + al(b_nb) + al(b_vol);
    KIWI_TRY(scratch_t(ctx, S_PART, (size_t)std::max<int64_t>(8 * n, 1), &dpart));
    KIWI_TRY(scratch_t(ctx, S_VOR_HOME, (size_t)std::max<int64_t>(n, 1), &dhome));
    KIWI_TRY(scratch_t(ctx, S_VOR_CSR, geo_bytes, &dgeo));
    KIWI_TRY(scratch_t(ctx, S_OUT, (size_t)(raw4 ? 8 : 4) * std::max<int64_t>(nc, 1), &dout));
    double* dinv = nullptr;  // inverse check: cell masses (given), recovered masses, coverage
    if (inv) KIWI_TRY(scratch_t(ctx, S_INV_OUT, (size_t)(std::max<int64_t>(nc, 1) + 2 * std::max<int64_t>(n, 1)), &dinv));
    KIWI_CUDA(ctx, cudaEventRecord(ctx->ev[2], ctx->stream));
    const double* src[8] = {particles->x, particles->y, particles->z, particles->vx,
                            particles->vy, particles->vz, particles->m, particles->h};
    for (int a = 0; a < 8 && n > 0; ++a)
        KIWI_CUDA(ctx, cudaMemcpyAsync(dpart + a * n, src[a], sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
    if (n > 0) KIWI_CUDA(ctx, cudaMemcpyAsync(dhome, home_cell, sizeof(int32_t) * n, cudaMemcpyHostToDevice, ctx->stream));
    unsigned char* q = dgeo;
    int64_t* d_fo = (int64_t*)q; q += al(b_fo);
    int64_t* d_vo = (int64_t*)q; q += al(b_vo);
    double* d_v = (double*)q; q += al(b_v);
    int32_t* d_nb = (int32_t*)q; q += al(b_nb);
    double* d_vol = (double*)q;
    if (nc > 0) {
        KIWI_CUDA(ctx, cudaMemcpyAsync(d_fo, cells->face_off, b_fo, cudaMemcpyHostToDevice, ctx->stream));
        KIWI_CUDA(ctx, cudaMemcpyAsync(d_vo, cells->vert_off, b_vo, cudaMemcpyHostToDevice, ctx->stream));
        if (nv > 0) KIWI_CUDA(ctx, cudaMemcpyAsync(d_v, cells->vxyz, b_v, cudaMemcpyHostToDevice, ctx->stream));
        if (nf > 0) KIWI_CUDA(ctx, cudaMemcpyAsync(d_nb, cells->face_nbr, b_nb, cudaMemcpyHostToDevice, ctx->stream));
        KIWI_CUDA(ctx, cudaMemcpyAsync(d_vol, cells->volume, b_vol, cudaMemcpyHostToDevice, ctx->stream));
    }
    DevParticles P{n, dpart, dpart + n, dpart + 2 * n, dpart + 3 * n, dpart + 4 * n, dpart + 5 * n, dpart + 6 * n,
                   dpart + 7 * n};
    KiwiVoronoiCells dc{nc, d_fo, d_vo, d_v, d_nb, d_vol};
    CartOutputs out{dout, dout + nc, dout + 2 * nc, dout + 3 * nc, raw4 ? dout + 4 * nc : nullptr, nullptr};
    VorInverse dinv_v{nullptr, nullptr, nullptr};
    if (inv) {
        double* d_cm = dinv;
        dinv_v.m_recovered = dinv + std::max<int64_t>(nc, 1);
        dinv_v.coverage = dinv_v.m_recovered + std::max<int64_t>(n, 1);
        if (n > 0) {
            KIWI_CUDA(ctx, cudaMemsetAsync(dinv_v.m_recovered, 0, sizeof(double) * n, ctx->stream));
            KIWI_CUDA(ctx, cudaMemsetAsync(dinv_v.coverage, 0, sizeof(double) * n, ctx->stream));
        }
        if (inv->cell_mass && nc > 0) {
            KIWI_CUDA(ctx, cudaMemcpyAsync(d_cm, inv->cell_mass, sizeof(double) * nc, cudaMemcpyHostToDevice, ctx->stream));
            dinv_v.cell_mass = d_cm;
        }
    }
    KIWI_TRY(voronoi_map_dev(ctx, P, dhome, dc, kc, out, stats, inv ? &dinv_v : nullptr));
    if (inv && n > 0) {
        KIWI_CUDA(ctx, cudaMemcpyAsync(inv->m_recovered, dinv_v.m_recovered, sizeof(double) * n, cudaMemcpyDeviceToHost,
                                       ctx->stream));
        if (inv->coverage)
            KIWI_CUDA(ctx, cudaMemcpyAsync(inv->coverage, dinv_v.coverage, sizeof(double) * n, cudaMemcpyDeviceToHost,
                                           ctx->stream));
    }
    double* dst[4] = {density, vx, vy, vz};
    for (int a = 0; a < 4 && nc > 0; ++a)
        if (dst[a])
            KIWI_CUDA(ctx, cudaMemcpyAsync(dst[a], dout + a * nc, sizeof(double) * nc, cudaMemcpyDeviceToHost, ctx->stream));
    if (raw4 && nc > 0)
        KIWI_CUDA(ctx, cudaMemcpyAsync(raw4, dout + 4 * nc, sizeof(double) * 4 * nc, cudaMemcpyDeviceToHost, ctx->stream));
    KIWI_CUDA(ctx, cudaEventRecord(ctx->ev[3], ctx->stream));
    KIWI_CUDA(ctx, cudaEventSynchronize(ctx->ev[3]));
    if (stats) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]);
        stats->total_ms = ms;
    }
    if (inv && inv->totals3) {
        // the totals of src/mapping.cpp:675-682, summed in particle and cell order on the host: the
        // original masses (every particle), the grid mass sum of m_i, the recovered masses
        double t_orig = 0.0, t_grid = 0.0, t_rec = 0.0;
        for (int64_t i = 0; i < n; ++i) {
            t_orig += particles->m[i];
            t_rec += inv->m_recovered[i];
        }
        if (inv->cell_mass) {
            for (int64_t c = 0; c < nc; ++c) t_grid += inv->cell_mass[c];
        } else if (density) {
            for (int64_t c = 0; c < nc; ++c) t_grid += density[c] * cells->volume[c];
        }
        inv->totals3[0] = t_orig;
        inv->totals3[1] = t_grid;
        inv->totals3[2] = t_rec;
    }
    return KIWI_OK;
}

}  // namespace

extern "C" {

int kiwi_map_voronoi(KiwiCtx* ctx, const KiwiParticles* particles, const int32_t* home_cell,
                     const KiwiVoronoiCells* cells, const KiwiKernelSel* kernel, int precision, double* density,
                     double* vx, double* vy, double* vz, double* raw4, KiwiStats* stats) {
    return map_voronoi_host(ctx, particles, home_cell, cells, kernel, precision, density, vx, vy, vz, raw4, stats,
                            nullptr);
}

int kiwi_map_voronoi_device(KiwiCtx* ctx, const KiwiParticles* particles, const int32_t* home_cell,
                            const KiwiVoronoiCells* cells, const KiwiKernelSel* kernel, int precision, double* density,
                            double* vx, double* vy, double* vz, double* raw4, KiwiStats* stats) {
    KIWI_TRY(check_ctx(ctx));
    int rc = KIWI_OK;
    if (!particles_ok(ctx, particles, &rc)) return rc;
    KernelChoice kc;
    KIWI_TRY(resolve_kernel(ctx, kernel, &kc));
    if ((precision & KIWI_FORM_MASK) != KIWI_FP64 && (precision & KIWI_FORM_MASK) != KIWI_FP64_REFERENCE_ORDER)
        return set_err(ctx, KIWI_ERR_UNSUPPORTED, "the Voronoi map is available in the FP64 form only");
    if (kc.tabulated) KIWI_TRY(table_ensure(ctx, &kc.tab));
    if (!cells || cells->n_cells < 0 || (cells->n_cells > 0 && (!cells->face_off || !cells->vert_off ||
                                                                 !cells->vxyz || !cells->face_nbr || !cells->volume)))
        return set_err(ctx, KIWI_ERR_ARG, "cell geometry is incomplete");
    if (particles->n > 0 && !home_cell) return set_err(ctx, KIWI_ERR_ARG, "home_cell is null");
    if (cells->n_cells >= (1LL << 31)) return set_err(ctx, KIWI_ERR_ARG, "too many cells");
    KIWI_CUDA(ctx, cudaEventRecord(ctx->ev[2], ctx->stream));
    DevParticles P{particles->n, particles->x, particles->y, particles->z, particles->vx,
                   particles->vy, particles->vz, particles->m, particles->h};
    CartOutputs out{density, vx, vy, vz, raw4, nullptr};
    KIWI_TRY(voronoi_map_dev(ctx, P, home_cell, *cells, kc, out, stats));
    KIWI_CUDA(ctx, cudaEventRecord(ctx->ev[3], ctx->stream));
    KIWI_CUDA(ctx, cudaEventSynchronize(ctx->ev[3]));
    if (stats) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]);
        stats->total_ms = ms;
    }
    return KIWI_OK;
}

int kiwi_inverse_map_voronoi(KiwiCtx* ctx, const KiwiParticles* particles, const int32_t* home_cell,
                             const KiwiVoronoiCells* cells, const KiwiKernelSel* kernel, int precision,
                             const double* cell_mass, double* m_recovered, double* coverage, double* totals3,
                             double* density, KiwiStats* stats) {
    if (ctx && particles && particles->n > 0 && !m_recovered)
        return set_err(ctx, KIWI_ERR_ARG, "inverse map: m_recovered is null");
    // the grid-mass total without given cell masses needs the forward densities on the host
    std::vector<double> dens_tmp;
    if (!cell_mass && totals3 && !density && cells && cells->n_cells > 0) {
        dens_tmp.resize((size_t)cells->n_cells);
        density = dens_tmp.data();
    }
    const InverseHost inv{cell_mass, m_recovered, coverage, totals3};
    return map_voronoi_host(ctx, particles, home_cell, cells, kernel, precision, density, nullptr, nullptr, nullptr,
                            nullptr, stats, &inv);
}

}  // extern "C"
