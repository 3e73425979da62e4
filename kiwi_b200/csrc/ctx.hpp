// Host-side context of the C ABI: device, stream, events, error text and a grow-only scratch arena.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <string>

#include "../../include/kiwi_b200.h"

namespace kiwi_b200 {
// A density lookup table in device memory (DensityLookupTable, include/kiwi/kernel_integral.hpp:21-72):
// the sub-grid sizes and split points of its three axes and the values, laid out as the reference does.
struct TabDev {
    const double* v = nullptr;
    int nr01 = 0, nR_01 = 0, nphi1 = 0, nr02 = 0, nR_02 = 0, nphi2 = 0, nr0 = 0, nR_0 = 0, nphi = 0;
    double rl = 0.0, mul = 0.0, cphil = 0.0;
};
}  // namespace kiwi_b200

struct KiwiCtx {
    int device = -1;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    std::string err;
    int64_t launches = 0;  // kernels launched on this context (for the stats of a call)
    // Scratch slots: each is grown on demand and reused by later calls on this context.
    static constexpr int kSlots = 64;
    void* slot_ptr[kSlots] = {};
    size_t slot_bytes[kSlots] = {};
    // Fixed arena mode (used only by the allocation-free entry point): when `arena` is set, scratch
    // slots are carved from it instead of allocated, and a request that does not fit is an error.
    unsigned char* arena = nullptr;
    size_t arena_bytes = 0, arena_used = 0;
    // The density lookup table of the tabulated integral (generated or loaded on demand; tab.v owns
    // tab_bytes of device memory).
    kiwi_b200::TabDev tab;
    size_t tab_bytes = 0;
    // Voronoi maps: each face value evaluated once through per-(pair, face) tables (kiwi_ctx_set_voronoi_face_tables)
    bool face_tables = true;
    // Voronoi maps: the pair and face totals of the last map, the sizes the next map's single walk reserves
    int64_t vor_pairs_hint = 0, vor_faces_hint = 0;
};

namespace kiwi_b200 {

inline int set_err(KiwiCtx* ctx, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (ctx) ctx->err = buf;
    return code;
}

#define KIWI_CUDA(ctx, call)                                                                              \
    do {                                                                                                  \
        cudaError_t e_ = (call);                                                                          \
        if (e_ != cudaSuccess) {                                                                          \
            cudaGetLastError(); /* a non-sticky error must not resurface at the next launch check */      \
            return ::kiwi_b200::set_err((ctx), KIWI_ERR_CUDA, "%s failed: %s (%s:%d)", #call,              \
                                        cudaGetErrorString(e_), __FILE__, __LINE__);                      \
        }                                                                                                 \
    } while (0)

#define KIWI_LAUNCHED(ctx)                                                                                \
    do {                                                                                                  \
        ++(ctx)->launches;                                                                                \
        cudaError_t e_ = cudaGetLastError();                                                              \
        if (e_ != cudaSuccess)                                                                            \
            return ::kiwi_b200::set_err((ctx), KIWI_ERR_CUDA, "kernel launch failed: %s (%s:%d)",          \
                                        cudaGetErrorString(e_), __FILE__, __LINE__);                      \
    } while (0)

#define KIWI_TRY(expr)          \
    do {                        \
        int rc_ = (expr);       \
        if (rc_ != KIWI_OK) return rc_; \
    } while (0)

// Device scratch of at least `bytes` in slot `slot` (grow-only; contents are not preserved on growth).
inline int scratch(KiwiCtx* ctx, int slot, size_t bytes, void** out) {
    if (bytes == 0) bytes = 256;
    if (ctx->arena && ctx->slot_bytes[slot] < bytes) {
        const size_t start = (ctx->arena_used + 255) & ~(size_t)255;
        if (start > ctx->arena_bytes || bytes > ctx->arena_bytes - start)
            return set_err(ctx, KIWI_ERR_LIMIT,
                           "input too large for the fixed scratch area: it needs more than %zu bytes (%zu requested "
                           "at offset %zu)", ctx->arena_bytes, bytes, start);
        ctx->slot_ptr[slot] = ctx->arena + start;
        ctx->slot_bytes[slot] = bytes;
        ctx->arena_used = start + bytes;
    }
    if (ctx->slot_bytes[slot] < bytes) {
        if (ctx->slot_ptr[slot]) {
            cudaStreamSynchronize(ctx->stream);
            cudaFree(ctx->slot_ptr[slot]);
            ctx->slot_ptr[slot] = nullptr;
            ctx->slot_bytes[slot] = 0;
        }
        size_t want = bytes + bytes / 4;
        cudaError_t e = cudaMalloc(&ctx->slot_ptr[slot], want);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return set_err(ctx, KIWI_ERR_ALLOC, "cudaMalloc of %zu bytes of scratch failed: %s", want,
                           cudaGetErrorString(e));
        }
        ctx->slot_bytes[slot] = want;
    }
    *out = ctx->slot_ptr[slot];
    return KIWI_OK;
}

template <class T>
inline int scratch_t(KiwiCtx* ctx, int slot, size_t count, T** out) {
    void* p = nullptr;
    int rc = scratch(ctx, slot, count * sizeof(T), &p);
    *out = static_cast<T*>(p);
    return rc;
}

// Scratch slot numbers (fixed so that a call never overwrites a buffer it still needs).
enum ScratchSlot {
    S_PART = 0,      // staged particle SoA (host entry points)
    S_OUT,           // staged outputs
    S_BOX,           // per-particle clamped bounding boxes
    S_COUNT,         // per-particle tile counts
    S_OFFS,          // per-particle tile-pair offsets
    S_KEYS0,
    S_VALS0,
    S_KEYS1,
    S_VALS1,
    S_HIST,          // radix histograms
    S_SCAN,          // scan partials
    S_TILE_RANGE,    // per-tile [begin, end)
    S_STATS,         // device counters
    S_MEANV,         // mean velocity
    S_MISC0,
    S_MISC1,
    S_MISC2,
    S_MISC3,
    S_VOR_MARK,      // Voronoi walk: visited markers per work slot
    S_VOR_QUEUE,     // Voronoi walk: queues per work slot
    S_VOR_PAIRS,     // Voronoi walk: visited cells of every particle
    S_VOR_NEXT,      // Voronoi walk: particle counter
    S_VOR_CSR,       // staged cell geometry (host entry point)
    S_VOR_HOME,      // staged home cells (host entry point)
    S_CELL_ERR,      // FP32-mixed form: per-cell rounding bound
    S_CELL_MASS,     // FP32-mixed form: per-cell raw mass
    S_TILE_MAP,      // FP32-mixed form: tiles recomputed in FP64
    S_STATS2,        // device counters of a second pass
    S_VOR_MASK,      // Voronoi walk: per pair, the faces whose neighbour was processed earlier
    S_ADJ_PART,      // adjoint: partial gradients per (tile, particle) entry
    S_VOR_PVAL,      // inverse map: each visited pair's cell integral
    S_VOR_CMASS,     // inverse map: per-cell mass m_i
    S_INV_OUT,       // inverse map: given cell masses, recovered masses and coverage (host entry point)
    S_PART_W,        // part split: per-tile entry counts
    S_PART_PREFIX,   // part split: their prefix sums
    S_PART_FLAGS,    // part split: tiles of this part
    S_PART_OFFS,     // part split: compaction offsets
    S_FLAG_PEAK,     // FP32-mixed guarantee: peak cell mass
    S_FLAG_FLAGS,    // FP32-mixed guarantee: tiles to recompute
    S_FLAG_OFFS,     // FP32-mixed guarantee: compaction offsets
    S_NMAP,          // FP32-mixed guarantee: number of tiles to recompute
    S_VOR_FCOUNT,    // Voronoi walk: per particle, the faces of its visited cells
    S_VOR_FOFFS,     // Voronoi walk: their prefix sums
    S_VOR_PFOFF,     // Voronoi walk: per pair, the offset of its cell's faces in the face tables
    S_VOR_FSRC,      // Voronoi walk: per (pair, face), where its value comes from
    S_VOR_FVAL,      // Voronoi map: per (pair, face), the face's integral
    S_VOR_LINKS,     // Voronoi map: per face, its earlier twin in the cell and the neighbour's face back
    S_VOR_STAGE,     // Voronoi walk: the single walk's staging area
    S_LPT_K0,        // heaviest-first tile order: sort keys and values (two buffers each)
    S_LPT_V0,
    S_LPT_K1,
    S_LPT_V1,
};
static_assert(S_LPT_V1 < KiwiCtx::kSlots, "scratch slots");

}  // namespace kiwi_b200
