// The lattice-factorised gather of the plain FP64 form (cubic spline closed form and table-driven generic
// kernels) and the batch's persistent kernel for those two families.  This translation unit is built with
// FMA contraction: the lattice form regroups the reference's sum (lattice_tile.cuh) and evaluates its tiers
// in the triangles' own lengths (lattice_math.cuh), so it does not follow the reference's operation order
// and gains nothing from rounding each product on its own; the quantities that integer results depend on
// (bounding boxes, lattice planes, cell centres, the support test of the pair counters) are formed with
// explicitly rounded operations (cart_common.cuh), as in every other form.
#include <cuda_runtime.h>

#include "engine.hpp"
#include "kernel_tables.h"

namespace kiwi_b200 {
static __constant__ KiwiKernelTable c_tables[KIWI_NUM_KERNELS];
}  // namespace kiwi_b200

#include "lattice_tile.cuh"

namespace kiwi_b200 {

int lattice_init_tables(KiwiCtx* ctx) {
    KIWI_CUDA(ctx, cudaMemcpyToSymbol(c_tables, kiwi_kernel_tables, sizeof(kiwi_kernel_tables)));
    return KIWI_OK;
}

namespace {

// Resident CTAs per SM the register budget is sized for: two for both kernels (128 registers).  The cubic
// kernel's shared memory would fit three, but at the 80 registers three need, its point-wise tiers spill:
// 3.59 G support pairs/s at three against 3.84 G at two on the 2 M-particle log-normal cube.
#ifndef KIWI_LATTICE_MIN_BLOCKS
#define KIWI_LATTICE_MIN_BLOCKS 2
#endif
#ifndef KIWI_LATTICE_GEN_MIN_BLOCKS
#define KIWI_LATTICE_GEN_MIN_BLOCKS 2
#endif
constexpr int kLatMinBlocks = KIWI_LATTICE_MIN_BLOCKS;
constexpr int kLatGenMinBlocks = KIWI_LATTICE_GEN_MIN_BLOCKS;
constexpr size_t kLatMergedDynSmem = kLatDynSmem > kLatGenDynSmem ? kLatDynSmem : kLatGenDynSmem;

template <bool CULL>
__global__ void __launch_bounds__(kLatThreads, kLatMinBlocks) k_cart_lattice(CartGeom g, DevParticles P,
                                                                             const uint32_t* __restrict__ list,
                                                                             const int64_t* __restrict__ range,
                                                                             const int32_t* __restrict__ tile_map,
                                                                             CartOutputs out, DevStats* __restrict__ st) {
    const int64_t t = tile_map ? (int64_t)tile_map[blockIdx.x] : (int64_t)blockIdx.x;
    lattice_tile<CULL>(g, P, list, range, t, t, out, st);
}

// The FP32-mixed form of the cubic lattice kernel (support cells only): edge pairs and lattice points
// evaluated with FP32 tiers (FP64 islands where a plane lies within 1e-3 h of the particle), cell assembly
// and per-cell sums in FP64.
__global__ void __launch_bounds__(kLatThreads, kLatMinBlocks) k_cart_lattice_mixed(CartGeom g, DevParticles P,
                                                                                const uint32_t* __restrict__ list,
                                                                                const int64_t* __restrict__ range,
                                                                                const int32_t* __restrict__ tile_map,
                                                                                CartOutputs out,
                                                                                DevStats* __restrict__ st) {
    const int64_t t = tile_map ? (int64_t)tile_map[blockIdx.x] : (int64_t)blockIdx.x;
    lattice_tile<true, false, false, true>(g, P, list, range, t, t, out, st);
}

// The lattice form for the generic kernels (support cells only).
__global__ void __launch_bounds__(kLatThreads, kLatGenMinBlocks) k_cart_lattice_generic(CartGeom g, DevParticles P,
                                                                                     int kernel,
                                                                                     const uint32_t* __restrict__ list,
                                                                                     const int64_t* __restrict__ range,
                                                                                     const int32_t* __restrict__ tile_map,
                                                                                     CartOutputs out,
                                                                                     DevStats* __restrict__ st) {
    const int64_t t = tile_map ? (int64_t)tile_map[blockIdx.x] : (int64_t)blockIdx.x;
    lattice_tile<true, true>(g, P, list, range, t, t, out, st, &c_tables[kernel]);
}

// The FP32-mixed form of the generic lattice kernel: edge records and vertex tiers in FP32 (FP64 islands
// where a plane lies within 1e-3 h of the particle), records, cell assembly and per-cell sums in FP64.
__global__ void __launch_bounds__(kLatThreads, kLatGenMinBlocks)
    k_cart_lattice_generic_mixed(CartGeom g, DevParticles P, int kernel, const uint32_t* __restrict__ list,
                                 const int64_t* __restrict__ range, const int32_t* __restrict__ tile_map,
                                 CartOutputs out, DevStats* __restrict__ st) {
    const int64_t t = tile_map ? (int64_t)tile_map[blockIdx.x] : (int64_t)blockIdx.x;
    lattice_tile<true, true, false, true>(g, P, list, range, t, t, out, st, &c_tables[kernel]);
}

// The tiles of a batch of grids, one persistent launch per lattice family, or one for both
// (kBatchFamilyLatticeMerged: each tile takes its item's body): each CTA takes the next of the launch's
// tiles (order[w]) from the work counter and runs the same tile body as the single-grid kernel, so every
// cell's summation order is that of a single-grid call.  MIXED: the FP32-mixed tile bodies.
template <int FAMILY, bool MIXED>
__global__ void __launch_bounds__(kLatThreads, 2) k_batch_lattice(const BatchItemDev* __restrict__ items,
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
        if (FAMILY == kBatchFamilyLattice || (FAMILY == kBatchFamilyLatticeMerged && it.mode == kBatchLattice))
            lattice_tile<true, false, false, MIXED>(it.g, it.P, list, range, tg, tl, it.out, it.st);
        else
            lattice_tile<true, true, false, MIXED>(it.g, it.P, list, range, tg, tl, it.out, it.st,
                                                   &c_tables[it.kernel]);
        __syncthreads();
    }
}

}  // namespace

int lattice_cart_gather(KiwiCtx* ctx, const CartGeom& g, const DevParticles& P, const KernelChoice& k,
                        const TileLists& tl, const CartOutputs& out, DevStats* d_stats, bool full_box) {
    const dim3 grid((unsigned)(tl.map ? tl.nmap : tl.ntiles));
    if (k.cubic) {
        if (full_box) {
            KIWI_CUDA(ctx, cudaFuncSetAttribute(k_cart_lattice<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                (int)kLatDynSmem));
            KIWI_CUDA(ctx, cudaFuncSetAttribute(k_cart_lattice<false>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                                (int)kLatCarveout));
            k_cart_lattice<false><<<grid, kLatThreads, kLatDynSmem, ctx->stream>>>(g, P, tl.list, tl.range, tl.map,
                                                                                   out, d_stats);
        } else {
            KIWI_CUDA(ctx, cudaFuncSetAttribute(k_cart_lattice<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                (int)kLatDynSmem));
            KIWI_CUDA(ctx, cudaFuncSetAttribute(k_cart_lattice<true>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                                (int)kLatCarveout));
            k_cart_lattice<true><<<grid, kLatThreads, kLatDynSmem, ctx->stream>>>(g, P, tl.list, tl.range, tl.map,
                                                                                  out, d_stats);
        }
    } else {
        KIWI_CUDA(ctx, cudaFuncSetAttribute(k_cart_lattice_generic, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)kLatGenDynSmem));
        k_cart_lattice_generic<<<grid, kLatThreads, kLatGenDynSmem, ctx->stream>>>(g, P, k.kernel, tl.list, tl.range,
                                                                                   tl.map, out, d_stats);
    }
    KIWI_LAUNCHED(ctx);
    return KIWI_OK;
}

int lattice_mixed_gather(KiwiCtx* ctx, const CartGeom& g, const DevParticles& P, const KernelChoice& k,
                         const TileLists& tl, const CartOutputs& out, DevStats* d_stats) {
    if (tl.ntiles <= 0 || (tl.map && tl.nmap <= 0)) return KIWI_OK;
    const dim3 grid((unsigned)(tl.map ? tl.nmap : tl.ntiles));
    if (!k.cubic) {
        KIWI_CUDA(ctx, cudaFuncSetAttribute(k_cart_lattice_generic_mixed, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)kLatGenDynSmem));
        KIWI_CUDA(ctx, cudaFuncSetAttribute(k_cart_lattice_generic_mixed,
                                            cudaFuncAttributePreferredSharedMemoryCarveout,
                                            (int)kLatCarveout));
        k_cart_lattice_generic_mixed<<<grid, kLatThreads, kLatGenDynSmem, ctx->stream>>>(
            g, P, k.kernel, tl.list, tl.range, tl.map, out, d_stats);
        KIWI_LAUNCHED(ctx);
        return KIWI_OK;
    }
    KIWI_CUDA(ctx, cudaFuncSetAttribute(k_cart_lattice_mixed, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)kLatDynSmem));
    KIWI_CUDA(ctx, cudaFuncSetAttribute(k_cart_lattice_mixed, cudaFuncAttributePreferredSharedMemoryCarveout,
                                        (int)kLatCarveout));
    k_cart_lattice_mixed<<<grid, kLatThreads, kLatDynSmem, ctx->stream>>>(g, P, tl.list, tl.range, tl.map, out,
                                                                          d_stats);
    KIWI_LAUNCHED(ctx);
    return KIWI_OK;
}

template <bool MIXED>
static int batch_prepare_t(KiwiCtx* ctx) {
    KIWI_CUDA(ctx, cudaFuncSetAttribute(k_batch_lattice<kBatchFamilyLattice, MIXED>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLatDynSmem));
    KIWI_CUDA(ctx, cudaFuncSetAttribute(k_batch_lattice<kBatchFamilyLatticeGeneric, MIXED>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLatGenDynSmem));
    KIWI_CUDA(ctx, cudaFuncSetAttribute(k_batch_lattice<kBatchFamilyLatticeMerged, MIXED>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLatMergedDynSmem));
    return KIWI_OK;
}

int lattice_batch_prepare(KiwiCtx* ctx) {
    KIWI_TRY(batch_prepare_t<false>(ctx));
    return batch_prepare_t<true>(ctx);
}

template <bool MIXED>
static void batch_launch_t(KiwiCtx* ctx, int family, const BatchItemDev* d_items, const int32_t* d_item_of_tile,
                           const int32_t* d_order, int64_t ntiles, const uint32_t* list, const int64_t* range,
                           unsigned long long* d_next, int blocks) {
    if (family == kBatchFamilyLattice)
        k_batch_lattice<kBatchFamilyLattice, MIXED><<<blocks, kLatThreads, kLatDynSmem, ctx->stream>>>(
            d_items, d_item_of_tile, d_order, ntiles, list, range, d_next);
    else if (family == kBatchFamilyLatticeMerged)
        k_batch_lattice<kBatchFamilyLatticeMerged, MIXED><<<blocks, kLatThreads, kLatMergedDynSmem, ctx->stream>>>(
            d_items, d_item_of_tile, d_order, ntiles, list, range, d_next);
    else
        k_batch_lattice<kBatchFamilyLatticeGeneric, MIXED><<<blocks, kLatThreads, kLatGenDynSmem, ctx->stream>>>(
            d_items, d_item_of_tile, d_order, ntiles, list, range, d_next);
}

int lattice_batch_gather(KiwiCtx* ctx, int family, const BatchItemDev* d_items, const int32_t* d_item_of_tile,
                         const int32_t* d_order, int64_t ntiles, const uint32_t* list, const int64_t* range,
                         unsigned long long* d_next, int blocks, bool mixed) {
    if (mixed)
        batch_launch_t<true>(ctx, family, d_items, d_item_of_tile, d_order, ntiles, list, range, d_next, blocks);
    else
        batch_launch_t<false>(ctx, family, d_items, d_item_of_tile, d_order, ntiles, list, range, d_next, blocks);
    KIWI_LAUNCHED(ctx);
    return KIWI_OK;
}

}  // namespace kiwi_b200
