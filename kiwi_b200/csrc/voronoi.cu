// Voronoi-cell mapping: the particle loop of run_mapping_stage (src/mapping.cpp:400-502) on the GPU.
//
//  (1) k_vor_bfs, one warp per particle (persistent, particles pulled from a counter): the breadth-first
//      walk of src/mapping.cpp:441-460 over the cell-neighbour graph from the particle's home cell,
//      entering a neighbour when the shared face's closest point lies within the support radius
//      (face_reachable: the out_vert rule of src/kernel_integral.cpp:636-645 and
//      src/mapping.cpp:187-193).  It needs no integrals.  Run twice: first it counts each particle's
//      visited cells, then it writes them at the particle's offset, so the (cell, particle) pairs come
//      out grouped by particle in ascending particle order.
//  (2) a stable radix sort by cell index: every cell's particles stay in ascending order.
//  (3) k_vor_gather, one CTA per cell: the cell's faces are staged in shared memory, each thread takes
//      one particle of the cell's list and evaluates compute_cell_integral (src/mapping.cpp:105-206): the
//      sum over the cell's faces of the face walk, clamped at 0; the values are then added in particle
//      order -- the reference's single-threaded summation order, no atomics -- and finalised as
//      src/mapping.cpp:482-502 does.
// The reference evaluates a face shared by two visited cells once per particle and reuses its negation
// on the other side (src/mapping.cpp:56-93); here each side evaluates it: the two agree to rounding.
#include <cuda_runtime.h>

#include <algorithm>

#include "../../include/kiwi_b200.h"
#include "engine.hpp"
#include "kiwi_math.cuh"
#include "prims.cuh"

namespace kiwi_b200 {

// kernel tables of this translation unit (constant memory is per translation unit)
__constant__ KiwiKernelTable c_vor_tables[KIWI_NUM_KERNELS];

int voronoi_init_tables(KiwiCtx* ctx) {
    KIWI_CUDA(ctx, cudaMemcpyToSymbol(c_vor_tables, kiwi_kernel_tables, sizeof(kiwi_kernel_tables)));
    return KIWI_OK;
}

namespace {

struct VorCells {
    int64_t n_cells;
    const int64_t* face_off;
    const int64_t* vert_off;
    const double* vxyz;
    const int32_t* face_nbr;
    const double* volume;
};

constexpr int kBfsWarpsPerBlock = 4;
constexpr int kGatherThreads = 128;
constexpr int kGatherVertCap = 1536;  // vertices staged in shared memory per cell (36 KB)

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// marker value of particle p in pass `pass`: distinct for every (particle, pass), never -1
__device__ __forceinline__ int marker(int64_t p, int pass) { return (int)(2 * p + pass); }

__global__ void __launch_bounds__(32 * kBfsWarpsPerBlock) k_vor_bfs(VorCells C, DevParticles P,
                                                                    const int32_t* __restrict__ home,
                                                                    double support_in_h, int pass,
                                                                    unsigned long long* __restrict__ next,
                                                                    int* __restrict__ mark_base,
                                                                    int32_t* __restrict__ queue_base,
                                                                    int64_t* __restrict__ counts,
                                                                    const int64_t* __restrict__ offs,
                                                                    int32_t* __restrict__ pair_cells,
                                                                    DevStats* __restrict__ st) {
    __shared__ int s_tail[kBfsWarpsPerBlock];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t slot = (int64_t)blockIdx.x * kBfsWarpsPerBlock + warp;
    int* mark = mark_base + slot * C.n_cells;
    int32_t* queue = queue_base + slot * C.n_cells;
    unsigned long long n_unresolved = 0, n_unmapped = 0, n_limit = 0;
    for (;;) {
        unsigned long long p = 0;
        if (lane == 0) p = atomicAdd(next, 1ull);
        p = __shfl_sync(0xffffffffu, p, 0);
        if (p >= (unsigned long long)P.n) break;
        const double h = P.h[p];
        const int32_t k0 = home[p];
        if (!(h > 0.0) || k0 < 0 || k0 >= C.n_cells) {
            if (lane == 0) {
                if (pass == 0) counts[p] = 0;
                if (h > 0.0) ++n_unresolved;
            }
            continue;
        }
        const double x0 = P.x[p], y0 = P.y[p], z0 = P.z[p];
        const double radius = mul_rn(support_in_h, h);
        const int mk = marker((int64_t)p, pass);
        if (lane == 0) {
            queue[0] = k0;
            mark[k0] = mk;
            s_tail[warp] = 1;
        }
        __syncwarp();
        int head = 0, tail = 1;
        int64_t guard = 0;
        while (head < tail) {
            if (++guard > C.n_cells + 1) {  // cannot happen: each cell enters the queue once
                n_limit += (lane == 0);
                break;
            }
            const int batch = min(32, tail - head);
            if (lane < batch) {
                const int32_t cell = queue[head + lane];
                for (int64_t f = C.face_off[cell]; f < C.face_off[cell + 1]; ++f) {
                    const int32_t nb = C.face_nbr[f];
                    if (nb < 0 || nb >= C.n_cells) continue;
                    if (mark[nb] == mk) continue;
                    const FlatVerts V{C.vxyz + 3 * C.vert_off[f]};
                    const int nv = (int)(C.vert_off[f + 1] - C.vert_off[f]);
                    if (!face_reachable(x0, y0, z0, radius, V, nv)) continue;
                    if (atomicExch(&mark[nb], mk) != mk) {
                        const int pos = atomicAdd(&s_tail[warp], 1);
                        queue[pos] = nb;
                    }
                }
            }
            __syncwarp();
            head += batch;
            tail = s_tail[warp];
            __syncwarp();
        }
        if (pass == 0) {
            if (lane == 0) {
                counts[p] = tail;
                if (tail == 1) ++n_unmapped;
            }
        } else {
            const int64_t o = offs[p];
            for (int i = lane; i < tail; i += 32) pair_cells[o + i] = queue[i];
        }
        __syncwarp();
    }
    n_unresolved = warp_sum_u64(n_unresolved);
    n_unmapped = warp_sum_u64(n_unmapped);
    n_limit = warp_sum_u64(n_limit);
    if (lane == 0 && pass == 0) {
        if (n_unresolved) atomicAdd(&st->skipped_outside, n_unresolved);
        if (n_unmapped) atomicAdd(&st->tile_pairs, n_unmapped);  // reported as "unmapped" by the caller
    }
    if (lane == 0 && n_limit) atomicAdd(&st->limit_hit, n_limit);
}

// pair index of particle p's k-th visited cell -> (key = cell, value = particle)
__global__ void k_vor_pairs(const int32_t* __restrict__ pair_cells, int64_t total, const int64_t* __restrict__ offs,
                            int64_t n, uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= total) return;
    int64_t lo = 0, hi = n - 1;
    while (lo < hi) {
        const int64_t mid = (lo + hi + 1) >> 1;
        if (offs[mid] <= k) lo = mid; else hi = mid - 1;
    }
    keys[k] = (uint32_t)pair_cells[k];
    vals[k] = (uint32_t)lo;
}

__global__ void k_cell_ranges(const uint32_t* __restrict__ keys, int64_t total, int64_t* __restrict__ range) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const uint32_t k = keys[i];
    if (i == 0 || keys[i - 1] != k) range[2 * (int64_t)k] = i;
    if (i == total - 1 || keys[i + 1] != k) range[2 * (int64_t)k + 1] = i + 1;
}

template <bool CUBIC>
__global__ void __launch_bounds__(kGatherThreads) k_vor_gather(VorCells C, DevParticles P, int kernel,
                                                                double support_in_h,
                                                                const uint32_t* __restrict__ plist,
                                                                const int64_t* __restrict__ range,
                                                                CartOutputs out, DevStats* __restrict__ st) {
    __shared__ double s_v[3 * kGatherVertCap];
    __shared__ double s_val[kGatherThreads], s_m[kGatherThreads], s_vx[kGatherThreads], s_vy[kGatherThreads],
        s_vz[kGatherThreads];
    const int64_t cell = blockIdx.x;
    const int64_t f0 = C.face_off[cell], f1 = C.face_off[cell + 1];
    const int64_t v0 = C.vert_off[f0], v1 = C.vert_off[f1];
    const bool staged = (v1 - v0) <= kGatherVertCap;
    if (staged)
        for (int64_t i = threadIdx.x; i < 3 * (v1 - v0); i += kGatherThreads) s_v[i] = C.vxyz[3 * v0 + i];
    __syncthreads();
    const int64_t beg = range[2 * cell], end = range[2 * cell + 1];
    double M = 0.0, Px = 0.0, Py = 0.0, Pz = 0.0;
    unsigned long long n_neg = 0, n_warn = 0;
    for (int64_t base = beg; base < end; base += kGatherThreads) {
        const int64_t k = base + threadIdx.x;
        double msum = 0.0;
        if (k < end) {
            const uint32_t p = plist[k];
            const double x0 = P.x[p], y0 = P.y[p], z0 = P.z[p], h = P.h[p];
            const double radius = mul_rn(support_in_h, h);
            if (CUBIC) {
                CubicEval ev;
                ev.h = h;
#pragma unroll 1
                for (int64_t f = f0; f < f1; ++f) {
                    const FlatVerts V{staged ? s_v + 3 * (C.vert_off[f] - v0) : C.vxyz + 3 * C.vert_off[f]};
                    msum += face_integral(x0, y0, z0, 2 * h, V, (int)(C.vert_off[f + 1] - C.vert_off[f]), (int*)nullptr, ev);
                }
            } else {
                GenericEval ev;
                ev.K = &c_vor_tables[kernel];
                ev.H = radius;
#pragma unroll 1
                for (int64_t f = f0; f < f1; ++f) {
                    const FlatVerts V{staged ? s_v + 3 * (C.vert_off[f] - v0) : C.vxyz + 3 * C.vert_off[f]};
                    msum += face_integral(x0, y0, z0, radius, V, (int)(C.vert_off[f + 1] - C.vert_off[f]), (int*)nullptr, ev);
                }
            }
            if (msum < 0.0) {
                ++n_neg;
                if (msum <= -0.01) ++n_warn;
                msum = 0.0;
            }
            s_m[threadIdx.x] = P.m[p];
            s_vx[threadIdx.x] = P.vx[p];
            s_vy[threadIdx.x] = P.vy[p];
            s_vz[threadIdx.x] = P.vz[p];
        }
        s_val[threadIdx.x] = msum;
        __syncthreads();
        if (threadIdx.x == 0) {
            const int cnt = (end - base < kGatherThreads) ? (int)(end - base) : kGatherThreads;
            for (int i = 0; i < cnt; ++i) {  // in particle order, as the reference's loop adds them
                const double mm = s_val[i] * s_m[i];
                M += mm;
                Px += mm * s_vx[i];
                Py += mm * s_vy[i];
                Pz += mm * s_vz[i];
            }
        }
        __syncthreads();
    }
    n_neg = warp_sum_u64(n_neg);
    n_warn = warp_sum_u64(n_warn);
    if ((threadIdx.x & 31) == 0) {
        if (n_neg) atomicAdd(&st->neg_clamped, n_neg);
        if (n_warn) atomicAdd(&st->neg_warned, n_warn);
    }
    if (threadIdx.x == 0) {
        const double vol = C.volume[cell];
        if (out.density) out.density[cell] = (vol > 0.0) ? M / vol : 0.0;
        const bool has = M > 0.0;
        if (out.vx) out.vx[cell] = has ? Px / M : out.meanv[0];
        if (out.vy) out.vy[cell] = has ? Py / M : out.meanv[1];
        if (out.vz) out.vz[cell] = has ? Pz / M : out.meanv[2];
        if (out.raw4) {
            out.raw4[cell] = M;
            out.raw4[C.n_cells + cell] = Px;
            out.raw4[2 * C.n_cells + cell] = Py;
            out.raw4[3 * C.n_cells + cell] = Pz;
        }
    }
}

}  // namespace

int voronoi_map_dev(KiwiCtx* ctx, const DevParticles& P, const int32_t* d_home, const KiwiVoronoiCells& cells,
                    const KernelChoice& kc, const CartOutputs& out_in, KiwiStats* stats) {
    const int64_t launches0 = ctx->launches;
    const int64_t n = P.n, nc = cells.n_cells;
    VorCells C{nc, cells.face_off, cells.vert_off, cells.vxyz, cells.face_nbr, cells.volume};
    DevStats* d_stats = nullptr;
    double* d_meanv = nullptr;
    unsigned long long* d_next = nullptr;
    KIWI_TRY(scratch_t(ctx, S_STATS, 1, &d_stats));
    KIWI_TRY(scratch_t(ctx, S_MEANV, 4, &d_meanv));
    KIWI_TRY(scratch_t(ctx, S_VOR_NEXT, 2, &d_next));
    KIWI_CUDA(ctx, cudaMemsetAsync(d_stats, 0, sizeof(DevStats), ctx->stream));
    CartOutputs out = out_in;
    out.meanv = d_meanv;
    KIWI_TRY(fp64_mean_velocity(ctx, P, d_meanv));
    if (nc <= 0) return KIWI_OK;

    // BFS work slots: a visited marker and a queue of n_cells entries each
    int sms = 0;
    KIWI_CUDA(ctx, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    int64_t slots = (int64_t)sms * 8;
    const int64_t budget = (int64_t)16 << 30;  // bytes of BFS scratch at most
    while (slots > kBfsWarpsPerBlock && slots * nc * 8 > budget) slots /= 2;
    slots = std::max<int64_t>(kBfsWarpsPerBlock, (slots / kBfsWarpsPerBlock) * kBfsWarpsPerBlock);
    const int blocks = (int)(slots / kBfsWarpsPerBlock);
    int* mark = nullptr;
    int32_t* queue = nullptr;
    int64_t *counts = nullptr, *offs = nullptr, *range = nullptr;
    KIWI_TRY(scratch_t(ctx, S_VOR_MARK, (size_t)(slots * nc), &mark));
    KIWI_TRY(scratch_t(ctx, S_VOR_QUEUE, (size_t)(slots * nc), &queue));
    KIWI_TRY(scratch_t(ctx, S_COUNT, (size_t)std::max<int64_t>(n, 1) * 2, &counts));
    KIWI_TRY(scratch_t(ctx, S_OFFS, (size_t)std::max<int64_t>(n, 1) + 1, &offs));
    KIWI_TRY(scratch_t(ctx, S_TILE_RANGE, (size_t)(2 * nc), &range));
    int64_t* d_total = offs + std::max<int64_t>(n, 1);
    KIWI_CUDA(ctx, cudaMemsetAsync(mark, 0xff, sizeof(int) * slots * nc, ctx->stream));
    KIWI_CUDA(ctx, cudaMemsetAsync(range, 0, sizeof(int64_t) * 2 * nc, ctx->stream));

    const double sup = kc.support_in_h;
    // pass 0: count
    KIWI_CUDA(ctx, cudaMemsetAsync(d_next, 0, sizeof(unsigned long long), ctx->stream));
    if (n > 0) {
        k_vor_bfs<<<blocks, 32 * kBfsWarpsPerBlock, 0, ctx->stream>>>(C, P, d_home, sup, 0, d_next, mark, queue,
                                                                     counts, nullptr, nullptr, d_stats);
        KIWI_LAUNCHED(ctx);
    }
    KIWI_TRY(exclusive_scan<int64_t>(ctx, counts, n, offs, d_total));
    int64_t total = 0;
    KIWI_CUDA(ctx, cudaMemcpyAsync(&total, d_total, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
    KIWI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (total >= (1LL << 32)) return set_err(ctx, KIWI_ERR_LIMIT, "too many (cell, particle) pairs: %lld", (long long)total);
    int32_t* pair_cells = nullptr;
    uint32_t *k0, *v0, *k1, *v1;
    KIWI_TRY(scratch_t(ctx, S_VOR_PAIRS, (size_t)std::max<int64_t>(total, 1), &pair_cells));
    KIWI_TRY(scratch_t(ctx, S_KEYS0, (size_t)std::max<int64_t>(total, 1), &k0));
    KIWI_TRY(scratch_t(ctx, S_VALS0, (size_t)std::max<int64_t>(total, 1), &v0));
    KIWI_TRY(scratch_t(ctx, S_KEYS1, (size_t)std::max<int64_t>(total, 1), &k1));
    KIWI_TRY(scratch_t(ctx, S_VALS1, (size_t)std::max<int64_t>(total, 1), &v1));
    const uint32_t* plist = v0;
    if (total > 0) {
        // pass 1: write each particle's visited cells at its offset
        KIWI_CUDA(ctx, cudaMemsetAsync(d_next, 0, sizeof(unsigned long long), ctx->stream));
        k_vor_bfs<<<blocks, 32 * kBfsWarpsPerBlock, 0, ctx->stream>>>(C, P, d_home, sup, 1, d_next, mark, queue,
                                                                     counts, offs, pair_cells, d_stats);
        KIWI_LAUNCHED(ctx);
        k_vor_pairs<<<(unsigned)((total + 255) / 256), 256, 0, ctx->stream>>>(pair_cells, total, offs, n, k0, v0);
        KIWI_LAUNCHED(ctx);
        int key_bits = 1;
        while ((1LL << key_bits) < nc) ++key_bits;
        bool second = false;
        KIWI_TRY(radix_sort_pairs(ctx, k0, v0, k1, v1, total, key_bits, &second));
        const uint32_t* sk = second ? k1 : k0;
        plist = second ? v1 : v0;
        k_cell_ranges<<<(unsigned)((total + 255) / 256), 256, 0, ctx->stream>>>(sk, total, range);
        KIWI_LAUNCHED(ctx);
    }
    KIWI_CUDA(ctx, cudaEventRecord(ctx->ev[0], ctx->stream));
    if (nc > 0x7fffffffLL) return set_err(ctx, KIWI_ERR_ARG, "too many cells (%lld)", (long long)nc);
    if (kc.cubic)
        k_vor_gather<true><<<(unsigned)nc, kGatherThreads, 0, ctx->stream>>>(C, P, kc.kernel, sup, plist, range, out, d_stats);
    else
        k_vor_gather<false><<<(unsigned)nc, kGatherThreads, 0, ctx->stream>>>(C, P, kc.kernel, sup, plist, range, out, d_stats);
    KIWI_LAUNCHED(ctx);
    KIWI_CUDA(ctx, cudaEventRecord(ctx->ev[1], ctx->stream));
    DevStats hs;
    KIWI_CUDA(ctx, cudaMemcpyAsync(&hs, d_stats, sizeof hs, cudaMemcpyDeviceToHost, ctx->stream));
    KIWI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (hs.limit_hit) return set_err(ctx, KIWI_ERR_LIMIT, "the cell walk hit its iteration cap");
    if (stats) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
        stats->bbox_pairs = total;
        stats->sphere_pairs = total;
        stats->evaluated_pairs = total;
        stats->skipped_outside = (int64_t)hs.skipped_outside;  // particles whose home cell is unresolved
        stats->neg_clamped = (int64_t)hs.neg_clamped;
        stats->neg_warned = (int64_t)hs.neg_warned;
        stats->tile_pairs = (int64_t)hs.tile_pairs;  // particles whose walk never left the home cell
        stats->gather_ms = ms;
        stats->launches = ctx->launches - launches0;
    }
    return KIWI_OK;
}

}  // namespace kiwi_b200
