// Device primitives for the binning step: an exclusive prefix sum and a stable LSD radix sort of
// (uint32 key, uint32 value) pairs.  Both are deterministic (no floating point, and the sort's
// stability keeps equal keys in input order, which is what makes every tile's particle list come out
// in ascending particle order).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "ctx.hpp"

namespace kiwi_b200 {

// ------------------------------------------------------------------ exclusive scan (int64)

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanSeg = kScanThreads * kScanItems;

template <class T>
__device__ __forceinline__ int64_t block_sum_i64(int64_t v, int64_t* sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[w] = v;
    __syncthreads();
    if (w == 0) {
        v = (l < (int)(blockDim.x >> 5)) ? sh[l] : 0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    __syncthreads();
    return v;  // valid in thread 0
}

template <class T>
__global__ void k_scan_partials(const T* __restrict__ in, int64_t n, int64_t* __restrict__ partial) {
    __shared__ int64_t sh[32];
    const int64_t base = (int64_t)blockIdx.x * kScanSeg;
    int64_t s = 0;
    for (int i = threadIdx.x; i < kScanSeg; i += kScanThreads) {
        const int64_t k = base + i;
        if (k < n) s += (int64_t)in[k];
    }
    s = block_sum_i64<T>(s, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// Single block: exclusive scan of the block partials in place, total to *total.
static __global__ void k_scan_partials_scan(int64_t* __restrict__ partial, int64_t nblocks, int64_t* __restrict__ total) {
    __shared__ int64_t sh[kScanThreads];
    __shared__ int64_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int64_t base = 0; base < nblocks; base += kScanThreads) {
        const int64_t k = base + threadIdx.x;
        const int64_t v = (k < nblocks) ? partial[k] : 0;
        sh[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < kScanThreads; o <<= 1) {
            int64_t t = (threadIdx.x >= o) ? sh[threadIdx.x - o] : 0;
            __syncthreads();
            sh[threadIdx.x] += t;
            __syncthreads();
        }
        if (k < nblocks) partial[k] = carry + sh[threadIdx.x] - v;
        __syncthreads();
        if (threadIdx.x == kScanThreads - 1) carry += sh[threadIdx.x];
        __syncthreads();
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

template <class T>
__global__ void k_scan_apply(const T* __restrict__ in, int64_t n, const int64_t* __restrict__ partial,
                             int64_t* __restrict__ out) {
    __shared__ int64_t vals[kScanSeg];
    __shared__ int64_t tsum[kScanThreads];
    const int64_t base = (int64_t)blockIdx.x * kScanSeg;
    for (int i = threadIdx.x; i < kScanSeg; i += kScanThreads) {
        const int64_t k = base + i;
        vals[i] = (k < n) ? (int64_t)in[k] : 0;
    }
    __syncthreads();
    int64_t run = 0;
    const int first = threadIdx.x * kScanItems;
    for (int i = 0; i < kScanItems; ++i) run += vals[first + i];
    tsum[threadIdx.x] = run;
    __syncthreads();
    for (int o = 1; o < kScanThreads; o <<= 1) {
        int64_t t = (threadIdx.x >= o) ? tsum[threadIdx.x - o] : 0;
        __syncthreads();
        tsum[threadIdx.x] += t;
        __syncthreads();
    }
    int64_t acc = partial[blockIdx.x] + tsum[threadIdx.x] - run;
    for (int i = 0; i < kScanItems; ++i) {
        const int64_t k = base + first + i;
        const int64_t v = vals[first + i];
        if (k < n) out[k] = acc;
        acc += v;
    }
}

// out[i] = sum_{j<i} in[j]; *d_total = sum of all (device).  Scratch: S_SCAN.
template <class T>
inline int exclusive_scan(KiwiCtx* ctx, const T* d_in, int64_t n, int64_t* d_out, int64_t* d_total) {
    const int64_t nb = (n + kScanSeg - 1) / kScanSeg;
    int64_t* partial = nullptr;
    KIWI_TRY(scratch_t(ctx, S_SCAN, (size_t)(nb > 0 ? nb : 1), &partial));
    if (n == 0) {
        KIWI_CUDA(ctx, cudaMemsetAsync(d_total, 0, sizeof(int64_t), ctx->stream));
        return KIWI_OK;
    }
    k_scan_partials<T><<<(unsigned)nb, kScanThreads, 0, ctx->stream>>>(d_in, n, partial);
    KIWI_LAUNCHED(ctx);
    k_scan_partials_scan<<<1, kScanThreads, 0, ctx->stream>>>(partial, nb, d_total);
    KIWI_LAUNCHED(ctx);
    k_scan_apply<T><<<(unsigned)nb, kScanThreads, 0, ctx->stream>>>(d_in, n, partial, d_out);
    KIWI_LAUNCHED(ctx);
    return KIWI_OK;
}

// ------------------------------------------------------------------ stable LSD radix sort

constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;
constexpr int kSortThreads = 256;
constexpr int kSortRounds = 8;
constexpr int kSortSeg = kSortThreads * kSortRounds;  // elements per block segment

static __global__ void k_radix_hist(const uint32_t* __restrict__ keys, int64_t n, int shift, uint32_t* __restrict__ hist,
                             int nblocks) {
    __shared__ uint32_t h[kRadix];
    for (int i = threadIdx.x; i < kRadix; i += kSortThreads) h[i] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kSortSeg;
    for (int i = threadIdx.x; i < kSortSeg; i += kSortThreads) {
        const int64_t k = base + i;
        if (k < n) atomicAdd(&h[(keys[k] >> shift) & (kRadix - 1)], 1u);
    }
    __syncthreads();
    // digit-major layout: hist[d * nblocks + b]
    for (int d = threadIdx.x; d < kRadix; d += kSortThreads) hist[(int64_t)d * nblocks + blockIdx.x] = h[d];
}

// Stable scatter: element order inside a block segment is round-major, then thread order, i.e. the
// input order; ranks among equal digits follow that order.
static __global__ void k_radix_scatter(const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin, int64_t n,
                                int shift, const int64_t* __restrict__ offs, int nblocks, uint32_t* __restrict__ kout,
                                uint32_t* __restrict__ vout) {
    __shared__ int64_t base_off[kRadix];
    __shared__ uint32_t wcount[kSortThreads / 32][kRadix];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int d = threadIdx.x; d < kRadix; d += kSortThreads) base_off[d] = offs[(int64_t)d * nblocks + blockIdx.x];
    for (int i = threadIdx.x; i < (kSortThreads / 32) * kRadix; i += kSortThreads) (&wcount[0][0])[i] = 0;
    __syncthreads();
    const unsigned lt_mask = (1u << lane) - 1u;
    const int64_t seg = (int64_t)blockIdx.x * kSortSeg;
    for (int r = 0; r < kSortRounds; ++r) {
        const int64_t k = seg + (int64_t)r * kSortThreads + threadIdx.x;
        const bool valid = k < n;
        uint32_t key = 0, val = 0;
        int digit = kRadix;  // invalid lanes form their own group and are never counted
        if (valid) {
            key = kin[k];
            val = vin[k];
            digit = (key >> shift) & (kRadix - 1);
        }
        const unsigned peers = __match_any_sync(0xffffffffu, digit);
        const int rank_in_warp = __popc(peers & lt_mask);
        const int leader = __ffs(peers) - 1;
        if (valid && lane == leader) wcount[warp][digit] = __popc(peers);
        __syncthreads();
        if (valid) {
            int64_t pos = base_off[digit] + rank_in_warp;
            for (int w = 0; w < warp; ++w) pos += wcount[w][digit];
            kout[pos] = key;
            vout[pos] = val;
        }
        __syncthreads();
        for (int d = threadIdx.x; d < kRadix; d += kSortThreads) {
            uint32_t s = 0;
            for (int w = 0; w < kSortThreads / 32; ++w) {
                s += wcount[w][d];
                wcount[w][d] = 0;
            }
            base_off[d] += s;
        }
        __syncthreads();
    }
}

// Sorts (keys, vals) by key, stably, over the low `key_bits` bits.  Ping-pongs between the given
// buffers; *result_is_second tells which pair holds the result.
inline int radix_sort_pairs(KiwiCtx* ctx, uint32_t* k0, uint32_t* v0, uint32_t* k1, uint32_t* v1, int64_t n,
                            int key_bits, bool* result_is_second) {
    *result_is_second = false;
    if (n <= 1) return KIWI_OK;
    const int nblocks = (int)((n + kSortSeg - 1) / kSortSeg);
    uint32_t* hist = nullptr;
    int64_t* offs = nullptr;
    KIWI_TRY(scratch_t(ctx, S_HIST, (size_t)kRadix * nblocks, &hist));
    KIWI_TRY(scratch_t(ctx, S_MISC3, (size_t)kRadix * nblocks + 1, &offs));
    int64_t* d_total = offs + (size_t)kRadix * nblocks;
    int passes = (key_bits + kRadixBits - 1) / kRadixBits;
    if (passes < 1) passes = 1;
    uint32_t *ki = k0, *vi = v0, *ko = k1, *vo = v1;
    for (int p = 0; p < passes; ++p) {
        const int shift = p * kRadixBits;
        k_radix_hist<<<nblocks, kSortThreads, 0, ctx->stream>>>(ki, n, shift, hist, nblocks);
        KIWI_LAUNCHED(ctx);
        KIWI_TRY(exclusive_scan<uint32_t>(ctx, hist, (int64_t)kRadix * nblocks, offs, d_total));
        k_radix_scatter<<<nblocks, kSortThreads, 0, ctx->stream>>>(ki, vi, n, shift, offs, nblocks, ko, vo);
        KIWI_LAUNCHED(ctx);
        uint32_t* t;
        t = ki; ki = ko; ko = t;
        t = vi; vi = vo; vo = t;
    }
    *result_is_second = (ki == k1);
    return KIWI_OK;
}

}  // namespace kiwi_b200
