// The point-set stage's coverage-grid buffer (add_coverage_grid_buffer, src/point_set.cpp:198-262): the
// cell-centred lattice of candidate points over the domain (generate_cartesian_lattice, :166-195) keeps the
// candidates that no particle's coverage sphere (radius factor x h_i) reaches, renumbered from n + 1 in
// lattice order.
//
// GPU form: the particles are binned with the reference's own bin arithmetic (floor(x / (factor x h_max))
// per axis) into a dense box of bins, stably radix-sorted by bin; one thread per candidate scans its bin and
// the 26 around it (binary searches in the sorted keys), which finds every particle whose sphere can reach
// it, exactly as the reference's hash does; a scan of the "uncovered" flags then places the survivors in
// lattice order.  Built with --fmad=false, like the other FP64 units.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>

#include "engine.hpp"
#include "prims.cuh"

using namespace kiwi_b200;

namespace {

struct Lattice {
    double x0, y0, z0, spacing;
    int nx, ny, nz;
};

// generate_cartesian_lattice's shape (src/point_set.cpp:166-180): spacing = fraction x the smallest extent,
// round(extent / spacing) candidates per axis (at least 1).
Lattice lattice_of(const double* b, double spacing_fraction) {
    const double ex = b[1] - b[0], ey = b[3] - b[2], ez = b[5] - b[4];
    Lattice L;
    L.spacing = spacing_fraction * std::min(std::min(ex, ey), ez);
    L.nx = std::max(1, (int)std::round(ex / L.spacing));
    L.ny = std::max(1, (int)std::round(ey / L.spacing));
    L.nz = std::max(1, (int)std::round(ez / L.spacing));
    L.x0 = b[0];
    L.y0 = b[2];
    L.z0 = b[4];
    return L;
}

struct PBins {
    double size;  // factor x h_max
    long long bx0, by0, bz0;
    long long nbx, nby, nbz;
};

__device__ __forceinline__ long long pbin(double v, double size) { return (long long)floor(v / size); }

__global__ void k_hmax_bins(int64_t n, const double* __restrict__ x, const double* __restrict__ y,
                            const double* __restrict__ z, double size, long long* __restrict__ mm) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long bx = pbin(x[i], size), by = pbin(y[i], size), bz = pbin(z[i], size);
    atomicMin(&mm[0], bx);
    atomicMin(&mm[1], by);
    atomicMin(&mm[2], bz);
    atomicMax(&mm[3], bx);
    atomicMax(&mm[4], by);
    atomicMax(&mm[5], bz);
}

__global__ void k_hmax(int64_t n, const double* __restrict__ h, unsigned long long* __restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double v = h[i];
    // h_max = max(0, h_i): positive doubles order like their bit patterns
    if (v > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(v));
}

__global__ void k_pkeys(int64_t n, const double* __restrict__ x, const double* __restrict__ y,
                        const double* __restrict__ z, PBins B, uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long bx = pbin(x[i], B.size) - B.bx0, by = pbin(y[i], B.size) - B.by0, bz = pbin(z[i], B.size) - B.bz0;
    keys[i] = (uint32_t)((bx * B.nby + by) * B.nbz + bz);
    vals[i] = (uint32_t)i;
}

__device__ __forceinline__ int64_t lower_bound_u32(const uint32_t* a, int64_t n, uint32_t key) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (a[mid] < key) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// 1 if no particle covers candidate c (src/point_set.cpp:234-249).
__global__ void k_uncovered(Lattice L, int64_t n, const double* __restrict__ x, const double* __restrict__ y,
                            const double* __restrict__ z, const double* __restrict__ h, double factor, PBins B,
                            const uint32_t* __restrict__ skeys, const uint32_t* __restrict__ sidx,
                            uint32_t* __restrict__ flags) {
    const int64_t nc = (int64_t)L.nx * L.ny * L.nz;
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    const int k = (int)(c % L.nz), j = (int)((c / L.nz) % L.ny), i = (int)(c / ((int64_t)L.nz * L.ny));
    const double cx = L.x0 + L.spacing * (i + 0.5), cy = L.y0 + L.spacing * (j + 0.5), cz = L.z0 + L.spacing * (k + 0.5);
    const long long bx = pbin(cx, B.size) - B.bx0, by = pbin(cy, B.size) - B.by0, bz = pbin(cz, B.size) - B.bz0;
    bool covered = false;
    for (int dx = -1; dx <= 1 && !covered; ++dx)
        for (int dy = -1; dy <= 1 && !covered; ++dy)
            for (int dz = -1; dz <= 1 && !covered; ++dz) {
                const long long qx = bx + dx, qy = by + dy, qz = bz + dz;
                if (qx < 0 || qy < 0 || qz < 0 || qx >= B.nbx || qy >= B.nby || qz >= B.nbz) continue;
                const uint32_t key = (uint32_t)((qx * B.nby + qy) * B.nbz + qz);
                for (int64_t p = lower_bound_u32(skeys, n, key); p < n && skeys[p] == key; ++p) {
                    const uint32_t q = sidx[p];
                    const double ddx = x[q] - cx, ddy = y[q] - cy, ddz = z[q] - cz;
                    const double r = factor * h[q];
                    if (ddx * ddx + ddy * ddy + ddz * ddz <= r * r) {
                        covered = true;
                        break;
                    }
                }
            }
    flags[c] = covered ? 0u : 1u;
}

__global__ void k_emit_buffer(Lattice L, const uint32_t* __restrict__ flags, const int64_t* __restrict__ offs,
                              int64_t id_base, double* __restrict__ ox, double* __restrict__ oy,
                              double* __restrict__ oz, int32_t* __restrict__ oid) {
    const int64_t nc = (int64_t)L.nx * L.ny * L.nz;
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc || !flags[c]) return;
    const int k = (int)(c % L.nz), j = (int)((c / L.nz) % L.ny), i = (int)(c / ((int64_t)L.nz * L.ny));
    const int64_t o = offs[c];
    ox[o] = L.x0 + L.spacing * (i + 0.5);
    oy[o] = L.y0 + L.spacing * (j + 0.5);
    oz[o] = L.z0 + L.spacing * (k + 0.5);
    oid[o] = (int32_t)(id_base + o + 1);
}

}  // namespace

extern "C" int64_t kiwi_coverage_grid_candidates(const double* bounds6, double spacing_fraction, int32_t* dims3) {
    if (!bounds6 || !(spacing_fraction > 0.0)) return -1;
    const Lattice L = lattice_of(bounds6, spacing_fraction);
    if (dims3) {
        dims3[0] = L.nx;
        dims3[1] = L.ny;
        dims3[2] = L.nz;
    }
    return (int64_t)L.nx * L.ny * L.nz;
}

extern "C" int kiwi_coverage_grid_buffer(KiwiCtx* ctx, int64_t n, const double* x, const double* y, const double* z,
                                         const double* h, const double* bounds6, double spacing_fraction,
                                         double coverage_radius_factor, int64_t capacity, double* out_x,
                                         double* out_y, double* out_z, int32_t* out_id, int64_t* n_added) {
    if (!ctx) return KIWI_ERR_ARG;
    KIWI_CUDA(ctx, cudaSetDevice(ctx->device));
    if (!n_added || !bounds6) return set_err(ctx, KIWI_ERR_ARG, "coverage buffer: a null argument");
    if (n < 0 || (n > 0 && (!x || !y || !z || !h))) return set_err(ctx, KIWI_ERR_ARG, "coverage buffer: bad particle arrays");
    if (!(bounds6[0] < bounds6[1]) || !(bounds6[2] < bounds6[3]) || !(bounds6[4] < bounds6[5]))
        return set_err(ctx, KIWI_ERR_ARG, "domain bounds must satisfy min < max on every axis");
    if (!(spacing_fraction > 0.0)) return set_err(ctx, KIWI_ERR_ARG, "buffer.coverage_grid.spacing_fraction must be > 0");
    const Lattice L = lattice_of(bounds6, spacing_fraction);
    const int64_t nc = (int64_t)L.nx * L.ny * L.nz;
    if (nc > (1LL << 31)) return set_err(ctx, KIWI_ERR_LIMIT, "coverage buffer: too many lattice candidates (%lld)", (long long)nc);
    const int64_t np = std::max<int64_t>(n, 1);
    // stage the particles
    double* d = nullptr;
    KIWI_TRY(scratch_t(ctx, S_PART, (size_t)(4 * np), &d));
    const size_t b = sizeof(double) * (size_t)n;
    if (n > 0) {
        KIWI_CUDA(ctx, cudaMemcpyAsync(d, x, b, cudaMemcpyHostToDevice, ctx->stream));
        KIWI_CUDA(ctx, cudaMemcpyAsync(d + np, y, b, cudaMemcpyHostToDevice, ctx->stream));
        KIWI_CUDA(ctx, cudaMemcpyAsync(d + 2 * np, z, b, cudaMemcpyHostToDevice, ctx->stream));
        KIWI_CUDA(ctx, cudaMemcpyAsync(d + 3 * np, h, b, cudaMemcpyHostToDevice, ctx->stream));
    }
    // h_max and the particles' bin box
    long long* mm = nullptr;
    KIWI_TRY(scratch_t(ctx, S_MISC2, 8, &mm));
    unsigned long long* hm = reinterpret_cast<unsigned long long*>(mm + 6);
    KIWI_CUDA(ctx, cudaMemsetAsync(hm, 0, sizeof(unsigned long long), ctx->stream));
    const unsigned gp = (unsigned)((np + 255) / 256);
    if (n > 0) {
        k_hmax<<<gp, 256, 0, ctx->stream>>>(n, d + 3 * np, hm);
        KIWI_LAUNCHED(ctx);
    }
    unsigned long long hbits = 0;
    KIWI_CUDA(ctx, cudaMemcpyAsync(&hbits, hm, sizeof hbits, cudaMemcpyDeviceToHost, ctx->stream));
    KIWI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    double h_max = 0.0;
    std::memcpy(&h_max, &hbits, sizeof h_max);
    if (!(h_max > 0.0)) return set_err(ctx, KIWI_ERR_ARG, "add_coverage_grid_buffer: all smoothing lengths are <= 0");
    PBins B;
    B.size = coverage_radius_factor * h_max;
    if (!(B.size > 0.0)) return set_err(ctx, KIWI_ERR_ARG, "buffer.coverage_grid.coverage_radius_factor must be > 0");
    long long init[6] = {LLONG_MAX, LLONG_MAX, LLONG_MAX, LLONG_MIN, LLONG_MIN, LLONG_MIN};
    KIWI_CUDA(ctx, cudaMemcpyAsync(mm, init, sizeof init, cudaMemcpyHostToDevice, ctx->stream));
    k_hmax_bins<<<gp, 256, 0, ctx->stream>>>(n, d, d + np, d + 2 * np, B.size, mm);
    KIWI_LAUNCHED(ctx);
    long long box[6];
    KIWI_CUDA(ctx, cudaMemcpyAsync(box, mm, sizeof box, cudaMemcpyDeviceToHost, ctx->stream));
    KIWI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    B.bx0 = box[0];
    B.by0 = box[1];
    B.bz0 = box[2];
    B.nbx = box[3] - box[0] + 1;
    B.nby = box[4] - box[1] + 1;
    B.nbz = box[5] - box[2] + 1;
    if ((double)B.nbx * (double)B.nby * (double)B.nbz >= 4294967295.0)
        return set_err(ctx, KIWI_ERR_LIMIT,
                       "coverage buffer: the particles span more than 2^32 coverage bins (factor x h_max is tiny "
                       "against their extent)");
    const int64_t nbins = B.nbx * B.nby * B.nbz;
    // particles sorted by bin (stable: ascending particle index within a bin)
    uint32_t *k0, *v0, *k1, *v1;
    KIWI_TRY(scratch_t(ctx, S_KEYS0, (size_t)np, &k0));
    KIWI_TRY(scratch_t(ctx, S_VALS0, (size_t)np, &v0));
    KIWI_TRY(scratch_t(ctx, S_KEYS1, (size_t)np, &k1));
    KIWI_TRY(scratch_t(ctx, S_VALS1, (size_t)np, &v1));
    k_pkeys<<<gp, 256, 0, ctx->stream>>>(n, d, d + np, d + 2 * np, B, k0, v0);
    KIWI_LAUNCHED(ctx);
    int key_bits = 1;
    while (key_bits < 32 && (1LL << key_bits) < nbins) ++key_bits;
    bool second = false;
    KIWI_TRY(radix_sort_pairs(ctx, k0, v0, k1, v1, n, key_bits, &second));
    const uint32_t* sk = second ? k1 : k0;
    const uint32_t* sv = second ? v1 : v0;
    // candidates: uncovered flags, their scan, the survivors in lattice order
    uint32_t* flags = nullptr;
    int64_t* offs = nullptr;
    KIWI_TRY(scratch_t(ctx, S_COUNT, (size_t)std::max<int64_t>(nc, 1), &flags));
    KIWI_TRY(scratch_t(ctx, S_OFFS, (size_t)nc + 1, &offs));
    const unsigned gc = (unsigned)((nc + 255) / 256);
    k_uncovered<<<gc, 256, 0, ctx->stream>>>(L, n, d, d + np, d + 2 * np, d + 3 * np, coverage_radius_factor, B, sk,
                                             sv, flags);
    KIWI_LAUNCHED(ctx);
    KIWI_TRY(exclusive_scan<uint32_t>(ctx, flags, nc, offs, offs + nc));
    int64_t added = 0;
    KIWI_CUDA(ctx, cudaMemcpyAsync(&added, offs + nc, sizeof added, cudaMemcpyDeviceToHost, ctx->stream));
    KIWI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *n_added = added;
    if (!out_x && !out_y && !out_z && !out_id) return KIWI_OK;  // count only
    if (!out_x || !out_y || !out_z || !out_id)
        return set_err(ctx, KIWI_ERR_ARG, "coverage buffer: give all four output arrays or none");
    if (added > capacity)
        return set_err(ctx, KIWI_ERR_ARG, "coverage buffer: %lld points do not fit the output arrays (%lld)",
                       (long long)added, (long long)capacity);
    double* o = nullptr;
    int32_t* oi = nullptr;
    KIWI_TRY(scratch_t(ctx, S_OUT, (size_t)(3 * std::max<int64_t>(added, 1)), &o));
    KIWI_TRY(scratch_t(ctx, S_VOR_HOME, (size_t)std::max<int64_t>(added, 1), &oi));
    const int64_t na = std::max<int64_t>(added, 1);
    k_emit_buffer<<<gc, 256, 0, ctx->stream>>>(L, flags, offs, n, o, o + na, o + 2 * na, oi);
    KIWI_LAUNCHED(ctx);
    if (added > 0) {
        const size_t ba = sizeof(double) * (size_t)added;
        KIWI_CUDA(ctx, cudaMemcpyAsync(out_x, o, ba, cudaMemcpyDeviceToHost, ctx->stream));
        KIWI_CUDA(ctx, cudaMemcpyAsync(out_y, o + na, ba, cudaMemcpyDeviceToHost, ctx->stream));
        KIWI_CUDA(ctx, cudaMemcpyAsync(out_z, o + 2 * na, ba, cudaMemcpyDeviceToHost, ctx->stream));
        KIWI_CUDA(ctx, cudaMemcpyAsync(out_id, oi, sizeof(int32_t) * (size_t)added, cudaMemcpyDeviceToHost, ctx->stream));
    }
    KIWI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return KIWI_OK;
}
