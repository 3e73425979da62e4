// The density lookup table of the tabulated cubic integral: generation on the GPU
// (generate_density_table, src/kernel_integral.cpp:57-119), loading from the reference's text format
// (load_density_table, :20-55), the batched scalar lookup (gridded_integral, :136-190) and the C ABI
// around them.  A context holds at most one table; a tabulated call on a context without one generates
// the canonical table first, as load_or_generate_density_table (src/mapping.cpp:281-300) does when no
// table file is configured.  Built with --fmad=false, like the other FP64 units.
#include <cuda_runtime.h>

#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "engine.hpp"
#include "kiwi_math.cuh"
#include "tabulated.cuh"

using namespace kiwi_b200;

namespace {

// One thread per table entry (i in [1, nr0], j in [0, nR_0), k in [0, nphi)) of the canonical shape:
// the cubic pyramid mass at h = 1 on the table's grid of (r0, mu0, phi).  At j = 0, mu0 = 0 and R_0 is
// +inf, which the closed form takes to the finite limit, as in the reference.  Row nr0 is also written to
// the padding row nr0 + 1.
__global__ void k_tab_generate(TabDev t, double* __restrict__ v) {
    const int64_t per_i = (int64_t)t.nR_0 * t.nphi;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)t.nr0 * per_i) return;
    const int i = 1 + (int)(e / per_i);
    const int j = (int)((e % per_i) / t.nphi), k = (int)(e % t.nphi);
    const int n = t.nR_01;  // one sub-grid size for the mu0 and phi axes (150 in the canonical shape)
    const double h = 1.0;
    const double r0 = (i <= t.nr01) ? (t.rl / t.nr01) * i * h : t.rl + ((2.0 - t.rl) / t.nr02) * (i - t.nr01) * h;
    const double mu0 = (j < n) ? (t.mul / (n - 1)) * j : t.mul + ((1.0 - t.mul) / n) * (j - n + 1);
    const double R_0 = r0 * sqrt(1.0 - mu0 * mu0) / mu0;
    const double phi = (k < n) ? acos((t.cphil / (n - 1)) * k) : acos(t.cphil + ((1.0 - t.cphil) / n) * (k - n + 1));
    const double val = cubic_full_integral(h, phi, r0, R_0);
    const int64_t row = (int64_t)(t.nR_0 + 1) * (t.nphi + 1);
    const int64_t at = (int64_t)i * row + (int64_t)j * (t.nphi + 1) + k;
    v[at] = val;
    if (i == t.nr0) v[at + row] = val;
}

__global__ void k_gridded_batch(TabDev t, int64_t n, const double* __restrict__ h, const double* __restrict__ phi,
                                const double* __restrict__ r0, const double* __restrict__ R0, double* __restrict__ out,
                                unsigned long long* __restrict__ clamps) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned nc = 0;
    if (i < n) out[i] = tab_gridded(t, h[i], phi[i], r0[i], R0[i], nc);
    unsigned long long v = nc;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(clamps, v);
}

int64_t table_values(const TabDev& t) { return (int64_t)(t.nr0 + 2) * (t.nR_0 + 1) * (t.nphi + 1); }

void table_release(KiwiCtx* ctx) {
    if (ctx->tab.v) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(const_cast<double*>(ctx->tab.v));
    }
    ctx->tab = TabDev{};
    ctx->tab_bytes = 0;
}

// Shape check beyond the reference's reader (which divides by nR_01 - 1 and nphi1 - 1 and sizes the
// table from the header without bounds): every sub-grid non-empty, the first mu0 and phi sub-grids of at
// least 2 points, split points inside (0, top), and at most 2^31 values.
int table_shape(KiwiCtx* ctx, TabDev& t) {
    if (t.nr01 < 1 || t.nr02 < 1 || t.nR_01 < 2 || t.nR_02 < 1 || t.nphi1 < 2 || t.nphi2 < 1 ||
        !(t.rl > 0.0 && t.rl < 2.0) || !(t.mul > 0.0 && t.mul < 1.0) || !(t.cphil > 0.0 && t.cphil < 1.0))
        return set_err(ctx, KIWI_ERR_ARG, "density lookup table shape is not usable");
    t.nr0 = t.nr01 + t.nr02;
    t.nR_0 = t.nR_01 + t.nR_02;
    t.nphi = t.nphi1 + t.nphi2;
    if ((double)(t.nr0 + 2) * (t.nR_0 + 1) * (t.nphi + 1) > 2147483648.0)
        return set_err(ctx, KIWI_ERR_ARG, "density lookup table is too large (%d x %d x %d)", t.nr0, t.nR_0, t.nphi);
    return KIWI_OK;
}

int table_alloc(KiwiCtx* ctx, TabDev& t) {
    const size_t bytes = sizeof(double) * (size_t)table_values(t);
    double* d = nullptr;
    cudaError_t e = cudaMalloc(&d, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_err(ctx, KIWI_ERR_ALLOC, "cudaMalloc of %zu bytes for the density lookup table failed: %s", bytes,
                       cudaGetErrorString(e));
    }
    t.v = d;
    ctx->tab = t;
    ctx->tab_bytes = bytes;
    return KIWI_OK;
}

int table_generate(KiwiCtx* ctx) {
    table_release(ctx);
    TabDev t;
    t.nr01 = 50; t.nr02 = 199;
    t.nR_01 = 150; t.nR_02 = 150;
    t.nphi1 = 150; t.nphi2 = 150;
    t.rl = 0.1; t.mul = 0.98; t.cphil = 0.98;
    KIWI_TRY(table_shape(ctx, t));
    KIWI_TRY(table_alloc(ctx, t));
    double* v = const_cast<double*>(ctx->tab.v);
    KIWI_CUDA(ctx, cudaMemsetAsync(v, 0, ctx->tab_bytes, ctx->stream));
    const int64_t n = (int64_t)t.nr0 * t.nR_0 * t.nphi;
    k_tab_generate<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(ctx->tab, v);
    KIWI_LAUNCHED(ctx);
    KIWI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return KIWI_OK;
}

// Whitespace-separated tokens of a text buffer, read like the reference's formatted extraction.
struct Tokens {
    const char* p;
    const char* end;
    bool next_int(int& out) {
        skip();
        if (p >= end) return false;
        char* q = nullptr;
        errno = 0;
        const long v = strtol(p, &q, 10);
        if (q == p || errno || v < -2147483647L || v > 2147483647L) return false;
        p = q;
        out = (int)v;
        return true;
    }
    bool next_double(double& out) {
        skip();
        if (p >= end) return false;
        char* q = nullptr;
        out = strtod(p, &q);
        if (q == p) return false;
        p = q;
        return true;
    }
    void skip() {
        while (p < end && (*p == ' ' || *p == '\n' || *p == '\t' || *p == '\r' || *p == '\v' || *p == '\f')) ++p;
    }
};

int table_load(KiwiCtx* ctx, const char* path) {
    if (!path) return set_err(ctx, KIWI_ERR_ARG, "density lookup table path is null");
    FILE* f = fopen(path, "rb");
    if (!f) return set_err(ctx, KIWI_ERR_ARG, "could not open density lookup table: %s", path);
    std::string text;
    char buf[1 << 16];
    size_t got;
    while ((got = fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, got);
    fclose(f);
    text.push_back('\0');  // strtod/strtol stop at the terminator
    Tokens tk{text.data(), text.data() + text.size() - 1};
    TabDev t;
    if (!(tk.next_int(t.nr01) && tk.next_int(t.nR_01) && tk.next_int(t.nphi1) && tk.next_double(t.rl) &&
          tk.next_double(t.mul) && tk.next_double(t.cphil) && tk.next_int(t.nr02) && tk.next_int(t.nR_02) &&
          tk.next_int(t.nphi2)))
        return set_err(ctx, KIWI_ERR_ARG, "density lookup table header is malformed: %s", path);
    KIWI_TRY(table_shape(ctx, t));
    // rows 1..nr0 of the file, j < nR_0, k < nphi; row 0, the last j and k slices stay zero and row nr0 + 1
    // repeats row nr0
    std::vector<double> h((size_t)table_values(t), 0.0);
    const int64_t row = (int64_t)(t.nR_0 + 1) * (t.nphi + 1);
    for (int i = 1; i <= t.nr0; ++i)
        for (int j = 0; j < t.nR_0; ++j)
            for (int k = 0; k < t.nphi; ++k)
                if (!tk.next_double(h[(size_t)(i * row + (int64_t)j * (t.nphi + 1) + k)]))
                    return set_err(ctx, KIWI_ERR_ARG, "density lookup table is truncated (short read): %s", path);
    for (int j = 0; j < t.nR_0; ++j)
        for (int k = 0; k < t.nphi; ++k) {
            const size_t a = (size_t)(t.nr0 * row + (int64_t)j * (t.nphi + 1) + k);
            h[a + row] = h[a];
        }
    table_release(ctx);
    KIWI_TRY(table_alloc(ctx, t));
    KIWI_CUDA(ctx, cudaMemcpyAsync(const_cast<double*>(ctx->tab.v), h.data(), ctx->tab_bytes, cudaMemcpyHostToDevice,
                                   ctx->stream));
    KIWI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return KIWI_OK;
}

}  // namespace

namespace kiwi_b200 {

int table_ensure(KiwiCtx* ctx, TabDev* out) {
    if (!ctx->tab.v) KIWI_TRY(table_generate(ctx));
    *out = ctx->tab;
    return KIWI_OK;
}

void table_free(KiwiCtx* ctx) { table_release(ctx); }

}  // namespace kiwi_b200

extern "C" {

int kiwi_density_table_generate(KiwiCtx* ctx) {
    if (!ctx) return KIWI_ERR_ARG;
    KIWI_CUDA(ctx, cudaSetDevice(ctx->device));
    return table_generate(ctx);
}

int kiwi_density_table_load(KiwiCtx* ctx, const char* path) {
    if (!ctx) return KIWI_ERR_ARG;
    KIWI_CUDA(ctx, cudaSetDevice(ctx->device));
    return table_load(ctx, path);
}

int kiwi_density_table_set(KiwiCtx* ctx, const KiwiDensityTableInfo* info, const double* values) {
    if (!ctx || !info || !values) return KIWI_ERR_ARG;
    KIWI_CUDA(ctx, cudaSetDevice(ctx->device));
    TabDev t;
    t.nr01 = info->nr01; t.nR_01 = info->nR_01; t.nphi1 = info->nphi1;
    t.nr02 = info->nr02; t.nR_02 = info->nR_02; t.nphi2 = info->nphi2;
    t.rl = info->rl; t.mul = info->mul; t.cphil = info->cphil;
    KIWI_TRY(table_shape(ctx, t));
    if (info->n_values != table_values(t))
        return set_err(ctx, KIWI_ERR_ARG, "n_values %lld does not match the table's shape (%lld)",
                       (long long)info->n_values, (long long)table_values(t));
    table_release(ctx);
    KIWI_TRY(table_alloc(ctx, t));
    KIWI_CUDA(ctx, cudaMemcpyAsync(const_cast<double*>(ctx->tab.v), values, ctx->tab_bytes, cudaMemcpyHostToDevice,
                                   ctx->stream));
    KIWI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return KIWI_OK;
}

int kiwi_density_table_info(KiwiCtx* ctx, KiwiDensityTableInfo* info) {
    if (!ctx || !info) return KIWI_ERR_ARG;
    if (!ctx->tab.v) return set_err(ctx, KIWI_ERR_ARG, "the context holds no density lookup table");
    const TabDev& t = ctx->tab;
    info->nr01 = t.nr01; info->nR_01 = t.nR_01; info->nphi1 = t.nphi1;
    info->nr02 = t.nr02; info->nR_02 = t.nR_02; info->nphi2 = t.nphi2;
    info->rl = t.rl; info->mul = t.mul; info->cphil = t.cphil;
    info->n_values = table_values(t);
    return KIWI_OK;
}

int kiwi_density_table_read(KiwiCtx* ctx, double* values, int64_t n) {
    if (!ctx) return KIWI_ERR_ARG;
    if (!ctx->tab.v) return set_err(ctx, KIWI_ERR_ARG, "the context holds no density lookup table");
    if (!values || n != table_values(ctx->tab))
        return set_err(ctx, KIWI_ERR_ARG, "values must hold the table's %lld values", (long long)table_values(ctx->tab));
    KIWI_CUDA(ctx, cudaSetDevice(ctx->device));
    KIWI_CUDA(ctx, cudaMemcpyAsync(values, ctx->tab.v, ctx->tab_bytes, cudaMemcpyDeviceToHost, ctx->stream));
    KIWI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return KIWI_OK;
}

void kiwi_density_table_release(KiwiCtx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    table_release(ctx);
}

int kiwi_gridded_integral_batch(KiwiCtx* ctx, int64_t n, const double* h, const double* phi, const double* r0,
                                const double* R_0, double* out, int64_t* clamps) {
    if (!ctx) return KIWI_ERR_ARG;
    KIWI_CUDA(ctx, cudaSetDevice(ctx->device));
    if (n < 0 || (n > 0 && (!h || !phi || !r0 || !R_0 || !out))) return set_err(ctx, KIWI_ERR_ARG, "bad arrays");
    TabDev t;
    KIWI_TRY(table_ensure(ctx, &t));
    if (clamps) *clamps = 0;
    if (n == 0) return KIWI_OK;
    double* d = nullptr;
    KIWI_TRY(scratch_t(ctx, S_MISC0, (size_t)(5 * n), &d));
    unsigned long long* dc = nullptr;
    KIWI_TRY(scratch_t(ctx, S_MISC1, 1, &dc));
    const size_t b = sizeof(double) * (size_t)n;
    KIWI_CUDA(ctx, cudaMemcpyAsync(d, h, b, cudaMemcpyHostToDevice, ctx->stream));
    KIWI_CUDA(ctx, cudaMemcpyAsync(d + n, phi, b, cudaMemcpyHostToDevice, ctx->stream));
    KIWI_CUDA(ctx, cudaMemcpyAsync(d + 2 * n, r0, b, cudaMemcpyHostToDevice, ctx->stream));
    KIWI_CUDA(ctx, cudaMemcpyAsync(d + 3 * n, R_0, b, cudaMemcpyHostToDevice, ctx->stream));
    KIWI_CUDA(ctx, cudaMemsetAsync(dc, 0, sizeof *dc, ctx->stream));
    k_gridded_batch<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(t, n, d, d + n, d + 2 * n, d + 3 * n,
                                                                          d + 4 * n, dc);
    KIWI_LAUNCHED(ctx);
    unsigned long long hc = 0;
    KIWI_CUDA(ctx, cudaMemcpyAsync(out, d + 4 * n, b, cudaMemcpyDeviceToHost, ctx->stream));
    KIWI_CUDA(ctx, cudaMemcpyAsync(&hc, dc, sizeof hc, cudaMemcpyDeviceToHost, ctx->stream));
    KIWI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (clamps) *clamps = (int64_t)hc;
    return KIWI_OK;
}

}  // extern "C"
