// Adjoint of the Cartesian sph-to-grid stage (no counterpart in the reference, which has no gradients).
//
// The forward pass produces, per cell c, the raw sums M_c = sum_p m_p K_pc and P_c = sum_p m_p K_pc v_p,
// where K_pc = max(Msum_pc, 0) is the particle's kernel mass inside the cell (src/cartesian_grid.cpp:
// 256-277).  Given the cotangents gM_c = dL/dM_c and gP_c = dL/dP_c, the adjoint returns per particle
//   dL/dm_p     = sum_c K_pc (gM_c + v_p . gP_c)
//   dL/dv_p     = m_p sum_c K_pc gP_c
//   dL/dtheta_p = m_p sum_c dK_pc/dtheta (gM_c + v_p . gP_c),   theta = x, y, z, h.
// The per-pair cell integrals are recomputed, not stored: the face walk is instantiated with the Dual4
// type, which carries d/dx, d/dy, d/dz, d/dh of every intermediate through the same operations, so the
// value part equals the forward's Msum bit for bit and the derivative part is the exact derivative of the
// evaluated formula (branch choices are taken on values).  A clamped pair (Msum < 0) has K = 0 and no
// gradient.  The pairs are those of the forward's default evaluation: the cells of the particle's
// support bounding box whose closest point lies within the support radius.
//
// One warp per particle: the lanes stride over the particle's support cells and the eight per-lane sums
// are combined by a fixed xor-shuffle tree, so the result is deterministic and no atomics touch the
// gradients.
#include <cuda_runtime.h>

#include "cart_common.cuh"
#include "ctx.hpp"
#include "dual.cuh"
#include "engine.hpp"
#include "kiwi_math.cuh"

namespace kiwi_b200 {

namespace {

constexpr int kAdjThreads = 128;
constexpr int kAdjWarps = kAdjThreads / 32;

struct AdjGrads {
    double *x, *y, *z, *h, *m, *vx, *vy, *vz;
};

__global__ void __launch_bounds__(kAdjThreads) k_cart_adjoint(DevParticles P, CartGeom g,
                                                             const double* __restrict__ cot, AdjGrads G,
                                                             DevStats* __restrict__ st) {
    const int lane = threadIdx.x & 31;
    const int64_t nwarps = (int64_t)gridDim.x * kAdjWarps;
    const int64_t ncell = (int64_t)g.nx * g.ny * g.nz;
    unsigned long long n_eval = 0, n_neg = 0;
    for (int64_t p = (int64_t)blockIdx.x * kAdjWarps + threadIdx.x / 32; p < P.n; p += nwarps) {
        const double x0 = P.x[p], y0 = P.y[p], z0 = P.z[p], h = P.h[p];
        const double pvx = P.vx[p], pvy = P.vy[p], pvz = P.vz[p], pm = P.m[p];
        // 0: sum K gs; 1-4: sum dK/d(x,y,z,h) gs; 5-7: sum K gP   (gs = gM + v . gP)
        double acc[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[k] = 0.0;
        CellBox b;
        bool outside;
        if (particle_cell_box(g, x0, y0, z0, h, b, &outside)) {
            const int dy = b.y1 - b.y0 + 1, dz = b.z1 - b.z0 + 1;
            const int64_t nb = (int64_t)(b.x1 - b.x0 + 1) * dy * dz;
            const double radius = mul_rn(g.support_in_h, h);
            for (int64_t k = lane; k < nb; k += 32) {
                const int iz = b.z0 + (int)(k % dz);
                const int iy = b.y0 + (int)((k / dz) % dy);
                const int ix = b.x0 + (int)(k / ((int64_t)dz * dy));
                const double cx = cell_centre(g.x_min, ix, g.dpx);
                const double cy = cell_centre(g.y_min, iy, g.dpy);
                const double cz = cell_centre(g.z_min, iz, g.dpz);
                const double ex = fmax(fabs(x0 - cx) - g.hpx, 0.0);
                const double ey = fmax(fabs(y0 - cy) - g.hpy, 0.0);
                const double ez = fmax(fabs(z0 - cz) - g.hpz, 0.0);
                if (!(ex * ex + ey * ey + ez * ez < radius * radius)) continue;
                CubicEvalT<Dual4> ev;
                ev.h = Dual4::seed(h, 3);
                const Dual4 msum = box_cell_msum<Dual4>(Dual4::seed(x0, 0), Dual4::seed(y0, 1), Dual4::seed(z0, 2),
                                                        2 * ev.h, cx, cy, cz, g.hpx, g.hpy, g.hpz, ev);
                ++n_eval;
                if (msum.v < 0.0) {
                    ++n_neg;
                    continue;
                }
                if (msum.v == 0.0) continue;
                const int64_t i3 = ((int64_t)ix * g.ny + iy) * g.nz + iz;
                const double gM = cot[i3], gx = cot[ncell + i3], gy = cot[2 * ncell + i3], gz = cot[3 * ncell + i3];
                const double gs = gM + pvx * gx + pvy * gy + pvz * gz;
                acc[0] += msum.v * gs;
                acc[1] += msum.d[0] * gs;
                acc[2] += msum.d[1] * gs;
                acc[3] += msum.d[2] * gs;
                acc[4] += msum.d[3] * gs;
                acc[5] += msum.v * gx;
                acc[6] += msum.v * gy;
                acc[7] += msum.v * gz;
            }
        }
#pragma unroll
        for (int k = 0; k < 8; ++k)
            for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
        if (lane == 0) {
            if (G.m) G.m[p] = acc[0];
            if (G.x) G.x[p] = pm * acc[1];
            if (G.y) G.y[p] = pm * acc[2];
            if (G.z) G.z[p] = pm * acc[3];
            if (G.h) G.h[p] = pm * acc[4];
            if (G.vx) G.vx[p] = pm * acc[5];
            if (G.vy) G.vy[p] = pm * acc[6];
            if (G.vz) G.vz[p] = pm * acc[7];
        }
    }
    if (n_eval) atomicAdd(&st->evaluated_pairs, n_eval);
    if (n_neg) atomicAdd(&st->neg_clamped, n_neg);
}

}  // namespace

int cart_adjoint_dev(KiwiCtx* ctx, const DevParticles& P, const CartGeom& g, const KernelChoice& kc,
                     const double* d_cot, const AdjointOutputs& out, KiwiStats* stats) {
    if (!kc.cubic)
        return set_err(ctx, KIWI_ERR_UNSUPPORTED,
                       "the adjoint is available for the cubic spline kernel with support 2h (generic_path unset)");
    DevStats* d_st = nullptr;
    KIWI_TRY(scratch(ctx, S_MISC3, sizeof(DevStats), (void**)&d_st));
    KIWI_CUDA(ctx, cudaMemsetAsync(d_st, 0, sizeof(DevStats), ctx->stream));
    if (P.n > 0) {
        int dev_sms = 148;
        cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, ctx->device);
        const int64_t want = (P.n + kAdjWarps - 1) / kAdjWarps;
        const int64_t cap = (int64_t)dev_sms * 16;
        const int blocks = (int)(want < cap ? want : cap);
        AdjGrads G{out.x, out.y, out.z, out.h, out.m, out.vx, out.vy, out.vz};
        k_cart_adjoint<<<blocks, kAdjThreads, 0, ctx->stream>>>(P, g, d_cot, G, d_st);
        KIWI_LAUNCHED(ctx);
    }
    if (stats) {
        DevStats h;
        KIWI_CUDA(ctx, cudaMemcpyAsync(&h, d_st, sizeof(DevStats), cudaMemcpyDeviceToHost, ctx->stream));
        KIWI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        stats->evaluated_pairs = (int64_t)h.evaluated_pairs;
        stats->neg_clamped = (int64_t)h.neg_clamped;
    }
    return KIWI_OK;
}

}  // namespace kiwi_b200
