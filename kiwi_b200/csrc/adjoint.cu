// Adjoint of the Cartesian sph-to-grid stage (no counterpart in the reference, which has no gradients).
//
// The forward pass produces, per cell c, the raw sums M_c = sum_p m_p K_pc and P_c = sum_p m_p K_pc v_p,
// where K_pc = max(Msum_pc, 0) is the particle's kernel mass inside the cell (src/cartesian_grid.cpp:
// 256-277).  Given the cotangents gM_c = dL/dM_c and gP_c = dL/dP_c, the adjoint returns per particle
//   dL/dm_p     = sum_c K_pc (gM_c + v_p . gP_c)
//   dL/dv_p     = m_p sum_c K_pc gP_c
//   dL/dtheta_p = m_p sum_c dK_pc/dtheta (gM_c + v_p . gP_c),   theta = x, y, z, h.
// The per-pair cell integrals are recomputed, not stored: the forward kernel's lattice tiers (lattice_edge,
// lattice_corner) are instantiated with the Dual4 type, which carries d/dx, d/dy, d/dz, d/dh of every
// intermediate through the same operations, so the
// value part equals the forward's Msum bit for bit and the derivative part is the exact derivative of the
// evaluated formula (branch choices are taken on values).  A clamped pair (Msum < 0) has K = 0 and no
// gradient.  The pairs are those of the forward's default evaluation: the cells of the particle's
// support bounding box whose closest point lies within the support radius.
//
// The evaluation is the lattice form of the forward pass (lattice.cuh) in Dual4: one CTA per 8^3-cell
// tile walks the tile's particles in chunks; (A) the edge tiers of every (plane, edge line) and (B) the
// corner values of every (plane, lattice point) are computed once per particle with their derivatives;
// (C) for each particle, each thread assembles the cells it owns from the 24 corner values (value and
// derivatives alike), weighs them with the cells' cotangents, and a fixed-order block reduction writes the
// particle's partial gradient for this tile to its (tile, particle) entry.  (D) Each particle's entries
// are then added in tile order.  Deterministic, no atomics on the gradients.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>

#include "binning.cuh"
#include "cart_common.cuh"
#include "ctx.hpp"
#include "dual.cuh"
#include "engine.hpp"
#include "kiwi_math.cuh"
#include "lattice.cuh"
#include "prims.cuh"

namespace kiwi_b200 {

namespace {

constexpr int kAdjLatThreads = 256;
constexpr int kAdjCellsPerThread = kTileCells / kAdjLatThreads;
constexpr int kAdjPMax = 32;
constexpr int kAdjECap = 512;   // edge entries per chunk (a full 8^3 particle box needs 486)
constexpr int kAdjSCap = 2304;  // corner entries per chunk (a full 8^3 particle box needs 2187)
constexpr int kAdjERec = 10;    // D2, D3 as Dual4
constexpr int kAdjSRec = 5;     // S as Dual4
constexpr size_t kAdjDynSmem = sizeof(double) * (kAdjERec * kAdjECap + kAdjSRec * kAdjSCap);
constexpr int kAdjPtCap = kAdjSCap / 3;  // lattice points per chunk (three corner items each)

struct AdjGrads {
    double *x, *y, *z, *h, *m, *vx, *vy, *vz;
};

__device__ __forceinline__ Dual4 dual_abs_offset(double off, int axis) {
    // |plane - x_axis| and its derivative with respect to the particle's coordinate on that axis
    Dual4 r(fabs(off));
    r.d[axis] = off > 0.0 ? -1.0 : (off < 0.0 ? 1.0 : 0.0);
    return r;
}

__device__ __forceinline__ Dual4 load_dual(const double* p) {
    Dual4 r(p[0]);
    r.d[0] = p[1];
    r.d[1] = p[2];
    r.d[2] = p[3];
    r.d[3] = p[4];
    return r;
}

__device__ __forceinline__ void store_dual(double* p, const Dual4& v) {
    p[0] = v.v;
    p[1] = v.d[0];
    p[2] = v.d[1];
    p[3] = v.d[2];
    p[4] = v.d[3];
}

__device__ __forceinline__ unsigned long long block_count(unsigned long long v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// (A)-(C) for one tile: list holds (tile, particle) entry indices (the entries of particle p are
// offs[p] .. offs[p+1]-1); part receives 8 doubles per entry: dL/dm, dL/d(x, y, z, h), dL/d(vx, vy, vz)
// over this tile's cells.
__global__ void __launch_bounds__(kAdjLatThreads, 1) k_cart_adjoint_lattice(CartGeom g, DevParticles P,
                                                                          const uint32_t* __restrict__ list,
                                                                          const int64_t* __restrict__ range,
                                                                          const int64_t* __restrict__ offs,
                                                                          const double* __restrict__ cot,
                                                                          double* __restrict__ part,
                                                                          DevStats* __restrict__ st) {
    __shared__ double s_x[kAdjPMax], s_y[kAdjPMax], s_z[kAdjPMax], s_h[kAdjPMax], s_m[kAdjPMax], s_vx[kAdjPMax],
        s_vy[kAdjPMax], s_vz[kAdjPMax];
    __shared__ int s_lo[kAdjPMax][3], s_dim[kAdjPMax][3], s_eoff[kAdjPMax], s_soff[kAdjPMax];
    __shared__ uint32_t s_entry[kAdjPMax];
    __shared__ uint32_t s_mag[kAdjPMax][4];  // div_magic of n0, n1, n2 and n1 n2
    __shared__ uint32_t s_blist[kAdjPtCap];
    __shared__ int s_np, s_etot, s_stot, s_nexp, s_ncheap;
    __shared__ double s_red[kAdjLatThreads / 32][8];
    extern __shared__ double s_adj[];
    double* s_E = s_adj;
    double* s_S = s_adj + kAdjERec * kAdjECap;

    const int64_t t = blockIdx.x;
    const int tz = (int)(t % g.ntz), ty = (int)((t / g.ntz) % g.nty), tx = (int)(t / ((int64_t)g.ntz * g.nty));
    const int bx = tx * kTileX, by = ty * kTileY, bz = tz * kTileZ;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t ncell = (int64_t)g.nx * g.ny * g.nz;
    unsigned long long n_eval = 0, n_neg = 0;
    const int64_t beg = range[2 * t], end = range[2 * t + 1];

    for (int64_t pos = beg; pos < end;) {
        if (warp == 0) {
            const int64_t idx = pos + lane;
            int ne = 0, ns = 0, lo0 = 0, lo1 = 0, lo2 = 0, d0 = 0, d1 = 0, d2 = 0;
            double px = 0, py = 0, pz = 0, ph = 0, pm = 0, pvx = 0, pvy = 0, pvz = 0;
            uint32_t e = 0;
            if (idx < end) {
                e = list[idx];
                int64_t lo = 0, hi = P.n - 1;  // the entry's particle: the last p with offs[p] <= e
                while (lo < hi) {
                    const int64_t mid = (lo + hi + 1) >> 1;
                    if (offs[mid] <= (int64_t)e) lo = mid; else hi = mid - 1;
                }
                const int64_t p = lo;
                px = P.x[p]; py = P.y[p]; pz = P.z[p]; ph = P.h[p];
                pm = P.m[p]; pvx = P.vx[p]; pvy = P.vy[p]; pvz = P.vz[p];
                CellBox b;
                bool outside;
                particle_cell_box(g, px, py, pz, ph, b, &outside);
                lo0 = max(b.x0, bx); lo1 = max(b.y0, by); lo2 = max(b.z0, bz);
                d0 = min(b.x1, bx + kTileX - 1) - lo0 + 1;
                d1 = min(b.y1, by + kTileY - 1) - lo1 + 1;
                d2 = min(b.z1, bz + kTileZ - 1) - lo2 + 1;
                const int n0 = d0 + 1, n1 = d1 + 1, n2 = d2 + 1;
                ne = 2 * (n0 * n1 + n0 * n2 + n1 * n2);
                ns = 3 * n0 * n1 * n2;
            }
            int ie = ne, is = ns;
            for (int o = 1; o < 32; o <<= 1) {
                const int ve = __shfl_up_sync(0xffffffffu, ie, o), vs = __shfl_up_sync(0xffffffffu, is, o);
                if (lane >= o) {
                    ie += ve;
                    is += vs;
                }
            }
            const bool take = (idx < end) && ie <= kAdjECap && is <= kAdjSCap;
            const int np = __popc(__ballot_sync(0xffffffffu, take));
            if (take) {
                s_x[lane] = px; s_y[lane] = py; s_z[lane] = pz; s_h[lane] = ph;
                s_m[lane] = pm; s_vx[lane] = pvx; s_vy[lane] = pvy; s_vz[lane] = pvz;
                s_lo[lane][0] = lo0; s_lo[lane][1] = lo1; s_lo[lane][2] = lo2;
                s_dim[lane][0] = d0; s_dim[lane][1] = d1; s_dim[lane][2] = d2;
                s_eoff[lane] = ie - ne;
                s_soff[lane] = is - ns;
                s_entry[lane] = e;
                s_mag[lane][0] = div_magic(d0 + 1);
                s_mag[lane][1] = div_magic(d1 + 1);
                s_mag[lane][2] = div_magic(d2 + 1);
                s_mag[lane][3] = div_magic((d1 + 1) * (d2 + 1));
            }
            if (lane == np - 1) {
                s_np = np;
                s_etot = ie;
                s_stot = is;
                s_nexp = s_ncheap = 0;
            }
        }
        __syncthreads();
        const int np = s_np, etot = s_etot, stot = s_stot;

        // (A) edge tiers with derivatives
        for (int it = threadIdx.x; it < etot; it += kAdjLatThreads) {
            const int j = chunk_search(s_eoff, np, it);
            int e = it - s_eoff[j];
            const int n[3] = {s_dim[j][0] + 1, s_dim[j][1] + 1, s_dim[j][2] + 1};
            int a = 0, bax = 1;
            {
                const int sz[6] = {n[0] * n[1], n[0] * n[2], n[1] * n[0], n[1] * n[2], n[2] * n[0], n[2] * n[1]};
                const int aa[6] = {0, 0, 1, 1, 2, 2}, bb[6] = {1, 2, 0, 2, 0, 1};
                int blk = 0;
                while (e >= sz[blk]) {
                    e -= sz[blk];
                    ++blk;
                }
                a = aa[blk];
                bax = bb[blk];
            }
            const int p = e / n[bax], q = e % n[bax];
            const double mn[3] = {g.x_min, g.y_min, g.z_min}, dd[3] = {g.dpx, g.dpy, g.dpz};
            const double pc[3] = {s_x[j], s_y[j], s_z[j]};
            const Dual4 r0 = dual_abs_offset(lattice_offset(mn[a], dd[a], s_lo[j][a] + p, pc[a]), a);
            const Dual4 R0 = dual_abs_offset(lattice_offset(mn[bax], dd[bax], s_lo[j][bax] + q, pc[bax]), bax);
            const Dual4 hD = Dual4::seed(s_h[j], 3);
            // the forward kernel's edge tier (lattice_edge) in Dual4; zero beyond 2h and for zero offsets
            Dual4 D2(0.0), D3(0.0);
            if (r0 != 0.0 && R0 != 0.0 && r0.v * r0.v + R0.v * R0.v <= 4.0 * (s_h[j] * s_h[j])) {
                const LatticeEdgeT<Dual4> ed = lattice_edge(hD, 1.0 / hD, r0, R0);
                D2 = ed.D2;
                D3 = ed.D3;
            }
            store_dual(s_E + kAdjERec * it, D2);
            store_dual(s_E + kAdjERec * it + 5, D3);
        }

        // (B0) the corner items, listed lattice point by lattice point as in the forward kernel: corners
        // that no evaluated cell reads left out (the same padded test), corners beyond 2h (or zero) from
        // the end of s_blist so that they run in warps of their own; a list entry packs (particle, i, j, k).
        {
            const int ptot = stot / 3;
            const int poff_l = lane < np ? s_soff[lane] / 3 : INT_MAX;
            for (int base = warp * 32; base < ptot; base += kAdjLatThreads) {
                const int pt = base + lane;
                int cls = -1;  // -1 none, 0 general, 1 cheap
                uint32_t rec = 0;
                const int jp = warp_owner(base, poff_l, lane);
                const int poff = __shfl_sync(0xffffffffu, poff_l, jp & 31);
                if (pt < ptot) {
                    const int lp = pt - poff;
                    const int n2 = s_dim[jp][2] + 1, n12 = (s_dim[jp][1] + 1) * n2;
                    const int i = div_by(lp, s_mag[jp][3]), rem = lp - i * n12;
                    const int jj = div_by(rem, s_mag[jp][2]), k = rem - jj * n2;
                    const double ux = lattice_offset(g.x_min, g.dpx, s_lo[jp][0] + i, s_x[jp]);
                    const double uy = lattice_offset(g.y_min, g.dpy, s_lo[jp][1] + jj, s_y[jp]);
                    const double uz = lattice_offset(g.z_min, g.dpz, s_lo[jp][2] + k, s_z[jp]);
                    const double h = s_h[jp], radius = mul_rn(g.support_in_h, h);
                    const double ex = fmax(fabs(ux) - kNeedPad * g.dpx, 0.0);
                    const double ey = fmax(fabs(uy) - kNeedPad * g.dpy, 0.0);
                    const double ez = fmax(fabs(uz) - kNeedPad * g.dpz, 0.0);
                    if (ex * ex + ey * ey + ez * ez < radius * radius) {
                        const bool zero = ux == 0.0 || uy == 0.0 || uz == 0.0;
                        cls = (zero || !(ux * ux + uy * uy + uz * uz < 4.0 * (h * h))) ? 1 : 0;
                        rec = (uint32_t)jp | (uint32_t)i << 5 | (uint32_t)jj << 9 | (uint32_t)k << 13;
                    }
                }
                const unsigned me = __ballot_sync(0xffffffffu, cls == 0), mc = __ballot_sync(0xffffffffu, cls == 1);
                int pe = 0, pcb = 0;
                if (lane == 0) {
                    if (me) pe = atomicAdd(&s_nexp, __popc(me));
                    if (mc) pcb = atomicAdd(&s_ncheap, __popc(mc));
                }
                pe = __shfl_sync(0xffffffffu, pe, 0);
                pcb = __shfl_sync(0xffffffffu, pcb, 0);
                const unsigned below = (1u << lane) - 1;
                if (cls >= 0) s_blist[cls == 0 ? pe + __popc(me & below) : kAdjPtCap - 1 - pcb - __popc(mc & below)] = rec;
            }
        }
        __syncthreads();

        // (B) corner values with derivatives
        const int nexp = s_nexp, ncheap = s_ncheap;
        for (int li = threadIdx.x; li < 3 * (nexp + ncheap); li += kAdjLatThreads) {
            const int pli = li / 3, axis = li - 3 * pli;
            const uint32_t rec = s_blist[pli < nexp ? pli : kAdjPtCap - ncheap + (pli - nexp)];
            const int jp = (int)(rec & 31u), i = (int)((rec >> 5) & 15u), jj = (int)((rec >> 9) & 15u),
                      k = (int)((rec >> 13) & 15u);
            const int n0 = s_dim[jp][0] + 1, n1 = s_dim[jp][1] + 1, n2 = s_dim[jp][2] + 1;
            const int it = s_soff[jp] + axis * (n0 * n1 * n2) + (i * n1 + jj) * n2 + k;
            const double ux = lattice_offset(g.x_min, g.dpx, s_lo[jp][0] + i, s_x[jp]);
            const double uy = lattice_offset(g.y_min, g.dpy, s_lo[jp][1] + jj, s_y[jp]);
            const double uz = lattice_offset(g.z_min, g.dpz, s_lo[jp][2] + k, s_z[jp]);
            const int eb = s_eoff[jp];
            const int nxy = n0 * n1, nxz = n0 * n2, nyz = n1 * n2;
            double ua, u1, u2;
            int ax1, ax2, e1, e2;
            if (axis == 0) {
                ua = ux; u1 = uy; u2 = uz; ax1 = 1; ax2 = 2;
                e1 = eb + i * n1 + jj;
                e2 = eb + nxy + i * n2 + k;
            } else if (axis == 1) {
                ua = uy; u1 = ux; u2 = uz; ax1 = 0; ax2 = 2;
                e1 = eb + nxy + nxz + jj * n0 + i;
                e2 = eb + 2 * nxy + nxz + jj * n2 + k;
            } else {
                ua = uz; u1 = ux; u2 = uy; ax1 = 0; ax2 = 1;
                e1 = eb + 2 * nxy + nxz + nyz + k * n0 + i;
                e2 = eb + 2 * nxy + 2 * nxz + nyz + k * n1 + jj;
            }
            Dual4 f(0.0);
            const double sg = sgn(u1) * sgn(u2);
            if (sg != 0.0 && ua != 0.0) {
                const Dual4 r0 = dual_abs_offset(ua, axis);
                const Dual4 a1 = dual_abs_offset(u1, ax1), a2 = dual_abs_offset(u2, ax2);
                const Dual4 hD = Dual4::seed(s_h[jp], 3);
                // the forward kernel's corner pair (lattice_corner) in Dual4
                f = lattice_corner(hD, 1.0 / hD, r0, a1, a2, load_dual(s_E + kAdjERec * e1), load_dual(s_E + kAdjERec * e1 + 5),
                                   load_dual(s_E + kAdjERec * e2), load_dual(s_E + kAdjERec * e2 + 5));
            }
            store_dual(s_S + kAdjSRec * it, sg * f);
        }
        __syncthreads();

        // (C) per particle: the cells' values and derivatives from the corners, weighed by the cotangents
        for (int j = 0; j < np; ++j) {
            double acc[8];
#pragma unroll
            for (int c = 0; c < 8; ++c) acc[c] = 0.0;
            const double x0 = s_x[j], y0 = s_y[j], z0 = s_z[j];
            const double radius = mul_rn(g.support_in_h, s_h[j]);
            const int n1 = s_dim[j][1] + 1, n2 = s_dim[j][2] + 1;
            const int L = (s_dim[j][0] + 1) * n1 * n2;
            const double* Sx = s_S + kAdjSRec * s_soff[j];
            const double* Sy = Sx + kAdjSRec * L;
            const double* Sz = Sy + kAdjSRec * L;
#pragma unroll
            for (int c = 0; c < kAdjCellsPerThread; ++c) {
                const int li = threadIdx.x + c * kAdjLatThreads;
                const int gz = bz + li % kTileZ, gy = by + (li / kTileZ) % kTileY, gx = bx + li / (kTileZ * kTileY);
                const int i = gx - s_lo[j][0], jj = gy - s_lo[j][1], k = gz - s_lo[j][2];
                if (i < 0 || jj < 0 || k < 0 || i >= s_dim[j][0] || jj >= s_dim[j][1] || k >= s_dim[j][2]) continue;
                const double ex = fmax(fabs(x0 - cell_centre(g.x_min, gx, g.dpx)) - g.hpx, 0.0);
                const double ey = fmax(fabs(y0 - cell_centre(g.y_min, gy, g.dpy)) - g.hpy, 0.0);
                const double ez = fmax(fabs(z0 - cell_centre(g.z_min, gz, g.dpz)) - g.hpz, 0.0);
                if (!(ex * ex + ey * ey + ez * ez < radius * radius)) continue;
                ++n_eval;
                const double sx1 = sgn(lattice_offset(g.x_min, g.dpx, gx + 1, x0)), sx0 = sgn(lattice_offset(g.x_min, g.dpx, gx, x0));
                const double sy1 = sgn(lattice_offset(g.y_min, g.dpy, gy + 1, y0)), sy0 = sgn(lattice_offset(g.y_min, g.dpy, gy, y0));
                const double sz1 = sgn(lattice_offset(g.z_min, g.dpz, gz + 1, z0)), sz0 = sgn(lattice_offset(g.z_min, g.dpz, gz, z0));
                // component comp of the cell's Msum: 0 the value (the forward's sum, same order), 1..4 d/d(x, y, z, h)
                auto cell_sum = [&](int comp) {
                    auto at = [&](const double* S, int a, int b, int cc) { return S[kAdjSRec * ((a * n1 + b) * n2 + cc) + comp]; };
                    double m = 0.0;
                    m += sx1 * (at(Sx, i + 1, jj + 1, k + 1) - at(Sx, i + 1, jj, k + 1) - at(Sx, i + 1, jj + 1, k) + at(Sx, i + 1, jj, k));
                    m -= sx0 * (at(Sx, i, jj + 1, k + 1) - at(Sx, i, jj, k + 1) - at(Sx, i, jj + 1, k) + at(Sx, i, jj, k));
                    m += sy1 * (at(Sy, i + 1, jj + 1, k + 1) - at(Sy, i, jj + 1, k + 1) - at(Sy, i + 1, jj + 1, k) + at(Sy, i, jj + 1, k));
                    m -= sy0 * (at(Sy, i + 1, jj, k + 1) - at(Sy, i, jj, k + 1) - at(Sy, i + 1, jj, k) + at(Sy, i, jj, k));
                    m += sz1 * (at(Sz, i + 1, jj + 1, k + 1) - at(Sz, i, jj + 1, k + 1) - at(Sz, i + 1, jj, k + 1) + at(Sz, i, jj, k + 1));
                    m -= sz0 * (at(Sz, i + 1, jj + 1, k) - at(Sz, i, jj + 1, k) - at(Sz, i + 1, jj, k) + at(Sz, i, jj, k));
                    return m;
                };
                const double msum = cell_sum(0);
                if (msum < 0.0) {
                    ++n_neg;
                    continue;
                }
                if (msum == 0.0) continue;
                const int64_t i3 = ((int64_t)gx * g.ny + gy) * g.nz + gz;
                const double gM = cot[i3], gx_ = cot[ncell + i3], gy_ = cot[2 * ncell + i3], gz_ = cot[3 * ncell + i3];
                const double gs = gM + s_vx[j] * gx_ + s_vy[j] * gy_ + s_vz[j] * gz_;
                acc[0] += msum * gs;
#pragma unroll 1
                for (int comp = 1; comp <= 4; ++comp) acc[comp] += cell_sum(comp) * gs;
                acc[5] += msum * gx_;
                acc[6] += msum * gy_;
                acc[7] += msum * gz_;
            }
            // fixed-order block reduction: xor tree within each warp, then the warps in order
#pragma unroll
            for (int c = 0; c < 8; ++c)
                for (int o = 16; o > 0; o >>= 1) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o);
            if (lane == 0)
#pragma unroll
                for (int c = 0; c < 8; ++c) s_red[warp][c] = acc[c];
            __syncthreads();
            if (threadIdx.x < 8) {
                double v = 0.0;
                for (int w = 0; w < kAdjLatThreads / 32; ++w) v += s_red[w][threadIdx.x];
                const double pm = s_m[j];
                part[8 * (int64_t)s_entry[j] + threadIdx.x] = (threadIdx.x == 0) ? v : pm * v;
            }
            __syncthreads();
        }
        pos += np;
    }
    n_eval = block_count(n_eval);
    n_neg = block_count(n_neg);
    if (lane == 0) {
        if (n_eval) atomicAdd(&st->evaluated_pairs, n_eval);
        if (n_neg) atomicAdd(&st->neg_clamped, n_neg);
    }
}

// (D) each particle's gradient: its entries' partial sums in tile order.
__global__ void k_adjoint_reduce(int64_t n, const int64_t* __restrict__ offs, const double* __restrict__ part,
                                 AdjGrads G) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    double acc[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) acc[c] = 0.0;
    for (int64_t e = offs[p]; e < offs[p + 1]; ++e)
#pragma unroll
        for (int c = 0; c < 8; ++c) acc[c] += part[8 * e + c];
    if (G.m) G.m[p] = acc[0];
    if (G.x) G.x[p] = acc[1];
    if (G.y) G.y[p] = acc[2];
    if (G.z) G.z[p] = acc[3];
    if (G.h) G.h[p] = acc[4];
    if (G.vx) G.vx[p] = acc[5];
    if (G.vy) G.vy[p] = acc[6];
    if (G.vz) G.vz[p] = acc[7];
}

}  // namespace

int cart_adjoint_dev(KiwiCtx* ctx, const DevParticles& P, const CartGeom& g, const KernelChoice& kc,
                     const double* d_cot, const AdjointOutputs& out, KiwiStats* stats) {
    if (!kc.cubic || kc.tabulated)
        return set_err(ctx, KIWI_ERR_UNSUPPORTED,
                       "the adjoint is available for the analytic cubic spline integral with support 2h (generic_path "
                       "and tabulated unset)");
    DevStats* d_st = nullptr;
    KIWI_TRY(scratch_t(ctx, S_STATS, 1, &d_st));
    KIWI_CUDA(ctx, cudaMemsetAsync(d_st, 0, sizeof(DevStats), ctx->stream));
    const int64_t n = P.n;
    const int64_t ntiles = (int64_t)g.ntx * g.nty * g.ntz;
    // binning as the forward pass, with the sort carrying each (tile, particle) entry's index
    uint32_t* counts = nullptr;
    TileBox* boxes = nullptr;
    int64_t *offs = nullptr, *range = nullptr;
    KIWI_TRY(scratch_t(ctx, S_COUNT, (size_t)std::max<int64_t>(n, 1), &counts));
    KIWI_TRY(scratch_t(ctx, S_BOX, (size_t)std::max<int64_t>(n, 1), &boxes));
    KIWI_TRY(scratch_t(ctx, S_OFFS, (size_t)std::max<int64_t>(n, 1) + 1, &offs));
    KIWI_TRY(scratch_t(ctx, S_TILE_RANGE, (size_t)(2 * ntiles), &range));
    int64_t* d_total = offs + std::max<int64_t>(n, 1);
    KIWI_CUDA(ctx, cudaMemsetAsync(range, 0, sizeof(int64_t) * 2 * ntiles, ctx->stream));
    if (n > 0) {
        k_tile_counts<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(g, P, counts, boxes, d_st);
        KIWI_LAUNCHED(ctx);
    }
    KIWI_TRY(exclusive_scan<uint32_t>(ctx, counts, n, offs, d_total));
    int64_t total = 0;
    KIWI_CUDA(ctx, cudaMemcpyAsync(&total, d_total, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
    KIWI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (total >= (1LL << 32)) return set_err(ctx, KIWI_ERR_LIMIT, "too many (tile, particle) entries: %lld", (long long)total);
    uint32_t *k0, *v0, *k1, *v1;
    double* part = nullptr;
    KIWI_TRY(scratch_t(ctx, S_KEYS0, (size_t)std::max<int64_t>(total, 1), &k0));
    KIWI_TRY(scratch_t(ctx, S_VALS0, (size_t)std::max<int64_t>(total, 1), &v0));
    KIWI_TRY(scratch_t(ctx, S_KEYS1, (size_t)std::max<int64_t>(total, 1), &k1));
    KIWI_TRY(scratch_t(ctx, S_VALS1, (size_t)std::max<int64_t>(total, 1), &v1));
    KIWI_TRY(scratch_t(ctx, S_ADJ_PART, (size_t)8 * std::max<int64_t>(total, 1), &part));
    if (total > 0) {
        k_tile_emit<<<(unsigned)((total + 255) / 256), 256, 0, ctx->stream>>>(g, n, offs, boxes, 0, total, 0u, k0, v0,
                                                                              true);
        KIWI_LAUNCHED(ctx);
        int key_bits = 1;
        while ((1LL << key_bits) < ntiles) ++key_bits;
        bool second = false;
        KIWI_TRY(radix_sort_pairs(ctx, k0, v0, k1, v1, total, key_bits, &second));
        k_tile_ranges<<<(unsigned)((total + 255) / 256), 256, 0, ctx->stream>>>(second ? k1 : k0, total, range);
        KIWI_LAUNCHED(ctx);
        KIWI_CUDA(ctx, cudaFuncSetAttribute(k_cart_adjoint_lattice, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)kAdjDynSmem));
        k_cart_adjoint_lattice<<<(unsigned)ntiles, kAdjLatThreads, kAdjDynSmem, ctx->stream>>>(
            g, P, second ? v1 : v0, range, offs, d_cot, part, d_st);
        KIWI_LAUNCHED(ctx);
    }
    if (n > 0) {
        AdjGrads G{out.x, out.y, out.z, out.h, out.m, out.vx, out.vy, out.vz};
        k_adjoint_reduce<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(n, offs, part, G);
        KIWI_LAUNCHED(ctx);
    }
    if (stats) {
        DevStats h;
        KIWI_CUDA(ctx, cudaMemcpyAsync(&h, d_st, sizeof(DevStats), cudaMemcpyDeviceToHost, ctx->stream));
        KIWI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        stats->evaluated_pairs = (int64_t)h.evaluated_pairs;
        stats->neg_clamped = (int64_t)h.neg_clamped;
        stats->skipped_outside = (int64_t)h.skipped_outside;
        stats->tile_pairs = total;
    }
    return KIWI_OK;
}

}  // namespace kiwi_b200
