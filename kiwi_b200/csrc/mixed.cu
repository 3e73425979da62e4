// FP32-mixed form of the Cartesian cell integrals (cubic spline, support 2h).
//
// The lattice factorisation of the FP64 form (lattice.cuh) with its two expensive phases in FP32: the
// edge tiers (D2, D3) of every (plane, edge line) and the corner values S of every (plane, lattice
// point) are evaluated by mixed_math.cuh with T = float, from plane offsets taken relative to the
// particle in FP64 and then rounded to FP32 (so large domain coordinates cost no precision).  The cell
// assembly -- 24 signed corner values per (particle, cell) -- and the per-cell sums of m K and m K v are
// done in FP64, in the same fixed particle order per cell as the FP64 kernels (no atomics).
//
// Each corner value carries the sum of the magnitudes of the terms it was computed from; the cell's
// rounding-error bound is kBoundScale x sum over particles of m x (the sum of those magnitudes over the
// cell's 24 corner values).  The closed form is a signed sum of pyramid masses that can be many orders of
// magnitude above the cell's mass (the pyramids of a cell's near and far faces nearly cancel), so the
// FP32 result is only as good as that bound says; with the guarantee option, tiles holding a cell whose
// bound exceeds the requested relative tolerance are recomputed by the FP64 lattice kernel.
#include <cuda_runtime.h>

#include "engine.hpp"
#include "lattice.cuh"
#include "mixed_math.cuh"
#include "prims.cuh"

namespace kiwi_b200 {

namespace {

using mixed::MxEdge;
using mixed::MxWall;

constexpr int kMxThreads = 256;
constexpr int kMxCellsPerThread = kTileCells / kMxThreads;
static_assert(kTileCells % kMxThreads == 0, "tile cells must split evenly over the threads");
constexpr int kMxPMax = 32;
constexpr int kMxECap = 1536;  // edge entries per chunk (a full 8^3 particle box needs 486)
constexpr int kMxSCap = 4096;  // corner entries per chunk (a full 8^3 particle box needs 2187)
constexpr size_t kMxDynSmem = sizeof(float) * (4 * kMxECap + 2 * kMxSCap);
// Rounding-error bound per unit of term magnitude: 4 x the FP32 unit roundoff 2^-24 (measured on 11M
// pairs of the lognormal-cube workload: |error| <= 0.5 x 2^-24 x magnitude for 99.9% of the pairs and
// <= 1.96 x 2^-24 x magnitude for all of them).
constexpr double kBoundScale = 4.0 * 5.9604644775390625e-08;
// FP64 islands: planes closer to the particle than this fraction of h are evaluated in FP64 (the wall
// tier's (h/r0)^3 and the edge ratio a = R0/r0 grow without bound as r0 -> 0, beyond FP32's range).
constexpr double kIslandFrac = 1e-3;

__device__ __forceinline__ void add_stat(unsigned long long* dst, unsigned long long v) {
    if (v) atomicAdd(dst, v);
}

__device__ __forceinline__ float fsgn(double v) { return (v > 0.0) ? 1.0f : ((v < 0.0) ? -1.0f : 0.0f); }

__global__ void __launch_bounds__(kMxThreads, 2) k_cart_lattice_f32(CartGeom g, DevParticles P,
                                                                    const uint32_t* __restrict__ list,
                                                                    const int64_t* __restrict__ range,
                                                                    const int32_t* __restrict__ tile_map,
                                                                    CartOutputs out, double* __restrict__ cell_err,
                                                                    double* __restrict__ cell_mass,
                                                                    DevStats* __restrict__ st) {
    __shared__ double s_x[kMxPMax], s_y[kMxPMax], s_z[kMxPMax], s_m[kMxPMax], s_vx[kMxPMax], s_vy[kMxPMax],
        s_vz[kMxPMax];
    __shared__ float s_h[kMxPMax];
    __shared__ double s_hd[kMxPMax];
    __shared__ int s_lo[kMxPMax][3], s_dim[kMxPMax][3], s_eoff[kMxPMax], s_soff[kMxPMax];
    __shared__ int s_np, s_etot, s_stot;
    extern __shared__ float s_dynf[];
    float* s_D2 = s_dynf;
    float* s_D3 = s_dynf + kMxECap;
    float* s_A2 = s_dynf + 2 * kMxECap;
    float* s_A3 = s_dynf + 3 * kMxECap;
    float* s_S = s_dynf + 4 * kMxECap;
    float* s_Sa = s_S + kMxSCap;

    const int64_t t = tile_map ? (int64_t)tile_map[blockIdx.x] : (int64_t)blockIdx.x;
    const int tz = (int)(t % g.ntz), ty = (int)((t / g.ntz) % g.nty), tx = (int)(t / ((int64_t)g.ntz * g.nty));
    const int bx = tx * kTileX, by = ty * kTileY, bz = tz * kTileZ;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    (void)warp;

    double acc[kMxCellsPerThread][5];
#pragma unroll
    for (int c = 0; c < kMxCellsPerThread; ++c)
        acc[c][0] = acc[c][1] = acc[c][2] = acc[c][3] = acc[c][4] = 0.0;
    unsigned long long n_bbox = 0, n_sphere = 0, n_eval = 0, n_neg = 0, n_warn = 0, n_vp = 0;
    unsigned long long n_eo = 0, n_em = 0, n_ei = 0, n_island = 0;
    const int64_t beg = range[2 * t], end = range[2 * t + 1];

    for (int64_t pos = beg; pos < end;) {
        if (threadIdx.x < 32) {
            const int64_t idx = pos + lane;
            int ne = 0, ns = 0, lo0 = 0, lo1 = 0, lo2 = 0, d0 = 0, d1 = 0, d2 = 0;
            double px = 0, py = 0, pz = 0, ph = 0, pm = 0, pvx = 0, pvy = 0, pvz = 0;
            if (idx < end) {
                const uint32_t p = list[idx];
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
            const bool take = (idx < end) && ie <= kMxECap && is <= kMxSCap;
            const int np = __popc(__ballot_sync(0xffffffffu, take));
            if (take) {
                s_x[lane] = px; s_y[lane] = py; s_z[lane] = pz; s_h[lane] = (float)ph; s_hd[lane] = ph;
                s_m[lane] = pm; s_vx[lane] = pvx; s_vy[lane] = pvy; s_vz[lane] = pvz;
                s_lo[lane][0] = lo0; s_lo[lane][1] = lo1; s_lo[lane][2] = lo2;
                s_dim[lane][0] = d0; s_dim[lane][1] = d1; s_dim[lane][2] = d2;
                s_eoff[lane] = ie - ne;
                s_soff[lane] = is - ns;
            }
            if (lane == np - 1) {
                s_np = np;
                s_etot = ie;
                s_stot = is;
            }
        }
        __syncthreads();
        const int np = s_np, etot = s_etot, stot = s_stot;

        // (A) edge tiers in FP32: block (a, b) holds r0 along axis a, R_0 along axis b
        for (int it = threadIdx.x; it < etot; it += kMxThreads) {
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
            const double r0d = fabs(lattice_offset(mn[a], dd[a], s_lo[j][a] + p, pc[a]));
            const float r0 = (float)r0d;
            const float R0 = (float)fabs(lattice_offset(mn[bax], dd[bax], s_lo[j][bax] + q, pc[bax]));
            const float h = s_h[j];
            MxEdge<float> ed;
            ed.D2 = ed.D3 = ed.A2 = ed.A3 = 0.0f;
            // (an island plane's edge tiers are evaluated in FP64 by the corner pass itself; the island
            // test is the corner pass's own, on the FP64 offset)
            if (r0 > 0.0f && R0 > 0.0f && !(r0d < kIslandFrac * s_hd[j])) ed = mixed::mx_edge(mixed::mx_wall(h, r0), R0);
            s_D2[it] = ed.D2;
            s_D3[it] = ed.D3;
            s_A2[it] = ed.A2;
            s_A3[it] = ed.A3;
            const float ld2 = r0 * r0 + R0 * R0;
            if (ld2 > 4.0f * h * h) ++n_eo;
            else if (ld2 > h * h) ++n_em;
            else ++n_ei;
        }
        __syncthreads();

        // (B) corner values in FP32, with their term magnitudes
        for (int it = threadIdx.x; it < stot; it += kMxThreads) {
            const int jp = chunk_search(s_soff, np, it);
            const int s = it - s_soff[jp];
            const int n0 = s_dim[jp][0] + 1, n1 = s_dim[jp][1] + 1, n2 = s_dim[jp][2] + 1;
            const int L = n0 * n1 * n2;
            const int axis = s / L, rem = s % L;
            const int i = rem / (n1 * n2), jj = (rem / n2) % n1, k = rem % n2;
            const double ux = lattice_offset(g.x_min, g.dpx, s_lo[jp][0] + i, s_x[jp]);
            const double uy = lattice_offset(g.y_min, g.dpy, s_lo[jp][1] + jj, s_y[jp]);
            const double uz = lattice_offset(g.z_min, g.dpz, s_lo[jp][2] + k, s_z[jp]);
            const int eb = s_eoff[jp];
            const int nxy = n0 * n1, nxz = n0 * n2, nyz = n1 * n2;
            double r0d, u1d, u2d;
            int e1, e2;
            if (axis == 0) {
                r0d = ux; u1d = uy; u2d = uz;
                e1 = eb + i * n1 + jj;
                e2 = eb + nxy + i * n2 + k;
            } else if (axis == 1) {
                r0d = uy; u1d = ux; u2d = uz;
                e1 = eb + nxy + nxz + jj * n0 + i;
                e2 = eb + 2 * nxy + nxz + jj * n2 + k;
            } else {
                r0d = uz; u1d = ux; u2d = uy;
                e1 = eb + 2 * nxy + nxz + nyz + k * n0 + i;
                e2 = eb + 2 * nxy + 2 * nxz + nyz + k * n1 + jj;
            }
            float f = 0.0f, fa = 0.0f;
            const float sg = fsgn(u1d) * fsgn(u2d);
            const float r0 = (float)fabs(r0d);
            if (sg != 0.0f && r0d != 0.0 && fabs(r0d) < kIslandFrac * s_hd[jp]) {
                // FP64 island: the whole corner (its wall, both edge tiers and both vertex pyramids)
                const double hd = s_hd[jp], a1 = fabs(u1d), a2 = fabs(u2d);
                const MxWall<double> w = mixed::mx_wall(hd, fabs(r0d));
                double ab1, ab2;
                const double fd = mixed::mx_vertex(w, mixed::mx_edge(w, a1), a1, a2, &ab1) +
                                  mixed::mx_vertex(w, mixed::mx_edge(w, a2), a2, a1, &ab2);
                f = (float)fd;
                // rounding scale: the FP32 storage of the value, plus the FP64 terms' own (2^-53, not 2^-24)
                fa = 0.25f * fabsf(f) + (float)((ab1 + ab2) * 1e-9);
                ++n_island;
            } else if (sg != 0.0f && r0 > 0.0f) {
                const float a1 = (float)fabs(u1d), a2 = (float)fabs(u2d);
                const MxWall<float> w = mixed::mx_wall(s_h[jp], r0);
                MxEdge<float> E1, E2;
                E1.D2 = s_D2[e1]; E1.D3 = s_D3[e1]; E1.A2 = s_A2[e1]; E1.A3 = s_A3[e1];
                E2.D2 = s_D2[e2]; E2.D3 = s_D3[e2]; E2.A2 = s_A2[e2]; E2.A3 = s_A3[e2];
                float ab1, ab2;
                f = mixed::mx_vertex(w, E1, a1, a2, &ab1) + mixed::mx_vertex(w, E2, a2, a1, &ab2);
                fa = ab1 + ab2;
                n_vp += 2;
            }
            s_S[it] = sg * f;
            s_Sa[it] = fa;
        }
        __syncthreads();

        // (C) cells in FP64: 6 faces x inclusion-exclusion over 4 corners, in particle order
#pragma unroll
        for (int c = 0; c < kMxCellsPerThread; ++c) {
            const int li = threadIdx.x + c * kMxThreads;
            const int gz = bz + li % kTileZ, gy = by + (li / kTileZ) % kTileY, gx = bx + li / (kTileZ * kTileY);
            for (int j = 0; j < np; ++j) {
                const int i = gx - s_lo[j][0], jj = gy - s_lo[j][1], k = gz - s_lo[j][2];
                if (i < 0 || jj < 0 || k < 0 || i >= s_dim[j][0] || jj >= s_dim[j][1] || k >= s_dim[j][2]) continue;
                ++n_bbox;
                const double x0 = s_x[j], y0 = s_y[j], z0 = s_z[j];
                const double radius = mul_rn(g.support_in_h, s_hd[j]);
                const double ex = fmax(fabs(x0 - cell_centre(g.x_min, gx, g.dpx)) - g.hpx, 0.0);
                const double ey = fmax(fabs(y0 - cell_centre(g.y_min, gy, g.dpy)) - g.hpy, 0.0);
                const double ez = fmax(fabs(z0 - cell_centre(g.z_min, gz, g.dpz)) - g.hpz, 0.0);
                const bool in = ex * ex + ey * ey + ez * ez < radius * radius;
                n_sphere += in;
                if (!in) continue;
                ++n_eval;
                const int n1 = s_dim[j][1] + 1, n2 = s_dim[j][2] + 1;
                const int L = (s_dim[j][0] + 1) * n1 * n2;
                const float* Sx = s_S + s_soff[j];
                const float* Sy = Sx + L;
                const float* Sz = Sy + L;
                const float* Ax = s_Sa + s_soff[j];
                auto at = [&](const float* S, int a, int b, int cc) { return (double)S[(a * n1 + b) * n2 + cc]; };
                const double sx1 = sgn(lattice_offset(g.x_min, g.dpx, gx + 1, x0)), sx0 = sgn(lattice_offset(g.x_min, g.dpx, gx, x0));
                const double sy1 = sgn(lattice_offset(g.y_min, g.dpy, gy + 1, y0)), sy0 = sgn(lattice_offset(g.y_min, g.dpy, gy, y0));
                const double sz1 = sgn(lattice_offset(g.z_min, g.dpz, gz + 1, z0)), sz0 = sgn(lattice_offset(g.z_min, g.dpz, gz, z0));
                double msum = 0.0;
                msum += sx1 * (at(Sx, i + 1, jj + 1, k + 1) - at(Sx, i + 1, jj, k + 1) - at(Sx, i + 1, jj + 1, k) + at(Sx, i + 1, jj, k));
                msum -= sx0 * (at(Sx, i, jj + 1, k + 1) - at(Sx, i, jj, k + 1) - at(Sx, i, jj + 1, k) + at(Sx, i, jj, k));
                msum += sy1 * (at(Sy, i + 1, jj + 1, k + 1) - at(Sy, i, jj + 1, k + 1) - at(Sy, i + 1, jj + 1, k) + at(Sy, i, jj + 1, k));
                msum -= sy0 * (at(Sy, i + 1, jj, k + 1) - at(Sy, i, jj, k + 1) - at(Sy, i + 1, jj, k) + at(Sy, i, jj, k));
                msum += sz1 * (at(Sz, i + 1, jj + 1, k + 1) - at(Sz, i, jj + 1, k + 1) - at(Sz, i + 1, jj, k + 1) + at(Sz, i, jj, k + 1));
                msum -= sz0 * (at(Sz, i + 1, jj + 1, k) - at(Sz, i, jj + 1, k) - at(Sz, i + 1, jj, k) + at(Sz, i, jj, k));
                // the magnitudes of the 24 corner values' terms (the x-, y- and z-plane tables of one
                // lattice point are L entries apart)
                float mag = 0.0f;
#pragma unroll
                for (int ax = 0; ax < 3; ++ax) {
                    const float* A = Ax + ax * L;
                    const int di = ax == 0 ? 1 : 0, dj = ax == 1 ? 1 : 0, dk = ax == 2 ? 1 : 0;
                    // the two faces normal to this axis: planes at lower index and lower index + 1
#pragma unroll
                    for (int f = 0; f < 2; ++f) {
                        const int pi = i + f * di, pj = jj + f * dj, pk = k + f * dk;
                        const int qi = ax == 0 ? 0 : 1, qj = ax == 1 ? 0 : 1, qk = ax == 2 ? 0 : 1;
                        // the face's four corners: the two in-plane axes take offsets 0/1
                        if (ax == 0) {
                            mag += A[(pi * n1 + jj) * n2 + k] + A[(pi * n1 + jj + qj) * n2 + k] +
                                   A[(pi * n1 + jj) * n2 + k + qk] + A[(pi * n1 + jj + qj) * n2 + k + qk];
                        } else if (ax == 1) {
                            mag += A[(i * n1 + pj) * n2 + k] + A[((i + qi) * n1 + pj) * n2 + k] +
                                   A[(i * n1 + pj) * n2 + k + qk] + A[((i + qi) * n1 + pj) * n2 + k + qk];
                        } else {
                            mag += A[(i * n1 + jj) * n2 + pk] + A[((i + qi) * n1 + jj) * n2 + pk] +
                                   A[(i * n1 + jj + qj) * n2 + pk] + A[((i + qi) * n1 + jj + qj) * n2 + pk];
                        }
                    }
                }
                if (msum < 0.0) {
                    ++n_neg;
                    if (msum <= -0.01) ++n_warn;
                    msum = 0.0;
                }
                const double pm = s_m[j];
                acc[c][4] += pm * (double)mag;
                if (msum == 0.0) continue;
                const double mm = msum * pm;
                acc[c][0] += mm;
                acc[c][1] += mm * s_vx[j];
                acc[c][2] += mm * s_vy[j];
                acc[c][3] += mm * s_vz[j];
            }
        }
        __syncthreads();
        pos += np;
    }

    const double mvx = out.meanv[0], mvy = out.meanv[1], mvz = out.meanv[2];
    const int64_t ncell = (int64_t)g.nx * g.ny * g.nz;
    unsigned long long n_flag = 0;
#pragma unroll
    for (int c = 0; c < kMxCellsPerThread; ++c) {
        const int li = threadIdx.x + c * kMxThreads;
        const int ix = bx + li / (kTileZ * kTileY), iy = by + (li / kTileZ) % kTileY, iz = bz + li % kTileZ;
        if (ix >= g.nx || iy >= g.ny || iz >= g.nz) continue;
        const int64_t i3 = ((int64_t)ix * g.ny + iy) * g.nz + iz;
        const double M = acc[c][0];
        const double E = kBoundScale * acc[c][4];
        if (cell_err) cell_err[i3] = E;
        if (cell_mass) cell_mass[i3] = M;
        n_flag += (M > 0.0 && E > 1e-6 * M);
        if (out.density) out.density[i3] = M / g.cell_volume;
        const bool has = M > 0.0;
        if (out.vx) out.vx[i3] = has ? acc[c][1] / M : mvx;
        if (out.vy) out.vy[i3] = has ? acc[c][2] / M : mvy;
        if (out.vz) out.vz[i3] = has ? acc[c][3] / M : mvz;
        if (out.raw4) {
            out.raw4[i3] = M;
            out.raw4[ncell + i3] = acc[c][1];
            out.raw4[2 * ncell + i3] = acc[c][2];
            out.raw4[3 * ncell + i3] = acc[c][3];
        }
    }
    add_stat(&st->bbox_pairs, n_bbox);
    add_stat(&st->sphere_pairs, n_sphere);
    add_stat(&st->evaluated_pairs, n_eval);
    add_stat(&st->neg_clamped, n_neg);
    add_stat(&st->neg_warned, n_warn);
    add_stat(&st->edge_outer, n_eo);
    add_stat(&st->edge_middle, n_em);
    add_stat(&st->edge_inner, n_ei);
    add_stat(&st->vertex_pyramids, n_vp);
    add_stat(&st->fp64_fallback, n_flag);
}

// Peak cell mass (max over cells; max is order-independent, so deterministic).
__global__ void k_max_mass(const double* __restrict__ M, int64_t n, unsigned long long* __restrict__ peak_bits) {
    double v = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        v = fmax(v, M[i]);
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    // non-negative doubles order like their bit patterns
    if ((threadIdx.x & 31) == 0) atomicMax(peak_bits, (unsigned long long)__double_as_longlong(v));
}

// One thread per tile: 1 if a cell of the tile that may lie above floor_frac x peak has bound > rel_tol x mass.
__global__ void k_flag_tiles(CartGeom g, const double* __restrict__ E, const double* __restrict__ M,
                             const unsigned long long* __restrict__ peak_bits, double rel_tol, double floor_frac,
                             uint32_t* __restrict__ flags) {
    const int64_t ntiles = (int64_t)g.ntx * g.nty * g.ntz;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntiles) return;
    const double floor_m = floor_frac * __longlong_as_double((long long)*peak_bits);
    const int tz = (int)(t % g.ntz), ty = (int)((t / g.ntz) % g.nty), tx = (int)(t / ((int64_t)g.ntz * g.nty));
    uint32_t f = 0;
    for (int lx = 0; lx < kTileX && !f; ++lx)
        for (int ly = 0; ly < kTileY && !f; ++ly)
            for (int lz = 0; lz < kTileZ; ++lz) {
                const int ix = tx * kTileX + lx, iy = ty * kTileY + ly, iz = tz * kTileZ + lz;
                if (ix >= g.nx || iy >= g.ny || iz >= g.nz) continue;
                const int64_t i3 = ((int64_t)ix * g.ny + iy) * g.nz + iz;
                // a cell counts if its mass can be at the floor or above (its FP32 mass plus the error
                // bound), and fails if the bound exceeds rel_tol of its mass
                const double m = M[i3], e = E[i3];
                if (m + e >= floor_m && m + e > 0.0 && e > rel_tol * m) {
                    f = 1;
                    break;
                }
            }
    flags[t] = f;
}

__global__ void k_compact_tiles(const uint32_t* __restrict__ flags, const int64_t* __restrict__ offs, int64_t n,
                                int32_t* __restrict__ map) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n && flags[t]) map[offs[t]] = (int32_t)t;
}

// FP32 FMA throughput probe: 8 independent fma chains per thread.
__global__ void __launch_bounds__(256) k_ffma_peak(int iters, float seed, float* __restrict__ sink) {
    float a0 = seed + threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6,
          a7 = a0 + 7;
    const float m = 0.999999f, c = 1e-7f;
    for (int i = 0; i < iters; ++i) {
        a0 = fmaf(a0, m, c); a1 = fmaf(a1, m, c); a2 = fmaf(a2, m, c); a3 = fmaf(a3, m, c);
        a4 = fmaf(a4, m, c); a5 = fmaf(a5, m, c); a6 = fmaf(a6, m, c); a7 = fmaf(a7, m, c);
    }
    const float s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (s == 12345.678f) sink[threadIdx.x] = s;  // keeps the chains live
}

}  // namespace

int fp32_measure_peak(KiwiCtx* ctx, double* tflops) {
    int sms = 0;
    KIWI_CUDA(ctx, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    float* sink = nullptr;
    KIWI_TRY(scratch_t(ctx, S_MISC0, 256, &sink));
    const int blocks = sms * 8, iters = 1 << 15;
    k_ffma_peak<<<blocks, 256, 0, ctx->stream>>>(256, 1.0f, sink);  // warm-up
    KIWI_LAUNCHED(ctx);
    KIWI_CUDA(ctx, cudaEventRecord(ctx->ev[0], ctx->stream));
    k_ffma_peak<<<blocks, 256, 0, ctx->stream>>>(iters, 1.0f, sink);
    KIWI_LAUNCHED(ctx);
    KIWI_CUDA(ctx, cudaEventRecord(ctx->ev[1], ctx->stream));
    KIWI_CUDA(ctx, cudaEventSynchronize(ctx->ev[1]));
    float ms = 0.f;
    KIWI_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]));
    *tflops = 2.0 * 8.0 * iters * (double)blocks * 256.0 / (ms * 1e-3) / 1e12;
    return KIWI_OK;
}

int mixed_cart_gather(KiwiCtx* ctx, const CartGeom& g, const DevParticles& P, const TileLists& tl,
                      const CartOutputs& out, double* cell_err, double* cell_mass, DevStats* d_stats) {
    if (tl.ntiles <= 0) return KIWI_OK;
    if (tl.ntiles > 0x7fffffffLL) return set_err(ctx, KIWI_ERR_ARG, "too many cell tiles (%lld)", (long long)tl.ntiles);
    KIWI_CUDA(ctx, cudaFuncSetAttribute(k_cart_lattice_f32, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)kMxDynSmem));
    if (tl.map && tl.nmap <= 0) return KIWI_OK;
    const unsigned grid = (unsigned)(tl.map ? tl.nmap : tl.ntiles);
    k_cart_lattice_f32<<<grid, kMxThreads, kMxDynSmem, ctx->stream>>>(g, P, tl.list, tl.range, tl.map, out, cell_err,
                                                                      cell_mass, d_stats);
    KIWI_LAUNCHED(ctx);
    return KIWI_OK;
}

int mixed_flag_tiles(KiwiCtx* ctx, const CartGeom& g, const double* cell_err, const double* cell_mass,
                     double rel_tol, double floor_frac, int32_t* map, int64_t* d_nmap) {
    const int64_t ncell = (int64_t)g.nx * g.ny * g.nz;
    const int64_t ntiles = (int64_t)g.ntx * g.nty * g.ntz;
    unsigned long long* peak = nullptr;
    uint32_t* flags = nullptr;
    int64_t* offs = nullptr;
    KIWI_TRY(scratch_t(ctx, S_FLAG_PEAK, 1, &peak));
    KIWI_TRY(scratch_t(ctx, S_FLAG_FLAGS, (size_t)ntiles, &flags));
    KIWI_TRY(scratch_t(ctx, S_FLAG_OFFS, (size_t)ntiles + 1, &offs));
    KIWI_CUDA(ctx, cudaMemsetAsync(peak, 0, sizeof(unsigned long long), ctx->stream));
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    const int64_t want = (ncell + 255) / 256;
    const int blocks = (int)(want < (int64_t)sms * 8 ? want : (int64_t)sms * 8);
    k_max_mass<<<blocks > 0 ? blocks : 1, 256, 0, ctx->stream>>>(cell_mass, ncell, peak);
    KIWI_LAUNCHED(ctx);
    k_flag_tiles<<<(unsigned)((ntiles + 127) / 128), 128, 0, ctx->stream>>>(g, cell_err, cell_mass, peak, rel_tol,
                                                                             floor_frac, flags);
    KIWI_LAUNCHED(ctx);
    KIWI_TRY(exclusive_scan<uint32_t>(ctx, flags, ntiles, offs, d_nmap));
    k_compact_tiles<<<(unsigned)((ntiles + 255) / 256), 256, 0, ctx->stream>>>(flags, offs, ntiles, map);
    KIWI_LAUNCHED(ctx);
    return KIWI_OK;
}

}  // namespace kiwi_b200
