// The tile body of the lattice-factorised gather (one CTA = one 8 x 8 x 8 cell tile), shared by the
// single-grid kernels and the batch's persistent kernel.  A translation unit that includes this defines
// `c_tables` (its __constant__ copy of the kernel tables) first.
//
// Per particle of the tile's list, the box of its support clipped to the tile (n0 x n1 x n2 cells) has
// (n0 + 1)(n1 + 1)(n2 + 1) lattice points and 2 (n0' n1' + n0' n2' + n1' n2') edge lines (n' = n + 1):
// every edge line of a plane, in the six orientation blocks xy, xz, yx, yz, zx, zy (block "ab": the wall
// at distance |u_a| along axis a, the line at in-plane distance |u_b| along axis b).  The two edges of a
// block pair (xy[i][j] and yx[j][i], ...) are the two orientations of one (|u_a|, |u_b|) pair and are
// evaluated together (lattice_edge_pair).  A lattice point's octant value (the kernel mass of the box
// spanned by the particle and the point, lattice_point) is sgn(ux) sgn(uy) sgn(uz) times the sum of its
// three corner values; a cell's mass is the alternating sum of its eight corners' octant values, which is
// the reference's sum over the cell's 6 faces x 4 edges x 2 vertex pyramids regrouped by corner
// (src/cartesian_grid.cpp:246-259, src/kernel_integral.cpp:471-647).
#pragma once

#include <climits>

#include "engine.hpp"
#include "f32.cuh"
#include "lattice.cuh"
#include "tabulated.cuh"

namespace kiwi_b200 {

#ifndef KIWI_LAT_THREADS
#define KIWI_LAT_THREADS 256
#endif
constexpr int kLatThreads = KIWI_LAT_THREADS;
constexpr int kLatCellsPerThread = kTileCells / kLatThreads;
static_assert(kTileCells % kLatThreads == 0, "tile cells must split evenly over the threads");
// Chunk capacities (defaults sized for two CTAs per SM; a full 8^3 particle box has 729 lattice points and
// 486 edge lines).
#ifndef KIWI_LAT_PT_CAP
#define KIWI_LAT_PT_CAP 2304
#endif
#ifndef KIWI_LAT_E_CAP
#define KIWI_LAT_E_CAP 2048
#endif
constexpr int kLatPtCap = KIWI_LAT_PT_CAP;  // lattice points per chunk
constexpr int kLatECap2 = KIWI_LAT_E_CAP;   // cubic edge tiers per chunk
static_assert(kTileX <= 15 && kTileY <= 15 && kTileZ <= 15 && kLatPMax <= 32, "packed point-list entries");
static_assert(kLatECap2 <= 2048 && kLatGenECap <= 2048, "packed edge-pair entries (11-bit slots)");
// (C1) keeps a chunk's (particle, cell) pair values in its edge-tier buffer: a box has fewer cells than
// lattice points, so ctot < ptot <= kLatPtCap
static_assert(2 * kLatECap2 >= kLatPtCap && kLatGenERec * kLatGenECap >= kLatPtCap, "pair values fit the edge buffer");
// Each edge pair's in-plane angle formed once (1) or every point's walls forming theirs (0).
#ifndef KIWI_LAT_ANGLES
#define KIWI_LAT_ANGLES 1
#endif
constexpr bool kLatAngles = KIWI_LAT_ANGLES != 0;
// Shared-memory carveout preference of the lattice kernels, percent of the SM's maximum (what is not
// carved out is L1, which holds the tiers' register spills).
#ifndef KIWI_LAT_CARVEOUT
#define KIWI_LAT_CARVEOUT 100
#endif
constexpr int kLatCarveout = KIWI_LAT_CARVEOUT;
// dynamic shared memory: the owned cells' sums (4 per cell), then the chunk's edge tiers and octant values
constexpr size_t kLatAccSmem = sizeof(double) * 4 * kTileCells;
constexpr size_t kLatDynSmem = kLatAccSmem + sizeof(double) * ((kLatAngles ? 3 : 2) * kLatECap2 + kLatPtCap);
constexpr size_t kLatGenDynSmem = kLatAccSmem + sizeof(double) * (kLatGenERec * kLatGenECap + kLatPtCap);
constexpr size_t kLatTabDynSmem = kLatAccSmem + sizeof(double) * kLatPtCap;

// The six edge tiers of a lattice point (slots of the chunk's D2 / D3 tables in PointEdge order), read where
// lattice_point uses them, as the real type T it is evaluated in.
template <class T>
struct SmemPointEdges {
    const double* d2;
    const double* d3;
    const double* ang;  // per edge pair (at its ab slot): the smaller in-plane angle, or < 0 if not formed
    int slot[6];
    __device__ __forceinline__ T D2(int e) const { return T(d2[slot[e]]); }
    __device__ __forceinline__ T D3(int e) const { return T(d3[slot[e]]); }
    // leg_angles from the pair's stored angle atan(min(a1, a2) / max(a1, a2)); a pair that (A2) did not
    // evaluate (its legs' rounded square sum beyond 2h while the point's is within) forms it here
    __device__ __forceinline__ void leg_angles(int e, T a1, T ia1, T a2, T ia2, T& pa, T& pb) const {
        const double t = ang ? ang[slot[e]] : -1.0;
        if (t < 0.0) {
            kiwi_b200::leg_angles(a1, ia1, a2, ia2, pa, pb);
            return;
        }
        const bool lo = a2 <= a1;
        const T tq = T(t), tc = 0.5 * kPi - tq;
        pa = lo ? tq : tc;
        pb = lo ? tc : tq;
    }
};

// FP32-mixed form: planes closer to the particle than this fraction of h are evaluated in FP64 (the wall
// tier's (h/r0)^3 and the edge ratio R_0/r0 grow without bound as r0 -> 0).
constexpr double kMixedIslandFrac = 1e-3;

__device__ __forceinline__ void lat_add_stat(unsigned long long* dst, unsigned long long v) {
    // warp-aggregate, then one atomic per warp
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(dst, v);
}

// One chunk of a tile's particle list as the lattice tile holds it in shared memory: the particles' data,
// their cell boxes clipped to the tile (lo, dim), their edge-slot and point offsets, the magic divisors of
// their lattice dimensions, and the chunk's counts.
struct LatChunk {
    double x[kLatPMax], y[kLatPMax], z[kLatPMax], h[kLatPMax], m[kLatPMax], vx[kLatPMax], vy[kLatPMax], vz[kLatPMax],
        ih[kLatPMax];
    int lo[kLatPMax][3], dim[kLatPMax][3], eoff[kLatPMax], poff[kLatPMax], coff[kLatPMax];
    uint32_t mag[kLatPMax][4];   // div_magic of n0', n1', n2' and n1' n2'
    uint32_t cmag[kLatPMax][2];  // div_magic of n2 and n1 n2 (the box's cells)
    int np, etot, ptot, ctot;
};

// The chunk of a tile's particle list (ascending particle index) is walked in four phases separated by
// barriers: (A) classify every edge pair, listing those within the support; (B0) list the lattice points
// that some evaluated cell reads (the cheap ones -- beyond the support -- from the end of the list) and set
// the octant value of the points on a particle plane to 0; (A2) the listed edge pairs; (B) the listed
// points' octant values; (C) each thread adds, for the cells it owns, the chunk's particles in list order
// -- every cell's sum runs over its particles in ascending index order with no atomics.  The chunks are
// double-buffered: while warps 1-7 classify the current chunk's edge pairs and points, warp 0 loads the next
// chunk (the particles' data, boxes and offsets) into the other buffer.
// GENERIC: the table-driven tiers of kernel K (support radius support_in_h x h) instead of the cubic closed
// form; edge tiers are lattice_generic_edge records.  TAB: the tabulated cubic integral (lookups in `tab`):
// no edge tiers, and the points run in their natural order.  List order never affects the results.
template <bool CULL, bool GENERIC = false, bool TAB = false, bool MIXED = false>
__device__ __forceinline__ void lattice_tile(const CartGeom& g, const DevParticles& P,
                                             const uint32_t* __restrict__ list, const int64_t* __restrict__ range,
                                             int64_t t_range, int64_t t, const CartOutputs& out,
                                             DevStats* __restrict__ st, const KiwiKernelTable* K = nullptr,
                                             const TabDev tab = TabDev{}) {
    __shared__ LatChunk s_cp[2];
    __shared__ TabWidths s_tw;               // TAB: the table's bin widths and their reciprocals
    if (TAB && threadIdx.x == 0) s_tw = tab_widths(tab);  // read after the chunk load's barrier
    __shared__ int s_nexp, s_ncheap, s_nheavy, s_ninner;
    __shared__ uint32_t s_plist[TAB ? 1 : kLatPtCap];
    __shared__ uint32_t s_hlist[TAB ? 1 : kLatECap2 / 2];
    static_assert(kLatGenECap / 2 <= kLatECap2 / 2, "generic edge pairs fit the pair list");
    extern __shared__ double s_dyn[];
    constexpr int kECap = GENERIC ? kLatGenECap : (TAB ? 0 : kLatECap2);
    // the owned cells' sums M, Px, Py, Pz: each thread's own entries (no sharing, no barrier), held in
    // registers only while (C) adds a chunk -- the point phase needs the registers
    double* s_acc = s_dyn;
    double* s_chunk = s_dyn + 4 * kTileCells;
    double* s_D2 = s_chunk;
    double* s_D3 = s_chunk + kLatECap2;
    double* s_E = s_chunk;  // generic edge records
    double* s_T = s_chunk + (GENERIC ? kLatGenERec * kLatGenECap : (TAB ? 0 : 2 * kLatECap2));
    // cubic: each edge pair's smaller in-plane angle (at its ab slot), or none
    double* s_A = kLatAngles ? s_T + kLatPtCap : nullptr;

    const int tz = (int)(t % g.ntz), ty = (int)((t / g.ntz) % g.nty), tx = (int)(t / ((int64_t)g.ntz * g.nty));
    const int bx = tx * kTileX, by = ty * kTileY, bz = tz * kTileZ;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // the tile's lattice planes (every particle box is clipped to the tile, so its planes are these) and
    // cell centres, formed as the reference forms them; read after the first barrier
    __shared__ double s_pl[3][kTileX + 1], s_cc[3][kTileX];
    static_assert(kTileX == kTileY && kTileX == kTileZ, "cubic tiles");
    if (threadIdx.x < 3 * (kTileX + 1)) {
        const int a = threadIdx.x / (kTileX + 1), l = threadIdx.x % (kTileX + 1);
        const double mn = a == 0 ? g.x_min : (a == 1 ? g.y_min : g.z_min), d = a == 0 ? g.dpx : (a == 1 ? g.dpy : g.dpz);
        const int b0 = a == 0 ? bx : (a == 1 ? by : bz);
        s_pl[a][l] = add_rn(mn, mul_rn((double)(b0 + l), d));
        if (l < kTileX) s_cc[a][l] = cell_centre(mn, b0 + l, d);
    }

#pragma unroll
    for (int c = 0; c < kLatCellsPerThread; ++c) {
        const int li = threadIdx.x + c * kLatThreads;
        s_acc[li] = s_acc[kTileCells + li] = s_acc[2 * kTileCells + li] = s_acc[3 * kTileCells + li] = 0.0;
    }
    // work counters: 32-bit per thread (a chunk adds at most a few hundred to any of them), flushed to the
    // 64-bit totals every 2^16 chunks and at the end
    unsigned n_bbox = 0, n_sphere = 0, n_eval = 0, n_neg = 0, n_warn = 0;
    unsigned n_eo = 0, n_em = 0, n_ei = 0, n_vp = 0, n_clamp = 0, n_chunks = 0, n_island = 0;
    auto flush = [&]() {
        lat_add_stat(&st->bbox_pairs, n_bbox);
        lat_add_stat(&st->sphere_pairs, n_sphere);
        lat_add_stat(&st->evaluated_pairs, n_eval);
        lat_add_stat(&st->neg_clamped, n_neg);
        lat_add_stat(&st->neg_warned, n_warn);
        lat_add_stat(&st->edge_outer, n_eo);
        lat_add_stat(&st->edge_middle, n_em);
        lat_add_stat(&st->edge_inner, n_ei);
        lat_add_stat(&st->vertex_pyramids, n_vp);
        if (TAB) lat_add_stat(&st->table_clamps, n_clamp);
        if (MIXED) lat_add_stat(&st->fp64_fallback, n_island);
        n_bbox = n_sphere = n_eval = n_neg = n_warn = n_eo = n_em = n_ei = n_vp = n_clamp = n_island = 0;
    };
    const int64_t beg = range[2 * t_range], end = range[2 * t_range + 1];
    const double sup_in_h = g.support_in_h;

    // warp 0: the chunk of the particle list starting at `at` into *dst (as many particles as the edge and
    // point capacities take, at most 32)
    auto load_chunk = [&](LatChunk* dst, int64_t at) {
        const int64_t idx = at + lane;
        int ne = 0, npt = 0, ncl = 0, lo0 = 0, lo1 = 0, lo2 = 0, d0 = 0, d1 = 0, d2 = 0;
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
            ne = TAB ? 0 : 2 * (n0 * n1 + n0 * n2 + n1 * n2);
            npt = n0 * n1 * n2;
            ncl = d0 * d1 * d2;
        }
        int ie = ne, ip = npt, ic = ncl;
        for (int o = 1; o < 32; o <<= 1) {
            const int ve = __shfl_up_sync(0xffffffffu, ie, o), vp = __shfl_up_sync(0xffffffffu, ip, o);
            const int vc = __shfl_up_sync(0xffffffffu, ic, o);
            if (lane >= o) {
                ie += ve;
                ip += vp;
                ic += vc;
            }
        }
        const bool take = (idx < end) && ie <= kECap && ip <= kLatPtCap;
        const int np = __popc(__ballot_sync(0xffffffffu, take));
        if (take) {
            dst->x[lane] = px; dst->y[lane] = py; dst->z[lane] = pz; dst->h[lane] = ph; dst->ih[lane] = 1.0 / ph;
            dst->m[lane] = pm; dst->vx[lane] = pvx; dst->vy[lane] = pvy; dst->vz[lane] = pvz;
            dst->lo[lane][0] = lo0; dst->lo[lane][1] = lo1; dst->lo[lane][2] = lo2;
            dst->dim[lane][0] = d0; dst->dim[lane][1] = d1; dst->dim[lane][2] = d2;
            dst->eoff[lane] = ie - ne;
            dst->poff[lane] = ip - npt;
            dst->mag[lane][0] = div_magic(d0 + 1);
            dst->mag[lane][1] = div_magic(d1 + 1);
            dst->mag[lane][2] = div_magic(d2 + 1);
            dst->mag[lane][3] = div_magic((d1 + 1) * (d2 + 1));
            dst->coff[lane] = ic - ncl;
            dst->cmag[lane][0] = div_magic(d2);
            dst->cmag[lane][1] = div_magic(d1 * d2);
        }
        if (lane == np - 1) {
            dst->np = np;
            dst->etot = ie;
            dst->ptot = ip;
            dst->ctot = ic;
        }
    };
    LatChunk* cp = &s_cp[0];
    if (warp == 0 && beg < end) load_chunk(cp, beg);
    if (threadIdx.x == 0) s_nexp = s_ncheap = s_nheavy = s_ninner = 0;
    __syncthreads();

    for (int64_t pos = beg; pos < end;) {
        LatChunk* const nx = cp == &s_cp[0] ? &s_cp[1] : &s_cp[0];
        const int np = cp->np, etot = cp->etot, ptot = cp->ptot;

        if (warp == 0) {
            // the next chunk, into the other buffer (read after the barrier that ends the current chunk)
            if (pos + np < end) load_chunk(nx, pos + np);
        } else {
            // (A) edge pairs: pair block 0 = (x, y) over n0' x n1', 1 = (x, z) over n0' x n2', 2 = (y, z) over
            // n1' x n2'; pair (p, q) of block (a, b) is edge ab[p][q] and edge ba[q][p].  Cubic: pairs beyond 2h
            // (and zero ones) get D2 = D3 = 0 here; the others are listed (slot ab | slot ba << 11 | particle <<
            // 22) with |u_a|, |u_b| parked in slot ab, and evaluated in (A2).  Generic: both records here.
            if (!TAB) {
                const int qtot = etot >> 1;
                const int qoff_l = lane < np ? (cp->eoff[lane] >> 1) : INT_MAX;
                for (int base = (warp - 1) * 32; base < qtot; base += kLatThreads - 32) {
                    const int it = base + lane;
                    bool heavy = false, inner = false;
                    uint32_t hrec = 0;
                    const int j = warp_owner(base, qoff_l, lane);
                    const int qoff = __shfl_sync(0xffffffffu, qoff_l, j & 31);
                    if (it < qtot) {
                        int e = it - qoff;
                        const int n0 = cp->dim[j][0] + 1, n1 = cp->dim[j][1] + 1, n2 = cp->dim[j][2] + 1;
                        const int nxy = n0 * n1, nxz = n0 * n2, nyz = n1 * n2;
                        const int blk = (e >= nxy) + (e >= nxy + nxz);
                        e -= blk == 0 ? 0 : (blk == 1 ? nxy : nxy + nxz);
                        const int a = blk == 2 ? 1 : 0, b = blk == 0 ? 1 : 2;
                        const int nb = b == 1 ? n1 : n2, na = a == 0 ? n0 : n1;
                        const int pi = div_by(e, cp->mag[j][b]), qi = e - pi * nb;
                        const int eb = cp->eoff[j];
                        const int sab = eb + (blk == 0 ? 0 : (blk == 1 ? nxy : 2 * nxy + nxz)) + pi * nb + qi;
                        const int sba = eb + (blk == 0 ? nxy + nxz : (blk == 1 ? 2 * nxy + nxz + nyz : 2 * nxy + 2 * nxz + nyz)) +
                                        qi * na + pi;
                        const int la = cp->lo[j][a] - (a == 0 ? bx : by), lb = cp->lo[j][b] - (b == 1 ? by : bz);
                        const double pa = a == 0 ? cp->x[j] : cp->y[j], pb = b == 1 ? cp->y[j] : cp->z[j];
                        const double vp = fabs(s_pl[a][la + pi] - pa), vq = fabs(s_pl[b][lb + qi] - pb);
                        if (GENERIC) {
                            // the records of a pair whose edge line crosses a region boundary (the expensive
                            // ones: per boundary an arccosine, a sine and cosine and two series) are listed
                            // and evaluated in (A2) by all warps, those crossing two or more from the end of
                            // the list; the others (zero, or one region) here
                            const double H = mul_rn(sup_in_h, cp->h[j]);
                            int nseg = 0;
                            if (vp != 0.0 && vq != 0.0) {
                                const double q0 = vp / H, qR = vq / H;
                                nseg = K->nreg - generic_region(K, sqrt(q0 * q0 + qR * qR)) + 1;
                            }
                            if (nseg <= 1) {
                                lattice_generic_edge(K, H, vp, vq, s_E + kLatGenERec * sab);
                                lattice_generic_edge(K, H, vq, vp, s_E + kLatGenERec * sba);
                            } else {
                                heavy = true;
                                inner = nseg >= 3;
                                s_E[kLatGenERec * sab] = vp;
                                s_E[kLatGenERec * sab + 1] = vq;
                                hrec = (uint32_t)sab | (uint32_t)sba << 11 | (uint32_t)j << 22;
                            }
                            n_ei += 2;
                        } else {
                            const double h2 = cp->h[j] * cp->h[j];
                            const double ld2 = add_rn(mul_rn(vp, vp), mul_rn(vq, vq));
                            heavy = vp != 0.0 && vq != 0.0 && ld2 <= 4.0 * h2;
                            inner = heavy && !(ld2 > h2);
                            if (heavy) {
                                if (ld2 > h2) n_em += 2;
                                else n_ei += 2;
                                s_D2[sab] = vp;
                                s_D3[sab] = vq;
                                hrec = (uint32_t)sab | (uint32_t)sba << 11 | (uint32_t)j << 22;
                            } else {
                                n_eo += 2;
                                s_D2[sab] = s_D3[sab] = 0.0;
                                s_D2[sba] = s_D3[sba] = 0.0;
                                if (kLatAngles) s_A[sab] = -1.0;
                            }
                        }
                    }
                    {
                        // pairs within h (two passes of the edge tiers; generic: two or more region
                        // boundaries) from the end of the list, the others from the front, so that each kind
                        // runs in warps of its own
                        const unsigned mm = __ballot_sync(0xffffffffu, heavy && !inner);
                        const unsigned mi = __ballot_sync(0xffffffffu, inner);
                        int hp = 0, hi = 0;
                        if (lane == 0) {
                            if (mm) hp = atomicAdd(&s_nheavy, __popc(mm));
                            if (mi) hi = atomicAdd(&s_ninner, __popc(mi));
                        }
                        hp = __shfl_sync(0xffffffffu, hp, 0);
                        hi = __shfl_sync(0xffffffffu, hi, 0);
                        const unsigned below = (1u << lane) - 1;
                        if (heavy)
                            s_hlist[inner ? kLatECap2 / 2 - 1 - hi - __popc(mi & below) : hp + __popc(mm & below)] = hrec;
                    }
                }
            }

            // (B0) the lattice points some evaluated cell reads: with CULL, a point none of whose eight cells
            // meets the support sphere is left out (the test bounds the distance to the 2 x 2 x 2 cells around
            // the point, their half-widths padded by 1e-6 of a cell so that rounding never drops a point an
            // evaluated cell reads).  A point on a particle plane (an offset of 0) has octant value 0, written
            // here; the others are listed, those within the support from the front of s_plist, those beyond it
            // from the end, so that each kind runs in warps of its own.  An entry packs (particle, i, j, k):
            // 5 + 3 x 4 bits.
            if (!TAB) {
                const int poff_l = lane < np ? cp->poff[lane] : INT_MAX;
                for (int base = (warp - 1) * 32; base < ptot; base += kLatThreads - 32) {
                    const int pt = base + lane;
                    int cls = -1;  // -1 none, 0 within the support, 1 beyond
                    uint32_t rec = 0;
                    const int jp = warp_owner(base, poff_l, lane);
                    const int poff = __shfl_sync(0xffffffffu, poff_l, jp & 31);
                    if (pt < ptot) {
                        const int lp = pt - poff;
                        const int n2 = cp->dim[jp][2] + 1, n12 = (cp->dim[jp][1] + 1) * n2;
                        const int i = div_by(lp, cp->mag[jp][3]), rem = lp - i * n12;
                        const int jj = div_by(rem, cp->mag[jp][2]), k = rem - jj * n2;
                        const double ux = s_pl[0][cp->lo[jp][0] - bx + i] - cp->x[jp];
                        const double uy = s_pl[1][cp->lo[jp][1] - by + jj] - cp->y[jp];
                        const double uz = s_pl[2][cp->lo[jp][2] - bz + k] - cp->z[jp];
                        const double h = cp->h[jp];
                        bool keep = true;
                        if (CULL) {
                            const double radius = mul_rn(sup_in_h, h);
                            const double ex = fmax(fabs(ux) - kNeedPad * g.dpx, 0.0);
                            const double ey = fmax(fabs(uy) - kNeedPad * g.dpy, 0.0);
                            const double ez = fmax(fabs(uz) - kNeedPad * g.dpz, 0.0);
                            keep = ex * ex + ey * ey + ez * ez < radius * radius;
                        }
                        if (keep) {
                            if (ux == 0.0 || uy == 0.0 || uz == 0.0) {
                                s_T[pt] = 0.0;
                            } else {
                                const double H = GENERIC ? mul_rn(sup_in_h, h) : 2.0 * h;
                                cls = (ux * ux + uy * uy + uz * uz < H * H) ? 0 : 1;
                                rec = (uint32_t)jp | (uint32_t)i << 5 | (uint32_t)jj << 9 | (uint32_t)k << 13;
                            }
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
                    if (cls >= 0) s_plist[cls == 0 ? pe + __popc(me & below) : kLatPtCap - 1 - pcb - __popc(mc & below)] = rec;
                }
            }
        }
        __syncthreads();

        // (A2) the listed edge pairs
        if (GENERIC) {
            const int nmid = s_nheavy, ninner = s_ninner;
            for (int li = threadIdx.x; li < nmid + ninner; li += kLatThreads) {
                const uint32_t rec = s_hlist[li < nmid ? li : kLatECap2 / 2 - ninner + (li - nmid)];
                const int sab = (int)(rec & 2047u), sba = (int)((rec >> 11) & 2047u), j = (int)(rec >> 22);
                const double vp = s_E[kLatGenERec * sab], vq = s_E[kLatGenERec * sab + 1];
                const double H = mul_rn(sup_in_h, cp->h[j]);
                if (MIXED && fmin(vp, vq) >= kMixedIslandFrac * cp->h[j]) {
                    lattice_generic_edge(K, H, F32(vp), F32(vq), s_E + kLatGenERec * sab);
                    lattice_generic_edge(K, H, F32(vq), F32(vp), s_E + kLatGenERec * sba);
                } else {
                    lattice_generic_edge(K, H, vp, vq, s_E + kLatGenERec * sab);
                    lattice_generic_edge(K, H, vq, vp, s_E + kLatGenERec * sba);
                }
            }
            __syncthreads();
        }
        if (!GENERIC && !TAB) {
            const int nmid = s_nheavy, ninner = s_ninner;
            for (int li = threadIdx.x; li < nmid + ninner; li += kLatThreads) {
                const uint32_t rec = s_hlist[li < nmid ? li : kLatECap2 / 2 - ninner + (li - nmid)];
                const int sab = (int)(rec & 2047u), sba = (int)((rec >> 11) & 2047u), j = (int)(rec >> 22);
                LatticeEdge e_pq, e_qp;
                const double vp = s_D2[sab], vq = s_D3[sab];
                // the pair's smaller in-plane angle (FP64 in every form: FP64 island points read it too),
                // which the walls with legs along a and b read
                const double vmin = fmin(vp, vq), vmax = fmax(vp, vq);
                if (kLatAngles) s_A[sab] = atan(vmin / vmax);
                if (MIXED && vmin >= kMixedIslandFrac * cp->h[j]) {
                    LatticeEdgeT<F32> f_pq, f_qp;
                    lattice_edge_pair(F32(cp->h[j]), F32(cp->ih[j]), F32(vp), F32(vq), f_pq, f_qp);
                    e_pq = {(double)f_pq.D2.v, (double)f_pq.D3.v};
                    e_qp = {(double)f_qp.D2.v, (double)f_qp.D3.v};
                } else {
                    lattice_edge_pair(cp->h[j], cp->ih[j], vp, vq, e_pq, e_qp);
                }
                s_D2[sab] = e_pq.D2;
                s_D3[sab] = e_pq.D3;
                s_D2[sba] = e_qp.D2;
                s_D3[sba] = e_qp.D3;
            }
            __syncthreads();
        }
        const int nexp = s_nexp, ncheap = s_ncheap;
        const int nplist = TAB ? ptot : nexp + ncheap;

        // (B) octant values of the listed points
        for (int li = threadIdx.x; li < nplist; li += kLatThreads) {
            int jp, i, jj, k, it;
            if (TAB) {
                it = li;
                jp = chunk_search(cp->poff, np, it);
                const int lp = it - cp->poff[jp];
                const int n2 = cp->dim[jp][2] + 1, n12 = (cp->dim[jp][1] + 1) * n2;
                i = div_by(lp, cp->mag[jp][3]);
                const int rem = lp - i * n12;
                jj = div_by(rem, cp->mag[jp][2]);
                k = rem - jj * n2;
            } else {
                const uint32_t rec = s_plist[li < nexp ? li : kLatPtCap - ncheap + (li - nexp)];
                jp = (int)(rec & 31u);
                i = (int)((rec >> 5) & 15u);
                jj = (int)((rec >> 9) & 15u);
                k = (int)((rec >> 13) & 15u);
                it = cp->poff[jp] + (i * (cp->dim[jp][1] + 1) + jj) * (cp->dim[jp][2] + 1) + k;
            }
            const double ux = s_pl[0][cp->lo[jp][0] - bx + i] - cp->x[jp];
            const double uy = s_pl[1][cp->lo[jp][1] - by + jj] - cp->y[jp];
            const double uz = s_pl[2][cp->lo[jp][2] - bz + k] - cp->z[jp];
            const double sg = sgn(ux) * sgn(uy) * sgn(uz);
            double f = 0.0;
            if (sg != 0.0) {
                const double ax = fabs(ux), ay = fabs(uy), az = fabs(uz);
                if (TAB) {
                    // two right-triangle vertex pyramids per wall; cos(phi) from the legs
                    const double ih = cp->ih[jp];
                    f = tab_pair(tab, s_tw, ih, ax, ay, az, n_clamp) + tab_pair(tab, s_tw, ih, ay, ax, az, n_clamp) +
                        tab_pair(tab, s_tw, ih, az, ax, ay, n_clamp);
                } else {
                    const int n0 = cp->dim[jp][0] + 1, n1 = cp->dim[jp][1] + 1, n2 = cp->dim[jp][2] + 1;
                    const int nxy = n0 * n1, nxz = n0 * n2, nyz = n1 * n2;
                    const int eb = cp->eoff[jp];
                    const int exy = eb + i * n1 + jj, exz = eb + nxy + i * n2 + k;
                    const int eyx = eb + nxy + nxz + jj * n0 + i, eyz = eb + 2 * nxy + nxz + jj * n2 + k;
                    const int ezx = eb + 2 * nxy + nxz + nyz + k * n0 + i, ezy = eb + 2 * nxy + 2 * nxz + nyz + k * n1 + jj;
                    if (GENERIC) {
                        const double H = mul_rn(sup_in_h, cp->h[jp]);
                        const double *rxy = s_E + kLatGenERec * exy, *rxz = s_E + kLatGenERec * exz;
                        const double *ryx = s_E + kLatGenERec * eyx, *ryz = s_E + kLatGenERec * eyz;
                        const double *rzx = s_E + kLatGenERec * ezx, *rzy = s_E + kLatGenERec * ezy;
                        if (MIXED && fmin(ax, fmin(ay, az)) >= kMixedIslandFrac * cp->h[jp]) {
                            const F32 fx(ax), fy(ay), fz(az);
                            f = (double)(lattice_generic_corner(K, H, fx, fy, fz, rxy, rxz) +
                                         lattice_generic_corner(K, H, fy, fx, fz, ryx, ryz) +
                                         lattice_generic_corner(K, H, fz, fx, fy, rzx, rzy)).v;
                        } else {
                            f = lattice_generic_corner(K, H, ax, ay, az, rxy, rxz) +
                                lattice_generic_corner(K, H, ay, ax, az, ryx, ryz) +
                                lattice_generic_corner(K, H, az, ax, ay, rzx, rzy);
                            if (MIXED) ++n_island;
                        }
                    } else {
                        if (MIXED && fmin(ax, fmin(ay, az)) >= kMixedIslandFrac * cp->h[jp]) {
                            const SmemPointEdges<F32> E{s_D2, s_D3, s_A, {exy, exz, eyx, eyz, ezx, ezy}};
                            f = (double)lattice_point(F32(cp->h[jp]), F32(cp->ih[jp]), F32(ax), F32(ay), F32(az), E).v;
                        } else {
                            const SmemPointEdges<double> E{s_D2, s_D3, s_A, {exy, exz, eyx, eyz, ezx, ezy}};
                            f = lattice_point(cp->h[jp], cp->ih[jp], ax, ay, az, E);
                            if (MIXED) ++n_island;
                        }
                    }
                }
                n_vp += 6;
            }
            s_T[it] = sg * f;
        }
        __syncthreads();

        // the next chunk's list counters (the lists of this one are read)
        if (threadIdx.x == 0) s_nexp = s_ncheap = s_nheavy = s_ninner = 0;

        // (C) cells: the alternating sum of the 8 corners' octant values, added in particle order.  (C1) every
        // (particle, cell of its box) pair of the chunk, as one flat list over all threads: the support test,
        // the counters and the clamped alternating sum, into the chunk's edge-tier buffer (dead after (B));
        // (C2) each thread adds, for the cells it owns, the chunk's pairs in particle order.  The tabulated
        // body (no edge buffer) does both in the owners' loop.
        if (TAB) {
#pragma unroll
    #pragma unroll
            for (int c = 0; c < kLatCellsPerThread; ++c) {
                const int li = threadIdx.x + c * kLatThreads;
                const int lx = li / (kTileZ * kTileY), ly = (li / kTileZ) % kTileY, lz = li % kTileZ;
                const int gx = bx + lx, gy = by + ly, gz = bz + lz;
                double a0 = s_acc[li], a1 = s_acc[kTileCells + li];
                double a2 = s_acc[2 * kTileCells + li], a3 = s_acc[3 * kTileCells + li];
                for (int j = 0; j < np; ++j) {
                    const int i = gx - cp->lo[j][0], jj = gy - cp->lo[j][1], k = gz - cp->lo[j][2];
                    if (i < 0 || jj < 0 || k < 0 || i >= cp->dim[j][0] || jj >= cp->dim[j][1] || k >= cp->dim[j][2]) continue;
                    ++n_bbox;
                    const double radius = mul_rn(sup_in_h, cp->h[j]);
                    const double ex = fmax(fabs(cp->x[j] - s_cc[0][lx]) - g.hpx, 0.0);
                    const double ey = fmax(fabs(cp->y[j] - s_cc[1][ly]) - g.hpy, 0.0);
                    const double ez = fmax(fabs(cp->z[j] - s_cc[2][lz]) - g.hpz, 0.0);
                    // the support test of the pair counters, rounded as the host restatement rounds it
                    const bool in = add_rn(add_rn(mul_rn(ex, ex), mul_rn(ey, ey)), mul_rn(ez, ez)) < mul_rn(radius, radius);
                    n_sphere += in;
                    if (CULL && !in) continue;
                    ++n_eval;
                    const int n2 = cp->dim[j][2] + 1, n12 = (cp->dim[j][1] + 1) * n2;
                    const double* Tp = s_T + cp->poff[j] + (i * (cp->dim[j][1] + 1) + jj) * n2 + k;
                    const double m1 = (Tp[n12 + n2 + 1] - Tp[n12 + n2]) - (Tp[n12 + 1] - Tp[n12]);
                    const double m0 = (Tp[n2 + 1] - Tp[n2]) - (Tp[1] - Tp[0]);
                    double msum = m1 - m0;
                    if (msum < 0.0) {
                        ++n_neg;
                        if (msum <= -0.01) ++n_warn;
                        msum = 0.0;
                    }
                    if (msum == 0.0) continue;
                    const double mm = msum * cp->m[j];
                    a0 += mm;
                    a1 += mm * cp->vx[j];
                    a2 += mm * cp->vy[j];
                    a3 += mm * cp->vz[j];
                }
                s_acc[li] = a0;
                s_acc[kTileCells + li] = a1;
                s_acc[2 * kTileCells + li] = a2;
                s_acc[3 * kTileCells + li] = a3;
            }
        } else {
            double* const s_cm = s_chunk;  // (particle, cell) pair values at coff[j] + the cell's box index
            const int ctot = cp->ctot;
            const int coff_l = lane < np ? cp->coff[lane] : INT_MAX;
            for (int base = warp * 32; base < ctot; base += kLatThreads) {
                const int it = base + lane;
                const int j = warp_owner(base, coff_l, lane);
                const int cof = __shfl_sync(0xffffffffu, coff_l, j & 31);
                if (it < ctot) {
                    const int lc = it - cof;
                    const int d1 = cp->dim[j][1], d2 = cp->dim[j][2];
                    const int i = div_by(lc, cp->cmag[j][1]), rem = lc - i * (d1 * d2);
                    const int jj = div_by(rem, cp->cmag[j][0]), k = rem - jj * d2;
                    const int lx = cp->lo[j][0] - bx + i, ly = cp->lo[j][1] - by + jj, lz = cp->lo[j][2] - bz + k;
                    ++n_bbox;
                    const double radius = mul_rn(sup_in_h, cp->h[j]);
                    const double ex = fmax(fabs(cp->x[j] - s_cc[0][lx]) - g.hpx, 0.0);
                    const double ey = fmax(fabs(cp->y[j] - s_cc[1][ly]) - g.hpy, 0.0);
                    const double ez = fmax(fabs(cp->z[j] - s_cc[2][lz]) - g.hpz, 0.0);
                    // the support test of the pair counters, rounded as the host restatement rounds it
                    const bool in = add_rn(add_rn(mul_rn(ex, ex), mul_rn(ey, ey)), mul_rn(ez, ez)) < mul_rn(radius, radius);
                    n_sphere += in;
                    double msum = 0.0;
                    if (!CULL || in) {
                        ++n_eval;
                        const int n2 = d2 + 1, n12 = (d1 + 1) * n2;
                        const double* Tp = s_T + cp->poff[j] + (i * (d1 + 1) + jj) * n2 + k;
                        const double m1 = (Tp[n12 + n2 + 1] - Tp[n12 + n2]) - (Tp[n12 + 1] - Tp[n12]);
                        const double m0 = (Tp[n2 + 1] - Tp[n2]) - (Tp[1] - Tp[0]);
                        msum = m1 - m0;
                        if (msum < 0.0) {
                            ++n_neg;
                            if (msum <= -0.01) ++n_warn;
                            msum = 0.0;
                        }
                    }
                    s_cm[it] = msum;
                }
            }
            __syncthreads();
#pragma unroll
            for (int c = 0; c < kLatCellsPerThread; ++c) {
                const int li = threadIdx.x + c * kLatThreads;
                const int gx = bx + li / (kTileZ * kTileY), gy = by + (li / kTileZ) % kTileY, gz = bz + li % kTileZ;
                double a0 = s_acc[li], a1 = s_acc[kTileCells + li];
                double a2 = s_acc[2 * kTileCells + li], a3 = s_acc[3 * kTileCells + li];
                for (int j = 0; j < np; ++j) {
                    const int i = gx - cp->lo[j][0], jj = gy - cp->lo[j][1], k = gz - cp->lo[j][2];
                    const int d1 = cp->dim[j][1], d2 = cp->dim[j][2];
                    if (i < 0 || jj < 0 || k < 0 || i >= cp->dim[j][0] || jj >= d1 || k >= d2) continue;
                    const double msum = s_cm[cp->coff[j] + (i * d1 + jj) * d2 + k];
                    if (msum == 0.0) continue;
                    const double mm = msum * cp->m[j];
                    a0 += mm;
                    a1 += mm * cp->vx[j];
                    a2 += mm * cp->vy[j];
                    a3 += mm * cp->vz[j];
                }
                s_acc[li] = a0;
                s_acc[kTileCells + li] = a1;
                s_acc[2 * kTileCells + li] = a2;
                s_acc[3 * kTileCells + li] = a3;
            }
        }
        __syncthreads();
        pos += np;
        cp = nx;
        if (++n_chunks == (1u << 16)) {
            flush();
            n_chunks = 0;
        }
    }

    const double mvx = out.meanv[0], mvy = out.meanv[1], mvz = out.meanv[2];
    const int64_t ncell = (int64_t)g.nx * g.ny * g.nz;
#pragma unroll
    for (int c = 0; c < kLatCellsPerThread; ++c) {
        const int li = threadIdx.x + c * kLatThreads;
        const int ix = bx + li / (kTileZ * kTileY), iy = by + (li / kTileZ) % kTileY, iz = bz + li % kTileZ;
        if (ix >= g.nx || iy >= g.ny || iz >= g.nz) continue;
        const int64_t i3 = ((int64_t)ix * g.ny + iy) * g.nz + iz;
        const double M = s_acc[li];
        if (out.density) out.density[i3] = M / g.cell_volume;
        const bool has = M > 0.0;
        const double P1 = s_acc[kTileCells + li], P2 = s_acc[2 * kTileCells + li], P3 = s_acc[3 * kTileCells + li];
        if (out.vx) out.vx[i3] = has ? P1 / M : mvx;
        if (out.vy) out.vy[i3] = has ? P2 / M : mvy;
        if (out.vz) out.vz[i3] = has ? P3 / M : mvz;
        if (out.raw4) {
            out.raw4[i3] = M;
            out.raw4[ncell + i3] = P1;
            out.raw4[2 * ncell + i3] = P2;
            out.raw4[3 * ncell + i3] = P3;
        }
    }
    flush();
}

}  // namespace kiwi_b200
