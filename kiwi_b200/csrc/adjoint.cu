// Adjoint of the Cartesian sph-to-grid stage (no counterpart in the reference, which has no gradients).
//
// The forward pass produces, per cell c, the raw sums M_c = sum_p m_p K_pc and P_c = sum_p m_p K_pc v_p,
// where K_pc = max(Msum_pc, 0) is the particle's kernel mass inside the cell (src/cartesian_grid.cpp:
// 256-277).  Given the cotangents gM_c = dL/dM_c and gP_c = dL/dP_c, the adjoint returns per particle
//   dL/dm_p     = sum_c K_pc (gM_c + v_p . gP_c)
//   dL/dv_p     = m_p sum_c K_pc gP_c
//   dL/dtheta_p = m_p sum_c dK_pc/dtheta (gM_c + v_p . gP_c),   theta = x, y, z, h.
// The per-pair cell integrals are recomputed, not stored: the forward kernel's lattice tiers
// (lattice_edge_pair, lattice_point) are instantiated with the Dual3 type, which carries d/dx, d/dy, d/dz of
// every intermediate through the same operations (d/dh follows from them, see k_cart_adjoint_lattice), so the
// derivative part is the exact derivative of the evaluated formula (branch choices are taken on values).  A clamped pair (Msum < 0) has K = 0 and no
// gradient.  The pairs are those of the forward's default evaluation: the cells of the particle's
// support bounding box whose closest point lies within the support radius.
//
// The evaluation is the lattice form of the forward pass (lattice_tile.cuh) with derivatives: one CTA per
// 8^3-cell tile walks the tile's particles in chunks; (A) the edge tiers of every (plane, edge line), in
// swapped pairs, and (B) the octant value of every lattice point are computed once per particle with their
// derivatives; (C) for each particle, each thread assembles the cells it owns from their 8 corners' octant
// values (value and derivatives alike), weighs them with the cells' cotangents, and a fixed-order block
// reduction writes the particle's partial gradient for this tile to its (tile, particle) entry.  (D) Each
// particle's entries are then added in tile order.  Deterministic, no atomics on the gradients.
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
#include "lattice_dual.cuh"
#include "prims.cuh"

namespace kiwi_b200 {

namespace {

constexpr int kAdjLatThreads = 256;
constexpr int kAdjCellsPerThread = kTileCells / kAdjLatThreads;
constexpr int kAdjPMax = 32;
constexpr int kAdjECap = 1536;  // edge slots per chunk (a full 8^3 particle box has 486)
constexpr int kAdjPtCap = 2304; // lattice points per chunk (a full 8^3 particle box has 729)
constexpr int kAdjERec = 8;     // D2, D3 as Dual3
constexpr int kAdjTRec = 5;     // octant value and its derivatives with respect to x, y, z, h
constexpr size_t kAdjDynSmem = sizeof(double) * (kAdjERec * kAdjECap + kAdjTRec * kAdjPtCap);
static_assert(kAdjECap <= 2048, "packed edge-pair entries (11-bit slots)");
// generic kernels: edge records of lattice_generic_edge in Dual3 (offsets with derivatives)
constexpr int kAdjGenECap = kLatGenECap;
constexpr int kAdjGenERec = lat_gen_dual_rec<3>();
constexpr size_t kAdjGenDynSmem = sizeof(double) * (kAdjGenERec * kAdjGenECap + kAdjTRec * kAdjPtCap);

static __constant__ KiwiKernelTable c_adj_tables[KIWI_NUM_KERNELS];

struct AdjGrads {
    double *x, *y, *z, *h, *m, *vx, *vy, *vz;
};

// |plane - x_axis| with its derivative with respect to the particle's coordinate on that axis
__device__ __forceinline__ Dual3 dual_abs_offset(double off, int axis) {
    Dual3 r(fabs(off));
    r.d[axis] = off > 0.0 ? -1.0 : (off < 0.0 ? 1.0 : 0.0);
    return r;
}

__device__ __forceinline__ Dual3 load_dual(const double* p) {
    Dual3 r(p[0]);
    r.d[0] = p[1];
    r.d[1] = p[2];
    r.d[2] = p[3];
    return r;
}

__device__ __forceinline__ void store_dual(double* p, const Dual3& v) {
    p[0] = v.v;
    p[1] = v.d[0];
    p[2] = v.d[1];
    p[3] = v.d[2];
}

// The six edge tiers (with derivatives) of a lattice point, read from the chunk's table where lattice_point
// uses them: slots in PointEdge order, D2 at +0 and D3 at +4 of each record.
struct SmemDualEdges {
    const double* rec;
    int slot[6];
    __device__ __forceinline__ Dual3 D2(int e) const { return load_dual(rec + kAdjERec * slot[e]); }
    __device__ __forceinline__ Dual3 D3(int e) const { return load_dual(rec + kAdjERec * slot[e] + 4); }
    __device__ __forceinline__ void leg_angles(int, const Dual3& a1, const Dual3& ia1, const Dual3& a2,
                                               const Dual3& ia2, Dual3& pa, Dual3& pb) const {
        kiwi_b200::leg_angles(a1, ia1, a2, ia2, pa, pb);
    }
};

__device__ __forceinline__ unsigned long long block_count(unsigned long long v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// (A)-(C) for one tile: list holds (tile, particle) entry indices (the entries of particle p are
// offs[p] .. offs[p+1]-1); part receives 8 doubles per entry: dL/dm, dL/d(x, y, z, h), dL/d(vx, vy, vz)
// over this tile's cells.
//
// The octant value T of a lattice point at offsets u = (ux, uy, uz) from the particle is sgn(ux) sgn(uy)
// sgn(uz) G(|ux|, |uy|, |uz|), with G the kernel mass of the box spanned by the particle and the point
// (lattice_point).  G is a mass fraction of a kernel of scale h, so G(a, b, c; h) = G(a/h, b/h, c/h; 1): it is
// homogeneous of degree 0 in (a, b, c, h), whence dT/dh = (ux dT/dx + uy dT/dy + uz dT/dz) / h with the
// derivatives taken with respect to the particle's coordinates (u = plane - particle).  The tiers are
// therefore evaluated with three forward derivatives (Dual3, h held fixed) and dT/dh follows from them.
//
// GENERIC: the table-driven tiers of kernel `kernel` (support g.support_in_h x h): every edge line's record
// (lattice_generic_edge in Dual3) in (A), the points' six vertex tiers together (lattice_generic_point in
// Dual3) in (B).  The same homogeneity gives d/dh.
template <bool GENERIC>
__global__ void __launch_bounds__(kAdjLatThreads, 1) k_cart_adjoint_lattice(CartGeom g, DevParticles P, int kernel,
                                                                          const uint32_t* __restrict__ list,
                                                                          const int64_t* __restrict__ range,
                                                                          const int64_t* __restrict__ offs,
                                                                          const double* __restrict__ cot,
                                                                          double* __restrict__ part,
                                                                          DevStats* __restrict__ st) {
    __shared__ double s_x[kAdjPMax], s_y[kAdjPMax], s_z[kAdjPMax], s_h[kAdjPMax], s_ih[kAdjPMax], s_m[kAdjPMax],
        s_vx[kAdjPMax], s_vy[kAdjPMax], s_vz[kAdjPMax];
    __shared__ int s_lo[kAdjPMax][3], s_dim[kAdjPMax][3], s_eoff[kAdjPMax], s_poff[kAdjPMax];
    __shared__ uint32_t s_entry[kAdjPMax];
    __shared__ uint32_t s_mag[kAdjPMax][4];  // div_magic of n0', n1', n2' and n1' n2'
    __shared__ uint32_t s_plist[kAdjPtCap];
    __shared__ uint32_t s_hlist[kAdjECap / 2];
    __shared__ int s_np, s_etot, s_ptot, s_nexp, s_ncheap, s_nheavy, s_ninner;
    __shared__ double s_red[kAdjLatThreads / 32][8];
    __shared__ double s_pl[3][kTileX + 1];
    extern __shared__ double s_adj[];
    constexpr int kERec = GENERIC ? kAdjGenERec : kAdjERec;
    constexpr int kECap = GENERIC ? kAdjGenECap : kAdjECap;
    const KiwiKernelTable* K = GENERIC ? &c_adj_tables[kernel] : nullptr;
    double* s_E = s_adj;
    double* s_T = s_adj + kERec * kECap;

    const int64_t t = blockIdx.x;
    const int tz = (int)(t % g.ntz), ty = (int)((t / g.ntz) % g.nty), tx = (int)(t / ((int64_t)g.ntz * g.nty));
    const int bx = tx * kTileX, by = ty * kTileY, bz = tz * kTileZ;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t ncell = (int64_t)g.nx * g.ny * g.nz;
    unsigned long long n_eval = 0, n_neg = 0;
    const int64_t beg = range[2 * t], end = range[2 * t + 1];
    if (threadIdx.x < 3 * (kTileX + 1)) {
        const int a = threadIdx.x / (kTileX + 1), l = threadIdx.x % (kTileX + 1);
        const double mn = a == 0 ? g.x_min : (a == 1 ? g.y_min : g.z_min), d = a == 0 ? g.dpx : (a == 1 ? g.dpy : g.dpz);
        s_pl[a][l] = add_rn(mn, mul_rn((double)((a == 0 ? bx : (a == 1 ? by : bz)) + l), d));
    }

    for (int64_t pos = beg; pos < end;) {
        if (warp == 0) {
            const int64_t idx = pos + lane;
            int ne = 0, npt = 0, lo0 = 0, lo1 = 0, lo2 = 0, d0 = 0, d1 = 0, d2 = 0;
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
                npt = n0 * n1 * n2;
            }
            int ie = ne, ip = npt;
            for (int o = 1; o < 32; o <<= 1) {
                const int ve = __shfl_up_sync(0xffffffffu, ie, o), vp = __shfl_up_sync(0xffffffffu, ip, o);
                if (lane >= o) {
                    ie += ve;
                    ip += vp;
                }
            }
            const bool take = (idx < end) && ie <= kECap && ip <= kAdjPtCap;
            const int np = __popc(__ballot_sync(0xffffffffu, take));
            if (take) {
                s_x[lane] = px; s_y[lane] = py; s_z[lane] = pz; s_h[lane] = ph; s_ih[lane] = 1.0 / ph;
                s_m[lane] = pm; s_vx[lane] = pvx; s_vy[lane] = pvy; s_vz[lane] = pvz;
                s_lo[lane][0] = lo0; s_lo[lane][1] = lo1; s_lo[lane][2] = lo2;
                s_dim[lane][0] = d0; s_dim[lane][1] = d1; s_dim[lane][2] = d2;
                s_eoff[lane] = ie - ne;
                s_poff[lane] = ip - npt;
                s_entry[lane] = e;
                s_mag[lane][0] = div_magic(d0 + 1);
                s_mag[lane][1] = div_magic(d1 + 1);
                s_mag[lane][2] = div_magic(d2 + 1);
                s_mag[lane][3] = div_magic((d1 + 1) * (d2 + 1));
            }
            if (lane == np - 1) {
                s_np = np;
                s_etot = ie;
                s_ptot = ip;
                s_nexp = s_ncheap = s_nheavy = s_ninner = 0;
            }
        }
        __syncthreads();
        const int np = s_np, etot = s_etot, ptot = s_ptot;

        // (A) edge pairs, as the forward kernel walks them: pairs beyond 2h (or zero) get D2 = D3 = 0; the
        // others are listed (slot ab | slot ba << 11 | particle << 22 | pair block << 27) with the two signed
        // offsets parked in slot ab, and evaluated in (A2) by full warps.
        {
            const int qtot = etot >> 1;
            const int qoff_l = lane < np ? (s_eoff[lane] >> 1) : INT_MAX;
            for (int base = warp * 32; base < qtot; base += kAdjLatThreads) {
                const int it = base + lane;
                bool heavy = false, inner = false;
                uint32_t hrec = 0;
                const int j = warp_owner(base, qoff_l, lane);
                const int qoff = __shfl_sync(0xffffffffu, qoff_l, j & 31);
                if (it < qtot) {
                    int e = it - qoff;
                    const int n0 = s_dim[j][0] + 1, n1 = s_dim[j][1] + 1, n2 = s_dim[j][2] + 1;
                    const int nxy = n0 * n1, nxz = n0 * n2, nyz = n1 * n2;
                    const int blk = (e >= nxy) + (e >= nxy + nxz);
                    e -= blk == 0 ? 0 : (blk == 1 ? nxy : nxy + nxz);
                    const int a = blk == 2 ? 1 : 0, b = blk == 0 ? 1 : 2;
                    const int nb = b == 1 ? n1 : n2, na = a == 0 ? n0 : n1;
                    const int pi = div_by(e, s_mag[j][b]), qi = e - pi * nb;
                    const int eb = s_eoff[j];
                    const int sab = eb + (blk == 0 ? 0 : (blk == 1 ? nxy : 2 * nxy + nxz)) + pi * nb + qi;
                    const int sba = eb + (blk == 0 ? nxy + nxz : (blk == 1 ? 2 * nxy + nxz + nyz : 2 * nxy + 2 * nxz + nyz)) +
                                    qi * na + pi;
                    const int la = s_lo[j][a] - (a == 0 ? bx : by), lb = s_lo[j][b] - (b == 1 ? by : bz);
                    const double oa = s_pl[a][la + pi] - (a == 0 ? s_x[j] : s_y[j]);
                    const double ob = s_pl[b][lb + qi] - (b == 1 ? s_y[j] : s_z[j]);
                    const double h = s_h[j];
                    if (GENERIC) {
                        // both orientations' records, evaluated here (no pair list)
                        const double H = mul_rn(g.support_in_h, h);
                        const Dual3 pD = dual_abs_offset(oa, a), qD = dual_abs_offset(ob, b);
                        lattice_generic_edge_dual<3>(K, H, pD, qD, s_E + kERec * sab);
                        lattice_generic_edge_dual<3>(K, H, qD, pD, s_E + kERec * sba);
                    } else {
                    heavy = oa != 0.0 && ob != 0.0 && oa * oa + ob * ob <= 4.0 * (h * h);
                    inner = heavy && oa * oa + ob * ob <= h * h;
                    if (heavy) {
                        s_E[kAdjERec * sab] = oa;
                        s_E[kAdjERec * sab + 1] = ob;
                        hrec = (uint32_t)sab | (uint32_t)sba << 11 | (uint32_t)j << 22 | (uint32_t)blk << 27;
                    } else {
#pragma unroll
                        for (int k = 0; k < kAdjERec; ++k) s_E[kAdjERec * sab + k] = s_E[kAdjERec * sba + k] = 0.0;
                    }
                    }
                }
                // pairs within h (two passes of the edge tiers) from the end of the list, the others from the
                // front, so that each kind runs in warps of its own
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
                if (heavy) s_hlist[inner ? kAdjECap / 2 - 1 - hi - __popc(mi & below) : hp + __popc(mm & below)] = hrec;
            }
        }

        // (B0) the lattice points some evaluated cell reads, listed as in the forward kernel (the same padded
        // test); a point on a particle plane has octant value 0 and no derivative, written here.
        {
            const int poff_l = lane < np ? s_poff[lane] : INT_MAX;
            for (int base = warp * 32; base < ptot; base += kAdjLatThreads) {
                const int pt = base + lane;
                int cls = -1;  // -1 none, 0 within 2h, 1 beyond
                uint32_t rec = 0;
                const int jp = warp_owner(base, poff_l, lane);
                const int poff = __shfl_sync(0xffffffffu, poff_l, jp & 31);
                if (pt < ptot) {
                    const int lp = pt - poff;
                    const int n2 = s_dim[jp][2] + 1, n12 = (s_dim[jp][1] + 1) * n2;
                    const int i = div_by(lp, s_mag[jp][3]), rem = lp - i * n12;
                    const int jj = div_by(rem, s_mag[jp][2]), k = rem - jj * n2;
                    const double ux = s_pl[0][s_lo[jp][0] - bx + i] - s_x[jp];
                    const double uy = s_pl[1][s_lo[jp][1] - by + jj] - s_y[jp];
                    const double uz = s_pl[2][s_lo[jp][2] - bz + k] - s_z[jp];
                    const double h = s_h[jp], radius = mul_rn(g.support_in_h, h);
                    const double ex = fmax(fabs(ux) - kNeedPad * g.dpx, 0.0);
                    const double ey = fmax(fabs(uy) - kNeedPad * g.dpy, 0.0);
                    const double ez = fmax(fabs(uz) - kNeedPad * g.dpz, 0.0);
                    if (ex * ex + ey * ey + ez * ez < radius * radius) {
                        if (ux == 0.0 || uy == 0.0 || uz == 0.0) {
#pragma unroll
                            for (int c = 0; c < kAdjTRec; ++c) s_T[kAdjTRec * pt + c] = 0.0;
                        } else {
                            cls = (ux * ux + uy * uy + uz * uz < (GENERIC ? radius * radius : 4.0 * (h * h))) ? 0 : 1;
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
                if (cls >= 0) s_plist[cls == 0 ? pe + __popc(me & below) : kAdjPtCap - 1 - pcb - __popc(mc & below)] = rec;
            }
        }
        __syncthreads();

        // (A2) the listed edge pairs with their derivatives (the forward kernel's lattice_edge_pair in Dual3)
        {
            const int nmid = s_nheavy, ninner = s_ninner;
            for (int li = threadIdx.x; li < nmid + ninner; li += kAdjLatThreads) {
                const uint32_t rec = s_hlist[li < nmid ? li : kAdjECap / 2 - ninner + (li - nmid)];
                const int sab = (int)(rec & 2047u), sba = (int)((rec >> 11) & 2047u), j = (int)((rec >> 22) & 31u);
                const int blk = (int)(rec >> 27);
                const int a = blk == 2 ? 1 : 0, b = blk == 0 ? 1 : 2;
                const Dual3 pD = dual_abs_offset(s_E[kAdjERec * sab], a);
                const Dual3 qD = dual_abs_offset(s_E[kAdjERec * sab + 1], b);
                LatticeEdgeT<Dual3> e_pq, e_qp;
                lattice_edge_pair(Dual3(s_h[j]), Dual3(s_ih[j]), pD, qD, e_pq, e_qp);
                store_dual(s_E + kAdjERec * sab, e_pq.D2);
                store_dual(s_E + kAdjERec * sab + 4, e_pq.D3);
                store_dual(s_E + kAdjERec * sba, e_qp.D2);
                store_dual(s_E + kAdjERec * sba + 4, e_qp.D3);
            }
        }
        __syncthreads();

        // (B) octant values with their derivatives
        const int nexp = s_nexp, ncheap = s_ncheap;
        for (int li = threadIdx.x; li < nexp + ncheap; li += kAdjLatThreads) {
            const uint32_t rec = s_plist[li < nexp ? li : kAdjPtCap - ncheap + (li - nexp)];
            const int jp = (int)(rec & 31u), i = (int)((rec >> 5) & 15u), jj = (int)((rec >> 9) & 15u),
                      k = (int)((rec >> 13) & 15u);
            const int n0 = s_dim[jp][0] + 1, n1 = s_dim[jp][1] + 1, n2 = s_dim[jp][2] + 1;
            const int it = s_poff[jp] + (i * n1 + jj) * n2 + k;
            const double ux = s_pl[0][s_lo[jp][0] - bx + i] - s_x[jp];
            const double uy = s_pl[1][s_lo[jp][1] - by + jj] - s_y[jp];
            const double uz = s_pl[2][s_lo[jp][2] - bz + k] - s_z[jp];
            const int eb = s_eoff[jp];
            const int nxy = n0 * n1, nxz = n0 * n2, nyz = n1 * n2;
            const int slots[6] = {eb + i * n1 + jj, eb + nxy + i * n2 + k, eb + nxy + nxz + jj * n0 + i,
                                  eb + 2 * nxy + nxz + jj * n2 + k, eb + 2 * nxy + nxz + nyz + k * n0 + i,
                                  eb + 2 * nxy + 2 * nxz + nyz + k * n1 + jj};
            const double sg = sgn(ux) * sgn(uy) * sgn(uz);
            Dual3 f;
            if (GENERIC) {
                const GenEdgeRecsDual<3> R{s_E, {slots[0], slots[1], slots[2], slots[3], slots[4], slots[5]}};
                f = sg * lattice_generic_point(K, mul_rn(g.support_in_h, s_h[jp]), dual_abs_offset(ux, 0),
                                               dual_abs_offset(uy, 1), dual_abs_offset(uz, 2), R);
            } else {
                const SmemDualEdges PE{s_E, {slots[0], slots[1], slots[2], slots[3], slots[4], slots[5]}};
                f = sg * lattice_point(Dual3(s_h[jp]), Dual3(s_ih[jp]), dual_abs_offset(ux, 0),
                                       dual_abs_offset(uy, 1), dual_abs_offset(uz, 2), PE);
            }
            double* o = s_T + kAdjTRec * it;
            o[0] = f.v;
            o[1] = f.d[0];
            o[2] = f.d[1];
            o[3] = f.d[2];
            o[4] = (ux * f.d[0] + uy * f.d[1] + uz * f.d[2]) * s_ih[jp];
        }
        __syncthreads();

        // (C) per particle: each cell's value and derivatives as the alternating sum of its 8 corners,
        // weighed by the cell's cotangents
        for (int j = 0; j < np; ++j) {
            double acc[8];
#pragma unroll
            for (int c = 0; c < 8; ++c) acc[c] = 0.0;
            const double x0 = s_x[j], y0 = s_y[j], z0 = s_z[j];
            const double radius = mul_rn(g.support_in_h, s_h[j]);
            const int n2 = s_dim[j][2] + 1, n12 = (s_dim[j][1] + 1) * n2;
#pragma unroll
            for (int c = 0; c < kAdjCellsPerThread; ++c) {
                const int li = threadIdx.x + c * kAdjLatThreads;
                const int gz = bz + li % kTileZ, gy = by + (li / kTileZ) % kTileY, gx = bx + li / (kTileZ * kTileY);
                const int i = gx - s_lo[j][0], jj = gy - s_lo[j][1], k = gz - s_lo[j][2];
                if (i < 0 || jj < 0 || k < 0 || i >= s_dim[j][0] || jj >= s_dim[j][1] || k >= s_dim[j][2]) continue;
                const double ex = fmax(fabs(x0 - cell_centre(g.x_min, gx, g.dpx)) - g.hpx, 0.0);
                const double ey = fmax(fabs(y0 - cell_centre(g.y_min, gy, g.dpy)) - g.hpy, 0.0);
                const double ez = fmax(fabs(z0 - cell_centre(g.z_min, gz, g.dpz)) - g.hpz, 0.0);
                if (!(add_rn(add_rn(mul_rn(ex, ex), mul_rn(ey, ey)), mul_rn(ez, ez)) < mul_rn(radius, radius))) continue;
                ++n_eval;
                const double* Tp = s_T + kAdjTRec * (s_poff[j] + (i * (s_dim[j][1] + 1) + jj) * n2 + k);
                // component comp of the cell's Msum: 0 the value, 1..4 d/d(x, y, z, h)
                auto cell_sum = [&](int comp) {
                    auto at = [&](int off) { return Tp[kAdjTRec * off + comp]; };
                    const double m1 = (at(n12 + n2 + 1) - at(n12 + n2)) - (at(n12 + 1) - at(n12));
                    const double m0 = (at(n2 + 1) - at(n2)) - (at(1) - at(0));
                    return m1 - m0;
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
#pragma unroll
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

int adjoint_init_tables(KiwiCtx* ctx) {
    KIWI_CUDA(ctx, cudaMemcpyToSymbol(c_adj_tables, kiwi_kernel_tables, sizeof(kiwi_kernel_tables)));
    return KIWI_OK;
}

int cart_adjoint_dev(KiwiCtx* ctx, const DevParticles& P, const CartGeom& g, const KernelChoice& kc,
                     const double* d_cot, const AdjointOutputs& out, KiwiStats* stats) {
    if (kc.tabulated)
        return set_err(ctx, KIWI_ERR_UNSUPPORTED,
                       "the adjoint is available for the analytic integrals (cubic closed form and the generic "
                       "kernels' tables), not for the tabulated one");
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
        if (kc.cubic) {
            KIWI_CUDA(ctx, cudaFuncSetAttribute(k_cart_adjoint_lattice<false>,
                                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kAdjDynSmem));
            k_cart_adjoint_lattice<false><<<(unsigned)ntiles, kAdjLatThreads, kAdjDynSmem, ctx->stream>>>(
                g, P, 0, second ? v1 : v0, range, offs, d_cot, part, d_st);
        } else {
            KIWI_CUDA(ctx, cudaFuncSetAttribute(k_cart_adjoint_lattice<true>,
                                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kAdjGenDynSmem));
            k_cart_adjoint_lattice<true><<<(unsigned)ntiles, kAdjLatThreads, kAdjGenDynSmem, ctx->stream>>>(
                g, P, kc.kernel, second ? v1 : v0, range, offs, d_cot, part, d_st);
        }
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
