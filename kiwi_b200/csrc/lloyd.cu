// The point-set stage's Lloyd step (lloyd_step, src/point_set.cpp:265-293): every site the Voro++
// container keeps moves to the centroid of its Voronoi cell (the cell clipped to the domain box), and the
// sites come out in the container's walk order.
//
// GPU form: one thread builds one cell.  The cell starts as the domain box, held in the dual form of a
// convex polyhedron -- its planes, and its vertices as triangles of three plane indices ordered
// counter-clockwise seen from outside -- and is clipped by the bisector plane of each neighbouring site,
// taken shell by shell from a uniform bin grid around the site, each shell's sites nearest first (so the
// cell shrinks fast and few planes are spent on sites that later clips make irrelevant; dense bins are
// scanned in several passes of at most 128 candidates): a clip removes the
// vertices beyond the plane and closes the hole with one new vertex per crossing edge (the removed vertices' edges whose
// twin edge belongs to a kept vertex).  The search stops once no unsearched site can be nearer than twice
// the cell's radius (any farther site's bisector misses the cell).  Volume and centroid come from a fan of
// tetrahedra from the site over each face polygon, walked around the face through the triangles that
// share its plane.  The walk order is the container's: blocks in index order, each block's sites in input
// order (a stable radix sort by block).  Built with --fmad=false, like the other FP64 units.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "engine.hpp"
#include "prims.cuh"
#include "sitebins.cuh"

using namespace kiwi_b200;

namespace {

constexpr int kPMax = 128;  // planes of one cell (6 walls + the bisectors that cut it)
constexpr int kTMax = 192;  // vertices of one cell

enum CellStatus { kCellOk = 0, kCellEmpty = 1, kCellCapacity = 2, kCellWalk = 3 };

struct Cell {
    double pl[kPMax][4];  // outward normal and offset: n . v <= d inside (site at the origin)
    unsigned char t[kTMax][3];
    double v[kTMax][3];
    int np, nt;
};

__host__ __device__ inline bool vertex_of(const Cell& c, int a, int b, int d, double* out) {
    const double* A = c.pl[a];
    const double* B = c.pl[b];
    const double* D = c.pl[d];
    const double bc0 = B[1] * D[2] - B[2] * D[1], bc1 = B[2] * D[0] - B[0] * D[2], bc2 = B[0] * D[1] - B[1] * D[0];
    const double ca0 = D[1] * A[2] - D[2] * A[1], ca1 = D[2] * A[0] - D[0] * A[2], ca2 = D[0] * A[1] - D[1] * A[0];
    const double ab0 = A[1] * B[2] - A[2] * B[1], ab1 = A[2] * B[0] - A[0] * B[2], ab2 = A[0] * B[1] - A[1] * B[0];
    const double det = A[0] * bc0 + A[1] * bc1 + A[2] * bc2;
    if (det == 0.0) return false;
    out[0] = (A[3] * bc0 + B[3] * ca0 + D[3] * ab0) / det;
    out[1] = (A[3] * bc1 + B[3] * ca1 + D[3] * ab1) / det;
    out[2] = (A[3] * bc2 + B[3] * ca2 + D[3] * ab2) / det;
    return true;
}

// The domain box around a site at (sx, sy, sz): planes 0..5 = -x, +x, -y, +y, -z, +z walls; its 8 corners
// with their planes ordered so that det(n_a, n_b, n_c) > 0 (counter-clockwise seen from outside).
__host__ __device__ void cell_box(Cell& c, const VoroBlocks& V, double sx, double sy, double sz) {
    const double lo[3] = {V.ax - sx, V.ay - sy, V.az - sz}, hi[3] = {V.bx - sx, V.by - sy, V.bz - sz};
    for (int a = 0; a < 3; ++a) {
        for (int s = 0; s < 2; ++s) {
            double* P = c.pl[2 * a + s];
            P[0] = P[1] = P[2] = 0.0;
            P[a] = s ? 1.0 : -1.0;
            P[3] = s ? hi[a] : -lo[a];
        }
    }
    c.np = 6;
    c.nt = 0;
    for (int ix = 0; ix < 2; ++ix)
        for (int iy = 0; iy < 2; ++iy)
            for (int iz = 0; iz < 2; ++iz) {
                // sign of det(n_x, n_y, n_z) for normals (+-1, 0, 0), (0, +-1, 0), (0, 0, +-1)
                const int sgn = (ix ? 1 : -1) * (iy ? 1 : -1) * (iz ? 1 : -1);
                unsigned char* T = c.t[c.nt];
                T[0] = (unsigned char)(0 + ix);
                T[1] = (unsigned char)(sgn > 0 ? 2 + iy : 4 + iz);
                T[2] = (unsigned char)(sgn > 0 ? 4 + iz : 2 + iy);
                c.v[c.nt][0] = ix ? hi[0] : lo[0];
                c.v[c.nt][1] = iy ? hi[1] : lo[1];
                c.v[c.nt][2] = iz ? hi[2] : lo[2];
                ++c.nt;
            }
}

// Clips the cell by n . v <= d (n = the neighbour's offset, d = |n|^2 / 2).  Returns a CellStatus; *r2 is
// updated to the largest squared vertex distance when the cell changed.
__host__ __device__ int cell_clip(Cell& c, double nx, double ny, double nz, double d, double eps, double* r2) {
    unsigned out_mask[(kTMax + 31) / 32];
    int n_out = 0;
    for (int w = 0; w < (kTMax + 31) / 32; ++w) out_mask[w] = 0u;
    for (int i = 0; i < c.nt; ++i) {
        const double g = nx * c.v[i][0] + ny * c.v[i][1] + nz * c.v[i][2] - d;
        if (g > eps) {
            out_mask[i >> 5] |= 1u << (i & 31);
            ++n_out;
        }
    }
    if (n_out == 0) return kCellOk;
    if (n_out == c.nt) return kCellEmpty;
    if (c.np >= kPMax) return kCellCapacity;
    const int p = c.np++;
    c.pl[p][0] = nx;
    c.pl[p][1] = ny;
    c.pl[p][2] = nz;
    c.pl[p][3] = d;
    // crossing edges: directed edges of removed vertices whose twin belongs to a kept vertex
    unsigned char be_a[kTMax], be_b[kTMax];
    int nb = 0;
    for (int i = 0; i < c.nt; ++i) {
        if (!((out_mask[i >> 5] >> (i & 31)) & 1u)) continue;
        for (int e = 0; e < 3; ++e) {
            const int a = c.t[i][e], b = c.t[i][(e + 1) % 3];
            bool interior = false;
            for (int j = 0; j < c.nt && !interior; ++j) {
                if (j == i || !((out_mask[j >> 5] >> (j & 31)) & 1u)) continue;
                const unsigned char* T = c.t[j];
                interior = (T[0] == b && T[1] == a) || (T[1] == b && T[2] == a) || (T[2] == b && T[0] == a);
            }
            if (!interior) {
                if (nb >= kTMax) return kCellCapacity;
                be_a[nb] = (unsigned char)a;
                be_b[nb] = (unsigned char)b;
                ++nb;
            }
        }
    }
    // keep the inside vertices, append one per crossing edge
    int k = 0;
    for (int i = 0; i < c.nt; ++i) {
        if ((out_mask[i >> 5] >> (i & 31)) & 1u) continue;
        if (k != i) {
            c.t[k][0] = c.t[i][0];
            c.t[k][1] = c.t[i][1];
            c.t[k][2] = c.t[i][2];
            c.v[k][0] = c.v[i][0];
            c.v[k][1] = c.v[i][1];
            c.v[k][2] = c.v[i][2];
        }
        ++k;
    }
    if (k + nb > kTMax) return kCellCapacity;
    for (int e = 0; e < nb; ++e) {
        c.t[k][0] = be_a[e];
        c.t[k][1] = be_b[e];
        c.t[k][2] = (unsigned char)p;
        if (!vertex_of(c, be_a[e], be_b[e], p, c.v[k])) return kCellEmpty;
        ++k;
    }
    c.nt = k;
    double m = 0.0;
    for (int i = 0; i < c.nt; ++i) m = fmax(m, c.v[i][0] * c.v[i][0] + c.v[i][1] * c.v[i][1] + c.v[i][2] * c.v[i][2]);
    *r2 = m;
    return kCellOk;
}

// Volume and centroid (site-relative) by tetrahedra from the site over each face's polygon.
__host__ __device__ int cell_moments(const Cell& c, double* vol, double* cen) {
    double v6 = 0.0, cx = 0.0, cy = 0.0, cz = 0.0;
    for (int p = 0; p < c.np; ++p) {
        // a vertex on plane p, rotated to (p, a, b)
        int t0 = -1, b = 0;
        for (int i = 0; i < c.nt && t0 < 0; ++i)
            for (int e = 0; e < 3; ++e)
                if (c.t[i][e] == p) {
                    t0 = i;
                    b = c.t[i][(e + 2) % 3];
                    break;
                }
        if (t0 < 0) continue;  // a plane the later clips removed
        const double* v0 = c.v[t0];
        const double* vprev = nullptr;
        int steps = 0;
        for (;;) {
            // the vertex after (p, a, b) around p is the one holding the directed edge (p, b)
            int nxt = -1, nb = 0;
            for (int i = 0; i < c.nt && nxt < 0; ++i)
                for (int e = 0; e < 3; ++e)
                    if (c.t[i][e] == p && c.t[i][(e + 1) % 3] == b) {
                        nxt = i;
                        nb = c.t[i][(e + 2) % 3];
                        break;
                    }
            if (nxt < 0 || ++steps > c.nt) return kCellWalk;
            if (nxt == t0) break;
            const double* v1 = c.v[nxt];
            if (vprev) {
                const double d6 = v0[0] * (vprev[1] * v1[2] - vprev[2] * v1[1]) +
                                  v0[1] * (vprev[2] * v1[0] - vprev[0] * v1[2]) +
                                  v0[2] * (vprev[0] * v1[1] - vprev[1] * v1[0]);
                v6 += d6;
                cx += d6 * (v0[0] + vprev[0] + v1[0]);
                cy += d6 * (v0[1] + vprev[1] + v1[1]);
                cz += d6 * (v0[2] + vprev[2] + v1[2]);
            }
            vprev = v1;
            b = nb;
        }
    }
    if (!(v6 != 0.0)) return kCellEmpty;
    *vol = fabs(v6) / 6.0;
    cen[0] = cx / (4.0 * v6);
    cen[1] = cy / (4.0 * v6);
    cen[2] = cz / (4.0 * v6);
    return kCellOk;
}

constexpr int kCandMax = 128;  // neighbour candidates held (sorted) at a time

// (d, i) < (e, j) in the order candidates are clipped: by squared distance, then by sorted index.
__host__ __device__ inline bool cand_less(double d, int64_t i, double e, int64_t j) { return d < e || (d == e && i < j); }

// The Voronoi cell in the box of the q-th kept site of B.  Neighbours come shell by shell of search bins;
// within a shell they are clipped nearest first: a pass keeps the kCandMax nearest not yet clipped, clips
// them, and scans the shell again while it had to leave some out (dense bins).  Stops once every unsearched
// site is at least twice the cell's radius away.  Returns a CellStatus; the centroid (absolute) and volume
// on success.
__host__ __device__ int build_cell(Cell& c, const SiteBins& B, const VoroBlocks& V, int64_t q, double eps,
                                   double* cen, double* vol) {
    const double sx = B.sx[q], sy = B.sy[q], sz = B.sz[q];
    const int32_t self = B.sidx[q];
    cell_box(c, V, sx, sy, sz);
    double r2 = 0.0;
    for (int i = 0; i < c.nt; ++i) r2 = fmax(r2, c.v[i][0] * c.v[i][0] + c.v[i][1] * c.v[i][1] + c.v[i][2] * c.v[i][2]);
    const int bx = bin_of(sx, B.x0, B.wx, B.nbx), by = bin_of(sy, B.y0, B.wy, B.nby), bz = bin_of(sz, B.z0, B.wz, B.nbz);
    const int rmax = max(max(B.nbx, B.nby), B.nbz);
    double cd[kCandMax];
    int64_t ci[kCandMax];
    for (int r = 0; r <= rmax; ++r) {
        const int i0 = max(bx - r, 0), i1 = min(bx + r, B.nbx - 1);
        const int j0 = max(by - r, 0), j1 = min(by + r, B.nby - 1);
        const int k0 = max(bz - r, 0), k1 = min(bz + r, B.nbz - 1);
        double done_d = -1.0;  // candidates up to (done_d, done_i) are clipped already
        int64_t done_i = -1;
        for (int pass = 0;; ++pass) {
            int nc = 0;
            bool left_out = false;
            for (int i = i0; i <= i1; ++i)
                for (int j = j0; j <= j1; ++j) {
                    const bool face = (i == bx - r || i == bx + r || j == by - r || j == by + r);
                    const int64_t row = ((int64_t)i * B.nby + j) * B.nbz;
                    for (int k = k0; k <= k1; ++k) {
                        if (!face && k != bz - r && k != bz + r) continue;
                        const int64_t bin = row + k;
                        const int64_t e = B.range[2 * bin + 1];
                        for (int64_t s = B.range[2 * bin]; s < e; ++s) {
                            if (B.sidx[s] == self) continue;
                            const double dx = B.sx[s] - sx, dy = B.sy[s] - sy, dz = B.sz[s] - sz;
                            const double dd = dx * dx + dy * dy + dz * dz;
                            if (dd == 0.0 || dd >= 4.0 * r2) continue;  // a coincident site, or beyond reach
                            if (!cand_less(done_d, done_i, dd, s)) continue;  // clipped in an earlier pass
                            // insert into the sorted buffer, keeping the kCandMax nearest
                            if (nc == kCandMax) {
                                left_out = true;
                                if (!cand_less(dd, s, cd[nc - 1], ci[nc - 1])) continue;
                                --nc;
                            }
                            int m = nc++;
                            while (m > 0 && cand_less(dd, s, cd[m - 1], ci[m - 1])) {
                                cd[m] = cd[m - 1];
                                ci[m] = ci[m - 1];
                                --m;
                            }
                            cd[m] = dd;
                            ci[m] = s;
                        }
                    }
                }
            for (int m = 0; m < nc; ++m) {
                if (cd[m] >= 4.0 * r2) break;  // sorted: the rest are beyond reach too
                const int64_t s = ci[m];
                const int st = cell_clip(c, B.sx[s] - sx, B.sy[s] - sy, B.sz[s] - sz, 0.5 * cd[m], eps * sqrt(cd[m]), &r2);
                if (st != kCellOk) return st;
            }
            if (!left_out || pass > 1000000) break;
            done_d = cd[nc - 1];
            done_i = ci[nc - 1];
        }
        if (i0 == 0 && j0 == 0 && k0 == 0 && i1 == B.nbx - 1 && j1 == B.nby - 1 && k1 == B.nbz - 1) break;
        double dmin = INFINITY;
        if (i0 > 0) dmin = fmin(dmin, sx - (B.x0 + i0 * B.wx));
        if (i1 < B.nbx - 1) dmin = fmin(dmin, (B.x0 + (i1 + 1) * B.wx) - sx);
        if (j0 > 0) dmin = fmin(dmin, sy - (B.y0 + j0 * B.wy));
        if (j1 < B.nby - 1) dmin = fmin(dmin, (B.y0 + (j1 + 1) * B.wy) - sy);
        if (k0 > 0) dmin = fmin(dmin, sz - (B.z0 + k0 * B.wz));
        if (k1 < B.nbz - 1) dmin = fmin(dmin, (B.z0 + (k1 + 1) * B.wz) - sz);
        dmin = fmax(dmin - B.margin, 0.0);
        if (dmin * dmin >= 4.0 * r2) break;  // every unsearched site is at least 2R away
    }
    double cc[3] = {0.0, 0.0, 0.0};
    const int st = cell_moments(c, vol, cc);
    cen[0] = sx + cc[0];
    cen[1] = sy + cc[1];
    cen[2] = sz + cc[2];
    return st;
}

// One thread per kept site (in search-bin order).
__global__ void __launch_bounds__(128) k_voronoi_cells(int64_t n_kept, SiteBins B, VoroBlocks V, double eps,
                                                       double* __restrict__ cen, double* __restrict__ vol,
                                                       int* __restrict__ status) {
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n_kept) return;
    Cell c;
    double cc[3] = {0.0, 0.0, 0.0}, vv = 0.0;
    const int st = build_cell(c, B, V, q, eps, cc, &vv);
    const int64_t o = B.sidx[q];
    cen[3 * o] = cc[0];
    cen[3 * o + 1] = cc[1];
    cen[3 * o + 2] = cc[2];
    vol[o] = vv;
    status[o] = st;
}

__global__ void k_block_keys(int64_t n, const double* __restrict__ xyz, VoroBlocks V, uint32_t* __restrict__ keys,
                             uint32_t* __restrict__ vals) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t b = voro_block(V, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    keys[i] = b < 0 ? 0xffffffffu : (uint32_t)b;
    vals[i] = (uint32_t)i;
}

// keep[w] = 1 for the w-th site of the walk order whose cell was built
__global__ void k_walk_flags(int64_t n, const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                             const int* __restrict__ status, uint32_t* __restrict__ keep) {
    const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= n) return;
    keep[w] = (keys[w] != 0xffffffffu && status[vals[w]] == kCellOk) ? 1u : 0u;
}

__global__ void k_walk_emit(int64_t n, const uint32_t* __restrict__ vals, const uint32_t* __restrict__ keep,
                            const int64_t* __restrict__ offs, const double* __restrict__ cen,
                            const double* __restrict__ vol, const int32_t* __restrict__ ids, int64_t np,
                            double* __restrict__ oxyz, double* __restrict__ ovol, int32_t* __restrict__ oid) {
    const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= n || !keep[w]) return;
    const int64_t s = vals[w], o = offs[w];
    if (o >= np) return;
    oxyz[3 * o] = cen[3 * s];
    oxyz[3 * o + 1] = cen[3 * s + 1];
    oxyz[3 * o + 2] = cen[3 * s + 2];
    ovol[o] = vol[s];
    oid[o] = ids ? ids[s] : (int32_t)s;
}

}  // namespace

extern "C" int kiwi_lloyd_step(KiwiCtx* ctx, int64_t n, const int32_t* ids, const double* xyz, const double* bounds6,
                               double block_scale_factor, int32_t* out_id, double* out_xyz, double* out_volume,
                               int64_t* n_out, int64_t* n_failed, KiwiStats* stats) {
    if (!ctx) return KIWI_ERR_ARG;
    KIWI_CUDA(ctx, cudaSetDevice(ctx->device));
    if (!n_out || !out_id || !out_xyz) return set_err(ctx, KIWI_ERR_ARG, "lloyd step: a null output");
    if (n < 0 || (n > 0 && !xyz)) return set_err(ctx, KIWI_ERR_ARG, "lloyd step: bad site arrays");
    if (n >= (1LL << 31)) return set_err(ctx, KIWI_ERR_ARG, "lloyd step: too many sites");
    if (!bounds6 || !(bounds6[0] < bounds6[1]) || !(bounds6[2] < bounds6[3]) || !(bounds6[4] < bounds6[5]))
        return set_err(ctx, KIWI_ERR_ARG, "domain bounds must satisfy min < max on every axis");
    if (block_scale_factor == 0.0) block_scale_factor = 3.0;
    if (!(block_scale_factor > 0.0)) return set_err(ctx, KIWI_ERR_ARG, "grid_blocks.block_scale_factor must be > 0");
    const int64_t launches0 = ctx->launches;
    const VoroBlocks V = voro_blocks_for(bounds6, n, xyz, block_scale_factor);
    if ((double)V.nx * V.ny * V.nz >= 4294967295.0) return set_err(ctx, KIWI_ERR_LIMIT, "lloyd step: too many blocks");
    int64_t n_kept = 0;
    for (int64_t i = 0; i < n; ++i) n_kept += voro_block(V, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]) >= 0;
    SiteBins B;
    site_bins_shape(bounds6, n_kept, B);
    const int64_t nbins = (int64_t)B.nbx * B.nby * B.nbz;
    const int64_t ns = std::max<int64_t>(n, 1);
    double* d = nullptr;    // xyz (3), sorted xyz (3), centroids (3), volumes (1)
    int32_t* di = nullptr;  // ids, sorted index, status
    int64_t* range = nullptr;
    KIWI_TRY(scratch_t(ctx, S_PART, (size_t)(10 * ns), &d));
    KIWI_TRY(scratch_t(ctx, S_VOR_HOME, (size_t)(3 * ns), &di));
    KIWI_TRY(scratch_t(ctx, S_TILE_RANGE, (size_t)(2 * nbins), &range));
    KIWI_CUDA(ctx, cudaEventRecord(ctx->ev[2], ctx->stream));
    if (n > 0) {
        KIWI_CUDA(ctx, cudaMemcpyAsync(d, xyz, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, ctx->stream));
        if (ids) KIWI_CUDA(ctx, cudaMemcpyAsync(di, ids, sizeof(int32_t) * n, cudaMemcpyHostToDevice, ctx->stream));
    }
    double* cen = d + 6 * ns;
    double* vol = d + 9 * ns;
    int* status = di + 2 * ns;
    KIWI_CUDA(ctx, cudaMemsetAsync(status, 0xff, sizeof(int) * ns, ctx->stream));
    KIWI_CUDA(ctx, cudaEventRecord(ctx->ev[0], ctx->stream));
    KIWI_TRY(build_site_bins(ctx, n, d, V, B, d + 3 * ns, di + ns, range));
    // the clip test's tolerance: 1e-12 of the domain's size, as a distance (the test's value is n . v - d with
    // |n| = the neighbour distance)
    const double ext = std::max(bounds6[1] - bounds6[0], std::max(bounds6[3] - bounds6[2], bounds6[5] - bounds6[4]));
    if (n_kept > 0) {
        k_voronoi_cells<<<(unsigned)((n_kept + 127) / 128), 128, 0, ctx->stream>>>(n_kept, B, V, 1e-12 * ext, cen, vol,
                                                                                    status);
        KIWI_LAUNCHED(ctx);
    }
    // the container's walk order: stable sort by block
    uint32_t *k0, *v0, *k1, *v1, *keep;
    int64_t* offs = nullptr;
    KIWI_TRY(scratch_t(ctx, S_KEYS0, (size_t)ns, &k0));
    KIWI_TRY(scratch_t(ctx, S_VALS0, (size_t)ns, &v0));
    KIWI_TRY(scratch_t(ctx, S_KEYS1, (size_t)ns, &k1));
    KIWI_TRY(scratch_t(ctx, S_VALS1, (size_t)ns, &v1));
    KIWI_TRY(scratch_t(ctx, S_COUNT, (size_t)ns, &keep));
    KIWI_TRY(scratch_t(ctx, S_OFFS, (size_t)ns + 1, &offs));
    int64_t produced = 0;
    if (n > 0) {
        const unsigned g = (unsigned)((n + 255) / 256);
        k_block_keys<<<g, 256, 0, ctx->stream>>>(n, d, V, k0, v0);
        KIWI_LAUNCHED(ctx);
        bool second = false;
        KIWI_TRY(radix_sort_pairs(ctx, k0, v0, k1, v1, n, 32, &second));
        const uint32_t* sk = second ? k1 : k0;
        const uint32_t* sv = second ? v1 : v0;
        k_walk_flags<<<g, 256, 0, ctx->stream>>>(n, sk, sv, status, keep);
        KIWI_LAUNCHED(ctx);
        KIWI_TRY(exclusive_scan<uint32_t>(ctx, keep, n, offs, offs + n));
        KIWI_CUDA(ctx, cudaMemcpyAsync(&produced, offs + n, sizeof produced, cudaMemcpyDeviceToHost, ctx->stream));
        KIWI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        double* o = nullptr;
        int32_t* oi = nullptr;
        const int64_t np = std::max<int64_t>(produced, 1);
        KIWI_TRY(scratch_t(ctx, S_OUT, (size_t)(4 * np), &o));
        KIWI_TRY(scratch_t(ctx, S_MISC2, (size_t)np, &oi));
        k_walk_emit<<<g, 256, 0, ctx->stream>>>(n, sv, keep, offs, cen, vol, ids ? di : nullptr, np, o, o + 3 * np, oi);
        KIWI_LAUNCHED(ctx);
        KIWI_CUDA(ctx, cudaEventRecord(ctx->ev[1], ctx->stream));
        if (produced > 0) {
            KIWI_CUDA(ctx, cudaMemcpyAsync(out_xyz, o, sizeof(double) * 3 * produced, cudaMemcpyDeviceToHost, ctx->stream));
            KIWI_CUDA(ctx, cudaMemcpyAsync(out_id, oi, sizeof(int32_t) * produced, cudaMemcpyDeviceToHost, ctx->stream));
            if (out_volume)
                KIWI_CUDA(ctx, cudaMemcpyAsync(out_volume, o + 3 * np, sizeof(double) * produced, cudaMemcpyDeviceToHost,
                                               ctx->stream));
        }
    } else {
        KIWI_CUDA(ctx, cudaEventRecord(ctx->ev[1], ctx->stream));
    }
    KIWI_CUDA(ctx, cudaEventRecord(ctx->ev[3], ctx->stream));
    KIWI_CUDA(ctx, cudaEventSynchronize(ctx->ev[3]));
    *n_out = produced;
    if (n_failed) *n_failed = n_kept - produced;
    if (stats) {
        *stats = KiwiStats{};
        float ms = 0.f, tot = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
        cudaEventElapsedTime(&tot, ctx->ev[2], ctx->ev[3]);
        stats->gather_ms = ms;
        stats->total_ms = tot;
        stats->evaluated_pairs = n_kept;
        stats->skipped_outside = n - n_kept;
        stats->launches = ctx->launches - launches0;
    }
    return KIWI_OK;
}
