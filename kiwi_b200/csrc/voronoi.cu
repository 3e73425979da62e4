// Voronoi-cell mapping: the particle loop of run_mapping_stage (src/mapping.cpp:400-502) on the GPU.
//
//  (1) k_vor_bfs, one warp per particle (persistent, particles pulled from a counter): the breadth-first
//      walk of src/mapping.cpp:441-460 over the cell-neighbour graph from the particle's home cell, in
//      the reference's queue order, entering a neighbour when the shared face's closest point lies within
//      the support radius (face_reachable: the out_vert rule of src/kernel_integral.cpp:636-645 and
//      src/mapping.cpp:187-193).  It needs no integrals.  Run twice: first it counts each particle's
//      visited cells, then it writes them (in walk order) at the particle's offset with, per visited
//      cell, which of its faces lead to a cell the walk processed earlier.
//  (2) a stable radix sort of the pairs by cell index: every cell's particles stay in ascending order.
//  (3) k_vor_gather, one CTA per cell: the cell's faces are staged in shared memory, each thread takes
//      one particle of the cell's list and evaluates compute_cell_integral (src/mapping.cpp:105-206): the
//      sum over the cell's faces of the face walk, clamped at 0; the values are then added in particle
//      order -- the reference's single-threaded summation order, no atomics -- and finalised as
//      src/mapping.cpp:482-502 does.
// The reference keeps a per-particle cache of face values keyed by the pair of cells (src/mapping.cpp:
// 56-93): a face towards a cell the walk processed earlier takes that cell's value of their shared face,
// negated.  Voro++ computes each cell separately, so the two sides' vertices of a shared face can differ
// (by ~1e-8 in near-degenerate spots), and the side the cache picks shows in the result; the gather
// therefore takes the same side.
#include <cuda_runtime.h>

#include <algorithm>

#include "../../include/kiwi_b200.h"
#include "engine.hpp"
#include "kiwi_math.cuh"
#include "lattice.cuh"
#include "prims.cuh"
#include "tabulated.cuh"

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
    // per face f of cell c towards a cell nb (k_face_links): twin[f] the local index of c's first face
    // before f towards nb, or -1; back[f] the index of nb's first face towards c, or -1 (both -1 when nb
    // is no cell)
    const int32_t* twin;
    const int64_t* back;
};

// The face links of every cell (one thread per cell): what the walk and the gathers would otherwise look
// up by scanning a cell's faces for every (particle, face).
__global__ void k_face_links(int64_t n_cells, const int64_t* __restrict__ face_off,
                             const int32_t* __restrict__ face_nbr, int32_t* __restrict__ twin,
                             int64_t* __restrict__ back) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_cells) return;
    const int64_t f0 = face_off[c], f1 = face_off[c + 1];
    for (int64_t f = f0; f < f1; ++f) {
        const int32_t nb = face_nbr[f];
        int32_t tw = -1;
        int64_t bk = -1;
        if (nb >= 0 && nb < n_cells) {
            for (int64_t e = f0; e < f; ++e)
                if (face_nbr[e] == nb) {
                    tw = (int32_t)(e - f0);
                    break;
                }
            for (int64_t g = face_off[nb]; g < face_off[nb + 1]; ++g)
                if (face_nbr[g] == (int32_t)c) {
                    bk = g;
                    break;
                }
        }
        twin[f] = tw;
        back[f] = bk;
    }
}

constexpr int kBfsWarpsPerBlock = 4;
constexpr int kBfsCandCap = 512;  // a batch's discovery candidates listed per warp (larger batches: lane 0)
constexpr int kGatherThreads = 128;
constexpr int kGatherVertCap = 1536;  // vertices staged in shared memory per cell (36 KB)
// k_vor_faces: a face item packs (pair slot << 7 | face), for cells of at most 128 faces
constexpr int kFaceItemMaxFaces = 128;
constexpr int kFaceItemCap = 2048;  // 4 KB of items beside the 36 KB of staged vertices
// k_vor_faces: CTAs per SM the register allocation leaves room for (4: 128 registers a thread, a few
// spilled; 8 % faster than 3 CTAs at 166 registers)
#ifndef KIWI_VOR_FACES_MIN_BLOCKS
#define KIWI_VOR_FACES_MIN_BLOCKS 4
#endif

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// marker value of particle p in pass `pass` (0, 1 or 2): distinct for every (particle, pass), never -1
__device__ __forceinline__ int marker(int64_t p, int pass) { return (int)(3 * p + pass); }

// The single walk's staging area (pass 2): each particle's pairs and face sources, at places reserved in
// walk-completion order with two atomic counters; k_vor_remap then lays them out particle by particle.
struct VorStage {
    unsigned long long* ctr;  // [0] pairs reserved, [1] faces reserved, [2] overflow
    int64_t cap_pairs, cap_faces;
    int32_t* cells;
    unsigned long long* mask;
    int64_t* floc;   // the pair's first face, relative to its particle's first face
    int32_t* fsrc;
    int64_t* start;  // per particle: its first pair and its first face in the staging area
    int64_t* fstart;
};

// One warp per particle: the particle's BFS over the cell graph in the reference's order
// (src/mapping.cpp:441-460): cells are processed first in, first out; a processed cell's faces are taken
// in order, and each unvisited neighbour whose face the kernel reaches is appended.  The lanes process 32
// queued cells at a time and the appends are made in (cell, face) order, so the queue is the reference's
// sequential queue.  A face whose neighbour already appeared on an earlier face of the same cell is a
// face-cache hit in the reference and discovers nothing.  mark[cell] = (marker << 32) | queue position.
// Cells of more than 128 faces are refused (KIWI_ERR_LIMIT).
// Pass 1 also records per (particle, cell) the faces whose neighbour the walk processed earlier (bit i:
// face i of the cell, first 64 faces): the reference reuses that neighbour's cached, negated face value.
// With face tables (fcounts in pass 0; foffs, pair_foff, fsrc in pass 1), pass 0 also counts the faces of
// each particle's visited cells, and pass 1 gives every (pair, face) its place in the face tables
// (pair_foff: the pair's first face, the particle's cells back to back in walk order) and its source
// (fsrc): -1 the face is evaluated for this pair; q >= 0 it takes, negated, the value of the neighbour's
// first face towards this cell, the neighbour being the particle's q-th visited cell; -2 - e it takes the
// value of this cell's earlier face e towards the same neighbour -- the reference's face cache
// (src/mapping.cpp:56-93), decided here once so that the map evaluates each face value once.
__global__ void __launch_bounds__(32 * kBfsWarpsPerBlock) k_vor_bfs(VorCells C, DevParticles P,
                                                                    const int32_t* __restrict__ home,
                                                                    double support_in_h, int pass,
                                                                    unsigned long long* __restrict__ next,
                                                                    long long* __restrict__ mark_base,
                                                                    int32_t* __restrict__ queue_base,
                                                                    int64_t* __restrict__ counts,
                                                                    const int64_t* __restrict__ offs,
                                                                    int32_t* __restrict__ pair_cells,
                                                                    unsigned long long* __restrict__ pair_mask,
                                                                    DevStats* __restrict__ st,
                                                                    int64_t* __restrict__ fcounts,
                                                                    const int64_t* __restrict__ foffs,
                                                                    int64_t* __restrict__ pair_foff,
                                                                    int32_t* __restrict__ fsrc, VorStage stg) {
    __shared__ int32_t s_cand[kBfsWarpsPerBlock][kBfsCandCap];
    __shared__ unsigned long long s_reach[kBfsWarpsPerBlock][32][2];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t slot = (int64_t)blockIdx.x * kBfsWarpsPerBlock + warp;
    long long* mark = mark_base + slot * C.n_cells;
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
                if (pass != 1) counts[p] = 0;
                if (pass != 1 && fcounts) fcounts[p] = 0;
                if (h > 0.0) ++n_unresolved;
            }
            continue;
        }
        const double x0 = P.x[p], y0 = P.y[p], z0 = P.z[p];
        const double radius = mul_rn(support_in_h, h);
        const long long mk = marker((int64_t)p, pass);
        const int64_t o = (pass == 1) ? offs[p] : 0;
        if (lane == 0) {
            queue[0] = k0;
            mark[k0] = mk << 32;
        }
        __syncwarp();
        int head = 0, tail = 1;
        int64_t nface = 0;                                  // pass 0: this lane's share of the face count
        int64_t fcarry = (pass == 1 && fsrc) ? foffs[p] : 0;  // pass 1: the next cell's first face
        while (head < tail) {
            if (head > C.n_cells) {  // cannot happen: each cell enters the queue once
                n_limit += (lane == 0);
                break;
            }
            // The lanes take the next (up to) 32 queued cells, one each, and mark the faces to test: faces
            // towards a neighbour not yet in the queue, skipping a face whose neighbour an earlier face of
            // the same cell already named (a face-cache hit in the reference, which discovers nothing).  The
            // warp tests them (the kernel reaches the face or not); the reachable ones are the discovery
            // candidates, appended in (cell, face) order, skipping neighbours queued meanwhile: the
            // reference's sequential queue.
            const int batch = min(32, tail - head);
            int64_t fa = 0, nf = 0;
            unsigned long long cand0 = 0, cand1 = 0, earlier = 0, test0 = 0, test1 = 0;
            if (lane < batch) {
                const int rank = head + lane;
                const int32_t cell = queue[rank];
                fa = C.face_off[cell];
                const int64_t fz = C.face_off[cell + 1];
                nf = fz - fa;
                nface += nf;
                if (fz - fa > 128) n_limit += 1;  // a cell of more than 128 faces is not supported
                for (int64_t f = fa; f < fz && f - fa < 128; ++f) {
                    const int32_t nb = C.face_nbr[f];
                    if (nb < 0 || nb >= C.n_cells) continue;
                    const long long mv = mark[nb];
                    const bool seen = (mv >> 32) == mk;
                    if (seen) {
                        if ((int)(mv & 0xffffffffLL) < rank && f - fa < 64) earlier |= 1ull << (f - fa);
                        continue;
                    }
                    if (C.twin[f] >= 0) continue;  // an earlier face of this cell named nb already
                    if (f - fa < 64) test0 |= 1ull << (f - fa);
                    else test1 |= 1ull << (f - fa - 64);
                }
                if (pass == 1) {
                    pair_cells[o + rank] = cell;
                    pair_mask[o + rank] = earlier;
                }
            }
            {
                // The faces left to test (neighbour not queued, not a twin) as one list over the warp, in
                // (cell, face) order, each lane testing every 32nd: a lane's own cell would leave the others
                // idle through its faces, and the early batches hold one cell or a few.  A batch of more
                // tests than the list holds is tested lane by lane.
                const int nt_l = __popcll(test0) + __popcll(test1);
                int t_incl = nt_l;
                for (int d = 1; d < 32; d <<= 1) {
                    const int v = __shfl_up_sync(0xffffffffu, t_incl, d);
                    if (lane >= d) t_incl += v;
                }
                const int n_test = __shfl_sync(0xffffffffu, t_incl, 31);
                if (n_test <= kBfsCandCap) {
                    int32_t* items = s_cand[warp];
                    int o_t = t_incl - nt_l;
                    for (int w = 0; w < 2; ++w) {
                        unsigned long long bits = w == 0 ? test0 : test1;
                        while (bits) {
                            const int b = __ffsll((long long)bits) - 1;
                            bits &= bits - 1;
                            items[o_t++] = lane << 7 | (64 * w + b);
                        }
                    }
                    s_reach[warp][lane][0] = 0;
                    s_reach[warp][lane][1] = 0;
                    __syncwarp();
                    for (int base = 0; base < n_test; base += 32) {
                        const int i = base + lane;
                        const int item = i < n_test ? items[i] : 0;
                        const int src = item >> 7, fl = item & 127;
                        const int64_t f = __shfl_sync(0xffffffffu, fa, src) + fl;
                        if (i < n_test) {
                            const FlatVerts V{C.vxyz + 3 * C.vert_off[f]};
                            if (face_reachable(x0, y0, z0, radius, V, (int)(C.vert_off[f + 1] - C.vert_off[f])))
                                atomicOr(&s_reach[warp][src][fl >> 6], 1ull << (fl & 63));
                        }
                    }
                    __syncwarp();
                    cand0 = s_reach[warp][lane][0];
                    cand1 = s_reach[warp][lane][1];
                    __syncwarp();
                } else {
                    for (int w = 0; w < 2; ++w) {
                        unsigned long long bits = w == 0 ? test0 : test1;
                        while (bits) {
                            const int b = __ffsll((long long)bits) - 1;
                            bits &= bits - 1;
                            const int64_t f = fa + 64 * w + b;
                            const FlatVerts V{C.vxyz + 3 * C.vert_off[f]};
                            if (face_reachable(x0, y0, z0, radius, V, (int)(C.vert_off[f + 1] - C.vert_off[f]))) {
                                if (w == 0) cand0 |= 1ull << b;
                                else cand1 |= 1ull << b;
                            }
                        }
                    }
                }
            }
            if (pass == 1 && fsrc) {
                // the cells' places in the face tables (a warp prefix sum in walk order) and each face's source
                int64_t incl = nf;
                for (int d = 1; d < 32; d <<= 1) {
                    const int64_t v = __shfl_up_sync(0xffffffffu, incl, d);
                    if (lane >= d) incl += v;
                }
                if (lane < batch) {
                    const int rank = head + lane;
                    const int64_t pf = fcarry + incl - nf;
                    pair_foff[o + rank] = pf;
                    for (int64_t f = fa; f < fa + nf; ++f) {
                        const int32_t nb = C.face_nbr[f];
                        int32_t code = -1;
                        if (nb >= 0 && nb < C.n_cells) {
                            const long long mv = mark[nb];
                            if ((mv >> 32) == mk && (int)(mv & 0xffffffffLL) < rank && C.back[f] >= 0)
                                code = (int32_t)(mv & 0xffffffffLL);
                            if (code < 0 && C.twin[f] >= 0) code = -2 - C.twin[f];
                        }
                        fsrc[pf + (f - fa)] = code;
                    }
                }
                fcarry += __shfl_sync(0xffffffffu, incl, 31);
            }
            int t = tail;
            // the batch's candidates in (cell, face) order; each is queued if no earlier candidate names the
            // same cell and it is not queued yet -- the sequential appends' queue, with every lane at work
            const int nc_l = __popcll(cand0) + __popcll(cand1);
            int c_incl = nc_l;
            for (int d = 1; d < 32; d <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, c_incl, d);
                if (lane >= d) c_incl += v;
            }
            const int n_cand = __shfl_sync(0xffffffffu, c_incl, 31);
            if (n_cand <= kBfsCandCap) {
                int32_t* cl = s_cand[warp];
                int o = c_incl - nc_l;
                for (int w = 0; w < 2; ++w) {
                    unsigned long long bits = w == 0 ? cand0 : cand1;
                    while (bits) {
                        const int b = __ffsll((long long)bits) - 1;
                        bits &= bits - 1;
                        cl[o++] = C.face_nbr[fa + 64 * w + b];
                    }
                }
                __syncwarp();
                for (int base = 0; base < n_cand; base += 32) {
                    const int i = base + lane;
                    int32_t nb = -1;
                    bool keep = false;
                    if (i < n_cand) {
                        nb = cl[i];
                        keep = (mark[nb] >> 32) != mk;
                        for (int j = 0; keep && j < i; ++j) keep = cl[j] != nb;
                    }
                    const unsigned kb = __ballot_sync(0xffffffffu, keep);
                    if (keep) {
                        const int pos = t + __popc(kb & ((1u << lane) - 1));
                        mark[nb] = (mk << 32) | (long long)pos;
                        queue[pos] = nb;
                    }
                    t += __popc(kb);
                }
                __syncwarp();
            } else {
            for (int L = 0; L < batch; ++L) {
                unsigned long long c0 = __shfl_sync(0xffffffffu, cand0, L);
                unsigned long long c1 = __shfl_sync(0xffffffffu, cand1, L);
                const int64_t fl = __shfl_sync(0xffffffffu, fa, L);
                if (lane == 0) {
                    for (int w = 0; w < 2; ++w) {
                        unsigned long long bits = w == 0 ? c0 : c1;
                        while (bits) {
                            const int b = __ffsll((long long)bits) - 1;
                            bits &= bits - 1;
                            const int32_t nb = C.face_nbr[fl + 64 * w + b];
                            if ((mark[nb] >> 32) != mk) {
                                mark[nb] = (mk << 32) | (long long)t;
                                queue[t++] = nb;
                            }
                        }
                    }
                }
            }
            }
            tail = __shfl_sync(0xffffffffu, t, 0);
            head += batch;
            __syncwarp();
        }
        if (pass != 1 && fcounts) {
            for (int d = 16; d > 0; d >>= 1) nface += __shfl_down_sync(0xffffffffu, nface, d);
            nface = __shfl_sync(0xffffffffu, nface, 0);
            if (lane == 0) fcounts[p] = nface;
        }
        if (pass != 1 && lane == 0) {
            counts[p] = tail;
            if (tail == 1) ++n_unmapped;
        }
        if (pass == 2) {
            // the single walk: reserve this particle's pairs and faces, then write them.  The marks hold
            // every visited cell's queue position, so each face's source is decided as pass 1 decides it
            // during its walk (a neighbour processed earlier is one with a smaller queue position).
            unsigned long long s0 = 0, fs0 = 0;
            if (lane == 0) {
                s0 = atomicAdd(&stg.ctr[0], (unsigned long long)tail);
                fs0 = atomicAdd(&stg.ctr[1], (unsigned long long)nface);
            }
            s0 = __shfl_sync(0xffffffffu, s0, 0);
            fs0 = __shfl_sync(0xffffffffu, fs0, 0);
            if (s0 + tail > (unsigned long long)stg.cap_pairs || fs0 + nface > (unsigned long long)stg.cap_faces) {
                if (lane == 0) atomicOr(&stg.ctr[2], 1ull);
            } else {
                if (lane == 0) {
                    stg.start[p] = (int64_t)s0;
                    stg.fstart[p] = (int64_t)fs0;
                }
                int64_t fc = 0;
                for (int base = 0; base < tail; base += 32) {
                    const int r = base + lane;
                    int32_t cell = 0;
                    int64_t fa = 0, nf = 0;
                    if (r < tail) {
                        cell = queue[r];
                        fa = C.face_off[cell];
                        nf = C.face_off[cell + 1] - fa;
                    }
                    int64_t incl = nf;
                    for (int d = 1; d < 32; d <<= 1) {
                        const int64_t v = __shfl_up_sync(0xffffffffu, incl, d);
                        if (lane >= d) incl += v;
                    }
                    if (r < tail) {
                        const int64_t fl = fc + incl - nf;
                        unsigned long long earlier = 0;
                        for (int64_t f = fa; f < fa + nf; ++f) {
                            const int32_t nb = C.face_nbr[f];
                            int32_t code = -1;
                            if (nb >= 0 && nb < C.n_cells) {
                                const long long mv = mark[nb];
                                const bool before = (mv >> 32) == mk && (int)(mv & 0xffffffffLL) < r;
                                if (before && f - fa < 64) earlier |= 1ull << (f - fa);
                                if (before && C.back[f] >= 0) code = (int32_t)(mv & 0xffffffffLL);
                                if (code < 0 && C.twin[f] >= 0) code = -2 - C.twin[f];
                            }
                            stg.fsrc[fs0 + fl + (f - fa)] = code;
                        }
                        stg.cells[s0 + r] = cell;
                        stg.mask[s0 + r] = earlier;
                        stg.floc[s0 + r] = fl;
                    }
                    fc += __shfl_sync(0xffffffffu, incl, 31);
                }
            }
        }
        __syncwarp();
    }
    n_unresolved = warp_sum_u64(n_unresolved);
    n_unmapped = warp_sum_u64(n_unmapped);
    n_limit = warp_sum_u64(n_limit);
    if (lane == 0 && pass != 1) {
        if (n_unresolved) atomicAdd(&st->skipped_outside, n_unresolved);
        if (n_unmapped) atomicAdd(&st->tile_pairs, n_unmapped);  // reported as "unmapped" by the caller
    }
    if (lane == 0 && n_limit) atomicAdd(&st->limit_hit, n_limit);
}

// The single walk's staging area laid out particle by particle (one warp per particle): the same arrays as
// the two-pass walk writes -- pair_cells, pair_mask, pair_foff at offs[p], the face sources at foffs[p].
__global__ void k_vor_remap(int64_t n, VorStage stg, const int64_t* __restrict__ counts,
                            const int64_t* __restrict__ fcounts, const int64_t* __restrict__ offs,
                            const int64_t* __restrict__ foffs, int32_t* __restrict__ pair_cells,
                            unsigned long long* __restrict__ pair_mask, int64_t* __restrict__ pair_foff,
                            int32_t* __restrict__ fsrc) {
    const int64_t p = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (p >= n) return;
    const int64_t cnt = counts[p], fcnt = fcounts[p];
    if (cnt == 0) return;
    const int64_t s0 = stg.start[p], d0 = offs[p], fs0 = stg.fstart[p], fd0 = foffs[p];
    for (int64_t r = lane; r < cnt; r += 32) {
        pair_cells[d0 + r] = stg.cells[s0 + r];
        pair_mask[d0 + r] = stg.mask[s0 + r];
        if (pair_foff) pair_foff[d0 + r] = fd0 + stg.floc[s0 + r];
    }
    if (fsrc)
        for (int64_t q = lane; q < fcnt; q += 32) fsrc[fd0 + q] = stg.fsrc[fs0 + q];
}

// pair k (particle p's visited cells in BFS order, at offs[p]) -> (key = cell, value = k)
__global__ void k_vor_pairs(const int32_t* __restrict__ pair_cells, int64_t total, uint32_t* __restrict__ keys,
                            uint32_t* __restrict__ vals) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= total) return;
    keys[k] = (uint32_t)pair_cells[k];
    vals[k] = (uint32_t)k;
}

// The particle of pair k: the last p with offs[p] <= k.
__device__ __forceinline__ int64_t pair_particle(const int64_t* __restrict__ offs, int64_t n, int64_t k) {
    int64_t lo = 0, hi = n - 1;
    while (lo < hi) {
        const int64_t mid = (lo + hi + 1) >> 1;
        if (offs[mid] <= k) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// One face's integral for one particle (the face walk with the kernel's evaluator).  MODE: kVorGeneric,
// kVorCubic (closed form) or kVorTab (lookups in tab; clamped indices counted in *nclamp).
constexpr int kVorGeneric = 0, kVorCubic = 1, kVorTab = 2;
template <int MODE>
static __device__ __noinline__ double vor_face(const double* verts, int nv, double x0, double y0, double z0, double h,
                                               double radius, int kernel, const TabDev& tab, unsigned* nclamp) {
    const FlatVerts V{verts};
    if (MODE == kVorTab) {
        TabEval ev{tab, h, 0.0, 0.0, nclamp};
        return face_integral(x0, y0, z0, 2 * h, V, nv, (int*)nullptr, ev);
    }
    if (MODE == kVorCubic) {
        LenCubicEval ev;
        ev.h = h;
        ev.ih = 1.0 / h;
        return face_integral(x0, y0, z0, 2 * h, V, nv, (int*)nullptr, ev);
    }
    GenericEval ev;
    ev.K = &c_vor_tables[kernel];
    ev.H = radius;
    return face_integral(x0, y0, z0, radius, V, nv, (int*)nullptr, ev);
}

__global__ void k_cell_ranges(const uint32_t* __restrict__ keys, int64_t total, int64_t* __restrict__ range) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const uint32_t k = keys[i];
    if (i == 0 || keys[i - 1] != k) range[2 * (int64_t)k] = i;
    if (i == total - 1 || keys[i + 1] != k) range[2 * (int64_t)k + 1] = i + 1;
}

template <int MODE>
__global__ void __launch_bounds__(kGatherThreads) k_vor_gather(VorCells C, DevParticles P, int kernel,
                                                                double support_in_h, const TabDev tab,
                                                                const uint32_t* __restrict__ plist,
                                                                const int64_t* __restrict__ range,
                                                                const int64_t* __restrict__ offs,
                                                                const int32_t* __restrict__ pair_cells,
                                                                const unsigned long long* __restrict__ pair_mask,
                                                                CartOutputs out, DevStats* __restrict__ st,
                                                                double* __restrict__ pair_val) {
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
    unsigned n_clamp = 0;
    for (int64_t base = beg; base < end; base += kGatherThreads) {
        const int64_t k = base + threadIdx.x;
        double msum = 0.0;
        if (k < end) {
            const int64_t pk = plist[k];
            const int64_t p = pair_particle(offs, P.n, pk);
            const int64_t seg = offs[p], rank = pk - seg;
            const unsigned long long mask = pair_mask[pk];
            const double x0 = P.x[p], y0 = P.y[p], z0 = P.z[p], h = P.h[p];
            const double radius = mul_rn(support_in_h, h);
            // compute_cell_integral (src/mapping.cpp:105-206) with its per-particle face cache: a face whose
            // neighbour this particle's walk processed earlier takes the neighbour's value of their shared
            // face, negated; a second face towards the same neighbour takes the first one's value; every
            // other face is evaluated here.  (The two sides' copies of a face can differ in their vertices,
            // so the choice shows in the result.)
#pragma unroll 1
            for (int64_t f = f0; f < f1; ++f) {
                const int32_t nb = C.face_nbr[f];
                int64_t src = f;  // the face whose value this face contributes
                double sign = 1.0;
                if (nb >= 0 && nb < C.n_cells) {
                    bool before;
                    if (f - f0 < 64) {
                        before = (mask >> (f - f0)) & 1ull;
                    } else {
                        before = false;
                        for (int64_t q = 0; q < rank; ++q)
                            if (pair_cells[seg + q] == nb) {
                                before = true;
                                break;
                            }
                    }
                    const int64_t g = before ? C.back[f] : -1;
                    if (g >= 0) {
                        src = g;
                        sign = -1.0;
                    } else if (C.twin[f] >= 0) {
                        src = f0 + C.twin[f];
                    }
                }
                const int nv = (int)(C.vert_off[src + 1] - C.vert_off[src]);
                const double* verts = (src >= f0 && src < f1 && staged) ? s_v + 3 * (C.vert_off[src] - v0)
                                                                         : C.vxyz + 3 * C.vert_off[src];
                const double val = vor_face<MODE>(verts, nv, x0, y0, z0, h, radius, kernel, tab, &n_clamp);
                if (sign < 0.0) msum -= val; else msum += val;
            }
            if (msum < 0.0) {
                ++n_neg;
                if (msum <= -0.01) ++n_warn;
                msum = 0.0;
            }
            if (pair_val) pair_val[pk] = msum;
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
    const unsigned long long n_cl = warp_sum_u64(n_clamp);
    if ((threadIdx.x & 31) == 0) {
        if (n_neg) atomicAdd(&st->neg_clamped, n_neg);
        if (n_warn) atomicAdd(&st->neg_warned, n_warn);
        if (n_cl) atomicAdd(&st->table_clamps, n_cl);
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

// The face-table form of k_vor_gather, in two launches.  (a) k_vor_faces, one CTA per cell: each of the
// cell's pairs evaluates the faces whose source is the pair itself (fsrc = -1) and stores their values.
// (b) k_vor_sum, one CTA per cell: each pair adds its faces' values from the tables -- its own, an earlier
// face's of its own cell, or the neighbour pair's value negated -- in face order, clamps at 0 and the
// cell's pairs are added in particle order: the same operations on the same values as k_vor_gather, with
// every face value evaluated once per particle instead of once per side.
template <int MODE>
__global__ void __launch_bounds__(kGatherThreads, KIWI_VOR_FACES_MIN_BLOCKS)
    k_vor_faces(VorCells C, DevParticles P, int kernel, double support_in_h, const TabDev tab,
                const uint32_t* __restrict__ plist, const int64_t* __restrict__ range,
                const int64_t* __restrict__ pair_foff, const int32_t* __restrict__ fsrc,
                const int64_t* __restrict__ offs, double* __restrict__ fval, DevStats* __restrict__ st) {
    __shared__ double s_v[3 * kGatherVertCap];
    const int64_t cell = blockIdx.x;
    const int64_t f0 = C.face_off[cell], f1 = C.face_off[cell + 1];
    const int64_t v0 = C.vert_off[f0], v1 = C.vert_off[f1];
    const bool staged = (v1 - v0) <= kGatherVertCap;
    if (staged)
        for (int64_t i = threadIdx.x; i < 3 * (v1 - v0); i += kGatherThreads) s_v[i] = C.vxyz[3 * v0 + i];
    __syncthreads();
    const int64_t beg = range[2 * cell], end = range[2 * cell + 1];
    const int nf = (int)(f1 - f0);
    unsigned n_clamp = 0;
    if (nf > kFaceItemMaxFaces) {
        // (a cell of more faces than an item packs; the walk refuses such a map afterwards)
        for (int64_t k = beg + threadIdx.x; k < end; k += kGatherThreads) {
            const int64_t pk = plist[k];
            const int64_t p = pair_particle(offs, P.n, pk);
            const double h = P.h[p];
            const int64_t pf = pair_foff[pk];
#pragma unroll 1
            for (int64_t f = f0; f < f1; ++f) {
                if (fsrc[pf + (f - f0)] != -1) continue;
                const int nv = (int)(C.vert_off[f + 1] - C.vert_off[f]);
                fval[pf + (f - f0)] = vor_face<MODE>(C.vxyz + 3 * C.vert_off[f], nv, P.x[p], P.y[p], P.z[p], h,
                                                     mul_rn(support_in_h, h), kernel, tab, &n_clamp);
            }
        }
    } else {
        // The cell's pairs in groups: each thread takes one pair and marks the faces it evaluates itself
        // (its walk did not borrow them); the group's (pair, face) items are listed face by face (a
        // counting sort by face) and evaluated by all threads at once, so that no lane idles through a
        // face another pair evaluates and a warp's lanes walk the same face (same vertex count, same
        // staged vertices) for different particles.  Each value goes to its own place in the tables, so
        // the order within a face's bucket does not matter.
        __shared__ double s_px[kGatherThreads], s_py[kGatherThreads], s_pz[kGatherThreads], s_ph[kGatherThreads];
        __shared__ int64_t s_pf[kGatherThreads];
        __shared__ uint16_t s_items[kFaceItemCap];
        __shared__ int s_fpos[kFaceItemMaxFaces];
        __shared__ int s_total;
        const int group = min(kGatherThreads, kFaceItemCap / max(nf, 1));
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        for (int64_t base = beg; base < end; base += group) {
            for (int f = threadIdx.x; f < nf; f += kGatherThreads) s_fpos[f] = 0;
            __syncthreads();
            const int64_t k = base + threadIdx.x;
            unsigned long long own0 = 0, own1 = 0;  // faces 0..63 and 64..127 this pair evaluates
            if (threadIdx.x < group && k < end) {
                const int64_t pk = plist[k];
                const int64_t p = pair_particle(offs, P.n, pk);
                const int64_t pf = pair_foff[pk];
                s_px[threadIdx.x] = P.x[p];
                s_py[threadIdx.x] = P.y[p];
                s_pz[threadIdx.x] = P.z[p];
                s_ph[threadIdx.x] = P.h[p];
                s_pf[threadIdx.x] = pf;
                for (int f = 0; f < nf; ++f)
                    if (fsrc[pf + f] == -1) {
                        if (f < 64) own0 |= 1ull << f;
                        else own1 |= 1ull << (f - 64);
                        atomicAdd(&s_fpos[f], 1);
                    }
            }
            __syncthreads();
            if (warp == 0) {
                // exclusive scan of the per-face counts (nf <= 128: four faces per lane)
                int c[4], sum = 0;
                for (int q = 0; q < 4; ++q) {
                    const int f = 4 * lane + q;
                    c[q] = f < nf ? s_fpos[f] : 0;
                    sum += c[q];
                }
                int incl = sum;
                for (int d = 1; d < 32; d <<= 1) {
                    const int v = __shfl_up_sync(0xffffffffu, incl, d);
                    if (lane >= d) incl += v;
                }
                int run = incl - sum;
                for (int q = 0; q < 4; ++q) {
                    const int f = 4 * lane + q;
                    if (f < nf) s_fpos[f] = run;
                    run += c[q];
                }
                if (lane == 31) s_total = incl;
            }
            __syncthreads();
            const int total = s_total;
            for (int w = 0; w < 2; ++w) {
                unsigned long long bits = w == 0 ? own0 : own1;
                while (bits) {
                    const int f = 64 * w + __ffsll((long long)bits) - 1;
                    bits &= bits - 1;
                    s_items[atomicAdd(&s_fpos[f], 1)] = (uint16_t)(threadIdx.x << 7 | f);
                }
            }
            __syncthreads();
            for (int it = threadIdx.x; it < total; it += kGatherThreads) {
                const int item = s_items[it];
                const int t = item >> 7, fl = item & 127;
                const int64_t f = f0 + fl;
                const int nv = (int)(C.vert_off[f + 1] - C.vert_off[f]);
                const double* verts = staged ? s_v + 3 * (C.vert_off[f] - v0) : C.vxyz + 3 * C.vert_off[f];
                const double h = s_ph[t];
                fval[s_pf[t] + fl] = vor_face<MODE>(verts, nv, s_px[t], s_py[t], s_pz[t], h,
                                                    mul_rn(support_in_h, h), kernel, tab, &n_clamp);
            }
            __syncthreads();
        }
    }
    const unsigned long long n_cl = warp_sum_u64(n_clamp);
    if ((threadIdx.x & 31) == 0 && n_cl) atomicAdd(&st->table_clamps, n_cl);
}

__global__ void __launch_bounds__(kGatherThreads) k_vor_sum(VorCells C, DevParticles P,
                                                             const uint32_t* __restrict__ plist,
                                                             const int64_t* __restrict__ range,
                                                             const int64_t* __restrict__ offs,
                                                             const int64_t* __restrict__ pair_foff,
                                                             const int32_t* __restrict__ fsrc,
                                                             const double* __restrict__ fval, CartOutputs out,
                                                             DevStats* __restrict__ st, double* __restrict__ pair_val) {
    __shared__ double s_val[kGatherThreads], s_m[kGatherThreads], s_vx[kGatherThreads], s_vy[kGatherThreads],
        s_vz[kGatherThreads];
    const int64_t cell = blockIdx.x;
    const int64_t f0 = C.face_off[cell], f1 = C.face_off[cell + 1];
    const int64_t beg = range[2 * cell], end = range[2 * cell + 1];
    double M = 0.0, Px = 0.0, Py = 0.0, Pz = 0.0;
    unsigned long long n_neg = 0, n_warn = 0;
    for (int64_t base = beg; base < end; base += kGatherThreads) {
        const int64_t k = base + threadIdx.x;
        double msum = 0.0;
        if (k < end) {
            const int64_t pk = plist[k];
            const int64_t p = pair_particle(offs, P.n, pk);
            const int64_t seg = offs[p];
            const int64_t pf = pair_foff[pk];
#pragma unroll 1
            for (int64_t f = f0; f < f1; ++f) {
                const int32_t code = fsrc[pf + (f - f0)];
                if (code >= 0) {
                    // the neighbour's first face towards this cell, from the neighbour's pair
                    const int32_t nb = C.face_nbr[f];
                    msum -= fval[pair_foff[seg + code] + (C.back[f] - C.face_off[nb])];
                } else {
                    msum += fval[pf + (code == -1 ? f - f0 : (int64_t)(-2 - code))];
                }
            }
            if (msum < 0.0) {
                ++n_neg;
                if (msum <= -0.01) ++n_warn;
                msum = 0.0;
            }
            if (pair_val) pair_val[pk] = msum;
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

// m_i = density * volume per cell (the forward map's cell mass, as run_inverse_mapping_test_stage forms
// it from the mapping's rows, src/mapping.cpp:554-561).
__global__ void k_vor_cell_mass(int64_t nc, const double* __restrict__ density, const double* __restrict__ volume,
                                double* __restrict__ cmass) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < nc) cmass[c] = density[c] * volume[c];
}

// Per particle, the inverse-mapping sum over its visited cells in the walk's order
// (src/mapping.cpp:635-661): recovered += (integral m / m_i) m_i for cells with m_i > 0; coverage =
// recovered / m (0 for m <= 0).  Particles without pairs (h <= 0, unresolved home cell) recover 0.
__global__ void k_vor_recover(DevParticles P, const int64_t* __restrict__ offs, const int32_t* __restrict__ pair_cells,
                              const double* __restrict__ pair_val, const double* __restrict__ cmass,
                              double* __restrict__ recovered, double* __restrict__ coverage) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P.n) return;
    const double m = P.m[p];
    double r = 0.0;
    for (int64_t k = offs[p]; k < offs[p + 1]; ++k) {
        const double mi = cmass[pair_cells[k]];
        if (mi > 0.0) r += (pair_val[k] * m / mi) * mi;
    }
    recovered[p] = r;
    coverage[p] = (m > 0.0) ? r / m : 0.0;
}

}  // namespace

int voronoi_map_dev(KiwiCtx* ctx, const DevParticles& P, const int32_t* d_home, const KiwiVoronoiCells& cells,
                    const KernelChoice& kc, const CartOutputs& out_in, KiwiStats* stats, const VorInverse* inv) {
    const int64_t launches0 = ctx->launches;
    const int64_t n = P.n, nc = cells.n_cells;
    VorCells C{nc, cells.face_off, cells.vert_off, cells.vxyz, cells.face_nbr, cells.volume, nullptr, nullptr};
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

    // the faces' links (earlier twin, the neighbour's face back)
    int64_t n_faces = 0;
    KIWI_CUDA(ctx, cudaMemcpyAsync(&n_faces, cells.face_off + nc, sizeof(int64_t), cudaMemcpyDeviceToHost,
                                   ctx->stream));
    KIWI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    unsigned char* links = nullptr;
    const size_t nf_alloc = (size_t)std::max<int64_t>(n_faces, 1);
    KIWI_TRY(scratch_t(ctx, S_VOR_LINKS, nf_alloc * (sizeof(int64_t) + sizeof(int32_t)), &links));
    int64_t* d_back = reinterpret_cast<int64_t*>(links);
    int32_t* d_twin = reinterpret_cast<int32_t*>(links + nf_alloc * sizeof(int64_t));
    k_face_links<<<(unsigned)((nc + 255) / 256), 256, 0, ctx->stream>>>(nc, cells.face_off, cells.face_nbr, d_twin,
                                                                        d_back);
    KIWI_LAUNCHED(ctx);
    C.twin = d_twin;
    C.back = d_back;

    // BFS work slots: a visited marker and a queue of n_cells entries each
    int sms = 0;
    KIWI_CUDA(ctx, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    int64_t slots = (int64_t)sms * 8;
    const int64_t budget = (int64_t)16 << 30;  // bytes of BFS scratch at most
    while (slots > kBfsWarpsPerBlock && slots * nc * 12 > budget) slots /= 2;
    slots = std::max<int64_t>(kBfsWarpsPerBlock, (slots / kBfsWarpsPerBlock) * kBfsWarpsPerBlock);
    const int blocks = (int)(slots / kBfsWarpsPerBlock);
    long long* mark = nullptr;
    int32_t* queue = nullptr;
    int64_t *counts = nullptr, *offs = nullptr, *range = nullptr;
    KIWI_TRY(scratch_t(ctx, S_VOR_MARK, (size_t)(slots * nc), &mark));
    KIWI_TRY(scratch_t(ctx, S_VOR_QUEUE, (size_t)(slots * nc), &queue));
    KIWI_TRY(scratch_t(ctx, S_COUNT, (size_t)std::max<int64_t>(n, 1) * 2, &counts));
    KIWI_TRY(scratch_t(ctx, S_OFFS, (size_t)std::max<int64_t>(n, 1) + 1, &offs));
    KIWI_TRY(scratch_t(ctx, S_TILE_RANGE, (size_t)(2 * nc), &range));
    int64_t* d_total = offs + std::max<int64_t>(n, 1);
    KIWI_CUDA(ctx, cudaMemsetAsync(mark, 0xff, sizeof(long long) * slots * nc, ctx->stream));
    KIWI_CUDA(ctx, cudaMemsetAsync(range, 0, sizeof(int64_t) * 2 * nc, ctx->stream));

    const double sup = kc.support_in_h;
    // pass 0: count the visited cells and their faces
    int64_t *fcounts = nullptr, *foffs = nullptr;
    KIWI_TRY(scratch_t(ctx, S_VOR_FCOUNT, (size_t)std::max<int64_t>(n, 1), &fcounts));
    KIWI_TRY(scratch_t(ctx, S_VOR_FOFFS, (size_t)std::max<int64_t>(n, 1) + 1, &foffs));
    int64_t* d_ftotal = foffs + std::max<int64_t>(n, 1);
    // One walk when an earlier map on this context gave the totals to reserve (with room to spare): each
    // particle's pairs and face sources go to a staging area and are laid out particle by particle after;
    // otherwise (or if the reservation overflows) one walk counts and a second writes.
    VorStage stg{};
    bool single = false;
    if (n > 0 && ctx->face_tables && ctx->vor_pairs_hint > 0) {
        const int64_t cap_p = ctx->vor_pairs_hint + ctx->vor_pairs_hint / 4 + 4096;
        const int64_t cap_f = ctx->vor_faces_hint + ctx->vor_faces_hint / 4 + 65536;
        const size_t bytes = 3 * sizeof(unsigned long long) + 2 * sizeof(int64_t) * (size_t)n +
                             (size_t)cap_p * (sizeof(unsigned long long) + sizeof(int64_t) + sizeof(int32_t)) +
                             (size_t)cap_f * sizeof(int32_t);
        if (bytes <= ((size_t)24 << 30)) {
            unsigned char* blob = nullptr;
            KIWI_TRY(scratch_t(ctx, S_VOR_STAGE, bytes, &blob));
            unsigned char* q = blob;
            stg.ctr = reinterpret_cast<unsigned long long*>(q), q += 3 * sizeof(unsigned long long);
            stg.start = reinterpret_cast<int64_t*>(q), q += sizeof(int64_t) * (size_t)n;
            stg.fstart = reinterpret_cast<int64_t*>(q), q += sizeof(int64_t) * (size_t)n;
            stg.mask = reinterpret_cast<unsigned long long*>(q), q += sizeof(unsigned long long) * (size_t)cap_p;
            stg.floc = reinterpret_cast<int64_t*>(q), q += sizeof(int64_t) * (size_t)cap_p;
            stg.cells = reinterpret_cast<int32_t*>(q), q += sizeof(int32_t) * (size_t)cap_p;
            stg.fsrc = reinterpret_cast<int32_t*>(q);
            stg.cap_pairs = cap_p;
            stg.cap_faces = cap_f;
            KIWI_CUDA(ctx, cudaMemsetAsync(stg.ctr, 0, 3 * sizeof(unsigned long long), ctx->stream));
            KIWI_CUDA(ctx, cudaMemsetAsync(d_next, 0, sizeof(unsigned long long), ctx->stream));
            k_vor_bfs<<<blocks, 32 * kBfsWarpsPerBlock, 0, ctx->stream>>>(C, P, d_home, sup, 2, d_next, mark, queue,
                                                                         counts, nullptr, nullptr, nullptr, d_stats,
                                                                         fcounts, nullptr, nullptr, nullptr, stg);
            KIWI_LAUNCHED(ctx);
            unsigned long long ovf = 0;
            KIWI_CUDA(ctx, cudaMemcpyAsync(&ovf, stg.ctr + 2, sizeof ovf, cudaMemcpyDeviceToHost, ctx->stream));
            KIWI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            single = ovf == 0;
            if (!single) KIWI_CUDA(ctx, cudaMemsetAsync(d_stats, 0, sizeof(DevStats), ctx->stream));
        }
    }
    if (!single) {
        KIWI_CUDA(ctx, cudaMemsetAsync(d_next, 0, sizeof(unsigned long long), ctx->stream));
        if (n > 0) {
            k_vor_bfs<<<blocks, 32 * kBfsWarpsPerBlock, 0, ctx->stream>>>(C, P, d_home, sup, 0, d_next, mark, queue,
                                                                         counts, nullptr, nullptr, nullptr, d_stats,
                                                                         fcounts, nullptr, nullptr, nullptr,
                                                                         VorStage{});
            KIWI_LAUNCHED(ctx);
        }
    }
    KIWI_TRY(exclusive_scan<int64_t>(ctx, counts, n, offs, d_total));
    KIWI_TRY(exclusive_scan<int64_t>(ctx, fcounts, n, foffs, d_ftotal));
    int64_t total = 0, total_faces = 0;
    KIWI_CUDA(ctx, cudaMemcpyAsync(&total, d_total, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
    KIWI_CUDA(ctx, cudaMemcpyAsync(&total_faces, d_ftotal, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
    KIWI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->vor_pairs_hint = total;
    ctx->vor_faces_hint = total_faces;
    // the face tables (each (pair, face) value evaluated once) when they fit a memory budget; else the
    // single-launch gather, which evaluates a shared face on both sides
    const int64_t face_bytes = total_faces * (int64_t)(sizeof(double) + sizeof(int32_t)) + total * 8;
    const bool tables = ctx->face_tables && face_bytes <= ((int64_t)48 << 30);
    int64_t* pair_foff = nullptr;
    int32_t* fsrc = nullptr;
    double* fval = nullptr;
    if (tables && total > 0) {
        KIWI_TRY(scratch_t(ctx, S_VOR_PFOFF, (size_t)total, &pair_foff));
        KIWI_TRY(scratch_t(ctx, S_VOR_FSRC, (size_t)std::max<int64_t>(total_faces, 1), &fsrc));
        KIWI_TRY(scratch_t(ctx, S_VOR_FVAL, (size_t)std::max<int64_t>(total_faces, 1), &fval));
    }
    if (total >= (1LL << 32)) return set_err(ctx, KIWI_ERR_LIMIT, "too many (cell, particle) pairs: %lld", (long long)total);
    int32_t* pair_cells = nullptr;
    unsigned long long* pair_mask = nullptr;
    uint32_t *k0, *v0, *k1, *v1;
    KIWI_TRY(scratch_t(ctx, S_VOR_PAIRS, (size_t)std::max<int64_t>(total, 1), &pair_cells));
    KIWI_TRY(scratch_t(ctx, S_VOR_MASK, (size_t)std::max<int64_t>(total, 1), &pair_mask));
    KIWI_TRY(scratch_t(ctx, S_KEYS0, (size_t)std::max<int64_t>(total, 1), &k0));
    KIWI_TRY(scratch_t(ctx, S_VALS0, (size_t)std::max<int64_t>(total, 1), &v0));
    KIWI_TRY(scratch_t(ctx, S_KEYS1, (size_t)std::max<int64_t>(total, 1), &k1));
    KIWI_TRY(scratch_t(ctx, S_VALS1, (size_t)std::max<int64_t>(total, 1), &v1));
    const uint32_t* plist = v0;
    if (total > 0) {
        if (single) {
            // the staged pairs and face sources, particle by particle
            k_vor_remap<<<(unsigned)((n * 32 + 255) / 256), 256, 0, ctx->stream>>>(
                n, stg, counts, fcounts, offs, foffs, pair_cells, pair_mask, pair_foff, fsrc);
            KIWI_LAUNCHED(ctx);
        } else {
            // pass 1: write each particle's visited cells at its offset
            KIWI_CUDA(ctx, cudaMemsetAsync(d_next, 0, sizeof(unsigned long long), ctx->stream));
            k_vor_bfs<<<blocks, 32 * kBfsWarpsPerBlock, 0, ctx->stream>>>(C, P, d_home, sup, 1, d_next, mark, queue,
                                                                         counts, offs, pair_cells, pair_mask, d_stats,
                                                                         nullptr, foffs, pair_foff, fsrc, VorStage{});
            KIWI_LAUNCHED(ctx);
        }
        k_vor_pairs<<<(unsigned)((total + 255) / 256), 256, 0, ctx->stream>>>(pair_cells, total, k0, v0);
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
    double* pair_val = nullptr;
    if (inv) KIWI_TRY(scratch_t(ctx, S_VOR_PVAL, (size_t)std::max<int64_t>(total, 1), &pair_val));
    if (fsrc) {
        if (kc.tabulated)
            k_vor_faces<kVorTab><<<(unsigned)nc, kGatherThreads, 0, ctx->stream>>>(
                C, P, kc.kernel, sup, kc.tab, plist, range, pair_foff, fsrc, offs, fval, d_stats);
        else if (kc.cubic)
            k_vor_faces<kVorCubic><<<(unsigned)nc, kGatherThreads, 0, ctx->stream>>>(
                C, P, kc.kernel, sup, kc.tab, plist, range, pair_foff, fsrc, offs, fval, d_stats);
        else
            k_vor_faces<kVorGeneric><<<(unsigned)nc, kGatherThreads, 0, ctx->stream>>>(
                C, P, kc.kernel, sup, kc.tab, plist, range, pair_foff, fsrc, offs, fval, d_stats);
        KIWI_LAUNCHED(ctx);
        k_vor_sum<<<(unsigned)nc, kGatherThreads, 0, ctx->stream>>>(C, P, plist, range, offs, pair_foff, fsrc, fval,
                                                                     out, d_stats, pair_val);
        KIWI_LAUNCHED(ctx);
    } else {
        if (kc.tabulated)
            k_vor_gather<kVorTab><<<(unsigned)nc, kGatherThreads, 0, ctx->stream>>>(
                C, P, kc.kernel, sup, kc.tab, plist, range, offs, pair_cells, pair_mask, out, d_stats, pair_val);
        else if (kc.cubic)
            k_vor_gather<kVorCubic><<<(unsigned)nc, kGatherThreads, 0, ctx->stream>>>(
                C, P, kc.kernel, sup, kc.tab, plist, range, offs, pair_cells, pair_mask, out, d_stats, pair_val);
        else
            k_vor_gather<kVorGeneric><<<(unsigned)nc, kGatherThreads, 0, ctx->stream>>>(
                C, P, kc.kernel, sup, kc.tab, plist, range, offs, pair_cells, pair_mask, out, d_stats, pair_val);
        KIWI_LAUNCHED(ctx);
    }
    if (inv && n > 0) {
        const double* cmass = inv->cell_mass;
        if (!cmass) {
            if (!out.density) return set_err(ctx, KIWI_ERR_ARG, "inverse map: no cell masses and no density output");
            double* cm = nullptr;
            KIWI_TRY(scratch_t(ctx, S_VOR_CMASS, (size_t)nc, &cm));
            k_vor_cell_mass<<<(unsigned)((nc + 255) / 256), 256, 0, ctx->stream>>>(nc, out.density, cells.volume, cm);
            KIWI_LAUNCHED(ctx);
            cmass = cm;
        }
        k_vor_recover<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(P, offs, pair_cells, pair_val, cmass,
                                                                            inv->m_recovered, inv->coverage);
        KIWI_LAUNCHED(ctx);
    }
    KIWI_CUDA(ctx, cudaEventRecord(ctx->ev[1], ctx->stream));
    DevStats hs;
    KIWI_CUDA(ctx, cudaMemcpyAsync(&hs, d_stats, sizeof hs, cudaMemcpyDeviceToHost, ctx->stream));
    KIWI_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (hs.limit_hit)
        return set_err(ctx, KIWI_ERR_LIMIT, "the cell walk hit a limit (a cell of more than 128 faces, or its iteration cap)");
    if (stats) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
        stats->bbox_pairs = total;
        stats->sphere_pairs = total;
        stats->evaluated_pairs = total;
        stats->skipped_outside = (int64_t)hs.skipped_outside;  // particles whose home cell is unresolved
        stats->neg_clamped = (int64_t)hs.neg_clamped;
        stats->neg_warned = (int64_t)hs.neg_warned;
        stats->table_clamps = (int64_t)hs.table_clamps;
        stats->tile_pairs = (int64_t)hs.tile_pairs;  // particles whose walk never left the home cell
        stats->gather_ms = ms;
        stats->launches = ctx->launches - launches0;
    }
    return KIWI_OK;
}

}  // namespace kiwi_b200
