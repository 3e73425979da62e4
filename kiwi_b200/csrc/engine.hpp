// Interfaces between the C-ABI layer (capi.cu) and the translation units holding the device kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "cart_common.cuh"
#include "ctx.hpp"

namespace kiwi_b200 {

// Device SoA view of a particle snapshot.
struct DevParticles {
    int64_t n;
    const double *x, *y, *z, *vx, *vy, *vz, *m, *h;
};

// Resolved kernel choice: cubic closed form (support 2h) or generic table `kernel` with support
// support_in_h * h.
struct KernelChoice {
    bool cubic;
    bool tabulated;
    int kernel;
    double support_in_h;
    TabDev tab;  // the context's density table when tabulated (set by table_ensure)
};

// tabulated.cu: the context's density table, generating the canonical one if it holds none.
int table_ensure(KiwiCtx* ctx, TabDev* out);
void table_free(KiwiCtx* ctx);

// Tile lists built by the binning step: tile t owns list[range[2t] .. range[2t+1]) (particle indices in
// ascending order).
struct TileLists {
    const uint32_t* list;
    const int64_t* range;
    int64_t ntiles;
    const int32_t* map = nullptr;  // optional: run only tiles map[0 .. nmap) (device array)
    int64_t nmap = 0;
};

struct CartOutputs {
    double *density, *vx, *vy, *vz;  // finalised fields (any may be null)
    double* raw4;                     // optional raw sums, 4 * ncell
    const double* meanv;              // device, 3 doubles: mean particle velocity
};

// Gradient outputs of the adjoint (device, one double per particle each; any may be null).
struct AdjointOutputs {
    double *x, *y, *z, *h, *m, *vx, *vy, *vz;
};

// capi.cu: argument resolution and the device pipeline of one sph-to-grid call
int resolve_kernel(KiwiCtx* ctx, const KiwiKernelSel* sel, KernelChoice* out);
int make_geom(KiwiCtx* ctx, const KiwiCartGrid* grid, double support_in_h, CartGeom* g);
bool particles_ok(KiwiCtx* ctx, const KiwiParticles* p, int* rc);
// part / n_parts: evaluate only the cell tiles owned by part `part` of `n_parts` (contiguous runs of the
// tile order with near-equal (tile, particle) entry counts); n_parts = 1 evaluates every tile.
int sph_to_grid_dev(KiwiCtx* ctx, const DevParticles& P, const CartGeom& g, const KernelChoice& kc, int precision,
                    const CartOutputs& out, KiwiStats* stats, int part = 0, int n_parts = 1);

// adjoint.cu
int cart_adjoint_dev(KiwiCtx* ctx, const DevParticles& P, const CartGeom& g, const KernelChoice& kc,
                     const double* d_cot, const AdjointOutputs& out, KiwiStats* stats);

// One grid of a batch (batch.cu): its geometry, particles and outputs, how its tiles are evaluated,
// and where its tiles start in the batch's concatenated tile lists.
enum BatchMode { kBatchLattice = 0, kBatchGatherCubic = 1, kBatchGatherGeneric = 2, kBatchLatticeGeneric = 3 };
// tile-body families, one persistent launch each
enum BatchFamily { kBatchFamilyLattice = 0, kBatchFamilyLatticeGeneric = 1, kBatchFamilyGather = 2, kBatchFamilies = 3 };
// launch-only family: the tiles of both lattice families in one persistent launch, each tile taking its
// item's body
constexpr int kBatchFamilyLatticeMerged = 3;
inline int batch_family(int mode) {
    return mode == kBatchLattice ? kBatchFamilyLattice
                                 : (mode == kBatchLatticeGeneric ? kBatchFamilyLatticeGeneric : kBatchFamilyGather);
}
struct BatchItemDev {
    CartGeom g;
    DevParticles P;
    CartOutputs out;
    int kernel;
    int mode;
    int64_t tile_base;
    DevStats* st;
};

// kiwi_fp64.cu: one persistent launch over the tiles order[0 .. ntiles) (global tile indices) of the items
// of one family, taken from the work counter *next (zero before the launch); mixed: the lattice families'
// FP32-mixed tile bodies.
int fp64_batch_prepare(KiwiCtx* ctx);
int fp64_batch_gather(KiwiCtx* ctx, int family, const BatchItemDev* d_items, const int32_t* d_item_of_tile,
                      const int32_t* d_order, int64_t ntiles, const uint32_t* list, const int64_t* range,
                      unsigned long long* d_next, int blocks, bool mixed);

// mixed.cu: the FP32-mixed form (cubic spline).  cell_err (device, ncell doubles) receives each cell's
// rounding-error bound and cell_mass (ncell doubles) its raw mass sum M.
int mixed_cart_gather(KiwiCtx* ctx, const CartGeom& g, const DevParticles& P, const TileLists& tl,
                      const CartOutputs& out, double* cell_err, double* cell_mass, DevStats* d_stats);
// Tiles holding a cell above floor_frac of the peak cell mass whose bound exceeds rel_tol of its mass:
// writes their indices to map (ascending) and their count to *d_nmap (device).
int mixed_flag_tiles(KiwiCtx* ctx, const CartGeom& g, const double* cell_err, const double* cell_mass,
                     double rel_tol, double floor_frac, int32_t* map, int64_t* d_nmap);
int fp32_measure_peak(KiwiCtx* ctx, double* tflops);

// voronoi.cu
int voronoi_init_tables(KiwiCtx* ctx);
// The inverse-mapping check's outputs (run_inverse_mapping_test_stage, src/mapping.cpp:540-701): per
// particle the mass recovered from the cells it reaches and its coverage fraction (device arrays of n);
// cell_mass: m_i per cell (device), or null for density x volume of the same call's forward map.
struct VorInverse {
    const double* cell_mass;
    double* m_recovered;
    double* coverage;
};
int voronoi_map_dev(KiwiCtx* ctx, const DevParticles& P, const int32_t* d_home, const KiwiVoronoiCells& cells,
                    const KernelChoice& kc, const CartOutputs& out, KiwiStats* stats,
                    const VorInverse* inv = nullptr);

// kiwi_fp64.cu
int fp64_init_tables(KiwiCtx* ctx);
int fp64_cart_gather(KiwiCtx* ctx, const CartGeom& g, const DevParticles& P, const KernelChoice& k,
                     const TileLists& tl, const CartOutputs& out, DevStats* d_stats, bool full_box,
                     bool reference_order);
int fp64_full_integral(KiwiCtx* ctx, int kernel, int64_t n, const double* arg0, const double* phi, const double* r0,
                       const double* R0, double* out);
int fp64_tier_constants(KiwiCtx* ctx, int kernel, int64_t n, const double* arg0, const double* r0, const double* R0,
                        double* wall, double* edge);
int fp64_face_integral(KiwiCtx* ctx, const KernelChoice& k, int64_t n, const double* particle,
                       const int64_t* vert_off, const double* verts, double* out, int32_t* out_vert);
int fp64_mean_velocity(KiwiCtx* ctx, const DevParticles& P, double* d_meanv);
int fp64_measure_peak(KiwiCtx* ctx, double* tflops);

// lattice.cu: the lattice-factorised gather of the plain FP64 form for the cubic spline (every cell of the
// support boxes with full_box, else the cells the supports reach) and the generic kernels (the cells the
// supports reach), and the batch's persistent launches of those two families.
int lattice_init_tables(KiwiCtx* ctx);
int adjoint_init_tables(KiwiCtx* ctx);
int lattice_cart_gather(KiwiCtx* ctx, const CartGeom& g, const DevParticles& P, const KernelChoice& k,
                        const TileLists& tl, const CartOutputs& out, DevStats* d_stats, bool full_box);
// The FP32-mixed form of the cubic lattice gather (FP32 tiers with FP64 islands, FP64 assembly); the number
// of lattice points evaluated in FP64 (islands) is added to d_stats->fp64_fallback.
int lattice_mixed_gather(KiwiCtx* ctx, const CartGeom& g, const DevParticles& P, const KernelChoice& k,
                         const TileLists& tl, const CartOutputs& out, DevStats* d_stats);
int lattice_batch_prepare(KiwiCtx* ctx);
int lattice_batch_gather(KiwiCtx* ctx, int family, const BatchItemDev* d_items, const int32_t* d_item_of_tile,
                         const int32_t* d_order, int64_t ntiles, const uint32_t* list, const int64_t* range,
                         unsigned long long* d_next, int blocks, bool mixed);

}  // namespace kiwi_b200
