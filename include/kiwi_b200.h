/* kiwi_b200: C ABI of the B200-native KIWI kernel-integral engine (libkiwi_b200.so).
 *
 * Every entry point below replaces a piece of the reference's C++ kernel-integral layer or one of its
 * two mapping stages; the comment on each names the reference interface (path within mapetkova/kiwi,
 * file:line).  Conventions:
 *   - plain pointers and sizes only; all arrays are caller-owned;
 *   - return value 0 (KIWI_OK) or a negative KIWI_ERR_* code; kiwi_last_error() explains it.  This is
 *     the C form of the reference's exceptions (std::runtime_error / ConfigError, turned into one
 *     "[kiwi] error: <what>" line by src/main.cpp:241-244);
 *   - one context per host thread; every call is synchronous with respect to the host unless its name
 *     ends in _device, in which case it is stream-ordered on the context's stream;
 *   - results are deterministic: each cell's sum is taken over its particles in ascending particle
 *     order, with no floating-point atomics, so repeated calls are bitwise identical;
 *   - there is no CPU fallback: without a usable sm_100 GPU every compute call fails with
 *     KIWI_ERR_NODEV.  The host-only helpers (kernel lookups, kiwi_part_rows, kiwi_snapshot_work,
 *     kiwi_voronoi_cell_owners, kiwi_voronoi_part_particles, the file readers and writers) need no GPU.
 */
#ifndef KIWI_B200_H
#define KIWI_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KIWI_OK 0
#define KIWI_ERR_ARG (-1)         /* invalid argument (the reference's ConfigError / runtime_error) */
#define KIWI_ERR_CUDA (-2)        /* a CUDA call failed */
#define KIWI_ERR_NODEV (-3)       /* no usable GPU */
#define KIWI_ERR_ALLOC (-4)       /* memory allocation failed (device; host in the host-only helpers) */
#define KIWI_ERR_LIMIT (-5)       /* a bounded device loop hit its iteration cap */
#define KIWI_ERR_UNSUPPORTED (-6) /* option not available in this library */

/* Arithmetic forms of the cell integrals (the low byte of a `precision` argument).
 * KIWI_FP64: all FP64.  The tiers are shared between the cells of a particle's box (each edge tier once
 * per plane and edge line, each lattice point's octant value once, a cell the alternating sum of its 8
 * corners' values), which is algebraically the reference's per-cell sum; the cubic closed form and the
 * generic kernels' tables alike.
 * KIWI_FP64_REFERENCE_ORDER: all FP64 in the reference's per-cell evaluation order, operation by
 * operation (6 faces x 4 edges x 2 vertices per cell, src/kernel_integral.cpp:471-647).
 * KIWI_FP32_MIXED: the edge tiers and octant values of the lattice form in FP32 (cubic closed form or the
 * generic kernels' tables), evaluated from FP64 plane offsets relative to the particle; the cell assembly
 * and the per-cell totals in FP64; lattice points and edge lines with a plane within 1e-3 h of the
 * particle in FP64 throughout (fp64_fallback in KiwiStats counts those points).  The closed form
 * subtracts octant values that can exceed the cell's mass by orders of magnitude, so the FP32 error grows
 * in the cells far from the particle: an approximate form with a stated error, not within 1e-6. */
#define KIWI_FP64 0
#define KIWI_FP32_MIXED 1
#define KIWI_FP64_REFERENCE_ORDER 2
#define KIWI_FORM_MASK 0xff
/* Flag: evaluate every cell of each particle's support bounding box, as the reference does
 * (src/cartesian_grid.cpp:213-243).  Without it only cells whose closest point lies within the support
 * radius are evaluated; the others hold no kernel mass and the reference's values for them are
 * rounding noise around zero (clamped at 0). */
#define KIWI_FULL_BOX 0x100
/* Flag for KIWI_FP32_MIXED (cubic spline with support 2h): evaluate the FP32 terms with their magnitudes,
 * so that each cell gets a bound on its rounding error (4 x 2^-24 x the summed magnitudes of its FP32
 * terms), and recompute in FP64 (lattice form) every 8x8x8 cell tile holding a cell whose mass is at least
 * 1e-6 of the peak cell mass and whose bound exceeds 1e-6 of its mass, so that those cells are within 1e-6
 * relative by construction.  KiwiStats.fp64_tiles counts the tiles, fp64_fallback the cells whose bound
 * exceeds 1e-6 of their mass. */
#define KIWI_FP32_GUARANTEE 0x200

typedef struct KiwiCtx KiwiCtx;

/* Particle snapshot, SoA (the SPHSnapshot fields the hot path reads, include/kiwi/snapshot.hpp:70-77). */
typedef struct KiwiParticles {
    int64_t n;
    const double *x, *y, *z;    /* positions */
    const double *vx, *vy, *vz; /* velocities */
    const double *m, *h;        /* mass, smoothing length (h <= 0: no contribution, as the reference) */
} KiwiParticles;

/* Uniform Cartesian grid (Domain + CartesianGridConfig resolved nx/ny/nz, include/kiwi/config.hpp:24-30,
 * 209-216; src/cartesian_grid.cpp:89-97).  Cell (ix,iy,iz) is stored at (ix*ny + iy)*nz + iz. */
typedef struct KiwiCartGrid {
    double bounds[6]; /* x_min, x_max, y_min, y_max, z_min, z_max */
    int32_t nx, ny, nz;
} KiwiCartGrid;

/* Kernel selection (KernelConfig + the dispatch of make_kernel_integrator,
 * include/kiwi/kernel_integrator.hpp:14-45 and src/config.cpp:267-277): the cubic closed form is used iff
 * kernel == M4, the support is 2h and generic_path == 0; otherwise the generic table-driven integral. */
typedef struct KiwiKernelSel {
    int32_t kernel;       /* kiwi_kernel_index(): 0 M4, 1 M5, 2 M6, 3 WC2, 4 WC4, 5 WC6 */
    double support_in_h;  /* kernel support radius in units of h; 0 = the kernel's default radkern */
    int32_t generic_path; /* force the generic integral for M4 */
    int32_t tabulated;    /* cubic path only: trilinear lookup in the context's density table instead of the
                           * closed form (the canonical table is generated on first use if none is loaded) */
} KiwiKernelSel;

typedef struct KiwiStats {
    int64_t bbox_pairs;      /* (particle, cell) pairs in the clamped support bounding boxes */
    int64_t sphere_pairs;    /* of those, cells whose closest point lies within the support radius */
    int64_t evaluated_pairs; /* pairs whose integral was evaluated */
    int64_t skipped_outside; /* particles whose support misses the grid (src/cartesian_grid.cpp:234-237) */
    int64_t neg_clamped;     /* pair integrals < 0 clamped to 0 (src/cartesian_grid.cpp:264-269) */
    int64_t neg_warned;      /* of those, <= -0.01 (the reference prints a warning for each) */
    int64_t fp64_fallback;   /* KIWI_FP32_MIXED: lattice points evaluated in FP64 (a plane within 1e-3 h);
                              * with KIWI_FP32_GUARANTEE: cells whose FP32 rounding bound exceeds 1e-6 of
                              * their mass */
    int64_t tile_pairs;      /* (tile, particle) list entries built by the binning step */
    int64_t launches;        /* GPU kernels launched by this call */
    double gather_ms;        /* device time of the cell-integral kernel(s) of this call (CUDA events) */
    double total_ms;         /* device time of the whole call, copies included for the host variants */
    /* work items of the lattice-factorised FP64 evaluation (0 for the other forms): edge tiers by the
     * distance of the edge line (beyond 2h, between h and 2h, within h) and vertex pyramids */
    int64_t edge_tiers_outer, edge_tiers_middle, edge_tiers_inner, vertex_pyramids;
    int64_t fp64_tiles;      /* KIWI_FP32_GUARANTEE: cell tiles recomputed in FP64 */
    int64_t table_clamps;    /* tabulated integral: lookup indices clamped into the table (the reference
                              * prints a warning for each, src/kernel_integral.cpp:125-133) */
} KiwiStats;

/* ---- context --------------------------------------------------------------------------------- */
int kiwi_ctx_create(int device, KiwiCtx** out);
void kiwi_ctx_destroy(KiwiCtx* ctx);
const char* kiwi_last_error(const KiwiCtx* ctx); /* message of the last failed call on ctx */
void* kiwi_ctx_stream(KiwiCtx* ctx);             /* the context's cudaStream_t */
int kiwi_ctx_synchronize(KiwiCtx* ctx);
/* Voronoi maps on this context: enable = 1 (the default) evaluates every face value once per particle
 * through per-(pair, face) tables (12 bytes per face of every visited cell; a map whose tables would
 * exceed 48 GB runs without them), and a map after an earlier one on the same context walks the cell
 * graph once, into space reserved from the earlier map's totals (another ~24 bytes per visited pair and
 * 4 per face; a map that outgrows the reservation walks twice); enable = 0 walks twice and runs one
 * launch that evaluates a face shared by two visited cells on both sides.  Every path gives the same
 * results bit for bit.  No counterpart in the reference. */
int kiwi_ctx_set_voronoi_face_tables(KiwiCtx* ctx, int enable);
const char* kiwi_version(void);
/* Measured FP64 FMA throughput of the context's GPU in TFLOP/s (a short probe kernel).  No counterpart in
 * the reference: it provides the roofline denominator of the FP64 cell-integral kernels. */
int kiwi_measure_fp64_peak(KiwiCtx* ctx, double* tflops);
/* The same for FP32 FMA throughput (the roofline denominator of the FP32-mixed form's kernel). */
int kiwi_measure_fp32_peak(KiwiCtx* ctx, double* tflops);

/* ---- kernel tables (include/kiwi/kernel_spec.hpp:18-44, src/kernel_spec_data.cpp:175-187) ----- */
/* get_kernel(name): index 0..5 for a key or alias ("M4", "cubic_spline", "wendland_c4", ...), -1 if
 * unknown (the reference throws std::invalid_argument). */
int kiwi_kernel_index(const char* name);
/* Kernel constants: out7 = {nreg, A2_pi, A3_pi, radkern, hfact, c[0], c[1]}. */
int kiwi_kernel_info(int kernel, double* out7);

/* ---- scalar integral layer, batched on the GPU ----------------------------------------------- */
/* full_integral_new(h, phi, r0, R_0) (include/kiwi/kernel_integral.hpp:80) when kernel < 0, with arg0 = h;
 * generic_full_integral(K, H, phi, r0, R_0) (include/kiwi/kernel_integral_generic.hpp:56) when
 * kernel >= 0, with arg0 = H.  Host arrays of length n. */
int kiwi_full_integral_batch(KiwiCtx* ctx, int kernel, int64_t n, const double* arg0, const double* phi,
                             const double* r0, const double* R_0, double* out);

/* The tier constants of n (r0, R_0) pairs, as the reference's structs hold them (host arrays).  kernel < 0:
 * the cubic spline with arg0 = h -- compute_wall_constants (src/kernel_integral.cpp:222-247) into
 * KIWI_CUBIC_WALL_DOUBLES per item {valid, r0, h, h2, r03, r0h2, r0h3, r0h_2, r0h_3, B1, B2, B3} and
 * compute_edge_constants (:253-350) into KIWI_CUBIC_EDGE_DOUBLES {valid, R_0, a, a2, D2, D3}
 * (include/kiwi/kernel_integral.hpp:108-127).  kernel >= 0: arg0 = H -- generic_wall_constants
 * (src/kernel_integral_generic.cpp:96-117) into KIWI_GENERIC_WALL_DOUBLES {valid, H, r0, q0, j,
 * coef[4][15], bphi[4]} and generic_edge_constants (:119-148) into KIWI_GENERIC_EDGE_DOUBLES {valid, R_0, a,
 * a2, nseg, region[4], phi_end[4], offset[4]} (include/kiwi/kernel_integral_generic.hpp:27-48). */
#define KIWI_CUBIC_WALL_DOUBLES 12
#define KIWI_CUBIC_EDGE_DOUBLES 6
#define KIWI_GENERIC_WALL_DOUBLES 69
#define KIWI_GENERIC_EDGE_DOUBLES 17
int kiwi_tier_constants_batch(KiwiCtx* ctx, int kernel, int64_t n, const double* arg0, const double* r0,
                              const double* R_0, double* wall_out, double* edge_out);

/* compute_face_integral / compute_face_integral_generic (include/kiwi/kernel_integral.hpp:182-193) for
 * n_faces independent (particle, face) items.  particle: 4 doubles per item (x0, y0, z0, h); face i has
 * vertices vert_off[i]..vert_off[i+1]-1 of verts (xyz each, absolute, in the face's winding).  out_vert
 * (may be NULL) receives the reference's out_vert per item. */
int kiwi_face_integral_batch(KiwiCtx* ctx, const KiwiKernelSel* kernel, int64_t n_faces, const double* particle,
                             const int64_t* vert_off, const double* verts, double* out, int32_t* out_vert);

/* ---- tabulated cubic integral (DensityLookupTable, include/kiwi/kernel_integral.hpp:21-72) ------ */
/* The shape of a density lookup table: three axes (r0/h, mu0, cos phi), each two uniform sub-grids split
 * at rl, mul, cphil (the header of the reference's table file). */
typedef struct KiwiDensityTableInfo {
    int32_t nr01, nR_01, nphi1, nr02, nR_02, nphi2;
    double rl, mul, cphil;
    int64_t n_values; /* (nr01 + nr02 + 2) (nR_01 + nR_02 + 1) (nphi1 + nphi2 + 1) */
} KiwiDensityTableInfo;
/* generate_density_table (src/kernel_integral.cpp:57-119): the canonical 251 x 301 x 301 table, computed on
 * the GPU into the context (replacing any table it holds). */
int kiwi_density_table_generate(KiwiCtx* ctx);
/* load_density_table (src/kernel_integral.cpp:20-55): the reference's text format, into the context.
 * Errors (KIWI_ERR_ARG) carry the reference's messages; shapes the reference would divide by zero on or
 * that exceed 2^31 values are rejected too. */
int kiwi_density_table_load(KiwiCtx* ctx, const char* path);
/* A caller's table (DensityLookupTable's header fields and its values, laid out as
 * DensityLookupTable::at, include/kiwi/kernel_integral.hpp:27-40) copied into the context, replacing any table
 * it holds; the shape is checked as the loader checks it. */
int kiwi_density_table_set(KiwiCtx* ctx, const KiwiDensityTableInfo* info, const double* values);
/* Shape of the context's table (KIWI_ERR_ARG if it holds none). */
int kiwi_density_table_info(KiwiCtx* ctx, KiwiDensityTableInfo* info);
/* Copy the table's n_values values to host memory, laid out as the reference's DensityLookupTable::at. */
int kiwi_density_table_read(KiwiCtx* ctx, double* values, int64_t n);
void kiwi_density_table_release(KiwiCtx* ctx);
/* gridded_integral(table, h, phi, r0, R_0) (src/kernel_integral.cpp:136-190) for n items (host arrays);
 * clamps (may be NULL) receives the number of lookup indices clamped into the table. */
int kiwi_gridded_integral_batch(KiwiCtx* ctx, int64_t n, const double* h, const double* phi, const double* r0,
                                const double* R_0, double* out, int64_t* clamps);

/* ---- sph-to-grid stage (run_sph_to_grid_stage, src/cartesian_grid.cpp:76-321) ---------------- */
/* Host arrays in, host arrays out (density, vx, vy, vz as CartesianGridResult holds them,
 * include/kiwi/cartesian_grid.hpp:53-71).  raw4 (may be NULL): the unnormalised sums
 * sum m*Msum, sum m*Msum*v{x,y,z} (4 * ncells doubles). */
int kiwi_sph_to_grid(KiwiCtx* ctx, const KiwiParticles* particles, const KiwiCartGrid* grid,
                     const KiwiKernelSel* kernel, int precision, double* density, double* vx, double* vy,
                     double* vz, double* raw4, KiwiStats* stats);

/* Same with every pointer (particles and outputs) in device memory, on the context's stream. */
int kiwi_sph_to_grid_device(KiwiCtx* ctx, const KiwiParticles* particles, const KiwiCartGrid* grid,
                            const KiwiKernelSel* kernel, int precision, double* density, double* vx, double* vy,
                            double* vz, double* raw4, KiwiStats* stats);

/* One part of kiwi_sph_to_grid_device, for splitting one grid over several GPUs (one process or context
 * per GPU, each with every particle; no counterpart in the reference, whose OpenMP loop splits
 * particles inside one process).  The 8x8x8-cell tiles are split into n_parts contiguous runs of the
 * tile order (tile (tx, ty, tz) at index (tx * nty + ty) * ntz + tz, so each run covers a slab of x rows)
 * holding near-equal numbers of (tile, particle) entries; part `part` computes and writes only the cells
 * of its own tiles, each equal bit for bit to the whole call's.  The other cells of the outputs are left
 * as they were.  KIWI_FP32_GUARANTEE needs n_parts = 1.  1 <= n_parts <= 65536. */
int kiwi_sph_to_grid_device_part(KiwiCtx* ctx, const KiwiParticles* particles, const KiwiCartGrid* grid,
                                 const KiwiKernelSel* kernel, int precision, int part, int n_parts, double* density,
                                 double* vx, double* vy, double* vz, double* raw4, KiwiStats* stats);

/* Host only, no GPU work (no counterpart in the reference): the x rows [*ix0, *ix1) of cells that part
 * `part` of kiwi_sph_to_grid_device_part writes (its tiles' cells lie in these rows, contiguous in the
 * output layout), from HOST arrays x, y, z, h of the same particles: the same support boxes and ownership
 * rule, so that each rank knows which rows to copy back before it runs.  *ix0 = *ix1 = 0 if the part owns
 * no tile.  ctx may be NULL (no message). */
int kiwi_part_rows(KiwiCtx* ctx, const KiwiParticles* particles, const KiwiCartGrid* grid,
                   const KiwiKernelSel* kernel, int part, int n_parts, int* ix0, int* ix1);

/* Host only, no GPU work (no counterpart in the reference): a snapshot's (particle, cell) pairs within the
 * particles' clamped support boxes (src/cartesian_grid.cpp:211-237; KiwiStats.bbox_pairs of the
 * reference-order form), from HOST arrays x, y, z, h -- the work estimate by which a batch of snapshots is
 * dealt to GPUs, longest first.  ctx may be NULL (no message). */
int kiwi_snapshot_work(KiwiCtx* ctx, const KiwiParticles* particles, const KiwiCartGrid* grid,
                       const KiwiKernelSel* kernel, int64_t* bbox_pairs);

/* Adjoint of the sph-to-grid raw sums.  It has no counterpart in the reference (which has no gradients).
 * With M_c = sum_p m_p K_pc and P_c = sum_p m_p K_pc v_p the raw sums of kiwi_sph_to_grid_device
 * (K_pc the particle's kernel mass in cell c, clamped at 0), and raw4 the cotangents dL/dM, dL/dPx,
 * dL/dPy, dL/dPz (4 * ncells doubles, the raw4 layout), it writes per particle dL/dx, dL/dy, dL/dz,
 * dL/dh, dL/dm, dL/dvx, dL/dvy, dL/dvz (any output may be NULL).  The per-pair integrals are recomputed
 * in FP64 with forward-mode derivatives, over the pairs of the default (support-culled) evaluation.
 * Every pointer is in device memory; runs on the context's stream and returns when done.  The cubic
 * closed form and the generic kernels' tables (every kernel of kiwi_kernel_spec); the tabulated integral
 * returns KIWI_ERR_UNSUPPORTED. */
int kiwi_sph_to_grid_adjoint_device(KiwiCtx* ctx, const KiwiParticles* particles, const KiwiCartGrid* grid,
                                    const KiwiKernelSel* kernel, const double* raw4, double* dx, double* dy,
                                    double* dz, double* dh, double* dm, double* dvx, double* dvy, double* dvz,
                                    KiwiStats* stats);

/* Allocation-free variant of kiwi_sph_to_grid_device.  It has no counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc: codes that hand all device memory to their own pool
 * allocator (an SPH simulation mapping its particles in situ between steps, a rank with a hard memory
 * budget) and latency-sensitive callers that cannot absorb the device-wide synchronisation a cudaMalloc
 * or cudaFree may cause.  It allocates nothing: every scratch buffer comes from one fixed device array of
 * KIWI_NOALLOC_SCRATCH_BYTES inside the library, which every GPU that loads the library holds until the
 * process exits.  The caller passes the particle arrays and the output arrays, all in device memory, and
 * the stream to run on (NULL: the legacy default stream); no KiwiCtx is needed.  It works on the current
 * device.  Its first call on a device does a one-off set-up there (the scratch array's device address,
 * the kernel tables, two timing events); make that first call before any stream capture.  Inputs whose
 * scratch needs exceed the array (roughly 36 bytes per particle plus 18 bytes per (tile, particle)
 * entry plus 16 bytes per 8x8x8-cell tile) are rejected with KIWI_ERR_LIMIT and a message in err (if
 * err_len > 0).  Every call reuses the same array and leaves the last call's contents in it, so calls
 * whose GPU work overlaps -- on different streams or from different host threads -- race and must be
 * serialised by the caller.  A call that fails waits for the work it had queued on the stream before it
 * returns, so nothing of it still writes the array afterwards.  Results equal kiwi_sph_to_grid_device's. */
#define KIWI_NOALLOC_SCRATCH_BYTES (32u << 20)
int kiwi_sph_to_grid_device_noalloc(void* stream, const KiwiParticles* particles, const KiwiCartGrid* grid,
                                    const KiwiKernelSel* kernel, int precision, double* density, double* vx,
                                    double* vy, double* vz, double* raw4, KiwiStats* stats, char* err,
                                    size_t err_len);

/* ---- batches of sph-to-grid problems (no counterpart in the reference) ----------------------- */
/* Many snapshots, each mapped onto its own grid with its own kernel, in one persistent launch per
 * evaluation family (cubic lattice, generic lattice, per-cell gather) recorded as one CUDA graph.  The reference maps one snapshot per run; a caller with many (a time series, a
 * parameter sweep, a set of zoom regions) would otherwise pay one launch sequence per snapshot and leave
 * the GPU idle on the small ones.  Every pointer of an item is in device memory. */
typedef struct KiwiBatchItem {
    KiwiParticles particles;
    KiwiCartGrid grid;
    KiwiKernelSel kernel;
    double *density, *vx, *vy, *vz; /* outputs, ncells each (any may be NULL) */
    double* raw4;                   /* optional raw sums, 4 * ncells */
} KiwiBatchItem;
typedef struct KiwiBatch KiwiBatch;

/* Bins every item's particles into the cell tiles of its grid (one scan and one sort over all items),
 * orders the tiles longest-first, and records the graph.  precision: KIWI_FP64 (lattice form),
 * KIWI_FP64_REFERENCE_ORDER or KIWI_FP32_MIXED (the lattice form's FP32-mixed tiles); no flags.  The plan
 * holds the tile lists of the particles' positions and smoothing lengths at creation: masses and velocities may change between runs, positions and smoothing
 * lengths may not.  Results equal kiwi_sph_to_grid_device's for each item: bit for bit in
 * KIWI_FP64_REFERENCE_ORDER; in the lattice form to rounding (within 1e-12 of the item's largest value;
 * it is compiled with FMA contraction, which the compiler forms per kernel), with equal counts. */
int kiwi_batch_create(KiwiCtx* ctx, const KiwiBatchItem* items, int n_items, int precision, KiwiBatch** out);
/* Replays the graph on the context's stream and waits for it.  item_stats (n_items entries) and total
 * may be NULL; gather_ms / total_ms hold the device time of the whole batch. */
int kiwi_batch_run(KiwiBatch* batch, KiwiStats* item_stats, KiwiStats* total);
/* Times the launch shapes (the two lattice families -- cubic and table-driven kernels -- in one persistent
 * launch or one each, when the batch holds both x longest-first or natural tile order x 1 or 2 resident
 * CTAs per SM; one run each) and keeps the fastest; *chosen = 0x10000 if merged | 0x100 if longest-first
 * | CTAs per SM. */
int kiwi_batch_tune(KiwiBatch* batch, int* chosen);
void kiwi_batch_destroy(KiwiBatch* batch);

/* ---- stage output files (host only; no GPU needed) ------------------------------------------- */
/* save_cartesian_grid (src/cartesian_grid.cpp:323-347): the VGTCGRD2 binary file -- "VGTCGRD2", int32 nx,
 * ny, nz, 6 doubles of bounds, then density, vx, vy, vz (nx*ny*nz doubles each, x-major).  Errors:
 * KIWI_ERR_ARG with the reference's message in err (if err_len > 0). */
int kiwi_save_cartesian_grid(const char* path, int32_t nx, int32_t ny, int32_t nz, const double* bounds6,
                             const double* density, const double* vx, const double* vy, const double* vz, char* err,
                             size_t err_len);
/* load_cartesian_grid (src/cartesian_grid.cpp:349-394).  With all four arrays NULL only the header is read
 * (nxyz[3], bounds6 may be NULL), so the caller can size the arrays; otherwise all four are filled. */
int kiwi_load_cartesian_grid(const char* path, int32_t* nxyz, double* bounds6, double* density, double* vx,
                             double* vy, double* vz, char* err, size_t err_len);
/* save_mapping (src/mapping.cpp:307-315): mapping.dat, "id x y z volume density vx vy vz" per cell with
 * 15 significant digits. */
int kiwi_save_mapping(const char* path, int64_t n_cells, const int64_t* id, const double* x, const double* y,
                      const double* z, const double* volume, const double* density, const double* vx, const double* vy,
                      const double* vz, char* err, size_t err_len);

/* save_cartesian_map / load_cartesian_map (src/cartesian_map.cpp:202-279): the VGTCMAP1 file of a cartesian
 * map; the loader reads the header only when all five arrays are NULL. */
int kiwi_save_cartesian_map(const char* path, int32_t res, const double* bounds6, const double* density,
                            const double* vx, const double* vy, const double* vz, const int32_t* voronoi_cell_id,
                            char* err, size_t err_len);
int kiwi_load_cartesian_map(const char* path, int32_t* res, double* bounds6, double* density, double* vx, double* vy,
                            double* vz, int32_t* voronoi_cell_id, char* err, size_t err_len);
/* save_inverse_mapping_test (src/mapping.cpp:505-513): inverse-mapping-test.dat, a '#' header, the totals
 * (original, grid, recovered mass) and "id m_original m_recovered coverage_fraction" per particle, with 15
 * significant digits. */
int kiwi_save_inverse_mapping_test(const char* path, int64_t n, const int64_t* id, const double* m_original,
                                   const double* m_recovered, const double* coverage, const double* totals3, char* err,
                                   size_t err_len);
/* load_inverse_mapping_test (src/mapping.cpp:519-538): *n receives the row count; rows are stored while
 * they fit in `capacity` (id may be NULL to count only); the reference's messages on a bad file. */
int kiwi_load_inverse_mapping_test(const char* path, int64_t* n, double* totals3, int64_t* id, double* m_original,
                                   double* m_recovered, double* coverage, int64_t capacity, char* err, size_t err_len);

/* ---- Voronoi map stage (run_mapping_stage's particle loop, src/mapping.cpp:105-206, 400-502) --- */
/* Cell geometry in CSR form: the plain data of CellFaceGeometry (src/mapping.cpp:49-54) with vertex
 * coordinates made absolute as src/mapping.cpp:168-175 does and neighbour ids resolved to cell indices. */
typedef struct KiwiVoronoiCells {
    int64_t n_cells;
    const int64_t* face_off; /* n_cells + 1 */
    const int64_t* vert_off; /* n_faces + 1 */
    const double* vxyz;      /* 3 per vertex */
    const int32_t* face_nbr; /* neighbour cell index, or -1 for a wall / unresolved neighbour */
    const double* volume;    /* n_cells */
} KiwiVoronoiCells;

/* home_cell: per particle the cell containing it (container::find_voronoi_cell resolved through
 * reverse_id_list, src/mapping.cpp:434-439), or -1 (skipped, "unresolved").  Outputs per cell in the
 * geometry's order: density = M/volume (0 if volume <= 0), velocity = P/M or the mean velocity. */
int kiwi_map_voronoi(KiwiCtx* ctx, const KiwiParticles* particles, const int32_t* home_cell,
                     const KiwiVoronoiCells* cells, const KiwiKernelSel* kernel, int precision, double* density,
                     double* vx, double* vy, double* vz, double* raw4, KiwiStats* stats);

/* kiwi_map_voronoi with every array in device memory -- particles, home cells, the cell geometry and the
 * outputs -- on the context's stream (returns when done): a caller that maps several snapshots, or several
 * quantities, on one tessellation copies its geometry to the GPU once.  The geometry's offsets and
 * neighbour indices are not checked here (kiwi_map_voronoi checks them on the host); they must satisfy the
 * same rules: face_off and vert_off start at 0 and do not decrease, face_nbr < n_cells, home_cell < n_cells. */
int kiwi_map_voronoi_device(KiwiCtx* ctx, const KiwiParticles* particles, const int32_t* home_cell,
                            const KiwiVoronoiCells* cells, const KiwiKernelSel* kernel, int precision, double* density,
                            double* vx, double* vy, double* vz, double* raw4, KiwiStats* stats);

/* A Voronoi map over several GPUs (no counterpart in the reference), host only, no GPU work.
 * kiwi_voronoi_cell_owners: owner[c] in [0, n_parts), the cells split into spatial slabs along `axis`
 * (0, 1, 2): ordered by the midpoint (lo + hi) / 2 of their vertices' extent along it (ties by cell index;
 * coordinates must be finite) and cut into runs of near-equal counts (rank k -> part k n_parts / n_cells).
 * kiwi_voronoi_part_particles: select[i] = 1 for the particles whose walk can reach a cell of `part` --
 * home cell owned by it, or support sphere within 1.001 radii of the box around its cells' vertices --
 * and the count in *n_selected.  A rank that maps these particles (in their order) with kiwi_map_voronoi
 * gets its own cells bit for bit as the whole snapshot gives them; a cell no particle reaches takes the
 * whole snapshot's mean velocity.  Every array is a HOST array; ctx may be NULL (no message). */
int kiwi_voronoi_cell_owners(KiwiCtx* ctx, const KiwiVoronoiCells* cells, int n_parts, int axis, int32_t* owner);
int kiwi_voronoi_part_particles(KiwiCtx* ctx, const KiwiParticles* particles, const int32_t* home_cell,
                                const KiwiVoronoiCells* cells, const KiwiKernelSel* kernel, const int32_t* owner,
                                int part, uint8_t* select, int64_t* n_selected);

/* The inverse-mapping check (run_inverse_mapping_test_stage's particle loop, src/mapping.cpp:540-701): the
 * same cell walk and cell integrals as kiwi_map_voronoi, summed per particle instead of per cell, in the
 * walk's order: m_recovered[i] = sum over the cells i reaches of (integral m_i' / M_c) M_c over cells with
 * M_c > 0, coverage[i] = m_recovered[i] / m_i (0 if m_i <= 0); particles with h <= 0 or an unresolved home
 * cell recover 0.  cell_mass (may be NULL): M_c per cell, density x volume of the forward mapping (the
 * reference takes mapping.dat's rows); NULL uses this call's own forward map.  totals3 (may be NULL):
 * total original mass, total grid mass (sum of M_c), total recovered mass, summed in order.  density (may
 * be NULL) receives the forward map's densities.  Host arrays. */
int kiwi_inverse_map_voronoi(KiwiCtx* ctx, const KiwiParticles* particles, const int32_t* home_cell,
                             const KiwiVoronoiCells* cells, const KiwiKernelSel* kernel, int precision,
                             const double* cell_mass, double* m_recovered, double* coverage, double* totals3,
                             double* density, KiwiStats* stats);

/* ---- point-set stage (src/point_set.cpp) ------------------------------------------------------ */
/* The candidate lattice of the coverage-grid buffer (generate_cartesian_lattice, src/point_set.cpp:166-195):
 * spacing = spacing_fraction x the smallest extent, round(extent / spacing) (at least 1) cell-centred
 * candidates per axis; returns their count (-1 on bad arguments), dims3 (may be NULL) the per-axis counts.
 * Host only. */
int64_t kiwi_coverage_grid_candidates(const double* bounds6, double spacing_fraction, int32_t* dims3);
/* add_coverage_grid_buffer (src/point_set.cpp:198-262): the lattice candidates that no particle covers
 * (squared distance <= (coverage_radius_factor x h_i)^2), in lattice order, with ids n + 1, n + 2, ...
 * (host arrays).  *n_added receives their count; with all four outputs NULL only the count is computed,
 * else they must hold capacity >= *n_added points.  KIWI_ERR_ARG with the reference's message if every
 * h <= 0. */
int kiwi_coverage_grid_buffer(KiwiCtx* ctx, int64_t n, const double* x, const double* y, const double* z,
                              const double* h, const double* bounds6, double spacing_fraction,
                              double coverage_radius_factor, int64_t capacity, double* out_x, double* out_y,
                              double* out_z, int32_t* out_id, int64_t* n_added);

/* lloyd_step (src/point_set.cpp:265-293): every site the reference's Voro++ container keeps (see
 * kiwi_cartesian_map) moves to the centroid of its Voronoi cell clipped to the domain; the moved sites come
 * out in the container's walk order (blocks in index order, each block's sites in input order), ids carried
 * along (ids may be NULL: the input index).  out_id / out_xyz (3 per site) / out_volume (the cell volumes,
 * may be NULL) must hold n entries; *n_out receives the count, *n_failed (may be NULL) the kept sites whose
 * cell could not be built (dropped, as Voro++ drops a cell it cannot compute).  block_scale_factor: as for
 * kiwi_cartesian_map.  Host arrays. */
int kiwi_lloyd_step(KiwiCtx* ctx, int64_t n, const int32_t* ids, const double* xyz, const double* bounds6,
                    double block_scale_factor, int32_t* out_id, double* out_xyz, double* out_volume, int64_t* n_out,
                    int64_t* n_failed, KiwiStats* stats);

/* ---- cartesian-map stage (run_cartesian_map_stage's point location, src/cartesian_map.cpp:84-200) ---- */
/* Every cell centre of a resolution^3 grid over bounds6 takes the values of its nearest site (the Voronoi
 * cell it lies in: container::find_voronoi_cell) and that site's id.  Sites (3 doubles each, host arrays)
 * the reference's container drops are ignored: outside bounds6, or in a block index past the last (a site
 * on an upper wall can be; block_scale_factor is grid_blocks.block_scale_factor, 0 = its default 3, which
 * sets the container's block grid); site_id (may be NULL: the site index) gives the
 * ids written to voronoi_cell_id; cell_density / cell_vx / cell_vy / cell_vz hold each site's mapping row and
 * mapped (may be NULL: all) marks the sites that have one.  Outputs are host arrays of resolution^3 in the
 * x-major order (ix*res + iy)*res + iz; cells with no site (no sites at all) keep 0 and id 0, cells whose
 * site has no mapping row keep 0 with the site's id.  counts2 (may be NULL) receives those two counts (the
 * reference's "unresolved" and "unmapped" warnings).  Exactly equidistant sites resolve to the smallest
 * site index. */
int kiwi_cartesian_map(KiwiCtx* ctx, int64_t n_sites, const double* site_xyz, const int32_t* site_id,
                       const double* cell_density, const double* cell_vx, const double* cell_vy,
                       const double* cell_vz, const uint8_t* mapped, const double* bounds6, int32_t resolution,
                       double block_scale_factor, double* density, double* vx, double* vy, double* vz,
                       int32_t* voronoi_cell_id, int64_t* counts2, KiwiStats* stats);

#ifdef __cplusplus
}
#endif
#endif
