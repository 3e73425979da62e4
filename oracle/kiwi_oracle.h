/* CPU oracle for the KIWI kernel-integral hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, all-FP64 restatement of the reference's algorithm, written to follow its arithmetic
 * operation by operation so that its results can stand in for the reference's own CPU output.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it, and only as the
 * checker: nothing in the product (kiwi_b200/) links, loads or calls it.
 *
 * Parity pin: tests/test_oracle_pins.py checks this file against the reference's own known answers
 * (tools/test_generic_kernel.cpp:163-297: normalisation, brute-force quadrature, box-mass identities)
 * and, where the reference has been built from its sources by oracle/Makefile into oracle/_ref/,
 * against the reference library itself.
 */
#ifndef KIWI_ORACLE_H
#define KIWI_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- scalar tiers ---------------------------------------------------------------------------- */

/* full_integral_new(h, phi, r0, R_0): src/kernel_integral.cpp:410-418 */
double or_full_integral_new(double h, double phi, double r0, double R_0);
/* generic_full_integral(K, H, phi, r0, R_0): src/kernel_integral_generic.cpp:216-221 */
double or_generic_full_integral(int kernel, double H, double phi, double r0, double R_0);
/* gridded_integral on the canonical in-memory table: src/kernel_integral.cpp:57-190 */
double or_gridded_integral(double h, double phi, double r0, double R_0);

/* compute_face_integral{,_generic}: src/kernel_integral.cpp:471-662.
 * kernel < 0: cubic closed form with support 2h (tabulated != 0 selects the lookup table);
 * kernel >= 0: generic path with support H = support (h is unused). */
double or_face_integral(double x0, double y0, double z0, int kernel, double h, double support, int tabulated,
                        const double* verts, int n, int* out_vert);

/* Generic-kernel tier internals, exposed for the continuity pin (tools/test_generic_kernel.cpp:224-238). */
int or_generic_edge_breaks(int kernel, double H, double r0, double R_0, double* phi_end, int max_n);
double or_generic_vertex(int kernel, double H, double r0, double R_0, double phi);

/* ---- sph-to-grid stage (src/cartesian_grid.cpp:76-321) --------------------------------------- */

typedef struct OrStats {
    int64_t bbox_pairs;      /* (particle, cell) pairs in the clamped bounding boxes */
    int64_t sphere_pairs;    /* of those, cells whose closest point is within the support radius */
    int64_t skipped_outside; /* particles whose support box misses the grid */
    int64_t neg_clamped;     /* pairs with Msum < 0 clamped to 0 */
    int64_t neg_warned;      /* of those, Msum <= -0.01 */
} OrStats;

/* kernel < 0: cubic fast path; else generic table kernel index (0..5) with support = support_in_h*h.
 * If mass_out (4 arrays) is non-null, the raw per-cell sums m*Msum, m*Msum*v are written there too.
 * p_begin/p_end select a particle sub-range for the loop (the mean velocity still uses all n). */
int or_sph_to_grid(int64_t n, const double* x, const double* y, const double* z, const double* vx,
                   const double* vy, const double* vz, const double* m, const double* h, const double bounds[6],
                   int nx, int ny, int nz, int kernel, double support_in_h, int tabulated, int64_t p_begin,
                   int64_t p_end, double* density, double* gvx, double* gvy, double* gvz, double* raw4,
                   OrStats* stats);

/* ---- Voronoi map stage (src/mapping.cpp:105-206, 400-502) ----------------------------------- */

/* Cell geometry in CSR form (the plain-data equivalent of CellFaceGeometry, src/mapping.cpp:49-54):
 * cell c has faces face_off[c]..face_off[c+1]-1; face f has vertices vert_off[f]..vert_off[f+1]-1 with
 * absolute coordinates vxyz[3*v..3*v+2] (already site + relative offset, as src/mapping.cpp:168-175 builds
 * them); face_nbr[f] is the neighbouring cell index or -1 for a wall / unresolved neighbour. */
int or_map_voronoi(int64_t n, const int32_t* home_cell, const double* x, const double* y, const double* z,
                   const double* vx, const double* vy, const double* vz, const double* m, const double* h,
                   int64_t n_cells, const int64_t* face_off, const int64_t* vert_off, const double* vxyz,
                   const int32_t* face_nbr, const double* volume, int kernel, double support_in_h, int tabulated,
                   double* density, double* gvx, double* gvy, double* gvz, double* raw4, int64_t* visited_pairs);

#ifdef __cplusplus
}
#endif
#endif
