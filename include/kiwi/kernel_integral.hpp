// kiwi_b200's C++ drop-in for the reference's cubic-spline kernel-integral layer
// (include/kiwi/kernel_integral.hpp:21-193): the same declarations, with every integral evaluated by
// libkiwi_b200.so's sm_100a kernels through its C ABI (include/kiwi_b200.h) on a per-thread GPU context
// (device 0, or KIWI_B200_DEVICE).  Each scalar call is one small GPU batch: the API exists for drop-in
// compatibility and tests; bulk work goes through the C ABI's sph-to-grid and map entry points.  Failures
// throw std::runtime_error with the library's message.  There is no CPU path: without a usable GPU every
// call throws.
#pragma once

#include <string>
#include <vector>

#include "kiwi/kernel_spec.hpp"

namespace kiwi {

// The reference's density lookup table (include/kiwi/kernel_integral.hpp:27-40): header fields, derived
// sizes, and the (nr0 + 2) x (nR_0 + 1) x (nphi + 1) values.
struct DensityLookupTable {
    int nr01 = 0, nR_01 = 0, nphi1 = 0;
    int nr02 = 0, nR_02 = 0, nphi2 = 0;
    double rl = 0, mul = 0, cphil = 0;
    int nr0 = 0, nR_0 = 0, nphi = 0;
    std::vector<double> values;

    double at(int i, int j, int k) const;
    double& at(int i, int j, int k);
};

// Reads a table file in the reference's text format (parsed and checked on the GPU side's loader).
DensityLookupTable load_density_table(const std::string& path);
// The canonical 251 x 301 x 301 table, generated on the GPU.
DensityLookupTable generate_density_table();
// Trilinear lookup in `table` (uploaded to the GPU on first use of that table's contents).
double gridded_integral(const DensityLookupTable& table, double h, double phi, double r0_old, double R_0_old);
// The closed-form vertex-pyramid integral of the cubic spline.
double full_integral_new(double h, double phi, double r0, double R_0);

// The three tiers of full_integral_new (include/kiwi/kernel_integral.hpp:108-131).  The constants are
// computed on the GPU; vertex_integral evaluates full_integral_new(wall.h, phi, wall.r0, edge.R_0), which
// is the same sequence of operations as the reference's tiers.
struct WallIntegralConstants {
    bool valid = false;
    double r0 = 0.0, h = 0.0;
    double h2 = 0.0, r03 = 0.0, r0h2 = 0.0, r0h3 = 0.0, r0h_2 = 0.0, r0h_3 = 0.0;
    double B1 = 0.0, B2 = 0.0, B3 = 0.0;
};

struct EdgeIntegralConstants {
    bool valid = false;
    double R_0 = 0.0;
    double a = 0.0, a2 = 0.0;
    double D2 = 0.0, D3 = 0.0;
};

WallIntegralConstants compute_wall_constants(double h, double r0);
EdgeIntegralConstants compute_edge_constants(const WallIntegralConstants& wall, double R_0);
double vertex_integral(const WallIntegralConstants& wall, const EdgeIntegralConstants& edge, double phi);

// Kernel mass of one planar convex face (absolute vertex coordinates, flattened xyz, in the winding the
// reference's face walk needs -- see its box_cell_faces) for a particle at (x0, y0, z0): the cubic spline
// with smoothing length h (support 2h), analytic or tabulated; out_vert (optional) receives the number of
// the face's edges whose closest point is at or beyond the support.
double compute_face_integral(double x0, double y0, double z0, double h, bool use_tabulated_integral,
                             const DensityLookupTable* table, const std::vector<double>& vertices,
                             int* out_vert = nullptr);

// The same for any kernel of kernel_spec.hpp with support radius H.
double compute_face_integral_generic(double x0, double y0, double z0, const KernelSpec& K, double H,
                                     const std::vector<double>& vertices, int* out_vert = nullptr);

}  // namespace kiwi
