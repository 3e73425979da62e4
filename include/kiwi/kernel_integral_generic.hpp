// kiwi_b200's C++ drop-in for the reference's generic-kernel tiers (include/kiwi/kernel_integral_generic.hpp:
// 27-56): the same structs and functions, computed by libkiwi_b200.so's sm_100a kernels (see
// kernel_integral.hpp for the calling model).  generic_vertex_integral evaluates
// generic_full_integral(*wall.K, wall.H, phi, wall.r0, edge.R_0), the same sequence of operations as the
// reference's tiers.
#pragma once

#include "kiwi/kernel_spec.hpp"

namespace kiwi {

struct GenericWallConstants {
    bool valid = false;
    const KernelSpec* K = nullptr;
    double H = 0.0, r0 = 0.0, q0 = 0.0;
    int j = 0;  // kernel region of q0 = r0 / H (1-based)
    double coef[KernelSpec::MAX_REGIONS][KernelSpec::NI];  // per vertex region: A3 a q0^(1-i) at index 1 - i
    double bphi[KernelSpec::MAX_REGIONS];                   // per vertex region: the coefficient of phi
};

struct GenericEdgeConstants {
    bool valid = false;
    double R_0 = 0.0, a = 0.0, a2 = 0.0;
    int nseg = 0;                              // kernel regions the edge line passes through
    int region[KernelSpec::MAX_REGIONS];       // the region of each segment
    double phi_end[KernelSpec::MAX_REGIONS];   // angle where each segment ends (the last at pi/2)
    double offset[KernelSpec::MAX_REGIONS];    // continuity offset of each segment
};

GenericWallConstants generic_wall_constants(const KernelSpec& K, double H, double r0);
GenericEdgeConstants generic_edge_constants(const GenericWallConstants& wall, double R_0);
double generic_vertex_integral(const GenericWallConstants& wall, const GenericEdgeConstants& edge, double phi);
double generic_full_integral(const KernelSpec& K, double H, double phi, double r0, double R_0);

}  // namespace kiwi
