// kiwi_b200's C++ drop-in for the reference's integrator dispatch (include/kiwi/kernel_integrator.hpp:14-45):
// the same struct and rule -- the generic face integral iff the configuration asks for a kernel other than
// the cubic spline, another support radius or the generic path; else the cubic fast path, analytic or
// tabulated.  make_kernel_integrator takes any configuration type with the reference's Config accessors
// (kernel_support_in_h(), use_generic_kernel_path(), kernel_spec()), so the reference's own Config works
// unchanged without this header depending on it.
#pragma once

#include <vector>

#include "kiwi/kernel_integral.hpp"
#include "kiwi/kernel_integral_generic.hpp"

namespace kiwi {

struct KernelIntegrator {
    const KernelSpec* generic = nullptr;  // null: the cubic-spline fast path
    double support_in_h = 2.0;            // support radius in units of h
    bool tabulated = false;               // the cubic fast path's lookup table
    const DensityLookupTable* table = nullptr;

    double face(double x0, double y0, double z0, double h, const std::vector<double>& vertices,
                int* out_vert = nullptr) const {
        if (generic) return compute_face_integral_generic(x0, y0, z0, *generic, support_in_h * h, vertices, out_vert);
        return compute_face_integral(x0, y0, z0, h, tabulated, table, vertices, out_vert);
    }

    double support(double h) const { return support_in_h * h; }
};

template <class ConfigT>
KernelIntegrator make_kernel_integrator(const ConfigT& cfg, bool tabulated, const DensityLookupTable* table) {
    KernelIntegrator ki;
    ki.support_in_h = cfg.kernel_support_in_h();
    if (cfg.use_generic_kernel_path()) {
        ki.generic = &cfg.kernel_spec();
    } else {
        ki.tabulated = tabulated;
        ki.table = table;
    }
    return ki;
}

}  // namespace kiwi
