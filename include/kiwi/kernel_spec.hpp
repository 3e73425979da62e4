// kiwi_b200's C++ drop-in for the reference's kernel tables (include/kiwi/kernel_spec.hpp:18-44): the same
// struct, field for field and in the same order, and the same lookup functions, served by libkiwi_b200.so.
// The values are the exact rationals of the six kernel definitions rounded once to double
// (kiwi_b200/tables/gen_kernel_tables.py), equal to the reference's kKernels bit for bit.
#pragma once

#include <string>
#include <vector>

namespace kiwi {

struct KernelSpec {
    static constexpr int MAX_REGIONS = 4;  // pieces + 1
    static constexpr int NI = 15;          // exponents i = 1, 0, -1, ..., -13 at index 1 - i
    static constexpr int NB = 16;          // powers of q0 in the B polynomials

    const char* key;   // "M4", "M5", "M6", "WC2", "WC4", "WC6"
    const char* name;  // "Cubic spline", ...
    int nreg;          // regions = pieces + 1
    double c[MAX_REGIONS];  // piece boundaries in units of the support radius H; the last one is 1
    double A2_pi, A3_pi;    // 2-D and 3-D normalisation constants times pi
    double radkern;         // H in units of the smoothing length h
    double hfact;           // h = hfact (m / rho)^(1/3)
    double a[MAX_REGIONS][NI];               // vertex-pyramid series coefficients per region
    double B[MAX_REGIONS][MAX_REGIONS][NB];  // wall polynomials per (wall region, vertex region)
};

// A kernel by key or alias ("M4", "cubic_spline", "wendland_c4", ...); throws std::invalid_argument for an
// unknown name, as the reference does (src/kernel_spec_data.cpp:175-187).
const KernelSpec& get_kernel(const std::string& name);

// The six kernels in table order.
const std::vector<const KernelSpec*>& all_kernels();

}  // namespace kiwi
