// Test-only: the compute of the reference's sph-to-grid stage (src/cartesian_grid.cpp:149-347) as a KIWI
// maintainer replaces it with kiwi_b200 (INTEGRATION.md's replacement of the particle loop): a plain_ascii
// snapshot in (9 columns per particle: x y z vx vy vz m h rho), one kiwi_sph_to_grid call, the grid written
// with kiwi_save_cartesian_grid (the VGTCGRD2 file of save_cartesian_grid).  Compiled and run by
// tests/test_gpu_cpp_dropin.py.
//
// Usage: sph_to_grid_stage <snapshot> <out.dat> x_min x_max y_min y_max z_min z_max nx ny nz [kernel]
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "kiwi_b200.h"

static void kiwi_check(KiwiCtx* ctx, int rc) {
    if (rc != KIWI_OK) throw std::runtime_error(kiwi_last_error(ctx));
}

int main(int argc, char** argv) {
    try {
        if (argc < 12) throw std::runtime_error("usage: sph_to_grid_stage <snapshot> <out.dat> bounds[6] nx ny nz [kernel]");
        std::vector<double> x, y, z, vx, vy, vz, m, h;
        std::ifstream in(argv[1]);
        double c[9];
        while (in >> c[0] >> c[1] >> c[2] >> c[3] >> c[4] >> c[5] >> c[6] >> c[7] >> c[8]) {
            x.push_back(c[0]); y.push_back(c[1]); z.push_back(c[2]);
            vx.push_back(c[3]); vy.push_back(c[4]); vz.push_back(c[5]);
            m.push_back(c[6]); h.push_back(c[7]);
        }
        double b[6];
        for (int i = 0; i < 6; ++i) b[i] = std::strtod(argv[3 + i], nullptr);
        const int nx = std::atoi(argv[9]), ny = std::atoi(argv[10]), nz = std::atoi(argv[11]);
        const char* kernel = argc > 12 ? argv[12] : "cubic_spline";
        const size_t nc = (size_t)nx * ny * nz;
        std::vector<double> density(nc), gvx(nc), gvy(nc), gvz(nc);

        // -- the replacement of the reference's per-thread grids, particle loop and reduction
        KiwiCtx* ctx = nullptr;
        if (kiwi_ctx_create(0, &ctx) != KIWI_OK) throw std::runtime_error("kiwi_b200: no usable sm_100 GPU");
        KiwiParticles p{(int64_t)x.size(), x.data(), y.data(), z.data(), vx.data(), vy.data(), vz.data(), m.data(),
                        h.data()};
        KiwiCartGrid g{{b[0], b[1], b[2], b[3], b[4], b[5]}, nx, ny, nz};
        KiwiKernelSel k{kiwi_kernel_index(kernel), 0.0, 0, 0};
        KiwiStats st{};
        kiwi_check(ctx, kiwi_sph_to_grid(ctx, &p, &g, &k, KIWI_FP64, density.data(), gvx.data(), gvy.data(),
                                         gvz.data(), nullptr, &st));
        std::cerr << "[kiwi] sph-to-grid: " << st.skipped_outside
                  << " particle(s)' kernel support did not overlap the grid at all\n";
        kiwi_ctx_destroy(ctx);
        // -- unchanged: the reference's writer
        char err[256] = {0};
        if (kiwi_save_cartesian_grid(argv[2], nx, ny, nz, b, density.data(), gvx.data(), gvy.data(), gvz.data(), err,
                                     sizeof err) != KIWI_OK)
            throw std::runtime_error(err);
        return 0;
    } catch (const std::exception& e) {
        std::cerr << "[kiwi] error: " << e.what() << "\n";
        return 1;
    }
}
