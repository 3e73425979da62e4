// The C++ drop-in of the reference's kernel-integral layer (include/kiwi/kernel_spec.hpp,
// kernel_integral.hpp, kernel_integral_generic.hpp under this repository's include/kiwi/): each function
// forwards to libkiwi_b200.so's C ABI, whose sm_100a kernels evaluate it, on a context owned by the calling
// thread (created on the thread's first call, on device KIWI_B200_DEVICE or 0, destroyed at thread exit).
// Errors throw std::runtime_error carrying the library's message (std::invalid_argument for an unknown
// kernel name or a kernel table this library does not hold, as the reference's get_kernel throws).
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "kernel_tables.h"
#include "kiwi/kernel_integral.hpp"
#include "kiwi/kernel_integral_generic.hpp"
#include "kiwi/kernel_spec.hpp"
#include "../../include/kiwi_b200.h"

namespace {

static_assert(kiwi::KernelSpec::MAX_REGIONS == KIWI_MAX_REGIONS && kiwi::KernelSpec::NI == KIWI_NI &&
                  kiwi::KernelSpec::NB == KIWI_NB,
              "KernelSpec and the library's kernel tables have the same shape");

struct ThreadCtx {
    KiwiCtx* ctx = nullptr;
    // identity of the host table last copied into this context's density table
    const double* table_data = nullptr;
    size_t table_size = 0;
    ~ThreadCtx() {
        if (ctx) kiwi_ctx_destroy(ctx);
    }
};

ThreadCtx& tls() {
    static thread_local ThreadCtx t;
    return t;
}

KiwiCtx* ctx() {
    ThreadCtx& t = tls();
    if (!t.ctx) {
        const char* dev = std::getenv("KIWI_B200_DEVICE");
        const int rc = kiwi_ctx_create(dev ? std::atoi(dev) : 0, &t.ctx);
        if (rc != KIWI_OK) {
            t.ctx = nullptr;
            throw std::runtime_error("kiwi_b200: no usable sm_100 GPU for the kernel-integral layer (error " +
                                     std::to_string(rc) + ")");
        }
    }
    return t.ctx;
}

void check(int rc) {
    if (rc != KIWI_OK) throw std::runtime_error(std::string("kiwi_b200: ") + kiwi_last_error(tls().ctx));
}

// The six kernels as KernelSpec, copied from the library's tables once.
const kiwi::KernelSpec* specs() {
    static const std::vector<kiwi::KernelSpec> v = [] {
        std::vector<kiwi::KernelSpec> out(KIWI_NUM_KERNELS);
        for (int i = 0; i < KIWI_NUM_KERNELS; ++i) {
            const KiwiKernelTable& t = kiwi_kernel_tables[i];
            kiwi::KernelSpec& s = out[i];
            s.key = t.key;
            s.name = t.name;
            s.nreg = t.nreg;
            std::memcpy(s.c, t.c, sizeof s.c);
            s.A2_pi = t.A2_pi;
            s.A3_pi = t.A3_pi;
            s.radkern = t.radkern;
            s.hfact = t.hfact;
            std::memcpy(s.a, t.a, sizeof s.a);
            std::memcpy(s.B, t.B, sizeof s.B);
        }
        return out;
    }();
    return v.data();
}

// Index of K in the library's tables: K itself (get_kernel / all_kernels) or a copy of one of them.
int kernel_index(const kiwi::KernelSpec& K) {
    const kiwi::KernelSpec* s = specs();
    if (&K >= s && &K < s + KIWI_NUM_KERNELS) return (int)(&K - s);
    const int i = K.key ? kiwi_kernel_index(K.key) : -1;
    if (i < 0 || std::memcmp(K.a, s[i].a, sizeof K.a) != 0 || std::memcmp(K.B, s[i].B, sizeof K.B) != 0)
        throw std::invalid_argument("kiwi_b200: kernel table '" + std::string(K.key ? K.key : "?") +
                                    "' is not one of the library's six kernels");
    return i;
}

// The table's contents on the GPU: copied when the caller's table differs from the last one copied (by
// its storage and size; a table changed in place after use is not seen).
void table_on_device(const kiwi::DensityLookupTable& t) {
    KiwiCtx* c = ctx();
    ThreadCtx& s = tls();
    if (s.table_data == t.values.data() && s.table_size == t.values.size() && !t.values.empty()) return;
    KiwiDensityTableInfo info;
    info.nr01 = t.nr01; info.nR_01 = t.nR_01; info.nphi1 = t.nphi1;
    info.nr02 = t.nr02; info.nR_02 = t.nR_02; info.nphi2 = t.nphi2;
    info.rl = t.rl; info.mul = t.mul; info.cphil = t.cphil;
    info.n_values = (int64_t)t.values.size();
    check(kiwi_density_table_set(c, &info, t.values.data()));
    s.table_data = t.values.data();
    s.table_size = t.values.size();
}

// The context's table copied back into a host DensityLookupTable.
kiwi::DensityLookupTable read_table() {
    KiwiCtx* c = ctx();
    KiwiDensityTableInfo info;
    check(kiwi_density_table_info(c, &info));
    kiwi::DensityLookupTable t;
    t.nr01 = info.nr01; t.nR_01 = info.nR_01; t.nphi1 = info.nphi1;
    t.nr02 = info.nr02; t.nR_02 = info.nR_02; t.nphi2 = info.nphi2;
    t.rl = info.rl; t.mul = info.mul; t.cphil = info.cphil;
    t.nr0 = t.nr01 + t.nr02;
    t.nR_0 = t.nR_01 + t.nR_02;
    t.nphi = t.nphi1 + t.nphi2;
    t.values.resize((size_t)info.n_values);
    check(kiwi_density_table_read(c, t.values.data(), info.n_values));
    tls().table_data = t.values.data();
    tls().table_size = t.values.size();
    return t;
}

double face(const KiwiKernelSel& sel, double x0, double y0, double z0, double h, const std::vector<double>& v,
            int* out_vert) {
    if (v.size() < 9 || v.size() % 3 != 0)
        throw std::invalid_argument("kiwi_b200: a face needs at least 3 vertices given as x, y, z triples");
    const double particle[4] = {x0, y0, z0, h};
    const int64_t off[2] = {0, (int64_t)(v.size() / 3)};
    double out = 0.0;
    int32_t ov = 0;
    check(kiwi_face_integral_batch(ctx(), &sel, 1, particle, off, v.data(), &out, &ov));
    if (out_vert) *out_vert = ov;
    return out;
}

}  // namespace

namespace kiwi {

const KernelSpec& get_kernel(const std::string& name) {
    const int i = kiwi_kernel_index(name.c_str());
    if (i < 0)
        throw std::invalid_argument("unknown kernel '" + name +
                                    "' (known: cubic_spline, quartic_spline, quintic_spline, wendland_c2, "
                                    "wendland_c4, wendland_c6)");
    return specs()[i];
}

const std::vector<const KernelSpec*>& all_kernels() {
    static const std::vector<const KernelSpec*> v = [] {
        std::vector<const KernelSpec*> out;
        for (int i = 0; i < KIWI_NUM_KERNELS; ++i) out.push_back(specs() + i);
        return out;
    }();
    return v;
}

double DensityLookupTable::at(int i, int j, int k) const {
    return values[((size_t)i * (nR_0 + 1) + j) * (nphi + 1) + k];
}

double& DensityLookupTable::at(int i, int j, int k) { return values[((size_t)i * (nR_0 + 1) + j) * (nphi + 1) + k]; }

DensityLookupTable load_density_table(const std::string& path) {
    check(kiwi_density_table_load(ctx(), path.c_str()));
    return read_table();
}

DensityLookupTable generate_density_table() {
    check(kiwi_density_table_generate(ctx()));
    return read_table();
}

double gridded_integral(const DensityLookupTable& table, double h, double phi, double r0_old, double R_0_old) {
    table_on_device(table);
    double out = 0.0;
    check(kiwi_gridded_integral_batch(ctx(), 1, &h, &phi, &r0_old, &R_0_old, &out, nullptr));
    return out;
}

double full_integral_new(double h, double phi, double r0, double R_0) {
    double out = 0.0;
    check(kiwi_full_integral_batch(ctx(), -1, 1, &h, &phi, &r0, &R_0, &out));
    return out;
}

WallIntegralConstants compute_wall_constants(double h, double r0) {
    double w[KIWI_CUBIC_WALL_DOUBLES], e[KIWI_CUBIC_EDGE_DOUBLES];
    const double R0 = 0.0;
    check(kiwi_tier_constants_batch(ctx(), -1, 1, &h, &r0, &R0, w, e));
    WallIntegralConstants c;
    c.valid = w[0] != 0.0;
    c.r0 = w[1]; c.h = w[2]; c.h2 = w[3]; c.r03 = w[4]; c.r0h2 = w[5]; c.r0h3 = w[6];
    c.r0h_2 = w[7]; c.r0h_3 = w[8]; c.B1 = w[9]; c.B2 = w[10]; c.B3 = w[11];
    return c;
}

EdgeIntegralConstants compute_edge_constants(const WallIntegralConstants& wall, double R_0) {
    double w[KIWI_CUBIC_WALL_DOUBLES], e[KIWI_CUBIC_EDGE_DOUBLES];
    check(kiwi_tier_constants_batch(ctx(), -1, 1, &wall.h, &wall.r0, &R_0, w, e));
    EdgeIntegralConstants c;
    c.valid = wall.valid && e[0] != 0.0;
    c.R_0 = e[1]; c.a = e[2]; c.a2 = e[3]; c.D2 = e[4]; c.D3 = e[5];
    return c;
}

double vertex_integral(const WallIntegralConstants& wall, const EdgeIntegralConstants& edge, double phi) {
    if (!wall.valid || !edge.valid) return 0.0;
    return full_integral_new(wall.h, phi, wall.r0, edge.R_0);
}

double compute_face_integral(double x0, double y0, double z0, double h, bool use_tabulated_integral,
                             const DensityLookupTable* table, const std::vector<double>& vertices, int* out_vert) {
    KiwiKernelSel sel{0, 2.0, 0, use_tabulated_integral ? 1 : 0};
    if (use_tabulated_integral) {
        if (!table) throw std::invalid_argument("kiwi_b200: the tabulated face integral needs a density table");
        table_on_device(*table);
    }
    return face(sel, x0, y0, z0, h, vertices, out_vert);
}

double compute_face_integral_generic(double x0, double y0, double z0, const KernelSpec& K, double H,
                                     const std::vector<double>& vertices, int* out_vert) {
    // support radius H given directly: smoothing length H with a support of 1 x H
    KiwiKernelSel sel{kernel_index(K), 1.0, 1, 0};
    return face(sel, x0, y0, z0, H, vertices, out_vert);
}

GenericWallConstants generic_wall_constants(const KernelSpec& K, double H, double r0) {
    const int k = kernel_index(K);
    double w[KIWI_GENERIC_WALL_DOUBLES], e[KIWI_GENERIC_EDGE_DOUBLES];
    const double R0 = 0.0;
    check(kiwi_tier_constants_batch(ctx(), k, 1, &H, &r0, &R0, w, e));
    GenericWallConstants c;
    c.valid = w[0] != 0.0;
    c.K = &K;
    c.H = w[1]; c.r0 = w[2]; c.q0 = w[3]; c.j = (int)w[4];
    for (int r = 0; r < KernelSpec::MAX_REGIONS; ++r) {
        for (int i = 0; i < KernelSpec::NI; ++i) c.coef[r][i] = w[5 + KernelSpec::NI * r + i];
        c.bphi[r] = w[5 + KernelSpec::NI * KernelSpec::MAX_REGIONS + r];
    }
    return c;
}

GenericEdgeConstants generic_edge_constants(const GenericWallConstants& wall, double R_0) {
    GenericEdgeConstants c;
    c.R_0 = R_0;
    if (!wall.valid || !wall.K) return c;
    const int k = kernel_index(*wall.K);
    double w[KIWI_GENERIC_WALL_DOUBLES], e[KIWI_GENERIC_EDGE_DOUBLES];
    check(kiwi_tier_constants_batch(ctx(), k, 1, &wall.H, &wall.r0, &R_0, w, e));
    c.valid = e[0] != 0.0;
    c.a = e[2]; c.a2 = e[3];
    c.nseg = (int)e[4];
    for (int s = 0; s < KernelSpec::MAX_REGIONS; ++s) {
        c.region[s] = (int)e[5 + s];
        c.phi_end[s] = e[5 + KernelSpec::MAX_REGIONS + s];
        c.offset[s] = e[5 + 2 * KernelSpec::MAX_REGIONS + s];
    }
    return c;
}

double generic_vertex_integral(const GenericWallConstants& wall, const GenericEdgeConstants& edge, double phi) {
    if (!wall.valid || !edge.valid || !wall.K) return 0.0;
    return generic_full_integral(*wall.K, wall.H, phi, wall.r0, edge.R_0);
}

double generic_full_integral(const KernelSpec& K, double H, double phi, double r0, double R_0) {
    double out = 0.0;
    check(kiwi_full_integral_batch(ctx(), kernel_index(K), 1, &H, &phi, &r0, &R_0, &out));
    return out;
}

}  // namespace kiwi
