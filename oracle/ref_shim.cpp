// C-ABI shim over the reference KIWI library, built from the reference's own sources by
// oracle/Makefile into oracle/_ref/libkiwi_ref.so -- TEST INFRASTRUCTURE ONLY.
//
// It lets the tests and bench.py's CPU-baseline leg call the unmodified reference code:
//  - the scalar integral API (include/kiwi/kernel_integral.hpp:72-193,
//    include/kiwi/kernel_integral_generic.hpp:47-56);
//  - run_sph_to_grid_stage (src/cartesian_grid.cpp:76) on arrays, through a temporary plain_ascii
//    snapshot (written with 17 significant digits, so it reads back bit-exact) and a Config built in code;
//  - the Voronoi cell geometry exactly as src/mapping.cpp:222-269 extracts it from Voro++, and
//    run_mapping_stage (src/mapping.cpp:331) on arrays.
#include <omp.h>
#include <unistd.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "kiwi/cartesian_grid.hpp"
#include "kiwi/snapshot.hpp"
#include "kiwi/config.hpp"
#include "kiwi/kernel_integral.hpp"
#include "kiwi/kernel_integral_generic.hpp"
#include "kiwi/kernel_integrator.hpp"
#include "kiwi/kernel_spec.hpp"
#include "kiwi/cartesian_map.hpp"
#include "kiwi/mapping.hpp"
#include "kiwi/point_set.hpp"
#include "kiwi/voro_grid.hpp"
#include "voro++.hh"

namespace {

const kiwi::KernelSpec& kernel_by_index(int k) { return *kiwi::all_kernels().at(k); }

std::string g_err;

std::string make_tmpdir() {
    char tmpl[] = "/tmp/kiwi_ref_XXXXXX";
    char* d = mkdtemp(tmpl);
    return d ? std::string(d) : std::string("/tmp");
}

void rm_rf(const std::string& dir) {
    std::string cmd = "rm -rf '" + dir + "'";
    int rc = std::system(cmd.c_str());
    (void)rc;
}

void write_snapshot(const std::string& path, long n, const double* x, const double* y, const double* z,
                    const double* vx, const double* vy, const double* vz, const double* m, const double* h) {
    FILE* f = std::fopen(path.c_str(), "w");
    for (long i = 0; i < n; ++i)
        std::fprintf(f, "%.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g 1\n", x[i], y[i], z[i], vx[i], vy[i],
                     vz[i], m[i], h[i]);
    std::fclose(f);
}

kiwi::Config base_config(const std::string& dir, const double b[6], const char* kernel, double support_in_h,
                         int generic_path) {
    kiwi::Config c;
    c.run_name = "ref";
    c.domain.x_min = b[0]; c.domain.x_max = b[1];
    c.domain.y_min = b[2]; c.domain.y_max = b[3];
    c.domain.z_min = b[4]; c.domain.z_max = b[5];
    c.input_snapshot = dir + "/snap.txt";
    c.input_snapshot_format = "plain_ascii";
    c.work_folder = dir + "/runs";
    c.kernel.name = kernel ? kernel : "cubic_spline";
    c.kernel.support_radius_in_h = support_in_h;
    c.kernel.generic_path = generic_path != 0;
    return c;
}

}  // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

double ref_full_integral_new(double h, double phi, double r0, double R_0) {
    return kiwi::full_integral_new(h, phi, r0, R_0);
}

double ref_generic_full_integral(int kernel, double H, double phi, double r0, double R_0) {
    return kiwi::generic_full_integral(kernel_by_index(kernel), H, phi, r0, R_0);
}

double ref_gridded_integral(double h, double phi, double r0, double R_0) {
    static kiwi::DensityLookupTable table = kiwi::generate_density_table();
    return kiwi::gridded_integral(table, h, phi, r0, R_0);
}

// load_density_table(path), then gridded_integral with it on n items.  0, or -1 with the reference's
// exception message in ref_last_error().
int ref_table_load_gridded(const char* path, int64_t n, const double* h, const double* phi, const double* r0,
                           const double* R_0, double* out) {
    try {
        const kiwi::DensityLookupTable t = kiwi::load_density_table(path);
        for (int64_t i = 0; i < n; ++i) out[i] = kiwi::gridded_integral(t, h[i], phi[i], r0[i], R_0[i]);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// The values of generate_density_table(), laid out as DensityLookupTable::at (out may be NULL to ask for
// their count).
int64_t ref_table_values(double* out) {
    static kiwi::DensityLookupTable table = kiwi::generate_density_table();
    const int64_t n = (int64_t)table.values.size();
    if (out)
        for (int64_t i = 0; i < n; ++i) out[i] = table.values[i];
    return n;
}

// kernel < 0: compute_face_integral (support 2h); else compute_face_integral_generic with H = support.
double ref_face_integral(double x0, double y0, double z0, int kernel, double h, double support, int tabulated,
                         const double* verts, int n, int* out_vert) {
    std::vector<double> v(verts, verts + 3 * n);
    if (kernel < 0) {
        static kiwi::DensityLookupTable table;
        static bool have = false;
        if (tabulated && !have) {
            table = kiwi::generate_density_table();
            have = true;
        }
        return kiwi::compute_face_integral(x0, y0, z0, h, tabulated != 0, &table, v, out_vert);
    }
    return kiwi::compute_face_integral_generic(x0, y0, z0, kernel_by_index(kernel), support, v, out_vert);
}

// run_sph_to_grid_stage on arrays. kernel: a kernel name accepted by get_kernel ("cubic_spline", ...).
int ref_sph_to_grid(long n, const double* x, const double* y, const double* z, const double* vx, const double* vy,
                    const double* vz, const double* m, const double* h, const double bounds[6], int nx, int ny,
                    int nz, const char* kernel, double support_in_h, int generic_path, int tabulated, int threads,
                    double* density, double* gvx, double* gvy, double* gvz) {
    std::string dir = make_tmpdir();
    try {
        write_snapshot(dir + "/snap.txt", n, x, y, z, vx, vy, vz, m, h);
        kiwi::Config c = base_config(dir, bounds, kernel, support_in_h, generic_path);
        c.cartesian_grid.resolution_x = nx;
        c.cartesian_grid.resolution_y = ny;
        c.cartesian_grid.resolution_z = nz;
        c.cartesian_grid.use_tabulated_integral = tabulated != 0;
        if (threads > 0) omp_set_num_threads(threads);
        kiwi::CartesianGridResult g = kiwi::run_sph_to_grid_stage(c);
        const size_t nc = static_cast<size_t>(nx) * ny * nz;
        std::memcpy(density, g.density.data(), nc * sizeof(double));
        std::memcpy(gvx, g.vx.data(), nc * sizeof(double));
        std::memcpy(gvy, g.vy.data(), nc * sizeof(double));
        std::memcpy(gvz, g.vz.data(), nc * sizeof(double));
    } catch (const std::exception& e) {
        g_err = e.what();
        rm_rf(dir);
        return -1;
    }
    rm_rf(dir);
    return 0;
}

// The reference's per-(particle, cell) work of run_sph_to_grid_stage (src/cartesian_grid.cpp:188-281)
// over the particles [p_begin, p_end), OpenMP-parallel over particles with schedule(dynamic, 256) as
// the reference's loop is, through the KernelIntegrator the reference's make_kernel_integrator builds
// (include/kiwi/kernel_integrator.hpp:35-45).  The six box faces are wound as src/cartesian_grid.cpp:54-72
// winds them.  Only the per-cell accumulation differs: each thread sums m*Msum into one scalar instead
// of a full-size grid replica, so that the time measured is that of the pair integrals.
// Returns wall seconds; *pairs_out = bounding-box pairs evaluated, *sphere_out = those whose cell's
// closest point lies within the support radius; *checksum = sum of m*Msum.
double ref_pair_sample(long n, const double* x, const double* y, const double* z, const double* m, const double* h,
                       const double bounds[6], int nx, int ny, int nz, const char* kernel, double support_in_h,
                       int generic_path, int threads, long p_begin, long p_end, long* pairs_out, long* sphere_out,
                       double* checksum) {
    std::string dir = make_tmpdir();
    kiwi::Config c = base_config(dir, bounds, kernel, support_in_h, generic_path);
    rm_rf(dir);
    kiwi::DensityLookupTable table;
    const kiwi::KernelIntegrator ki = kiwi::make_kernel_integrator(c, false, &table);
    if (threads > 0) omp_set_num_threads(threads);
    const double dpx = (bounds[1] - bounds[0]) / nx, dpy = (bounds[3] - bounds[2]) / ny, dpz = (bounds[5] - bounds[4]) / nz;
    const double hpx = 0.5 * dpx, hpy = 0.5 * dpy, hpz = 0.5 * dpz;
    long pairs = 0, sphere = 0;
    double sum = 0.0;
    if (p_end < 0 || p_end > n) p_end = n;
    const double t0 = omp_get_wtime();
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : pairs, sphere, sum)
    for (long i = p_begin; i < p_end; ++i) {
        if (h[i] <= 0.0) continue;
        const double radius = ki.support(h[i]);
        int ix0 = std::max(static_cast<int>(std::floor((x[i] - radius - bounds[0]) / dpx)), 0);
        int ix1 = std::min(static_cast<int>(std::floor((x[i] + radius - bounds[0]) / dpx)), nx - 1);
        int iy0 = std::max(static_cast<int>(std::floor((y[i] - radius - bounds[2]) / dpy)), 0);
        int iy1 = std::min(static_cast<int>(std::floor((y[i] + radius - bounds[2]) / dpy)), ny - 1);
        int iz0 = std::max(static_cast<int>(std::floor((z[i] - radius - bounds[4]) / dpz)), 0);
        int iz1 = std::min(static_cast<int>(std::floor((z[i] + radius - bounds[4]) / dpz)), nz - 1);
        for (int ix = ix0; ix <= ix1; ++ix) {
            const double cx = bounds[0] + (ix + 0.5) * dpx;
            for (int iy = iy0; iy <= iy1; ++iy) {
                const double cy = bounds[2] + (iy + 0.5) * dpy;
                for (int iz = iz0; iz <= iz1; ++iz) {
                    const double cz = bounds[4] + (iz + 0.5) * dpz;
                    const double xm = cx - hpx, xp = cx + hpx, ym = cy - hpy, yp = cy + hpy, zm = cz - hpz, zp = cz + hpz;
                    std::vector<double> faces[6];
                    faces[0] = {xp, ym, zp, xp, yp, zp, xp, yp, zm, xp, ym, zm};
                    faces[1] = {xm, yp, zm, xm, yp, zp, xm, ym, zp, xm, ym, zm};
                    faces[2] = {xp, yp, zm, xp, yp, zp, xm, yp, zp, xm, yp, zm};
                    faces[3] = {xm, ym, zp, xp, ym, zp, xp, ym, zm, xm, ym, zm};
                    faces[4] = {xm, yp, zp, xp, yp, zp, xp, ym, zp, xm, ym, zp};
                    faces[5] = {xp, ym, zm, xp, yp, zm, xm, yp, zm, xm, ym, zm};
                    double Msum = 0.0;
                    for (int f = 0; f < 6; ++f) Msum += ki.face(x[i], y[i], z[i], h[i], faces[f]);
                    if (Msum < 0.0) Msum = 0.0;
                    sum += Msum * m[i];
                    ++pairs;
                    {
                        const double ex = std::max(std::fabs(x[i] - cx) - hpx, 0.0), ey = std::max(std::fabs(y[i] - cy) - hpy, 0.0),
                                     ez = std::max(std::fabs(z[i] - cz) - hpz, 0.0);
                        if (ex * ex + ey * ey + ez * ez < radius * radius) ++sphere;
                    }
                }
            }
        }
    }
    const double t1 = omp_get_wtime();
    if (pairs_out) *pairs_out = pairs;
    if (sphere_out) *sphere_out = sphere;
    if (checksum) *checksum = sum;
    return t1 - t0;
}

int ref_max_threads() { return omp_get_max_threads(); }

// load_sph_snapshot (src/snapshot.cpp:511) on a snapshot file, format detected as the reference detects it.
// With out == nullptr returns the particle count; else fills out[8][n] (x y z vx vy vz m h) and returns n.
// Returns -1 on error (ref_last_error()).
long ref_load_snapshot(const char* path, double hfact, double* const* out) {
    try {
        kiwi::SPHSnapshot s = kiwi::load_sph_snapshot(path, "auto", hfact);
        const long n = static_cast<long>(s.size());
        if (out) {
            const std::vector<double>* cols[8] = {&s.x, &s.y, &s.z, &s.vx, &s.vy, &s.vz, &s.m, &s.h};
            for (int k = 0; k < 8; ++k) std::memcpy(out[k], cols[k]->data(), n * sizeof(double));
        }
        return n;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// ---- Voronoi --------------------------------------------------------------------------------------

struct RefVoronoi {
    std::vector<int> id;
    std::vector<double> site;               // 3 per cell
    std::vector<double> volume;
    std::vector<long> face_off, vert_off;   // CSR
    std::vector<double> vxyz;               // absolute vertex coordinates
    std::vector<int> face_nbr;              // resolved cell index or -1
    std::vector<int> home;                  // per particle: cell index or -1
    std::vector<double> density, vx, vy, vz;
    // run_map == 2: run_inverse_mapping_test_stage's rows (per particle, snapshot order), its totals and
    // the cell masses it used (density x volume of the cached mapping rows, geometry order)
    std::vector<double> inv_recovered, inv_coverage, inv_cell_mass;
    double inv_totals[3] = {0.0, 0.0, 0.0};
};

// Tessellates the point set the way src/mapping.cpp:222-269 does (same container and block setup) into R's
// CSR geometry, vertices made absolute as src/mapping.cpp:168-175 does, plus each particle's home cell as
// src/mapping.cpp:434-439 finds it; returns the largest site id.
static int tessellate(const kiwi::Config& c, const kiwi::PointSet& pts, long n, const double* x, const double* y,
                      const double* z, RefVoronoi* R, std::vector<int>& reverse) {
    const kiwi::Domain& d = c.domain;
    voro::pre_container pcon(d.x_min, d.x_max, d.y_min, d.y_max, d.z_min, d.z_max, false, false, false);
    for (size_t i = 0; i < pts.size(); ++i) pcon.put(pts.id[i], pts.x[i], pts.y[i], pts.z[i]);
    int bx, by, bz;
    kiwi::guess_scaled_blocks(pcon, c.grid_blocks.block_scale_factor, bx, by, bz);
    voro::container con(d.x_min, d.x_max, d.y_min, d.y_max, d.z_min, d.z_max, bx, by, bz, false, false, false, 8);
    pcon.setup(con);
    int max_id = 0;
    for (int pid : pts.id) max_id = std::max(max_id, pid);
    reverse.assign(max_id + 1, -1);
    std::vector<std::vector<int>> fvert_all, nlist_all;
    std::vector<std::vector<double>> fcoord_all;
    voro::voronoicell_neighbor cell;
    voro::c_loop_all clo(con);
    double px, py, pz;
    if (clo.start()) do {
        if (con.compute_cell(cell, clo)) {
            int idx = static_cast<int>(R->id.size());
            R->id.push_back(clo.pid());
            reverse[clo.pid()] = idx;
            clo.pos(px, py, pz);
            R->site.push_back(px);
            R->site.push_back(py);
            R->site.push_back(pz);
            std::vector<int> fv, nl;
            std::vector<double> fc;
            cell.face_vertices(fv);
            cell.vertices(fc);
            cell.neighbors(nl);
            R->volume.push_back(cell.volume());
            fvert_all.push_back(std::move(fv));
            fcoord_all.push_back(std::move(fc));
            nlist_all.push_back(std::move(nl));
        }
    } while (clo.inc());
    R->face_off.push_back(0);
    R->vert_off.push_back(0);
    for (size_t ci = 0; ci < R->id.size(); ++ci) {
        const std::vector<int>& fv = fvert_all[ci];
        const std::vector<double>& fc = fcoord_all[ci];
        const std::vector<int>& nl = nlist_all[ci];
        const double sx = R->site[3 * ci], sy = R->site[3 * ci + 1], sz = R->site[3 * ci + 2];
        size_t it = 0;
        int fi = 0;
        while (it < fv.size()) {
            int cnt = fv[it];
            for (int k = 0; k < cnt; ++k) {
                int ci2 = fv[it + 1 + k];
                R->vxyz.push_back(fc[3 * ci2] + sx);
                R->vxyz.push_back(fc[3 * ci2 + 1] + sy);
                R->vxyz.push_back(fc[3 * ci2 + 2] + sz);
            }
            R->vert_off.push_back(R->vert_off.back() + cnt);
            int nb = nl[fi];
            R->face_nbr.push_back(nb >= 0 && nb <= max_id ? reverse[nb] : -1);
            it += cnt + 1;
            ++fi;
        }
        R->face_off.push_back(R->face_off.back() + fi);
    }
    for (long i = 0; i < n; ++i) {
        double fx, fy, fz;
        int sid;
        bool found = con.find_voronoi_cell(x[i], y[i], z[i], fx, fy, fz, sid);
        R->home.push_back((found && sid >= 0 && sid <= max_id) ? reverse[sid] : -1);
    }
    return max_id;
}

// Builds the cell geometry (tessellate) of the final point set (after buffer/Lloyd) -- taken from
// run_point_set_stage on the same snapshot, as run_mapping_stage does.  With run_map, then runs
// run_mapping_stage itself and keeps its per-cell rows (matched by site id to the geometry order).  With
// run_map == 2, runs run_inverse_mapping_test_stage after it in the same work folder, as
// `kiwi inverse-mapping-test` does, and returns instead the geometry that stage tessellated (from the point
// set cached by the forward stage), with the cell masses it used and its per-particle results.
void* ref_voronoi_build(long n, const double* x, const double* y, const double* z, const double* vx,
                        const double* vy, const double* vz, const double* m, const double* h,
                        const double bounds[6], int buffer_enabled, double spacing_fraction, int lloyd_iterations,
                        const char* kernel, double support_in_h, int generic_path, int threads, int run_map) {
    std::string dir = make_tmpdir();
    auto* R = new RefVoronoi();
    try {
        write_snapshot(dir + "/snap.txt", n, x, y, z, vx, vy, vz, m, h);
        kiwi::Config c = base_config(dir, bounds, kernel, support_in_h, generic_path);
        c.buffer.enabled = buffer_enabled != 0;
        c.buffer.strategy = "coverage_grid";
        if (spacing_fraction > 0) c.buffer.coverage_grid.spacing_fraction = spacing_fraction;
        c.lloyd.iterations = lloyd_iterations;
        if (threads > 0) omp_set_num_threads(threads);
        kiwi::PointSet pts = kiwi::run_point_set_stage(c);
        std::vector<int> reverse;
        int max_id = tessellate(c, pts, n, x, y, z, R, reverse);
        if (run_map) {
            // A fresh run of the stage in its own work folder, as `kiwi map` on an empty folder runs it:
            // it recomputes the point set and uses it in memory (reusing the cached point-set file above
            // would give it the 15-digit rounded points instead).
            kiwi::Config cm = c;
            cm.work_folder = dir + "/runs_map";
            kiwi::MappingResult mr = kiwi::run_mapping_stage(cm);
            const size_t nc = R->id.size();
            R->density.assign(nc, 0.0);
            R->vx.assign(nc, 0.0);
            R->vy.assign(nc, 0.0);
            R->vz.assign(nc, 0.0);
            for (const auto& row : mr.cells) {
                if (row.id < 0 || row.id > max_id || reverse[row.id] < 0) continue;
                int ci = reverse[row.id];
                R->density[ci] = row.density;
                R->vx[ci] = row.vx;
                R->vy[ci] = row.vy;
                R->vz[ci] = row.vz;
            }
            if (run_map == 2) {
                kiwi::InverseMappingTestResult ir = kiwi::run_inverse_mapping_test_stage(cm);
                kiwi::MappingResult cached = kiwi::run_mapping_stage(cm);       // the rows the stage read
                kiwi::PointSet cached_pts = kiwi::run_point_set_stage(cm);      // the points it tessellated
                auto* G = new RefVoronoi();
                max_id = tessellate(cm, cached_pts, n, x, y, z, G, reverse);
                G->inv_cell_mass.assign(G->id.size(), 0.0);
                for (const auto& row : cached.cells) {
                    if (row.id < 0 || row.id > max_id || reverse[row.id] < 0) continue;
                    G->inv_cell_mass[reverse[row.id]] = row.density * row.volume;
                }
                for (const auto& p : ir.particles) {
                    G->inv_recovered.push_back(p.m_recovered);
                    G->inv_coverage.push_back(p.coverage_fraction);
                }
                G->inv_totals[0] = ir.total_original_mass;
                G->inv_totals[1] = ir.total_grid_mass;
                G->inv_totals[2] = ir.total_recovered_mass;
                delete R;
                R = G;
            }
        }
    } catch (const std::exception& e) {
        g_err = e.what();
        rm_rf(dir);
        delete R;
        return nullptr;
    }
    rm_rf(dir);
    return R;
}

// run_cartesian_map_stage (src/cartesian_map.cpp:84-200) on a fresh work folder, plus the point set and the
// mapping rows it used, each recomputed the same way in a fresh folder of its own (they are deterministic;
// reading them back from the stage's cache files would give their 15-digit rounded copies).  The stage
// locates against the point set it computed in memory, and its mapping stage tessellates the point set
// as cached by then.
struct RefCartMap {
    std::vector<int> pt_id;
    std::vector<double> pt_xyz;
    std::vector<int> row_id;
    std::vector<double> row_density, row_vx, row_vy, row_vz;
    std::vector<double> density, vx, vy, vz;
    std::vector<int> cell_id;
};

void* ref_cartesian_map(long n, const double* x, const double* y, const double* z, const double* vx,
                        const double* vy, const double* vz, const double* m, const double* h,
                        const double bounds[6], int resolution, int threads) {
    std::string dir = make_tmpdir();
    auto* R = new RefCartMap();
    try {
        write_snapshot(dir + "/snap.txt", n, x, y, z, vx, vy, vz, m, h);
        kiwi::Config c = base_config(dir, bounds, "cubic_spline", 0.0, 0);
        c.buffer.enabled = false;
        c.lloyd.iterations = 0;
        c.cartesian_map.resolution = resolution;
        if (threads > 0) omp_set_num_threads(threads);
        kiwi::Config c1 = c, c2 = c, c3 = c;
        c1.work_folder = dir + "/runs_points";
        c2.work_folder = dir + "/runs_mapping";
        c3.work_folder = dir + "/runs_cmap";
        kiwi::PointSet pts = kiwi::run_point_set_stage(c1);
        for (size_t i = 0; i < pts.size(); ++i) {
            R->pt_id.push_back(pts.id[i]);
            R->pt_xyz.push_back(pts.x[i]);
            R->pt_xyz.push_back(pts.y[i]);
            R->pt_xyz.push_back(pts.z[i]);
        }
        // as inside the stage: the point-set stage runs (and caches its points) first, so the mapping stage
        // tessellates the cached points
        kiwi::run_point_set_stage(c2);
        kiwi::MappingResult mr = kiwi::run_mapping_stage(c2);
        for (const auto& row : mr.cells) {
            R->row_id.push_back(row.id);
            R->row_density.push_back(row.density);
            R->row_vx.push_back(row.vx);
            R->row_vy.push_back(row.vy);
            R->row_vz.push_back(row.vz);
        }
        kiwi::CartesianMap cm = kiwi::run_cartesian_map_stage(c3);
        R->density = cm.density;
        R->vx = cm.vx;
        R->vy = cm.vy;
        R->vz = cm.vz;
        R->cell_id.assign(cm.voronoi_cell_id.begin(), cm.voronoi_cell_id.end());
    } catch (const std::exception& e) {
        g_err = e.what();
        rm_rf(dir);
        delete R;
        return nullptr;
    }
    rm_rf(dir);
    return R;
}

// Sizes: [points, mapping rows, grid cells]
void ref_cartesian_map_sizes(void* h, long* out3) {
    auto* R = static_cast<RefCartMap*>(h);
    out3[0] = (long)R->pt_id.size();
    out3[1] = (long)R->row_id.size();
    out3[2] = (long)R->cell_id.size();
}

void ref_cartesian_map_copy(void* h, int* pt_id, double* pt_xyz, int* row_id, double* row_density, double* row_vx,
                            double* row_vy, double* row_vz, double* density, double* vx, double* vy, double* vz,
                            int* cell_id) {
    auto* R = static_cast<RefCartMap*>(h);
    auto cp = [](auto* dst, const auto& v) {
        if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
    };
    cp(pt_id, R->pt_id);
    cp(pt_xyz, R->pt_xyz);
    cp(row_id, R->row_id);
    cp(row_density, R->row_density);
    cp(row_vx, R->row_vx);
    cp(row_vy, R->row_vy);
    cp(row_vz, R->row_vz);
    cp(density, R->density);
    cp(vx, R->vx);
    cp(vy, R->vy);
    cp(vz, R->vz);
    cp(cell_id, R->cell_id);
}

void ref_cartesian_map_free(void* h) { delete static_cast<RefCartMap*>(h); }

// The cartesian-map stage's point location over the x-slabs [ix_begin, ix_end) of a res^3 grid, as the
// stage runs it (src/cartesian_map.cpp:146-184: one Voro++ container per OpenMP thread, collapse(2) over
// ix, iy): the owning site id per cell into out_ids, and the wall time in seconds, container builds
// included (*build_s, if given, receives the container builds' share).  The CPU baseline of the GPU point
// location.
double ref_locate_sample(long n_sites, const int* ids, const double* xyz, const double b[6], int res, int ix_begin,
                         int ix_end, int threads, int* out_ids, double* build_s) {
    kiwi::Config c;
    c.domain.x_min = b[0]; c.domain.x_max = b[1];
    c.domain.y_min = b[2]; c.domain.y_max = b[3];
    c.domain.z_min = b[4]; c.domain.z_max = b[5];
    if (threads > 0) omp_set_num_threads(threads);
    const double t0 = omp_get_wtime();
    const int nt = omp_get_max_threads();
    std::vector<std::unique_ptr<voro::container>> cons(nt);
    const kiwi::Domain& d = c.domain;
#pragma omp parallel for
    for (int t = 0; t < nt; ++t) {
        voro::pre_container pcon(d.x_min, d.x_max, d.y_min, d.y_max, d.z_min, d.z_max, false, false, false);
        for (long i = 0; i < n_sites; ++i) pcon.put(ids[i], xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
        int bx, by, bz;
        kiwi::guess_scaled_blocks(pcon, c.grid_blocks.block_scale_factor, bx, by, bz);
        cons[t] = std::make_unique<voro::container>(d.x_min, d.x_max, d.y_min, d.y_max, d.z_min, d.z_max, bx, by, bz,
                                                    false, false, false, 8);
        pcon.setup(*cons[t]);
    }
    if (build_s) *build_s = omp_get_wtime() - t0;
    const double dpx = (d.x_max - d.x_min) / res, dpy = (d.y_max - d.y_min) / res, dpz = (d.z_max - d.z_min) / res;
#pragma omp parallel for collapse(2) schedule(dynamic)
    for (int ix = ix_begin; ix < ix_end; ++ix) {
        for (int iy = 0; iy < res; ++iy) {
            voro::container& con = *cons[omp_get_thread_num()];
            const double x = d.x_min + (ix + 0.5) * dpx;
            const double y = d.y_min + (iy + 0.5) * dpy;
            for (int iz = 0; iz < res; ++iz) {
                const double z = d.z_min + (iz + 0.5) * dpz;
                double rx, ry, rz;
                int pid = 0;
                if (!con.find_voronoi_cell(x, y, z, rx, ry, rz, pid)) pid = 0;
                out_ids[((size_t)(ix - ix_begin) * res + iy) * res + iz] = pid;
            }
        }
    }
    return omp_get_wtime() - t0;
}

// add_coverage_grid_buffer (src/point_set.cpp:198-262) on the particles as the point set (ids 1..n): the
// appended points and their ids; the count, or -1 with the reference's message.
long ref_coverage_grid_buffer(long n, const double* x, const double* y, const double* z, const double* h,
                              const double b[6], double spacing_fraction, double factor, double* out_xyz, int* out_id,
                              long capacity) {
    try {
        kiwi::PointSet pts;
        for (long i = 0; i < n; ++i) pts.append((int)(i + 1), x[i], y[i], z[i]);
        std::vector<double> hv(h, h + n);
        kiwi::Domain d;
        d.x_min = b[0]; d.x_max = b[1];
        d.y_min = b[2]; d.y_max = b[3];
        d.z_min = b[4]; d.z_max = b[5];
        kiwi::CoverageGridBufferParams params;
        params.spacing_fraction = spacing_fraction;
        params.coverage_radius_factor = factor;
        kiwi::PointSet out = kiwi::add_coverage_grid_buffer(pts, hv, d, params);
        long k = 0;
        for (size_t i = (size_t)n; i < out.size() && k < capacity; ++i, ++k) {
            out_xyz[3 * k] = out.x[i];
            out_xyz[3 * k + 1] = out.y[i];
            out_xyz[3 * k + 2] = out.z[i];
            out_id[k] = out.id[i];
        }
        return k;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// lloyd_step (src/point_set.cpp:265-293) on the given point set: the moved points in the container's walk
// order (ids and positions, out_xyz 3 per point); returns their count, or -1 with the reference's message.
long ref_lloyd_step(long n, const int* ids, const double* xyz, const double b[6], double scale, int* out_id,
                    double* out_xyz, long capacity) {
    try {
        kiwi::PointSet pts;
        for (long i = 0; i < n; ++i) pts.append(ids[i], xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
        kiwi::Domain d;
        d.x_min = b[0]; d.x_max = b[1];
        d.y_min = b[2]; d.y_max = b[3];
        d.z_min = b[4]; d.z_max = b[5];
        kiwi::GridBlocks blocks;
        blocks.block_scale_factor = scale;
        kiwi::PointSet out = kiwi::lloyd_step(pts, d, blocks);
        long k = 0;
        for (size_t i = 0; i < out.size() && k < capacity; ++i, ++k) {
            out_id[k] = out.id[i];
            out_xyz[3 * k] = out.x[i];
            out_xyz[3 * k + 1] = out.y[i];
            out_xyz[3 * k + 2] = out.z[i];
        }
        return k;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// A container built as the reference builds it (pre_container -> guess_scaled_blocks -> setup, ids = site
// indices): the site indices it keeps, in its c_loop_all walk order; returns their count.
long ref_container_order(long n, const double* xyz, const double b[6], double scale, long* out) {
    voro::pre_container pcon(b[0], b[1], b[2], b[3], b[4], b[5], false, false, false);
    for (long i = 0; i < n; ++i) pcon.put((int)i, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    int bx, by, bz;
    kiwi::guess_scaled_blocks(pcon, scale, bx, by, bz);
    voro::container con(b[0], b[1], b[2], b[3], b[4], b[5], bx, by, bz, false, false, false, 8);
    pcon.setup(con);
    voro::c_loop_all clo(con);
    long k = 0;
    if (clo.start()) do {
        out[k++] = clo.pid();
    } while (clo.inc());
    return k;
}

// save_cartesian_map (src/cartesian_map.cpp:202-229).
int ref_save_cartesian_map(const char* path, int res, const double* b, const double* density, const double* vx,
                           const double* vy, const double* vz, const int* cell_id) {
    try {
        kiwi::CartesianMap cm;
        cm.resolution = res;
        cm.domain.x_min = b[0]; cm.domain.x_max = b[1];
        cm.domain.y_min = b[2]; cm.domain.y_max = b[3];
        cm.domain.z_min = b[4]; cm.domain.z_max = b[5];
        const size_t nq = (size_t)res * res * res;
        cm.density.assign(density, density + nq);
        cm.vx.assign(vx, vx + nq);
        cm.vy.assign(vy, vy + nq);
        cm.vz.assign(vz, vz + nq);
        cm.voronoi_cell_id.assign(cell_id, cell_id + nq);
        kiwi::save_cartesian_map(cm, path);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// Sizes: [n_cells, n_faces, n_vertices, n_particles]
void ref_voronoi_sizes(void* h, long* out4) {
    auto* R = static_cast<RefVoronoi*>(h);
    out4[0] = static_cast<long>(R->id.size());
    out4[1] = static_cast<long>(R->face_nbr.size());
    out4[2] = static_cast<long>(R->vxyz.size() / 3);
    out4[3] = static_cast<long>(R->home.size());
}

void ref_voronoi_copy(void* h, int* id, double* site, double* volume, long* face_off, long* vert_off, double* vxyz,
                      int* face_nbr, int* home, double* density, double* vx, double* vy, double* vz) {
    auto* R = static_cast<RefVoronoi*>(h);
    auto cp = [](auto* dst, const auto& v) {
        if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
    };
    cp(id, R->id);
    cp(site, R->site);
    cp(volume, R->volume);
    cp(face_off, R->face_off);
    cp(vert_off, R->vert_off);
    cp(vxyz, R->vxyz);
    cp(face_nbr, R->face_nbr);
    cp(home, R->home);
    cp(density, R->density);
    cp(vx, R->vx);
    cp(vy, R->vy);
    cp(vz, R->vz);
}

// The inverse-mapping results of a run_map == 2 build: per particle recovered mass and coverage, the three
// totals, and per cell the mass the stage used.
void ref_voronoi_inverse_copy(void* h, double* recovered, double* coverage, double* totals3, double* cell_mass) {
    auto* R = static_cast<RefVoronoi*>(h);
    auto cp = [](double* dst, const std::vector<double>& v) {
        if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(double));
    };
    cp(recovered, R->inv_recovered);
    cp(coverage, R->inv_coverage);
    cp(cell_mass, R->inv_cell_mass);
    if (totals3) std::memcpy(totals3, R->inv_totals, sizeof(R->inv_totals));
}

void ref_voronoi_free(void* h) { delete static_cast<RefVoronoi*>(h); }

// The reference's own stage-file writers (src/cartesian_grid.cpp:323-347, src/mapping.cpp:307-315).
int ref_save_cartesian_grid(const char* path, int nx, int ny, int nz, const double* b, const double* density,
                            const double* vx, const double* vy, const double* vz) {
    try {
        kiwi::CartesianGridResult g;
        g.nx = nx;
        g.ny = ny;
        g.nz = nz;
        g.domain.x_min = b[0];
        g.domain.x_max = b[1];
        g.domain.y_min = b[2];
        g.domain.y_max = b[3];
        g.domain.z_min = b[4];
        g.domain.z_max = b[5];
        const size_t n = (size_t)nx * ny * nz;
        g.density.assign(density, density + n);
        g.vx.assign(vx, vx + n);
        g.vy.assign(vy, vy + n);
        g.vz.assign(vz, vz + n);
        kiwi::save_cartesian_grid(g, path);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// save_inverse_mapping_test (src/mapping.cpp:505-513).
int ref_save_inverse_mapping_test(const char* path, long n, const long* id, const double* m_original,
                                  const double* m_recovered, const double* coverage, const double* totals3) {
    try {
        kiwi::InverseMappingTestResult r;
        r.total_original_mass = totals3[0];
        r.total_grid_mass = totals3[1];
        r.total_recovered_mass = totals3[2];
        for (long i = 0; i < n; ++i) {
            kiwi::InverseMappingTestRow row;
            row.id = (int)id[i];
            row.m_original = m_original[i];
            row.m_recovered = m_recovered[i];
            row.coverage_fraction = coverage[i];
            r.particles.push_back(row);
        }
        kiwi::save_inverse_mapping_test(r, path);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

int ref_save_mapping(const char* path, long n, const long* id, const double* x, const double* y, const double* z,
                     const double* volume, const double* density, const double* vx, const double* vy,
                     const double* vz) {
    try {
        kiwi::MappingResult m;
        for (long i = 0; i < n; ++i) {
            kiwi::CellMapping c;
            c.id = (int)id[i];
            c.x = x[i];
            c.y = y[i];
            c.z = z[i];
            c.volume = volume[i];
            c.density = density[i];
            c.vx = vx[i];
            c.vy = vy[i];
            c.vz = vz[i];
            m.cells.push_back(c);
        }
        kiwi::save_mapping(m, path);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

}  // extern "C"
