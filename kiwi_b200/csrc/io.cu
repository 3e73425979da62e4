// Output files of the two stages (host code only): the binary Cartesian grid file and the text mapping
// file, in the reference's formats so that its readers and downstream writers take them unchanged.
//
//   VGTCGRD2 grid file (src/cartesian_grid.cpp:323-394): the 8 bytes "VGTCGRD2", int32 nx, ny, nz, six
//   doubles of domain bounds (x_min, x_max, y_min, y_max, z_min, z_max), then density, vx, vy, vz as nx*ny*nz
//   doubles each in the x-major cell order, all in the machine's (little-endian) byte order.
//   mapping.dat (src/mapping.cpp:307-315): one line per cell, "id x y z volume density vx vy vz", the
//   numbers printed by an ostream with precision 15.
//   cartesian_map.dat (src/cartesian_map.cpp:202-279): the 8 bytes "VGTCMAP1", int32 resolution, six doubles
//   of domain bounds, density, vx, vy, vz as res^3 doubles each and the Voronoi cell ids as res^3 int32.
//   inverse-mapping-test.dat (src/mapping.cpp:505-538): a '#' header line, the three totals, then one line
//   per particle, "id m_original m_recovered coverage_fraction", precision 15.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <string>

#include "../../include/kiwi_b200.h"

namespace {

const char kGridMagic[8] = {'V', 'G', 'T', 'C', 'G', 'R', 'D', '2'};
const char kMapMagic[8] = {'V', 'G', 'T', 'C', 'M', 'A', 'P', '1'};

int io_err(char* err, size_t len, int code, const std::string& what) {
    if (err && len > 0) std::snprintf(err, len, "%s", what.c_str());
    return code;
}

}  // namespace

extern "C" {

int kiwi_save_cartesian_grid(const char* path, int32_t nx, int32_t ny, int32_t nz, const double* bounds6,
                             const double* density, const double* vx, const double* vy, const double* vz, char* err,
                             size_t err_len) {
    if (!path || !bounds6 || !density || !vx || !vy || !vz)
        return io_err(err, err_len, KIWI_ERR_ARG, "save_cartesian_grid: a null argument");
    if (nx <= 0 || ny <= 0 || nz <= 0)
        return io_err(err, err_len, KIWI_ERR_ARG, "save_cartesian_grid: nx/ny/nz must be > 0");
    std::ofstream f(path, std::ios::binary);
    if (!f) return io_err(err, err_len, KIWI_ERR_ARG, std::string("could not open output file: ") + path);
    f.write(kGridMagic, sizeof(kGridMagic));
    f.write(reinterpret_cast<const char*>(&nx), sizeof(nx));
    f.write(reinterpret_cast<const char*>(&ny), sizeof(ny));
    f.write(reinterpret_cast<const char*>(&nz), sizeof(nz));
    f.write(reinterpret_cast<const char*>(bounds6), 6 * sizeof(double));
    const std::streamsize bytes = (std::streamsize)((size_t)nx * ny * nz * sizeof(double));
    for (const double* a : {density, vx, vy, vz}) f.write(reinterpret_cast<const char*>(a), bytes);
    if (!f) return io_err(err, err_len, KIWI_ERR_ARG, std::string("failed writing output file (disk full?): ") + path);
    return KIWI_OK;
}

int kiwi_load_cartesian_grid(const char* path, int32_t* nxyz, double* bounds6, double* density, double* vx,
                             double* vy, double* vz, char* err, size_t err_len) {
    if (!path || !nxyz) return io_err(err, err_len, KIWI_ERR_ARG, "load_cartesian_grid: a null argument");
    std::ifstream f(path, std::ios::binary);
    if (!f) return io_err(err, err_len, KIWI_ERR_ARG, std::string("could not open cartesian grid file: ") + path);
    char magic[8];
    f.read(magic, sizeof(magic));
    if (!f || std::memcmp(magic, kGridMagic, sizeof(magic)) != 0)
        return io_err(err, err_len, KIWI_ERR_ARG,
                      std::string("cartesian grid file has an unrecognized header (wrong format or corrupt): ") + path);
    int32_t n[3] = {0, 0, 0};
    f.read(reinterpret_cast<char*>(n), sizeof(n));
    if (!f || n[0] <= 0 || n[1] <= 0 || n[2] <= 0)
        return io_err(err, err_len, KIWI_ERR_ARG,
                      std::string("cartesian grid file has an invalid resolution (nx/ny/nz): ") + path);
    double b[6];
    f.read(reinterpret_cast<char*>(b), sizeof(b));
    if (!f) return io_err(err, err_len, KIWI_ERR_ARG, std::string("cartesian grid file is truncated (domain bounds): ") + path);
    nxyz[0] = n[0];
    nxyz[1] = n[1];
    nxyz[2] = n[2];
    if (bounds6) std::memcpy(bounds6, b, sizeof(b));
    if (!density && !vx && !vy && !vz) return KIWI_OK;  // header only: the caller sizes its arrays
    if (!density || !vx || !vy || !vz)
        return io_err(err, err_len, KIWI_ERR_ARG, "load_cartesian_grid: give all four arrays or none");
    const std::streamsize bytes = (std::streamsize)((size_t)n[0] * n[1] * n[2] * sizeof(double));
    for (double* a : {density, vx, vy, vz}) f.read(reinterpret_cast<char*>(a), bytes);
    if (!f) return io_err(err, err_len, KIWI_ERR_ARG, std::string("cartesian grid file is truncated/corrupt: ") + path);
    return KIWI_OK;
}

int kiwi_save_mapping(const char* path, int64_t n_cells, const int64_t* id, const double* x, const double* y,
                      const double* z, const double* volume, const double* density, const double* vx, const double* vy,
                      const double* vz, char* err, size_t err_len) {
    if (!path || n_cells < 0 || (n_cells > 0 && (!id || !x || !y || !z || !volume || !density || !vx || !vy || !vz)))
        return io_err(err, err_len, KIWI_ERR_ARG, "save_mapping: a null argument");
    std::ofstream f(path);
    if (!f) return io_err(err, err_len, KIWI_ERR_ARG, std::string("could not open mapping file for writing: ") + path);
    f << std::setprecision(15);
    for (int64_t c = 0; c < n_cells; ++c)
        f << id[c] << " " << x[c] << " " << y[c] << " " << z[c] << " " << volume[c] << " " << density[c] << " "
          << vx[c] << " " << vy[c] << " " << vz[c] << "\n";
    if (!f) return io_err(err, err_len, KIWI_ERR_ARG, std::string("failed writing mapping file: ") + path);
    return KIWI_OK;
}

int kiwi_save_cartesian_map(const char* path, int32_t res, const double* bounds6, const double* density,
                            const double* vx, const double* vy, const double* vz, const int32_t* voronoi_cell_id,
                            char* err, size_t err_len) {
    if (!path || res <= 0 || !bounds6 || !density || !vx || !vy || !vz || !voronoi_cell_id)
        return io_err(err, err_len, KIWI_ERR_ARG, "save_cartesian_map: a null argument");
    std::ofstream f(path, std::ios::binary);
    if (!f) return io_err(err, err_len, KIWI_ERR_ARG, std::string("could not open output file: ") + path);
    f.write(kMapMagic, sizeof(kMapMagic));
    f.write(reinterpret_cast<const char*>(&res), sizeof(res));
    f.write(reinterpret_cast<const char*>(bounds6), 6 * sizeof(double));
    const std::streamsize n = (std::streamsize)((size_t)res * res * res);
    for (const double* a : {density, vx, vy, vz}) f.write(reinterpret_cast<const char*>(a), n * (std::streamsize)sizeof(double));
    f.write(reinterpret_cast<const char*>(voronoi_cell_id), n * (std::streamsize)sizeof(int32_t));
    if (!f) return io_err(err, err_len, KIWI_ERR_ARG, std::string("failed writing output file (disk full?): ") + path);
    return KIWI_OK;
}

int kiwi_load_cartesian_map(const char* path, int32_t* res, double* bounds6, double* density, double* vx, double* vy,
                            double* vz, int32_t* voronoi_cell_id, char* err, size_t err_len) {
    if (!path || !res) return io_err(err, err_len, KIWI_ERR_ARG, "load_cartesian_map: a null argument");
    std::ifstream f(path, std::ios::binary);
    if (!f) return io_err(err, err_len, KIWI_ERR_ARG, std::string("could not open cartesian map file: ") + path);
    char magic[8];
    f.read(magic, sizeof(magic));
    if (!f || std::memcmp(magic, kMapMagic, sizeof(magic)) != 0)
        return io_err(err, err_len, KIWI_ERR_ARG,
                      std::string("cartesian map file has an unrecognized header (wrong format or corrupt): ") + path);
    int32_t r = 0;
    f.read(reinterpret_cast<char*>(&r), sizeof(r));
    if (!f || r <= 0)
        return io_err(err, err_len, KIWI_ERR_ARG, std::string("cartesian map file has an invalid resolution: ") + path);
    double b[6];
    f.read(reinterpret_cast<char*>(b), sizeof(b));
    if (!f) return io_err(err, err_len, KIWI_ERR_ARG, std::string("cartesian map file is truncated (domain bounds): ") + path);
    *res = r;
    if (bounds6) std::memcpy(bounds6, b, sizeof(b));
    if (!density && !vx && !vy && !vz && !voronoi_cell_id) return KIWI_OK;  // header only
    if (!density || !vx || !vy || !vz || !voronoi_cell_id)
        return io_err(err, err_len, KIWI_ERR_ARG, "load_cartesian_map: give all five arrays or none");
    const std::streamsize n = (std::streamsize)((size_t)r * r * r);
    for (double* a : {density, vx, vy, vz}) f.read(reinterpret_cast<char*>(a), n * (std::streamsize)sizeof(double));
    f.read(reinterpret_cast<char*>(voronoi_cell_id), n * (std::streamsize)sizeof(int32_t));
    if (!f) return io_err(err, err_len, KIWI_ERR_ARG, std::string("cartesian map file is truncated/corrupt: ") + path);
    return KIWI_OK;
}

int kiwi_save_inverse_mapping_test(const char* path, int64_t n, const int64_t* id, const double* m_original,
                                   const double* m_recovered, const double* coverage, const double* totals3, char* err,
                                   size_t err_len) {
    if (!path || !totals3 || n < 0 || (n > 0 && (!id || !m_original || !m_recovered || !coverage)))
        return io_err(err, err_len, KIWI_ERR_ARG, "save_inverse_mapping_test: a null argument");
    std::ofstream f(path);
    if (!f)
        return io_err(err, err_len, KIWI_ERR_ARG,
                      std::string("could not open inverse-mapping-test file for writing: ") + path);
    f << std::setprecision(15);
    f << "# total_original_mass total_grid_mass total_recovered_mass\n";
    f << totals3[0] << " " << totals3[1] << " " << totals3[2] << "\n";
    for (int64_t i = 0; i < n; ++i)
        f << id[i] << " " << m_original[i] << " " << m_recovered[i] << " " << coverage[i] << "\n";
    if (!f) return io_err(err, err_len, KIWI_ERR_ARG, std::string("failed writing inverse-mapping-test file: ") + path);
    return KIWI_OK;
}

int kiwi_load_inverse_mapping_test(const char* path, int64_t* n, double* totals3, int64_t* id, double* m_original,
                                   double* m_recovered, double* coverage, int64_t capacity, char* err, size_t err_len) {
    if (!path || !n) return io_err(err, err_len, KIWI_ERR_ARG, "load_inverse_mapping_test: a null argument");
    std::ifstream f(path);
    if (!f) return io_err(err, err_len, KIWI_ERR_ARG, std::string("could not open inverse-mapping-test file: ") + path);
    std::string header;
    if (!std::getline(f, header) || header.empty() || header[0] != '#')
        return io_err(err, err_len, KIWI_ERR_ARG,
                      std::string("inverse-mapping-test file missing expected '#' totals header: ") + path);
    double t[3];
    if (!(f >> t[0] >> t[1] >> t[2]))
        return io_err(err, err_len, KIWI_ERR_ARG,
                      std::string("could not read totals line from inverse-mapping-test file: ") + path);
    if (totals3) std::memcpy(totals3, t, sizeof(t));
    int64_t rows = 0;
    long long rid;
    double a, b, c;
    while (f >> rid >> a >> b >> c) {
        if (id && rows < capacity) {
            id[rows] = (int64_t)rid;
            if (m_original) m_original[rows] = a;
            if (m_recovered) m_recovered[rows] = b;
            if (coverage) coverage[rows] = c;
        }
        ++rows;
    }
    if (rows == 0)
        return io_err(err, err_len, KIWI_ERR_ARG,
                      std::string("inverse-mapping-test file contained no particle rows (wrong format?): ") + path);
    *n = rows;
    if (id && rows > capacity)
        return io_err(err, err_len, KIWI_ERR_ARG, "load_inverse_mapping_test: more rows than the arrays hold");
    return KIWI_OK;
}

}  // extern "C"
