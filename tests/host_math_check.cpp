// Test-only: compiles the device maths header kiwi_b200/csrc/kiwi_math.cuh for the host (glibc libm,
// -ffp-contract=off) so that tests/test_host_math.py can check its transcription of the reference's
// formulas against the oracle bit for bit, without a GPU.  Never part of the product library.
#include <cmath>
#include <cstdint>

#include "../kiwi_b200/csrc/kiwi_math.cuh"
#include "../kiwi_b200/csrc/dual.cuh"
#include "../kiwi_b200/csrc/lattice_math.cuh"
#include "../kiwi_b200/csrc/lattice_dual.cuh"
#include "../kiwi_b200/csrc/f32.cuh"

using namespace kiwi_b200;

extern "C" {

double hm_full_integral(int kernel, double arg0, double phi, double r0, double R0) {
    return kernel < 0 ? cubic_full_integral(arg0, phi, r0, R0)
                      : generic_full_integral(&kiwi_kernel_tables[kernel], arg0, phi, r0, R0);
}

double hm_face_integral(double x0, double y0, double z0, int kernel, double h, double support, const double* verts,
                        int n, int* out_vert) {
    FlatVerts V{verts};
    if (kernel < 0) {
        CubicEval ev;
        ev.h = h;
        return face_integral(x0, y0, z0, 2 * h, V, n, out_vert, ev);
    }
    static GenericEval ev;
    ev.K = &kiwi_kernel_tables[kernel];
    ev.H = support;
    return face_integral(x0, y0, z0, support, V, n, out_vert, ev);
}

int hm_face_reachable(double x0, double y0, double z0, double support, const double* verts, int n) {
    FlatVerts V{verts};
    return face_reachable(x0, y0, z0, support, V, n) ? 1 : 0;
}

// One box cell's Msum for one particle (cubic spline, support 2h) by the double evaluation and by the
// Dual4 evaluation of the adjoint: out[0] = double Msum, out[1] = Dual4 value, out[2..5] = d/dx0, d/dy0,
// d/dz0, d/dh.
void hm_cell_grad(double x0, double y0, double z0, double h, double cx, double cy, double cz, double hx, double hy,
                  double hz, double* out) {
    CubicEval ev;
    ev.h = h;
    out[0] = box_cell_msum(x0, y0, z0, 2 * h, cx, cy, cz, hx, hy, hz, ev);
    CubicEvalT<Dual4> evd;
    evd.h = Dual4::seed(h, 3);
    const Dual4 X = Dual4::seed(x0, 0), Y = Dual4::seed(y0, 1), Z = Dual4::seed(z0, 2);
    const Dual4 m = box_cell_msum<Dual4>(X, Y, Z, 2 * evd.h, cx, cy, cz, hx, hy, hz, evd);
    out[1] = m.v;
    for (int k = 0; k < 4; ++k) out[2 + k] = m.d[k];
}

// The lattice kernels' tiers: one edge tier, both orientations of an edge pair, one wall's corner value,
// and a lattice point's three corner values together.
void hm_lattice_edge(double h, double r0, double R0, double* out2) {
    const LatticeEdge e = lattice_edge(h, 1.0 / h, r0, R0);
    out2[0] = e.D2;
    out2[1] = e.D3;
}

void hm_lattice_edge_pair(double h, double p, double q, double* out4) {
    LatticeEdge a, b;
    lattice_edge_pair(h, 1.0 / h, p, q, a, b);
    out4[0] = a.D2;
    out4[1] = a.D3;
    out4[2] = b.D2;
    out4[3] = b.D3;
}

double hm_lattice_corner(double h, double r0, double a1, double a2, const double* d4) {
    return lattice_corner(h, 1.0 / h, r0, a1, a2, d4[0], d4[1], d4[2], d4[3]);
}

// edges: D2, D3 of xy, xz, yx, yz, zx, zy
double hm_lattice_point(double h, double ax, double ay, double az, const double* e) {
    PointEdges<double> E;
    for (int k = 0; k < 6; ++k) {
        E.d2[k] = e[2 * k];
        E.d3[k] = e[2 * k + 1];
    }
    return lattice_point(h, 1.0 / h, ax, ay, az, E);
}

// Generic kernels: one edge record (kLatGenERec doubles), one wall's two vertex tiers, and a lattice
// point's six vertex tiers together (recs: the six edge records in PointEdge order, back to back).
void hm_lattice_generic_edge(int kernel, double H, double r0, double R0, double* rec) {
    lattice_generic_edge(&kiwi_kernel_tables[kernel], H, r0, R0, rec);
}

double hm_lattice_generic_corner(int kernel, double H, double r0, double a1, double a2, const double* rec1,
                                 const double* rec2) {
    return lattice_generic_corner(&kiwi_kernel_tables[kernel], H, r0, a1, a2, rec1, rec2);
}

double hm_lattice_generic_point(int kernel, double H, double ax, double ay, double az, const double* recs) {
    const GenEdgeRecs rec{recs, {0, 1, 2, 3, 4, 5}};
    return lattice_generic_point(&kiwi_kernel_tables[kernel], H, ax, ay, az, rec);
}

// The same point in Dual3 (d/dax, d/day, d/daz): the six edge records with derivatives
// (lattice_generic_edge_dual) and the point value.  out4 = value, d/dax, d/day, d/daz.
void hm_lattice_generic_point_grad(int kernel, double H, double ax, double ay, double az, double* out4) {
    const KiwiKernelTable* K = &kiwi_kernel_tables[kernel];
    const Dual3 X = Dual3::seed(ax, 0), Y = Dual3::seed(ay, 1), Z = Dual3::seed(az, 2);
    constexpr int R = lat_gen_dual_rec<3>();
    double recs[6 * R];
    const Dual3 r0s[6] = {X, X, Y, Y, Z, Z}, R0s[6] = {Y, Z, X, Z, X, Y};
    for (int e = 0; e < 6; ++e) lattice_generic_edge_dual<3>(K, H, r0s[e], R0s[e], recs + R * e);
    const GenEdgeRecsDual<3> rd{recs, {0, 1, 2, 3, 4, 5}};
    const Dual3 f = lattice_generic_point(K, H, X, Y, Z, rd);
    out4[0] = f.v;
    for (int k = 0; k < 3; ++k) out4[1 + k] = f.d[k];
}

// FP32 instances (the FP32 type of f32.cuh): a cubic lattice point with FP32 edge pairs, and a generic
// lattice point as three FP32 corners over FP32 edge records -- for measuring what FP32 does to the
// octant values.
double hm_lattice_point_f32(double h, double ax, double ay, double az) {
    const F32 H(h), IH(1.0 / h);
    const F32 a[3] = {F32(ax), F32(ay), F32(az)};
    PointEdges<F32> E;
    // PointEdge order xy, xz, yx, yz, zx, zy: (wall, edge line) = (p, q) pairs of axes
    const int pw[6] = {0, 0, 1, 1, 2, 2}, pq[6] = {1, 2, 0, 2, 0, 1};
    for (int e = 0; e < 6; ++e) {
        const F32 p = a[pw[e]], q = a[pq[e]];
        if ((double)(p.v * p.v + q.v * q.v) <= 4.0 * h * h) {
            LatticeEdgeT<F32> ab, ba;
            lattice_edge_pair(H, IH, p, q, ab, ba);
            E.d2[e] = ab.D2;
            E.d3[e] = ab.D3;
        } else {
            E.d2[e] = E.d3[e] = F32(0.0);
        }
    }
    return (double)lattice_point(H, IH, a[0], a[1], a[2], E).v;
}

struct GenEdgeWriterF32 {
    double* rec;
    void set_packed(double v) { rec[0] = v; }
    void set_segment(int s, F32 phi_end, F32 off) {
        rec[1 + s] = (double)phi_end.v;
        rec[4 + s] = (double)off.v;
    }
};

double hm_lattice_generic_point_f32(int kernel, double H, double ax, double ay, double az) {
    const KiwiKernelTable* K = &kiwi_kernel_tables[kernel];
    const F32 a[3] = {F32(ax), F32(ay), F32(az)};
    double recs[6][kLatGenERec];
    const int pw[6] = {0, 0, 1, 1, 2, 2}, pq[6] = {1, 2, 0, 2, 0, 1};
    for (int e = 0; e < 6; ++e) {
        for (int i = 0; i < kLatGenERec; ++i) recs[e][i] = 0.0;
        GenEdgeWriterF32 w{recs[e]};
        lattice_generic_edge_t(K, H, a[pw[e]], a[pq[e]], w);
    }
    const F32 f = lattice_generic_corner(K, H, a[0], a[1], a[2], recs[0], recs[1]) +
                  lattice_generic_corner(K, H, a[1], a[0], a[2], recs[2], recs[3]) +
                  lattice_generic_corner(K, H, a[2], a[0], a[1], recs[4], recs[5]);
    return (double)f.v;
}
}
