// Kernel-integral maths, FP64, shared by every kernel of the plain (all-FP64) form.
//
// The exact kernel mass of one SPH particle inside one polygonal face's "vertex pyramids", following the
// reference's three-tier decomposition operation by operation so that the plain GPU form reproduces the
// reference's CPU results to rounding (compile the translation units that include this with
// --fmad=false: the reference's x86-64 build does not contract a*b+c):
//   wall tier   -- once per face:   src/kernel_integral.cpp:222-247   (cubic)   / kernel_integral_generic.cpp:96-117
//   edge tier   -- once per edge:   src/kernel_integral.cpp:253-350             / kernel_integral_generic.cpp:119-148
//   vertex tier -- twice per edge:  src/kernel_integral.cpp:356-400             / kernel_integral_generic.cpp:150-156
//   face walk                        src/kernel_integral.cpp:471-647
// The header is also compiled for the host by the test-only transcription check
// (tests/host_math_check.cpp), never by the product library's host code.
#pragma once

#include <math.h>
#include <stdint.h>

#include <type_traits>

#include "kernel_tables.h"

#ifdef __CUDACC__
#define KIWI_HD __host__ __device__ __forceinline__
#define KIWI_HD_NOINLINE static __host__ __device__ __noinline__
#else
#define KIWI_HD inline
#define KIWI_HD_NOINLINE static inline
#endif

namespace kiwi_b200 {

constexpr double kPi = 3.14159265358979323846;

// ------------------------------------------------------------------ cubic spline closed form

// Every function of the cubic closed form and of the face walk is written once over the real type T:
// T = double is the FP64 evaluation (the reference's operations one by one), T = Dual4 (dual.cuh) carries
// the derivatives with respect to the particle's position and smoothing length for the adjoint.
template <class T>
struct CubicWallT {
    bool valid;
    T r0, h, h2, r03, r0h2, r0h3, r0h_2, r0h_3, B1, B2, B3;
};
using CubicWall = CubicWallT<double>;

template <class T>
struct CubicEdgeT {
    bool valid;
    T R_0, a, a2, D2, D3;
};
using CubicEdge = CubicEdgeT<double>;

template <class T>
KIWI_HD CubicWallT<T> cubic_wall_t(T h, T r0) {
    CubicWallT<T> w;
    w.valid = false;
    w.h = h;
    w.r0 = r0;
    w.h2 = w.r03 = w.r0h2 = w.r0h3 = w.r0h_2 = w.r0h_3 = 0.0;
    w.B1 = w.B2 = w.B3 = 0.0;
    if (r0 == 0.0) return w;
    w.valid = true;
    w.h2 = h * h;
    w.r03 = r0 * r0 * r0;
    w.r0h2 = r0 / h * r0 / h;
    w.r0h3 = w.r0h2 * r0 / h;
    w.r0h_2 = h / r0 * h / r0;
    w.r0h_3 = w.r0h_2 * h / r0;
    if (r0 >= 2.0 * h) {
        w.B3 = w.h2 * h / 4.;
    } else if (r0 > h) {
        w.B3 = w.r03 / 4. * (-4. / 3. + (r0 / h) - 0.3 * w.r0h2 + 1. / 30. * w.r0h3 - 1. / 15. * w.r0h_3 + 8. / 5. * w.r0h_2);
        w.B2 = w.r03 / 4. * (-4. / 3. + (r0 / h) - 0.3 * w.r0h2 + 1. / 30. * w.r0h3 - 1. / 15. * w.r0h_3);
    } else {
        w.B3 = w.r03 / 4. * (-2. / 3. + 0.3 * w.r0h2 - 0.1 * w.r0h3 + 7. / 5. * w.r0h_2);
        w.B2 = w.r03 / 4. * (-2. / 3. + 0.3 * w.r0h2 - 0.1 * w.r0h3 - 1. / 5. * w.r0h_2);
        w.B1 = w.r03 / 4. * (-2. / 3. + 0.3 * w.r0h2 - 0.1 * w.r0h3);
    }
    return w;
}
KIWI_HD CubicWall cubic_wall(double h, double r0) { return cubic_wall_t<double>(h, r0); }

// The I-series at one angle (src/kernel_integral.cpp:278-294 and 372-386), with the sincos of the angle
// it starts from.  This is the bulk of the transcendental work of every tier; it is kept out of line so
// that a single copy of it serves the edge tier's two angles and the vertex tier's two vertices (inlined
// four times per edge it overflows the instruction cache).
template <class T>
struct PhiSeriesT {
    T I0, I_2, I_4, I1, I_1, I_3, I_5, cosp;
};
using PhiSeries = PhiSeriesT<double>;

template <class T>
KIWI_HD_NOINLINE PhiSeriesT<T> phi_series_sc(T phi, T sinp, T cosp, T a, T a2) {
    PhiSeriesT<T> s;
    s.cosp = cosp;
    const T cosp2 = cosp * cosp;
    const T mu = cosp / a / sqrt(1. + cosp2 / a2);
    const T tanp = sinp / cosp;
    s.I0 = phi;
    s.I_2 = phi + a2 * tanp;
    s.I_4 = phi + 2 * a2 * tanp + 1. / 3. * a2 * a2 * tanp * (2. + 1. / cosp2);
    const T u = sinp * sqrt(1 - mu * mu);
    const T logs = log(1 + u) - log(1 - u);
    s.I1 = atan(u / a);
    s.I_1 = a / 2. * logs + s.I1;
    s.I_3 = s.I_1 + a * (1. + a2) / 4. * (2 * u / (1 - u * u) + logs);
    s.I_5 = s.I_3 + a * (1. + a2) * (1. + a2) / 16. * ((10 * u - 6 * u * u * u) / (1 - u * u) / (1 - u * u) + 3. * logs);
    return s;
}

// The series at phi, with the sincos of phi (the edge tier's h and 2h angles).
template <class T>
KIWI_HD_NOINLINE PhiSeriesT<T> phi_series(T phi, T a, T a2) {
    T sinp, cosp;
    sincos(phi, &sinp, &cosp);
    return phi_series_sc<T>(phi, sinp, cosp, a, a2);
}

template <class T>
KIWI_HD CubicEdgeT<T> cubic_edge_t(const CubicWallT<T>& w, T R_0) {
    CubicEdgeT<T> e;
    e.valid = false;
    e.R_0 = R_0;
    e.a = e.a2 = e.D2 = e.D3 = 0.0;
    if (!w.valid || R_0 == 0.0) return e;
    e.valid = true;
    const T h = w.h, r0 = w.r0, h2 = w.h2;
    const T r03 = w.r03, r0h2 = w.r0h2, r0h3 = w.r0h3, r0h_3 = w.r0h_3;
    T D2 = 0.0, D3 = 0.0;
    const T a = R_0 / r0;
    const T a2 = a * a;
    e.a = a;
    e.a2 = a2;
    const T linedist2 = r0 * r0 + R_0 * R_0;
    if (linedist2 <= 4.0 * h2) {
        // pass 0: the angle where the vertex radius reaches h (inner edges only) -> D2;
        // pass 1: the angle where it reaches 2h -> D3
#pragma unroll 1
        for (int pass = (linedist2 <= h2) ? 0 : 1; pass < 2; ++pass) {
            const T hh = (pass == 0) ? h * h : 4.0 * h * h;
            const T phik = acos(R_0 / sqrt(hh - r0 * r0));
            const PhiSeriesT<T> s = phi_series<T>(phik, a, a2);
            if (pass == 0)
                D2 = -1. / 6. * s.I_2 + 0.25 * (r0 / h) * s.I_3 - 0.15 * r0h2 * s.I_4 + 1. / 30. * r0h3 * s.I_5 - 1. / 60. * r0h_3 * s.I1 + (w.B1 - w.B2) / r03 * s.I0;
            else
                D3 = 1. / 3. * s.I_2 - 0.25 * (r0 / h) * s.I_3 + 3. / 40. * r0h2 * s.I_4 - 1. / 120. * r0h3 * s.I_5 + 4. / 15. * r0h_3 * s.I1 + (w.B2 - w.B3) / r03 * s.I0 + D2;
        }
    }
    e.D2 = D2;
    e.D3 = D3;
    return e;
}
KIWI_HD CubicEdge cubic_edge(const CubicWall& w, double R_0) { return cubic_edge_t<double>(w, R_0); }

template <class T>
KIWI_HD T cubic_vertex_t(const CubicWallT<T>& w, const CubicEdgeT<T>& e, T phi) {
    if (!w.valid || !e.valid) return T(0.0);
    if (phi == 0.0) return T(0.0);
    const T r0 = w.r0, h = w.h, r03 = w.r03, r0h2 = w.r0h2, r0h3 = w.r0h3, r0h_3 = w.r0h_3;
    // (the full series in every region: a per-lane shortcut for the outer region only diverges warps here)
    const PhiSeriesT<T> s = phi_series<T>(phi, e.a, e.a2);
    const T R = e.R_0 / s.cosp;
    const T r2 = r0 * r0 + R * R;
    T full_int;
    if (r2 < w.h2) {
        full_int = r0h3 / kPi * (1. / 6. * s.I_2 - 3. / 40. * r0h2 * s.I_4 + 1. / 40. * r0h3 * s.I_5 + w.B1 / r03 * s.I0);
    } else if (r2 < 4.0 * w.h2) {
        full_int = r0h3 / kPi * (0.25 * (4. / 3. * s.I_2 - (r0 / h) * s.I_3 + 0.3 * r0h2 * s.I_4 - 1. / 30. * r0h3 * s.I_5 + 1. / 15. * r0h_3 * s.I1) + w.B2 / r03 * s.I0 + e.D2);
    } else {
        full_int = r0h3 / kPi * (-0.25 * r0h_3 * s.I1 + w.B3 / r03 * s.I0 + e.D3);
    }
    return full_int;
}
KIWI_HD double cubic_vertex(const CubicWall& w, const CubicEdge& e, double phi) { return cubic_vertex_t<double>(w, e, phi); }

// full_integral_new (src/kernel_integral.cpp:410-418)
KIWI_HD double cubic_full_integral(double h, double phi, double r0, double R_0) {
    if (r0 == 0.0 || R_0 == 0.0 || phi == 0.0) return 0.0;
    const CubicWall w = cubic_wall(h, r0);
    const CubicEdge e = cubic_edge(w, R_0);
    return cubic_vertex(w, e, phi);
}

// ------------------------------------------------------------------ generic table-driven kernels

struct GenericWall {
    bool valid;
    const KiwiKernelTable* K;
    double H, r0, q0;
    int j;
    double coef[KIWI_MAX_REGIONS][KIWI_NI];
    double bphi[KIWI_MAX_REGIONS];
};

struct GenericEdge {
    bool valid;
    double R_0, a, a2;
    int nseg;
    int region[KIWI_MAX_REGIONS];
    double phi_end[KIWI_MAX_REGIONS];
    double offset[KIWI_MAX_REGIONS];
};

// I_i(phi) = int_0^phi mu^i dphi', i = 1, 0, -1, ..., imin, stored at out[1 - i]
// (src/kernel_integral_generic.cpp:19-66).
// With sin(phi) and cos(phi) given (the lattice form knows them from the legs of its right triangles).
KIWI_HD void generic_basis_sc(double a, double a2, double phi, double sinp, double cosp, int imin, double* out) {
    const double den = a2 + cosp * cosp;
    const double u = a * sinp / sqrt(den);
    const double one_minus_u2 = cosp * cosp * (1.0 + a2) / den;
    out[0] = atan(u / a);
    out[1] = phi;
    const int mmax = (-imin - 1) / 2;
    double Iodd = out[0];
    double K = atanh(u);
    double pow1a2 = 1.0;
    for (int m = 0; m <= mmax && -2 * m - 1 >= imin; ++m) {
        if (m > 0) {
            const int n = m;
            K = u / (2.0 * n * pow(one_minus_u2, (double)n)) + (2.0 * n - 1.0) / (2.0 * n) * K;
            pow1a2 *= (1.0 + a2);
        }
        Iodd += a * pow1a2 * K;
        out[1 + (2 * m + 1)] = Iodd;
    }
    const int kmax = -imin / 2;
    if (kmax >= 1) {
        double J[KIWI_NI];
        const double t = sinp / cosp, s = 1.0 / cosp;
        J[0] = phi;
        J[2] = t;
        double spow = 1.0;
        for (int l = 2; l <= kmax; ++l) {
            const int m = 2 * l;
            spow *= s * s;
            J[m] = spow * t / (m - 1.0) + (m - 2.0) / (m - 1.0) * J[m - 2];
        }
        for (int k = 1; k <= kmax; ++k) {
            double sum = J[0], apow = 1.0, b = 1.0;
            for (int l = 1; l <= k; ++l) {
                b = b * (k - l + 1) / l;
                apow *= a2;
                sum += b * apow * J[2 * l];
            }
            out[1 + 2 * k] = sum;
        }
    }
}

KIWI_HD void generic_basis(double a, double a2, double phi, int imin, double* out) {
    const double sinp = sin(phi), cosp = cos(phi);
    generic_basis_sc(a, a2, phi, sinp, cosp, imin, out);
}

KIWI_HD int generic_region(const KiwiKernelTable* K, double q) {
    for (int k = 0; k < K->nreg - 1; ++k)
        if (q <= K->c[k]) return k + 1;
    return K->nreg;
}

KIWI_HD int generic_imin(const GenericWall& w, int k) {
    for (int idx = KIWI_NI - 1; idx >= 0; --idx)
        if (w.coef[k - 1][idx] != 0.0) return 1 - idx;
    return 1;
}

// G_k(phi): antiderivative of dI_P/dphi in region k (src/kernel_integral_generic.cpp:82-92).
KIWI_HD_NOINLINE double generic_G(const GenericWall& w, const GenericEdge& e, int k, double phi) {
    const int imin = generic_imin(w, k);
    double I[KIWI_NI];
    generic_basis(e.a, e.a2, phi, imin, I);
    double sum = w.bphi[k - 1] * phi;
    for (int idx = 0; idx < KIWI_NI; ++idx) {
        const double c = w.coef[k - 1][idx];
        if (c != 0.0) sum += c * I[idx];
    }
    return sum;
}

KIWI_HD void generic_wall(GenericWall& w, const KiwiKernelTable* K, double H, double r0) {
    w.valid = false;
    w.K = K;
    w.H = H;
    w.r0 = r0;
    w.q0 = 0.0;
    w.j = 0;
    if (r0 == 0.0) return;
    w.valid = true;
    w.q0 = r0 / H;
    w.j = generic_region(K, w.q0);
    const double A3 = K->A3_pi / kPi;
    for (int k = 1; k <= K->nreg; ++k) {
        for (int idx = 0; idx < KIWI_NI; ++idx) {
            const double a = K->a[k - 1][idx];
            w.coef[k - 1][idx] = (a == 0.0) ? 0.0 : A3 * a * pow(w.q0, (double)idx);
        }
        double b = 0.0;
        if (k >= w.j)
            for (int p = KIWI_NB - 1; p >= 0; --p) b = b * w.q0 + K->B[w.j - 1][k - 1][p];
        w.bphi[k - 1] = A3 * b;
    }
}

KIWI_HD void generic_edge(GenericEdge& e, const GenericWall& w, double R_0) {
    e.valid = false;
    e.R_0 = R_0;
    e.nseg = 0;
    e.a = e.a2 = 0.0;
    if (!w.valid || R_0 == 0.0) return;
    e.valid = true;
    e.a = R_0 / w.r0;
    e.a2 = e.a * e.a;
    const KiwiKernelTable* K = w.K;
    const double qR = R_0 / w.H;
    const double r_start = sqrt(w.q0 * w.q0 + qR * qR);
    int k = generic_region(K, r_start);
    for (; k <= K->nreg; ++k) {
        e.region[e.nseg] = k;
        if (k == K->nreg) {
            e.phi_end[e.nseg] = 0.5 * kPi;
        } else {
            const double c = K->c[k - 1];
            e.phi_end[e.nseg] = acos(fmin(1.0, qR / sqrt(c * c - w.q0 * w.q0)));
        }
        ++e.nseg;
    }
    e.offset[0] = 0.0;
    for (int s = 0; s + 1 < e.nseg; ++s) {
        const double pb = e.phi_end[s];
        e.offset[s + 1] = e.offset[s] + generic_G(w, e, e.region[s], pb) - generic_G(w, e, e.region[s + 1], pb);
    }
}

KIWI_HD double generic_vertex(const GenericWall& w, const GenericEdge& e, double phi) {
    if (!w.valid || !e.valid) return 0.0;
    if (phi == 0.0) return 0.0;
    int s = 0;
    while (s + 1 < e.nseg && phi > e.phi_end[s]) ++s;
    return e.offset[s] + generic_G(w, e, e.region[s], phi);
}

KIWI_HD double generic_full_integral(const KiwiKernelTable* K, double H, double phi, double r0, double R_0) {
    if (r0 == 0.0 || R_0 == 0.0 || phi == 0.0) return 0.0;
    GenericWall w;
    GenericEdge e;
    generic_wall(w, K, H, r0);
    generic_edge(e, w, R_0);
    return generic_vertex(w, e, phi);
}

// ------------------------------------------------------------------ face walk

// Evaluator hooks (the strategy of src/kernel_integral.cpp:433-467): set_wall once per face with the
// unsigned wall distance, set_edge once per edge with the in-plane distance to the edge line, at(phi)
// once per edge vertex.
template <class T>
struct CubicEvalT {
    T h;
    CubicWallT<T> w;
    CubicEdgeT<T> e;
    KIWI_HD void set_wall(T ar0) { w = cubic_wall_t<T>(h, ar0); }
    KIWI_HD void set_edge(T R_0) { e = cubic_edge_t<T>(w, R_0); }
    KIWI_HD T at(T phi) const { return cubic_vertex_t<T>(w, e, phi); }
};
using CubicEval = CubicEvalT<double>;

struct GenericEval {
    const KiwiKernelTable* K;
    double H;
    GenericWall w;
    GenericEdge e;
    KIWI_HD void set_wall(double ar0) { generic_wall(w, K, H, ar0); }
    KIWI_HD void set_edge(double R_0) { generic_edge(e, w, R_0); }
    KIWI_HD double at(double phi) const { return generic_vertex(w, e, phi); }
};

KIWI_HD double dmax2(double a, double b) { return a > b ? a : b; }
KIWI_HD double dmin2(double a, double b) { return a < b ? a : b; }
template <class T>
KIWI_HD T vmax2(const T& a, const T& b) { return a > b ? a : b; }
template <class T>
KIWI_HD T vmin2(const T& a, const T& b) { return a < b ? a : b; }

// Vertex source for the face walk: VX(i), VY(i), VZ(i) give vertex i of the face (n vertices, n >= 3).
// Whether a face-walk evaluator takes the vertex pyramid's leg along the edge (at_len(t)) instead of its
// angle (at(phi)).
template <class E, class = void>
struct EvalUsesLengths : std::false_type {};
template <class E>
struct EvalUsesLengths<E, std::void_t<decltype(E::kLengths)>> : std::integral_constant<bool, E::kLengths> {};

// face_integral_impl of src/kernel_integral.cpp:471-647, including the out_vert reachability rule.
// T is the type of the particle's coordinates (the face's vertices are plain doubles): double, or Dual4
// for the derivatives of the face integral with respect to the particle.
template <class T, class Verts, class Eval>
KIWI_HD T face_integral(T x0, T y0, T z0, T support_radius, const Verts& V, int n, int* out_vert, Eval& ev) {
    if (n < 3) {
        if (out_vert) *out_vert = 0;
        return T(0.0);
    }
    T face_Msum = 0.0;
    const double x1 = V.x(0), y1 = V.y(0), z1 = V.z(0);
    const double x2s = V.x(1), y2s = V.y(1), z2s = V.z(1);
    const double x3s = V.x(2), y3s = V.y(2), z3s = V.z(2);
    const double A = (y2s - y1) * (z3s - z1) - (y3s - y1) * (z2s - z1);
    const double B = (z2s - z1) * (x3s - x1) - (z3s - z1) * (x2s - x1);
    const double C = (x2s - x1) * (y3s - y1) - (x3s - x1) * (y2s - y1);
    const double D = -A * x1 - B * y1 - C * z1;
    const double norm = sqrt(A * A + B * B + C * C);
    const T r0 = (A * x0 + B * y0 + C * z0 + D) / norm;
    const T ar0 = fabs(r0);
    const T xp = x0 - r0 * A / norm;
    const T yp = y0 - r0 * B / norm;
    const T zp = z0 - r0 * C / norm;
    const T x1r = x1 - x0, y1r = y1 - y0, z1r = z1 - z0;
    const T x2sr = x2s - x0, y2sr = y2s - y0, z2sr = z2s - z0;
    const T x3sr = x3s - x0, y3sr = y3s - y0, z3sr = z3s - z0;
    const T s2 = x1r * (y2sr * z3sr - z2sr * y3sr) + y1r * (z2sr * x3sr - x2sr * z3sr) + z1r * (x2sr * y3sr - y2sr * x3sr);
    ev.set_wall(ar0);
    bool inside_polygon = true, have_sign = false;
    T sign_ref = 0.0;
    T min_edge_dist = INFINITY;
    for (int j = 0; j < n; ++j) {
        const double x2 = V.x(j), y2 = V.y(j), z2 = V.z(j);
        const int jn = (j == n - 1) ? 0 : j + 1;
        const double x3 = V.x(jn), y3 = V.y(jn), z3 = V.z(jn);
        const double r23 = sqrt((x3 - x2) * (x3 - x2) + (y3 - y2) * (y3 - y2) + (z3 - z2) * (z3 - z2));
        const T r12 = sqrt((xp - x2) * (xp - x2) + (yp - y2) * (yp - y2) + (zp - z2) * (zp - z2));
        const T r13 = sqrt((xp - x3) * (xp - x3) + (yp - y3) * (yp - y3) + (zp - z3) * (zp - z3));
        const T cosa = ((x3 - x2) * (xp - x2) + (y3 - y2) * (yp - y2) + (z3 - z2) * (zp - z2)) / r12 / r23;
        const T R_0 = (fabs(cosa) < 1.0) ? r12 * sqrt(1 - cosa * cosa) : T(0.0);
        const T xpr = xp - x0, ypr = yp - y0, zpr = zp - z0;
        const T x2r = x2 - x0, y2r = y2 - y0, z2r = z2 - z0;
        const T x3r = x3 - x0, y3r = y3 - y0, z3r = z3 - z0;
        const T s1 = xpr * (y2r * z3r - z2r * y3r) + ypr * (z2r * x3r - x2r * z3r) + zpr * (x2r * y3r - y2r * x3r);
        const double ex = x3 - x2, ey = y3 - y2, ez = z3 - z2;
        const T tpx = xp - x2, tpy = yp - y2, tpz = zp - z2;
        const T side = (ey * tpz - ez * tpy) * A + (ez * tpx - ex * tpz) * B + (ex * tpy - ey * tpx) * C;
        const T side_eps = 1e-9 * norm * r23 * vmax2(vmax2(fabs(tpx), fabs(tpy)), vmax2(fabs(tpz), T(1.0)));
        if (fabs(side) > side_eps) {
            if (!have_sign) {
                sign_ref = side;
                have_sign = true;
            } else if ((side > 0) != (sign_ref > 0)) {
                inside_polygon = false;
            }
        }
        bool foot_beyond_endpoint, first_wider;
        T I1v = 0.0, I2v = 0.0;
        if constexpr (EvalUsesLengths<Eval>::value) {
            // the legs along the edge line from each vertex to the foot: r12 |cos a| and |r23 - r12 cos a|
            // (the reference's r12 sin(phi1) and r13 sin(phi2)); phi1 >= phi2 iff t1 >= t2
            const T t1 = r12 * fabs(cosa), t2 = fabs(r23 - r12 * cosa);
            foot_beyond_endpoint = (t1 >= r23) || (t2 >= r23);
            first_wider = t1 >= t2;
            ev.set_edge(R_0);
            I1v = ev.at_len(t1);
            I2v = ev.at_len(t2);
        } else {
            const T phi1 = (R_0 < r12) ? acos(R_0 / r12) : T(0.0);
            const T phi2 = (R_0 < r13) ? acos(R_0 / r13) : T(0.0);
            foot_beyond_endpoint = (r12 * sin(phi1) >= r23) || (r13 * sin(phi2) >= r23);
            first_wider = phi1 >= phi2;
            ev.set_edge(R_0);
#pragma unroll 1
            for (int v = 0; v < 2; ++v) {
                const T t = ev.at(v == 0 ? phi1 : phi2);
                if (v == 0) I1v = t; else I2v = t;
            }
        }
        const T in_plane_dist = foot_beyond_endpoint ? vmin2(r12, r13) : R_0;
        min_edge_dist = vmin2(min_edge_dist, in_plane_dist);
        T M = (s1 * s2 * r0 <= 0) ? T(-1.0) : T(1.0);
        if (foot_beyond_endpoint) {
            M = first_wider ? M * (I1v - I2v) : M * (I2v - I1v);
        } else {
            M = M * (I1v + I2v);
        }
        face_Msum += M;
    }
    if (out_vert) {
        const T face_dist = inside_polygon ? ar0 : sqrt(r0 * r0 + min_edge_dist * min_edge_dist);
        *out_vert = (face_dist >= support_radius) ? n : 0;
    }
    return face_Msum;
}

// The reachability half of the face walk alone (src/kernel_integral.cpp:533-645, no integrals): true iff
// the face's closest point to the particle lies within the support radius, i.e. iff the reference's
// out_vert != n, the condition under which its BFS enqueues the neighbour behind the face
// (src/mapping.cpp:187-193).  Same operations as face_integral's geometry.
template <class Verts>
KIWI_HD bool face_reachable(double x0, double y0, double z0, double support_radius, const Verts& V, int n) {
    if (n < 3) return true;  // out_vert = 0 != n
    const double x1 = V.x(0), y1 = V.y(0), z1 = V.z(0);
    const double x2s = V.x(1), y2s = V.y(1), z2s = V.z(1);
    const double x3s = V.x(2), y3s = V.y(2), z3s = V.z(2);
    const double A = (y2s - y1) * (z3s - z1) - (y3s - y1) * (z2s - z1);
    const double B = (z2s - z1) * (x3s - x1) - (z3s - z1) * (x2s - x1);
    const double C = (x2s - x1) * (y3s - y1) - (x3s - x1) * (y2s - y1);
    const double D = -A * x1 - B * y1 - C * z1;
    const double norm = sqrt(A * A + B * B + C * C);
    const double r0 = (A * x0 + B * y0 + C * z0 + D) / norm;
    const double ar0 = fabs(r0);
    // The face is no closer than its plane: face_dist below is ar0 or sqrt(r0^2 + d^2), and a correctly
    // rounded sqrt(r0 * r0) is |r0| in binary floating point, so sqrt(r0^2 + d^2) >= ar0 as rounded too.
    // (A NaN ar0 goes on to the walk, as in the reference.)
    if (ar0 >= support_radius) return false;
    const double xp = x0 - r0 * A / norm;
    const double yp = y0 - r0 * B / norm;
    const double zp = z0 - r0 * C / norm;
    bool inside_polygon = true, have_sign = false;
    double sign_ref = 0.0;
    double min_edge_dist = INFINITY;
    for (int j = 0; j < n; ++j) {
        const double x2 = V.x(j), y2 = V.y(j), z2 = V.z(j);
        const int jn = (j == n - 1) ? 0 : j + 1;
        const double x3 = V.x(jn), y3 = V.y(jn), z3 = V.z(jn);
        const double r23 = sqrt((x3 - x2) * (x3 - x2) + (y3 - y2) * (y3 - y2) + (z3 - z2) * (z3 - z2));
        const double r12 = sqrt((xp - x2) * (xp - x2) + (yp - y2) * (yp - y2) + (zp - z2) * (zp - z2));
        const double r13 = sqrt((xp - x3) * (xp - x3) + (yp - y3) * (yp - y3) + (zp - z3) * (zp - z3));
        const double cosa = ((x3 - x2) * (xp - x2) + (y3 - y2) * (yp - y2) + (z3 - z2) * (zp - z2)) / r12 / r23;
        const double R_0 = (fabs(cosa) < 1.0) ? r12 * sqrt(1 - cosa * cosa) : 0.0;
        const double phi1 = (R_0 < r12) ? acos(R_0 / r12) : 0.0;
        const double phi2 = (R_0 < r13) ? acos(R_0 / r13) : 0.0;
        const double ex = x3 - x2, ey = y3 - y2, ez = z3 - z2;
        const double tpx = xp - x2, tpy = yp - y2, tpz = zp - z2;
        const double side = (ey * tpz - ez * tpy) * A + (ez * tpx - ex * tpz) * B + (ex * tpy - ey * tpx) * C;
        const double side_eps = 1e-9 * norm * r23 * dmax2(dmax2(fabs(tpx), fabs(tpy)), dmax2(fabs(tpz), 1.0));
        if (fabs(side) > side_eps) {
            if (!have_sign) {
                sign_ref = side;
                have_sign = true;
            } else if ((side > 0) != (sign_ref > 0)) {
                inside_polygon = false;
            }
        }
        const bool foot_beyond_endpoint = (r12 * sin(phi1) >= r23) || (r13 * sin(phi2) >= r23);
        const double in_plane_dist = foot_beyond_endpoint ? dmin2(r12, r13) : R_0;
        min_edge_dist = dmin2(min_edge_dist, in_plane_dist);
    }
    const double face_dist = inside_polygon ? ar0 : sqrt(r0 * r0 + min_edge_dist * min_edge_dist);
    return !(face_dist >= support_radius);
}

// Flattened xyz vertex array (a Voronoi face, or a face handed over by the scalar API).
struct FlatVerts {
    const double* p;
    KIWI_HD double x(int i) const { return p[3 * i]; }
    KIWI_HD double y(int i) const { return p[3 * i + 1]; }
    KIWI_HD double z(int i) const { return p[3 * i + 2]; }
};

// One of the six faces of an axis-aligned box cell, in the winding of src/cartesian_grid.cpp:54-72
// (the winding the face walk needs): bit 0/1/2 of kBoxFace[f][v] selects the + side of x/y/z.
struct BoxFace {
    double xm, xp, ym, yp, zm, zp;
    unsigned pat;  // 4 vertices x 3 bits
    KIWI_HD double x(int i) const { return ((pat >> (3 * i)) & 1u) ? xp : xm; }
    KIWI_HD double y(int i) const { return ((pat >> (3 * i + 1)) & 1u) ? yp : ym; }
    KIWI_HD double z(int i) const { return ((pat >> (3 * i + 2)) & 1u) ? zp : zm; }
};

// Vertex sign patterns of the six box faces (+x, -x, +y, -y, +z, -z), vertex v in bits 3v..3v+2.
#define KIWI_V(px, py, pz) ((px) | ((py) << 1) | ((pz) << 2))
#define KIWI_F(a, b, c, d) ((a) | ((b) << 3) | ((c) << 6) | ((d) << 9))
KIWI_HD unsigned box_face_pattern(int f) {
    switch (f) {
        case 0: return KIWI_F(KIWI_V(1, 0, 1), KIWI_V(1, 1, 1), KIWI_V(1, 1, 0), KIWI_V(1, 0, 0));  // +x
        case 1: return KIWI_F(KIWI_V(0, 1, 0), KIWI_V(0, 1, 1), KIWI_V(0, 0, 1), KIWI_V(0, 0, 0));  // -x
        case 2: return KIWI_F(KIWI_V(1, 1, 0), KIWI_V(1, 1, 1), KIWI_V(0, 1, 1), KIWI_V(0, 1, 0));  // +y
        case 3: return KIWI_F(KIWI_V(0, 0, 1), KIWI_V(1, 0, 1), KIWI_V(1, 0, 0), KIWI_V(0, 0, 0));  // -y
        case 4: return KIWI_F(KIWI_V(0, 1, 1), KIWI_V(1, 1, 1), KIWI_V(1, 0, 1), KIWI_V(0, 0, 1));  // +z
        default: return KIWI_F(KIWI_V(1, 0, 0), KIWI_V(1, 1, 0), KIWI_V(0, 1, 0), KIWI_V(0, 0, 0));  // -z
    }
}
#undef KIWI_V
#undef KIWI_F

// Msum of one box cell for one particle: the 6 faces summed in order, then the clamp of
// src/cartesian_grid.cpp:256-269 (the caller counts the clamps).
template <class T, class Eval>
KIWI_HD T box_cell_msum(T x0, T y0, T z0, T support, double cx, double cy, double cz, double hx, double hy,
                        double hz, Eval& ev) {
    BoxFace bf;
    bf.xm = cx - hx;
    bf.xp = cx + hx;
    bf.ym = cy - hy;
    bf.yp = cy + hy;
    bf.zm = cz - hz;
    bf.zp = cz + hz;
    T Msum = 0.0;
#pragma unroll 1
    for (int f = 0; f < 6; ++f) {
        bf.pat = box_face_pattern(f);
        Msum += face_integral<T>(x0, y0, z0, support, bf, 4, (int*)nullptr, ev);
    }
    return Msum;
}

}  // namespace kiwi_b200
