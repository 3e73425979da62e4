// The tabulated cubic integral: a trilinear lookup of the vertex-pyramid mass in a (r0/h, mu0, cos phi)
// table (DensityLookupTable, include/kiwi/kernel_integral.hpp:21-72; gridded_integral,
// src/kernel_integral.cpp:136-190).  The table lives in device memory (182 MB for the canonical
// 251 x 301 x 301 shape); every lookup reads 8 neighbouring entries.
#pragma once

#include "ctx.hpp"
#include "kiwi_math.cuh"

namespace kiwi_b200 {

// value (i, j, k) at ((i * (nR_0 + 1) + j) * (nphi + 1) + k): i in [0, nr0 + 1] (row 0 zero, row nr0 + 1 a
// copy of row nr0), j in [0, nR_0] and k in [0, nphi] (the last of each zero), as the reference lays it out.
KIWI_HD double tab_at(const TabDev& t, int i, int j, int k) {
    return t.v[((size_t)i * (t.nR_0 + 1) + j) * (t.nphi + 1) + k];
}

// The index of v on a two-piece uniform axis: bins of width lo / n1d below lo (n1d = nr01 for r0, nR_01 - 1
// and nphi1 - 1 for mu0 and cos phi), then bins of width (top - lo) / n2 from lo; clamped to [0, imax] (clamps
// counted: the reference prints a warning for each).
KIWI_HD int tab_index(double v, double lo, int n1d, double top, int n2, int first2, int imax, unsigned& nclamp) {
    int i;
    if (v < lo) i = (int)(v / (lo / n1d));
    else i = first2 + (int)((v - lo) / ((top - lo) / n2));
    if (i < 0 || i > imax) {
        ++nclamp;
        i = i < 0 ? 0 : imax;
    }
    return i;
}

// gridded_integral(t, h, phi, r0, R_0) with cos(phi) given (cphi; the caller returns 0 for phi == 0).
KIWI_HD double tab_gridded_c(const TabDev& t, double h, double cphi, double r0_old, double R_0_old,
                             unsigned& nclamp) {
    if (r0_old == 0.0 || R_0_old == 0.0) return 0.0;
    double r0 = r0_old / h;
    double R_0 = R_0_old / h;
    if (r0 < 0.0) r0 = 0.0;
    if (R_0 < 0.0) R_0 = 0.0;
    const double mu0 = r0 / sqrt(r0 * r0 + R_0 * R_0);
    if (r0 > 2.0) r0 = 2.0;  // beyond 2h the pyramid mass depends on the angles alone
    const double rl = t.rl, mul = t.mul, cphil = t.cphil;
    const int i = tab_index(r0, rl, t.nr01, 2.0, t.nr02, t.nr01, t.nr0, nclamp);
    const int j = tab_index(mu0, mul, t.nR_01 - 1, 1.0, t.nR_02, t.nR_01 - 1, t.nR_0 - 1, nclamp);
    const int k = tab_index(cphi, cphil, t.nphi1 - 1, 1.0, t.nphi2, t.nphi1 - 1, t.nphi - 1, nclamp);
    // fractional positions inside the bins, then x (r0), y (mu0), z (cos phi) interpolation in that order
    double fr;
    if (r0 < rl) fr = (r0 - (rl / t.nr01) * i) / (rl / t.nr01);
    else fr = (r0 - rl - ((2.0 - rl) / t.nr02) * (i - t.nr01)) / ((2.0 - rl) / t.nr02);
    const double x00 = fr * tab_at(t, i + 1, j, k) + (1 - fr) * tab_at(t, i, j, k);
    const double x10 = fr * tab_at(t, i + 1, j + 1, k) + (1 - fr) * tab_at(t, i, j + 1, k);
    const double x01 = fr * tab_at(t, i + 1, j, k + 1) + (1 - fr) * tab_at(t, i, j, k + 1);
    const double x11 = fr * tab_at(t, i + 1, j + 1, k + 1) + (1 - fr) * tab_at(t, i, j + 1, k + 1);
    if (mu0 < mul) fr = (mu0 - mul / (t.nR_01 - 1) * j) / (mul / (t.nR_01 - 1));
    else fr = (mu0 - mul - (1.0 - mul) / t.nR_02 * (j - t.nR_01 + 1)) / ((1.0 - mul) / t.nR_02);
    const double y0 = fr * x10 + (1 - fr) * x00;
    const double y1 = fr * x11 + (1 - fr) * x01;
    if (cphi < cphil) fr = (cphi - cphil / (t.nphi1 - 1) * k) / (cphil / (t.nphi1 - 1));
    else fr = (cphi - cphil - (1.0 - cphil) / t.nphi2 * (k - t.nphi1 + 1)) / ((1.0 - cphil) / t.nphi2);
    const double z = fr * y1 + (1 - fr) * y0;
    // the last mu0 bin (R_0 -> 0) and the last cos phi bin (phi -> 0) evaluate to 0
    if (j == t.nR_01 + t.nR_02 - 1 || k == t.nphi1 + t.nphi2 - 1) return 0.0;
    return z;
}

// Bin widths of the table's three axes (two uniform pieces each: below and above rl / mul / cphil) and
// their reciprocals, for the lattice kernel's pair lookups.
struct TabWidths {
    double w[3][2], iw[3][2];
};
KIWI_HD TabWidths tab_widths(const TabDev& t) {
    TabWidths W;
    W.w[0][0] = t.rl / t.nr01;
    W.w[0][1] = (2.0 - t.rl) / t.nr02;
    W.w[1][0] = t.mul / (t.nR_01 - 1);
    W.w[1][1] = (1.0 - t.mul) / t.nR_02;
    W.w[2][0] = t.cphil / (t.nphi1 - 1);
    W.w[2][1] = (1.0 - t.cphil) / t.nphi2;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 2; ++b) W.iw[a][b] = 1.0 / W.w[a][b];
    return W;
}

// tab_index and the fraction inside the bin on axis a, with the widths' reciprocals in place of the
// divisions (an index that rounds to the neighbouring bin at a bin face gives the same interpolated
// value: the trilinear interpolation is continuous across bin faces).
KIWI_HD int tab_index_fr(const TabWidths& W, int a, double v, double lo, int first2, int imax, double& fr,
                         unsigned& nclamp) {
    int i = v < lo ? (int)(v * W.iw[a][0]) : first2 + (int)((v - lo) * W.iw[a][1]);
    if (i < 0 || i > imax) {
        ++nclamp;
        i = i < 0 ? 0 : imax;
    }
    fr = v < lo ? (v - W.w[a][0] * i) * W.iw[a][0] : (v - lo - W.w[a][1] * (i - first2)) * W.iw[a][1];
    return i;
}

// The two lookups of a lattice corner (tab_gridded_c at (cos phi = a1 / r, R_0 = a1) and (a2 / r, a2), r the
// distance in the wall to the corner): the r0 axis's index and fraction are shared, and the ratios come
// from the reciprocals of h (ih) and of r.  r0, a1, a2 > 0.
KIWI_HD double tab_pair(const TabDev& t, const TabWidths& W, double ih, double r0_old, double a1, double a2,
                        unsigned& nclamp) {
    double r0 = r0_old * ih;
    if (r0 > 2.0) r0 = 2.0;  // beyond 2h the pyramid mass depends on the angles alone
    double fx;
    const int i = tab_index_fr(W, 0, r0, t.rl, t.nr01, t.nr0, fx, nclamp);
    const double irr = 1.0 / sqrt(a1 * a1 + a2 * a2);
    double sum = 0.0;
#pragma unroll 1
    for (int q = 0; q < 2; ++q) {
        const double R = q ? a2 : a1;
        const double mu0 = r0_old / sqrt(r0_old * r0_old + R * R);
        const double cphi = R * irr;
        double fy, fz;
        const int j = tab_index_fr(W, 1, mu0, t.mul, t.nR_01 - 1, t.nR_0 - 1, fy, nclamp);
        const int k = tab_index_fr(W, 2, cphi, t.cphil, t.nphi1 - 1, t.nphi - 1, fz, nclamp);
        // the last mu0 bin (R_0 -> 0) and the last cos phi bin (phi -> 0) evaluate to 0
        if (j == t.nR_01 + t.nR_02 - 1 || k == t.nphi1 + t.nphi2 - 1) continue;
        const double x00 = fx * tab_at(t, i + 1, j, k) + (1 - fx) * tab_at(t, i, j, k);
        const double x10 = fx * tab_at(t, i + 1, j + 1, k) + (1 - fx) * tab_at(t, i, j + 1, k);
        const double x01 = fx * tab_at(t, i + 1, j, k + 1) + (1 - fx) * tab_at(t, i, j, k + 1);
        const double x11 = fx * tab_at(t, i + 1, j + 1, k + 1) + (1 - fx) * tab_at(t, i, j + 1, k + 1);
        const double y0 = fy * x10 + (1 - fy) * x00;
        const double y1 = fy * x11 + (1 - fy) * x01;
        sum += fz * y1 + (1 - fz) * y0;
    }
    return sum;
}

// gridded_integral at the angle phi (the face walk's form).
KIWI_HD double tab_gridded(const TabDev& t, double h, double phi, double r0, double R_0, unsigned& nclamp) {
    if (r0 == 0.0 || R_0 == 0.0 || phi == 0.0) return 0.0;
    return tab_gridded_c(t, h, cos(phi), r0, R_0, nclamp);
}

// Face-walk evaluator of the tabulated path (CubicFaceEvaluator with tabulated set,
// src/kernel_integral.cpp:433-458): no wall or edge constants, one lookup per vertex.
struct TabEval {
    TabDev t;
    double h;
    double ar0 = 0.0, R_0 = 0.0;
    unsigned* nclamp;
    KIWI_HD void set_wall(double a) { ar0 = a; }
    KIWI_HD void set_edge(double R) { R_0 = R; }
    KIWI_HD double at(double phi) const { return tab_gridded(t, h, phi, ar0, R_0, *nclamp); }
};

}  // namespace kiwi_b200
