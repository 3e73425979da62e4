/* CPU oracle for the KIWI kernel-integral hot path -- TEST INFRASTRUCTURE ONLY (see kiwi_oracle.h).
 *
 * Every function restates the reference's arithmetic in the same operation order (FP64, no FMA
 * contraction: build with -ffp-contract=off), citing the reference file:line it follows.  The kernel
 * coefficient tables come from kiwi_b200/csrc/kernel_tables.h, which tests/test_kernel_tables.py pins
 * against the reference's src/kernel_spec_data.cpp values.
 */
#define _GNU_SOURCE
#include "kiwi_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "../kiwi_b200/csrc/kernel_tables.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ============================ cubic spline closed form ======================================== */

typedef struct {
    int valid;
    double r0, h, h2, r03, r0h2, r0h3, r0h_2, r0h_3, B1, B2, B3;
} Wall;

typedef struct {
    int valid;
    double R_0, a, a2, D2, D3;
} Edge;

/* compute_wall_constants: src/kernel_integral.cpp:222-247 */
static Wall wall_constants(double h, double r0) {
    Wall w;
    memset(&w, 0, sizeof w);
    w.h = h;
    w.r0 = r0;
    if (r0 == 0.0) return w;
    w.valid = 1;
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

/* The phi-series shared by the edge and vertex tiers (src/kernel_integral.cpp:278-294, 367-386). */
typedef struct {
    double I0, I_2, I_4, I1, I_1, I_3, I_5;
} Series;

static Series series_at(double phi, double sinp, double cosp, double a, double a2) {
    Series s;
    double cosp2 = cosp * cosp;
    double mu = cosp / a / sqrt(1. + cosp2 / a2);
    double tanp = sinp / cosp;
    s.I0 = phi;
    s.I_2 = phi + a2 * tanp;
    s.I_4 = phi + 2 * a2 * tanp + 1. / 3. * a2 * a2 * tanp * (2. + 1. / cosp2);
    double u = sinp * sqrt(1 - mu * mu);
    double logs = log(1 + u) - log(1 - u);
    s.I1 = atan(u / a);
    s.I_1 = a / 2. * logs + s.I1;
    s.I_3 = s.I_1 + a * (1. + a2) / 4. * (2 * u / (1 - u * u) + logs);
    s.I_5 = s.I_3 + a * (1. + a2) * (1. + a2) / 16. * ((10 * u - 6 * u * u * u) / (1 - u * u) / (1 - u * u) + 3. * logs);
    return s;
}

/* compute_edge_constants: src/kernel_integral.cpp:253-350 */
static Edge edge_constants(const Wall* w, double R_0) {
    Edge e;
    memset(&e, 0, sizeof e);
    e.R_0 = R_0;
    if (!w->valid || R_0 == 0.0) return e;
    e.valid = 1;
    const double h = w->h, r0 = w->r0, h2 = w->h2;
    const double r03 = w->r03, r0h2 = w->r0h2, r0h3 = w->r0h3, r0h_3 = w->r0h_3;
    const double B1 = w->B1, B2 = w->B2, B3 = w->B3;
    double D2 = 0.0, D3 = 0.0, sinp, cosp;
    double a = R_0 / r0;
    double a2 = a * a;
    e.a = a;
    e.a2 = a2;
    double linedist2 = r0 * r0 + R_0 * R_0;
    if (linedist2 <= h2) {
        double phi1 = acos(R_0 / sqrt(h * h - r0 * r0));
        sincos(phi1, &sinp, &cosp);
        Series s = series_at(phi1, sinp, cosp, a, a2);
        D2 = -1. / 6. * s.I_2 + 0.25 * (r0 / h) * s.I_3 - 0.15 * r0h2 * s.I_4 + 1. / 30. * r0h3 * s.I_5 - 1. / 60. * r0h_3 * s.I1 + (B1 - B2) / r03 * s.I0;
        double phi2 = acos(R_0 / sqrt(4.0 * h * h - r0 * r0));
        sincos(phi2, &sinp, &cosp);
        s = series_at(phi2, sinp, cosp, a, a2);
        D3 = 1. / 3. * s.I_2 - 0.25 * (r0 / h) * s.I_3 + 3. / 40. * r0h2 * s.I_4 - 1. / 120. * r0h3 * s.I_5 + 4. / 15. * r0h_3 * s.I1 + (B2 - B3) / r03 * s.I0 + D2;
    } else if (linedist2 <= 4.0 * h2) {
        double phi2 = acos(R_0 / sqrt(4.0 * h * h - r0 * r0));
        sincos(phi2, &sinp, &cosp);
        Series s = series_at(phi2, sinp, cosp, a, a2);
        D3 = 1. / 3. * s.I_2 - 0.25 * (r0 / h) * s.I_3 + 3. / 40. * r0h2 * s.I_4 - 1. / 120. * r0h3 * s.I_5 + 4. / 15. * r0h_3 * s.I1 + (B2 - B3) / r03 * s.I0 + D2;
    }
    e.D2 = D2;
    e.D3 = D3;
    return e;
}

/* vertex_integral: src/kernel_integral.cpp:356-400 */
static double vertex_integral(const Wall* w, const Edge* e, double phi) {
    if (!w->valid || !e->valid) return 0.0;
    if (phi == 0.0) return 0.0;
    const double pi = M_PI;
    const double h2 = w->h2, r03 = w->r03, r0h2 = w->r0h2, r0h3 = w->r0h3, r0h_3 = w->r0h_3;
    const double B1 = w->B1, B2 = w->B2, B3 = w->B3, r0 = w->r0, h = w->h;
    const double R_0 = e->R_0, a = e->a, a2 = e->a2, D2 = e->D2, D3 = e->D3;
    double sinp, cosp;
    sincos(phi, &sinp, &cosp);
    double R = R_0 / cosp;
    double r2 = r0 * r0 + R * R;
    Series s = series_at(phi, sinp, cosp, a, a2);
    double full_int;
    if (r2 < h2) {
        full_int = r0h3 / pi * (1. / 6. * s.I_2 - 3. / 40. * r0h2 * s.I_4 + 1. / 40. * r0h3 * s.I_5 + B1 / r03 * s.I0);
    } else if (r2 < 4.0 * h2) {
        full_int = r0h3 / pi * (0.25 * (4. / 3. * s.I_2 - (r0 / h) * s.I_3 + 0.3 * r0h2 * s.I_4 - 1. / 30. * r0h3 * s.I_5 + 1. / 15. * r0h_3 * s.I1) + B2 / r03 * s.I0 + D2);
    } else {
        full_int = r0h3 / pi * (-0.25 * r0h_3 * s.I1 + B3 / r03 * s.I0 + D3);
    }
    return full_int;
}

/* full_integral_new: src/kernel_integral.cpp:410-418 */
double or_full_integral_new(double h, double phi, double r0, double R_0) {
    if (r0 == 0.0) return 0.0;
    if (R_0 == 0.0) return 0.0;
    if (phi == 0.0) return 0.0;
    Wall w = wall_constants(h, r0);
    Edge e = edge_constants(&w, R_0);
    return vertex_integral(&w, &e, phi);
}

/* ============================ tabulated cubic integral ======================================== */

/* The canonical table of generate_density_table(): src/kernel_integral.cpp:57-119. */
typedef struct {
    int nr01, nR_01, nphi1, nr02, nR_02, nphi2, nr0, nR_0, nphi;
    double rl, mul, cphil;
    double* v;
} Table;

static Table g_table;

static double* tab_at(Table* t, int i, int j, int k) {
    return &t->v[((size_t)i * (t->nR_0 + 1) + j) * (t->nphi + 1) + k];
}

static void table_build(void) {
    if (g_table.v) return;
    Table t;
    memset(&t, 0, sizeof t);
    t.nr01 = 50; t.nr02 = 199; t.nR_01 = 150; t.nR_02 = 150; t.nphi1 = 150; t.nphi2 = 150;
    t.rl = 0.1; t.mul = 0.98; t.cphil = 0.98;
    t.nr0 = t.nr01 + t.nr02; t.nR_0 = t.nR_01 + t.nR_02; t.nphi = t.nphi1 + t.nphi2;
    const double h = 1.0;
    t.v = (double*)calloc((size_t)(t.nr0 + 2) * (t.nR_0 + 1) * (t.nphi + 1), sizeof(double));
    const int n = t.nR_01;
    for (int i = 1; i <= t.nr0; ++i) {
        const double r0 = (i <= t.nr01) ? (t.rl / t.nr01) * i * h : t.rl + ((2.0 - t.rl) / t.nr02) * (i - t.nr01) * h;
        for (int j = 0; j < t.nR_0; ++j) {
            const double mu0 = (j < n) ? (t.mul / (n - 1)) * j : t.mul + ((1.0 - t.mul) / n) * (j - n + 1);
            const double R_0 = r0 * sqrt(1.0 - mu0 * mu0) / mu0;
            for (int k = 0; k < t.nphi; ++k) {
                const double phi = (k < n) ? acos((t.cphil / (n - 1)) * k) : acos(t.cphil + ((1.0 - t.cphil) / n) * (k - n + 1));
                *tab_at(&t, i, j, k) = or_full_integral_new(h, phi, r0, R_0);
            }
        }
    }
    for (int j = 0; j < t.nR_0; ++j)
        for (int k = 0; k < t.nphi; ++k) *tab_at(&t, t.nr0 + 1, j, k) = *tab_at(&t, t.nr0, j, k);
    g_table = t;
}

static int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* gridded_integral: src/kernel_integral.cpp:136-190 (warnings of the clamp are not reproduced) */
double or_gridded_integral(double h, double phi, double r0_old, double R_0_old) {
    if (r0_old == 0.0) return 0.0;
    if (R_0_old == 0.0) return 0.0;
    if (phi == 0.0) return 0.0;
    table_build();
    Table* t = &g_table;
    double r0 = r0_old / h, R_0 = R_0_old / h, cphi = cos(phi);
    if (r0 < 0.0) r0 = 0.0;
    if (R_0 < 0.0) R_0 = 0.0;
    double mu0 = r0 / sqrt(r0 * r0 + R_0 * R_0);
    if (r0 > 2.0) r0 = 2.0;
    const int nr01 = t->nr01, nr02 = t->nr02, nR_01 = t->nR_01, nR_02 = t->nR_02, nphi1 = t->nphi1, nphi2 = t->nphi2;
    const double rl = t->rl, mul = t->mul, cphil = t->cphil;
    int i, j, k;
    double frac;
    if (r0 < rl) i = (int)(r0 / (rl / nr01)); else i = nr01 + (int)((r0 - rl) / ((2.0 - rl) / nr02));
    if (mu0 < mul) j = (int)(mu0 / (mul / (nR_01 - 1))); else j = nR_01 - 1 + (int)((mu0 - mul) / ((1.0 - mul) / nR_02));
    if (cphi < cphil) k = (int)(cphi / (cphil / (nphi1 - 1))); else k = nphi1 - 1 + (int)((cphi - cphil) / ((1.0 - cphil) / nphi2));
    i = clampi(i, 0, t->nr0);
    j = clampi(j, 0, t->nR_0 - 1);
    k = clampi(k, 0, t->nphi - 1);
    if (r0 < rl) frac = (r0 - (rl / nr01) * i) / (rl / nr01);
    else frac = (r0 - rl - ((2.0 - rl) / nr02) * (i - nr01)) / ((2.0 - rl) / nr02);
    double fx1 = frac * *tab_at(t, i + 1, j, k) + (1 - frac) * *tab_at(t, i, j, k);
    double fx2 = frac * *tab_at(t, i + 1, j + 1, k) + (1 - frac) * *tab_at(t, i, j + 1, k);
    double fx3 = frac * *tab_at(t, i + 1, j, k + 1) + (1 - frac) * *tab_at(t, i, j, k + 1);
    double fx4 = frac * *tab_at(t, i + 1, j + 1, k + 1) + (1 - frac) * *tab_at(t, i, j + 1, k + 1);
    if (mu0 < mul) frac = (mu0 - mul / (nR_01 - 1) * j) / (mul / (nR_01 - 1));
    else frac = (mu0 - mul - (1.0 - mul) / nR_02 * (j - nR_01 + 1)) / ((1.0 - mul) / nR_02);
    double fy1 = frac * fx2 + (1 - frac) * fx1;
    double fy2 = frac * fx4 + (1 - frac) * fx3;
    if (cphi < cphil) frac = (cphi - cphil / (nphi1 - 1) * k) / (cphil / (nphi1 - 1));
    else frac = (cphi - cphil - (1.0 - cphil) / nphi2 * (k - nphi1 + 1)) / ((1.0 - cphil) / nphi2);
    double fz = frac * fy2 + (1 - frac) * fy1;
    if ((j == (nR_01 + nR_02 - 1)) || (k == (nphi1 + nphi2 - 1))) fz = 0.0;
    return fz;
}

/* ============================ generic table-driven kernels ==================================== */

#define NI KIWI_NI
#define NB KIWI_NB
#define MAXR KIWI_MAX_REGIONS

typedef struct {
    int valid;
    const KiwiKernelTable* K;
    double H, r0, q0;
    int j;
    double coef[MAXR][NI];
    double bphi[MAXR];
} GWall;

typedef struct {
    int valid;
    double R_0, a, a2;
    int nseg;
    int region[MAXR];
    double phi_end[MAXR];
    double offset[MAXR];
} GEdge;

/* basis_integrals: src/kernel_integral_generic.cpp:19-66 */
static void basis_integrals(double a, double a2, double phi, int imin, double* out) {
    const double sinp = sin(phi), cosp = cos(phi);
    const double den = a2 + cosp * cosp;
    const double u = a * sinp / sqrt(den);
    const double one_minus_u2 = cosp * cosp * (1.0 + a2) / den;
    out[0] = atan(u / a);
    out[1] = phi;
    const int mmax = (-imin - 1) / 2;
    double Ioddprev = out[0];
    double K = atanh(u);
    double pow1a2 = 1.0;
    for (int m = 0; m <= mmax && -2 * m - 1 >= imin; ++m) {
        if (m > 0) {
            const int n = m;
            K = u / (2.0 * n * pow(one_minus_u2, n)) + (2.0 * n - 1.0) / (2.0 * n) * K;
            pow1a2 *= (1.0 + a2);
        }
        Ioddprev += a * pow1a2 * K;
        out[1 + (2 * m + 1)] = Ioddprev;
    }
    const int kmax = -imin / 2;
    if (kmax >= 1) {
        double J[NI];
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

/* region_of: src/kernel_integral_generic.cpp:68-72 */
static int region_of(const KiwiKernelTable* K, double q) {
    for (int k = 0; k < K->nreg - 1; ++k)
        if (q <= K->c[k]) return k + 1;
    return K->nreg;
}

/* imin_of: src/kernel_integral_generic.cpp:75-79 */
static int imin_of(const GWall* w, int k) {
    for (int idx = NI - 1; idx >= 0; --idx)
        if (w->coef[k - 1][idx] != 0.0) return 1 - idx;
    return 1;
}

/* G: src/kernel_integral_generic.cpp:82-92 */
static double Gk(const GWall* w, const GEdge* e, int k, double phi) {
    const int imin = imin_of(w, k);
    double I[NI];
    basis_integrals(e->a, e->a2, phi, imin, I);
    double sum = w->bphi[k - 1] * phi;
    for (int idx = 0; idx < NI; ++idx) {
        const double c = w->coef[k - 1][idx];
        if (c != 0.0) sum += c * I[idx];
    }
    return sum;
}

/* generic_wall_constants: src/kernel_integral_generic.cpp:96-117 */
static void gwall(GWall* w, const KiwiKernelTable* K, double H, double r0) {
    memset(w, 0, sizeof *w);
    w->K = K;
    w->H = H;
    w->r0 = r0;
    if (r0 == 0.0) return;
    w->valid = 1;
    w->q0 = r0 / H;
    w->j = region_of(K, w->q0);
    const double A3 = K->A3_pi / M_PI;
    for (int k = 1; k <= K->nreg; ++k) {
        for (int idx = 0; idx < NI; ++idx) {
            const double a = K->a[k - 1][idx];
            w->coef[k - 1][idx] = (a == 0.0) ? 0.0 : A3 * a * pow(w->q0, idx);
        }
        double b = 0.0;
        if (k >= w->j)
            for (int p = NB - 1; p >= 0; --p) b = b * w->q0 + K->B[w->j - 1][k - 1][p];
        w->bphi[k - 1] = A3 * b;
    }
}

/* generic_edge_constants: src/kernel_integral_generic.cpp:119-148 */
static void gedge(GEdge* e, const GWall* w, double R_0) {
    memset(e, 0, sizeof *e);
    e->R_0 = R_0;
    if (!w->valid || R_0 == 0.0) return;
    e->valid = 1;
    e->a = R_0 / w->r0;
    e->a2 = e->a * e->a;
    const KiwiKernelTable* K = w->K;
    const double qR = R_0 / w->H;
    const double r_start = sqrt(w->q0 * w->q0 + qR * qR);
    int k = region_of(K, r_start);
    e->nseg = 0;
    for (; k <= K->nreg; ++k) {
        e->region[e->nseg] = k;
        if (k == K->nreg) {
            e->phi_end[e->nseg] = 0.5 * M_PI;
        } else {
            const double c = K->c[k - 1];
            e->phi_end[e->nseg] = acos(fmin(1.0, qR / sqrt(c * c - w->q0 * w->q0)));
        }
        ++e->nseg;
    }
    e->offset[0] = 0.0;
    for (int s = 0; s + 1 < e->nseg; ++s) {
        const double pb = e->phi_end[s];
        e->offset[s + 1] = e->offset[s] + Gk(w, e, e->region[s], pb) - Gk(w, e, e->region[s + 1], pb);
    }
}

/* generic_vertex_integral: src/kernel_integral_generic.cpp:150-156 */
static double gvertex(const GWall* w, const GEdge* e, double phi) {
    if (!w->valid || !e->valid) return 0.0;
    if (phi == 0.0) return 0.0;
    int s = 0;
    while (s + 1 < e->nseg && phi > e->phi_end[s]) ++s;
    return e->offset[s] + Gk(w, e, e->region[s], phi);
}

double or_generic_full_integral(int kernel, double H, double phi, double r0, double R_0) {
    if (r0 == 0.0 || R_0 == 0.0 || phi == 0.0) return 0.0;
    GWall w;
    GEdge e;
    gwall(&w, &kiwi_kernel_tables[kernel], H, r0);
    gedge(&e, &w, R_0);
    return gvertex(&w, &e, phi);
}

int or_generic_edge_breaks(int kernel, double H, double r0, double R_0, double* phi_end, int max_n) {
    GWall w;
    GEdge e;
    gwall(&w, &kiwi_kernel_tables[kernel], H, r0);
    gedge(&e, &w, R_0);
    int n = e.nseg < max_n ? e.nseg : max_n;
    for (int s = 0; s < n; ++s) phi_end[s] = e.phi_end[s];
    return e.nseg;
}

double or_generic_vertex(int kernel, double H, double r0, double R_0, double phi) {
    GWall w;
    GEdge e;
    gwall(&w, &kiwi_kernel_tables[kernel], H, r0);
    gedge(&e, &w, R_0);
    return gvertex(&w, &e, phi);
}

/* ============================ face walk ======================================================= */

/* The evaluator hooks of src/kernel_integral.cpp:433-467 folded into one tagged struct. */
typedef struct {
    int kind; /* 0 cubic analytic, 1 cubic tabulated, 2 generic */
    double h, ar0, R_0;
    Wall w;
    Edge e;
    GWall gw;
    GEdge ge;
} Eval;

static void ev_set_wall(Eval* ev, double ar0) {
    ev->ar0 = ar0;
    if (ev->kind == 0) ev->w = wall_constants(ev->h, ar0);
    else if (ev->kind == 2) gwall(&ev->gw, ev->gw.K, ev->gw.H, ar0);
}

static void ev_set_edge(Eval* ev, double R_0) {
    ev->R_0 = R_0;
    if (ev->kind == 0) ev->e = edge_constants(&ev->w, R_0);
    else if (ev->kind == 2) gedge(&ev->ge, &ev->gw, R_0);
}

static double ev_at(const Eval* ev, double phi) {
    if (ev->kind == 0) return vertex_integral(&ev->w, &ev->e, phi);
    if (ev->kind == 1) return or_gridded_integral(ev->h, phi, ev->ar0, ev->R_0);
    return gvertex(&ev->gw, &ev->ge, phi);
}

static double dmax(double a, double b) { return a > b ? a : b; }
static double dmin(double a, double b) { return a < b ? a : b; }

/* face_integral_impl: src/kernel_integral.cpp:471-647 */
static double face_impl(double x0, double y0, double z0, double support_radius, const double* V, int n,
                        int* out_vert, Eval* ev) {
    int out_vert_count = 0;
    double face_Msum = 0.0;
    if (n < 3) {
        if (out_vert) *out_vert = out_vert_count;
        return face_Msum;
    }
#define VX(i) V[3 * (i)]
#define VY(i) V[3 * (i) + 1]
#define VZ(i) V[3 * (i) + 2]
    const double x1 = VX(0), y1 = VY(0), z1 = VZ(0);
    const double x2s = VX(1), y2s = VY(1), z2s = VZ(1);
    const double x3s = VX(2), y3s = VY(2), z3s = VZ(2);
    double A = (y2s - y1) * (z3s - z1) - (y3s - y1) * (z2s - z1);
    double B = (z2s - z1) * (x3s - x1) - (z3s - z1) * (x2s - x1);
    double C = (x2s - x1) * (y3s - y1) - (x3s - x1) * (y2s - y1);
    double D = -A * x1 - B * y1 - C * z1;
    double norm = sqrt(A * A + B * B + C * C);
    double r0 = (A * x0 + B * y0 + C * z0 + D) / norm;
    double ar0 = fabs(r0);
    double xp = x0 - r0 * A / norm;
    double yp = y0 - r0 * B / norm;
    double zp = z0 - r0 * C / norm;
    const double x1r = x1 - x0, y1r = y1 - y0, z1r = z1 - z0;
    const double x2sr = x2s - x0, y2sr = y2s - y0, z2sr = z2s - z0;
    const double x3sr = x3s - x0, y3sr = y3s - y0, z3sr = z3s - z0;
    double s2 = x1r * (y2sr * z3sr - z2sr * y3sr) + y1r * (z2sr * x3sr - x2sr * z3sr) + z1r * (x2sr * y3sr - y2sr * x3sr);
    ev_set_wall(ev, ar0);
    int inside_polygon = 1, have_sign = 0;
    double sign_ref = 0.0;
    double min_edge_dist = INFINITY;
    for (int j = 0; j < n; ++j) {
        double x2 = VX(j), y2 = VY(j), z2 = VZ(j);
        double x3, y3, z3;
        if (j == n - 1) {
            x3 = x1; y3 = y1; z3 = z1;
        } else {
            x3 = VX(j + 1); y3 = VY(j + 1); z3 = VZ(j + 1);
        }
        double r23 = sqrt((x3 - x2) * (x3 - x2) + (y3 - y2) * (y3 - y2) + (z3 - z2) * (z3 - z2));
        double r12 = sqrt((xp - x2) * (xp - x2) + (yp - y2) * (yp - y2) + (zp - z2) * (zp - z2));
        double r13 = sqrt((xp - x3) * (xp - x3) + (yp - y3) * (yp - y3) + (zp - z3) * (zp - z3));
        double cosa = ((x3 - x2) * (xp - x2) + (y3 - y2) * (yp - y2) + (z3 - z2) * (zp - z2)) / r12 / r23;
        double R_0;
        if (fabs(cosa) < 1.0) R_0 = r12 * sqrt(1 - cosa * cosa);
        else R_0 = 0.0;
        const double xpr = xp - x0, ypr = yp - y0, zpr = zp - z0;
        const double x2r = x2 - x0, y2r = y2 - y0, z2r = z2 - z0;
        const double x3r = x3 - x0, y3r = y3 - y0, z3r = z3 - z0;
        double s1 = xpr * (y2r * z3r - z2r * y3r) + ypr * (z2r * x3r - x2r * z3r) + zpr * (x2r * y3r - y2r * x3r);
        double phi1 = (R_0 < r12) ? acos(R_0 / r12) : 0.0;
        double phi2 = (R_0 < r13) ? acos(R_0 / r13) : 0.0;
        double ex = x3 - x2, ey = y3 - y2, ez = z3 - z2;
        double tpx = xp - x2, tpy = yp - y2, tpz = zp - z2;
        double side = (ey * tpz - ez * tpy) * A + (ez * tpx - ex * tpz) * B + (ex * tpy - ey * tpx) * C;
        const double side_eps = 1e-9 * norm * r23 * dmax(dmax(fabs(tpx), fabs(tpy)), dmax(fabs(tpz), 1.0));
        if (fabs(side) > side_eps) {
            if (!have_sign) {
                sign_ref = side;
                have_sign = 1;
            } else if ((side > 0) != (sign_ref > 0)) {
                inside_polygon = 0;
            }
        }
        int foot_beyond_endpoint = (r12 * sin(phi1) >= r23) || (r13 * sin(phi2) >= r23);
        double in_plane_dist = foot_beyond_endpoint ? dmin(r12, r13) : R_0;
        min_edge_dist = dmin(min_edge_dist, in_plane_dist);
        double M = (s1 * s2 * r0 <= 0) ? -1.0 : 1.0;
        ev_set_edge(ev, R_0);
        if (foot_beyond_endpoint) {
            if (phi1 >= phi2) M = M * (ev_at(ev, phi1) - ev_at(ev, phi2));
            else M = M * (ev_at(ev, phi2) - ev_at(ev, phi1));
        } else {
            M = M * (ev_at(ev, phi1) + ev_at(ev, phi2));
        }
        face_Msum += M;
    }
#undef VX
#undef VY
#undef VZ
    double face_dist = inside_polygon ? ar0 : sqrt(r0 * r0 + min_edge_dist * min_edge_dist);
    out_vert_count = (face_dist >= support_radius) ? n : 0;
    if (out_vert) *out_vert = out_vert_count;
    return face_Msum;
}

double or_face_integral(double x0, double y0, double z0, int kernel, double h, double support, int tabulated,
                        const double* verts, int n, int* out_vert) {
    static __thread Eval ev; /* GWall is large; keep it off the stack */
    memset(&ev, 0, sizeof ev);
    if (kernel < 0) {
        ev.kind = tabulated ? 1 : 0;
        ev.h = h;
        return face_impl(x0, y0, z0, 2 * h, verts, n, out_vert, &ev);
    }
    ev.kind = 2;
    ev.gw.K = &kiwi_kernel_tables[kernel];
    ev.gw.H = support;
    return face_impl(x0, y0, z0, support, verts, n, out_vert, &ev);
}

/* ============================ sph-to-grid ===================================================== */

/* box_cell_faces: src/cartesian_grid.cpp:54-72 (the winding the face walk needs) */
static void box_cell_faces(double cx, double cy, double cz, double hx, double hy, double hz, double f[6][12]) {
    const double xm = cx - hx, xp = cx + hx;
    const double ym = cy - hy, yp = cy + hy;
    const double zm = cz - hz, zp = cz + hz;
    const double F[6][12] = {
        {xp, ym, zp, xp, yp, zp, xp, yp, zm, xp, ym, zm},
        {xm, yp, zm, xm, yp, zp, xm, ym, zp, xm, ym, zm},
        {xp, yp, zm, xp, yp, zp, xm, yp, zp, xm, yp, zm},
        {xm, ym, zp, xp, ym, zp, xp, ym, zm, xm, ym, zm},
        {xm, yp, zp, xp, yp, zp, xp, ym, zp, xm, ym, zp},
        {xp, ym, zm, xp, yp, zm, xm, yp, zm, xm, ym, zm},
    };
    memcpy(f, F, sizeof F);
}

static int imax(int a, int b) { return a > b ? a : b; }
static int imin(int a, int b) { return a < b ? a : b; }

/* run_sph_to_grid_stage's particle loop and finalisation: src/cartesian_grid.cpp:184-317 */
int or_sph_to_grid(int64_t n, const double* x, const double* y, const double* z, const double* vx,
                   const double* vy, const double* vz, const double* m, const double* h, const double bounds[6],
                   int nx, int ny, int nz, int kernel, double support_in_h, int tabulated, int64_t p_begin,
                   int64_t p_end, double* density, double* gvx, double* gvy, double* gvz, double* raw4,
                   OrStats* stats) {
    const double x_min = bounds[0], x_max = bounds[1], y_min = bounds[2], y_max = bounds[3];
    const double z_min = bounds[4], z_max = bounds[5];
    if (nx <= 0 || ny <= 0 || nz <= 0) return -1;
    const double dpx = (x_max - x_min) / nx, dpy = (y_max - y_min) / ny, dpz = (z_max - z_min) / nz;
    const size_t ncell = (size_t)nx * (size_t)ny * (size_t)nz;
    double* dens = (double*)calloc(ncell, sizeof(double));
    double* px = (double*)calloc(ncell, sizeof(double));
    double* py = (double*)calloc(ncell, sizeof(double));
    double* pz = (double*)calloc(ncell, sizeof(double));
    if (!dens || !px || !py || !pz) return -2;
    const double hpx = 0.5 * dpx, hpy = 0.5 * dpy, hpz = 0.5 * dpz;
    const double cell_volume = dpx * dpy * dpz;
    double vx_mean = 0, vy_mean = 0, vz_mean = 0;
    OrStats st;
    memset(&st, 0, sizeof st);
    if (p_end < 0 || p_end > n) p_end = n;
    for (int64_t idx = 0; idx < n; ++idx) {
        vx_mean += vx[idx];
        vy_mean += vy[idx];
        vz_mean += vz[idx];
    }
    double faces[6][12];
    for (int64_t idx = p_begin; idx < p_end; ++idx) {
        const double x0 = x[idx], y0 = y[idx], z0 = z[idx];
        const double mm = m[idx], hh = h[idx];
        if (hh <= 0.0) continue;
        const double radius = support_in_h * hh;
        int ixmin = (int)floor((x0 - radius - x_min) / dpx);
        int ixmax = (int)floor((x0 + radius - x_min) / dpx);
        int iymin = (int)floor((y0 - radius - y_min) / dpy);
        int iymax = (int)floor((y0 + radius - y_min) / dpy);
        int izmin = (int)floor((z0 - radius - z_min) / dpz);
        int izmax = (int)floor((z0 + radius - z_min) / dpz);
        ixmin = imax(ixmin, 0); ixmax = imin(ixmax, nx - 1);
        iymin = imax(iymin, 0); iymax = imin(iymax, ny - 1);
        izmin = imax(izmin, 0); izmax = imin(izmax, nz - 1);
        if (ixmin > ixmax || iymin > iymax || izmin > izmax) {
            ++st.skipped_outside;
            continue;
        }
        for (int ix = ixmin; ix <= ixmax; ++ix) {
            const double cx = x_min + (ix + 0.5) * dpx;
            for (int iy = iymin; iy <= iymax; ++iy) {
                const double cy = y_min + (iy + 0.5) * dpy;
                for (int iz = izmin; iz <= izmax; ++iz) {
                    const double cz = z_min + (iz + 0.5) * dpz;
                    ++st.bbox_pairs;
                    {   /* closest point of the cell to the particle, for the sphere-pair count */
                        double ddx = fabs(x0 - cx) - hpx, ddy = fabs(y0 - cy) - hpy, ddz = fabs(z0 - cz) - hpz;
                        ddx = ddx > 0 ? ddx : 0; ddy = ddy > 0 ? ddy : 0; ddz = ddz > 0 ? ddz : 0;
                        if (ddx * ddx + ddy * ddy + ddz * ddz < radius * radius) ++st.sphere_pairs;
                    }
                    box_cell_faces(cx, cy, cz, hpx, hpy, hpz, faces);
                    double Msum = 0.0;
                    for (int f = 0; f < 6; ++f)
                        Msum += or_face_integral(x0, y0, z0, kernel, hh, radius, tabulated, faces[f], 4, NULL);
                    if (Msum < 0.0) {
                        ++st.neg_clamped;
                        if (Msum <= -0.01) ++st.neg_warned;
                        Msum = 0.0;
                    }
                    if (Msum == 0.0) continue;
                    const size_t i3 = ((size_t)ix * ny + (size_t)iy) * nz + (size_t)iz;
                    dens[i3] += Msum * mm;
                    px[i3] += Msum * mm * vx[idx];
                    py[i3] += Msum * mm * vy[idx];
                    pz[i3] += Msum * mm * vz[idx];
                }
            }
        }
    }
    if (n > 0) {
        vx_mean /= (double)n;
        vy_mean /= (double)n;
        vz_mean /= (double)n;
    }
    for (size_t i = 0; i < ncell; ++i) {
        if (density) density[i] = dens[i] / cell_volume;
        double ux = vx_mean, uy = vy_mean, uz = vz_mean;
        if (dens[i] > 0.0) {
            ux = px[i] / dens[i];
            uy = py[i] / dens[i];
            uz = pz[i] / dens[i];
        }
        if (gvx) gvx[i] = ux;
        if (gvy) gvy[i] = uy;
        if (gvz) gvz[i] = uz;
        if (raw4) {
            raw4[i] = dens[i];
            raw4[ncell + i] = px[i];
            raw4[2 * ncell + i] = py[i];
            raw4[3 * ncell + i] = pz[i];
        }
    }
    free(dens); free(px); free(py); free(pz);
    if (stats) *stats = st;
    return 0;
}

/* ============================ Voronoi map ===================================================== */

/* Per-particle face cache: open addressing on the unordered cell pair (src/mapping.cpp:56-93). */
typedef struct {
    int64_t* key;
    int32_t* owner;
    double* val;
    int64_t* used;
    int64_t nused, cap;
} FCache;

static void fc_init(FCache* c, int64_t cap) {
    c->cap = 1;
    while (c->cap < cap) c->cap <<= 1;
    c->key = (int64_t*)malloc(sizeof(int64_t) * c->cap);
    c->owner = (int32_t*)malloc(sizeof(int32_t) * c->cap);
    c->val = (double*)malloc(sizeof(double) * c->cap);
    c->used = (int64_t*)malloc(sizeof(int64_t) * c->cap);
    for (int64_t i = 0; i < c->cap; ++i) c->key[i] = -1;
    c->nused = 0;
}

static void fc_clear(FCache* c) {
    for (int64_t i = 0; i < c->nused; ++i) c->key[c->used[i]] = -1;
    c->nused = 0;
}

static void fc_free(FCache* c) { free(c->key); free(c->owner); free(c->val); free(c->used); }

static int64_t fc_slot(const FCache* c, int64_t k) {
    uint64_t hsh = (uint64_t)k * 0x9E3779B97F4A7C15ull;
    int64_t i = (int64_t)(hsh >> 20) & (c->cap - 1);
    while (c->key[i] != -1 && c->key[i] != k) i = (i + 1) & (c->cap - 1);
    return i;
}

static int64_t pair_key(int32_t a, int32_t b) {
    int32_t lo = a < b ? a : b, hi = a < b ? b : a;
    return ((int64_t)lo << 32) | (uint32_t)hi;
}

/* run_mapping_stage's particle BFS and finalisation: src/mapping.cpp:105-206, 400-502 */
int or_map_voronoi(int64_t n, const int32_t* home_cell, const double* x, const double* y, const double* z,
                   const double* vx, const double* vy, const double* vz, const double* m, const double* h,
                   int64_t n_cells, const int64_t* face_off, const int64_t* vert_off, const double* vxyz,
                   const int32_t* face_nbr, const double* volume, int kernel, double support_in_h, int tabulated,
                   double* density, double* gvx, double* gvy, double* gvz, double* raw4, int64_t* visited_pairs) {
    double* dens = (double*)calloc(n_cells, sizeof(double));
    double* px = (double*)calloc(n_cells, sizeof(double));
    double* py = (double*)calloc(n_cells, sizeof(double));
    double* pz = (double*)calloc(n_cells, sizeof(double));
    int64_t* mark = (int64_t*)calloc(n_cells, sizeof(int64_t));
    int32_t* queue = (int32_t*)malloc(sizeof(int32_t) * (n_cells > 0 ? n_cells : 1));
    int64_t max_faces = 0;
    for (int64_t c = 0; c < n_cells; ++c) max_faces += face_off[c + 1] - face_off[c];
    FCache fc;
    fc_init(&fc, 2 * max_faces + 16);
    double* fv = (double*)malloc(sizeof(double) * 3 * 4096);
    double vx_mean = 0, vy_mean = 0, vz_mean = 0;
    int64_t visits = 0;
    for (int64_t idx = 0; idx < n; ++idx) {
        vx_mean += vx[idx];
        vy_mean += vy[idx];
        vz_mean += vz[idx];
        const double hh = h[idx];
        if (hh <= 0.0) continue;
        const int32_t k0 = home_cell[idx];
        if (k0 < 0) continue;
        const int64_t ind = idx + 1;
        const double x0 = x[idx], y0 = y[idx], z0 = z[idx], radius = support_in_h * hh;
        int64_t top = 1, bottom = 0;
        queue[0] = k0;
        mark[k0] = ind;
        fc_clear(&fc);
        while (bottom < top) {
            const int32_t cell = queue[bottom];
            double Msum = 0.0;
            for (int64_t f = face_off[cell]; f < face_off[cell + 1]; ++f) {
                const int32_t nb = face_nbr[f];
                const int nv = (int)(vert_off[f + 1] - vert_off[f]);
                int64_t slot = -1;
                if (nb >= 0) {
                    int64_t key = pair_key(cell, nb);
                    slot = fc_slot(&fc, key);
                    if (fc.key[slot] == key) {
                        Msum += (fc.owner[slot] == cell) ? fc.val[slot] : -fc.val[slot];
                        continue;
                    }
                }
                for (int v = 0; v < nv && v < 4096; ++v) {
                    fv[3 * v] = vxyz[3 * (vert_off[f] + v)];
                    fv[3 * v + 1] = vxyz[3 * (vert_off[f] + v) + 1];
                    fv[3 * v + 2] = vxyz[3 * (vert_off[f] + v) + 2];
                }
                int ov = 0;
                double fm = or_face_integral(x0, y0, z0, kernel, hh, radius, tabulated, fv, nv, &ov);
                Msum += fm;
                if (nb >= 0) {
                    fc.key[slot] = pair_key(cell, nb);
                    fc.owner[slot] = cell;
                    fc.val[slot] = fm;
                    fc.used[fc.nused++] = slot;
                }
                if (ov != nv && nb >= 0 && mark[nb] != ind) {
                    queue[top++] = nb;
                    mark[nb] = ind;
                }
            }
            if (Msum < 0.0) Msum = 0.0;
            dens[cell] += Msum * m[idx];
            px[cell] += Msum * m[idx] * vx[idx];
            py[cell] += Msum * m[idx] * vy[idx];
            pz[cell] += Msum * m[idx] * vz[idx];
            ++bottom;
        }
        visits += top;
    }
    if (n > 0) {
        vx_mean /= (double)n;
        vy_mean /= (double)n;
        vz_mean /= (double)n;
    }
    for (int64_t i = 0; i < n_cells; ++i) {
        if (density) density[i] = (volume[i] > 0.0) ? dens[i] / volume[i] : 0.0;
        double ux = vx_mean, uy = vy_mean, uz = vz_mean;
        if (dens[i] > 0.0) {
            ux = px[i] / dens[i];
            uy = py[i] / dens[i];
            uz = pz[i] / dens[i];
        }
        if (gvx) gvx[i] = ux;
        if (gvy) gvy[i] = uy;
        if (gvz) gvz[i] = uz;
        if (raw4) {
            raw4[i] = dens[i];
            raw4[n_cells + i] = px[i];
            raw4[2 * n_cells + i] = py[i];
            raw4[3 * n_cells + i] = pz[i];
        }
    }
    if (visited_pairs) *visited_pairs = visits;
    fc_free(&fc);
    free(fv); free(queue); free(mark); free(dens); free(px); free(py); free(pz);
    return 0;
}
