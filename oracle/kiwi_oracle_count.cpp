// Operation-counting instance of the oracle -- TEST / MEASUREMENT INFRASTRUCTURE ONLY.
//
// oracle_core.inc compiled with R = Counted, a double that counts every arithmetic operation it takes
// part in: each +, -, *, / and sqrt is one flop; each sin, cos, acos, atan, atanh, log and pow is one
// transcendental (sincos counts as two).  Running it over a sample of a workload's (particle, cell)
// pairs gives the algorithmic work per pair, F_pair (flops) and T_pair (transcendentals), of the
// reference's evaluation order -- the numerator of the cell-integral kernel's roofline.
#include <math.h>
#include <stdio.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../kiwi_b200/csrc/kernel_tables.h"

extern "C" {
typedef struct OrStats {
    int64_t bbox_pairs, sphere_pairs, skipped_outside, neg_clamped, neg_warned;
} OrStats;
}

static thread_local uint64_t g_flops = 0, g_trans = 0;

struct Counted {
    double v;
    Counted() = default;
    constexpr Counted(double x) : v(x) {}
    explicit operator double() const { return v; }
    explicit operator int() const { return (int)v; }
};
static inline Counted mk(double x) { return Counted(x); }
#define BIN(op)                                                                            \
    static inline Counted operator op(Counted a, Counted b) { ++g_flops; return mk(a.v op b.v); } \
    static inline Counted operator op(Counted a, double b) { ++g_flops; return mk(a.v op b); }    \
    static inline Counted operator op(double a, Counted b) { ++g_flops; return mk(a op b.v); }    \
    static inline Counted operator op(Counted a, int b) { ++g_flops; return mk(a.v op b); }       \
    static inline Counted operator op(int a, Counted b) { ++g_flops; return mk(a op b.v); }
BIN(+)
BIN(-)
BIN(*)
BIN(/)
#undef BIN
static inline Counted operator-(Counted a) { return mk(-a.v); }
#define CMP(op)                                                                  \
    static inline bool operator op(Counted a, Counted b) { return a.v op b.v; }  \
    static inline bool operator op(Counted a, double b) { return a.v op b; }     \
    static inline bool operator op(double a, Counted b) { return a op b.v; }
CMP(<)
CMP(>)
CMP(<=)
CMP(>=)
CMP(==)
CMP(!=)
#undef CMP
#define ASG(op, bop)                                                                         \
    static inline Counted& operator op(Counted& a, Counted b) { a = a bop b; return a; }     \
    static inline Counted& operator op(Counted& a, double b) { a = a bop b; return a; }
ASG(+=, +)
ASG(-=, -)
ASG(*=, *)
ASG(/=, /)
#undef ASG

static inline Counted c_sqrt(Counted a) { ++g_flops; return mk(sqrt(a.v)); }
static inline Counted c_acos(Counted a) { ++g_trans; return mk(acos(a.v)); }
static inline Counted c_atan(Counted a) { ++g_trans; return mk(atan(a.v)); }
static inline Counted c_log(Counted a) { ++g_trans; return mk(log(a.v)); }
static inline Counted c_sin(Counted a) { ++g_trans; return mk(sin(a.v)); }
static inline Counted c_cos(Counted a) { ++g_trans; return mk(cos(a.v)); }
static inline Counted c_atanh(Counted a) { ++g_trans; return mk(atanh(a.v)); }
static inline Counted c_pow(Counted a, Counted b) { ++g_trans; return mk(pow(a.v, b.v)); }
static inline Counted c_fabs(Counted a) { return mk(fabs(a.v)); }
static inline Counted c_fmin(Counted a, Counted b) { return mk(fmin(a.v, b.v)); }
static inline Counted c_floor(Counted a) { return mk(floor(a.v)); }
static inline void c_sincos(Counted a, Counted* s, Counted* c) { g_trans += 2; s->v = sin(a.v); c->v = cos(a.v); }

typedef Counted R;
#define R_PI Counted(M_PI)
#define Q(a, b) Counted((double)(a) / (double)(b))
#define F_SQRT c_sqrt
#define F_ACOS c_acos
#define F_ATAN c_atan
#define F_LOG c_log
#define F_SIN c_sin
#define F_COS c_cos
#define F_FABS c_fabs
#define F_ATANH c_atanh
#define F_POW c_pow
#define F_FMIN c_fmin
#define F_FLOOR c_floor
#define F_SINCOS c_sincos
#define API(name) orc_##name

extern "C" {
#include "oracle_core.inc"

void orc_reset(void) { g_flops = g_trans = 0; }
void orc_counts(uint64_t* flops, uint64_t* trans) { *flops = g_flops; *trans = g_trans; }
}

// Per-item costs of the lattice-factorised evaluation (kiwi_b200/csrc/lattice.cuh): one edge tier
// (wall tier + edge tier for a (plane, edge line)) and one lattice vertex pyramid (wall tier, the right-
// triangle angle and its sine and cosine, the I-series and the region formula).
extern "C" void orc_edge_cost(double h, double r0, double R0, uint64_t* f, uint64_t* t) {
    g_flops = g_trans = 0;
    Wall w = wall_constants(h, r0);
    Edge e = edge_constants(&w, R0);
    (void)e;
    *f = g_flops;
    *t = g_trans;
}

extern "C" void orc_lattice_vertex_cost(double h, double r0d, double R0d, double td, uint64_t* f, uint64_t* t) {
    g_flops = g_trans = 0;
    const Counted r0(r0d), R_0(R0d), tt(td);
    Wall w = wall_constants(h, r0);
    Edge e = edge_constants(&w, R_0);  // D2, D3 come from the shared edge tier: not counted here
    g_flops = g_trans = 0;
    w = wall_constants(h, r0);
    const Counted a = R_0 / r0;
    const Counted a2 = a * a;
    const Counted s2 = R_0 * R_0 + tt * tt;
    const Counted rr = c_sqrt(s2);
    ++g_trans;  // atan2(t, R_0)
    const Counted phi(atan2(td, R0d));
    Series s = series_at(phi, tt / rr, R_0 / rr, a, a2);
    const Counted r2 = r0 * r0 + s2;
    Counted full;
    if (r2 < w.h2)
        full = w.r0h3 / R_PI * (Q(1, 6) * s.I_2 - Q(3, 40) * w.r0h2 * s.I_4 + Q(1, 40) * w.r0h3 * s.I_5 + w.B1 / w.r03 * s.I0);
    else if (r2 < 4.0 * w.h2)
        full = w.r0h3 / R_PI * (0.25 * (Q(4, 3) * s.I_2 - (r0 / h) * s.I_3 + Q(3, 10) * w.r0h2 * s.I_4 - Q(1, 30) * w.r0h3 * s.I_5 + Q(1, 15) * w.r0h_3 * s.I1) + w.B2 / w.r03 * s.I0 + e.D2);
    else
        full = w.r0h3 / R_PI * (-0.25 * w.r0h_3 * s.I1 + w.B3 / w.r03 * s.I0 + e.D3);
    (void)full;
    *f = g_flops;
    *t = g_trans;
}
