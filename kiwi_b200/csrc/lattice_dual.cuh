// Generic-kernel edge records with forward derivatives, for the adjoint's lattice form: the record of
// lattice_generic_edge_t evaluated in DualN<N>.  The segment boundaries phi_end are only compared with the
// vertices' angles (a choice taken on values), so they are kept as values; the continuity offsets carry
// their derivatives.  Layout, kLatGenDualRec(N) doubles: [0] = nseg + 8 x first region, [1..3] = phi_end of
// segments 0..2, then the offsets of segments 1..3 as (value, d[0..N-1]) each.
#pragma once

#include "dual.cuh"
#include "lattice_math.cuh"

namespace kiwi_b200 {

template <int N>
constexpr int lat_gen_dual_rec() {
    return 4 + 3 * (N + 1);
}

template <int N>
struct GenEdgeWriterDual {
    double* rec;
    KIWI_HD void set_packed(double v) { rec[0] = v; }
    KIWI_HD void set_segment(int s, const DualN<N>& phi_end, const DualN<N>& off) {
        rec[1 + s] = phi_end.v;
        double* o = rec + 4 + (N + 1) * s;
        o[0] = off.v;
#pragma unroll
        for (int k = 0; k < N; ++k) o[1 + k] = off.d[k];
    }
};

// lattice_generic_edge in DualN<N>: r0 and R0 carry their derivatives; H is held fixed.
template <int N>
KIWI_LAT void lattice_generic_edge_dual(const KiwiKernelTable* K, double H, const DualN<N>& r0, const DualN<N>& R0,
                                        double* rec) {
    for (int i = 0; i < lat_gen_dual_rec<N>(); ++i) rec[i] = 0.0;
    GenEdgeWriterDual<N> w{rec};
    lattice_generic_edge_t(K, H, r0, R0, w);
}

// The six dual edge records of a lattice point (lattice_generic_point's reader): base + kLatGenDualRec x
// slot, in PointEdge order.
template <int N>
struct GenEdgeRecsDual {
    const double* base;
    int slot[6];
    KIWI_HD const double* rec(int e) const {
        const int sl = e < 3 ? (e == 0 ? slot[0] : (e == 1 ? slot[1] : slot[2]))
                             : (e == 3 ? slot[3] : (e == 4 ? slot[4] : slot[5]));
        return base + lat_gen_dual_rec<N>() * sl;
    }
    KIWI_HD int packed(const double* r) const { return (int)r[0]; }
    KIWI_HD double phi_end(const double* r, int s) const { return r[1 + s]; }
    KIWI_HD DualN<N> offset(const double* r, int s) const {  // segment s >= 1
        const double* o = r + 4 + (N + 1) * (s - 1);
        DualN<N> v(o[0]);
#pragma unroll
        for (int k = 0; k < N; ++k) v.d[k] = o[1 + k];
        return v;
    }
};

}  // namespace kiwi_b200
