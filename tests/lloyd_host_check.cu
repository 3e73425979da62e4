// Host build of the Lloyd step's per-cell algorithm (kiwi_b200/csrc/lloyd.cu: search bins, shells of
// candidates clipped nearest first, face-fan moments), for a CPU check against the reference's lloyd_step.
// Test infrastructure: compiled by tests/test_lloyd_host.py.
#include "lloyd.cu"
#include <vector>
#include <algorithm>
#include <numeric>
extern "C" int host_full(long n, const double* xyz, const double* b, double* cen, double* vol, int* status) {
    VoroBlocks V = voro_blocks_for(b, n, xyz, 3.0);
    long n_kept = 0;
    for (long i = 0; i < n; ++i) n_kept += voro_block(V, xyz[3*i], xyz[3*i+1], xyz[3*i+2]) >= 0;
    SiteBins B; site_bins_shape(b, n_kept, B);
    const long nbins = (long)B.nbx * B.nby * B.nbz;
    std::vector<long> key(n), ord(n);
    for (long i = 0; i < n; ++i) {
        key[i] = nbins;
        if (voro_block(V, xyz[3*i], xyz[3*i+1], xyz[3*i+2]) >= 0)
            key[i] = ((long)bin_of(xyz[3*i], B.x0, B.wx, B.nbx) * B.nby + bin_of(xyz[3*i+1], B.y0, B.wy, B.nby)) * B.nbz + bin_of(xyz[3*i+2], B.z0, B.wz, B.nbz);
    }
    std::iota(ord.begin(), ord.end(), 0);
    std::stable_sort(ord.begin(), ord.end(), [&](long a, long c) { return key[a] < key[c]; });
    std::vector<double> sx(n), sy(n), sz(n); std::vector<int32_t> sidx(n); std::vector<int64_t> range(2 * nbins, 0);
    for (long i = 0; i < n; ++i) { long s = ord[i]; sx[i] = xyz[3*s]; sy[i] = xyz[3*s+1]; sz[i] = xyz[3*s+2]; sidx[i] = (int32_t)s;
        long k = key[s]; if (k >= nbins) continue;
        if (i == 0 || key[ord[i-1]] != k) range[2*k] = i;
        if (i == n-1 || key[ord[i+1]] != k) range[2*k+1] = i + 1; }
    B.range = range.data(); B.sx = sx.data(); B.sy = sy.data(); B.sz = sz.data(); B.sidx = sidx.data();
    const double ext = std::max(b[1] - b[0], std::max(b[3] - b[2], b[5] - b[4]));
    Cell* c = new Cell;
    for (long i = 0; i < n; ++i) status[i] = -1;
    for (long q = 0; q < n_kept; ++q) {
        double cc[3], vv = 0;
        int st = build_cell(*c, B, V, q, 1e-12 * ext, cc, &vv);
        long o = sidx[q];
        cen[3*o] = cc[0]; cen[3*o+1] = cc[1]; cen[3*o+2] = cc[2]; vol[o] = vv; status[o] = st;
    }
    delete c;
    return 0;
}
