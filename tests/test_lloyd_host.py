"""The Lloyd step's per-cell algorithm (kiwi_b200/csrc/lloyd.cu), compiled for the host and run on the CPU,
against the reference's own lloyd_step (tests/golden/lloyd_*.npz): the same search bins, shells, nearest-
first clipping and face-fan moments the kernel runs, so a fault in the cell construction shows here without
a GPU.  The walk order comes from the oracle's restatement of the container (pinned in
tests/test_cartmap_oracle.py)."""
import ctypes as C
import glob
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "lloyd_*.npz")))
_dp = C.POINTER(C.c_double)


@pytest.fixture(scope="module")
def cells(tmp_path_factory):
    out = tmp_path_factory.mktemp("lloyd") / "liblloyd_host.so"
    nvcc = os.environ.get("NVCC", "nvcc")
    subprocess.run([nvcc, "-O2", "-std=c++17", "--expt-relaxed-constexpr", "--fmad=false",
                    "-I" + os.path.join(ROOT, "include"), "-I" + os.path.join(ROOT, "kiwi_b200", "csrc"),
                    "-Xcompiler", "-fPIC", "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", str(out),
                    os.path.join(ROOT, "tests", "lloyd_host_check.cu"), "-cudart", "static"], check=True)
    L = C.CDLL(str(out))

    def run(xyz, b):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        n = len(xyz)
        bb = np.asarray(b, dtype=np.float64)
        cen, vol, st = np.zeros((max(n, 1), 3)), np.zeros(max(n, 1)), np.zeros(max(n, 1), np.int32)
        L.host_full(C.c_long(n), xyz.ctypes.data_as(_dp), bb.ctypes.data_as(_dp), cen.ctypes.data_as(_dp),
                    vol.ctypes.data_as(_dp), st.ctypes.data_as(C.POINTER(C.c_int)))
        return cen[:n], vol[:n], st[:n]

    return run


@pytest.mark.parametrize("fn", GOLDEN, ids=[os.path.basename(f)[6:-4] for f in GOLDEN])
def test_cells_match_reference(cells, oracle, fn):
    d = np.load(fn)
    b = d["bounds"]
    order = oracle.container_order(d["xyz"], b)
    assert np.array_equal(d["ids"][order], d["ref_id"])
    cen, vol, st = cells(d["xyz"], b)
    assert np.all(st[order] == 0)
    ext = max(b[1] - b[0], b[3] - b[2], b[5] - b[4])
    assert np.abs(cen[order] - d["ref_xyz"]).max() <= 1e-12 * ext
    dom = (b[1] - b[0]) * (b[3] - b[2]) * (b[5] - b[4])
    assert abs(vol[order].sum() - dom) <= 1e-12 * dom


def test_clustered_cells_tile_the_domain(cells, oracle):
    rng = np.random.default_rng(11)
    n = 20_000
    xyz = np.concatenate([rng.normal(5.0, 0.7, (n // 2, 3)), rng.uniform(0, 10, (n // 2, 3))])
    b = (0.0, 10.0, 0.0, 10.0, 0.0, 10.0)
    order = oracle.container_order(xyz, b)
    cen, vol, st = cells(xyz, b)
    assert np.all(st[order] == 0)
    assert abs(vol[order].sum() - 1000.0) <= 1e-10 * 1000.0


def test_dense_cells_match_an_independent_construction(cells, reflib):
    """Dense clustered sites (a filament, as in the column recipe): interior cells against qhull's
    Voronoi regions (scipy), an independent construction.  Here the reference's Voro++ centroids can sit
    ~1e-8 from both (its vertex tolerance), so the reference is compared with that looser bound."""
    from scipy.spatial import ConvexHull, Voronoi

    rng = np.random.default_rng(12)
    n = 4000
    xyz = np.column_stack([1.0 + 0.05 * rng.standard_normal(n), 1.0 + 0.05 * rng.standard_normal(n), rng.random(n) * 2])
    xyz = np.concatenate([xyz, rng.random((500, 3)) * 2])
    b = (0.0, 2.0, 0.0, 2.0, 0.0, 2.0)
    cen, vol, st = cells(xyz, b)
    vor = Voronoi(xyz)
    inner = np.nonzero((np.abs(xyz[:, 0] - 1) < 0.03) & (np.abs(xyz[:, 1] - 1) < 0.03) &
                       (xyz[:, 2] > 0.3) & (xyz[:, 2] < 1.7))[0][:200]
    worst = 0.0
    for s in inner:
        reg = vor.regions[vor.point_region[s]]
        assert -1 not in reg
        V = vor.vertices[reg]
        hull = ConvexHull(V)
        acc, tot = np.zeros(3), 0.0
        for simp in hull.simplices:
            a, p, q = V[simp]
            v = abs(np.dot(a - xyz[s], np.cross(p - xyz[s], q - xyz[s]))) / 6
            tot += v
            acc += v * (xyz[s] + a + p + q) / 4
        worst = max(worst, np.abs(cen[s] - acc / tot).max() / np.cbrt(tot))
        assert abs(vol[s] - hull.volume) <= 1e-10 * hull.volume
    assert worst <= 1e-11, worst
    rid, rxyz = reflib.lloyd_step(xyz, np.arange(len(xyz), dtype=np.int32), b)
    assert np.abs(cen[rid] - rxyz).max() <= 1e-6
