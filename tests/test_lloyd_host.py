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
