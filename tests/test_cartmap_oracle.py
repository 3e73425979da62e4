"""The oracle's brute-force restatement of the cartesian-map stage's point location
(run_cartesian_map_stage, src/cartesian_map.cpp:84-200) pinned to the reference's own stage
(tests/golden/cmap_*.npz, made by tests/golden/make_cartmap_fixtures.py with the reference library): every
cell's owning site id and its copied mapping values, bit for bit."""
import glob
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "cmap_*.npz")))


def site_values(d):
    """Per site (point-set order): its mapping row's values and whether it has one."""
    row = {int(i): k for k, i in enumerate(d["row_id"])}
    k = np.array([row.get(int(i), -1) for i in d["pt_id"]])
    has = k >= 0
    vals = [np.where(has, d["row_" + f][np.maximum(k, 0)], 0.0) for f in ("density", "vx", "vy", "vz")]
    return vals, has


@pytest.mark.parametrize("fn", GOLDEN, ids=[os.path.basename(f)[5:-4] for f in GOLDEN])
def test_oracle_matches_reference_stage(oracle, fn):
    d = np.load(fn)
    res = int(d["resolution"])
    near = oracle.cartesian_map_nearest(d["pt_xyz"], d["bounds"], res)
    assert np.all(near >= 0)
    assert np.array_equal(d["pt_id"][near], d["out_cell_id"])
    vals, has = site_values(d)
    for f, v in zip(("density", "vx", "vy", "vz"), vals):
        assert np.array_equal(np.where(has[near], v[near], 0.0), d["out_" + f]), f
    # sites outside the domain are in the point set but never own a cell
    b = d["bounds"]
    xyz = d["pt_xyz"].reshape(-1, 3)
    outside = ~((xyz[:, 0] >= b[0]) & (xyz[:, 0] <= b[1]) & (xyz[:, 1] >= b[2]) & (xyz[:, 1] <= b[3]) &
                (xyz[:, 2] >= b[4]) & (xyz[:, 2] <= b[5]))
    assert not np.isin(np.nonzero(outside)[0], near).any()


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_container_filter_and_order_match_reference(oracle, reflib, seed):
    """Which sites the reference's Voro++ container keeps (a site on an upper wall falls out) and the order
    it walks them in, restated by the oracle, against a container built as the reference builds it."""
    rng = np.random.default_rng(seed)
    xyz = rng.uniform(-0.1, 1.1, (400, 3))
    xyz[:20, 0] = 1.0
    xyz[20:40, 1] = 0.0
    xyz[40:45] = [1.0, 1.0, 1.0]
    xyz[45:50] = [0.0, 0.0, 0.0]
    for b in ((0.0, 1.0, 0.0, 1.0, 0.0, 1.0), (0.0, 1.0, -0.3, 1.0, 0.0, 0.7)):
        for scale in (3.0, 1.0):
            assert np.array_equal(oracle.container_order(xyz, b, scale), reflib.container_order(xyz, b, scale))
