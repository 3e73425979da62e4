"""GPU parity of the cartesian-map stage's point location (run_cartesian_map_stage,
src/cartesian_map.cpp:84-200; kiwi_cartesian_map) against the reference's own stage
(tests/golden/cmap_*.npz, made by tests/golden/make_cartmap_fixtures.py with the reference library) and
against the oracle's brute-force nearest-site search and an independent k-d tree: the owning site of every
cell is an exact, integer result, so the bar is equality (distances equal to the nearest distance at scale,
where exact ties may differ only in the chosen index)."""
import glob
import os

import numpy as np
import pytest

from test_cartmap_oracle import site_values

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "cmap_*.npz")))


@pytest.mark.parametrize("fn", GOLDEN, ids=[os.path.basename(f)[5:-4] for f in GOLDEN])
def test_matches_reference_stage(kiwi, ctx, fn):
    d = np.load(fn)
    vals, has = site_values(d)
    m = kiwi.cartesian_map(d["pt_xyz"].reshape(-1, 3), d["bounds"], int(d["resolution"]), *vals,
                           site_id=d["pt_id"], mapped=has, ctx=ctx)
    assert np.array_equal(m.voronoi_cell_id, d["out_cell_id"])
    for f in ("density", "vx", "vy", "vz"):
        assert np.array_equal(getattr(m, f), d["out_" + f]), f
    assert m.stats["unresolved"] == 0
    row_ids = set(d["row_id"].tolist())
    assert m.stats["unmapped"] == int(sum(1 for i in d["out_cell_id"].tolist() if i not in row_ids))


def _grid_centres(bounds, res):
    b = np.asarray(bounds, float)
    ax = [b[2 * a] + (np.arange(res) + 0.5) * ((b[2 * a + 1] - b[2 * a]) / res) for a in range(3)]
    X, Y, Z = np.meshgrid(*ax, indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)


@pytest.mark.parametrize("case", ["uniform", "clustered", "noncube"])
def test_random_sites_vs_oracle(kiwi, ctx, oracle, case):
    rng = np.random.default_rng({"uniform": 1, "clustered": 2, "noncube": 3}[case])
    if case == "uniform":
        bounds, res, xyz = (0.0, 1.0, 0.0, 1.0, 0.0, 1.0), 20, rng.random((500, 3))
    elif case == "clustered":
        bounds, res = (-2.0, 2.0, -2.0, 2.0, -2.0, 2.0), 17
        xyz = np.concatenate([rng.normal(0, 0.1, (400, 3)), rng.uniform(-2.2, 2.2, (100, 3))])
    else:
        bounds, res = (-36.0, -34.0, -60.0, -57.5, 1.4, 2.0), 15
        xyz = rng.uniform([-36.2, -60.1, 1.3], [-33.9, -57.4, 2.1], (300, 3))
        xyz[:15, 0] = -34.0  # on the upper x wall: the container drops some or all of them
        xyz[15:30, 2] = 1.4  # on the lower z wall: kept
    n = len(xyz)
    vals = [rng.random(n) for _ in range(4)]
    m = kiwi.cartesian_map(xyz, bounds, res, *vals, ctx=ctx)
    near = oracle.cartesian_map_nearest(xyz, bounds, res)
    assert np.array_equal(m.voronoi_cell_id, near)
    assert np.array_equal(m.density, vals[0][near])


def test_ties_go_to_the_smallest_index(kiwi, ctx, oracle):
    """Sites on a lattice whose cell centres sit exactly between two or more of them."""
    g = (np.arange(4) + 0.0) / 4
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    xyz = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
    perm = np.random.default_rng(5).permutation(len(xyz))
    xyz = xyz[perm]
    bounds, res = (0.0, 1.0, 0.0, 1.0, 0.0, 1.0), 8
    vals = [np.arange(len(xyz), dtype=float)] * 4
    m = kiwi.cartesian_map(xyz, bounds, res, *vals, ctx=ctx)
    assert np.array_equal(m.voronoi_cell_id, oracle.cartesian_map_nearest(xyz, bounds, res))


def test_at_scale_vs_kdtree(kiwi, ctx):
    from scipy.spatial import cKDTree

    rng = np.random.default_rng(7)
    n = 200_000
    xyz = np.concatenate([rng.normal(5.0, 0.8, (n // 2, 3)), rng.uniform(0, 10, (n // 2, 3))])
    bounds, res = (0.0, 10.0, 0.0, 10.0, 0.0, 10.0), 96
    inside = np.all((xyz >= 0) & (xyz <= 10), axis=1)
    vals = [np.zeros(n)] * 4
    m = kiwi.cartesian_map(xyz, bounds, res, *vals, ctx=ctx)
    q = _grid_centres(bounds, res)
    d_kd, _ = cKDTree(xyz[inside]).query(q, k=1)
    s = m.voronoi_cell_id
    assert inside[s].all()
    diff = xyz[s] - q
    d_gpu = (diff[:, 0] * diff[:, 0] + diff[:, 1] * diff[:, 1]) + diff[:, 2] * diff[:, 2]
    assert np.all(d_gpu <= d_kd * d_kd * (1 + 1e-12) + 1e-300)
    print(f"{res ** 3} cells, {n} sites: gather {m.stats['gather_ms']:.2f} ms")


def test_edge_cases(kiwi, ctx):
    bounds = (0.0, 1.0, 0.0, 1.0, 0.0, 1.0)
    # no sites: every cell unresolved, id 0
    m = kiwi.cartesian_map(np.zeros((0, 3)), bounds, 4, *[np.zeros(0)] * 4, ctx=ctx)
    assert m.stats["unresolved"] == 64 and not m.voronoi_cell_id.any() and not m.density.any()
    # sites outside the domain only: the same
    m = kiwi.cartesian_map(np.array([[2.0, 0.5, 0.5], [-0.1, 0.5, 0.5]]), bounds, 3, *[np.ones(2)] * 4, ctx=ctx)
    assert m.stats["unresolved"] == 27
    # the reference's container drops a site on the domain's upper corner and keeps one on the lower corner
    m = kiwi.cartesian_map(np.array([[1.0, 1.0, 1.0]]), bounds, 1, *[np.array([7.0])] * 4, site_id=[42], ctx=ctx)
    assert m.stats["unresolved"] == 1 and m.voronoi_cell_id[0] == 0
    m = kiwi.cartesian_map(np.array([[0.0, 0.0, 0.0]]), bounds, 1, *[np.array([7.0])] * 4, site_id=[42], ctx=ctx)
    assert m.voronoi_cell_id[0] == 42 and m.density[0] == 7.0
    # unmapped sites: their cells keep 0 and carry the id
    xyz = np.array([[0.25, 0.5, 0.5], [0.75, 0.5, 0.5]])
    m = kiwi.cartesian_map(xyz, bounds, 2, *[np.array([1.0, 2.0])] * 4, site_id=[10, 11], mapped=[1, 0], ctx=ctx)
    assert set(m.voronoi_cell_id.tolist()) == {10, 11} and m.stats["unmapped"] == 4
    assert np.all(m.density[m.voronoi_cell_id == 11] == 0.0) and np.all(m.density[m.voronoi_cell_id == 10] == 1.0)
    with pytest.raises(kiwi.KiwiError):
        kiwi.cartesian_map(xyz, bounds, 0, *[np.ones(2)] * 4, ctx=ctx)
