"""GPU parity of the coverage-grid buffer (add_coverage_grid_buffer, src/point_set.cpp:198-262;
kiwi_coverage_grid_buffer) against the reference's own function (tests/golden/pset_*.npz, made by
tests/golden/make_pointset_fixtures.py with the reference library) and the oracle's brute force: the
appended points (lattice positions) and ids are exact results, so the bar is equality."""
import glob
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "pset_*.npz")))


@pytest.mark.parametrize("fn", GOLDEN, ids=[os.path.basename(f)[5:-4] for f in GOLDEN])
def test_matches_reference(kiwi, ctx, fn):
    d = np.load(fn)
    P = {k: d[k] for k in ("x", "y", "z", "h")}
    xyz, ids = kiwi.coverage_grid_buffer(P, d["bounds"], float(d["spacing_fraction"]), float(d["factor"]), ctx=ctx)
    assert np.array_equal(xyz, d["ref_xyz"]) and np.array_equal(ids, d["ref_id"])


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_random_vs_oracle(kiwi, ctx, oracle, seed):
    rng = np.random.default_rng(seed)
    n = 800
    P = {"x": rng.normal(1.0, 0.4, n), "y": rng.normal(1.0, 0.4, n), "z": rng.uniform(0, 2, n),
         "h": rng.lognormal(-2.5, 0.6, n)}
    P["h"][::37] = -P["h"][::37]  # a negative h covers like |h| (the squared radius)
    P["h"][::41] = 0.0
    bounds = (-0.2, 2.3, -0.1, 2.1, 0.0, 2.0)
    a = kiwi.coverage_grid_buffer(P, bounds, 0.03, 2.0, ctx=ctx)
    b = oracle.coverage_grid_buffer(P, bounds, 0.03, 2.0)
    assert len(a[1]) > 0 and np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_edge_cases(kiwi, ctx):
    P = {"x": np.array([0.5]), "y": np.array([0.5]), "z": np.array([0.5]), "h": np.array([0.0])}
    with pytest.raises(kiwi.KiwiError, match="all smoothing lengths are <= 0"):
        kiwi.coverage_grid_buffer(P, (0, 1, 0, 1, 0, 1), ctx=ctx)
    # one particle covering everything: no buffer points
    P["h"][0] = 10.0
    xyz, ids = kiwi.coverage_grid_buffer(P, (0, 1, 0, 1, 0, 1), ctx=ctx)
    assert len(ids) == 0
    # a particle far outside: every candidate is kept, ids 2..k+1 in lattice order
    P = {"x": np.array([50.0]), "y": np.array([0.5]), "z": np.array([0.5]), "h": np.array([0.1])}
    xyz, ids = kiwi.coverage_grid_buffer(P, (0, 1, 0, 1, 0, 1), spacing_fraction=0.25, ctx=ctx)
    assert len(ids) == 64 and np.array_equal(ids, np.arange(2, 66))
    assert np.array_equal(xyz[0], [0.125, 0.125, 0.125]) and np.array_equal(xyz[1], [0.125, 0.125, 0.375])
