"""The oracle's brute-force restatement of the coverage-grid buffer (add_coverage_grid_buffer,
src/point_set.cpp:198-262) pinned to the reference's own function (tests/golden/pset_*.npz, made by
tests/golden/make_pointset_fixtures.py with the reference library): the appended points and ids, bit for
bit."""
import glob
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "pset_*.npz")))


@pytest.mark.parametrize("fn", GOLDEN, ids=[os.path.basename(f)[5:-4] for f in GOLDEN])
def test_oracle_matches_reference(oracle, fn):
    d = np.load(fn)
    P = {k: d[k] for k in ("x", "y", "z", "h")}
    xyz, ids = oracle.coverage_grid_buffer(P, d["bounds"], float(d["spacing_fraction"]), float(d["factor"]))
    assert len(ids) > 0
    assert np.array_equal(xyz, d["ref_xyz"]) and np.array_equal(ids, d["ref_id"])


def test_all_h_nonpositive(oracle, reflib):
    P = {"x": np.array([0.5]), "y": np.array([0.5]), "z": np.array([0.5]), "h": np.array([0.0])}
    assert oracle.coverage_grid_buffer(P, (0, 1, 0, 1, 0, 1)) is None
    with pytest.raises(RuntimeError, match="all smoothing lengths are <= 0"):
        reflib.coverage_grid_buffer(P, (0, 1, 0, 1, 0, 1))
