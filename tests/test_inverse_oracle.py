"""The oracle's restatement of the inverse-mapping check (run_inverse_mapping_test_stage's particle loop,
src/mapping.cpp:540-701) pinned to the reference's own stage: per-particle recovered masses and coverage
fractions bit for bit on the stage's own geometry (tests/golden/inv_*.npz, made by
tests/golden/make_inverse_fixtures.py with the reference library), and the totals in order."""
import glob
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "inv_*.npz")))


def load_inverse_fixture(fn):
    d = np.load(fn)
    P = {k: d[k] for k in ("x", "y", "z", "vx", "vy", "vz", "m", "h")}
    geo = {k[4:]: d[k] for k in d.files if k.startswith("geo_")}
    return d, P, geo


@pytest.mark.parametrize("fn", GOLDEN, ids=[os.path.basename(f)[4:-4] for f in GOLDEN])
def test_oracle_matches_reference_stage(oracle, fn):
    d, P, geo = load_inverse_fixture(fn)
    rec, cov = oracle.inverse_map(P, d["home"], geo, cell_mass=d["ref_cell_mass"])
    assert np.array_equal(rec, d["ref_m_recovered"])
    assert np.array_equal(cov, d["ref_coverage"])
    # the stage's totals, summed in particle / cell order (np.cumsum adds in order; Python's sum() of
    # floats is compensated)
    t = d["ref_totals"]
    assert np.cumsum(P["m"])[-1] == t[0]
    assert np.cumsum(d["ref_cell_mass"])[-1] == t[1]
    assert np.cumsum(rec)[-1] == t[2]


def test_reference_invariants_hold_on_fixtures():
    """tests/inverse_mapping_test.py:68-93: in a domain wider than the cloud every particle recovers its mass;
    in one that cuts it, particles outside recover nothing and none recovers more than its mass."""
    d, P, _ = load_inverse_fixture(os.path.join(ROOT, "tests", "golden", "inv_wide.npz"))
    assert np.all(np.abs(d["ref_coverage"] - 1.0) < 1e-8)
    d, P, _ = load_inverse_fixture(os.path.join(ROOT, "tests", "golden", "inv_tight.npz"))
    cov = d["ref_coverage"]
    assert np.all(cov[d["home"] < 0] == 0.0) and (d["home"] < 0).any()
    assert ((cov > 0) & (cov < 0.99)).any() and cov.max() < 1.0 + 1e-8
