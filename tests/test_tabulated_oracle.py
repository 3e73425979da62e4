"""The oracle's restatement of the tabulated cubic integral (the density lookup table and
gridded_integral, src/kernel_integral.cpp:13-190) pinned to the reference library built from its own
sources: the canonical table, lookups in a loaded table, the loader's errors, and sph-to-grid with the
tabulated integral against the reference's own outputs (tests/golden/tab_grid_*.npz)."""
import glob
import os

import numpy as np
import pytest

from conftest import table_probe_points, write_table_file

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "tab_grid_*.npz")))


def test_canonical_table_bit_identical(oracle, reflib):
    oracle.table_reset()
    a, b = oracle.table_values(), reflib.table_values()
    assert a.shape == b.shape == (251 * 301 * 301,)
    assert np.array_equal(a, b)


def test_loaded_table_lookups_bit_identical(oracle, reflib, tmp_path):
    fn = str(tmp_path / "small.tab")
    vals = write_table_file(fn, seed=3)
    assert oracle.table_load(fn) == 0
    try:
        v = oracle.table_values().reshape(4 + 7 + 2, 5 + 3 + 1, 6 + 4 + 1)
        assert np.array_equal(v[1:-1, :-1, :-1].reshape(-1), vals)
        assert np.array_equal(v[-1], v[-2]) and not v[0].any() and not v[:, -1].any() and not v[:, :, -1].any()
        h, phi, r0, R0 = table_probe_points(3000, 4)
        ours = np.array([oracle.gridded_integral(*t) for t in zip(h, phi, r0, R0)])
        assert np.array_equal(ours, reflib.table_load_gridded(fn, h, phi, r0, R0))
    finally:
        oracle.table_reset()


def test_loader_errors(oracle, reflib, tmp_path):
    missing = str(tmp_path / "missing.tab")
    assert oracle.table_load(missing) == -1
    with pytest.raises(RuntimeError, match="could not open density lookup table"):
        reflib.table_load_gridded(missing, 1.0, 0.5, 0.5, 0.5)
    bad = str(tmp_path / "bad.tab")
    write_table_file(bad, header="4 5 six\n")
    assert oracle.table_load(bad) == -2
    with pytest.raises(RuntimeError, match="header is malformed"):
        reflib.table_load_gridded(bad, 1.0, 0.5, 0.5, 0.5)
    short = str(tmp_path / "short.tab")
    write_table_file(short, truncate=5)
    assert oracle.table_load(short) == -3
    with pytest.raises(RuntimeError, match="truncated"):
        reflib.table_load_gridded(short, 1.0, 0.5, 0.5, 0.5)
    oracle.table_reset()


@pytest.mark.parametrize("fn", GOLDEN, ids=[os.path.basename(f)[9:-4] for f in GOLDEN])
def test_oracle_tabulated_sph_to_grid_matches_fixture(oracle, fn):
    d = np.load(fn)
    P = {k: d[k] for k in ("x", "y", "z", "vx", "vy", "vz", "m", "h")}
    oracle.table_reset()
    dens, vx, vy, vz, _, _ = oracle.sph_to_grid(P, d["bounds"], tuple(d["shape"]), tabulated=True)
    assert np.array_equal(dens, d["out_density"])
    for name, v in (("vx", vx), ("vy", vy), ("vz", vz)):
        assert np.array_equal(v, d["out_" + name]), name
