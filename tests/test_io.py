"""Stage output files (no GPU): the VGTCGRD2 grid file and mapping.dat, byte for byte as the reference's own
writers produce them (src/cartesian_grid.cpp:323-394, src/mapping.cpp:307-315), plus round trips and the
reader's error cases."""
import struct

import numpy as np
import pytest


def _grid(kiwi, shape=(3, 4, 5), seed=0):
    rng = np.random.default_rng(seed)
    nc = int(np.prod(shape))
    return kiwi.CartesianGridResult(shape[0], shape[1], shape[2], (-1.0, 2.5, 0.0, 1.0, 3.0, 7.25),
                                    rng.random(nc) * 1e3, rng.normal(size=nc), rng.normal(size=nc), rng.normal(size=nc))


def test_grid_file_layout_and_round_trip(kiwi, tmp_path):
    g = _grid(kiwi)
    p = str(tmp_path / "grid.bin")
    kiwi.save_cartesian_grid(g, p)
    raw = open(p, "rb").read()
    # the layout the reference's readers expect (tests/phantom_dump_test.py reads the same header)
    expect = (b"VGTCGRD2" + struct.pack("<3i", 3, 4, 5) + struct.pack("<6d", *g.bounds) +
              g.density.astype("<f8").tobytes() + g.vx.astype("<f8").tobytes() + g.vy.astype("<f8").tobytes() +
              g.vz.astype("<f8").tobytes())
    assert raw == expect
    r = kiwi.load_cartesian_grid(p)
    assert (r.nx, r.ny, r.nz) == (3, 4, 5) and r.bounds == g.bounds
    for k in ("density", "vx", "vy", "vz"):
        assert np.array_equal(getattr(r, k), getattr(g, k))


def test_grid_file_equals_reference_writer(kiwi, reflib, tmp_path):
    g = _grid(kiwi, (7, 2, 9), seed=3)
    a, b = str(tmp_path / "ours.bin"), str(tmp_path / "ref.bin")
    kiwi.save_cartesian_grid(g, a)
    reflib.save_cartesian_grid(b, (g.nx, g.ny, g.nz), g.bounds, g.density, g.vx, g.vy, g.vz)
    assert open(a, "rb").read() == open(b, "rb").read()


def test_mapping_file_equals_reference_writer(kiwi, reflib, tmp_path):
    rng = np.random.default_rng(5)
    n = 200
    ids = rng.permutation(1000)[:n]
    sites = rng.normal(size=(n, 3)) * [1e-3, 1.0, 1e5]
    vol = rng.random(n) ** 3
    res = kiwi.MappingResult(rng.random(n) * 1e-20, rng.normal(size=n), np.zeros(n), rng.normal(size=n) * 1e10)
    res.density[:3] = [0.0, 1.0, 123456789.123456789]
    a, b = str(tmp_path / "ours.dat"), str(tmp_path / "ref.dat")
    kiwi.save_mapping(a, ids, sites, vol, res)
    reflib.save_mapping(b, ids, sites[:, 0], sites[:, 1], sites[:, 2], vol, res.density, res.vx, res.vy, res.vz)
    assert open(a).read() == open(b).read()


def test_grid_reader_errors(kiwi, tmp_path):
    p = tmp_path / "bad.bin"
    p.write_bytes(b"NOTAGRID" + b"\0" * 64)
    with pytest.raises(kiwi.KiwiError, match="unrecognized header"):
        kiwi.load_cartesian_grid(str(p))
    p.write_bytes(b"VGTCGRD2" + struct.pack("<3i", 0, 4, 4) + b"\0" * 48)
    with pytest.raises(kiwi.KiwiError, match="invalid resolution"):
        kiwi.load_cartesian_grid(str(p))
    p.write_bytes(b"VGTCGRD2" + struct.pack("<3i", 2, 2, 2) + struct.pack("<6d", 0, 1, 0, 1, 0, 1) + b"\0" * 40)
    with pytest.raises(kiwi.KiwiError, match="truncated"):
        kiwi.load_cartesian_grid(str(p))
    with pytest.raises(kiwi.KiwiError, match="could not open"):
        kiwi.load_cartesian_grid(str(tmp_path / "missing.bin"))


def _inverse(kiwi, n=57, seed=3):
    rng = np.random.default_rng(seed)
    m = rng.uniform(0.001, 0.05, n)
    rec = m * rng.uniform(0.0, 1.0 + 1e-9, n)
    rec[::7] = 0.0
    cov = np.where(m > 0, rec / m, 0.0)
    r = kiwi.InverseMappingResult(m, rec, cov, float(m.sum()), float(rec.sum()) * (1 + 1e-12), float(rec.sum()))
    return np.arange(1, n + 1, dtype=np.int64) * 3, r


def test_inverse_mapping_file_equals_reference_writer(kiwi, reflib, tmp_path):
    ids, r = _inverse(kiwi)
    a, b = str(tmp_path / "a.dat"), str(tmp_path / "b.dat")
    kiwi.save_inverse_mapping_test(a, ids, r)
    reflib.save_inverse_mapping_test(b, ids, r.m_original, r.m_recovered, r.coverage,
                                     [r.total_original_mass, r.total_grid_mass, r.total_recovered_mass])
    assert open(a, "rb").read() == open(b, "rb").read()


def test_inverse_mapping_file_round_trip_and_errors(kiwi, tmp_path):
    ids, r = _inverse(kiwi)
    p = str(tmp_path / "inv.dat")
    kiwi.save_inverse_mapping_test(p, ids, r)
    ids2, r2 = kiwi.load_inverse_mapping_test(p)
    assert np.array_equal(ids2, ids)
    for k in ("m_original", "m_recovered", "coverage"):
        assert np.allclose(getattr(r2, k), getattr(r, k), rtol=1e-14, atol=0)  # 15 significant digits
    with pytest.raises(kiwi.KiwiError, match="could not open inverse-mapping-test file"):
        kiwi.load_inverse_mapping_test(str(tmp_path / "missing.dat"))
    bad = tmp_path / "bad.dat"
    bad.write_text("1 2 3\n")
    with pytest.raises(kiwi.KiwiError, match="missing expected '#' totals header"):
        kiwi.load_inverse_mapping_test(str(bad))
    bad.write_text("# totals\nx y z\n")
    with pytest.raises(kiwi.KiwiError, match="could not read totals line"):
        kiwi.load_inverse_mapping_test(str(bad))
    bad.write_text("# totals\n1 2 3\n")
    with pytest.raises(kiwi.KiwiError, match="contained no particle rows"):
        kiwi.load_inverse_mapping_test(str(bad))


def _cmap(kiwi, res=5, seed=4):
    rng = np.random.default_rng(seed)
    nq = res ** 3
    return kiwi.CartesianMap(res, (-1.0, 2.0, 0.5, 3.5, 1.0, 4.0), rng.random(nq), rng.normal(size=nq),
                             rng.normal(size=nq), rng.normal(size=nq), rng.integers(0, 1000, nq).astype(np.int32))


def test_cartesian_map_file_equals_reference_writer(kiwi, reflib, tmp_path):
    m = _cmap(kiwi)
    a, b = str(tmp_path / "a.dat"), str(tmp_path / "b.dat")
    kiwi.save_cartesian_map(m, a)
    reflib.save_cartesian_map(b, m.resolution, m.bounds, m.density, m.vx, m.vy, m.vz, m.voronoi_cell_id)
    assert open(a, "rb").read() == open(b, "rb").read()


def test_cartesian_map_file_round_trip_and_errors(kiwi, tmp_path):
    m = _cmap(kiwi)
    p = str(tmp_path / "m.dat")
    kiwi.save_cartesian_map(m, p)
    r = kiwi.load_cartesian_map(p)
    assert r.resolution == m.resolution and r.bounds == m.bounds
    for k in ("density", "vx", "vy", "vz", "voronoi_cell_id"):
        assert np.array_equal(getattr(r, k), getattr(m, k)), k
    with pytest.raises(kiwi.KiwiError, match="could not open cartesian map file"):
        kiwi.load_cartesian_map(str(tmp_path / "missing.dat"))
    bad = tmp_path / "bad.dat"
    bad.write_bytes(b"VGTCGRD2" + struct.pack("<i", 5))
    with pytest.raises(kiwi.KiwiError, match="unrecognized header"):
        kiwi.load_cartesian_map(str(bad))
    bad.write_bytes(b"VGTCMAP1" + struct.pack("<i", 0))
    with pytest.raises(kiwi.KiwiError, match="invalid resolution"):
        kiwi.load_cartesian_map(str(bad))
    raw = open(p, "rb").read()
    bad.write_bytes(raw[:-9])
    with pytest.raises(kiwi.KiwiError, match="truncated"):
        kiwi.load_cartesian_map(str(bad))
