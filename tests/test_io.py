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
