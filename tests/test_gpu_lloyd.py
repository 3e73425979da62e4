"""GPU parity of the point-set stage's Lloyd step (lloyd_step, src/point_set.cpp:265-293; kiwi_lloyd_step)
against the reference's own function (tests/golden/lloyd_*.npz, made by tests/golden/make_lloyd_fixtures.py
with the reference library): the sites kept and their order exactly (the container's filter and walk
order), the moved positions to 1e-12 of the domain's size (centroids computed in a different order of
operations), plus the invariant that the cells tile the domain (their volumes sum to its volume)."""
import glob
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "lloyd_*.npz")))


def _volume(b):
    return (b[1] - b[0]) * (b[3] - b[2]) * (b[5] - b[4])


@pytest.mark.parametrize("fn", GOLDEN, ids=[os.path.basename(f)[6:-4] for f in GOLDEN])
def test_matches_reference(kiwi, ctx, fn):
    d = np.load(fn)
    b = d["bounds"]
    ids, xyz, vol, st = kiwi.lloyd_step(d["xyz"], b, ids=d["ids"], ctx=ctx)
    assert st["failed"] == 0
    assert np.array_equal(ids, d["ref_id"])
    ext = max(b[1] - b[0], b[3] - b[2], b[5] - b[4])
    err = np.abs(xyz - d["ref_xyz"]).max()
    print(f"{os.path.basename(fn)}: {len(ids)} sites, max |diff| {err:.3e}")
    assert err <= 1e-12 * ext
    assert abs(vol.sum() - _volume(b)) <= 1e-12 * _volume(b)
    assert st["dropped"] == len(d["ids"]) - len(d["ref_id"])


def test_at_scale_cells_tile_the_domain(kiwi, ctx):
    rng = np.random.default_rng(9)
    n = 200_000
    xyz = np.concatenate([rng.normal(5.0, 1.0, (n // 2, 3)), rng.uniform(0, 10, (n // 2, 3))])
    b = (0.0, 10.0, 0.0, 10.0, 0.0, 10.0)
    ids, out, vol, st = kiwi.lloyd_step(xyz, b, ctx=ctx)
    inside = np.all((xyz >= 0) & (xyz < 10), axis=1)
    assert st["failed"] == 0 and len(ids) == inside.sum()
    assert abs(vol.sum() - 1000.0) <= 1e-9 * 1000.0
    assert np.all((out >= 0) & (out <= 10))
    # a centroid lies nearer its own site than the cell radius: its cell is convex and contains both
    assert np.all(np.linalg.norm(out - xyz[ids], axis=1) <= np.cbrt(vol) * 3)
    a = kiwi.lloyd_step(xyz, b, ctx=ctx)
    assert np.array_equal(a[0], ids) and np.array_equal(a[1], out)
    print(f"{n} sites: {st['gather_ms']:.2f} ms on the device, {st['total_ms']:.2f} ms end to end")


def test_edge_cases(kiwi, ctx):
    b = (0.0, 1.0, 0.0, 1.0, 0.0, 1.0)
    ids, xyz, vol, st = kiwi.lloyd_step(np.zeros((0, 3)), b, ctx=ctx)
    assert len(ids) == 0
    # one site: its cell is the whole box, its centroid the box centre
    ids, xyz, vol, st = kiwi.lloyd_step(np.array([[0.1, 0.2, 0.3]]), b, ctx=ctx)
    assert np.allclose(xyz[0], [0.5, 0.5, 0.5], atol=1e-15) and abs(vol[0] - 1.0) < 1e-15
    # a lattice of sites (every neighbour plane through cell vertices): cells are the lattice cubes
    g = (np.arange(4) + 0.5) / 4
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    sites = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
    ids, xyz, vol, st = kiwi.lloyd_step(sites, b, ctx=ctx)
    assert st["failed"] == 0 and np.allclose(xyz, sites[ids], atol=1e-14) and np.allclose(vol, 1 / 64, rtol=1e-12)
    with pytest.raises(kiwi.KiwiError):
        kiwi.lloyd_step(sites, (1.0, 0.0, 0.0, 1.0, 0.0, 1.0), ctx=ctx)
