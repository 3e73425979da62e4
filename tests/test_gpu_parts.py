"""One grid split over several parts (kiwi_sph_to_grid_device_part), run here one part after another on
one GPU: each part writes exactly the cells of the tiles the host-side rule (kiwi_b200.shard) gives it,
and together the parts reproduce the whole call bit for bit."""
import numpy as np
import pytest

from conftest import random_particles

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

KEYS = ("x", "y", "z", "vx", "vy", "vz", "m", "h")


@pytest.mark.parametrize("precision,kname", [("fp64", "cubic_spline"), ("fp64", "wendland_c4"),
                                             ("fp64_reference_order", "cubic_spline"), ("fp32_mixed", "cubic_spline")])
@pytest.mark.parametrize("n_parts", [2, 3, 7])
def test_parts_reproduce_the_whole_grid(kiwi, ctx, precision, kname, n_parts):
    from kiwi_b200 import shard

    P = random_particles(500, 31, hmin=0.02, hmax=0.35)
    b, shape = (0.0, 2.0, 0.0, 2.0, 0.0, 2.0), (40, 24, 33)
    ki = kiwi.make_kernel_integrator(kname)
    dP = {k: torch.tensor(P[k], device="cuda") for k in KEYS}
    nc = int(np.prod(shape))

    def fresh(v):
        return {k: torch.full((nc,), v, dtype=torch.float64, device="cuda") for k in ("density", "vx", "vy", "vz")}

    whole = fresh(0.0)
    st = kiwi.sph_to_grid_device(dP, b, shape, whole, kernel=ki, precision=precision, ctx=ctx)
    own = shard.tile_owners(shard.tile_entry_counts(P, b, shape, ki.support_in_h or kiwi.get_kernel(kname).radkern),
                            n_parts)
    merged = fresh(float("nan"))
    pairs = 0
    for p in range(n_parts):
        part = fresh(float("nan"))
        sp = kiwi.sph_to_grid_device(dP, b, shape, part, kernel=ki, precision=precision, ctx=ctx, part=p,
                                     n_parts=n_parts)
        pairs += sp["sphere_pairs"]
        written = ~torch.isnan(part["density"]).cpu().numpy()
        assert np.array_equal(written, shard.cells_of_part(own, p, shape)), p
        for k in part:
            m = ~torch.isnan(part[k])
            merged[k][m] = part[k][m]
    for k in whole:
        assert torch.equal(merged[k], whole[k]), k
    assert pairs == st["sphere_pairs"]


def test_part_arguments_are_checked(kiwi, ctx):
    P = random_particles(10, 1)
    dP = {k: torch.tensor(P[k], device="cuda") for k in KEYS}
    out = {k: torch.zeros(512, dtype=torch.float64, device="cuda") for k in ("density", "vx", "vy", "vz")}
    for part, n in ((2, 2), (-1, 2), (0, 0)):
        with pytest.raises(kiwi.KiwiError):
            kiwi.sph_to_grid_device(dP, (0, 2, 0, 2, 0, 2), (8, 8, 8), out, ctx=ctx, part=part, n_parts=n)
    with pytest.raises(kiwi.KiwiError):
        kiwi.sph_to_grid_device(dP, (0, 2, 0, 2, 0, 2), (8, 8, 8), out, ctx=ctx, precision="fp32_mixed_guaranteed",
                                part=0, n_parts=2)


@pytest.mark.parametrize("precision,kname", [("fp64", "cubic_spline"), ("fp64", "wendland_c4"),
                                             ("fp64_reference_order", "cubic_spline"), ("fp32_mixed", "cubic_spline")])
def test_part_particles_reproduce_their_cells(kiwi, ctx, precision, kname):
    """A rank that holds only the particles reaching its tiles (shard.part_particles) and maps them with the
    whole-grid call gets its own cells bit for bit as the whole snapshot gives them (densities everywhere,
    velocities wherever a particle reaches the cell)."""
    from kiwi_b200 import shard

    P = random_particles(500, 32, hmin=0.02, hmax=0.35)
    b, shape, n_parts = (0.0, 2.0, 0.0, 2.0, 0.0, 2.0), (40, 24, 33), 3
    ki = kiwi.make_kernel_integrator(kname)
    sup = ki.support_in_h or kiwi.get_kernel(kname).radkern
    nc = int(np.prod(shape))

    def run(Q):
        dQ = {k: torch.tensor(np.ascontiguousarray(Q[k]), device="cuda") for k in KEYS}
        out = {k: torch.zeros(nc, dtype=torch.float64, device="cuda") for k in ("density", "vx", "vy", "vz")}
        kiwi.sph_to_grid_device(dQ, b, shape, out, kernel=ki, precision=precision, ctx=ctx)
        return {k: v.cpu().numpy() for k, v in out.items()}

    whole = run(P)
    own = shard.tile_owners(shard.tile_entry_counts(P, b, shape, sup), n_parts)
    for p in range(n_parts):
        idx = shard.part_particles(P, b, shape, sup, own, p)
        assert 0 < len(idx) < len(P["x"])
        part = run({k: v[idx] for k, v in P.items()})
        cells = shard.cells_of_part(own, p, shape)
        assert np.array_equal(part["density"][cells], whole["density"][cells]), p
        reached = cells & (whole["density"] > 0)
        for k in ("vx", "vy", "vz"):
            assert np.array_equal(part[k][reached], whole[k][reached]), (p, k)
