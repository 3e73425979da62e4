"""Batches (kiwi_batch_create / run / tune): many snapshots on their own grids with their own kernels in
one persistent, graph-recorded launch.  The batch runs the same tile bodies with the same per-cell particle
order as a single-grid call: in the reference-order form (compiled without FMA contraction) each item's
output equals the single call's bit for bit; the lattice form is compiled with FMA contraction, which the
compiler forms per kernel, so the batch kernel's results agree with the single-grid kernel's to rounding
(within 1e-12 of the item's largest value; the FP32-mixed form within its own error level), every count is
equal, and the clamped-cell count (cells whose sum rounds below zero) agrees to within the cells whose sum
is within rounding of zero."""
import numpy as np
import pytest

from conftest import random_particles

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

KEYS = ("x", "y", "z", "vx", "vy", "vz", "m", "h")


def _items(kiwi):
    rng = np.random.default_rng(77)
    specs = [
        (600, (16, 16, 16), "cubic_spline", 0.02, 0.25),
        (50, (9, 20, 7), "quintic_spline", 0.05, 0.3),
        (0, (8, 8, 8), "cubic_spline", 0.05, 0.2),          # empty snapshot
        (300, (24, 12, 12), "wendland_c4", 0.03, 0.2),
        (40, (5, 5, 5), "cubic_spline", 0.05, 0.1),         # every particle outside the grid (below)
        (1500, (32, 32, 32), "cubic_spline", 0.01, 0.15),
    ]
    items = []
    for i, (n, shape, kname, hmin, hmax) in enumerate(specs):
        P = random_particles(n, seed=100 + i, hmin=hmin, hmax=hmax)
        if i == 4:
            P["x"] = P["x"] + 10.0
        b = (0.0, 2.0, -0.1, 2.0, 0.05, 1.9)
        dP = {k: torch.tensor(np.asarray(P[k], dtype=np.float64), device="cuda") for k in KEYS}
        nc = int(np.prod(shape))
        out = {k: torch.full((nc,), float(rng.normal()), dtype=torch.float64, device="cuda")
               for k in ("density", "vx", "vy", "vz")}
        out["raw4"] = torch.full((4 * nc,), -1.0, dtype=torch.float64, device="cuda")
        items.append({"particles": dP, "bounds": b, "shape": shape, "kernel": kiwi.make_kernel_integrator(kname),
                      "out": out})
    return items


# agreement of a batch item with the single-grid call, relative to the item's largest value: the FP64
# lattice form to rounding; the FP32-mixed form within its own error level (the densest cells are within
# 1e-3 of the exact integral in either kernel)
TOL = {"fp64": 1e-12, "fp32_mixed": 2e-3}
VTOL = {"fp64": 1e-9, "fp32_mixed": 2e-2}


def _same(a, b, precision):
    """Bitwise equal in the reference-order form; within TOL of the largest value in the lattice forms."""
    if precision == "fp64_reference_order":
        return torch.equal(a, b)
    scale = float(b.abs().max()) if b.numel() else 0.0
    d = float((a - b).abs().max()) if b.numel() else 0.0
    return d <= TOL[precision] * scale


def _same_outputs(out, ref, precision):
    """Every output of an item against the single-grid call's: the raw sums and densities as _same; the
    finalised velocities (ratios of two sums, as sensitive as the cell's mass is small) bitwise in the
    reference-order form, and in the lattice forms within VTOL of the largest velocity where the density is
    above 1e-3 of its peak."""
    bad = [k for k in ("density", "raw4") if not _same(out[k], ref[k], precision)]
    if precision == "fp64_reference_order":
        return bad + [k for k in ("vx", "vy", "vz") if not torch.equal(out[k], ref[k])]
    if ref["density"].numel():
        m = ref["density"] >= 1e-3 * ref["density"].max()
        for k in ("vx", "vy", "vz"):
            scale = float(ref[k].abs().max())
            if m.any() and float((out[k][m] - ref[k][m]).abs().max()) > VTOL[precision] * scale:
                bad.append(k)
    return bad


def _single(kiwi, ctx, it, precision):
    nc = int(np.prod(it["shape"]))
    out = {k: torch.empty(nc, dtype=torch.float64, device="cuda") for k in ("density", "vx", "vy", "vz")}
    out["raw4"] = torch.empty(4 * nc, dtype=torch.float64, device="cuda")
    st = kiwi.sph_to_grid_device(it["particles"], it["bounds"], it["shape"], out, kernel=it["kernel"],
                                 precision=precision, ctx=ctx)
    return out, st


@pytest.mark.parametrize("precision", ["fp64", "fp64_reference_order", "fp32_mixed"])
def test_batch_equals_single_calls(kiwi, ctx, precision):
    items = _items(kiwi)
    batch = kiwi.Batch(items, precision=precision, ctx=ctx)
    try:
        for rep in range(2):
            per, tot = batch.run()
            torch.cuda.synchronize()
            for i, it in enumerate(items):
                ref, st = _single(kiwi, ctx, it, precision)
                assert not _same_outputs(it["out"], ref, precision), (rep, i, _same_outputs(it["out"], ref, precision))
                for k in ("bbox_pairs", "sphere_pairs", "evaluated_pairs", "skipped_outside", "tile_pairs",
                          "vertex_pyramids"):
                    assert per[i][k] == st[k], (rep, i, k, per[i][k], st[k])
                # a clamped cell is one whose alternating sum rounds below zero: in the lattice form, cells
                # at the support's edge whose sum is within rounding of zero may round to either side
                tol = {"fp64_reference_order": 0, "fp64": max(8, st["neg_clamped"] // 50),
                       "fp32_mixed": max(64, st["neg_clamped"] // 5)}[precision]
                assert abs(per[i]["neg_clamped"] - st["neg_clamped"]) <= tol, (rep, i, per[i]["neg_clamped"],
                                                                            st["neg_clamped"])
            assert tot["sphere_pairs"] == sum(p["sphere_pairs"] for p in per)
            assert per[4]["skipped_outside"] == 40 and per[2]["sphere_pairs"] == 0
        # the launch-shape tuning keeps the results
        lpt, ctas = batch.tune()
        assert ctas in (1, 2)
        for it in items:
            for k in it["out"]:
                it["out"][k].fill_(123.0)
        batch.run()
        torch.cuda.synchronize()
        for i, it in enumerate(items):
            ref, _ = _single(kiwi, ctx, it, precision)
            assert _same(it["out"]["density"], ref["density"], precision), i
    finally:
        batch.close()


def test_batch_masses_may_change_between_runs(kiwi, ctx):
    items = _items(kiwi)[:2]
    batch = kiwi.Batch(items, ctx=ctx)
    try:
        batch.run()
        items[0]["particles"]["m"].mul_(2.0)
        batch.run()
        torch.cuda.synchronize()
        ref, _ = _single(kiwi, ctx, items[0], "fp64")
        assert _same(items[0]["out"]["density"], ref["density"], "fp64")
    finally:
        batch.close()


def test_batch_rejects_bad_arguments(kiwi, ctx):
    items = _items(kiwi)[:1]
    with pytest.raises(kiwi.KiwiError):
        kiwi.Batch(items, precision="fp32_mixed_guaranteed", ctx=ctx)
    bad = dict(items[0])
    bad["bounds"] = (1.0, 0.0, 0.0, 1.0, 0.0, 1.0)
    with pytest.raises(kiwi.KiwiError):
        kiwi.Batch([bad], ctx=ctx)
    with pytest.raises(kiwi.KiwiError):
        kiwi.Batch([], ctx=ctx)


@pytest.mark.parametrize("precision", ["fp64", "fp64_reference_order"])
def test_snapshots_dealt_to_gpus_equal_the_whole_batch(kiwi, ctx, precision):
    """A batch split over GPUs by whole snapshots, longest first (shard.assign_snapshots_lpt on
    shard.snapshot_work), run here part after part: each part's batch gives its items' outputs as the
    whole batch does."""
    from kiwi_b200 import shard

    items = _items(kiwi)
    full = kiwi.Batch(items, precision=precision, ctx=ctx)
    try:
        full.run()
        torch.cuda.synchronize()
        ref = [{k: v.clone() for k, v in it["out"].items()} for it in items]
    finally:
        full.close()
    work = [shard.snapshot_work({k: it["particles"][k].cpu().numpy() for k in ("x", "y", "z", "h")}, it["bounds"],
                                it["shape"], it["kernel"].support_in_h or 2.0) for it in items]
    parts = shard.assign_snapshots_lpt(work, 2)
    assert all(len(q) for q in parts)
    for q in parts:
        sub = [items[i] for i in q]
        for it in sub:
            for k in it["out"]:
                it["out"][k].fill_(123.0)
        b = kiwi.Batch(sub, precision=precision, ctx=ctx)
        try:
            b.run()
            torch.cuda.synchronize()
        finally:
            b.close()
        for i in q:
            assert not _same_outputs(items[i]["out"], ref[i], precision), (i, _same_outputs(items[i]["out"], ref[i],
                                                                                            precision))
