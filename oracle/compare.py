"""Cell-by-cell comparison of two density grids, per density band -- TEST INFRASTRUCTURE ONLY (used by the
GPU parity tests and by bench.py's CPU-baseline leg, which compares the GPU with the reference).

Bands are fractions of the reference grid's peak density: > 1e-2, 1e-4..1e-2, 1e-6..1e-4, and the cells at
or below 1e-6 of the peak, whose differences are taken relative to the peak."""
import numpy as np

BANDS = ((1e-2, np.inf), (1e-4, 1e-2), (1e-6, 1e-4))


def band_stats(x, ref, bands=BANDS):
    """Per band: cells, fraction within 1e-12 relative, median and largest relative difference."""
    x, ref = np.asarray(x), np.asarray(ref)
    peak = float(np.abs(ref).max())
    out = []
    for lo, hi in bands:
        m = (np.abs(ref) > lo * peak) & (np.abs(ref) <= hi * peak)
        rel = np.abs(x[m] - ref[m]) / np.abs(ref[m])
        out.append({"band": f">{lo:g} of peak" if hi == np.inf else f"{lo:g}..{hi:g} of peak", "cells": int(m.sum()),
                    "frac_le_1e-12": float(np.mean(rel <= 1e-12)) if m.any() else None,
                    "median": float(np.median(rel)) if m.any() else None,
                    "max": float(rel.max()) if m.any() else None})
    low = np.abs(ref) <= bands[-1][0] * peak
    rel = np.abs(x[low] - ref[low]) / peak
    out.append({"band": f"<={bands[-1][0]:g} of peak (abs/peak)", "cells": int(low.sum()),
                "frac_le_1e-12": float(np.mean(rel <= 1e-12)) if low.any() else None,
                "median": float(np.median(rel)) if low.any() else None, "max": float(rel.max()) if low.any() else None})
    return out


def covering_particles(P, bounds, shape, cell, support_in_h=2.0):
    """Indices of the particles whose clamped support bounding box contains the cell (the pairs the
    reference evaluates for it, src/cartesian_grid.cpp:211-243)."""
    idx = (cell // (shape[1] * shape[2]), (cell // shape[2]) % shape[1], cell % shape[2])
    keep = np.ones(len(P["x"]), dtype=bool)
    for a, k in enumerate("xyz"):
        d = (bounds[2 * a + 1] - bounds[2 * a]) / shape[a]
        r = support_in_h * P["h"]
        lo = np.clip(np.floor((P[k] - r - bounds[2 * a]) / d), 0, shape[a] - 1)
        hi = np.clip(np.floor((P[k] + r - bounds[2 * a]) / d), 0, shape[a] - 1)
        keep &= (lo <= idx[a]) & (hi >= idx[a])
    return np.nonzero(keep)[0]


def exact_cells(P, bounds, shape, cells, truth):
    """The exact (__float128) density and velocity of each given cell: the cell alone as a 1 x 1 x 1 grid over
    the particles that cover it, evaluated by `truth` (oracle.Oracle(quad=True))."""
    out = []
    for c in cells:
        idx = (c // (shape[1] * shape[2]), (c // shape[2]) % shape[1], c % shape[2])
        cb = []
        for a in range(3):
            d = (bounds[2 * a + 1] - bounds[2 * a]) / shape[a]
            cb += [bounds[2 * a] + idx[a] * d, bounds[2 * a] + (idx[a] + 1) * d]
        sel = covering_particles(P, bounds, shape, c)
        Ps = {k: np.ascontiguousarray(v[sel]) for k, v in P.items()}
        r = truth.sph_to_grid(Ps, cb, (1, 1, 1))
        out.append({"cell": int(c), "particles": int(len(sel)), "density": float(r[0][0]),
                    "v": [float(r[1][0]), float(r[2][0]), float(r[3][0])]})
    return out


def exact_check(P, bounds, shape, gpu, ref, truth, n_worst=8, n_random=40, seed=5):
    """The GPU's and the reference's distance from the exact integral, per cell, on the n_worst cells where the
    two disagree most (relative, cells above 1e-2 of the peak) and on n_random random cells of each band above
    1e-2, 1e-4 and 1e-6 of the peak (those present).  gpu and ref are (density, vx, vy, vz) grids.  Per group:
    median and largest relative density error, and the largest absolute velocity error, of each."""
    gd, rd = np.asarray(gpu[0]), np.asarray(ref[0])
    peak = rd.max()
    top = np.nonzero(rd > 1e-2 * peak)[0]
    rel = np.abs(gd[top] - rd[top]) / rd[top]
    rng = np.random.default_rng(seed)
    groups = {"worst_disagreement": top[np.argsort(rel)[-n_worst:]]}
    for name, lo, hi in (("band_gt_1e-2", 1e-2, np.inf), ("band_1e-4_1e-2", 1e-4, 1e-2), ("band_1e-6_1e-4", 1e-6, 1e-4)):
        m = np.nonzero((rd > lo * peak) & (rd <= hi * peak))[0]
        if len(m):
            groups[name] = rng.choice(m, min(n_random, len(m)), replace=False)
    res = {}
    for name, cells in groups.items():
        ex = exact_cells(P, bounds, shape, cells, truth)
        eg = np.array([abs(gd[e["cell"]] - e["density"]) / e["density"] for e in ex])
        er = np.array([abs(rd[e["cell"]] - e["density"]) / e["density"] for e in ex])
        vg = max(abs(float(np.asarray(gpu[1 + k])[e["cell"]]) - e["v"][k]) for e in ex for k in range(3))
        vr = max(abs(float(np.asarray(ref[1 + k])[e["cell"]]) - e["v"][k]) for e in ex for k in range(3))
        res[name] = {"cells": len(ex), "gpu_err_median": float(np.median(eg)), "gpu_err_max": float(eg.max()),
                     "ref_err_median": float(np.median(er)), "ref_err_max": float(er.max()),
                     "gpu_velocity_err_max": vg, "ref_velocity_err_max": vr}
    return res
