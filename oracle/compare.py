"""Cell-by-cell comparison of two density grids, per density band -- TEST INFRASTRUCTURE ONLY (used by the
GPU parity tests and by bench.py's CPU-baseline leg, which runs the reference as the checker).

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
