"""Comparison helpers shared by the GPU parity tests."""
import numpy as np

# Per-cell tolerance of the all-FP64 form against the reference / oracle: relative, on every cell whose
# density is above FLOOR x the peak; cells below the floor are held to the same bound in absolute terms
# relative to the peak.
FP64_REL = 1e-12
FLOOR = 1e-6


def cell_errors(gpu, ref, floor=FLOOR):
    gpu, ref = np.asarray(gpu), np.asarray(ref)
    peak = float(np.max(np.abs(ref))) if ref.size else 0.0
    if peak == 0.0:
        return 0.0, float(np.max(np.abs(gpu))) if gpu.size else 0.0
    mask = np.abs(ref) > floor * peak
    rel = float(np.max(np.abs(gpu[mask] - ref[mask]) / np.abs(ref[mask]))) if mask.any() else 0.0
    low = float(np.max(np.abs(gpu[~mask] - ref[~mask])) / peak) if (~mask).any() else 0.0
    return rel, low


def velocity_errors(gpu_v, ref_v, ref_density, floor=FLOOR):
    ref_density = np.asarray(ref_density)
    peak = float(np.max(ref_density)) if ref_density.size else 0.0
    mask = ref_density > floor * peak
    if not mask.any():
        return 0.0
    g, r = np.asarray(gpu_v)[mask], np.asarray(ref_v)[mask]
    return float(np.max(np.abs(g - r) / np.maximum(np.abs(r), 1.0)))


def assert_grid_match(res, dens, vx, vy, vz, tol=FP64_REL, label=""):
    rel, low = cell_errors(res.density, dens)
    assert rel <= tol and low <= tol, f"{label}: density rel {rel:.3e} low {low:.3e}"
    for name, g, r in (("vx", res.vx, vx), ("vy", res.vy, vy), ("vz", res.vz, vz)):
        e = velocity_errors(g, r, dens)
        assert e <= 1e3 * tol, f"{label}: {name} err {e:.3e}"
