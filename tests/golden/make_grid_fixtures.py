#!/usr/bin/env python3
"""Generates the sph-to-grid golden fixtures ``grid_*.npz`` by running the reference library itself
(oracle/_ref/libkiwi_ref.so, built from the reference sources by oracle/Makefile) on small seeded cases.

Each fixture holds the particle arrays, the grid (bounds, shape), the kernel selection, the reference's
output fields (density, vx, vy, vz) as run_sph_to_grid_stage computed them with one thread, and
``truth_raw``: the raw per-cell sums (sum m*Msum, sum m*Msum*v) of the same algorithm evaluated in
__float128 with exact constants (oracle/liboracle_q.so) -- the yardstick against which the reference's
and the GPU's FP64 errors are both measured.
Run from the repository root:  python tests/golden/make_grid_fixtures.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle.oracle import KERNEL_NAMES, Oracle, RefLib  # noqa: E402

RADKERN = [2.0, 2.5, 3.0, 2.0, 2.0, 2.0]


def particles(n, seed, lo, hi, hmin, hmax):
    rng = np.random.default_rng(seed)
    P = {k: rng.uniform(lo[i], hi[i], n) for i, k in enumerate(("x", "y", "z"))}
    for k in ("vx", "vy", "vz"):
        P[k] = rng.standard_normal(n)
    P["m"] = rng.uniform(0.02, 0.08, n)
    P["h"] = rng.uniform(hmin, hmax, n)
    return P


def _truth_part(args):
    P, bounds, shape, kern, sup, lo, hi = args
    q = Oracle(quad=True)
    return q.sph_to_grid(P, bounds, shape, kernel=kern, support_in_h=sup, p_range=(lo, hi))[4]


def truth_raw(P, bounds, shape, kern, sup, workers=8):
    """Raw sums in __float128 (rounded once to double per particle range), split over processes."""
    import multiprocessing as mp
    n = len(P["x"])
    cuts = np.linspace(0, n, workers + 1).astype(int)
    jobs = [(P, bounds, shape, kern, sup, int(cuts[i]), int(cuts[i + 1])) for i in range(workers)]
    with mp.get_context("spawn").Pool(workers) as pool:
        parts = pool.map(_truth_part, jobs)
    return np.sum(parts, axis=0)


def main():
    ref = RefLib()
    out_dir = os.path.dirname(os.path.abspath(__file__))
    cases = []
    # cubic spline on a cube
    cases.append(("cubic_cube", particles(240, 11, (0, 0, 0), (2, 2, 2), 0.05, 0.3), (0, 2, 0, 2, 0, 2), (16, 16, 16),
                  0, False))
    # ragged grid (no axis a multiple of the tile size), far-from-origin coordinates as the example
    # cutout has, particles partly outside the domain, some with h <= 0
    P = particles(200, 12, (-36.3, -60.2, 1.2), (-33.7, -57.8, 4.8), 0.04, 0.35)
    P["h"][::17] = 0.0
    P["h"][5] = -1.0
    cases.append(("cubic_ragged", P, (-36.0, -34.0, -60.0, -58.0, 1.4, 4.6), (13, 7, 19), 0, False))
    # cubic through the generic integral
    cases.append(("generic_m4", particles(150, 13, (0, 0, 0), (2, 2, 2), 0.08, 0.3), (0, 2, 0, 2, 0, 2), (12, 12, 12),
                  0, True))
    for k in range(1, 6):
        Pk = particles(120, 20 + k, (0, 0, 0), (2, 2, 2), 0.06, 0.25)
        cases.append((KERNEL_NAMES[k], Pk, (0, 2, 0, 2, 0, 2), (12, 12, 12), k, True))
    # padded domain: every support inside the grid, so the grid holds all the mass
    Pp = particles(80, 30, (0.6, 0.6, 0.6), (1.4, 1.4, 1.4), 0.05, 0.2)
    cases.append(("cubic_padded", Pp, (0, 2, 0, 2, 0, 2), (10, 10, 10), 0, False))
    for name, P, bounds, shape, k, generic in cases:
        d, vx, vy, vz = ref.sph_to_grid(P, bounds, shape, kernel=KERNEL_NAMES[k], generic_path=generic and k == 0,
                                        threads=1)
        tr = truth_raw(P, bounds, shape, k if (generic or k > 0) else -1, RADKERN[k])
        np.savez_compressed(os.path.join(out_dir, f"grid_{name}.npz"), **P, bounds=np.array(bounds, float),
                            shape=np.array(shape), kernel_index=k, support_in_h=RADKERN[k], generic=generic,
                            out_density=d, out_vx=vx, out_vy=vy, out_vz=vz, truth_raw=tr)
        print(name, d.sum() * np.prod([(bounds[2 * i + 1] - bounds[2 * i]) / shape[i] for i in range(3)]))


if __name__ == "__main__":
    main()
