#!/usr/bin/env python3
"""Generates the tabulated-integral golden fixtures ``tab_grid_*.npz`` by running the reference library
itself (oracle/_ref/libkiwi_ref.so, built from the reference sources by oracle/Makefile) with
cartesian_grid.use_tabulated_integral set and no table file, so that the reference generates its canonical
table (generate_density_table, src/kernel_integral.cpp:57-119) and looks every vertex pyramid up in it.

Each fixture holds the particle arrays, the grid (bounds, shape) and the reference's output fields
(density, vx, vy, vz) computed with one thread.  Run from the repository root:
    python tests/golden/make_tabulated_fixtures.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle.oracle import RefLib  # noqa: E402


def particles(n, seed, lo, hi, hmin, hmax):
    rng = np.random.default_rng(seed)
    P = {k: rng.uniform(lo[i], hi[i], n) for i, k in enumerate(("x", "y", "z"))}
    for k in ("vx", "vy", "vz"):
        P[k] = rng.standard_normal(n)
    P["m"] = rng.uniform(0.02, 0.08, n)
    P["h"] = rng.uniform(hmin, hmax, n)
    return P


def main():
    ref = RefLib()
    out_dir = os.path.dirname(os.path.abspath(__file__))
    cases = [("cube", particles(240, 41, (0, 0, 0), (2, 2, 2), 0.05, 0.3), (0, 2, 0, 2, 0, 2), (16, 16, 16))]
    # ragged grid, particles partly outside the domain, some with h <= 0
    P = particles(200, 42, (-36.3, -60.2, 1.2), (-33.7, -57.8, 4.8), 0.04, 0.35)
    P["h"][::17] = 0.0
    P["h"][5] = -1.0
    cases.append(("ragged", P, (-36.0, -34.0, -60.0, -58.0, 1.4, 4.6), (13, 7, 19)))
    # padded domain: every support inside the grid
    cases.append(("padded", particles(80, 43, (0.6, 0.6, 0.6), (1.4, 1.4, 1.4), 0.05, 0.2), (0, 2, 0, 2, 0, 2),
                  (10, 10, 10)))
    for name, P, bounds, shape in cases:
        d, vx, vy, vz = ref.sph_to_grid(P, bounds, shape, tabulated=True, threads=1)
        np.savez_compressed(os.path.join(out_dir, f"tab_grid_{name}.npz"), **P, bounds=np.array(bounds, float),
                            shape=np.array(shape), out_density=d, out_vx=vx, out_vy=vy, out_vz=vz)
        print(name, d.sum() * np.prod([(bounds[2 * i + 1] - bounds[2 * i]) / shape[i] for i in range(3)]))


if __name__ == "__main__":
    main()
