#!/usr/bin/env python3
"""Generates the Voronoi-map golden fixtures ``vor_*.npz`` with the reference library itself
(oracle/_ref/libkiwi_ref.so, built from the reference sources by oracle/Makefile).

For each seeded case the reference's own code builds the point set (optionally with the coverage-grid
buffer and Lloyd steps), tessellates it with its vendored Voro++ exactly as src/mapping.cpp:222-269 does,
locates every particle's home cell, and runs run_mapping_stage; the fixture keeps the cell geometry in CSR
form (absolute vertex coordinates, neighbour indices), the home cells, the reference's per-cell density
and velocity (mapping.dat), and ``truth_raw``: the raw per-cell sums of the same algorithm in __float128
(oracle/liboracle_q.so).  Run from the repository root:  python tests/golden/make_voronoi_fixtures.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle.oracle import KERNEL_NAMES, Oracle, RefLib  # noqa: E402

RADKERN = [2.0, 2.5, 3.0, 2.0, 2.0, 2.0]


def particles(n, seed, centre, sigma, hscale):
    rng = np.random.default_rng(seed)
    pos = centre + sigma * rng.standard_normal((n, 3))
    P = {"x": pos[:, 0].copy(), "y": pos[:, 1].copy(), "z": pos[:, 2].copy()}
    for k in ("vx", "vy", "vz"):
        P[k] = rng.standard_normal(n)
    P["m"] = np.full(n, 0.01)
    r2 = ((pos - centre) ** 2).sum(1)
    rho = np.maximum(n * 0.01 / (2 * np.pi * sigma * sigma) ** 1.5 * np.exp(-0.5 * r2 / sigma ** 2), 1e-3)
    P["h"] = hscale * 1.2 * (0.01 / rho) ** (1.0 / 3.0)
    return P


def _truth_part(args):
    P, home, geo, kern, sup = args
    return Oracle(quad=True).map_voronoi(P, home, geo, kernel=kern, support_in_h=sup)[4]


def truth_raw(P, home, geo, kern, sup, workers=8):
    import multiprocessing as mp
    n = len(P["x"])
    cuts = np.linspace(0, n, workers + 1).astype(int)
    jobs = [({k: v[cuts[i]:cuts[i + 1]] for k, v in P.items()}, home[cuts[i]:cuts[i + 1]], geo, kern, sup)
            for i in range(workers)]
    with mp.get_context("spawn").Pool(workers) as pool:
        parts = pool.map(_truth_part, jobs)
    return np.sum(parts, axis=0)


def main():
    ref = RefLib()
    out_dir = os.path.dirname(os.path.abspath(__file__))
    cases = [
        # name, particles, bounds, buffer, lloyd, kernel
        ("vor_blob_cubic", particles(220, 21, 1.0, 0.3, 1.0), (0, 2, 0, 2, 0, 2), False, 0, 0),
        ("vor_buffer_lloyd_cubic", particles(160, 22, 1.0, 0.25, 1.0), (0, 2, 0, 2, 0, 2), True, 1, 0),
        ("vor_blob_wc4", particles(150, 23, 1.0, 0.3, 1.0), (0, 2, 0, 2, 0, 2), False, 0, 4),
    ]
    for name, P, bounds, buf, lloyd, k in cases:
        geo, res = ref.voronoi(P, bounds, buffer=buf, spacing_fraction=0.1 if buf else 0.0, lloyd=lloyd,
                               kernel=KERNEL_NAMES[k], threads=1)
        home = geo["home"]
        tr = truth_raw(P, home, geo, k if k > 0 else -1, RADKERN[k])
        np.savez_compressed(os.path.join(out_dir, f"{name}.npz"), **P, bounds=np.array(bounds, float),
                            kernel_index=k, support_in_h=RADKERN[k], home=home,
                            **{"geo_" + key: v for key, v in geo.items() if key != "home"},
                            out_density=res[0], out_vx=res[1], out_vy=res[2], out_vz=res[3], truth_raw=tr)
        print(name, "cells", len(geo["volume"]), "faces", len(geo["face_nbr"]), "mass on cells",
              float((res[0] * geo["volume"]).sum()), "particle mass", float(P["m"].sum()))


if __name__ == "__main__":
    main()
