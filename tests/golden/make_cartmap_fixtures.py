#!/usr/bin/env python3
"""Generates the cartesian-map golden fixtures ``cmap_*.npz`` with the reference library itself
(oracle/_ref/libkiwi_ref.so, built from the reference sources by oracle/Makefile): run_cartesian_map_stage
on seeded snapshots, with the point set and the mapping rows it located against (each recomputed in a fresh
work folder, as the stage computes them in memory).  Run from the repository root:
    python tests/golden/make_cartmap_fixtures.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from make_voronoi_fixtures import particles  # noqa: E402
from oracle.oracle import RefLib  # noqa: E402


def main():
    ref = RefLib()
    out_dir = os.path.dirname(os.path.abspath(__file__))
    cases = [
        # a cube domain: the blob and its outskirts
        ("cmap_blob", particles(300, 41, 1.0, 0.35, 1.0), (0.0, 2.0, 0.0, 2.0, 0.0, 2.0), 24),
        # a non-cube domain that cuts the cloud (particles outside it are not sites); odd resolution
        ("cmap_cut", particles(250, 42, 1.0, 0.3, 1.0), (0.5, 1.7, 0.4, 1.5, 0.6, 1.4), 19),
    ]
    for name, P, bounds, res in cases:
        pts, rows, mp = ref.cartesian_map(P, bounds, res)
        np.savez_compressed(os.path.join(out_dir, f"{name}.npz"), **P, bounds=np.array(bounds, float),
                            resolution=res, pt_id=pts["id"], pt_xyz=pts["xyz"],
                            **{"row_" + k: v for k, v in rows.items()}, **{"out_" + k: v for k, v in mp.items()})
        print(name, "sites", len(pts["id"]), "rows", len(rows["id"]), "cells", res ** 3,
              "distinct owners", len(np.unique(mp["cell_id"])))


if __name__ == "__main__":
    main()
