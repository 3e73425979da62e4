#!/usr/bin/env python3
"""Generates the coverage-buffer golden fixtures ``pset_*.npz`` with the reference library itself
(oracle/_ref/libkiwi_ref.so, built from the reference sources by oracle/Makefile): add_coverage_grid_buffer
(src/point_set.cpp:198-262) on seeded snapshots, the particles standing as the point set with ids 1..n.
Run from the repository root:  python tests/golden/make_pointset_fixtures.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from make_voronoi_fixtures import particles  # noqa: E402
from oracle.oracle import RefLib  # noqa: E402

from kiwi_b200.workloads import column_snapshot  # noqa: E402


def main():
    ref = RefLib()
    out_dir = os.path.dirname(os.path.abspath(__file__))
    P1, b1 = column_snapshot(n=3000, seed=1001, box=(2.0, 2.0, 8.2))
    cases = [
        # the column in a padded domain: buffer points fill the padding
        ("pset_column", P1, (b1[0] - 1.0, b1[1] + 1.0, b1[2] - 1.0, b1[3] + 1.0, b1[4] - 1.0, b1[5] + 1.0), 0.05, 2.0),
        ("pset_blob", particles(500, 51, 1.0, 0.25, 0.35), (0.0, 2.0, 0.0, 2.0, 0.0, 2.0), 0.04, 2.0),
        ("pset_noncube", particles(400, 52, 1.0, 0.3, 0.3), (-0.3, 2.4, 0.1, 1.9, 0.0, 2.0), 0.03, 2.5),
    ]
    for name, P, bounds, sf, factor in cases:
        xyz, ids = ref.coverage_grid_buffer(P, bounds, sf, factor)
        np.savez_compressed(os.path.join(out_dir, f"{name}.npz"), **{k: P[k] for k in ("x", "y", "z", "h")},
                            bounds=np.array(bounds, float), spacing_fraction=sf, factor=factor, ref_xyz=xyz,
                            ref_id=ids)
        print(name, "particles", len(P["x"]), "buffer points", len(ids))


if __name__ == "__main__":
    main()
