#!/usr/bin/env python3
"""Generates the Lloyd-step golden fixtures ``lloyd_*.npz`` with the reference library itself
(oracle/_ref/libkiwi_ref.so, built from the reference sources by oracle/Makefile): lloyd_step
(src/point_set.cpp:265-293) on seeded point sets -- the moved points in the container's walk order.
Run from the repository root:  python tests/golden/make_lloyd_fixtures.py
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
    P = particles(400, 61, 1.0, 0.3, 1.0)
    blob = np.stack([P["x"], P["y"], P["z"]], axis=1)
    blob[:6, 0] = 2.0  # on the upper x wall: the container drops them
    blob[6:10, 2] = 0.0  # on the lower z wall: kept
    # the column recipe with its coverage-grid buffer points (the reference's own buffer), as the point-set
    # stage hands them to the Lloyd step
    C, b = column_snapshot(n=1500, seed=1003, box=(2.0, 2.0, 4.0))
    pb = (b[0] - 0.5, b[1] + 0.5, b[2] - 0.5, b[3] + 0.5, b[4] - 0.5, b[5] + 0.5)
    bxyz, _ = ref.coverage_grid_buffer(C, pb, 0.05, 2.0)
    col = np.concatenate([np.stack([C["x"], C["y"], C["z"]], axis=1), bxyz])
    rng = np.random.default_rng(62)
    cases = [
        ("lloyd_blob", blob, (0.0, 2.0, 0.0, 2.0, 0.0, 2.0)),
        ("lloyd_column_buffer", col, pb),
        ("lloyd_uniform_noncube", rng.uniform([0, 0, 0], [3.0, 1.0, 2.0], (500, 3)), (0.0, 3.0, 0.0, 1.0, 0.0, 2.0)),
    ]
    for name, xyz, bounds in cases:
        ids = np.arange(1, len(xyz) + 1, dtype=np.int32)
        oid, oxyz = ref.lloyd_step(xyz, ids, bounds)
        np.savez_compressed(os.path.join(out_dir, f"{name}.npz"), xyz=xyz, ids=ids, bounds=np.array(bounds, float),
                            ref_id=oid, ref_xyz=oxyz)
        print(name, "sites", len(xyz), "moved", len(oid))


if __name__ == "__main__":
    main()
