#!/usr/bin/env python3
"""Writes ``cutout_particles.npz``: the particles of the reference's real-data cutout
(``tests/data/brick_03927_cutout.ascii`` of a KIWI checkout: a SPLASH ascii export of a Phantom snapshot,
gas particles with -36 <= x <= -34 pc and -60 <= y <= -58 pc) as the reference's own snapshot reader
(load_sph_snapshot, src/snapshot.cpp:511, through oracle/_ref) returns them, together with the grid of the
checkout's ``configs/example-cutout.json`` (100 x 100 x 410 cells of 0.02 pc over the cutout's column).

The GPU parity test (tests/test_gpu_parity_full.py) maps these particles with the GPU and with the
reference's run_sph_to_grid_stage (oracle/_ref) on the same machine and compares the two grids cell by
cell; the reference checkout itself is not needed there.

Usage: python tests/golden/make_cutout_fixture.py <KIWI checkout>   (or set KIWI_REF)
Needs oracle/_ref built (make -C oracle REF=<KIWI checkout>).
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle.oracle import load_ref  # noqa: E402


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("KIWI_REF")
    if not ref_root:
        sys.exit("usage: make_cutout_fixture.py <KIWI checkout>  (or set KIWI_REF)")
    ref = load_ref()
    if ref is None:
        sys.exit("oracle/_ref/libkiwi_ref.so is not built: make -C oracle REF=<KIWI checkout>")
    with open(os.path.join(ref_root, "configs", "example-cutout.json")) as f:
        cfg = json.load(f)
    P = ref.load_snapshot(os.path.join(ref_root, cfg["input_snapshot"]))
    d, g = cfg["domain"], cfg["cartesian_grid"]
    bounds = np.array([d["x_min"], d["x_max"], d["y_min"], d["y_max"], d["z_min"], d["z_max"]])
    shape = np.array([g["resolution_x"], g["resolution_y"], g["resolution_z"]], dtype=np.int64)
    out = os.path.join(HERE, "cutout_particles.npz")
    np.savez_compressed(out, bounds=bounds, shape=shape, **P)
    print(f"{out}: {len(P['x'])} particles, grid {tuple(shape)}, bounds {tuple(bounds)}")


if __name__ == "__main__":
    main()
