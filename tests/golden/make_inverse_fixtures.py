#!/usr/bin/env python3
"""Generates the inverse-mapping golden fixtures ``inv_*.npz`` with the reference library itself
(oracle/_ref/libkiwi_ref.so, built from the reference sources by oracle/Makefile).

For each seeded case the reference's own code runs run_mapping_stage and then run_inverse_mapping_test_stage
in the same work folder, as `kiwi inverse-mapping-test` does.  The inverse stage tessellates the point set
the forward stage cached (15 significant digits), so the fixture keeps that geometry (CSR, rebuilt by the
same Voro++ calls from the cached points) and its home cells, the cell masses the stage used (density x
volume of the cached mapping rows), and the stage's per-particle recovered masses, coverage fractions and
three totals.
The cases follow the reference's own test (tests/inverse_mapping_test.py): a domain wider than the cloud
(every particle recovers its mass) and one that cuts the cloud.
Run from the repository root:  python tests/golden/make_inverse_fixtures.py
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
        ("inv_wide", particles(200, 31, 1.0, 0.3, 1.0), (-8.0, 10.0, -8.0, 10.0, -8.0, 10.0)),
        ("inv_cut", particles(200, 31, 1.0, 0.3, 1.0), (-2.0, 4.0, -2.0, 4.0, -2.0, 4.0)),
        ("inv_tight", particles(200, 32, 1.0, 0.3, 1.0), (0.6, 1.4, 0.55, 1.45, 0.6, 1.4)),
    ]
    for name, P, bounds in cases:
        geo, _, inv = ref.voronoi(P, bounds, kernel="cubic_spline", threads=1, run_map=2)
        np.savez_compressed(os.path.join(out_dir, f"{name}.npz"), **P, bounds=np.array(bounds, float),
                            home=geo["home"], **{"geo_" + k: v for k, v in geo.items() if k != "home"},
                            ref_m_recovered=inv["m_recovered"], ref_coverage=inv["coverage"],
                            ref_totals=inv["totals"], ref_cell_mass=inv["cell_mass"])
        cov = inv["coverage"]
        print(name, "cells", len(geo["volume"]), "coverage range", cov.min(), cov.max(), "totals", inv["totals"])


if __name__ == "__main__":
    main()
