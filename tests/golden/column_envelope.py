#!/usr/bin/env python3
"""Measures the reference's own FP64 error on the 7,300-particle column workload (the example-cutout
configuration: 2 x 2 x 8.2 pc, 100 x 100 x 410 cells) for the seeded 6-particle subset the GPU tests
use, against the __float128 oracle, per density band (> 1e-2, 1e-4..1e-2, 1e-6..1e-4 of the peak; and
cells below, in absolute terms relative to the peak).  The GPU test bounds |gpu - reference| by 4x these.
Takes ~4 minutes (the float128 oracle is slow).  Run from the repository root.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))
from gpu_checks import band_max_rel  # noqa: E402
from kiwi_b200.workloads import column_snapshot, subset  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402

P, b = column_snapshot()
idx = np.sort(np.random.default_rng(0).choice(len(P["x"]), 6, replace=False))
Ps = subset(P, idx)
ref = Oracle().sph_to_grid(Ps, b, (100, 100, 410))[0]
tru = Oracle(quad=True).sph_to_grid(Ps, b, (100, 100, 410))[0]
print(band_max_rel(ref, tru))
