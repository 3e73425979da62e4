#!/usr/bin/env python3
"""Measures the algorithmic work per (particle, cell) pair -- F_pair flops and T_pair transcendentals
in the reference's evaluation order -- with the operation-counting oracle, on a seeded sample of a
benchmark workload's particles.  Each +, -, *, /, sqrt is one flop; each sin, cos, acos, atan, atanh,
log, pow one transcendental (sincos: two).  Output: JSON on stdout.

  python oracle/count_work.py [--workload lognormal|column] [--kernel 0] [--sample 40]
"""
import argparse
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
from oracle.oracle import CountingOracle  # noqa: E402
from kiwi_b200.workloads import column_snapshot, lognormal_cube, subset  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="lognormal")
    ap.add_argument("--kernel", type=int, default=-1, help="-1: cubic closed form; 0..5 generic table kernel")
    ap.add_argument("--sample", type=int, default=40)
    ap.add_argument("--n", type=int, default=2_000_000)
    ap.add_argument("--res", type=int, default=256)
    a = ap.parse_args()
    if a.workload == "lognormal":
        P, b = lognormal_cube(n=a.n)
        shape = (a.res,) * 3
    else:
        P, b = column_snapshot()
        shape = (100, 100, 410)
    idx = np.sort(np.random.default_rng(7).choice(len(P["x"]), a.sample, replace=False))
    Ps = subset(P, idx)
    co = CountingOracle()
    sup = [2.0, 2.5, 3.0, 2.0, 2.0, 2.0][max(a.kernel, 0)]
    out = {"workload": a.workload, "kernel": a.kernel, "sample_particles": a.sample}
    for label, only in (("bbox", 0), ("support", 1)):
        co.lib.orc_set_support_cells_only(only)
        co.reset()
        st = co.sph_to_grid(Ps, b, shape, kernel=a.kernel, support_in_h=sup)[5]
        f, t = co.counts()
        n = st.sphere_pairs if only else st.bbox_pairs
        out.update({f"{label}_pairs": n, f"F_pair_{label}": f / n, f"T_pair_{label}": t / n})
    co.lib.orc_set_support_cells_only(0)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
