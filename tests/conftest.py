import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU and the built libkiwi_b200.so")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reflib():
    from oracle.oracle import load_ref
    r = load_ref()
    if r is None:
        pytest.skip("reference library oracle/_ref/libkiwi_ref.so not built on this machine")
    return r


@pytest.fixture(scope="session")
def kiwi():
    import kiwi_b200
    return kiwi_b200


@pytest.fixture(scope="session")
def ctx(kiwi):
    return kiwi.Context(0)


def box_faces(lo, hi):
    """The 6 faces of an axis-aligned box in the winding of src/cartesian_grid.cpp:54-72."""
    xm, ym, zm = lo
    xp, yp, zp = hi
    return [
        [xp, ym, zp, xp, yp, zp, xp, yp, zm, xp, ym, zm],
        [xm, yp, zm, xm, yp, zp, xm, ym, zp, xm, ym, zm],
        [xp, yp, zm, xp, yp, zp, xm, yp, zp, xm, yp, zm],
        [xm, ym, zp, xp, ym, zp, xp, ym, zm, xm, ym, zm],
        [xm, yp, zp, xp, yp, zp, xp, ym, zp, xm, ym, zp],
        [xp, ym, zm, xp, yp, zm, xm, yp, zm, xm, ym, zm],
    ]


def random_particles(n, seed, box=(0.0, 2.0), hmin=0.05, hmax=0.3):
    rng = np.random.default_rng(seed)
    P = {k: rng.uniform(box[0], box[1], n) for k in ("x", "y", "z")}
    for k in ("vx", "vy", "vz"):
        P[k] = rng.standard_normal(n)
    P["m"] = rng.uniform(0.5, 1.5, n)
    P["h"] = rng.uniform(hmin, hmax, n)
    return P


def scaled_err(a, b, abs_tol=1e-12, rel_tol=1e-9):
    """The combined error measure of tools/test_generic_kernel.cpp:114-118."""
    a, b = np.asarray(a), np.asarray(b)
    return np.abs(a - b) / (abs_tol / rel_tol + np.maximum(np.abs(a), np.abs(b)))


# A small density lookup table in the reference's text format (load_density_table,
# src/kernel_integral.cpp:20-55): header nr01 nR_01 nphi1 / rl mul cphil / nr02 nR_02 nphi2, then the
# nr0 x nR_0 x nphi values with k fastest.
SMALL_TABLE = dict(nr01=4, nR_01=5, nphi1=6, rl=0.3, mul=0.9, cphil=0.85, nr02=7, nR_02=3, nphi2=4)


def write_table_file(path, seed=0, shape=SMALL_TABLE, truncate=0, header=None):
    s = shape
    nr0, nR0, nphi = s["nr01"] + s["nr02"], s["nR_01"] + s["nR_02"], s["nphi1"] + s["nphi2"]
    vals = np.random.default_rng(seed).uniform(0.0, 0.15, nr0 * nR0 * nphi)
    if truncate:
        vals = vals[:-truncate]
    with open(path, "w") as f:
        f.write(header if header is not None else
                f"{s['nr01']} {s['nR_01']} {s['nphi1']}\n{s['rl']!r} {s['mul']!r} {s['cphil']!r}\n"
                f"{s['nr02']} {s['nR_02']} {s['nphi2']}\n")
        for i in range(0, len(vals), 7):
            f.write(" ".join(repr(float(v)) for v in vals[i:i + 7]) + "\n")
    return vals


def table_probe_points(n, seed):
    """(h, phi, r0, R_0) spanning the table's axes, its edges and beyond (r0 > 2h, R_0 -> 0, phi -> 0)."""
    rng = np.random.default_rng(seed)
    h = rng.uniform(0.2, 3.0, n)
    r0 = h * rng.uniform(0.0, 2.6, n)
    R0 = h * np.exp(rng.uniform(-9.0, 1.5, n))
    phi = rng.uniform(0.0, np.pi / 2, n)
    phi[::11] = rng.uniform(0.0, 0.02, phi[::11].size)
    r0[::13] = 2.0 * h[::13]
    r0[::17] = 0.0
    R0[::19] = 0.0
    phi[::23] = 0.0
    return h, phi, r0, R0
