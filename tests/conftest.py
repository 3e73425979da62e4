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
