"""The device maths header compiled for the host must reproduce the oracle (= the reference) bit for bit:
a CPU check of every transcribed formula of the cubic and generic tiers, the face walk and the
reachability rule (tests/host_math_check.cpp)."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from conftest import box_faces

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def hm(tmp_path_factory):
    out = tmp_path_factory.mktemp("hm") / "libhm.so"
    src = os.path.join(ROOT, "tests", "host_math_check.cpp")
    subprocess.run(["g++", "-O2", "-fPIC", "-shared", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-o",
                    str(out), src], check=True)
    L = C.CDLL(str(out))
    L.hm_full_integral.restype = C.c_double
    L.hm_full_integral.argtypes = [C.c_int] + [C.c_double] * 4
    dp = C.POINTER(C.c_double)
    L.hm_face_integral.restype = C.c_double
    L.hm_face_integral.argtypes = [C.c_double] * 3 + [C.c_int, C.c_double, C.c_double, dp, C.c_int,
                                                      C.POINTER(C.c_int)]
    L.hm_face_reachable.argtypes = [C.c_double] * 4 + [dp, C.c_int]
    L.hm_cell_grad.argtypes = [C.c_double] * 10 + [dp]
    return L


def test_tiers_bit_identical(hm, oracle):
    rng = np.random.default_rng(11)
    for _ in range(4000):
        H = 0.5 + 6.0 * rng.random()
        r0, R0 = H * (0.01 + 1.6 * rng.random()), H * (0.01 + 2.0 * rng.random())
        phi = 1e-3 + (np.pi / 2 - 2e-3) * rng.random()
        assert hm.hm_full_integral(-1, H / 2, phi, r0, R0) == oracle.full_integral_new(H / 2, phi, r0, R0)
        for k in range(6):
            assert hm.hm_full_integral(k, H, phi, r0, R0) == oracle.generic_full_integral(k, H, phi, r0, R0)


def test_face_walk_bit_identical(hm, oracle):
    rng = np.random.default_rng(12)
    for _ in range(400):
        p = rng.normal(size=3)
        lo = rng.normal(size=3) * 2
        hi = lo + 0.05 + rng.random(3) * 2
        for f in box_faces(lo, hi):
            v = np.ascontiguousarray(f, dtype=np.float64)
            for k in (-1, 0, 2, 5):
                ov = C.c_int(0)
                a = hm.hm_face_integral(*p, k, 0.7, 1.7, v.ctypes.data_as(C.POINTER(C.c_double)), 4, C.byref(ov))
                b, ovo = oracle.face_integral(*p, f, kernel=k, h=0.7, support=1.7)
                assert a == b and ov.value == ovo
                reach = hm.hm_face_reachable(*p, 1.4 if k < 0 else 1.7, v.ctypes.data_as(C.POINTER(C.c_double)), 4)
                assert reach == (ovo != 4)


def test_dual_cell_gradient(hm, oracle):
    """The adjoint's forward-mode evaluation of one cell's Msum (kiwi_b200/csrc/dual.cuh through the
    templated face walk): its value equals the FP64 evaluation bit for bit, and its derivatives with
    respect to x0, y0, z0, h agree with central differences of the exact (__float128) cell integral."""
    from oracle.oracle import load_truth

    truth = load_truth()
    rng = np.random.default_rng(21)
    bounds, n = [0.0, 1.0] * 3, 8
    d = 1.0 / n
    out = (C.c_double * 6)()
    worst = 0.0
    for _ in range(10):
        h = 0.05 + 0.15 * rng.random()
        th = np.array([*(0.2 + 0.6 * rng.random(3)), h])

        def M(t):
            P = dict(x=[t[0]], y=[t[1]], z=[t[2]], vx=[0.0], vy=[0.0], vz=[0.0], m=[1.0], h=[t[3]])
            return truth.sph_to_grid(P, bounds, (n, n, n))[4][0]

        fd = np.zeros((4, n ** 3))
        for k in range(4):
            step = 1e-6 * max(abs(th[k]), h)
            a, b = th.copy(), th.copy()
            a[k] += step
            b[k] -= step
            fd[k] = (M(a) - M(b)) / (2 * step)
        g = np.zeros((4, n ** 3))
        for c in np.nonzero(M(th))[0]:
            ix, iy, iz = c // (n * n), (c // n) % n, c % n
            hm.hm_cell_grad(*th, (ix + 0.5) * d, (iy + 0.5) * d, (iz + 0.5) * d, d / 2, d / 2, d / 2, out)
            assert out[0] == out[1]
            if out[1] > 0:
                g[:, c] = out[2:]
        worst = max(worst, (np.abs(g - fd) / np.abs(fd).max(axis=1, keepdims=True)).max())
    assert worst < 1e-7, worst

