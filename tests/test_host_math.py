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
