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
    L.hm_lattice_edge.argtypes = [C.c_double] * 3 + [dp]
    L.hm_lattice_edge_pair.argtypes = [C.c_double] * 3 + [dp]
    L.hm_lattice_corner.restype = C.c_double
    L.hm_lattice_corner.argtypes = [C.c_double] * 4 + [dp]
    L.hm_lattice_point.restype = C.c_double
    L.hm_lattice_point.argtypes = [C.c_double] * 4 + [dp]
    L.hm_lattice_generic_edge.argtypes = [C.c_int] + [C.c_double] * 3 + [dp]
    L.hm_lattice_generic_corner.restype = C.c_double
    L.hm_lattice_generic_corner.argtypes = [C.c_int] + [C.c_double] * 4 + [dp, dp]
    L.hm_lattice_generic_point.restype = C.c_double
    L.hm_lattice_generic_point.argtypes = [C.c_int] + [C.c_double] * 4 + [dp]
    L.hm_lattice_generic_point_grad.argtypes = [C.c_int] + [C.c_double] * 4 + [dp]
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



def _lattice_cases(n, seed):
    """Random lattice-point offsets within and beyond the support of a particle with h = 0.8, a part of
    them with one offset shrunk towards the particle's planes."""
    rng = np.random.default_rng(seed)
    h = 0.8
    for it in range(n):
        a = 2.4 * h * rng.random(3)
        if it % 7 == 0:
            a[0] *= 1e-3
        if it % 11 == 0:
            a[1] *= 1e-6
        yield h, a


def test_lattice_edge_pair(hm):
    """The edge tiers of a (p, q) pair evaluated together (lattice_edge_pair: shared half-chord, log term and
    reciprocal) equal the two single tiers (lattice_edge) to rounding.  The tiers enter a corner value
    multiplied by (r0/h)^3 / pi, so the differences are compared at that scale."""
    dp = C.POINTER(C.c_double)
    worst = 0.0
    for h, a in _lattice_cases(20000, 31):
        p, q = a[0], a[1]
        if not (p * p + q * q <= 4 * h * h):
            continue
        pair, one, two = np.zeros(4), np.zeros(2), np.zeros(2)
        hm.hm_lattice_edge_pair(h, p, q, pair.ctypes.data_as(dp))
        hm.hm_lattice_edge(h, p, q, one.ctypes.data_as(dp))
        hm.hm_lattice_edge(h, q, p, two.ctypes.data_as(dp))
        K = np.array([p, p, q, q]) ** 3 / h ** 3 / np.pi
        worst = max(worst, float(np.abs(K * (pair - np.concatenate([one, two]))).max()))
    assert worst < 4e-15, worst


def test_lattice_point(hm):
    """A lattice point's three corner values evaluated together (lattice_point: one root, two reciprocals,
    three log terms for the six pyramids) equal the sum of the three single corner values (lattice_corner)
    to rounding, inside the support, beyond it, and next to the particle's planes."""
    dp = C.POINTER(C.c_double)
    worst = 0.0
    for h, a in _lattice_cases(20000, 32):
        ax, ay, az = a
        E = {}
        for nm, (r0, R0) in dict(xy=(ax, ay), xz=(ax, az), yx=(ay, ax), yz=(ay, az), zx=(az, ax), zy=(az, ay)).items():
            E[nm] = np.zeros(2)
            if r0 * r0 + R0 * R0 <= 4 * h * h:
                hm.hm_lattice_edge(h, r0, R0, E[nm].ctypes.data_as(dp))
        e = np.concatenate([E[k] for k in ("xy", "xz", "yx", "yz", "zx", "zy")])
        point = hm.hm_lattice_point(h, ax, ay, az, e.ctypes.data_as(dp))
        corners = sum(hm.hm_lattice_corner(h, r0, a1, a2, np.concatenate([E[e1], E[e2]]).ctypes.data_as(dp))
                      for r0, a1, a2, e1, e2 in ((ax, ay, az, "xy", "xz"), (ay, ax, az, "yx", "yz"),
                                                 (az, ax, ay, "zx", "zy")))
        worst = max(worst, abs(point - corners))
    assert worst < 4e-15, worst


def test_lattice_generic_point(hm):
    """A lattice point's six generic vertex tiers evaluated together (lattice_generic_point: shared 1/r, 1/a_c,
    three atanh terms, the first basis integral from the three walls' angles) equal the sum of the three walls'
    vertex pairs (lattice_generic_corner) to the latter's own rounding, for every kernel of the table, inside
    the support, beyond it and next to the particle's planes.  The generic tiers sum terms that cancel (the
    kernel's polynomial coefficients times powers of q0), so that rounding level depends on the kernel: it is
    measured as the change of the corner sum when every offset moves by one ulp (the function itself moves
    by ~1e-16 there), and the point-wise form must stay within 1.5x of it."""
    dp = C.POINTER(C.c_double)

    def evaluate(kern, H, ax, ay, az):
        R = {}
        for nm, (r0, R0) in dict(xy=(ax, ay), xz=(ax, az), yx=(ay, ax), yz=(ay, az), zx=(az, ax),
                                 zy=(az, ay)).items():
            R[nm] = np.zeros(7)
            hm.hm_lattice_generic_edge(kern, H, r0, R0, R[nm].ctypes.data_as(dp))
        recs = np.concatenate([R[k] for k in ("xy", "xz", "yx", "yz", "zx", "zy")])
        point = hm.hm_lattice_generic_point(kern, H, ax, ay, az, recs.ctypes.data_as(dp))
        corners = sum(hm.hm_lattice_generic_corner(kern, H, r0, a1, a2, R[e1].ctypes.data_as(dp),
                                                   R[e2].ctypes.data_as(dp))
                      for r0, a1, a2, e1, e2 in ((ax, ay, az, "xy", "xz"), (ay, ax, az, "yx", "yz"),
                                                 (az, ax, ay, "zx", "zy")))
        return point, corners

    for kern in range(6):
        diff, noise = [], []
        for h, a in _lattice_cases(2500, 40 + kern):
            point, corners = evaluate(kern, 2.0 * h, *a)
            _, moved = evaluate(kern, 2.0 * h, *np.nextafter(a, 9.0))
            diff.append(abs(point - corners))
            noise.append(abs(moved - corners))
        diff, noise = np.array(diff), np.array(noise)
        print(f"kernel {kern}: point vs corners max {diff.max():.2e} q99 {np.quantile(diff, 0.99):.2e}; "
              f"corner rounding max {noise.max():.2e} q99 {np.quantile(noise, 0.99):.2e}")
        assert diff.max() <= 1.5 * noise.max() + 1e-15, kern
        assert np.quantile(diff, 0.99) <= 1.5 * np.quantile(noise, 0.99) + 1e-15, kern


def test_lattice_generic_point_derivatives(hm):
    """The generic lattice point in dual numbers (the adjoint's instantiation: edge records with derivatives
    of their continuity offsets, the point's six vertex tiers) has the double form's value and derivatives
    that match central differences of the double form (records recomputed at each offset)."""
    dp = C.POINTER(C.c_double)

    def value(kern, H, a):
        recs = np.zeros(6 * 7)
        for e, (r0, R0) in enumerate(((a[0], a[1]), (a[0], a[2]), (a[1], a[0]), (a[1], a[2]), (a[2], a[0]),
                                      (a[2], a[1]))):
            hm.hm_lattice_generic_edge(kern, H, r0, R0, recs[7 * e:].ctypes.data_as(dp))
        return hm.hm_lattice_generic_point(kern, H, a[0], a[1], a[2], recs.ctypes.data_as(dp))

    def fd(kern, H, a, c, d):
        ap, am = a.copy(), a.copy()
        ap[c] += d
        am[c] -= d
        return (value(kern, H, ap) - value(kern, H, am)) / (2 * d)

    rng = np.random.default_rng(61)
    worst_v, worst_d = 0.0, 0.0
    for kern in range(6):
        for _ in range(150):
            H = 1.6
            a = H * (0.05 + 0.9 * rng.random(3))
            out = np.zeros(4)
            hm.hm_lattice_generic_point_grad(kern, H, a[0], a[1], a[2], out.ctypes.data_as(dp))
            worst_v = max(worst_v, abs(out[0] - value(kern, H, a)))
            for c in range(3):
                # Richardson-extrapolated central differences (step 1e-4 H and half of it): truncation ~1e-13,
                # rounding (the generic tiers' ~1e-13 noise over the step) ~1e-9
                d = 1e-4 * H
                est = (4.0 * fd(kern, H, a, c, d / 2) - fd(kern, H, a, c, d)) / 3.0
                worst_d = max(worst_d, abs(out[1 + c] - est) * H)
    print(f"dual vs double value {worst_v:.2e}; derivative vs central differences (x H) {worst_d:.2e}")
    assert worst_v < 1e-13
    assert worst_d < 1e-8


def _plane_distance(p, v):
    """|r0| of the face walk (src/kernel_integral.cpp:481-495) in the same IEEE operations, in numpy."""
    (x1, y1, z1), (x2, y2, z2), (x3, y3, z3) = (tuple(float(c) for c in v[i]) for i in range(3))
    A = (y2 - y1) * (z3 - z1) - (y3 - y1) * (z2 - z1)
    B = (z2 - z1) * (x3 - x1) - (z3 - z1) * (x2 - x1)
    Cc = (x2 - x1) * (y3 - y1) - (x3 - x1) * (y2 - y1)
    D = -A * x1 - B * y1 - Cc * z1
    norm = np.sqrt(A * A + B * B + Cc * Cc)
    return abs((A * p[0] + B * p[1] + Cc * p[2] + D) / norm)


def test_reachability_at_the_plane_distance(hm, oracle):
    """face_reachable rejects a face whose plane lies at or beyond the support before its vertex loop.  On
    convex polygons of 3 to 9 vertices in random orientations, with the support equal to the plane
    distance, one ulp either side of it and 1e-12 .. 1e-3 relative either side, and with the foot of the
    perpendicular inside and outside the polygon, its decision is the reference's (out_vert != n) every time."""
    rng = np.random.default_rng(13)
    dp = C.POINTER(C.c_double)
    checked = 0
    for _ in range(400):
        n = int(rng.integers(3, 10))
        ang = np.sort(rng.random(n)) * 2 * np.pi
        rad = 0.2 + rng.random()
        q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        off = rng.normal(size=3)
        verts = np.ascontiguousarray(np.stack([rad * np.cos(ang), rad * np.sin(ang), np.zeros(n)], axis=1) @ q.T
                                     + off)
        local = np.array([rng.normal() * rad, rng.normal() * rad, (0.05 + rng.random()) * rng.choice([-1, 1])])
        p = q @ local + off
        d = _plane_distance(p, verts)
        sups = [d, np.nextafter(d, 0), np.nextafter(d, np.inf)]
        sups += [d * (1 + s * e) for e in (1e-12, 1e-9, 1e-6, 1e-3) for s in (-1, 1)]
        for sup in sups:
            r = hm.hm_face_reachable(*p, sup, verts.ctypes.data_as(dp), n)
            _, ov = oracle.face_integral(*p, verts, kernel=0, h=sup / 2, support=sup)
            assert r == (ov != n), (n, sup / d - 1)
            checked += 1
    assert checked == 400 * 11
