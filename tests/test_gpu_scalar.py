"""GPU parity of the batched scalar integral layer (full_integral_new, generic_full_integral and the face
walk) against the CPU oracle, on the reference test's sampling (tools/test_generic_kernel.cpp:178-259)."""
import numpy as np
import pytest

from conftest import box_faces

pytestmark = pytest.mark.gpu

TOL = 1e-13  # relative per value (plus an absolute floor of 1e-16 for values near zero)


def _close(a, b, tol=TOL):
    a, b = np.asarray(a), np.asarray(b)
    return np.abs(a - b) <= tol * np.maximum(np.abs(b), 1e-3)


def test_full_integral_cubic_and_generic(kiwi, ctx, oracle):
    rng = np.random.default_rng(12345)
    n = 20000
    H = 0.5 + 6.0 * rng.random(n)
    r0 = H * (0.01 + 1.6 * rng.random(n))
    R0 = H * (0.01 + 2.0 * rng.random(n))
    phi = 1e-3 + (np.pi / 2 - 2e-3) * rng.random(n)
    # include the guards: r0 == 0, R_0 == 0, phi == 0
    r0[:3] = 0.0
    R0[3:6] = 0.0
    phi[6:9] = 0.0
    g = kiwi.full_integral_new(H / 2, phi, r0, R0, ctx=ctx)
    o = np.array([oracle.full_integral_new(a, b, c, d) for a, b, c, d in zip(H / 2, phi, r0, R0)])
    assert np.all(_close(g, o)), np.max(np.abs(g - o))
    assert np.all(g[:9] == 0.0)
    for k in range(6):
        gk = kiwi.generic_full_integral(kiwi.KernelSpec(k), H, phi, r0, R0, ctx=ctx)
        ok = np.array([oracle.generic_full_integral(k, a, b, c, d) for a, b, c, d in zip(H, phi, r0, R0)])
        assert np.all(_close(gk, ok)), (k, np.max(np.abs(gk - ok)))


@pytest.mark.parametrize("kernel", [-1, 0, 1, 2, 3, 4, 5])
def test_face_integrals_and_out_vert(kiwi, ctx, oracle, kernel):
    rng = np.random.default_rng(77 + kernel)
    parts, faces, ref, ref_ov = [], [], [], []
    for _ in range(300):
        H = 0.5 + 3.0 * rng.random()
        c = H * (rng.random(3) - 0.5) * 3.0
        half = H * (0.05 + 1.2 * rng.random(3))
        p = H * (rng.random(3) - 0.5) * 0.8
        for f in box_faces(c - half, c + half):
            parts.append([p[0], p[1], p[2], H / 2 if kernel < 0 else H])
            faces.append(np.array(f).reshape(4, 3))
            v, ov = oracle.face_integral(*p, f, kernel=kernel, h=H / 2, support=H)
            ref.append(v)
            ref_ov.append(ov)
    if kernel < 0:
        vals, ov = kiwi.face_integrals(parts, faces, kernel=0, support_in_h=2.0, ctx=ctx)
    else:
        vals, ov = kiwi.face_integrals(parts, faces, kernel=kernel, support_in_h=1.0, generic_path=True, ctx=ctx)
    assert np.all(_close(vals, ref)), np.max(np.abs(vals - np.array(ref)))
    assert np.array_equal(ov, np.array(ref_ov))


def test_polygon_faces(kiwi, ctx, oracle):
    """Non-rectangular faces (regular n-gons in random planes), as a Voronoi cell has."""
    rng = np.random.default_rng(5)
    parts, faces, ref = [], [], []
    for _ in range(400):
        nv = int(rng.integers(3, 9))
        centre = rng.normal(size=3)
        nrm = rng.normal(size=3)
        nrm /= np.linalg.norm(nrm)
        u = np.cross(nrm, [1.0, 0.0, 0.0] if abs(nrm[0]) < 0.9 else [0.0, 1.0, 0.0])
        u /= np.linalg.norm(u)
        v = np.cross(nrm, u)
        rad = 0.2 + rng.random()
        ang = np.sort(rng.random(nv)) * 2 * np.pi
        poly = np.array([centre + rad * (np.cos(a) * u + np.sin(a) * v) for a in ang])
        p = centre + rng.normal(size=3) * 0.7
        h = 0.3 + 0.5 * rng.random()
        parts.append([p[0], p[1], p[2], h])
        faces.append(poly)
        ref.append(oracle.face_integral(*p, poly.reshape(-1), kernel=-1, h=h)[0])
    vals, _ = kiwi.face_integrals(parts, faces, kernel=0, support_in_h=2.0, ctx=ctx)
    assert np.all(_close(vals, ref)), np.max(np.abs(vals - np.array(ref)))


def test_invalid_arguments_raise(kiwi, ctx):
    with pytest.raises(kiwi.KiwiError):
        kiwi.get_kernel("gaussian")
    with pytest.raises(kiwi.KiwiError):
        kiwi.face_integrals([[0, 0, 0, 1]], [np.zeros((4, 3))], kernel=9, ctx=ctx)
