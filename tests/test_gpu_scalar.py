"""GPU parity of the batched scalar integral layer (full_integral_new, generic_full_integral and the face
walk) on the reference test's sampling (tools/test_generic_kernel.cpp:178-259).  Both the GPU and the FP64
oracle (bit-identical to the reference) are measured against the __float128 oracle: the GPU's error
distribution (max, 99.9th percentile, median) must match the reference's, and most values must agree
with the reference to the last bit."""
import numpy as np
import pytest

from conftest import box_faces

pytestmark = pytest.mark.gpu


def _rel(x, t):
    x, t = np.asarray(x), np.asarray(t)
    return np.abs(x - t) / np.maximum(np.abs(t), 1e-300)


def assert_same_error_distribution(gpu, ref, truth, label, min_identical=0.0, floor=1e-15):
    """The largest error within 4x the reference's, the 99.9th percentile and the median within 2x."""
    eg, er = _rel(gpu, truth), _rel(ref, truth)
    for q, factor in ((1.0, 4.0), (0.999, 2.0), (0.5, 2.0)):
        g, r = np.quantile(eg, q), np.quantile(er, q)
        assert g <= factor * r + floor, f"{label}: quantile {q}: GPU {g:.3e} vs reference {r:.3e}"
    same = np.mean(np.asarray(gpu) == np.asarray(ref))
    assert same >= min_identical, f"{label}: only {same:.2f} of the values bit-identical to the reference"


def _sample(n, seed):
    rng = np.random.default_rng(seed)
    H = 0.5 + 6.0 * rng.random(n)
    r0 = H * (0.01 + 1.6 * rng.random(n))
    R0 = H * (0.01 + 2.0 * rng.random(n))
    phi = 1e-3 + (np.pi / 2 - 2e-3) * rng.random(n)
    return H, r0, R0, phi


def test_full_integral_cubic_and_generic(kiwi, ctx, oracle):
    from oracle.oracle import Oracle
    q = Oracle(quad=True)
    H, r0, R0, phi = _sample(4000, 12345)
    g = kiwi.full_integral_new(H / 2, phi, r0, R0, ctx=ctx)
    o = np.array([oracle.full_integral_new(a, b, c, d) for a, b, c, d in zip(H / 2, phi, r0, R0)])
    t = np.array([q.full_integral_new(a, b, c, d) for a, b, c, d in zip(H / 2, phi, r0, R0)])
    assert_same_error_distribution(g, o, t, "cubic", min_identical=0.6)
    for k in range(6):
        gk = kiwi.generic_full_integral(kiwi.KernelSpec(k), H, phi, r0, R0, ctx=ctx)
        ok = np.array([oracle.generic_full_integral(k, a, b, c, d) for a, b, c, d in zip(H, phi, r0, R0)])
        tk = np.array([q.generic_full_integral(k, a, b, c, d) for a, b, c, d in zip(H, phi, r0, R0)])
        assert_same_error_distribution(gk, ok, tk, f"generic kernel {k}", min_identical=0.5)


def test_full_integral_guards(kiwi, ctx):
    """r0 == 0, R_0 == 0 and phi == 0 give exactly 0 (src/kernel_integral.cpp:410-413)."""
    z = np.zeros(3)
    o = np.ones(3)
    assert np.all(kiwi.full_integral_new(o, o, z, o, ctx=ctx) == 0.0)
    assert np.all(kiwi.full_integral_new(o, o, o, z, ctx=ctx) == 0.0)
    assert np.all(kiwi.full_integral_new(o, z, o, o, ctx=ctx) == 0.0)
    assert np.all(kiwi.generic_full_integral(kiwi.KernelSpec(4), o, z, o, o, ctx=ctx) == 0.0)


@pytest.mark.parametrize("kernel", [-1, 0, 1, 2, 3, 4, 5])
def test_face_integrals_and_out_vert(kiwi, ctx, oracle, kernel):
    from oracle.oracle import Oracle
    q = Oracle(quad=True)
    rng = np.random.default_rng(77 + kernel)
    parts, faces, ref, ref_ov, tru = [], [], [], [], []
    for _ in range(120):
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
            tru.append(q.face_integral(*p, f, kernel=kernel, h=H / 2, support=H)[0])
    if kernel < 0:
        vals, ov = kiwi.face_integrals(parts, faces, kernel=0, support_in_h=2.0, ctx=ctx)
    else:
        vals, ov = kiwi.face_integrals(parts, faces, kernel=kernel, support_in_h=1.0, generic_path=True, ctx=ctx)
    assert_same_error_distribution(vals, ref, tru, f"faces kernel {kernel}")
    assert np.array_equal(ov, np.array(ref_ov))


def test_polygon_faces(kiwi, ctx, oracle):
    """Non-rectangular faces (regular n-gons in random planes), as a Voronoi cell has."""
    from oracle.oracle import Oracle
    q = Oracle(quad=True)
    rng = np.random.default_rng(5)
    parts, faces, ref, tru = [], [], [], []
    for _ in range(300):
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
        tru.append(q.face_integral(*p, poly.reshape(-1), kernel=-1, h=h)[0])
    vals, _ = kiwi.face_integrals(parts, faces, kernel=0, support_in_h=2.0, ctx=ctx)
    assert_same_error_distribution(vals, ref, tru, "polygons")


def test_invalid_arguments_raise(kiwi, ctx):
    with pytest.raises(kiwi.KiwiError):
        kiwi.get_kernel("gaussian")
    with pytest.raises(kiwi.KiwiError):
        kiwi.face_integrals([[0, 0, 0, 1]], [np.zeros((4, 3))], kernel=9, ctx=ctx)
