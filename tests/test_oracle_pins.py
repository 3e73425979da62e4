"""Pins the CPU oracle (oracle/kiwi_oracle.c) to the reference's own known answers -- the checks of
tools/test_generic_kernel.cpp:163-297 (normalisation, brute-force quadrature, region continuity, box-mass
identities, generic vs closed-form cubic) -- and, where oracle/_ref is built, to the reference library
itself (bit-exact) and to the committed reference fixtures under tests/golden/."""
import glob
import os

import numpy as np
import pytest

from conftest import box_faces, scaled_err

REL_TOL = 1e-9
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# ---------------------------------------------------------------- brute-force reference of the maths
# Kernel shape functions w(q) straight from their definitions (B-splines M4/M5/M6, Wendland C2/C4/C6).


def w_direct(key, q):
    q = np.asarray(q, dtype=float)
    p = lambda x, n: np.where(x > 0, np.abs(x) ** n, 0.0)
    if key == "M4":
        w = p(1 - q, 3) - 4 * p(0.5 - q, 3)
    elif key == "M5":
        w = p(1 - q, 4) - 5 * p(0.6 - q, 4) + 10 * p(0.2 - q, 4)
    elif key == "M6":
        w = p(1 - q, 5) - 6 * p(2.0 / 3 - q, 5) + 15 * p(1.0 / 3 - q, 5)
    elif key == "WC2":
        w = p(1 - q, 4) * (1 + 4 * q)
    elif key == "WC4":
        w = p(1 - q, 6) * (1 + 6 * q + 35.0 / 3 * q * q)
    else:
        w = p(1 - q, 8) * (1 + 8 * q + 25 * q * q + 32 * q ** 3)
    return np.where(q >= 1.0, 0.0, w)


BREAKS = {"M4": [0.5, 1.0], "M5": [0.2, 0.6, 1.0], "M6": [1 / 3, 2 / 3, 1.0], "WC2": [1.0], "WC4": [1.0],
          "WC6": [1.0]}
KEYS = ["M4", "M5", "M6", "WC2", "WC4", "WC6"]


def gauss_legendre(n):
    x, w = np.polynomial.legendre.leggauss(n)
    return x, w


GL12, GL48 = gauss_legendre(12), gauss_legendre(48)


def integrate(f, a, b, gl):
    x, w = gl
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    h = 0.5 * (b - a)
    m = 0.5 * (b + a)
    pts = m[..., None] + h[..., None] * x
    return h * np.sum(w * f(pts), axis=-1)


def enclosed(key, A, rho):
    """m(rho) = A int_0^rho w(s) s^2 ds (H = 1), vectorised over rho."""
    rho = np.asarray(rho, float)
    cuts = [0.0] + BREAKS[key]
    tot = np.zeros_like(rho)
    for lo, hi in zip(cuts[:-1], cuts[1:]):
        b = np.clip(rho, lo, hi)
        tot += np.where(b > lo, integrate(lambda s: w_direct(key, s) * s * s, np.full_like(b, lo), b, GL12), 0.0)
    return A * tot


def pyramid(key, A, r0, R0, phi):
    """Kernel mass of the vertex pyramid by nested Gauss-Legendre quadrature (H = 1)."""
    pc = [0.0]
    for c in BREAKS[key]:
        if c * c - r0 * r0 > R0 * R0:
            pc.append(np.arccos(R0 / np.sqrt(c * c - r0 * r0)))
    pc = sorted(x for x in pc if x < phi) + [phi]
    total = 0.0
    for lo, hi in zip(pc[:-1], pc[1:]):
        xs, ws = GL48
        ph = 0.5 * (hi + lo) + 0.5 * (hi - lo) * xs
        vals = []
        for p_ in ph:
            Rmax = R0 / np.cos(p_)
            rc = [0.0]
            for c in BREAKS[key]:
                if c * c > r0 * r0 and np.sqrt(c * c - r0 * r0) < Rmax:
                    rc.append(np.sqrt(c * c - r0 * r0))
            g = r0 * 0.5
            while g < Rmax:
                rc.append(g)
                g *= 2.0
            rc = sorted(rc) + [Rmax]
            rc = np.array(rc)
            lo_, hi_ = rc[:-1], rc[1:]

            def f(R):
                rho2 = r0 * r0 + R * R
                return enclosed(key, A, np.sqrt(rho2)) * r0 * R / (rho2 * np.sqrt(rho2))

            vals.append(np.sum(integrate(f, lo_, hi_, GL48)))
        total += 0.5 * (hi - lo) * np.sum(ws * np.array(vals))
    return total


@pytest.fixture(scope="module")
def a3():
    import json
    t = json.load(open(os.path.join(ROOT, "tests", "golden", "kernel_spec_ref.json")))
    return {k["key"]: k["A3_pi"] / np.pi for k in t}


# ---------------------------------------------------------------- pins


def test_normalisation(a3):
    for key in KEYS:
        norm = 4 * np.pi * enclosed(key, a3[key], 1.0)
        assert abs(norm - 1.0) < 1e-12, key


def test_generic_vs_cubic_closed_form(oracle):
    rng = np.random.default_rng(12345)
    worst = 0.0
    for _ in range(800):
        H = 0.5 + 6.0 * rng.random()
        r0, R0 = H * (0.01 + 1.6 * rng.random()), H * (0.01 + 2.0 * rng.random())
        phi = 1e-3 + (np.pi / 2 - 2e-3) * rng.random()
        ref = oracle.full_integral_new(H / 2, phi, r0, R0)
        gen = oracle.generic_full_integral(0, H, phi, r0, R0)
        worst = max(worst, float(scaled_err(gen, ref)))
    assert worst <= REL_TOL, worst


@pytest.mark.parametrize("k", range(6))
def test_generic_vs_quadrature(oracle, a3, k):
    key = KEYS[k]
    rng = np.random.default_rng(100 + k)
    worst = 0.0
    for _ in range(6):
        r0, R0, phi = 0.02 + 1.4 * rng.random(), 0.02 + 1.6 * rng.random(), 0.05 + 1.5 * rng.random()
        ref = pyramid(key, a3[key], r0, R0, phi)
        gen = oracle.generic_full_integral(k, 1.0, phi, r0, R0)
        worst = max(worst, float(scaled_err(gen, ref)))
    assert worst <= REL_TOL, (key, worst)


@pytest.mark.parametrize("k", range(6))
def test_region_continuity(oracle, k):
    rng = np.random.default_rng(200 + k)
    worst = 0.0
    for _ in range(40):
        r0, R0 = 0.05 + 0.9 * rng.random(), 0.05 + 0.5 * rng.random()
        ends = oracle.generic_edge_breaks(k, 1.0, r0, R0)
        for pb in ends[:-1]:
            lo = oracle.generic_vertex(k, 1.0, r0, R0, pb - 1e-9)
            hi = oracle.generic_vertex(k, 1.0, r0, R0, pb + 1e-9)
            worst = max(worst, abs(hi - lo))
    assert worst <= 1e-7, worst


def box_mass(oracle, p, lo, hi, kernel, H):
    tot = 0.0
    for f in box_faces(lo, hi):
        v, _ = oracle.face_integral(p[0], p[1], p[2], f, kernel=kernel, h=H / 2, support=H)
        tot += v
    return tot


@pytest.mark.parametrize("k", range(6))
def test_box_mass_identities(oracle, k):
    rng = np.random.default_rng(300 + k)
    w1 = wpart = wgrid = 0.0
    for n in range(12):
        H = 0.5 + 3.0 * rng.random()
        p = H * (rng.random(3) - 0.5) * 2.0
        lo = p - H * (1.0 + 2.0 * rng.random(3))
        hi = p + H * (1.0 + 2.0 * rng.random(3))
        w1 = max(w1, abs(box_mass(oracle, p, lo, hi, k, H) - 1.0))
        c = H * (rng.random(3) - 0.5) * 2.0
        half = H * (0.1 + 0.9 * rng.random(3))
        blo, bhi = c - half, c + half
        ax = n % 3
        cut = blo[ax] + (bhi[ax] - blo[ax]) * (0.2 + 0.6 * rng.random())
        hi1, lo2 = bhi.copy(), blo.copy()
        hi1[ax] = cut
        lo2[ax] = cut
        whole = box_mass(oracle, p, blo, bhi, k, H)
        parts = box_mass(oracle, p, blo, hi1, k, H) + box_mass(oracle, p, lo2, bhi, k, H)
        wpart = max(wpart, abs(whole - parts))
        glo, ghi = p - 1.3 * H, p + 1.3 * H
        mid = glo + (ghi - glo) * (0.2 + 0.6 * rng.random(3))
        tot = 0.0
        for cidx in range(8):
            up = [(cidx >> d) & 1 for d in range(3)]
            cl = np.where(up, mid, glo)
            ch = np.where(up, ghi, mid)
            tot += box_mass(oracle, p, cl, ch, k, H)
        wgrid = max(wgrid, abs(tot - 1.0))
    assert w1 <= 1e-10 and wpart <= 1e-10 and wgrid <= 1e-10, (w1, wpart, wgrid)


def test_cubic_box_mass_generic_vs_closed_form(oracle):
    rng = np.random.default_rng(400)
    worst = 0.0
    for _ in range(60):
        H = 0.5 + 3.0 * rng.random()
        c = H * (rng.random(3) - 0.5) * 3.0
        half = H * (0.05 + 1.2 * rng.random(3))
        p = H * (rng.random(3) - 0.5) * 0.8
        mg = mc = 0.0
        for f in box_faces(c - half, c + half):
            mg += oracle.face_integral(*p, f, kernel=0, h=H / 2, support=H)[0]
            mc += oracle.face_integral(*p, f, kernel=-1, h=H / 2)[0]
        worst = max(worst, float(scaled_err(mg, mc)))
    assert worst <= REL_TOL, worst


# ---------------------------------------------------------------- against the reference itself


def test_bitexact_vs_reference_scalar(oracle, reflib):
    rng = np.random.default_rng(7)
    for _ in range(3000):
        H = 0.5 + 6 * rng.random()
        r0, R0 = H * (0.01 + 1.6 * rng.random()), H * (0.01 + 2 * rng.random())
        phi = 1e-3 + (np.pi / 2 - 2e-3) * rng.random()
        assert oracle.full_integral_new(H / 2, phi, r0, R0) == reflib.full_integral_new(H / 2, phi, r0, R0)
        for k in range(6):
            assert oracle.generic_full_integral(k, H, phi, r0, R0) == reflib.generic_full_integral(k, H, phi, r0, R0)


def test_bitexact_vs_reference_faces(oracle, reflib):
    rng = np.random.default_rng(8)
    for _ in range(500):
        p = rng.normal(size=3)
        lo = rng.normal(size=3) * 2
        hi = lo + rng.random(3) * 2
        for f in box_faces(lo, hi):
            for k in (-1, 0, 3, 5):
                assert oracle.face_integral(*p, f, kernel=k, h=0.7, support=1.7) == \
                    reflib.face_integral(*p, f, kernel=k, h=0.7, support=1.7)


def test_oracle_matches_golden_fixtures(oracle):
    files = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "grid_*.npz")))
    assert files, "no golden grid fixtures"
    for fn in files:
        d = np.load(fn)
        P = {k: d[k] for k in ("x", "y", "z", "vx", "vy", "vz", "m", "h")}
        kern = int(d["kernel_index"])
        sup = float(d["support_in_h"])
        generic = bool(d["generic"])
        dens, vx, vy, vz, _, _ = oracle.sph_to_grid(P, d["bounds"], tuple(d["shape"]),
                                                    kernel=kern if generic else -1, support_in_h=sup)
        for name, a in (("density", dens), ("vx", vx), ("vy", vy), ("vz", vz)):
            assert np.array_equal(a, d["out_" + name]), (fn, name)
