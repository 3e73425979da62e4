"""GPU parity of the tabulated cubic integral (the density lookup table and gridded_integral,
src/kernel_integral.cpp:13-190; CubicFaceEvaluator's tabulated branch, :433-458) against the oracle,
which is pinned bit for bit to the reference (tests/test_tabulated_oracle.py), and against the reference's
own sph-to-grid outputs (tests/golden/tab_grid_*.npz, made by tests/golden/make_tabulated_fixtures.py):
the GPU-generated canonical table, lookups in it and in a loaded table, the loader's errors, face
integrals, sph-to-grid in both FP64 forms, the Voronoi map, and the reference's own check that the
tabulated total mass is within 1e-3 of the analytic one (tests/real_data_test.py:191-196).

Agreement bars.  Table entries: the closed form's terms cancel, and the GPU's CUDA libm may differ from
glibc in the last bit, so an entry is held to 4x the reference's own error against the exact value.
Lookups in a loaded table (the same entries on both sides) agree to 1e-13 relative; in the generated
table, to the entries' differences (at most a few 1e-13).  Grids: the cell sums cancel as the analytic ones do, so the per-density-band relative
tolerances of the analytic parity tests apply (4x the reference's own FP64 error envelope there)."""
import glob
import math
import os

import numpy as np
import pytest

from conftest import SMALL_TABLE, box_faces, random_particles, table_probe_points, write_table_file
from gpu_checks import assert_band_tolerance

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "tab_grid_*.npz")))
GRID_TOLS = (4e-10, 4e-9, 1e-7, 1e-12)
KEYS = ("x", "y", "z", "vx", "vy", "vz", "m", "h")


def _tab(kiwi):
    return kiwi.make_kernel_integrator("cubic_spline", use_tabulated_integral=True)


def _expected_clamps(h, phi, r0, R0, s):
    """How many of the three lookup indices of each item fall outside the table (numpy restatement of the
    index arithmetic, the expected value of the GPU's count)."""
    n = 0
    for hh, p, a, b in zip(h, phi, r0, R0):
        if a == 0.0 or b == 0.0 or p == 0.0:
            continue
        r, R, c = a / hh, b / hh, np.cos(p)
        mu = r / np.sqrt(r * r + R * R)
        r = min(r, 2.0)
        i = int(r / (s["rl"] / s["nr01"])) if r < s["rl"] else s["nr01"] + int((r - s["rl"]) / ((2.0 - s["rl"]) / s["nr02"]))
        j = (int(mu / (s["mul"] / (s["nR_01"] - 1))) if mu < s["mul"] else
             s["nR_01"] - 1 + int((mu - s["mul"]) / ((1.0 - s["mul"]) / s["nR_02"])))
        k = (int(c / (s["cphil"] / (s["nphi1"] - 1))) if c < s["cphil"] else
             s["nphi1"] - 1 + int((c - s["cphil"]) / ((1.0 - s["cphil"]) / s["nphi2"])))
        n += (i > s["nr01"] + s["nr02"]) + (j > s["nR_01"] + s["nR_02"] - 1) + (k > s["nphi1"] + s["nphi2"] - 1)
    return n


def _entry_args(flat):
    """(phi, r0, R_0) of canonical-table entries by flat index (the grid of generate_density_table,
    src/kernel_integral.cpp:84-112, restated in numpy)."""
    i, rem = np.divmod(flat, 301 * 301)
    j, k = np.divmod(rem, 301)
    n, rl, mul, cphil = 150, 0.1, 0.98, 0.98
    r0 = np.where(i <= 50, (rl / 50) * i * 1.0, rl + ((2.0 - rl) / 199) * (i - 50) * 1.0)
    mu0 = np.where(j < n, (mul / (n - 1)) * j, mul + ((1.0 - mul) / n) * (j - n + 1))
    with np.errstate(divide="ignore"):
        R0 = r0 * np.sqrt(1.0 - mu0 * mu0) / mu0
    # the C library's acos, as the table's generator calls it (numpy's vectorised arccos may round differently)
    phi = np.array([math.acos((cphil / (n - 1)) * kk) if kk < n else math.acos(cphil + ((1.0 - cphil) / n) * (kk - n + 1))
                    for kk in k.tolist()])
    return phi, r0, R0


def test_generated_table_matches_reference(kiwi, ctx, oracle):
    """Entries are closed-form pyramid masses, whose terms cancel; where the GPU's entry differs from the
    reference's, both are measured against the exact value (__float128 oracle): the GPU's error is at most
    4x the reference's plus a few ulp of the table's scale."""
    from oracle.oracle import Oracle

    info = kiwi.generate_density_table(ctx=ctx)
    assert (info["nr01"], info["nR_01"], info["nphi1"], info["nr02"], info["nR_02"], info["nphi2"]) == \
        (50, 150, 150, 199, 150, 150)
    assert info["n_values"] == 251 * 301 * 301
    g = kiwi.density_table_values(ctx=ctx).reshape(-1)
    oracle.table_reset()
    o = oracle.table_values()
    assert np.all(np.isfinite(g))
    diff = np.abs(g - o)
    same = np.mean(g == o)
    print(f"table: {same:.4f} of the entries bit-identical, max |diff| {diff.max():.3e}")
    assert same > 0.5
    # the 2000 largest differences and 2000 random entries, against the exact value
    rng = np.random.default_rng(1)
    idx = np.unique(np.concatenate([np.argsort(diff)[-2000:], rng.integers(0, o.size, 2000)]))
    idx = idx[(idx // (301 * 301) >= 1) & (idx // (301 * 301) <= 249) & (idx // 301 % 301 < 300) & (idx % 301 < 300)]
    phi, r0, R0 = _entry_args(idx)
    q = Oracle(quad=True)
    tru = np.array([q.full_integral_new(1.0, *a) for a in zip(phi, r0, R0)])
    ge, re_ = np.abs(g[idx] - tru), np.abs(o[idx] - tru)
    print(f"table vs exact: GPU max {ge.max():.3e}, reference max {re_.max():.3e}")
    # entry by entry either side can be the closer one; the error distributions must match
    for q in (0.5, 0.9, 0.99, 1.0):
        gq, rq = np.quantile(ge, q), np.quantile(re_, q)
        assert gq <= 4.0 * rq + 4 * 2.0 ** -52 * 0.125, (q, gq, rq)


def test_lookups_match_oracle(kiwi, ctx, oracle):
    kiwi.generate_density_table(ctx=ctx)
    oracle.table_reset()
    h, phi, r0, R0 = table_probe_points(20000, 5)
    g, clamps = kiwi.gridded_integral(h, phi, r0, R0, ctx=ctx, return_clamps=True)
    o = np.array([oracle.gridded_integral(*t) for t in zip(h, phi, r0, R0)])
    assert np.all(g[(r0 == 0) | (R0 == 0) | (phi == 0)] == 0.0)
    # the GPU's table entries differ from the reference's by at most a few 1e-13 (see above); a lookup is a
    # convex combination of 8 entries
    err = np.abs(g - o)
    print(f"lookups: {np.mean(g == o):.4f} bit-identical, max |diff| {err.max():.3e}, clamps {clamps}")
    assert err.max() <= 1e-12
    canon = dict(nr01=50, nR_01=150, nphi1=150, rl=0.1, mul=0.98, cphil=0.98, nr02=199, nR_02=150, nphi2=150)
    # a clamp can only come from rounding at the tops of the axes; the GPU's cos(phi) may round the other
    # way from numpy's on one of them
    assert abs(clamps - _expected_clamps(h, phi, r0, R0, canon)) <= 2


def test_loaded_table(kiwi, ctx, oracle, tmp_path):
    fn = str(tmp_path / "small.tab")
    vals = write_table_file(fn, seed=9)
    info = kiwi.load_density_table(fn, ctx=ctx)
    assert info["nr01"] == SMALL_TABLE["nr01"] and info["cphil"] == SMALL_TABLE["cphil"]
    v = kiwi.density_table_values(ctx=ctx)
    assert v.shape == (13, 9, 11)
    assert np.array_equal(v[1:-1, :-1, :-1].reshape(-1), vals)
    assert np.array_equal(v[-1], v[-2]) and not v[0].any() and not v[:, -1].any() and not v[:, :, -1].any()
    assert oracle.table_load(fn) == 0
    try:
        h, phi, r0, R0 = table_probe_points(5000, 6)
        g, clamps = kiwi.gridded_integral(h, phi, r0, R0, ctx=ctx, return_clamps=True)
        o = np.array([oracle.gridded_integral(*t) for t in zip(h, phi, r0, R0)])
    finally:
        oracle.table_reset()
    err = np.abs(g - o) / np.maximum(np.abs(o), 1e-3)
    assert err.max() <= 1e-13, err.max()
    assert abs(clamps - _expected_clamps(h, phi, r0, R0, SMALL_TABLE)) <= 2
    kiwi.release_density_table(ctx=ctx)
    with pytest.raises(kiwi.KiwiError):
        kiwi.density_table_info(ctx=ctx)


def test_loader_errors(kiwi, ctx, tmp_path):
    missing = str(tmp_path / "missing.tab")
    with pytest.raises(kiwi.KiwiError, match="could not open density lookup table") as e:
        kiwi.load_density_table(missing, ctx=ctx)
    assert e.value.code == -1
    bad = str(tmp_path / "bad.tab")
    write_table_file(bad, header="4 5 six\n")
    with pytest.raises(kiwi.KiwiError, match="header is malformed"):
        kiwi.load_density_table(bad, ctx=ctx)
    short = str(tmp_path / "short.tab")
    write_table_file(short, truncate=5)
    with pytest.raises(kiwi.KiwiError, match=r"truncated \(short read\)"):
        kiwi.load_density_table(short, ctx=ctx)
    # a shape the reference would divide by zero on
    zero = str(tmp_path / "zero.tab")
    write_table_file(zero, shape=dict(SMALL_TABLE, nR_01=1))
    with pytest.raises(kiwi.KiwiError, match="shape is not usable"):
        kiwi.load_density_table(zero, ctx=ctx)


def test_face_integrals(kiwi, ctx, oracle):
    kiwi.generate_density_table(ctx=ctx)
    oracle.table_reset()
    rng = np.random.default_rng(21)
    parts, faces, ref = [], [], []
    for _ in range(300):
        p = rng.normal(size=3)
        lo = rng.normal(size=3) * 1.5
        hi = lo + 0.05 + rng.random(3) * 1.5
        h = 0.2 + rng.random()
        for f in box_faces(lo, hi):
            parts.append([*p, h])
            faces.append(np.asarray(f).reshape(-1, 3))
            ref.append(oracle.face_integral(*p, f, kernel=-1, h=h, tabulated=True)[0])
    vals, _ = kiwi.face_integrals(np.array(parts), faces, kernel=0, support_in_h=2.0, ctx=ctx, tabulated=True)
    ref = np.array(ref)
    # up to 8 lookups per face, each within 1e-12 of the reference's (the tables' entries differ)
    err = np.abs(vals - ref)
    print(f"faces: max |diff| {err.max():.3e}")
    assert err.max() <= 1e-11, err.max()


@pytest.mark.parametrize("form", ["fp64", "fp64_reference_order"])
@pytest.mark.parametrize("fn", GOLDEN, ids=[os.path.basename(f)[9:-4] for f in GOLDEN])
def test_matches_reference_fixture(kiwi, ctx, fn, form):
    d = np.load(fn)
    P = {k: d[k] for k in KEYS}
    kiwi.generate_density_table(ctx=ctx)
    res = kiwi.sph_to_grid(P, d["bounds"], tuple(d["shape"]), kernel=_tab(kiwi), ctx=ctx, precision=form)
    errs = assert_band_tolerance(res.density, d["out_density"], GRID_TOLS, label=os.path.basename(fn))
    print(f"{os.path.basename(fn)} {form}: band errors {errs}")
    m = d["out_density"] > 1e-2 * d["out_density"].max()
    for name in ("vx", "vy", "vz"):
        assert np.max(np.abs(getattr(res, name)[m] - d["out_" + name][m])) <= 1e-8, name
    assert res.stats["table_clamps"] >= 0


@pytest.mark.parametrize("form", ["fp64", "fp64_reference_order"])
def test_random_cases_vs_oracle(kiwi, ctx, oracle, form):
    kiwi.generate_density_table(ctx=ctx)
    oracle.table_reset()
    for seed, shape in ((71, (12, 12, 12)), (72, (9, 14, 11))):
        P = random_particles(150, seed, hmin=0.05, hmax=0.35)
        bounds = (0.0, 2.0, 0.0, 2.0, 0.0, 2.0)
        res = kiwi.sph_to_grid(P, bounds, shape, kernel=_tab(kiwi), ctx=ctx, precision=form, raw=True)
        dens = oracle.sph_to_grid(P, bounds, shape, tabulated=True)[0]
        assert_band_tolerance(res.density, dens, GRID_TOLS, label=f"seed {seed}")


def test_lattice_and_reference_order_agree(kiwi, ctx):
    P = random_particles(400, 73, hmin=0.04, hmax=0.3)
    bounds, shape = (0.0, 2.0, 0.0, 2.0, 0.0, 2.0), (20, 20, 20)
    a = kiwi.sph_to_grid(P, bounds, shape, kernel=_tab(kiwi), ctx=ctx, precision="fp64")
    b = kiwi.sph_to_grid(P, bounds, shape, kernel=_tab(kiwi), ctx=ctx, precision="fp64_reference_order")
    assert_band_tolerance(a.density, b.density, GRID_TOLS, label="lattice vs per-cell")
    # every cell of the particles' bounding boxes is evaluated in both forms
    assert a.stats["evaluated_pairs"] == b.stats["evaluated_pairs"] == a.stats["bbox_pairs"]


def test_tabulated_mass_close_to_analytic(kiwi, ctx):
    """tests/real_data_test.py:191-196: the tabulated total mass within 1e-3 of the analytic one."""
    d = np.load(os.path.join(ROOT, "tests", "golden", "tab_grid_padded.npz"))
    P = {k: d[k] for k in KEYS}
    tab = kiwi.sph_to_grid(P, d["bounds"], tuple(d["shape"]), kernel=_tab(kiwi), ctx=ctx)
    ana = kiwi.sph_to_grid(P, d["bounds"], tuple(d["shape"]), ctx=ctx)
    vol = np.prod([(d["bounds"][2 * i + 1] - d["bounds"][2 * i]) / d["shape"][i] for i in range(3)])
    mt, ma = tab.density.sum() * vol, ana.density.sum() * vol
    assert abs(mt - ma) / ma < 1e-3
    assert abs(ma - P["m"].sum()) / P["m"].sum() < 1e-12


def test_voronoi_map_vs_oracle(kiwi, ctx, oracle):
    fn = os.path.join(ROOT, "tests", "golden", "vor_blob_cubic.npz")
    d = np.load(fn)
    P = {k: d[k] for k in KEYS}
    geo = {k[4:]: d[k] for k in d.files if k.startswith("geo_")}
    kiwi.generate_density_table(ctx=ctx)
    oracle.table_reset()
    res = kiwi.map_voronoi(P, d["home"], geo, kernel=_tab(kiwi), raw=True, ctx=ctx)
    dens = oracle.map_voronoi(P, d["home"], geo, kernel=-1, support_in_h=2.0, tabulated=True)[0]
    assert_band_tolerance(res.density, dens, GRID_TOLS, label="voronoi tabulated")
    # the tabulated mass differs from the analytic one by the table's interpolation error (1.3e-3 on this
    # blob, a property of the reference's algorithm), and equals the oracle's
    vol = geo["volume"]
    ana = kiwi.map_voronoi(P, d["home"], geo, raw=True, ctx=ctx)
    m_gpu, m_or, m_ana = (res.density * vol).sum(), (dens * vol).sum(), (ana.density * vol).sum()
    assert abs(m_gpu - m_or) <= 1e-12 * m_or
    assert abs(m_gpu - m_ana) <= 5e-3 * m_ana


def test_deterministic_and_forms_without_tabulated(kiwi, ctx):
    P = random_particles(200, 74)
    bounds, shape = (0.0, 2.0, 0.0, 2.0, 0.0, 2.0), (12, 12, 12)
    a = kiwi.sph_to_grid(P, bounds, shape, kernel=_tab(kiwi), ctx=ctx, raw=True)
    b = kiwi.sph_to_grid(P, bounds, shape, kernel=_tab(kiwi), ctx=ctx, raw=True)
    assert np.array_equal(a.raw, b.raw)
    with pytest.raises(kiwi.KiwiError) as e:
        kiwi.sph_to_grid(P, bounds, shape, kernel=_tab(kiwi), ctx=ctx, precision="fp32_mixed")
    assert e.value.code == -6
    with pytest.raises(kiwi.KiwiError) as e:
        kiwi.sph_to_grid(P, bounds, shape, kernel=kiwi.make_kernel_integrator("wendland_c4",
                                                                             use_tabulated_integral=True), ctx=ctx)
    assert e.value.code == -1
    import torch

    dP = {k: torch.tensor(P[k], device="cuda") for k in KEYS}
    cot = torch.zeros(4 * 12 ** 3, dtype=torch.float64, device="cuda")
    with pytest.raises(kiwi.KiwiError) as e:
        kiwi.sph_to_grid_adjoint_device(dP, bounds, shape, cot, {"x": torch.empty_like(dP["x"])}, kernel=_tab(kiwi),
                                        ctx=ctx)
    assert e.value.code == -6
    out = {k: torch.empty(12 ** 3, dtype=torch.float64, device="cuda") for k in ("density", "vx", "vy", "vz")}
    with pytest.raises(kiwi.KiwiError) as e:
        kiwi.Batch([dict(particles=dP, bounds=bounds, shape=shape, kernel=_tab(kiwi), out=out)], ctx=ctx)
    assert e.value.code == -6
