"""The hand-written adjoint of the sph-to-grid raw sums (kiwi_sph_to_grid_adjoint_device and its
torch.autograd.Function binding) against central finite differences: of the GPU forward pass, of the
FP64 oracle (the reference's CPU path restated operation by operation) and of the __float128 oracle.

Finite differences use the relative step 1e-6 * max(|theta|, h) (the stated FD recipe).  The derivative of
the loss with respect to one particle's inputs depends on that particle alone (the raw sums are sums of
per-particle terms), so each particle's FD is taken on a forward pass of that particle alone: its
rounding noise is then the particle's own, ~1e-16 |L| / step."""
import numpy as np
import pytest

from conftest import random_particles

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

KEYS = ("x", "y", "z", "h", "m", "vx", "vy", "vz")
FD_TOL = 1e-5  # adjoint vs finite differences, relative to the particle's gradient scale


def _dev(P):
    return {k: torch.tensor(np.asarray(P[k], dtype=np.float64), device="cuda") for k in KEYS}


def _adjoint(kiwi, ctx, P, bounds, shape, cot):
    Pd = _dev(P)
    g = {k: torch.empty_like(Pd[k]) for k in KEYS}
    st = kiwi.sph_to_grid_adjoint_device(Pd, bounds, shape, torch.tensor(cot, device="cuda"), g, ctx=ctx)
    return {k: g[k].cpu().numpy() for k in KEYS}, st


def _one(P, i):
    return {k: np.array([P[k][i]], dtype=np.float64) for k in ("x", "y", "z", "vx", "vy", "vz", "m", "h")}


def _fd(loss, P1, h):
    """Central differences of loss(P1) in every input of a one-particle snapshot."""
    out = {}
    for k in KEYS:
        t = float(P1[k][0])
        d = 1e-6 * max(abs(t), h)
        a = {kk: vv.copy() for kk, vv in P1.items()}
        b = {kk: vv.copy() for kk, vv in P1.items()}
        a[k][0] = t + d
        b[k][0] = t - d
        out[k] = (loss(a) - loss(b)) / (2 * d)
    return out


def _rel_errors(ad, fd, i):
    """Per particle: the largest |ad - fd| over the geometric inputs (x, y, z, h; one unit, one scale),
    over m, and over v, each relative to that group's largest |fd|."""
    errs = []
    for group in (("x", "y", "z", "h"), ("m",), ("vx", "vy", "vz")):
        scale = max(abs(fd[k]) for k in group)
        if scale == 0.0:
            errs.append(max(abs(ad[k][i]) for k in group))
            continue
        errs.append(max(abs(ad[k][i] - fd[k]) for k in group) / scale)
    return errs


def test_adjoint_matches_fd_of_gpu_forward(kiwi, ctx):
    bounds, shape = (0.0, 2.0, 0.0, 2.0, 0.0, 2.0), (20, 20, 20)
    P = random_particles(300, seed=41, hmin=0.06, hmax=0.35)
    rng = np.random.default_rng(7)
    cot = rng.standard_normal(4 * int(np.prod(shape)))
    ad, st = _adjoint(kiwi, ctx, P, bounds, shape, cot)
    assert st["evaluated_pairs"] > 0 and st["launches"] >= 1

    def loss(P1):
        r = kiwi.sph_to_grid(P1, bounds, shape, raw=True, ctx=ctx, precision="fp64")
        return float(r.raw.reshape(-1) @ cot)

    worst = np.zeros(3)
    for i in rng.choice(len(P["x"]), 40, replace=False):
        fd = _fd(loss, _one(P, i), float(P["h"][i]))
        worst = np.maximum(worst, _rel_errors(ad, fd, i))
    print(f"adjoint vs FD of the GPU forward (x/y/z/h, m, v): {worst}")
    assert worst.max() <= FD_TOL, worst


def test_adjoint_matches_fd_of_oracle(kiwi, ctx, oracle):
    """FD of the FP64 oracle (bit-identical to the reference's CPU sph-to-grid) and of the exact
    (__float128) integral on a small grid."""
    from oracle.oracle import load_truth

    truth = load_truth()
    bounds, shape = (0.0, 1.0, 0.0, 1.0, 0.0, 1.0), (8, 8, 8)
    P = random_particles(6, seed=5, box=(0.15, 0.85), hmin=0.06, hmax=0.2)
    rng = np.random.default_rng(8)
    cot = rng.standard_normal(4 * 512)
    ad, _ = _adjoint(kiwi, ctx, P, bounds, shape, cot)
    worst_ref, worst_truth = np.zeros(3), np.zeros(3)
    for i in range(len(P["x"])):
        fd_ref = _fd(lambda P1: float(oracle.sph_to_grid(P1, bounds, shape)[4].reshape(-1) @ cot), _one(P, i),
                     float(P["h"][i]))
        fd_tru = _fd(lambda P1: float(truth.sph_to_grid(P1, bounds, shape)[4].reshape(-1) @ cot), _one(P, i),
                     float(P["h"][i]))
        worst_ref = np.maximum(worst_ref, _rel_errors(ad, fd_ref, i))
        worst_truth = np.maximum(worst_truth, _rel_errors(ad, fd_tru, i))
    print(f"adjoint vs FD of the FP64 oracle: {worst_ref}; vs FD of the exact integral: {worst_truth}")
    assert worst_ref.max() <= FD_TOL, worst_ref
    assert worst_truth.max() <= 1e-7, worst_truth


def test_autograd_function_gradcheck(kiwi, ctx):
    from kiwi_b200.autograd import sph_to_grid_raw

    bounds, shape = (0.0, 1.0, 0.0, 1.0, 0.0, 1.0), (6, 6, 6)
    P = random_particles(3, seed=9, box=(0.25, 0.75), hmin=0.1, hmax=0.2)
    ins = [torch.tensor(P[k], device="cuda", dtype=torch.float64, requires_grad=True) for k in KEYS]

    def f(*t):
        return sph_to_grid_raw(*t, bounds, shape, precision="fp64_reference_order", ctx=ctx)

    assert torch.autograd.gradcheck(f, tuple(ins), eps=1e-7, atol=1e-6, rtol=1e-4, fast_mode=True)


def test_density_loss_gradient(kiwi, ctx):
    """A projected-density loss through the torch binding, L = sum_xy (sum_z rho dz - T_xy)^2, against
    central differences of the same loss."""
    from kiwi_b200.autograd import sph_to_grid

    bounds, shape = (0.0, 1.0, 0.0, 1.0, 0.0, 1.0), (16, 16, 16)
    P = random_particles(400, seed=2004, box=(0.05, 0.95), hmin=0.04, hmax=0.12)
    rng = np.random.default_rng(3)
    T = torch.tensor(rng.uniform(0.0, 400.0, (16, 16)), device="cuda")
    dz = 1.0 / 16

    def loss_of(tensors):
        rho = sph_to_grid(*tensors, bounds, shape, ctx=ctx)[0]
        return ((rho.sum(dim=2) * dz - T) ** 2).sum()

    ins = [torch.tensor(P[k], device="cuda", dtype=torch.float64, requires_grad=True) for k in KEYS]
    L = loss_of(ins)
    L.backward()
    ad = {k: t.grad.cpu().numpy() for k, t in zip(KEYS, ins)}
    worst = 0.0
    for i in rng.choice(400, 12, replace=False):
        g = np.array([ad[k][i] for k in ("x", "y", "z", "h")])
        fd = []
        for j, k in enumerate(("x", "y", "z", "h")):
            t = float(P[k][i])
            d = 1e-6 * max(abs(t), float(P["h"][i]))
            vals = []
            for s in (1, -1):
                Q = {kk: np.array(vv, dtype=np.float64) for kk, vv in P.items()}
                Q[k][i] = t + s * d
                with torch.no_grad():
                    vals.append(float(loss_of([torch.tensor(Q[kk], device="cuda") for kk in KEYS])))
            fd.append((vals[0] - vals[1]) / (2 * d))
        fd = np.array(fd)
        worst = max(worst, np.abs(g - fd).max() / np.abs(fd).max())
    print(f"projected-density loss: autograd vs FD {worst:.3e}")
    assert worst <= FD_TOL, worst


def test_adjoint_deterministic_and_edge_cases(kiwi, ctx):
    bounds, shape = (0.0, 2.0, 0.0, 2.0, 0.0, 2.0), (12, 12, 12)
    P = random_particles(200, seed=12)
    # one particle far outside the grid, one with h = 0, one with h < 0: no mass on the grid, no gradient
    P["x"][0], P["h"][1], P["h"][2] = 50.0, 0.0, -0.1
    rng = np.random.default_rng(1)
    cot = rng.standard_normal(4 * 12 ** 3)
    a, _ = _adjoint(kiwi, ctx, P, bounds, shape, cot)
    b, _ = _adjoint(kiwi, ctx, P, bounds, shape, cot)
    for k in KEYS:
        assert np.array_equal(a[k], b[k]), k
        assert a[k][0] == 0.0 and a[k][1] == 0.0 and a[k][2] == 0.0, k
    # the gradient of the total mass (cotangent 1 on M) with respect to m is each particle's mass fraction
    # inside the grid: 1 for particles whose support lies inside it
    ones = np.concatenate([np.ones(12 ** 3), np.zeros(3 * 12 ** 3)])
    c, _ = _adjoint(kiwi, ctx, P, bounds, shape, ones)
    inside = ((P["x"] - 2 * P["h"] > 0) & (P["x"] + 2 * P["h"] < 2) & (P["y"] - 2 * P["h"] > 0) &
              (P["y"] + 2 * P["h"] < 2) & (P["z"] - 2 * P["h"] > 0) & (P["z"] + 2 * P["h"] < 2) & (P["h"] > 0))
    assert inside.sum() > 20
    assert np.abs(c["m"][inside] - 1.0).max() < 1e-12
    # and mass inside the grid does not move when a fully enclosed particle moves or changes h: the cell
    # derivatives (each up to ~m/h) cancel to rounding; the cancellation inside the face walk leaves
    # ~1e-10 of m/h (measured up to 7.5e-11)
    scale = P["m"][inside] / P["h"][inside]
    for k in ("x", "y", "z", "h"):
        assert np.abs(c[k][inside] / scale).max() < 1e-9, k
    # empty snapshot
    E = {k: np.zeros(0) for k in P}
    e, st = _adjoint(kiwi, ctx, E, bounds, shape, cot)
    assert st["evaluated_pairs"] == 0


@pytest.mark.parametrize("kname", ["wendland_c4", "quintic_spline", "cubic_generic"])
def test_generic_kernel_adjoint_matches_fd(kiwi, ctx, kname):
    """The generic kernels' adjoint (edge records and lattice points in dual numbers over the kernel's
    tables) against central differences of the GPU forward with the same kernel, and of the FP64 oracle on
    a small grid."""
    ki = (kiwi.make_kernel_integrator("cubic_spline", generic_path=True) if kname == "cubic_generic"
          else kiwi.make_kernel_integrator(kname))
    bounds, shape = (0.0, 2.0, 0.0, 2.0, 0.0, 2.0), (16, 16, 16)
    P = random_particles(120, seed=43, hmin=0.06, hmax=0.3)
    rng = np.random.default_rng(17)
    cot = rng.standard_normal(4 * int(np.prod(shape)))
    Pd = _dev(P)
    g = {k: torch.empty_like(Pd[k]) for k in KEYS}
    st = kiwi.sph_to_grid_adjoint_device(Pd, bounds, shape, torch.tensor(cot, device="cuda"), g, kernel=ki, ctx=ctx)
    ad = {k: g[k].cpu().numpy() for k in KEYS}
    assert st["evaluated_pairs"] > 0

    def loss(P1):
        r = kiwi.sph_to_grid(P1, bounds, shape, raw=True, ctx=ctx, precision="fp64", kernel=ki)
        return float(r.raw.reshape(-1) @ cot)

    worst = np.zeros(3)
    for i in rng.choice(len(P["x"]), 20, replace=False):
        fd = _fd(loss, _one(P, i), float(P["h"][i]))
        worst = np.maximum(worst, _rel_errors(ad, fd, i))
    print(f"{kname}: adjoint vs FD of the GPU forward (x/y/z/h, m, v): {worst}")
    assert worst.max() <= FD_TOL, worst


def test_generic_kernel_adjoint_matches_fd_of_oracle(kiwi, ctx, oracle):
    bounds, shape = (0.0, 1.0, 0.0, 1.0, 0.0, 1.0), (8, 8, 8)
    P = random_particles(5, seed=6, box=(0.15, 0.85), hmin=0.06, hmax=0.2)
    rng = np.random.default_rng(9)
    cot = rng.standard_normal(4 * 512)
    ki = kiwi.make_kernel_integrator("wendland_c4")
    Pd = _dev(P)
    g = {k: torch.empty_like(Pd[k]) for k in KEYS}
    kiwi.sph_to_grid_adjoint_device(Pd, bounds, shape, torch.tensor(cot, device="cuda"), g, kernel=ki, ctx=ctx)
    ad = {k: g[k].cpu().numpy() for k in KEYS}
    spec = kiwi.get_kernel("wendland_c4")
    worst = np.zeros(3)
    for i in range(len(P["x"])):
        fd = _fd(lambda P1: float(oracle.sph_to_grid(P1, bounds, shape, kernel=spec.index,
                                                     support_in_h=spec.radkern)[4].reshape(-1) @ cot),
                 _one(P, i), float(P["h"][i]))
        worst = np.maximum(worst, _rel_errors(ad, fd, i))
    print(f"wendland_c4: adjoint vs FD of the FP64 oracle: {worst}")
    assert worst.max() <= FD_TOL, worst


def test_adjoint_rejects_tabulated(kiwi, ctx):
    P = random_particles(4, seed=1)
    Pd = _dev(P)
    g = {"x": torch.empty_like(Pd["x"])}
    cot = torch.zeros(4 * 8 ** 3, dtype=torch.float64, device="cuda")
    with pytest.raises(kiwi.KiwiError) as e:
        kiwi.sph_to_grid_adjoint_device(Pd, (0, 2, 0, 2, 0, 2), (8, 8, 8), cot, g,
                                        kernel=kiwi.make_kernel_integrator("cubic_spline", use_tabulated_integral=True),
                                        ctx=ctx)
    assert e.value.code == -6
