"""Seeded synthetic SPH snapshots with the shapes, sizes and value distributions of the benchmark
configurations (no dataset is read: every input is generated here from a seed).

  column_snapshot   7,300 equal-mass gas particles (m = 0.05 Msun) in a 2 x 2 x 8.2 pc column: 60 % uniform,
                    40 % from a Gaussian filament (sigma = 0.15 pc) along z through (1, 1); velocities
                    i.i.d. N(0, 1) km/s; grid 100 x 100 x 410 cells of 0.02 pc, unpadded.
  lognormal_cube    N particles in a 10 pc cube sampling a log-normal density field (sigma_ln rho = 1.5,
                    P(k) ~ k^-4 Gaussian random field on a mesh), equal masses, domain padded by max(2h),
                    grid res^3 over the padded box.
Smoothing lengths follow the 57-nearest-neighbour recipe: rho = 57 m / (4/3 pi r57^3) (r57: distance to the
57th neighbour, self excluded) and h = hfact (m / rho)^(1/3) with the kernel's hfact (1.2 for M4).
"""
from __future__ import annotations

import numpy as np

N_NEIGH = 57


def knn_smoothing_lengths(pos: np.ndarray, m: np.ndarray, hfact: float = 1.2, k: int = N_NEIGH) -> np.ndarray:
    from scipy.spatial import cKDTree

    tree = cKDTree(pos)
    d, _ = tree.query(pos, k=k + 1, workers=-1)
    r = d[:, -1]
    rho = k * m / (4.0 / 3.0 * np.pi * r ** 3)
    return hfact * (m / rho) ** (1.0 / 3.0)


def _pack(pos, vel, m, h):
    return {"x": np.ascontiguousarray(pos[:, 0]), "y": np.ascontiguousarray(pos[:, 1]),
            "z": np.ascontiguousarray(pos[:, 2]), "vx": np.ascontiguousarray(vel[:, 0]),
            "vy": np.ascontiguousarray(vel[:, 1]), "vz": np.ascontiguousarray(vel[:, 2]),
            "m": np.ascontiguousarray(m), "h": np.ascontiguousarray(h)}


def column_snapshot(n: int = 7300, seed: int = 1001, box=(2.0, 2.0, 8.2), mass: float = 0.05,
                    uniform_frac: float = 0.6, sigma: float = 0.15, hfact: float = 1.2):
    """Returns (particles, bounds)."""
    rng = np.random.default_rng(seed)
    nu = int(round(uniform_frac * n))
    pos = np.empty((n, 3))
    pos[:nu] = rng.random((nu, 3)) * np.asarray(box)
    nf = n - nu
    fil = np.empty((0, 3))
    while len(fil) < nf:
        c = np.column_stack([box[0] / 2 + sigma * rng.standard_normal(2 * nf),
                             box[1] / 2 + sigma * rng.standard_normal(2 * nf),
                             rng.random(2 * nf) * box[2]])
        ok = (c[:, 0] >= 0) & (c[:, 0] <= box[0]) & (c[:, 1] >= 0) & (c[:, 1] <= box[1])
        fil = np.concatenate([fil, c[ok]])
    pos[nu:] = fil[:nf]
    m = np.full(n, mass)
    h = knn_smoothing_lengths(pos, m, hfact)
    vel = rng.standard_normal((n, 3))
    return _pack(pos, vel, m, h), (0.0, box[0], 0.0, box[1], 0.0, box[2])


def gaussian_random_field(res: int, seed: int, slope: float = -4.0) -> np.ndarray:
    """Unit-variance Gaussian random field on a res^3 periodic mesh with P(k) ~ k^slope."""
    rng = np.random.default_rng(seed)
    white = rng.standard_normal((res, res, res))
    fk = np.fft.rfftn(white)
    kx = np.fft.fftfreq(res)[:, None, None]
    ky = np.fft.fftfreq(res)[None, :, None]
    kz = np.fft.rfftfreq(res)[None, None, :]
    k2 = kx * kx + ky * ky + kz * kz
    k2[0, 0, 0] = np.inf
    fk *= k2 ** (slope / 4.0)  # amplitude ~ sqrt(P) = k^(slope/2)
    g = np.fft.irfftn(fk, s=(res, res, res))
    g -= g.mean()
    g /= g.std()
    return g


def lognormal_cube(n: int = 2_000_000, seed: int = 1002, size: float = 10.0, sigma_ln: float = 1.5,
                   mesh: int = 256, hfact: float = 1.2):
    """Returns (particles, padded bounds).  Equal-mass particles sample a log-normal field: particles are
    distributed multinomially over mesh cells with probability ~ rho, then jittered uniformly in the cell."""
    rng = np.random.default_rng(seed + 7)
    g = gaussian_random_field(mesh, seed)
    rho = np.exp(sigma_ln * g - 0.5 * sigma_ln ** 2)
    p = (rho / rho.sum()).reshape(-1)
    counts = rng.multinomial(n, p)
    cells = np.repeat(np.arange(mesh ** 3), counts)
    ix, iy, iz = np.unravel_index(cells, (mesh, mesh, mesh))
    dx = size / mesh
    pos = (np.column_stack([ix, iy, iz]) + rng.random((n, 3))) * dx
    m = np.full(n, 1.0 / n * 1000.0)  # total mass 1000 (arbitrary units)
    h = knn_smoothing_lengths(pos, m, hfact)
    vel = rng.standard_normal((n, 3))
    pad = 2.0 * h.max()
    b = (-pad, size + pad, -pad, size + pad, -pad, size + pad)
    return _pack(pos, vel, m, h), b


def subset(P: dict, idx) -> dict:
    return {k: np.ascontiguousarray(v[idx]) for k, v in P.items()}
