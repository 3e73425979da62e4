"""Splitting work over several GPUs: the host side of kiwi_sph_to_grid_device_part, the Voronoi map's
spatial slabs, and snapshots dealt to GPUs.

The library splits a grid's 8x8x8-cell tiles into n parts, each a contiguous run of the tile order
(tile (tx, ty, tz) at index (tx * nty + ty) * ntz + tz) with a near-equal number of (tile, particle)
entries: tile t belongs to part floor(prefix(t) * n / W) (capped at n - 1), prefix(t) being the entries of
the tiles before t and W their total; with W = 0 the tiles split evenly by number.  This module restates
that rule on the host -- the entry counts from the particles' clamped support boxes, exactly as the
binning computes them -- so that a rank knows which x rows of the grid it owns (to copy back only those)
before the GPU has run, and every rank agrees on the split without talking to the others.  A Voronoi
map splits by spatial slabs of cells (each rank maps the particles that can reach its slab and keeps its
cells), and a batch of snapshots by whole snapshots, longest first.  It also holds the max-over-ranks
reduction of a step's timing.
"""
from __future__ import annotations

import numpy as np

TILE = 8


def tile_grid(shape):
    nx, ny, nz = (int(s) for s in shape)
    return (nx + TILE - 1) // TILE, (ny + TILE - 1) // TILE, (nz + TILE - 1) // TILE


def _support_boxes(particles: dict, bounds, shape, support_in_h: float):
    """Per particle: whether its clamped support box (src/cartesian_grid.cpp:211-237) holds a cell, and
    the box's inclusive cell range [lo, hi] on each axis (as floats; meaningful where it holds a cell)."""
    nx, ny, nz = (int(s) for s in shape)
    x, y, z, h = (np.asarray(particles[k], dtype=np.float64) for k in ("x", "y", "z", "h"))
    b = [float(v) for v in bounds]
    d = [(b[1] - b[0]) / nx, (b[3] - b[2]) / ny, (b[5] - b[4]) / nz]
    ok = h > 0
    radius = support_in_h * h
    lo, hi = [], []
    for c, mn, dd, n in ((x, b[0], d[0], nx), (y, b[2], d[1], ny), (z, b[4], d[2], nz)):
        with np.errstate(invalid="ignore", over="ignore"):
            a0 = np.clip(np.floor((c - radius - mn) / dd), -2e9, 2e9)
            a1 = np.clip(np.floor((c + radius - mn) / dd), -2e9, 2e9)
        a0 = np.maximum(a0, 0)
        a1 = np.minimum(a1, n - 1)
        ok &= a0 <= a1
        lo.append(a0)
        hi.append(a1)
    return ok, lo, hi


def _support_tiles(particles: dict, bounds, shape, support_in_h: float):
    """Per particle: whether its clamped support box holds a cell, and the tile range [t0, t1) of that box
    on each axis."""
    ok, lo, hi = _support_boxes(particles, bounds, shape, support_in_h)
    t0 = [np.where(ok, lo[i], 0).astype(np.int64) // TILE for i in range(3)]
    t1 = [np.where(ok, hi[i], 0).astype(np.int64) // TILE + 1 for i in range(3)]
    return ok, t0, t1


def _box_sums(table: np.ndarray, t0, t1) -> np.ndarray:
    """Sum of table[t0x:t1x, t0y:t1y, t0z:t1z] per box, from the 3-D prefix sums (inclusion-exclusion)."""
    S = np.zeros(tuple(n + 1 for n in table.shape), dtype=np.int64)
    S[1:, 1:, 1:] = table.astype(np.int64).cumsum(0).cumsum(1).cumsum(2)
    out = np.zeros(len(t0[0]), dtype=np.int64)
    for sx, ix in ((1, t1[0]), (-1, t0[0])):
        for sy, iy in ((1, t1[1]), (-1, t0[1])):
            for sz, iz in ((1, t1[2]), (-1, t0[2])):
                out += sx * sy * sz * S[ix, iy, iz]
    return out


def tile_entry_counts(particles: dict, bounds, shape, support_in_h: float) -> np.ndarray:
    """(tile, particle) entries per tile, in tile order: the number of particles whose clamped support
    box (src/cartesian_grid.cpp:211-237) touches the tile."""
    ntx, nty, ntz = tile_grid(shape)
    ok, t0, t1 = _support_tiles(particles, bounds, shape, support_in_h)
    t0 = [t[ok] for t in t0]
    t1 = [t[ok] for t in t1]
    cnt = np.zeros((ntx + 1, nty + 1, ntz + 1), dtype=np.int64)
    # 3-D difference array: +1 on the box's corners with inclusion-exclusion signs
    for sx, ix in ((1, t0[0]), (-1, t1[0])):
        for sy, iy in ((1, t0[1]), (-1, t1[1])):
            for sz, iz in ((1, t0[2]), (-1, t1[2])):
                np.add.at(cnt, (ix, iy, iz), sx * sy * sz)
    cnt = cnt.cumsum(0).cumsum(1).cumsum(2)[:ntx, :nty, :ntz]
    return cnt.reshape(-1)


def part_particles(particles: dict, bounds, shape, support_in_h: float, owner: np.ndarray,
                   part: int) -> np.ndarray:
    """Indices (ascending) of the particles whose clamped support box touches a tile of `part`: every
    particle that contributes to a cell of the part.  A rank that maps only these particles (in this
    order) gets its own cells' sums exactly as the whole snapshot gives them -- each cell adds its
    particles in ascending order and the others add nothing -- and keeps `cells_of_part` of the result.
    A cell no particle reaches takes the snapshot's mean velocity (src/cartesian_grid.cpp:302-315), which
    needs the whole snapshot."""
    ntx, nty, ntz = tile_grid(shape)
    ok, t0, t1 = _support_tiles(particles, bounds, shape, support_in_h)
    mine = (np.asarray(owner) == part).reshape(ntx, nty, ntz)
    hit = _box_sums(mine, t0, t1) > 0
    return np.nonzero(ok & hit)[0]


def tile_owners(weights: np.ndarray, n_parts: int) -> np.ndarray:
    """The part of every tile (the library's rule, integer arithmetic as on the device)."""
    w = np.minimum(np.asarray(weights, dtype=np.int64), 0xFFFFFFFF)
    n = len(w)
    prefix = np.concatenate([[0], np.cumsum(w)[:-1]]) if n else np.zeros(0, dtype=np.int64)
    W = int(w.sum())
    if W > 0:
        owner = (prefix * n_parts) // W
    else:
        owner = (np.arange(n, dtype=np.int64) * n_parts) // max(n, 1)
    return np.minimum(owner, n_parts - 1)


def part_rows(owner: np.ndarray, part: int, shape) -> tuple[int, int]:
    """The x rows [ix0, ix1) of cells that cover every tile of `part` (empty if it owns none).  The cells
    of rows ix0 .. ix1 - 1 are contiguous in the (ix * ny + iy) * nz + iz layout."""
    nx = int(shape[0])
    ntx, nty, ntz = tile_grid(shape)
    mine = np.nonzero(owner == part)[0]
    if len(mine) == 0:
        return 0, 0
    tx0, tx1 = int(mine[0]) // (nty * ntz), int(mine[-1]) // (nty * ntz)
    return tx0 * TILE, min(nx, (tx1 + 1) * TILE)


def cells_of_part(owner: np.ndarray, part: int, shape) -> np.ndarray:
    """Boolean mask over the cells (x-major) of the tiles owned by `part`."""
    nx, ny, nz = (int(s) for s in shape)
    ntx, nty, ntz = tile_grid(shape)
    t = (owner == part).reshape(ntx, nty, ntz)
    m = np.repeat(np.repeat(np.repeat(t, TILE, 0), TILE, 1), TILE, 2)[:nx, :ny, :nz]
    return m.reshape(-1)


def _cell_vertex_rows(cells: dict):
    """Per cell, its vertex rows [start, end) in vxyz (a cell's faces, and their vertices, are contiguous)."""
    fo = np.asarray(cells["face_off"], dtype=np.int64)
    vo = np.asarray(cells["vert_off"], dtype=np.int64)
    return vo[fo[:-1]], vo[fo[1:]]


def _cell_midpoints(cells: dict, axis: int) -> np.ndarray:
    """Per cell, the midpoint (lo + hi) / 2 of its vertices' extent along `axis` (0 for a cell without
    vertices): min, max and one sum, so that every restatement of it rounds alike."""
    start, end = _cell_vertex_rows(cells)
    coord = np.asarray(cells["vxyz"], dtype=np.float64).reshape(-1, 3)[:, axis]
    mid = np.zeros(len(start))
    has = end > start
    if has.any():
        # the cells' rows are back to back in cell order (CSR), so the non-empty cells' starts delimit them
        s = start[has]
        mid[has] = (np.minimum.reduceat(coord, s) + np.maximum.reduceat(coord, s)) * 0.5
    return mid


def voronoi_cell_owners(cells: dict, n_parts: int, axis: int = 0) -> np.ndarray:
    """Voronoi cells split into n_parts spatial slabs along `axis`: the cells ordered by the midpoint of
    their vertices' extent along it (ties by cell index), cut into runs of near-equal cell counts (the cell
    of rank k goes to part floor(k n / n_cells))."""
    nc = len(np.asarray(cells["face_off"])) - 1
    if nc <= 0:
        return np.zeros(0, dtype=np.int64)
    centre = _cell_midpoints(cells, axis)
    order = np.argsort(centre, kind="stable")
    owner = np.empty(nc, dtype=np.int64)
    owner[order] = (np.arange(nc, dtype=np.int64) * n_parts) // nc
    return owner


def voronoi_part_particles(particles: dict, home_cell, cells: dict, owner: np.ndarray, part: int,
                           support_in_h: float) -> np.ndarray:
    """Indices (ascending) of the particles whose cell walk can reach a cell of `part`: those whose home
    cell is the part's, and those whose support sphere comes within 1.001 radii of the box around the
    part's cell vertices.  A walk visits the home cell and otherwise only cells behind a face within the
    support radius (src/mapping.cpp:187-193), so every (cell, particle) pair of the part's cells comes from
    these particles; a walk depends on its particle alone and a cell adds its pairs in particle order, so a
    rank that maps only these particles (in this order) gets its own cells bit for bit as the whole
    snapshot gives them.  A cell no particle reaches takes the snapshot's mean velocity
    (src/mapping.cpp:490-500), which needs the whole snapshot."""
    start, end = _cell_vertex_rows(cells)
    owner = np.asarray(owner)
    v = np.asarray(cells["vxyz"], dtype=np.float64).reshape(-1, 3)
    rows = np.repeat(owner == part, end - start)
    home = np.asarray(home_cell, dtype=np.int64)
    n = len(home)
    valid = (home >= 0) & (home < len(owner))
    sel = np.zeros(n, dtype=bool)
    sel[valid] = owner[home[valid]] == part
    if rows.any():
        lo, hi = v[rows].min(axis=0), v[rows].max(axis=0)
        d2 = np.zeros(n)
        for a, k in enumerate("xyz"):
            c = np.asarray(particles[k], dtype=np.float64)
            d2 += np.maximum(np.maximum(lo[a] - c, c - hi[a]), 0.0) ** 2
        r = 1.001 * support_in_h * np.asarray(particles["h"], dtype=np.float64)
        sel |= d2 <= r * r
    return np.nonzero(sel)[0]


def snapshot_work(particles: dict, bounds, shape, support_in_h: float) -> int:
    """A snapshot's (particle, cell) pairs within the particles' clamped support boxes
    (src/cartesian_grid.cpp:211-237): the work estimate by which snapshots are dealt to GPUs."""
    ok, lo, hi = _support_boxes(particles, bounds, shape, support_in_h)
    cells = np.ones(int(ok.sum()), dtype=np.int64)
    for a in range(3):
        cells *= (hi[a][ok] - lo[a][ok] + 1).astype(np.int64)
    return int(cells.sum())


def assign_snapshots_lpt(work, n_parts: int) -> list[np.ndarray]:
    """Whole snapshots dealt to n_parts GPUs, longest processing time first: by work descending (ties by
    index), each to the part with the least work so far (ties to the lowest part).  Every rank computes
    the same assignment from the same work list.  Returns each part's snapshot indices, ascending.
    A batch that mixes kernels should weigh each snapshot's pairs by its kernel's cost per pair: on one
    B200 the generic kernels run at 0.99 G (Wendland C4) and 0.68 G (M6) support pairs/s against 4.89 G/s
    for the cubic spline's closed form."""
    work = np.asarray(work, dtype=np.int64)
    load = np.zeros(n_parts, dtype=np.int64)
    parts = [[] for _ in range(n_parts)]
    for i in np.argsort(-work, kind="stable"):
        p = int(np.argmin(load))
        parts[p].append(int(i))
        load[p] += work[i]
    return [np.array(sorted(q), dtype=np.int64) for q in parts]


def reduce_step(ms: float, pairs: float, device=None):
    """(max over ranks of ms, sum over ranks of pairs) through torch.distributed (NCCL or gloo)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([ms, pairs], dtype=torch.float64, device=device)
    mx = t.clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(mx[0]), float(t[1])
