"""Host side of splitting one grid over several GPUs (kiwi_b200.shard): the tile entry counts, the
ownership rule, and the multi-rank agreement and timing reduction over gloo with two ranks on the CPU."""
import glob
import os
import socket

import numpy as np
import pytest

from conftest import random_particles
from kiwi_b200 import shard


def _brute_counts(P, bounds, shape, sup):
    nx, ny, nz = shape
    ntx, nty, ntz = [(s + 7) // 8 for s in shape]
    d = [(bounds[1] - bounds[0]) / nx, (bounds[3] - bounds[2]) / ny, (bounds[5] - bounds[4]) / nz]
    mn = [bounds[0], bounds[2], bounds[4]]
    cnt = np.zeros((ntx, nty, ntz), dtype=np.int64)
    for i in range(len(P["x"])):
        h = P["h"][i]
        if not h > 0:
            continue
        r = sup * h
        lo, hi = [], []
        for c, k, n in ((P["x"][i], 0, nx), (P["y"][i], 1, ny), (P["z"][i], 2, nz)):
            a0 = max(int(np.floor((c - r - mn[k]) / d[k])), 0)
            a1 = min(int(np.floor((c + r - mn[k]) / d[k])), n - 1)
            lo.append(a0)
            hi.append(a1)
        if any(a > b for a, b in zip(lo, hi)):
            continue
        cnt[lo[0] // 8:hi[0] // 8 + 1, lo[1] // 8:hi[1] // 8 + 1, lo[2] // 8:hi[2] // 8 + 1] += 1
    return cnt.reshape(-1)


def test_tile_entry_counts_match_brute_force():
    from kiwi_b200 import shard

    for seed, shape in ((1, (20, 17, 33)), (2, (8, 8, 8)), (3, (41, 9, 16))):
        P = random_particles(300, seed, box=(-0.3, 2.3), hmin=0.01, hmax=0.6)
        P["h"][:5] = 0.0
        P["h"][5:8] = -1.0
        b = (0.0, 2.0, 0.1, 1.9, -0.2, 2.0)
        assert np.array_equal(shard.tile_entry_counts(P, b, shape, 2.0), _brute_counts(P, b, shape, 2.0))


def test_tile_owners_cover_contiguous_balanced():
    from kiwi_b200 import shard

    rng = np.random.default_rng(4)
    for n in (1, 2, 3, 8, 64):
        w = rng.integers(0, 1000, 500)
        own = shard.tile_owners(w, n)
        assert own.min() >= 0 and own.max() <= n - 1
        assert np.all(np.diff(own) >= 0)  # contiguous runs in tile order
        W = w.sum()
        for p in range(n):
            assert w[own == p].sum() <= W / n + w.max() + 1
    # no entries at all: split evenly by tile count
    own = shard.tile_owners(np.zeros(10, dtype=np.int64), 3)
    assert list(np.bincount(own, minlength=3)) == [4, 3, 3]


def test_part_rows_cover_the_part():
    from kiwi_b200 import shard

    shape = (40, 24, 16)
    ntx, nty, ntz = shard.tile_grid(shape)
    own = shard.tile_owners(np.arange(ntx * nty * ntz) % 7, 4)
    for p in range(4):
        ix0, ix1 = shard.part_rows(own, p, shape)
        m = shard.cells_of_part(own, p, shape).reshape(shape)
        rows = np.nonzero(m.any(axis=(1, 2)))[0]
        assert rows.min() >= ix0 and rows.max() < ix1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import torch

        from kiwi_b200 import shard

        # every rank builds the same snapshot from the seed and derives the split on its own
        P = random_particles(400, 11, hmin=0.02, hmax=0.3)
        shape = (48, 40, 24)
        own = shard.tile_owners(shard.tile_entry_counts(P, (0, 2, 0, 2, 0, 2), shape, 2.0), world)
        mine = torch.tensor((own == rank).astype(np.int64))
        allm = [torch.zeros_like(mine) for _ in range(world)]
        dist.all_gather(allm, mine)
        ownt = torch.tensor(own)
        allo = [torch.zeros_like(ownt) for _ in range(world)]
        dist.all_gather(allo, ownt)
        ms, pairs = shard.reduce_step(10.0 + rank, 100.0 * (rank + 1))
        q.put((rank, [a.numpy() for a in allm], [a.numpy() for a in allo], ms, pairs))
    finally:
        dist.destroy_process_group()


def test_two_ranks_agree_on_the_split_gloo():
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, masks, owners, ms, pairs in out:
        assert np.array_equal(owners[0], owners[1])  # both ranks derived the same split
        cover = masks[0] + masks[1]
        assert np.all(cover == 1)  # disjoint and complete
        assert ms == 11.0 and pairs == 300.0  # max of the times, sum of the pairs


def test_part_particles_cover_the_part():
    """part_particles holds every particle whose support box reaches a cell of the part (brute force over
    the cells), in ascending order, and no particle that reaches none of its tiles."""
    P = random_particles(300, 21, hmin=0.02, hmax=0.25)
    bounds, shape, sup = (0, 2, 0, 2, 0, 2), (40, 24, 20), 2.0
    own = shard.tile_owners(shard.tile_entry_counts(P, bounds, shape, sup), 3)
    ntx, nty, ntz = shard.tile_grid(shape)
    d = [2.0 / s for s in shape]
    for part in range(3):
        idx = shard.part_particles(P, bounds, shape, sup, own, part)
        assert np.all(np.diff(idx) > 0)
        mine = (own == part).reshape(ntx, nty, ntz)
        want = []
        for i in range(len(P["x"])):
            r = sup * P["h"][i]
            lo = [max(int(np.floor((P[k][i] - r) / d[a])), 0) for a, k in enumerate("xyz")]
            hi = [min(int(np.floor((P[k][i] + r) / d[a])), shape[a] - 1) for a, k in enumerate("xyz")]
            if any(lo[a] > hi[a] for a in range(3)):
                continue
            if mine[lo[0] // 8:hi[0] // 8 + 1, lo[1] // 8:hi[1] // 8 + 1, lo[2] // 8:hi[2] // 8 + 1].any():
                want.append(i)
        assert np.array_equal(idx, np.array(want, dtype=idx.dtype))


def _rank_compute(rank, world, port, q):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import torch

        from kiwi_b200 import shard
        from oracle.oracle import Oracle

        # every rank builds the snapshot, derives the split, and maps only the particles that reach its
        # tiles (the oracle stands in for the per-part device call), then the cells are gathered on rank 0
        P = random_particles(500, 17, hmin=0.02, hmax=0.15)
        bounds, shape, sup = (0, 2, 0, 2, 0, 2), (40, 24, 16), 2.0
        own = shard.tile_owners(shard.tile_entry_counts(P, bounds, shape, sup), world)
        idx = shard.part_particles(P, bounds, shape, sup, own, rank)
        sub = {k: np.ascontiguousarray(v[idx]) for k, v in P.items()}
        dens, vx, vy, vz, raw, _ = Oracle().sph_to_grid(sub, bounds, shape)
        cells = shard.cells_of_part(own, rank, shape)
        mine = torch.tensor(np.stack([np.where(cells, a, 0.0) for a in (dens, vx, vy, vz, *raw.reshape(4, -1))]))
        parts = [torch.zeros_like(mine) for _ in range(world)]
        dist.all_gather(parts, mine)
        q.put((rank, len(idx), [t.numpy() for t in parts] if rank == 0 else None))
    finally:
        dist.destroy_process_group()


def test_two_ranks_map_their_parts_gloo(oracle):
    """Two gloo ranks each map the particles of their own part and keep their own cells; the assembled
    grid equals the whole snapshot's map bit for bit (densities and raw sums everywhere, velocities in
    every cell a particle reaches)."""
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_compute, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted([q.get(timeout=300) for _ in procs], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    P = random_particles(500, 17, hmin=0.02, hmax=0.15)
    dens, vx, vy, vz, raw, _ = oracle.sph_to_grid(P, (0, 2, 0, 2, 0, 2), (40, 24, 16))
    assert out[0][1] < 500 and out[1][1] < 500  # each rank maps a proper subset
    assembled = out[0][2][0] + out[0][2][1]  # the parts' cells are disjoint, zero elsewhere
    whole = np.stack([dens, vx, vy, vz, *raw.reshape(4, -1)])
    reached = raw.reshape(4, -1)[0] > 0
    for f in (0, 4, 5, 6, 7):
        assert np.array_equal(assembled[f], whole[f])
    for f in (1, 2, 3):
        assert np.array_equal(assembled[f][reached], whole[f][reached])


VOR_GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "vor_*.npz")))


def _vor_fixture(fn):
    d = np.load(fn)
    P = {k: d[k] for k in ("x", "y", "z", "vx", "vy", "vz", "m", "h")}
    geo = {k[4:]: d[k] for k in d.files if k.startswith("geo_")}
    k = int(d["kernel_index"])
    return d, P, geo, (k if k > 0 else -1), float(d["support_in_h"])


def test_voronoi_slabs_are_balanced_and_ordered():
    _, _, geo, _, _ = _vor_fixture(VOR_GOLDEN[0])
    start, end = shard._cell_vertex_rows(geo)
    v = geo["vxyz"].reshape(-1, 3)
    centre = np.array([(v[a:b, 0].min() + v[a:b, 0].max()) * 0.5 for a, b in zip(start, end)])
    for n in (2, 3, 5):
        own = shard.voronoi_cell_owners(geo, n)
        counts = np.bincount(own, minlength=n)
        assert counts.max() - counts.min() <= 1
        for p in range(n - 1):
            assert centre[own == p].max() <= centre[own == p + 1].min() + 1e-12


def _check_voronoi_slabs(oracle, P, home, geo, k, sup, parts=(2, 3)):
    """Each slab's particles, mapped on their own (the oracle, the reference's algorithm), give the slab's
    cells bit for bit as the whole snapshot gives them (raw sums and densities everywhere, velocities where
    a particle reaches the cell).  Returns the slabs' particle counts."""
    whole = oracle.map_voronoi(P, home, geo, kernel=k, support_in_h=sup)
    sizes = []
    for n in parts:
        own = shard.voronoi_cell_owners(geo, n)
        for p in range(n):
            idx = shard.voronoi_part_particles(P, home, geo, own, p, sup)
            sizes.append(len(idx))
            part = oracle.map_voronoi({q: v[idx] for q, v in P.items()}, home[idx], geo, kernel=k, support_in_h=sup)
            cells = own == p
            assert np.array_equal(part[4][:, cells], whole[4][:, cells]), (n, p)
            assert np.array_equal(part[0][cells], whole[0][cells]), (n, p)
            reached = cells & (whole[4][0] > 0)
            for i in (1, 2, 3):
                assert np.array_equal(part[i][reached], whole[i][reached]), (n, p, i)
    return sizes


@pytest.mark.parametrize("fn", VOR_GOLDEN, ids=[os.path.basename(f)[4:-4] for f in VOR_GOLDEN])
def test_voronoi_part_particles_reproduce_their_cells(oracle, fn):
    d, P, geo, k, sup = _vor_fixture(fn)
    _check_voronoi_slabs(oracle, P, d["home"], geo, k, sup)


def test_voronoi_slab_particles_on_a_larger_tessellation(oracle, reflib):
    """2,000 particles with small supports on the reference's own Voro++ tessellation: every slab maps a
    proper subset of the particles and its cells come out bit for bit."""
    P = random_particles(2000, 23, hmin=0.02, hmax=0.06)
    geo, _ = reflib.voronoi(P, (0, 2, 0, 2, 0, 2), run_map=False)
    sizes = _check_voronoi_slabs(oracle, P, geo["home"], geo, -1, 2.0, parts=(2, 4))
    assert max(sizes) < 2000 and min(sizes) > 0


def test_snapshot_work_is_the_bounding_box_pair_count(oracle):
    """shard.snapshot_work and kiwi_snapshot_work (C ABI, host only) both equal the oracle's bounding-box
    pair count."""
    import ctypes as C

    import kiwi_b200 as kb

    lib = C.CDLL(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "kiwi_b200",
                              "libkiwi_b200.so"))
    lib.kiwi_snapshot_work.argtypes = [C.c_void_p, C.POINTER(kb.KiwiParticles), C.POINTER(kb.KiwiCartGrid),
                                       C.POINTER(kb.KiwiKernelSel), C.POINTER(C.c_int64)]
    dp = C.POINTER(C.c_double)
    for seed in (3, 4, 5):
        P = random_particles(200, seed, hmin=0.02, hmax=0.3)
        if seed == 5:
            P["x"][:50] += 3.0  # outside the domain
        b, shape = (0, 2, 0, 2, 0, 2), (20, 12, 9)
        st = oracle.sph_to_grid(P, b, shape)[5]
        assert shard.snapshot_work(P, b, shape, 2.0) == st.bbox_pairs
        arrs = {k: np.ascontiguousarray(P[k], dtype=np.float64) for k in ("x", "y", "z", "vx", "vy", "vz", "m", "h")}
        parts = kb.KiwiParticles(200, *[arrs[k].ctypes.data_as(dp) for k in ("x", "y", "z", "vx", "vy", "vz", "m", "h")])
        grid = kb.KiwiCartGrid((C.c_double * 6)(*b), *shape)
        w = C.c_int64(-1)
        assert lib.kiwi_snapshot_work(None, C.byref(parts), C.byref(grid), C.byref(kb.KiwiKernelSel(0, 0.0, 0, 0)),
                                      C.byref(w)) == 0
        assert w.value == st.bbox_pairs


def test_snapshots_dealt_longest_first():
    rng = np.random.default_rng(5)
    work = rng.integers(1, 10_000, 64) ** 2
    for n in (1, 2, 3, 8):
        parts = shard.assign_snapshots_lpt(work, n)
        allp = np.concatenate(parts)
        assert np.array_equal(np.sort(allp), np.arange(64))  # disjoint and complete
        loads = [int(work[q].sum()) for q in parts]
        assert max(loads) <= work.sum() / n + work.max()  # the greedy bound
        again = shard.assign_snapshots_lpt(work.copy(), n)  # deterministic: every rank derives the same
        assert all(np.array_equal(a, b) for a, b in zip(parts, again))


def _rank_voronoi(rank, world, port, fn, q):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import torch

        from oracle.oracle import Oracle

        # every rank loads the tessellation, derives the slabs, and maps only the particles that can reach
        # its own slab (the oracle standing in for the device call); the slabs' raw sums go to rank 0
        d, P, geo, k, sup = _vor_fixture(fn)
        own = shard.voronoi_cell_owners(geo, world)
        idx = shard.voronoi_part_particles(P, d["home"], geo, own, rank, sup)
        raw = Oracle().map_voronoi({q_: v[idx] for q_, v in P.items()}, d["home"][idx], geo, kernel=k,
                                   support_in_h=sup)[4]
        mine = torch.tensor(np.where(own == rank, raw, 0.0))
        parts = [torch.zeros_like(mine) for _ in range(world)]
        dist.all_gather(parts, mine)
        q.put((rank, [t.numpy() for t in parts] if rank == 0 else None))
    finally:
        dist.destroy_process_group()


def test_two_ranks_map_their_voronoi_slabs_gloo(oracle):
    """Two gloo ranks each map their slab's particles; the gathered raw sums equal the whole map's bit for
    bit."""
    import multiprocessing as mp

    fn = VOR_GOLDEN[0]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_voronoi, args=(r, 2, port, fn, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted([q.get(timeout=300) for _ in procs], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    d, P, geo, k, sup = _vor_fixture(fn)
    whole = oracle.map_voronoi(P, d["home"], geo, kernel=k, support_in_h=sup)[4]
    assert np.array_equal(out[0][1][0] + out[0][1][1], whole)


def test_c_abi_part_rows_match_the_host_rule():
    """kiwi_part_rows (host only, no GPU) gives the rows of shard.part_rows: the C ABI's restatement of the
    split for C and C++ callers, on random, clustered and out-of-domain particles and several kernels."""
    import ctypes as C

    import kiwi_b200 as kb

    lib = C.CDLL(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "kiwi_b200",
                              "libkiwi_b200.so"))
    lib.kiwi_part_rows.argtypes = [C.c_void_p, C.POINTER(kb.KiwiParticles), C.POINTER(kb.KiwiCartGrid),
                                   C.POINTER(kb.KiwiKernelSel), C.c_int, C.c_int, C.POINTER(C.c_int),
                                   C.POINTER(C.c_int)]
    rng = np.random.default_rng(9)
    dp = C.POINTER(C.c_double)
    for case in range(12):
        n = int(rng.integers(0, 3000))
        P = random_particles(n, 40 + case, hmin=0.01, hmax=0.4)
        if case % 3 == 1:  # clustered
            for k in "xyz":
                P[k] = 1.0 + 0.1 * rng.standard_normal(n)
        if case % 3 == 2 and n:  # some outside the domain, some with h <= 0
            P["x"][: n // 5] += 5.0
            P["h"][n // 5: n // 4] = 0.0
        shape = tuple(int(v) for v in rng.integers(5, 70, 3))
        b = (0.0, 2.0, -0.3, 2.1, 0.1, 1.7)
        kernel, sup = [(0, 2.0), (4, 2.0), (2, 0.0)][case % 3]
        sup_h = sup or kb.get_kernel("quintic_spline").radkern
        arrs = {k: np.ascontiguousarray(P[k], dtype=np.float64) for k in ("x", "y", "z", "vx", "vy", "vz", "m", "h")}
        parts = kb.KiwiParticles(n, *[arrs[k].ctypes.data_as(dp) for k in ("x", "y", "z", "vx", "vy", "vz", "m", "h")])
        grid = kb.KiwiCartGrid((C.c_double * 6)(*b), *shape)
        sel = kb.KiwiKernelSel(kernel, sup, 0, 0)
        for n_parts in (1, 2, 3, 7):
            own = shard.tile_owners(shard.tile_entry_counts(arrs, b, shape, sup_h), n_parts)
            for p in range(n_parts):
                a0, a1 = C.c_int(-1), C.c_int(-1)
                assert lib.kiwi_part_rows(None, C.byref(parts), C.byref(grid), C.byref(sel), p, n_parts,
                                          C.byref(a0), C.byref(a1)) == 0
                assert (a0.value, a1.value) == shard.part_rows(own, p, shape), (case, n_parts, p)
    a0, a1 = C.c_int(), C.c_int()
    assert lib.kiwi_part_rows(None, C.byref(parts), C.byref(grid), C.byref(sel), 3, 3, C.byref(a0), C.byref(a1)) < 0


def test_c_abi_voronoi_slabs_match_the_host_rule(reflib):
    """kiwi_voronoi_cell_owners and kiwi_voronoi_part_particles (host only, no GPU) give the owners and
    particle sets of shard.voronoi_cell_owners / voronoi_part_particles, on every axis and several part
    counts, on the Voronoi fixtures and on a 2,000-particle Voro++ tessellation."""
    import ctypes as C

    import kiwi_b200 as kb

    lib = C.CDLL(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "kiwi_b200",
                              "libkiwi_b200.so"))
    i32p, i64p, dp = C.POINTER(C.c_int32), C.POINTER(C.c_int64), C.POINTER(C.c_double)
    lib.kiwi_voronoi_cell_owners.argtypes = [C.c_void_p, C.POINTER(kb.KiwiVoronoiCells), C.c_int, C.c_int, i32p]
    lib.kiwi_voronoi_part_particles.argtypes = [C.c_void_p, C.POINTER(kb.KiwiParticles), i32p,
                                                C.POINTER(kb.KiwiVoronoiCells), C.POINTER(kb.KiwiKernelSel), i32p,
                                                C.c_int, C.POINTER(C.c_uint8), i64p]
    cases = []
    for fn in VOR_GOLDEN:
        d, P, geo, _, sup = _vor_fixture(fn)
        cases.append((P, d["home"], geo, int(d["kernel_index"]), sup))
    P = random_particles(2000, 23, hmin=0.02, hmax=0.06)
    g, _ = reflib.voronoi(P, (0, 2, 0, 2, 0, 2), run_map=False)
    cases.append((P, g["home"], g, 0, 2.0))
    for P, home, geo, kernel, sup in cases:
        fo = np.ascontiguousarray(geo["face_off"], dtype=np.int64)
        vo = np.ascontiguousarray(geo["vert_off"], dtype=np.int64)
        vx = np.ascontiguousarray(geo["vxyz"], dtype=np.float64).reshape(-1)
        nb = np.ascontiguousarray(geo["face_nbr"], dtype=np.int32)
        vol = np.ascontiguousarray(geo["volume"], dtype=np.float64)
        cells = kb.KiwiVoronoiCells(len(vol), fo.ctypes.data_as(i64p), vo.ctypes.data_as(i64p), vx.ctypes.data_as(dp),
                                    nb.ctypes.data_as(i32p), vol.ctypes.data_as(dp))
        arrs = {k: np.ascontiguousarray(P[k], dtype=np.float64) for k in ("x", "y", "z", "vx", "vy", "vz", "m", "h")}
        parts = kb.KiwiParticles(len(arrs["x"]), *[arrs[k].ctypes.data_as(dp)
                                                   for k in ("x", "y", "z", "vx", "vy", "vz", "m", "h")])
        hm = np.ascontiguousarray(home, dtype=np.int32)
        sel = kb.KiwiKernelSel(kernel, 0.0, 0, 0)
        for axis in (0, 1, 2):
            for n in (1, 2, 3, 5):
                own_c = np.zeros(len(vol), dtype=np.int32)
                assert lib.kiwi_voronoi_cell_owners(None, C.byref(cells), n, axis, own_c.ctypes.data_as(i32p)) == 0
                own = shard.voronoi_cell_owners(geo, n, axis=axis)
                assert np.array_equal(own_c, own), (axis, n)
                for p in range(n):
                    s = np.zeros(len(arrs["x"]), dtype=np.uint8)
                    cnt = C.c_int64(-1)
                    assert lib.kiwi_voronoi_part_particles(None, C.byref(parts), hm.ctypes.data_as(i32p),
                                                           C.byref(cells), C.byref(sel), own_c.ctypes.data_as(i32p),
                                                           p, s.ctypes.data_as(C.POINTER(C.c_uint8)),
                                                           C.byref(cnt)) == 0
                    want = shard.voronoi_part_particles(P, home, geo, own, p, sup)
                    assert np.array_equal(np.nonzero(s)[0], want) and cnt.value == len(want), (axis, n, p)


def test_voronoi_split_edge_cases(oracle):
    """More parts than cells (some parts own none and map no particle), a snapshot without particles, and
    particles with h <= 0 or no home cell: the parts still reproduce the whole map."""
    d, P, geo, k, sup = _vor_fixture(VOR_GOLDEN[0])
    nc = len(geo["volume"])
    own = shard.voronoi_cell_owners(geo, nc + 3)
    assert np.bincount(own, minlength=nc + 3).max() == 1  # at most one cell per part
    empty = [p for p in range(nc + 3) if not np.any(own == p)]
    assert len(empty) == 3
    for p in empty:
        assert len(shard.voronoi_part_particles(P, d["home"], geo, own, p, sup)) == 0
    P0 = {q: v[:0] for q, v in P.items()}
    assert len(shard.voronoi_part_particles(P0, d["home"][:0], geo, shard.voronoi_cell_owners(geo, 2), 0, sup)) == 0
    home = d["home"].copy()
    home[:10] = -1
    P2 = {q: v.copy() for q, v in P.items()}
    P2["h"][10:20] = 0.0
    whole = oracle.map_voronoi(P2, home, geo, kernel=k, support_in_h=sup)[4]
    own = shard.voronoi_cell_owners(geo, 3, axis=2)
    for p in range(3):
        idx = shard.voronoi_part_particles(P2, home, geo, own, p, sup)
        part = oracle.map_voronoi({q: v[idx] for q, v in P2.items()}, home[idx], geo, kernel=k, support_in_h=sup)[4]
        assert np.array_equal(part[:, own == p], whole[:, own == p]), p
