"""Host side of splitting one grid over several GPUs (kiwi_b200.shard): the tile entry counts, the
ownership rule, and the multi-rank agreement and timing reduction over gloo with two ranks on the CPU."""
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
