#!/usr/bin/env python3
"""Benchmark of the kernel-integral mapping hot path (sph-to-grid) on B200.

Metric: particle-cell integrals per second -- a pair is one (particle, cell) pair whose cell's closest
point lies within the particle's support radius (the cells that can receive mass); the bounding-box
pair count the reference evaluates is reported beside it.

Workload (one GPU): the 2,000,000-particle log-normal cube (sigma_ln rho = 1.5, P(k) ~ k^-4, 10 pc,
domain padded by max 2h) on a 256^3 grid, cubic spline (M4) -- seeded synthetic input.  With N GPUs
(torchrun, one process per GPU) the ranks split that one grid (--multi tiles, the default: each rank
computes the cell tiles of its part, kiwi_sph_to_grid_device_part, a weight-balanced run of x rows; strong
scaling, no data-path collective) or each maps its own independently seeded snapshot of the same size
(--multi replicas: weak scaling).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|fp32_mixed] [--impl reference]

One JSON line is printed by rank 0.  `value` is timed with CUDA events on the engine's stream with the
inputs resident in HBM; `e2e` is the same metric through the public host API (pinned host arrays in,
host arrays out, copies inside the timed region).  `cpu_baseline` / --impl reference time the
reference's own OpenMP pair-integral loop (built from its sources into oracle/_ref) on a bounded particle
sample of the same workload on this machine's host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# Algorithmic work of one evaluated (particle, cell) pair in the reference's evaluation order, measured
# with the operation-counting oracle (`python oracle/count_work.py --workload lognormal --sample 60`):
# per support pair (the cells the support reaches, evaluated by default) 10,166 flops (+ - * / sqrt) and
# 481.9 transcendentals (sin cos acos atan atanh log pow); per bounding-box pair (every cell of the box,
# --full-box) 9,143 flops and 435.6 transcendentals.  Roofline convention: one FP64 transcendental =
# 20 flop-equivalents.
TRANS_FLOPS = 20.0
WORK_PER_SUPPORT_PAIR = 10166.4 + TRANS_FLOPS * 481.9
WORK_PER_BBOX_PAIR = 9142.7 + TRANS_FLOPS * 435.6
# The lattice-factorised kernel's own work items (orc_edge_cost / orc_lattice_vertex_cost of the counting
# oracle, averaged over 3,000 random inputs per class): an edge tier beyond 2h 37 flops; between h and 2h
# 127 flops + 6 transcendentals; within h 209 flops + 12; a vertex pyramid 121 flops + 4; the assembly of
# one cell from 24 corner values ~60 flops.
EDGE_OUTER = 37.0
EDGE_MIDDLE = 127.0 + TRANS_FLOPS * 6
EDGE_INNER = 209.0 + TRANS_FLOPS * 12
VERTEX_PYRAMID = 121.0 + TRANS_FLOPS * 4
CELL_ASSEMBLY = 60.0

# DRAM bytes (read + write) of one k_cart_lattice launch on the default workload (2 M particles, 256^3) from
# a one-pass ncu capture, and the commit whose kernel was captured.
LATTICE_TRAFFIC = {"bytes": 948.439296e6 + 511.081984e6, "commit": "9c39bf1", "kernel": "k_cart_lattice"}

L2_BYTES = 126 * 1024 * 1024
# the tabulated integral: one trilinear lookup reads 8 table entries
TAB_BYTES_PER_LOOKUP = 64.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="kiwi", choices=["kiwi", "reference"])
    ap.add_argument("--precision", default="fp64",
                    choices=["fp64", "fp32_mixed", "fp32_mixed_guaranteed", "fp64_reference_order"])
    ap.add_argument("--full-box", action="store_true",
                    help="evaluate every cell of each support bounding box, as the reference does")
    ap.add_argument("--n", type=int, default=2_000_000)
    ap.add_argument("--res", type=int, default=256)
    ap.add_argument("--kernel", default="cubic_spline")
    ap.add_argument("--tabulated", action="store_true",
                    help="the cubic spline's tabulated integral (lookups in the GPU-generated canonical table) "
                         "instead of its closed form; every cell of each support bounding box, as the reference")
    ap.add_argument("--seed", type=int, default=1002)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip parity_c1: the 7,300-particle column on the GPU and through the reference's stage "
                         "(~3 min of host CPU)")
    ap.add_argument("--no-fp32-compare", action="store_true",
                    help="with --precision fp64: skip timing the FP32-mixed form beside it")
    ap.add_argument("--multi", default="tiles", choices=["tiles", "replicas"],
                    help="with N > 1 GPUs: split one grid by cell tiles (strong scaling) or map one snapshot per "
                         "rank (weak scaling)")
    ap.add_argument("--fd-particles", type=int, default=200, help="adjoint workload: particles checked by FD")
    ap.add_argument("--adj-n", type=int, default=500_000, help="adjoint workload: particles")
    ap.add_argument("--adj-res", type=int, default=128, help="adjoint workload: grid cells per axis")
    ap.add_argument("--vor-n", type=int, default=200_000, help="voronoi workload: particles")
    ap.add_argument("--cmap-n", type=int, default=1_000_000, help="cartesian_map workload: sites")
    ap.add_argument("--cmap-res", type=int, default=256, help="cartesian_map workload: grid cells per axis")
    ap.add_argument("--lloyd-n", type=int, default=1_000_000, help="lloyd workload: particles")
    ap.add_argument("--workload", default="lognormal",
                    choices=["lognormal", "batch", "adjoint", "voronoi", "cartesian_map", "lloyd"],
                    help="batch: many column snapshots of log-uniform sizes on grids of log-uniform resolution, "
                         "kernels cycling M4 / M6 / WC4, in one persistent graph-recorded launch")
    ap.add_argument("--batch-items", type=int, default=64)
    ap.add_argument("--batch-nmin", type=int, default=10_000)
    ap.add_argument("--batch-nmax", type=int, default=2_000_000)
    ap.add_argument("--batch-resmin", type=int, default=64)
    ap.add_argument("--batch-resmax", type=int, default=256)
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def hbm_peak_gbs():
    """HBM copy bandwidth for the roofline: MEASURED_PEAKS.json's hbm_gbs (measured on this pool's B200s),
    else the pool's earlier measurement of 6.65 TB/s, marked as the fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (of measured)"
    except (OSError, ValueError, KeyError):
        return 6650.0, "fallback 6.65 TB/s (MEASURED_PEAKS.json absent; of fallback)"


def _standalone(name, relpath):
    """Loads one pure-Python file of the package by path, without importing the package itself (so that the
    reference arm maps no kiwi_b200 shared library into its process)."""
    import importlib.util

    spec = importlib.util.spec_from_file_location(name, os.path.join(ROOT, relpath))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def kernel_hfact(kernel_name):
    """hfact of a kernel, from the kernel-table generator's definitions (pure Python)."""
    gen = _standalone("kiwi_kernel_table_gen", "kiwi_b200/tables/gen_kernel_tables.py")
    for K in gen.KERNELS:
        if kernel_name in (K.key, K.key.lower(), K.name.lower().replace(" ", "_")):
            return K.hfact
    raise ValueError(f"unknown kernel {kernel_name!r}")


def make_workload(n, res, seed, kernel_name):
    wl = _standalone("kiwi_workloads", "kiwi_b200/workloads.py")
    P, bounds = wl.lognormal_cube(n=n, seed=seed, mesh=min(res, 256), hfact=kernel_hfact(kernel_name))
    return P, bounds, (res, res, res)


def workload_config(args, nc=None, ws=1, split=False):
    """The `config` object of the sph-to-grid line, shared by both arms."""
    cfg = {"workload": f"lognormal_cube n={args.n} sigma_ln=1.5 P(k)~k^-4 10pc padded, grid {args.res}^3, "
                       f"kernel {args.kernel}" + (", tabulated integral" if args.tabulated else ""),
           "precision": args.precision, "particles_per_gpu": args.n, "cells": nc or args.res ** 3,
           "l2": "flushed between timed steps (256 MB write) and inputs+outputs > L2",
           "parallelism": (f"cell-tile parts x{ws} of one grid" if split else f"replicas x{ws}")
           if ws > 1 else "single GPU"}
    return cfg


# The reference's pair loop runs OpenMP schedule(dynamic, 256) over particles; a sample step gives every
# thread this many 256-particle chunks, so that the idle tail of the last chunks stays a small part of it.
REF_CHUNKS_PER_THREAD = 6


def ref_sample(P, bounds, shape, kernel_name, ref, threads, steps, warmup):
    """The reference's own OpenMP pair loop (oracle/_ref: its KernelIntegrator::face over the six box faces
    of every bounding-box cell, schedule(dynamic, 256), per-cell sums into a scalar instead of the grid) on
    consecutive ranges of a seeded permutation of the workload's particles: `warmup` untimed ranges of one
    chunk per thread, then `steps` timed ranges of REF_CHUNKS_PER_THREAD chunks per thread.
    Returns (seconds, bbox pairs, support pairs, particles per step) summed over the timed ranges."""
    n = len(P["x"])
    perm = np.random.default_rng(99).permutation(n)
    Ps = {k: np.ascontiguousarray(v[perm]) for k, v in P.items()}
    pos = 0
    for _ in range(warmup):
        m = min(256 * threads, n - pos)
        ref.pair_sample(Ps, bounds, shape, kernel=kernel_name, threads=threads, p_range=(pos, pos + m))
        pos = (pos + m) % n
    per_step = min(n, REF_CHUNKS_PER_THREAD * 256 * threads)
    tt, bb, ss = 0.0, 0, 0
    for _ in range(steps):
        if pos + per_step > n:
            pos = 0
        t, b, s, _ = ref.pair_sample(Ps, bounds, shape, kernel=kernel_name, threads=threads,
                                     p_range=(pos, pos + per_step))
        pos += per_step
        tt, bb, ss = tt + t, bb + b, ss + s
    return tt, bb, ss, per_step


def cpu_baseline(P, bounds, shape, kernel_name):
    """One step of the reference arm (below) timed on this machine's host cores: the reported CPU baseline."""
    from oracle.oracle import load_ref

    ref = load_ref()
    if ref is None:
        return None
    threads = ref.max_threads()
    t, b, s, per = ref_sample(P, bounds, shape, kernel_name, ref, threads, steps=1, warmup=1)
    return {"value": s / t, "unit": "pair-integrals/s", "cores": threads, "kind": "reference",
            "sample": f"{per} of {len(P['x'])} particles (seeded permutation; {REF_CHUNKS_PER_THREAD} chunks of 256 "
                      f"per thread), {b} bounding-box / {s} support pairs, {t:.1f} s wall on {threads} OpenMP "
                      f"threads; the reference's KernelIntegrator::face over each cell's six box faces",
            "bbox_pairs_per_s": b / t}


def cpu_baseline_c1(kiwi_b200, ctx):
    """The 7,300-particle column on its 100 x 100 x 410 grid of 0.02 pc cells (the workload small enough for
    the reference's own stage) mapped twice: on the GPU through the public host API (host arrays in and out), and by the
    reference's own run_sph_to_grid_stage (oracle/_ref) on all host cores -- its stage wall time is the CPU
    baseline of this workload, and its grid is compared with the GPU's, cell by cell per density band
    (parity_c1)."""
    from oracle.compare import band_stats, exact_check
    from oracle.oracle import load_ref, load_truth

    ref = load_ref()
    if ref is None:
        return None
    wl = _standalone("kiwi_workloads", "kiwi_b200/workloads.py")
    P, b = wl.column_snapshot()
    shape = (100, 100, 410)
    kiwi_b200.sph_to_grid(P, b, shape, ctx=ctx)  # warm-up
    t0 = time.perf_counter()
    r = kiwi_b200.sph_to_grid(P, b, shape, ctx=ctx)
    gpu_s = time.perf_counter() - t0
    threads = ref.max_threads()
    t0 = time.perf_counter()
    rd = ref.sph_to_grid(P, b, shape, threads=threads)
    ref_s = time.perf_counter() - t0
    sig = rd[0] > 1e-6 * rd[0].max()
    dv = max(float(np.max(np.abs(getattr(r, k)[sig] - v[sig]))) for k, v in zip(("vx", "vy", "vz"), rd[1:]))
    pairs, bbox = r.stats["sphere_pairs"], r.stats["bbox_pairs"]
    exact = exact_check(P, b, shape, (r.density, r.vx, r.vy, r.vz), rd, load_truth())
    return {"workload": "column n=7300 (60% uniform + 40% filament, h from 57-NN), grid 100x100x410 of 0.02 pc",
            "support_pairs": int(pairs), "bbox_pairs": int(bbox),
            "gpu_e2e_s": gpu_s, "gpu_e2e_pairs_per_s": pairs / gpu_s,
            "reference_stage_s": ref_s, "reference_stage_pairs_per_s": pairs / ref_s, "reference_cores": threads,
            "against": "the reference's run_sph_to_grid_stage (oracle/_ref) on the same particles, every cell",
            "density_bands": band_stats(r.density, rd[0]),
            "max_abs_velocity_diff_above_1e-6_peak_km_s": dv,
            "total_mass_rel_diff": float(abs(r.density.sum() - rd[0].sum()) / rd[0].sum()),
            "vs_exact": {"how": "__float128 evaluation of the reference's algorithm, each cell alone over the "
                                "particles covering it; relative density error of the GPU and of the reference",
                         **exact}}


def run_reference(args):
    """The reference arm: the reference's own CPU implementation of the path (oracle/_ref, built from its
    sources) on the host cores, for the same workload, metric and unit as the GPU arm.  Imports nothing of
    the kiwi_b200 package: the workload generator and the kernel's hfact are loaded as plain files."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    from oracle.oracle import load_ref

    ref = load_ref()
    if ref is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libkiwi_ref.so was not built"}))
        return 0
    P, bounds, shape = make_workload(args.n, args.res, args.seed, args.kernel)
    threads = ref.max_threads()
    tt, bb, ss, per_step = ref_sample(P, bounds, shape, args.kernel, ref, threads, args.steps, args.warmup)
    value = ss / tt
    sample = (f"{per_step} of {args.n} particles per step (consecutive ranges of a seeded permutation, "
              f"{REF_CHUNKS_PER_THREAD} chunks of 256 per thread); {bb} bounding-box / {ss} support pairs over "
              f"{args.steps} steps; the reference's KernelIntegrator::face over each cell's six box faces in its "
              f"OpenMP schedule(dynamic, 256) particle loop, per-cell sums into a scalar instead of the grid")
    line = {"metric": "particle-cell integrals/s (support pairs), sph-to-grid", "value": value,
            "unit": "pair-integrals/s", "impl": "reference", "n_gpus": 0, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * tt / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(args),
            "cpu_baseline": {"value": value, "unit": "pair-integrals/s", "cores": threads, "kind": "reference",
                             "sample": sample},
            "pairs": {"bbox_pairs_per_s": bb / tt, "sample_particles_per_step": per_step},
            "e2e": {"value": value, "unit": "pair-integrals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_adjoint(args):
    """Differentiable sph-to-grid: 500,000 column-recipe particles (60 % uniform, 40 % filament) in a 4 pc
    cube (seed 1004), 128^3 grid, loss L = sum_xy (sum_z rho dz - T_xy)^2 with T the projected density of
    the seed-2004 realisation.  Times the forward pass (FP32-mixed and FP64) and the adjoint, and checks
    dL/d(x, y, z, h, m) of --fd-particles random particles against central differences (step 1e-6 max(|t|, h))
    of the particle's own contribution through the FP64 forward pass (the loss is linear in each particle's
    raw sums at fixed residual, so this is the exact dL/dtheta)."""
    import torch

    import kiwi_b200
    from kiwi_b200.workloads import column_snapshot

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    n, res, box = args.adj_n, args.adj_res, (4.0, 4.0, 4.0)
    P, bounds = column_snapshot(n=n, seed=1004, box=box)
    Tp, _ = column_snapshot(n=n, seed=2004, box=box)
    shape = (res, res, res)
    nc = res ** 3
    dz = box[2] / res
    vol = (box[0] / res) * (box[1] / res) * dz
    ctx = kiwi_b200.Context(0)
    keys = ("x", "y", "z", "vx", "vy", "vz", "m", "h")
    dP = {k: torch.from_numpy(P[k]).to(dev) for k in keys}
    dT = {k: torch.from_numpy(Tp[k]).to(dev) for k in keys}
    outT = {"density": torch.empty(nc, dtype=torch.float64, device=dev)}
    kiwi_b200.sph_to_grid_device(dT, bounds, shape, outT, ctx=ctx)
    T = outT["density"].view(res, res, res).sum(dim=2) * dz
    raw = torch.empty(4 * nc, dtype=torch.float64, device=dev)
    times = {}
    for prec in ("fp32_mixed", "fp64"):
        for _ in range(2):
            kiwi_b200.sph_to_grid_device(dP, bounds, shape, {"raw4": raw}, precision=prec, ctx=ctx)
        ms, pairs = 0.0, 0
        for _ in range(args.steps):
            st = kiwi_b200.sph_to_grid_device(dP, bounds, shape, {"raw4": raw}, precision=prec, ctx=ctx)
            ms += st["total_ms"]
            pairs += st["sphere_pairs"]
        times[prec] = (ms / args.steps, pairs / args.steps)
    # cotangent of the raw sums: dL/dM = dL/drho / V, with dL/drho_xyz = 2 (proj_xy - T_xy) dz
    M = raw.view(4, res, res, res)[0]
    resid = (M / vol).sum(dim=2) * dz - T
    loss = float((resid ** 2).sum())
    cot = torch.zeros(4, res, res, res, dtype=torch.float64, device=dev)
    cot[0] = (2.0 * resid * dz / vol)[:, :, None].expand(res, res, res)
    cot = cot.reshape(-1).contiguous()
    grads = {k: torch.empty(n, dtype=torch.float64, device=dev) for k in ("x", "y", "z", "h", "m", "vx", "vy", "vz")}
    for _ in range(max(args.warmup, 1)):
        st = kiwi_b200.sph_to_grid_adjoint_device(dP, bounds, shape, cot, grads, ctx=ctx)
    ms_adj = 0.0
    for _ in range(args.steps):
        st = kiwi_b200.sph_to_grid_adjoint_device(dP, bounds, shape, cot, grads, ctx=ctx)
        ms_adj += st["total_ms"]
    ms_adj /= args.steps
    adj_pairs = st["evaluated_pairs"]
    g = {k: v.cpu().numpy() for k, v in grads.items()}

    # FD of each sampled particle's own contribution (one-particle forward passes, FP64)
    rng = np.random.default_rng(7)
    worst = 0.0
    one = {k: torch.empty(1, dtype=torch.float64, device=dev) for k in keys}
    raw1 = torch.empty(4 * nc, dtype=torch.float64, device=dev)

    def contrib(vals):
        for k in keys:
            one[k].fill_(float(vals[k]))
        kiwi_b200.sph_to_grid_device(one, bounds, shape, {"raw4": raw1}, ctx=ctx)
        return float(torch.dot(raw1, cot))

    for i in rng.choice(n, args.fd_particles, replace=False):
        base = {k: float(P[k][i]) for k in keys}
        fd = {}
        for k in ("x", "y", "z", "h", "m"):
            d = 1e-6 * max(abs(base[k]), base["h"])
            a, b = dict(base), dict(base)
            a[k] += d
            b[k] -= d
            fd[k] = (contrib(a) - contrib(b)) / (2 * d)
        scale = max(abs(fd[k]) for k in ("x", "y", "z", "h"))
        if scale > 0:
            worst = max(worst, max(abs(g[k][i] - fd[k]) for k in ("x", "y", "z", "h")) / scale)
        if abs(fd["m"]) > 0:
            worst = max(worst, abs(g["m"][i] - fd["m"]) / abs(fd["m"]))
    line = {
        "metric": "adjoint particle-cell pairs/s (support pairs), differentiable sph-to-grid",
        "value": adj_pairs / (ms_adj * 1e-3), "unit": "pair-integrals/s", "n_gpus": 1, "steps": args.steps,
        "warmup": max(args.warmup, 1), "ms_per_step": ms_adj, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 (forward-mode derivatives)", "data": "synthetic",
        "config": {"workload": f"{n} column-recipe particles in a 4 pc cube (seed 1004), grid {res}^3, "
                               "L = sum_xy (sum_z rho dz - T_xy)^2, T from the seed-2004 realisation"},
        "forward_ms": {k: v[0] for k, v in times.items()},
        "forward_pairs_per_s": {k: v[1] / (v[0] * 1e-3) for k, v in times.items()},
        "loss": loss, "fd_particles": args.fd_particles, "fd_max_rel_err": worst,
        "fd_recipe": "central, step 1e-6 max(|theta|, h), per particle through one-particle FP64 forward passes",
    }
    print(json.dumps(line), flush=True)
    return 0


def run_voronoi(args):
    """Voronoi-cell map: --vor-n column-recipe particles on a 5 pc cube (filament through the centre, seed
    1003), coverage_grid buffer points (spacing 0.05 x 5 pc) and one Lloyd iteration; the tessellation is
    built on the host by the reference's own point-set stage and Voro++ (oracle/_ref, as the reference
    keeps it on the host), which also runs the reference's OpenMP mapping loop as the CPU baseline.  The
    GPU map is timed through kiwi_map_voronoi (geometry and particles staged from host arrays)."""
    import torch

    import kiwi_b200
    from kiwi_b200.workloads import column_snapshot
    from oracle.oracle import load_ref

    ref = load_ref()
    if ref is None:
        print(json.dumps({"workload": "voronoi", "unavailable": "oracle/_ref (the reference library) is not built"}))
        return 0
    torch.cuda.set_device(0)
    P, bounds = column_snapshot(n=args.vor_n, seed=1003, box=(5.0, 5.0, 5.0))
    threads = ref.max_threads()
    t0 = time.perf_counter()
    geo, _ = ref.voronoi(P, bounds, buffer=True, spacing_fraction=0.05, lloyd=1, threads=threads, run_map=False)
    t_geo = time.perf_counter() - t0
    geo2, ref_res, t_ref_map = geo, None, None
    if not args.no_cpu_baseline:  # the reference's own map (its geometry is built again, then mapped)
        t0 = time.perf_counter()
        geo2, ref_res = ref.voronoi(P, bounds, buffer=True, spacing_fraction=0.05, lloyd=1, threads=threads,
                                    run_map=True)
        t_ref_map = max(time.perf_counter() - t0 - t_geo, 1e-9)
    cells = {k: geo2[k] for k in ("face_off", "vert_off", "vxyz", "face_nbr", "volume")}
    ctx = kiwi_b200.Context(0)
    for _ in range(max(args.warmup, 1)):
        r = kiwi_b200.map_voronoi(P, geo2["home"], cells, ctx=ctx)  # warm-up
    g_ms, t_ms = [], []
    for _ in range(args.steps):
        r = kiwi_b200.map_voronoi(P, geo2["home"], cells, ctx=ctx)
        g_ms.append(r.stats["gather_ms"])
        t_ms.append(r.stats["total_ms"])
    pairs = r.stats["evaluated_pairs"]
    # the same map with the particles and the tessellation already resident on the GPU (staged once)
    dev = torch.device("cuda", 0)
    dP = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in P.items()}
    dgeo = {k: torch.from_numpy(np.ascontiguousarray(geo2[k]).reshape(-1)).to(dev)
            for k in ("face_off", "vert_off", "vxyz", "face_nbr", "volume")}
    dhome = torch.from_numpy(np.ascontiguousarray(geo2["home"], dtype=np.int32)).to(dev)
    ncv = len(geo2["volume"])
    dout = {k: torch.empty(ncv, dtype=torch.float64, device=dev) for k in ("density", "vx", "vy", "vz")}
    kiwi_b200.map_voronoi_device(dP, dhome, dgeo, dout, ctx=ctx)
    r_ms = []
    for _ in range(args.steps):
        r_ms.append(kiwi_b200.map_voronoi_device(dP, dhome, dgeo, dout, ctx=ctx)["total_ms"])
    # the single-launch gather (a face shared by two visited cells evaluated on both sides), for comparison
    ctx.set_voronoi_face_tables(False)
    kiwi_b200.map_voronoi_device(dP, dhome, dgeo, dout, ctx=ctx)
    s_ms = [kiwi_b200.map_voronoi_device(dP, dhome, dgeo, dout, ctx=ctx)["gather_ms"] for _ in range(args.steps)]
    ctx.set_voronoi_face_tables(True)
    line = {
        "metric": "particle-cell integrals/s (BFS-visited pairs), Voronoi map", "value": pairs / (np.mean(g_ms) * 1e-3),
        "unit": "pair-integrals/s", "n_gpus": 1, "steps": args.steps, "warmup": max(args.warmup, 1),
        "ms_per_step": float(np.mean(g_ms)), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{args.vor_n} column-recipe particles, 5 pc cube, coverage_grid buffer 0.05, "
                               "1 Lloyd iteration, cubic spline", "cells": int(len(geo2["volume"])),
                   "faces": int(len(geo2["vert_off"]) - 1)},
        "visited_pairs": int(pairs),
        "single_launch_gather": {"value": pairs / (np.mean(s_ms) * 1e-3), "ms_per_step": float(np.mean(s_ms)),
                                 "note": "kiwi_ctx_set_voronoi_face_tables(ctx, 0): each shared face evaluated on "
                                         "both sides, no face tables"},
        "e2e": {"value": pairs / (np.mean(t_ms) * 1e-3), "unit": "pair-integrals/s",
                "ms_per_step": float(np.mean(t_ms)), "note": "host arrays in and out (kiwi_map_voronoi)"},
        "device_resident": {"value": pairs / (np.mean(r_ms) * 1e-3), "unit": "pair-integrals/s",
                            "ms_per_step": float(np.mean(r_ms)),
                            "note": "particles and tessellation staged on the GPU once (kiwi_map_voronoi_device): "
                                    "walk, sort and gather of every call"},
        "cpu_baseline": None, "agreement_with_reference": None,
    }
    if ref_res is not None:
        d_ref = ref_res[0]
        m = d_ref > 1e-2 * d_ref.max()
        line["cpu_baseline"] = {"value": pairs / t_ref_map, "unit": "pair-integrals/s", "cores": threads,
                                "kind": "reference",
                                "sample": f"the whole map: run_mapping_stage's loop, {t_ref_map:.1f} s (geometry "
                                          f"build {t_geo:.1f} s excluded)"}
        line["agreement_with_reference"] = {
            "max_rel_density_diff_top_band": float(np.max(np.abs(r.density[m] - d_ref[m]) / d_ref[m])),
            "cells_compared": int(m.sum())}
    print(json.dumps(line), flush=True)
    return 0


def run_cartesian_map(args):
    """Cartesian-map point location: --cmap-n column-recipe particle positions on a 5 pc cube as the sites
    (seed 1003), a --cmap-res^3 grid; each cell centre takes its nearest site's values and id
    (kiwi_cartesian_map: host arrays in and out).  `value` is cells located per second over the device time
    of the binning and location kernels; the CPU baseline is the reference stage's own loop (one Voro++
    container per OpenMP thread, find_voronoi_cell per cell) over a bounded sample of x-slabs, container
    builds included, and the GPU's owners are checked against it there."""
    import torch

    import kiwi_b200
    from kiwi_b200.workloads import column_snapshot
    from oracle.oracle import load_ref

    torch.cuda.set_device(0)
    P, bounds = column_snapshot(n=args.cmap_n, seed=1003, box=(5.0, 5.0, 5.0))
    xyz = np.stack([P["x"], P["y"], P["z"]], axis=1)
    n = len(P["x"])
    ids = np.arange(n, dtype=np.int32)
    rng = np.random.default_rng(1)
    vals = [rng.random(n) for _ in range(4)]
    res = args.cmap_res
    ctx = kiwi_b200.Context(0)
    for _ in range(max(args.warmup, 1)):
        m = kiwi_b200.cartesian_map(xyz, bounds, res, *vals, site_id=ids, ctx=ctx)
    g_ms, t_ms, launches = [], [], 0
    clocks = ClockSampler(0)
    clocks.start()
    for _ in range(args.steps):
        m = kiwi_b200.cartesian_map(xyz, bounds, res, *vals, site_id=ids, ctx=ctx)
        g_ms.append(m.stats["gather_ms"])
        t_ms.append(m.stats["total_ms"])
        launches += m.stats["launches"]
    clk = clocks.stop()
    nq = res ** 3
    cpu, agree = None, None
    ref = load_ref()
    if ref is not None and not args.no_cpu_baseline:
        threads = ref.max_threads()
        slabs = max(1, res // 32)
        i0 = res // 2 - slabs // 2
        sec, rid, build = ref.locate_sample(xyz, ids, bounds, res, i0, i0 + slabs, threads=threads)
        q = sec - build
        whole = build + q * res / slabs  # the stage over the whole grid: one set of builds, every slab's queries
        cpu = {"value": nq / whole, "unit": "cells/s", "cores": threads, "kind": "reference",
               "sample": f"x-slabs {i0}..{i0 + slabs - 1} of {res} ({slabs * res * res} cells, through the filament): "
                         f"{q:.2f} s of queries, scaled to the whole grid, plus {build:.2f} s of per-thread container "
                         f"builds; sample rate {slabs * res * res / q:.4g} cells/s without the builds"}
        gpu_ids = m.voronoi_cell_id.reshape(res, res, res)[i0:i0 + slabs].reshape(-1)
        agree = {"cells_compared": int(rid.size), "owners_equal": int(np.sum(gpu_ids == rid))}
    line = {
        "metric": "cartesian-map cells located/s (nearest-site point location)", "value": nq / (np.mean(g_ms) * 1e-3),
        "unit": "cells/s", "n_gpus": 1, "steps": args.steps, "warmup": max(args.warmup, 1),
        "ms_per_step": float(np.mean(g_ms)), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{n} column-recipe sites, 5 pc cube, grid {res}^3", "sites": n, "cells": nq},
        "gpu_launches": int(launches), "clocks": clk,
        "e2e": {"value": nq / (np.mean(t_ms) * 1e-3), "unit": "cells/s", "ms_per_step": float(np.mean(t_ms)),
                "h2d_bytes_per_step": int(n * (7 * 8 + 4)), "d2h_bytes_per_step": int(nq * (4 * 8 + 4))},
        "cpu_baseline": cpu, "agreement_with_reference": agree,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_lloyd(args):
    """Point-set stage on the GPU: --lloyd-n column-recipe particles on a 5 pc cube (seed 1003), their
    coverage-grid buffer (spacing 0.05 x 5 pc, kiwi_coverage_grid_buffer) and one Lloyd step
    (kiwi_lloyd_step: every kept site's Voronoi cell built and its centroid taken).  `value` is Voronoi cells
    built per second over the Lloyd step's device time; the CPU baseline is the reference's own lloyd_step
    (single-threaded Voro++, as the reference runs it) on the sites of a sub-box holding a bounded sample."""
    import torch

    import kiwi_b200
    from kiwi_b200.workloads import column_snapshot
    from oracle.oracle import load_ref

    torch.cuda.set_device(0)
    P, bounds = column_snapshot(n=args.lloyd_n, seed=1003, box=(5.0, 5.0, 5.0))
    ctx = kiwi_b200.Context(0)
    t0 = time.perf_counter()
    bxyz, bids = kiwi_b200.coverage_grid_buffer(P, bounds, 0.05, 2.0, ctx=ctx)
    t_buf = time.perf_counter() - t0
    xyz = np.concatenate([np.stack([P["x"], P["y"], P["z"]], axis=1), bxyz])
    ids = np.arange(1, len(xyz) + 1, dtype=np.int32)
    for _ in range(max(args.warmup, 1)):
        r = kiwi_b200.lloyd_step(xyz, bounds, ids=ids, ctx=ctx)
    g_ms, t_ms, launches = [], [], 0
    clocks = ClockSampler(0)
    clocks.start()
    for _ in range(args.steps):
        r = kiwi_b200.lloyd_step(xyz, bounds, ids=ids, ctx=ctx)
        g_ms.append(r[3]["gather_ms"])
        t_ms.append(r[3]["total_ms"])
        launches += r[3]["launches"]
    clk = clocks.stop()
    cells = len(r[0])
    vol_err = abs(r[2].sum() - np.prod([bounds[2 * a + 1] - bounds[2 * a] for a in range(3)]))
    cpu, agree = None, None
    ref = load_ref()
    if ref is not None and not args.no_cpu_baseline:
        # the sites of a centred sub-box (its own domain), about 20 k of them
        frac = min(1.0, (20_000 / len(xyz)) ** (1 / 3))
        c = [(bounds[2 * a] + bounds[2 * a + 1]) / 2 for a in range(3)]
        half = [(bounds[2 * a + 1] - bounds[2 * a]) * frac / 2 for a in range(3)]
        sb = tuple(v for a in range(3) for v in (c[a] - half[a], c[a] + half[a]))
        m = np.all((xyz >= [sb[0], sb[2], sb[4]]) & (xyz <= [sb[1], sb[3], sb[5]]), axis=1)
        t0 = time.perf_counter()
        rid, rxyz = ref.lloyd_step(xyz[m], ids[m], sb)
        sec = time.perf_counter() - t0
        cpu = {"value": len(rid) / sec, "unit": "cells/s", "cores": 1, "kind": "reference",
               "sample": f"lloyd_step on the {int(m.sum())} sites of a centred sub-box (its own domain), {sec:.2f} s"}
        gid, gxyz, _, _ = kiwi_b200.lloyd_step(xyz[m], sb, ids=ids[m], ctx=ctx)
        agree = {"sites": int(len(rid)), "order_equal": bool(np.array_equal(gid, rid)),
                 "max_abs_position_diff": float(np.abs(gxyz - rxyz).max()) if np.array_equal(gid, rid) else None}
    line = {
        "metric": "Voronoi cells built/s (Lloyd step)", "value": cells / (np.mean(g_ms) * 1e-3), "unit": "cells/s",
        "n_gpus": 1, "steps": args.steps, "warmup": max(args.warmup, 1), "ms_per_step": float(np.mean(g_ms)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{args.lloyd_n} column-recipe particles + {len(bids)} coverage-grid buffer points, "
                               "5 pc cube, one Lloyd step", "sites": int(len(xyz)), "cells": int(cells)},
        "failed_cells": int(r[3]["failed"]), "cell_volume_sum_minus_domain": float(vol_err),
        "coverage_buffer_s_end_to_end": t_buf, "gpu_launches": int(launches), "clocks": clk,
        "e2e": {"value": cells / (np.mean(t_ms) * 1e-3), "unit": "cells/s", "ms_per_step": float(np.mean(t_ms)),
                "h2d_bytes_per_step": int(len(xyz) * 28), "d2h_bytes_per_step": int(cells * 36)},
        "cpu_baseline": cpu, "agreement_with_reference": agree,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_batch(args):
    """Batched sph-to-grid: args.batch_items column snapshots (item i seeded 5000 + i), N log-uniform in
    [nmin, nmax], grid res^3 with res log-uniform in [resmin, resmax], kernels cycling M4 / M6 / WC4; one
    kiwi_batch_create, then timed graph replays.  Also times the same items as one sph-to-grid call each."""
    import torch

    import kiwi_b200
    from kiwi_b200.workloads import column_snapshot

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(5000)
    kernels = ["cubic_spline", "quintic_spline", "wendland_c4"]
    items, t_gen = [], time.perf_counter()
    for i in range(args.batch_items):
        n = int(round(np.exp(rng.uniform(np.log(args.batch_nmin), np.log(args.batch_nmax)))))
        res = int(round(np.exp(rng.uniform(np.log(args.batch_resmin), np.log(args.batch_resmax)))))
        kname = kernels[i % 3]
        P, bounds = column_snapshot(n=n, seed=5000 + i, hfact=kiwi_b200.get_kernel(kname).hfact)
        dP = {k: torch.from_numpy(v).to(dev) for k, v in P.items()}
        nc = res ** 3
        out = {k: torch.empty(nc, dtype=torch.float64, device=dev) for k in ("density", "vx", "vy", "vz")}
        items.append({"particles": dP, "bounds": bounds, "shape": (res, res, res),
                      "kernel": kiwi_b200.make_kernel_integrator(kname), "out": out, "n": n})
    t_gen = time.perf_counter() - t_gen
    ctx = kiwi_b200.Context(0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    batch = kiwi_b200.Batch(items, precision=args.precision, ctx=ctx)
    create_s = time.perf_counter() - t0
    batch.run()
    lpt, ctas = batch.tune()
    for _ in range(max(args.warmup - 1, 0)):
        batch.run()
    peak_fp64 = kiwi_b200.measure_fp64_peak(ctx)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)
    clocks = ClockSampler(0)
    clocks.start()
    ms, pairs, cells = [], 0, 0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        per, tot = batch.run()
        ms.append(tot["gather_ms"])
        pairs += tot["sphere_pairs"]
    clk = clocks.stop()
    ncells = sum(int(np.prod(it["shape"])) for it in items)
    # the same items as one call each (the unbatched baseline)
    torch.cuda.synchronize()
    t_single, single_pairs = 0.0, 0
    for it in items:
        st = kiwi_b200.sph_to_grid_device(it["particles"], it["bounds"], it["shape"], it["out"], kernel=it["kernel"],
                                          precision=args.precision, ctx=ctx)
        t_single += st["total_ms"]
        single_pairs += st["sphere_pairs"]
    batch.close()
    errors = batch_item_errors(items, args) if not args.no_cpu_baseline else None
    tot_ms = float(np.sum(ms))
    line = {
        "metric": "particle-cell integrals/s (support pairs), batched sph-to-grid", "value": pairs / (tot_ms * 1e-3),
        "unit": "pair-integrals/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": tot_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{args.batch_items} column snapshots (C1 recipe, seeds 5000+i), N log-uniform in "
                               f"[{args.batch_nmin}, {args.batch_nmax}], grids res^3 with res log-uniform in "
                               f"[{args.batch_resmin}, {args.batch_resmax}], kernels cycling M4/M6/WC4",
                   "precision": args.precision, "particles": int(sum(it["n"] for it in items)), "cells": ncells,
                   "l2": "flushed between timed steps (256 MB write)"},
        "cells_per_s": ncells * args.steps / (tot_ms * 1e-3),
        "pairs_per_step": pairs / args.steps,
        "launch_shape": {"longest_first": lpt, "ctas_per_sm": ctas},
        "plan_create_s": create_s, "generate_s": t_gen,
        "unbatched": {"ms": t_single, "value": single_pairs / (t_single * 1e-3),
                      "note": "the same items as one kiwi_sph_to_grid_device call each, binning included"},
        "fp64_peak_tflops": peak_fp64, "clocks": clk, "gpu_launches": int(per[0]["launches"]) if per else 0,
    }
    if errors is not None:
        line["per_snapshot_error"] = errors
    print(json.dumps(line), flush=True)
    return 0


def batch_item_errors(items, args, pair_cap=200_000):
    """Per snapshot of the batch: a seeded subset of its particles (random order, taken while the subset's
    bounding-box pairs stay under pair_cap) mapped on the snapshot's own grid by the GPU (one call, FP64 and
    FP32-mixed) and by the CPU oracle (the C restatement of the reference, bit-identical to it); per density
    band of the oracle's grid, the largest relative difference.  The batch's own outputs agree with one call
    per item to rounding (within 1e-12 of the item's peak, tests/test_gpu_batch.py), so this is the batch's
    error."""
    import kiwi_b200
    from oracle.compare import band_stats
    from oracle.oracle import Oracle

    orc = Oracle()
    ctx = kiwi_b200.Context(0)
    rng = np.random.default_rng(77)
    out, worst64, worst32 = [], [0.0] * 4, [0.0] * 4
    for it in items:
        P = {k: v.cpu().numpy() for k, v in it["particles"].items()}
        b, shape = it["bounds"], it["shape"]
        d = [(b[2 * a + 1] - b[2 * a]) / shape[a] for a in range(3)]
        kidx = it["kernel"].kernel
        spec = kiwi_b200.KernelSpec(kidx)
        sup = it["kernel"].support_in_h or spec.radkern
        box = np.ones(len(P["x"]))
        for a, k in enumerate("xyz"):
            lo = np.clip(np.floor((P[k] - sup * P["h"] - b[2 * a]) / d[a]), 0, shape[a] - 1)
            hi = np.clip(np.floor((P[k] + sup * P["h"] - b[2 * a]) / d[a]), 0, shape[a] - 1)
            box *= np.maximum(hi - lo + 1, 0)
        take, tot = [], 0.0
        for i in rng.permutation(len(box)):
            if tot + box[i] > pair_cap:
                continue
            take.append(i)
            tot += box[i]
            if len(take) >= 64:
                break
        sub = {k: np.ascontiguousarray(v[np.sort(take)]) for k, v in P.items()}
        cubic = kidx == 0 and sup == 2.0
        dens = orc.sph_to_grid(sub, b, shape, kernel=-1 if cubic else kidx, support_in_h=sup)[0]
        rec = {"kernel": spec.key, "grid": shape[0], "particles": len(P["x"]), "subset": len(take),
               "subset_bbox_pairs": int(tot)}
        for prec, worst in (("fp64", worst64), ("fp32_mixed", worst32)):
            g = kiwi_b200.sph_to_grid(sub, b, shape, kernel=it["kernel"], precision=prec, ctx=ctx).density
            st = band_stats(g, dens)
            rec[prec] = [s["max"] for s in st]
            for k in range(4):
                if st[k]["max"] is not None:
                    worst[k] = max(worst[k], st[k]["max"])
        out.append(rec)
    return {"against": "the CPU oracle (the reference's algorithm restated, bit-identical to it) on a seeded "
                       "particle subset of each snapshot, the snapshot's grid and kernel",
            "bands": [">1e-2 of peak", "1e-4..1e-2", "1e-6..1e-4", "<=1e-6 (abs/peak)"],
            "max_over_snapshots_fp64": worst64, "max_over_snapshots_fp32_mixed": worst32, "items": out}


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "adjoint":
        return run_adjoint(args)
    if args.workload == "voronoi":
        return run_voronoi(args)
    if args.workload == "cartesian_map":
        return run_cartesian_map(args)
    if args.workload == "lloyd":
        return run_lloyd(args)
    ws, rank, local = dist_env()
    import torch

    import kiwi_b200

    dist = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", torch.cuda.current_device())

    split = ws > 1 and args.multi == "tiles"
    P, bounds, shape = make_workload(args.n, args.res, args.seed + (0 if split else 1000 * rank), args.kernel)
    ki = kiwi_b200.make_kernel_integrator(args.kernel, use_tabulated_integral=args.tabulated)
    part, n_parts = (rank, ws) if split else (0, 1)
    ctx = kiwi_b200.Context(dev.index)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    dP = {k: torch.from_numpy(v).to(dev) for k, v in P.items()}
    nc = shape[0] * shape[1] * shape[2]
    out = {k: torch.empty(nc, dtype=torch.float64, device=dev) for k in ("density", "vx", "vy", "vz")}
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()

    for _ in range(args.warmup):
        kiwi_b200.sph_to_grid_device(dP, bounds, shape, out, kernel=ki, precision=args.precision, full_box=args.full_box,
                                     ctx=ctx, part=part, n_parts=n_parts)
    peak_fp64 = kiwi_b200.measure_fp64_peak(ctx)

    clocks = ClockSampler(dev.index)
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    t_wall = time.perf_counter()
    step_ms, gather_ms, sph_pairs, bbox_pairs, evaluated, launches = [], [], 0, 0, 0, 0
    items = {}
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()  # L2 flush between steps, outside the timed events
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        st = kiwi_b200.sph_to_grid_device(dP, bounds, shape, out, kernel=ki, precision=args.precision,
                                          full_box=args.full_box, ctx=ctx, part=part, n_parts=n_parts)
        with torch.cuda.stream(stream):
            e1.record(stream)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        gather_ms.append(st["gather_ms"])
        sph_pairs += st["sphere_pairs"]
        bbox_pairs += st["bbox_pairs"]
        evaluated += st["evaluated_pairs"]
        launches += st["launches"]
        for key in ("edge_tiers_outer", "edge_tiers_middle", "edge_tiers_inner", "vertex_pyramids"):
            items[key] = items.get(key, 0) + st[key]
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    wall = time.perf_counter() - t_wall
    clk = clocks.stop()

    tot_ms = float(np.sum(step_ms))
    if ws > 1:
        t = torch.tensor([tot_ms, float(sph_pairs), float(bbox_pairs)], dtype=torch.float64, device=dev)
        tmax = t.clone()
        dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        job_ms, job_pairs, job_bbox = float(tmax[0]), float(t[1]), float(t[2])
    else:
        job_ms, job_pairs, job_bbox = tot_ms, float(sph_pairs), float(bbox_pairs)
    value = job_pairs / (job_ms * 1e-3)

    def fp32_accuracy(g, r, st_last, precision):
        """Per-cell and total-mass error of FP32-form densities g against FP64-form densities r."""
        msk = r >= 1e-6 * r.max()
        rel = ((g[msk] - r[msk]).abs() / r[msk]).double()
        acc = {"against": "the FP64 form (lattice), same input", "cells_above_1e-6_peak": int(msk.sum()),
               "nonfinite_cells": int((~torch.isfinite(g)).sum()),
               "max_rel_cell_err": float(rel.max()), "median_rel_cell_err": float(rel.median()),
               "q99_rel_cell_err": float(torch.quantile(rel[: 1 << 24].float(), 0.99)),
               "cells_over_1e-6": int((rel > 1e-6).sum()),
               "total_mass_rel_err": float(abs(g.sum() - r.sum()) / r.sum())}
        if precision == "fp32_mixed_guaranteed":
            acc.update({"cells_fp32_bound_over_1e-6": int(st_last["fp64_fallback"]),
                        "fp64_tiles": int(st_last["fp64_tiles"])})
        else:
            # points and edge pairs with a plane within 1e-3 h of the particle, evaluated in FP64
            acc["fp64_island_points"] = int(st_last["fp64_fallback"])
        return acc

    # accuracy of an FP32 form: against the FP64 form on the same input (untimed)
    accuracy = None
    if args.precision.startswith("fp32") and not split:
        ref = {k: torch.empty(nc, dtype=torch.float64, device=dev) for k in ("density", "vx", "vy", "vz")}
        kiwi_b200.sph_to_grid_device(dP, bounds, shape, ref, kernel=ki, precision="fp64", ctx=ctx)
        torch.cuda.synchronize()
        accuracy = fp32_accuracy(out["density"], ref["density"], st, args.precision)

    # the FP32-mixed form timed beside the FP64 form (same input, same step protocol), with its error
    # against this run's FP64 output: the FP32-mixed vs FP64 comparison of the metric
    fp32_side = None
    if (args.precision == "fp64" and not args.no_fp32_compare and args.kernel == "cubic_spline" and not args.full_box
            and not split and not args.tabulated):
        # both FP32 forms on the same input, timed like the FP64 steps (the guaranteed one over fewer steps)
        fp32_side = {}
        o32 = {k: torch.empty(nc, dtype=torch.float64, device=dev) for k in ("density", "vx", "vy", "vz")}
        for prec in ("fp32_mixed", "fp32_mixed_guaranteed"):
            steps32 = args.steps if prec == "fp32_mixed" else min(args.steps, 2)
            for _ in range(min(args.warmup, 2)):
                kiwi_b200.sph_to_grid_device(dP, bounds, shape, o32, kernel=ki, precision=prec, ctx=ctx)
            ms32, pairs32 = 0.0, 0
            for _ in range(steps32):
                with torch.cuda.stream(stream):
                    flush.zero_()
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                st32 = kiwi_b200.sph_to_grid_device(dP, bounds, shape, o32, kernel=ki, precision=prec, ctx=ctx)
                with torch.cuda.stream(stream):
                    e1.record(stream)
                e1.synchronize()
                ms32 += e0.elapsed_time(e1)
                pairs32 += st32["sphere_pairs"]
            acc32 = fp32_accuracy(o32["density"], out["density"], st32, prec)
            v32 = pairs32 / (ms32 * 1e-3)
            fp32_side[prec] = {"precision": prec, "value": v32 * ws, "unit": "pair-integrals/s", "steps": steps32,
                               "ms_per_step": ms32 / steps32,
                               "ratio_vs_fp64": v32 / (tot_ms and sph_pairs / (tot_ms * 1e-3)),
                               "meets_1e-6_per_cell": acc32["max_rel_cell_err"] <= 1e-6, "accuracy": acc32}
        del o32

    # end to end through the public host API: pinned host arrays in, host arrays out
    e2e = None
    if args.e2e_steps > 0 and split:
        # each rank: the whole snapshot host -> device, its part, its x rows device -> host; max over ranks
        from kiwi_b200 import shard

        sup = ki.support_in_h or kiwi_b200.get_kernel(args.kernel).radkern
        own = shard.tile_owners(shard.tile_entry_counts(P, bounds, shape, sup), ws)
        ix0, ix1 = shard.part_rows(own, rank, shape)
        c0, c1 = ix0 * shape[1] * shape[2], ix1 * shape[1] * shape[2]
        hP = {k: torch.from_numpy(v).pin_memory() for k, v in P.items()}
        hout = {k: torch.empty(c1 - c0, dtype=torch.float64).pin_memory() for k in out}
        e_ms, e_pairs = 0.0, 0
        for i in range(args.e2e_steps + 1):
            dist.barrier()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for k in dP:
                dP[k].copy_(hP[k], non_blocking=True)
            torch.cuda.synchronize()
            st = kiwi_b200.sph_to_grid_device(dP, bounds, shape, out, kernel=ki, precision=args.precision,
                                              full_box=args.full_box, ctx=ctx, part=part, n_parts=n_parts)
            for k in out:
                hout[k].copy_(out[k][c0:c1], non_blocking=True)
            torch.cuda.synchronize()
            if i > 0:  # the first pass is a warm-up
                e_ms += (time.perf_counter() - t0) * 1e3
                e_pairs += st["sphere_pairs"]
        from kiwi_b200.shard import reduce_step

        e_max, e_all = reduce_step(e_ms, float(e_pairs), device=dev)
        e2e = {"value": e_all / (e_max * 1e-3), "unit": "pair-integrals/s",
               "h2d_bytes_per_step": int(8 * 8 * len(P["x"])) * ws, "d2h_bytes_per_step": int(4 * 8 * nc),
               "ms_per_step": e_max / args.e2e_steps,
               "note": "max over ranks of the wall time of each rank's copies in, part, and its rows out"}
    elif args.e2e_steps > 0:
        hP = {k: torch.from_numpy(v).pin_memory().numpy() for k, v in P.items()}
        hout = [torch.empty(nc, dtype=torch.float64).pin_memory().numpy() for _ in range(4)]
        kiwi_b200.sph_to_grid(hP, bounds, shape, kernel=ki, precision=args.precision, full_box=args.full_box, ctx=ctx, out=hout)
        e_ms, e_pairs = 0.0, 0
        for _ in range(args.e2e_steps):
            r = kiwi_b200.sph_to_grid(hP, bounds, shape, kernel=ki, precision=args.precision, full_box=args.full_box, ctx=ctx, out=hout)
            e_ms += r.stats["total_ms"]
            e_pairs += r.stats["sphere_pairs"]
        e2e = {"value": e_pairs / (e_ms * 1e-3) * ws, "unit": "pair-integrals/s",
               "h2d_bytes_per_step": int(8 * 8 * len(P["x"])), "d2h_bytes_per_step": int(4 * 8 * nc),
               "ms_per_step": e_ms / args.e2e_steps}

    cpu = None
    parity_c1 = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline and not args.tabulated:
        cpu = cpu_baseline(P, bounds, shape, args.kernel)
        if not args.no_parity and args.kernel == "cubic_spline" and args.precision == "fp64":
            parity_c1 = cpu_baseline_c1(kiwi_b200, ctx)

    if rank == 0:
        g_ms = float(np.mean(gather_ms))
        evaluated_per_launch = evaluated / args.steps
        is32 = args.precision.startswith("fp32")
        if items.get("vertex_pyramids", 0) > 0:
            # lattice-factorised kernel: its own work items x their measured costs
            kname = ("k_cart_lattice_f32 (FP32 lattice tiers with rounding bounds; flagged tiles recomputed in FP64)"
                     if args.precision == "fp32_mixed_guaranteed" else
                     "k_cart_lattice_mixed (FP32 lattice tiers, FP64 islands and assembly)" if is32 else
                     "k_cart_lattice (FP64 lattice-factorised cell-integral gather)" if args.kernel == "cubic_spline"
                     else "k_cart_lattice_generic (FP64 lattice form, table-driven tiers; work items costed at the "
                          "cubic tiers' rates)")
            work = (items["edge_tiers_outer"] * EDGE_OUTER + items["edge_tiers_middle"] * EDGE_MIDDLE +
                    items["edge_tiers_inner"] * EDGE_INNER + items["vertex_pyramids"] * VERTEX_PYRAMID +
                    evaluated * CELL_ASSEMBLY) / args.steps
            work_per_pair = work / max(evaluated_per_launch, 1)
        else:
            kname = "k_cart_gather (FP64 cell-integral gather, reference evaluation order)"
            work_per_pair = WORK_PER_BBOX_PAIR if args.full_box else WORK_PER_SUPPORT_PAIR
            work = evaluated_per_launch * work_per_pair
        achieved = work / (g_ms * 1e-3) / 1e12
        peak = kiwi_b200.measure_fp32_peak(ctx) if is32 else peak_fp64
        # DRAM traffic of the kernel per launch: an ncu capture of this exact workload (one pass,
        # dram__bytes_read.sum + dram__bytes_write.sum), stated with the commit it was captured at; the
        # bench cannot count DRAM bytes itself, so other workloads report None
        traffic, traffic_src = None, None
        if (not is32 and args.n == 2_000_000 and args.res == 256 and args.kernel == "cubic_spline" and
                not args.full_box and args.precision == "fp64" and ws == 1 and not args.tabulated):
            traffic = LATTICE_TRAFFIC["bytes"]
            traffic_src = (f"ncu dram__bytes_read.sum + dram__bytes_write.sum of one {LATTICE_TRAFFIC['kernel']} "
                           f"launch of this workload, captured at commit {LATTICE_TRAFFIC['commit']}")
        hbm_peak, hbm_src = hbm_peak_gbs()
        tab_roofline = None
        if args.tabulated:
            # each vertex pyramid is one trilinear lookup: 8 table entries (64 bytes) from a 182 MB table
            lookups = items.get("vertex_pyramids", 0) / args.steps
            ach = lookups * TAB_BYTES_PER_LOOKUP / (g_ms * 1e-3) / 1e9
            tab_roofline = {"bound": "hbm", "kernel": "k_cart_lattice_tab (FP64 lattice form, tabulated integral)",
                            "achieved": ach, "peak": hbm_peak, "unit": "GB/s",
                            "frac": ach / hbm_peak if hbm_peak else None, "traffic": None,
                            "algorithmic_bytes": "64 bytes (8 table entries) per lookup x lookups per launch",
                            "lookups_per_launch": lookups, "peak_source": hbm_src,
                            "gather_ms_per_launch": g_ms}
        line = {
            "metric": "particle-cell integrals/s (support pairs), sph-to-grid", "value": value,
            "unit": "pair-integrals/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": job_ms / args.steps, "higher_is_better": True,
            # --multi tiles: the same grid at every N (total work fixed); replicas: one grid per rank
            "scaling": "strong" if args.multi == "tiles" else "weak",
            "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
            "data": "synthetic",
            "config": workload_config(args, nc, ws, split),
            "pairs": {"support_pairs_per_step": job_pairs / args.steps / ws,
                      "bbox_pairs_per_step": job_bbox / args.steps / ws,
                      "bbox_pairs_per_s": job_bbox / (job_ms * 1e-3)},
            "roofline": {"bound": "fp32" if is32 else "fp64", "kernel": kname, "work_items_per_launch":
                         {k: v / args.steps for k, v in items.items()},
                         "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak if peak else None, "traffic": traffic,
                         "traffic_source": traffic_src,
                         "hbm": ({"achieved_gbs": traffic / (g_ms * 1e-3) / 1e9, "peak_gbs": hbm_peak,
                                  "frac": traffic / (g_ms * 1e-3) / 1e9 / hbm_peak, "peak_source": hbm_src}
                                 if traffic and hbm_peak else None),
                         "work_per_pair_flops": work_per_pair, "evaluated_pairs_per_launch": evaluated_per_launch,
                         "peak_source": ("measured FP32 FMA probe (kiwi_measure_fp32_peak)" if is32 else
                                         "measured FP64 FMA probe (kiwi_measure_fp64_peak)") +
                                        " in this run; MEASURED_PEAKS.json has no FP64/FP32 figure",
                         "gather_ms_per_launch": g_ms},
            "clocks": clk, "gpu_launches": int(launches), "wall_s_timed_region": wall,
            "e2e": e2e, "cpu_baseline": cpu,
        }
        if tab_roofline is not None:
            line["roofline"] = tab_roofline
        if accuracy is not None:
            line["accuracy"] = accuracy
        if parity_c1 is not None:
            line["parity_c1"] = parity_c1
        if fp32_side is not None:
            # the FP32 lattice kernel evaluates the same lattice work items as the FP64 one
            peak32 = kiwi_b200.measure_fp32_peak(ctx)
            side = fp32_side["fp32_mixed"]
            a32 = work_per_pair * side["value"] / ws / 1e12
            side["roofline"] = {"bound": "fp32", "kernel": "k_cart_lattice_mixed", "achieved": a32, "peak": peak32,
                                "unit": "TFLOP/s", "frac": a32 / peak32 if peak32 else None,
                                "peak_source": "measured FP32 FMA probe (kiwi_measure_fp32_peak) in this run"}
            line["fp32_mixed"] = side
            line["fp32_mixed_guaranteed"] = fp32_side["fp32_mixed_guaranteed"]
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
