"""ctypes bindings of the CPU oracles -- TEST INFRASTRUCTURE ONLY.

``Oracle`` wraps oracle/liboracle.so (the C restatement of the reference's algorithm) and ``RefLib``
wraps oracle/_ref/libkiwi_ref.so (the reference KIWI library built from its own sources by
oracle/Makefile).  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this
module; the product package (kiwi_b200) never does.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
ORACLE_Q_SO = os.path.join(HERE, "liboracle_q.so")
REF_SO = os.path.join(HERE, "_ref", "libkiwi_ref.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_i32p = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)


def _d(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class OrStats(C.Structure):
    _fields_ = [("bbox_pairs", C.c_int64), ("sphere_pairs", C.c_int64), ("skipped_outside", C.c_int64),
                ("neg_clamped", C.c_int64), ("neg_warned", C.c_int64)]


class Oracle:
    """The C restatement (oracle/kiwi_oracle.c, FP64, bit-identical to the reference).  With quad=True the
    same algorithm in __float128 with exact constants (oracle/kiwi_oracle_q.c): the error yardstick."""

    def __init__(self, path: str | None = None, quad: bool = False, prefix: str | None = None):
        path = path or (ORACLE_Q_SO if quad else ORACLE_SO)
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        L = self.lib = C.CDLL(path)
        pfx = prefix or ("orq_" if quad else "or_")
        for name in ("full_integral_new", "generic_full_integral", "gridded_integral", "face_integral",
                     "generic_edge_breaks", "generic_vertex", "sph_to_grid", "map_voronoi"):
            setattr(L, "or_" + name, getattr(L, pfx + name))
        L.or_full_integral_new.restype = C.c_double
        L.or_full_integral_new.argtypes = [C.c_double] * 4
        L.or_generic_full_integral.restype = C.c_double
        L.or_generic_full_integral.argtypes = [C.c_int] + [C.c_double] * 4
        L.or_gridded_integral.restype = C.c_double
        L.or_gridded_integral.argtypes = [C.c_double] * 4
        L.or_face_integral.restype = C.c_double
        L.or_face_integral.argtypes = [C.c_double] * 3 + [C.c_int, C.c_double, C.c_double, C.c_int, _dp, C.c_int, _ip]
        L.or_generic_edge_breaks.restype = C.c_int
        L.or_generic_edge_breaks.argtypes = [C.c_int] + [C.c_double] * 3 + [_dp, C.c_int]
        L.or_generic_vertex.restype = C.c_double
        L.or_generic_vertex.argtypes = [C.c_int] + [C.c_double] * 4
        L.or_sph_to_grid.restype = C.c_int
        L.or_sph_to_grid.argtypes = ([C.c_int64] + [_dp] * 8 + [_dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                                                C.c_int, C.c_int64, C.c_int64] + [_dp] * 5 +
                                     [C.POINTER(OrStats)])
        L.or_inverse_map = getattr(L, pfx + "inverse_map")
        L.or_inverse_map.restype = C.c_int
        L.or_inverse_map.argtypes = ([C.c_int64, _i32p] + [_dp] * 8 + [C.c_int64, _i64p, _i64p, _dp, _i32p, _dp,
                                                                       C.c_int, C.c_double, C.c_int] + [_dp] * 3)
        L.or_coverage_grid_buffer = getattr(L, pfx + "coverage_grid_buffer")
        L.or_coverage_grid_buffer.restype = C.c_int64
        L.or_coverage_grid_buffer.argtypes = [C.c_int64] + [_dp] * 5 + [C.c_double, C.c_double, _dp, _i32p]
        L.or_container_order = getattr(L, pfx + "container_order")
        L.or_container_order.restype = C.c_int64
        L.or_container_order.argtypes = [C.c_int64, _dp, _dp, C.c_double, _i64p]
        L.or_cartesian_map_nearest = getattr(L, pfx + "cartesian_map_nearest")
        L.or_cartesian_map_nearest.restype = C.c_int
        L.or_cartesian_map_nearest.argtypes = [C.c_int64, _dp, _dp, C.c_int, _i32p]
        for name in ("table_load", "table_reset", "table_values"):
            setattr(L, "or_" + name, getattr(L, pfx + name))
        L.or_table_load.restype = C.c_int
        L.or_table_load.argtypes = [C.c_char_p]
        L.or_table_reset.restype = None
        L.or_table_reset.argtypes = []
        L.or_table_values.restype = C.c_int64
        L.or_table_values.argtypes = [_dp]
        L.or_map_voronoi.restype = C.c_int
        L.or_map_voronoi.argtypes = ([C.c_int64, _i32p] + [_dp] * 8 + [C.c_int64, _i64p, _i64p, _dp, _i32p, _dp,
                                                                      C.c_int, C.c_double, C.c_int] + [_dp] * 5 +
                                     [_i64p])

    def full_integral_new(self, h, phi, r0, R0):
        return self.lib.or_full_integral_new(h, phi, r0, R0)

    def generic_full_integral(self, kernel, H, phi, r0, R0):
        return self.lib.or_generic_full_integral(kernel, H, phi, r0, R0)

    def gridded_integral(self, h, phi, r0, R0):
        return self.lib.or_gridded_integral(h, phi, r0, R0)

    def inverse_map(self, P, home, geo, kernel=-1, support_in_h=2.0, tabulated=False, cell_mass=None):
        """run_inverse_mapping_test_stage's particle loop: (m_recovered, coverage) per particle."""
        arrs = [_f64(P[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "m", "h")]
        n = len(arrs[0])
        home = np.ascontiguousarray(home, dtype=np.int32)
        fo = np.ascontiguousarray(geo["face_off"], dtype=np.int64)
        vo = np.ascontiguousarray(geo["vert_off"], dtype=np.int64)
        vx_ = _f64(geo["vxyz"]).reshape(-1)
        fn = np.ascontiguousarray(geo["face_nbr"], dtype=np.int32)
        vol = _f64(geo["volume"])
        cm = _f64(cell_mass) if cell_mass is not None else None
        rec, cov = np.zeros(n), np.zeros(n)
        self.lib.or_inverse_map(n, home.ctypes.data_as(_i32p), *[_d(a) for a in arrs], len(vol),
                                fo.ctypes.data_as(_i64p), vo.ctypes.data_as(_i64p), _d(vx_),
                                fn.ctypes.data_as(_i32p), _d(vol), kernel, support_in_h, int(tabulated), _d(cm),
                                _d(rec), _d(cov))
        return rec, cov

    def coverage_grid_buffer(self, P, bounds, spacing_fraction=0.05, factor=2.0):
        """add_coverage_grid_buffer by brute force: (xyz (k, 3), ids (k,)), or None if every h <= 0."""
        a = [_f64(P[k]) for k in ("x", "y", "z", "h")]
        b = _f64(bounds)
        ex, ey, ez = b[1] - b[0], b[3] - b[2], b[5] - b[4]
        sp = spacing_fraction * min(ex, ey, ez)
        cap = max(1, int(round(ex / sp))) * max(1, int(round(ey / sp))) * max(1, int(round(ez / sp)))
        xyz = np.zeros(3 * cap)
        ids = np.zeros(cap, dtype=np.int32)
        k = self.lib.or_coverage_grid_buffer(len(a[0]), *[_d(v) for v in a], _d(b), spacing_fraction, factor, _d(xyz),
                                             ids.ctypes.data_as(_i32p))
        if k < 0:
            return None
        return xyz[:3 * k].reshape(-1, 3), ids[:k]

    def container_order(self, sites, bounds, scale=3.0):
        """The site indices the reference's Voro++ container keeps, in its walk order."""
        xyz = _f64(np.asarray(sites, dtype=np.float64).reshape(-1, 3))
        out = np.zeros(max(len(xyz), 1), dtype=np.int64)
        k = self.lib.or_container_order(len(xyz), _d(xyz), _d(_f64(bounds)), scale, out.ctypes.data_as(_i64p))
        return out[:k]

    def cartesian_map_nearest(self, sites, bounds, res):
        """Nearest site index of every cell centre of the res^3 grid (-1 without sites), brute force."""
        xyz = _f64(np.asarray(sites, dtype=np.float64).reshape(-1, 3))
        out = np.zeros(res ** 3, dtype=np.int32)
        self.lib.or_cartesian_map_nearest(xyz.shape[0], _d(xyz), _d(_f64(bounds)), res, out.ctypes.data_as(_i32p))
        return out

    def table_load(self, path) -> int:
        """load_density_table restated: 0, or -1 / -2 / -3 (cannot open / header malformed / truncated)."""
        return self.lib.or_table_load(os.fsencode(path))

    def table_reset(self):
        """Back to the canonical (generated) table."""
        self.lib.or_table_reset()

    def table_values(self) -> np.ndarray:
        """The values of the table in use, flat, laid out as DensityLookupTable::at."""
        n = self.lib.or_table_values(None)
        out = np.empty(n)
        self.lib.or_table_values(_d(out))
        return out

    def face_integral(self, x0, y0, z0, verts, kernel=-1, h=1.0, support=None, tabulated=False):
        v = _f64(verts).reshape(-1)
        ov = C.c_int(0)
        sup = support if support is not None else 2.0 * h
        r = self.lib.or_face_integral(x0, y0, z0, kernel, h, sup, int(tabulated), _d(v), len(v) // 3, C.byref(ov))
        return r, ov.value

    def generic_edge_breaks(self, kernel, H, r0, R0):
        out = np.zeros(8)
        n = self.lib.or_generic_edge_breaks(kernel, H, r0, R0, _d(out), 8)
        return out[:n]

    def generic_vertex(self, kernel, H, r0, R0, phi):
        return self.lib.or_generic_vertex(kernel, H, r0, R0, phi)

    def sph_to_grid(self, P, bounds, shape, kernel=-1, support_in_h=2.0, tabulated=False, p_range=None):
        """P: dict of arrays x y z vx vy vz m h.  Returns (density, vx, vy, vz, raw[4], stats)."""
        arrs = [_f64(P[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "m", "h")]
        n = len(arrs[0])
        nx, ny, nz = shape
        nc = nx * ny * nz
        outs = [np.zeros(nc) for _ in range(4)]
        raw = np.zeros(4 * nc)
        st = OrStats()
        b = _f64(bounds)
        pb, pe = (0, n) if p_range is None else p_range
        rc = self.lib.or_sph_to_grid(n, *[_d(a) for a in arrs], _d(b), nx, ny, nz, kernel, support_in_h,
                                     int(tabulated), pb, pe, *[_d(o) for o in outs], _d(raw), C.byref(st))
        if rc != 0:
            raise RuntimeError(f"or_sph_to_grid failed: {rc}")
        return outs[0], outs[1], outs[2], outs[3], raw.reshape(4, nc), st

    def map_voronoi(self, P, home, geo, kernel=-1, support_in_h=2.0, tabulated=False):
        arrs = [_f64(P[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "m", "h")]
        n = len(arrs[0])
        home = np.ascontiguousarray(home, dtype=np.int32)
        fo = np.ascontiguousarray(geo["face_off"], dtype=np.int64)
        vo = np.ascontiguousarray(geo["vert_off"], dtype=np.int64)
        vx = _f64(geo["vxyz"]).reshape(-1)
        fn = np.ascontiguousarray(geo["face_nbr"], dtype=np.int32)
        vol = _f64(geo["volume"])
        nc = len(vol)
        outs = [np.zeros(nc) for _ in range(4)]
        raw = np.zeros(4 * nc)
        vis = C.c_int64(0)
        rc = self.lib.or_map_voronoi(n, home.ctypes.data_as(_i32p), *[_d(a) for a in arrs], nc,
                                     fo.ctypes.data_as(_i64p), vo.ctypes.data_as(_i64p), _d(vx),
                                     fn.ctypes.data_as(_i32p), _d(vol), kernel, support_in_h, int(tabulated),
                                     *[_d(o) for o in outs], _d(raw), C.byref(vis))
        if rc != 0:
            raise RuntimeError(f"or_map_voronoi failed: {rc}")
        return outs[0], outs[1], outs[2], outs[3], raw.reshape(4, nc), vis.value


KERNEL_NAMES = ["cubic_spline", "quartic_spline", "quintic_spline", "wendland_c2", "wendland_c4", "wendland_c6"]


class RefLib:
    """The reference library compiled from its own sources (oracle/_ref/libkiwi_ref.so)."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle` where the reference is present")
        L = self.lib = C.CDLL(path)
        L.ref_last_error.restype = C.c_char_p
        L.ref_full_integral_new.restype = C.c_double
        L.ref_full_integral_new.argtypes = [C.c_double] * 4
        L.ref_generic_full_integral.restype = C.c_double
        L.ref_generic_full_integral.argtypes = [C.c_int] + [C.c_double] * 4
        L.ref_gridded_integral.restype = C.c_double
        L.ref_gridded_integral.argtypes = [C.c_double] * 4
        L.ref_face_integral.restype = C.c_double
        L.ref_face_integral.argtypes = [C.c_double] * 3 + [C.c_int, C.c_double, C.c_double, C.c_int, _dp, C.c_int, _ip]
        L.ref_sph_to_grid.restype = C.c_int
        L.ref_sph_to_grid.argtypes = ([C.c_long] + [_dp] * 8 + [_dp, C.c_int, C.c_int, C.c_int, C.c_char_p, C.c_double,
                                                               C.c_int, C.c_int, C.c_int] + [_dp] * 4)
        L.ref_voronoi_build.restype = C.c_void_p
        L.ref_voronoi_build.argtypes = ([C.c_long] + [_dp] * 8 + [_dp, C.c_int, C.c_double, C.c_int, C.c_char_p,
                                                                 C.c_double, C.c_int, C.c_int, C.c_int])
        L.ref_voronoi_sizes.argtypes = [C.c_void_p, C.POINTER(C.c_long)]
        L.ref_voronoi_copy.argtypes = [C.c_void_p, _ip, _dp, _dp, C.POINTER(C.c_long), C.POINTER(C.c_long), _dp, _ip,
                                       _ip, _dp, _dp, _dp, _dp]
        L.ref_voronoi_free.argtypes = [C.c_void_p]
        L.ref_pair_sample.restype = C.c_double
        L.ref_pair_sample.argtypes = ([C.c_long] + [_dp] * 5 + [_dp, C.c_int, C.c_int, C.c_int, C.c_char_p, C.c_double,
                                                              C.c_int, C.c_int, C.c_long, C.c_long,
                                                              C.POINTER(C.c_long), C.POINTER(C.c_long), _dp])
        L.ref_max_threads.restype = C.c_int
        L.ref_save_cartesian_grid.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int] + [_dp] * 5
        L.ref_save_mapping.argtypes = [C.c_char_p, C.c_long, C.POINTER(C.c_long)] + [_dp] * 8
        L.ref_voronoi_inverse_copy.argtypes = [C.c_void_p] + [_dp] * 4
        L.ref_voronoi_inverse_copy.restype = None
        L.ref_table_load_gridded.restype = C.c_int
        L.ref_table_load_gridded.argtypes = [C.c_char_p, C.c_int64] + [_dp] * 5
        L.ref_table_values.restype = C.c_int64
        L.ref_table_values.argtypes = [_dp]

    def cartesian_map(self, P, bounds, resolution, threads=1):
        """run_cartesian_map_stage on a fresh work folder: (points {id, xyz}, mapping rows {id, density, vx,
        vy, vz}, map {density, vx, vy, vz, cell_id})."""
        L = self.lib
        L.ref_cartesian_map.restype = C.c_void_p
        L.ref_cartesian_map.argtypes = [C.c_long] + [_dp] * 8 + [_dp, C.c_int, C.c_int]
        L.ref_cartesian_map_sizes.argtypes = [C.c_void_p, C.POINTER(C.c_long)]
        L.ref_cartesian_map_copy.argtypes = [C.c_void_p, _ip, _dp, _ip] + [_dp] * 8 + [_ip]
        L.ref_cartesian_map_free.argtypes = [C.c_void_p]
        arrs = [_f64(P[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "m", "h")]
        hnd = L.ref_cartesian_map(len(arrs[0]), *[_d(a) for a in arrs], _d(_f64(bounds)), int(resolution), threads)
        if not hnd:
            raise RuntimeError("reference cartesian map failed: " + L.ref_last_error().decode())
        sz = (C.c_long * 3)()
        L.ref_cartesian_map_sizes(hnd, sz)
        npt, nrow, nq = sz[0], sz[1], sz[2]
        pts = {"id": np.zeros(npt, np.int32), "xyz": np.zeros(3 * npt)}
        rows = {"id": np.zeros(nrow, np.int32), **{k: np.zeros(nrow) for k in ("density", "vx", "vy", "vz")}}
        mp = {**{k: np.zeros(nq) for k in ("density", "vx", "vy", "vz")}, "cell_id": np.zeros(nq, np.int32)}
        L.ref_cartesian_map_copy(hnd, pts["id"].ctypes.data_as(_ip), _d(pts["xyz"]), rows["id"].ctypes.data_as(_ip),
                                 *[_d(rows[k]) for k in ("density", "vx", "vy", "vz")],
                                 *[_d(mp[k]) for k in ("density", "vx", "vy", "vz")], mp["cell_id"].ctypes.data_as(_ip))
        L.ref_cartesian_map_free(hnd)
        return pts, rows, mp

    def coverage_grid_buffer(self, P, bounds, spacing_fraction=0.05, factor=2.0):
        """The reference's add_coverage_grid_buffer on the particles as the point set: the appended points,
        (xyz (k, 3), ids (k,)) (RuntimeError with its message when it throws)."""
        f = self.lib.ref_coverage_grid_buffer
        f.restype = C.c_long
        f.argtypes = [C.c_long] + [_dp] * 5 + [C.c_double, C.c_double, _dp, _ip, C.c_long]
        a = [_f64(P[k]) for k in ("x", "y", "z", "h")]
        cap = 1 << 22
        xyz = np.zeros(3 * cap)
        ids = np.zeros(cap, dtype=np.int32)
        k = f(len(a[0]), *[_d(v) for v in a], _d(_f64(bounds)), spacing_fraction, factor, _d(xyz),
              ids.ctypes.data_as(_ip), cap)
        if k < 0:
            raise RuntimeError(self.lib.ref_last_error().decode())
        return xyz[:3 * k].reshape(-1, 3).copy(), ids[:k].copy()

    def container_order(self, sites, bounds, scale=3.0):
        """The site indices a container built as the reference builds it keeps, in c_loop_all order."""
        f = self.lib.ref_container_order
        f.restype = C.c_long
        f.argtypes = [C.c_long, _dp, _dp, C.c_double, C.POINTER(C.c_long)]
        xyz = _f64(np.asarray(sites, dtype=np.float64).reshape(-1))
        n = len(xyz) // 3
        out = np.zeros(max(n, 1), dtype=np.int64)
        k = f(n, _d(xyz), _d(_f64(bounds)), scale, out.ctypes.data_as(C.POINTER(C.c_long)))
        return out[:k]

    def lloyd_step(self, xyz, ids, bounds, scale=3.0):
        """The reference's lloyd_step: (ids, xyz (k, 3)) in the container's walk order."""
        f = self.lib.ref_lloyd_step
        f.restype = C.c_long
        f.argtypes = [C.c_long, _ip, _dp, _dp, C.c_double, _ip, _dp, C.c_long]
        xyz = _f64(np.asarray(xyz, dtype=np.float64).reshape(-1))
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        n = len(ids)
        oid = np.zeros(max(n, 1), dtype=np.int32)
        oxyz = np.zeros(3 * max(n, 1))
        k = f(n, ids.ctypes.data_as(_ip), _d(xyz), _d(_f64(bounds)), scale, oid.ctypes.data_as(_ip), _d(oxyz), n)
        if k < 0:
            raise RuntimeError(self.lib.ref_last_error().decode())
        return oid[:k].copy(), oxyz[:3 * k].reshape(-1, 3).copy()

    def locate_sample(self, xyz, ids, bounds, res, ix_begin, ix_end, threads=0):
        """The stage's point location over x-slabs [ix_begin, ix_end): (seconds, owning site id per cell,
        seconds of it spent building the per-thread containers)."""
        f = self.lib.ref_locate_sample
        f.restype = C.c_double
        f.argtypes = [C.c_long, _ip, _dp, _dp, C.c_int, C.c_int, C.c_int, C.c_int, _ip, _dp]
        xyz = _f64(np.asarray(xyz, dtype=np.float64).reshape(-1))
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        out = np.zeros((ix_end - ix_begin) * res * res, dtype=np.int32)
        build = C.c_double(0.0)
        sec = f(len(ids), ids.ctypes.data_as(_ip), _d(xyz), _d(_f64(bounds)), int(res), int(ix_begin), int(ix_end),
                int(threads), out.ctypes.data_as(_ip), C.byref(build))
        return sec, out, build.value

    def save_cartesian_map(self, path, res, bounds, density, vx, vy, vz, cell_id):
        f = self.lib.ref_save_cartesian_map
        f.argtypes = [C.c_char_p, C.c_int] + [_dp] * 5 + [_ip]
        cid = np.ascontiguousarray(cell_id, dtype=np.int32)
        if f(path.encode(), int(res), *[_d(_f64(a)) for a in (bounds, density, vx, vy, vz)],
             cid.ctypes.data_as(_ip)) != 0:
            raise RuntimeError(self.lib.ref_last_error().decode())

    def table_load_gridded(self, path, h, phi, r0, R0):
        """load_density_table(path), then gridded_integral with that table over the arrays (RuntimeError
        with the reference's message when loading fails)."""
        a = [_f64(np.atleast_1d(v)) for v in (h, phi, r0, R0)]
        out = np.empty(a[0].size)
        if self.lib.ref_table_load_gridded(os.fsencode(path), out.size, *[_d(v) for v in a], _d(out)) != 0:
            raise RuntimeError(self.lib.ref_last_error().decode())
        return out

    def table_values(self) -> np.ndarray:
        """generate_density_table()'s values, flat, laid out as DensityLookupTable::at."""
        n = self.lib.ref_table_values(None)
        out = np.empty(n)
        self.lib.ref_table_values(_d(out))
        return out

    def save_cartesian_grid(self, path, shape, bounds, density, vx, vy, vz):
        arrs = [_f64(a) for a in (bounds, density, vx, vy, vz)]
        if self.lib.ref_save_cartesian_grid(path.encode(), *[int(s) for s in shape], *[_d(a) for a in arrs]) != 0:
            raise RuntimeError(self.lib.ref_last_error().decode())

    def save_inverse_mapping_test(self, path, ids, m_original, m_recovered, coverage, totals):
        ids = np.ascontiguousarray(ids, dtype=np.int64)
        arrs = [_f64(a) for a in (m_original, m_recovered, coverage, totals)]
        f = self.lib.ref_save_inverse_mapping_test
        f.argtypes = [C.c_char_p, C.c_long, C.POINTER(C.c_long)] + [_dp] * 4
        if f(path.encode(), len(ids), ids.ctypes.data_as(C.POINTER(C.c_long)), *[_d(a) for a in arrs]) != 0:
            raise RuntimeError(self.lib.ref_last_error().decode())

    def save_mapping(self, path, ids, x, y, z, volume, density, vx, vy, vz):
        ids = np.ascontiguousarray(ids, dtype=np.int64)
        arrs = [_f64(a) for a in (x, y, z, volume, density, vx, vy, vz)]
        if self.lib.ref_save_mapping(path.encode(), len(ids), ids.ctypes.data_as(C.POINTER(C.c_long)),
                                     *[_d(a) for a in arrs]) != 0:
            raise RuntimeError(self.lib.ref_last_error().decode())

    def max_threads(self):
        return self.lib.ref_max_threads()

    def load_snapshot(self, path, hfact=1.2):
        """The reference's own snapshot reader (load_sph_snapshot, format detected): dict of x y z vx vy vz m h."""
        self.lib.ref_load_snapshot.restype = C.c_long
        self.lib.ref_load_snapshot.argtypes = [C.c_char_p, C.c_double, C.c_void_p]
        n = self.lib.ref_load_snapshot(path.encode(), hfact, None)
        if n < 0:
            raise RuntimeError("reference snapshot reader failed: " + self.lib.ref_last_error().decode())
        keys = ("x", "y", "z", "vx", "vy", "vz", "m", "h")
        cols = [np.zeros(n) for _ in keys]
        ptrs = (C.POINTER(C.c_double) * 8)(*[_d(c) for c in cols])
        if self.lib.ref_load_snapshot(path.encode(), hfact, C.cast(ptrs, C.c_void_p)) != n:
            raise RuntimeError("reference snapshot reader failed: " + self.lib.ref_last_error().decode())
        return dict(zip(keys, cols))

    def pair_sample(self, P, bounds, shape, kernel="cubic_spline", support_in_h=0.0, generic_path=False, threads=0,
                    p_range=None):
        """The reference's pair-integral loop over a particle range, OpenMP: (seconds, bbox pairs, sphere
        pairs, checksum)."""
        arrs = [_f64(P[k]) for k in ("x", "y", "z", "m", "h")]
        n = len(arrs[0])
        pb, pe = (0, n) if p_range is None else p_range
        pairs = C.c_long(0)
        sphere = C.c_long(0)
        cs = C.c_double(0)
        b = _f64(bounds)
        t = self.lib.ref_pair_sample(n, *[_d(a) for a in arrs], _d(b), *[int(s) for s in shape], kernel.encode(),
                                     support_in_h, int(generic_path), threads, pb, pe, C.byref(pairs), C.byref(sphere),
                                     C.byref(cs))
        return t, pairs.value, sphere.value, cs.value

    def full_integral_new(self, h, phi, r0, R0):
        return self.lib.ref_full_integral_new(h, phi, r0, R0)

    def generic_full_integral(self, kernel, H, phi, r0, R0):
        return self.lib.ref_generic_full_integral(kernel, H, phi, r0, R0)

    def gridded_integral(self, h, phi, r0, R0):
        return self.lib.ref_gridded_integral(h, phi, r0, R0)

    def face_integral(self, x0, y0, z0, verts, kernel=-1, h=1.0, support=None, tabulated=False):
        v = _f64(verts).reshape(-1)
        ov = C.c_int(0)
        sup = support if support is not None else 2.0 * h
        r = self.lib.ref_face_integral(x0, y0, z0, kernel, h, sup, int(tabulated), _d(v), len(v) // 3, C.byref(ov))
        return r, ov.value

    def sph_to_grid(self, P, bounds, shape, kernel="cubic_spline", support_in_h=0.0, generic_path=False,
                    tabulated=False, threads=0):
        arrs = [_f64(P[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "m", "h")]
        n = len(arrs[0])
        nx, ny, nz = shape
        nc = nx * ny * nz
        outs = [np.zeros(nc) for _ in range(4)]
        b = _f64(bounds)
        rc = self.lib.ref_sph_to_grid(n, *[_d(a) for a in arrs], _d(b), nx, ny, nz, kernel.encode(), support_in_h,
                                      int(generic_path), int(tabulated), threads, *[_d(o) for o in outs])
        if rc != 0:
            raise RuntimeError("reference sph-to-grid failed: " + self.lib.ref_last_error().decode())
        return tuple(outs)

    def voronoi(self, P, bounds, buffer=False, spacing_fraction=0.0, lloyd=0, kernel="cubic_spline",
                support_in_h=0.0, generic_path=False, threads=0, run_map=True):
        """Cell geometry (CSR, as src/mapping.cpp builds it), home cells and, if run_map, the reference's
        own mapping.dat values per cell; with run_map=2 also the inverse-mapping check's results
        (run_inverse_mapping_test_stage: per-particle recovered mass and coverage, totals, cell masses)."""
        arrs = [_f64(P[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "m", "h")]
        n = len(arrs[0])
        b = _f64(bounds)
        hnd = self.lib.ref_voronoi_build(n, *[_d(a) for a in arrs], _d(b), int(buffer), spacing_fraction, lloyd,
                                         kernel.encode(), support_in_h, int(generic_path), threads, int(run_map))
        if not hnd:
            raise RuntimeError("reference voronoi failed: " + self.lib.ref_last_error().decode())
        sz = (C.c_long * 4)()
        self.lib.ref_voronoi_sizes(hnd, sz)
        nc, nf, nv, npart = sz[0], sz[1], sz[2], sz[3]
        g = {
            "id": np.zeros(nc, np.int32), "site": np.zeros(3 * nc), "volume": np.zeros(nc),
            "face_off": np.zeros(nc + 1, np.int64), "vert_off": np.zeros(nf + 1, np.int64),
            "vxyz": np.zeros(3 * nv), "face_nbr": np.zeros(nf, np.int32), "home": np.zeros(npart, np.int32),
        }
        res = [np.zeros(nc) for _ in range(4)]
        lp = C.POINTER(C.c_long)
        self.lib.ref_voronoi_copy(hnd, g["id"].ctypes.data_as(_ip), _d(g["site"]), _d(g["volume"]),
                                  g["face_off"].ctypes.data_as(lp), g["vert_off"].ctypes.data_as(lp), _d(g["vxyz"]),
                                  g["face_nbr"].ctypes.data_as(_ip), g["home"].ctypes.data_as(_ip),
                                  *[_d(r) for r in res])
        if run_map == 2:
            inv = {"m_recovered": np.zeros(npart), "coverage": np.zeros(npart), "totals": np.zeros(3),
                   "cell_mass": np.zeros(nc)}
            self.lib.ref_voronoi_inverse_copy(hnd, _d(inv["m_recovered"]), _d(inv["coverage"]), _d(inv["totals"]),
                                              _d(inv["cell_mass"]))
            self.lib.ref_voronoi_free(hnd)
            return g, res, inv
        self.lib.ref_voronoi_free(hnd)
        return g, (res if run_map else None)


def load_oracle():
    return Oracle()


ORACLE_COUNT_SO = os.path.join(HERE, "liboracle_count.so")


class CountingOracle(Oracle):
    """The oracle over an operation-counting double (oracle/kiwi_oracle_count.cpp)."""

    def __init__(self, path: str = ORACLE_COUNT_SO):
        super().__init__(path=path, prefix="orc_")
        self.lib.orc_counts.argtypes = [C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]

    def reset(self):
        self.lib.orc_reset()

    def counts(self):
        f, t = C.c_uint64(0), C.c_uint64(0)
        self.lib.orc_counts(C.byref(f), C.byref(t))
        return f.value, t.value


def load_truth():
    """The __float128 oracle (the error yardstick)."""
    return Oracle(quad=True)


def load_ref():
    """The reference library, or None when it was not built on this machine."""
    try:
        return RefLib()
    except (FileNotFoundError, OSError):
        return None
