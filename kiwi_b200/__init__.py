"""kiwi_b200: B200-native KIWI kernel-integral engine -- Python host binding over the C ABI.

The names mirror the reference's C++ kernel-integral layer and stages (mapetkova/kiwi):

  get_kernel(name)                                      include/kiwi/kernel_spec.hpp:41-44
  full_integral_new(h, phi, r0, R_0)                    include/kiwi/kernel_integral.hpp:80
  generic_full_integral(K, H, phi, r0, R_0)             include/kiwi/kernel_integral_generic.hpp:56
  compute_face_integral(x0, y0, z0, h, verts)           include/kiwi/kernel_integral.hpp:182-184
  compute_face_integral_generic(x0, y0, z0, K, H, v)    include/kiwi/kernel_integral.hpp:192-193
  KernelIntegrator / make_kernel_integrator             include/kiwi/kernel_integrator.hpp:14-45
  sph_to_grid(...) -> CartesianGridResult               src/cartesian_grid.cpp:76-321 (the stage's compute)

Every call runs on the GPU through libkiwi_b200.so (hand-written sm_100a kernels).  There is no CPU
fallback: if the library or a usable GPU is missing, calls raise KiwiError.  Scalar functions accept
NumPy arrays and evaluate them as one batched launch.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("KIWI_B200_LIB") or os.path.join(HERE, "libkiwi_b200.so")

KIWI_FP64 = 0
KIWI_FP32_MIXED = 1
KIWI_FP64_REFERENCE_ORDER = 2
KIWI_FP32_GUARANTEE = 0x200
PRECISIONS = {"fp64": KIWI_FP64, "fp32_mixed": KIWI_FP32_MIXED, "fp64_reference_order": KIWI_FP64_REFERENCE_ORDER,
              "fp32_mixed_guaranteed": KIWI_FP32_MIXED | KIWI_FP32_GUARANTEE}

KERNEL_KEYS = ["M4", "M5", "M6", "WC2", "WC4", "WC6"]
KERNEL_NAMES = ["cubic_spline", "quartic_spline", "quintic_spline", "wendland_c2", "wendland_c4", "wendland_c6"]

_ERRORS = {-1: "invalid argument", -2: "CUDA error", -3: "no usable GPU", -4: "device allocation failed",
           -5: "iteration limit hit", -6: "unsupported option"}


class KiwiError(RuntimeError):
    """Raised for any failed call: the Python form of the reference's `[kiwi] error: <what>`."""

    def __init__(self, code: int, what: str):
        super().__init__(f"[kiwi] error: {what}")
        self.code = code


_dp = C.POINTER(C.c_double)
_i32p = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)


class KiwiParticles(C.Structure):
    _fields_ = [("n", C.c_int64)] + [(k, _dp) for k in ("x", "y", "z", "vx", "vy", "vz", "m", "h")]


class KiwiCartGrid(C.Structure):
    _fields_ = [("bounds", C.c_double * 6), ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32)]


class KiwiKernelSel(C.Structure):
    _fields_ = [("kernel", C.c_int32), ("support_in_h", C.c_double), ("generic_path", C.c_int32),
                ("tabulated", C.c_int32)]


class KiwiStats(C.Structure):
    _fields_ = [("bbox_pairs", C.c_int64), ("sphere_pairs", C.c_int64), ("evaluated_pairs", C.c_int64),
                ("skipped_outside", C.c_int64), ("neg_clamped", C.c_int64), ("neg_warned", C.c_int64),
                ("fp64_fallback", C.c_int64), ("tile_pairs", C.c_int64), ("launches", C.c_int64), ("gather_ms", C.c_double),
                ("total_ms", C.c_double), ("edge_tiers_outer", C.c_int64), ("edge_tiers_middle", C.c_int64),
                ("edge_tiers_inner", C.c_int64), ("vertex_pyramids", C.c_int64), ("fp64_tiles", C.c_int64),
                ("table_clamps", C.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class KiwiDensityTableInfo(C.Structure):
    _fields_ = [(k, C.c_int32) for k in ("nr01", "nR_01", "nphi1", "nr02", "nR_02", "nphi2")] + \
               [(k, C.c_double) for k in ("rl", "mul", "cphil")] + [("n_values", C.c_int64)]


class KiwiBatchItem(C.Structure):
    _fields_ = [("particles", KiwiParticles), ("grid", KiwiCartGrid), ("kernel", KiwiKernelSel),
                ("density", _dp), ("vx", _dp), ("vy", _dp), ("vz", _dp), ("raw4", _dp)]


class KiwiVoronoiCells(C.Structure):
    _fields_ = [("n_cells", C.c_int64), ("face_off", _i64p), ("vert_off", _i64p), ("vxyz", _dp),
                ("face_nbr", _i32p), ("volume", _dp)]


_lib = None


def load_library(path: str = LIB_PATH):
    """Loads libkiwi_b200.so (built in-tree by kiwi_b200.build); raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise KiwiError(-6, f"{path} is missing: build it with `python -m kiwi_b200.build`")
    L = C.CDLL(path)
    L.kiwi_version.restype = C.c_char_p
    L.kiwi_ctx_create.argtypes = [C.c_int, C.POINTER(C.c_void_p)]
    L.kiwi_ctx_destroy.argtypes = [C.c_void_p]
    L.kiwi_last_error.restype = C.c_char_p
    L.kiwi_last_error.argtypes = [C.c_void_p]
    L.kiwi_ctx_stream.restype = C.c_void_p
    L.kiwi_ctx_stream.argtypes = [C.c_void_p]
    L.kiwi_ctx_synchronize.argtypes = [C.c_void_p]
    L.kiwi_ctx_set_voronoi_face_tables.argtypes = [C.c_void_p, C.c_int]
    L.kiwi_kernel_index.argtypes = [C.c_char_p]
    L.kiwi_kernel_info.argtypes = [C.c_int, _dp]
    L.kiwi_full_integral_batch.argtypes = [C.c_void_p, C.c_int, C.c_int64, _dp, _dp, _dp, _dp, _dp]
    L.kiwi_face_integral_batch.argtypes = [C.c_void_p, C.POINTER(KiwiKernelSel), C.c_int64, _dp, _i64p, _dp, _dp,
                                           _i32p]
    sig = [C.c_void_p, C.POINTER(KiwiParticles), C.POINTER(KiwiCartGrid), C.POINTER(KiwiKernelSel), C.c_int,
           _dp, _dp, _dp, _dp, _dp, C.POINTER(KiwiStats)]
    L.kiwi_sph_to_grid.argtypes = sig
    L.kiwi_sph_to_grid_device.argtypes = sig
    L.kiwi_sph_to_grid_device_part.argtypes = sig[:5] + [C.c_int, C.c_int] + sig[5:]
    L.kiwi_sph_to_grid_adjoint_device.argtypes = ([C.c_void_p, C.POINTER(KiwiParticles), C.POINTER(KiwiCartGrid),
                                                   C.POINTER(KiwiKernelSel), _dp] + [_dp] * 8 +
                                                  [C.POINTER(KiwiStats)])
    L.kiwi_batch_create.argtypes = [C.c_void_p, C.POINTER(KiwiBatchItem), C.c_int, C.c_int, C.POINTER(C.c_void_p)]
    L.kiwi_batch_run.argtypes = [C.c_void_p, C.POINTER(KiwiStats), C.POINTER(KiwiStats)]
    L.kiwi_batch_tune.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
    L.kiwi_batch_destroy.argtypes = [C.c_void_p]
    L.kiwi_map_voronoi.argtypes = [C.c_void_p, C.POINTER(KiwiParticles), _i32p, C.POINTER(KiwiVoronoiCells),
                                   C.POINTER(KiwiKernelSel), C.c_int, _dp, _dp, _dp, _dp, _dp, C.POINTER(KiwiStats)]
    L.kiwi_density_table_generate.argtypes = [C.c_void_p]
    L.kiwi_density_table_load.argtypes = [C.c_void_p, C.c_char_p]
    L.kiwi_density_table_info.argtypes = [C.c_void_p, C.POINTER(KiwiDensityTableInfo)]
    L.kiwi_density_table_read.argtypes = [C.c_void_p, _dp, C.c_int64]
    L.kiwi_density_table_release.argtypes = [C.c_void_p]
    L.kiwi_density_table_release.restype = None
    L.kiwi_gridded_integral_batch.argtypes = [C.c_void_p, C.c_int64, _dp, _dp, _dp, _dp, _dp, C.POINTER(C.c_int64)]
    _lib = L
    return L


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _p(a):
    return a.ctypes.data_as(_dp) if a is not None else None


class KernelSpec:
    """A kernel of the table (the KernelSpec of include/kiwi/kernel_spec.hpp:18-44)."""

    def __init__(self, index: int):
        out = (C.c_double * 7)()
        rc = load_library().kiwi_kernel_info(index, out)
        if rc != 0:
            raise KiwiError(rc, f"unknown kernel index {index}")
        self.index = index
        self.key = KERNEL_KEYS[index]
        self.name = KERNEL_NAMES[index]
        self.nreg = int(out[0])
        self.A2_pi, self.A3_pi, self.radkern, self.hfact = out[1], out[2], out[3], out[4]

    def __repr__(self):
        return f"KernelSpec({self.key})"


def get_kernel(name: str) -> KernelSpec:
    """Kernel by key or alias, case-insensitive; unknown names raise (std::invalid_argument)."""
    k = load_library().kiwi_kernel_index(str(name).encode())
    if k < 0:
        raise KiwiError(-1, f"kernel.name: unknown kernel '{name}' (expected one of: cubic_spline, quartic_spline, "
                            "quintic_spline, wendland_c2, wendland_c4, wendland_c6)")
    return KernelSpec(k)


class Context:
    """One GPU context (stream, scratch memory).  One per host thread."""

    def __init__(self, device: int = 0):
        L = load_library()
        h = C.c_void_p()
        rc = L.kiwi_ctx_create(int(device), C.byref(h))
        if rc != 0:
            raise KiwiError(rc, f"kiwi_ctx_create(device={device}) failed: {_ERRORS.get(rc, rc)}")
        self._h = h
        self._L = L

    @property
    def handle(self):
        return self._h

    @property
    def stream(self) -> int:
        return self._L.kiwi_ctx_stream(self._h)

    def check(self, rc: int, what: str = ""):
        if rc != 0:
            msg = self._L.kiwi_last_error(self._h).decode()
            raise KiwiError(rc, (what + ": " if what else "") + (msg or _ERRORS.get(rc, str(rc))))

    def synchronize(self):
        self.check(self._L.kiwi_ctx_synchronize(self._h))

    def set_voronoi_face_tables(self, enable: bool):
        """Voronoi maps: each face value evaluated once through per-(pair, face) tables (True, the default)
        or in one launch that evaluates a shared face on both sides (False); the results are equal."""
        self.check(self._L.kiwi_ctx_set_voronoi_face_tables(self._h, int(bool(enable))))

    def close(self):
        if getattr(self, "_h", None):
            self._L.kiwi_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(int(os.environ.get("KIWI_DEVICE", "0")))
    return _default_ctx


# ---------------------------------------------------------------------------------------------- scalar API

def _batch(fn_kernel: int, arg0, phi, r0, R0, ctx=None):
    ctx = ctx or default_context()
    a0, ph, a, b = np.broadcast_arrays(_f64(arg0), _f64(phi), _f64(r0), _f64(R0))
    shape = a0.shape
    a0, ph, a, b = (_f64(x).reshape(-1) for x in (a0, ph, a, b))
    out = np.empty(a0.size)
    ctx.check(ctx._L.kiwi_full_integral_batch(ctx.handle, fn_kernel, a0.size, _p(a0), _p(ph), _p(a), _p(b), _p(out)),
              "full_integral")
    return out.reshape(shape) if shape else float(out[0])


def full_integral_new(h, phi, r0, R_0, ctx=None):
    """Closed-form cubic-spline vertex-pyramid integral (src/kernel_integral.cpp:410-418), batched."""
    return _batch(-1, h, phi, r0, R_0, ctx)


def generic_full_integral(K, H, phi, r0, R_0, ctx=None):
    """Generic-kernel vertex-pyramid integral (src/kernel_integral_generic.cpp:216-221), batched."""
    k = K.index if isinstance(K, KernelSpec) else get_kernel(K).index
    return _batch(k, H, phi, r0, R_0, ctx)


def _sel(kernel=0, support_in_h=0.0, generic_path=False, tabulated=False) -> KiwiKernelSel:
    k = kernel.index if isinstance(kernel, KernelSpec) else (kernel if isinstance(kernel, int) else get_kernel(kernel).index)
    return KiwiKernelSel(k, float(support_in_h), int(bool(generic_path)), int(bool(tabulated)))


def face_integrals(particles, faces, kernel=0, support_in_h=0.0, generic_path=False, ctx=None, tabulated=False):
    """Batched face integrals: particles (n, 4) = (x0, y0, z0, h); faces: list of (nv, 3) vertex arrays in
    the face's winding.  Returns (values, out_vert).  tabulated: the cubic spline's lookup table (the
    context's density table) instead of its closed form."""
    ctx = ctx or default_context()
    part = _f64(particles).reshape(-1, 4)
    n = part.shape[0]
    if len(faces) != n:
        raise KiwiError(-1, "one face per particle row is required")
    nv = np.array([len(np.asarray(f).reshape(-1, 3)) for f in faces], dtype=np.int64)
    off = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(nv, out=off[1:])
    verts = _f64(np.concatenate([_f64(f).reshape(-1) for f in faces]) if n else np.zeros(0))
    out = np.empty(n)
    ov = np.empty(n, dtype=np.int32)
    sel = _sel(kernel, support_in_h, generic_path, tabulated)
    ctx.check(ctx._L.kiwi_face_integral_batch(ctx.handle, C.byref(sel), n, _p(part), off.ctypes.data_as(_i64p),
                                              _p(verts), _p(out), ov.ctypes.data_as(_i32p)), "face_integral")
    return out, ov


def compute_face_integral(x0, y0, z0, h, vertices, out_vert=False, ctx=None, tabulated=False):
    """compute_face_integral(x0, y0, z0, h, tabulated, table, vertices, &out_vert): cubic spline, support 2h;
    with tabulated, the lookups go to the context's density table."""
    v, ov = face_integrals([[x0, y0, z0, h]], [vertices], kernel=0, support_in_h=2.0, ctx=ctx, tabulated=tabulated)
    return (float(v[0]), int(ov[0])) if out_vert else float(v[0])


def compute_face_integral_generic(x0, y0, z0, K, H, vertices, out_vert=False, ctx=None):
    """compute_face_integral_generic(x0, y0, z0, K, H, vertices, &out_vert)."""
    k = K if isinstance(K, KernelSpec) else get_kernel(K)
    # H is passed as h = H / support_in_h with support_in_h = 1 on the generic path
    v, ov = face_integrals([[x0, y0, z0, H]], [vertices], kernel=k.index, support_in_h=1.0, generic_path=True, ctx=ctx)
    return (float(v[0]), int(ov[0])) if out_vert else float(v[0])


# ---- tabulated cubic integral (DensityLookupTable, include/kiwi/kernel_integral.hpp:21-72)

def generate_density_table(ctx=None):
    """generate_density_table (src/kernel_integral.cpp:57-119): the canonical table, computed on the GPU into
    the context.  Returns its shape (density_table_info)."""
    ctx = ctx or default_context()
    ctx.check(ctx._L.kiwi_density_table_generate(ctx.handle), "generate_density_table")
    return density_table_info(ctx)


def load_density_table(path, ctx=None):
    """load_density_table (src/kernel_integral.cpp:20-55): the reference's text format, into the context
    (KiwiError with the reference's messages on a missing, malformed or truncated file)."""
    ctx = ctx or default_context()
    ctx.check(ctx._L.kiwi_density_table_load(ctx.handle, os.fsencode(path)), "load_density_table")
    return density_table_info(ctx)


def density_table_info(ctx=None) -> dict:
    ctx = ctx or default_context()
    info = KiwiDensityTableInfo()
    ctx.check(ctx._L.kiwi_density_table_info(ctx.handle, C.byref(info)), "density_table_info")
    return {k: getattr(info, k) for k, _ in info._fields_}


def density_table_values(ctx=None) -> np.ndarray:
    """The context's table values, shape (nr0 + 2, nR_0 + 1, nphi + 1), indexed as DensityLookupTable::at."""
    ctx = ctx or default_context()
    d = density_table_info(ctx)
    out = np.empty(d["n_values"])
    ctx.check(ctx._L.kiwi_density_table_read(ctx.handle, _p(out), out.size), "density_table_read")
    return out.reshape(d["nr01"] + d["nr02"] + 2, d["nR_01"] + d["nR_02"] + 1, d["nphi1"] + d["nphi2"] + 1)


def release_density_table(ctx=None):
    ctx = ctx or default_context()
    ctx._L.kiwi_density_table_release(ctx.handle)


def gridded_integral(h, phi, r0, R_0, ctx=None, return_clamps=False):
    """gridded_integral(table, h, phi, r0, R_0) (src/kernel_integral.cpp:136-190), batched over broadcast
    arrays, with the context's density table (the canonical one is generated if none is loaded).  With
    return_clamps, also the number of lookup indices clamped into the table (the reference prints a
    warning for each)."""
    ctx = ctx or default_context()
    a = np.broadcast_arrays(*[np.asarray(v, dtype=np.float64) for v in (h, phi, r0, R_0)])
    shape = a[0].shape
    a = [_f64(v.reshape(-1)) for v in a]
    n = a[0].size
    out = np.empty(n)
    cl = C.c_int64(0)
    ctx.check(ctx._L.kiwi_gridded_integral_batch(ctx.handle, n, *[_p(v) for v in a], _p(out), C.byref(cl)),
              "gridded_integral")
    res = out.reshape(shape) if shape else float(out[0])
    return (res, cl.value) if return_clamps else res


@dataclass
class KernelIntegrator:
    """Dispatch of make_kernel_integrator (include/kiwi/kernel_integrator.hpp:35-45)."""
    kernel: int = 0
    support_in_h: float = 0.0
    generic_path: bool = False
    tabulated: bool = False

    @property
    def generic(self) -> bool:
        s = self.support_in_h or KernelSpec(self.kernel).radkern
        return self.generic_path or self.kernel != 0 or s != 2.0

    def support(self, h):
        return (self.support_in_h or KernelSpec(self.kernel).radkern) * h

    def sel(self) -> KiwiKernelSel:
        return _sel(self.kernel, self.support_in_h, self.generic_path, self.tabulated)


def make_kernel_integrator(name="cubic_spline", support_radius_in_h=0.0, generic_path=False,
                           use_tabulated_integral=False) -> KernelIntegrator:
    return KernelIntegrator(get_kernel(name).index, float(support_radius_in_h), bool(generic_path),
                            bool(use_tabulated_integral))


# ---------------------------------------------------------------------------------------------- stages

@dataclass
class CartesianGridResult:
    """include/kiwi/cartesian_grid.hpp:53-71; arrays are flat, x-major: (ix*ny + iy)*nz + iz."""
    nx: int
    ny: int
    nz: int
    bounds: tuple
    density: np.ndarray
    vx: np.ndarray
    vy: np.ndarray
    vz: np.ndarray
    raw: np.ndarray | None = None
    stats: dict = field(default_factory=dict)


def _particles_struct(P: dict, device: bool = False):
    keys = ("x", "y", "z", "vx", "vy", "vz", "m", "h")
    if device:
        ptrs = [C.cast(C.c_void_p(int(P[k].data_ptr())), _dp) for k in keys]
        n = int(P["x"].numel())
        keep = None
    else:
        keep = [_f64(P[k]) for k in keys]
        n = len(keep[0])
        for a in keep:
            if len(a) != n:
                raise KiwiError(-1, "particle arrays differ in length")
        ptrs = [_p(a) for a in keep]
    return KiwiParticles(n, *ptrs), keep


KIWI_FULL_BOX = 0x100


def precision_code(precision="fp64", full_box=False) -> int:
    """The C ABI's precision argument: the arithmetic form, plus KIWI_FULL_BOX to evaluate every cell of
    each particle's support bounding box as the reference does (default: only the cells the support
    reaches)."""
    code = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
    return code | (KIWI_FULL_BOX if full_box else 0)


def sph_to_grid(particles: dict, bounds, shape, kernel=None, precision="fp64", raw=False, ctx=None, out=None,
                full_box=False):
    """Density and mass-weighted velocity of an SPH snapshot on a Cartesian grid -- the compute of
    run_sph_to_grid_stage (src/cartesian_grid.cpp:76-321) on host arrays.  `particles` maps x y z vx vy
    vz m h to 1-D arrays; `bounds` = (x_min, x_max, y_min, y_max, z_min, z_max); `shape` = (nx, ny, nz);
    `kernel` a KernelIntegrator (default: cubic spline); `out`: optional preallocated float64 arrays
    (density, vx, vy, vz), e.g. in pinned memory."""
    ctx = ctx or default_context()
    ki = kernel or KernelIntegrator()
    Ps, keep = _particles_struct(particles)
    nx, ny, nz = (int(s) for s in shape)
    grid = KiwiCartGrid((C.c_double * 6)(*[float(b) for b in bounds]), nx, ny, nz)
    nc = nx * ny * nz
    if out is not None:
        outs = list(out)
        if len(outs) != 4 or any(o.dtype != np.float64 or o.size != nc or not o.flags.c_contiguous for o in outs):
            raise KiwiError(-1, "out must be 4 contiguous float64 arrays of nx*ny*nz cells")
    else:
        outs = [np.empty(nc) for _ in range(4)]
    rawa = np.empty(4 * nc) if raw else None
    st = KiwiStats()
    sel = ki.sel()
    ctx.check(ctx._L.kiwi_sph_to_grid(ctx.handle, C.byref(Ps), C.byref(grid), C.byref(sel),
                                      precision_code(precision, full_box), *[_p(o) for o in outs], _p(rawa),
                                      C.byref(st)), "sph-to-grid")
    return CartesianGridResult(nx, ny, nz, tuple(bounds), *outs, raw=rawa.reshape(4, nc) if raw else None,
                               stats=st.as_dict())


def sph_to_grid_device(particles: dict, bounds, shape, out: dict, kernel=None, precision="fp64", ctx=None,
                       full_box=False, part=0, n_parts=1):
    """Device variant: `particles` and `out` (density, vx, vy, vz[, raw4]) hold CUDA tensors (float64,
    contiguous).  Runs on the context's stream and returns the call's stats.  With n_parts > 1 only the
    cells of the tiles owned by `part` are computed and written (kiwi_sph_to_grid_device_part): one part
    per GPU splits one grid over several GPUs."""
    ctx = ctx or default_context()
    ki = kernel or KernelIntegrator()
    Ps, _ = _particles_struct(particles, device=True)
    nx, ny, nz = (int(s) for s in shape)
    grid = KiwiCartGrid((C.c_double * 6)(*[float(b) for b in bounds]), nx, ny, nz)
    st = KiwiStats()
    sel = ki.sel()

    def dp(t):
        return C.cast(C.c_void_p(int(t.data_ptr())), _dp) if t is not None else None

    outs = [dp(out.get(k)) for k in ("density", "vx", "vy", "vz", "raw4")]
    if n_parts == 1:
        ctx.check(ctx._L.kiwi_sph_to_grid_device(ctx.handle, C.byref(Ps), C.byref(grid), C.byref(sel),
                                                 precision_code(precision, full_box), *outs, C.byref(st)),
                  "sph-to-grid")
    else:
        ctx.check(ctx._L.kiwi_sph_to_grid_device_part(ctx.handle, C.byref(Ps), C.byref(grid), C.byref(sel),
                                                      precision_code(precision, full_box), int(part), int(n_parts),
                                                      *outs, C.byref(st)), "sph-to-grid part")
    return st.as_dict()


def sph_to_grid_adjoint_device(particles: dict, bounds, shape, raw4_cot, grads: dict, kernel=None, ctx=None):
    """Adjoint of the raw sums (no counterpart in the reference): `particles` holds CUDA float64 tensors,
    `raw4_cot` the cotangents dL/dM, dL/dPx, dL/dPy, dL/dPz (4 * ncells, CUDA float64), `grads` maps any of
    x y z h m vx vy vz to CUDA float64 tensors that receive dL/d(that input).  Returns the call's stats."""
    ctx = ctx or default_context()
    ki = kernel or KernelIntegrator()
    Ps, _ = _particles_struct(particles, device=True)
    nx, ny, nz = (int(s) for s in shape)
    grid = KiwiCartGrid((C.c_double * 6)(*[float(b) for b in bounds]), nx, ny, nz)
    st = KiwiStats()
    sel = ki.sel()

    def dp(t):
        return C.cast(C.c_void_p(int(t.data_ptr())), _dp) if t is not None else None

    outs = [dp(grads.get(k)) for k in ("x", "y", "z", "h", "m", "vx", "vy", "vz")]
    ctx.check(ctx._L.kiwi_sph_to_grid_adjoint_device(ctx.handle, C.byref(Ps), C.byref(grid), C.byref(sel),
                                                     dp(raw4_cot), *outs, C.byref(st)), "sph-to-grid adjoint")
    return st.as_dict()


class Batch:
    """Many sph-to-grid problems in one persistent, graph-recorded launch (kiwi_batch_create / run /
    tune / destroy; no counterpart in the reference).  `items` is a list of dicts with `particles` (CUDA
    float64 tensors x y z vx vy vz m h), `bounds`, `shape`, optional `kernel` (KernelIntegrator) and `out`
    (CUDA float64 tensors density vx vy vz [raw4]).  The tensors must stay alive while the batch is used;
    positions and smoothing lengths must not change after creation."""

    def __init__(self, items, precision="fp64", ctx=None):
        self.ctx = ctx or default_context()
        self._keep = []
        arr = (KiwiBatchItem * len(items))()

        def dp(t):
            return C.cast(C.c_void_p(int(t.data_ptr())), _dp) if t is not None else None

        for i, it in enumerate(items):
            Ps, _ = _particles_struct(it["particles"], device=True)
            nx, ny, nz = (int(v) for v in it["shape"])
            grid = KiwiCartGrid((C.c_double * 6)(*[float(b) for b in it["bounds"]]), nx, ny, nz)
            sel = (it.get("kernel") or KernelIntegrator()).sel()
            out = it.get("out", {})
            arr[i] = KiwiBatchItem(Ps, grid, sel, dp(out.get("density")), dp(out.get("vx")), dp(out.get("vy")),
                                   dp(out.get("vz")), dp(out.get("raw4")))
            self._keep.append((it["particles"], out))
        self.n_items = len(items)
        h = C.c_void_p()
        self.ctx.check(self.ctx._L.kiwi_batch_create(self.ctx.handle, arr, len(items),
                                                     precision_code(precision), C.byref(h)), "batch create")
        self._h = h

    def run(self):
        """Runs the batch; returns (per-item stats, total stats)."""
        st = (KiwiStats * self.n_items)()
        tot = KiwiStats()
        self.ctx.check(self.ctx._L.kiwi_batch_run(self._h, st, C.byref(tot)), "batch run")
        return [s.as_dict() for s in st], tot.as_dict()

    def tune(self):
        """Times the launch shapes and keeps the fastest; returns (longest_first, ctas_per_sm) and sets
        self.merged (both lattice families in one persistent launch)."""
        c = C.c_int(0)
        self.ctx.check(self.ctx._L.kiwi_batch_tune(self._h, C.byref(c)), "batch tune")
        self.merged = bool(c.value & 0x10000)
        return bool(c.value & 0x100), c.value & 0xff

    def close(self):
        if getattr(self, "_h", None):
            self.ctx._L.kiwi_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class MappingResult:
    """Per-cell results of the Voronoi map in the geometry's cell order (the MappingResult rows of
    include/kiwi/mapping.hpp:17-30 without the site coordinates)."""
    density: np.ndarray
    vx: np.ndarray
    vy: np.ndarray
    vz: np.ndarray
    raw: np.ndarray | None = None
    stats: dict = field(default_factory=dict)


def _io_lib():
    L = load_library()
    L.kiwi_save_cartesian_grid.argtypes = [C.c_char_p, C.c_int32, C.c_int32, C.c_int32] + [_dp] * 5 + [C.c_char_p,
                                                                                                   C.c_size_t]
    L.kiwi_load_cartesian_grid.argtypes = [C.c_char_p, C.POINTER(C.c_int32)] + [_dp] * 5 + [C.c_char_p, C.c_size_t]
    L.kiwi_save_mapping.argtypes = ([C.c_char_p, C.c_int64, _i64p] + [_dp] * 8 + [C.c_char_p, C.c_size_t])
    L.kiwi_save_cartesian_map.argtypes = [C.c_char_p, C.c_int32, _dp, _dp, _dp, _dp, _dp, _i32p, C.c_char_p,
                                          C.c_size_t]
    L.kiwi_load_cartesian_map.argtypes = [C.c_char_p, C.POINTER(C.c_int32), _dp, _dp, _dp, _dp, _dp, _i32p,
                                          C.c_char_p, C.c_size_t]
    L.kiwi_save_inverse_mapping_test.argtypes = ([C.c_char_p, C.c_int64, _i64p] + [_dp] * 4 +
                                                 [C.c_char_p, C.c_size_t])
    L.kiwi_load_inverse_mapping_test.argtypes = ([C.c_char_p, C.POINTER(C.c_int64), _dp, _i64p] + [_dp] * 3 +
                                                 [C.c_int64, C.c_char_p, C.c_size_t])
    return L


def _io_check(rc, err):
    if rc != 0:
        raise KiwiError(rc, err.value.decode() or "file error")


def save_cartesian_grid(result: CartesianGridResult, path: str):
    """save_cartesian_grid (src/cartesian_grid.cpp:323-347): the VGTCGRD2 file of a CartesianGridResult."""
    L = _io_lib()
    err = C.create_string_buffer(512)
    arrs = [_f64(a) for a in (result.density, result.vx, result.vy, result.vz)]
    b = _f64(result.bounds)
    _io_check(L.kiwi_save_cartesian_grid(path.encode(), result.nx, result.ny, result.nz, _p(b), *[_p(a) for a in arrs],
                                         err, len(err)), err)


def load_cartesian_grid(path: str) -> CartesianGridResult:
    """load_cartesian_grid (src/cartesian_grid.cpp:349-394)."""
    L = _io_lib()
    err = C.create_string_buffer(512)
    n = (C.c_int32 * 3)()
    b = np.zeros(6)
    _io_check(L.kiwi_load_cartesian_grid(path.encode(), n, _p(b), None, None, None, None, err, len(err)), err)
    nc = n[0] * n[1] * n[2]
    arrs = [np.empty(nc) for _ in range(4)]
    _io_check(L.kiwi_load_cartesian_grid(path.encode(), n, _p(b), *[_p(a) for a in arrs], err, len(err)), err)
    return CartesianGridResult(n[0], n[1], n[2], tuple(b), *arrs)


def save_mapping(path: str, ids, sites, volume, result):
    """save_mapping (src/mapping.cpp:307-315): mapping.dat rows "id x y z volume density vx vy vz" for the
    cells of a MappingResult (ids and site coordinates from the caller's tessellation)."""
    L = _io_lib()
    err = C.create_string_buffer(512)
    ids = np.ascontiguousarray(ids, dtype=np.int64)
    sites = np.asarray(sites, dtype=np.float64)
    arrs = [_f64(sites[:, 0]), _f64(sites[:, 1]), _f64(sites[:, 2]), _f64(volume), _f64(result.density),
            _f64(result.vx), _f64(result.vy), _f64(result.vz)]
    _io_check(L.kiwi_save_mapping(path.encode(), len(ids), ids.ctypes.data_as(_i64p), *[_p(a) for a in arrs], err,
                                  len(err)), err)


def map_voronoi(particles: dict, home_cell, cells: dict, kernel=None, precision="fp64", raw=False, ctx=None):
    """Density and mass-weighted velocity of an SPH snapshot on Voronoi cells -- the particle loop of
    run_mapping_stage (src/mapping.cpp:400-502).  `cells` holds the CSR geometry: face_off (n_cells+1),
    vert_off (n_faces+1), vxyz (absolute vertex coordinates, 3 per vertex, in each face's winding),
    face_nbr (neighbour cell index or -1), volume.  `home_cell[i]` is the cell containing particle i, or -1."""
    ctx = ctx or default_context()
    ki = kernel or KernelIntegrator()
    Ps, keep = _particles_struct(particles)
    home = np.ascontiguousarray(home_cell, dtype=np.int32)
    fo = np.ascontiguousarray(cells["face_off"], dtype=np.int64)
    vo = np.ascontiguousarray(cells["vert_off"], dtype=np.int64)
    vx_ = _f64(cells["vxyz"]).reshape(-1)
    nb = np.ascontiguousarray(cells["face_nbr"], dtype=np.int32)
    vol = _f64(cells["volume"])
    nc = len(vol)
    cs = KiwiVoronoiCells(nc, fo.ctypes.data_as(_i64p), vo.ctypes.data_as(_i64p), _p(vx_), nb.ctypes.data_as(_i32p),
                          _p(vol))
    outs = [np.empty(nc) for _ in range(4)]
    rawa = np.empty(4 * nc) if raw else None
    st = KiwiStats()
    sel = ki.sel()
    ctx.check(ctx._L.kiwi_map_voronoi(ctx.handle, C.byref(Ps), home.ctypes.data_as(_i32p), C.byref(cs), C.byref(sel),
                                      precision_code(precision), *[_p(o) for o in outs], _p(rawa), C.byref(st)),
              "map")
    d = st.as_dict()
    d["unresolved"] = d["skipped_outside"]
    d["unmapped"] = d["tile_pairs"]
    d["visited_pairs"] = d["evaluated_pairs"]
    return MappingResult(*outs, raw=rawa.reshape(4, nc) if raw else None, stats=d)


def map_voronoi_device(particles: dict, home_cell, cells: dict, out: dict, kernel=None, precision="fp64",
                       ctx=None):
    """Device variant of map_voronoi: `particles` (x y z vx vy vz m h), `home_cell` (int32), `cells`
    (face_off, vert_off int64; vxyz, volume float64; face_nbr int32) and `out` (density, vx, vy, vz[, raw4])
    are contiguous CUDA tensors, so that one tessellation staged on the GPU serves many calls.  Runs on the
    context's stream and returns the call's stats."""
    ctx = ctx or default_context()
    ki = kernel or KernelIntegrator()
    Ps, _ = _particles_struct(particles, device=True)

    def ptr(t, typ):
        return C.cast(C.c_void_p(int(t.data_ptr())), typ) if t is not None else None

    nc = int(cells["volume"].numel())
    cs = KiwiVoronoiCells(nc, ptr(cells["face_off"], _i64p), ptr(cells["vert_off"], _i64p), ptr(cells["vxyz"], _dp),
                          ptr(cells["face_nbr"], _i32p), ptr(cells["volume"], _dp))
    st = KiwiStats()
    sel = ki.sel()
    outs = [ptr(out.get(k), _dp) for k in ("density", "vx", "vy", "vz", "raw4")]
    ctx.check(ctx._L.kiwi_map_voronoi_device(ctx.handle, C.byref(Ps), ptr(home_cell, _i32p), C.byref(cs), C.byref(sel),
                                             precision_code(precision), *outs, C.byref(st)), "map (device)")
    d = st.as_dict()
    d["unresolved"] = d["skipped_outside"]
    d["unmapped"] = d["tile_pairs"]
    d["visited_pairs"] = d["evaluated_pairs"]
    return d


@dataclass
class InverseMappingResult:
    """run_inverse_mapping_test_stage's results (include/kiwi/mapping.hpp:88-106): per particle, in snapshot
    order, the mass recovered from the cells its kernel reaches and its coverage fraction; the totals of the
    original masses, the grid's cell masses and the recovered masses."""
    m_original: np.ndarray
    m_recovered: np.ndarray
    coverage: np.ndarray
    total_original_mass: float
    total_grid_mass: float
    total_recovered_mass: float
    density: np.ndarray | None = None
    stats: dict = field(default_factory=dict)


def inverse_map_voronoi(particles: dict, home_cell, cells: dict, kernel=None, cell_mass=None, precision="fp64",
                        ctx=None) -> InverseMappingResult:
    """The inverse-mapping check (run_inverse_mapping_test_stage's particle loop, src/mapping.cpp:540-701):
    the cell walk and cell integrals of map_voronoi, summed per particle.  `cell_mass`: M_c per cell
    (density x volume of the forward mapping's rows, as the stage reads them from mapping.dat); None uses
    this call's own forward map."""
    ctx = ctx or default_context()
    ki = kernel or KernelIntegrator()
    Ps, keep = _particles_struct(particles)
    n = int(Ps.n)
    home = np.ascontiguousarray(home_cell, dtype=np.int32)
    fo = np.ascontiguousarray(cells["face_off"], dtype=np.int64)
    vo = np.ascontiguousarray(cells["vert_off"], dtype=np.int64)
    vx_ = _f64(cells["vxyz"]).reshape(-1)
    nb = np.ascontiguousarray(cells["face_nbr"], dtype=np.int32)
    vol = _f64(cells["volume"])
    nc = len(vol)
    cs = KiwiVoronoiCells(nc, fo.ctypes.data_as(_i64p), vo.ctypes.data_as(_i64p), _p(vx_), nb.ctypes.data_as(_i32p),
                          _p(vol))
    cm = _f64(cell_mass) if cell_mass is not None else None
    rec, cov, tot, dens = np.zeros(n), np.zeros(n), np.zeros(3), np.empty(nc)
    st = KiwiStats()
    sel = ki.sel()
    ctx._L.kiwi_inverse_map_voronoi.argtypes = [C.c_void_p, C.POINTER(KiwiParticles), _i32p,
                                                C.POINTER(KiwiVoronoiCells), C.POINTER(KiwiKernelSel), C.c_int,
                                                _dp, _dp, _dp, _dp, _dp, C.POINTER(KiwiStats)]
    ctx.check(ctx._L.kiwi_inverse_map_voronoi(ctx.handle, C.byref(Ps), home.ctypes.data_as(_i32p), C.byref(cs),
                                              C.byref(sel), precision_code(precision), _p(cm), _p(rec), _p(cov),
                                              _p(tot), _p(dens), C.byref(st)), "inverse map")
    d = st.as_dict()
    d["unresolved"] = d["skipped_outside"]
    d["visited_pairs"] = d["evaluated_pairs"]
    return InverseMappingResult(_f64(particles["m"]).copy(), rec, cov, float(tot[0]), float(tot[1]), float(tot[2]),
                                density=dens, stats=d)


def save_inverse_mapping_test(path: str, ids, result: InverseMappingResult):
    """save_inverse_mapping_test (src/mapping.cpp:505-513): inverse-mapping-test.dat."""
    L = _io_lib()
    err = C.create_string_buffer(512)
    ids = np.ascontiguousarray(ids, dtype=np.int64)
    arrs = [_f64(result.m_original), _f64(result.m_recovered), _f64(result.coverage)]
    tot = np.array([result.total_original_mass, result.total_grid_mass, result.total_recovered_mass])
    _io_check(L.kiwi_save_inverse_mapping_test(path.encode(), len(ids), ids.ctypes.data_as(_i64p),
                                               *[_p(a) for a in arrs], _p(tot), err, len(err)), err)


def load_inverse_mapping_test(path: str):
    """load_inverse_mapping_test (src/mapping.cpp:519-538): (ids, InverseMappingResult)."""
    L = _io_lib()
    err = C.create_string_buffer(512)
    n = C.c_int64(0)
    tot = np.zeros(3)
    _io_check(L.kiwi_load_inverse_mapping_test(path.encode(), C.byref(n), _p(tot), None, None, None, None, 0, err,
                                               len(err)), err)
    ids = np.zeros(n.value, dtype=np.int64)
    arrs = [np.zeros(n.value) for _ in range(3)]
    _io_check(L.kiwi_load_inverse_mapping_test(path.encode(), C.byref(n), _p(tot), ids.ctypes.data_as(_i64p),
                                               *[_p(a) for a in arrs], n.value, err, len(err)), err)
    return ids, InverseMappingResult(*arrs, float(tot[0]), float(tot[1]), float(tot[2]))


@dataclass
class CartesianMap:
    """CartesianMap (include/kiwi/cartesian_map.hpp): a resolution^3 grid over the domain, each cell holding
    the mapping values of the Voronoi cell its centre lies in and that cell's site id."""
    resolution: int
    bounds: tuple
    density: np.ndarray
    vx: np.ndarray
    vy: np.ndarray
    vz: np.ndarray
    voronoi_cell_id: np.ndarray
    stats: dict = field(default_factory=dict)


def cartesian_map(sites, bounds, resolution, cell_density, cell_vx, cell_vy, cell_vz, site_id=None, mapped=None,
                  block_scale_factor=3.0, ctx=None) -> CartesianMap:
    """run_cartesian_map_stage's point location (src/cartesian_map.cpp:84-200) on the GPU: `sites` (n, 3)
    the point set, `cell_*` each site's mapping row, `site_id` the ids written to voronoi_cell_id (default:
    the site index), `mapped` which sites have a mapping row (default: all); sites the reference's
    container drops (outside the domain, or past its last block) own no cell."""
    ctx = ctx or default_context()
    xyz = _f64(np.asarray(sites, dtype=np.float64).reshape(-1, 3))
    n = xyz.shape[0]
    vals = [_f64(v) for v in (cell_density, cell_vx, cell_vy, cell_vz)]
    sid = np.ascontiguousarray(site_id, dtype=np.int32) if site_id is not None else None
    mp = np.ascontiguousarray(mapped, dtype=np.uint8) if mapped is not None else None
    b = _f64(bounds)
    res = int(resolution)
    nq = res ** 3 if res > 0 else 0
    outs = [np.empty(nq) for _ in range(4)]
    cid = np.empty(nq, dtype=np.int32)
    counts = np.zeros(2, dtype=np.int64)
    st = KiwiStats()
    f = ctx._L.kiwi_cartesian_map
    f.argtypes = [C.c_void_p, C.c_int64, _dp, _i32p, _dp, _dp, _dp, _dp, C.POINTER(C.c_uint8), _dp, C.c_int32,
                  C.c_double, _dp, _dp, _dp, _dp, _i32p, _i64p, C.POINTER(KiwiStats)]
    ctx.check(f(ctx.handle, n, _p(xyz), sid.ctypes.data_as(_i32p) if sid is not None else None, *[_p(v) for v in vals],
                mp.ctypes.data_as(C.POINTER(C.c_uint8)) if mp is not None else None, _p(b), res,
                float(block_scale_factor),
                *[_p(o) for o in outs], cid.ctypes.data_as(_i32p), counts.ctypes.data_as(_i64p), C.byref(st)),
              "cartesian_map")
    d = st.as_dict()
    d["unresolved"], d["unmapped"] = int(counts[0]), int(counts[1])
    return CartesianMap(res, tuple(float(v) for v in b), *outs, cid, stats=d)


def save_cartesian_map(m: CartesianMap, path: str):
    """save_cartesian_map (src/cartesian_map.cpp:202-229): the VGTCMAP1 file."""
    L = _io_lib()
    err = C.create_string_buffer(512)
    b = _f64(m.bounds)
    arrs = [_f64(a) for a in (m.density, m.vx, m.vy, m.vz)]
    cid = np.ascontiguousarray(m.voronoi_cell_id, dtype=np.int32)
    _io_check(L.kiwi_save_cartesian_map(path.encode(), m.resolution, _p(b), *[_p(a) for a in arrs],
                                        cid.ctypes.data_as(_i32p), err, len(err)), err)


def load_cartesian_map(path: str) -> CartesianMap:
    """load_cartesian_map (src/cartesian_map.cpp:231-277)."""
    L = _io_lib()
    err = C.create_string_buffer(512)
    r = C.c_int32(0)
    b = np.zeros(6)
    _io_check(L.kiwi_load_cartesian_map(path.encode(), C.byref(r), _p(b), None, None, None, None, None, err, len(err)),
              err)
    nq = r.value ** 3
    arrs = [np.empty(nq) for _ in range(4)]
    cid = np.empty(nq, dtype=np.int32)
    _io_check(L.kiwi_load_cartesian_map(path.encode(), C.byref(r), _p(b), *[_p(a) for a in arrs],
                                        cid.ctypes.data_as(_i32p), err, len(err)), err)
    return CartesianMap(r.value, tuple(b), *arrs, cid)


def coverage_grid_buffer(particles: dict, bounds, spacing_fraction=0.05, coverage_radius_factor=2.0, ctx=None):
    """add_coverage_grid_buffer (src/point_set.cpp:198-262) on the GPU: the cell-centred lattice candidates
    no particle's sphere of radius coverage_radius_factor x h reaches, in lattice order, ids from n + 1.
    `particles` holds x y z h.  Returns (xyz (k, 3), ids (k,))."""
    ctx = ctx or default_context()
    L = ctx._L
    L.kiwi_coverage_grid_candidates.restype = C.c_int64
    L.kiwi_coverage_grid_candidates.argtypes = [_dp, C.c_double, _i32p]
    L.kiwi_coverage_grid_buffer.argtypes = [C.c_void_p, C.c_int64, _dp, _dp, _dp, _dp, _dp, C.c_double, C.c_double,
                                            C.c_int64, _dp, _dp, _dp, _i32p, _i64p]
    b = _f64(bounds)
    cap = L.kiwi_coverage_grid_candidates(_p(b), float(spacing_fraction), None)
    if cap < 0:
        raise KiwiError(-1, "coverage buffer: bad domain or spacing_fraction")
    a = [_f64(particles[k]) for k in ("x", "y", "z", "h")]
    n = len(a[0])
    out = [np.empty(max(cap, 1)) for _ in range(3)]
    ids = np.empty(max(cap, 1), dtype=np.int32)
    na = C.c_int64(0)
    ctx.check(L.kiwi_coverage_grid_buffer(ctx.handle, n, *[_p(v) for v in a], _p(b), float(spacing_fraction),
                                          float(coverage_radius_factor), cap, *[_p(o) for o in out],
                                          ids.ctypes.data_as(_i32p), C.byref(na)), "coverage buffer")
    k = na.value
    return np.stack([o[:k] for o in out], axis=1), ids[:k].copy()


def lloyd_step(sites, bounds, ids=None, block_scale_factor=3.0, ctx=None):
    """lloyd_step (src/point_set.cpp:265-293) on the GPU: the sites the reference's container keeps, each
    moved to its Voronoi cell's centroid, in the container's walk order.  Returns (ids, xyz (k, 3), cell
    volumes (k,), stats)."""
    ctx = ctx or default_context()
    xyz = _f64(np.asarray(sites, dtype=np.float64).reshape(-1, 3))
    n = xyz.shape[0]
    sid = np.ascontiguousarray(ids, dtype=np.int32) if ids is not None else None
    oid = np.empty(max(n, 1), dtype=np.int32)
    oxyz = np.empty((max(n, 1), 3))
    ovol = np.empty(max(n, 1))
    k, failed = C.c_int64(0), C.c_int64(0)
    st = KiwiStats()
    f = ctx._L.kiwi_lloyd_step
    f.argtypes = [C.c_void_p, C.c_int64, _i32p, _dp, _dp, C.c_double, _i32p, _dp, _dp, _i64p, _i64p,
                  C.POINTER(KiwiStats)]
    ctx.check(f(ctx.handle, n, sid.ctypes.data_as(_i32p) if sid is not None else None, _p(xyz), _p(_f64(bounds)),
                float(block_scale_factor), oid.ctypes.data_as(_i32p), _p(oxyz), _p(ovol), C.byref(k), C.byref(failed),
                C.byref(st)), "lloyd step")
    d = st.as_dict()
    d["failed"] = failed.value
    d["dropped"] = d["skipped_outside"]
    m = k.value
    return oid[:m].copy(), oxyz[:m].copy(), ovol[:m].copy(), d


def version() -> str:
    return load_library().kiwi_version().decode()


def measure_fp64_peak(ctx=None) -> float:
    """Measured FP64 FMA throughput (TFLOP/s) of the context's GPU."""
    ctx = ctx or default_context()
    v = C.c_double(0.0)
    ctx._L.kiwi_measure_fp64_peak.argtypes = [C.c_void_p, _dp]
    ctx.check(ctx._L.kiwi_measure_fp64_peak(ctx.handle, C.byref(v)), "fp64 peak")
    return v.value


def measure_fp32_peak(ctx=None) -> float:
    """Measured FP32 FMA throughput (TFLOP/s) of the context's GPU."""
    ctx = ctx or default_context()
    v = C.c_double(0.0)
    ctx._L.kiwi_measure_fp32_peak.argtypes = [C.c_void_p, _dp]
    ctx.check(ctx._L.kiwi_measure_fp32_peak(ctx.handle, C.byref(v)), "fp32 peak")
    return v.value
