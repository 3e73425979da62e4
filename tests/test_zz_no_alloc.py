"""The allocation-free sph-to-grid entry point, called through the C ABI.

kiwi_sph_to_grid_device_noalloc serves callers that cannot call cudaMalloc -- codes whose device memory
is all handed to their own pool allocator (a simulation mapping its particles in situ), and callers
that cannot absorb the device-wide synchronisation an allocation may cause.  Its scratch lives in a
fixed device array inside the library.  This test checks that two calls in a row, on different inputs,
give exactly what the allocating entry point (kiwi_sph_to_grid_device) gives -- bitwise, which is
within every tolerance the parity tests use -- and that an input too large for the fixed array is
rejected with a clear error.  The file sorts last so that a stop-at-first-failure run has already run
every other test when it gets here.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KIWI_ERR_LIMIT = -5


def _noalloc_fn():
    import kiwi_b200

    L = kiwi_b200.load_library()
    f = L.kiwi_sph_to_grid_device_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.POINTER(kiwi_b200.KiwiParticles), C.POINTER(kiwi_b200.KiwiCartGrid),
                  C.POINTER(kiwi_b200.KiwiKernelSel), C.c_int] + [C.POINTER(C.c_double)] * 5 + \
                 [C.POINTER(kiwi_b200.KiwiStats), C.c_char_p, C.c_size_t]
    return f


def _dptr(t):
    return C.cast(C.c_void_p(int(t.data_ptr())), C.POINTER(C.c_double)) if t is not None else None


def _device_particles(torch, n, seed):
    rng = np.random.default_rng(seed)
    P = {k: rng.uniform(0.0, 2.0, n) for k in ("x", "y", "z")}
    for k in ("vx", "vy", "vz"):
        P[k] = rng.standard_normal(n)
    P["m"] = rng.uniform(0.5, 1.5, n)
    P["h"] = rng.uniform(0.02, 0.25, n)
    return {k: torch.from_numpy(v).cuda() for k, v in P.items()}


def _call_noalloc(kiwi_b200, f, dP, bounds, shape, out, precision=None):
    Ps, _ = kiwi_b200._particles_struct(dP, device=True)
    grid = kiwi_b200.KiwiCartGrid((C.c_double * 6)(*bounds), *shape)
    sel = kiwi_b200.KernelIntegrator().sel()
    st = kiwi_b200.KiwiStats()
    err = C.create_string_buffer(512)
    prec = kiwi_b200.KIWI_FP64 if precision is None else precision
    rc = f(None, C.byref(Ps), C.byref(grid), C.byref(sel), prec, _dptr(out["density"]),
           _dptr(out["vx"]), _dptr(out["vy"]), _dptr(out["vz"]), _dptr(out["raw4"]), C.byref(st), err, 512)
    return rc, st, err.value.decode()


def test_noalloc_matches_allocating_entry_point_on_two_calls():
    import torch

    import kiwi_b200

    f = _noalloc_fn()
    ctx = kiwi_b200.Context(0)
    bounds, shape = (0.0, 2.0, 0.0, 2.0, 0.0, 2.0), (40, 36, 44)
    nc = shape[0] * shape[1] * shape[2]
    for call, (n, seed) in enumerate(((3000, 1), (1700, 2))):
        dP = _device_particles(torch, n, seed)
        ref = {k: torch.zeros(nc, dtype=torch.float64, device="cuda") for k in ("density", "vx", "vy", "vz")}
        ref["raw4"] = torch.zeros(4 * nc, dtype=torch.float64, device="cuda")
        st_ref = kiwi_b200.sph_to_grid_device(dP, bounds, shape, ref, ctx=ctx)
        out = {k: torch.full_like(v, np.nan) for k, v in ref.items()}
        torch.cuda.synchronize()
        rc, st, msg = _call_noalloc(kiwi_b200, f, dP, bounds, shape, out)
        torch.cuda.synchronize()
        assert rc == 0, msg
        for k in ref:
            assert torch.equal(out[k], ref[k]), (call, k)
        assert st.bbox_pairs == st_ref["bbox_pairs"] and st.sphere_pairs == st_ref["sphere_pairs"]


def test_noalloc_allocates_no_device_memory():
    """After a first (set-up) call, further calls -- plain FP64 and FP32-mixed, whose mixed kernel takes its
    own scratch -- leave the device's free memory unchanged, and the FP32-mixed call equals the allocating
    entry point's FP32-mixed result bit for bit."""
    import torch

    import kiwi_b200

    f = _noalloc_fn()
    ctx = kiwi_b200.Context(0)
    bounds, shape = (0.0, 2.0, 0.0, 2.0, 0.0, 2.0), (32, 32, 32)
    nc = shape[0] * shape[1] * shape[2]
    dP = _device_particles(torch, 2500, 3)
    out = {k: torch.zeros(nc, dtype=torch.float64, device="cuda") for k in ("density", "vx", "vy", "vz")}
    out["raw4"] = torch.zeros(4 * nc, dtype=torch.float64, device="cuda")
    ref = {k: torch.zeros_like(v) for k, v in out.items()}
    kiwi_b200.sph_to_grid_device(dP, bounds, shape, ref, precision="fp32_mixed", ctx=ctx)
    rc, _, msg = _call_noalloc(kiwi_b200, f, dP, bounds, shape, out)
    assert rc == 0, msg
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for prec in (kiwi_b200.KIWI_FP64, kiwi_b200.KIWI_FP32_MIXED, kiwi_b200.KIWI_FP32_MIXED):
        rc, _, msg = _call_noalloc(kiwi_b200, f, dP, bounds, shape, out, precision=prec)
        assert rc == 0, msg
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] >= free0
    for k in ref:
        assert torch.equal(out[k], ref[k]), k


def test_noalloc_rejects_input_beyond_the_scratch_limit():
    import torch

    import kiwi_b200

    f = _noalloc_fn()
    n = 1_000_000  # ~36 bytes of scratch per particle: beyond the 32 MiB fixed area
    dP = {k: torch.zeros(n, dtype=torch.float64, device="cuda") for k in ("x", "y", "z", "vx", "vy", "vz", "m", "h")}
    out = {k: torch.zeros(64, dtype=torch.float64, device="cuda") for k in ("density", "vx", "vy", "vz")}
    out["raw4"] = None
    rc, _, msg = _call_noalloc(kiwi_b200, f, dP, (0.0, 1.0, 0.0, 1.0, 0.0, 1.0), (4, 4, 4), out)
    torch.cuda.synchronize()
    assert rc == KIWI_ERR_LIMIT
    assert "scratch" in msg
