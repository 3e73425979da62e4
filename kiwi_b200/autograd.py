"""Differentiable sph-to-grid for checking gradients: a torch.autograd.Function whose forward is the GPU
sph-to-grid stage (kiwi_sph_to_grid_device) and whose backward is the hand-written adjoint kernel
(kiwi_sph_to_grid_adjoint_device).  The reference has no gradients; this binding exists to differentiate
the gridded density and momentum with respect to the particles' positions, smoothing lengths, masses and
velocities, and to check those derivatives against finite differences.

The C calls run on the library context's stream and return when their work is done; the binding
synchronises torch's current stream before each call so that the inputs are complete.
"""
from __future__ import annotations

import torch

from . import KernelIntegrator, default_context, sph_to_grid_adjoint_device, sph_to_grid_device

_KEYS = ("x", "y", "z", "h", "m", "vx", "vy", "vz")


class SphToGridRaw(torch.autograd.Function):
    """raw4 = (M, Px, Py, Pz) per cell, shape (4, nx, ny, nz): M_c = sum_p m_p K_pc, P_c = sum_p m_p K_pc v_p
    (src/cartesian_grid.cpp:272-277 accumulates exactly these)."""

    @staticmethod
    def forward(fctx, x, y, z, h, m, vx, vy, vz, bounds, shape, kernel, precision, kctx):
        ins = (x, y, z, h, m, vx, vy, vz)
        for t in ins:
            if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
                raise ValueError("particle tensors must be contiguous float64 CUDA tensors")
        nx, ny, nz = (int(s) for s in shape)
        raw4 = torch.empty(4 * nx * ny * nz, dtype=torch.float64, device=x.device)
        torch.cuda.current_stream(x.device).synchronize()
        sph_to_grid_device(dict(zip(_KEYS, ins)), bounds, shape, {"raw4": raw4}, kernel=kernel,
                           precision=precision, ctx=kctx)
        fctx.save_for_backward(*ins)
        fctx.bounds, fctx.shape, fctx.kernel, fctx.kctx = bounds, (nx, ny, nz), kernel, kctx
        return raw4.view(4, nx, ny, nz)

    @staticmethod
    def backward(fctx, g):
        ins = fctx.saved_tensors
        cot = g.contiguous().view(-1)
        grads = {k: (torch.empty_like(t) if fctx.needs_input_grad[i] else None)
                 for i, (k, t) in enumerate(zip(_KEYS, ins))}
        torch.cuda.current_stream(cot.device).synchronize()
        sph_to_grid_adjoint_device(dict(zip(_KEYS, ins)), fctx.bounds, fctx.shape, cot, grads,
                                   kernel=fctx.kernel, ctx=fctx.kctx)
        return tuple(grads[k] for k in _KEYS) + (None, None, None, None, None)


def sph_to_grid_raw(x, y, z, h, m, vx, vy, vz, bounds, shape, kernel=None, precision="fp64", ctx=None):
    """The raw sums (M, Px, Py, Pz), differentiable in every particle input."""
    return SphToGridRaw.apply(x, y, z, h, m, vx, vy, vz, bounds, shape, kernel or KernelIntegrator(), precision,
                              ctx or default_context())


def sph_to_grid(x, y, z, h, m, vx, vy, vz, bounds, shape, kernel=None, precision="fp64", ctx=None):
    """(density, vx, vy, vz) on the grid as run_sph_to_grid_stage finalises them (src/cartesian_grid.cpp:
    294-317): density = M / cell volume; velocity = P / M where M > 0, else the mean particle velocity."""
    raw = sph_to_grid_raw(x, y, z, h, m, vx, vy, vz, bounds, shape, kernel, precision, ctx)
    nx, ny, nz = (int(s) for s in shape)
    vol = ((bounds[1] - bounds[0]) / nx) * ((bounds[3] - bounds[2]) / ny) * ((bounds[5] - bounds[4]) / nz)
    M = raw[0]
    has = M > 0
    Msafe = torch.where(has, M, torch.ones_like(M))
    vel = [torch.where(has, raw[1 + i] / Msafe, v.mean()) for i, v in enumerate((vx, vy, vz))]
    return (M / vol, *vel)
