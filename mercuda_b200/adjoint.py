"""Gradients through the MVS and HYBRID test-particle integrations as
torch.autograd.Functions.

The library's mercury_b200_adjoint_* entry points run the forward integration
of massless particles (keeping a checkpoint every K steps) and the reverse
sweep. Tensors stay on the GPU: inputs and outputs are float64 CUDA tensors
passed to the C ABI by device pointer. The library keeps the checkpoints of one
forward run, so a backward pass belongs to the most recent forward call.

    x_final, v_final = mvs_trajectory(x0, v0, yar, big, h=8.0, nsteps=1000, K=50)
    loss = (x_final ** 2).sum()
    loss.backward()          # x0.grad, v0.grad, yar.grad

hybrid_trajectory() does the same through mdt_hy (democratic-heliocentric
coordinates, changeover radii rcrit, encounter tolerance tol); its forward run
goes through the library's HYBRID path and replaces the resident system.
"""
from __future__ import annotations

import ctypes as C
import itertools

import numpy as np
import torch

from .backend import BackendError, _p, load_library

_run_ids = itertools.count(1)
_last_run = 0
_last_hybrid_run = 0


def _ptr(t: torch.Tensor | None):
    if t is None:
        return None
    if t.dtype != torch.float64 or not t.is_cuda or not t.is_contiguous():
        raise BackendError("adjoint tensors must be contiguous float64 CUDA tensors")
    return C.c_void_p(t.data_ptr())


class MvsTrajectory(torch.autograd.Function):
    """(x0, v0, yar) -> (x_final, v_final) of nsteps MVS steps about fixed Big bodies."""

    @staticmethod
    def forward(ctx, x0, v0, yar, big_m, big_x, big_v, h, nsteps, checkpoint_every):
        global _last_run
        lib = load_library()
        x0 = x0.detach().contiguous()
        v0 = v0.detach().contiguous()
        yar_d = yar.detach().contiguous() if yar is not None else None
        np_ = x0.shape[0]
        xf = torch.empty_like(x0)
        vf = torch.empty_like(v0)
        m = np.ascontiguousarray(big_m, dtype=np.float64)
        bx = np.ascontiguousarray(big_x, dtype=np.float64)
        bv = np.ascontiguousarray(big_v, dtype=np.float64)
        torch.cuda.synchronize(x0.device)
        rc = lib.mercury_b200_adjoint_forward(len(m), _p(m), _p(bx), _p(bv), np_, _ptr(x0), _ptr(v0), _ptr(yar_d),
                                              float(h), int(nsteps), int(checkpoint_every), _ptr(xf), _ptr(vf))
        if rc != 0:
            raise BackendError("adjoint forward run failed")
        ctx.run = next(_run_ids)
        _last_run = ctx.run
        # the library reads x0, v0, yar again in the backward sweep
        ctx.keep = (x0, v0, yar_d)
        ctx.has_yar = yar is not None
        return xf, vf

    @staticmethod
    def backward(ctx, gx, gv):
        if ctx.run != _last_run:
            raise BackendError("the library holds the checkpoints of a later forward run")
        lib = load_library()
        x0 = ctx.keep[0]
        gx = gx.contiguous() if gx is not None else torch.zeros_like(x0)
        gv = gv.contiguous() if gv is not None else None
        dx0 = torch.empty_like(x0)
        dv0 = torch.empty_like(x0)
        dyar = torch.empty(x0.shape[0], dtype=torch.float64, device=x0.device) if ctx.has_yar else None
        torch.cuda.synchronize(x0.device)
        if lib.mercury_b200_adjoint_backward(_ptr(gx), _ptr(gv), _ptr(dx0), _ptr(dv0), _ptr(dyar)) != 0:
            raise BackendError("adjoint backward sweep failed")
        return dx0, dv0, dyar, None, None, None, None, None, None


def mvs_trajectory(x0, v0, yar, big, h: float, nsteps: int, checkpoint_every: int = 50):
    """big = (m, x, v) of the central body and the Big bodies (host arrays)."""
    m, bx, bv = big
    return MvsTrajectory.apply(x0, v0, yar, m, bx, bv, h, nsteps, checkpoint_every)


class HybridTrajectory(torch.autograd.Function):
    """(x0, v0, yar) -> (x_final, v_final) of nsteps mdt_hy steps about the Big bodies."""

    @staticmethod
    def forward(ctx, x0, v0, yar, big_m, big_x, big_v, big_rcrit, rcrit, h, tol, nsteps, checkpoint_every):
        global _last_hybrid_run
        lib = load_library()
        x0 = x0.detach().contiguous()
        v0 = v0.detach().contiguous()
        yar_d = yar.detach().contiguous() if yar is not None else None
        np_ = x0.shape[0]
        xf = torch.empty_like(x0)
        vf = torch.empty_like(v0)
        m = np.ascontiguousarray(big_m, dtype=np.float64)
        bx = np.ascontiguousarray(big_x, dtype=np.float64)
        bv = np.ascontiguousarray(big_v, dtype=np.float64)
        brc = np.ascontiguousarray(big_rcrit, dtype=np.float64)
        rc = np.ascontiguousarray(rcrit, dtype=np.float64)
        if rc.shape != (np_,) or brc.shape != (len(m),):
            raise BackendError("rcrit must hold one changeover radius per body")
        torch.cuda.synchronize(x0.device)
        if lib.mercury_b200_hybrid_adjoint_forward(len(m), _p(m), _p(bx), _p(bv), _p(brc), np_, _ptr(x0), _ptr(v0),
                                                   _ptr(yar_d), _p(rc), float(h), float(tol), int(nsteps),
                                                   int(checkpoint_every), _ptr(xf), _ptr(vf)) != 0:
            raise BackendError("HYBRID adjoint forward run failed")
        ctx.run = next(_run_ids)
        _last_hybrid_run = ctx.run
        ctx.keep = (x0, v0, yar_d)
        ctx.has_yar = yar is not None
        return xf, vf

    @staticmethod
    def backward(ctx, gx, gv):
        if ctx.run != _last_hybrid_run:
            raise BackendError("the library holds the records of a later HYBRID forward run")
        lib = load_library()
        x0 = ctx.keep[0]
        gx = gx.contiguous() if gx is not None else torch.zeros_like(x0)
        gv = gv.contiguous() if gv is not None else None
        dx0 = torch.empty_like(x0)
        dv0 = torch.empty_like(x0)
        dyar = torch.empty(x0.shape[0], dtype=torch.float64, device=x0.device) if ctx.has_yar else None
        torch.cuda.synchronize(x0.device)
        if lib.mercury_b200_hybrid_adjoint_backward(_ptr(gx), _ptr(gv), _ptr(dx0), _ptr(dv0), _ptr(dyar)) != 0:
            raise BackendError("HYBRID adjoint backward sweep failed")
        return dx0, dv0, dyar, None, None, None, None, None, None, None, None, None


def hybrid_trajectory(x0, v0, yar, big, rcrit, h: float, nsteps: int, tol: float = 1e-12,
                      checkpoint_every: int = 50):
    """big = (m, x, v, rcrit) of the central body and the Big bodies (host
    arrays, democratic-heliocentric); rcrit = the particles' changeover radii."""
    m, bx, bv, brc = big
    return HybridTrajectory.apply(x0, v0, yar, m, bx, bv, brc, rcrit, h, tol, nsteps, checkpoint_every)


def hybrid_timing():
    """(forward wall ms, backward device ms, encounter-member steps) of the last HYBRID run."""
    lib = load_library()
    f, b, k = C.c_double(0.0), C.c_double(0.0), C.c_int64(0)
    lib.mercury_b200_hybrid_adjoint_timing(C.byref(f), C.byref(b), C.byref(k))
    return f.value, b.value, k.value


def timing():
    lib = load_library()
    f, b = C.c_double(0.0), C.c_double(0.0)
    lib.mercury_b200_adjoint_timing(C.byref(f), C.byref(b))
    return f.value, b.value
