"""Gradient of the wall-pressure objective through torch.autograd.

J(P0, Mach) = sum over the cells of one block face of p * A after `nsteps`
time-accurate SSP-RK steps of the explicit inviscid scheme, started from the
interior state P0 with the 405 inflow at Mach `mach`.  The forward runs the
fused GPU steps keeping a checkpoint every `interval` steps (sqrt(nsteps) by
default); the backward recomputes each segment from its checkpoint and runs
the hand-written discrete adjoint kernels (C ABI mose_gpu_adjoint_*) back
through it.  Single-block 2-D domains, HLLC with minmod, van Leer or van
Albada.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from .cases import GC, to_ref_layout


class WallPressure(torch.autograd.Function):
    """J = WallPressure.apply(prim0, mach, solver, nsteps, interval, block, face)

    prim0: float64 tensor (nk, nj, ni, 5) -- interior primitives (rho, u, v, w, p)
    mach:  float64 scalar tensor -- inflow Mach of the 405 faces
    """

    @staticmethod
    def forward(ctx, prim0, mach, solver, nsteps, interval=None, block=1, face=3):
        interval = interval or max(1, int(round(math.sqrt(nsteps))))
        ref = to_ref_layout(prim0.detach().cpu().numpy().astype(np.float64))
        solver.upload_prim(block, ref)
        solver.set_time(0.0, 0)
        solver.set_inflow_mach(float(mach))
        J = solver.adjoint_forward(nsteps, interval, block, face)
        ctx.solver, ctx.block = solver, block
        ctx.dev, ctx.shape = prim0.device, prim0.shape
        return torch.tensor(J, dtype=torch.float64, device=prim0.device)

    @staticmethod
    def backward(ctx, gJ):
        s = ctx.solver
        dM = s.adjoint_backward()
        lam = s.download_adjoint(ctx.block)[GC:-GC, GC:-GC, GC:-GC]
        dP = torch.from_numpy(np.ascontiguousarray(lam)).to(ctx.dev).reshape(ctx.shape)
        return gJ * dP, gJ * torch.tensor(dM, dtype=torch.float64, device=ctx.dev), None, None, None, None, None


def wall_pressure(prim0, mach, solver, nsteps, interval=None, block=1, face=3):
    """J(prim0, mach) with a gradient (see WallPressure)."""
    return WallPressure.apply(prim0, mach, solver, nsteps, interval, block, face)
