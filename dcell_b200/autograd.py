"""Differentiable SL transport: torch.autograd.Function over the hand-written
adjoint kernel (dcell_sl_adjoint), with checkpoint-and-recompute.

Forward: K dense SL steps phi_{n+1} = SL(phi_n; vel, dt_n).  Only every
`every`-th state is kept; backward recomputes each segment's states from its
checkpoint and runs the adjoint steps in reverse, accumulating dL/dvel over
all steps and returning dL/dphi_0.  Memory: K/every + every grids instead of
K.  The reference has no derivatives; this is new capability on the same
transport operator (DCELL_LINEAR or the Catmull-Rom cubic).
"""
from __future__ import annotations

import ctypes
import math
from typing import Sequence

import numpy as np
import torch

from . import _lib, fields
from ._lib import BACKTRACE, INTERP, check, geom, lib
from .levelset import sl_step


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


def sl_adjoint(phi0, vel, dt, h, grad_phi, grad_phi0, grad_vel, interp="cubic_separable", backtrace="midpoint"):
    """Accumulate one step's adjoint into grad_phi0 / grad_vel (in place)."""
    g = geom(tuple(phi0.shape), h)
    dtype = _lib.F64 if phi0.dtype == torch.float64 else _lib.F32
    check(lib().dcell_sl_adjoint(ctypes.byref(g), dtype, _vp(phi0), _vp(vel), float(dt),
                                 INTERP[interp] if isinstance(interp, str) else int(interp),
                                 BACKTRACE[backtrace] if isinstance(backtrace, str) else int(backtrace),
                                 _vp(grad_phi), _vp(grad_phi0), _vp(grad_vel),
                                 ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))


class SLTransport(torch.autograd.Function):
    """phi_K = SL^K(phi_0; vel).  Arguments: phi0 (nz,ny,nx), vel (nz,ny,nx,3),
    dts (sequence of K step sizes with any time factor folded in), h,
    interp, backtrace, every (checkpoint interval)."""

    @staticmethod
    def forward(ctx, phi0, vel, dts: Sequence[float], h, interp="cubic_separable", backtrace="midpoint", every=10):
        dts = [float(d) for d in dts]
        x = phi0.detach().contiguous()
        v = vel.detach().contiguous()
        ckpts = [x]
        for i, dt in enumerate(dts):
            x = sl_step(x, v, dt, h, interp=interp, backtrace=backtrace)
            if (i + 1) % every == 0 and i + 1 < len(dts):
                ckpts.append(x)
        ctx.save_for_backward(v, *ckpts)
        ctx.cfg = (dts, h, interp, backtrace, every)
        return x

    @staticmethod
    def backward(ctx, grad_out):
        v, *ckpts = ctx.saved_tensors
        dts, h, interp, backtrace, every = ctx.cfg
        g = grad_out.contiguous().clone()
        gvel = torch.zeros_like(v)
        K = len(dts)
        for seg in reversed(range(len(ckpts))):
            s, e = seg * every, min((seg + 1) * every, K)
            states = [ckpts[seg]]
            for i in range(s, e - 1):
                states.append(sl_step(states[-1], v, dts[i], h, interp=interp, backtrace=backtrace))
            for i in reversed(range(s, e)):
                gprev = torch.zeros_like(g)
                sl_adjoint(states[i - s], v, dts[i], h, g, gprev, gvel, interp, backtrace)
                g = gprev
        return g, gvel, None, None, None, None, None


def transport(phi0, vel, dts, h, interp="cubic_separable", backtrace="midpoint", every=10):
    return SLTransport.apply(phi0, vel, list(dts), h, interp, backtrace, every)


def heaviside(phi, eps):
    """Smoothed Heaviside whose derivative is the reference's smoothed delta
    (LevelSetDiracDelta, NormalDirection.c:36-57)."""
    x = (phi / eps).clamp(-1.0, 1.0)
    return 0.5 * (1.0 + x + torch.sin(math.pi * x) / math.pi)


class FourierVelocity(torch.nn.Module):
    """vel = sum_m c_m B_m with B_m fixed divergence-free MAC fields (discrete
    curls of one Fourier mode each) and c the learnable coefficients."""

    def __init__(self, shape, nmodes=16, seed=5, device="cuda", dtype=torch.float32):
        super().__init__()
        k, a, ph = fields.fourier_modes(nmodes, seed)
        scale = 1.0 / (2 * math.pi * np.linalg.norm(k, axis=1))
        basis = []
        for m in range(nmodes):
            e = np.zeros(nmodes)
            e[m] = scale[m]
            basis.append(fields.fourier_velocity(shape, e, (k, a, ph), device=device).to(dtype))
        self.register_buffer("basis", torch.stack(basis))
        self.coeffs = torch.nn.Parameter(torch.ones(nmodes, dtype=dtype, device=device))

    def forward(self, coeffs=None):
        c = self.coeffs if coeffs is None else coeffs
        return torch.einsum("m,m...->...", c.to(self.basis.dtype), self.basis).contiguous()


def c5_loss(phi_T, phi_target, h):
    eps = 1.5 * h
    return ((heaviside(phi_T, eps) - heaviside(phi_target, eps)) ** 2).sum()
