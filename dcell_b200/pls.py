"""Particle level set on the GPU -- the reference's LevelSetMethod/ParticleLS.c,
ParticleLS2D.c and ParticleLS3D.c over torch device memory.

Particles are (capacity, 4) device tensors of the level set's dtype, rows
X.x, X.y, X.z (global index space) and the signed radius (struct _Particle,
LSM_private.h:45-48); ``count`` rows are live.  Random draws follow the
reference's PETSCRAND48 stream (the C library's drand48): ``rng`` is a
one-element int64 device tensor holding the 48-bit state; srand48(0x12345678),
PETSc's default seed on rank 0, is ``SEED_STATE``.

Low-level calls: ``advect``, ``correct``, ``adjust_radii``, ``seed``,
``reseed``.  Reference-named entry points on a ``levelset.LevelSet``:
``LevelSetInitializeParticles``, ``LevelSetAdvectPLS``,
``LevelSetAdvectPLSRK2HalfStep`` / ``FullStep`` and ``ParticleLS_*``.
Seeding and reseeding are 2D, as the reference's (its attraction step reads
phi through 2D pointers).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Optional

import torch

from . import _lib
from . import levelset as L
from ._lib import DcellError, check, geom, lib

SEED_STATE = 0x12345678330E


def params(dim: int = 2, **kw) -> _lib.PlsParams:
    """LevelSetInitializeParticles' defaults (ParticleLS.c:21-27), overridable by keyword."""
    p = _lib.PlsParams()
    lib().dcell_pls_default_params(int(dim), ctypes.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


class _Scratch:
    """A device byte buffer with a 256-byte aligned start (the C ABI's rule)."""

    def __init__(self, nbytes: int, device):
        self.buf = torch.empty(max(int(nbytes), 1) + 256, dtype=torch.uint8, device=device)
        base = self.buf.data_ptr()
        self.ptr = ctypes.c_void_p(base + (-base) % 256)
        self.nbytes = max(int(nbytes), 1)


def _scratch(nbytes: int, device) -> _Scratch:
    return _Scratch(nbytes, device)


def _flags_arg(flags):
    return L._ptr(flags) if flags is not None else None


def advect(particles: torch.Tensor, n: int, vel: torch.Tensor, dt: float, h, origin=(0, 0, 0), flags=None):
    """ParticleLS_AdvectParticles2D/3D (ParticleLS2D.c:6-36, ParticleLS3D.c:6-36)
    on the first n particles, in place.  vel: the level set's velocity grid."""
    L._require_cuda(particles, vel)
    shape = tuple(vel.shape[:-1])
    g = geom(shape, h, origin)
    check(lib().dcell_pls_advect(ctypes.byref(g), L._dtype_code(particles), L._ptr(vel), L._ptr(particles), int(n),
                                 float(dt), _flags_arg(flags), L._stream()))


def correct(phi: torch.Tensor, band: torch.Tensor, particles: torch.Tensor, n: int, h, origin=(0, 0, 0),
            flags=None, scratch: Optional[_Scratch] = None):
    """ParticleLS_ErrorCorrection2D/3D (ParticleLS2D.c:40-115,
    ParticleLS3D.c:40-116): phi corrected at the band points, in place."""
    L._require_cuda(phi, particles)
    g = geom(tuple(phi.shape), h, origin)
    dt = L._dtype_code(phi)
    need = lib().dcell_pls_correct_scratch_bytes(ctypes.byref(g), dt)
    if scratch is None or scratch.nbytes < need:
        scratch = _scratch(need, phi.device)
    nb = int(band.shape[0]) if band is not None else 0
    check(lib().dcell_pls_correct(ctypes.byref(g), dt, L._ptr(phi), L._ptr(band) if nb else None, nb,
                                  L._ptr(particles), int(n), scratch.ptr, scratch.nbytes, _flags_arg(flags),
                                  L._stream()))


def adjust_radii(phi: torch.Tensor, particles: torch.Tensor, n: int, h=1.0, origin=(0, 0, 0), prm=None, flags=None):
    """ParticleLS_AdjustRadii (ParticleLS.c:158-185), in place."""
    L._require_cuda(phi, particles)
    g = geom(tuple(phi.shape), h, origin)
    prm = prm or params(phi.dim())
    check(lib().dcell_pls_adjust_radii(ctypes.byref(g), L._dtype_code(phi), L._ptr(phi), L._ptr(particles), int(n),
                                       ctypes.byref(prm), _flags_arg(flags), L._stream()))


def new_rng(state: int = SEED_STATE, device="cuda") -> torch.Tensor:
    return torch.tensor([int(state)], dtype=torch.int64, device=device)


def seed(phi: torch.Tensor, band: torch.Tensor, rng: torch.Tensor, h=1.0, origin=(0, 0, 0), prm=None,
         capacity: Optional[int] = None, flags=None):
    """LevelSetInitializeParticles' seeding (ParticleLS.c:36-75), 2D.
    Returns (particles (capacity, 4), count); rng is advanced in place."""
    L._require_cuda(phi, band, rng)
    prm = prm or params(phi.dim())
    g = geom(tuple(phi.shape), h, origin)
    nb = int(band.shape[0])
    cap = int(capacity) if capacity is not None else max(nb * prm.s_init, 1)
    parts = torch.zeros((max(cap, 1), 4), dtype=phi.dtype, device=phi.device)
    count = torch.zeros(1, dtype=torch.int64, device=phi.device)
    need = lib().dcell_pls_scratch_bytes(ctypes.byref(g), nb, 0)
    scr = _scratch(need, phi.device)
    check(lib().dcell_pls_seed(ctypes.byref(g), L._dtype_code(phi), L._ptr(phi), L._ptr(band) if nb else None, nb,
                               ctypes.byref(prm), L._ptr(rng), L._ptr(parts), cap, L._ptr(count), scr.ptr,
                               scr.nbytes, _flags_arg(flags), L._stream()))
    return parts, int(count.item())


def reseed(phi: torch.Tensor, band: torch.Tensor, particles: torch.Tensor, n: int, rng: torch.Tensor, h=1.0,
           origin=(0, 0, 0), prm=None, flags=None):
    """ParticleLS_ReseedParticles (ParticleLS.c:202-295), 2D, on the first n
    particles.  Returns (particles, count): the same tensor when it has room
    for every new particle, else a larger copy; rng is advanced in place."""
    L._require_cuda(phi, band, particles, rng)
    prm = prm or params(phi.dim())
    g = geom(tuple(phi.shape), h, origin)
    nb = int(band.shape[0])
    cap = int(n) + nb * prm.s_init
    if particles.shape[0] < cap:
        grown = torch.zeros((cap, 4), dtype=particles.dtype, device=particles.device)
        grown[:n] = particles[:n]
        particles = grown
    count = torch.zeros(1, dtype=torch.int64, device=phi.device)
    need = lib().dcell_pls_scratch_bytes(ctypes.byref(g), nb, int(n))
    scr = _scratch(need, phi.device)
    check(lib().dcell_pls_reseed(ctypes.byref(g), L._dtype_code(phi), L._ptr(phi), L._ptr(band) if nb else None, nb,
                                 ctypes.byref(prm), L._ptr(rng), L._ptr(particles), int(n), int(particles.shape[0]),
                                 L._ptr(count), scr.ptr, scr.nbytes, _flags_arg(flags), L._stream()))
    return particles, int(count.item())


# ---------------------------------------------------------------------------
# struct _ParticleLS and the reference-named entry points

@dataclass
class ParticleLS:
    """Mirror of struct _ParticleLS (LSM_private.h:50-67) on the device."""
    prm: _lib.PlsParams
    particles: torch.Tensor
    count: int
    rng: torch.Tensor
    particles0: Optional[torch.Tensor] = None
    count0: int = 0
    scratch: Optional[_Scratch] = field(default=None, repr=False)

    @property
    def live(self) -> torch.Tensor:
        return self.particles[:self.count]


def LevelSetInitializeParticles(ls: L.LevelSet, rng_state: int = SEED_STATE, prm=None) -> ParticleLS:
    """LevelSetInitializeParticles (ParticleLS.c:6-88): seed from the band,
    adjust radii, and make LevelSetAdvectPLS the level set's Advect."""
    prm = prm or params(2 if ls.is2D else 3)
    rng = new_rng(rng_state, ls.phi.device)
    parts, count = seed(ls.phi, ls.band, rng, ls.h, ls.origin, prm, flags=ls.flags)
    ls.pls = ParticleLS(prm=prm, particles=parts, count=count, rng=rng)
    ls.Advect = LevelSetAdvectPLS
    return ls.pls


def ParticleLS_AdvectParticles(ls: L.LevelSet, velgrid: torch.Tensor, dt: float):
    advect(ls.pls.particles, ls.pls.count, velgrid, dt, ls.h, ls.origin, flags=ls.flags)


def ParticleLS_ErrorCorrection(ls: L.LevelSet):
    p = ls.pls
    g = geom(tuple(ls.phi.shape), ls.h, ls.origin)
    need = lib().dcell_pls_correct_scratch_bytes(ctypes.byref(g), L._dtype_code(ls.phi))
    if p.scratch is None or p.scratch.nbytes < need:
        p.scratch = _scratch(need, ls.phi.device)
    correct(ls.phi, ls.band, p.particles, p.count, ls.h, ls.origin, flags=ls.flags, scratch=p.scratch)


def ParticleLS_AdjustRadii(ls: L.LevelSet):
    adjust_radii(ls.phi, ls.pls.particles, ls.pls.count, ls.h, ls.origin, ls.pls.prm, flags=ls.flags)


def ParticleLS_ReseedParticles(ls: L.LevelSet):
    p = ls.pls
    p.particles, p.count = reseed(ls.phi, ls.band, p.particles, p.count, p.rng, ls.h, ls.origin, p.prm,
                                  flags=ls.flags)


def _reinit(ls: L.LevelSet):
    if ls.Reinitialize is None:
        raise DcellError(_lib.ERR_UNSUPPORTED, "reinitialisation threshold reached but no Reinitialize hook is set")
    ls.Reinitialize(ls)


def LevelSetAdvectPLS(ls: L.LevelSet, velgrid: torch.Tensor, dt: float):
    """LevelSetAdvectPLS (ParticleLS.c:299-329): particles by RK2, phi by SL,
    error correction, irregular nodes, CFL count; at the threshold
    reinitialise and reseed; adjust radii."""
    ParticleLS_AdvectParticles(ls, velgrid, dt)
    ls.phi0.copy_(ls.phi)
    L.LevelSetAdvectSL(ls, velgrid, dt)
    ParticleLS_ErrorCorrection(ls)
    L.LevelSetUpdateIrregularNodeList(ls)
    L.LevelSetCFLIncrement(ls, velgrid, dt)
    if ls.AdvectCount >= ls.AdvectThres or ls.CFLcount >= ls.CFLthres:
        _reinit(ls)
        ParticleLS_ReseedParticles(ls)
        ls.CFLcount = 0.0
        ls.AdvectCount = 0
    ParticleLS_AdjustRadii(ls)


def LevelSetAdvectPLSRK2HalfStep(ls: L.LevelSet, velgrid: torch.Tensor, dt: float):
    """ParticleLS.c:333-349: particles0 <- particles, advect, phi0 <- phi,
    SL, error correction, irregular nodes.  (The reference calls the 2D
    particle advection here in any dimension; this calls the level set's.)"""
    p = ls.pls
    p.particles0 = p.particles.clone()
    p.count0 = p.count
    ParticleLS_AdvectParticles(ls, velgrid, dt)
    ls.phi0.copy_(ls.phi)
    L.LevelSetAdvectSL(ls, velgrid, dt)
    ParticleLS_ErrorCorrection(ls)
    L.LevelSetUpdateIrregularNodeList(ls)


def LevelSetAdvectPLSRK2FullStep(ls: L.LevelSet, velgrid: torch.Tensor, dt: float):
    """ParticleLS.c:353-375: particles <- particles0, advect, SL from the same
    phi0, error correction, irregular nodes, CFL; at the threshold
    reinitialise, correct again and reseed; adjust radii."""
    p = ls.pls
    p.particles = p.particles0.clone()
    p.count = p.count0
    ParticleLS_AdvectParticles(ls, velgrid, dt)
    L.LevelSetAdvectSL(ls, velgrid, dt)
    ParticleLS_ErrorCorrection(ls)
    L.LevelSetUpdateIrregularNodeList(ls)
    L.LevelSetCFLIncrement(ls, velgrid, dt)
    if ls.AdvectCount >= ls.AdvectThres or ls.CFLcount >= ls.CFLthres:
        _reinit(ls)
        ParticleLS_ErrorCorrection(ls)
        ParticleLS_ReseedParticles(ls)
        ls.CFLcount = 0.0
        ls.AdvectCount = 0
    ParticleLS_AdjustRadii(ls)
