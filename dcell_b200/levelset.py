"""Host-side mirror of the reference's LevelSet interface over the C ABI.

Device memory comes from torch (CUDA tensors); every computation is a
kernel of ``libdcell_ls.so`` launched on torch's current stream.  Names and
argument meanings follow LevelSetMethod/LevelSetMethod.h:57-94:

    LevelSetCreate(dh, pos, size)                  LevelSet.c:6-37
    LevelSetAdvectSL(ls, velgrid, dt)              AdvectSL.c:6-19
    LevelSetAdvectSLRK2HalfStep / FullStep         AdvectRK2.c:5-26
    LevelSetUpdateIrregularNodeList(ls)            IrregularNodes.c:9-28
    LevelSetCFLIncrement / LevelSet_MaxVelocity    Advect.c:54-111
    LevelSetAdvectAndReinit(ls, velgrid, dt)       Advect.c:33-50

Errors raise :class:`dcell_b200.DcellError` (the reference returns a
PetscErrorCode).  Reinitialisation stays the reference's CPU fast marching:
``LevelSetAdvectAndReinit`` calls ``ls.Reinitialize(ls)``, a hook the caller
supplies, when the reference's thresholds trigger.

Layout: phi tensors are (nz, ny, nx) or (ny, nx); velocity grids append the
MAC components (3 or 2) innermost; bands are (nb, 3) int32 GLOBAL indices.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Callable, Optional

import numpy as np
import torch

from . import _lib
from ._lib import BACKTRACE, INTERP, NODE_DTYPE, DcellError, check, geom, lib


def _ptr(t: Optional[torch.Tensor]):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _dtype_code(t: torch.Tensor) -> int:
    if t.dtype == torch.float32:
        return _lib.F32
    if t.dtype == torch.float64:
        return _lib.F64
    raise DcellError(_lib.ERR_ARG, f"unsupported dtype {t.dtype} (float32 or float64)")


def _require_cuda(*ts):
    for t in ts:
        if t is None:
            continue
        if not t.is_cuda:
            raise DcellError(_lib.ERR_ARG, "tensors must live on a CUDA device (no CPU fallback)")
        if not t.is_contiguous():
            raise DcellError(_lib.ERR_ARG, "tensors must be contiguous")


def sl_step(phi0: torch.Tensor, vel: torch.Tensor, dt: float, h, origin=(0, 0, 0), band=None,
            interp="linear", backtrace="euler", out: Optional[torch.Tensor] = None,
            flags: Optional[torch.Tensor] = None) -> torch.Tensor:
    """One semi-Lagrangian step phi[X] = interp(phi0, S(X)) on the band (or everywhere).

    ``out`` (default: a copy of phi0) is updated in place at the advected points."""
    _require_cuda(phi0, vel, band, out, flags)
    dof = 3 if phi0.dim() == 3 else 2
    if tuple(vel.shape) != tuple(phi0.shape) + (dof,):
        raise DcellError(_lib.ERR_ARG, f"velocity shape {tuple(vel.shape)} != {tuple(phi0.shape) + (dof,)}")
    if vel.dtype != phi0.dtype:
        raise DcellError(_lib.ERR_ARG, "phi0 and velocity dtypes differ")
    if out is None:
        out = phi0.clone()
    if band is not None and (band.dtype != torch.int32 or band.dim() != 2 or band.shape[1] != 3):
        raise DcellError(_lib.ERR_ARG, "band must be an (nb, 3) int32 tensor")
    g = geom(phi0.shape, h, origin)
    nb = int(band.shape[0]) if band is not None else 0
    check(lib().dcell_sl_step(ctypes.byref(g), _dtype_code(phi0), _ptr(phi0), _ptr(vel), float(dt), _ptr(band), nb,
                              INTERP[interp] if isinstance(interp, str) else int(interp),
                              BACKTRACE[backtrace] if isinstance(backtrace, str) else int(backtrace),
                              _ptr(out), _ptr(flags), _stream()))
    return out


def split_bf16(phi: torch.Tensor, out: Optional[torch.Tensor] = None) -> torch.Tensor:
    """Packed BF16 hi/lo split of an FP32 grid (int32 words, see dcell_split_bf16)."""
    _require_cuda(phi, out)
    if phi.dtype != torch.float32:
        raise DcellError(_lib.ERR_ARG, "split_bf16 takes an FP32 grid")
    out = torch.empty(phi.shape, dtype=torch.int32, device=phi.device) if out is None else out
    g = geom(phi.shape, 1.0)
    check(lib().dcell_split_bf16(ctypes.byref(g), _ptr(phi), _ptr(out), _stream()))
    return out


def sl_step_tc_split(phi0_split: torch.Tensor, vel: torch.Tensor, dt: float, h, origin=(0, 0, 0), band=None,
                     backtrace="midpoint", out: Optional[torch.Tensor] = None,
                     out_split: Optional[torch.Tensor] = None, flags: Optional[torch.Tensor] = None):
    """Tensor-core step on a split-state level set; returns (phi, phi_split)."""
    _require_cuda(phi0_split, vel, band, out, out_split, flags)
    if phi0_split.dtype != torch.int32 or vel.dtype != torch.float32 or phi0_split.dim() != 3:
        raise DcellError(_lib.ERR_ARG, "phi0_split (int32 3D) and an FP32 velocity are required")
    if out is None:
        out = torch.empty(phi0_split.shape, dtype=torch.float32, device=phi0_split.device)
    g = geom(phi0_split.shape, h, origin)
    nb = int(band.shape[0]) if band is not None else 0
    check(lib().dcell_sl_step_tc_split(ctypes.byref(g), _ptr(phi0_split), _ptr(vel), float(dt), _ptr(band), nb,
                                       BACKTRACE[backtrace] if isinstance(backtrace, str) else int(backtrace),
                                       _ptr(out), _ptr(out_split), _ptr(flags), _stream()))
    return out, out_split


def sl_step_tc_split_planes(phi0_split: torch.Tensor, vel: torch.Tensor, dt: float, h, z_begin: int, z_end: int,
                            out: torch.Tensor, out_split: Optional[torch.Tensor] = None, origin=(0, 0, 0),
                            backtrace="midpoint", flags: Optional[torch.Tensor] = None):
    """The split-state tensor-core step on arrival planes [z_begin, z_end)
    only (multiples of the 8-plane brick depth, or z_end = nz): writes those
    planes of out / out_split, reads phi0_split wherever their departures
    reach (dcell_sl_step_tc_split_planes)."""
    _require_cuda(phi0_split, vel, out, out_split, flags)
    g = geom(phi0_split.shape, h, origin)
    check(lib().dcell_sl_step_tc_split_planes(ctypes.byref(g), _ptr(phi0_split), _ptr(vel), float(dt), int(z_begin),
                                              int(z_end),
                                              BACKTRACE[backtrace] if isinstance(backtrace, str) else int(backtrace),
                                              _ptr(out), _ptr(out_split), _ptr(flags), _stream()))
    return out, out_split


def nodes_to_numpy(raw: torch.Tensor, count: int) -> np.ndarray:
    """Device node buffer (uint8, 120 B/node) -> numpy structured array."""
    n = int(count)
    return np.frombuffer(raw[: n * NODE_DTYPE.itemsize].cpu().numpy().tobytes(), dtype=NODE_DTYPE)


def nodes_to_rows(nodes: np.ndarray) -> np.ndarray:
    """Structured nodes -> (n, 18) float64 rows: pos, axis, shift, signCenter,
    signFace, d, X, op, n, k (the row layout the test checkers use)."""
    r = np.zeros((len(nodes), 18))
    r[:, 0:3] = nodes["pos"]
    r[:, 3] = nodes["axis"]
    r[:, 4] = nodes["shift"]
    r[:, 5] = nodes["signCenter"]
    r[:, 6] = nodes["signFace"]
    r[:, 7] = nodes["d"]
    r[:, 8:11] = nodes["X"]
    r[:, 11:14] = nodes["op"]
    r[:, 14:17] = nodes["n"]
    r[:, 17] = nodes["k"]
    return r


def irregular_nodes(phi: torch.Tensor, h, band: torch.Tensor, origin=(0, 0, 0), with_surface=True,
                    capacity: Optional[int] = None, flags: Optional[torch.Tensor] = None):
    """Irregular-node pass; returns (raw uint8 node buffer, device int32 count tensor)."""
    _require_cuda(phi, band, flags)
    nb = int(band.shape[0])
    cap = capacity if capacity is not None else max(16, (10 if phi.dim() == 3 else 5) * nb)
    dev = phi.device
    raw = torch.empty(max(cap, 1) * NODE_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    count = torch.zeros(1, dtype=torch.int32, device=dev)
    sb = lib().dcell_irregular_nodes_scratch_bytes(nb)
    scratch = torch.empty(max(int(sb), 16), dtype=torch.uint8, device=dev)
    g = geom(phi.shape, h, origin)
    check(lib().dcell_irregular_nodes(ctypes.byref(g), _dtype_code(phi), _ptr(phi), _ptr(band), nb,
                                      1 if with_surface else 0, _ptr(raw), cap, _ptr(count), _ptr(scratch),
                                      scratch.numel(), _ptr(flags), _stream()))
    return raw, count


def max_velocity(vel: torch.Tensor, h, raw_nodes: torch.Tensor, count: torch.Tensor, origin=(0, 0, 0)):
    _require_cuda(vel, raw_nodes, count)
    shape = tuple(vel.shape[:-1])
    g = geom(shape, h, origin)
    out = torch.zeros(1, dtype=torch.float64, device=vel.device)
    cap = raw_nodes.numel() // NODE_DTYPE.itemsize
    check(lib().dcell_max_velocity(ctypes.byref(g), _dtype_code(vel), _ptr(vel), _ptr(raw_nodes), _ptr(count), cap,
                                   _ptr(out), _stream()))
    return out


def reinitialize(phi: torch.Tensor, raw_nodes: torch.Tensor, count, band_width: float = 6.0, bucket: float = 1.0 / 64,
                 origin=(0, 0, 0), flags: Optional[torch.Tensor] = None):
    """Narrow-band reinitialisation of phi in place (cell units; the
    reference's LevelSetReinitialize, LevelSetMethod/FastMarching.c:11-146,
    after its LevelSetResize) from the irregular nodes of phi (raw buffer and
    count as irregular_nodes returns them).  Returns the band, (nb, 3) int32
    global indices in grid order."""
    _require_cuda(phi, raw_nodes, flags)
    nn = int(count.item()) if isinstance(count, torch.Tensor) else int(count)
    cap = phi.numel()
    band = torch.empty((max(cap, 1), 3), dtype=torch.int32, device=phi.device)
    nb = torch.zeros(1, dtype=torch.int32, device=phi.device)
    g = geom(phi.shape, 1.0, origin)
    sb = int(lib().dcell_reinit_scratch_bytes(ctypes.byref(g), _dtype_code(phi)))
    scratch = torch.empty(sb + 256, dtype=torch.uint8, device=phi.device)
    base = scratch.data_ptr()
    off = (-base) % 256
    check(lib().dcell_reinitialize(ctypes.byref(g), _dtype_code(phi), _ptr(phi), _ptr(raw_nodes), nn,
                                   float(band_width), float(bucket), _ptr(band), cap, _ptr(nb),
                                   ctypes.c_void_p(base + off), sb, _ptr(flags), _stream()))
    return band[: int(nb.item())]


def _field_dims(global_field: torch.Tensor):
    if global_field.dim() == 4:
        gz, gy, gx, gdof = global_field.shape
    elif global_field.dim() == 3:
        gy, gx, gdof = global_field.shape
        gz = 1
    else:
        raise DcellError(_lib.ERR_ARG, "global field must be [z][y][x][c] or [y][x][c]")
    return (ctypes.c_int * 3)(int(gx), int(gy), int(gz)), int(gdof)


def velocity_box(global_field: torch.Tensor, origin, shape, first: int = 1):
    """The velocity grid of a level set's phi box (global index `origin`
    (x, y(, z)), extents `shape` (nz, ny, nx) or (ny, nx)) from the fluid's
    global field: the reference's LevelSetGetVelocity (Advect.c:145-192) with
    the Global Array on the device.  Components first .. first+dim-1; zero
    outside the field.  Returns shape + (dim,)."""
    _require_cuda(global_field)
    gd, gdof = _field_dims(global_field)
    dim = len(shape)
    out = torch.empty(tuple(shape) + (dim,), dtype=global_field.dtype, device=global_field.device)
    g = geom(shape, 1.0, origin)
    check(lib().dcell_velocity_box(ctypes.byref(g), _dtype_code(global_field), _ptr(global_field), gd, gdof, int(first),
                                   _ptr(out), _stream()))
    return out


def velocity_boxes(global_field: torch.Tensor, boxes, first: int = 1):
    """velocity_box for a list of (origin, shape) boxes in one launch; returns
    one tensor per box (views of one packed buffer)."""
    _require_cuda(global_field)
    gd, gdof = _field_dims(global_field)
    dim = global_field.dim() - 1
    rec = np.zeros(len(boxes), dtype=_lib.BOX_DTYPE)
    off, sizes = 0, []
    for b, (o, sh) in enumerate(boxes):
        n = int(np.prod(sh))
        rec[b]["offset"] = off
        rec[b]["p"] = tuple(int(v) for v in o) + (0,) * (3 - len(o))
        rec[b]["n"] = tuple(int(v) for v in reversed(sh)) + (1,) * (3 - len(sh))
        sizes.append(n)
        off += n
    out = torch.empty(max(off, 1) * dim, dtype=global_field.dtype, device=global_field.device)
    d_rec = torch.from_numpy(np.frombuffer(rec.tobytes(), dtype=np.uint8).copy()).to(global_field.device)
    check(lib().dcell_velocity_boxes(_ptr(d_rec), len(boxes), dim, _dtype_code(global_field), _ptr(global_field), gd,
                                     gdof, int(first), max(sizes, default=0), _ptr(out), _stream()))
    res, start = [], 0
    for (o, sh), n in zip(boxes, sizes):
        res.append(out[start * dim:(start + n) * dim].view(tuple(sh) + (dim,)))
        start += n
    return res


def volume(phi: torch.Tensor, h, eps: float):
    """Enclosed volume through the smoothed Heaviside (FP64, deterministic)."""
    _require_cuda(phi)
    g = geom(phi.shape, h)
    out = torch.zeros(1, dtype=torch.float64, device=phi.device)
    sb = int(lib().dcell_volume_scratch_bytes())
    scratch = torch.empty(sb, dtype=torch.uint8, device=phi.device)
    check(lib().dcell_volume(ctypes.byref(g), _dtype_code(phi), _ptr(phi), float(eps), _ptr(out), _ptr(scratch), sb,
                             _stream()))
    return out


def advect_mac(phi: torch.Tensor, u: torch.Tensor, v: torch.Tensor, w: Optional[torch.Tensor], dt: float, h,
               origin=(0, 0, 0), out: Optional[torch.Tensor] = None) -> torch.Tensor:
    """One first-order conservative upwind step on MAC faces
    (LevelSetAdvectMAC / LevelSetAdvectMAC_3D, LevelSetMethod/AdvectMAC.c:
    18-111): phi, u, v (, w in 3D) share the grid at global `origin`; u[k, j,
    i] is the face between cells i-1 and i.  Writes the updated range
    [max(p, 0), p + n - 1) of each axis into `out` (default: a copy of phi,
    so the other points keep phi's values) and returns it."""
    is3 = phi.dim() == 3
    ts = (phi, u, v, w) if is3 else (phi, u, v)
    _require_cuda(*ts)
    for t in ts[1:]:
        if t.shape != phi.shape or t.dtype != phi.dtype or not t.is_contiguous():
            raise ValueError("u, v (, w) must be contiguous, with phi's shape and dtype")
    if not phi.is_contiguous():
        raise ValueError("phi must be contiguous")
    if out is None:
        out = phi.clone()
    elif out.shape != phi.shape or out.dtype != phi.dtype or not out.is_contiguous():
        raise ValueError("out must be contiguous, with phi's shape and dtype")
    g = geom(phi.shape, h, origin)
    check(lib().dcell_advect_mac(ctypes.byref(g), _dtype_code(phi), _ptr(phi), _ptr(u), _ptr(v),
                                 _ptr(w) if is3 else None, float(dt), _ptr(out), _stream()))
    return out


# ---------------------------------------------------------------------------
# LevelSet object and the reference-named entry points
@dataclass
class LevelSet:
    """Mirror of struct _LevelSet (LevelSetMethod.h:10-26) with device grids."""
    phi: torch.Tensor
    phi0: torch.Tensor
    h: tuple
    origin: tuple
    band: torch.Tensor
    bandWidth: float = 6.0
    PHI_INF: float = 7.5
    CFLthres: float = 3.0
    CFLcount: float = 0.0
    AdvectThres: int = 1000
    AdvectCount: int = 0
    maxVel: float = 0.0
    interp: str = "linear"
    backtrace: str = "euler"
    irregularNodes: Optional[torch.Tensor] = None
    irregularCount: Optional[torch.Tensor] = None
    Advect: Optional[Callable] = None
    Reinitialize: Optional[Callable] = None
    flags: Optional[torch.Tensor] = field(default=None)
    pls: Optional[object] = None  # dcell_b200.pls.ParticleLS once particles are seeded

    @property
    def is2D(self) -> bool:
        return self.phi.dim() == 2


def LevelSetCreate(dh, pos, size, dtype=torch.float32, device="cuda") -> LevelSet:
    """LevelSetCreate (LevelSet.c:6-37): zeroed phi/phi0 on [pos, pos+size), bandwidth 6."""
    nx, ny, nz = (int(v) for v in size)
    shape = (ny, nx) if nz < 2 else (nz, ny, nx)
    phi = torch.zeros(shape, dtype=dtype, device=device)
    ls = LevelSet(phi=phi, phi0=phi.clone(), h=tuple(np.broadcast_to(np.asarray(dh, float), (3,))),
                  origin=tuple(int(v) for v in pos), band=torch.zeros((0, 3), dtype=torch.int32, device=device))
    LevelSetSetBandWidth(ls, 6.0)
    ls.Advect = LevelSetAdvectAndReinit
    ls.flags = torch.zeros(1, dtype=torch.int32, device=device)
    return ls


def LevelSetSetBandWidth(ls: LevelSet, bandwidth: float):
    """LevelSetSetBandWidth (LevelSet.c:60-66): PHI_INF = bandWidth + 1.5."""
    ls.bandWidth = float(bandwidth)
    ls.PHI_INF = ls.bandWidth + 1.5


def LevelSetAdvectSL(ls: LevelSet, velgrid: torch.Tensor, dt: float):
    """phi[band] <- SL(phi0, velgrid, dt) (AdvectSL.c:6-89)."""
    sl_step(ls.phi0, velgrid, dt, ls.h, ls.origin, band=ls.band, interp=ls.interp, backtrace=ls.backtrace,
            out=ls.phi, flags=ls.flags)


def LevelSetUpdateIrregularNodeList(ls: LevelSet, with_surface: bool = False):
    raw, count = irregular_nodes(ls.phi, ls.h, ls.band, ls.origin, with_surface=with_surface, flags=ls.flags)
    ls.irregularNodes, ls.irregularCount = raw, count


def LevelSetAdvectSLRK2HalfStep(ls: LevelSet, velgrid: torch.Tensor, dt: float):
    """AdvectRK2.c:5-14: phi0 <- phi; SL(dt); irregular nodes."""
    ls.phi0.copy_(ls.phi)
    LevelSetAdvectSL(ls, velgrid, dt)
    LevelSetUpdateIrregularNodeList(ls)


def LevelSetAdvectSLRK2FullStep(ls: LevelSet, velgrid: torch.Tensor, dt: float):
    """AdvectRK2.c:18-26: SL(dt) from the same phi0; irregular nodes."""
    LevelSetAdvectSL(ls, velgrid, dt)
    LevelSetUpdateIrregularNodeList(ls)


def LevelSet_MaxVelocity(ls: LevelSet, velgrid: torch.Tensor) -> float:
    """Advect.c:70-111: max |V| over the irregular nodes' positions."""
    if ls.irregularNodes is None:
        ls.maxVel = 0.0
        return 0.0
    ls.maxVel = float(max_velocity(velgrid, ls.h, ls.irregularNodes, ls.irregularCount, ls.origin).item())
    return ls.maxVel


def LevelSetCFLIncrement(ls: LevelSet, velgrid: torch.Tensor, dt: float):
    """Advect.c:54-66."""
    LevelSet_MaxVelocity(ls, velgrid)
    ls.CFLcount += dt * ls.maxVel / ls.h[0]
    ls.AdvectCount += 1


def LevelSetAdvectAndReinit(ls: LevelSet, velgrid: torch.Tensor, dt: float):
    """Advect.c:33-50: copy, SL, CFL bookkeeping, irregular nodes, reinit trigger."""
    ls.phi0.copy_(ls.phi)
    LevelSetAdvectSL(ls, velgrid, dt)
    LevelSetCFLIncrement(ls, velgrid, dt)
    LevelSetUpdateIrregularNodeList(ls)
    if ls.AdvectCount > ls.AdvectThres or ls.CFLcount > ls.CFLthres:
        ls.CFLcount = 0.0
        ls.AdvectCount = 0
        if ls.Reinitialize is None:
            raise DcellError(_lib.ERR_UNSUPPORTED, "reinitialisation threshold reached but no Reinitialize hook is "
                             "set (fast marching stays the reference's CPU LevelSetReinitialize)")
        ls.Reinitialize(ls)


def LevelSetAdvectMAC(ls: LevelSet, d, dt: float, u: torch.Tensor, v: torch.Tensor, new: LevelSet):
    """LevelSetAdvectMAC (AdvectMAC.c:18-60): one upwind step of ls.phi into
    new.phi on the MAC faces u, v of ls's grid (d: the spacing)."""
    advect_mac(ls.phi, u, v, None, dt, d, ls.origin, out=new.phi)


def LevelSetAdvectMAC_3D(ls: LevelSet, d, dt: float, u: torch.Tensor, v: torch.Tensor, w: torch.Tensor,
                         new: LevelSet):
    """LevelSetAdvectMAC_3D (AdvectMAC.c:62-111)."""
    advect_mac(ls.phi, u, v, w, dt, d, ls.origin, out=new.phi)


def LevelSetReinitializeGPU(ls: LevelSet, bucket: float = 1.0 / 64):
    """A Reinitialize hook on the GPU: the reference's LevelSetReinitialize
    (FastMarching.c:11-146) without its LevelSetResize -- bucketed fast
    marching from the irregular nodes of phi, new band in grid order."""
    raw, count = irregular_nodes(ls.phi, ls.h, ls.band, ls.origin, with_surface=False, flags=ls.flags)
    ls.band = reinitialize(ls.phi, raw, count, ls.bandWidth, bucket, ls.origin, flags=ls.flags)


class ResidentLevelSet:
    """A level set kept on the device across LevelSetAdvectAndReinit steps
    (Advect.c:33-50) through the host-buffer C ABI (dcell_ls_resident_*):
    phi and its band go up once, each step uploads only its velocity.

        r = ResidentLevelSet(phi_host, h, origin, band_host, precision="f32")
        for s in range(steps):
            r.advect_and_reinit(vel_host, dt, interp="cubic_tc", backtrace="midpoint")
        phi_host, band_host = r.get()
    """

    def __init__(self, phi: np.ndarray, h, origin=(0, 0, 0), band=None, precision="f64", device: int = 0,
                 bandWidth: float = 6.0, CFLthres: float = 3.0, AdvectThres: int = 1000):
        self.shape = tuple(phi.shape)
        self.g = geom(self.shape, h, origin)
        self.s = ctypes.c_void_p()
        check(lib().dcell_session_create(int(device), ctypes.byref(self.s)))
        self.loop = _lib.LsLoop(CFLcount=0.0, CFLthres=float(CFLthres), maxVel=0.0, bandWidth=float(bandWidth),
                                AdvectCount=0, AdvectThres=int(AdvectThres), reinitialized=0, band=0)
        p = np.ascontiguousarray(phi, dtype=np.float64)
        b = np.ascontiguousarray(band if band is not None else np.zeros((0, 3)), dtype=np.int32).reshape(-1, 3)
        self.precision = _lib.F32 if precision in ("f32", _lib.F32) else _lib.F64
        check(lib().dcell_ls_resident_set(self.s, ctypes.byref(self.g), p.ctypes.data_as(ctypes.c_void_p),
                                          b.ctypes.data_as(ctypes.c_void_p), b.shape[0], self.precision))

    def advect_and_reinit(self, vel, dt: float, interp="linear", backtrace="euler", dense: bool = False):
        """One step; vel a host array (numpy or CPU tensor, FP32 or FP64,
        (..., dof) in the reference's layout).  Returns the loop counters."""
        v = vel.numpy() if isinstance(vel, torch.Tensor) else vel
        v = np.ascontiguousarray(v)
        vdt = _lib.F32 if v.dtype == np.float32 else _lib.F64
        if vdt == _lib.F64:
            v = np.ascontiguousarray(v, dtype=np.float64)
        ptr = ctypes.c_void_p(vel.data_ptr()) if isinstance(vel, torch.Tensor) and vel.is_contiguous() and \
            vel.dtype in (torch.float32, torch.float64) else v.ctypes.data_as(ctypes.c_void_p)
        check(lib().dcell_ls_resident_advect_and_reinit(
            self.s, ctypes.byref(self.g), ptr, vdt, float(dt), INTERP[interp] if isinstance(interp, str) else
            int(interp), BACKTRACE[backtrace] if isinstance(backtrace, str) else int(backtrace), int(dense),
            ctypes.byref(self.loop)))
        return self.loop

    def get(self, out=None):
        """(phi (FP64 host array), band (nb, 3) int32).  `out`: a C-contiguous
        FP64 host array (numpy, or a CPU tensor, pinned for the full copy
        rate) of the grid's shape that receives phi; a new array otherwise."""
        if out is None:
            phi = np.empty(self.shape, dtype=np.float64)
            ptr = phi.ctypes.data_as(ctypes.c_void_p)
        else:
            phi = out
            if isinstance(out, torch.Tensor):
                if out.device.type != "cpu" or out.dtype != torch.float64 or not out.is_contiguous() or \
                        tuple(out.shape) != self.shape:
                    raise ValueError("out must be a contiguous CPU float64 tensor of the grid's shape")
                ptr = ctypes.c_void_p(out.data_ptr())
            else:
                if out.dtype != np.float64 or not out.flags["C_CONTIGUOUS"] or tuple(out.shape) != self.shape:
                    raise ValueError("out must be a C-contiguous float64 array of the grid's shape")
                ptr = out.ctypes.data_as(ctypes.c_void_p)
        n = ctypes.c_int()
        check(lib().dcell_ls_resident_get(self.s, ctypes.byref(self.g), ptr, None, 0, ctypes.byref(n)))
        band = np.empty((max(n.value, 1), 3), dtype=np.int32)
        check(lib().dcell_ls_resident_get(self.s, ctypes.byref(self.g), None, band.ctypes.data_as(ctypes.c_void_p),
                                          n.value, ctypes.byref(n)))
        return phi, band[: n.value]

    def close(self):
        if self.s:
            lib().dcell_session_destroy(self.s)
            self.s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def status(ls: LevelSet) -> int:
    """Read and clear the device status flags of ``ls`` (DCELL_FLAG_* bits)."""
    v = int(ls.flags.item())
    ls.flags.zero_()
    return v
