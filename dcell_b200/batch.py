"""Batched cells: many DCells' level sets of uneven sizes advanced together.

The reference advances the level sets of a rank's cells one after another
(DWorld/DCellsArray.c:50-102, each through LevelSetAdvect).  Here the cells'
grids are packed into one FP32 buffer, covered by a queue of fixed-size
tiles, and one persistent kernel walks the queue per SL step
(dcell_batch_sl_step); several steps are captured into one CUDA graph and
replayed.  The tile shape and the number of persistent CTAs per SM are
chosen by a small autotuner that times the candidates on the batch itself.
"""
from __future__ import annotations

import ctypes
import json
import math
import os
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _lib, fields
from ._lib import BACKTRACE, INTERP, DcellError, check, lib
from .levelset import split_bf16

CELL_DTYPE = np.dtype([("offset", "<i8"), ("n", "<i4", 3), ("pad", "<i4"), ("h", "<f8", 3), ("dt", "<f8")])
TILE_DTYPE = np.dtype([("cell", "<i4"), ("x0", "<i4"), ("y0", "<i4"), ("z0", "<i4")])
assert CELL_DTYPE.itemsize == 56 and TILE_DTYPE.itemsize == 16

# 128-point tiles for the tensor-core path (one MMA row block per tile)
TC_TILES = [(32, 2, 2), (16, 4, 2), (16, 2, 4), (8, 4, 4), (8, 8, 2), (4, 4, 8), (32, 4, 1), (64, 2, 1)]
CORE_TILES = [(32, 4, 2), (32, 2, 4), (16, 4, 4), (32, 8, 1), (64, 2, 2), (8, 8, 4)]


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class CellBatch:
    """A packed batch of 3D cell grids (FP32) on one device."""

    def __init__(self, phis: Sequence[torch.Tensor], vels: Sequence[torch.Tensor], hs, dts, device="cuda",
                 padded: bool = False):
        """padded: rows padded to multiples of 4 points (the extra columns
        hold copies of each cell's last column) for the TMA-staged batched
        split-state step (step_tc_split_tma); the other steps need the
        unpadded packing."""
        if len(phis) != len(vels):
            raise DcellError(_lib.ERR_ARG, "one velocity per cell")
        self.device = torch.device(device)
        self.ncells = len(phis)
        self.padded = bool(padded)
        self.shapes = [tuple(int(v) for v in p.shape) for p in phis]
        # stored shapes: the padded row length in x
        self.stored = [(s[0], s[1], (s[2] + 3) // 4 * 4 if padded else s[2]) for s in self.shapes]
        sizes = [int(np.prod(s)) for s in self.stored]
        self.offsets = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
        self.npoints = int(sum(sizes))
        if 3 * self.npoints >= 2 ** 31:
            raise DcellError(_lib.ERR_ARG, "batch too large for 32-bit velocity offsets")
        self.phi = torch.empty(self.npoints, dtype=torch.float32, device=self.device)
        self.vel = torch.empty(3 * self.npoints, dtype=torch.float32, device=self.device)
        for i, (p, v) in enumerate(zip(phis, vels)):
            o, n = int(self.offsets[i]), sizes[i]
            if tuple(v.shape) != self.shapes[i] + (3,):
                raise DcellError(_lib.ERR_ARG, f"cell {i}: velocity shape {tuple(v.shape)}")
            nx, sx = self.shapes[i][2], self.stored[i][2]
            pp = p.to(self.device, torch.float32)
            vv = v.to(self.device, torch.float32)
            if sx > nx:  # pad columns: copies of the last column
                pp = torch.cat([pp, pp[..., -1:].expand(*pp.shape[:2], sx - nx)], dim=2)
                vv = torch.cat([vv, vv[..., -1:, :].expand(*vv.shape[:2], sx - nx, 3)], dim=2)
            self.phi[o:o + n] = pp.reshape(-1)
            self.vel[3 * o:3 * (o + n)] = vv.reshape(-1)
        cells = np.zeros(self.ncells, dtype=CELL_DTYPE)
        cells["offset"] = self.offsets
        cells["n"] = [(s[2], s[1], s[0]) for s in self.shapes]
        if padded:
            cells["pad"] = [s[2] for s in self.stored]
        hs = np.broadcast_to(np.asarray(hs, dtype=np.float64).reshape(-1, 3) if np.ndim(hs) > 1 else
                             np.asarray(hs, dtype=np.float64), (self.ncells, 3))
        cells["h"] = hs
        cells["dt"] = np.broadcast_to(np.asarray(dts, dtype=np.float64), (self.ncells,))
        self.cells_host = cells
        self.cells = torch.as_tensor(cells.view(np.uint8), device=self.device)
        self._plans = {}
        self.tuned = {}

    def _unpadded(self):
        if self.padded:
            raise DcellError(_lib.ERR_ARG, "this step reads the unpadded packing: use step_tc_split_tma on a "
                                           "padded batch")

    # ------------------------------------------------------------------
    def plan(self, tile):
        """Device tile queue covering every point once (dcell_batch_plan)."""
        tile = tuple(int(v) for v in tile)
        if tile not in self._plans:
            n = ctypes.c_int()
            L = lib()
            rc = L.dcell_batch_plan(self.cells_host.ctypes.data_as(ctypes.c_void_p), self.ncells, *tile, None, 0,
                                    ctypes.byref(n))
            if rc not in (_lib.OK, _lib.ERR_CAPACITY):
                check(rc)
            tiles = np.zeros(n.value, dtype=TILE_DTYPE)
            check(L.dcell_batch_plan(self.cells_host.ctypes.data_as(ctypes.c_void_p), self.ncells, *tile,
                                     tiles.ctypes.data_as(ctypes.c_void_p), n.value, ctypes.byref(n)))
            self._plans[tile] = (torch.as_tensor(tiles.view(np.uint8), device=self.device), n.value)
        return self._plans[tile]

    def step(self, phi0, phi, interp="cubic_tc", backtrace="midpoint", tile=None, ctas_per_sm=None, flags=None):
        """One SL step of every cell: phi <- SL(phi0) in one persistent launch."""
        self._unpadded()
        mode = INTERP[interp] if isinstance(interp, str) else int(interp)
        if tile is None or ctas_per_sm is None:
            t, c = self.tuned.get((mode, BACKTRACE[backtrace] if isinstance(backtrace, str) else backtrace),
                                  ((32, 2, 2), 4) if mode == _lib.CUBIC_TC else ((32, 4, 2), 4))
            tile = tile or t
            ctas_per_sm = ctas_per_sm or c
        tiles, ntiles = self.plan(tile)
        check(lib().dcell_batch_sl_step(_vp(self.cells), self.ncells, _vp(tiles), ntiles, *tile, int(ctas_per_sm),
                                        _vp(phi0), _vp(self.vel), _vp(phi), mode,
                                        BACKTRACE[backtrace] if isinstance(backtrace, str) else int(backtrace),
                                        _vp(flags) if flags is not None else None, _stream()))
        return phi

    def step_per_cell(self, phi0, phi, interp="cubic_tc", backtrace="midpoint"):
        """The comparator: one dcell_sl_step launch per cell."""
        self._unpadded()
        mode = INTERP[interp] if isinstance(interp, str) else int(interp)
        bt = BACKTRACE[backtrace] if isinstance(backtrace, str) else int(backtrace)
        L = lib()
        st = _stream()
        for i, s in enumerate(self.shapes):
            c = self.cells_host[i]
            g = _lib.geom(s, tuple(c["h"]))
            o = int(self.offsets[i])
            check(L.dcell_sl_step(ctypes.byref(g), _lib.F32, ctypes.c_void_p(phi0.data_ptr() + 4 * o),
                                  ctypes.c_void_p(self.vel.data_ptr() + 12 * o), float(c["dt"]), None, 0, mode, bt,
                                  ctypes.c_void_p(phi.data_ptr() + 4 * o), None, st))
        return phi

    # ------------------------------------------------------------------
    BRICK = (32, 4, 8)  # the brick kernel's points per brick (x, y, z)

    def split(self, phi=None):
        """Packed BF16 hi/lo words of the packed FP32 phi (the split state)."""
        phi = self.phi if phi is None else phi
        return split_bf16(phi.view(1, 1, -1)).view(-1)

    def step_tc_split(self, phi0_split, phi, phi_split, backtrace="midpoint", flags=None):
        """One split-state tensor-core step of every cell in ONE launch over
        bricks of 32 x 4 x 8 points (dcell_batch_sl_step_tc_split): phi and
        phi_split (the next step's input) receive the new state."""
        self._unpadded()
        bricks, n = self.plan(self.BRICK)
        check(lib().dcell_batch_sl_step_tc_split(_vp(self.cells), self.ncells, _vp(bricks), n, _vp(phi0_split),
                                                 _vp(self.vel), BACKTRACE[backtrace] if isinstance(backtrace, str)
                                                 else int(backtrace), _vp(phi), _vp(phi_split),
                                                 _vp(flags) if flags is not None else None, _stream()))
        return phi, phi_split

    def step_tc_split_per_cell(self, phi0_split, phi, phi_split, backtrace="midpoint"):
        """The comparator: dcell_sl_step_tc_split launched once per cell."""
        self._unpadded()
        bt = BACKTRACE[backtrace] if isinstance(backtrace, str) else int(backtrace)
        L = lib()
        st = _stream()
        for i, s in enumerate(self.shapes):
            c = self.cells_host[i]
            g = _lib.geom(s, tuple(c["h"]))
            o = int(self.offsets[i])
            check(L.dcell_sl_step_tc_split(ctypes.byref(g), ctypes.c_void_p(phi0_split.data_ptr() + 4 * o),
                                           ctypes.c_void_p(self.vel.data_ptr() + 12 * o), float(c["dt"]), None, 0,
                                           bt, ctypes.c_void_p(phi.data_ptr() + 4 * o),
                                           ctypes.c_void_p(phi_split.data_ptr() + 4 * o), None, st))
        return phi, phi_split

    def cell_view(self, flat, i):
        """Cell i's grid in a packed array (its real columns when padded)."""
        o, st = int(self.offsets[i]), self.stored[i]
        return flat[o:o + int(np.prod(st))].view(st)[..., :self.shapes[i][2]]

    def step_tc_split_tma(self, phi0_split, phi, phi_split, backtrace="midpoint", flags=None):
        """One split-state tensor-core step of every cell of a padded batch
        in ONE launch over bricks of 32 x 4 x 8 points, the boxes staged by
        TMA with a tensor map per cell (dcell_batch_sl_step_tc_split_tma);
        the maps of each (phi0_split, velocity) buffer pair are built once."""
        if not self.padded:
            raise DcellError(_lib.ERR_ARG, "the TMA-staged batched step needs CellBatch(..., padded=True)")
        bricks, n = self.plan(self.BRICK)
        key = (phi0_split.data_ptr(), self.vel.data_ptr())
        maps = self._maps.get(key) if hasattr(self, "_maps") else None
        if maps is None:
            if not hasattr(self, "_maps"):
                self._maps = {}
            maps = torch.empty(int(lib().dcell_batch_tma_maps_bytes(self.ncells)), dtype=torch.uint8,
                               device=self.device)
            check(lib().dcell_batch_tma_maps(self.cells_host.ctypes.data_as(ctypes.c_void_p), self.ncells,
                                             _vp(phi0_split), _vp(self.vel), _vp(maps), _stream()))
            self._maps[key] = maps
        check(lib().dcell_batch_sl_step_tc_split_tma(_vp(self.cells), self.ncells, _vp(bricks), n, _vp(maps),
                                                     _vp(phi0_split), _vp(self.vel),
                                                     BACKTRACE[backtrace] if isinstance(backtrace, str)
                                                     else int(backtrace), _vp(phi), _vp(phi_split),
                                                     _vp(flags) if flags is not None else None, _stream()))
        return phi, phi_split

    # ------------------------------------------------------------------
    def autotune(self, interp="cubic_tc", backtrace="midpoint", candidates=None, ctas=None, reps=3, cache=None):
        """Time every (tile shape, CTAs per SM) candidate on this batch; keep the fastest."""
        mode = INTERP[interp] if isinstance(interp, str) else int(interp)
        bt = BACKTRACE[backtrace] if isinstance(backtrace, str) else int(backtrace)
        key = self.signature(mode, bt)
        if cache and os.path.exists(cache):
            saved = json.load(open(cache)).get(key)
            if saved:
                self.tuned[(mode, bt)] = (tuple(saved["tile"]), saved["ctas_per_sm"])
                return self.tuned[(mode, bt)], []
        candidates = candidates or (TC_TILES if mode == _lib.CUBIC_TC else CORE_TILES)
        ctas = ctas or ([2, 3, 4] if mode == _lib.CUBIC_TC else [2, 4, 8])
        a, b = self.phi.clone(), torch.empty_like(self.phi)
        results = []
        for tile in candidates:
            for c in ctas:
                self.step(a, b, interp, backtrace, tile, c)  # warm-up (also builds the plan)
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                for _ in range(reps):
                    self.step(a, b, interp, backtrace, tile, c)
                e1.record()
                torch.cuda.synchronize()
                results.append((e0.elapsed_time(e1) / reps, tile, c))
        results.sort()
        best = results[0]
        self.tuned[(mode, bt)] = (best[1], best[2])
        if cache:
            d = json.load(open(cache)) if os.path.exists(cache) else {}
            d[key] = {"tile": list(best[1]), "ctas_per_sm": best[2], "ms": best[0]}
            os.makedirs(os.path.dirname(os.path.abspath(cache)), exist_ok=True)
            json.dump(d, open(cache, "w"), indent=1)
        return self.tuned[(mode, bt)], results

    def signature(self, mode, bt):
        name = torch.cuda.get_device_name(self.device)
        h = hash(tuple(self.shapes)) & 0xFFFFFFFF
        return f"{name}|cells={self.ncells}|points={self.npoints}|shapes={h:08x}|interp={mode}|bt={bt}"

    def capture(self, nsteps, interp="cubic_tc", backtrace="midpoint"):
        """CUDA graph of nsteps batched steps (ping-pong between two buffers);
        returns (graph, buffers) -- replay advances self.phi-like buffer a."""
        a = self.phi.clone()
        b = torch.empty_like(a)
        s = torch.cuda.Stream(device=self.device)
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):  # warm-up outside capture
            self.step(a, b, interp, backtrace)
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            x, y = a, b
            for _ in range(nsteps):
                self.step(x, y, interp, backtrace)
                x, y = y, x
        out = a if nsteps % 2 == 0 else b
        return g, (a, b, out)


def c4_workload(ncells=512, seed=2024, emin=32, emax=96, nmodes=8, device="cuda", dtype=torch.float32):
    """The batching workload: `ncells` cells with per-axis edges drawn
    uniformly from [emin, emax] (seeded); each a randomly centred ellipsoid
    with semi-axes in [0.2, 0.4] of its box, in its own divergence-free MAC
    velocity from `nmodes` random Fourier modes (unit amplitude, wave numbers
    1..4).  Each cell's box is [0,1]^3; dt is the CFL-0.5 step of the fastest
    cell.  Returns (phis, vels, hs, dt)."""
    rng = np.random.default_rng(seed)
    phis, vels, hs = [], [], []
    vmax = 0.0
    for i in range(ncells):
        nx, ny, nz = (int(v) for v in rng.integers(emin, emax + 1, size=3))
        semi = rng.uniform(0.2, 0.4, size=3)
        center = rng.uniform(semi.max(), 1 - semi.max(), size=3) if semi.max() < 0.5 else np.full(3, 0.5)
        phi = fields.ellipsoid_sdf((nz, ny, nx), center, semi, device=device)
        k, a, ph = fields.fourier_modes(nmodes, seed * 100003 + i)
        coeffs = 1.0 / (2 * math.pi * np.linalg.norm(k, axis=1))  # unit velocity amplitude per mode
        vel = fields.fourier_velocity((nz, ny, nx), coeffs, (k, a, ph), device=device)
        h = (1.0 / nx, 1.0 / ny, 1.0 / nz)
        vmax = max(vmax, max(float(vel[..., d].abs().max()) / h[d] for d in range(3)))
        phis.append(phi.to(dtype))
        vels.append(vel.to(dtype))
        hs.append(h)
    dt = 0.5 / vmax
    return phis, vels, np.array(hs), dt
