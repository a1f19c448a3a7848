"""Multi-GPU transport: one process per GPU over torch.distributed.

Two decompositions of the level-set transport step:

* **cells over ranks** -- the reference's own parallelism (each MPI rank owns
  whole DCells, DWorld/DCellsArray.c:50-64; a level set is never split):
  cells go to ranks largest-first onto the least-loaded rank, every rank
  advances its cells with no collective on the data path, and only the
  per-step diagnostics (enclosed volume, max |V| for the CFL count) are
  all-reduced.
* **z-slabs of one large grid** -- each rank owns a contiguous z-range plus
  `halo` planes on each side; before every step the halo planes of phi0 are
  exchanged with the z-neighbours (point-to-point, NCCL over NVLink on GPUs),
  the velocity halos once.  `halo` must cover the departure reach:
  ceil(max |w| dt / h_z) + 2 planes for the cubic stencil.

The per-slab / per-cell step is a callable (default: the CUDA kernels via
dcell_b200.levelset.sl_step), so the same host logic runs on GPUs with NCCL
and in CPU tests with gloo.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Callable, List, Sequence

import numpy as np
import torch
import torch.distributed as dist


def partition_cells(sizes: Sequence[int], world: int) -> List[List[int]]:
    """Largest-first greedy assignment of cells (by point count) to ranks."""
    loads = [0] * world
    parts: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i)):
        r = min(range(world), key=lambda k: (loads[k], k))
        parts[r].append(i)
        loads[r] += int(sizes[i])
    return [sorted(p) for p in parts]


def allreduce_diagnostics(volume: float, maxvel: float, device="cpu"):
    """Sum of enclosed volumes and max of |V| over ranks (one collective each)."""
    v = torch.tensor([volume], dtype=torch.float64, device=device)
    m = torch.tensor([maxvel], dtype=torch.float64, device=device)
    dist.all_reduce(v, op=dist.ReduceOp.SUM)
    dist.all_reduce(m, op=dist.ReduceOp.MAX)
    return float(v.item()), float(m.item())


def halo_for(max_w: float, dt: float, hz: float, cubic: bool = True) -> int:
    """Planes each slab needs from its neighbours for one step."""
    return int(math.ceil(abs(max_w) * dt / hz)) + (2 if cubic else 1)


@dataclass
class Slab:
    """Rank `rank`'s share [z0, z1) of nz planes, stored with halos as [lo, hi)."""
    nz: int
    world: int
    rank: int
    halo: int

    def __post_init__(self):
        counts = [self.nz // self.world + (1 if r < self.nz % self.world else 0) for r in range(self.world)]
        if min(counts) < self.halo:
            raise ValueError(f"slabs of {min(counts)} planes are thinner than the halo ({self.halo})")
        self.z0 = sum(counts[: self.rank])
        self.z1 = self.z0 + counts[self.rank]
        self.lo = max(0, self.z0 - self.halo)
        self.hi = min(self.nz, self.z1 + self.halo)

    def local(self, global_array):
        """This rank's planes [lo, hi) of a global (nz, ...) array."""
        return global_array[self.lo:self.hi].clone()

    def interior(self, local):
        return local[self.z0 - self.lo:self.z1 - self.lo]

    def exchange(self, local: torch.Tensor):
        """Refresh the halo planes of `local` from the z-neighbours."""
        ops = []
        bufs = []
        lo_in, hi_in = self.z0 - self.lo, self.z1 - self.lo
        if self.rank > 0:  # my first planes -> lower neighbour's upper halo; its last planes -> my lower halo
            send = local[lo_in:lo_in + (self.z0 - self.lo)].contiguous()
            recv = torch.empty_like(local[:lo_in])
            ops += [dist.P2POp(dist.isend, send, self.rank - 1), dist.P2POp(dist.irecv, recv, self.rank - 1)]
            bufs.append((0, recv))
        if self.rank < self.world - 1:
            nh = self.hi - self.z1
            send = local[hi_in - nh:hi_in].contiguous()
            recv = torch.empty_like(local[hi_in:])
            ops += [dist.P2POp(dist.isend, send, self.rank + 1), dist.P2POp(dist.irecv, recv, self.rank + 1)]
            bufs.append((hi_in, recv))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        for start, recv in bufs:
            local[start:start + recv.shape[0]] = recv
        return local


def default_stepper(interp="cubic_tc", backtrace="midpoint"):
    from .levelset import sl_step

    def step(phi0, vel, dt, h, origin):
        return sl_step(phi0.contiguous(), vel.contiguous(), dt, h, origin, interp=interp, backtrace=backtrace)
    return step


def slab_steps(slab: Slab, phi_local: torch.Tensor, vel_local: torch.Tensor, dts: Sequence[float], h,
               stepper: Callable):
    """Advance this rank's slab by len(dts) steps with a halo exchange before
    each; returns the local array (interior planes valid)."""
    x = phi_local
    for dt in dts:
        slab.exchange(x)
        x = stepper(x, vel_local, dt, h, (0, 0, slab.lo))
    return x


def gather_interiors(slab: Slab, local: torch.Tensor, nz: int):
    """Collect every rank's interior planes on all ranks (all_gather of equal-size padded blocks)."""
    inner = slab.interior(local).contiguous()
    maxp = nz // slab.world + 1
    pad = torch.zeros((maxp,) + tuple(inner.shape[1:]), dtype=inner.dtype, device=inner.device)
    pad[: inner.shape[0]] = inner
    out = [torch.empty_like(pad) for _ in range(slab.world)]
    dist.all_gather(out, pad)
    counts = [nz // slab.world + (1 if r < nz % slab.world else 0) for r in range(slab.world)]
    return torch.cat([o[:c] for o, c in zip(out, counts)], dim=0)
