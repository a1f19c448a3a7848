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

* **velocity acquisition** -- the fluid's velocity field is z-slab
  distributed over the ranks (like the reference's Global Array); every rank
  sends the parts of the cells' velocity boxes that lie in its slab to the
  cells' owners in one all_to_all (LevelSetGetVelocity's NGA_Get,
  LevelSetMethod/Advect.c:145-192), and each owner assembles its boxes with
  zeros outside the field.

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


def slab_ranges(nz: int, world: int):
    """Planes [z0, z1) of each rank in a block distribution of nz planes (the
    first nz % world ranks hold one plane more)."""
    base, extra = divmod(nz, world)
    out, z = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append((z, z + n))
        z += n
    return out


def _box_part(box, gdims, z0: int, z1: int):
    """Global index range (lo, hi per axis x, y, z) of the part of a box
    ((x, y, z) origin, (nz, ny, nx) shape) inside the field and planes [z0, z1); None if empty."""
    o, sh = box
    lo = [max(0, int(o[0])), max(0, int(o[1])), max(z0, int(o[2]))]
    hi = [min(int(gdims[0]), int(o[0]) + int(sh[2])), min(int(gdims[1]), int(o[1]) + int(sh[1])),
          min(z1, int(gdims[2]), int(o[2]) + int(sh[0]))]
    if any(h <= l for l, h in zip(lo, hi)):
        return None
    return lo, hi


def gather_velocity_boxes(local_field: torch.Tensor, gdims, boxes, owner, first: int = 1):
    """Velocity grids of the boxes this rank owns, from a z-slab distributed
    global field.

    local_field: this rank's planes slab_ranges(gdims[2], world)[rank] of the
    global [z][y][x][c] field; gdims = (gx, gy, gz); boxes: list of ((x, y, z)
    origin, (nz, ny, nx) shape), the same list on every rank; owner[b]: the
    rank that owns box b.  Components first .. first+2.  Returns {b: tensor
    shape + (3,)} for the boxes owned here, zero outside the field (GridResize
    zeroes the velocity grid before NGA_Get, Common/Grid.c:146).  One
    all_to_all_single carries every part; the receive sizes follow from the
    box list and the slab ranges, so no size exchange is needed."""
    rank, world = dist.get_rank(), dist.get_world_size()
    ranges = slab_ranges(int(gdims[2]), world)
    z0, z1 = ranges[rank]
    dim = 3
    send_chunks = [[] for _ in range(world)]
    for b, box in enumerate(boxes):
        part = _box_part(box, gdims, z0, z1)
        if part is None:
            continue
        lo, hi = part
        blk = local_field[lo[2] - z0:hi[2] - z0, lo[1]:hi[1], lo[0]:hi[0], first:first + dim]
        send_chunks[owner[b]].append(blk.reshape(-1))
    send_sizes = [sum(c.numel() for c in ch) for ch in send_chunks]
    flat = [c for ch in send_chunks for c in ch]
    send = torch.cat(flat) if flat else local_field.new_empty(0)
    recv_sizes = [0] * world
    for src, (s0, s1) in enumerate(ranges):
        for b, box in enumerate(boxes):
            if owner[b] != rank:
                continue
            part = _box_part(box, gdims, s0, s1)
            if part is not None:
                lo, hi = part
                recv_sizes[src] += (hi[0] - lo[0]) * (hi[1] - lo[1]) * (hi[2] - lo[2]) * dim
    recv = local_field.new_empty(sum(recv_sizes))
    dist.all_to_all_single(recv, send.contiguous(), recv_sizes, send_sizes)
    out = {b: local_field.new_zeros(tuple(int(v) for v in box[1]) + (dim,))
           for b, box in enumerate(boxes) if owner[b] == rank}
    pos = 0
    for src, (s0, s1) in enumerate(ranges):
        for b, box in enumerate(boxes):
            if owner[b] != rank:
                continue
            part = _box_part(box, gdims, s0, s1)
            if part is None:
                continue
            lo, hi = part
            o = box[0]
            ext = (hi[2] - lo[2], hi[1] - lo[1], hi[0] - lo[0], dim)
            n = ext[0] * ext[1] * ext[2] * dim
            out[b][lo[2] - o[2]:hi[2] - o[2], lo[1] - o[1]:hi[1] - o[1], lo[0] - o[0]:hi[0] - o[0]] = \
                recv[pos:pos + n].view(ext)
            pos += n
    return out
