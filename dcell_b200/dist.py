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

The per-slab / per-cell step is a callable (default: the CUDA kernels --
the split-state tensor-core brick stepper for slabs, stepping a plane range
so that the interior overlaps the halo exchange, and the batched brick
stepper for a rank's cells), so the same host logic runs on GPUs with NCCL
and in CPU tests with gloo.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Callable, List, Optional, Sequence

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


def cells_steps(phis: Sequence[torch.Tensor], vels: Sequence[torch.Tensor], hs, dt: float, nsteps: int,
                advance: Optional[Callable] = None, diagnose: Optional[Callable] = None, device="cuda",
                diag_every: int = 1):
    """The reference's cells-over-ranks loop (DWorld/DCellsArray.c:50-64: each
    rank advects its own cells, then a barrier) for one process per GPU.

    Cells (the same list on every rank) are assigned largest-first
    (partition_cells); this rank advances its share `nsteps` times and, every
    `diag_every` steps, all-reduces the diagnostics of its cells (enclosed
    volume sum, max |V| / h for the CFL count) -- the only collective.

    advance(phis, vels, hs, dt, k) -> the phis of this rank's cells after k
    steps; the default packs them into one CellBatch and runs the split-state
    tensor-core brick stepper over all of them, one launch per step
    (CellBatch.step_tc_split).  diagnose(phis, vels, hs) -> (volume, vmax)
    of a list of cells (default: FP64 smoothed-Heaviside volume on the
    device, eps = 1.5 h_x).  Returns (this rank's cell indices, their final
    phis, [(step, volume sum, max |V| / h)] identical on every rank)."""
    rank, world = dist.get_rank(), dist.get_world_size()
    parts = partition_cells([int(p.numel()) for p in phis], world)
    mine = parts[rank]
    hs = np.broadcast_to(np.asarray(hs, dtype=np.float64).reshape(-1, 3) if np.ndim(hs) > 1 else
                         np.asarray(hs, dtype=np.float64), (len(phis), 3))
    my_phis, my_vels, my_hs = [phis[i] for i in mine], [vels[i] for i in mine], hs[mine]
    advance = advance or _batch_advance(device)
    diagnose = diagnose or _device_diagnostics
    diags = []
    done = 0
    while done < nsteps:
        k = min(diag_every, nsteps - done)
        my_phis = advance(my_phis, my_vels, my_hs, dt, k) if my_phis else my_phis
        done += k
        vol, vmax = diagnose(my_phis, my_vels, my_hs) if my_phis else (0.0, 0.0)
        v, m = allreduce_diagnostics(vol, vmax, device=device if dist.get_backend() == "nccl" else "cpu")
        diags.append((done, v, m))
    return mine, my_phis, diags


def _batch_advance(device):
    """This rank's cells in one CellBatch, split-state bricks, one launch per step."""
    def advance(phis, vels, hs, dt, k):
        from .batch import CellBatch
        b = CellBatch(phis, vels, hs, dt, device=device)
        sa, sb = b.split(), torch.empty(b.npoints, dtype=torch.int32, device=b.device)
        out = torch.empty_like(b.phi)
        for _ in range(k):
            b.step_tc_split(sa, out, sb)
            sa, sb = sb, sa
        return [b.cell_view(out, i).clone() for i in range(b.ncells)]
    return advance


def _device_diagnostics(phis, vels, hs):
    from .levelset import volume
    vol, vmax = 0.0, 0.0
    for p, v, h in zip(phis, vels, hs):
        vol += float(volume(p.contiguous(), tuple(h), 1.5 * float(h[0])).item())
        vmax = max(vmax, max(float(v[..., d].abs().max()) / float(h[d]) for d in range(3)))
    return vol, vmax


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

    def exchange_start(self, local: torch.Tensor):
        """Post the halo exchange of `local` with the z-neighbours (my edge
        planes out, their edge planes into my halo planes); returns what
        exchange_finish needs.  The interior planes may be read meanwhile."""
        ops, bufs = [], []
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
        reqs = dist.batch_isend_irecv(ops) if ops else []
        return reqs, bufs

    def exchange_finish(self, local: torch.Tensor, pending):
        reqs, bufs = pending
        for req in reqs:
            req.wait()
        for start, recv in bufs:
            local[start:start + recv.shape[0]] = recv
        return local

    def exchange(self, local: torch.Tensor):
        """Refresh the halo planes of `local` from the z-neighbours."""
        return self.exchange_finish(local, self.exchange_start(local))

    def step_ranges(self, reach: int, align: int = 1):
        """Local plane ranges of one overlapped step: (interior, edges).  The
        interior range reads no halo plane (its departures reach `reach`
        planes), so it can step while the exchange is in flight; the edge
        ranges step after it.  Ranges are widened to multiples of `align`
        (the local grid's last plane ends the last range) and together cover
        the owned planes [z0 - lo, z1 - lo)."""
        n = self.hi - self.lo
        lo_in, hi_in = self.z0 - self.lo, self.z1 - self.lo
        up = lambda v: min(n, -(-v // align) * align)  # noqa: E731
        down = lambda v: (v // align) * align  # noqa: E731
        a, b = up(lo_in + reach), down(hi_in - reach)
        start, end = down(lo_in), up(hi_in)
        if a >= b:  # too thin to overlap: everything after the exchange
            return None, [(start, end)]
        return (a, b), [r for r in ((start, a), (b, end)) if r[1] > r[0]]


def default_stepper(interp="cubic_tc", backtrace="midpoint"):
    """Whole-array stepper over the CUDA kernels: step(phi0, vel, dt, h,
    origin) -> phi."""
    from .levelset import sl_step

    def step(phi0, vel, dt, h, origin):
        return sl_step(phi0.contiguous(), vel.contiguous(), dt, h, origin, interp=interp, backtrace=backtrace)
    return step


def slab_steps(slab: Slab, phi_local: torch.Tensor, vel_local: torch.Tensor, dts: Sequence[float], h,
               stepper: Callable):
    """Advance this rank's slab by len(dts) steps with a blocking halo
    exchange before each (whole-array stepper); returns the local array
    (interior planes valid)."""
    x = phi_local
    for dt in dts:
        slab.exchange(x)
        x = stepper(x, vel_local, dt, h, (0, 0, slab.lo))
    return x


class SplitStateSlab:
    """The dense split-state tensor-core stepper on a z-slab (the benchmark's
    brick kernel): the state carried between steps is the packed BF16 hi/lo
    words, so only they cross the halo exchange (4 bytes per halo point); the
    FP32 phi of each step is a side output.  step(x_in, vel, dt, h, origin,
    z_begin, z_end, x_out) advances local planes [z_begin, z_end) (multiples
    of the 8-plane brick depth) into x_out and self.phi."""

    align = 8

    def __init__(self, shape, device, backtrace="midpoint"):
        self.phi = torch.empty(shape, dtype=torch.float32, device=device)
        self.backtrace = backtrace

    def __call__(self, x_in, vel, dt, h, origin, z_begin, z_end, x_out):
        from .levelset import sl_step_tc_split_planes
        sl_step_tc_split_planes(x_in, vel, dt, h, z_begin, z_end, self.phi, x_out, origin=origin,
                                backtrace=self.backtrace)


def slab_steps_overlapped(slab: Slab, state: torch.Tensor, vel_local: torch.Tensor, dts: Sequence[float], h,
                          stepper: Callable, reach: int, align: int = 1):
    """Advance this rank's slab by len(dts) steps, each overlapping its halo
    exchange with the interior planes: post the exchange of the state's edge
    planes, step the planes that read no halo plane (`reach` = the planes a
    departure reaches), wait, step the planes next to the halos.  `stepper`
    advances a plane range: stepper(x_in, vel, dt, h, origin, z_begin, z_end,
    x_out).  On GPUs the exchange runs on NCCL's stream while the interior
    kernel runs on the compute stream.  Returns the final state (interior
    planes valid)."""
    x, y = state, torch.empty_like(state)
    inner, edges = slab.step_ranges(reach, align)
    origin = (0, 0, slab.lo)
    for dt in dts:
        pending = slab.exchange_start(x)
        if inner:
            stepper(x, vel_local, dt, h, origin, inner[0], inner[1], y)
        slab.exchange_finish(x, pending)
        for a, b in edges:
            stepper(x, vel_local, dt, h, origin, a, b, y)
        x, y = y, x
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
