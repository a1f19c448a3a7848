"""Multi-process host logic of the multi-GPU path on CPU (gloo, world size 2):
z-slab decomposition with halo exchange, cells over ranks with all-reduced
diagnostics, and a peer that dies between steps.  The per-slab step is the
CPU oracle here; on GPUs it is the CUDA kernel over NCCL."""
import datetime
import os
import socket
import tempfile

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from dcell_b200 import dist as D


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _init(rank, world, port, timeout=30):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=timeout))


def _problem():
    import oracle  # noqa: F401  (checker)
    rng = np.random.default_rng(4)
    nz, ny, nx = 26, 18, 20
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    phi = np.sqrt((x - 9.3) ** 2 + (y - 8.1) ** 2 + (z - 12.7) ** 2) - 6.2
    vel = 0.6 * np.sin(0.3 * x + 0.2 * y + 0.1 * z)[..., None] * rng.uniform(-1, 1, size=3)
    vel = np.ascontiguousarray(vel + 0.1 * rng.uniform(-1, 1, size=vel.shape))
    return phi, vel, [0.9, 0.8, 1.0], 1.0


def _oracle_stepper(phi0, vel, dt, h, origin):
    import oracle
    out = oracle.sl_step(phi0.numpy(), vel.numpy(), dt, h, origin=origin, interp="cubic", backtrace="midpoint")
    return torch.from_numpy(out)


def _slab_worker(rank, world, port, result):
    _init(rank, world, port)
    import oracle
    phi, vel, dts, h = _problem()
    halo = D.halo_for(max_w=float(np.abs(vel[..., 2]).max()), dt=max(dts), hz=h)
    slab = D.Slab(phi.shape[0], world, rank, halo)
    out = D.slab_steps(slab, slab.local(torch.from_numpy(phi)), slab.local(torch.from_numpy(vel)), dts, h,
                       _oracle_stepper)
    full = D.gather_interiors(slab, out, phi.shape[0])
    if rank == 0:
        ref = phi
        for dt in dts:
            ref = oracle.sl_step(ref, vel, dt, h, interp="cubic", backtrace="midpoint")
        np.save(result, np.array([np.abs(full.numpy() - ref).max()]))
    dist.barrier()
    dist.destroy_process_group()


def _oracle_plane_stepper(x_in, vel, dt, h, origin, z0, z1, x_out):
    """Planes [z0, z1) of the local arrays stepped by the oracle (a band of
    those planes), written into x_out."""
    import oracle
    nz, ny, nx = x_in.shape
    zs, ys, xs = np.meshgrid(np.arange(z0, z1), np.arange(ny), np.arange(nx), indexing="ij")
    band = np.stack([xs.ravel() + origin[0], ys.ravel() + origin[1], zs.ravel() + origin[2]], 1).astype(np.int32)
    out = oracle.sl_step(x_in.numpy(), vel.numpy(), dt, h, origin=origin, band=band, interp="cubic",
                         backtrace="midpoint")
    x_out[z0:z1] = torch.from_numpy(out[z0:z1])


def _overlap_worker(rank, world, port, result, align):
    _init(rank, world, port)
    import oracle
    phi, vel, dts, h = _problem()
    halo = D.halo_for(max_w=float(np.abs(vel[..., 2]).max()), dt=max(dts), hz=h)
    slab = D.Slab(phi.shape[0], world, rank, halo)
    out = D.slab_steps_overlapped(slab, slab.local(torch.from_numpy(phi)), slab.local(torch.from_numpy(vel)), dts,
                                  h, _oracle_plane_stepper, reach=halo, align=align)
    full = D.gather_interiors(slab, out, phi.shape[0])
    if rank == 0:
        ref = phi
        for dt in dts:
            ref = oracle.sl_step(ref, vel, dt, h, interp="cubic", backtrace="midpoint")
        np.save(result, np.array([np.abs(full.numpy() - ref).max()]))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("align", [1, 4])
def test_overlapped_slab_steps_match_single_domain(align):
    """The overlapped form (interior planes stepped while the halo exchange
    is in flight, the planes next to the halos after it; plane ranges widened
    to `align`, as the 8-plane bricks of the GPU stepper are) reproduces the
    single-domain steps bit for bit."""
    with tempfile.TemporaryDirectory() as d:
        result = os.path.join(d, "err.npy")
        mp.spawn(_overlap_worker, args=(2, _port(), result, align), nprocs=2, join=True)
        assert float(np.load(result)[0]) == 0.0


def test_step_ranges_cover_the_owned_planes():
    for nz, world, halo, reach, align in [(26, 2, 3, 3, 1), (64, 3, 4, 4, 8), (40, 4, 5, 5, 8), (26, 2, 3, 3, 4),
                                          (17, 2, 3, 3, 8)]:
        for rank in range(world):
            slab = D.Slab(nz, world, rank, halo)
            inner, edges = slab.step_ranges(reach, align)
            n = slab.hi - slab.lo
            covered = set()
            for a, b in ([inner] if inner else []) + edges:
                assert 0 <= a < b <= n and (a % align == 0) and (b % align == 0 or b == n)
                covered |= set(range(a, b))
            assert set(range(slab.z0 - slab.lo, slab.z1 - slab.lo)) <= covered
            if inner:  # the interior range reads no halo plane
                assert inner[0] - reach >= slab.z0 - slab.lo and inner[1] + reach <= slab.z1 - slab.lo


def _cells_steps_worker(rank, world, port, result):
    _init(rank, world, port)
    phis, vels, hs, dt = _cells_problem()
    mine, out, diags = D.cells_steps(phis, vels, hs, dt, 3, advance=_oracle_advance, diagnose=_oracle_diagnose,
                                     device="cpu")
    np.save(result + f".{rank}.npy", np.array([float(x) for x in np.concatenate(
        [np.array(mine, dtype=np.float64)] + [o.numpy().ravel() for o in out] +
        [np.array(diags, dtype=np.float64).ravel()])]))
    dist.barrier()
    dist.destroy_process_group()


def _cells_problem():
    rng = np.random.default_rng(12)
    phis, vels, hs = [], [], []
    for _ in range(5):
        nz, ny, nx = (int(v) for v in rng.integers(8, 14, size=3))
        z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        phis.append(torch.from_numpy(np.sqrt((x - nx / 2) ** 2 + (y - ny / 2) ** 2 + (z - nz / 2) ** 2) - 3.0))
        vels.append(torch.from_numpy(rng.uniform(-0.4, 0.4, size=(nz, ny, nx, 3))))
        hs.append((1.0, 1.0, 1.0))
    return phis, vels, np.array(hs), 1.0


def _oracle_advance(phis, vels, hs, dt, k):
    import oracle
    out = []
    for p, v, h in zip(phis, vels, hs):
        x = p.numpy()
        for _ in range(k):
            x = oracle.sl_step(x, v.numpy(), dt, tuple(h), interp="cubic", backtrace="midpoint")
        out.append(torch.from_numpy(x))
    return out


def _oracle_diagnose(phis, vels, hs):
    import oracle
    vol = sum(oracle.volume(p.numpy(), tuple(h), 1.5 * float(h[0])) for p, h in zip(phis, hs))
    vmax = max(float(v[..., d].abs().max()) / float(h[d]) for v, h in zip(vels, hs) for d in range(3))
    return vol, vmax


def test_cells_over_ranks_steps_match_one_process():
    """cells_steps at world size 2: each rank advances its largest-first
    share of the cells; the cells' final level sets equal the one-process run
    and the all-reduced diagnostics (volume sum, max |V| / h) after every step
    equal the one-process sums."""
    phis, vels, hs, dt = _cells_problem()
    ref, vols = [], []
    xs = [p for p in phis]
    for step in range(3):
        xs = _oracle_advance(xs, vels, hs, dt, 1)
        vols.append(_oracle_diagnose(xs, vels, hs))
    with tempfile.TemporaryDirectory() as d:
        result = os.path.join(d, "cells")
        mp.spawn(_cells_steps_worker, args=(2, _port(), result), nprocs=2, join=True)
        got = {}
        parts = D.partition_cells([int(p.numel()) for p in phis], 2)
        for r in range(2):
            a = np.load(result + f".{r}.npy")
            n = len(parts[r])
            assert list(a[:n].astype(int)) == parts[r]
            pos = n
            for i in parts[r]:
                m = phis[i].numel()
                got[i] = a[pos:pos + m].reshape(tuple(phis[i].shape))
                pos += m
            diags = a[pos:].reshape(-1, 3)
            assert diags.shape[0] == 3
            for k in range(3):
                assert diags[k, 0] == k + 1
                assert abs(diags[k, 1] - vols[k][0]) <= 1e-12 * vols[k][0] and diags[k, 2] == vols[k][1]
        for i in range(len(phis)):
            assert np.array_equal(got[i], xs[i].numpy())


def test_slab_decomposition_matches_single_domain():
    with tempfile.TemporaryDirectory() as d:
        result = os.path.join(d, "err.npy")
        mp.spawn(_slab_worker, args=(2, _port(), result), nprocs=2, join=True)
        assert float(np.load(result)[0]) == 0.0


def _cells_worker(rank, world, port, result):
    _init(rank, world, port)
    import oracle
    rng = np.random.default_rng(8)
    shapes = [tuple(int(v) for v in rng.integers(8, 20, size=3)) for _ in range(7)]
    parts = D.partition_cells([int(np.prod(s)) for s in shapes], world)
    vol, vmax = 0.0, 0.0
    for i in parts[rank]:
        nz, ny, nx = shapes[i]
        z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        phi = np.sqrt((x - nx / 2) ** 2 + (y - ny / 2) ** 2 + (z - nz / 2) ** 2) - min(shapes[i]) / 4
        vol += oracle.volume(phi, 1.0, 1.5)
        vmax = max(vmax, float(i + 1))
    v, m = D.allreduce_diagnostics(vol, vmax)
    if rank == 0:
        np.save(result, np.array([v, m]))
    dist.barrier()
    dist.destroy_process_group()


def test_cells_over_ranks_diagnostics():
    import oracle
    rng = np.random.default_rng(8)
    shapes = [tuple(int(v) for v in rng.integers(8, 20, size=3)) for _ in range(7)]
    total = 0.0
    for s in shapes:
        nz, ny, nx = s
        z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        total += oracle.volume(np.sqrt((x - nx / 2) ** 2 + (y - ny / 2) ** 2 + (z - nz / 2) ** 2) - min(s) / 4, 1.0, 1.5)
    with tempfile.TemporaryDirectory() as d:
        result = os.path.join(d, "diag.npy")
        mp.spawn(_cells_worker, args=(2, _port(), result), nprocs=2, join=True)
        v, m = np.load(result)
        assert abs(v - total) <= 1e-12 * total and m == 7.0


def test_partition_is_balanced_and_complete():
    sizes = [96 * 96 * 96, 32 ** 3, 64 ** 3, 50 ** 3, 80 ** 3, 33 ** 3, 90 ** 3, 40 ** 3]
    parts = D.partition_cells(sizes, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(sizes)))
    loads = [sum(sizes[i] for i in p) for p in parts]
    assert max(loads) <= 1.35 * (sum(sizes) / 3)


def _dead_peer_worker(rank, world, port, result):
    _init(rank, world, port, timeout=5)
    phi, vel, dts, h = _problem()
    slab = D.Slab(phi.shape[0], world, rank, 3)
    local = slab.local(torch.from_numpy(phi))
    if rank == 1:
        os._exit(0)  # leaves between steps, before the halo exchange
    try:
        slab.exchange(local)
        np.save(result, np.array([0]))
    except Exception:
        np.save(result, np.array([1]))  # the survivor sees an error, not a hang
    os._exit(0)


def test_dead_peer_is_an_error_not_a_hang():
    with tempfile.TemporaryDirectory() as d:
        result = os.path.join(d, "dead.npy")
        ctx = mp.get_context("spawn")
        port = _port()
        procs = [ctx.Process(target=_dead_peer_worker, args=(r, 2, port, result)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=60)
        alive = [p.is_alive() for p in procs]
        for p, a in zip(procs, alive):
            if a:
                p.kill()
        assert not any(alive)
        assert int(np.load(result)[0]) == 1
