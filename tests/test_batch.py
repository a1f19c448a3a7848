"""Batched cells: the tile planner (host, CPU) and the persistent batched
step (GPU) against one launch per cell, eager and CUDA-graph replay."""
import ctypes

import numpy as np
import pytest
import torch

from dcell_b200 import _lib
from dcell_b200.batch import CELL_DTYPE, TILE_DTYPE


def _cells(shapes):
    cells = np.zeros(len(shapes), dtype=CELL_DTYPE)
    off = 0
    for i, (nz, ny, nx) in enumerate(shapes):
        cells[i]["offset"] = off
        cells[i]["n"] = (nx, ny, nz)
        cells[i]["h"] = (1.0 / nx, 1.0 / ny, 1.0 / nz)
        cells[i]["dt"] = 0.01
        off += nx * ny * nz
    return cells, off


def _plan(cells, tile):
    L = _lib.lib()
    n = ctypes.c_int()
    rc = L.dcell_batch_plan(cells.ctypes.data_as(ctypes.c_void_p), len(cells), *tile, None, 0, ctypes.byref(n))
    assert rc == _lib.ERR_CAPACITY or (rc == _lib.OK and n.value == 0)
    tiles = np.zeros(n.value, dtype=TILE_DTYPE)
    _lib.check(L.dcell_batch_plan(cells.ctypes.data_as(ctypes.c_void_p), len(cells), *tile,
                                  tiles.ctypes.data_as(ctypes.c_void_p), n.value, ctypes.byref(n)))
    return tiles


@pytest.mark.parametrize("tile", [(32, 2, 2), (8, 4, 4), (5, 3, 7), (128, 1, 1)])
def test_plan_covers_every_point_once(tile):
    rng = np.random.default_rng(1)
    shapes = [tuple(int(v) for v in rng.integers(3, 40, size=3)) for _ in range(23)]
    cells, total = _cells(shapes)
    tiles = _plan(cells, tile)
    hits = np.zeros(total, dtype=np.int64)
    tx, ty, tz = tile
    for t in tiles:
        c = cells[t["cell"]]
        nx, ny, nz = c["n"]
        xs = np.arange(t["x0"], min(t["x0"] + tx, nx))
        ys = np.arange(t["y0"], min(t["y0"] + ty, ny))
        zs = np.arange(t["z0"], min(t["z0"] + tz, nz))
        Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
        np.add.at(hits, c["offset"] + (Z * ny + Y) * nx + X, 1)
    assert hits.min() == 1 and hits.max() == 1


def test_plan_rejects_bad_arguments():
    L = _lib.lib()
    cells, _ = _cells([(4, 4, 4)])
    n = ctypes.c_int()
    assert L.dcell_batch_plan(cells.ctypes.data_as(ctypes.c_void_p), 1, 0, 1, 1, None, 0, ctypes.byref(n)) == \
        _lib.ERR_ARG
    cells[0]["n"] = (0, 4, 4)
    assert L.dcell_batch_plan(cells.ctypes.data_as(ctypes.c_void_p), 1, 4, 4, 4, None, 0, ctypes.byref(n)) == \
        _lib.ERR_ARG


@pytest.mark.gpu
@pytest.mark.parametrize("interp", ["cubic_tc", "cubic_separable", "cubic_plain", "linear"])
def test_batched_step_equals_per_cell_launches(cuda, interp):
    from dcell_b200.batch import CellBatch, c4_workload
    phis, vels, hs, dt = c4_workload(ncells=12, emin=20, emax=40, seed=7, device=cuda)
    b = CellBatch(phis, vels, hs, dt, device=cuda)
    out_b = torch.zeros_like(b.phi)
    out_c = torch.zeros_like(b.phi)
    tile = (16, 4, 2) if interp == "cubic_tc" else (32, 4, 2)
    b.step(b.phi, out_b, interp, "midpoint", tile=tile, ctas_per_sm=2)
    b.step_per_cell(b.phi, out_c, interp, "midpoint")
    torch.cuda.synchronize()
    if interp == "linear":  # per-cell linear is the reference-order kernel: equal to rounding
        assert float((out_b - out_c).abs().max()) <= 1e-6 * float(out_c.abs().max())
    else:
        assert torch.equal(out_b, out_c)


@pytest.mark.gpu
def test_autotune_and_graph_replay(cuda):
    from dcell_b200.batch import CellBatch, c4_workload
    phis, vels, hs, dt = c4_workload(ncells=16, emin=24, emax=48, seed=3, device=cuda)
    b = CellBatch(phis, vels, hs, dt, device=cuda)
    (tile, ctas), results = b.autotune("cubic_tc", "midpoint", reps=1)
    assert tile[0] * tile[1] * tile[2] == 128 and len(results) > 4
    g, (a, _, out) = b.capture(4, "cubic_tc", "midpoint")
    g.replay()
    torch.cuda.synchronize()
    x, y = b.phi.clone(), torch.empty_like(b.phi)
    for _ in range(4):
        b.step(x, y, "cubic_tc", "midpoint")
        x, y = y, x
    torch.cuda.synchronize()
    assert torch.equal(out, x)


@pytest.mark.gpu
@pytest.mark.parametrize("backtrace", ["midpoint", "euler"])
def test_batched_split_bricks_equal_per_cell_split_steps(cuda, backtrace):
    """The batched split-state brick kernel (cp.async-staged boxes clamped to
    each cell) gives every cell the bits of dcell_sl_step_tc_split on that
    cell alone -- cells narrower, shorter and shallower than a brick box,
    widths not a multiple of 4, and cells the brick kernel of the single-grid
    path would take -- over three consecutive steps, also at 3x the CFL (the
    global fallback)."""
    from dcell_b200.batch import CellBatch, c4_workload
    phis, vels, hs, dt = c4_workload(ncells=10, emin=5, emax=70, seed=11, device=cuda)
    shapes = [tuple(p.shape) for p in phis]
    assert any(s[2] % 4 for s in shapes) and any(min(s) < 12 for s in shapes)
    for scale in (1.0, 3.0):
        b = CellBatch(phis, vels, hs, [d * scale for d in dt] if np.ndim(dt) else dt * scale, device=cuda)
        s0 = b.split()
        a_phi, a_s = torch.empty_like(b.phi), torch.empty_like(s0)
        c_phi, c_s = torch.empty_like(b.phi), torch.empty_like(s0)
        xa, xc = s0.clone(), s0.clone()
        for _ in range(3):
            b.step_tc_split(xa, a_phi, a_s, backtrace)
            b.step_tc_split_per_cell(xc, c_phi, c_s, backtrace)
            torch.cuda.synchronize()
            assert torch.equal(a_phi, c_phi)
            assert torch.equal(a_s, c_s)
            xa, xc = a_s.clone(), c_s.clone()


@pytest.mark.gpu
@pytest.mark.parametrize("backtrace", ["midpoint", "euler"])
def test_tma_batched_split_bricks_equal_per_cell_split_steps(cuda, backtrace):
    """The TMA-staged batched step on a padded batch (rows padded to 4
    points, pad columns copies of each cell's last column, a tensor map per
    cell) gives every cell's real points the bits of dcell_sl_step_tc_split
    on that cell alone, and keeps the pad columns copies of the new last
    column, over three consecutive steps, also at 3x the CFL (the global
    fallback)."""
    from dcell_b200.batch import CellBatch, c4_workload
    phis, vels, hs, dt = c4_workload(ncells=10, emin=5, emax=70, seed=11, device=cuda)
    assert any(p.shape[2] % 4 for p in phis)
    for scale in (1.0, 3.0):
        dts = dt * scale
        ref = CellBatch(phis, vels, hs, dts, device=cuda)
        b = CellBatch(phis, vels, hs, dts, device=cuda, padded=True)
        xr, xb = ref.split(), b.split()
        r_phi, r_s = torch.empty_like(ref.phi), torch.empty_like(xr)
        b_phi, b_s = torch.empty_like(b.phi), torch.empty_like(xb)
        for _ in range(3):
            ref.step_tc_split_per_cell(xr, r_phi, r_s, backtrace)
            b.step_tc_split_tma(xb, b_phi, b_s, backtrace)
            torch.cuda.synchronize()
            for i in range(b.ncells):
                assert torch.equal(b.cell_view(b_phi, i), ref.cell_view(r_phi, i)), i
                assert torch.equal(b.cell_view(b_s, i), ref.cell_view(r_s, i)), i
                full = b_s[int(b.offsets[i]):int(b.offsets[i]) + int(np.prod(b.stored[i]))].view(b.stored[i])
                nx = b.shapes[i][2]
                assert torch.equal(full[..., nx:], full[..., nx - 1:nx].expand_as(full[..., nx:])), i
            xr, xb = r_s.clone(), b_s.clone()
