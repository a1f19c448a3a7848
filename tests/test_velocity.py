"""Velocity acquisition -- the reference's LevelSetGetVelocity
(LevelSetMethod/Advect.c:145-192): the velocity grid of a level set's phi box
is zeroed (GridResize, Common/Grid.c:146) and the part of the box inside the
fluid's Global Array is fetched with NGA_Get, components U_FACE.. of the
global field.

Pinning: the oracle (oracle.velocity_box) against the compiled reference's
LevelSetGetVelocity over a one-process Global Array (golden fixture
tests/golden/velocity.npz: boxes inside, straddling and outside the field, 3D
and 2D).  The CUDA copy kernels equal the golden boxes bit for bit (FP64) and
their FP32 rounding (FP32).  The multi-rank exchange (z-slab distributed field,
all_to_all to the boxes' owners) runs on gloo ranks against the oracle."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
from dcell_b200 import dist as D


def _cases(golden, d):
    g = golden("velocity")
    n = len([k for k in g if k.startswith("vel%s_" % d)])
    return g["global" + d], [(tuple(int(v) for v in g["origin%s_%d" % (d, i)]),
                              tuple(int(v) for v in g["shape%s_%d" % (d, i)]), g["vel%s_%d" % (d, i)])
                             for i in range(n)]


@pytest.mark.parametrize("d", ["3", "2"])
def test_oracle_velocity_box_vs_reference_golden(golden, d):
    gf, cases = _cases(golden, d)
    outside = 0
    for origin, shape, want in cases:
        got = oracle.velocity_box(gf, origin, shape, first=1)
        assert got.shape == want.shape
        assert np.array_equal(got, want)
        outside += int(np.count_nonzero(np.all(want == 0, axis=-1)))
    assert outside > 0  # the fixture has box points outside the field


def _getvel_case():
    """The reference's own GetVelocity test (LevelSetMethod/tests/getVel.c):
    a 10x10 2D field with 3 values per point, g[j][i][0] = i, g[j][i][1] = j,
    and a 19x19 box at (-5, -5).  GetVelocity takes components U_FACE..V_FACE
    (1..2), so inside the field the box holds (j, 0), zero elsewhere."""
    g = np.zeros((10, 10, 3))
    j, i = np.meshgrid(np.arange(10), np.arange(10), indexing="ij")
    g[..., 0], g[..., 1] = i, j
    want = np.zeros((19, 19, 2))
    want[5:15, 5:15, 0] = j
    return g, want


def test_getvel_known_answer():
    from oracle import reference as R
    g, want = _getvel_case()
    assert np.array_equal(oracle.velocity_box(g, (-5, -5), (19, 19), first=1), want)
    if R.available():
        ls = R.RefLevelSet.create(1.0, (-5, -5), (19, 19))
        assert np.array_equal(ls.get_velocity(g), want)
        ls.close()


def test_slab_ranges_and_box_part():
    assert D.slab_ranges(10, 3) == [(0, 4), (4, 7), (7, 10)]
    assert D.slab_ranges(2, 4) == [(0, 1), (1, 2), (2, 2), (2, 2)]
    box = ((-2, 3, 5), (6, 4, 5))  # x -2..2, y 3..6, z 5..10
    assert D._box_part(box, (10, 10, 20), 0, 8) == ([0, 3, 5], [3, 7, 8])
    assert D._box_part(box, (10, 10, 20), 11, 20) is None
    assert D._box_part(((12, 0, 0), (1, 1, 1)), (10, 10, 20), 0, 20) is None


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


GDIMS = (22, 18, 20)
BOXES = [((2, 3, 1), (8, 6, 7)), ((-3, -2, 15), (9, 7, 6)), ((10, 5, 6), (10, 9, 8)), ((30, 0, 0), (2, 2, 2)),
         ((0, 0, 0), (20, 18, 22))]
OWNER = [0, 1, 1, 0, 1]


def _field():
    rng = np.random.default_rng(11)
    return rng.uniform(-1, 1, size=(GDIMS[2], GDIMS[1], GDIMS[0], 4))


def _exchange_worker(rank, world, port, result):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    try:
        f = _field()
        z0, z1 = D.slab_ranges(GDIMS[2], world)[rank]
        got = D.gather_velocity_boxes(torch.from_numpy(f[z0:z1].copy()), GDIMS, BOXES, OWNER, first=1)
        assert sorted(got) == [b for b in range(len(BOXES)) if OWNER[b] == rank]
        for b, t in got.items():
            want = oracle.velocity_box(f, BOXES[b][0], BOXES[b][1], first=1)
            assert np.array_equal(t.numpy(), want), b
        result[rank] = "ok"
    except Exception as e:  # reported to the parent
        result[rank] = repr(e)
    finally:
        dist.destroy_process_group()


def test_gather_velocity_boxes_two_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        result = m.dict()
        port = _port()
        procs = [ctx.Process(target=_exchange_worker, args=(r, 2, port, result)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        assert all(p.exitcode == 0 for p in procs)
        assert dict(result) == {0: "ok", 1: "ok"}


# ---------------------------------------------------------------------------
# GPU: the copy kernels against the reference's boxes

@pytest.mark.gpu
@pytest.mark.parametrize("d", ["3", "2"])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_gpu_velocity_box_vs_reference_golden(golden, cuda, d, dtype):
    from dcell_b200 import levelset as L
    gf, cases = _cases(golden, d)
    g = torch.from_numpy(gf).to(cuda, dtype)
    for origin, shape, want in cases:
        got = L.velocity_box(g, origin, shape, first=1)
        assert got.dtype == dtype and tuple(got.shape) == want.shape
        assert np.array_equal(got.cpu().numpy(), want.astype(got.cpu().numpy().dtype))
    outs = L.velocity_boxes(g, [(o, s) for o, s, _ in cases], first=1)
    for t, (_, _, want) in zip(outs, cases):
        assert np.array_equal(t.cpu().numpy(), want.astype(t.cpu().numpy().dtype))


@pytest.mark.gpu
def test_gpu_getvel_known_answer(cuda):
    from dcell_b200 import levelset as L
    g, want = _getvel_case()
    got = L.velocity_box(torch.from_numpy(g).to(cuda), (-5, -5), (19, 19), first=1)
    assert np.array_equal(got.cpu().numpy(), want)


@pytest.mark.gpu
def test_gpu_velocity_boxes_many_cells(cuda):
    """512 cells' boxes (some straddling the domain edge) from a 128^3 field
    in one launch, each against the oracle."""
    from dcell_b200 import levelset as L
    rng = np.random.default_rng(5)
    G = 128
    gf = rng.standard_normal((G, G, G, 4))
    boxes = []
    for _ in range(512):
        sh = tuple(int(v) for v in rng.integers(4, 24, size=3))
        o = tuple(int(v) for v in rng.integers(-8, G - 4, size=3))
        boxes.append((o, sh))
    g = torch.from_numpy(gf).to(cuda)
    outs = L.velocity_boxes(g, boxes)
    for t, (o, sh) in zip(outs, boxes):
        assert np.array_equal(t.cpu().numpy(), oracle.velocity_box(gf, o, sh, first=1))


@pytest.mark.gpu
@pytest.mark.parametrize("gdof,first", [(4, 0), (4, 1), (5, 2), (3, 0)])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_gpu_velocity_box_record_layouts(cuda, gdof, first, dtype):
    """Vector-load records (four components: 16 B FP32, 32 B FP64) and
    per-component loads (other widths), any first component, against the oracle."""
    from dcell_b200 import levelset as L
    rng = np.random.default_rng(gdof * 10 + first)
    gf = rng.standard_normal((21, 19, 37, gdof))
    want_dtype = np.float64 if dtype == torch.float64 else np.float32
    g = torch.from_numpy(gf).to(cuda, dtype)
    boxes = [((-5, 3, 2), (9, 11, 50)), ((30, -2, 18), (6, 25, 13)), ((0, 0, 0), (21, 19, 37)), ((40, 0, 0), (2, 3, 4))]
    outs = L.velocity_boxes(g, boxes, first=first)
    for (o, sh), t in zip(boxes, outs):
        want = oracle.velocity_box(gf.astype(want_dtype), o, sh, first=first).astype(want_dtype)
        assert np.array_equal(L.velocity_box(g, o, sh, first=first).cpu().numpy(), want)
        assert np.array_equal(t.cpu().numpy(), want)
