"""GPU irregular-node pass (with orthogonal projection, normals, curvature),
max-velocity reduction and smoothed-Heaviside volume vs the reference's
outputs (golden) and the oracle."""
import numpy as np
import pytest
import torch

import oracle
from dcell_b200 import _lib, fields
from dcell_b200 import levelset as L

pytestmark = pytest.mark.gpu
EXACT = [0, 1, 2, 3, 4, 5, 6, 7]


def _nodes(g, dev, dtype, key="phi", with_surface=True):
    phi = torch.as_tensor(g[key], dtype=dtype, device=dev)
    band = torch.as_tensor(g["band"], dtype=torch.int32, device=dev)
    flags = torch.zeros(1, dtype=torch.int32, device=dev)
    raw, count = L.irregular_nodes(phi, float(g["h"]), band, tuple(g["origin"]), with_surface=with_surface,
                                   flags=flags)
    torch.cuda.synchronize()
    assert int(flags.item()) == 0
    return raw, count, L.nodes_to_rows(L.nodes_to_numpy(raw, int(count.item())))


@pytest.mark.parametrize("case", ["sl3d_linear", "sl2d_linear"])
def test_irregular_fp64_vs_reference(golden, cuda, case):
    g = golden(case)
    _, _, rows = _nodes(g, cuda, torch.float64)
    ref = g["nodes"]
    assert rows.shape == ref.shape
    assert np.array_equal(rows[:, EXACT], ref[:, EXACT])
    face = ref[:, 3] != -1
    assert np.array_equal(rows[face, 8:11], ref[face, 8:11])          # face-node positions: exact
    assert np.abs(rows[:, 8:14] - ref[:, 8:14]).max() < 1e-11          # projections: evaluation order only
    assert np.array_equal(rows[face, 14:18], ref[face, 14:18])        # normals, curvature at face nodes: exact
    assert np.abs(rows[:, 14:17] - ref[:, 14:17]).max() < 1e-11
    assert np.allclose(rows[:, 17], ref[:, 17], rtol=1e-9, atol=1e-9)


@pytest.mark.parametrize("case", ["sl3d_linear", "sl2d_linear"])
def test_irregular_fp32_topology(golden, cuda, case):
    """FP32 input: same node set wherever no FP32 sign flip occurs (inputs are FP32-exact here)."""
    g = golden(case)
    _, _, rows = _nodes(g, cuda, torch.float32, key="phi0")
    ref = oracle.irregular_nodes(g["phi0"], float(g["h"]), g["band"], origin=g["origin"])
    assert rows.shape == ref.shape
    assert np.array_equal(rows[:, [0, 1, 2, 3, 4, 5, 6]], ref[:, [0, 1, 2, 3, 4, 5, 6]])
    assert np.abs(rows[:, 7] - ref[:, 7]).max() < 1e-5
    assert np.abs(rows[:, 8:14] - ref[:, 8:14]).max() < 2e-3


@pytest.mark.parametrize("case", ["sl3d_linear", "sl2d_linear"])
def test_max_velocity_exact(golden, cuda, case):
    g = golden(case)
    raw, count, _ = _nodes(g, cuda, torch.float64)
    vel = torch.as_tensor(g["vel"], dtype=torch.float64, device=cuda)
    mv = L.max_velocity(vel, float(g["h"]), raw, count, tuple(g["origin"]))
    assert float(mv.item()) == float(g["maxvel"])


def test_capacity_overflow_is_reported(golden, cuda):
    g = golden("sl3d_linear")
    phi = torch.as_tensor(g["phi"], dtype=torch.float64, device=cuda)
    band = torch.as_tensor(g["band"], dtype=torch.int32, device=cuda)
    flags = torch.zeros(1, dtype=torch.int32, device=cuda)
    raw, count = L.irregular_nodes(phi, float(g["h"]), band, tuple(g["origin"]), capacity=100, flags=flags)
    torch.cuda.synchronize()
    assert int(count.item()) == g["nodes"].shape[0]
    assert int(flags.item()) & _lib.FLAG_CAPACITY
    rows = L.nodes_to_rows(L.nodes_to_numpy(raw, 100))
    assert np.array_equal(rows[:, EXACT], g["nodes"][:100, EXACT])


def test_empty_band(cuda):
    phi = torch.zeros((8, 8, 8), dtype=torch.float64, device=cuda)
    band = torch.zeros((0, 3), dtype=torch.int32, device=cuda)
    raw, count = L.irregular_nodes(phi, 0.1, band)
    torch.cuda.synchronize()
    assert int(count.item()) == 0


def test_curvature_of_sphere(cuda):
    """Known answer: curvature 2/r and outward normals on a sphere's nodes."""
    N = 64
    h = 1.0 / N
    phi = fields.sphere_sdf(N, center=(0.5, 0.5, 0.5), r=0.25, device=cuda)
    band = fields.band_of(phi, 3 * h).to(cuda)
    raw, count = L.irregular_nodes(phi, h, band)
    rows = L.nodes_to_rows(L.nodes_to_numpy(raw, int(count.item())))
    proj = rows[rows[:, 3] == -1]
    assert len(proj) > 1000
    assert np.abs(np.median(proj[:, 17]) - 2 / 0.25) < 0.02 * 8
    X = (proj[:, 8:11] + 0.5) * h
    nrm = (X - 0.5) / np.linalg.norm(X - 0.5, axis=1, keepdims=True)
    assert np.abs((proj[:, 14:17] * nrm).sum(1) - 1).max() < 1e-3
    # projection points lie on the sphere
    assert np.abs(np.linalg.norm(X - 0.5, axis=1) - 0.25).max() < 0.05 * h


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_volume_vs_oracle(cuda, dtype):
    N = 48
    h = 1.0 / N
    phi = fields.sphere_sdf(N, device=cuda)
    v = float(L.volume(phi.to(dtype), h, 1.5 * h).item())
    ref = oracle.volume(phi.cpu().numpy(), h, 1.5 * h)
    assert abs(v - ref) <= (1e-12 if dtype == torch.float64 else 1e-6) * ref
    assert abs(ref - 4 / 3 * np.pi * 0.15 ** 3) < 0.03 * ref  # smoothing bias O((eps/r)^2)
    v2 = float(L.volume(phi.to(dtype), h, 1.5 * h).item())
    assert v == v2  # deterministic
