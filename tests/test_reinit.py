"""Narrow-band reinitialisation (bucketed fast marching) -- the reference's
LevelSetReinitialize (LevelSetMethod/FastMarching.c:11-146).

Pinning: the oracle's restatement (oracle.reinit) against the reference's own
FMM (golden fixture tests/golden/reinit.npz, made by running the compiled
reference; and live through oracle/_ref where it is built).  The heap is
replaced by buckets, so the pin is a tolerance: in the band, mean |diff|
<= 2e-4 and max <= 2e-2 cells, identical band sets and identical +/-PHI_INF
outside.  The CUDA kernels run the same bucketed procedure: FP64 results
equal the oracle's bit for bit (phi and band), FP32 within 1e-4 cells."""
import numpy as np
import pytest

import oracle
from oracle import reference as R

BUCKET = 1.0 / 64


def _case(golden, d):
    g = golden("reinit")
    return (g["phi_in" + d], g["nodes" + d], tuple(int(v) for v in g["origin" + d]), g["phi" + d], g["band" + d],
            float(g["band_width" + d]))


def _band_set(b):
    return set(map(tuple, np.asarray(b).reshape(-1, 3).tolist()))


def _check_vs_reference(phi, band, phi_ref, band_ref, bw):
    inf = bw + 1.5
    inb = np.abs(phi_ref) < inf
    assert _band_set(band) == _band_set(band_ref)
    d = np.abs(phi - phi_ref)[inb]
    assert d.mean() <= 2e-4 and d.max() <= 2e-2, (d.mean(), d.max())
    assert np.array_equal(phi[~inb], phi_ref[~inb])  # +/-PHI_INF outside the band


@pytest.mark.parametrize("d", ["3", "2"])
def test_oracle_reinit_vs_reference_golden(golden, d):
    phi_in, nodes, origin, phi_ref, band_ref, bw = _case(golden, d)
    phi, band = oracle.reinit(phi_in, nodes, bw, BUCKET, origin=origin)
    _check_vs_reference(phi, band, phi_ref, band_ref, bw)
    # grid order (x fastest) and seeds in the band
    lin = (band[:, 2] * phi_in.shape[-2] + band[:, 1]) * phi_in.shape[-1] + band[:, 0]
    assert np.all(np.diff(lin) > 0)
    seeds = nodes[nodes[:, 3] == -1][:, :3].astype(np.int32)
    assert _band_set(seeds) <= _band_set(band)


@pytest.mark.skipif(not R.available(), reason="oracle/_ref not built")
def test_oracle_reinit_vs_reference_live_and_exact_distance():
    """A larger sphere through the reference itself, and both against the
    exact distance: the bucketed march is no less accurate than the heap."""
    h, c, r = 1 / 64., (0.3512, 0.3371, 0.3618), 0.15
    ls = R.RefLevelSet.sphere(h, c, r)
    nodes = ls.irregular_nodes(surface=False)
    phi_in, origin = ls.get_phi().copy(), ls.origin
    ls.reinitialize()
    phi_ref, band_ref = ls.get_phi().copy(), ls.band().copy()
    ls.close()
    phi, band = oracle.reinit(phi_in, nodes, 6.0, BUCKET, origin=origin)
    _check_vs_reference(phi, band, phi_ref, band_ref, 6.0)
    nz, ny, nx = phi_in.shape
    z, y, x = np.meshgrid(np.arange(nz) + origin[2], np.arange(ny) + origin[1], np.arange(nx) + origin[0],
                          indexing="ij")
    exact = (np.sqrt((x * h - c[0]) ** 2 + (y * h - c[1]) ** 2 + (z * h - c[2]) ** 2) - r) / h
    inb = np.abs(phi_ref) < 6.0
    e_ref = np.abs(phi_ref - exact)[inb].max()
    e_orc = np.abs(phi - exact)[inb].max()
    assert e_orc <= e_ref + 0.01, (e_orc, e_ref)


def test_oracle_reinit_without_seeds_and_bucket_independence(golden):
    phi_in, nodes, origin, phi_ref, band_ref, bw = _case(golden, "2")
    phi, band = oracle.reinit(phi_in, nodes[:0], bw, BUCKET, origin=origin)
    assert band.shape == (0, 3)
    assert np.all(np.abs(phi) == bw + 1.5)
    # finer buckets move towards the heap's order, never away from the reference tolerance
    fine, _ = oracle.reinit(phi_in, nodes, bw, BUCKET / 4, origin=origin)
    inb = np.abs(phi_ref) < bw + 1.5
    assert np.abs(fine - phi_ref)[inb].max() <= 2e-2


# ---------------------------------------------------------------------------
# GPU: the CUDA kernels against the oracle (same nodes, same procedure)

def _raw_nodes(rows, torch, dev):
    from dcell_b200._lib import NODE_DTYPE
    a = np.zeros(len(rows), dtype=NODE_DTYPE)
    a["pos"] = rows[:, 0:3].astype(np.int32)
    a["axis"] = rows[:, 3].astype(np.int32)
    a["shift"] = rows[:, 4].astype(np.int32)
    a["signCenter"] = rows[:, 5].astype(np.int32)
    a["signFace"] = rows[:, 6].astype(np.int32)
    a["d"] = rows[:, 7]
    a["X"] = rows[:, 8:11]
    a["op"] = rows[:, 11:14]
    a["n"] = rows[:, 14:17]
    a["k"] = rows[:, 17]
    raw = torch.from_numpy(np.frombuffer(a.tobytes(), dtype=np.uint8).copy()).to(dev)
    return raw, len(rows)


@pytest.mark.gpu
@pytest.mark.parametrize("d", ["3", "2"])
def test_gpu_reinit_fp64_equals_oracle(golden, cuda, d):
    import torch

    from dcell_b200 import levelset as L
    phi_in, nodes, origin, phi_ref, band_ref, bw = _case(golden, d)
    raw, n = _raw_nodes(nodes, torch, cuda)
    phi = torch.from_numpy(phi_in.copy()).to(cuda)
    flags = torch.zeros(1, dtype=torch.int32, device=cuda)
    band = L.reinitialize(phi, raw, n, bw, BUCKET, origin=origin, flags=flags)
    torch.cuda.synchronize()
    assert int(flags.item()) == 0
    want_phi, want_band = oracle.reinit(phi_in, nodes, bw, BUCKET, origin=origin)
    assert np.array_equal(phi.cpu().numpy(), want_phi)
    assert np.array_equal(band.cpu().numpy(), want_band)
    _check_vs_reference(phi.cpu().numpy(), band.cpu().numpy(), phi_ref, band_ref, bw)


@pytest.mark.gpu
@pytest.mark.parametrize("d", ["3", "2"])
def test_gpu_reinit_fp32(golden, cuda, d):
    import torch

    from dcell_b200 import levelset as L
    phi_in, nodes, origin, phi_ref, band_ref, bw = _case(golden, d)
    raw, n = _raw_nodes(nodes, torch, cuda)
    phi = torch.from_numpy(phi_in.astype(np.float32)).to(cuda)
    band = L.reinitialize(phi, raw, n, bw, BUCKET, origin=origin)
    want, want_band = oracle.reinit(phi_in, nodes, bw, BUCKET, origin=origin)
    got = phi.double().cpu().numpy()
    inb = np.abs(want) < bw + 1.5
    assert np.abs(got - want)[inb].max() <= 1e-4
    assert len(_band_set(band.cpu().numpy()) ^ _band_set(want_band)) <= 2  # points at the band edge may flip


@pytest.mark.gpu
def test_gpu_pipeline_irregular_nodes_then_reinit(cuda):
    """phi -> GPU irregular nodes -> GPU reinitialisation, against the oracle
    fed the very node list the GPU produced (FP64: bit for bit)."""
    import torch

    from dcell_b200 import fields
    from dcell_b200 import levelset as L
    N = 48
    phi = (fields.sphere_sdf(N, center=(0.47, 0.52, 0.44), r=0.23, device=cuda) * N).contiguous()  # cell units
    band = fields.band_of(phi, 6.0, margin=3).to(cuda)
    raw, count = L.irregular_nodes(phi, 1.0, band, with_surface=False)
    rows = L.nodes_to_rows(L.nodes_to_numpy(raw, count))
    phi_in = phi.cpu().numpy().copy()
    out = phi.clone()
    got_band = L.reinitialize(out, raw, count, 6.0, BUCKET)
    want, want_band = oracle.reinit(phi_in, rows, 6.0, BUCKET)
    assert np.array_equal(out.cpu().numpy(), want)
    assert np.array_equal(got_band.cpu().numpy(), want_band)
    # distance quality: the exact sphere distance in cell units
    inb = np.abs(want) < 6.0
    exact = phi_in
    assert np.abs(want - exact)[inb].max() < 0.5


@pytest.mark.gpu
def test_gpu_reinit_without_seeds(cuda):
    import torch

    from dcell_b200 import levelset as L
    phi = torch.linspace(-3, 3, 40 * 40, dtype=torch.float64, device=cuda).reshape(40, 40)
    raw = torch.zeros(120, dtype=torch.uint8, device=cuda)
    flags = torch.zeros(1, dtype=torch.int32, device=cuda)
    band = L.reinitialize(phi, raw, 0, 6.0, BUCKET, flags=flags)
    assert band.shape[0] == 0 and int(flags.item()) == 0
    assert torch.all(phi.abs() == 7.5)
