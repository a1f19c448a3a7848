"""The drop-in: the reference's own C host with dcell_b200/host/levelset_b200.c
linked in place of its CPU LevelSetAdvectSL / LevelSetUpdateIrregularNodeList /
LevelSet_MaxVelocity (oracle/_ref/libdcell_ref_b200.so, built by
`make -C oracle dropin REF=<reference tree>`), driven through the very same reference call
sequence as the unmodified reference library.  FP64 linear is bit-identical.
"""
import numpy as np
import pytest

from oracle import reference as R

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (R.available() and R.available(R.DROPIN_PATH)),
                                 reason="reference libraries (oracle/_ref) not built")]

EXACT = [0, 1, 2, 3, 4, 5, 6, 7]


def _pair(g, key="phi0"):
    out = []
    for path in (R.PATH, R.DROPIN_PATH):
        ls = R.RefLevelSet.create(float(g["h"]), tuple(g["origin"]), g[key].shape, path=path)
        ls.set_phi(g[key])
        ls.set_band(g["band"])
        ls.set_velocity(g["vel"])
        out.append(ls)
    return out


@pytest.mark.parametrize("case", ["sl3d_linear", "sl2d_linear"])
def test_dropin_advect_irregular_maxvel(golden, cuda, case):
    g = golden(case)
    ref, b200 = _pair(g)
    for ls in (ref, b200):
        ls.copy_phi_to_phi0()
        ls.advect_sl(float(g["dt"]))
    assert np.array_equal(ref.get_phi(), b200.get_phi())
    assert np.array_equal(b200.get_phi(), g["phi"])
    nr, nb = ref.irregular_nodes(surface=False), b200.irregular_nodes(surface=False)
    assert nr.shape == nb.shape
    assert np.array_equal(nr[:, EXACT], nb[:, EXACT])
    assert np.abs(nr[:, 8:14] - nb[:, 8:14]).max() < 1e-11
    face = nr[:, 3] != -1
    assert np.array_equal(nr[face, 8:11], nb[face, 8:11])
    assert ref.max_velocity() == b200.max_velocity() == float(g["maxvel"])
    for ls in (ref, b200):
        ls.cfl_increment(float(g["dt"]))
    assert ref.param("CFLcount") == b200.param("CFLcount")
    ref.close()
    b200.close()


def test_dropin_rk2_half_full(golden, cuda):
    """AdvectRK2.c unchanged: its LevelSetAdvectSL / irregular-node calls land on the GPU."""
    g = golden("sl3d_rk2")
    ref, b200 = _pair(g)
    dt = float(g["dt"])
    for ls in (ref, b200):
        ls.rk2_half(dt / 2)
    assert np.array_equal(ref.get_phi(), b200.get_phi())
    for ls in (ref, b200):
        ls.set_velocity(g["vel_half"])
        ls.rk2_full(dt)
    assert np.array_equal(ref.get_phi(), b200.get_phi())
    assert np.array_equal(b200.get_phi(), g["phi_full"])
    ref.close()
    b200.close()


def test_dropin_advect_and_reinit_sequence(cuda):
    """Reference initialiser + LevelSetAdvectAndReinit steps (CPU fast marching
    in between, triggered by the reference's CFL threshold)."""
    rng = np.random.default_rng(7)
    h = 1.0 / 40
    libs = [R.RefLevelSet.sphere(h, (0.5, 0.5, 0.5), 0.16, path=p) for p in (R.PATH, R.DROPIN_PATH)]
    ref, b200 = libs
    # the initialiser already ran the (GPU resp. CPU) irregular-node pass and FMM
    assert ref.shape == b200.shape
    assert np.abs(ref.get_phi() - b200.get_phi()).max() < 1e-11
    vel = np.ascontiguousarray(rng.uniform(-1, 1, size=ref.shape + (3,)).astype(np.float32).astype(np.float64))
    for ls in libs:
        ls.set_velocity(vel)
    for step in range(6):
        for ls in libs:
            ls.advect_and_reinit(0.45 * h)
        assert ref.band().shape == b200.band().shape
        assert np.abs(ref.get_phi() - b200.get_phi()).max() < 1e-9, step
    ref.close()
    b200.close()


def test_reference_cpu_advect_vs_gpu_fp32_linear_slotted_disk(cuda):
    """Config C1's inputs through the reference's own CPU LevelSetAdvectSL
    (FP64, linear, Euler, narrow band) and the FP32 GPU linear kernel on the
    same band: 50 steps stay within FP32 rounding of each other."""
    import math

    import torch

    from dcell_b200 import fields
    from dcell_b200 import levelset as L
    N = 128
    h = 1.0 / N
    phi0 = fields.slotted_disk_sdf(N, device=cuda)
    vel = fields.rotation_velocity_2d(N, device=cuda)
    dt = 1.0 / int(math.ceil(2 * math.pi / h))
    band = fields.band_of(phi0, 6 * h)
    ls = R.RefLevelSet.create(h, (0, 0), (N, N))
    ls.set_phi(phi0.cpu().numpy())
    ls.set_band(band.cpu().numpy())
    ls.set_velocity(vel.cpu().numpy())
    a, v, b = phi0.float().contiguous(), vel.float().contiguous(), band.to(cuda)
    for _ in range(50):
        ls.copy_phi_to_phi0()
        ls.advect_sl(dt)
        a = L.sl_step(a, v, dt, h, band=b, out=a.clone())
    ref = torch.as_tensor(ls.get_phi(), device=cuda)
    ls.close()
    sel = torch.zeros_like(phi0, dtype=torch.bool)
    sel[band[:, 1].long(), band[:, 0].long()] = True
    err = (a.double() - ref).abs()[sel]
    assert float(err.max()) <= 5e-6, float(err.max())


def test_dropin_gpu_reinitialize(cuda, monkeypatch):
    """DCELL_LS_REINIT=gpu: the drop-in's LevelSetReinitialize runs the GPU's
    bucketed march; against the unmodified reference (heap FMM) on the same
    level set the band is the same set of points and phi agrees within the
    bucketing tolerance (mean <= 2e-4, max <= 2e-2 cells).  Unset, the drop-in
    calls the reference's own code (fed the GPU's irregular nodes, whose
    projections agree to ~1e-11)."""
    h, c, r = 1 / 48., (0.4512, 0.3371, 0.5618), 0.2
    ref = R.RefLevelSet.sphere(h, c, r)
    b200 = R.RefLevelSet.sphere(h, c, r, path=R.DROPIN_PATH)
    for ls in (ref, b200):
        ls.update_irregular()
    ref.reinitialize()
    b200.reinitialize()  # default: the reference's CPU code
    assert np.abs(ref.get_phi() - b200.get_phi()).max() < 1e-9
    assert set(map(tuple, ref.band().tolist())) == set(map(tuple, b200.band().tolist()))
    for ls in (ref, b200):
        ls.update_irregular()
    monkeypatch.setenv("DCELL_LS_REINIT", "gpu")
    b200.reinitialize()
    monkeypatch.delenv("DCELL_LS_REINIT")
    ref.reinitialize()
    pr, pb = ref.get_phi(), b200.get_phi()
    assert pr.shape == pb.shape
    inb = np.abs(pr) < ref.param("bandWidth") + 1.5
    d = np.abs(pr - pb)[inb]
    assert d.mean() <= 2e-4 and d.max() <= 2e-2, (d.mean(), d.max())
    assert set(map(tuple, ref.band().tolist())) == set(map(tuple, b200.band().tolist()))
    ref.close()
    b200.close()


def test_dropin_particle_level_set(golden, cuda):
    """LevelSetInitializeParticles + LevelSetAdvectPLS (ParticleLS.c) with the
    GPU's seeding, particle advection, error correction, radius adjustment
    and reseeding linked in: bit-identical to the unmodified reference until
    the CFL threshold triggers the fast marching (fed the GPU's irregular
    nodes, projections within ~1e-11), then within 1e-6 cells with the same
    particle count and random-number state."""
    g = golden("pls")
    h, o = float(g["h2"]), tuple(int(v) for v in g["origin2"])
    ny, nx = g["phi2"].shape
    y, x = np.meshgrid(np.arange(ny) + o[1], np.arange(nx) + o[0], indexing="ij")
    c = (o[0] + nx / 2.0, o[1] + ny / 2.0)
    vel = np.zeros((ny, nx, 2))  # a rotation; about 1.2 CFL per step, so the third step reinitialises
    vel[..., 0] = -2 * np.pi * h * (y - c[1])
    vel[..., 1] = 2 * np.pi * h * (x - c[0])
    dt = 5.3 * h / np.abs(vel).max()
    runs = []
    for path in (R.PATH, R.DROPIN_PATH):  # one after the other: both draw from the C library's drand48 state
        ls = R.RefLevelSet.create(h, o, g["phi2"].shape, path=path)
        ls.set_phi(g["phi2"])
        ls.set_band(g["band2"])
        ls.pls_init()
        rec = [(ls.particles(), ls.get_phi(), R.rand48_state(path))]
        ls.set_velocity(vel)
        for _ in range(5):
            ls.pls_step(dt)
            rec.append((ls.particles(), ls.get_phi(), R.rand48_state(path), ls.param("CFLcount")))
        runs.append(rec)
        ls.close()
    ref, b200 = runs
    assert np.array_equal(ref[0][0], b200[0][0]) and ref[0][2] == b200[0][2]
    assert np.array_equal(ref[0][0], g["init2"])
    triggered = False
    for a, b in zip(ref[1:], b200[1:]):
        assert a[0].shape == b[0].shape and a[2] == b[2]
        triggered = triggered or a[3] == 0.0  # this step reinitialised and reseeded
        if not triggered:
            assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
        else:
            assert np.abs(a[0] - b[0]).max() <= 1e-6 and np.abs(a[1] - b[1]).max() <= 1e-9
    assert triggered  # the reinitialisation and reseeding ran
