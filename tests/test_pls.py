"""Particle level set -- the reference's LevelSetMethod/ParticleLS.c,
ParticleLS2D.c, ParticleLS3D.c: RK2 particle advection, escaped-particle
error correction, radius adjustment, seeding and reseeding.

Pinning: the oracle's restatement (oracle.pls_*) against the reference
compiled from its own sources (golden fixture tests/golden/pls.npz, made by
make_golden.py; and live through oracle/_ref where it is built), bit for bit
in FP64 including the drand48 stream the reference's PETSCRAND48 draws from.
The CUDA kernels equal the oracle bit for bit in FP64 (positions, radii, the
corrected phi and the random-number state), FP32 within FP32 rounding."""
import numpy as np
import pytest

import oracle
from oracle import reference as R

SEED_STATE = 0x12345678330E  # srand48(0x12345678): PETSc's default seed on rank 0


def _g(golden):
    return golden("pls")


def _corrected(base, idx, val):
    out = base.copy().ravel()
    out[idx] = val
    return out.reshape(base.shape)


def test_oracle_pls2d_vs_reference_golden(golden):
    g = _g(golden)
    o, h = tuple(int(v) for v in g["origin2"]), float(g["h2"])
    init, rng = oracle.pls_init(g["phi2"], g["band2"], SEED_STATE, h, origin=o)
    assert np.array_equal(init, g["init2"]) and rng == int(g["rng_init2"])
    adv = oracle.pls_advect(g["vel2"].astype(np.float64), init, float(g["dt2"]), h, origin=o)
    assert np.array_equal(adv, g["adv2"])
    phi_corr, skipped = oracle.pls_correct(g["phi_sl2"], g["band2"], adv, h, origin=o)
    assert skipped == 0
    assert np.array_equal(phi_corr, _corrected(g["phi_sl2"], g["corr_idx2"], g["corr_val2"]))
    adj = oracle.pls_adjust(phi_corr, adv, h, origin=o)
    assert np.array_equal(adj[:, 3], g["adj_radius2"]) and np.array_equal(adj[:, :3], adv[:, :3])
    res, rng2, miss = oracle.pls_reseed(phi_corr, g["band2"], adj, rng, h, origin=o)
    assert miss == 0
    assert np.array_equal(res, g["reseed2"]) and rng2 == int(g["rng_reseed2"])


def test_oracle_pls3d_vs_reference_golden(golden):
    g = _g(golden)
    o, h = tuple(int(v) for v in g["origin3"]), float(g["h3"])
    adv = oracle.pls_advect(g["vel3"].astype(np.float64), g["parts3"], float(g["dt3"]), h, origin=o)
    assert np.array_equal(adv, g["adv3"])
    phi_corr, skipped = oracle.pls_correct(g["phi3"], g["band3"], adv, h, origin=o)
    assert skipped == 0
    assert np.array_equal(phi_corr, _corrected(g["phi3"], g["corr_idx3"], g["corr_val3"]))
    adj = oracle.pls_adjust(phi_corr, adv, h, origin=o, params=oracle.pls_params(3))
    assert np.array_equal(adj[:, 3], g["adj_radius3"])


def test_oracle_pls_known_answers():
    # one particle in a linear field phi = x - 3.3: five drand48 draws (POSIX
    # X <- 0x5DEECE66D X + 0xB mod 2^48 after srand48(0x12345678)); the
    # attraction moves it along x only and an accepted step zeroes its z
    phi = np.tile(np.arange(8.0) - 3.3, (8, 1))
    init, rng = oracle.pls_init(phi, [[3, 3, 0]], SEED_STATE, params=oracle.pls_params(2, s_init=1))
    assert init.shape == (1, 4) and rng == _skip(SEED_STATE, 5)
    assert init[0, 1] == _skip(SEED_STATE, 2) / 2.0 ** 48 + (3 - 0.5)
    assert init[0, 2] == 0.0 and abs(init[0, 3]) in (0.1, 0.5) or 0.1 < abs(init[0, 3]) < 0.5
    # zero velocity: particles stay; a uniform velocity translates by dt V / h exactly
    parts = np.array([[3.25, 4.5, 0.0, 0.3], [5.75, 2.125, 0.0, -0.2]])
    vel0 = np.zeros((10, 10, 2))
    assert np.array_equal(oracle.pls_advect(vel0, parts, 0.1, 0.5), parts)
    vel = np.zeros((10, 10, 2))
    vel[..., 0], vel[..., 1] = 0.25, -0.5
    moved = oracle.pls_advect(vel, parts, 0.5, 0.5)
    assert np.array_equal(moved[:, :2], parts[:, :2] + [0.25, -0.5])
    # no particles: correction leaves phi, reseeding fills every band cell
    phi = np.linspace(-2, 2, 100).reshape(10, 10)
    band = np.array([[i, j, 0] for j in range(3, 7) for i in range(3, 7)], dtype=np.int32)
    same, _ = oracle.pls_correct(phi, band, np.zeros((0, 4)))
    assert np.array_equal(same, phi)
    res, _, _ = oracle.pls_reseed(phi, band, np.zeros((0, 4)), SEED_STATE)
    assert len(res) == 16 * int((np.abs(phi[3:7, 3:7]) <= 3.0).sum())


def _skip(x, k):
    for _ in range(k):
        x = (0x5DEECE66D * x + 0xB) % (1 << 48)
    return x


@pytest.mark.skipif(not R.available(), reason="oracle/_ref not built")
def test_oracle_pls_vs_reference_live():
    """A larger circle through the reference itself: seeding, three
    advect / correct / adjust rounds and a reseed."""
    h = 1 / 48.
    ls = R.RefLevelSet.circle(h, (0.47, 0.52), 0.22)
    p, _ = ls.geometry()
    phi, band = ls.get_phi().copy(), ls.band().copy()
    ls.pls_init()
    parts, rng = oracle.pls_init(phi, band, SEED_STATE, h, origin=p)
    assert np.array_equal(parts, ls.particles()) and rng == R.rand48_state()
    ny, nx = ls.shape
    r = np.random.default_rng(2)
    vel = r.uniform(-1, 1, (ny, nx, 2))
    ls.set_velocity(vel)
    for _ in range(3):
        ls.pls_advect(h)
        parts = oracle.pls_advect(vel, parts, h, h, origin=p)
        assert np.array_equal(parts, ls.particles())
        ls.pls_correct()
        phi, _ = oracle.pls_correct(phi, band, parts, h, origin=p)
        assert np.array_equal(phi, ls.get_phi())
        ls.pls_adjust()
        parts = oracle.pls_adjust(phi, parts, h, origin=p)
        assert np.array_equal(parts, ls.particles())
    rng = R.rand48_state()
    ls.pls_reseed()
    parts, rng, _ = oracle.pls_reseed(phi, band, parts, rng, h, origin=p)
    assert np.array_equal(parts, ls.particles()) and rng == R.rand48_state()
    ls.close()


# ---------------------------------------------------------------------------
# GPU: the CUDA kernels against the reference's golden records and the oracle

def _dev(a, cuda, dtype=None):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a)).to(cuda)
    return t.to(dtype) if dtype is not None else t


@pytest.mark.gpu
def test_gpu_pls2d_fp64_equals_reference(golden, cuda):
    import torch

    from dcell_b200 import pls
    g = _g(golden)
    o, h = tuple(int(v) for v in g["origin2"]), float(g["h2"])
    phi = _dev(g["phi2"], cuda)
    band = _dev(g["band2"].astype(np.int32), cuda)
    rng = pls.new_rng(SEED_STATE, cuda)
    flags = torch.zeros(1, dtype=torch.int32, device=cuda)
    parts, n = pls.seed(phi, band, rng, h, o, flags=flags)
    assert n == len(g["init2"]) and int(rng.item()) == int(g["rng_init2"])
    assert np.array_equal(parts[:n].cpu().numpy(), g["init2"])
    vel = _dev(g["vel2"].astype(np.float64), cuda)
    pls.advect(parts, n, vel, float(g["dt2"]), h, o, flags=flags)
    assert np.array_equal(parts[:n].cpu().numpy(), g["adv2"])
    phi_sl = _dev(g["phi_sl2"], cuda)
    pls.correct(phi_sl, band, parts, n, h, o, flags=flags)
    want = _corrected(g["phi_sl2"], g["corr_idx2"], g["corr_val2"])
    assert np.array_equal(phi_sl.cpu().numpy(), want)
    pls.adjust_radii(phi_sl, parts, n, h, o, flags=flags)
    assert np.array_equal(parts[:n, 3].cpu().numpy(), g["adj_radius2"])
    parts, n2 = pls.reseed(phi_sl, band, parts, n, rng, h, o, flags=flags)
    assert n2 == len(g["reseed2"]) and int(rng.item()) == int(g["rng_reseed2"])
    assert np.array_equal(parts[:n2].cpu().numpy(), g["reseed2"])
    assert int(flags.item()) == 0


@pytest.mark.gpu
def test_gpu_pls3d_fp64_equals_reference(golden, cuda):
    import torch

    from dcell_b200 import pls
    g = _g(golden)
    o, h = tuple(int(v) for v in g["origin3"]), float(g["h3"])
    parts = _dev(g["parts3"], cuda)
    n = parts.shape[0]
    flags = torch.zeros(1, dtype=torch.int32, device=cuda)
    pls.advect(parts, n, _dev(g["vel3"].astype(np.float64), cuda), float(g["dt3"]), h, o, flags=flags)
    assert np.array_equal(parts.cpu().numpy(), g["adv3"])
    phi = _dev(g["phi3"], cuda)
    pls.correct(phi, _dev(g["band3"].astype(np.int32), cuda), parts, n, h, o, flags=flags)
    assert np.array_equal(phi.cpu().numpy(), _corrected(g["phi3"], g["corr_idx3"], g["corr_val3"]))
    pls.adjust_radii(phi, parts, n, h, o, pls.params(3), flags=flags)
    assert np.array_equal(parts[:, 3].cpu().numpy(), g["adj_radius3"])
    assert int(flags.item()) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("d", ["2", "3"])
def test_gpu_pls_fp32_within_rounding(golden, cuda, d):
    """FP32 particles: advection within 1e-4 cells of the reference's FP64,
    corrected phi within 1e-5 cells, radii within 1e-5."""
    import torch

    from dcell_b200 import pls
    g = _g(golden)
    o, h = tuple(int(v) for v in g["origin" + d]), float(g["h" + d])
    f32 = torch.float32
    start = g["init2"] if d == "2" else g["parts3"]
    base = g["phi_sl2"] if d == "2" else g["phi3"]
    parts = _dev(start, cuda, f32)
    n = parts.shape[0]
    pls.advect(parts, n, _dev(g["vel" + d], cuda, f32), float(g["dt" + d]), h, o)
    adv = g["adv" + d]
    assert np.abs(parts.double().cpu().numpy() - adv).max() <= 1e-4
    phi = _dev(base, cuda, f32)
    pls.correct(phi, _dev(g["band" + d].astype(np.int32), cuda), _dev(adv, cuda, f32), n, h, o)
    want = _corrected(base, g["corr_idx" + d], g["corr_val" + d])
    assert np.abs(phi.double().cpu().numpy() - want).max() <= 1e-5
    adj = _dev(adv, cuda, f32)
    pls.adjust_radii(_dev(want, cuda, f32), adj, n, h, o, pls.params(int(d)))
    assert np.abs(adj[:, 3].double().cpu().numpy() - g["adj_radius" + d]).max() <= 1e-5


@pytest.mark.gpu
def test_gpu_pls_larger_case_equals_oracle(cuda):
    """A 160^2 circle: GPU seeding, three advect / correct / adjust rounds in
    a random velocity, and a reseed that deletes and adds many particles --
    FP64 bit for bit against the oracle."""
    import torch

    from dcell_b200 import pls
    N, h = 160, 1 / 160.
    y, x = np.meshgrid(np.arange(N), np.arange(N), indexing="ij")
    phi_np = np.sqrt((x - 77.3) ** 2 + (y - 81.6) ** 2) - 40.2
    band_np = np.stack([x[np.abs(phi_np) < 6], y[np.abs(phi_np) < 6], 0 * x[np.abs(phi_np) < 6]], 1).astype(np.int32)
    rng_np = np.random.default_rng(7)
    vel_np = rng_np.uniform(-1, 1, (N, N, 2))
    phi, band, vel = _dev(phi_np, cuda), _dev(band_np, cuda), _dev(vel_np, cuda)
    rng = pls.new_rng(SEED_STATE, cuda)
    parts, n = pls.seed(phi, band, rng, h)
    want, want_rng = oracle.pls_init(phi_np, band_np, SEED_STATE, h)
    assert n == len(want) and int(rng.item()) == want_rng
    assert np.array_equal(parts[:n].cpu().numpy(), want)
    for _ in range(3):
        pls.advect(parts, n, vel, 2 * h, h)
        want = oracle.pls_advect(vel_np, want, 2 * h, h)
        pls.correct(phi, band, parts, n, h)
        phi_np, _ = oracle.pls_correct(phi_np, band_np, want, h)
        pls.adjust_radii(phi, parts, n, h)
        want = oracle.pls_adjust(phi_np, want, h)
    assert np.array_equal(parts[:n].cpu().numpy(), want)
    assert np.array_equal(phi.cpu().numpy(), phi_np)
    parts, n2 = pls.reseed(phi, band, parts, n, rng, h)
    want, want_rng, _ = oracle.pls_reseed(phi_np, band_np, want, want_rng, h)
    assert n2 == len(want) and int(rng.item()) == want_rng
    assert np.array_equal(parts[:n2].cpu().numpy(), want)


@pytest.mark.gpu
def test_gpu_pls_host_buffer_abi(golden, cuda):
    """dcell_ls_pls_* on host arrays (the drop-in's calls) reproduce the
    reference's golden records."""
    import ctypes

    from dcell_b200 import _lib, pls
    L = _lib.lib()
    g = _g(golden)
    o, h = tuple(int(v) for v in g["origin2"]), float(g["h2"])
    sess = ctypes.c_void_p()
    _lib.check(L.dcell_session_create(0, ctypes.byref(sess)))
    try:
        geo = _lib.geom(g["phi2"].shape, h, o)
        prm = pls.params(2)
        band = np.ascontiguousarray(g["band2"], dtype=np.int32)
        p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        cap = len(band) * prm.s_init
        parts = np.zeros((cap, 4))
        rng, count = ctypes.c_ulonglong(SEED_STATE), ctypes.c_longlong(0)
        _lib.check(L.dcell_ls_pls_seed(sess, ctypes.byref(geo), p(g["phi2"]), p(band), len(band), ctypes.byref(prm),
                                       ctypes.byref(rng), p(parts), cap, ctypes.byref(count)))
        n = count.value
        assert np.array_equal(parts[:n], g["init2"]) and rng.value == int(g["rng_init2"])
        vel = np.ascontiguousarray(g["vel2"], dtype=np.float64)
        _lib.check(L.dcell_ls_pls_advect(sess, ctypes.byref(geo), p(vel), p(parts), n, float(g["dt2"])))
        assert np.array_equal(parts[:n], g["adv2"])
        phi = g["phi_sl2"].copy()
        _lib.check(L.dcell_ls_pls_correct(sess, ctypes.byref(geo), p(phi), p(band), len(band), p(parts), n))
        assert np.array_equal(phi, _corrected(g["phi_sl2"], g["corr_idx2"], g["corr_val2"]))
        _lib.check(L.dcell_ls_pls_adjust_radii(sess, ctypes.byref(geo), p(phi), p(parts), n, ctypes.byref(prm)))
        cap2 = n + cap
        big = np.zeros((cap2, 4))
        big[:n] = parts[:n]
        _lib.check(L.dcell_ls_pls_reseed(sess, ctypes.byref(geo), p(phi), p(band), len(band), ctypes.byref(prm),
                                         ctypes.byref(rng), p(big), n, cap2, ctypes.byref(count)))
        assert np.array_equal(big[:count.value], g["reseed2"]) and rng.value == int(g["rng_reseed2"])
        # too small a buffer: the count is reported, nothing past the capacity is written
        small = np.zeros((3, 4))
        rc = L.dcell_ls_pls_seed(sess, ctypes.byref(geo), p(g["phi2"]), p(band), len(band), ctypes.byref(prm),
                                 ctypes.byref(ctypes.c_ulonglong(SEED_STATE)), p(small), 3, ctypes.byref(count))
        assert rc == _lib.ERR_CAPACITY and count.value == n
    finally:
        L.dcell_session_destroy(sess)


@pytest.mark.gpu
def test_gpu_pls_edge_cases(cuda):
    import torch

    from dcell_b200 import pls
    from dcell_b200._lib import DcellError
    phi = _dev(np.linspace(-2, 2, 100).reshape(10, 10), cuda)
    band = _dev(np.array([[i, j, 0] for j in range(3, 7) for i in range(3, 7)], dtype=np.int32), cuda)
    empty = torch.zeros((0, 4), dtype=torch.float64, device=cuda)
    before = phi.clone()
    pls.correct(phi, band, empty, 0, 1.0)
    assert torch.equal(phi, before)
    rng = pls.new_rng(SEED_STATE, cuda)
    parts, n = pls.reseed(phi, band, torch.zeros((1, 4), dtype=torch.float64, device=cuda), 0, rng)
    want, want_rng, _ = oracle.pls_reseed(phi.cpu().numpy(), band.cpu().numpy(), np.zeros((0, 4)), SEED_STATE)
    assert n == len(want) and int(rng.item()) == want_rng and np.array_equal(parts[:n].cpu().numpy(), want)
    # a particle whose stencil leaves the grid is flagged, not read out of bounds
    out = _dev(np.array([[0.2, 8.9, 0.0, 0.3]]), cuda)
    flags = torch.zeros(1, dtype=torch.int32, device=cuda)
    pls.advect(out, 1, _dev(np.ones((10, 10, 2)), cuda), 0.5, 1.0, flags=flags)
    assert int(flags.item()) & 64
    # seeding is 2D
    with pytest.raises(DcellError):
        pls.seed(_dev(np.zeros((4, 4, 4)), cuda), band, rng)


@pytest.mark.gpu
@pytest.mark.skipif(not R.available(), reason="oracle/_ref not built")
def test_gpu_levelset_advect_pls_equals_reference(golden, cuda):
    """dcell_b200.pls.LevelSetAdvectPLS (GPU SL, correction, irregular nodes,
    CFL count, radius adjustment) against the reference's LevelSetAdvectPLS
    for steps below the reinitialisation threshold: FP64 bit for bit."""
    import torch

    from dcell_b200 import levelset as L
    from dcell_b200 import pls
    g = _g(golden)
    h, o = float(g["h2"]), tuple(int(v) for v in g["origin2"])
    ny, nx = g["phi2"].shape
    y, x = np.meshgrid(np.arange(ny) + o[1], np.arange(nx) + o[0], indexing="ij")
    vel = np.zeros((ny, nx, 2))
    vel[..., 0] = -2 * np.pi * h * (y - (o[1] + ny / 2.0))
    vel[..., 1] = 2 * np.pi * h * (x - (o[0] + nx / 2.0))
    dt = 1.5 * h / np.abs(vel).max()
    ref = R.RefLevelSet.create(h, o, (ny, nx))
    ref.set_phi(g["phi2"])
    ref.set_band(g["band2"])
    ref.pls_init()
    ref.set_velocity(vel)
    ls = L.LevelSetCreate((h, h, h), o + (0,), (nx, ny, 0), dtype=torch.float64, device=cuda)
    ls.phi.copy_(_dev(g["phi2"], cuda))
    ls.band = _dev(g["band2"].astype(np.int32), cuda)
    pls.LevelSetInitializeParticles(ls)
    assert ls.Advect is pls.LevelSetAdvectPLS
    v = _dev(vel, cuda)
    for _ in range(2):
        ref.pls_step(dt)
        ls.Advect(ls, v, dt)
        assert np.array_equal(ls.pls.live.cpu().numpy(), ref.particles())
        assert np.array_equal(ls.phi.cpu().numpy(), ref.get_phi())
        assert abs(ls.CFLcount - ref.param("CFLcount")) <= 1e-12
    ref.close()


@pytest.mark.gpu
@pytest.mark.skipif(not R.available(), reason="oracle/_ref not built")
def test_gpu_pls_rk2_half_full_equals_reference(golden, cuda):
    """LevelSetAdvectPLSRK2HalfStep / FullStep (ParticleLS.c:333-375): the
    particles restart from particles0 for the full step, SL from the same
    phi0 -- FP64 bit for bit against the reference below the threshold."""
    import torch

    from dcell_b200 import levelset as L
    from dcell_b200 import pls
    g = _g(golden)
    h, o = float(g["h2"]), tuple(int(v) for v in g["origin2"])
    ny, nx = g["phi2"].shape
    rng = np.random.default_rng(12)
    vel_n = rng.uniform(-0.5, 0.5, (ny, nx, 2)) * h
    vel_half = vel_n + rng.uniform(-0.05, 0.05, (ny, nx, 2)) * h
    dt = 1.0
    ref = R.RefLevelSet.create(h, o, (ny, nx))
    ref.set_phi(g["phi2"])
    ref.set_band(g["band2"])
    ref.pls_init()
    ls = L.LevelSetCreate((h, h, h), o + (0,), (nx, ny, 0), dtype=torch.float64, device=cuda)
    ls.phi.copy_(_dev(g["phi2"], cuda))
    ls.band = _dev(g["band2"].astype(np.int32), cuda)
    pls.LevelSetInitializeParticles(ls)
    ref.set_velocity(vel_n)
    ref.pls_rk2_half(dt / 2)
    pls.LevelSetAdvectPLSRK2HalfStep(ls, _dev(vel_n, cuda), dt / 2)
    assert np.array_equal(ls.pls.live.cpu().numpy(), ref.particles())
    assert np.array_equal(ls.phi.cpu().numpy(), ref.get_phi())
    ref.set_velocity(vel_half)
    ref.pls_rk2_full(dt)
    pls.LevelSetAdvectPLSRK2FullStep(ls, _dev(vel_half, cuda), dt)
    assert np.array_equal(ls.pls.live.cpu().numpy(), ref.particles())
    assert np.array_equal(ls.phi.cpu().numpy(), ref.get_phi())
    ref.close()
