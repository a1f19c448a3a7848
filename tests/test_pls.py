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
