"""Pins the FP64 oracle restatement to the reference's own outputs.

The golden fixtures were produced by the reference's C compiled from its own
sources (tests/golden/make_golden.py); where the compiled reference is present
(oracle/_ref) the oracle is also compared with it directly on fresh inputs.
"""
import numpy as np
import pytest

import oracle
from oracle import reference as R

EXACT_FIELDS = [0, 1, 2, 3, 4, 5, 6, 7]  # pos, axis, shift, signCenter, signFace, d


def test_sl3d_linear_bit_exact(golden):
    g = golden("sl3d_linear")
    out = oracle.sl_step(g["phi0"], g["vel"], float(g["dt"]), float(g["h"]), origin=g["origin"], band=g["band"],
                         phi=g["phi0"])
    assert np.array_equal(out, g["phi"])


def test_sl2d_linear_bit_exact(golden):
    g = golden("sl2d_linear")
    out = oracle.sl_step(g["phi0"], g["vel"], float(g["dt"]), float(g["h"]), origin=g["origin"], band=g["band"],
                         phi=g["phi0"])
    assert np.array_equal(out, g["phi"])


def test_rk2_half_full_bit_exact(golden):
    """advectSLRK2.c:27-36 driver: half step dt/2 with u^n, full step dt with u^{n+1/2} from the same phi0."""
    g = golden("sl3d_rk2")
    dt, h, o = float(g["dt"]), float(g["h"]), g["origin"]
    half = oracle.sl_step(g["phi0"], g["vel"], dt / 2, h, origin=o, band=g["band"], phi=g["phi0"])
    assert np.array_equal(half, g["phi_half"])
    full = oracle.sl_step(g["phi0"], g["vel_half"], dt, h, origin=o, band=g["band"], phi=half)
    assert np.array_equal(full, g["phi_full"])


@pytest.mark.parametrize("case", ["sl3d_linear", "sl2d_linear"])
def test_irregular_nodes(golden, case):
    g = golden(case)
    nodes = oracle.irregular_nodes(g["phi"], float(g["h"]), g["band"], origin=g["origin"], surface=True)
    ref = g["nodes"]
    assert nodes.shape == ref.shape
    assert np.array_equal(nodes[:, EXACT_FIELDS], ref[:, EXACT_FIELDS])
    # face nodes' X is exact; projection nodes differ only by the polynomial evaluation order
    assert np.abs(nodes[:, 8:14] - ref[:, 8:14]).max() < 1e-11
    assert np.abs(nodes[:, 14:17] - ref[:, 14:17]).max() < 1e-11
    face = ref[:, 3] != -1
    assert np.array_equal(nodes[face, 8:11], ref[face, 8:11])
    assert np.array_equal(nodes[face, 17], ref[face, 17])
    assert np.allclose(nodes[:, 17], ref[:, 17], rtol=1e-9, atol=1e-9)


@pytest.mark.parametrize("case", ["sl3d_linear", "sl2d_linear"])
def test_max_velocity_and_cfl(golden, case):
    g = golden(case)
    mv = oracle.max_velocity(g["vel"], g["nodes"], float(g["h"]), origin=g["origin"])
    assert mv == float(g["maxvel"])
    assert float(g["dt"]) * mv / float(g["h"]) == float(g["cflcount"])


def test_tricubic_operator_matches_reference_header(golden):
    M = golden("operators")["tricubic_M"]
    assert np.array_equal(oracle.catmull_rom_operator(3), M)
    assert int((M != 0).sum()) == 1331
    C = np.array([[0, 1, 0, 0], [-.5, 0, .5, 0], [1, -2.5, 2, -.5], [-.5, 1.5, -1.5, .5]])
    assert np.array_equal(np.kron(C, np.kron(C, C)), M)


def test_orthogonal_projection_3d(golden):
    g = golden("operators")
    for p3, p5, op in zip(g["ortho_phi3"], g["ortho_phi5"], g["ortho_op"]):
        assert np.abs(oracle.ortho3d(p3, p5) - op).max() < 1e-11


def test_grid_function_samples(golden):
    g = golden("operators")
    phi0 = golden("sl3d_linear")["phi0"]
    for fn in range(6):
        got = oracle.sample(phi0, fn, g["sample_X"], float(g["sample_h"]), origin=g["sample_origin"])
        assert np.array_equal(got, g["samples"][:, fn]) if fn in (0, 1, 2, 3, 4) else \
            np.allclose(got, g["samples"][:, fn], rtol=1e-14, atol=1e-15)


def test_linear_reproduces_linear_fields():
    """Known answer: trilinear SL of a linear field under uniform velocity is exact."""
    n = 12
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    phi = 0.25 * x - 0.5 * y + 0.125 * z
    vel = np.zeros((n, n, n, 3))
    vel[..., 0], vel[..., 1], vel[..., 2] = 0.5, -0.25, 0.75
    band = np.stack([x[3:-3, 3:-3, 3:-3].ravel(), y[3:-3, 3:-3, 3:-3].ravel(), z[3:-3, 3:-3, 3:-3].ravel()], 1)
    out = oracle.sl_step(phi, vel, 0.5, 1.0, band=band, interp="cubic")
    dt = 0.5
    shift = (0.25 * 0.5 - 0.5 * (-0.25) + 0.125 * 0.75) * dt  # phi(X - V dt) = phi(X) - grad.V dt
    expect = phi - shift
    sel = (slice(3, -3),) * 3
    assert np.abs(out[sel] - expect[sel]).max() < 1e-13


@pytest.mark.skipif(not R.available(), reason="compiled reference (oracle/_ref) not present")
def test_oracle_matches_compiled_reference_fresh_inputs():
    rng = np.random.default_rng(5)
    ls = R.RefLevelSet.sphere(1 / 48, (0.5, 0.47, 0.52), 0.13)
    p = ls.origin
    phi, band = ls.get_phi(), ls.band()
    vel = rng.uniform(-1, 1, size=ls.shape + (3,))
    ls.set_velocity(vel)
    ls.copy_phi_to_phi0()
    ls.advect_sl(0.33 / 48)
    ref = ls.get_phi()
    mine = oracle.sl_step(phi, vel, 0.33 / 48, 1 / 48, origin=p, band=band, phi=phi)
    assert np.array_equal(ref, mine)
    nr = ls.irregular_nodes()
    nm = oracle.irregular_nodes(ref, 1 / 48, band, origin=p)
    assert np.array_equal(nr[:, EXACT_FIELDS], nm[:, EXACT_FIELDS])
    ls.close()
