"""Generate the golden fixtures in tests/golden/ from the reference's OWN code.

Runs the reference's level-set C (compiled by ``make -C oracle ref`` from the
reference tree against oracle/shim) on small seeded inputs and stores inputs
and outputs as .npz.  The fixtures let the GPU box, where the reference tree
is absent, pin both the oracle and the CUDA path to the reference.

All inputs are FP32-representable (stored as float32; widen to float64
exactly), so FP32 and FP64 kernels see the very same data the FP64
reference saw.

    python tests/golden/make_golden.py        # needs oracle/_ref/libdcell_ref.so
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import reference as R  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def f32(a):
    return np.asarray(a, dtype=np.float32).astype(np.float64)


def sphere_case(shape, origin, h, center, r, seed, margin=3, cutoff=4.0):
    """Signed distance of a sphere (in grid-cell units, as after the
    reference's FMM), random MAC velocity, band = |phi| < cutoff points at
    least `margin` cells inside the grid, in lexicographic order."""
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    z, y, x = np.meshgrid(np.arange(nz) + origin[2], np.arange(ny) + origin[1], np.arange(nx) + origin[0],
                          indexing="ij")
    phi = f32(np.sqrt((x - center[0]) ** 2 + (y - center[1]) ** 2 + (z - center[2]) ** 2) - r)
    vel = f32(rng.uniform(-1.0, 1.0, size=shape + (3,)))
    inner = np.zeros(shape, bool)
    inner[margin:-margin, margin:-margin, margin:-margin] = True
    sel = inner & (np.abs(phi) < cutoff)
    band = np.stack([x[sel], y[sel], z[sel]], axis=1).astype(np.int32)
    return phi, vel, band


def circle_case(shape, origin, center, r, seed, margin=3, cutoff=4.0):
    rng = np.random.default_rng(seed)
    ny, nx = shape
    y, x = np.meshgrid(np.arange(ny) + origin[1], np.arange(nx) + origin[0], indexing="ij")
    phi = f32(np.sqrt((x - center[0]) ** 2 + (y - center[1]) ** 2) - r)
    vel = f32(rng.uniform(-1.0, 1.0, size=shape + (2,)))
    inner = np.zeros(shape, bool)
    inner[margin:-margin, margin:-margin] = True
    sel = inner & (np.abs(phi) < cutoff)
    band = np.stack([x[sel], y[sel], np.zeros_like(x[sel])], axis=1).astype(np.int32)
    return phi, vel, band


def run_sl(phi, vel, band, h, origin, dt):
    ls = R.RefLevelSet.create(h, origin, phi.shape)
    ls.set_phi(phi)
    ls.set_band(band)
    ls.set_velocity(vel)
    ls.copy_phi_to_phi0()
    ls.advect_sl(dt)
    out = ls.get_phi()
    nodes = ls.irregular_nodes(surface=True)
    maxv = ls.max_velocity()
    ls.cfl_increment(dt)
    cfl = ls.param("CFLcount")
    ls.close()
    return out, nodes, maxv, cfl


def run_rk2(phi, vel_n, vel_half, band, h, origin, dt):
    """advectSLRK2.c:27-36 driver shape: HalfStep(dt/2, u^n) then FullStep(dt, u^{n+1/2})."""
    ls = R.RefLevelSet.create(h, origin, phi.shape)
    ls.set_phi(phi)
    ls.set_band(band)
    ls.set_velocity(vel_n)
    ls.rk2_half(dt / 2)
    half = ls.get_phi()
    nodes_half = ls.nodes_no_update(R.lib().dref_update_irregular(ls.h))
    ls.set_velocity(vel_half)
    ls.rk2_full(dt)
    full = ls.get_phi()
    nodes_full = ls.irregular_nodes(surface=True)
    ls.close()
    return half, full, nodes_half, nodes_full


def run_reinit(ls):
    """LevelSetReinitialize (FastMarching.c:11-41) of a reference level set
    after an irregular-node pass: its input phi and nodes, output phi and band."""
    nodes = ls.irregular_nodes(surface=False)
    phi_in, origin, shape = ls.get_phi().copy(), ls.origin, ls.shape
    ls.reinitialize()
    assert ls.shape == shape and ls.origin == origin, "fixture case must not trigger LevelSetResize"
    return dict(phi_in=phi_in, nodes=nodes, origin=np.array(origin), phi=ls.get_phi().copy(), band=ls.band().copy(),
                band_width=ls.param("bandWidth"))


def main():
    assert R.available(), "build oracle/_ref first: make -C oracle ref"
    # fast-marching reinitialisation: a sphere and a circle as the reference's
    # own initialisers build them (off-grid centres, no symmetric ties)
    r3 = run_reinit(R.RefLevelSet.sphere(1.0 / 20, (0.4512, 0.3371, 0.5618), 0.2))
    r2 = run_reinit(R.RefLevelSet.circle(1.0 / 64, (0.4512, 0.5371), 0.2))
    np.savez_compressed(os.path.join(OUT, "reinit.npz"), **{k + "3": v for k, v in r3.items()},
                        **{k + "2": v for k, v in r2.items()})

    # velocity acquisition: LevelSetGetVelocity (Advect.c:145-192) through the
    # shim's one-process Global Array, for boxes inside, across and beyond the
    # fluid domain (components CELL_CENTER, U, V(, W) per cell)
    rng = np.random.default_rng(21)
    g3 = f32(rng.uniform(-2.0, 2.0, size=(20, 24, 28, 4)))
    boxes3 = [((-3, 5, 12), (14, 16, 22)), ((4, 3, 2), (6, 7, 8)), ((20, -6, -2), (12, 9, 10)), ((30, 30, 30), (4, 4, 4))]
    out3 = [R.RefLevelSet.create(0.05, o, s).get_velocity(g3) for o, s in boxes3]
    g2 = f32(rng.uniform(-2.0, 2.0, size=(30, 26, 3)))
    boxes2 = [((20, -4), (15, 12)), ((3, 7), (10, 9))]
    out2 = [R.RefLevelSet.create(0.05, o, s).get_velocity(g2) for o, s in boxes2]
    np.savez_compressed(os.path.join(OUT, "velocity.npz"), global3=g3.astype(np.float32),
                        global2=g2.astype(np.float32),
                        **{f"origin3_{i}": np.array(o) for i, (o, s) in enumerate(boxes3)},
                        **{f"shape3_{i}": np.array(s) for i, (o, s) in enumerate(boxes3)},
                        **{f"vel3_{i}": v.astype(np.float32) for i, v in enumerate(out3)},
                        **{f"origin2_{i}": np.array(o) for i, (o, s) in enumerate(boxes2)},
                        **{f"shape2_{i}": np.array(s) for i, (o, s) in enumerate(boxes2)},
                        **{f"vel2_{i}": v.astype(np.float32) for i, v in enumerate(out2)})

    h3 = 1.0 / 40
    # 3D: non-cubic grid, non-zero (partly negative) global origin
    shape3, origin3 = (20, 22, 24), (5, -3, 7)
    phi, vel, band = sphere_case(shape3, origin3, h3, center=(16.3, 7.6, 16.9), r=5.2, seed=11)
    dt = f32(0.45 * h3)
    out, nodes, maxv, cfl = run_sl(phi, vel, band, h3, origin3, dt)
    np.savez_compressed(os.path.join(OUT, "sl3d_linear.npz"), h=h3, origin=np.array(origin3), dt=dt, phi0=phi.astype(np.float32),
                        vel=vel.astype(np.float32), band=band, phi=out, nodes=nodes, maxvel=maxv, cflcount=cfl)

    vel_half = f32(vel * 0.8 + 0.1)
    half, full, nh, nf = run_rk2(phi, vel, vel_half, band, h3, origin3, f32(0.6 * h3))
    np.savez_compressed(os.path.join(OUT, "sl3d_rk2.npz"), h=h3, origin=np.array(origin3), dt=f32(0.6 * h3),
                        phi0=phi.astype(np.float32), vel=vel.astype(np.float32), vel_half=vel_half.astype(np.float32), band=band, phi_half=half, phi_full=full,
                        nodes_half=nh, nodes_full=nf)

    # 2D circle
    h2 = 1.0 / 64
    shape2, origin2 = (40, 44), (-2, 9)
    phi2, vel2, band2 = circle_case(shape2, origin2, center=(19.7, 28.4), r=11.3, seed=12)
    dt2 = f32(0.4 * h2)
    out2, nodes2, maxv2, cfl2 = run_sl(phi2, vel2, band2, h2, origin2, dt2)
    np.savez_compressed(os.path.join(OUT, "sl2d_linear.npz"), h=h2, origin=np.array(origin2), dt=dt2, phi0=phi2.astype(np.float32),
                        vel=vel2.astype(np.float32), band=band2, phi=out2, nodes=nodes2, maxvel=maxv2, cflcount=cfl2)

    # Catmull-Rom tricubic operator of TricubicInverse.h (64 unit stencils)
    M = np.zeros((64, 64))
    for s in range(64):
        e = np.zeros(64)
        e[s] = 1.0
        M[:, s] = R.tricubic_coefs(e)
    # orthogonal projections at the sphere's surface points (OrthogonalProjection3D)
    rng = np.random.default_rng(13)
    P = np.pad(phi, 2, mode="edge")
    picks = nodes[nodes[:, 3] == -1][:, :3].astype(int)
    picks = picks[rng.permutation(len(picks))[:48]]
    st5, st3, ops = [], [], []
    for (x, y, z) in picks:
        i, j, k = x - origin3[0] + 2, y - origin3[1] + 2, z - origin3[2] + 2
        p5 = P[k - 2:k + 3, j - 2:j + 3, i - 2:i + 3]
        p3 = P[k - 1:k + 2, j - 1:j + 2, i - 1:i + 2]
        st5.append(p5)
        st3.append(p3)
        ops.append(R.ortho3d(p3, p5))
    # sampled grid functions (Bilinear3D of identity, d/dx.., curvature, delta)
    ls = R.RefLevelSet.create(h3, origin3, shape3)
    ls.set_phi(phi)
    Xs = np.stack([rng.uniform(origin3[0] + 3, origin3[0] + shape3[2] - 4, 64),
                   rng.uniform(origin3[1] + 3, origin3[1] + shape3[1] - 4, 64),
                   rng.uniform(origin3[2] + 3, origin3[2] + shape3[0] - 4, 64)], axis=1)
    samples = np.stack([ls.sample(fn, Xs) for fn in range(6)], axis=1)
    ls.close()
    np.savez_compressed(os.path.join(OUT, "operators.npz"), tricubic_M=M, ortho_phi5=np.array(st5),
                        ortho_phi3=np.array(st3), ortho_op=np.array(ops), sample_X=Xs, samples=samples,
                        sample_h=h3, sample_origin=np.array(origin3))
    print("golden fixtures written to", OUT)


if __name__ == "__main__":
    main()
