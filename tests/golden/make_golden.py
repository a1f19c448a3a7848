"""Generate the golden fixtures in tests/golden/ from the reference's OWN code.

Runs the reference's level-set C (compiled by ``make -C oracle ref REF=<reference tree>`` from the
reference tree against oracle/shim) on small seeded inputs and stores inputs
and outputs as .npz.  The fixtures let a GPU machine, where the reference tree
is absent, pin both the oracle and the CUDA path to the reference.

All inputs are FP32-representable (stored as float32; widen to float64
exactly), so FP32 and FP64 kernels see the very same data the FP64
reference saw.

    python tests/golden/make_golden.py        # needs oracle/_ref/libdcell_ref.so
    python tests/golden/make_golden.py mac    # only mac.npz
    python tests/golden/make_golden.py writer # only writer.npz
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


def _swirl(shape, origin, seed, noise):
    rng = np.random.default_rng(seed)
    idx = np.meshgrid(*[np.arange(n) + o for n, o in zip(shape, reversed(origin[:len(shape)]))], indexing="ij")
    if len(shape) == 2:
        y, x = idx
        v = np.stack([np.sin(0.3 * x) * np.cos(0.2 * y), -np.cos(0.3 * x) * np.sin(0.2 * y)], -1)
    else:
        z, y, x = idx
        v = np.stack([np.sin(0.3 * y), np.cos(0.2 * z), np.sin(0.25 * x)], -1)
    return f32(v + noise * rng.standard_normal(v.shape))


def run_pls2d():
    h = 1.0 / 24
    ls = R.RefLevelSet.circle(h, (0.4512, 0.5371), 0.1)
    p, _ = ls.geometry()
    phi, band = ls.get_phi().copy(), ls.band().copy()
    ls.pls_init()  # PetscRandomSetType seeds drand48 with 0x12345678 (state 0x12345678330E)
    init, rng_init = ls.particles(), R.rand48_state()
    vel = _swirl(ls.shape, p, 31, 0.3)
    dt = 2 * h
    ls.set_velocity(vel)
    ls.pls_advect(dt)
    adv = ls.particles()
    ls.L.dref_copy_phi_to_phi0(ls.h)
    ls.L.dref_advect_sl(ls.h, ls._vel, dt)
    phi_sl = ls.get_phi().copy()
    ls.pls_correct()
    corr = np.flatnonzero(ls.get_phi() != phi_sl)
    phi_corr = ls.get_phi().ravel()[corr]
    ls.pls_adjust()
    adj = ls.particles()
    assert np.array_equal(adj[:, :3], adv[:, :3])
    ls.pls_reseed()
    reseed, rng_reseed = ls.particles(), R.rand48_state()
    ls.close()
    return dict(origin2=np.array(p[:2]), h2=h, phi2=phi, band2=band, init2=init,
                rng_init2=np.uint64(rng_init), vel2=vel.astype(np.float32), dt2=dt, adv2=adv, phi_sl2=phi_sl,
                corr_idx2=corr, corr_val2=phi_corr, adj_radius2=adj[:, 3], reseed2=reseed,
                rng_reseed2=np.uint64(rng_reseed))


def run_pls3d():
    """A 20x18x16 (z, y, x) box at global origin (3, 1, 0) around a sphere of
    radius 3.4 cells, band |phi| < 4 cells, 1000 particles in the band.  The
    reference takes the corner z of an escaped particle from floor(X.y)
    (ParticleLS3D.c:76), so the z range covers the particles' y range (the
    reference writes out of bounds otherwise)."""
    h = 1.0 / 16
    shape, origin = (20, 18, 16), (3, 1, 0)
    z, y, x = np.meshgrid(*[np.arange(n) + o for n, o in zip(shape, reversed(origin))], indexing="ij")
    phi = f32(np.sqrt((x - 10.6) ** 2 + (y - 9.7) ** 2 + (z - 10.2) ** 2) - 3.4)
    inner = np.zeros(shape, bool)
    inner[2:-2, 2:-2, 2:-2] = True
    sel = inner & (np.abs(phi) < 4)
    band = np.stack([x[sel], y[sel], z[sel]], 1).astype(np.int32)
    ls = R.RefLevelSet.create(h, origin, shape)
    ls.set_phi(phi)
    ls.set_band(band)
    ls.pls_create_empty()
    rng = np.random.default_rng(33)
    pick = band[rng.choice(len(band), 1000)]
    parts = np.concatenate([pick + rng.uniform(-0.5, 0.5, pick.shape), rng.uniform(-0.6, 0.6, (len(pick), 1))], 1)
    ls.set_particles(parts)
    vel = _swirl(shape, origin, 35, 0.2)
    dt = 0.05
    ls.set_velocity(vel)
    ls.pls_advect(dt)
    adv = ls.particles()
    ls.pls_correct()
    corr = np.flatnonzero(ls.get_phi() != phi)
    phi_corr = ls.get_phi().ravel()[corr]
    ls.pls_adjust()
    adj = ls.particles()
    assert np.array_equal(adj[:, :3], adv[:, :3])
    ls.close()
    return dict(origin3=np.array(origin), h3=h, phi3=phi, band3=band, parts3=parts, vel3=vel.astype(np.float32),
                dt3=dt, adv3=adv, corr_idx3=corr, corr_val3=phi_corr, adj_radius3=adj[:, 3])


MAC_CASES = [  # (shape (z, y, x) or (y, x), global origin x, y(, z), spacing)
    ((11, 13, 17), (0, 0, 0), (0.05, 0.04, 0.03)),
    ((9, 12, 10), (-3, -1, -4), (0.05, 0.05, 0.05)),
    ((3, 3, 3), (0, 0, 0), (0.1, 0.2, 0.3)),
    ((23, 19), (0, 0), (0.02, 0.03, 1.0)),
    ((15, 21), (-5, -2), (0.04, 0.04, 1.0)),
]


def run_mac():
    """LevelSetAdvectMAC / _3D (LevelSetMethod/AdvectMAC.c:18-111), compiled
    from its own source against oracle/shim/mac: random phi, random face
    velocities of both signs (with exact zeros), out pre-filled with other
    values so untouched points are visible; dt chosen per case."""
    rng = np.random.default_rng(31)
    res = {}
    for c, (shape, origin, h) in enumerate(MAC_CASES):
        phi = f32(rng.uniform(-1.0, 1.0, size=shape))
        comps = [f32(rng.uniform(-2.0, 2.0, size=shape) * (rng.random(shape) > 0.1)) for _ in range(len(shape))]
        out0 = f32(rng.uniform(5.0, 6.0, size=shape))
        dt = f32(0.3 * min(h[:len(shape)]))
        w = comps[2] if len(shape) == 3 else None
        out = R.advect_mac(phi, comps[0], comps[1], w, dt, h, origin, out=out0)
        res.update({f"phi_{c}": phi.astype(np.float32), f"out0_{c}": out0.astype(np.float32), f"out_{c}": out,
                    f"origin_{c}": np.array(origin), f"h_{c}": np.array(h), f"dt_{c}": dt,
                    **{f"vel{a}_{c}": comps[a].astype(np.float32) for a in range(len(shape))}})
    res["ncases"] = len(MAC_CASES)
    return res


def run_writer():
    """The reference's own writers, into a scratch directory: GridWrite
    (Common/Serialize.c:23-55; two writes of one grid, so .pos / .size hold two
    lines; a velocity grid of dof 3 and one of dof 2), the node lists of a 3D
    and a 2D level set (LevelSetWriteIrregularNodeList,
    IrregularNodes.c:145-246; nodes from the reference's own irregular-node
    pass with normals and curvature stored in them) and a particle Array
    (ArrayWrite, Common/Array.c:134-150).  Stored: the inputs, and every file's
    bytes under "file:<name>"."""
    import tempfile
    out = {}
    with tempfile.TemporaryDirectory() as d:
        wd, tmp = os.path.join(d, "wd"), os.path.join(d, "tmp")
        os.makedirs(wd)
        os.makedirs(tmp)
        # 3D: a sphere (cell units) on a 16 x 18 x 20 (z, y, x) box at origin (-3, 2, 1)
        phi3, vel3, band3 = sphere_case((16, 18, 20), (-3, 2, 1), 0.1, (6.3, 10.6, 8.4), 4.7, seed=21)
        ls = R.RefLevelSet.create(0.1, (-3, 2, 1), phi3.shape)
        ls.set_output_dirs(wd, tmp)
        ls.set_phi(phi3)
        ls.set_band(band3)
        ls.update_irregular()
        ls.set_surface()
        nodes3 = ls.nodes_no_update(ls.update_irregular(), surface=True)
        ls.set_surface()
        ls.grid_write("ls3", 0)
        ls.set_phi(f32(phi3 * 0.5))
        ls.grid_write("ls3", 1)
        ls.set_phi(phi3)
        ls.write_irregular(2)
        ls.set_velocity(vel3)
        ls.velocity_write("vel3", 4)
        ls.close()
        # 2D: a circle on a 26 x 30 (y, x) box at origin (5, -4)
        phi2, vel2, band2 = circle_case((26, 30), (5, -4), (18.3, 8.6), 6.2, seed=22)
        ls = R.RefLevelSet.create(0.1, (5, -4), phi2.shape)
        ls.set_output_dirs(wd, tmp)
        ls.set_phi(phi2)
        ls.set_band(band2)
        n2 = ls.update_irregular()
        ls.set_surface()
        nodes2 = ls.nodes_no_update(n2, surface=True)
        ls.grid_write("ls2", 7)
        ls.write_irregular(0)
        ls.set_velocity(vel2)
        ls.velocity_write("vel2", 1)
        ls.close()
        # particles: the reference's own 2D seeding of a circle
        ls = R.RefLevelSet.circle(1.0 / 24, (0.4512, 0.5371), 0.1)
        ls.set_output_dirs(wd, tmp)
        ls.pls_init()
        parts = ls.particles()
        ls.write_particles(3)
        ls.close()
        for sub, base in (("wd", wd), ("tmp", tmp)):
            for name in sorted(os.listdir(base)):
                with open(os.path.join(base, name), "rb") as f:
                    out[f"file:{sub}/{name}"] = np.frombuffer(f.read(), dtype=np.uint8)
    out.update(phi3=phi3, vel3=vel3, nodes3=nodes3, phi2=phi2, vel2=vel2, nodes2=nodes2, particles=parts)
    return out


def main(only=None):
    assert R.available(), "build oracle/_ref first: make -C oracle ref REF=<reference tree>"
    if only == "mac":
        np.savez_compressed(os.path.join(OUT, "mac.npz"), **run_mac())
        print("mac.npz written to", OUT)
        return
    if only == "writer":
        np.savez_compressed(os.path.join(OUT, "writer.npz"), **run_writer())
        print("writer.npz written to", OUT)
        return
    np.savez_compressed(os.path.join(OUT, "writer.npz"), **run_writer())
    np.savez_compressed(os.path.join(OUT, "mac.npz"), **run_mac())
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

    # particle level set (ParticleLS*.c): 2D seeding from the reference's own
    # rand48 stream, RK2 particle advection in a noisy swirl, SL advection of
    # phi, escaped-particle correction, radius adjustment and reseeding; 3D
    # advection / correction / adjustment of particles seeded here (the
    # reference's seeding is 2D code)
    np.savez_compressed(os.path.join(OUT, "pls.npz"), **run_pls2d(), **run_pls3d())

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
    main(sys.argv[1] if len(sys.argv) > 1 else None)  # "mac": that fixture only
