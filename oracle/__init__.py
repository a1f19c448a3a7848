"""CPU oracle for the level-set transport path -- TEST INFRASTRUCTURE ONLY.

Two libraries sit behind this module:

* ``liboracle.so`` -- our FP64 C restatement of the reference's hot path
  (``oracle/sl_oracle.c``; every function cites the reference file:line it
  follows).
* ``_ref/libdcell_ref.so`` -- the reference's OWN C sources compiled against
  ``oracle/shim`` (see ``oracle/Makefile``); present only where the reference
  tree was available at build time.  ``oracle.reference`` wraps it.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may use this package, and only to check results / as the timed CPU baseline.
The product path (``dcell_b200``) never imports it.

Array conventions: phi is (nz, ny, nx) or (ny, nx) float64, x fastest;
velocity is (nz, ny, nx, 3) or (ny, nx, 2) with the MAC components innermost
(u at x-face i-1/2, v at y-face j-1/2, w at z-face k-1/2); band is an
(nb, 3) int32 array of GLOBAL (x, y, z) indices; ``origin`` is the global
index of element 0 (the reference Grid's ``p``).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

NODE_FIELDS = ("px", "py", "pz", "axis", "shift", "signCenter", "signFace", "d",
               "Xx", "Xy", "Xz", "opx", "opy", "opz", "nx", "ny", "nz", "k")
NODE_W = len(NODE_FIELDS)


class Geom(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("px", ctypes.c_int), ("py", ctypes.c_int), ("pz", ctypes.c_int),
                ("hx", ctypes.c_double), ("hy", ctypes.c_double), ("hz", ctypes.c_double)]


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def lib():
    """Load liboracle.so, compiling it with gcc first if it is missing."""
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        src = os.path.join(HERE, "sl_oracle.c")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
            subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
        L = ctypes.CDLL(path)
        vp, i, d, l = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_long
        L.orc_sl_step.argtypes = [vp, vp, vp, d, vp, i, i, i, vp]
        L.orc_sl_step.restype = i
        L.orc_interp_velocity.argtypes = [vp, vp, vp, i, vp]
        L.orc_tricubic_coefs.argtypes = [vp, vp]
        L.orc_bicubic_coefs.argtypes = [vp, vp]
        L.orc_sample.argtypes = [vp, vp, i, d, d, d]
        L.orc_sample.restype = d
        L.orc_ortho2d.argtypes = [vp, vp, vp]
        L.orc_ortho3d.argtypes = [vp, vp, vp]
        L.orc_irregular_nodes.argtypes = [vp, vp, vp, i, vp, l]
        L.orc_irregular_nodes.restype = l
        L.orc_node_surface.argtypes = [vp, vp, vp, l]
        L.orc_max_velocity.argtypes = [vp, vp, vp, l]
        L.orc_max_velocity.restype = d
        L.orc_volume.argtypes = [vp, vp, d]
        L.orc_volume.restype = d
        L.orc_reinit.argtypes = [vp, vp, vp, l, d, d, vp, l]
        L.orc_reinit.restype = l
        L.orc_pls_advect.argtypes = [vp, vp, vp, l, d]
        L.orc_pls_correct.argtypes = [vp, vp, vp, l, vp, l]
        L.orc_pls_correct.restype = l
        L.orc_pls_adjust.argtypes = [vp, vp, vp, l, vp]
        L.orc_pls_init.argtypes = [vp, vp, vp, l, vp, vp, vp, l]
        L.orc_pls_init.restype = l
        L.orc_pls_reseed.argtypes = [vp, vp, vp, l, vp, vp, vp, l, l, vp]
        L.orc_advect_mac.argtypes = [vp, vp, vp, vp, vp, d, vp]
        L.orc_pls_reseed.restype = l
        _LIB = L
    return _LIB


def geom(shape, h, origin=(0, 0, 0)):
    """Geom from a phi shape ((nz,ny,nx) or (ny,nx)), spacing and origin."""
    if len(shape) == 2:
        ny, nx = shape
        nz = 1
    else:
        nz, ny, nx = shape
    h = np.broadcast_to(np.asarray(h, dtype=np.float64), (3,))
    o = tuple(origin) + (0,) * (3 - len(origin))
    return Geom(int(nx), int(ny), int(nz), int(o[0]), int(o[1]), int(0 if nz == 1 else o[2]),
                float(h[0]), float(h[1]), float(h[2]))


def _band(band):
    if band is None:
        return None, 0
    b = np.ascontiguousarray(band, dtype=np.int32).reshape(-1, 3)
    return b, b.shape[0]


def sl_step(phi0, vel, dt, h, origin=(0, 0, 0), band=None, interp="linear", backtrace="euler", phi=None):
    """One semi-Lagrangian step (AdvectSL.c:23-89 for linear/euler)."""
    phi0 = np.ascontiguousarray(phi0, dtype=np.float64)
    vel = np.ascontiguousarray(vel, dtype=np.float64)
    out = phi0.copy() if phi is None else np.ascontiguousarray(phi, dtype=np.float64).copy()
    g = geom(phi0.shape, h, origin)
    b, nb = _band(band)
    rc = lib().orc_sl_step(ctypes.byref(g), _ptr(phi0), _ptr(vel), float(dt), _ptr(b), nb,
                           {"linear": 0, "cubic": 1}[interp], {"euler": 0, "midpoint": 1}[backtrace],
                           _ptr(out))
    assert rc == 0
    return out


def interp_velocity(vel, X, h=1.0, origin=(0, 0, 0)):
    vel = np.ascontiguousarray(vel, dtype=np.float64)
    shape = vel.shape[:-1]
    X = np.ascontiguousarray(X, dtype=np.float64).reshape(-1, 3)
    V = np.zeros_like(X)
    g = geom(shape, h, origin)
    lib().orc_interp_velocity(ctypes.byref(g), _ptr(vel), _ptr(X), X.shape[0], _ptr(V))
    return V


def tricubic_coefs(stencil64):
    s = np.ascontiguousarray(stencil64, dtype=np.float64).reshape(64)
    a = np.zeros(64)
    lib().orc_tricubic_coefs(_ptr(s), _ptr(a))
    return a


def bicubic_coefs(stencil16):
    s = np.ascontiguousarray(stencil16, dtype=np.float64).reshape(16)
    a = np.zeros(16)
    lib().orc_bicubic_coefs(_ptr(s), _ptr(a))
    return a


def catmull_rom_operator(dim=3):
    """Dense (4^dim x 4^dim) matrix M with a = M @ stencil (a[px+4py+16pz])."""
    n = 4 ** dim
    M = np.zeros((n, n))
    f = tricubic_coefs if dim == 3 else bicubic_coefs
    for s in range(n):
        e = np.zeros(n)
        e[s] = 1.0
        M[:, s] = f(e)
    return M


def sample(phi, fn, X, h, origin=(0, 0, 0)):
    """Bilinear/trilinear sample of a grid function at index-space points X.
    fn: 0 identity, 1-3 d/dx,d/dy,d/dz, 4 curvature, 5 smoothed delta."""
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    g = geom(phi.shape, h, origin)
    X = np.asarray(X, dtype=np.float64).reshape(-1, 3)
    return np.array([lib().orc_sample(ctypes.byref(g), _ptr(phi), int(fn), *map(float, x)) for x in X])


def ortho3d(phi3, phi5):
    a3 = np.ascontiguousarray(phi3, dtype=np.float64).reshape(27)
    a5 = np.ascontiguousarray(phi5, dtype=np.float64).reshape(125)
    op = np.zeros(3)
    lib().orc_ortho3d(_ptr(a3), _ptr(a5), _ptr(op))
    return op


def ortho2d(phi3, phi5):
    a3 = np.ascontiguousarray(phi3, dtype=np.float64).reshape(9)
    a5 = np.ascontiguousarray(phi5, dtype=np.float64).reshape(25)
    op = np.zeros(3)
    lib().orc_ortho2d(_ptr(a3), _ptr(a5), _ptr(op))
    return op


def irregular_nodes(phi, h, band, origin=(0, 0, 0), surface=True):
    """Irregular-node list (IrregularNodes.c:32-141 / IrregularNodes3D.c:6-117),
    optionally with normals and curvature; (n, 18) float64, NODE_FIELDS order."""
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    g = geom(phi.shape, h, origin)
    b, nb = _band(band)
    cap = max(16, 13 * nb)
    out = np.zeros((cap, NODE_W))
    n = lib().orc_irregular_nodes(ctypes.byref(g), _ptr(phi), _ptr(b), nb, _ptr(out), cap)
    assert n <= cap
    out = np.ascontiguousarray(out[:n])
    if surface and n:
        lib().orc_node_surface(ctypes.byref(g), _ptr(phi), _ptr(out), n)
    return out


def max_velocity(vel, nodes, h=1.0, origin=(0, 0, 0)):
    vel = np.ascontiguousarray(vel, dtype=np.float64)
    g = geom(vel.shape[:-1], h, origin)
    nodes = np.ascontiguousarray(nodes, dtype=np.float64)
    return lib().orc_max_velocity(ctypes.byref(g), _ptr(vel), _ptr(nodes), nodes.shape[0])


def volume(phi, h, eps):
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    g = geom(phi.shape, h)
    return lib().orc_volume(ctypes.byref(g), _ptr(phi), float(eps))


def reinit(phi, nodes, band_width=6.0, bucket=1.0 / 64, origin=(0, 0, 0)):
    """Bucketed fast-marching reinitialisation (orc_reinit; the reference's
    LevelSetReinitialize, FastMarching.c:11-146, with buckets of width
    `bucket` cells in place of its heap).  phi in cell units; nodes: (n, 18)
    irregular-node rows of phi.  Returns (phi, band (nb, 3) int32, grid order)."""
    phi = np.array(phi, dtype=np.float64, copy=True, order="C")
    g = geom(phi.shape, 1.0, origin)
    nodes = np.ascontiguousarray(nodes, dtype=np.float64).reshape(-1, NODE_W)
    cap = phi.size
    band = np.zeros((cap, 3), dtype=np.int32)
    n = lib().orc_reinit(ctypes.byref(g), _ptr(phi), _ptr(nodes), nodes.shape[0], float(band_width), float(bucket),
                         _ptr(band), cap)
    if n == -1:
        raise FloatingPointError("fast-marching update is not a number")
    if n < 0:
        raise RuntimeError("fast marching did not settle within the buckets")
    return phi, band[:n].copy()


def velocity_box(global_field, origin, shape, first=1):
    """The velocity grid of a level set whose phi box starts at global index
    `origin` (x, y(, z)) with extents `shape` ((nz, ny, nx) or (ny, nx)):
    components first .. first+dim-1 of the fluid's global field ([z][y][x][c]
    or [y][x][c]) where the box overlaps the global domain, zero elsewhere
    (LevelSetGetVelocity, Advect.c:145-192: GridResize zeroes the grid, then
    NGA_Get fills the part of the box inside the global array)."""
    gf = np.asarray(global_field, dtype=np.float64)
    dim = len(shape)
    out = np.zeros(tuple(shape) + (dim,))
    lo = [max(0, int(origin[a])) for a in range(dim)]                            # x, y(, z)
    hi = [min(int(origin[a]) + int(shape[dim - 1 - a]), gf.shape[dim - 1 - a]) for a in range(dim)]
    if any(h <= l for l, h in zip(lo, hi)):
        return out
    src = tuple(slice(lo[a], hi[a]) for a in reversed(range(dim)))
    dst = tuple(slice(lo[a] - int(origin[a]), hi[a] - int(origin[a])) for a in reversed(range(dim)))
    out[dst] = gf[src + (slice(first, first + dim),)]
    return out


# ---------------------------------------------------------------------------
# particle level set (LevelSetMethod/ParticleLS*.c); particles are (n, 4)
# float64 rows X.x, X.y, X.z, radius in global index space

class PlsParams(ctypes.Structure):
    """LevelSetInitializeParticles' parameters (ParticleLS.c:21-27)."""
    _fields_ = [("r_min", ctypes.c_double), ("r_max", ctypes.c_double), ("d_init", ctypes.c_double),
                ("g_tol", ctypes.c_double), ("e_dist", ctypes.c_double), ("s_init", ctypes.c_int),
                ("l_max", ctypes.c_int)]


def pls_params(dim=2, **kw):
    p = PlsParams(0.1, 0.5, 3.0, 1e-3, 0.5, 16 if dim == 2 else 32, 30)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _parts(parts):
    return np.array(parts, dtype=np.float64, copy=True, order="C").reshape(-1, 4)


def pls_advect(vel, parts, dt, h, origin=(0, 0, 0)):
    """RK2-midpoint particle advection (ParticleLS2D.c:6-36 / ParticleLS3D.c:6-36)."""
    vel = np.ascontiguousarray(vel, dtype=np.float64)
    out = _parts(parts)
    g = geom(vel.shape[:-1], h, origin)
    lib().orc_pls_advect(ctypes.byref(g), _ptr(vel), _ptr(out), out.shape[0], float(dt))
    return out


def pls_correct(phi, band, parts, h=1.0, origin=(0, 0, 0)):
    """Escaped-particle error correction of phi at the band points
    (ParticleLS2D.c:40-115 / ParticleLS3D.c:40-116).  Returns (phi, number
    of corners skipped outside the grid)."""
    phi = np.array(phi, dtype=np.float64, copy=True, order="C")
    g = geom(phi.shape, h, origin)
    b, _ = _band(band)
    P = _parts(parts)
    skipped = lib().orc_pls_correct(ctypes.byref(g), _ptr(phi), _ptr(b), b.shape[0], _ptr(P), P.shape[0])
    return phi, skipped


def pls_adjust(phi, parts, h=1.0, origin=(0, 0, 0), params=None):
    """ParticleLS_AdjustRadii (ParticleLS.c:158-185)."""
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    g = geom(phi.shape, h, origin)
    P = _parts(parts)
    prm = params or pls_params(phi.ndim)
    lib().orc_pls_adjust(ctypes.byref(g), _ptr(phi), _ptr(P), P.shape[0], ctypes.byref(prm))
    return P


def pls_init(phi, band, rng, h=1.0, origin=(0, 0, 0), params=None):
    """LevelSetInitializeParticles (ParticleLS.c:6-88), 2D.  rng: the drand48
    state.  Returns (particles, rng after)."""
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    g = geom(phi.shape, h, origin)
    b, _ = _band(band)
    prm = params or pls_params(2)
    st = ctypes.c_uint64(int(rng))
    cap = b.shape[0] * prm.s_init
    out = np.zeros((max(cap, 1), 4))
    n = lib().orc_pls_init(ctypes.byref(g), _ptr(phi), _ptr(b), b.shape[0], ctypes.byref(prm), ctypes.byref(st),
                           _ptr(out), cap)
    if n < 0:
        raise ValueError("particle seeding is 2D")
    return out[:n].copy(), st.value


def pls_reseed(phi, band, parts, rng, h=1.0, origin=(0, 0, 0), params=None):
    """ParticleLS_ReseedParticles (ParticleLS.c:202-295), 2D.  Returns
    (particles, rng after, particles not counted because outside the box)."""
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    g = geom(phi.shape, h, origin)
    b, _ = _band(band)
    prm = params or pls_params(2)
    P0 = _parts(parts)
    cap = P0.shape[0] + b.shape[0] * prm.s_init
    P = np.zeros((max(cap, 1), 4))
    P[:P0.shape[0]] = P0
    st = ctypes.c_uint64(int(rng))
    miss = ctypes.c_long(0)
    n = lib().orc_pls_reseed(ctypes.byref(g), _ptr(phi), _ptr(b), b.shape[0], ctypes.byref(prm), ctypes.byref(st),
                             _ptr(P), P0.shape[0], cap, ctypes.byref(miss))
    if n < 0:
        raise ValueError("particle reseeding is 2D")
    return P[:n].copy(), st.value, miss.value


# ---------------------------------------------------------------------------
# first-order conservative upwind step on MAC faces (LevelSetMethod/AdvectMAC.c)

def advect_mac(phi, u, v, w, dt, h, origin=(0, 0, 0), out=None):
    """LevelSetAdvectMAC (2D, phi (ny, nx)) / LevelSetAdvectMAC_3D (phi
    (nz, ny, nx)), AdvectMAC.c:18-111: phi, u, v (, w) share one grid at
    global `origin`; returns a copy of `out` (default phi) with the updated
    points replaced, or None where the reference would read outside its grid
    (an axis with a non-empty range and origin > 0 or extent < 3)."""
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    u = np.ascontiguousarray(u, dtype=np.float64)
    v = np.ascontiguousarray(v, dtype=np.float64)
    w = np.ascontiguousarray(w, dtype=np.float64) if phi.ndim == 3 else None
    res = (phi if out is None else np.asarray(out, dtype=np.float64)).copy()
    g = geom(phi.shape, h, origin)
    rc = lib().orc_advect_mac(ctypes.byref(g), _ptr(phi), _ptr(u), _ptr(v), _ptr(w), float(dt), _ptr(res))
    return None if rc else res
