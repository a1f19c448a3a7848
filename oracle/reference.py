"""ctypes wrapper over the reference's own level-set C (oracle/_ref) --
TEST INFRASTRUCTURE ONLY.

``_ref/libdcell_ref.so`` is the reference's unmodified hot-path sources plus
``oracle/ref_driver.c``, compiled by ``make -C oracle ref REF=<reference tree>`` where the
reference tree is present.  ``available()`` says whether it was built.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import NODE_W

HERE = os.path.dirname(os.path.abspath(__file__))
PATH = os.path.join(HERE, "_ref", "libdcell_ref.so")
# the same reference sources linked with the B200 drop-in (make -C oracle dropin REF=<reference tree>)
DROPIN_PATH = os.path.join(HERE, "_ref", "libdcell_ref_b200.so")
_LIBS = {}


def available(path=PATH) -> bool:
    return os.path.exists(path)


def lib(path=PATH):
    if path not in _LIBS:
        L = ctypes.CDLL(path)
        vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.dref_ls_create.restype = vp
        L.dref_ls_create.argtypes = [d, d, d, i, i, i, i, i, i]
        L.dref_ls_destroy.argtypes = [vp]
        L.dref_ls_geometry.argtypes = [vp, vp, vp]
        L.dref_ls_set_phi.argtypes = [vp, vp, i]
        L.dref_ls_get_phi.argtypes = [vp, vp, i]
        L.dref_ls_set_band.argtypes = [vp, vp, i]
        L.dref_ls_band_length.argtypes = [vp]
        L.dref_ls_get_band.argtypes = [vp, vp]
        L.dref_ls_param.argtypes = [vp, i]
        L.dref_ls_param.restype = d
        L.dref_vel_create.restype = vp
        L.dref_vel_create.argtypes = [vp, vp]
        L.dref_vel_destroy.argtypes = [vp]
        for f in ("dref_advect_sl", "dref_rk2_half", "dref_rk2_full", "dref_advect_and_reinit",
                  "dref_cfl_increment"):
            getattr(L, f).argtypes = [vp, vp, d]
        L.dref_copy_phi_to_phi0.argtypes = [vp]
        L.dref_max_velocity.argtypes = [vp, vp]
        L.dref_max_velocity.restype = d
        L.dref_update_irregular.argtypes = [vp]
        L.dref_reinitialize.argtypes = [vp]
        L.dref_get_irregular.argtypes = [vp, vp, i]
        L.dref_init_sphere.restype = vp
        L.dref_init_sphere.argtypes = [d, d, d, d, d]
        L.dref_init_circle.restype = vp
        L.dref_init_circle.argtypes = [d, d, d, d]
        L.dref_sample.argtypes = [vp, i, d, d, d]
        L.dref_sample.restype = d
        L.dref_interp_velocity.argtypes = [vp, d, d, d, vp]
        L.dref_ortho3d.argtypes = [vp, vp, vp]
        L.dref_ortho2d.argtypes = [vp, vp, vp]
        L.dref_tricubic_coefs.argtypes = [vp, vp]
        L.dref_get_velocity.argtypes = [vp, vp, ctypes.c_int, vp, vp]
        for f in ("dref_pls_init", "dref_pls_create_empty", "dref_pls_count", "dref_pls_correct",
                  "dref_pls_adjust", "dref_pls_reseed"):
            getattr(L, f).argtypes = [vp]
        L.dref_pls_params.argtypes = [vp, vp]
        L.dref_pls_get.argtypes = [vp, vp]
        L.dref_pls_set.argtypes = [vp, vp, i]
        for f in ("dref_pls_advect", "dref_pls_step", "dref_pls_rk2_half", "dref_pls_rk2_full"):
            getattr(L, f).argtypes = [vp, vp, d]
        L.dref_rand48_get.argtypes = [vp]
        L.dref_rand48_get.restype = None
        L.dref_rand48_set.argtypes = [vp]
        L.dref_rand48_set.restype = None
        if hasattr(L, "dref_grid_write"):  # the reference's writers (Common/Serialize.c, IrregularNodes.c, Array.c)
            L.dref_set_dirs.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
            L.dref_set_dirs.restype = None
            L.dref_grid_write.argtypes = [vp, ctypes.c_char_p, i]
            L.dref_vel_write.argtypes = [vp, ctypes.c_char_p, i]
            L.dref_set_surface.argtypes = [vp]
            L.dref_write_irregular.argtypes = [vp, i]
            L.dref_pls_write.argtypes = [vp, i]
        if hasattr(L, "dref_advect_mac"):  # the reference-only library (shim/mac)
            L.dref_advect_mac.argtypes = [vp, vp, vp, vp, vp, vp, vp, d, vp]
        _LIBS[path] = L
    return _LIBS[path]


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def rand48_state(path=PATH) -> int:
    """The C library's drand48 state (48 bits) that PETSCRAND48 draws from."""
    s = np.zeros(3, dtype=np.uint16)
    lib(path).dref_rand48_get(_p(s))
    return int(s[0]) | (int(s[1]) << 16) | (int(s[2]) << 32)


def set_rand48_state(x: int, path=PATH):
    s = np.array([x & 0xFFFF, (x >> 16) & 0xFFFF, (x >> 32) & 0xFFFF], dtype=np.uint16)
    lib(path).dref_rand48_set(_p(s))


class RefLevelSet:
    """A reference ``LevelSet`` (LevelSetMethod.h:10-26) driven from numpy."""

    def __init__(self, handle, path=PATH):
        self.h = handle
        self._vel = None
        self.L = lib(path)

    @classmethod
    def create(cls, h, origin, shape, path=PATH):
        """LevelSetCreate (LevelSet.c:6-37); shape (nz,ny,nx) or (ny,nx)."""
        if len(shape) == 2:
            ny, nx = shape
            nz = 0
        else:
            nz, ny, nx = shape
        o = tuple(origin) + (0,) * (3 - len(origin))
        hh = np.broadcast_to(np.asarray(h, dtype=np.float64), (3,))
        return cls(lib(path).dref_ls_create(*map(float, hh), *map(int, o), int(nx), int(ny), int(nz)), path)

    @classmethod
    def sphere(cls, h, center, r, path=PATH):
        return cls(lib(path).dref_init_sphere(float(h), *map(float, center), float(r)), path)

    @classmethod
    def circle(cls, h, center, r, path=PATH):
        return cls(lib(path).dref_init_circle(float(h), *map(float, center), float(r)), path)

    def close(self):
        if self._vel:
            self.L.dref_vel_destroy(self._vel)
            self._vel = None
        if self.h:
            self.L.dref_ls_destroy(self.h)
            self.h = None

    def geometry(self):
        p = (ctypes.c_int * 3)()
        n = (ctypes.c_int * 3)()
        self.L.dref_ls_geometry(self.h, p, n)
        return tuple(p), tuple(n)

    @property
    def shape(self):
        _, n = self.geometry()
        return (n[1], n[0]) if n[2] < 2 else (n[2], n[1], n[0])

    @property
    def origin(self):
        return self.geometry()[0]

    def get_phi(self, which=0):
        out = np.zeros(self.shape)
        self.L.dref_ls_get_phi(self.h, _p(out), which)
        return out

    def set_phi(self, phi, which=0):
        a = np.ascontiguousarray(phi, dtype=np.float64)
        assert a.shape == self.shape
        assert self.L.dref_ls_set_phi(self.h, _p(a), which) == 0

    def band(self):
        nb = self.L.dref_ls_band_length(self.h)
        out = np.zeros((nb, 3), dtype=np.int32)
        self.L.dref_ls_get_band(self.h, _p(out))
        return out

    def set_band(self, band):
        b = np.ascontiguousarray(band, dtype=np.int32).reshape(-1, 3)
        assert self.L.dref_ls_set_band(self.h, _p(b), b.shape[0]) == 0

    def set_velocity(self, vel):
        if self._vel:
            self.L.dref_vel_destroy(self._vel)
        v = np.ascontiguousarray(vel, dtype=np.float64)
        self._vel = self.L.dref_vel_create(self.h, _p(v))

    def param(self, which):
        return self.L.dref_ls_param(self.h, {"bandWidth": 0, "PHI_INF": 1, "CFLcount": 2,
                                            "AdvectCount": 3, "maxVel": 4}[which])

    def copy_phi_to_phi0(self):
        assert self.L.dref_copy_phi_to_phi0(self.h) == 0

    def advect_sl(self, dt):
        """LevelSetAdvectSL (AdvectSL.c:6): phi[band] <- SL(phi0, vel, dt)."""
        assert self.L.dref_advect_sl(self.h, self._vel, float(dt)) == 0

    def rk2_half(self, dt):
        assert self.L.dref_rk2_half(self.h, self._vel, float(dt)) == 0

    def rk2_full(self, dt):
        assert self.L.dref_rk2_full(self.h, self._vel, float(dt)) == 0

    def advect_and_reinit(self, dt):
        assert self.L.dref_advect_and_reinit(self.h, self._vel, float(dt)) == 0

    def cfl_increment(self, dt):
        assert self.L.dref_cfl_increment(self.h, self._vel, float(dt)) == 0

    def max_velocity(self):
        return self.L.dref_max_velocity(self.h, self._vel)

    def update_irregular(self):
        n = self.L.dref_update_irregular(self.h)
        assert n >= 0
        return n

    def irregular_nodes(self, surface=True):
        n = self.L.dref_update_irregular(self.h)
        out = np.zeros((max(n, 1), NODE_W))
        self.L.dref_get_irregular(self.h, _p(out), 1 if surface else 0)
        return out[:n]

    def nodes_no_update(self, n, surface=True):
        out = np.zeros((max(n, 1), NODE_W))
        self.L.dref_get_irregular(self.h, _p(out), 1 if surface else 0)
        return out[:n]

    def reinitialize(self):
        assert self.L.dref_reinitialize(self.h) == 0

    # output through the reference's own writers, into `wd` (grids, node
    # lists: DCellGetWorkingDirectory) and `tmp` (Arrays: PetscGetTmp)
    def set_output_dirs(self, wd, tmp):
        self.L.dref_set_dirs(wd.encode(), tmp.encode())

    def grid_write(self, name, t):
        """GridSetName + GridWrite (Common/Serialize.c:23-55) of phi."""
        assert self.L.dref_grid_write(self.h, name.encode(), int(t)) == 0

    def velocity_write(self, name, t):
        """GridWrite of the velocity grid set by set_velocity (dof 2 / 3)."""
        assert self.L.dref_vel_write(self._vel, name.encode(), int(t)) == 0

    def set_surface(self):
        """Store the node normals and curvature in the irregular nodes."""
        return self.L.dref_set_surface(self.h)

    def write_irregular(self, idx):
        """LevelSetWriteIrregularNodeList (IrregularNodes.c:224-246)."""
        assert self.L.dref_write_irregular(self.h, int(idx)) == 0

    def write_particles(self, t):
        """ArrayWrite (Common/Array.c:134-150) of the particle Array."""
        assert self.L.dref_pls_write(self.h, int(t)) == 0

    def get_velocity(self, global_field):
        """LevelSetGetVelocity (Advect.c:145-192) from a one-process Global
        Array holding `global_field` ([z][y][x][c] in 3D, [y][x][c] in 2D,
        c = CELL_CENTER, U_FACE, V_FACE(, W_FACE)); returns the velocity grid
        of the level set's phi box, (nz, ny, nx, 3) or (ny, nx, 2)."""
        gf = np.ascontiguousarray(global_field, dtype=np.float64)
        dims = np.array(gf.shape, dtype=np.int32)
        shape = self.shape
        out = np.zeros(shape + (len(shape),))
        assert self.L.dref_get_velocity(self.h, _p(gf), gf.ndim, _p(dims), _p(out)) == 0
        return out

    # particle level set (LevelSetMethod/ParticleLS*.c); particles are
    # (n, 4) float64 rows X.x, X.y, X.z, radius (struct _Particle)
    def pls_init(self):
        """LevelSetInitializeParticles (ParticleLS.c:6-88)."""
        assert self.L.dref_pls_init(self.h) == 0

    def pls_create_empty(self):
        assert self.L.dref_pls_create_empty(self.h) == 0

    def pls_params(self):
        out = np.zeros(7)
        assert self.L.dref_pls_params(self.h, _p(out)) == 0
        keys = ("R_MIN", "R_MAX", "D_INIT", "S_INIT", "L_MAX", "G_TOL", "E_DIST")
        return dict(zip(keys, out.tolist()))

    def particles(self):
        n = self.L.dref_pls_count(self.h)
        out = np.zeros((max(n, 0), 4))
        if n > 0:
            self.L.dref_pls_get(self.h, _p(out))
        return out

    def set_particles(self, parts):
        a = np.ascontiguousarray(parts, dtype=np.float64).reshape(-1, 4)
        assert self.L.dref_pls_set(self.h, _p(a), len(a)) == 0

    def pls_advect(self, dt):
        """pls->AdvectParticles (ParticleLS2D.c:6-36 / ParticleLS3D.c:6-36) on the set velocity."""
        assert self.L.dref_pls_advect(self.h, self._vel, float(dt)) == 0

    def pls_correct(self):
        """pls->ErrorCorrection (ParticleLS2D.c:40-115 / ParticleLS3D.c:40-116)."""
        assert self.L.dref_pls_correct(self.h) == 0

    def pls_adjust(self):
        """ParticleLS_AdjustRadii (ParticleLS.c:158-185)."""
        assert self.L.dref_pls_adjust(self.h) == 0

    def pls_reseed(self):
        """ParticleLS_ReseedParticles (ParticleLS.c:202-295)."""
        assert self.L.dref_pls_reseed(self.h) == 0

    def pls_step(self, dt):
        """LevelSetAdvectPLS (ParticleLS.c:299-329)."""
        assert self.L.dref_pls_step(self.h, self._vel, float(dt)) == 0

    def pls_rk2_half(self, dt):
        assert self.L.dref_pls_rk2_half(self.h, self._vel, float(dt)) == 0

    def pls_rk2_full(self, dt):
        assert self.L.dref_pls_rk2_full(self.h, self._vel, float(dt)) == 0

    def sample(self, fn, X):
        return np.array([self.L.dref_sample(self.h, int(fn), *map(float, x)) for x in np.reshape(X, (-1, 3))])

    def interp_velocity(self, X):
        out = np.zeros(3)
        res = []
        for x in np.reshape(X, (-1, 3)):
            self.L.dref_interp_velocity(self._vel, *map(float, x), _p(out))
            res.append(out.copy())
        return np.array(res)


def tricubic_coefs(stencil64):
    s = np.ascontiguousarray(stencil64, dtype=np.float64).reshape(64)
    a = np.zeros(64)
    lib().dref_tricubic_coefs(_p(s), _p(a))
    return a


def ortho3d(phi3, phi5):
    a3 = np.ascontiguousarray(phi3, dtype=np.float64).reshape(27)
    a5 = np.ascontiguousarray(phi5, dtype=np.float64).reshape(125)
    op = np.zeros(3)
    lib().dref_ortho3d(_p(a3), _p(a5), _p(op))
    return op


def ortho2d(phi3, phi5):
    a3 = np.ascontiguousarray(phi3, dtype=np.float64).reshape(9)
    a5 = np.ascontiguousarray(phi5, dtype=np.float64).reshape(25)
    op = np.zeros(3)
    lib().dref_ortho2d(_p(a3), _p(a5), _p(op))
    return op


def advect_mac(phi, u, v, w, dt, h, origin=(0, 0, 0), out=None):
    """The reference's LevelSetAdvectMAC (2D, phi (ny, nx)) or
    LevelSetAdvectMAC_3D (phi (nz, ny, nx)), LevelSetMethod/AdvectMAC.c:18-111,
    compiled from its own source: phi, u, v (, w) share the grid at global
    `origin` (x, y(, z)); returns a copy of `out` (default phi) with the
    updated points replaced.  Call only on grids where the routine stays in
    bounds (oracle.advect_mac returns None for the others)."""
    phi = np.ascontiguousarray(phi, dtype=np.float64)
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (u, v)]
    arrs.append(np.ascontiguousarray(w, dtype=np.float64) if phi.ndim == 3 else np.zeros(1))
    res = (phi if out is None else np.asarray(out, dtype=np.float64)).copy()
    shape = phi.shape if phi.ndim == 3 else (1,) + phi.shape
    n = np.array([shape[2], shape[1], shape[0]], dtype=np.int32)
    o = tuple(int(x) for x in origin) + (0,) * (3 - len(origin))
    pp = np.array([o[0], o[1], o[2] if phi.ndim == 3 else 0], dtype=np.int32)
    hh = np.broadcast_to(np.asarray(h, dtype=np.float64), (3,)).copy()
    rc = lib().dref_advect_mac(_p(n), _p(pp), _p(hh), _p(phi), _p(arrs[0]), _p(arrs[1]), _p(arrs[2]), float(dt),
                               _p(res))
    assert rc == 0
    return res
