"""ctypes binding of ``lib/libdcell_ls.so`` (the C ABI in include/dcell_ls.h).

Loading fails loudly when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libdcell_ls.so")

OK, ERR_ARG, ERR_CUDA, ERR_DEPARTURE, ERR_NONFINITE, ERR_TIMEOUT, ERR_CAPACITY, ERR_UNSUPPORTED, ERR_NOMEM = range(9)
F32, F64 = 0, 1
LINEAR, CUBIC_PLAIN, CUBIC_SEPARABLE, CUBIC_TC = 0, 1, 2, 3
EULER, MIDPOINT = 0, 1
FLAG_DEPARTURE_CLAMPED, FLAG_NONFINITE, FLAG_CAPACITY, FLAG_WAIT_TIMEOUT, FLAG_BAD_BAND = 1, 2, 4, 8, 16
FLAG_UNSETTLED = 32
FLAG_PARTICLE_OUTSIDE = 64

GATHER_FORM = 0x100  # OR'ed into interp: the global-gather form on dense FP32 grids
INTERP = {"linear": LINEAR, "cubic": CUBIC_PLAIN, "cubic_plain": CUBIC_PLAIN, "cubic_separable": CUBIC_SEPARABLE,
          "cubic_tc": CUBIC_TC, "linear_gather": LINEAR | GATHER_FORM,
          "cubic_plain_gather": CUBIC_PLAIN | GATHER_FORM, "cubic_separable_gather": CUBIC_SEPARABLE | GATHER_FORM}
BACKTRACE = {"euler": EULER, "midpoint": MIDPOINT}


class DcellError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"dcell error {code}: {msg}")
        self.code = code


class Geom(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int * 3), ("p", ctypes.c_int * 3), ("h", ctypes.c_double * 3)]


class IrregularNode(ctypes.Structure):
    _fields_ = [("pos", ctypes.c_int * 3), ("axis", ctypes.c_int), ("shift", ctypes.c_int),
                ("signCenter", ctypes.c_int), ("signFace", ctypes.c_int), ("pad", ctypes.c_int),
                ("d", ctypes.c_double), ("X", ctypes.c_double * 3), ("op", ctypes.c_double * 3),
                ("n", ctypes.c_double * 3), ("k", ctypes.c_double)]


class PlsParams(ctypes.Structure):
    """struct dcell_pls_params: LevelSetInitializeParticles' parameters (ParticleLS.c:21-27)."""
    _fields_ = [("r_min", ctypes.c_double), ("r_max", ctypes.c_double), ("d_init", ctypes.c_double),
                ("g_tol", ctypes.c_double), ("e_dist", ctypes.c_double), ("s_init", ctypes.c_int),
                ("l_max", ctypes.c_int)]


class LsLoop(ctypes.Structure):
    """struct dcell_ls_loop: the loop counters of struct _LevelSet (LevelSetMethod.h:10-26)."""
    _fields_ = [("CFLcount", ctypes.c_double), ("CFLthres", ctypes.c_double), ("maxVel", ctypes.c_double),
                ("bandWidth", ctypes.c_double), ("AdvectCount", ctypes.c_int), ("AdvectThres", ctypes.c_int),
                ("reinitialized", ctypes.c_int), ("band", ctypes.c_int)]


NODE_DTYPE = np.dtype([("pos", "<i4", 3), ("axis", "<i4"), ("shift", "<i4"), ("signCenter", "<i4"),
                       ("signFace", "<i4"), ("pad", "<i4"), ("d", "<f8"), ("X", "<f8", 3), ("op", "<f8", 3),
                       ("n", "<f8", 3), ("k", "<f8")])
assert NODE_DTYPE.itemsize == ctypes.sizeof(IrregularNode) == 120
BOX_DTYPE = np.dtype([("offset", "<i8"), ("p", "<i4", 3), ("n", "<i4", 3)])  # struct dcell_box
assert BOX_DTYPE.itemsize == 32


def geom(shape, h, origin=(0, 0, 0)) -> Geom:
    """Geom from a phi shape ((nz, ny, nx) or (ny, nx)), spacing and global origin."""
    if len(shape) == 2:
        ny, nx = shape
        nz = 1
    else:
        nz, ny, nx = shape
    hh = np.broadcast_to(np.asarray(h, dtype=np.float64), (3,))
    o = tuple(int(v) for v in origin) + (0,) * (3 - len(origin))
    g = Geom()
    g.n[:] = [int(nx), int(ny), int(nz)]
    g.p[:] = [o[0], o[1], o[2] if nz > 1 else 0]
    g.h[:] = [float(hh[0]), float(hh[1]), float(hh[2])]
    return g


_LIB = None


def lib():
    """The loaded C-ABI library (raises if it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m dcell_b200.build` "
                          "(the level-set kernels have no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    vp, i, d, sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_size_t
    G = ctypes.POINTER(Geom)
    L.dcell_last_error.restype = ctypes.c_char_p
    L.dcell_version.restype = i
    L.dcell_sl_step.argtypes = [G, i, vp, vp, d, vp, i, i, i, vp, vp, vp]
    L.dcell_irregular_nodes_scratch_bytes.argtypes = [i]
    L.dcell_irregular_nodes_scratch_bytes.restype = sz
    L.dcell_irregular_nodes.argtypes = [G, i, vp, vp, i, i, vp, i, vp, vp, sz, vp, vp]
    L.dcell_irregular_nodes_noalloc.argtypes = [G, i, vp, vp, i, i, vp, i, vp, vp, vp]
    L.dcell_max_velocity.argtypes = [G, i, vp, vp, vp, i, vp, vp]
    L.dcell_volume_scratch_bytes.restype = sz
    L.dcell_volume.argtypes = [G, i, vp, d, vp, vp, sz, vp]
    L.dcell_velocity_box.argtypes = [G, i, vp, vp, i, i, vp, vp]
    L.dcell_velocity_boxes.argtypes = [vp, i, i, i, vp, vp, i, i, ctypes.c_longlong, vp, vp]
    L.dcell_reinit_scratch_bytes.argtypes = [G, i]
    L.dcell_reinit_scratch_bytes.restype = sz
    L.dcell_reinitialize.argtypes = [G, i, vp, vp, i, d, d, vp, i, vp, vp, sz, vp, vp]
    L.dcell_session_create.argtypes = [i, ctypes.POINTER(vp)]
    L.dcell_session_destroy.argtypes = [vp]
    L.dcell_ls_advect_sl.argtypes = [vp, G, vp, vp, vp, i, d, i, i, i, vp]
    L.dcell_ls_update_irregular_nodes.argtypes = [vp, G, vp, vp, i, i, i, vp, i, vp]
    L.dcell_ls_advect_sl_rk2_half.argtypes = [vp, G, vp, vp, vp, i, d, i, i, i, vp, i, vp, i, vp]
    L.dcell_ls_advect_sl_rk2_full.argtypes = [vp, G, vp, vp, vp, i, d, i, i, i, vp, i, vp, i, vp]
    L.dcell_ls_max_velocity.argtypes = [vp, G, vp, vp, i, vp]
    L.dcell_ls_reinitialize.argtypes = [vp, G, vp, vp, i, d, i, vp, i, vp]
    L.dcell_advect_mac.argtypes = [G, i, vp, vp, vp, vp, d, vp, vp]
    L.dcell_ls_advect_mac.argtypes = [vp, G, vp, vp, vp, vp, d, i, vp]
    L.dcell_tc_gemm_check.argtypes = [vp, vp, vp, vp]
    L.dcell_wait_timeout_check.argtypes = [vp, vp]
    L.dcell_sl_adjoint.argtypes = [G, i, vp, vp, d, i, i, vp, vp, vp, vp]
    L.dcell_ls_resident_set.argtypes = [vp, G, vp, vp, i, i]
    L.dcell_ls_resident_advect_and_reinit.argtypes = [vp, G, vp, i, d, i, i, i, ctypes.POINTER(LsLoop)]
    L.dcell_ls_resident_get.argtypes = [vp, G, vp, vp, i, vp]
    L.dcell_split_bf16.argtypes = [G, vp, vp, vp]
    L.dcell_sl_step_tc_split.argtypes = [G, vp, vp, d, vp, i, i, vp, vp, vp, vp]
    L.dcell_sl_step_tc_split_planes.argtypes = [G, vp, vp, d, i, i, i, vp, vp, vp, vp]
    L.dcell_batch_plan.argtypes = [vp, i, i, i, i, vp, i, vp]
    L.dcell_batch_sl_step.argtypes = [vp, i, vp, i, i, i, i, i, vp, vp, vp, i, i, vp, vp]
    L.dcell_batch_sl_step_tc_split.argtypes = [vp, i, vp, i, vp, vp, i, vp, vp, vp, vp]
    L.dcell_batch_tma_maps_bytes.argtypes = [i]
    L.dcell_batch_tma_maps_bytes.restype = sz
    L.dcell_batch_tma_maps.argtypes = [vp, i, vp, vp, vp, vp]
    L.dcell_batch_sl_step_tc_split_tma.argtypes = [vp, i, vp, i, vp, vp, vp, i, vp, vp, vp, vp]
    ll, P = ctypes.c_longlong, ctypes.POINTER(PlsParams)
    L.dcell_pls_default_params.argtypes = [i, P]
    L.dcell_pls_default_params.restype = None
    L.dcell_pls_advect.argtypes = [G, i, vp, vp, ll, d, vp, vp]
    L.dcell_pls_correct_scratch_bytes.argtypes = [G, i]
    L.dcell_pls_correct_scratch_bytes.restype = sz
    L.dcell_pls_correct.argtypes = [G, i, vp, vp, ll, vp, ll, vp, sz, vp, vp]
    L.dcell_pls_adjust_radii.argtypes = [G, i, vp, vp, ll, P, vp, vp]
    L.dcell_pls_scratch_bytes.argtypes = [G, ll, ll]
    L.dcell_pls_scratch_bytes.restype = sz
    L.dcell_pls_seed.argtypes = [G, i, vp, vp, ll, P, vp, vp, ll, vp, vp, sz, vp, vp]
    L.dcell_pls_reseed.argtypes = [G, i, vp, vp, ll, P, vp, vp, ll, ll, vp, vp, sz, vp, vp]
    L.dcell_ls_pls_advect.argtypes = [vp, G, vp, vp, ll, d]
    L.dcell_ls_pls_correct.argtypes = [vp, G, vp, vp, i, vp, ll]
    L.dcell_ls_pls_adjust_radii.argtypes = [vp, G, vp, vp, ll, P]
    L.dcell_ls_pls_seed.argtypes = [vp, G, vp, vp, i, P, vp, vp, ll, vp]
    L.dcell_ls_pls_reseed.argtypes = [vp, G, vp, vp, i, P, vp, vp, ll, ll, vp]
    cp = ctypes.c_char_p
    L.dcell_writer_create.argtypes = [cp, cp, i, ctypes.POINTER(vp)]
    L.dcell_writer_flush.argtypes = [vp]
    L.dcell_writer_destroy.argtypes = [vp]
    L.dcell_writer_grid.argtypes = [vp, cp, i, G, i, i, vp, vp]
    L.dcell_writer_grid_host.argtypes = [vp, cp, i, G, i, vp]
    L.dcell_writer_irregular_nodes.argtypes = [vp, cp, i, i, vp, vp, i, vp]
    L.dcell_writer_irregular_nodes_host.argtypes = [vp, cp, i, i, vp, i]
    L.dcell_writer_particles.argtypes = [vp, cp, i, vp, ll, i, vp]
    L.dcell_writer_particles_host.argtypes = [vp, cp, i, vp, ll]
    for name in ("dcell_writer_create", "dcell_writer_flush", "dcell_writer_destroy", "dcell_writer_grid",
                 "dcell_writer_grid_host", "dcell_writer_irregular_nodes", "dcell_writer_irregular_nodes_host",
                 "dcell_writer_particles", "dcell_writer_particles_host"):
        getattr(L, name).restype = i
    for name in ("dcell_sl_step", "dcell_irregular_nodes", "dcell_irregular_nodes_noalloc", "dcell_max_velocity",
                 "dcell_volume", "dcell_reinitialize", "dcell_velocity_box", "dcell_velocity_boxes",
                 "dcell_session_create", "dcell_session_destroy", "dcell_ls_advect_sl",
                 "dcell_ls_update_irregular_nodes", "dcell_ls_max_velocity", "dcell_ls_reinitialize",
                 "dcell_ls_advect_sl_rk2_half", "dcell_ls_advect_sl_rk2_full",
                 "dcell_tc_gemm_check", "dcell_wait_timeout_check",
                 "dcell_sl_adjoint", "dcell_ls_resident_set", "dcell_ls_resident_advect_and_reinit",
                 "dcell_ls_resident_get", "dcell_batch_plan", "dcell_batch_sl_step", "dcell_split_bf16",
                 "dcell_batch_sl_step_tc_split", "dcell_batch_tma_maps", "dcell_batch_sl_step_tc_split_tma",
                 "dcell_sl_step_tc_split", "dcell_sl_step_tc_split_planes", "dcell_pls_advect", "dcell_pls_correct", "dcell_pls_adjust_radii",
                 "dcell_pls_seed", "dcell_pls_reseed", "dcell_ls_pls_advect", "dcell_ls_pls_correct",
                 "dcell_ls_pls_adjust_radii", "dcell_ls_pls_seed", "dcell_ls_pls_reseed", "dcell_advect_mac",
                 "dcell_ls_advect_mac"):
        getattr(L, name).restype = i
    _LIB = L
    return L


def check(rc: int):
    if rc != OK:
        raise DcellError(rc, lib().dcell_last_error().decode(errors="replace"))


def exported_symbols():
    """Names the public header declares (for the load/export test)."""
    hdr = os.path.join(os.path.dirname(PKG), "include", "dcell_ls.h")
    import re
    return re.findall(r"^DCELL_API [^(]*?\b(dcell_\w+)\(", open(hdr).read(), flags=re.M)
