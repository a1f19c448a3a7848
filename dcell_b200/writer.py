"""Output in the reference's file formats, written asynchronously from device
(or host) memory -- GridWrite (Common/Serialize.c:23-55),
LevelSetWriteIrregularNodeList (LevelSetMethod/IrregularNodes.c:145-246) and
the particle ArrayWrite (Common/Array.c:133-150).

    w = Writer("out")                 # grids and node lists in out/, particles in $PETSC_TMP or /tmp
    w.grid("phi", t, ls.phi, h, origin)        # snapshot on the current stream, written by a thread
    w.grid("vel", t, velgrid, h, origin, dof=3)
    w.irregular_nodes("phi", t, raw, count, dim=3)
    w.particles("particles", t, ls.pls.live)
    w.flush()                         # wait; raises the first error

Device tensors are snapshotted into device staging memory on the current
stream and copied to pinned memory on the writer's own stream, so the caller
may overwrite them right after the call returns.  ``read_real64`` reads a
grid file back the way the reference's own reader does
(Visualization/DCellVTK.py: two int32 header words, then big-endian FP64).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np
import torch

from . import _lib
from . import levelset as L
from ._lib import check, geom, lib


class Writer:
    def __init__(self, directory: str, tmpdir: str | None = None, device: int = 0):
        os.makedirs(directory, exist_ok=True)
        self._w = ctypes.c_void_p()
        check(lib().dcell_writer_create(directory.encode(), tmpdir.encode() if tmpdir else None, int(device),
                                        ctypes.byref(self._w)))

    def grid(self, name: str, t: int, data, h, origin=(0, 0, 0), dof: int = 1):
        """A level set's grid: data (nz, ny, nx) or (ny, nx) for dof 1, with a
        trailing axis of dof values otherwise (a velocity grid)."""
        shape = tuple(data.shape[:-1]) if dof > 1 else tuple(data.shape)
        if dof > 1 and data.shape[-1] != dof:
            raise ValueError("the last axis must hold the dof values")
        g = geom(shape, h, origin)
        if isinstance(data, torch.Tensor) and data.is_cuda:
            L._require_cuda(data)
            check(lib().dcell_writer_grid(self._w, name.encode(), int(t), ctypes.byref(g), dof, L._dtype_code(data),
                                          L._ptr(data), L._stream()))
        else:
            a = np.ascontiguousarray(np.asarray(data.cpu() if isinstance(data, torch.Tensor) else data,
                                                dtype=np.float64))
            check(lib().dcell_writer_grid_host(self._w, name.encode(), int(t), ctypes.byref(g), dof,
                                               a.ctypes.data_as(ctypes.c_void_p)))
            self._keep = a

    def irregular_nodes(self, name: str, idx: int, raw, count, dim: int = 3):
        """A node list as irregular_nodes returns it (raw device buffer and a
        device count), or a host NODE_DTYPE array with count = its length."""
        if isinstance(raw, torch.Tensor) and raw.is_cuda:
            cap = raw.numel() // _lib.NODE_DTYPE.itemsize
            check(lib().dcell_writer_irregular_nodes(self._w, name.encode(), int(idx), int(dim), L._ptr(raw),
                                                     L._ptr(count), cap, L._stream()))
        else:
            a = np.ascontiguousarray(raw, dtype=_lib.NODE_DTYPE)
            check(lib().dcell_writer_irregular_nodes_host(self._w, name.encode(), int(idx), int(dim),
                                                          a.ctypes.data_as(ctypes.c_void_p), int(count)))

    def particles(self, name: str, t: int, parts):
        if isinstance(parts, torch.Tensor) and parts.is_cuda:
            L._require_cuda(parts)
            check(lib().dcell_writer_particles(self._w, name.encode(), int(t), L._ptr(parts), int(parts.shape[0]),
                                               L._dtype_code(parts), L._stream()))
        else:
            a = np.ascontiguousarray(parts, dtype=np.float64).reshape(-1, 4)
            check(lib().dcell_writer_particles_host(self._w, name.encode(), int(t),
                                                    a.ctypes.data_as(ctypes.c_void_p), a.shape[0]))

    def flush(self):
        check(lib().dcell_writer_flush(self._w))

    def close(self):
        if self._w:
            rc = lib().dcell_writer_destroy(self._w)
            self._w = None
            check(rc)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


FILE_COUNT_START = 10000


def read_real64(path: str):
    """(class id, length, values) of a grid file: two int32 header words, then
    big-endian FP64 (the reference's reader, Visualization/DCellVTK.py)."""
    with open(path, "rb") as f:
        head = np.frombuffer(f.read(8), dtype=">i4")
        vals = np.frombuffer(f.read(), dtype=">f8")
    return int(head[0]), int(head[1]), vals
