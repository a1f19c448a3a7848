"""The allocation-free irregular-node entry point (dcell_irregular_nodes_noalloc).

It serves callers that cannot allocate device memory (their device memory is
owned by another allocator or a fixed pool, or they must not risk the device
synchronisation a cudaMalloc can cause): its scan scratch is a static array
inside the library.  This file is collected last on purpose so that a run
stopping at its first failure has run every other test before it.
"""
import ctypes

import numpy as np
import pytest
import torch

from dcell_b200 import _lib
from dcell_b200 import levelset as L

pytestmark = pytest.mark.gpu


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


def _noalloc(g, phi, band, cap, with_surface):
    geom = _lib.geom(tuple(phi.shape), float(g["h"]), tuple(g["origin"]))
    raw = torch.empty(cap * _lib.NODE_DTYPE.itemsize, dtype=torch.uint8, device=phi.device)
    count = torch.zeros(1, dtype=torch.int32, device=phi.device)
    flags = torch.zeros(1, dtype=torch.int32, device=phi.device)
    _lib.check(_lib.lib().dcell_irregular_nodes_noalloc(
        ctypes.byref(geom), _lib.F64 if phi.dtype == torch.float64 else _lib.F32, _vp(phi), _vp(band),
        int(band.shape[0]), with_surface, _vp(raw), cap, _vp(count), _vp(flags),
        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    assert int(flags.item()) == 0
    n = int(count.item())
    return n, raw[: n * _lib.NODE_DTYPE.itemsize].cpu().numpy()


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("case", ["sl3d_linear", "sl2d_linear"])
def test_noalloc_matches_scratch_entry_point_twice(golden, cuda, case, dtype):
    g = golden(case)
    phi = torch.as_tensor(g["phi"], dtype=dtype, device=cuda)
    band = torch.as_tensor(g["band"], dtype=torch.int32, device=cuda)
    raw, count = L.irregular_nodes(phi, float(g["h"]), band, tuple(g["origin"]), with_surface=True)
    torch.cuda.synchronize()
    n_ref = int(count.item())
    ref = L.nodes_to_rows(L.nodes_to_numpy(raw, n_ref))
    cap = raw.numel() // _lib.NODE_DTYPE.itemsize
    for _ in range(2):  # two calls in a row share (and reuse) the static scratch
        n, got = _noalloc(g, phi, band, cap, 1)
        assert n == n_ref
        rows = L.nodes_to_rows(np.frombuffer(got.tobytes(), dtype=_lib.NODE_DTYPE))
        assert np.array_equal(rows[:, :8], ref[:, :8])
        assert np.allclose(rows[:, 8:], ref[:, 8:], rtol=1e-12, atol=1e-12)


def test_noalloc_rejects_band_beyond_maximum(cuda):
    geom = _lib.geom((8, 8, 8), 0.1)
    dummy = torch.zeros(16, dtype=torch.int32, device=cuda)
    rc = _lib.lib().dcell_irregular_nodes_noalloc(ctypes.byref(geom), _lib.F32, _vp(dummy), _vp(dummy),
                                                  (1 << 20) + 1, 0, _vp(dummy), 1, _vp(dummy), None, None)
    assert rc == _lib.ERR_ARG
    assert b"maximum" in _lib.lib().dcell_last_error()
