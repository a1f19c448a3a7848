"""LevelSetAdvectMAC / LevelSetAdvectMAC_3D (LevelSetMethod/AdvectMAC.c:18-111):
the first-order conservative upwind step on MAC faces.

The oracle restatement is pinned to the reference's own routine (compiled
from its source against oracle/shim/mac) through tests/golden/mac.npz and,
where the reference tree is present, live on more shapes; the CUDA kernel
(dcell_advect_mac), the host-buffer entry (dcell_ls_advect_mac) and the
drop-in (LevelSetAdvectMAC in dcell_b200/host/levelset_b200.c) must give the
reference's FP64 bits."""
import ctypes
import os

import numpy as np
import pytest

import oracle
from oracle import reference as R

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "mac.npz")


def golden_cases():
    z = np.load(GOLDEN)
    for c in range(int(z["ncases"])):
        phi = z[f"phi_{c}"].astype(np.float64)
        vel = [z[f"vel{a}_{c}"].astype(np.float64) for a in range(phi.ndim)]
        yield dict(phi=phi, u=vel[0], v=vel[1], w=vel[2] if phi.ndim == 3 else None,
                   out0=z[f"out0_{c}"].astype(np.float64), out=z[f"out_{c}"], origin=tuple(z[f"origin_{c}"]),
                   h=tuple(z[f"h_{c}"]), dt=float(z[f"dt_{c}"]))


def test_oracle_matches_reference_golden():
    for case in golden_cases():
        got = oracle.advect_mac(case["phi"], case["u"], case["v"], case["w"], case["dt"], case["h"], case["origin"],
                                out=case["out0"])
        assert got is not None
        assert np.array_equal(got, case["out"])
        # the updated range is exactly [max(p, 0), p + n - 1) per axis
        changed = got != case["out0"]
        shape, origin = case["phi"].shape, case["origin"]
        for ax in range(len(shape)):
            a = len(shape) - 1 - ax  # array axis of x, y(, z)
            n, p = shape[a], origin[ax]
            keep = [i for i in range(n) if not (max(p, 0) <= p + i < p + n - 1)]
            assert not changed.take(keep, axis=a).any()


@pytest.mark.skipif(not R.available(), reason="reference not compiled here (make -C oracle ref REF=<reference tree>)")
@pytest.mark.parametrize("shape,origin", [((7, 8, 9), (-2, -1, -4)), ((6, 5, 4), (-1, 0, -2)), ((4, 3, 5), (0, -2, 0)),
                                          ((9, 11), (-3, -2)), ((4, 3), (-2, 0)), ((3, 7), (0, -6))])
def test_oracle_matches_reference_live(shape, origin):
    rng = np.random.default_rng(abs(sum(shape) + 7 * sum(origin)))
    phi, u, v, w, out0 = (rng.standard_normal(shape) for _ in range(5))
    u[rng.random(shape) < 0.2] = 0.0
    h = (0.1, 0.2, 0.3)
    w = w if len(shape) == 3 else None
    a = oracle.advect_mac(phi, u, v, w, 0.01, h, origin, out=out0)
    b = R.advect_mac(phi, u, v, w, 0.01, h, origin, out=out0)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("shape,origin", [((5, 5), (1, 0)), ((5, 5), (0, 2)), ((5, 2), (0, 0)), ((2, 5), (0, 0)),
                                          ((4, 4, 4), (0, 0, 3)), ((2, 4, 4), (0, 0, 0))])
def test_oracle_refuses_grids_the_reference_reads_outside(shape, origin):
    """An updated axis with origin > 0 reads phi one cell before the grid
    (AdvectMAC.c:83); one with fewer than 3 points reads it at the range's
    last point (:84)."""
    z = np.zeros(shape)
    assert oracle.advect_mac(z, z, z, z if len(shape) == 3 else None, 0.1, 1.0, origin) is None


def test_oracle_known_answer_uniform_flow():
    """phi = a x (global x), u = c > 0 on every face, v = w = 0: every updated
    point moves by -dt c a / h.x (the extrapolation at x = 0 continues the
    line)."""
    a, c, hx, dt = 0.25, 1.5, 0.1, 0.01
    nz, ny, nx = 5, 6, 8
    x = np.arange(nx, dtype=np.float64)[None, None, :] + np.zeros((nz, ny, 1))
    phi = a * x
    u = np.full(phi.shape, c)
    zero = np.zeros(phi.shape)
    out = oracle.advect_mac(phi, u, zero, zero, dt, (hx, 0.2, 0.3), (0, 0, 0), out=np.full(phi.shape, 9.0))
    upd = out[:nz - 1, :ny - 1, :nx - 1]
    assert np.allclose(upd, phi[:nz - 1, :ny - 1, :nx - 1] - dt * c * a / hx, rtol=0, atol=1e-15)
    assert (out[nz - 1] == 9.0).all() and (out[:, ny - 1] == 9.0).all() and (out[:, :, nx - 1] == 9.0).all()


def test_c_abi_argument_errors():
    """dcell_advect_mac / dcell_ls_advect_mac reject bad arguments with status
    codes before any device work (runs without a GPU)."""
    from dcell_b200 import _lib
    L = _lib.lib()
    d = ctypes.c_void_p(64)  # never dereferenced: every call below fails or has nothing to do first
    e = ctypes.c_void_p(128)
    g3 = _lib.geom((6, 6, 6), 0.1)
    g2 = _lib.geom((6, 6), 0.1)

    def rc(g, dtype=_lib.F64, phi=d, u=d, v=d, w=d, dt=0.1, out=e):
        return L.dcell_advect_mac(ctypes.byref(g) if g is not None else None, dtype, phi, u, v, w, dt, out, None)
    assert rc(None) == _lib.ERR_ARG
    assert rc(g3, dtype=7) == _lib.ERR_ARG
    assert rc(g3, phi=None) == _lib.ERR_ARG
    assert rc(g3, w=None) == _lib.ERR_ARG           # 3D needs w
    assert rc(g3, out=d) == _lib.ERR_ARG            # out aliases phi
    assert rc(g3, dt=float("nan")) == _lib.ERR_NONFINITE
    assert rc(_lib.geom((6, 6, 6), 0.1, (0, 2, 0))) == _lib.ERR_UNSUPPORTED
    assert b"outside its grid" in L.dcell_last_error()
    assert rc(_lib.geom((6, 2), 0.1)) == _lib.ERR_UNSUPPORTED
    assert rc(_lib.geom((6, 6, 6), 0.1, (0, -9, 0))) == _lib.OK  # empty y range: nothing to do, no launch
    assert rc(g2, u=None, w=None) == _lib.ERR_ARG
    assert L.dcell_ls_advect_mac(None, ctypes.byref(g3), d, d, d, d, 0.1, _lib.F64, e) == _lib.ERR_ARG


# --------------------------------------------------------------------------- GPU
def _mac_gpu(case, dtype, torch):
    from dcell_b200 import levelset as L
    dev = "cuda"
    t = lambda a: torch.tensor(a, dtype=dtype, device=dev)  # noqa: E731
    w = t(case["w"]) if case["w"] is not None else None
    out = t(case["out0"])
    L.advect_mac(t(case["phi"]), t(case["u"]), t(case["v"]), w, case["dt"], case["h"], case["origin"], out=out)
    torch.cuda.synchronize()
    return out.double().cpu().numpy()


@pytest.mark.gpu
def test_gpu_fp64_gives_the_reference_bits():
    import torch
    for case in golden_cases():
        assert np.array_equal(_mac_gpu(case, torch.float64, torch), case["out"])


@pytest.mark.gpu
def test_gpu_fp32_within_tolerance():
    """FP32 arithmetic on the same (FP32-exact) inputs: |out - reference| <=
    1e-5 (values of order 1, one update of order 1)."""
    import torch
    for case in golden_cases():
        got = _mac_gpu(case, torch.float32, torch)
        assert float(np.abs(got - case["out"]).max()) <= 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("shape,origin", [((64, 48, 80), (-5, 0, -7)), ((96, 130), (-3, -1)), ((3, 3, 300), (0, 0, 0))])
def test_gpu_fp64_equals_oracle_larger(shape, origin):
    import torch

    from dcell_b200 import levelset as L
    rng = np.random.default_rng(3)
    phi, u, v, w, out0 = (rng.standard_normal(shape) for _ in range(5))
    w = w if len(shape) == 3 else None
    want = oracle.advect_mac(phi, u, v, w, 0.02, (0.1, 0.2, 0.3), origin, out=out0)
    T = lambda a: torch.tensor(a, device="cuda")  # noqa: E731
    out = T(out0)
    L.advect_mac(T(phi), T(u), T(v), T(w) if w is not None else None, 0.02, (0.1, 0.2, 0.3), origin, out=out)
    assert np.array_equal(out.cpu().numpy(), want)


@pytest.mark.gpu
@pytest.mark.parametrize("shape,origin", [((5, 5), (1, 0)), ((5, 2), (0, 0)), ((4, 4, 4), (0, 0, 3))])
def test_gpu_refuses_out_of_bounds_grids(shape, origin):
    import torch

    from dcell_b200 import _lib
    from dcell_b200 import levelset as L
    z = torch.zeros(shape, dtype=torch.float64, device="cuda")
    out = torch.full(shape, 3.0, dtype=torch.float64, device="cuda")
    with pytest.raises(_lib.DcellError) as e:
        L.advect_mac(z, z, z, z if len(shape) == 3 else None, 0.1, 1.0, origin, out=out)
    assert e.value.code == _lib.ERR_UNSUPPORTED
    assert bool((out == 3.0).all())


@pytest.mark.gpu
def test_gpu_empty_range_and_alias():
    import torch

    from dcell_b200 import _lib
    from dcell_b200 import levelset as L
    # origin so negative that no point has a global index in [0, p + n - 1)
    z = torch.ones((4, 4, 4), dtype=torch.float64, device="cuda")
    out = torch.full_like(z, 2.0)
    L.advect_mac(z, z, z, z, 0.1, 1.0, (-6, 0, 0), out=out)
    assert bool((out == 2.0).all())
    with pytest.raises(_lib.DcellError) as e:
        L.advect_mac(z, z, z, z, 0.1, 1.0, (0, 0, 0), out=z)
    assert e.value.code == _lib.ERR_ARG


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_host_buffer_entry(precision):
    from dcell_b200 import _lib
    Lb = _lib.lib()
    sess = ctypes.c_void_p()
    _lib.check(Lb.dcell_session_create(0, ctypes.byref(sess)))
    try:
        for case in golden_cases():
            out = case["out0"].copy()
            g = _lib.geom(case["phi"].shape, case["h"], case["origin"])
            arrs = [np.ascontiguousarray(case[k]) for k in ("phi", "u", "v")]
            w = np.ascontiguousarray(case["w"]) if case["w"] is not None else None
            p = lambda a: a.ctypes.data_as(ctypes.c_void_p) if a is not None else None  # noqa: E731
            _lib.check(Lb.dcell_ls_advect_mac(sess, ctypes.byref(g), p(arrs[0]), p(arrs[1]), p(arrs[2]), p(w),
                                              case["dt"], _lib.F64 if precision == "f64" else _lib.F32, p(out)))
            if precision == "f64":
                assert np.array_equal(out, case["out"])
            else:
                assert float(np.abs(out - case["out"]).max()) <= 1e-5
    finally:
        Lb.dcell_session_destroy(sess)


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(R.DROPIN_PATH), reason="drop-in library not built (make -C oracle dropin REF=<reference tree>)")
def test_dropin_levelset_advect_mac():
    """The B200 LevelSetAdvectMAC / _3D in the reference's own C host, called
    as FluidField/tests/testSource.c calls the originals, gives the
    reference's bits."""
    L = ctypes.CDLL(R.DROPIN_PATH)
    vp = ctypes.c_void_p
    L.ddrop_advect_mac.argtypes = [vp, vp, vp, vp, vp, vp, vp, ctypes.c_double, vp]
    p = lambda a: a.ctypes.data_as(vp) if a is not None else None  # noqa: E731
    for case in golden_cases():
        phi = case["phi"]
        shape = phi.shape if phi.ndim == 3 else (1,) + phi.shape
        n = np.array([shape[2], shape[1], shape[0]], dtype=np.int32)
        o = tuple(case["origin"]) + (0,) * (3 - len(case["origin"]))
        pp = np.array([o[0], o[1], o[2] if phi.ndim == 3 else 0], dtype=np.int32)
        h = np.array(case["h"], dtype=np.float64)
        arrs = [np.ascontiguousarray(case[k]) for k in ("phi", "u", "v")]
        w = np.ascontiguousarray(case["w"]) if case["w"] is not None else None
        out = case["out0"].copy()
        assert L.ddrop_advect_mac(p(n), p(pp), p(h), p(arrs[0]), p(arrs[1]), p(arrs[2]), p(w), case["dt"], p(out)) == 0
        assert np.array_equal(out, case["out"])
