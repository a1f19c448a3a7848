"""GPU parity of the semi-Lagrangian step against the reference and the oracle.

* FP64 linear/Euler (the reference's own AdvectSL arithmetic) must reproduce
  the reference's outputs bit for bit (golden fixtures from its compiled C).
* FP32 paths: within FP32 rounding of the FP64 results.
* Cubic paths: against the oracle's FP64 Catmull-Rom restatement.
* Split-BF16 tensor-core path: max |error| <= 1e-5 (physical units) in the
  |phi| < 3h band on a smooth signed distance, vs the FP64 oracle.
"""
import numpy as np
import pytest
import torch

import oracle
from dcell_b200 import _lib, fields
from dcell_b200 import levelset as L

pytestmark = pytest.mark.gpu


def _t(a, dev, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=dev)


def _run(g, dev, dtype, interp="linear", backtrace="euler", vel_key="vel", dt=None, phi_in=None):
    phi0 = _t(g["phi0"], dev, dtype)
    vel = _t(g[vel_key], dev, dtype)
    band = torch.as_tensor(g["band"], dtype=torch.int32, device=dev)
    out = phi0.clone() if phi_in is None else _t(phi_in, dev, dtype)
    flags = torch.zeros(1, dtype=torch.int32, device=dev)
    L.sl_step(phi0, vel, float(g["dt"]) if dt is None else dt, float(g["h"]), tuple(g["origin"]), band=band,
              interp=interp, backtrace=backtrace, out=out, flags=flags)
    torch.cuda.synchronize()
    assert int(flags.item()) == 0
    return out.cpu().numpy().astype(np.float64)


@pytest.mark.parametrize("case", ["sl3d_linear", "sl2d_linear"])
def test_linear_fp64_bit_exact_vs_reference(golden, cuda, case):
    g = golden(case)
    out = _run(g, cuda, torch.float64)
    assert np.array_equal(out, g["phi"])


@pytest.mark.parametrize("case", ["sl3d_linear", "sl2d_linear"])
def test_linear_fp32_vs_reference(golden, cuda, case):
    g = golden(case)
    out = _run(g, cuda, torch.float32)
    scale = np.abs(g["phi"]).max()
    assert np.abs(out - g["phi"]).max() <= 4e-7 * scale


def _random_case(shape, cfl, dev, seed=3):
    """Smooth-ish FP32 phi and a random MAC velocity whose largest component
    moves cfl cells per unit step (dt = h = 1)."""
    g = torch.Generator(device="cpu").manual_seed(seed)
    nz, ny, nx = shape
    z, y, x = torch.meshgrid(torch.arange(nz), torch.arange(ny), torch.arange(nx), indexing="ij")
    phi = (torch.sin(0.37 * x) + torch.cos(0.29 * y) * torch.sin(0.41 * z) + 0.1 * torch.rand(shape, generator=g))
    vel = (torch.rand(shape + (3,), generator=g) * 2 - 1) * cfl
    return phi.float().to(dev).contiguous(), vel.float().to(dev).contiguous()


@pytest.mark.parametrize("interp", ["linear", "cubic_plain", "cubic_separable"])
@pytest.mark.parametrize("backtrace", ["euler", "midpoint"])
@pytest.mark.parametrize("shape,cfl", [((9, 20, 36), 0.5), ((40, 24, 64), 0.9), ((24, 16, 44), 3.0), ((3, 5, 8), 0.5),
                                       ((70, 9, 96), 1.7), ((12, 8, 40), 0.5)])
def test_fp32_staged_form_equals_gather_form(cuda, interp, backtrace, shape, cfl):
    """Dense FP32 steps: the shared-memory-staged forms (TMA z-march for the
    trilinear step, TMA bricks for the two cubic forms) give the same bits as
    their global-gather forms -- on partial tiles and bricks, grids smaller
    than a box, and departures beyond the staged boxes at CFL 1.7 and 3 (the
    warps' global path).  The linear gather form also equals the band form
    run on a band that lists every point."""
    phi, vel = _random_case(shape, cfl, cuda)
    staged = L.sl_step(phi, vel, 1.0, 1.0, interp=interp, backtrace=backtrace)
    gathered = L.sl_step(phi, vel, 1.0, 1.0, interp=interp + "_gather", backtrace=backtrace,
                         out=torch.full_like(phi, float("nan")))
    torch.cuda.synchronize()
    assert torch.equal(staged, gathered)
    if interp == "linear":
        band = fields.band_of(torch.zeros_like(phi), 1.0, margin=0).to(cuda)
        assert band.shape[0] == phi.numel()
        banded = L.sl_step(phi, vel, 1.0, 1.0, band=band, interp=interp, backtrace=backtrace,
                           out=torch.full_like(phi, float("nan")))
        torch.cuda.synchronize()
        assert torch.equal(staged, banded)


@pytest.mark.parametrize("rows,per_warp", [(8, 1), (8, 2), (16, 2), (16, 4)])
@pytest.mark.parametrize("backtrace", ["euler", "midpoint"])
def test_linear_march_shapes_equal_gather_form(cuda, backtrace, rows, per_warp, monkeypatch):
    """Every tile shape of the FP32 trilinear z-march (tile rows, rows per
    consumer warp) gives the gather form's bits: partial tiles in x and y,
    and departures beyond the staged box (CFL 3)."""
    monkeypatch.setenv("DCELL_LIN_TILE_ROWS", str(rows))
    monkeypatch.setenv("DCELL_LIN_ROWS_PER_WARP", str(per_warp))
    for shape, cfl in (((40, 24, 64), 0.9), ((21, 37, 44), 3.0)):
        phi, vel = _random_case(shape, cfl, cuda)
        staged = L.sl_step(phi, vel, 1.0, 1.0, interp="linear", backtrace=backtrace)
        gathered = L.sl_step(phi, vel, 1.0, 1.0, interp="linear_gather", backtrace=backtrace,
                             out=torch.full_like(phi, float("nan")))
        torch.cuda.synchronize()
        assert torch.equal(staged, gathered), (shape, cfl)


@pytest.mark.parametrize("backtrace", ["euler", "midpoint"])
def test_split_state_plane_ranges_equal_the_full_step(cuda, backtrace):
    """dcell_sl_step_tc_split_planes over brick-aligned plane ranges (the
    overlapped z-slab form: interior first, then the planes next to the
    halos, here on one GPU) gives the full dense step's phi and split words
    bit for bit, and writes nothing outside its ranges."""
    from dcell_b200 import dist as D
    phi, vel = _random_case((43, 24, 64), 0.9, cuda, seed=5)
    spl = L.split_bf16(phi)
    full, fspl = L.sl_step_tc_split(spl, vel, 1.0, 1.0, backtrace=backtrace, out_split=torch.empty_like(spl))
    out = torch.full_like(phi, float("nan"))
    ospl = torch.full_like(spl, -1)
    L.sl_step_tc_split_planes(spl, vel, 1.0, 1.0, 8, 24, out, ospl, backtrace=backtrace)
    torch.cuda.synchronize()
    assert torch.equal(out[8:24], full[8:24]) and torch.equal(ospl[8:24], fspl[8:24])
    assert bool(out[:8].isnan().all()) and bool(out[24:].isnan().all()) and bool((ospl[24:] == -1).all())
    L.sl_step_tc_split_planes(spl, vel, 1.0, 1.0, 0, 8, out, ospl, backtrace=backtrace)
    L.sl_step_tc_split_planes(spl, vel, 1.0, 1.0, 24, 43, out, ospl, backtrace=backtrace)
    torch.cuda.synchronize()
    assert torch.equal(out, full) and torch.equal(ospl, fspl)
    # the slab stepper over one rank's ranges (no neighbours: no exchange)
    st = D.SplitStateSlab(phi.shape, cuda, backtrace)
    slab = D.Slab(phi.shape[0], 1, 0, 3)
    inner, edges = slab.step_ranges(3, D.SplitStateSlab.align)
    y = torch.empty_like(spl)
    for a, b in ([inner] if inner else []) + edges:
        st(spl, vel, 1.0, 1.0, (0, 0, 0), a, b, y)
    torch.cuda.synchronize()
    assert torch.equal(st.phi, full) and torch.equal(y, fspl)


@pytest.mark.parametrize("backtrace", ["euler", "midpoint"])
def test_linear_fp32_dense_vs_fp64(cuda, backtrace):
    """Dense 64^3 sphere in the deformation field (FP32-representable
    inputs): the FP32 step within FP32 rounding of the FP64 reference-order
    step (Euler: the reference's own arithmetic; midpoint: its FP64 form)."""
    N = 64
    h, phi, vel, dt = _sphere_case(N, cuda)
    p32, v32 = phi.float().contiguous(), vel.float().contiguous()
    ref = L.sl_step(p32.double(), v32.double(), dt, h, interp="linear", backtrace=backtrace)
    out = L.sl_step(p32, v32, dt, h, interp="linear", backtrace=backtrace).double()
    assert float((out - ref).abs().max()) <= 4e-7 * float(ref.abs().max())


def test_rk2_half_full_fp64_bit_exact(golden, cuda):
    """AdvectRK2.c: HalfStep(dt/2, u^n) then FullStep(dt, u^{n+1/2}) from the same phi0."""
    g = golden("sl3d_rk2")
    dt = float(g["dt"])
    half = _run(g, cuda, torch.float64, dt=dt / 2)
    assert np.array_equal(half, g["phi_half"])
    full = _run(g, cuda, torch.float64, vel_key="vel_half", dt=dt, phi_in=half)
    assert np.array_equal(full, g["phi_full"])


@pytest.mark.parametrize("backtrace", ["euler", "midpoint"])
@pytest.mark.parametrize("case", ["sl3d_linear", "sl2d_linear"])
def test_cubic_fp64_vs_oracle(golden, cuda, case, backtrace):
    g = golden(case)
    ref = oracle.sl_step(g["phi0"], g["vel"], float(g["dt"]), float(g["h"]), origin=g["origin"], band=g["band"],
                         interp="cubic", backtrace=backtrace, phi=g["phi0"])
    for interp in ("cubic_plain", "cubic_separable"):
        out = _run(g, cuda, torch.float64, interp=interp, backtrace=backtrace)
        assert np.abs(out - ref).max() < 1e-12, interp


def test_linear_midpoint_fp64_vs_oracle(golden, cuda):
    g = golden("sl3d_linear")
    ref = oracle.sl_step(g["phi0"], g["vel"], float(g["dt"]), float(g["h"]), origin=g["origin"], band=g["band"],
                         interp="linear", backtrace="midpoint", phi=g["phi0"])
    out = _run(g, cuda, torch.float64, backtrace="midpoint")
    assert np.abs(out - ref).max() < 1e-12


@pytest.mark.parametrize("interp", ["cubic_plain", "cubic_separable", "cubic_tc"])
def test_cubic_fp32_vs_oracle_golden_case(golden, cuda, interp):
    """Cell-unit signed distance (|phi| up to ~12): FP32 relative accuracy."""
    g = golden("sl3d_linear")
    ref = oracle.sl_step(g["phi0"], g["vel"], float(g["dt"]), float(g["h"]), origin=g["origin"], band=g["band"],
                         interp="cubic", phi=g["phi0"])
    out = _run(g, cuda, torch.float32, interp=interp)
    tol = 2e-5 if interp == "cubic_tc" else 4e-6
    assert np.abs(out - ref).max() <= tol * np.abs(ref).max(), np.abs(out - ref).max()


def _sphere_case(N, dev):
    h = 1.0 / N
    phi = fields.sphere_sdf(N, device=dev)
    vel = fields.deformation_velocity(N, device=dev)
    dt = fields.cfl_dt((2.0, 1.0, 1.0), h) * fields.deformation_time_factor(0.37)
    return h, phi, vel, dt


@pytest.mark.parametrize("backtrace", ["euler", "midpoint"])
def test_tensor_core_dense_error_budget(cuda, backtrace):
    """Dense 64^3 sphere in the deformation field: split-BF16 TC and plain FP32
    vs the FP64 GPU oracle (itself checked against the CPU oracle on a sample)."""
    N = 64
    h, phi, vel, dt = _sphere_case(N, cuda)
    ref = L.sl_step(phi, vel, dt, h, interp="cubic_plain", backtrace=backtrace)
    # FP64 GPU oracle == CPU oracle
    cpu = oracle.sl_step(phi.cpu().numpy(), vel.cpu().numpy(), dt, h, interp="cubic", backtrace=backtrace)
    assert np.abs(ref.cpu().numpy() - cpu).max() < 1e-13
    band = (ref.abs() < 3 * h)
    p32, v32 = phi.float().contiguous(), vel.float().contiguous()
    for interp, tol in (("cubic_tc", 1e-5), ("cubic_plain", 1e-6), ("cubic_separable", 1e-6)):
        out = L.sl_step(p32, v32, dt, h, interp=interp, backtrace=backtrace).double()
        err = (out - ref).abs()
        assert float(err[band].max()) <= tol, (interp, float(err[band].max()))
        assert float(err.max()) <= 10 * tol, (interp, float(err.max()))


def test_tensor_core_band_mode_matches_dense(cuda):
    N = 48
    h, phi, vel, dt = _sphere_case(N, cuda)
    p32, v32 = phi.float().contiguous(), vel.float().contiguous()
    dense = L.sl_step(p32, v32, dt, h, interp="cubic_tc")
    band = fields.band_of(phi, 6 * h).to(cuda)
    banded = L.sl_step(p32, v32, dt, h, band=band, interp="cubic_tc", out=p32.clone())
    sel = torch.zeros_like(phi, dtype=torch.bool)
    sel[band[:, 2].long(), band[:, 1].long(), band[:, 0].long()] = True
    assert torch.equal(banded[sel], dense[sel])
    assert torch.equal(banded[~sel], p32[~sel])


def test_tc_gemm_layout(cuda):
    """The tensor-core operand layouts: D = bf16(A) M^T against a host product."""
    rng = np.random.default_rng(3)
    A = rng.normal(size=(128, 64)).astype(np.float32)
    Ab = torch.as_tensor(A).to(torch.bfloat16).float().numpy().astype(np.float64)
    M = oracle.catmull_rom_operator(3)
    a = torch.as_tensor(A, device=cuda)
    d = torch.zeros((128, 64), dtype=torch.float32, device=cuda)
    flags = torch.zeros(1, dtype=torch.int32, device=cuda)
    import ctypes
    _lib.check(_lib.lib().dcell_tc_gemm_check(ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(d.data_ptr()),
                                              ctypes.c_void_p(flags.data_ptr()),
                                              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    assert int(flags.item()) == 0
    expect = Ab @ M.T
    assert np.abs(d.cpu().numpy() - expect).max() < 1e-4 * np.abs(expect).max()


def test_bounded_waits_give_up_and_the_context_survives(cuda):
    """Failure detection without a fault: both bounded mbarrier waits of the
    tensor-core kernels, waiting on a phase that nothing completes, give up
    within their limits and say so; the context then still runs a
    tensor-core step."""
    import ctypes
    import time
    res = torch.full((1,), -1, dtype=torch.int32, device=cuda)
    t0 = time.perf_counter()
    _lib.check(_lib.lib().dcell_wait_timeout_check(ctypes.c_void_p(res.data_ptr()),
                                                   ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    took = time.perf_counter() - t0
    assert int(res.item()) == 3
    assert took < 30.0
    N = 24
    phi = fields.sphere_sdf(N, device=cuda).float().contiguous()
    vel = fields.deformation_velocity(N, device=cuda).float().contiguous()
    out, _ = L.sl_step_tc_split(L.split_bf16(phi), vel, 0.25 / N, 1.0 / N)
    torch.cuda.synchronize()
    assert bool(torch.isfinite(out).all())


def test_departure_outside_grid_is_flagged(cuda):
    """Band points whose departure leaves the grid raise the flag; a dense
    step treats the grid edge as the domain boundary and does not."""
    N = 16
    phi = torch.zeros((N, N, N), dtype=torch.float32, device=cuda)
    vel = torch.full((N, N, N, 3), 4.0, dtype=torch.float32, device=cuda)
    flags = torch.zeros(1, dtype=torch.int32, device=cuda)
    band = torch.tensor([[8, 8, 8], [2, 3, 2]], dtype=torch.int32, device=cuda)
    inner = torch.tensor([[8, 8, 8]], dtype=torch.int32, device=cuda)
    for interp in ("linear", "cubic_plain", "cubic_tc"):
        flags.zero_()
        L.sl_step(phi, vel, 1.0, 1.0, band=band, interp=interp, flags=flags)
        torch.cuda.synchronize()
        assert int(flags.item()) & _lib.FLAG_DEPARTURE_CLAMPED, interp
        flags.zero_()
        L.sl_step(phi, vel, 1.0, 1.0, band=inner, interp=interp, flags=flags)
        L.sl_step(phi, vel, 1.0, 1.0, interp=interp, flags=flags)
        torch.cuda.synchronize()
        assert int(flags.item()) == 0, interp


def test_zero_velocity_is_identity(cuda):
    N = 24
    phi = fields.sphere_sdf(N, device=cuda).float()
    vel = torch.zeros((N, N, N, 3), dtype=torch.float32, device=cuda)
    for interp in ("linear", "cubic_plain", "cubic_separable", "cubic_tc"):
        out = L.sl_step(phi, vel, 0.1, 1.0 / N, interp=interp)
        tol = 0 if interp != "cubic_tc" else 1e-7
        assert float((out - phi).abs().max()) <= tol, interp


def test_integer_shift_is_exact_translation(cuda):
    """u = 1 cell/step along x: departure = X - 1 exactly (fraction 0)."""
    N = 20
    phi = fields.sphere_sdf(N, device=cuda).float()
    vel = torch.zeros((N, N, N, 3), dtype=torch.float32, device=cuda)
    vel[..., 0] = 1.0
    for interp in ("linear", "cubic_plain", "cubic_separable", "cubic_tc"):
        out = L.sl_step(phi, vel, 1.0 / N, 1.0 / N, interp=interp)
        tol = 0 if interp != "cubic_tc" else 1e-7
        assert float((out[:, :, 1:] - phi[:, :, :-1]).abs().max()) <= tol, interp


def test_split_bf16_words(cuda):
    x = torch.randn(4, 8, 16, device=cuda) * torch.logspace(-6, 2, 16, device=cuda)
    w = L.split_bf16(x.contiguous())
    u = w.view(torch.int32).cpu().numpy().astype(np.uint32)
    hi = (u & 0xFFFF).astype(np.uint32) << 16
    lo = (u >> 16).astype(np.uint32) << 16
    v = hi.view(np.float32).astype(np.float64) + lo.view(np.float32).astype(np.float64)
    ref = x.double().cpu().numpy()
    assert np.all(np.abs(v - ref) <= 2.0 ** -16 * np.abs(ref))


@pytest.mark.parametrize("backtrace", ["euler", "midpoint"])
def test_tc_split_state_error_budget(cuda, backtrace):
    """Split-state TC step: <= 1e-5 in the |phi| < 3h band vs the FP64 oracle."""
    N = 64
    h, phi, vel, dt = _sphere_case(N, cuda)
    ref = L.sl_step(phi, vel, dt, h, interp="cubic_plain", backtrace=backtrace)
    p32, v32 = phi.float().contiguous(), vel.float().contiguous()
    out, spl = L.sl_step_tc_split(L.split_bf16(p32), v32, dt, h, backtrace=backtrace,
                                  out_split=torch.empty((N, N, N), dtype=torch.int32, device=cuda))
    band = ref.abs() < 3 * h
    err = (out.double() - ref).abs()
    assert float(err[band].max()) <= 1e-5, float(err[band].max())
    assert float(err.max()) <= 1e-4, float(err.max())
    assert torch.equal(spl, L.split_bf16(out))  # the written split is the next step's input


def test_tc_split_band_mode_and_multistep(cuda):
    N = 48
    h, phi, vel, dt = _sphere_case(N, cuda)
    p32, v32 = phi.float().contiguous(), vel.float().contiguous()
    band = fields.band_of(phi, 6 * h).to(cuda)
    dense, _ = L.sl_step_tc_split(L.split_bf16(p32), v32, dt, h)
    banded, _ = L.sl_step_tc_split(L.split_bf16(p32), v32, dt, h, band=band, out=p32.clone())
    sel = torch.zeros_like(phi, dtype=torch.bool)
    sel[band[:, 2].long(), band[:, 1].long(), band[:, 0].long()] = True
    assert torch.equal(banded[sel], dense[sel])
    # 10 steps split-state vs 10 FP64 steps
    a, s = p32, L.split_bf16(p32)
    ref = phi.clone()
    for k in range(10):
        a, s = L.sl_step_tc_split(s, v32, dt, h, out_split=torch.empty_like(s))
        ref = L.sl_step(ref, vel, dt, h, interp="cubic_plain", backtrace="midpoint")
    err = (a.double() - ref).abs()[ref.abs() < 3 * h]
    assert float(err.max()) <= 1e-5, float(err.max())


@pytest.mark.parametrize("shape", [(40, 48, 64), (37, 45, 68), (12, 8, 40), (20, 8, 40)])
@pytest.mark.parametrize("cfl_scale", [1.0, 3.0])
def test_tc_brick_path_equals_gather_path(cuda, cfl_scale, shape):
    """Dense split-state steps on grids with nx % 4 == 0 run the TMA-staged
    brick kernel; a band listing every point runs the global-gather kernel.
    Both must give the same bits (3x the CFL exercises the brick fallbacks;
    the odd shapes end in partial bricks on every axis, the smallest are one
    brick deep, so a CTA's first step is also its last brick's)."""
    nz, ny, nx = shape
    h = 1.0 / 64
    phi = fields.sphere_sdf(72, device=cuda)[:nz, :ny, :nx].contiguous().float()
    vel = fields.deformation_velocity(72, device=cuda)[:nz, :ny, :nx].contiguous().float()
    dt = cfl_scale * fields.cfl_dt((2.0, 1.0, 1.0), h)
    spl = L.split_bf16(phi)
    for bt in ("midpoint", "euler"):
        dense, dspl = L.sl_step_tc_split(spl, vel, dt, h, backtrace=bt, out_split=torch.empty_like(spl))
        band = fields.band_of(torch.zeros_like(phi), 1.0, margin=0).to(cuda)  # every point, x fastest
        assert band.shape[0] == nx * ny * nz
        banded, bspl = L.sl_step_tc_split(spl, vel, dt, h, band=band, backtrace=bt, out=torch.zeros_like(phi),
                                          out_split=torch.zeros_like(spl))
        torch.cuda.synchronize()
        assert torch.equal(dense, banded), float((dense - banded).abs().max())
        assert torch.equal(dspl, bspl)


@pytest.mark.gpu
def test_host_buffer_rk2_half_full_equal_reference(golden, cuda):
    """dcell_ls_advect_sl_rk2_half / _full (AdvectRK2.c:5-26) on host FP64
    arrays: the half step copies phi into phi0, and phi and the irregular-node
    list of each substep equal the reference's (golden)."""
    import ctypes
    g = golden("sl3d_rk2")
    Lb = _lib.lib()
    sess = ctypes.c_void_p()
    _lib.check(Lb.dcell_session_create(0, ctypes.byref(sess)))
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    try:
        geo = _lib.geom(g["phi0"].shape, float(g["h"]), tuple(int(v) for v in g["origin"]))
        phi = np.ascontiguousarray(g["phi0"], dtype=np.float64).copy()
        phi0 = np.zeros_like(phi)
        band = np.ascontiguousarray(g["band"], dtype=np.int32)
        cap = 10 * len(band)
        nodes = np.zeros(cap, dtype=_lib.NODE_DTYPE)
        count = ctypes.c_int()
        dt = float(g["dt"])
        for step, (vel, tau, want_phi, want_nodes) in enumerate(
                [(g["vel"], dt / 2, g["phi_half"], g["nodes_half"]), (g["vel_half"], dt, g["phi_full"], g["nodes_full"])]):
            v = np.ascontiguousarray(vel, dtype=np.float64)
            fn = Lb.dcell_ls_advect_sl_rk2_half if step == 0 else Lb.dcell_ls_advect_sl_rk2_full
            _lib.check(fn(sess, ctypes.byref(geo), p(phi0), p(v), p(band), len(band), tau, _lib.LINEAR, _lib.EULER,
                          _lib.F64, p(phi), 0, p(nodes), cap, ctypes.byref(count)))
            if step == 0:
                assert np.array_equal(phi0, g["phi0"])  # GridCopy(phi, phi0) before the half step
            assert np.array_equal(phi, want_phi)
            rows = L.nodes_to_rows(nodes[:count.value])
            assert rows.shape == want_nodes.shape
            assert np.array_equal(rows[:, :8], want_nodes[:, :8])
            assert np.abs(rows[:, 8:14] - want_nodes[:, 8:14]).max() < 1e-11
    finally:
        Lb.dcell_session_destroy(sess)


@pytest.mark.gpu
@pytest.mark.parametrize("speed", [1.0, 40.0])
def test_host_buffer_tc_step_pipelined_equals_device_step(cuda, speed):
    """dcell_ls_advect_sl (FP32 tensor-core, dense) on host FP64 arrays is
    stepped slab by slab while the inputs are still going up; its result
    equals the device-resident split-state step bit for bit -- also when the
    velocity is too fast for the staged halo (speed 40: every slab defers to
    the full-grid step)."""
    import ctypes

    N, nz = 64, 96
    h = 1.0 / N
    ramp = torch.linspace(-0.3, 0.3, nz, device=cuda, dtype=torch.float64)[:, None, None].expand(nz, N, N)
    phi = (ramp + torch.rand((nz, N, N), device=cuda, dtype=torch.float64) * 0.01).contiguous()
    vel = (torch.rand((nz, N, N, 3), device=cuda, dtype=torch.float64) - 0.5) * speed
    dt = 0.4 * h
    want = L.sl_step_tc_split(L.split_bf16(phi.float().contiguous()), vel.float().contiguous(), dt, h,
                              backtrace="midpoint")[0]
    Lb = _lib.lib()
    sess = ctypes.c_void_p()
    _lib.check(Lb.dcell_session_create(0, ctypes.byref(sess)))
    try:
        p0 = phi.cpu().pin_memory()
        v0 = vel.cpu().pin_memory()
        out = torch.empty_like(p0).pin_memory()
        g = _lib.geom(tuple(phi.shape), h)
        for _ in range(2):  # twice: buffers and streams reused
            _lib.check(Lb.dcell_ls_advect_sl(sess, ctypes.byref(g), ctypes.c_void_p(p0.data_ptr()),
                                             ctypes.c_void_p(v0.data_ptr()), None, 0, dt, _lib.CUBIC_TC,
                                             _lib.MIDPOINT, _lib.F32, ctypes.c_void_p(out.data_ptr())))
            assert torch.equal(out.to(cuda), want.double())
    finally:
        Lb.dcell_session_destroy(sess)
