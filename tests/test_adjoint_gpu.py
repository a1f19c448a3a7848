"""Hand-written SL adjoint vs FP64 central differences and vs the FP64
adjoint (the FP64 reference gradient), through torch.autograd."""
import numpy as np
import pytest
import torch

from dcell_b200 import fields
from dcell_b200.autograd import FourierVelocity, c5_loss, sl_adjoint, transport
from dcell_b200.levelset import sl_step

pytestmark = pytest.mark.gpu


def _dot(a, b):
    return float((a.double() * b.double()).sum())


@pytest.mark.parametrize("aggregate", ["none", "all"])
@pytest.mark.parametrize("interp", ["linear", "cubic_separable"])
@pytest.mark.parametrize("backtrace", ["euler", "midpoint"])
def test_single_step_adjoint_identity(cuda, interp, backtrace, aggregate, monkeypatch):
    """<SL'(phi0) dphi + SL_vel dvel, gbar> == <dphi, gphi0> + <dvel, gvel> (FP64, tiny steps),
    with per-lane and with warp-aggregated scatters."""
    monkeypatch.setenv("DCELL_ADJOINT_AGGREGATE", aggregate)
    N = 24
    h = 1.0 / N
    torch.manual_seed(0)
    phi0 = fields.sphere_sdf(N, center=(0.5, 0.5, 0.5), r=0.25, device=cuda)
    k, a, ph = fields.fourier_modes(4, 11)
    vel = fields.fourier_velocity((N, N, N), np.full(4, 0.05), (k, a, ph), device=cuda)
    dt = 0.3 * h
    gbar = torch.randn_like(phi0)
    gphi0, gvel = torch.zeros_like(phi0), torch.zeros_like(vel)
    sl_adjoint(phi0, vel, dt, h, gbar, gphi0, gvel, interp, backtrace)
    dphi, dvel = torch.randn_like(phi0), torch.randn_like(vel) * 0.05
    for eps in (1e-4,):
        fp = sl_step(phi0 + eps * dphi, vel + eps * dvel, dt, h, interp=interp, backtrace=backtrace)
        fm = sl_step(phi0 - eps * dphi, vel - eps * dvel, dt, h, interp=interp, backtrace=backtrace)
        lhs = _dot((fp - fm) / (2 * eps), gbar)
        rhs = _dot(dphi, gphi0) + _dot(dvel, gvel)
        assert abs(lhs - rhs) <= 1e-6 * max(abs(lhs), 1.0), (lhs, rhs)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("interp", ["linear", "cubic_separable"])
def test_aggregated_scatters_equal_per_lane_atomics(cuda, interp, dtype, monkeypatch):
    """The warp-aggregated scatters (phi0, velocity, both) give the per-lane
    atomics' gradients up to summation order, over a partial last warp
    (nx = 45) and 3x the CFL number (departures off the warp's row)."""
    nz, ny, nx = 20, 24, 45
    h = 1.0 / 48
    k, a, ph = fields.fourier_modes(4, 11)
    for cfl in (0.3, 3.0):
        phi0 = fields.sphere_sdf(48, center=(0.5, 0.5, 0.5), r=0.25, device=cuda)[:nz, :ny, :nx].contiguous().to(dtype)
        vel = fields.fourier_velocity((48, 48, 48), np.full(4, 0.05), (k, a, ph), device=cuda)[:nz, :ny, :nx]
        vel = vel.contiguous().to(dtype)
        gbar = torch.randn(phi0.shape, generator=torch.Generator().manual_seed(3), dtype=torch.float64).to(cuda, dtype)
        gbar[gbar.abs() < 0.3] = 0  # lanes that contribute nothing
        dt = cfl * h / float(vel.abs().max())
        res = {}
        for mode in ("none", "phi", "vel", "all"):
            monkeypatch.setenv("DCELL_ADJOINT_AGGREGATE", mode)
            gphi0, gvel = torch.zeros_like(phi0), torch.zeros_like(vel)
            sl_adjoint(phi0, vel, dt, h, gbar, gphi0, gvel, interp, "midpoint")
            res[mode] = (gphi0.double(), gvel.double())
        tol = 1e-12 if dtype == torch.float64 else 1e-5
        for mode in ("phi", "vel", "all"):
            for got, ref in zip(res[mode], res["none"]):
                assert float((got - ref).abs().max()) <= tol * float(ref.abs().max()), (mode, cfl)


def _c5(N, nsteps, dtype, cuda):
    h = 1.0 / N
    model = FourierVelocity((N, N, N), nmodes=16, seed=5, device=cuda, dtype=dtype)
    phi0 = fields.sphere_sdf(N, center=(0.5, 0.5, 0.5), r=0.2, device=cuda).to(dtype)
    with torch.no_grad():
        c_tg = torch.as_tensor(np.random.default_rng(9).normal(size=16), dtype=dtype, device=cuda)
        v_tg = model(c_tg)
        vmax = max(float(model(torch.ones(16, dtype=dtype, device=cuda))[..., d].abs().max()) for d in range(3))
        dt = 0.5 * h / max(vmax, float(v_tg.abs().max()))
        dts = [dt] * nsteps
        target = transport(phi0, v_tg, dts, h, "cubic_separable", "midpoint", 4)
    return h, model, phi0, target, dts


def test_gradient_matches_central_differences_fp64(cuda):
    """dL/dc (16 Fourier coefficients) by the adjoint vs FP64 central differences (delta 1e-3)."""
    N, K = 40, 12
    h, model, phi0, target, dts = _c5(N, K, torch.float64, cuda)
    loss = c5_loss(transport(phi0, model(), dts, h, "cubic_separable", "midpoint", 4), target, h)
    loss.backward()
    grad = model.coeffs.grad.detach().clone()
    fd = torch.zeros_like(grad)
    with torch.no_grad():
        for m in range(16):
            e = torch.zeros_like(grad)
            e[m] = 1e-3
            lp = c5_loss(transport(phi0, model(model.coeffs + e), dts, h, "cubic_separable", "midpoint", 4), target, h)
            lm = c5_loss(transport(phi0, model(model.coeffs - e), dts, h, "cubic_separable", "midpoint", 4), target, h)
            fd[m] = (lp - lm) / 2e-3
    rel = float((grad - fd).norm() / fd.norm())
    assert rel < 1e-4, (rel, grad.cpu().numpy(), fd.cpu().numpy())


def test_fp32_gradient_matches_fp64_reference_gradient(cuda):
    N, K = 40, 12
    grads = {}
    for dtype in (torch.float64, torch.float32):
        h, model, phi0, target, dts = _c5(N, K, dtype, cuda)
        loss = c5_loss(transport(phi0, model(), dts, h, "cubic_separable", "midpoint", 5), target, h)
        loss.backward()
        grads[dtype] = model.coeffs.grad.double()
    rel = float((grads[torch.float32] - grads[torch.float64]).norm() / grads[torch.float64].norm())
    assert rel < 1e-3, rel


def test_checkpoint_interval_does_not_change_gradient(cuda):
    N, K = 32, 10
    out = []
    for every in (1, 3, 10):
        h, model, phi0, target, dts = _c5(N, K, torch.float64, cuda)
        loss = c5_loss(transport(phi0, model(), dts, h, "cubic_separable", "midpoint", every), target, h)
        loss.backward()
        out.append(model.coeffs.grad.detach().clone())
    assert torch.allclose(out[0], out[1], rtol=1e-9, atol=1e-12)
    assert torch.allclose(out[0], out[2], rtol=1e-9, atol=1e-12)


def test_c5_configuration_as_stated(cuda):
    """The differentiation configuration itself: 128^3, 50 midpoint steps,
    velocity from 16 learnable Fourier coefficients, loss sum (H_eps(phi_T) -
    H_eps(phi_target))^2 with eps = 1.5h, checkpoints every 10.  The FP64
    adjoint gradient matches FP64 central differences (delta 1e-3, all 16
    coefficients) to 1e-4 relative, and the FP32 adjoint matches the FP64
    adjoint (the FP64 reference gradient) to 1e-4 relative."""
    from dcell_b200.configs import run_c5
    r = run_c5(N=128, steps=50, every=10, dev=cuda, fd_modes=16)
    print(f"\nC5 128^3 x 50: FP64 adjoint vs FD {r['fp64_adjoint_vs_fd_rel']:.2e}, FP32 vs FP64 adjoint "
          f"{r['fp32_adjoint_vs_fp64_adjoint_rel']:.2e}, forward+backward {r['forward_backward_s_float32'] * 1e3:.1f} ms "
          f"(FP32), {r['forward_backward_s_float64'] * 1e3:.1f} ms (FP64)")
    assert r["fp64_adjoint_vs_fd_rel"] <= 1e-4, r
    assert r["fp32_adjoint_vs_fp64_adjoint_rel"] <= 1e-4, r
