"""The device-resident LevelSetAdvectAndReinit loop (dcell_ls_resident_*,
LevelSetMethod/Advect.c:33-50): phi, band and irregular nodes stay on the
device between steps, only the velocity goes up.  Checked against the same
loop run step by step through the device API (levelset.LevelSetAdvectAndReinit
with the GPU reinitialisation hook): same phi bits, bands, counters."""
import ctypes
import math

import numpy as np
import pytest
import torch

from dcell_b200 import _lib, fields
from dcell_b200 import levelset as L


def test_resident_argument_errors():
    """No resident level set, a different geometry, bad dtypes: status codes,
    no device work."""
    lib = _lib.lib()
    g = _lib.geom((8, 8, 8), 0.1)
    loop = _lib.LsLoop()
    dummy = ctypes.c_void_p(64)
    assert lib.dcell_ls_resident_advect_and_reinit(None, ctypes.byref(g), dummy, 0, 0.1, 0, 0, 0,
                                                   ctypes.byref(loop)) == _lib.ERR_ARG
    assert lib.dcell_ls_resident_set(None, ctypes.byref(g), dummy, None, 0, 0) == _lib.ERR_ARG
    assert lib.dcell_ls_resident_get(None, ctypes.byref(g), None, None, 0, None) == _lib.ERR_ARG


def _case(N, dev):
    h = 1.0 / N
    phi = (fields.sphere_sdf(N, center=(0.5, 0.45, 0.55), r=0.2, device=dev) * N).contiguous()  # cell units
    vel = fields.deformation_velocity(N, device=dev).contiguous()
    band = fields.band_of(phi, 6.0, margin=3)
    return h, phi, vel, band


@pytest.mark.gpu
def test_resident_loop_equals_the_device_api_loop(cuda):
    """8 steps, FP64 linear Euler on the band, CFL threshold 1 so that the
    reinitialisation runs inside the loop: the resident loop gives the device
    API loop's phi and band bit for bit, and the same counters each step."""
    N = 48
    h, phi, vel, band = _case(N, cuda)
    dt = 0.9 * h
    ls = L.LevelSetCreate(h, (0, 0, 0), (N, N, N), dtype=torch.float64, device=cuda)
    ls.phi.copy_(phi)
    ls.band = band.to(cuda).contiguous()
    ls.CFLthres = 1.0
    ls.Reinitialize = L.LevelSetReinitializeGPU
    L.LevelSetUpdateIrregularNodeList(ls)
    r = L.ResidentLevelSet(phi.cpu().numpy(), h, band=band.cpu().numpy(), precision="f64", CFLthres=1.0)
    vhost = vel.cpu().numpy()
    reinits = 0
    for s in range(8):
        L.LevelSetAdvectAndReinit(ls, vel, dt)
        loop = r.advect_and_reinit(vhost, dt)
        assert loop.AdvectCount == ls.AdvectCount and loop.CFLcount == ls.CFLcount and loop.maxVel == ls.maxVel
        reinits += loop.reinitialized
    assert reinits >= 2
    got, gband = r.get()
    r.close()
    assert np.array_equal(got, ls.phi.cpu().numpy())
    assert np.array_equal(gband, ls.band.cpu().numpy())


@pytest.mark.gpu
@pytest.mark.parametrize("vel_dtype", ["f32", "f64"])
@pytest.mark.parametrize("cfl", [0.5, 4.0])
def test_resident_tc_loop_equals_split_state_steps(cuda, cfl, vel_dtype):
    """FP32, dense, split-BF16 tensor-core steps with FP32 or FP64 host
    velocity: the resident loop's phi after 5 steps equals 5
    dcell_sl_step_tc_split steps (the split state carried between them) bit
    for bit.  At 64^3 the loop steps z-slabs while the velocity planes go up;
    at 4x the CFL number the slabs' gate leaves them and the whole grid is
    stepped again once every plane is present."""
    N = 64
    h, phi, vel, band = _case(N, cuda)
    dt = cfl * h
    r = L.ResidentLevelSet(phi.cpu().numpy(), h, band=band.cpu().numpy(), precision="f32", CFLthres=1e9)
    v32 = vel.float().contiguous()
    vhost = v32.cpu().numpy() if vel_dtype == "f32" else v32.double().cpu().numpy()
    spl = L.split_bf16(phi.float().contiguous())
    out = None
    for s in range(5):
        r.advect_and_reinit(vhost, dt, interp="cubic_tc", backtrace="midpoint", dense=True)
        out, spl = L.sl_step_tc_split(spl, v32, dt, h, backtrace="midpoint", out_split=torch.empty_like(spl))
    got, _ = r.get()
    r.close()
    assert np.array_equal(got, out.double().cpu().numpy())


@pytest.mark.gpu
def test_resident_tc_loop_with_reinitialisation(cuda):
    """FP32 dense split-BF16 steps at 64^3 (the velocity upload overlapped with
    z-slab steps) with a CFL threshold low enough that the loop reinitialises
    twice.  The reinitialisation a step triggers runs at the start of the next
    call, under its upload, or in get(); phi, band and counters equal a
    step-by-step device loop that reinitialises at the end of the triggering
    step (split state carried, re-split after each reinitialisation)."""
    N = 64
    h, phi, vel, band = _case(N, cuda)
    dt = 0.5 * h
    v32 = vel.float().contiguous()
    r = L.ResidentLevelSet(phi.cpu().numpy(), h, band=band.cpu().numpy(), precision="f32", CFLthres=1.0)
    vhost = v32.cpu().numpy()
    p = phi.float().contiguous()
    b = band.to(cuda).contiguous()
    spl = L.split_bf16(p)
    raw, count = L.irregular_nodes(p, h, b, with_surface=False)
    cfl, reinits = 0.0, 0
    for s in range(10):
        loop = r.advect_and_reinit(vhost, dt, interp="cubic_tc", backtrace="midpoint", dense=True)
        p, spl = L.sl_step_tc_split(spl, v32, dt, h, backtrace="midpoint", out_split=torch.empty_like(spl))
        maxvel = float(L.max_velocity(v32, h, raw, count).item())
        cfl += dt * maxvel / h
        raw, count = L.irregular_nodes(p, h, b, with_surface=False)
        assert loop.maxVel == maxvel
        if cfl > 1.0:
            cfl = 0.0
            reinits += 1
            b = L.reinitialize(p, raw, count, 6.0)
            spl = L.split_bf16(p)
            assert loop.reinitialized == 1
        else:
            assert loop.reinitialized == 0
        assert loop.CFLcount == cfl
    assert reinits >= 2
    got, gband = r.get()
    r.close()
    assert np.array_equal(got, p.double().cpu().numpy())
    assert np.array_equal(gband, b.cpu().numpy())


@pytest.mark.gpu
def test_resident_loop_2d_equals_the_device_api_loop(cuda):
    """The 2D loop (Zalesak's disk in cell units, rigid rotation, FP64
    bilinear Euler on the band, CFL threshold 1 so that it reinitialises
    inside the loop): the resident loop's phi, band and counters equal the
    device API loop's, bit for bit."""
    N = 128
    h = 1.0 / N
    phi = (fields.slotted_disk_sdf(N, device=cuda) * N).contiguous()
    vel = fields.rotation_velocity_2d(N, device=cuda).contiguous()
    band = fields.band_of(phi, 6.0, margin=3)
    dt = 0.5 * h / math.pi
    ls = L.LevelSetCreate(h, (0, 0, 0), (N, N, 1), dtype=torch.float64, device=cuda)
    ls.phi.copy_(phi)
    ls.band = band.to(cuda).contiguous()
    ls.CFLthres = 1.0
    ls.Reinitialize = L.LevelSetReinitializeGPU
    L.LevelSetUpdateIrregularNodeList(ls)
    r = L.ResidentLevelSet(phi.cpu().numpy(), h, band=band.cpu().numpy(), precision="f64", CFLthres=1.0)
    vhost = vel.cpu().numpy()
    reinits = 0
    for s in range(12):
        L.LevelSetAdvectAndReinit(ls, vel, dt)
        loop = r.advect_and_reinit(vhost, dt)
        assert loop.AdvectCount == ls.AdvectCount and loop.CFLcount == ls.CFLcount and loop.maxVel == ls.maxVel
        reinits += loop.reinitialized
    assert reinits >= 2
    got, gband = r.get()
    r.close()
    assert np.array_equal(got, ls.phi.cpu().numpy())
    assert np.array_equal(gband, ls.band.cpu().numpy())
