"""The five benchmark configurations of the transport path, run end to end.

    python -m dcell_b200.configs [c1|c2|c3|c4|c5|all] [--out results.json]

Each runner returns a JSON-able dict with the errors (max and L2 of phi in
the |phi| < 3h band, enclosed-volume error) and timings it measured.  Every
field is synthetic (formulas and seeds; no dataset exists for this path):

c1  2D Zalesak slotted disk, 256^2, rigid rotation, one revolution, CFL 0.5,
    midpoint backtrace, bicubic: FP32 GPU vs the exact answer (the initial
    disk) and vs an FP64 GPU run.  (The reference's own CPU AdvectSL against
    the FP32 GPU linear kernel on this case is a GPU test, not a runner.)
c2  3D sphere in LeVeque's time-reversing deformation, 128^3, T=3, CFL 0.5,
    tricubic, midpoint: FP32 vs the FP64 GPU kernel; volume loss and max phi
    error after the return at t = T.
c3  the same field at 256^3 over the whole period (t = 0 .. T): the
    split-BF16 tensor-core step's one-step error vs the FP64 GPU kernel at
    every step (max, L2, volume), and the accumulated error of the
    split-state TC and plain FP32 trajectories at t = T.
c4  512 cells, edges U{32..96} (seeded), ellipsoids in 8-mode divergence-free
    Fourier velocities, 20 steps: one persistent CUDA-graph launch per step
    with autotuned tiles vs one launch per cell; the split-state bricks of
    all cells in one launch per step, staged by cp.async and, over a padded
    packing, by TMA.
vel velocity acquisition of 512 cells' boxes (edges U{32..96}, some
    straddling the domain edge) from a 512^3 fluid field [z][y][x][c] (FP32,
    c = CELL_CENTER, U, V, W) in one dcell_velocity_boxes launch: time,
    achieved bytes/s, and 8 boxes checked against slicing.
pls the particle level set at 256^3: ~3.5 M FP32 particles (32 per cell
    within 3 cells of a sphere of radius 0.15) in LeVeque's deformation field;
    per step RK2 particle advection, escaped-particle error correction and
    radius adjustment, timed on the device.
reinit  narrow-band reinitialisation (bucketed fast marching) of the
    workload sphere at 256^3 (cell units, band width 6), FP64 and FP32.
io  output: phi of the 256^3 workload (FP32) written 10 times in the
    reference's .Real64 format by the asynchronous writer -- the time the
    compute stream spends on each snapshot, and the drain rate to disk.
steps  K dense steps of one SL form at 256^3 (--interp, --backtrace, --steps):
    the command the kernel profiles capture.
c5  128^3, 50 midpoint steps, velocity from 16 learnable Fourier
    coefficients, loss sum (H_eps(phi_T) - H_eps(phi_target))^2: hand-written
    adjoint (checkpoints every 10) vs FP64 central differences (delta 1e-3)
    and vs the FP64 adjoint.
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np
import torch

from . import fields
from . import levelset as L


def _band_err(out, ref, h):
    band = ref.abs() < 3 * h
    e = (out.double() - ref.double()).abs()[band]
    return {"max": float(e.max()), "l2": float(e.pow(2).mean().sqrt()), "band_points": int(band.sum())}


def _events():
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def run_c1(N=256, dev="cuda"):
    h = 1.0 / N
    phi0 = fields.slotted_disk_sdf(N, device=dev)
    vel = fields.rotation_velocity_2d(N, device=dev)
    steps = int(math.ceil(2 * math.pi / h))  # one revolution at CFL 0.5 (max |u| = pi)
    dt = 1.0 / steps
    out = {"grid": [N, N], "steps": steps, "dt": dt}
    for name, dtype in (("fp32", torch.float32), ("fp64", torch.float64)):
        a = phi0.to(dtype).contiguous()
        v = vel.to(dtype).contiguous()
        e0, e1 = _events()
        e0.record()
        for _ in range(steps):
            a = L.sl_step(a, v, dt, h, interp="cubic_plain", backtrace="midpoint")
        e1.record()
        torch.cuda.synchronize()
        out[f"bicubic_{name}"] = {"vs_exact": _band_err(a, phi0, h), "ms": e0.elapsed_time(e1),
                                  "area_rel_err": abs(float(L.volume(a, h, 1.5 * h)) -
                                                      float(L.volume(phi0, h, 1.5 * h))) /
                                  float(L.volume(phi0, h, 1.5 * h))}
        out[f"_final_{name}"] = a
    out["bicubic_fp32_vs_fp64"] = _band_err(out.pop("_final_fp32"), out.pop("_final_fp64"), h)
    return out


def _deformation(N, dev):
    h = 1.0 / N
    return h, fields.sphere_sdf(N, device=dev), fields.deformation_velocity(N, device=dev)


def run_c2(N=128, dev="cuda", T=3.0):
    h, phi0, vel = _deformation(N, dev)
    dt0 = fields.cfl_dt((2.0, 1.0, 1.0), h)
    steps = int(math.ceil(T / dt0))
    dt = T / steps
    res = {"grid": [N] * 3, "steps": steps, "dt": dt}
    finals = {}
    for name, dtype, interp in (("fp32_plain", torch.float32, "cubic_plain"),
                                ("fp32_tc", torch.float32, "cubic_tc"),
                                ("fp64_gpu", torch.float64, "cubic_plain")):
        a = phi0.to(dtype).contiguous()
        v = vel.to(dtype).contiguous()
        e0, e1 = _events()
        e0.record()
        for s in range(steps):
            fac = math.cos(math.pi * (s + 0.5) * dt / T)
            a = L.sl_step(a, v, dt * fac, h, interp=interp, backtrace="midpoint")
        e1.record()
        torch.cuda.synchronize()
        v0 = float(L.volume(phi0, h, 1.5 * h))
        res[name] = {"return_error_vs_initial": _band_err(a, phi0, h), "ms": e0.elapsed_time(e1),
                     "volume_loss_rel": (v0 - float(L.volume(a, h, 1.5 * h))) / v0}
        finals[name] = a
    # the split-state stepper of the dense benchmark: phi carried between
    # steps as packed BF16 hi/lo words (fp32_tc splits the FP32 field inside
    # every step instead)
    v = vel.float().contiguous()
    spl = [L.split_bf16(phi0.float().contiguous()), None]
    spl[1] = torch.empty_like(spl[0])
    outs = [torch.empty(phi0.shape, dtype=torch.float32, device=phi0.device) for _ in range(2)]
    a = None
    e0, e1 = _events()
    e0.record()
    for s in range(steps):
        fac = math.cos(math.pi * (s + 0.5) * dt / T)
        a, _ = L.sl_step_tc_split(spl[s & 1], v, dt * fac, h, backtrace="midpoint", out=outs[s & 1],
                                  out_split=spl[(s + 1) & 1])
    e1.record()
    torch.cuda.synchronize()
    v0 = float(L.volume(phi0, h, 1.5 * h))
    res["fp32_tc_split_state"] = {"return_error_vs_initial": _band_err(a, phi0, h), "ms": e0.elapsed_time(e1),
                                  "volume_loss_rel": (v0 - float(L.volume(a, h, 1.5 * h))) / v0,
                                  "vs_fp64_gpu": _band_err(a, finals["fp64_gpu"], h)}
    res["fp32_plain_vs_fp64_gpu"] = _band_err(finals["fp32_plain"], finals["fp64_gpu"], h)
    res["fp32_tc_vs_fp64_gpu"] = _band_err(finals["fp32_tc"], finals["fp64_gpu"], h)
    return res


def run_c3(N=256, dev="cuda", T=3.0, steps=None):
    """C3 over the whole period of the time-reversing field (t = 0 .. T, the
    shape back where it started), FP64 tricubic GPU trajectory as the
    reference.  Every step k:
      * one-step error: the split-BF16 tensor-core step from the FP32
        rounding of the FP64 state phi_k vs the FP64 step from phi_k (max and
        L2 in the |phi| < 3h band, and the relative volume error) -- the
        per-step error that the 1e-5 bar is about;
    and at t = T (plus the worst over the run, sampled every 64 steps):
      * accumulated error: the split-state tensor-core trajectory (phi carried
        as packed BF16 hi/lo words between steps) and the plain FP32
        trajectory vs the FP64 trajectory;
      * the return error of each against the initial sphere (the exact
        answer at t = T) and their volume loss.
    `steps` < the period's step count stops early (same dt)."""
    h, phi0, vel = _deformation(N, dev)
    dt0 = fields.cfl_dt((2.0, 1.0, 1.0), h)
    period = int(math.ceil(T / dt0))
    dt = T / period
    steps = period if steps is None else min(int(steps), period)
    v64, v32 = vel.contiguous(), vel.float().contiguous()
    del vel
    ref = phi0.contiguous()
    spl = [L.split_bf16(phi0.float().contiguous()), None]
    spl[1] = torch.empty_like(spl[0])
    outs = [torch.empty(phi0.shape, dtype=torch.float32, device=phi0.device) for _ in range(2)]
    one_phi, one_spl = torch.empty_like(outs[0]), torch.empty_like(spl[0])
    pl = phi0.float().contiguous()
    tc = outs[0]
    loc_max, loc_l2, loc_vol, traj = [], [], [], []

    def band_stats(a, b):
        band = b.abs() < 3 * h
        e = (a.double() - b).abs() * band
        return e.max(), (e.pow(2).sum() / band.sum()).sqrt()

    t0 = time.perf_counter()
    for k in range(steps):
        d = dt * math.cos(math.pi * (k + 0.5) * dt / T)
        nxt = L.sl_step(ref, v64, d, h, interp="cubic_plain", backtrace="midpoint")
        L.sl_step_tc_split(L.split_bf16(ref.float()), v32, d, h, backtrace="midpoint", out=one_phi,
                           out_split=one_spl)
        m, l2 = band_stats(one_phi, nxt)
        vr = L.volume(nxt, h, 1.5 * h)
        loc_max.append(m)
        loc_l2.append(l2)
        loc_vol.append(((L.volume(one_phi, h, 1.5 * h) - vr) / vr).abs())
        tc, _ = L.sl_step_tc_split(spl[k & 1], v32, d, h, backtrace="midpoint", out=outs[k & 1],
                                   out_split=spl[(k + 1) & 1])
        pl = L.sl_step(pl, v32, d, h, interp="cubic_plain", backtrace="midpoint")
        ref = nxt
        if (k + 1) % 64 == 0 or k + 1 == steps:
            traj.append(torch.stack([band_stats(tc, ref)[0], band_stats(pl, ref)[0]]))
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    loc_max, loc_l2 = torch.stack(loc_max).cpu(), torch.stack(loc_l2).cpu()
    loc_vol = torch.cat(loc_vol).cpu()
    traj = torch.stack(traj).cpu()
    v0 = float(L.volume(phi0, h, 1.5 * h))

    def final(a):
        return {"vs_fp64": _band_err(a, ref, h), "return_error_vs_initial": _band_err(a, phi0, h),
                "volume_loss_rel": (v0 - float(L.volume(a, h, 1.5 * h))) / v0}
    worst = float(loc_max.max())
    return {"grid": [N] * 3, "steps": steps, "period_steps": period, "dt": dt, "T": T,
            "one_step_tc_vs_fp64": {"worst_max": worst, "worst_step": int(loc_max.argmax()) + 1,
                                    "worst_l2": float(loc_l2.max()), "mean_max": float(loc_max.mean()),
                                    "worst_volume_rel": float(loc_vol.max())},
            "tc_meets_1e-5_every_step": worst <= 1e-5,
            "accumulated": {"tc_split_state": final(tc), "plain_fp32": final(pl),
                            "fp64": {"return_error_vs_initial": _band_err(ref, phi0, h),
                                     "volume_loss_rel": (v0 - float(L.volume(ref, h, 1.5 * h))) / v0},
                            "tc_worst_max_vs_fp64_over_run": float(traj[:, 0].max()),
                            "plain_fp32_worst_max_vs_fp64_over_run": float(traj[:, 1].max())},
            "wall_s": wall}


def run_c4(dev="cuda", ncells=512, steps=20):
    from .batch import CellBatch, c4_workload
    phis, vels, hs, dt = c4_workload(ncells=ncells, device=dev)
    b = CellBatch(phis, vels, hs, dt, device=dev)
    res = {"cells": ncells, "points_per_step": b.npoints, "steps": steps, "dt": dt}
    for interp in ("cubic_tc", "cubic_separable"):
        (tile, ctas), table = b.autotune(interp, "midpoint", reps=2)
        g, (a, _, outbuf) = b.capture(steps, interp, "midpoint")
        g.replay()
        torch.cuda.synchronize()
        e0, e1 = _events()
        e0.record()
        g.replay()
        e1.record()
        torch.cuda.synchronize()
        ms_graph = e0.elapsed_time(e1)
        x, y = b.phi.clone(), torch.empty_like(b.phi)
        b.step_per_cell(x, y, interp, "midpoint")
        torch.cuda.synchronize()
        e0.record()
        for _ in range(steps):
            b.step_per_cell(x, y, interp, "midpoint")
            x, y = y, x
        e1.record()
        torch.cuda.synchronize()
        ms_cells = e0.elapsed_time(e1)
        res[interp] = {"tile": list(tile), "ctas_per_sm": ctas, "graph_ms": ms_graph, "per_cell_launch_ms": ms_cells,
                       "speedup": ms_cells / ms_graph, "updates_per_s": b.npoints * steps / (ms_graph / 1e3),
                       "autotune_top3": [[t[0], list(t[1]), t[2]] for t in table[:3]]}
    # split-state tensor-core steps over bricks of all cells (one launch per
    # step), against dcell_sl_step_tc_split per cell, and the error of both TC
    # forms against the FP64 tricubic step per cell after `steps` steps
    s0 = b.split()
    xa, ya = s0.clone(), torch.empty_like(s0)
    pa = torch.empty_like(b.phi)
    b.step_tc_split(xa, pa, ya)
    torch.cuda.synchronize()
    e0, e1 = _events()
    e0.record()
    for _ in range(steps):
        b.step_tc_split(xa, pa, ya)
        xa, ya = ya, xa
    e1.record()
    torch.cuda.synchronize()
    ms_bricks = e0.elapsed_time(e1)
    xc, yc, pc = s0.clone(), torch.empty_like(s0), torch.empty_like(b.phi)
    e0.record()
    for _ in range(steps):
        b.step_tc_split_per_cell(xc, pc, yc)
        xc, yc = yc, xc
    e1.record()
    torch.cuda.synchronize()
    ms_split_cells = e0.elapsed_time(e1)
    res["cubic_tc_split_bricks"] = {"ms": ms_bricks, "per_cell_launch_ms": ms_split_cells,
                                    "updates_per_s": b.npoints * steps / (ms_bricks / 1e3),
                                    "equal_to_per_cell": bool(torch.equal(pa, pc)),
                                    "how": "dcell_batch_sl_step_tc_split, one launch per step over bricks of all "
                                           "cells, split state, CUDA events"}
    # the same over a padded packing with the boxes staged by TMA (a tensor
    # map per cell); the real points must equal the unpadded run's
    bp = CellBatch(phis, vels, hs, dt, device=dev, padded=True)
    sp = bp.split()
    xp, yp, pp = sp.clone(), torch.empty_like(sp), torch.empty_like(bp.phi)
    bp.step_tc_split_tma(xp, pp, yp)  # warm-up (tensor maps of both buffers)
    bp.step_tc_split_tma(yp, pp, xp)
    xp.copy_(sp)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        bp.step_tc_split_tma(xp, pp, yp)
        xp, yp = yp, xp
    e1.record()
    torch.cuda.synchronize()
    ms_tma = e0.elapsed_time(e1)
    same = all(torch.equal(bp.cell_view(pp, i), b.cell_view(pa, i)) for i in range(b.ncells))
    res["cubic_tc_split_bricks_tma"] = {"ms": ms_tma, "updates_per_s": b.npoints * steps / (ms_tma / 1e3),
                                        "stored_points": bp.npoints, "equal_to_unpadded": same,
                                        "how": "dcell_batch_sl_step_tc_split_tma, rows padded to 4 points, TMA "
                                               "boxes through a tensor map per cell, CUDA events"}
    return res


def vel_workload(G=512, ncells=512, seed=7, dev="cuda"):
    """The field, the box records (host and device), the output buffer, the
    largest box's point count, the total points and the algorithmic bytes of
    one launch (12 B read per point inside the field, 12 B written per point)."""
    from . import _lib
    gen = torch.Generator(device=dev).manual_seed(seed)
    field = torch.rand((G, G, G, 4), dtype=torch.float32, device=dev, generator=gen)
    rng = np.random.default_rng(seed)
    rec = np.zeros(ncells, dtype=_lib.BOX_DTYPE)
    off, inside, maxp = 0, 0, 0
    for b in range(ncells):
        e = rng.integers(32, 97, size=3)
        o = np.array([rng.integers(-8, G - int(e[a]) + 9) for a in range(3)])
        rec[b]["offset"], rec[b]["p"], rec[b]["n"] = off, o, e
        n = int(np.prod(e))
        inside += int(np.prod([max(0, min(G, o[a] + e[a]) - max(0, o[a])) for a in range(3)]))
        off, maxp = off + n, max(maxp, n)
    d_rec = torch.from_numpy(np.frombuffer(rec.tobytes(), dtype=np.uint8).copy()).to(dev)
    out = torch.empty(off * 3, dtype=torch.float32, device=dev)
    return field, rec, d_rec, out, maxp, off, inside * 12 + off * 12


def run_vel(G=512, ncells=512, dev="cuda", K=10, W=3):
    import ctypes

    from . import _lib
    field, rec, d_rec, out, maxp, npts, nbytes = vel_workload(G, ncells, dev=dev)
    lib = _lib.lib()
    gd = (ctypes.c_int * 3)(G, G, G)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def launch():
        _lib.check(lib.dcell_velocity_boxes(ctypes.c_void_p(d_rec.data_ptr()), len(rec), 3, _lib.F32,
                                            ctypes.c_void_p(field.data_ptr()), gd, 4, 1, maxp,
                                            ctypes.c_void_p(out.data_ptr()), st))
    for _ in range(W):
        launch()
    e0, e1 = _events()
    torch.cuda.synchronize()
    e0.record()
    for _ in range(K):
        launch()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / K
    bad = 0
    for b in np.linspace(0, ncells - 1, 8).astype(int):
        o, n, at = rec[b]["p"], rec[b]["n"], int(rec[b]["offset"])
        want = torch.zeros((int(n[2]), int(n[1]), int(n[0]), 3), dtype=field.dtype, device=dev)
        lo = [max(0, int(o[a])) for a in range(3)]
        hi = [min(G, int(o[a] + n[a])) for a in range(3)]
        if all(h > l for l, h in zip(lo, hi)):
            want[lo[2] - o[2]:hi[2] - o[2], lo[1] - o[1]:hi[1] - o[1], lo[0] - o[0]:hi[0] - o[0]] = \
                field[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0], 1:4]
        got = out[at * 3:(at + int(np.prod(n))) * 3].view(want.shape)
        bad += int((got != want).sum().item())
    return {"workload": f"{ncells} cells, edges U{{32..96}}, from a {G}^3 x 4 FP32 field", "points": npts,
            "ms": ms, "algorithmic_bytes": nbytes, "achieved_gbs": nbytes / (ms / 1e3) / 1e9,
            "mismatches_in_8_boxes": bad,
            "how": "dcell_velocity_boxes, one launch for all boxes, CUDA events, mean of 10 (field + boxes > L2)"}


def run_mac(N=256, dev="cuda", K=10, W=3, return_fp64=False):
    """LevelSetAdvectMAC_3D (AdvectMAC.c:62-111) on the N^3 workload: the
    sphere's phi and the deformation field's three components as separate
    face arrays.  FP32 and FP64 dense steps timed with CUDA events (inputs
    larger than L2).  With return_fp64, also returns the FP64 inputs and
    result as numpy arrays (phi, u, v, w, dt, h, out) for a caller that
    compares them with a CPU implementation."""
    import ctypes

    from . import _lib
    phi64 = (fields.sphere_sdf(N, device=dev) * N).double().contiguous()
    vel = fields.deformation_velocity(N, device=dev).double()
    comps64 = [vel[..., a].contiguous() for a in range(3)]
    del vel
    h, dt = 1.0 / N, 0.5 / N
    upd = (N - 1) ** 3
    res = {"workload": f"{N}^3 sphere phi (cell units), LeVeque deformation faces, dt = 0.5 h",
           "points_updated": upd}
    lib = _lib.lib()
    got = None
    for name, dtype in (("fp32", torch.float32), ("fp64", torch.float64)):
        ph = phi64.to(dtype)
        u, v, w = (c.to(dtype) for c in comps64)
        out = ph.clone()
        g = _lib.geom(ph.shape, h)
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        args = [ctypes.byref(g), _lib.F32 if dtype == torch.float32 else _lib.F64] + \
            [ctypes.c_void_p(t.data_ptr()) for t in (ph, u, v, w)] + [dt, ctypes.c_void_p(out.data_ptr()), st]
        for _ in range(W):
            _lib.check(lib.dcell_advect_mac(*args))
        e0, e1 = _events()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(K):
            _lib.check(lib.dcell_advect_mac(*args))
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / K
        nbytes = upd * 5 * ph.element_size()  # read phi, u, v, w; write out (neighbour re-reads not counted)
        res[name] = {"ms": ms, "algorithmic_bytes": nbytes, "achieved_gbs": nbytes / (ms / 1e3) / 1e9}
        if dtype == torch.float64:
            got = out.cpu().numpy()
    res["how"] = "dcell_advect_mac, dense, CUDA events, mean of 10 (inputs > L2)"
    if not return_fp64:
        return res
    return res, [t.cpu().numpy() for t in [phi64] + comps64] + [dt, h, got]


def run_nodes(N=256, dev="cuda", reps=5, return_fp64=False):
    """The irregular-node pass (LevelSetUpdateIrregularNodeList,
    IrregularNodes3D.c:6-117: sign tests, orthogonal projections; plus the
    normals and curvature of IIM/SurfaceQuantities.c) on the |phi| < 6h band
    of the N^3 workload sphere, FP64 and FP32, CUDA events, median of `reps`
    calls.  With return_fp64, also returns (phi, band, node rows) of the FP64
    pass as numpy arrays for a caller that compares them with a CPU
    implementation."""
    import statistics
    h = 1.0 / N
    phi64 = fields.sphere_sdf(N, device=dev).double().contiguous()
    band = fields.band_of(phi64, 6 * h, margin=3).to(dev)
    res = {"workload": f"{N}^3 sphere r=0.15, band |phi| < 6h", "band_points": int(band.shape[0])}
    rows64 = None
    for name, dtype in (("fp64", torch.float64), ("fp32", torch.float32)):
        ph = phi64.to(dtype)
        L.irregular_nodes(ph, h, band, with_surface=True)  # warm-up (allocations)
        times = []
        for _ in range(reps):
            e0, e1 = _events()
            torch.cuda.synchronize()
            e0.record()
            raw, count = L.irregular_nodes(ph, h, band, with_surface=True)
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        res[name] = {"ms": statistics.median(times), "nodes": int(count.item())}
        if dtype == torch.float64:
            rows64 = L.nodes_to_rows(L.nodes_to_numpy(raw, int(count.item())))
    res["how"] = "levelset.irregular_nodes(with_surface=True): count, scan, write, projections, normals/curvature"
    if not return_fp64:
        return res
    return res, (phi64.cpu().numpy(), band.cpu().numpy(), rows64)


def pls_workload(N=256, per_cell=32, seed=5, dev="cuda", dtype=torch.float32):
    """phi (cell units) of the workload sphere, its band |phi| < 6 cells, the
    deformation velocity, and per_cell particles uniform in every cell with
    |phi| < 3 whose side is phi's sign there (the radius is set by the first
    adjustment)."""
    phi = (fields.sphere_sdf(N, device=dev) * N).to(dtype).contiguous()
    band = fields.band_of(phi, 6.0, margin=3).to(dev)
    vel = fields.deformation_velocity(N, device=dev).to(dtype).contiguous()
    near = band[phi[band[:, 2].long(), band[:, 1].long(), band[:, 0].long()].abs() < 3]
    gen = torch.Generator(device=dev).manual_seed(seed)
    cells = near.repeat_interleave(per_cell, dim=0).to(dtype)
    parts = torch.empty((cells.shape[0], 4), dtype=dtype, device=dev)
    parts[:, :3] = cells + torch.rand(cells.shape, generator=gen, device=dev, dtype=dtype) - 0.5
    side = phi[near[:, 2].long(), near[:, 1].long(), near[:, 0].long()].sign().repeat_interleave(per_cell)
    parts[:, 3] = torch.where(side == 0, torch.ones_like(side), side) * 0.3
    return phi, band, vel, parts.contiguous()


def run_pls(N=256, steps=10, warmup=3, dev="cuda", workload=None):
    import ctypes

    from . import _lib, pls
    phi, band, vel, parts = workload if workload is not None else pls_workload(N, dev=dev)
    parts = parts.clone()
    n = parts.shape[0]
    h = 1.0 / N
    dt = 0.5 * h / 1.0  # CFL 0.5 of the field's unit maximum speed
    prm = pls.params(3)
    g = _lib.geom(tuple(phi.shape), h)
    scr = pls._scratch(_lib.lib().dcell_pls_correct_scratch_bytes(ctypes.byref(g), _lib.F32), dev)
    pls.adjust_radii(phi, parts, n, h, prm=prm)
    work = phi.clone()

    def step():
        pls.advect(parts, n, vel, dt, h)
        pls.correct(work, band, parts, n, h, scratch=scr)
        pls.adjust_radii(work, parts, n, h, prm=prm)
    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    e0, e1 = _events()
    e0.record()
    for _ in range(steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    # the three kernels timed alone (advection dominates)
    parts_f = parts.clone()
    e0.record()
    for _ in range(steps):
        pls.advect(parts_f, n, vel, dt, h)
    e1.record()
    torch.cuda.synchronize()
    ms_adv = e0.elapsed_time(e1) / steps
    return {"grid": [N] * 3, "particles": n, "band_points": int(band.shape[0]), "dtype": "f32", "steps": steps,
            "ms_per_step": ms, "particle_updates_per_s": n / (ms / 1e3), "advect_ms": ms_adv,
            "advect_bytes_per_particle": 32, "advect_gbs": n * 32 / (ms_adv / 1e3) / 1e9,
            "how": "advect (RK2 midpoint) + error correction + adjust radii per step, CUDA events, phi held fixed"}


def run_reinit(N=256, reps=5, dev="cuda"):
    phi = (fields.sphere_sdf(N, device=dev) * N).contiguous()
    band = fields.band_of(phi, 6.0, margin=3).to(dev)
    raw, count = L.irregular_nodes(phi, 1.0, band, with_surface=False)
    nn = int(count.item())
    out = {"grid": [N] * 3, "seed_nodes": nn}
    for name, dt in (("fp64", torch.float64), ("fp32", torch.float32)):
        x = phi.to(dt)
        ms = []
        for k in range(reps + 1):
            y = x.clone()
            e0, e1 = _events()
            e0.record()
            b = L.reinitialize(y, raw, nn, 6.0, 1.0 / 64)
            e1.record()
            torch.cuda.synchronize()
            if k:
                ms.append(e0.elapsed_time(e1))
        ms.sort()
        out[name + "_ms"] = ms[len(ms) // 2]
        out["band_points"] = int(b.shape[0])
    out["how"] = "dcell_reinitialize, CUDA events, median of %d" % reps
    return out


def run_io(N=256, writes=10, directory=None, dev="cuda"):
    import shutil
    import tempfile

    from .writer import Writer
    phi = (fields.sphere_sdf(N, device=dev) * N).float().contiguous()
    h = 1.0 / N
    d = directory or tempfile.mkdtemp(prefix="dcell_io_")
    try:
        with Writer(d, tmpdir=d) as w:
            for t in range(writes):  # the snapshot pool grows to what `writes` pending snapshots need
                w.grid("warm", t, phi, h)
            w.flush()
            e0, e1 = _events()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            e0.record()
            for t in range(writes):
                w.grid("phi", t, phi, h)
            e1.record()
            torch.cuda.synchronize()
            stream_ms = e0.elapsed_time(e1) / writes
            w.flush()
            wall = time.perf_counter() - t0
        nbytes = phi.numel() * 8 + 8
    finally:
        if directory is None:
            shutil.rmtree(d, ignore_errors=True)
    return {"grid": [N] * 3, "writes": writes, "file_bytes": nbytes, "stream_ms_per_write": stream_ms,
            "snapshot_gbs": 2 * phi.numel() * 4 / (stream_ms / 1e3) / 1e9, "drain_s": wall,
            "drain_gbs": writes * nbytes / wall / 1e9,
            "how": "dcell_writer_grid after a warm-up round: device snapshot on the stream (CUDA events), file "
                   "writing by the writer thread (wall clock to the flush)"}


def run_c5(N=128, steps=50, every=10, dev="cuda", fd_modes=16):
    from .autograd import FourierVelocity, c5_loss, transport
    h = 1.0 / N
    res = {"grid": [N] * 3, "steps": steps, "checkpoint_every": every}
    grads = {}
    for dtype in (torch.float64, torch.float32):
        model = FourierVelocity((N, N, N), nmodes=16, seed=5, device=dev, dtype=dtype)
        phi0 = fields.sphere_sdf(N, center=(0.5, 0.5, 0.5), r=0.2, device=dev).to(dtype)
        with torch.no_grad():
            c_tg = torch.as_tensor(np.random.default_rng(9).normal(size=16), dtype=dtype, device=dev)
            v_tg = model(c_tg)
            vmax = max(float(model()[..., d].abs().max()) for d in range(3))
            dt = 0.5 * h / max(vmax, float(v_tg.abs().max()))
            dts = [dt] * steps
            target = transport(phi0, v_tg, dts, h, "cubic_separable", "midpoint", every)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        loss = c5_loss(transport(phi0, model(), dts, h, "cubic_separable", "midpoint", every), target, h)
        loss.backward()
        torch.cuda.synchronize()
        grads[dtype] = model.coeffs.grad.double().clone()
        res[f"loss_{str(dtype)[6:]}"] = float(loss)
        res[f"forward_backward_s_{str(dtype)[6:]}"] = time.perf_counter() - t0
        if dtype == torch.float64:
            fd = torch.zeros(16, dtype=torch.float64, device=dev)
            with torch.no_grad():
                for m in range(fd_modes):
                    e = torch.zeros(16, dtype=dtype, device=dev)
                    e[m] = 1e-3
                    lp = c5_loss(transport(phi0, model(model.coeffs + e), dts, h, "cubic_separable", "midpoint",
                                           every), target, h)
                    lm = c5_loss(transport(phi0, model(model.coeffs - e), dts, h, "cubic_separable", "midpoint",
                                           every), target, h)
                    fd[m] = (lp - lm) / 2e-3
            sel = slice(0, fd_modes)
            res["fp64_adjoint_vs_fd_rel"] = float((grads[dtype][sel] - fd[sel]).norm() / fd[sel].norm())
    res["fp32_adjoint_vs_fp64_adjoint_rel"] = float((grads[torch.float32] - grads[torch.float64]).norm() /
                                                   grads[torch.float64].norm())
    return res


def run_steps(N=256, interp="cubic_tc", backtrace="midpoint", steps=4, dev="cuda"):
    """`steps` dense steps of one form of the SL step (any `interp` name of
    levelset.sl_step, "_gather" forms included) on the benchmark's N^3
    workload (sphere in the deformation field, FP32, dt at CFL 0.5), the
    same input each step; CUDA events.  The command the kernel profiles
    capture."""
    h, phi0, vel = _deformation(N, dev)
    phi, v = phi0.float().contiguous(), vel.float().contiguous()
    del phi0, vel
    dt = fields.cfl_dt((2.0, 1.0, 1.0), h)
    out = torch.empty_like(phi)
    e0, e1 = _events()
    L.sl_step(phi, v, dt, h, interp=interp, backtrace=backtrace, out=out)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        L.sl_step(phi, v, dt, h, interp=interp, backtrace=backtrace, out=out)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    return {"grid": [N] * 3, "interp": interp, "backtrace": backtrace, "steps": steps, "ms_per_step": ms,
            "updates_per_s": N ** 3 / (ms / 1e3)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("which", nargs="?", default="all")
    ap.add_argument("--out", default=None)
    ap.add_argument("--grid", type=int, default=None, help="vel: edge of the fluid field (512); pls: grid edge (256)")
    ap.add_argument("--cells", type=int, default=512, help="vel: number of cell boxes; c4: number of cells")
    ap.add_argument("--steps", type=int, default=20, help="c4, steps: steps per timed run")
    ap.add_argument("--interp", default="cubic_tc", help="steps: the SL form (levelset.sl_step interp name)")
    ap.add_argument("--backtrace", default="midpoint", help="steps: euler or midpoint")
    a = ap.parse_args()
    todo = ["c1", "c2", "c3", "c4", "c5"] if a.which == "all" else a.which.split(",")
    results = {}
    for c in todo:
        t0 = time.time()
        results[c] = (run_vel(a.grid or 512, a.cells) if c == "vel" else
                      run_pls(a.grid or 256) if c == "pls" else run_io(a.grid or 256) if c == "io" else
                      run_reinit(a.grid or 256) if c == "reinit" else run_mac(a.grid or 256) if c == "mac" else
                      run_nodes(a.grid or 256) if c == "nodes" else run_c4(ncells=a.cells, steps=a.steps) if c == "c4" else
                      run_steps(a.grid or 256, a.interp, a.backtrace, a.steps) if c == "steps" else
                      globals()[f"run_{c}"]())
        results[c]["wall_s"] = time.time() - t0
        print(json.dumps({c: results[c]}, default=float), flush=True)
    if a.out:
        json.dump(results, open(a.out, "w"), indent=1, default=float)


if __name__ == "__main__":
    main()
