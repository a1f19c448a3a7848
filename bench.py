#!/usr/bin/env python
"""Benchmark: semi-Lagrangian level-set updates/s at 256^3 on B200.

Workload (one "step"): one SL step of a 256^3 FP32 signed distance (sphere
r = 0.15 at (0.35, 0.35, 0.35)) in LeVeque's time-reversing deformation
field (T = 3, dt at CFL 0.5), midpoint backtrace, Catmull-Rom tricubic
reconstruction with the coefficient solve as a split-BF16 tcgen05 GEMM --
every one of the 16,777,216 grid points is updated.  Inputs are synthetic
(formulas), resident in HBM, larger than L2 (no flush needed).

Also measured in the same run: the plain FP32 CUDA-core step (1331-nnz
coefficient form) and the separable FP32 step, each as global gathers and on
the tensor-core stepper's TMA bricks; the trilinear FP32 step (the
reference's own mode) against the HBM roofline; the error of the TC step vs
the FP64 GPU oracle in the |phi| < 3h band, one step and over the field's
whole period; the end-to-end rate through the reference-facing C ABI (the
reference's LevelSetAdvectAndReinit loop with the level set resident on the
device, and the one-call round trip of FP64 host buffers); the CPU oracle
port.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 (torchrun): every rank advects its own independent 256^3 level set
(independent DCells, no collective on the data path) -> weak scaling.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_DEFAULT = 256
BYTES_PER_UPDATE = 20          # FP32: read phi0 4 B + u,v,w 12 B, write phi 4 B
TC_FLOP_PER_UPDATE = 16384     # 2 * 64 * 64 per split term, hi + lo
T_PERIOD = 3.0
METRIC = "SL level-set updates/s @256^3: split-BF16 TC vs plain FP32 GPU at <=1e-5 err"


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), float(p["bf16_tflops"]), "measured"
    except Exception:
        return 6650.0, 1590.0, "fallback"


def profiled_traffic():
    """DRAM bytes per launch of the TC kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "sl_tc_brick_kernel_256.md")  # ncu capture summary
    try:
        for ln in open(path):
            if ln.startswith("dram_bytes_per_launch_256:"):
                return float(ln.split(":")[1])
    except OSError:
        pass
    return None


class ClockSampler:
    """SM clock, power and clock-event (throttle) reasons sampled through NVML
    every 5 ms while the timed region runs (reads only; changes nothing)."""

    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
               0x80: "hw_power_brake_slowdown"}

    def __init__(self, cuda_index):
        self.cuda_index, self.samples, self.max_mhz, self.stop = cuda_index, [], None, threading.Event()

    def __enter__(self):
        try:
            import pynvml as N
            import torch
            N.nvmlInit()
            uuid = str(torch.cuda.get_device_properties(self.cuda_index).uuid)
            try:
                self.h = N.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
            except Exception:
                self.h = N.nvmlDeviceGetHandleByIndex(self.cuda_index)
            self.N = N
            self.max_mhz = N.nvmlDeviceGetMaxClockInfo(self.h, N.NVML_CLOCK_SM)
            getr = getattr(N, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                N.nvmlDeviceGetCurrentClocksThrottleReasons

            def run():
                while not self.stop.is_set():
                    try:
                        self.samples.append((N.nvmlDeviceGetClockInfo(self.h, N.NVML_CLOCK_SM), getr(self.h),
                                             N.nvmlDeviceGetPowerUsage(self.h) / 1000.0))
                    except Exception:
                        pass
                    self.stop.wait(0.005)
            self.t = threading.Thread(target=run, daemon=True)
            self.t.start()
        except Exception:
            self.N = None
        return self

    def __exit__(self, *a):
        self.stop.set()
        if self.N is not None:
            self.t.join(timeout=2)

    def summary(self):
        sm = [s[0] for s in self.samples]
        reasons = sorted({name for s in self.samples for bit, name in self.REASONS.items() if s[1] & bit})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "power_w_max": max((s[2] for s in self.samples), default=None), "samples": len(sm),
                "source": "nvml, 5 ms period, during the timed region"}


def workload(N, dev):
    import torch

    from dcell_b200 import fields
    h = 1.0 / N
    phi = fields.sphere_sdf(N, device=dev).float().contiguous()
    vel = fields.deformation_velocity(N, device=dev).float().contiguous()
    dt = fields.cfl_dt((2.0, 1.0, 1.0), h)
    return h, phi, vel, dt, torch


def dt_at(step, dt):
    """velocity factor cos(pi t/T) at the step's mid time, folded into dt"""
    return dt * math.cos(math.pi * (step + 0.5) * dt / T_PERIOD)


def timed_steps(L, torch, phi, vel, h, dt, interp, K, W, dist=None, backtrace="midpoint"):
    a, b = phi.clone(), phi.clone()
    for s in range(W):
        L.sl_step(a, vel, dt_at(s, dt), h, interp=interp, backtrace=backtrace, out=b)
        a, b = b, a
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for s in range(K):
        L.sl_step(a, vel, dt_at(W + s, dt), h, interp=interp, backtrace=backtrace, out=b)
        a, b = b, a
    e1.record(st)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    return e0.elapsed_time(e1)


def timed_tc_split(L, torch, phi, vel, h, dt, K, W, dist=None, backtrace="midpoint"):
    """The headline loop: split-BF16 tensor-core steps on a split-state level
    set (each step writes phi and its packed BF16 split for the next step)."""
    a, b = phi.clone(), torch.empty_like(phi)
    sa, sb = L.split_bf16(phi), torch.empty(phi.shape, dtype=torch.int32, device=phi.device)
    for s in range(W):
        L.sl_step_tc_split(sa, vel, dt_at(s, dt), h, backtrace=backtrace, out=b, out_split=sb)
        a, b, sa, sb = b, a, sb, sa
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for s in range(K):
        L.sl_step_tc_split(sa, vel, dt_at(W + s, dt), h, backtrace=backtrace, out=b, out_split=sb)
        a, b, sa, sb = b, a, sb, sa
    e1.record(st)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    return e0.elapsed_time(e1)


def cpu_oracle_rate(phi, vel, h, dt, nplanes=24, threads=1):
    """FP64 oracle port (tricubic, midpoint) on `nplanes` z-planes of the grid."""
    import numpy as np

    import oracle
    N = phi.shape[0]
    p64 = phi.double().cpu().numpy()
    v64 = vel.double().cpu().numpy()
    z0 = N // 2 - nplanes // 2
    zs, ys, xs = np.meshgrid(np.arange(z0, z0 + nplanes), np.arange(N), np.arange(N), indexing="ij")
    pts = np.stack([xs.ravel(), ys.ravel(), zs.ravel()], 1).astype(np.int32)
    chunks = np.array_split(pts, threads)
    t0 = time.perf_counter()
    if threads == 1:
        oracle.sl_step(p64, v64, dt, h, band=pts, interp="cubic", backtrace="midpoint")
    else:
        from concurrent.futures import ThreadPoolExecutor
        with ThreadPoolExecutor(threads) as ex:  # ctypes releases the GIL
            list(ex.map(lambda c: oracle.sl_step(p64, v64, dt, h, band=c, interp="cubic", backtrace="midpoint"),
                        chunks))
    t = time.perf_counter() - t0
    return len(pts) / t, len(pts), t


def reference_linear_rate(phi, vel, h, dt, nplanes=24):
    """The reference's own LevelSetAdvectSL_3D (linear, Euler, FP64) on `nplanes` planes."""
    import numpy as np

    from oracle import reference as R
    if not R.available():
        return None
    N = phi.shape[0]
    ls = R.RefLevelSet.create(h, (0, 0, 0), (N, N, N))
    ls.set_phi(phi.double().cpu().numpy())
    z0 = N // 2 - nplanes // 2
    zs, ys, xs = np.meshgrid(np.arange(z0, z0 + nplanes), np.arange(N), np.arange(N), indexing="ij")
    ls.set_band(np.stack([xs.ravel(), ys.ravel(), zs.ravel()], 1).astype(np.int32))
    ls.set_velocity(vel.double().cpu().numpy())
    ls.copy_phi_to_phi0()
    t0 = time.perf_counter()
    ls.advect_sl(dt)
    t = time.perf_counter() - t0
    ls.close()
    return xs.size / t


def reinit_case(torch, N, dev):
    """The 256^3 sphere of the workload in cell units, its band (|phi| < 6
    cells, 3 cells inside the grid) and the GPU irregular nodes of it."""
    from dcell_b200 import fields
    from dcell_b200 import levelset as L
    phi = (fields.sphere_sdf(N, device=dev) * N).contiguous()
    band = fields.band_of(phi, 6.0, margin=3).to(dev)
    raw, count = L.irregular_nodes(phi, 1.0, band, with_surface=False)
    return phi, band, raw, count


def timed_reinit(torch, phi, raw, count, dtype, K=5):
    """GPU reinitialisation (bucketed fast marching, dcell_reinitialize) of the
    case, CUDA events around each call on a fresh copy; median ms and the
    result of the last call."""
    from dcell_b200 import levelset as L
    x = phi.to(dtype)
    nn = int(count.item())
    ms = []
    for k in range(K + 1):
        y = x.clone()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        band = L.reinitialize(y, raw, nn, 6.0, 1.0 / 64)
        e1.record()
        torch.cuda.synchronize()
        if k:
            ms.append(e0.elapsed_time(e1))
    ms.sort()
    return ms[len(ms) // 2], y, band


def reference_reinit(phi, band):
    """The reference's own LevelSetReinitialize (FastMarching.c:11-146, heap
    FMM, FP64, one core) on the same phi after its own irregular-node pass."""
    import numpy as np

    from oracle import reference as R
    if not R.available():
        return None
    N = phi.shape[0]
    ls = R.RefLevelSet.create(1.0 / N, (0, 0, 0), (N, N, N))
    ls.set_phi(phi.double().cpu().numpy())
    ls.set_band(band.cpu().numpy())
    ls.update_irregular()
    t0 = time.perf_counter()
    ls.reinitialize()
    t = time.perf_counter() - t0
    out = ls.get_phi().copy()
    nb = int(ls.L.dref_ls_band_length(ls.h))
    ls.close()
    return t, out, nb


def reference_pls_step(phi, band, vel, parts, h, dt):
    """One particle step of the reference's own FP64 code (ParticleLS3D.c
    AdvectParticles3D + ErrorCorrection3D, ParticleLS.c AdjustRadii) on the
    same particles, one core; seconds per routine."""
    from oracle import reference as R
    if not R.available():
        return None
    N = phi.shape[0]
    ls = R.RefLevelSet.create(h, (0, 0, 0), (N, N, N))
    ls.set_phi(phi.double().cpu().numpy())
    ls.set_band(band.cpu().numpy())
    ls.set_velocity(vel.double().cpu().numpy())
    ls.pls_create_empty()
    ls.set_particles(parts.double().cpu().numpy())
    ls.pls_adjust()
    t0 = time.perf_counter()
    ls.pls_advect(dt)
    t1 = time.perf_counter()
    ls.pls_correct()
    t2 = time.perf_counter()
    ls.pls_adjust()
    t3 = time.perf_counter()
    adv = ls.particles()
    ls.close()
    return {"advect_s": t1 - t0, "correct_s": t2 - t1, "adjust_s": t3 - t2, "step_s": t3 - t0}, adv


def reference_nodes(res, phi, band, rows64, h):
    """The reference's own LevelSetUpdateIrregularNodeList_3D and surface
    quantities (oracle/_ref, FP64, one core) on the same phi and band, timed,
    with its node list compared to the GPU's FP64 rows."""
    import numpy as np

    from oracle import reference as R
    if not R.available():
        return
    N = phi.shape[0]
    ls = R.RefLevelSet.create(h, (0, 0, 0), (N, N, N))
    ls.set_phi(phi)
    ls.set_band(band)
    t0 = time.perf_counter()
    n = ls.update_irregular()
    t1 = time.perf_counter()
    ref = ls.nodes_no_update(n, surface=True)
    t2 = time.perf_counter()
    ls.close()
    same = rows64.shape == ref.shape and bool(np.array_equal(rows64[:, :8], ref[:, :8]))
    res["reference_cpu"] = {"node_list_s": t1 - t0, "surface_s": t2 - t1, "cores": 1, "kind": "reference",
                            "nodes": int(n), "fp64_exact_fields_equal": same,
                            "fp64_max_projection_diff": float(np.abs(rows64[:, 8:14] - ref[:, 8:14]).max())
                            if same else None,
                            "gpu_fp64_speedup": (t2 - t0) * 1e3 / res["fp64"]["ms"]}


def reference_mac(res, phi, u, v, w, dt, h, got):
    """The reference's own LevelSetAdvectMAC_3D (oracle/_ref, one core, timed)
    on the FP64 inputs of the GPU leg, compared bit for bit with the GPU's
    FP64 result; the oracle restatement is the checker where the reference
    was not compiled."""
    from oracle import reference as R
    ref_ok = R.available()
    t0 = time.perf_counter()
    if ref_ok:
        want = R.advect_mac(phi, u, v, w, dt, h)
        t = time.perf_counter() - t0
        res["reference_cpu"] = {"s": t, "cores": 1, "kind": "reference", "updates_per_s": res["points_updated"] / t}
    else:
        import oracle
        want = oracle.advect_mac(phi, u, v, w, dt, h)
    res["fp64_mismatches"] = int((got != want).sum())
    res["fp64_checked_against"] = "reference" if ref_ok else "oracle"


def e2e_rate(phi, vel, h, dt, K, torch):
    """Through the reference-facing C ABI with pinned FP64 host buffers
    (reference Grid layout): H2D of phi0 + velocity, TC step, D2H of phi,
    per step; synchronous calls timed by the host clock."""
    from dcell_b200 import _lib
    L = _lib.lib()
    N = phi.shape[0]
    p0 = phi.double().cpu().pin_memory()
    v0 = vel.double().cpu().pin_memory()
    out = torch.empty_like(p0).pin_memory()
    sess = ctypes.c_void_p()
    _lib.check(L.dcell_session_create(torch.cuda.current_device(), ctypes.byref(sess)))
    g = _lib.geom((N, N, N), h)
    args = lambda s: (sess, ctypes.byref(g), ctypes.c_void_p(p0.data_ptr()), ctypes.c_void_p(v0.data_ptr()), None, 0,
                      dt_at(s, dt), _lib.CUBIC_TC, _lib.MIDPOINT, _lib.F32, ctypes.c_void_p(out.data_ptr()))
    _lib.check(L.dcell_ls_advect_sl(*args(0)))  # warm-up (device buffers allocated)
    t0 = time.perf_counter()
    for s in range(K):
        _lib.check(L.dcell_ls_advect_sl(*args(s)))
    t = time.perf_counter() - t0
    L.dcell_session_destroy(sess)
    n = N ** 3
    # the copy bound: the same bytes moved alone, uploads and the download on
    # two streams at once (pinned buffers, best of 3, host clock)
    dp, dv, do = torch.empty_like(p0, device="cuda"), torch.empty_like(v0, device="cuda"), \
        torch.empty_like(out, device="cuda")
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    best = float("inf")
    for _ in range(3):
        torch.cuda.synchronize()
        c0 = time.perf_counter()
        with torch.cuda.stream(s1):
            dp.copy_(p0, non_blocking=True)
            dv.copy_(v0, non_blocking=True)
        with torch.cuda.stream(s2):
            out.copy_(do, non_blocking=True)
        torch.cuda.synchronize()
        best = min(best, time.perf_counter() - c0)
    del dp, dv, do
    return n * K / t, {"h2d_bytes_per_step": n * 8 + n * 24, "d2h_bytes_per_step": n * 8,
                       "copy_bound": {"ms": best * 1e3, "updates_per_s": n / best, "frac": (n * K / t) / (n / best),
                                      "how": "the step's H2D bytes on one stream with its D2H bytes on another, "
                                             "pinned, no compute"}}


def e2e_resident_rate(phi, vel, h, dt, K, torch):
    """The reference's LevelSetAdvectAndReinit loop (Advect.c:33-50) through
    the C ABI with the level set resident on the device
    (dcell_ls_resident_*): phi (cell units, as after the reference's fast
    marching) and its band go up once before the timed region; every step
    uploads its velocity from pinned FP32 host memory (12 B per point) and
    reads back the step's diagnostics (max |V| and the CFL counters), and
    runs the split-BF16 tensor-core step, the CFL increment, the
    irregular-node list and, when the CFL count passes 3 (the reference's
    default), the device reinitialisation; phi comes down once at the end,
    inside the timed region, into a pinned FP64 host grid allocated
    beforehand.  The warm-up runs the loop through one reinitialisation.
    Host clock around the synchronous calls."""
    from dcell_b200 import fields
    from dcell_b200 import levelset as L
    N = phi.shape[0]
    n = N ** 3
    cells = (phi.double() * N).contiguous()
    band = fields.band_of(cells, 6.0, margin=3)
    vhost = vel.float().cpu().pin_memory()
    phi_out = torch.empty(tuple(phi.shape), dtype=torch.float64).pin_memory()  # the host grid phi comes down to
    r = L.ResidentLevelSet(cells.cpu().numpy(), h, band=band.cpu().numpy(), precision="f32", CFLthres=3.0)
    # warm-up: buffers, and steps up to and including a reinitialisation (its
    # scratch and kernels), as in a loop that has been running
    for s in range(20):
        if r.advect_and_reinit(vhost, dt_at(s, dt), "cubic_tc", "midpoint", dense=True).reinitialized:
            break
    r.get(out=phi_out)
    reinits = 0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for s in range(K):
        reinits += r.advect_and_reinit(vhost, dt_at(s + 1, dt), "cubic_tc", "midpoint", dense=True).reinitialized
    r.get(out=phi_out)
    t = time.perf_counter() - t0
    r.close()
    return n * K / t, {"h2d_bytes_per_step": n * 12, "d2h_bytes_per_step": 16 + n * 8 / K, "steps": K,
                       "reinitialisations": reinits,
                       "how": "dcell_ls_resident_advect_and_reinit per step (FP32 host velocity up, diagnostics "
                              "down; split-BF16 TC step, CFL increment, irregular nodes, device reinitialisation at "
                              "CFL count > 3), phi down once at the end into a pinned FP64 host grid; warm-up through "
                              "one reinitialisation; host clock"}


def c4_rates(torch, dev, steps=20, sample_cells=48):
    """C4 (512 cells of 32..96 points per axis, ellipsoids in their own
    Fourier velocities, midpoint tricubic steps): the GPU's TMA-staged
    split-state bricks of all cells, one launch per step (CUDA events, 20
    steps), against the FP64 oracle restatement of the same tricubic/midpoint
    step on a sample of the cells with one host thread per core (the
    reference advects its cells rank by rank; its SL has no tricubic form)."""
    import numpy as np

    import oracle
    from dcell_b200.batch import CellBatch, c4_workload
    phis, vels, hs, dt = c4_workload(ncells=512, device=dev)
    bp = CellBatch(phis, vels, hs, dt, device=dev, padded=True)
    sp = bp.split()
    x, y, p = sp.clone(), torch.empty_like(sp), torch.empty_like(bp.phi)
    bp.step_tc_split_tma(x, p, y)  # warm-up (tensor maps of both buffers)
    bp.step_tc_split_tma(y, p, x)
    x.copy_(sp)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        bp.step_tc_split_tma(x, p, y)
        x, y = y, x
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    idx = np.linspace(0, len(phis) - 1, sample_cells).astype(int)
    cells = [(phis[i].double().cpu().numpy(), vels[i].double().cpu().numpy(), hs[i]) for i in idx]
    threads = os.cpu_count() or 1
    from concurrent.futures import ThreadPoolExecutor
    t0 = time.perf_counter()
    with ThreadPoolExecutor(threads) as ex:  # ctypes releases the GIL
        list(ex.map(lambda c: oracle.sl_step(c[0], c[1], dt, c[2], interp="cubic", backtrace="midpoint"), cells))
    t = time.perf_counter() - t0
    npts = int(sum(c[0].size for c in cells))
    gpu = bp.npoints * steps / (ms / 1e3)
    cpu = npts / t
    return {"cells": len(phis), "points_per_step": int(bp.npoints), "steps": steps,
            "gpu": {"ms": ms, "updates_per_s": gpu, "how": "dcell_batch_sl_step_tc_split_tma, CUDA events"},
            "cpu_baseline": {"value": cpu, "unit": "updates/s", "cores": threads, "kind": "port",
                             "sample": f"{sample_cells} of the 512 cells ({npts} points), one step each, one host "
                                       f"thread per core, {t:.1f} s"},
            "gpu_over_cpu": gpu / cpu}


def error_check(L, torch, phi, vel, h, dt):
    a = L.sl_step_tc_split(L.split_bf16(phi), vel, dt_at(0, dt), h, backtrace="midpoint")[0].double()
    ref = L.sl_step(phi.double(), vel.double(), dt_at(0, dt), h, interp="cubic_plain", backtrace="midpoint")
    plain = L.sl_step(phi, vel, dt_at(0, dt), h, interp="cubic_plain", backtrace="midpoint").double()
    band = ref.abs() < 3 * h
    e_tc, e_pl = (a - ref).abs()[band], (plain - ref).abs()[band]
    vol_ref = float(L.volume(ref, h, 1.5 * h).item())
    vol_tc = float(L.volume(a, h, 1.5 * h).item())
    return {"max_err_band_tc": float(e_tc.max()), "l2_err_band_tc": float(e_tc.pow(2).mean().sqrt()),
            "max_err_band_plain_fp32": float(e_pl.max()), "volume_rel_err_tc": abs(vol_tc - vol_ref) / vol_ref,
            "band_points": int(band.sum())}


def run_reference(args, rank, world):
    """--impl reference: the CPU implementation of the path on the host cores."""
    if rank != 0:
        return
    import torch
    h, phi, vel, dt, _ = workload(args.size, "cpu")
    threads = os.cpu_count() or 1
    nplanes = 16
    times, npts = [], 0
    for s in range(args.warmup + args.steps):
        r, npts, t = cpu_oracle_rate(phi, vel, h, dt_at(s, dt), nplanes=nplanes, threads=threads)
        if s >= args.warmup:
            times.append(t)
    # a step is one bounded sample of the 256^3 step (nplanes z-planes):
    # ms_per_step is the measured time of such a sample, value the rate over
    # all timed samples
    value = npts * len(times) / sum(times)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": sum(times) / len(times) * 1e3,
            "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"sphere r=0.15 in LeVeque deformation, {args.size}^3, tricubic, midpoint SL",
                       "sample": f"{nplanes} z-planes ({nplanes * args.size ** 2} points) per step; "
                                 "ms_per_step is the time of one such sample"},
            "cpu_baseline": {"value": value, "unit": "updates/s", "cores": threads, "kind": "port",
                             "sample": f"{nplanes} of {args.size} z-planes per step; the reference has no tricubic "
                                       "SL, so its FP64 restatement (oracle/sl_oracle.c) is timed"},
            "e2e": {"value": value, "unit": "updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--size", type=int, default=N_DEFAULT)
    ap.add_argument("--no-extras", action="store_true", help="skip comparators, e2e and CPU baseline")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    from dcell_b200 import levelset as L
    h, phi, vel, dt, _ = workload(args.size, dev)
    n = args.size ** 3
    K, W = args.steps, args.warmup

    with ClockSampler(local) as clk:
        ms_tc = timed_tc_split(L, torch, phi, vel, h, dt, K, W, dist)
    ms = ms_tc
    if dist:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = n * K * world / (ms / 1e3)

    hbm, bf16, src = peaks()
    t_launch = ms_tc / K / 1e3
    tflops = TC_FLOP_PER_UPDATE * n / t_launch / 1e12
    gbs = BYTES_PER_UPDATE * n / t_launch / 1e9
    traffic = profiled_traffic()
    line = {"metric": METRIC, "value": value, "unit": "updates/s", "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 (bf16 hi+lo split operands, f32 accumulate)", "data": "synthetic",
            "config": {"workload": f"sphere r=0.15 in LeVeque deformation field, {args.size}^3 dense, tricubic "
                                   "(split-BF16 tcgen05 coefficient GEMM, split-state stepping), midpoint SL "
                                   "backtrace, CFL 0.5",
                       "grid": [args.size] * 3, "points_per_step": n, "l2": "inputs 268 MB > 126 MB L2, no flush",
                       "parallelism": f"independent level set per GPU x{world}"},
            # the binding roofline: 16,384 split-BF16 tensor FLOP per update (M=1 row x N=64 x K=128)
            # take longer at peak than the 20 HBM bytes per update
            "roofline": {"bound": "tensor", "achieved": tflops, "peak": bf16, "unit": "TFLOP/s",
                         "frac": tflops / bf16, "traffic": traffic, "peak_source": src,
                         "flop_per_update": TC_FLOP_PER_UPDATE,
                         "hbm": {"achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm,
                                 "bytes_per_update": BYTES_PER_UPDATE}},
            "gpu_launches": K, "clocks": clk.summary()}

    if not args.no_extras:
        # CUDA-core comparators in both data paths: global gathers (one thread
        # per point) and the tensor-core stepper's TMA bricks (equal data
        # movement, evaluation on CUDA cores)
        ms_pl = timed_steps(L, torch, phi, vel, h, dt, "cubic_plain_gather", K, W)
        ms_sep = timed_steps(L, torch, phi, vel, h, dt, "cubic_separable_gather", K, W)
        ms_pl_b = timed_steps(L, torch, phi, vel, h, dt, "cubic_plain", K, W)
        ms_sep_b = timed_steps(L, torch, phi, vel, h, dt, "cubic_separable", K, W)
        ms_tc_unsplit = timed_steps(L, torch, phi, vel, h, dt, "cubic_tc", K, W)
        ms_lin = timed_steps(L, torch, phi, vel, h, dt, "linear", K, W)
        ms_lin_e = timed_steps(L, torch, phi, vel, h, dt, "linear", K, W, backtrace="euler")
        # the reference's own backtrace (AdvectSL.c:56-89: S = X - V dt / h)
        ms_tc_e = timed_tc_split(L, torch, phi, vel, h, dt, K, W, backtrace="euler")
        ms_pl_e = timed_steps(L, torch, phi, vel, h, dt, "cubic_plain_gather", K, W, backtrace="euler")
        ms_sep_e = timed_steps(L, torch, phi, vel, h, dt, "cubic_separable_gather", K, W, backtrace="euler")
        ms_sep_b_e = timed_steps(L, torch, phi, vel, h, dt, "cubic_separable", K, W, backtrace="euler")

        def hbm_leg(ms):  # one dense FP32 step: 20 algorithmic bytes per update
            t = ms / K / 1e3
            return {"updates_per_s": n / t, "ms_per_step": t * 1e3, "achieved_gbs": BYTES_PER_UPDATE * n / t / 1e9,
                    "hbm_frac": BYTES_PER_UPDATE * n / t / 1e9 / hbm}
        line["comparators"] = {
            "plain_fp32_updates_per_s": n * K / (ms_pl / 1e3),
            "separable_fp32_updates_per_s": n * K / (ms_sep / 1e3),
            "plain_fp32_brick_updates_per_s": n * K / (ms_pl_b / 1e3),
            "separable_fp32_brick_updates_per_s": n * K / (ms_sep_b / 1e3),
            "linear_fp32_updates_per_s": n * K / (ms_lin / 1e3),
            "tc_unsplit_state_updates_per_s": n * K / (ms_tc_unsplit / 1e3),
            "tc_over_plain_fp32": ms_pl / ms_tc,
            "tc_over_separable_fp32": ms_sep / ms_tc,
            "tc_over_plain_fp32_brick": ms_pl_b / ms_tc,
            "tc_over_separable_fp32_brick": ms_sep_b / ms_tc,
            "forms": "plain/separable: global-gather form (one thread per point, the scope's plain FP32 CUDA SL "
                     "step); *_brick: the same arithmetic on the tensor-core stepper's TMA-staged bricks",
            # the reference's own mode (trilinear, Euler backtrace) and its
            # midpoint form: TMA z-march, HBM-bound
            "linear_fp32": {"euler": hbm_leg(ms_lin_e), "midpoint": hbm_leg(ms_lin),
                            "kernel": "sl_lin_march_kernel"},
            # the same forms with the reference's own (Euler) backtrace
            "euler_backtrace": {"tc_ms_per_step": ms_tc_e / K, "plain_fp32_ms_per_step": ms_pl_e / K,
                                "separable_fp32_ms_per_step": ms_sep_e / K,
                                "separable_fp32_brick_ms_per_step": ms_sep_b_e / K,
                                "tc_over_plain_fp32": ms_pl_e / ms_tc_e, "tc_over_separable_fp32": ms_sep_e / ms_tc_e,
                                "tc_over_separable_fp32_brick": ms_sep_b_e / ms_tc_e}}
        line["accuracy"] = error_check(L, torch, phi, vel, h, dt)
        if world == 1:
            # the whole period of the field (t = 0 .. T): one-step error of the
            # TC step at every step and the accumulated error at t = T, vs FP64
            from dcell_b200.configs import run_c3
            c3 = run_c3(args.size, dev=dev)
            line["accuracy"]["period"] = {k: c3[k] for k in ("steps", "one_step_tc_vs_fp64",
                                                             "tc_meets_1e-5_every_step", "accumulated", "wall_s")}
        # end to end on every rank at once (the ranks share the host's memory
        # and PCIe); the slowest rank's rate sets the job's
        if dist:
            dist.barrier()
        e2e_rt, by = e2e_rate(phi, vel, h, dt, min(K, 5), torch)
        e2e, by_res = e2e_resident_rate(phi, vel, h, dt, 10, torch)
        if dist:
            t = torch.tensor([e2e, e2e_rt], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MIN)
            e2e, e2e_rt = float(t[0].item()), float(t[1].item())
        if rank == 0:
            # the headline end-to-end form: the reference's time loop with the
            # level set resident on the device; beside it the one-call round
            # trip of phi0 and velocity up, phi down (FP64 host buffers)
            line["e2e"] = {"value": e2e * world, "unit": "updates/s",
                           "h2d_bytes_per_step": by_res["h2d_bytes_per_step"],
                           "d2h_bytes_per_step": by_res["d2h_bytes_per_step"], "resident_loop": by_res,
                           "round_trip": {"value": e2e_rt * world, "unit": "updates/s", **by,
                                          "how": "dcell_ls_advect_sl (C ABI) on pinned FP64 host buffers, FP32 TC "
                                                 "compute, host clock around synchronous calls"},
                           "ranks": "every rank at once, the slowest rank's rate times the ranks"}
            if world == 1:
                rate, npts, t = cpu_oracle_rate(phi, vel, h, dt, nplanes=24, threads=1)
                line["cpu_baseline"] = {"value": rate, "unit": "updates/s", "cores": 1, "kind": "port",
                                        "sample": f"{npts} points (24 z-planes) of the 256^3 step, FP64 "
                                                  f"oracle restatement, {t:.1f} s"}
                ref_lin = reference_linear_rate(phi, vel, h, dt, nplanes=24)
                if ref_lin:
                    line["cpu_baseline"]["reference_linear_advectsl_updates_per_s"] = ref_lin
            if world == 1:
                line["c4"] = c4_rates(torch, dev)
            # narrow-band reinitialisation of the same sphere (cell units), GPU vs the reference's heap FMM
            rphi, rband, raw, count = reinit_case(torch, args.size, dev)
            ms64, y64, b64 = timed_reinit(torch, rphi, raw, count, torch.float64)
            ms32, _, _ = timed_reinit(torch, rphi, raw, count, torch.float32)
            line["reinit"] = {"grid": [args.size] * 3, "band_points": int(b64.shape[0]),
                              "seed_nodes": int(count.item()), "gpu_fp64_ms": ms64, "gpu_fp32_ms": ms32,
                              "how": "dcell_reinitialize: bucketed fast marching (buckets of 1/64 cell), band "
                                     "width 6, CUDA events, median of 5"}
            if world == 1:
                ref = reference_reinit(rphi, rband)
                if ref:
                    t, out, nb = ref
                    import numpy as np
                    got = y64.cpu().numpy()
                    inb = np.abs(out) < 6.0
                    d = np.abs(got - out)[inb]
                    line["cpu_baseline"]["reference_fmm_reinit"] = {
                        "ms": t * 1e3, "cores": 1, "band_points": nb, "kind": "reference",
                        "gpu_fp64_vs_reference": {"max": float(d.max()), "mean": float(d.mean())},
                        "gpu_fp64_speedup": t * 1e3 / ms64}
        if rank == 0:
            # velocity acquisition of 512 cells' boxes from a 512^3 fluid field (HBM-bound copy)
            from dcell_b200.configs import run_vel
            v = run_vel(dev=dev)
            v.update({"peak_gbs": hbm, "frac": v["achieved_gbs"] / hbm})
            line["velocity_acquisition"] = v
            # particle level set: ~3.5 M particles around the workload sphere, GPU FP32 vs the reference's FP64
            from dcell_b200.configs import pls_workload, run_pls
            wl = pls_workload(args.size, dev=dev)
            pr = run_pls(args.size, workload=wl, dev=dev)
            pr.update({"peak_gbs": hbm, "advect_frac": pr["advect_gbs"] / hbm})
            if world == 1:
                ref = reference_pls_step(*wl, 1.0 / args.size, 0.5 / args.size)
                if ref:
                    times, _ = ref
                    pr["reference_cpu"] = {**times, "cores": 1, "kind": "reference",
                                           "particle_updates_per_s": pr["particles"] / times["step_s"],
                                           "gpu_speedup": times["step_s"] * 1e3 / pr["ms_per_step"]}
            line["pls"] = pr
            del wl
            # output in the reference's formats: the stream's cost of a 256^3 snapshot and the drain to disk
            from dcell_b200.configs import run_io
            line["io"] = run_io(args.size)
            # the irregular-node pass that follows the step (projections, normals, curvature)
            from dcell_b200.configs import run_nodes
            nres, ncase = run_nodes(args.size, dev=dev, return_fp64=True)
            if world == 1:
                reference_nodes(nres, *ncase, 1.0 / args.size)
            line["irregular_nodes"] = nres
            # first-order upwind step on MAC faces (LevelSetAdvectMAC_3D), HBM-bound stencil
            from dcell_b200.configs import run_mac
            m, mcase = run_mac(args.size, dev=dev, return_fp64=True)
            for k in ("fp32", "fp64"):
                m[k]["frac"] = m[k]["achieved_gbs"] / hbm
            reference_mac(m, *mcase)
            line["advect_mac"] = m
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
