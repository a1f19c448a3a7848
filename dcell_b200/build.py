"""Build the sm_100a shared library ``dcell_b200/lib/libdcell_ls.so``.

Every CUDA translation unit under ``dcell_b200/csrc`` is compiled with
``nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo`` and linked into one
C-ABI shared library (static CUDA runtime, so it loads on machines without a
GPU; kernels need a B200 to run).  ``sl_exact.cu`` and ``pls.cu`` are
compiled with ``-fmad=false`` so their FP64 kernels keep the reference's
one-rounding-per-operation arithmetic.

    python -m dcell_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libdcell_ls.so")
INCLUDE = os.path.join(os.path.dirname(PKG), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden", "-I", INCLUDE,
          "-I", CSRC, "--expt-relaxed-constexpr"]
# Kernels that keep tcgen05.ld results in flight across other code (the
# loaded registers are only valid after the tied tcgen05.wait::ld): the build
# fails if ptxas spills any of their registers, since a spill store placed
# between a load and its wait would save a register that is not yet written.
NO_SPILL = {"sl_tc.cu": ["sl_tc_brick_kernel"]}

UNITS = {
    "sl_exact.cu": ["-fmad=false"],
    "sl_lin.cu": [],
    "sl_cubic.cu": [],
    "sl_tc.cu": [],
    "sl_adjoint.cu": [],
    "velocity.cu": [],
    "pls.cu": ["-fmad=false"],
    "writer.cu": [],
    "capi.cu": [],
}


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build dcell_b200")


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _spilling(ptxas_log, names):
    """Kernels of `names` whose ptxas report shows spill stores or loads."""
    bad, cur = [], None
    for ln in ptxas_log.splitlines():
        if "Compiling entry function" in ln:
            cur = next((n for n in names if n in ln), None)
        elif cur and "spill stores" in ln:
            parts = ln.replace(",", "").split()
            stores = int(parts[parts.index("spill") - 2])
            loads = int(parts[parts.index("loads") - 3])
            if stores or loads:
                bad.append(cur)
            cur = None
    return sorted(set(bad))


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> str:
    """Compile all translation units and link the shared library; returns its path."""
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(LIBDIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h", ".inc"))]
    headers.append(os.path.join(INCLUDE, "dcell_ls.h"))
    objs = []
    cc = nvcc()
    for unit, extra in UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(objdir, unit.replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, [src] + headers + [__file__]):
            guard = NO_SPILL.get(unit)
            cmd = [cc] + ARCH + COMMON + extra + (["-Xptxas", "-v"] if ptxas_verbose or guard else []) + \
                ["-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            r = subprocess.run(cmd, stderr=subprocess.PIPE, text=True)
            if ptxas_verbose or r.returncode:
                sys.stderr.write(r.stderr)
            if r.returncode:
                raise subprocess.CalledProcessError(r.returncode, cmd)
            if guard:
                bad = _spilling(r.stderr, guard)
                if bad:
                    os.remove(obj)
                    raise RuntimeError(f"{unit}: ptxas spilled registers of {', '.join(bad)}")
    if force or _stale(LIB, objs):
        cmd = [cc] + ARCH + ["-shared", "-cudart", "static", "-Xcompiler", "-fPIC", "-o", LIB] + objs
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print register/smem usage per kernel")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose, ptxas_verbose=a.ptxas))
    sys.exit(0)
