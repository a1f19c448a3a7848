"""Synthetic level sets and MAC velocity fields of the benchmark workloads.

All fields live on cell-centred grids over [0,1]^d with N cells per axis:
cell i has its centre at x = (i + 1/2) h, h = 1/N.  MAC faces follow the
reference's staggering (Common/Common.h:26-30): the u value stored at index i
sits on the x-face i - 1/2 (physical x = i h), likewise v on y-faces and w on
z-faces.  Level sets are FP64 signed distances in physical units.

Workloads (no dataset is involved; everything is generated from formulas and
seeds):
  * Zalesak's slotted disk in a rigid rotation (2D),
  * a sphere in LeVeque's time-reversing deformation field (3D),
  * ellipsoids in divergence-free random Fourier velocities (batched cells),
  * a 16-mode Fourier velocity basis (differentiation workload).
"""
from __future__ import annotations

import math

import numpy as np
import torch


def _axes(N, dim, device, dtype=torch.float64):
    h = 1.0 / N
    c = (torch.arange(N, device=device, dtype=dtype) + 0.5) * h  # centres
    f = torch.arange(N, device=device, dtype=dtype) * h          # faces i - 1/2
    return h, c, f


def sphere_sdf(N, center=(0.35, 0.35, 0.35), r=0.15, device="cpu"):
    """(N, N, N) signed distance of a sphere (negative inside)."""
    h, c, _ = _axes(N, 3, device)
    z, y, x = torch.meshgrid(c, c, c, indexing="ij")
    return torch.sqrt((x - center[0]) ** 2 + (y - center[1]) ** 2 + (z - center[2]) ** 2) - r


def deformation_velocity(N, device="cpu"):
    """LeVeque's 3D deformation field without its cos(pi t / T) factor, on MAC
    faces: (N, N, N, 3) with [..., 0] = u at x-faces, 1 = v at y-faces,
    2 = w at z-faces.  Divergence-free; max |u| = 2, |v| = |w| = 1."""
    h, c, f = _axes(N, 3, device)
    s = torch.sin
    pi = math.pi
    vel = torch.empty((N, N, N, 3), dtype=torch.float64, device=device)
    z, y, x = torch.meshgrid(c, c, f, indexing="ij")
    vel[..., 0] = 2.0 * s(pi * x) ** 2 * s(2 * pi * y) * s(2 * pi * z)
    z, y, x = torch.meshgrid(c, f, c, indexing="ij")
    vel[..., 1] = -s(2 * pi * x) * s(pi * y) ** 2 * s(2 * pi * z)
    z, y, x = torch.meshgrid(f, c, c, indexing="ij")
    vel[..., 2] = -s(2 * pi * x) * s(2 * pi * y) * s(pi * z) ** 2
    return vel


def deformation_time_factor(t, T=3.0):
    return math.cos(math.pi * t / T)


def rotation_velocity_2d(N, device="cpu"):
    """Rigid rotation u = 2 pi (0.5 - y), v = 2 pi (x - 0.5) on MAC faces: (N, N, 2)."""
    h, c, f = _axes(N, 2, device)
    vel = torch.empty((N, N, 2), dtype=torch.float64, device=device)
    y, x = torch.meshgrid(c, f, indexing="ij")
    vel[..., 0] = 2 * math.pi * (0.5 - y)
    y, x = torch.meshgrid(f, c, indexing="ij")
    vel[..., 1] = 2 * math.pi * (x - 0.5)
    return vel


def _seg_dist(px, py, ax, ay, bx, by):
    dx, dy = bx - ax, by - ay
    t = ((px - ax) * dx + (py - ay) * dy) / (dx * dx + dy * dy)
    t = t.clamp(0.0, 1.0)
    return torch.sqrt((px - ax - t * dx) ** 2 + (py - ay - t * dy) ** 2)


def slotted_disk_sdf(N, center=(0.5, 0.75), r=0.15, width=0.05, depth=0.25, device="cpu"):
    """(N, N) exact signed distance of Zalesak's disk: a disk with a vertical
    slot of the given width cut `depth` deep from its bottom edge."""
    h, c, _ = _axes(N, 2, device)
    y, x = torch.meshgrid(c, c, indexing="ij")
    cx, cy = center
    xl, xr = cx - width / 2, cx + width / 2
    ytop = cy - r + depth
    y0 = cy - math.sqrt(r * r - (width / 2) ** 2)  # where the slot walls meet the circle
    rho = torch.sqrt((x - cx) ** 2 + (y - cy) ** 2)
    # nearest point of the full circle; valid unless it falls in the removed bottom arc
    qx = cx + r * (x - cx) / rho.clamp_min(1e-300)
    qy = cy + r * (y - cy) / rho.clamp_min(1e-300)
    removed = ((qx - cx).abs() < width / 2) & (qy < cy)
    d_end = torch.minimum(torch.sqrt((x - xl) ** 2 + (y - y0) ** 2), torch.sqrt((x - xr) ** 2 + (y - y0) ** 2))
    d_arc = torch.where(removed, d_end, (rho - r).abs())
    d = torch.minimum(d_arc, _seg_dist(x, y, xl, y0, xl, ytop))
    d = torch.minimum(d, _seg_dist(x, y, xr, y0, xr, ytop))
    d = torch.minimum(d, _seg_dist(x, y, xl, ytop, xr, ytop))
    inside = (rho < r) & ~(((x - cx).abs() < width / 2) & (y < ytop))
    return torch.where(inside, -d, d)


def cfl_dt(vmax_per_axis, h, cfl=0.5):
    """dt with the per-component CFL definition: cfl * h / max_a max|u_a|."""
    return cfl * h / max(vmax_per_axis)


def band_of(phi, width, origin=(0, 0, 0), margin=3):
    """(nb, 3) int32 global indices of points with |phi| < width, at least
    `margin` cells inside the grid, in x-fastest order."""
    dim = phi.dim()
    inner = torch.zeros_like(phi, dtype=torch.bool)
    sl = tuple(slice(margin, n - margin) for n in phi.shape)
    inner[sl] = True
    sel = inner & (phi.abs() < width)
    idx = torch.nonzero(sel)  # (nb, dim) in (z, y, x) order, lexicographic = x fastest
    if dim == 2:
        b = torch.stack([idx[:, 1] + origin[0], idx[:, 0] + origin[1], torch.zeros_like(idx[:, 0])], dim=1)
    else:
        b = torch.stack([idx[:, 2] + origin[0], idx[:, 1] + origin[1], idx[:, 0] + origin[2]], dim=1)
    return b.to(torch.int32).contiguous()


# ---------------------------------------------------------------------------
# divergence-free Fourier velocities (batched cells, differentiation)
def fourier_modes(nmodes, seed, kmin=1, kmax=4):
    """Random modes: integer wave vectors k in [kmin, kmax]^3 (random signs),
    unit vector-potential directions and phases."""
    rng = np.random.default_rng(seed)
    k = rng.integers(kmin, kmax + 1, size=(nmodes, 3)) * rng.choice([-1, 1], size=(nmodes, 3))
    a = rng.normal(size=(nmodes, 3))
    a /= np.linalg.norm(a, axis=1, keepdims=True)
    ph = rng.uniform(0, 2 * np.pi, size=nmodes)
    return k.astype(np.float64), a, ph


def fourier_velocity(shape, coeffs, modes, device="cpu", dtype=torch.float64):
    """MAC velocity = discrete curl of the edge-centred vector potential
    A(x) = sum_m c_m a_m sin(2 pi k_m . x + phase_m) on the box [0,1]^3 of the
    cell grid `shape` (nz, ny, nx): discretely divergence-free by construction.
    Returns (nz, ny, nx, 3)."""
    nz, ny, nx = shape
    hx, hy, hz = 1.0 / nx, 1.0 / ny, 1.0 / nz
    k, a, ph = modes
    xc = (torch.arange(nx, device=device, dtype=torch.float64) + 0.5) * hx
    yc = (torch.arange(ny, device=device, dtype=torch.float64) + 0.5) * hy
    zc = (torch.arange(nz, device=device, dtype=torch.float64) + 0.5) * hz
    xf, yf, zf = xc - 0.5 * hx, yc - 0.5 * hy, zc - 0.5 * hz

    def A(comp, X, Y, Z):
        out = torch.zeros(torch.broadcast_shapes(X.shape, Y.shape, Z.shape), dtype=torch.float64, device=device)
        for m in range(len(ph)):
            arg = 2 * math.pi * (k[m, 0] * X + k[m, 1] * Y + k[m, 2] * Z) + ph[m]
            out = out + float(coeffs[m]) * float(a[m, comp]) * torch.sin(arg)
        return out

    def grid(xs, ys, zs):
        Z, Y, X = torch.meshgrid(zs, ys, xs, indexing="ij")
        return X, Y, Z

    vel = torch.empty((nz, ny, nx, 3), dtype=torch.float64, device=device)
    # u at (xf, yc, zc) = dAz/dy - dAy/dz with Az on z-edges (xf, yf, zc), Ay on y-edges (xf, yc, zf)
    X, Y, Z = grid(xf, yc, zc)
    vel[..., 0] = (A(2, X, Y + 0.5 * hy, Z) - A(2, X, Y - 0.5 * hy, Z)) / hy - \
                  (A(1, X, Y, Z + 0.5 * hz) - A(1, X, Y, Z - 0.5 * hz)) / hz
    # v at (xc, yf, zc) = dAx/dz - dAz/dx
    X, Y, Z = grid(xc, yf, zc)
    vel[..., 1] = (A(0, X, Y, Z + 0.5 * hz) - A(0, X, Y, Z - 0.5 * hz)) / hz - \
                  (A(2, X + 0.5 * hx, Y, Z) - A(2, X - 0.5 * hx, Y, Z)) / hx
    # w at (xc, yc, zf) = dAy/dx - dAx/dy
    X, Y, Z = grid(xc, yc, zf)
    vel[..., 2] = (A(1, X + 0.5 * hx, Y, Z) - A(1, X - 0.5 * hx, Y, Z)) / hx - \
                  (A(0, X, Y + 0.5 * hy, Z) - A(0, X, Y - 0.5 * hy, Z)) / hy
    return vel.to(dtype)


def ellipsoid_sdf(shape, center, semi, device="cpu", dtype=torch.float64):
    """Approximate signed distance of an axis-aligned ellipsoid on the cell
    grid of `shape` over [0,1]^3: (|x/a| - 1) * min(a), exact on the surface
    and along the axes."""
    nz, ny, nx = shape
    xs = (torch.arange(nx, device=device, dtype=torch.float64) + 0.5) / nx
    ys = (torch.arange(ny, device=device, dtype=torch.float64) + 0.5) / ny
    zs = (torch.arange(nz, device=device, dtype=torch.float64) + 0.5) / nz
    Z, Y, X = torch.meshgrid(zs, ys, xs, indexing="ij")
    q = torch.sqrt(((X - center[0]) / semi[0]) ** 2 + ((Y - center[1]) / semi[1]) ** 2 +
                   ((Z - center[2]) / semi[2]) ** 2)
    return ((q - 1.0) * min(semi)).to(dtype)
