// Device helpers of the production semi-Lagrangian path (FP32 or FP64).
//
// The departure point is carried as an integer cell index plus a fractional
// offset in [0, 1): S = X + t with t = -V dt / h, cell = X + floor(t),
// frac = t - floor(t).  The fraction is therefore exact to the working
// precision of the displacement (not of the absolute coordinate), which is
// what keeps FP32 transport accurate on 256^3 grids.
#pragma once

#include "dcell_common.cuh"

namespace dcell {

// Index math of this path is 32-bit: the C ABI rejects grids with 3 * points
// >= 2^31.  Gathers take LOCAL indices (origin subtracted) and clamp only on
// the slow path, when a stencil touches the grid edge.

// Explicitly rounded arithmetic for the velocity interpolation, so every code
// path that interpolates the MAC field (global gathers, staged bricks,
// adjoint recomputation) produces the same bits whatever the compiler's
// contraction choices.
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float rsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double rsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float rfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double rfma(double a, double b, double c) { return __fma_rn(a, b, c); }

template <typename T>
__device__ __forceinline__ T face_mean(T a, T b) {
  return rfma(T(0.5), a, rmul(T(0.5), b));
}

// a + s (b - a): one subtraction and one fused multiply-add
template <typename T>
__device__ __forceinline__ T lerp(T a, T b, T s) {
  return rfma(s, rsub(b, a), a);
}

// bilinear in (x, y) of v[yx] with fractions s0, s1
template <typename T>
__device__ __forceinline__ T bilerp(T v00, T v10, T v01, T v11, T s0, T s1) {
  return lerp(lerp(v00, v10, s0), lerp(v01, v11, s0), s1);
}

template <typename T>
__device__ __forceinline__ T trilerp(T v000, T v100, T v010, T v110, T v001, T v101, T v011, T v111, const T s[3]) {
  return lerp(bilerp(v000, v100, v010, v110, s[0], s[1]), bilerp(v001, v101, v011, v111, s[0], s[1]), s[2]);
}

// MAC velocity at local node (x, y, z): each component is the mean of its two
// faces around the node -- InterpolateVelocity3D/2D
// (Common/InterpolateVelocity.c:35-67) at an integer point, where the
// off-axis trilinear weights vanish.
template <typename T, int DIM>
__device__ __forceinline__ void mac_vel_node(const Geom &g, const T *__restrict__ vel, int x, int y, int z, T V[3]) {
  const int q = (z * g.ny + y) * g.nx + x;
  const T *c = vel + DIM * q;
  const int dx = x + 1 < g.nx ? DIM : 0, dy = y + 1 < g.ny ? DIM * g.nx : 0;
  V[0] = face_mean(__ldg(c), __ldg(c + dx));
  V[1] = face_mean(__ldg(c + 1), __ldg(c + dy + 1));
  if (DIM == 3) {
    const int dz = z + 1 < g.nz ? 3 * g.nx * g.ny : 0;
    V[2] = face_mean(__ldg(c + 2), __ldg(c + dz + 2));
  } else {
    V[2] = T(0);
  }
}

// MAC velocity at local node + delta (|delta| small), trilinear per component
// with the component's half-cell stagger (Tensor1, Common/Common.h:26-30).
template <typename T, int DIM>
__device__ __forceinline__ void mac_vel_rel(const Geom &g, const T *__restrict__ vel, int x, int y, int z,
                                            const T dl[3], T V[3]) {
  const int X[3] = {x, y, z}, n[3] = {g.nx, g.ny, g.nz};
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    int b[3];
    T s[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      if (a == 2 && DIM == 2) { b[2] = 0; s[2] = T(0); continue; }
      const T t = dl[a] + (a == d ? T(0.5) : T(0));
      const T f = floor(t);
      b[a] = X[a] + (int)f;
      s[a] = t - f;
    }
    // offsets of the +1 neighbour per axis (0 when clamped at the upper edge)
    int o[3], bc[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      bc[a] = clampi(b[a], 0, n[a] - 1);
      const int up = clampi(b[a] + 1, 0, n[a] - 1) - bc[a];
      o[a] = up * (a == 0 ? DIM : a == 1 ? DIM * g.nx : DIM * g.nx * g.ny);
    }
    const T *c = vel + DIM * ((bc[2] * g.ny + bc[1]) * g.nx + bc[0]) + d;
    if (DIM == 3) {
      const T *c2 = c + o[2];
      V[d] = trilerp(__ldg(c), __ldg(c + o[0]), __ldg(c + o[1]), __ldg(c + o[1] + o[0]), __ldg(c2), __ldg(c2 + o[0]),
                     __ldg(c2 + o[1]), __ldg(c2 + o[1] + o[0]), s);
    } else {
      V[d] = bilerp(__ldg(c), __ldg(c + o[0]), __ldg(c + o[1]), __ldg(c + o[1] + o[0]), s[0], s[1]);
    }
  }
  if (DIM == 2) V[2] = T(0);
}

// Departure cell (LOCAL indices) and fraction for local arrival node (x, y, z).
// dth[a] = dt / h[a].  Returns true if the departure point left the grid.
template <typename T, int DIM>
__device__ __forceinline__ bool departure_cell(const Geom &g, const T *__restrict__ vel, const T dth[3], int backtrace,
                                               int x, int y, int z, int c[3], T f[3]) {
  T V[3];
  mac_vel_node<T, DIM>(g, vel, x, y, z, V);
  if (backtrace == DCELL_MIDPOINT) {  // products rounded explicitly: no path-dependent contraction
    const T dl[3] = {rmul(rmul(T(-0.5), V[0]), dth[0]), rmul(rmul(T(-0.5), V[1]), dth[1]),
                     DIM == 3 ? rmul(rmul(T(-0.5), V[2]), dth[2]) : T(0)};
    mac_vel_rel<T, DIM>(g, vel, x, y, z, dl, V);
  }
  const int X[3] = {x, y, z}, n[3] = {g.nx, g.ny, g.nz};
  bool out = false;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (a == 2 && DIM == 2) {
      c[2] = 0;
      f[2] = T(0);
      continue;
    }
    const T t = rmul(-V[a], dth[a]);
    const T fl = floor(t);
    c[a] = X[a] + (int)fl;
    f[a] = t - fl;
    out |= c[a] < 0 || c[a] + (f[a] > T(0) ? 1 : 0) > n[a] - 1;
  }
  return out;
}

// 4^3 (DIM 3) or 4^2 stencil of f around local cell c: s[x + 4y + 16z] =
// f[c - 1 + (x, y, z)], clamped to the grid.
template <typename T, int DIM>
__device__ __forceinline__ void gather_stencil(const Geom &g, const T *__restrict__ f, const int c[3], T *s) {
  const int x0 = c[0] - 1, y0 = c[1] - 1, z0 = DIM == 3 ? c[2] - 1 : 0;
  const int sy = g.nx, sz = g.nx * g.ny;
  const bool inside = x0 >= 0 && y0 >= 0 && x0 + 3 < g.nx && y0 + 3 < g.ny && (DIM == 2 || (z0 >= 0 && z0 + 3 < g.nz));
  if (inside) {
    const T *p = f + ((z0 * g.ny + y0) * g.nx + x0);
#pragma unroll
    for (int z = 0; z < (DIM == 3 ? 4 : 1); ++z)
#pragma unroll
      for (int y = 0; y < 4; ++y) {
        const T *r = p + z * sz + y * sy;
#pragma unroll
        for (int x = 0; x < 4; ++x) s[x + 4 * y + 16 * z] = __ldg(r + x);
      }
  } else {
    int xi[4], yo[4], zo[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      xi[i] = clampi(x0 + i, 0, g.nx - 1);
      yo[i] = clampi(y0 + i, 0, g.ny - 1) * sy;
      zo[i] = DIM == 3 ? clampi(z0 + i, 0, g.nz - 1) * sz : 0;
    }
#pragma unroll
    for (int z = 0; z < (DIM == 3 ? 4 : 1); ++z)
#pragma unroll
      for (int y = 0; y < 4; ++y)
#pragma unroll
        for (int x = 0; x < 4; ++x) s[x + 4 * y + 16 * z] = __ldg(f + zo[z] + yo[y] + xi[x]);
  }
}

// Catmull-Rom (Keys a = -1/2) cubic, the 1-D factor of the reference's
// TricubicInverse.h operator: rows = power 0..3, columns = offsets -1..2.
__host__ __device__ constexpr float cr_coef(int p, int s) {
  return p == 0 ? (s == 1 ? 1.f : 0.f)
       : p == 1 ? (s == 0 ? -0.5f : s == 2 ? 0.5f : 0.f)
       : p == 2 ? (s == 0 ? 1.f : s == 1 ? -2.5f : s == 2 ? 2.f : -0.5f)
                : (s == 0 ? -0.5f : s == 1 ? 1.5f : s == 2 ? -1.5f : 0.5f);
}

// Catmull-Rom weights of offsets -1..2 at fraction t: w = C^T [1 t t^2 t^3].
template <typename T>
__device__ __forceinline__ void cr_weights(T t, T w[4]) {
  const T t2 = t * t, t3 = t2 * t;
  w[0] = T(-0.5) * t + t2 - T(0.5) * t3;
  w[1] = T(1) - T(2.5) * t2 + T(1.5) * t3;
  w[2] = T(0.5) * t + T(2) * t2 - T(1.5) * t3;
  w[3] = T(-0.5) * t2 + T(0.5) * t3;
}

}  // namespace dcell
