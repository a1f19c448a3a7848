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

// MAC velocity at integer node (x, y, z): each component is the mean of its
// two faces around the node -- InterpolateVelocity3D/2D
// (Common/InterpolateVelocity.c:35-67) at an integer point, where the
// off-axis trilinear weights vanish.
template <typename T, int DIM>
__device__ __forceinline__ void mac_vel_node(const Geom &g, const T *__restrict__ vel, int x, int y, int z, T V[3]) {
  if (DIM == 3) {
    V[0] = T(0.5) * vel[gidx(g, x, y, z) * 3 + 0] + T(0.5) * vel[gidx(g, x + 1, y, z) * 3 + 0];
    V[1] = T(0.5) * vel[gidx(g, x, y, z) * 3 + 1] + T(0.5) * vel[gidx(g, x, y + 1, z) * 3 + 1];
    V[2] = T(0.5) * vel[gidx(g, x, y, z) * 3 + 2] + T(0.5) * vel[gidx(g, x, y, z + 1) * 3 + 2];
  } else {
    V[0] = T(0.5) * vel[gidx(g, x, y, 0) * 2 + 0] + T(0.5) * vel[gidx(g, x + 1, y, 0) * 2 + 0];
    V[1] = T(0.5) * vel[gidx(g, x, y, 0) * 2 + 1] + T(0.5) * vel[gidx(g, x, y + 1, 0) * 2 + 1];
    V[2] = T(0);
  }
}

// MAC velocity at node + delta (|delta| small), trilinear per component with
// the component's half-cell stagger (Tensor1, Common/Common.h:26-30).
template <typename T, int DIM>
__device__ __forceinline__ void mac_vel_rel(const Geom &g, const T *__restrict__ vel, int x, int y, int z,
                                            const T dl[3], T V[3]) {
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    int b[3];
    T s[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const T t = dl[a] + (a == d ? T(0.5) : T(0));
      const T f = floor(t);
      b[a] = (a == 0 ? x : a == 1 ? y : z) + (int)f;
      s[a] = t - f;
    }
    T sum = 0;
    if (DIM == 3) {
#pragma unroll
      for (int k = 0; k < 2; ++k)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
          for (int i = 0; i < 2; ++i) {
            const T w = (i ? s[0] : 1 - s[0]) * (j ? s[1] : 1 - s[1]) * (k ? s[2] : 1 - s[2]);
            sum += w * vel[gidx(g, b[0] + i, b[1] + j, b[2] + k) * 3 + d];
          }
    } else {
#pragma unroll
      for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const T w = (i ? s[0] : 1 - s[0]) * (j ? s[1] : 1 - s[1]);
          sum += w * vel[gidx(g, b[0] + i, b[1] + j, 0) * 2 + d];
        }
    }
    V[d] = sum;
  }
  if (DIM == 2) V[2] = T(0);
}

// Departure cell (global indices) and fraction for arrival node (x, y, z).
// dth[a] = dt / h[a].  Returns true if the departure point left the grid.
template <typename T, int DIM>
__device__ __forceinline__ bool departure_cell(const Geom &g, const T *__restrict__ vel, const T dth[3], int backtrace,
                                               int x, int y, int z, int c[3], T f[3]) {
  T V[3];
  mac_vel_node<T, DIM>(g, vel, x, y, z, V);
  if (backtrace == DCELL_MIDPOINT) {
    const T dl[3] = {T(-0.5) * V[0] * dth[0], T(-0.5) * V[1] * dth[1], DIM == 3 ? T(-0.5) * V[2] * dth[2] : T(0)};
    mac_vel_rel<T, DIM>(g, vel, x, y, z, dl, V);
  }
  const int X[3] = {x, y, z};
  bool out = false;
  const int lo[3] = {g.px, g.py, g.pz}, n[3] = {g.nx, g.ny, g.nz};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (a == 2 && DIM == 2) {
      c[2] = z;
      f[2] = T(0);
      continue;
    }
    const T t = -V[a] * dth[a];
    const T fl = floor(t);
    c[a] = X[a] + (int)fl;
    f[a] = t - fl;
    out |= c[a] < lo[a] || c[a] + (f[a] > T(0) ? 1 : 0) > lo[a] + n[a] - 1;
  }
  return out;
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
