// Adjoint of the dense 3D semi-Lagrangian step (FP32 or FP64).
//
// Forward (per arrival node X, index space):
//   phi1[X] = I(phi0; S),   S = X + t,   t_a = -(dt/h_a) U_a,
//   U = V(X)                         (Euler: mean of the two MAC faces)
//   U = V(Xm), Xm = X + d, d_a = -(dt/2h_a) V_a(X)   (midpoint; trilinear MAC)
// with I the trilinear or Catmull-Rom tricubic interpolant (the forward of
// dcell_sl_step for DCELL_LINEAR / the three cubic modes, which share one
// interpolant).  Given gbar = dL/dphi1 the kernel accumulates
//   dL/dphi0[c + o] += gbar[X] w_o(S)                    (transpose scatter)
//   dL/dU_a = gbar[X] dI/dS_a(S) (-dt/h_a)                (departure point)
//   dL/du  += dU/du^T dL/dU  through V(X) (Euler) or V(Xm) and, for the
//            midpoint, through Xm's dependence on V(X).
// Accumulation uses global atomics (RED): results agree with any ordering to
// rounding but are not bitwise reproducible in FP32.  Floors of the
// departure cell are treated as constants (the interpolants are continuous,
// the tricubic one C1).
#include "dcell_common.cuh"
#include "dcell_kernels.h"
#include "sl_device.cuh"

namespace dcell {

template <typename T>
__device__ __forceinline__ void cr_dweights(T t, T w[4]) {  // d/dt of cr_weights
  const T t2 = t * t;
  w[0] = T(-0.5) + T(2) * t - T(1.5) * t2;
  w[1] = T(-5) * t + T(4.5) * t2;
  w[2] = T(0.5) + T(4) * t - T(4.5) * t2;
  w[3] = T(-1) * t + T(1.5) * t2;
}

// 1-D weights (and derivatives) of the interpolant: cubic uses offsets -1..2,
// linear offsets 0..1 placed in slots 1..2.
template <typename T, bool CUBIC>
__device__ __forceinline__ void weights(T t, T w[4], T dw[4]) {
  if (CUBIC) {
    cr_weights<T>(t, w);
    cr_dweights<T>(t, dw);
  } else {
    w[0] = T(0); w[1] = 1 - t; w[2] = t; w[3] = T(0);
    dw[0] = T(0); dw[1] = T(-1); dw[2] = T(1); dw[3] = T(0);
  }
}

__device__ __forceinline__ void atomic_add(float *p, float v) { atomicAdd(p, v); }
__device__ __forceinline__ void atomic_add(double *p, double v) { atomicAdd(p, v); }

// Trilinear MAC interpolation of component d at node + dl, its weights'
// gradient wrt position, and the 8 face indices (clamped).
template <typename T>
__device__ __forceinline__ T mac_component(const Geom &g, const T *__restrict__ vel, int x, int y, int z, int d,
                                           const T dl[3], T grad[3], int idx[8], T w8[8]) {
  const int X[3] = {x, y, z}, n[3] = {g.nx, g.ny, g.nz};
  int b[3];
  T s[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const T t = dl[a] + (a == d ? T(0.5) : T(0));
    const T f = floor(t);
    b[a] = X[a] + (int)f;
    s[a] = t - f;
  }
  T val = 0, gx = 0, gy = 0, gz = 0;
#pragma unroll
  for (int k = 0; k < 2; ++k)
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int q = (clampi(b[2] + k, 0, n[2] - 1) * g.ny + clampi(b[1] + j, 0, n[1] - 1)) * g.nx +
                      clampi(b[0] + i, 0, n[0] - 1);
        const T wx = i ? s[0] : 1 - s[0], wy = j ? s[1] : 1 - s[1], wz = k ? s[2] : 1 - s[2];
        const T v = vel[3 * q + d];
        const int e = i + 2 * j + 4 * k;
        idx[e] = 3 * q + d;
        w8[e] = wx * wy * wz;
        val += w8[e] * v;
        gx += (i ? T(1) : T(-1)) * wy * wz * v;
        gy += wx * (j ? T(1) : T(-1)) * wz * v;
        gz += wx * wy * (k ? T(1) : T(-1)) * v;
      }
  grad[0] = gx; grad[1] = gy; grad[2] = gz;
  return val;
}

template <typename T, bool CUBIC>
__global__ void __launch_bounds__(256) sl_adjoint_kernel(Geom g, const T *__restrict__ phi0, const T *__restrict__ vel,
                                                         T dt, int backtrace, const T *__restrict__ gphi,
                                                         T *__restrict__ gphi0, T *__restrict__ gvel) {
  const long long npts = (long long)g.nx * g.ny * g.nz;
  const T dth[3] = {dt / (T)g.hx, dt / (T)g.hy, dt / (T)g.hz};
  const int sy = g.nx, sz = g.nx * g.ny;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < npts;
       q += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(q % g.nx), y = (int)((q / g.nx) % g.ny), z = (int)(q / sz);
    const T gb = gphi[q];
    if (gb == T(0)) continue;
    // ---- forward recomputation of the departure point
    T V0[3];
    mac_vel_node<T, 3>(g, vel, x, y, z, V0);
    T U[3] = {V0[0], V0[1], V0[2]};
    T dl[3] = {0, 0, 0}, J[3][3];  // J[a][b] = dU_a / dXm_b (midpoint)
    int idx[3][8];
    T w8[3][8];
    if (backtrace == DCELL_MIDPOINT) {
#pragma unroll
      for (int a = 0; a < 3; ++a) dl[a] = T(-0.5) * V0[a] * dth[a];
#pragma unroll
      for (int a = 0; a < 3; ++a) U[a] = mac_component<T>(g, vel, x, y, z, a, dl, J[a], idx[a], w8[a]);
    }
    int c[3];
    T f[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const T t = -U[a] * dth[a];
      const T fl = floor(t);
      c[a] = (a == 0 ? x : a == 1 ? y : z) + (int)fl;
      f[a] = t - fl;
    }
    T wx[4], wy[4], wz[4], dwx[4], dwy[4], dwz[4];
    weights<T, CUBIC>(f[0], wx, dwx);
    weights<T, CUBIC>(f[1], wy, dwy);
    weights<T, CUBIC>(f[2], wz, dwz);
    // ---- transpose scatter into dL/dphi0 and the interpolant's gradient
    int xi[4], yo[4], zo[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      xi[i] = clampi(c[0] - 1 + i, 0, g.nx - 1);
      yo[i] = clampi(c[1] - 1 + i, 0, g.ny - 1) * sy;
      zo[i] = clampi(c[2] - 1 + i, 0, g.nz - 1) * sz;
    }
    T gS[3] = {0, 0, 0};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (!CUBIC && (k == 0 || k == 3)) continue;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        if (!CUBIC && (j == 0 || j == 3)) continue;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          if (!CUBIC && (i == 0 || i == 3)) continue;
          const int p = zo[k] + yo[j] + xi[i];
          atomic_add(gphi0 + p, gb * wx[i] * wy[j] * wz[k]);
          const T v = phi0[p];
          gS[0] += dwx[i] * wy[j] * wz[k] * v;
          gS[1] += wx[i] * dwy[j] * wz[k] * v;
          gS[2] += wx[i] * wy[j] * dwz[k] * v;
        }
      }
    }
    // ---- velocity sensitivity: dL/dU_a = gb dI/dS_a (-dt/h_a)
    T gU[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) gU[a] = gb * gS[a] * (-dth[a]);
    T gV0[3] = {gU[0], gU[1], gU[2]};  // Euler: U = V(X)
    if (backtrace == DCELL_MIDPOINT) {
      // U_a = sum_e w8[a][e] u_a[idx[a][e]]
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int e = 0; e < 8; ++e) atomic_add(gvel + idx[a][e], gU[a] * w8[a][e]);
      // through Xm = X + d(V(X)):  dL/dd_b = sum_a gU_a J[a][b];  d_b = -(dt/2h_b) V0_b
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        T acc = 0;
#pragma unroll
        for (int a = 0; a < 3; ++a) acc += gU[a] * J[a][b];
        gV0[b] = acc * (T(-0.5) * dth[b]);
      }
    }
    if (backtrace == DCELL_EULER || backtrace == DCELL_MIDPOINT) {
      // V0_a = (u_a[node] + u_a[node + e_a]) / 2  (upper face clamped at the edge)
      const int qn = (z * g.ny + y) * g.nx + x;
      const int up[3] = {x + 1 < g.nx ? 1 : 0, y + 1 < g.ny ? g.nx : 0, z + 1 < g.nz ? sz : 0};
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        atomic_add(gvel + 3 * qn + a, T(0.5) * gV0[a]);
        atomic_add(gvel + 3 * (qn + up[a]) + a, T(0.5) * gV0[a]);
      }
    }
  }
}

}  // namespace dcell

using namespace dcell;

int launch_sl_adjoint(const Geom &g, int dtype, const void *phi0, const void *vel, double dt, int interp,
                      int backtrace, const void *gphi, void *gphi0, void *gvel, cudaStream_t st) {
  const long long n = (long long)g.nx * g.ny * g.nz;
  long long blocks = (n + 255) / 256;
  if (blocks > 148LL * 16) blocks = 148LL * 16;
  const bool cubic = interp != DCELL_LINEAR;
  if (dtype == DCELL_F64) {
    if (cubic)
      sl_adjoint_kernel<double, true><<<(int)blocks, 256, 0, st>>>(g, (const double *)phi0, (const double *)vel, dt,
                                                                   backtrace, (const double *)gphi, (double *)gphi0,
                                                                   (double *)gvel);
    else
      sl_adjoint_kernel<double, false><<<(int)blocks, 256, 0, st>>>(g, (const double *)phi0, (const double *)vel, dt,
                                                                    backtrace, (const double *)gphi, (double *)gphi0,
                                                                    (double *)gvel);
  } else {
    if (cubic)
      sl_adjoint_kernel<float, true><<<(int)blocks, 256, 0, st>>>(g, (const float *)phi0, (const float *)vel,
                                                                  (float)dt, backtrace, (const float *)gphi,
                                                                  (float *)gphi0, (float *)gvel);
    else
      sl_adjoint_kernel<float, false><<<(int)blocks, 256, 0, st>>>(g, (const float *)phi0, (const float *)vel,
                                                                   (float)dt, backtrace, (const float *)gphi,
                                                                   (float *)gphi0, (float *)gvel);
  }
  return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
}
