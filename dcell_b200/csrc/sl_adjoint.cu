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
// Accumulation uses global atomics (RED), one per lane and target by
// default.  The warp-aggregated form is built too (DCELL_ADJOINT_AGGREGATE =
// phi, vel or all): a warp's 32 lanes are consecutive arrival points of one
// grid row, and wherever the departure (or midpoint) cells of its
// contributing lanes are one row of consecutive cells, the contributions
// that land on one target -- the stencils of neighbouring lanes overlap in
// x -- are summed with shuffles first (a sliding window along the row), so
// each target of a stencil row gets one atomic per warp instead of one per
// lane: 35 instead of 128 per row of a tricubic stencil.  Other warps add per
// lane.  On the 128^3 differentiation workload the shuffles cost more than
// the atomics they save (FP32 backward 13.9 ms per lane, 15.9 ms
// aggregated), hence the default.  Results agree with any ordering to
// rounding but are not bitwise reproducible.  Floors of the departure cell
// are treated as constants (the interpolants are continuous, the tricubic
// one C1).
#include <stdlib.h>

#include <string>

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

constexpr unsigned kFull = 0xffffffffu;

// Warp-aggregated scatter of one stencil row.  Lane L holds v[i] (i < W) for
// the targets m = L + i of a row whose target m lives at dst + stride *
// clamp(m0 + m, 0, n - 1), dst and m0 the same in every lane: the sliding
// sums value(m) = sum_i v[i](lane m - i) for m = 0 .. 31 + W - 1 go out as
// one atomic each (lane m adds value(m); lanes 0 .. W - 2 add the tail m =
// 32 + lane), zero sums skipped.  Called by the whole warp.
template <int W, typename T>
__device__ __forceinline__ void warp_row_scatter(const T v[W], T *dst, int m0, int n, int stride, int lane) {
  T s = v[0];
#pragma unroll
  for (int i = 1; i < W; ++i) {
    const T u = __shfl_up_sync(kFull, v[i], i);
    if (lane >= i) s += u;
  }
  if (s != T(0)) atomic_add(dst + (long long)stride * clampi(m0 + lane, 0, n - 1), s);
  T t = T(0);
#pragma unroll
  for (int i = 1; i < W; ++i) {  // value(32 + lane) = sum_{i > lane} v[i](lane 32 + lane - i)
    const int src = 32 + lane - i;
    const T u = __shfl_sync(kFull, v[i], src & 31);
    if (src <= 31) t += u;
  }
  if (lane < W - 1 && t != T(0)) atomic_add(dst + (long long)stride * clampi(m0 + 32 + lane, 0, n - 1), t);
}

// Whether the contributing lanes (active) of the warp share the values a, b
// and have c - lane equal (their cells are consecutive along the row); the
// common c - lane goes to c0.
__device__ __forceinline__ bool warp_row(unsigned active, int a, int b, int c, int lane, int &c0) {
  const int ref = __ffs(active) - 1;
  const int ra = __shfl_sync(kFull, a, ref), rb = __shfl_sync(kFull, b, ref);
  c0 = __shfl_sync(kFull, c - lane, ref);
  const bool ok = !((active >> lane) & 1u) || (a == ra && b == rb && c - lane == c0);
  return __all_sync(kFull, ok);
}

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

// AGG_PHI / AGG_VEL: warp-aggregate the dL/dphi0 / the velocity scatters
// (per-lane atomics otherwise).
template <typename T, bool CUBIC, bool AGG_PHI, bool AGG_VEL>
__global__ void __launch_bounds__(256) sl_adjoint_kernel(Geom g, const T *__restrict__ phi0, const T *__restrict__ vel,
                                                         T dt, int backtrace, const T *__restrict__ gphi,
                                                         T *__restrict__ gphi0, T *__restrict__ gvel) {
  const long long npts = (long long)g.nx * g.ny * g.nz;
  const T dth[3] = {dt / (T)g.hx, dt / (T)g.hy, dt / (T)g.hz};
  const int sy = g.nx, sz = g.nx * g.ny;
  const int lane = threadIdx.x & 31;
  // whole warps step together (the scatters are warp-collective); lanes past
  // the grid's end compute the last point and contribute nothing
  for (long long wq = blockIdx.x * (long long)blockDim.x + threadIdx.x - lane; wq < npts;
       wq += (long long)gridDim.x * blockDim.x) {
    const long long q = wq + lane < npts ? wq + lane : npts - 1;
    const int x = (int)(q % g.nx), y = (int)((q / g.nx) % g.ny), z = (int)(q / sz);
    const T gb = wq + lane < npts ? gphi[q] : T(0);
    const unsigned active = __ballot_sync(kFull, gb != T(0));
    if (!active) continue;
    const bool on = (active >> lane) & 1u;  // this lane contributes
    const int ref = __ffs(active) - 1;      // a contributing lane: rows of the warp-wide scatters
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
    int xi[4], yo[4], zo[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      xi[i] = clampi(c[0] - 1 + i, 0, g.nx - 1);
      yo[i] = clampi(c[1] - 1 + i, 0, g.ny - 1) * sy;
      zo[i] = clampi(c[2] - 1 + i, 0, g.nz - 1) * sz;
    }
    // ---- the interpolant's gradient at S
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
          const T v = phi0[zo[k] + yo[j] + xi[i]];
          gS[0] += dwx[i] * wy[j] * wz[k] * v;
          gS[1] += wx[i] * dwy[j] * wz[k] * v;
          gS[2] += wx[i] * wy[j] * dwz[k] * v;
        }
      }
    }
    // ---- transpose scatter into dL/dphi0
    constexpr int I0 = CUBIC ? 0 : 1, W = CUBIC ? 4 : 2;
    int cx0;
    if (AGG_PHI && warp_row(active, c[1], c[2], c[0], lane, cx0)) {
#pragma unroll
      for (int k = I0; k < I0 + W; ++k)
#pragma unroll
        for (int j = I0; j < I0 + W; ++j) {
          T v[W];
#pragma unroll
          for (int i = 0; i < W; ++i) v[i] = on ? gb * wx[I0 + i] * wy[j] * wz[k] : T(0);
          warp_row_scatter<W, T>(v, gphi0 + __shfl_sync(kFull, zo[k] + yo[j], ref), cx0 - 1 + I0, g.nx, 1, lane);
        }
    } else if (on) {
#pragma unroll
      for (int k = I0; k < I0 + W; ++k)
#pragma unroll
        for (int j = I0; j < I0 + W; ++j)
#pragma unroll
          for (int i = I0; i < I0 + W; ++i) atomic_add(gphi0 + zo[k] + yo[j] + xi[i], gb * wx[i] * wy[j] * wz[k]);
    }
    // ---- velocity sensitivity: dL/dU_a = gb dI/dS_a (-dt/h_a)
    T gU[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) gU[a] = gb * gS[a] * (-dth[a]);
    T gV0[3] = {gU[0], gU[1], gU[2]};  // Euler: U = V(X)
    if (backtrace == DCELL_MIDPOINT) {
      // U_a = sum_e w8[a][e] u_a[idx[a][e]], e = i + 2j + 4k over the 2^3
      // corners of the midpoint cell b_a (x of corner i of lane L at
      // idx / 3 % nx = clamp(b_a.x + i))
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const int q0 = idx[a][0] / 3;  // corner (0, 0, 0), clamped
        const int bx = q0 % g.nx, byz = q0 / g.nx;
        const int byz11 = idx[a][6] / 3 / g.nx;  // row of corner (0, 1, 1), clamped
        const int bxu = (idx[a][1] / 3) % g.nx;  // corner (1, 0, 0): bx + 1 clamped
        int bx0;
        // one row when the contributing lanes share the corner rows and their
        // corners are consecutive, unclamped cells.  The rows of corners
        // (0, 0, 0) and (0, 1, 1) fix clamp(by), clamp(by + 1), clamp(bz)
        // and clamp(bz + 1), hence all four corner rows: at a y or z edge
        // lanes whose midpoint cells differ there can share the first row
        // alone.
        const bool interior = bxu == bx + 1;
        if (AGG_VEL && __all_sync(kFull, interior || !on) && warp_row(active, byz, byz11, bx, lane, bx0)) {
#pragma unroll
          for (int jk = 0; jk < 4; ++jk) {
            const T v[2] = {on ? gU[a] * w8[a][2 * jk] : T(0), on ? gU[a] * w8[a][2 * jk + 1] : T(0)};
            const int row = idx[a][2 * jk] / 3 - bx;  // corner (0, j, k) row start, this lane
            warp_row_scatter<2, T>(v, gvel + 3 * (long long)__shfl_sync(kFull, row, ref) + a, bx0, g.nx, 3, lane);
          }
        } else if (on) {
#pragma unroll
          for (int e = 0; e < 8; ++e) atomic_add(gvel + idx[a][e], gU[a] * w8[a][e]);
        }
      }
      // through Xm = X + d(V(X)):  dL/dd_b = sum_a gU_a J[a][b];  d_b = -(dt/2h_b) V0_b
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        T acc = 0;
#pragma unroll
        for (int a = 0; a < 3; ++a) acc += gU[a] * J[a][b];
        gV0[b] = acc * (T(-0.5) * dth[b]);
      }
    }
    // V0_a = (u_a[node] + u_a[node + e_a]) / 2  (upper face clamped at the edge):
    // the u faces of a row of nodes overlap between neighbouring lanes
    const int qn = (z * g.ny + y) * g.nx + x;
    const int up[3] = {x + 1 < g.nx ? 1 : 0, y + 1 < g.ny ? g.nx : 0, z + 1 < g.nz ? sz : 0};
    int x0;
    if (AGG_VEL && warp_row(active, y, z, x, lane, x0)) {
      const T hv = on ? T(0.5) * gV0[0] : T(0);
      const T v[2] = {hv, hv};
      warp_row_scatter<2, T>(v, gvel + 3 * (long long)__shfl_sync(kFull, (z * g.ny + y) * g.nx, ref), x0, g.nx, 3,
                             lane);
    } else if (on) {
      atomic_add(gvel + 3 * qn, T(0.5) * gV0[0]);
      atomic_add(gvel + 3 * (qn + up[0]), T(0.5) * gV0[0]);
    }
    if (on) {
#pragma unroll
      for (int a = 1; a < 3; ++a) {
        atomic_add(gvel + 3 * qn + a, T(0.5) * gV0[a]);
        atomic_add(gvel + 3 * (qn + up[a]) + a, T(0.5) * gV0[a]);
      }
    }
  }
}

}  // namespace dcell

using namespace dcell;

// Which scatters are warp-aggregated: DCELL_ADJOINT_AGGREGATE = none, phi,
// vel or all (default none: per-lane atomics measured faster).
static int adjoint_aggregate() {
  const char *e = getenv("DCELL_ADJOINT_AGGREGATE");
  if (!e) return 0;
  const std::string v(e);
  return v == "none" ? 0 : v == "phi" ? 1 : v == "vel" ? 2 : 3;
}

template <typename T, bool CUBIC>
static void launch_adjoint_t(int agg, int blocks, const Geom &g, const T *phi0, const T *vel, T dt, int backtrace,
                             const T *gphi, T *gphi0, T *gvel, cudaStream_t st) {
  switch (agg) {
    case 0: sl_adjoint_kernel<T, CUBIC, false, false><<<blocks, 256, 0, st>>>(g, phi0, vel, dt, backtrace, gphi, gphi0, gvel); break;
    case 1: sl_adjoint_kernel<T, CUBIC, true, false><<<blocks, 256, 0, st>>>(g, phi0, vel, dt, backtrace, gphi, gphi0, gvel); break;
    case 2: sl_adjoint_kernel<T, CUBIC, false, true><<<blocks, 256, 0, st>>>(g, phi0, vel, dt, backtrace, gphi, gphi0, gvel); break;
    default: sl_adjoint_kernel<T, CUBIC, true, true><<<blocks, 256, 0, st>>>(g, phi0, vel, dt, backtrace, gphi, gphi0, gvel);
  }
}

int launch_sl_adjoint(const Geom &g, int dtype, const void *phi0, const void *vel, double dt, int interp,
                      int backtrace, const void *gphi, void *gphi0, void *gvel, cudaStream_t st) {
  const long long n = (long long)g.nx * g.ny * g.nz;
  long long blocks = (n + 255) / 256;
  if (blocks > 148LL * 16) blocks = 148LL * 16;
  const bool cubic = interp != DCELL_LINEAR;
  const int agg = adjoint_aggregate();
  if (dtype == DCELL_F64) {
    if (cubic)
      launch_adjoint_t<double, true>(agg, (int)blocks, g, (const double *)phi0, (const double *)vel, dt, backtrace,
                                     (const double *)gphi, (double *)gphi0, (double *)gvel, st);
    else
      launch_adjoint_t<double, false>(agg, (int)blocks, g, (const double *)phi0, (const double *)vel, dt, backtrace,
                                      (const double *)gphi, (double *)gphi0, (double *)gvel, st);
  } else {
    if (cubic)
      launch_adjoint_t<float, true>(agg, (int)blocks, g, (const float *)phi0, (const float *)vel, (float)dt, backtrace,
                                    (const float *)gphi, (float *)gphi0, (float *)gvel, st);
    else
      launch_adjoint_t<float, false>(agg, (int)blocks, g, (const float *)phi0, (const float *)vel, (float)dt,
                                     backtrace, (const float *)gphi, (float *)gphi0, (float *)gvel, st);
  }
  return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
}
