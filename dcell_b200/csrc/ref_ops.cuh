// Reference-order device helpers shared by the translation units that must
// reproduce the reference's FP64 arithmetic bit for bit (compiled with
// -fmad=false: one rounding per operation, in the reference's order).
//
//   interp_vel2/3   InterpolateVelocity2D/3D (Common/InterpolateVelocity.c:7-67)
//   trilinear_ref   Bilinear3D + GridFunction3D_Identity (Common/Grid3D.c:4-36)
//   bilinear_ref    Bilinear2D + GridFunction2D_Identity (Common/Grid.c:190-217)
//   gf2/gf3         GridFunction2D_* (Grid.c:214-254), GridFunction3D_* (Grid3D.c:33-108)
//   sample_gf       Bilinear2D / Bilinear3D of a grid function
//   ord_bits        order-preserving integer images of floating-point values
#pragma once

#include <math.h>

#include "dcell_common.cuh"

namespace dcell {

// ---------------------------------------------------------------------------
// MAC velocity interpolation: InterpolateVelocity2D/3D
// (Common/InterpolateVelocity.c:7-67), same loop and operation order.
template <typename T>
__device__ __forceinline__ void interp_vel3(const Geom &g, const T *__restrict__ vel, const T X[3], T V[3]) {
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const T tx = d == 0 ? T(0.5) : T(0), ty = d == 1 ? T(0.5) : T(0), tz = d == 2 ? T(0.5) : T(0);
    const int xs = (int)floor(X[0] + tx), ys = (int)floor(X[1] + ty), zs = (int)floor(X[2] + tz);
    const T sx = X[0] - (T)xs + tx, sy = X[1] - (T)ys + ty, sz = X[2] - (T)zs + tz;
    T sum = 0;
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int i = 0; i < 2; ++i)
          sum += ((1 - sx) * (T)(1 - i) + (T)i * sx) * ((1 - sy) * (T)(1 - j) + (T)j * sy) *
                 ((1 - sz) * (T)(1 - k) + (T)k * sz) * vel[gidx(g, xs + i, ys + j, zs + k) * 3 + d];
    V[d] = sum;
  }
}

template <typename T>
__device__ __forceinline__ void interp_vel2(const Geom &g, const T *__restrict__ vel, const T X[3], T V[3]) {
#pragma unroll
  for (int d = 0; d < 2; ++d) {
    const T tx = d == 0 ? T(0.5) : T(0), ty = d == 1 ? T(0.5) : T(0);
    const int xs = (int)floor(X[0] + tx), ys = (int)floor(X[1] + ty);
    const T sx = X[0] - (T)xs + tx, sy = X[1] - (T)ys + ty;
    T sum = 0;
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int i = 0; i < 2; ++i)
        sum += ((1 - sx) * (T)(1 - i) + (T)i * sx) * ((1 - sy) * (T)(1 - j) + (T)j * sy) *
               vel[gidx(g, xs + i, ys + j, 0) * 2 + d];
    V[d] = sum;
  }
  V[2] = 0;
}

// Bilinear3D(GridFunction3D_Identity) (Grid3D.c:4-36).
template <typename T>
__device__ __forceinline__ T trilinear_ref(const Geom &g, const T *__restrict__ f, const T S[3]) {
  const int xs = (int)floor(S[0]), ys = (int)floor(S[1]), zs = (int)floor(S[2]);
  const T sx = S[0] - (T)xs, sy = S[1] - (T)ys, sz = S[2] - (T)zs;
  T sum = 0;
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const T xb = (T)i * sx + (T)(1 - i) * (1 - sx);
        const T yb = (T)j * sy + (T)(1 - j) * (1 - sy);
        const T zb = (T)k * sz + (T)(1 - k) * (1 - sz);
        sum += f[gidx(g, xs + i, ys + j, zs + k)] * xb * yb * zb;
      }
  return sum;
}

// Bilinear2D(GridFunction2D_Identity) (Grid.c:190-217).
template <typename T>
__device__ __forceinline__ T bilinear_ref(const Geom &g, const T *__restrict__ f, T x, T y) {
  const int xi = (int)floor(x), yi = (int)floor(y);
  const T xf = (T(2.) * (x - (T)xi) - T(1.)), yf = (T(2.) * (y - (T)yi) - T(1.));
  T sum = 0;
#pragma unroll
  for (int k = 0; k < 2; ++k)
#pragma unroll
    for (int l = 0; l < 2; ++l) {
      const T xb = T(1.) + (T(2.) * (T)k - T(1.)) * xf;
      const T yb = T(1.) + (T(2.) * (T)l - T(1.)) * yf;
      sum += f[gidx(g, xi + k, yi + l, 0)] * xb * yb;
    }
  sum /= T(4.);
  return sum;
}

// ---------------------------------------------------------------------------
// Grid functions (GridFunction2D_* Grid.c:214-254, GridFunction3D_* Grid3D.c:33-108).
template <typename T>
__device__ __forceinline__ T gf3(const Geom &g, const T *__restrict__ p, int fn, int i, int j, int k, T dx, T dy, T dz) {
#define P(a, b, c) p[gidx(g, (a), (b), (c))]
  switch (fn) {
    case 0: return P(i, j, k);
    case 1: return (P(i + 1, j, k) - P(i - 1, j, k)) / (T(2.0) * dx);
    case 2: return (P(i, j + 1, k) - P(i, j - 1, k)) / (T(2.0) * dy);
    case 3: return (P(i, j, k + 1) - P(i, j, k - 1)) / (T(2.0) * dz);
    default: {
      const T px = (P(i + 1, j, k) - P(i - 1, j, k)) / (T(2.0) * dx);
      const T py = (P(i, j + 1, k) - P(i, j - 1, k)) / (T(2.0) * dy);
      const T pz = (P(i, j, k + 1) - P(i, j, k - 1)) / (T(2.0) * dz);
      const T px2 = px * px, py2 = py * py, pz2 = pz * pz;
      const T ppp = px2 + py2 + pz2;
      const T pxx = (P(i - 1, j, k) - T(2.) * P(i, j, k) + P(i + 1, j, k)) / (dx * dx);
      const T pyy = (P(i, j - 1, k) - T(2.) * P(i, j, k) + P(i, j + 1, k)) / (dy * dy);
      const T pzz = (P(i, j, k - 1) - T(2.) * P(i, j, k) + P(i, j, k + 1)) / (dz * dz);
      const T pxy = (P(i - 1, j - 1, k) + P(i + 1, j + 1, k) - P(i - 1, j + 1, k) - P(i + 1, j - 1, k)) / (T(4.) * dx * dy);
      const T pxz = (P(i - 1, j, k - 1) + P(i + 1, j, k + 1) - P(i - 1, j, k + 1) - P(i + 1, j, k - 1)) / (T(4.) * dx * dz);
      const T pyz = (P(i, j - 1, k - 1) + P(i, j + 1, k + 1) - P(i, j - 1, k + 1) - P(i, j + 1, k - 1)) / (T(4.) * dy * dz);
      T c = px2 * (pyy + pzz) + py2 * (pxx + pzz) + pz2 * (pxx + pyy);
      c -= T(2.) * (px * py * pxy + px * pz * pxz + py * pz * pyz);
      c /= sqrt(ppp * ppp * ppp);
      if (c != c) c = 0;
      return c;
    }
  }
#undef P
}

template <typename T>
__device__ __forceinline__ T gf2(const Geom &g, const T *__restrict__ p, int fn, int i, int j, T dx, T dy) {
#define P(a, b) p[gidx(g, (a), (b), 0)]
  switch (fn) {
    case 0: return P(i, j);
    case 1: return (P(i + 1, j) - P(i - 1, j)) / (T(2.) * dx);
    case 2: return (P(i, j + 1) - P(i, j - 1)) / (T(2.) * dy);
    case 3: return 0;
    default: {
      const T px = (P(i + 1, j) - P(i - 1, j)) / (T(2.) * dx);
      const T py = (P(i, j + 1) - P(i, j - 1)) / (T(2.) * dy);
      const T px2 = px * px, py2 = py * py;
      const T pxx = (P(i - 1, j) - T(2.) * P(i, j) + P(i + 1, j)) / (dx * dx);
      const T pyy = (P(i, j - 1) - T(2.) * P(i, j) + P(i, j + 1)) / (dy * dy);
      const T pxy = (P(i - 1, j - 1) + P(i + 1, j + 1) - P(i - 1, j + 1) - P(i + 1, j - 1)) / (T(4.) * dx * dy);
      T k = (pxx * py2 - T(2.) * px * py * pxy + pyy * px2) / sqrt((px2 + py2) * (px2 + py2) * (px2 + py2));
      if (k != k) k = 0;
      return k;
    }
  }
#undef P
}

// Bilinear3D / Bilinear2D of grid function fn at X.
template <typename T, int DIM>
__device__ T sample_gf(const Geom &g, const T *__restrict__ p, int fn, const T X[3]) {
  const T dx = (T)g.hx, dy = (T)g.hy, dz = (T)g.hz;
  if (DIM == 2) {
    const int xi = (int)floor(X[0]), yi = (int)floor(X[1]);
    const T xf = (T(2.) * (X[0] - (T)xi) - T(1.)), yf = (T(2.) * (X[1] - (T)yi) - T(1.));
    T sum = 0;
    for (int k = 0; k < 2; ++k)
      for (int l = 0; l < 2; ++l) {
        const T xb = T(1.) + (T(2.) * (T)k - T(1.)) * xf;
        const T yb = T(1.) + (T(2.) * (T)l - T(1.)) * yf;
        sum += gf2<T>(g, p, fn, xi + k, yi + l, dx, dy) * xb * yb;
      }
    sum /= T(4.);
    return sum;
  }
  const int xs = (int)floor(X[0]), ys = (int)floor(X[1]), zs = (int)floor(X[2]);
  const T sx = X[0] - (T)xs, sy = X[1] - (T)ys, sz = X[2] - (T)zs;
  T sum = 0;
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j)
      for (int k = 0; k < 2; ++k) {
        const T xb = (T)i * sx + (T)(1 - i) * (1 - sx);
        const T yb = (T)j * sy + (T)(1 - j) * (1 - sy);
        const T zb = (T)k * sz + (T)(1 - k) * (1 - sz);
        sum += gf3<T>(g, p, fn, xs + i, ys + j, zs + k, dx, dy, dz) * xb * yb * zb;
      }
  return sum;
}

// order-preserving integer images of floating-point values (smaller value <=> smaller image)
__device__ __forceinline__ unsigned long long ord_bits(double v) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double ord_value(unsigned long long o) {
  const unsigned long long b = (o >> 63) ? (o & 0x7fffffffffffffffull) : ~o;
  return __longlong_as_double((long long)b);
}
__device__ __forceinline__ unsigned int ord_bits(float v) {
  const unsigned int b = __float_as_uint(v);
  return (b >> 31) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float ord_value(unsigned int o) {
  const unsigned int b = (o >> 31) ? (o & 0x7fffffffu) : ~o;
  return __uint_as_float(b);
}
template <typename T> struct OrdOf;
template <> struct OrdOf<double> { typedef unsigned long long type; };
template <> struct OrdOf<float> { typedef unsigned int type; };

}  // namespace dcell
