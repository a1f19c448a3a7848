// Shared device/host helpers for the level-set transport kernels (sm_100a).
//
// Grid convention (reference Common/Grid.c:69-93): a grid covers global
// indices [p, p+n) per axis with x fastest; a velocity grid keeps its MAC
// components innermost (u at x-face i-1/2, v at y-face j-1/2, w at z-face
// k-1/2, Common/Common.h:26-30).  2D grids have nz == 1.  All gathers clamp
// their indices to the grid so any departure point is safe to sample.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/dcell_ls.h"

namespace dcell {

// Unsigned 32-bit division by an invariant divisor d >= 1 (multiply-high and
// shifts, Granlund-Montgomery / Hacker's Delight 10-8): n / d for all n < 2^32.
struct FastDiv {
  uint32_t m, s1, s2;
};

static inline FastDiv make_fastdiv(uint32_t d) {
  uint32_t l = 0;
  while ((1ull << l) < d) ++l;
  FastDiv f;
  f.m = (uint32_t)(((1ull << 32) * ((1ull << l) - d)) / d + 1);
  f.s1 = l < 1 ? l : 1;
  f.s2 = l > 1 ? l - 1 : 0;
  return f;
}

__device__ __forceinline__ uint32_t fdiv(uint32_t n, const FastDiv &f) {
  const uint32_t t = __umulhi(f.m, n);
  return (t + ((n - t) >> f.s1)) >> f.s2;
}

struct Geom {
  int nx, ny, nz;
  int px, py, pz;
  double hx, hy, hz;
  FastDiv div_nx, div_nxny;  // dense-index decode
};

static inline Geom to_geom(const dcell_geom *g) {
  Geom r;
  r.nx = g->n[0]; r.ny = g->n[1]; r.nz = g->n[2] < 1 ? 1 : g->n[2];
  r.px = g->p[0]; r.py = g->p[1]; r.pz = r.nz == 1 ? 0 : g->p[2];
  r.hx = g->h[0]; r.hy = g->h[1]; r.hz = g->h[2];
  r.div_nx = make_fastdiv((uint32_t)r.nx);
  r.div_nxny = make_fastdiv((uint32_t)r.nx * (uint32_t)r.ny);
  return r;
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Flat index of global (i, j, k), clamped into the grid.
__device__ __forceinline__ long long gidx(const Geom &g, int i, int j, int k) {
  i = clampi(i - g.px, 0, g.nx - 1);
  j = clampi(j - g.py, 0, g.ny - 1);
  k = clampi(k - g.pz, 0, g.nz - 1);
  return ((long long)k * g.ny + j) * g.nx + i;
}

// Local (already origin-relative) indices, clamped.
__device__ __forceinline__ long long lidx(const Geom &g, int i, int j, int k) {
  i = clampi(i, 0, g.nx - 1);
  j = clampi(j, 0, g.ny - 1);
  k = clampi(k, 0, g.nz - 1);
  return ((long long)k * g.ny + j) * g.nx + i;
}

// Arrival point number q: band entry q (global coords) or dense point q.
__device__ __forceinline__ void arrival(const Geom &g, const int *__restrict__ band, long long q, int &x, int &y,
                                        int &z) {
  if (band) {
    x = band[3 * q];
    y = band[3 * q + 1];
    z = g.nz == 1 ? 0 : band[3 * q + 2];
  } else {
    x = g.px + (int)(q % g.nx);
    y = g.py + (int)((q / g.nx) % g.ny);
    z = g.pz + (int)(q / ((long long)g.nx * g.ny));
  }
}

// Local (origin-relative) arrival point of number q; false when a band entry
// lies outside the grid (the point is then skipped and flagged).
__device__ __forceinline__ bool arrival_local(const Geom &g, const int *__restrict__ band, long long q, int &x,
                                              int &y, int &z) {
  if (band) {
    x = band[3 * q] - g.px;
    y = band[3 * q + 1] - g.py;
    z = g.nz == 1 ? 0 : band[3 * q + 2] - g.pz;
    return (unsigned)x < (unsigned)g.nx && (unsigned)y < (unsigned)g.ny && (unsigned)z < (unsigned)g.nz;
  }
  const uint32_t n = (uint32_t)q, zq = fdiv(n, g.div_nxny), rem = n - zq * (uint32_t)(g.nx * g.ny);
  const uint32_t yq = fdiv(rem, g.div_nx);
  x = (int)(rem - yq * (uint32_t)g.nx);
  y = (int)yq;
  z = (int)zq;
  return true;
}

// Status bits a kernel may raise in its optional device flags word.
enum : int {
  FLAG_DEPARTURE_CLAMPED = 1,  // a departure point fell outside the grid
  FLAG_NONFINITE = 2,          // a non-finite value was produced
  FLAG_CAPACITY = 4,           // output list capacity exceeded
  FLAG_WAIT_TIMEOUT = 8,       // a bounded device wait gave up
  FLAG_BAD_BAND = 16,          // a band entry lies outside the grid (skipped)
  FLAG_UNSETTLED = 32,         // reinitialisation: points still tentative after the last bucket
  FLAG_PARTICLE_OUTSIDE = 64,  // a particle's stencil or cell left the grid (clamped / skipped)
  FLAG_PIPELINE_REDO = 128,    // internal: a gated z-slab launch left its slab to a full-grid step
};

__device__ __forceinline__ void raise_flag(int *flags, int bit) {
  if (flags) atomicOr(flags, bit);
}

}  // namespace dcell

// Host-side error plumbing shared by all translation units (capi.cu).
extern "C" void dcell_set_error(int code, const char *fmt, ...);
#define DCELL_CUDA_CHECK(expr)                                                                  \
  do {                                                                                          \
    cudaError_t _e = (expr);                                                                    \
    if (_e != cudaSuccess) {                                                                    \
      dcell_set_error(DCELL_ERR_CUDA, "%s failed: %s (%s:%d)", #expr, cudaGetErrorString(_e), \
                      __FILE__, __LINE__);                                                      \
      return DCELL_ERR_CUDA;                                                                    \
    }                                                                                           \
  } while (0)
