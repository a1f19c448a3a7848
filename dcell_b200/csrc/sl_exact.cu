// Reference-exact kernels of the level-set transport path.
//
// This translation unit is compiled with -fmad=false: every expression keeps
// the reference's operation order with one rounding per operation, so in
// FP64 the results are bit-identical to the reference's x86 double
// arithmetic (Common/Grid.c, Grid3D.c, InterpolateVelocity.c, AdvectSL.c,
// IrregularNodes*.c).  The FP32 instantiations follow the same order (the
// FP32 linear step itself runs the fast unit sl_lin.cu).
//
// Kernels:
//   sl_linear_kernel     LevelSetAdvectSL_2D/_3D (AdvectSL.c:23-89)
//   irr_count/irr_write  LevelSetUpdateIrregularNodeList_2D/_3D
//   ortho_kernel         OrthogonalProjection2D/3D (8 threads per node)
//   surface_kernel       IIMUpdateSurfaceQuantities normal + curvature
//   maxvel_kernel        LevelSet_MaxVelocity (Advect.c:70-111)
//   volume kernels       smoothed-Heaviside volume, deterministic FP64 sum
#include <cooperative_groups.h>
#include <math.h>
#include <stdlib.h>

#include <algorithm>
#include <mutex>

#include "dcell_common.cuh"
#include "dcell_kernels.h"
#include "ref_ops.cuh"

namespace dcell {

template <typename T>
__device__ __forceinline__ bool outside(const Geom &g, const T S[3]) {
  return S[0] < (T)g.px || S[0] > (T)(g.px + g.nx - 1) || S[1] < (T)g.py || S[1] > (T)(g.py + g.ny - 1) ||
         (g.nz > 1 && (S[2] < (T)g.pz || S[2] > (T)(g.pz + g.nz - 1)));
}

// Departure point of arrival X (AdvectSL.c:44-47 / :78-82; midpoint variant).
template <typename T, int DIM>
__device__ __forceinline__ void departure(const Geom &g, const T *__restrict__ vel, T dt, T hx, T hy, T hz,
                                          int backtrace, const T X[3], T S[3]) {
  T V[3];
  if (DIM == 3) interp_vel3<T>(g, vel, X, V); else interp_vel2<T>(g, vel, X, V);
  if (backtrace == DCELL_MIDPOINT) {
    const T half = T(0.5) * dt;
    T Xm[3] = {X[0] - V[0] * half / hx, X[1] - V[1] * half / hy, DIM == 3 ? X[2] - V[2] * half / hz : T(0)};
    if (DIM == 3) interp_vel3<T>(g, vel, Xm, V); else interp_vel2<T>(g, vel, Xm, V);
  }
  S[0] = X[0] - V[0] * dt / hx;
  S[1] = X[1] - V[1] * dt / hy;
  S[2] = DIM == 3 ? X[2] - V[2] * dt / hz : T(0);
}

template <typename T, int DIM>
__global__ void __launch_bounds__(256) sl_linear_kernel(Geom g, const T *__restrict__ phi0, const T *__restrict__ vel,
                                                        T dt, const int *__restrict__ band, long long npts, int backtrace,
                                                        T *__restrict__ phi, int *flags) {
  const T hx = (T)g.hx, hy = (T)g.hy, hz = (T)g.hz;
  bool clamped = false;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < npts;
       q += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    arrival(g, band, q, x, y, z);
    const T X[3] = {(T)x, (T)y, (T)z};
    T S[3];
    departure<T, DIM>(g, vel, dt, hx, hy, hz, backtrace, X, S);
    clamped |= outside<T>(g, S);
    phi[gidx(g, x, y, z)] = DIM == 3 ? trilinear_ref<T>(g, phi0, S) : bilinear_ref<T>(g, phi0, S[0], S[1]);
  }
  if (clamped && band) raise_flag(flags, FLAG_DEPARTURE_CLAMPED);  // dense grids: the edge is the domain boundary
}

// ---------------------------------------------------------------------------
// Catmull-Rom polynomial of a stencil for the orthogonal projection
// (OrthogonalProjection3D.c builds it with TricubicInverse.h == C (x) C (x) C,
// OrthogonalProjection.c:48-63 with C (x) C).  Here the operator is applied
// one axis at a time (x, then y, then z: 3 x 16 x 11 products instead of
// the 1331 of the full matrix) and the value and gradient are evaluated by
// nested Horner; both are fully unrolled so the 64 values stay in
// registers.  The coefficients and values equal the reference's up to
// rounding (the projection's tolerance is 1e-3 cells; the results agree with
// the reference's to ~1e-13).

// C[p][q]: row p = the monomial t^p, column q = stencil entry q - 1
__host__ __device__ constexpr double cr_c(int p, int q) {
  return p == 0 ? (q == 1 ? 1.0 : 0.0)
       : p == 1 ? (q == 0 ? -0.5 : q == 2 ? 0.5 : 0.0)
       : p == 2 ? (q == 0 ? 1.0 : q == 1 ? -2.5 : q == 2 ? 2.0 : -0.5)
                : (q == 0 ? -0.5 : q == 1 ? 1.5 : q == 2 ? -1.5 : 0.5);
}

// one axis of C on 4 values with stride `st` (compile-time after unrolling)
template <typename T>
__device__ __forceinline__ void cr_apply(const T *in, T *out, int st) {
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    T acc = T(0);
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if (cr_c(p, q) != 0.0) acc += (T)cr_c(p, q) * in[q * st];
    out[p * st] = acc;
  }
}

template <typename T>
__device__ __forceinline__ void cubic_coefs3(const T *s, T *a) {
  T t[64], u[64];
#pragma unroll
  for (int l = 0; l < 16; ++l) cr_apply(s + 4 * l, t + 4 * l, 1);  // x
#pragma unroll
  for (int l = 0; l < 16; ++l) cr_apply(t + (l & 3) + 16 * (l >> 2), u + (l & 3) + 16 * (l >> 2), 4);  // y
#pragma unroll
  for (int l = 0; l < 16; ++l) cr_apply(u + l, a + l, 16);  // z
}

template <typename T>
__device__ __forceinline__ void cubic_coefs2(const T *s, T *a) {
  T t[16];
#pragma unroll
  for (int l = 0; l < 4; ++l) cr_apply(s + 4 * l, t + 4 * l, 1);  // x
#pragma unroll
  for (int l = 0; l < 4; ++l) cr_apply(t + l, a + l, 4);  // y
}

// value and gradient of sum a[i + 4j + 16k] x^i y^j z^k
template <typename T>
__device__ __forceinline__ void cubic_eval3(const T *a, T x, T y, T z, T &p, T &gx, T &gy, T &gz) {
  T v = 0, vx = 0, vy = 0, vz = 0;
#pragma unroll
  for (int k = 3; k >= 0; --k) {
    T w = 0, wx = 0, wy = 0;  // the (x, y) polynomial of slice k, its x and y derivatives
#pragma unroll
    for (int j = 3; j >= 0; --j) {
      const T *c = a + 4 * j + 16 * k;
      const T px = ((c[3] * x + c[2]) * x + c[1]) * x + c[0];
      const T dpx = (T(3) * c[3] * x + T(2) * c[2]) * x + c[1];
      wy = wy * y + w;
      w = w * y + px;
      wx = wx * y + dpx;
    }
    vz = vz * z + v;
    v = v * z + w;
    vx = vx * z + wx;
    vy = vy * z + wy;
  }
  p = v; gx = vx; gy = vy; gz = vz;
}

template <typename T>
__device__ __forceinline__ void cubic_eval2(const T *a, T x, T y, T &p, T &gx, T &gy) {
  T v = 0, vx = 0, vy = 0;
#pragma unroll
  for (int j = 3; j >= 0; --j) {
    const T *c = a + 4 * j;
    const T px = ((c[3] * x + c[2]) * x + c[1]) * x + c[0];
    const T dpx = (T(3) * c[3] * x + T(2) * c[2]) * x + c[1];
    vy = vy * y + v;
    v = v * y + px;
    vx = vx * y + dpx;
  }
  p = v; gx = vx; gy = vy;
}

// ---------------------------------------------------------------------------
// Irregular nodes (IrregularNodes.c:32-141, IrregularNodes3D.c:6-117).
// STAGGERED_GRID (Common.h:42-47): CELL_CENTER {0,0,0}, U {-1,0,0}, V {0,-1,0}, W {0,0,-1}.
__device__ __forceinline__ int stag(int face, int axis) { return (face == axis + 1) ? -1 : 0; }

// Visits the nodes of one band point in the reference's emission order.
// EMIT(kind, args...) is a functor: kind 0 = projection node, 1 = cell-face
// node (axis), 2 = velocity-face node (face, axis, hi, lo).
template <typename T, int DIM, typename F>
__device__ __forceinline__ void visit_point(const Geom &g, const T *__restrict__ phi, int i, int j, int k, F &emit) {
  if (DIM == 3) {
    T s[3][3][3];
#pragma unroll
    for (int K = 0; K < 3; ++K)
#pragma unroll
      for (int J = 0; J < 3; ++J)
#pragma unroll
        for (int I = 0; I < 3; ++I) s[K][J][I] = phi[gidx(g, i + I - 1, j + J - 1, k + K - 1)];
    const T c = s[1][1][1];
    // STAR order (Common.h:49-51): +x, -x, +y, -y, +z, -z; first sign change only.
    const int star[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
#pragma unroll
    for (int m = 0; m < 6; ++m) {
      if (c * s[1 + star[m][2]][1 + star[m][1]][1 + star[m][0]] <= T(0.)) {
        emit.projection(c);
        break;
      }
    }
#pragma unroll
    for (int f = 1; f <= 3; ++f) {
      const T nb = s[1 + stag(f, 2)][1 + stag(f, 1)][1 + stag(f, 0)];
      if (c * nb <= T(0.)) emit.cell_face(f - 1, c, nb);
    }
#pragma unroll
    for (int face = 1; face <= 3; ++face) {
      const T hi = (s[1 + stag(face, 2)][1 + stag(face, 1)][1 + stag(face, 0)] + c) / T(2.);
#pragma unroll
      for (int axis = 1; axis <= 3; ++axis) {
        if (face == axis) continue;
        const T lo = (s[1 + stag(face, 2) + stag(axis, 2)][1 + stag(face, 1) + stag(axis, 1)]
                       [1 + stag(face, 0) + stag(axis, 0)] +
                      s[1 + stag(axis, 2)][1 + stag(axis, 1)][1 + stag(axis, 0)]) /
                     T(2.);
        if (hi * lo <= T(0.)) emit.vel_face(face, axis - 1, hi, lo);
      }
    }
  } else {
    T s[3][3];
#pragma unroll
    for (int J = 0; J < 3; ++J)
#pragma unroll
      for (int I = 0; I < 3; ++I) s[J][I] = phi[gidx(g, i + I - 1, j + J - 1, 0)];
    const T c = s[1][1];
    const int nei[4][2] = {{1, 0}, {-1, 0}, {0, -1}, {0, 1}};  // IrregularNodes.c:36
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      if (c * s[1 + nei[m][1]][1 + nei[m][0]] <= T(0.)) {
        emit.projection(c);
        break;
      }
    }
#pragma unroll
    for (int f = 1; f <= 2; ++f) {
      const T nb = s[1 + stag(f, 1)][1 + stag(f, 0)];
      if (c * nb <= T(0.)) emit.cell_face(f - 1, c, nb);
    }
    // U-velocity Laplacian (IrregularNodes.c:108-122), V (:124-138)
    T hi = (s[1][0] + s[1][1]) / T(2.), lo = (s[0][0] + s[0][1]) / T(2.);
    if (hi * lo <= T(0.)) emit.vel_face(1, 1, hi, lo);
    hi = (s[0][1] + s[1][1]) / T(2.);
    lo = (s[0][0] + s[1][0]) / T(2.);
    if (hi * lo <= T(0.)) emit.vel_face(2, 0, hi, lo);
  }
}

struct CountEmit {
  int n = 0;
  template <typename T> __device__ void projection(T) { ++n; }
  template <typename T> __device__ void cell_face(int, T, T) { ++n; }
  template <typename T> __device__ void vel_face(int, int, T, T) { ++n; }
};

template <typename T, int DIM>
struct WriteEmit {
  dcell_irregular_node *out;
  long long slot;
  long long cap;
  int i, j, k;
  __device__ dcell_irregular_node *next() {
    if (slot >= cap) { ++slot; return nullptr; }
    dcell_irregular_node *r = out + slot++;
    return r;
  }
  __device__ void base(dcell_irregular_node &r) {
    r.pos[0] = i; r.pos[1] = j; r.pos[2] = k;
    r.pad = 0;
    r.d = 0; r.X[0] = r.X[1] = r.X[2] = 0; r.op[0] = r.op[1] = r.op[2] = 0;
    r.n[0] = r.n[1] = r.n[2] = 0; r.k = 0;
    r.signFace = 0;
  }
  __device__ void projection(T c) {
    dcell_irregular_node *r = next();
    if (!r) return;
    dcell_irregular_node t; base(t);
    t.axis = -1; t.shift = -1; t.signCenter = c > T(0.) ? 1 : -1;
    t.X[0] = i; t.X[1] = j; t.X[2] = DIM == 3 ? k : 0;  // op (and X) filled by the projection kernel
    *r = t;
  }
  __device__ void cell_face(int axis, T c, T nb) {
    dcell_irregular_node *r = next();
    if (!r) return;
    dcell_irregular_node t; base(t);
    const T d = c / (c - nb);
    t.d = (double)d;
    t.signCenter = c > T(0.) ? 1 : -1;
    t.signFace = d < T(0.5) ? -t.signCenter : t.signCenter;
    t.shift = 0; t.axis = axis;
    // X = pos + d * STAGGERED_GRID[axis+1]  (the -1 component only)
    t.X[0] = (double)((T)i + d * (T)stag(axis + 1, 0));
    t.X[1] = (double)((T)j + d * (T)stag(axis + 1, 1));
    t.X[2] = DIM == 3 ? (double)((T)k + d * (T)stag(axis + 1, 2)) : 0.0;
    *r = t;
  }
  __device__ void vel_face(int face, int axis, T hi, T lo) {
    dcell_irregular_node *r = next();
    if (!r) return;
    dcell_irregular_node t; base(t);
    T d = hi / (hi - lo);
    if (DIM == 3 && d != d) d = 0;
    t.d = (double)d;
    t.signCenter = hi > T(0.) ? 1 : -1;
    t.signFace = d < T(0.5) ? -t.signCenter : t.signCenter;
    t.shift = face; t.axis = axis;
    if (DIM == 3) {
      t.X[0] = (double)((T)i + (T)stag(face, 0) / T(2.) + d * (T)stag(axis + 1, 0));
      t.X[1] = (double)((T)j + (T)stag(face, 1) / T(2.) + d * (T)stag(axis + 1, 1));
      t.X[2] = (double)((T)k + (T)stag(face, 2) / T(2.) + d * (T)stag(axis + 1, 2));
    } else if (face == 1) {  // U: X = (x - 1/2, y - d)
      t.X[0] = (double)((T)i + (T)stag(1, 0) / T(2.));
      t.X[1] = (double)((T)j + (T)stag(1, 1) / T(2.) - d);
    } else {                 // V: X = (x - d, y - 1/2)
      t.X[0] = (double)((T)i + (T)stag(2, 0) / T(2.) - d);
      t.X[1] = (double)((T)j + (T)stag(2, 1) / T(2.));
    }
    *r = t;
  }
};

template <typename T, int DIM>
__global__ void __launch_bounds__(256) irr_count_kernel(Geom g, const T *__restrict__ phi, const int *__restrict__ band,
                                                        int nband, int *__restrict__ counts) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nband) return;
  CountEmit e;
  visit_point<T, DIM>(g, phi, band[3 * b], band[3 * b + 1], DIM == 3 ? band[3 * b + 2] : 0, e);
  counts[b] = e.n;
}

template <typename T, int DIM>
__global__ void __launch_bounds__(256) irr_write_kernel(Geom g, const T *__restrict__ phi, const int *__restrict__ band,
                                                        int nband, const int *__restrict__ offsets,
                                                        dcell_irregular_node *__restrict__ out, int cap) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nband) return;
  WriteEmit<T, DIM> e;
  e.out = out; e.slot = offsets[b]; e.cap = cap;
  e.i = band[3 * b]; e.j = band[3 * b + 1]; e.k = DIM == 3 ? band[3 * b + 2] : band[3 * b + 2];
  visit_point<T, DIM>(g, phi, e.i, e.j, DIM == 3 ? e.k : 0, e);
}

// ---------------------------------------------------------------------------
// Block-level exclusive scan of int counts (3 passes): offsets[b], total.
constexpr int SCAN_BLOCK = 1024;

__global__ void __launch_bounds__(SCAN_BLOCK) scan_blocks_kernel(const int *__restrict__ in, int n,
                                                                 int *__restrict__ out, int *__restrict__ partial) {
  __shared__ int warp_sums[SCAN_BLOCK / 32];
  const int b = blockIdx.x * SCAN_BLOCK + threadIdx.x;
  const int v = b < n ? in[b] : 0;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += t;
  }
  if (lane == 31) warp_sums[w] = x;
  __syncthreads();
  if (w == 0) {
    int y = warp_sums[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, y, o);
      if (lane >= o) y += t;
    }
    warp_sums[lane] = y;
  }
  __syncthreads();
  const int incl = x + (w > 0 ? warp_sums[w - 1] : 0);
  if (b < n) out[b] = incl - v;
  if (threadIdx.x == SCAN_BLOCK - 1) partial[blockIdx.x] = incl;
}

// Single block: exclusive scan of the per-block totals in place; total at partial[nblk].
__global__ void __launch_bounds__(SCAN_BLOCK) scan_partials_kernel(int *__restrict__ partial, int nblk) {
  __shared__ int warp_sums[SCAN_BLOCK / 32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int base = 0; base < nblk; base += SCAN_BLOCK) {
    const int b = base + threadIdx.x;
    const int v = b < nblk ? partial[b] : 0;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += t;
    }
    if (lane == 31) warp_sums[w] = x;
    __syncthreads();
    if (w == 0) {
      int y = warp_sums[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, y, o);
        if (lane >= o) y += t;
      }
      warp_sums[lane] = y;
    }
    __syncthreads();
    const int incl = x + (w > 0 ? warp_sums[w - 1] : 0);
    const int c = carry;
    if (b < nblk) partial[b] = c + incl - v;
    __syncthreads();
    if (threadIdx.x == SCAN_BLOCK - 1) carry = c + incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[nblk] = carry;
}

__global__ void __launch_bounds__(SCAN_BLOCK) scan_add_kernel(int *__restrict__ out, int n,
                                                              const int *__restrict__ partial, int nblk,
                                                              int *__restrict__ total, int cap, int *flags) {
  const int b = blockIdx.x * SCAN_BLOCK + threadIdx.x;
  if (b < n) out[b] += partial[blockIdx.x];
  if (b == 0) {
    *total = partial[nblk];
    if (partial[nblk] > cap) raise_flag(flags, FLAG_CAPACITY);
  }
}

// ---------------------------------------------------------------------------
// Orthogonal projection (OrthogonalProjection.c, OrthogonalProjection3D.c):
// 8 threads per projection node, thread s = sub-cell (i,j,k) of the 2x2x2
// (2D: 2x2) patches; the closest converged in-cell root wins (ties resolve to
// the lowest sub-cell index, the reference's loop order).
template <typename T>
__device__ void ortho_quadratic3(const T s[3][3][3], T op[3]);
template <typename T>
__device__ void ortho_linear3(const T s[3][3][3], T op[3]) {
  const int star[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
  T mindist = 2;
  for (int i = 0; i < 6; ++i) {
    const T nb = s[star[i][2] + 1][star[i][1] + 1][star[i][0] + 1];
    if (s[1][1][1] * nb <= 0) {
      const T dist = s[1][1][1] / (s[1][1][1] - nb);
      if (dist < mindist) {
        mindist = dist;
        op[0] = dist * (T)star[i][0];
        op[1] = dist * (T)star[i][1];
        op[2] = dist * (T)star[i][2];
      }
    }
  }
}
template <typename T>
__device__ void ortho_quadratic3(const T s[3][3][3], T op[3]) {
  const T p = s[1][1][1];
  const T px = (s[1][1][2] - s[1][1][0]) / T(2.), py = (s[1][2][1] - s[1][0][1]) / T(2.),
          pz = (s[2][1][1] - s[0][1][1]) / T(2.);
  const T px2 = px * px, py2 = py * py, pz2 = pz * pz;
  const T pxx = (s[1][1][2] - T(2.) * p + s[1][1][0]);
  const T pyy = (s[1][2][1] - T(2.) * p + s[1][0][1]);
  const T pzz = (s[2][1][1] - T(2.) * p + s[0][1][1]);
  const T pxy = (s[1][0][0] + s[1][2][2] - s[1][2][0] - s[1][0][2]) / T(4.);
  const T pxz = (s[0][1][0] + s[2][1][2] - s[2][1][0] - s[0][1][2]) / T(4.);
  const T pyz = (s[0][0][1] + s[2][2][1] - s[2][0][1] - s[0][2][1]) / T(4.);
  const T pn = sqrt(px2 + py2 + pz2);
  const T c = (px2 * pxx + py2 * pyy + pz2 * pzz + T(2) * px * py * pxy + T(2) * px * pz * pxz +
               T(2) * py * pz * pyz) /
              (px2 + py2 + pz2);
  T a = 0;
  for (int m = 0; m < 5; ++m) {
    const T f = p + pn * a + T(0.5) * a * a * c;
    const T df = pn + a * c;
    a = a - f / df;
  }
  if (fabs(a) < T(1)) {
    op[0] = a * px / pn;
    op[1] = a * py / pn;
    op[2] = a * pz / pn;
  } else {
    ortho_linear3<T>(s, op);
  }
}

template <typename T>
__device__ void ortho_linear2(const T s[3][3], T op[3], T &mindist) {
  const int star[4][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}};
  mindist = 2;
  for (int i = 0; i < 4; ++i) {
    const T nb = s[star[i][1] + 1][star[i][0] + 1];
    if (s[1][1] * nb <= 0) {
      const T dist = s[1][1] / (s[1][1] - nb);
      if (dist < mindist) {
        mindist = dist;
        op[0] = dist * (T)star[i][0];
        op[1] = dist * (T)star[i][1];
      }
    }
  }
}

template <typename T, int DIM>
__global__ void __launch_bounds__(256, 3) ortho_kernel(Geom g, const T *__restrict__ phi,
                                                    dcell_irregular_node *__restrict__ nodes,
                                                    const int *__restrict__ count, int cap) {
  const int n = min(*count, cap);
  // a block-uniform loop over the nodes written (the launch is sized for the capacity)
  for (long long base = blockIdx.x * (long long)blockDim.x; base < 8LL * n;
       base += (long long)gridDim.x * blockDim.x) {
  const long long tid = base + threadIdx.x;
  const long long node = tid >> 3;
  const int sub = (int)(tid & 7);
  const bool active = node < n && nodes[node].axis == -1 && (DIM == 3 || sub < 4);
  const T TOL = T(1e-3), TOL2 = TOL * TOL;
  const double BIG = 1.7976931348623157e308;
  double dist = BIG;
  T res[3] = {0, 0, 0};
  int ci = 0, cj = 0, ck = 0;
  if (active) {
    ci = nodes[node].pos[0]; cj = nodes[node].pos[1]; ck = DIM == 3 ? nodes[node].pos[2] : 0;
    const int i = sub & 1, j = (sub >> 1) & 1, k = (sub >> 2) & 1;
    T x0[3] = {(T)(1 - i), (T)(1 - j), (T)(1 - k)}, x = x0[0], y = x0[1], z = x0[2];
    int m;
    if (DIM == 3) {
      T s[64], a[64];
#pragma unroll
      for (int zz = 0; zz < 4; ++zz)
#pragma unroll
        for (int yy = 0; yy < 4; ++yy)
#pragma unroll
          for (int xx = 0; xx < 4; ++xx)
            s[xx + 4 * yy + 16 * zz] = phi[gidx(g, ci - 2 + i + xx, cj - 2 + j + yy, ck - 2 + k + zz)];
      cubic_coefs3<T>(s, a);
      for (m = 0; m < 20; ++m) {
        T p, gx, gy, gz;
        cubic_eval3<T>(a, x, y, z, p, gx, gy, gz);
        const T pp = gx * gx + gy * gy + gz * gz;
        const T d1x = -p * gx / pp, d1y = -p * gy / pp, d1z = -p * gz / pp;
        const T xp = (x0[0] - x) * gx + (x0[1] - y) * gy + (x0[2] - z) * gz;
        const T d2x = (x0[0] - x) - xp / pp * gx, d2y = (x0[1] - y) - xp / pp * gy, d2z = (x0[2] - z) - xp / pp * gz;
        x += d1x + T(0.5) * d2x;
        y += d1y + T(0.5) * d2y;
        z += d1z + T(0.5) * d2z;
        const T norm = d1x * d1x + d1y * d1y + d1z * d1z + d2x * d2x + d2y * d2y + d2z * d2z;
        if (norm < TOL2) break;
      }
      if (m < 20 && !(x < -TOL || 1 + TOL < x || y < -TOL || 1 + TOL < y || z < -TOL || 1 + TOL < z))
        dist = (double)sqrt((x - x0[0]) * (x - x0[0]) + (y - x0[1]) * (y - x0[1]) + (z - x0[2]) * (z - x0[2]));
      res[0] = x + (T)i - 1; res[1] = y + (T)j - 1; res[2] = z + (T)k - 1;
    } else {
      T s[16], a[16];
#pragma unroll
      for (int yy = 0; yy < 4; ++yy)
#pragma unroll
        for (int xx = 0; xx < 4; ++xx) s[xx + 4 * yy] = phi[gidx(g, ci - 2 + i + xx, cj - 2 + j + yy, 0)];
      cubic_coefs2<T>(s, a);
      for (m = 0; m < 20; ++m) {
        T p, gx, gy;
        cubic_eval2<T>(a, x, y, p, gx, gy);
        const T pp = gx * gx + gy * gy;
        const T d1x = -p * gx / pp, d1y = -p * gy / pp;
        const T xp = (x0[0] - x) * gx + (x0[1] - y) * gy;
        const T d2x = (x0[0] - x) - xp / pp * gx, d2y = (x0[1] - y) - xp / pp * gy;
        x += d1x + T(0.5) * d2x;
        y += d1y + T(0.5) * d2y;
        const T norm = d1x * d1x + d1y * d1y + d2x * d2x + d2y * d2y;
        if (norm < TOL2) break;
      }
      if (m < 20 && !(x < -TOL || 1 + TOL < x || y < -TOL || 1 + TOL < y))
        dist = (double)sqrt((x - x0[0]) * (x - x0[0]) + (y - x0[1]) * (y - x0[1]));
      res[0] = x + (T)i - 1; res[1] = y + (T)j - 1; res[2] = 0;
    }
  }
  // min over the 8 sub-cells of this node (lanes 8q..8q+7), lowest index on ties
  int best = sub;
  double bd = dist;
#pragma unroll
  for (int o = 1; o < 8; o <<= 1) {
    const double od = __shfl_xor_sync(0xffffffffu, bd, o, 8);
    const int ob = __shfl_xor_sync(0xffffffffu, best, o, 8);
    if (od < bd || (od == bd && ob < best)) { bd = od; best = ob; }
  }
  T w0 = __shfl_sync(0xffffffffu, res[0], best, 8);
  T w1 = __shfl_sync(0xffffffffu, res[1], best, 8);
  T w2 = __shfl_sync(0xffffffffu, res[2], best, 8);
  if (!active || sub != 0) continue;
  T op[3] = {w0, w1, w2};
  if (DIM == 3) {
    if (bd == BIG) {  // no sub-cell converged: quadratic, then linear fallback
      T s3[3][3][3];
      for (int K = 0; K < 3; ++K)
        for (int J = 0; J < 3; ++J)
          for (int I = 0; I < 3; ++I) s3[K][J][I] = phi[gidx(g, ci + I - 1, cj + J - 1, ck + K - 1)];
      op[0] = op[1] = op[2] = 0;
      ortho_quadratic3<T>(s3, op);
    }
  } else {
    T s3[3][3], opl[3] = {0, 0, 0}, dl;
    for (int J = 0; J < 3; ++J)
      for (int I = 0; I < 3; ++I) s3[J][I] = phi[gidx(g, ci + I - 1, cj + J - 1, 0)];
    ortho_linear2<T>(s3, opl, dl);
    if (!(bd < (double)dl)) { op[0] = opl[0]; op[1] = opl[1]; op[2] = 0; }
  }
  dcell_irregular_node &r = nodes[node];
  r.op[0] = (double)op[0]; r.op[1] = (double)op[1]; r.op[2] = (double)op[2];
  r.X[0] = (double)((T)ci + op[0]);
  r.X[1] = (double)((T)cj + op[1]);
  r.X[2] = DIM == 3 ? (double)((T)ck + op[2]) : 0.0;
  }
}

// Normal and curvature at node X (IIM/SurfaceQuantities.c 2D:48-56, 3D:83-89,111):
// Bilinear3D / Bilinear2D samples of the gradient components and of the
// curvature grid function.  8 lanes per node, lane c = trilinear corner c in
// the reference's loop order (i, j, k nested; 2D: 4 lanes, x then y); each
// lane forms its corner's terms exactly as Bilinear3D does, and the node's
// first lane sums them in corner order -- the reference's bits, with the
// corners' divisions and square roots spread over the lanes.
template <typename T, int DIM>
__global__ void __launch_bounds__(128) surface_kernel(Geom g, const T *__restrict__ phi,
                                                      dcell_irregular_node *__restrict__ nodes,
                                                      const int *__restrict__ count, int cap) {
  constexpr int NC = DIM == 3 ? 8 : 4;  // corners
  const int n = min(*count, cap);
  const T dx = (T)g.hx, dy = (T)g.hy, dz = (T)g.hz;
  for (long long base = blockIdx.x * (long long)blockDim.x; base < 8LL * n;
       base += (long long)gridDim.x * blockDim.x) {
    const long long tid = base + threadIdx.x;
    const long long q = tid >> 3;
    const int c = (int)(tid & 7);
    const bool active = q < n;
    T t[4] = {0, 0, 0, 0};  // this corner's terms of d/dx, d/dy, d/dz, curvature
    if (active && c < NC) {
      const dcell_irregular_node &r = nodes[q];
      const T X[3] = {(T)r.X[0], (T)r.X[1], (T)r.X[2]};
      if (DIM == 3) {
        const int xs = (int)floor(X[0]), ys = (int)floor(X[1]), zs = (int)floor(X[2]);
        const T sx = X[0] - (T)xs, sy = X[1] - (T)ys, sz = X[2] - (T)zs;
        const int i = c >> 2, j = (c >> 1) & 1, k = c & 1;
        const T xb = (T)i * sx + (T)(1 - i) * (1 - sx);
        const T yb = (T)j * sy + (T)(1 - j) * (1 - sy);
        const T zb = (T)k * sz + (T)(1 - k) * (1 - sz);
#pragma unroll
        for (int f = 0; f < 4; ++f) t[f] = gf3<T>(g, phi, f + 1, xs + i, ys + j, zs + k, dx, dy, dz) * xb * yb * zb;
      } else {
        const int xi = (int)floor(X[0]), yi = (int)floor(X[1]);
        const T xf = (T(2.) * (X[0] - (T)xi) - T(1.)), yf = (T(2.) * (X[1] - (T)yi) - T(1.));
        const int k = c >> 1, l = c & 1;
        const T xb = T(1.) + (T(2.) * (T)k - T(1.)) * xf;
        const T yb = T(1.) + (T(2.) * (T)l - T(1.)) * yf;
        t[0] = gf2<T>(g, phi, 1, xi + k, yi + l, dx, dy) * xb * yb;
        t[1] = gf2<T>(g, phi, 2, xi + k, yi + l, dx, dy) * xb * yb;
        t[3] = gf2<T>(g, phi, 4, xi + k, yi + l, dx, dy) * xb * yb;
      }
    }
    T sum[4] = {0, 0, 0, 0};
#pragma unroll
    for (int f = 0; f < 4; ++f)
#pragma unroll
      for (int e = 0; e < NC; ++e) sum[f] += __shfl_sync(0xffffffffu, t[f], e, 8);
    if (!active || c != 0) continue;
    dcell_irregular_node &r = nodes[q];
    if (DIM == 2) {
      const T nx = sum[0] / T(4.), ny = sum[1] / T(4.);
      const T h = sqrt(nx * nx + ny * ny);
      r.n[0] = (double)(nx / h); r.n[1] = (double)(ny / h); r.n[2] = 0.0;
      r.k = (double)(sum[3] / T(4.));
    } else {
      T nx = sum[0], ny = sum[1], nz = sum[2];
      const T h = sqrt(nx * nx + ny * ny + nz * nz);
      nx /= h; ny /= h; nz /= h;
      r.n[0] = (double)nx; r.n[1] = (double)ny; r.n[2] = (double)nz;
      r.k = (double)sum[3];
    }
  }
}

// LevelSet_MaxVelocity: max |V(pos)| over nodes; non-negative doubles order
// like their bit patterns, so an integer atomicMax is exact and deterministic.
template <typename T, int DIM>
__global__ void __launch_bounds__(256) maxvel_kernel(Geom g, const T *__restrict__ vel,
                                                     const dcell_irregular_node *__restrict__ nodes,
                                                     const int *__restrict__ count, int cap,
                                                     unsigned long long *__restrict__ out) {
  const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int n = min(*count, cap);
  double mag = 0.0;
  if (q < n) {
    const T X[3] = {(T)nodes[q].pos[0], (T)nodes[q].pos[1], DIM == 3 ? (T)nodes[q].pos[2] : T(0)};
    T V[3];
    if (DIM == 3) {
      interp_vel3<T>(g, vel, X, V);
      mag = (double)sqrt(V[0] * V[0] + V[1] * V[1] + V[2] * V[2]);
    } else {
      interp_vel2<T>(g, vel, X, V);
      mag = (double)sqrt(V[0] * V[0] + V[1] * V[1]);
    }
  }
  unsigned long long bits = (unsigned long long)__double_as_longlong(mag);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long t = __shfl_xor_sync(0xffffffffu, bits, o);
    bits = t > bits ? t : bits;
  }
  if ((threadIdx.x & 31) == 0 && bits) atomicMax(out, bits);
}

// Smoothed-Heaviside volume: fixed grid, fixed per-thread strides and a fixed
// reduction tree -> bitwise reproducible.
constexpr int VOL_BLOCKS = 148 * 4;
constexpr int VOL_THREADS = 256;

template <typename T>
__global__ void __launch_bounds__(VOL_THREADS) volume_partial_kernel(const T *__restrict__ phi, long long n, double eps,
                                                                     double *__restrict__ partial) {
  __shared__ double ws[VOL_THREADS / 32];
  const double pi = 3.14159265358979323846264;
  double acc = 0.0;
  for (long long q = blockIdx.x * (long long)VOL_THREADS + threadIdx.x; q < n; q += (long long)VOL_BLOCKS * VOL_THREADS) {
    const double p = (double)phi[q];
    double H;
    if (p < -eps) H = 0.0;
    else if (p > eps) H = 1.0;
    else H = 0.5 * (1.0 + p / eps + sin(pi * p / eps) / pi);
    acc += 1.0 - H;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < VOL_THREADS / 32; ++w) s += ws[w];
    partial[blockIdx.x] = s;
  }
}

__global__ void __launch_bounds__(32) volume_final_kernel(const double *__restrict__ partial, double cell,
                                                          double *__restrict__ out) {
  double acc = 0.0;
  for (int b = threadIdx.x; b < VOL_BLOCKS; b += 32) acc += partial[b];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (threadIdx.x == 0) *out = acc * cell;
}


// ---------------------------------------------------------------------------
// Narrow-band reinitialisation by bucketed fast marching (replaces
// LevelSetReinitialize, LevelSetMethod/FastMarching.c:11-146, after its
// LevelSetResize).  The heap of FMM_SolveEikonal is replaced by buckets of
// width `bucket` cells: every tentative value below (b+1)*bucket (and <=
// bandWidth) is fixed together, then the neighbours of the newly fixed points
// are re-evaluated with the reference's second-order update (AccumulateCoef
// FastMarching2D.c:33-99, FMM_PushNeighbors2D/3D FastMarching2D.c:103-185,
// FastMarching3D.c:13-101) and keep the smallest value (atomicMin on an
// order-preserving integer image).  Each evaluation sees what the heap had
// fixed when it popped the pushing point: the seeds and the marched points
// whose value is not larger than the pusher's.  Evaluations read only fixed
// points, so the result is independent of thread order and identical to the
// oracle's restatement of the same procedure.  Compiled, like the rest of
// this file, without FMA contraction.
constexpr int REINIT_TAIL = 16;   // buckets past bandWidth in which the last pushes settle
constexpr int REINIT_THREADS = 256;

enum ReinitMark : int { RM_FAR = 0, RM_TENT = 1, RM_MARCHED = 2, RM_SEED = 3 };

struct ReinitState {
  int *mark;          // ReinitMark per point
  void *tent;         // OrdOf<T>::type per point
  int *near[2];       // tentative points below the window end (ping-pong)
  int *far[2];        // tentative points at or past it (ping-pong)
  int *acc;           // points fixed in the current bucket
  int *err;           // bit 1: an update was not a number, bit 2: unsettled (global)
};

// list lengths of one side's march, in shared memory
struct ReinitCounts {
  int near[2], far[2], acc[2];  // acc: ping-pong by bucket parity
};

template <typename T>
__device__ void fmm_accumulate_dev(T bw, const T *p, T &a, T &b, T &c) {
  const T D2p = (3 * p[0] - 4 * p[1] + p[2]) / T(2);
  const T D2m = (3 * p[0] - 4 * p[-1] + p[-2]) / T(2);
  const T D1p = p[0] - p[1];
  const T D1m = p[0] - p[-1];
  T Dm, am, bm, cm, Dp, ap, bp, cp, t;
  if (0 <= p[1] && p[1] < bw && 0 <= p[2] && p[2] < bw && D2p > 0) {
    t = (4 * p[1] - p[2]) / T(3);
    ap = T(9) / T(4);
    bp = -T(9) / T(2) * t;
    cp = T(9) / T(4) * t * t;
    Dp = D2p;
  } else if (0 <= p[1] && p[1] < bw && D1p > 0) {
    ap = 1;
    bp = -2 * p[1];
    cp = p[1] * p[1];
    Dp = D1p;
  } else {
    ap = bp = cp = Dp = 0;
  }
  if (0 <= p[-1] && p[-1] < bw && 0 <= p[-2] && p[-2] < bw && D2m > 0) {
    t = (4 * p[-1] - p[-2]) / T(3);
    am = T(9) / T(4);
    bm = -T(9) / T(2) * t;
    cm = T(9) / T(4) * t * t;
    Dm = D2m;
  } else if (0 <= p[-1] && p[-1] < bw && D1m > 0) {
    am = 1;
    bm = -2 * p[-1];
    cm = p[-1] * p[-1];
    Dm = D1m;
  } else {
    am = bm = cm = Dm = 0;
  }
  if (Dm > Dp) {
    a += am;
    b += bm;
    c += cm;
  } else {
    a += ap;
    b += bp;
    c += cp;
  }
}

// update of local point (x,y,z) on side `sign`, seeing seeds and marched points <= lim
template <typename T, int DIM>
__device__ T fmm_update_dev(const Geom &g, const T *__restrict__ phi, const int *__restrict__ mark, int x, int y,
                            int z, int sign, T inf, T lim) {
  T a = 0, b = 0, c = -1, line[7];
  const int X[3] = {x, y, z}, n[3] = {g.nx, g.ny, g.nz};
#pragma unroll
  for (int ax = 0; ax < DIM; ++ax) {
#pragma unroll
    for (int m = 0; m < 7; ++m) {
      int q[3] = {X[0], X[1], X[2]};
      q[ax] += m - 3;
      if (q[ax] < 0 || q[ax] >= n[ax]) {
        line[m] = inf;
      } else {
        const int r = (q[2] * g.ny + q[1]) * g.nx + q[0];
        const T v = sign * phi[r];
        line[m] = (mark[r] == RM_MARCHED && v > lim) ? inf : v;
      }
    }
    fmm_accumulate_dev<T>(inf, line + 3, a, b, c);
  }
  const T disc = sqrt(b * b - 4 * a * c);
  T d1 = (-b + disc) / (2 * a);
  if (d1 != d1) d1 = -b / (2 * a);
  return d1;
}

// Push neighbour s (STAR order) of (x,y,z): re-evaluate it if unfixed and
// keep the smaller value.  A point whose value dropped below the window end `win` goes
// on the near list (again, if it was there with a larger value: the first
// copy to be fixed wins); a point seen for the first time at or past it goes
// on the far list.  Values only fall and the window only grows, so a far
// point is either improved into the near list or moved there when the window
// passes it.  One relaxation returns which list the neighbour must join
// (RELAX_NEAR / RELAX_FAR, its index in *qn) or RELAX_NONE; the caller
// appends, warp-wide.
enum { RELAX_NONE = 0, RELAX_NEAR = 1, RELAX_FAR = 2 };

template <typename T, int DIM>
__device__ int fmm_relax_dev(const Geom &g, const T *__restrict__ phi, const ReinitState &st, int x, int y, int z,
                             int s, int sign, T bw, T inf, T lim, T win, int *qn) {
  typedef typename OrdOf<T>::type O;
  O *tent = (O *)st.tent;
  constexpr int kStarDev[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
  const int i = x + kStarDev[s][0], j = y + kStarDev[s][1], k = z + kStarDev[s][2];
  if (i < 0 || i >= g.nx || j < 0 || j >= g.ny || k < 0 || k >= g.nz) return RELAX_NONE;
  const int q = (k * g.ny + j) * g.nx + i;
  if (sign * phi[q] < bw) return RELAX_NONE;  // fixed, or the other side
  const T v = fmm_update_dev<T, DIM>(g, phi, st.mark, i, j, k, sign, inf, lim);
  if (v != v) {
    atomicOr(st.err, 1);
    return RELAX_NONE;
  }
  const O ov = ord_bits(v);
  const O old = atomicMin(&tent[q], ov);
  *qn = q;
  if (v < win) {
    if (ov < old) {
      atomicExch(&st.mark[q], RM_TENT);
      return RELAX_NEAR;
    }
  } else if (atomicCAS(&st.mark[q], RM_FAR, RM_TENT) == RM_FAR) {
    return RELAX_FAR;
  }
  return RELAX_NONE;
}

// Appends `value` of every lane that wants to, with one atomic per warp on
// the list's length (a counter in the cluster's distributed shared memory,
// which all eight CTAs of a side update); called by all 32 lanes.  The lists
// are sets -- which thread handles which entry does not change the march.
__device__ __forceinline__ void warp_append(int *list, int *count, bool want, int value) {
  const unsigned m = __ballot_sync(0xffffffffu, want);
  if (!m) return;
  const int lane = (int)(threadIdx.x & 31), leader = __ffs(m) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(count, __popc(m));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (want) list[base + __popc(m & ((1u << lane) - 1u))] = value;
}

template <typename T>
__global__ void __launch_bounds__(REINIT_THREADS) reinit_init_kernel(T *phi, long long n, T inf, int *mark,
                                                                   void *tent_v, int *err) {
  typedef typename OrdOf<T>::type O;
  O *tent = (O *)tent_v;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    phi[q] = phi[q] > 0 ? inf : -inf;  // FastMarching.c:28-30
    mark[q] = RM_FAR;
    tent[q] = ord_bits((T)INFINITY);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *err = 0;
}

template <typename T, int DIM>
__global__ void __launch_bounds__(REINIT_THREADS) reinit_seed_kernel(Geom g, T *phi, const dcell_irregular_node *nodes,
                                                                   int nnodes, int *mark) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nnodes) return;
  const dcell_irregular_node nd = nodes[r];
  if (nd.axis != -1) return;  // FastMarching.c:57-70
  const int x = nd.pos[0] - g.px, y = nd.pos[1] - g.py, z = DIM == 3 ? nd.pos[2] - g.pz : 0;
  if (x < 0 || x >= g.nx || y < 0 || y >= g.ny || z < 0 || z >= g.nz) return;
  const int q = (z * g.ny + y) * g.nx + x;
  const double len = DIM == 2 ? sqrt(nd.op[0] * nd.op[0] + nd.op[1] * nd.op[1])
                              : sqrt(nd.op[0] * nd.op[0] + nd.op[1] * nd.op[1] + nd.op[2] * nd.op[2]);
  phi[q] = (T)(nd.signCenter * len);
  mark[q] = RM_SEED;
}

// The whole march of one side in one CTA (blockIdx.x 0: sign -1, 1: sign +1):
// the sides touch disjoint points (each only ever reads the other's values,
// which are negative on its scale and so never "known"), so they march
// concurrently from one launch.  Tentative points below the window end
// (REINIT_WINDOW buckets ahead) sit on the near list, which each bucket
// scans; the far list is redistributed when the window moves on.  Per
// bucket: accept, block barrier, relax, block barrier -- no kernel launches;
// list lengths in shared memory.  Acceptance and values are those of the
// single-list procedure (the oracle's): a point is fixed in the bucket its
// value falls in, by the first of its near-list copies to get there.
constexpr int REINIT_MARCH_THREADS = 1024;
constexpr int REINIT_WINDOW = 16;

template <typename T, int DIM>
__global__ void __launch_bounds__(REINIT_MARCH_THREADS) reinit_march_kernel(Geom g, T *phi,
                                                                          const dcell_irregular_node *nodes,
                                                                          int nnodes, ReinitState s0, ReinitState s1,
                                                                          T bw, T inf, T bucket, int nb) {
  typedef typename OrdOf<T>::type O;
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();  // the CTAs of one side (a single CTA without clusters)
  const int rank = (int)cl.block_rank(), nrank = (int)cl.num_blocks();
  const int side = (int)blockIdx.x / nrank;
  const int sign = side == 0 ? -1 : 1;
  const ReinitState st = side == 0 ? s0 : s1;
  O *tent = (O *)st.tent;
  __shared__ ReinitCounts c_rank;
  ReinitCounts &c = *cl.map_shared_rank(&c_rank, 0);  // the side's list lengths, in rank 0's shared memory
  const int tid = rank * (int)blockDim.x + (int)threadIdx.x, nthr = nrank * (int)blockDim.x;
  const bool lead = rank == 0 && threadIdx.x == 0;
  if (lead) c.near[0] = c.near[1] = c.far[0] = c.far[1] = c.acc[0] = c.acc[1] = 0;
  cl.sync();
  int in = 0, fcur = 0;
  T win = bucket * (T)REINIT_WINDOW;
  // every loop below runs a warp-uniform number of rounds (t0 = the warp's
  // first index), so that the appends can be aggregated warp-wide
  const int wtid = tid - (int)(threadIdx.x & 31);
  for (int r0 = wtid; r0 < nnodes * 2 * DIM; r0 += nthr) {  // FastMarching.c:72-84, one neighbour each
    const int r = r0 + (int)(threadIdx.x & 31);
    int req = RELAX_NONE, qn = 0;
    if (r < nnodes * 2 * DIM) {
      const dcell_irregular_node nd = nodes[r / (2 * DIM)];
      const int x = nd.pos[0] - g.px, y = nd.pos[1] - g.py, z = DIM == 3 ? nd.pos[2] - g.pz : 0;
      if (nd.axis == -1 && x >= 0 && x < g.nx && y >= 0 && y < g.ny && z >= 0 && z < g.nz &&
          sign * phi[(z * g.ny + y) * g.nx + x] >= 0)
        req = fmm_relax_dev<T, DIM>(g, phi, st, x, y, z, r % (2 * DIM), sign, bw, inf, -(T)INFINITY, win, &qn);
    }
    warp_append(st.near[in], &c.near[in], req == RELAX_NEAR, qn);
    warp_append(st.far[fcur], &c.far[fcur], req == RELAX_FAR, qn);
  }
  cl.sync();
  for (int b = 0; b < nb; ++b) {
    const T thr = bucket * (T)(b + 1);
    // accept what falls below this bucket's threshold; keep the rest of the window
    const int n_in = c.near[in];
    for (int t0 = wtid; t0 < n_in; t0 += nthr) {
      const int t = t0 + (int)(threadIdx.x & 31);
      const int q = t < n_in ? st.near[in][t] : 0;
      bool acc = false, keep = false;
      if (t < n_in && st.mark[q] != RM_MARCHED) {
        const T v = ord_value(tent[q]);
        if (v < thr && v <= bw) {
          if (atomicCAS(&st.mark[q], RM_TENT, RM_MARCHED) == RM_TENT) {
            phi[q] = sign * v;
            acc = true;
          }
        } else if (v <= bw) {
          keep = true;
        } else {
          st.mark[q] = RM_FAR;  // past the band unless a later push lowers it
        }
      }
      warp_append(st.acc, &c.acc[b & 1], acc, q);
      warp_append(st.near[in ^ 1], &c.near[in ^ 1], keep, q);
    }
    cl.sync();
    const int n_acc = c.acc[b & 1];
    // nobody reads the consumed near list or the other parity's accept count
    // again before the barrier after the relax pass: reset them meanwhile
    if (lead) {
      c.near[in] = 0;
      c.acc[(b + 1) & 1] = 0;
    }
    for (int t0 = wtid; t0 < n_acc * 2 * DIM; t0 += nthr) {  // one (point, neighbour) pair each
      const int t = t0 + (int)(threadIdx.x & 31);
      int req = RELAX_NONE, qn = 0;
      if (t < n_acc * 2 * DIM) {
        const int q = st.acc[t / (2 * DIM)];
        const int x = q % g.nx, y = (q / g.nx) % g.ny, z = q / (g.nx * g.ny);
        req = fmm_relax_dev<T, DIM>(g, phi, st, x, y, z, t % (2 * DIM), sign, bw, inf, sign * phi[q], win, &qn);
      }
      warp_append(st.near[in ^ 1], &c.near[in ^ 1], req == RELAX_NEAR, qn);
      warp_append(st.far[fcur], &c.far[fcur], req == RELAX_FAR, qn);
    }
    cl.sync();
    in ^= 1;
    if ((b + 1) % REINIT_WINDOW == 0) {  // the window moves on: far points now inside it join the near list
      win = bucket * (T)(b + 1 + REINIT_WINDOW);
      const int n_far = c.far[fcur];
      for (int t0 = wtid; t0 < n_far; t0 += nthr) {
        const int t = t0 + (int)(threadIdx.x & 31);
        const int q = t < n_far ? st.far[fcur][t] : 0;
        bool to_near = false, stay = false;
        if (t < n_far && st.mark[q] != RM_MARCHED) {
          const T v = ord_value(tent[q]);
          if (v < win) {
            if (v <= bw) {
              st.mark[q] = RM_TENT;
              to_near = true;
            } else {
              st.mark[q] = RM_FAR;
            }
          } else {
            stay = true;
          }
        }
        warp_append(st.near[in], &c.near[in], to_near, q);
        warp_append(st.far[fcur ^ 1], &c.far[fcur ^ 1], stay, q);
      }
      cl.sync();
      // the consumed far list's length is read again only at the next
      // redistribution, many barriers later
      if (lead) c.far[fcur] = 0;
      fcur ^= 1;
    }
  }
  // still tentative (within the band) after the last bucket
  bool left = false;
  for (int t = tid; t < c.near[in]; t += nthr)
    if (st.mark[st.near[in][t]] == RM_TENT && ord_value(tent[st.near[in][t]]) <= bw) left = true;
  for (int t = tid; t < c.far[fcur]; t += nthr)
    if (st.mark[st.far[fcur][t]] == RM_TENT && ord_value(tent[st.far[fcur][t]]) <= bw) left = true;
  if (left) atomicOr(st.err, 2);
  cl.sync();  // rank 0's shared counters stay alive until every CTA of the side is done with them
}

__global__ void __launch_bounds__(REINIT_THREADS) reinit_band_flags_kernel(const int *mark, long long n, int *flag) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    flag[q] = mark[q] >= RM_MARCHED ? 1 : 0;
}

__global__ void __launch_bounds__(REINIT_THREADS) reinit_band_write_kernel(Geom g, const int *mark, const int *offs,
                                                                         long long n, int *band, int cap) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    if (mark[q] >= RM_MARCHED) {
      const int o = offs[q];
      if (o < cap) {
        band[3 * o + 0] = g.px + (int)(q % g.nx);
        band[3 * o + 1] = g.py + (int)((q / g.nx) % g.ny);
        band[3 * o + 2] = g.pz + (int)(q / ((long long)g.nx * g.ny));
      }
    }
}

__global__ void reinit_status_kernel(const int *err, int *flags) {
  if (*err & 1) raise_flag(flags, FLAG_NONFINITE);
  if (*err & 2) raise_flag(flags, FLAG_UNSETTLED);
}

// ---------------------------------------------------------------------------
// First-order conservative upwind step on MAC faces: LevelSetAdvectMAC and
// LevelSetAdvectMAC_3D (LevelSetMethod/AdvectMAC.c:18-111), the reference's
// expressions in its operation order (this unit is compiled without FMA
// contraction, so FP64 gives its bits).  u / v / w hold at (i, j, k) the face
// between cells i-1 and i along x / y / z.  At global index 0 and at the
// range's last point the missing neighbour is extrapolated as
// 2 phi - (the other neighbour) (AdvectMAC.c:83-88).  Every read stays in the
// grid: the caller admits only updated ranges [s, e) with p <= 0 and n >= 3.
//
// A thread owns one (i, j) column and marches kMacChunk planes of the updated
// z range upwards, carrying phi at k-1 and k and w at k in registers: per
// point it loads phi's four x/y neighbours and plane k+1, u at i and i+1, v at
// j and j+1 and w at k+1 (10 loads instead of 13), and the loads of the next
// planes do not wait for this plane's arithmetic.  Bound: HBM (4 arrays read
// and one written per point; the neighbour re-reads hit L1/L2).
constexpr int kMacChunk = 8;

template <typename T, int DIM>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 8 : 6)
    advect_mac_kernel(Geom g, const T *__restrict__ phi, const T *__restrict__ u, const T *__restrict__ v,
                      const T *__restrict__ w, T dt, int xs, int xe, int ys, int ye, int zs, int ze,
                      T *__restrict__ out) {
  const int i = xs + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= xe) return;
  const T hx = (T)g.hx, hy = (T)g.hy, hz = (T)g.hz;
  const int sy = g.nx, sz = g.nx * g.ny;
  for (int j = ys + (int)(blockIdx.y * blockDim.y + threadIdx.y); j < ye; j += (int)(gridDim.y * blockDim.y))
    for (int k0 = zs + (int)blockIdx.z * kMacChunk; k0 < ze; k0 += (int)gridDim.z * kMacChunk) {
      const int k1 = min(k0 + kMacChunk, ze);
      int c = (k0 - g.pz) * sz + (j - g.py) * sy + (i - g.px);
      T p = __ldg(phi + c), below = T(0), w0 = T(0);
      if (DIM == 3) {
        below = k0 > g.pz ? __ldg(phi + c - sz) : T(0);  // read where k > 0 or k == ze-1: both imply k0 > p_z
        w0 = __ldg(w + c);
      }
#pragma unroll(sizeof(T) == 4 ? 2 : 4)
      for (int k = k0; k < k1; ++k, c += sz) {
        const T am = i == 0 ? T(2) * p - __ldg(phi + c + 1) : __ldg(phi + c - 1);
        const T an = i == xe - 1 ? T(2) * p - __ldg(phi + c - 1) : __ldg(phi + c + 1);
        const T bm = j == 0 ? T(2) * p - __ldg(phi + c + sy) : __ldg(phi + c - sy);
        const T bn = j == ye - 1 ? T(2) * p - __ldg(phi + c - sy) : __ldg(phi + c + sy);
        const T u0 = __ldg(u + c), u1 = __ldg(u + c + 1);
        const T v0 = __ldg(v + c), v1 = __ldg(v + c + sy);
        T du = u0 > T(0) ? am * u0 : p * u0;
        T dv = v0 > T(0) ? bm * v0 : p * v0;
        du -= u1 > T(0) ? p * u1 : an * u1;
        dv -= v1 > T(0) ? p * v1 : bn * v1;
        if (DIM == 3) {
          const T above = __ldg(phi + c + sz);  // plane k+1 <= e is in the grid
          const T w1 = __ldg(w + c + sz);
          const T cm = k == 0 ? T(2) * p - above : below;
          const T cn = k == ze - 1 ? T(2) * p - below : above;
          T dw = w0 > T(0) ? cm * w0 : p * w0;
          dw -= w1 > T(0) ? p * w1 : cn * w1;
          out[c] = p + dt * (du / hx + dv / hy + dw / hz);
          below = p;
          p = above;
          w0 = w1;
        } else {
          out[c] = p + dt * (du / hx + dv / hy);
        }
      }
    }
}

}  // namespace dcell

// ===========================================================================
// Launchers (declared in dcell_kernels.h)
using namespace dcell;

size_t scan_partial_ints(long long n) { return (size_t)((n + SCAN_BLOCK - 1) / SCAN_BLOCK) + 1; }

int launch_scan_exclusive(const int *in, int n, int *out, int *partial, int *total, int cap, int *flags,
                          cudaStream_t st) {
  if (n <= 0) return cudaMemsetAsync(total, 0, sizeof(int), st) == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
  const int nblk = (n + SCAN_BLOCK - 1) / SCAN_BLOCK;
  scan_blocks_kernel<<<nblk, SCAN_BLOCK, 0, st>>>(in, n, out, partial);
  scan_partials_kernel<<<1, SCAN_BLOCK, 0, st>>>(partial, nblk);
  scan_add_kernel<<<nblk, SCAN_BLOCK, 0, st>>>(out, n, partial, nblk, total, cap, flags);
  return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
}


static inline int grid_for(long long n, int threads) {
  long long b = (n + threads - 1) / threads;
  if (b > 148LL * 64) b = 148LL * 64;
  return (int)(b < 1 ? 1 : b);
}

int launch_sl_linear(const Geom &g, int dtype, const void *phi0, const void *vel, double dt, const int *band,
                     long long npts, int backtrace, void *phi, int *flags, cudaStream_t st, bool gather) {
  const int threads = 256, blocks = grid_for(npts, threads);
  const bool is2d = g.nz == 1;
  // FP32 runs the fast unit (sl_lin.cu); this one keeps the reference's
  // FP64 operation order
  if (dtype == DCELL_F32)
    return launch_sl_lin_f32(g, (const float *)phi0, (const float *)vel, dt, band, npts, backtrace, (float *)phi,
                             flags, st, gather);
  if (is2d)
    sl_linear_kernel<double, 2><<<blocks, threads, 0, st>>>(g, (const double *)phi0, (const double *)vel, dt, band,
                                                            npts, backtrace, (double *)phi, flags);
  else
    sl_linear_kernel<double, 3><<<blocks, threads, 0, st>>>(g, (const double *)phi0, (const double *)vel, dt, band,
                                                            npts, backtrace, (double *)phi, flags);
  return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
}

size_t irregular_scratch_bytes(int nband) {
  const size_t nblk = ((size_t)nband + SCAN_BLOCK - 1) / SCAN_BLOCK;
  return sizeof(int) * ((size_t)nband + 1 + nblk + 1) + 256;
}

template <typename T, int DIM>
static void irr_launch(const Geom &g, const T *phi, const int *band, int nband, int with_surface,
                       dcell_irregular_node *nodes, int cap, int *count, int *offsets, int *partial, int *flags,
                       cudaStream_t st) {
  const int nblk = (nband + SCAN_BLOCK - 1) / SCAN_BLOCK;
  irr_count_kernel<T, DIM><<<(nband + 255) / 256, 256, 0, st>>>(g, phi, band, nband, offsets);
  scan_blocks_kernel<<<nblk, SCAN_BLOCK, 0, st>>>(offsets, nband, offsets, partial);
  scan_partials_kernel<<<1, SCAN_BLOCK, 0, st>>>(partial, nblk);
  scan_add_kernel<<<nblk, SCAN_BLOCK, 0, st>>>(offsets, nband, partial, nblk, count, cap, flags);
  irr_write_kernel<T, DIM><<<(nband + 255) / 256, 256, 0, st>>>(g, phi, band, nband, offsets, nodes, cap);
  // projection nodes: 8 threads each; bounded by the capacity
  // the node count is on the device: grids sized for the capacity, capped,
  // and the kernels loop over the nodes actually written
  const long long nthreads = 8LL * cap;
  const int ob = (int)std::min<long long>((nthreads + 255) / 256, 148LL * 24);
  const int sb = (int)std::min<long long>((nthreads + 127) / 128, 148LL * 48);
  ortho_kernel<T, DIM><<<ob < 1 ? 1 : ob, 256, 0, st>>>(g, phi, nodes, count, cap);
  if (with_surface) surface_kernel<T, DIM><<<sb < 1 ? 1 : sb, 128, 0, st>>>(g, phi, nodes, count, cap);
}

int launch_irregular(const Geom &g, int dtype, const void *phi, const int *band, int nband, int with_surface,
                     dcell_irregular_node *nodes, int cap, int *count, void *scratch, int *flags, cudaStream_t st) {
  int *offsets = (int *)scratch;
  int *partial = offsets + nband + 1;
  if (nband == 0) {
    cudaMemsetAsync(count, 0, sizeof(int), st);
    return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
  }
  const bool is2d = g.nz == 1;
  if (dtype == DCELL_F64) {
    if (is2d) irr_launch<double, 2>(g, (const double *)phi, band, nband, with_surface, nodes, cap, count, offsets, partial, flags, st);
    else irr_launch<double, 3>(g, (const double *)phi, band, nband, with_surface, nodes, cap, count, offsets, partial, flags, st);
  } else {
    if (is2d) irr_launch<float, 2>(g, (const float *)phi, band, nband, with_surface, nodes, cap, count, offsets, partial, flags, st);
    else irr_launch<float, 3>(g, (const float *)phi, band, nband, with_surface, nodes, cap, count, offsets, partial, flags, st);
  }
  return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
}

int launch_max_velocity(const Geom &g, int dtype, const void *vel, const dcell_irregular_node *nodes,
                        const int *count, int cap, double *out, cudaStream_t st) {
  cudaMemsetAsync(out, 0, sizeof(double), st);
  if (cap <= 0) return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
  const int blocks = (cap + 255) / 256;
  unsigned long long *o = (unsigned long long *)out;
  const bool is2d = g.nz == 1;
  if (dtype == DCELL_F64) {
    if (is2d) maxvel_kernel<double, 2><<<blocks, 256, 0, st>>>(g, (const double *)vel, nodes, count, cap, o);
    else maxvel_kernel<double, 3><<<blocks, 256, 0, st>>>(g, (const double *)vel, nodes, count, cap, o);
  } else {
    if (is2d) maxvel_kernel<float, 2><<<blocks, 256, 0, st>>>(g, (const float *)vel, nodes, count, cap, o);
    else maxvel_kernel<float, 3><<<blocks, 256, 0, st>>>(g, (const float *)vel, nodes, count, cap, o);
  }
  return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
}


int launch_advect_mac(const Geom &g, int dtype, const void *phi, const void *u, const void *v, const void *w, double dt,
                      const int range[6], void *out, cudaStream_t st) {
  const int X = range[1] - range[0], Y = range[3] - range[2], Z = range[5] - range[4];
  if (X <= 0 || Y <= 0 || Z <= 0) return DCELL_OK;
  const dim3 block(32, 8);
  const dim3 grid((unsigned)((X + 31) / 32), (unsigned)min((Y + 7) / 8, 65535),
                  (unsigned)min((Z + kMacChunk - 1) / kMacChunk, 65535));
  const bool is2d = g.nz == 1;
#define DCELL_MAC_LAUNCH(T, D)                                                                                    \
  advect_mac_kernel<T, D><<<grid, block, 0, st>>>(g, (const T *)phi, (const T *)u, (const T *)v, (const T *)w,   \
                                                  (T)dt, range[0], range[1], range[2], range[3], range[4], range[5], \
                                                  (T *)out)
  if (dtype == DCELL_F64) {
    if (is2d) DCELL_MAC_LAUNCH(double, 2);
    else DCELL_MAC_LAUNCH(double, 3);
  } else {
    if (is2d) DCELL_MAC_LAUNCH(float, 2);
    else DCELL_MAC_LAUNCH(float, 3);
  }
#undef DCELL_MAC_LAUNCH
  return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
}

// ---------------------------------------------------------------------------
// Reinitialisation.  Scratch layout (bytes, each part 256-aligned): mark
// int[n]; tentative values [n] (8 or 4 bytes; the sides touch disjoint
// points, so they share it); per side two near lists, two far lists and an
// accepted list, int[n] each; the error word; the band scan's block totals.
// The band scan reuses the first list.
static size_t align256(size_t v) { return (v + 255) / 256 * 256; }

size_t reinit_scratch_bytes(long long n, int dtype) {
  const size_t w = dtype == DCELL_F64 ? 8 : 4;
  const size_t nblk = ((size_t)n + SCAN_BLOCK - 1) / SCAN_BLOCK;
  return align256(sizeof(int) * n) + align256(w * n) + 10 * align256(sizeof(int) * n) + align256(sizeof(int) * 8) +
         align256(sizeof(int) * (nblk + 1));
}

// CTAs per side of the march (a thread-block cluster): 8, or
// DCELL_REINIT_CLUSTER (1, 2, 4 or 8)
static int reinit_cluster() {
  static int cl = 0;
  if (!cl) {
    const char *e = getenv("DCELL_REINIT_CLUSTER");
    const int v = e ? atoi(e) : 8;
    cl = (v == 1 || v == 2 || v == 4 || v == 8) ? v : 8;
  }
  return cl;
}

template <typename T, int DIM>
static void reinit_run(const Geom &g, T *phi, const dcell_irregular_node *nodes, int nnodes, T bw, T bucket,
                       int *band, int cap, int *count, uint8_t *sc, int *flags, cudaStream_t st) {
  const long long n = (long long)g.nx * g.ny * g.nz;
  size_t off = 0;
  int *mark = (int *)(sc + off); off += align256(sizeof(int) * n);
  void *tent = sc + off; off += align256(sizeof(T) * n);
  ReinitState side[2];
  for (int k = 0; k < 2; ++k) {
    side[k].mark = mark;
    side[k].tent = tent;
    for (int l = 0; l < 2; ++l) {
      side[k].near[l] = (int *)(sc + off); off += align256(sizeof(int) * n);
      side[k].far[l] = (int *)(sc + off); off += align256(sizeof(int) * n);
    }
    side[k].acc = (int *)(sc + off); off += align256(sizeof(int) * n);
  }
  int *err = (int *)(sc + off); off += align256(sizeof(int) * 8);
  side[0].err = side[1].err = err;
  int *partial = (int *)(sc + off);
  const T inf = bw + T(1.5);  // PHI_INF, LevelSet.c:64
  const int dense = grid_for(n, REINIT_THREADS);
  reinit_init_kernel<T><<<dense, REINIT_THREADS, 0, st>>>(phi, n, inf, mark, tent, err);
  if (nnodes > 0)
    reinit_seed_kernel<T, DIM><<<(nnodes + REINIT_THREADS - 1) / REINIT_THREADS, REINIT_THREADS, 0, st>>>(
        g, phi, nodes, nnodes, mark);
  const int nb = (int)ceil((double)bw / (double)bucket) + REINIT_TAIL;
  // each side a cluster of reinit_cluster() CTAs; one CTA per side where
  // clusters of that size cannot be scheduled
  bool launched = false;
  for (int cl = reinit_cluster(); cl > 1 && !launched; cl >>= 1) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(2 * cl);
    cfg.blockDim = dim3(REINIT_MARCH_THREADS);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cl;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    launched = cudaLaunchKernelEx(&cfg, reinit_march_kernel<T, DIM>, g, phi, nodes, nnodes, side[0], side[1], bw, inf,
                                  bucket, nb) == cudaSuccess;
    if (!launched) cudaGetLastError();
  }
  if (!launched)
    reinit_march_kernel<T, DIM><<<2, REINIT_MARCH_THREADS, 0, st>>>(g, phi, nodes, nnodes, side[0], side[1], bw, inf,
                                                                    bucket, nb);
  reinit_status_kernel<<<1, 1, 0, st>>>(err, flags);
  // band: the fixed points in grid order
  int *flag = side[0].near[0], *offs = side[0].near[0];
  const int nblk = (int)((n + SCAN_BLOCK - 1) / SCAN_BLOCK);
  reinit_band_flags_kernel<<<dense, REINIT_THREADS, 0, st>>>(mark, n, flag);
  scan_blocks_kernel<<<nblk, SCAN_BLOCK, 0, st>>>(flag, (int)n, offs, partial);
  scan_partials_kernel<<<1, SCAN_BLOCK, 0, st>>>(partial, nblk);
  scan_add_kernel<<<nblk, SCAN_BLOCK, 0, st>>>(offs, (int)n, partial, nblk, count, cap, flags);
  reinit_band_write_kernel<<<dense, REINIT_THREADS, 0, st>>>(g, mark, offs, n, band, cap);
}

int launch_reinit(const Geom &g, int dtype, void *phi, const dcell_irregular_node *nodes, int nnodes, double bw,
                  double bucket, int *band, int cap, int *count, void *scratch, int *flags, cudaStream_t st) {
  const bool is2d = g.nz == 1;
  uint8_t *sc = (uint8_t *)scratch;
  if (dtype == DCELL_F64) {
    if (is2d) reinit_run<double, 2>(g, (double *)phi, nodes, nnodes, bw, bucket, band, cap, count, sc, flags, st);
    else reinit_run<double, 3>(g, (double *)phi, nodes, nnodes, bw, bucket, band, cap, count, sc, flags, st);
  } else {
    if (is2d) reinit_run<float, 2>(g, (float *)phi, nodes, nnodes, (float)bw, (float)bucket, band, cap, count, sc, flags, st);
    else reinit_run<float, 3>(g, (float *)phi, nodes, nnodes, (float)bw, (float)bucket, band, cap, count, sc, flags, st);
  }
  return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
}

size_t volume_scratch_bytes() { return sizeof(double) * VOL_BLOCKS; }

int launch_volume(const Geom &g, int dtype, const void *phi, double eps, double *out, double *partial,
                  cudaStream_t st) {
  const long long n = (long long)g.nx * g.ny * g.nz;
  const double cell = g.hx * g.hy * (g.nz == 1 ? 1.0 : g.hz);
  if (dtype == DCELL_F64)
    volume_partial_kernel<double><<<VOL_BLOCKS, VOL_THREADS, 0, st>>>((const double *)phi, n, eps, partial);
  else
    volume_partial_kernel<float><<<VOL_BLOCKS, VOL_THREADS, 0, st>>>((const float *)phi, n, eps, partial);
  volume_final_kernel<<<1, 32, 0, st>>>(partial, cell, out);
  return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of the irregular-node pass.
//
// The scan scratch of launch_irregular lives in this file-scope device array
// instead of a caller buffer.  Every GPU that loads the library holds it
// (about 4 MiB) until the process exits; all calls on a device share it, so
// calls that overlap on the GPU race.  Every scratch entry is written before
// it is read, so nothing needs clearing between calls.  The host cannot use
// the array's name as a device address: its address is looked up once per
// device with cudaGetSymbolAddress, on the first call made with that device
// current.
static_assert(kNoAllocScratchInts >= kNoAllocMaxBand + 1 + (kNoAllocMaxBand + SCAN_BLOCK - 1) / SCAN_BLOCK + 1,
              "allocation-free scratch smaller than the scan layout of launch_irregular");
static __device__ __align__(256) int g_irr_noalloc_scratch[kNoAllocScratchInts];

namespace {
std::mutex g_noalloc_mu;
int *g_noalloc_ptr[kNoAllocMaxDevices] = {};
}  // namespace

static int noalloc_scratch(int **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    dcell_set_error(DCELL_ERR_CUDA, "cudaGetDevice failed: %s", cudaGetErrorString(e));
    return DCELL_ERR_CUDA;
  }
  if (dev < 0 || dev >= kNoAllocMaxDevices) {
    dcell_set_error(DCELL_ERR_UNSUPPORTED, "device %d beyond the %d devices the allocation-free path tracks", dev,
                    kNoAllocMaxDevices);
    return DCELL_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_irr_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      dcell_set_error(DCELL_ERR_CUDA, "cudaGetSymbolAddress of the allocation-free scratch failed: %s",
                      cudaGetErrorString(e));
      return DCELL_ERR_CUDA;
    }
    g_noalloc_ptr[dev] = (int *)p;
  }
  *out = g_noalloc_ptr[dev];
  return DCELL_OK;
}

int launch_irregular_noalloc(const Geom &g, int dtype, const void *phi, const int *band, int nband,
                             int with_surface, dcell_irregular_node *nodes, int cap, int *count, int *flags,
                             cudaStream_t st) {
  if (nband > kNoAllocMaxBand) {
    dcell_set_error(DCELL_ERR_ARG, "band of %d points exceeds the allocation-free maximum of %d", nband,
                    kNoAllocMaxBand);
    return DCELL_ERR_ARG;
  }
  int *scratch = nullptr;
  const int rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  return launch_irregular(g, dtype, phi, band, nband, with_surface, nodes, cap, count, scratch, flags, st);
}
