// Particle level set (LevelSetMethod/ParticleLS.c, ParticleLS2D.c,
// ParticleLS3D.c) on the GPU.
//
// Compiled with -fmad=false, like the other reference-exact kernels: in FP64
// every particle position, radius and corrected phi value is bit-identical to
// the reference's (the CPU restatement in the oracle pins both).  Particles
// are records of four values (X.x, X.y, X.z, radius), struct _Particle of
// LevelSetMethod/LSM_private.h:45-48, one thread per particle.
//
//   pls_advect_kernel    ParticleLS_AdvectParticles2D/3D: RK2 midpoint
//   pls_escape_kernel    ErrorCorrection: escaped particles raise phi+ / lower
//                        phi- at their cell corners (order-preserving integer
//                        atomics: max / min do not depend on particle order)
//   pls_merge_kernel     ErrorCorrection: band points take phi+ or phi-
//   pls_adjust_kernel    ParticleLS_AdjustRadii
//   pls_seed_kernel      LevelSetInitializeParticles' seeding: particle k uses
//                        draws 5k .. 5k+4 of the drand48 stream (jump-ahead)
//   reseed               ParticleLS_ReseedParticles: keep flags, a scan, the
//                        swap-with-last deletion order as a permutation, cell
//                        counts, per-cell deficits and their scan; one thread
//                        walks the random stream (its rejection loop makes the
//                        draw count data dependent), then every new particle
//                        is attracted in parallel.
#include <math.h>

#include "dcell_common.cuh"
#include "dcell_kernels.h"
#include "ref_ops.cuh"
#include "sl_device.cuh"

namespace dcell {

constexpr unsigned long long R48_A = 0x5DEECE66DULL, R48_C = 0xBULL, R48_MASK = 0xFFFFFFFFFFFFULL;
constexpr int REJECT_LIMIT = 1 << 20;  // bound of the phi_goal rejection loop (the reference has none)

// drand48 (POSIX): X <- (a X + c) mod 2^48, value X / 2^48 (exact in FP64).
__device__ __forceinline__ double r48_next(unsigned long long &x) {
  x = (R48_A * x + R48_C) & R48_MASK;
  return (double)x * (1.0 / 281474976710656.0);
}

// The state k draws after x: the affine map x -> a x + c composed k times by
// squaring (arithmetic mod 2^64, reduced mod 2^48 at the end).
__device__ __forceinline__ unsigned long long r48_skip(unsigned long long x, unsigned long long k) {
  unsigned long long A = 1, C = 0, a = R48_A, c = R48_C;
  while (k) {
    if (k & 1) {
      A = a * A;
      C = a * C + c;
    }
    c = a * c + c;
    a = a * a;
    k >>= 1;
  }
  return (A * x + C) & R48_MASK;
}

template <typename T>
__device__ __forceinline__ T psign(T a) {  // PetscSign
  return a >= T(0) ? (a == T(0) ? T(0) : T(1)) : T(-1);
}

// GridInterpolate2D/3D (Common/Grid.c:351-410), same loop and operation order.
template <typename T, int DIM>
__device__ __forceinline__ T grid_interp(const Geom &g, const T *__restrict__ f, const T X[3]) {
  const int xs = (int)floor(X[0]), ys = (int)floor(X[1]);
  const T sx = X[0] - (T)xs, sy = X[1] - (T)ys;
  T val = 0;
  if (DIM == 2) {
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int i = 0; i < 2; ++i)
        val += ((1 - sx) * (T)(1 - i) + (T)i * sx) * ((1 - sy) * (T)(1 - j) + (T)j * sy) * f[gidx(g, xs + i, ys + j, 0)];
    return val;
  }
  const int zs = (int)floor(X[2]);
  const T sz = X[2] - (T)zs;
#pragma unroll
  for (int k = 0; k < 2; ++k)
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int i = 0; i < 2; ++i)
        val += ((1 - sx) * (T)(1 - i) + (T)i * sx) * ((1 - sy) * (T)(1 - j) + (T)j * sy) *
               ((1 - sz) * (T)(1 - k) + (T)k * sz) * f[gidx(g, xs + i, ys + j, zs + k)];
  return val;
}

// The sampling used by the particle kernels: in FP64 the reference's own
// expressions (bit-identical results); in FP32 the production form of the SL
// kernels -- local coordinates, one subtraction and one fused multiply-add
// per linear interpolation (24 -> 7 operations per component), within FP32
// rounding of the reference.
template <typename T, int DIM>
__device__ __forceinline__ void vel_at(const Geom &g, const T *__restrict__ vel, const T X[3], T V[3]) {
  if constexpr (sizeof(T) == 4) {
    const T xl[3] = {X[0] - (T)g.px, X[1] - (T)g.py, DIM == 3 ? X[2] - (T)g.pz : T(0)};
    mac_vel_rel<T, DIM>(g, vel, 0, 0, 0, xl, V);
  } else if (DIM == 3) {
    interp_vel3<T>(g, vel, X, V);
  } else {
    interp_vel2<T>(g, vel, X, V);
  }
}

// FP32 MAC velocity at X and whether every stencil lies in the grid: per
// axis the cell and the half-staggered cell are floored once and shared by
// the three components and the test (the values equal mac_vel_rel's).
template <int DIM>
__device__ __forceinline__ void vel_at_f32(const Geom &g, const float *__restrict__ vel, const float X[3], float V[3],
                                           bool &inside) {
  const int p[3] = {g.px, g.py, g.pz}, n[3] = {g.nx, g.ny, g.nz};
  int i0[3] = {0, 0, 0}, i1[3] = {0, 0, 0};
  float s0[3] = {0.f, 0.f, 0.f}, s1[3] = {0.f, 0.f, 0.f};
#pragma unroll
  for (int a = 0; a < DIM; ++a) {
    const float xl = X[a] - (float)p[a], t1 = xl + 0.5f;
    const float f0 = floorf(xl), f1 = floorf(t1);
    i0[a] = (int)f0;
    i1[a] = (int)f1;
    s0[a] = xl - f0;
    s1[a] = t1 - f1;
    inside = inside && i0[a] >= 0 && i1[a] + 1 <= n[a] - 1;
  }
  const int pitch[3] = {DIM, DIM * g.nx, DIM * g.nx * g.ny};
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    int off = d, o[3] = {0, 0, 0};
    float s[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
      const int b = a == d ? i1[a] : i0[a];
      const int bc = clampi(b, 0, n[a] - 1);
      o[a] = (clampi(b + 1, 0, n[a] - 1) - bc) * pitch[a];
      off += bc * pitch[a];
      s[a] = a == d ? s1[a] : s0[a];
    }
    const float *c = vel + off;
    if (DIM == 3) {
      const float *c2 = c + o[2];
      V[d] = trilerp(__ldg(c), __ldg(c + o[0]), __ldg(c + o[1]), __ldg(c + o[1] + o[0]), __ldg(c2), __ldg(c2 + o[0]),
                     __ldg(c2 + o[1]), __ldg(c2 + o[1] + o[0]), s);
    } else {
      V[d] = bilerp(__ldg(c), __ldg(c + o[0]), __ldg(c + o[1]), __ldg(c + o[1] + o[0]), s[0], s[1]);
    }
  }
  if (DIM == 2) V[2] = 0.f;
}

template <typename T, int DIM>
__device__ __forceinline__ T phi_at(const Geom &g, const T *__restrict__ f, const T X[3]) {
  if constexpr (sizeof(T) == 4) {
    const int p[3] = {g.px, g.py, g.pz}, n[3] = {g.nx, g.ny, g.nz};
    int b[3], o[3];
    T s[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      if (a == 2 && DIM == 2) {
        b[2] = 0, o[2] = 0, s[2] = T(0);
        continue;
      }
      const T t = X[a] - (T)p[a], fl = floor(t);
      const int lo = (int)fl;
      b[a] = clampi(lo, 0, n[a] - 1);
      o[a] = clampi(lo + 1, 0, n[a] - 1) - b[a];
      s[a] = t - fl;
    }
    const T *c = f + ((long long)b[2] * g.ny + b[1]) * g.nx + b[0];
    const int ox = o[0], oy = o[1] * g.nx;
    if (DIM == 2) return bilerp(__ldg(c), __ldg(c + ox), __ldg(c + oy), __ldg(c + oy + ox), s[0], s[1]);
    const T *c2 = c + (long long)o[2] * g.nx * g.ny;
    return trilerp(__ldg(c), __ldg(c + ox), __ldg(c + oy), __ldg(c + oy + ox), __ldg(c2), __ldg(c2 + ox),
                   __ldg(c2 + oy), __ldg(c2 + oy + ox), s);
  } else {
    return grid_interp<T, DIM>(g, f, X);
  }
}

// Whether the 2^DIM stencils of X (cell and MAC-staggered) lie in the grid.
template <typename T, int DIM>
__device__ __forceinline__ bool stencil_inside(const Geom &g, const T X[3]) {
  const int p[3] = {g.px, g.py, g.pz}, n[3] = {g.nx, g.ny, g.nz};
#pragma unroll
  for (int a = 0; a < DIM; ++a) {
    const int lo = (int)floor(X[a]), hi = (int)floor(X[a] + T(0.5)) + 1;
    if (!(lo >= p[a] && hi <= p[a] + n[a] - 1)) return false;
  }
  return true;
}

// One particle record; VEC (FP32 records on a 16-byte aligned array, chosen
// at launch): one 16-byte access instead of four.
template <typename T, bool VEC = false>
__device__ __forceinline__ void load4(const T *__restrict__ parts, long long i, T p[4]) {
  if constexpr (VEC && sizeof(T) == 4) {
    const float4 v = reinterpret_cast<const float4 *>(parts)[i];
    p[0] = v.x;
    p[1] = v.y;
    p[2] = v.z;
    p[3] = v.w;
  } else {
#pragma unroll
    for (int c = 0; c < 4; ++c) p[c] = parts[4 * i + c];
  }
}
template <typename T, bool VEC = false>
__device__ __forceinline__ void store4(T *__restrict__ parts, long long i, const T p[4]) {
  if constexpr (VEC && sizeof(T) == 4) {
    reinterpret_cast<float4 *>(parts)[i] = make_float4(p[0], p[1], p[2], p[3]);
  } else {
#pragma unroll
    for (int c = 0; c < 4; ++c) parts[4 * i + c] = p[c];
  }
}

// ParticleLS_AdvectParticles2D/3D (ParticleLS2D.c:6-36, ParticleLS3D.c:6-36).
// FP64 keeps the reference's expressions (its bits); FP32 scales the
// velocities by kh = dt/(2h) and kf = dt/h, formed on the host in FP64 and
// rounded once (within FP32 rounding of the reference's divisions).
template <typename T, int DIM, bool VEC>
__global__ void __launch_bounds__(256) pls_advect_kernel(Geom g, const T *__restrict__ vel, T *__restrict__ parts,
                                                         long long n, T dt, float3 kh, float3 kf, int *flags) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  T p[4];
  load4<T, VEC>(parts, i, p);
  const T hx = (T)g.hx, hy = (T)g.hy, hz = (T)g.hz;
  T V1[3], V2[3], X[3];
  bool inside = true;
  if constexpr (sizeof(T) == 4) {
    vel_at_f32<DIM>(g, vel, p, V1, inside);
    X[0] = p[0] + V1[0] * kh.x;
    X[1] = p[1] + V1[1] * kh.y;
    X[2] = DIM == 3 ? p[2] + V1[2] * kh.z : p[2];
    vel_at_f32<DIM>(g, vel, X, V2, inside);
    p[0] += V2[0] * kf.x;
    p[1] += V2[1] * kf.y;
    if (DIM == 3) p[2] += V2[2] * kf.z;
  } else {
    inside = stencil_inside<T, DIM>(g, p);
    vel_at<T, DIM>(g, vel, p, V1);
    X[0] = p[0] + dt / T(2) * V1[0] / hx;
    X[1] = p[1] + dt / T(2) * V1[1] / hy;
    X[2] = DIM == 3 ? p[2] + dt / T(2) * V1[2] / hz : p[2];
    inside = inside && stencil_inside<T, DIM>(g, X);
    vel_at<T, DIM>(g, vel, X, V2);
    p[0] += dt * V2[0] / hx;
    p[1] += dt * V2[1] / hy;
    if (DIM == 3) p[2] += dt * V2[2] / hz;
  }
  store4<T, VEC>(parts, i, p);
  if (!inside) raise_flag(flags, FLAG_PARTICLE_OUTSIDE);
}

// ErrorCorrection, identification and phi+/phi- (ParticleLS2D.c:65-97,
// ParticleLS3D.c:65-98).  pos / neg hold order-preserving images of phi+ and
// phi- over phi's grid, 0 / all ones meaning "phi itself".
//
// FP32: the particles of a warp usually share a cell and so the same corners;
// their scatters are aggregated per (grid point, side) with warp reductions,
// one atomic per group (max and min do not depend on the order, so the result
// is the same).
template <typename T, int DIM, bool VEC>
__global__ void __launch_bounds__(256) pls_escape_kernel(Geom g, const T *__restrict__ phi,
                                                         const T *__restrict__ parts, long long n,
                                                         typename OrdOf<T>::type *pos, typename OrdOf<T>::type *neg,
                                                         int *flags) {
  const long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (m >= n) return;
  T p[4];
  load4<T, VEC>(parts, m, p);
  const T dist = phi_at<T, DIM>(g, phi, p);
  const T sign = psign(p[3]);
  const bool esc = sign * dist < T(0) && fabs(dist) > fabs(p[3]);
  if constexpr (sizeof(T) == 4) {
    const unsigned act = __activemask();  // the lanes with a particle
    if (!__any_sync(act, esc)) return;
    const int lane = threadIdx.x & 31;
    const int A[3] = {(int)floor(p[0]), (int)floor(p[1]), DIM == 3 ? (int)floor(p[1]) : 0};
    bool outside = false;
#pragma unroll
    for (int c = 0; c < (DIM == 3 ? 8 : 4); ++c) {
      const int a[3] = {A[0] + (c & 1), A[1] + ((c >> 1) & 1), A[2] + (c >> 2)};
      const int lx = a[0] - g.px, ly = a[1] - g.py, lz = DIM == 3 ? a[2] - g.pz : 0;
      const bool in = (unsigned)lx < (unsigned)g.nx && (unsigned)ly < (unsigned)g.ny && (unsigned)lz < (unsigned)g.nz;
      outside = outside || (esc && !in);
      T d2 = (p[0] - (T)a[0]) * (p[0] - (T)a[0]) + (p[1] - (T)a[1]) * (p[1] - (T)a[1]);
      if (DIM == 3) d2 = d2 + (p[2] - (T)a[2]) * (p[2] - (T)a[2]);
      const T phi_p = sign * (sign * p[3] - sqrt(d2));
      const unsigned bits = ord_bits(phi_p);
      const long long key = esc && in ? 2LL * ((lz * g.ny + ly) * g.nx + lx) + (sign > T(0) ? 1 : 0) : -1LL;
      unsigned pending = __ballot_sync(act, key >= 0);
      while (pending) {  // one round per distinct (grid point, side) in the warp
        const int leader = __ffs(pending) - 1;
        const long long lk = __shfl_sync(act, key, leader);
        const bool mine = key == lk;
        const unsigned vmax = __reduce_max_sync(act, mine ? bits : 0u);
        const unsigned vmin = __reduce_min_sync(act, mine ? bits : ~0u);
        if (lane == leader) {
          if (lk & 1) atomicMax(pos + (lk >> 1), vmax);
          else atomicMin(neg + (lk >> 1), vmin);
        }
        pending &= ~__ballot_sync(act, mine);
      }
    }
    if (outside) raise_flag(flags, FLAG_PARTICLE_OUTSIDE);
    return;
  }
  if (!esc) return;
  const int A[3] = {(int)floor(p[0]), (int)floor(p[1]), DIM == 3 ? (int)floor(p[1]) : 0};
  bool outside = false;
#pragma unroll
  for (int k = 0; k < (DIM == 3 ? 2 : 1); ++k)
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int a[3] = {A[0] + i, A[1] + j, A[2] + k};
        const int lx = a[0] - g.px, ly = a[1] - g.py, lz = DIM == 3 ? a[2] - g.pz : 0;
        if ((unsigned)lx >= (unsigned)g.nx || (unsigned)ly >= (unsigned)g.ny || (unsigned)lz >= (unsigned)g.nz) {
          outside = true;
          continue;
        }
        T d2 = (p[0] - (T)a[0]) * (p[0] - (T)a[0]) + (p[1] - (T)a[1]) * (p[1] - (T)a[1]);
        if (DIM == 3) d2 = d2 + (p[2] - (T)a[2]) * (p[2] - (T)a[2]);
        const T phi_p = sign * (sign * p[3] - sqrt(d2));
        const long long q = ((long long)lz * g.ny + ly) * g.nx + lx;
        if (sign > T(0))
          atomicMax(pos + q, ord_bits(phi_p));
        else
          atomicMin(neg + q, ord_bits(phi_p));
      }
  if (outside) raise_flag(flags, FLAG_PARTICLE_OUTSIDE);
}

// ErrorCorrection, merge at the band points (ParticleLS2D.c:103-112,
// ParticleLS3D.c:104-113): phi = phi+ if |phi+| <= |phi-| else phi-.
template <typename T>
__global__ void __launch_bounds__(256) pls_merge_kernel(Geom g, T *__restrict__ phi, const int *__restrict__ band,
                                                        long long nband, const typename OrdOf<T>::type *pos,
                                                        const typename OrdOf<T>::type *neg, int *flags) {
  typedef typename OrdOf<T>::type O;
  const long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (b >= nband) return;
  int x, y, z;
  if (!arrival_local(g, band, b, x, y, z)) {
    raise_flag(flags, FLAG_BAD_BAND);
    return;
  }
  const long long q = ((long long)z * g.ny + y) * g.nx + x;
  const T v = phi[q];
  T pp = v, pn = v;
  if (pos[q] != O(0)) {
    const T c = ord_value(pos[q]);
    pp = c < pp ? pp : c;  // PetscMax(phi_p, phi+)
  }
  if (neg[q] != ~O(0)) {
    const T c = ord_value(neg[q]);
    pn = c < pn ? c : pn;  // PetscMin(phi_p, phi-)
  }
  phi[q] = fabs(pp) <= fabs(pn) ? pp : pn;
}

// ParticleLS_AdjustRadii (ParticleLS.c:158-185).
template <typename T, int DIM, bool VEC>
__global__ void __launch_bounds__(256) pls_adjust_kernel(Geom g, const T *__restrict__ phi, T *__restrict__ parts,
                                                         long long n, const long long *dcount, T r_min, T r_max) {
  const long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (m >= n || (dcount && m >= *dcount)) return;
  T p[4];
  load4<T, VEC>(parts, m, p);
  const T dist = phi_at<T, DIM>(g, phi, p);
  const T sign = psign(p[3]);
  const T sphi = sign * dist;
  if (r_min < sphi && sphi < r_max)
    p[3] = sign * sphi;
  else if (sphi > r_max)
    p[3] = sign * r_max;
  else if (sphi < r_min)
    p[3] = sign * r_min;
  parts[4 * m + 3] = p[3];
}

// ParticleLS_AttractParticleToPhiGoal (ParticleLS.c:108-154), 2D: Bilinear2D
// samples of phi and its central differences; an accepted step copies the
// local Coor X, whose z stays 0.
template <typename T>
__device__ void attract2(const Geom &g, const T *__restrict__ phi, T p[4], T goal, T g_tol, int l_max) {
  T X[3] = {0, 0, 0}, lambda = 1, phi_X = 0;
  T phi_Xp = sample_gf<T, 2>(g, phi, 0, p);
  int l;
  for (l = 0; l < l_max; ++l) {
    T Nx = sample_gf<T, 2>(g, phi, 1, p);
    T Ny = sample_gf<T, 2>(g, phi, 2, p);
    const T mag = sqrt(Nx * Nx + Ny * Ny);
    Nx = Nx / mag;
    Ny = Ny / mag;
    const T sign = psign(goal - phi_Xp);
    X[0] = p[0] + sign * lambda * Nx;
    X[1] = p[1] + sign * lambda * Ny;
    phi_X = sample_gf<T, 2>(g, phi, 0, X);
    if (fabs(phi_X - goal) > fabs(phi_Xp - goal)) {
      lambda = lambda / T(2.);
    } else {
      p[0] = X[0];
      p[1] = X[1];
      p[2] = X[2];
      phi_Xp = phi_X;
    }
    if (fabs(phi_X - goal) < g_tol) break;
  }
  if (l == l_max) {
    phi_X = sample_gf<T, 2>(g, phi, 0, p);
    p[3] = psign(phi_X);
  }
}

// Seeding flags: s_init for a band cell with |phi| < d_init (ParticleLS.c:42-48).
template <typename T>
__global__ void __launch_bounds__(256) pls_seed_count_kernel(Geom g, const T *__restrict__ phi,
                                                             const int *__restrict__ band, int nband, double d_init,
                                                             int s_init, int *__restrict__ cnt, int *flags) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nband) return;
  int x, y, z;
  if (!arrival_local(g, band, b, x, y, z)) {
    cnt[b] = 0;
    raise_flag(flags, FLAG_BAD_BAND);
    return;
  }
  const double dist = fabs((double)phi[((long long)z * g.ny + y) * g.nx + x]);
  cnt[b] = (-d_init < dist && dist < d_init) ? s_init : 0;
}

// Seeding (ParticleLS.c:50-71): thread (b, m) makes particle offs[b] + m.
template <typename T>
__global__ void __launch_bounds__(128) pls_seed_kernel(Geom g, const T *__restrict__ phi, const int *__restrict__ band,
                                                       int nband, const int *__restrict__ cnt,
                                                       const int *__restrict__ offs, dcell_pls_params prm,
                                                       const unsigned long long *rng, T *__restrict__ parts,
                                                       long long cap) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int b = (int)(t / prm.s_init), m = (int)(t % prm.s_init);
  if (b >= nband || !cnt[b]) return;
  const long long k = (long long)offs[b] + m;
  if (k >= cap) return;
  unsigned long long x = r48_skip(*rng, 5ULL * (unsigned long long)k);
  double X0 = r48_next(x), X1 = r48_next(x), X2 = r48_next(x);
  X0 += band[3 * b] - 0.5;
  X1 += band[3 * b + 1] - 0.5;
  X2 += band[3 * b + 2] - 0.5;
  double sign = r48_next(x);
  sign = sign > 0.5 ? 1 : -1;
  double goal = r48_next(x);
  goal = (prm.d_init - prm.r_min) * goal + prm.r_min;
  goal *= sign;
  T p[4] = {(T)X0, (T)X1, (T)X2, (T)sign};
  attract2<T>(g, phi, p, (T)goal, (T)prm.g_tol, prm.l_max);
  store4(parts, k, p);
}

__global__ void pls_seed_finish_kernel(const int *total, unsigned long long *rng, long long *count, long long cap,
                                       int *flags) {
  const long long n = *total;
  *rng = r48_skip(*rng, 5ULL * (unsigned long long)n);
  *count = n;
  if (n > cap) raise_flag(flags, FLAG_CAPACITY);
}

// Reseeding, deletion (ParticleLS.c:228-240): keep flags.
template <typename T>
__global__ void __launch_bounds__(256) pls_keep_kernel(Geom g, const T *__restrict__ phi, const T *__restrict__ parts,
                                                       int n, double d_init, double e_dist, int *__restrict__ keep) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  T p[4];
  load4(parts, i, p);
  const T dist = phi_at<T, 2>(g, phi, p);
  const T sign = psign(p[3]);
  const T thres = sign * dist < T(0) ? (T)e_dist : (T)d_init;
  keep[i] = fabs(dist) > thres ? 0 : 1;
}

// The swap-with-last deletion (ArrayDelete1, Common/Array.c:272-285) run
// front to back leaves the kept particles of [0, L) in place and fills the
// deleted slots of [0, L), in increasing order, with the kept particles of
// [L, n) in decreasing order.  holes: slot of the r-th deleted index < L.
__global__ void __launch_bounds__(256) pls_holes_kernel(const int *__restrict__ keep, const int *__restrict__ excl,
                                                        int n, const int *kept, int *__restrict__ holes) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int L = *kept;
  if (i >= n || i >= L || keep[i]) return;
  holes[i - excl[i]] = i;
}

template <typename T>
__global__ void __launch_bounds__(256) pls_fill_kernel(T *__restrict__ parts, const int *__restrict__ keep,
                                                       const int *__restrict__ excl, int n, const int *kept,
                                                       const int *__restrict__ holes) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int L = *kept;
  if (j >= n || j < L || !keep[j]) return;
  const int r = L - excl[j] - 1;  // kept particles after j
  T p[4];
  load4(parts, j, p);
  store4(parts, holes[r], p);
}

// Reseeding, counts (ParticleLS.c:242-258): non-escaped particles per cell
// floor(X + 1/2), ArrayGetCoor's linear index over phi's box.
template <typename T>
__global__ void __launch_bounds__(256) pls_count_kernel(Geom g, const T *__restrict__ phi, const T *__restrict__ parts,
                                                        const int *kept, int *__restrict__ counts, int *flags) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= *kept) return;
  T p[4];
  load4(parts, i, p);
  const T v = phi_at<T, 2>(g, phi, p);
  if (p[3] * v < T(0)) return;
  const long long cx = (long long)floor(p[0] + T(0.5)), cy = (long long)floor(p[1] + T(0.5)),
                  cz = (long long)floor(p[2] + T(0.5));
  const long long idx = (cx - g.px) + (long long)g.nx * (cy - g.py) + (long long)g.nx * g.ny * (cz - g.pz);
  if (idx < 0 || idx >= (long long)g.nx * g.ny) {
    raise_flag(flags, FLAG_PARTICLE_OUTSIDE);
    return;
  }
  atomicAdd(counts + idx, 1);
}

// Reseeding, deficits (ParticleLS.c:261-267): s_init - count for band cells
// with |phi| <= d_init.
template <typename T>
__global__ void __launch_bounds__(256) pls_deficit_kernel(Geom g, const T *__restrict__ phi,
                                                          const int *__restrict__ band, int nband,
                                                          const int *__restrict__ counts, double d_init, int s_init,
                                                          int *__restrict__ def, int *flags) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nband) return;
  int x, y, z;
  if (!arrival_local(g, band, b, x, y, z)) {
    def[b] = 0;
    raise_flag(flags, FLAG_BAD_BAND);
    return;
  }
  const long long q = (long long)y * g.nx + x;
  const double dist = (double)phi[q];
  def[b] = fabs(dist) > d_init ? 0 : max(0, s_init - counts[q]);
}

// Reseeding, the random stream (ParticleLS.c:268-288), one thread: positions
// and phi goals of the new particles in band order.
template <typename T>
__global__ void pls_walk_kernel(Geom g, const T *__restrict__ phi, const int *__restrict__ band, int nband,
                                const int *__restrict__ def, const int *__restrict__ doff, const int *kept,
                                dcell_pls_params prm, unsigned long long *rng, T *__restrict__ parts, long long cap,
                                int *flags) {
  if (blockIdx.x || threadIdx.x) return;
  unsigned long long x = *rng;
  const long long base = *kept;
  for (int b = 0; b < nband; ++b) {
    const int d = def[b];
    if (!d) continue;
    const int bx = band[3 * b], by = band[3 * b + 1], bz = band[3 * b + 2];
    const double dist = (double)phi[(long long)(by - g.py) * g.nx + (bx - g.px)];
    for (int c = 0; c < d; ++c) {
      double X0 = r48_next(x), X1 = r48_next(x), X2 = r48_next(x);
      X0 += bx - 0.5;
      X1 += by - 0.5;
      X2 += bz - 0.5;
      double goal = 0;
      int tries = 0;
      for (;; ++tries) {
        goal = r48_next(x);
        const double phimax = prm.d_init < dist + 0.71 ? prm.d_init : dist + 0.71;
        const double phimin = -prm.d_init < dist - 0.71 ? dist - 0.71 : -prm.d_init;
        goal = (phimax - phimin) * goal + phimin;
        if (goal < -prm.r_min || prm.r_min < goal) break;
        if (tries >= REJECT_LIMIT) {
          raise_flag(flags, FLAG_WAIT_TIMEOUT);
          break;
        }
      }
      const long long k = base + doff[b] + c;
      if (k < cap) {
        const T p[4] = {(T)X0, (T)X1, (T)X2, (T)goal};
        store4(parts, k, p);
      }
    }
  }
  *rng = x;
}

// Reseeding, attraction of the new particles [L, L + M) to their goals (the
// radius field holds phi_goal, ParticleLS.c:288-289).
template <typename T>
__global__ void __launch_bounds__(128) pls_attract_new_kernel(Geom g, const T *__restrict__ phi, T *__restrict__ parts,
                                                              const int *kept, const int *added, long long cap,
                                                              dcell_pls_params prm) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= *added) return;
  const long long k = *kept + t;
  if (k >= cap) return;
  T p[4];
  load4(parts, k, p);
  attract2<T>(g, phi, p, p[3], (T)prm.g_tol, prm.l_max);
  store4(parts, k, p);
}

__global__ void pls_reseed_finish_kernel(const int *kept, const int *added, long long *count, long long cap,
                                         int *flags) {
  const long long n = (long long)*kept + *added;
  *count = n;
  if (n > cap) raise_flag(flags, FLAG_CAPACITY);
}

static inline unsigned blocks_for(long long n, int threads) {
  const long long b = (n + threads - 1) / threads;
  return (unsigned)(b < 1 ? 1 : b);
}

// 16-byte records: FP32 particles on a 16-byte aligned array
template <typename T>
static bool vec_records(const void *parts) {
  return sizeof(T) == 4 && ((uintptr_t)parts % 16) == 0;
}

template <typename T, int DIM>
static void advect_launch(const Geom &g, const void *vel, void *parts, long long n, double dt, int *flags,
                          cudaStream_t st) {
  const double d = (double)(T)dt;  // the kernels' dt
  const float3 kh = make_float3((float)(0.5 * d / g.hx), (float)(0.5 * d / g.hy), (float)(0.5 * d / g.hz));
  const float3 kf = make_float3((float)(d / g.hx), (float)(d / g.hy), (float)(d / g.hz));
  if (vec_records<T>(parts))
    pls_advect_kernel<T, DIM, true><<<blocks_for(n, 256), 256, 0, st>>>(g, (const T *)vel, (T *)parts, n, (T)dt, kh,
                                                                        kf, flags);
  else
    pls_advect_kernel<T, DIM, false><<<blocks_for(n, 256), 256, 0, st>>>(g, (const T *)vel, (T *)parts, n, (T)dt, kh,
                                                                         kf, flags);
}

template <typename T, int DIM>
static void correct_launch(const Geom &g, void *phi, const int *band, long long nband, const void *parts, long long n,
                           void *scratch, int *flags, cudaStream_t st) {
  typedef typename OrdOf<T>::type O;
  const long long npts = (long long)g.nx * g.ny * g.nz;
  O *pos = (O *)scratch, *neg = pos + npts;
  cudaMemsetAsync(pos, 0x00, npts * sizeof(O), st);
  cudaMemsetAsync(neg, 0xFF, npts * sizeof(O), st);
  if (n > 0 && vec_records<T>(parts))
    pls_escape_kernel<T, DIM, true><<<blocks_for(n, 256), 256, 0, st>>>(g, (const T *)phi, (const T *)parts, n, pos,
                                                                        neg, flags);
  else if (n > 0)
    pls_escape_kernel<T, DIM, false><<<blocks_for(n, 256), 256, 0, st>>>(g, (const T *)phi, (const T *)parts, n, pos,
                                                                         neg, flags);
  if (nband > 0) pls_merge_kernel<T><<<blocks_for(nband, 256), 256, 0, st>>>(g, (T *)phi, band, nband, pos, neg, flags);
}

template <typename T, int DIM>
static void adjust_launch(const Geom &g, const void *phi, void *parts, long long n, const long long *dcount,
                          const dcell_pls_params &prm, cudaStream_t st) {
  if (vec_records<T>(parts))
    pls_adjust_kernel<T, DIM, true><<<blocks_for(n, 256), 256, 0, st>>>(g, (const T *)phi, (T *)parts, n, dcount,
                                                                        (T)prm.r_min, (T)prm.r_max);
  else
    pls_adjust_kernel<T, DIM, false><<<blocks_for(n, 256), 256, 0, st>>>(g, (const T *)phi, (T *)parts, n, dcount,
                                                                         (T)prm.r_min, (T)prm.r_max);
}

// scratch of seeding / reseeding, ints: keep, excl, holes (n each), counts
// (npts), cnt/def, offs (nband each), scan partials, 4 small counters
struct PlsScratch {
  int *keep, *excl, *holes, *counts, *cnt, *offs, *partial, *small;
};
static PlsScratch pls_scratch(void *base, long long npts, long long nband, long long n) {
  PlsScratch s;
  int *p = (int *)base;
  s.small = p;
  p += 8;
  s.keep = p;
  p += n;
  s.excl = p;
  p += n;
  s.holes = p;
  p += n;
  s.counts = p;
  p += npts;
  s.cnt = p;
  p += nband;
  s.offs = p;
  p += nband;
  s.partial = p;
  return s;
}

template <typename T>
static int seed_launch(const Geom &g, const void *phi, const int *band, long long nband, const dcell_pls_params &prm,
                       unsigned long long *rng, void *parts, long long cap, long long *count, void *scratch,
                       int *flags, cudaStream_t st) {
  const long long npts = (long long)g.nx * g.ny;
  PlsScratch s = pls_scratch(scratch, npts, nband, 0);
  const int nb = (int)nband;
  if (nb > 0)
    pls_seed_count_kernel<T><<<blocks_for(nb, 256), 256, 0, st>>>(g, (const T *)phi, band, nb, prm.d_init, prm.s_init,
                                                                  s.cnt, flags);
  int rc = launch_scan_exclusive(s.cnt, nb, s.offs, s.partial, s.small, 0x7fffffff, nullptr, st);
  if (rc) return rc;
  if (nb > 0)
    pls_seed_kernel<T><<<blocks_for((long long)nb * prm.s_init, 128), 128, 0, st>>>(
        g, (const T *)phi, band, nb, s.cnt, s.offs, prm, rng, (T *)parts, cap);
  pls_seed_finish_kernel<<<1, 1, 0, st>>>(s.small, rng, count, cap, flags);
  // AdjustRadii over the seeded particles (ParticleLS.c:75), at most the capacity
  const long long nmax = (long long)nb * prm.s_init < cap ? (long long)nb * prm.s_init : cap;
  if (nmax > 0) adjust_launch<T, 2>(g, phi, parts, nmax, count, prm, st);
  return DCELL_OK;
}

template <typename T>
static int reseed_launch(const Geom &g, const void *phi, const int *band, long long nband,
                         const dcell_pls_params &prm, unsigned long long *rng, void *parts, long long n, long long cap,
                         long long *count, void *scratch, int *flags, cudaStream_t st) {
  const long long npts = (long long)g.nx * g.ny;
  PlsScratch s = pls_scratch(scratch, npts, nband, n);
  const int nn = (int)n, nb = (int)nband;
  int *kept = s.small, *added = s.small + 1;
  int rc;
  if (nn > 0) {
    pls_keep_kernel<T><<<blocks_for(nn, 256), 256, 0, st>>>(g, (const T *)phi, (const T *)parts, nn, prm.d_init,
                                                            prm.e_dist, s.keep);
  }
  if ((rc = launch_scan_exclusive(s.keep, nn, s.excl, s.partial, kept, 0x7fffffff, nullptr, st))) return rc;
  if (nn > 0) {
    pls_holes_kernel<<<blocks_for(nn, 256), 256, 0, st>>>(s.keep, s.excl, nn, kept, s.holes);
    pls_fill_kernel<T><<<blocks_for(nn, 256), 256, 0, st>>>((T *)parts, s.keep, s.excl, nn, kept, s.holes);
  }
  cudaMemsetAsync(s.counts, 0, npts * sizeof(int), st);
  if (nn > 0)
    pls_count_kernel<T><<<blocks_for(nn, 256), 256, 0, st>>>(g, (const T *)phi, (const T *)parts, kept, s.counts,
                                                             flags);
  if (nb > 0)
    pls_deficit_kernel<T><<<blocks_for(nb, 256), 256, 0, st>>>(g, (const T *)phi, band, nb, s.counts, prm.d_init,
                                                               prm.s_init, s.cnt, flags);
  if ((rc = launch_scan_exclusive(s.cnt, nb, s.offs, s.partial, added, 0x7fffffff, nullptr, st))) return rc;
  pls_walk_kernel<T><<<1, 1, 0, st>>>(g, (const T *)phi, band, nb, s.cnt, s.offs, kept, prm, rng, (T *)parts, cap,
                                      flags);
  const long long mmax = (long long)nb * prm.s_init;
  if (mmax > 0)
    pls_attract_new_kernel<T><<<blocks_for(mmax, 128), 128, 0, st>>>(g, (const T *)phi, (T *)parts, kept, added, cap,
                                                                      prm);
  pls_reseed_finish_kernel<<<1, 1, 0, st>>>(kept, added, count, cap, flags);
  return DCELL_OK;
}

}  // namespace dcell

using namespace dcell;

static inline int last_status() { return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA; }

int launch_pls_advect(const Geom &g, int dtype, const void *vel, void *parts, long long n, double dt, int *flags,
                      cudaStream_t st) {
  if (n <= 0) return DCELL_OK;
  const bool d3 = g.nz > 1;
  if (dtype == DCELL_F64)
    d3 ? advect_launch<double, 3>(g, vel, parts, n, dt, flags, st) : advect_launch<double, 2>(g, vel, parts, n, dt, flags, st);
  else
    d3 ? advect_launch<float, 3>(g, vel, parts, n, dt, flags, st) : advect_launch<float, 2>(g, vel, parts, n, dt, flags, st);
  return last_status();
}

size_t pls_correct_scratch_bytes(long long npts, int dtype) {
  return (size_t)npts * 2 * (dtype == DCELL_F64 ? sizeof(unsigned long long) : sizeof(unsigned int)) + 256;
}

int launch_pls_correct(const Geom &g, int dtype, void *phi, const int *band, long long nband, const void *parts,
                       long long n, void *scratch, int *flags, cudaStream_t st) {
  const bool d3 = g.nz > 1;
  if (dtype == DCELL_F64)
    d3 ? correct_launch<double, 3>(g, phi, band, nband, parts, n, scratch, flags, st)
       : correct_launch<double, 2>(g, phi, band, nband, parts, n, scratch, flags, st);
  else
    d3 ? correct_launch<float, 3>(g, phi, band, nband, parts, n, scratch, flags, st)
       : correct_launch<float, 2>(g, phi, band, nband, parts, n, scratch, flags, st);
  return last_status();
}

int launch_pls_adjust(const Geom &g, int dtype, const void *phi, void *parts, long long n, const dcell_pls_params &prm,
                      int *flags, cudaStream_t st) {
  (void)flags;
  if (n <= 0) return DCELL_OK;
  const bool d3 = g.nz > 1;
  if (dtype == DCELL_F64)
    d3 ? adjust_launch<double, 3>(g, phi, parts, n, nullptr, prm, st)
       : adjust_launch<double, 2>(g, phi, parts, n, nullptr, prm, st);
  else
    d3 ? adjust_launch<float, 3>(g, phi, parts, n, nullptr, prm, st)
       : adjust_launch<float, 2>(g, phi, parts, n, nullptr, prm, st);
  return last_status();
}

size_t pls_scratch_bytes(long long npts, long long nband, long long n) {
  const long long ints = 8 + 3 * n + npts + 2 * nband + (long long)scan_partial_ints(n > nband ? n : nband);
  return (size_t)ints * sizeof(int) + 256;
}

int launch_pls_seed(const Geom &g, int dtype, const void *phi, const int *band, long long nband,
                    const dcell_pls_params &prm, unsigned long long *rng, void *parts, long long cap, long long *count,
                    void *scratch, int *flags, cudaStream_t st) {
  const int rc = dtype == DCELL_F64 ? seed_launch<double>(g, phi, band, nband, prm, rng, parts, cap, count, scratch, flags, st)
                                    : seed_launch<float>(g, phi, band, nband, prm, rng, parts, cap, count, scratch, flags, st);
  return rc ? rc : last_status();
}

int launch_pls_reseed(const Geom &g, int dtype, const void *phi, const int *band, long long nband,
                      const dcell_pls_params &prm, unsigned long long *rng, void *parts, long long n, long long cap,
                      long long *count, void *scratch, int *flags, cudaStream_t st) {
  const int rc = dtype == DCELL_F64
                     ? reseed_launch<double>(g, phi, band, nband, prm, rng, parts, n, cap, count, scratch, flags, st)
                     : reseed_launch<float>(g, phi, band, nband, prm, rng, parts, n, cap, count, scratch, flags, st);
  return rc ? rc : last_status();
}
