// Cubic semi-Lagrangian kernels on CUDA cores (FP32 and FP64).
//
// Reconstruction at the departure point is the Catmull-Rom tricubic
// (bicubic in 2D) of the reference's TricubicInverse.h /
// OrthogonalProjection.c:48-63, which is the tensor product C (x) C (x) C of
// the 1-D Keys a=-1/2 matrix.  Two forms of the same interpolant:
//
//   PLAIN      per point: gather the 4^3 stencil, form the 64 coefficients
//              with the 1331 non-zeros of the 64x64 operator, evaluate the
//              64-term polynomial -- the reference's own arithmetic shape and
//              the "plain FP32 CUDA SL step";
//   SEPARABLE  per point: 4-tap weights per axis, 64 + 16 + 4 multiply-adds.
//
// Band structure and backtrace follow LevelSetAdvectSL_2D/_3D
// (LevelSetMethod/AdvectSL.c:23-89).  The FP64 instantiation of PLAIN is
// the GPU FP64 oracle used to measure errors on grids too large for the CPU.
//
// Two data paths: global gathers (one thread per point; bands, FP64, 2-D)
// and, for dense FP32 3-D grids, the bricks of the tensor-core stepper
// (brick_stage.cuh: TMA-staged boxes, edge replication, the same departure
// code) with the two forms evaluated on CUDA cores -- the equal-data-movement
// comparison for the tensor-core contraction.
#include "brick_stage.cuh"
#include "dcell_common.cuh"
#include "dcell_kernels.h"
#include "sl_device.cuh"
#include "catmull_rom_ops.inc"

namespace dcell {

// Coefficients with the 1331 non-zeros of M = C (x) C (x) C, then Horner per
// axis: the polynomial of stencil s (s[x + 4y + 16z]) at fraction f.
template <typename T>
__device__ __forceinline__ T plain_eval3(const T *s, const T f[3]) {
  T a[64];
  DCELL_CR_COEFS3(s, a);
  // p = sum a[i + 4j + 16k] x^i y^j z^k, Horner per axis
  T pz = T(0);
#pragma unroll
  for (int k = 3; k >= 0; --k) {
    T py = T(0);
#pragma unroll
    for (int j = 3; j >= 0; --j) {
      const T *r = a + 4 * j + 16 * k;
      const T px = ((r[3] * f[0] + r[2]) * f[0] + r[1]) * f[0] + r[0];
      py = py * f[1] + px;
    }
    pz = pz * f[2] + py;
  }
  return pz;
}

// 4-tap Catmull-Rom weights per axis applied to stencil s: 64 + 16 + 4
// multiply-adds.
template <typename T>
__device__ __forceinline__ T separable_eval3(const T *s, const T f[3]) {
  T wx[4], wy[4], wz[4];
  cr_weights<T>(f[0], wx);
  cr_weights<T>(f[1], wy);
  cr_weights<T>(f[2], wz);
  T acc = T(0);
#pragma unroll
  for (int z = 0; z < 4; ++z) {
    T accy = T(0);
#pragma unroll
    for (int y = 0; y < 4; ++y) {
      T accx = T(0);
#pragma unroll
      for (int x = 0; x < 4; ++x) accx += wx[x] * s[x + 4 * y + 16 * z];
      accy += wy[y] * accx;
    }
    acc += wz[z] * accy;
  }
  return acc;
}

template <typename T, int DIM>
__device__ __forceinline__ T cubic_plain(const Geom &g, const T *__restrict__ phi0, const int c[3], const T f[3]) {
  if (DIM == 3) {
    T s[64];
    gather_stencil<T, 3>(g, phi0, c, s);
    return plain_eval3<T>(s, f);
  } else {
    T s[16];
    gather_stencil<T, 2>(g, phi0, c, s);
    T a[16];
    DCELL_CR_COEFS2(s, a);
    T py = T(0);
#pragma unroll
    for (int j = 3; j >= 0; --j) {
      const T *r = a + 4 * j;
      const T px = ((r[3] * f[0] + r[2]) * f[0] + r[1]) * f[0] + r[0];
      py = py * f[1] + px;
    }
    return py;
  }
}

template <typename T, int DIM>
__device__ __forceinline__ T cubic_separable(const Geom &g, const T *__restrict__ phi0, const int c[3], const T f[3]) {
  T s[DIM == 3 ? 64 : 16];
  gather_stencil<T, DIM>(g, phi0, c, s);
  if (DIM == 3) return separable_eval3<T>(s, f);
  T wx[4], wy[4];
  cr_weights<T>(f[0], wx);
  cr_weights<T>(f[1], wy);
  T acc = T(0);
#pragma unroll
  for (int y = 0; y < 4; ++y) {
    T accx = T(0);
#pragma unroll
    for (int x = 0; x < 4; ++x) accx += wx[x] * s[x + 4 * y];
    acc += wy[y] * accx;
  }
  return acc;
}

template <typename T, int DIM, bool SEPARABLE>
__global__ void __launch_bounds__(256) sl_cubic_kernel(Geom g, const T *__restrict__ phi0, const T *__restrict__ vel,
                                                       T dt, const int *__restrict__ band, long long npts,
                                                       int backtrace, T *__restrict__ phi, int *flags) {
  const T dth[3] = {dt / (T)g.hx, dt / (T)g.hy, dt / (T)g.hz};
  bool clamped = false, bad = false;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < npts;
       q += (long long)gridDim.x * blockDim.x) {
    int x, y, z, c[3];
    T f[3];
    if (!arrival_local(g, band, q, x, y, z)) {
      bad = true;
      continue;
    }
    clamped |= departure_cell<T, DIM>(g, vel, dth, backtrace, x, y, z, c, f);
    phi[(z * g.ny + y) * g.nx + x] =
        SEPARABLE ? cubic_separable<T, DIM>(g, phi0, c, f) : cubic_plain<T, DIM>(g, phi0, c, f);
  }
  if (clamped && band) raise_flag(flags, FLAG_DEPARTURE_CLAMPED);  // dense grids: the edge is the domain boundary
  if (bad) raise_flag(flags, FLAG_BAD_BAND);
}

// Brick-staged CUDA-core step (dense FP32 3-D grids, nx % 4 == 0): the
// tensor-core stepper's 32 x 4 x 8 bricks and TMA boxes (phi staged as FP32
// here), double-buffered, edge-replicated, departures by brick_depart; the
// coefficient solve and evaluation on CUDA cores (PLAIN: the 1331 non-zeros
// and Horner; SEPARABLE: 4-tap weights).  256 threads: warp w owns tile row
// w & 3 and brick planes 4 (w >> 2) .. 4 (w >> 2) + 3, two points per step
// (the same (x, y) in consecutive planes), two steps per brick.  A warp whose
// stencils leave the boxes takes the global path for that step.  Thread 0
// issues the loads; one CTA barrier per brick frees its buffer.  Bounded
// waits; on a timeout the CTA raises FLAG_WAIT_TIMEOUT, waits (bounded) for
// its loads in flight and leaves.
constexpr int kCcThreads = 256;

template <int BT, bool SEP>
__global__ void __launch_bounds__(kCcThreads, 2)
    sl_cc_brick_kernel(const __grid_constant__ CUtensorMap tm_phi, const __grid_constant__ CUtensorMap tm_vel, Geom g,
                       BrickGrid bg, const float *__restrict__ phi0, const float *__restrict__ vel, float dt,
                       float *__restrict__ phi, int *flags) {
  using S = BrickBox<2>;
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t *const buf0 = smem, *const buf1 = smem + S::BufBytes;
  uint64_t *const tbar = reinterpret_cast<uint64_t *>(smem + 2 * S::BufBytes);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    mbar_init(&tbar[0], 1);
    mbar_init(&tbar[1], 1);
  }
  __syncthreads();
  const int nbricks = bg.nbx * bg.nby * bg.nbz;
  const int nmine = (int)blockIdx.x < nbricks ? (nbricks - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  int issued[2] = {nmine > 0 ? 1 : 0, nmine > 1 ? 1 : 0};  // loads per buffer (thread 0 issues them)
  if (tid == 0) {
    if (nmine > 0) issue_brick<S>(bg, blockIdx.x, buf0, &tm_phi, &tm_vel, &tbar[0]);
    if (nmine > 1) issue_brick<S>(bg, blockIdx.x + gridDim.x, buf1, &tm_phi, &tm_vel, &tbar[1]);
  }
  const float dth[3] = {dt / (float)g.hx, dt / (float)g.hy, dt / (float)g.hz};
  const float hdth[3] = {-0.5f * dth[0], -0.5f * dth[1], -0.5f * dth[2]};
  const int nn[3] = {g.nx, g.ny, g.nz};
  const int ly = warp & 3, zg = warp >> 2;
  int consumed[2] = {0, 0};
  bool err = false;
  for (int k = 0; k < nmine; ++k) {
    const int bs = k & 1;
    uint8_t *const cbuf = bs ? buf1 : buf0;
    const bool ok = mbar_wait_sleep(&tbar[bs], (uint32_t)(k >> 1) & 1u);
    if (__syncthreads_or(!ok)) {
      err = true;
      break;
    }
    ++consumed[bs];
    int x0, y0, z0;
    brick_origin<S>(bg, (int)blockIdx.x + k * (int)gridDim.x, x0, y0, z0);
    if (x0 < 4 || x0 + S::PX - 4 > g.nx || y0 < 2 || y0 + S::PY - 2 > g.ny || z0 < 2 || z0 + S::PZ - 2 > g.nz) {
      const int op[3] = {x0 - 4, y0 - 2, z0 - 2}, ov[3] = {x0 - 4, y0 - 1, z0 - 1};
      for (int axis = 0; axis < 3; ++axis) {
        replicate_pass<S::PX, S::PY, S::PZ, 1>(reinterpret_cast<uint32_t *>(cbuf), axis, op, nn, kCcThreads);
        replicate_pass<S::VX, S::VY, S::VZ, 3>(reinterpret_cast<uint32_t *>(cbuf + S::PhiBytes), axis, ov, nn,
                                               kCcThreads);
        __syncthreads();
      }
    }
    const float *pbox = reinterpret_cast<const float *>(cbuf);
    const float *vbox = reinterpret_cast<const float *>(cbuf + S::PhiBytes);
    const int x = min(x0 + lane, g.nx - 1), y = min(y0 + ly, g.ny - 1);
    const bool xy_valid = x0 + lane < g.nx && y0 + ly < g.ny;
#pragma unroll 1
    for (int st = 0; st < 2; ++st) {
      const int zl = 4 * zg + 2 * st;  // brick-local plane of point 0
      float f[2][3];
      int soff[2];
      const bool in = brick_depart<BT, S, 2>(vbox, x - x0 + 4, y - y0 + 1, zl + 1, x - x0 + 4, y - y0 + 2, zl + 2,
                                             dth, hdth, f, soff);
      float v[2];
      if (__all_sync(0xffffffffu, in)) {
#pragma unroll
        for (int p = 0; p < 2; ++p) {
          float sv[64];
          const float *q = pbox + soff[p];
#pragma unroll
          for (int e = 0; e < 64; ++e) sv[e] = q[((e >> 4) * S::PY + ((e >> 2) & 3)) * S::PX + (e & 3)];
          v[p] = SEP ? separable_eval3<float>(sv, f[p]) : plain_eval3<float>(sv, f[p]);
        }
      } else {
#pragma unroll
        for (int p = 0; p < 2; ++p) {
          int c[3];
          float fg[3];
          departure_cell<float, 3>(g, vel, dth, BT, x, y, min(z0 + zl + p, g.nz - 1), c, fg);
          v[p] = SEP ? cubic_separable<float, 3>(g, phi0, c, fg) : cubic_plain<float, 3>(g, phi0, c, fg);
        }
      }
#pragma unroll
      for (int p = 0; p < 2; ++p) {
        const int z = z0 + zl + p;
        if (xy_valid && z < g.nz) phi[(z * g.ny + y) * g.nx + x] = v[p];
      }
    }
    __syncthreads();  // the buffer read for the last time
    if (k + 2 < nmine) {
      if (tid == 0) issue_brick<S>(bg, (int)blockIdx.x + (k + 2) * (int)gridDim.x, cbuf, &tm_phi, &tm_vel, &tbar[bs]);
      ++issued[bs];
    }
  }
  if (err && tid == 0) {
    // the load still in flight per buffer, if any
    for (int b = 0; b < 2; ++b)
      if (issued[b] > consumed[b]) mbar_wait(&tbar[b], (uint32_t)(issued[b] - 1) & 1u);
    raise_flag(flags, FLAG_WAIT_TIMEOUT);
  }
}

// Trilinear sample on the production gather (batched linear mode).
template <typename T>
__device__ __forceinline__ T trilinear_fast(const Geom &g, const T *__restrict__ f, const int c[3], const T fr[3]) {
  T s[64];  // s[21] holds cell c itself (stencil origin c - 1)
  gather_stencil<T, 3>(g, f, c, s);
  const T x0 = 1 - fr[0], y0 = 1 - fr[1], z0 = 1 - fr[2];
  const T a = (x0 * s[21] + fr[0] * s[22]) * y0 + (x0 * s[25] + fr[0] * s[26]) * fr[1];
  const T b = (x0 * s[37] + fr[0] * s[38]) * y0 + (x0 * s[41] + fr[0] * s[42]) * fr[1];
  return a * z0 + b * fr[2];
}

// Batched cells on CUDA cores: one thread per point of a tile, a persistent
// grid walking the packed tile queue (see dcell_batch_sl_step).
template <int MODE>
__global__ void __launch_bounds__(1024) batch_cubic_kernel(const dcell_cell *__restrict__ cells,
                                                           const dcell_tile *__restrict__ tiles, int ntiles, int tx,
                                                           int ty, const float *__restrict__ phi0,
                                                           const float *__restrict__ vel, int backtrace,
                                                           float *__restrict__ phi) {
  const int lx = threadIdx.x % tx, ly = (threadIdx.x / tx) % ty, lz = threadIdx.x / (tx * ty);
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const dcell_tile T = tiles[t];
    const dcell_cell C = cells[T.cell];
    Geom g;
    g.nx = C.n[0]; g.ny = C.n[1]; g.nz = C.n[2];
    g.px = g.py = g.pz = 0;
    g.hx = C.h[0]; g.hy = C.h[1]; g.hz = C.h[2];
    const int x = T.x0 + lx, y = T.y0 + ly, z = T.z0 + lz;
    if (x >= g.nx || y >= g.ny || z >= g.nz) continue;
    const float dtf = (float)C.dt;  // same rounding as the single-grid kernels
    const float dth[3] = {dtf / (float)C.h[0], dtf / (float)C.h[1], dtf / (float)C.h[2]};
    const float *p0 = phi0 + C.offset;
    int c[3];
    float f[3];
    departure_cell<float, 3>(g, vel + 3 * C.offset, dth, backtrace, x, y, z, c, f);
    float out;
    if (MODE == DCELL_CUBIC_SEPARABLE) out = cubic_separable<float, 3>(g, p0, c, f);
    else if (MODE == DCELL_CUBIC_PLAIN) out = cubic_plain<float, 3>(g, p0, c, f);
    else out = trilinear_fast<float>(g, p0, c, f);
    phi[C.offset + (z * g.ny + y) * g.nx + x] = out;
  }
}

// FP64 <-> FP32 conversion and band gathers for the host-buffer entry points.
template <typename S, typename D>
__global__ void convert_kernel(const S *__restrict__ src, D *__restrict__ dst, long long n) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    dst[q] = (D)src[q];
}

template <typename T>
__global__ void gather_band_kernel(Geom g, const T *__restrict__ phi, const int *__restrict__ band, int nband,
                                   T *__restrict__ out) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < nband) out[b] = phi[gidx(g, band[3 * b], band[3 * b + 1], g.nz == 1 ? 0 : band[3 * b + 2])];
}

}  // namespace dcell

using namespace dcell;

static inline int blocks_for(long long n, int threads) {
  long long b = (n + threads - 1) / threads;
  if (b > 148LL * 32) b = 148LL * 32;
  return (int)(b < 1 ? 1 : b);
}

template <typename T>
static void cubic_dispatch(const Geom &g, const T *phi0, const T *vel, T dt, const int *band, long long npts,
                           int interp, int backtrace, T *phi, int *flags, cudaStream_t st) {
  const int threads = 256, blocks = blocks_for(npts, threads);
  const bool sep = interp == DCELL_CUBIC_SEPARABLE;
  if (g.nz == 1) {
    if (sep) sl_cubic_kernel<T, 2, true><<<blocks, threads, 0, st>>>(g, phi0, vel, dt, band, npts, backtrace, phi, flags);
    else sl_cubic_kernel<T, 2, false><<<blocks, threads, 0, st>>>(g, phi0, vel, dt, band, npts, backtrace, phi, flags);
  } else {
    if (sep) sl_cubic_kernel<T, 3, true><<<blocks, threads, 0, st>>>(g, phi0, vel, dt, band, npts, backtrace, phi, flags);
    else sl_cubic_kernel<T, 3, false><<<blocks, threads, 0, st>>>(g, phi0, vel, dt, band, npts, backtrace, phi, flags);
  }
}

// Brick-staged CUDA-core step; false when the grid does not admit it or no
// tensor maps could be made (the caller then runs the gather form).
static bool launch_cc_brick(const Geom &g, const float *phi0, const float *vel, double dt, int interp, int backtrace,
                            float *phi, int *flags, cudaStream_t st) {
  using S = BrickBox<2>;
  constexpr int smem = 2 * S::BufBytes + 16;
  if (!tc_brick_applicable(g, phi0, vel)) return false;
  static bool configured = false;
  if (!configured) {
    if (cudaFuncSetAttribute(sl_cc_brick_kernel<DCELL_EULER, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             smem) != cudaSuccess ||
        cudaFuncSetAttribute(sl_cc_brick_kernel<DCELL_EULER, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             smem) != cudaSuccess ||
        cudaFuncSetAttribute(sl_cc_brick_kernel<DCELL_MIDPOINT, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             smem) != cudaSuccess ||
        cudaFuncSetAttribute(sl_cc_brick_kernel<DCELL_MIDPOINT, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             smem) != cudaSuccess)
      return false;
    configured = true;
  }
  CUtensorMap tm_phi, tm_vel;
  if (!make_tensor_map_3d(&tm_phi, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, phi0, (uint64_t)g.nx, (uint64_t)g.ny,
                          (uint64_t)g.nz, S::PX, S::PY, S::PZ, 4) ||
      !make_tensor_map_3d(&tm_vel, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, vel, 3ull * g.nx, (uint64_t)g.ny, (uint64_t)g.nz,
                          3 * S::VX, S::VY, S::VZ, 4))
    return false;
  BrickGrid bg;
  bg.nbx = (g.nx + S::BX - 1) / S::BX;
  bg.nby = (g.ny + S::BY - 1) / S::BY;
  bg.nbz = (g.nz + S::BZ - 1) / S::BZ;
  bg.bz0 = 0;
  const long long nbricks = (long long)bg.nbx * bg.nby * bg.nbz;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = (int)(nbricks < 2LL * sms ? nbricks : 2LL * sms);
  const bool mid = backtrace == DCELL_MIDPOINT, sep = interp == DCELL_CUBIC_SEPARABLE;
  auto kern = mid ? (sep ? sl_cc_brick_kernel<DCELL_MIDPOINT, true> : sl_cc_brick_kernel<DCELL_MIDPOINT, false>)
                  : (sep ? sl_cc_brick_kernel<DCELL_EULER, true> : sl_cc_brick_kernel<DCELL_EULER, false>);
  kern<<<grid, kCcThreads, smem, st>>>(tm_phi, tm_vel, g, bg, phi0, vel, (float)dt, phi, flags);
  return true;
}

int launch_sl_cubic(const Geom &g, int dtype, const void *phi0, const void *vel, double dt, const int *band,
                    long long npts, int interp, int backtrace, void *phi, int *flags, cudaStream_t st, bool gather) {
  if (dtype == DCELL_F32 && !band && g.nz > 1 && !gather &&
      launch_cc_brick(g, (const float *)phi0, (const float *)vel, dt, interp, backtrace, (float *)phi, flags, st))
    return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
  if (dtype == DCELL_F64)
    cubic_dispatch<double>(g, (const double *)phi0, (const double *)vel, dt, band, npts, interp, backtrace,
                           (double *)phi, flags, st);
  else
    cubic_dispatch<float>(g, (const float *)phi0, (const float *)vel, (float)dt, band, npts, interp, backtrace,
                          (float *)phi, flags, st);
  return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
}

int launch_convert(const void *src, int src_dtype, void *dst, int dst_dtype, long long n, cudaStream_t st) {
  const int threads = 256, blocks = blocks_for(n, threads);
  if (src_dtype == DCELL_F64 && dst_dtype == DCELL_F32)
    convert_kernel<double, float><<<blocks, threads, 0, st>>>((const double *)src, (float *)dst, n);
  else if (src_dtype == DCELL_F32 && dst_dtype == DCELL_F64)
    convert_kernel<float, double><<<blocks, threads, 0, st>>>((const float *)src, (double *)dst, n);
  else
    return DCELL_ERR_ARG;
  return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
}

int launch_gather_band(const Geom &g, int dtype, const void *phi, const int *band, int nband, void *out,
                       cudaStream_t st) {
  if (nband <= 0) return DCELL_OK;
  if (dtype == DCELL_F64)
    gather_band_kernel<double><<<(nband + 255) / 256, 256, 0, st>>>(g, (const double *)phi, band, nband, (double *)out);
  else
    gather_band_kernel<float><<<(nband + 255) / 256, 256, 0, st>>>(g, (const float *)phi, band, nband, (float *)out);
  return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
}

int launch_batch_cuda_core(const dcell_cell *cells, const dcell_tile *tiles, int ntiles, int tx, int ty, int tz,
                           int ctas_per_sm, const float *phi0, const float *vel, int interp, int backtrace, float *phi,
                           int *flags, cudaStream_t st) {
  (void)flags;
  if (ntiles <= 0) return DCELL_OK;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int threads = tx * ty * tz;
  const int per = ctas_per_sm < 1 ? 1 : (ctas_per_sm > 8 ? 8 : ctas_per_sm);
  const int grid = per * sms < ntiles ? per * sms : ntiles;
  if (interp == DCELL_CUBIC_SEPARABLE)
    batch_cubic_kernel<DCELL_CUBIC_SEPARABLE><<<grid, threads, 0, st>>>(cells, tiles, ntiles, tx, ty, phi0, vel,
                                                                       backtrace, phi);
  else if (interp == DCELL_CUBIC_PLAIN)
    batch_cubic_kernel<DCELL_CUBIC_PLAIN><<<grid, threads, 0, st>>>(cells, tiles, ntiles, tx, ty, phi0, vel,
                                                                   backtrace, phi);
  else
    batch_cubic_kernel<DCELL_LINEAR><<<grid, threads, 0, st>>>(cells, tiles, ntiles, tx, ty, phi0, vel, backtrace,
                                                              phi);
  return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
}
