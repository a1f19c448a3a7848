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
#include "dcell_common.cuh"
#include "dcell_kernels.h"
#include "sl_device.cuh"
#include "catmull_rom_ops.inc"

namespace dcell {

template <typename T, int DIM>
__device__ __forceinline__ T cubic_plain(const Geom &g, const T *__restrict__ phi0, const int c[3], const T f[3]) {
  if (DIM == 3) {
    T s[64];
    gather_stencil<T, 3>(g, phi0, c, s);
    // a = M s with M = C (x) C (x) C: the 1331 non-zeros as straight-line code
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
  T wx[4], wy[4];
  cr_weights<T>(f[0], wx);
  cr_weights<T>(f[1], wy);
  T s[DIM == 3 ? 64 : 16];
  gather_stencil<T, DIM>(g, phi0, c, s);
  if (DIM == 3) {
    T wz[4];
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
  } else {
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

int launch_sl_cubic(const Geom &g, int dtype, const void *phi0, const void *vel, double dt, const int *band,
                    long long npts, int interp, int backtrace, void *phi, int *flags, cudaStream_t st) {
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
