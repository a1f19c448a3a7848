// Velocity acquisition: the velocity grid of a level set's box from the
// fluid's global MAC field -- LevelSetGetVelocity (LevelSetMethod/Advect.c:
// 145-192).  The reference resizes the velocity grid to the phi box (which
// zeroes it, Common/Grid.c:146) and NGA_Gets the part of the box inside the
// Global Array [z][y][x][c] (components U_FACE.. of the cell, CELL_CENTER
// first).  Here the global field is a device array and the copy is a kernel:
// one warp per row of the box, x fastest so the global reads and the box
// writes coalesce; zero outside the field.  The batched form
// fills many boxes (cells) in one launch: blockIdx.y picks the box.
#include <cuda_runtime.h>

#include "dcell_common.cuh"
#include "dcell_kernels.h"

namespace dcell {

struct VBox {
  long long offset;  // first point of the box in the packed output
  int px, py, pz;    // global index of the box's first point
  int nx, ny, nz;    // extents
};

__device__ __forceinline__ unsigned word32(const uint4 &q, int i) {
  return i == 0 ? q.x : i == 1 ? q.y : i == 2 ? q.z : q.w;
}

// Element j of a point record held as 16-byte words (j is a constant after unrolling).
template <typename T>
__device__ __forceinline__ T rec_elem(const uint4 *q, int j);
template <>
__device__ __forceinline__ float rec_elem<float>(const uint4 *q, int j) {
  return __uint_as_float(word32(q[0], j));
}
template <>
__device__ __forceinline__ double rec_elem<double>(const uint4 *q, int j) {
  const uint4 w = j < 2 ? q[0] : q[1];  // two words per FP64 record
  return __hiloint2double((int)word32(w, 2 * (j & 1) + 1), (int)word32(w, 2 * (j & 1)));
}

// One warp per (y, z) row of the box: the output row is nx * DIM contiguous
// values, the input row is the global row from x = px with gdof values per
// point.  A row is done in passes of 32 * U points (lane + 32 k: a warp
// instruction reads 32 neighbouring records).  NV > 0: a point's record is NV
// aligned 16-byte words (gdof * sizeof(T) = 16 or 32: FP32 or FP64 with four
// components) read with vector loads, the components picked in registers;
// NV = 0: one load per component.  The picked values go through the warp's
// slice of shared memory so that the stores are contiguous (consecutive
// lanes, consecutive values) instead of DIM-strided.  The passes are
// software-pipelined: the loads of the next pass are issued before the stores
// of the current one, so two passes' loads are in flight.  Rows advance by a
// fixed (dy, dz) step: no division per row.
constexpr int VEL_U = 2;

struct VPass {
  long long r;  // row index in the box (y + ny * z)
  int y, z, x0;
};

template <typename T, int DIM, int NV>
__device__ __forceinline__ void load_pass(const VBox &b, const VPass &p, const T *__restrict__ global, int gx, int gy,
                                          int gz, int gdof, int first, int xa, int xb, int lane,
                                          T (&v)[VEL_U][DIM]) {
  const int Y = b.py + p.y, Z = DIM == 3 ? b.pz + p.z : 0;
  const bool rowin = Y >= 0 && Y < gy && Z >= 0 && Z < gz;
  const int ra = rowin ? xa : 0, rb = rowin ? xb : 0;  // in-field columns of this row
  const T *row = global + (rowin ? (((long long)Z * gy + Y) * gx + b.px) * gdof : 0);
#pragma unroll
  for (int k = 0; k < VEL_U; ++k) {
    const int x = p.x0 + lane + 32 * k;
    const bool ok = x >= ra && x < rb;
    const T *rec = row + (long long)x * gdof;
    if constexpr (NV > 0) {
      constexpr int NT = NV * 16 / (int)sizeof(T);
      uint4 q[NV];
#pragma unroll
      for (int w = 0; w < NV; ++w) {
        q[w] = make_uint4(0, 0, 0, 0);
        if (ok) q[w] = __ldg(reinterpret_cast<const uint4 *>(rec) + w);
      }
      // first + DIM <= NT (checked by the caller): component c is one of
      // elements c .. c + NT - DIM of the record
#pragma unroll
      for (int c = 0; c < DIM; ++c) {
        T s = rec_elem<T>(q, c);
#pragma unroll
        for (int j = c + 1; j <= c + NT - DIM; ++j)
          if (j == first + c) s = rec_elem<T>(q, j);
        v[k][c] = s;
      }
    } else {
#pragma unroll
      for (int c = 0; c < DIM; ++c) v[k][c] = ok ? __ldg(rec + first + c) : T(0);
    }
  }
}

template <typename T, int DIM>
__device__ __forceinline__ void store_pass(const VBox &b, const VPass &p, T *__restrict__ out, T *stage, int lane,
                                           const T (&v)[VEL_U][DIM]) {
  __syncwarp();  // the previous pass has read the stage
#pragma unroll
  for (int k = 0; k < VEL_U; ++k)
#pragma unroll
    for (int c = 0; c < DIM; ++c) stage[(lane + 32 * k) * DIM + c] = v[k][c];
  __syncwarp();
  const int n = min(32 * VEL_U, b.nx - p.x0) * DIM;
  T *d = out + (b.offset + p.r * b.nx + p.x0) * DIM;
#pragma unroll
  for (int i = 0; i < VEL_U * DIM; ++i) {
    const int e = lane + 32 * i;
    if (e < n) d[e] = stage[e];
  }
}

template <typename T, int DIM, int NV>
__device__ __forceinline__ void copy_box(const VBox &b, const T *__restrict__ global, int gx, int gy, int gz, int gdof,
                                         int first, T *__restrict__ out, T *stage, long long warp0,
                                         long long nwarps) {
  const int lane = threadIdx.x & 31;
  const long long rows = (long long)b.ny * b.nz;
  if (warp0 >= rows || b.nx <= 0) return;
  const int xa = max(0, -b.px), xb = min(b.nx, gx - b.px);  // box columns inside the field
  const int dy = (int)(nwarps % b.ny);
  const int dz = (int)(nwarps / b.ny);
  VPass cur{warp0, (int)(warp0 % b.ny), (int)(warp0 / b.ny), 0};
  T v[VEL_U][DIM], w[VEL_U][DIM];
  load_pass<T, DIM, NV>(b, cur, global, gx, gy, gz, gdof, first, xa, xb, lane, v);
  for (;;) {
    VPass nxt = cur;
    nxt.x0 += 32 * VEL_U;
    if (nxt.x0 >= b.nx) {
      nxt.x0 = 0;
      nxt.r += nwarps;
      nxt.y += dy;
      nxt.z += dz;
      if (nxt.y >= b.ny) {
        nxt.y -= b.ny;
        ++nxt.z;
      }
    }
    const bool more = nxt.r < rows;
    if (more) load_pass<T, DIM, NV>(b, nxt, global, gx, gy, gz, gdof, first, xa, xb, lane, w);
    store_pass<T, DIM>(b, cur, out, stage, lane, v);
    if (!more) break;
    cur = nxt;
#pragma unroll
    for (int k = 0; k < VEL_U; ++k)
#pragma unroll
      for (int c = 0; c < DIM; ++c) v[k][c] = w[k][c];
  }
}

template <typename T, int DIM, int NV>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 6 : 4) velocity_box_kernel(VBox b, const T *__restrict__ global, int gx, int gy,
                                                           int gz, int gdof, int first, T *__restrict__ out) {
  __shared__ T stage[8][32 * VEL_U * DIM];
  copy_box<T, DIM, NV>(b, global, gx, gy, gz, gdof, first, out, stage[threadIdx.x >> 5],
                       (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5,
                       ((long long)gridDim.x * blockDim.x) >> 5);
}

template <typename T, int DIM, int NV>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 6 : 4) velocity_boxes_kernel(const dcell_box *__restrict__ boxes,
                                                             const T *__restrict__ global, int gx, int gy, int gz,
                                                             int gdof, int first, T *__restrict__ out) {
  const dcell_box d = boxes[blockIdx.y];
  VBox b;
  b.offset = d.offset;
  b.px = d.p[0];
  b.py = d.p[1];
  b.pz = d.p[2];
  b.nx = d.n[0];
  b.ny = d.n[1];
  b.nz = DIM == 3 ? d.n[2] : 1;
  __shared__ T stage[8][32 * VEL_U * DIM];
  copy_box<T, DIM, NV>(b, global, gx, gy, gz, gdof, first, out, stage[threadIdx.x >> 5],
                       (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5,
                       ((long long)gridDim.x * blockDim.x) >> 5);
}

// Record width in 16-byte words when the vector path applies, else 0.
template <typename T>
static int vec_words(const void *global, int gdof) {
  if (reinterpret_cast<uintptr_t>(global) % 16) return 0;
  const int bytes = gdof * (int)sizeof(T);
  return bytes == 16 ? 1 : bytes == 32 ? 2 : 0;
}

template <typename T, int DIM>
static void launch_one(dim3 grid, const VBox &b, const T *global, const int gd[3], int gdof, int first, T *vel,
                       cudaStream_t st) {
  constexpr int NV = sizeof(T) == 4 ? 1 : 2;  // 4 components: 16 B (FP32) or 32 B (FP64) per point
  if (vec_words<T>(global, gdof) == NV)
    velocity_box_kernel<T, DIM, NV><<<grid, 256, 0, st>>>(b, global, gd[0], gd[1], gd[2], gdof, first, vel);
  else
    velocity_box_kernel<T, DIM, 0><<<grid, 256, 0, st>>>(b, global, gd[0], gd[1], gd[2], gdof, first, vel);
}

template <typename T, int DIM>
static void launch_many(dim3 grid, const dcell_box *boxes, const T *global, const int gd[3], int gdof, int first,
                        T *vel, cudaStream_t st) {
  constexpr int NV = sizeof(T) == 4 ? 1 : 2;  // 4 components: 16 B (FP32) or 32 B (FP64) per point
  if (vec_words<T>(global, gdof) == NV)
    velocity_boxes_kernel<T, DIM, NV><<<grid, 256, 0, st>>>(boxes, global, gd[0], gd[1], gd[2], gdof, first, vel);
  else
    velocity_boxes_kernel<T, DIM, 0><<<grid, 256, 0, st>>>(boxes, global, gd[0], gd[1], gd[2], gdof, first, vel);
}

}  // namespace dcell

using namespace dcell;

int launch_velocity_box(const Geom &g, int dtype, const void *global, const int gdims[3], int gdof, int first,
                        void *vel, cudaStream_t st) {
  VBox b;
  b.offset = 0;
  b.px = g.px;
  b.py = g.py;
  b.pz = g.pz;
  b.nx = g.nx;
  b.ny = g.ny;
  b.nz = g.nz;
  const bool is2d = g.nz == 1 && gdims[2] <= 1;
  const int gd[3] = {gdims[0], gdims[1], is2d ? 1 : gdims[2]};
  const long long rows = (long long)g.ny * g.nz;
  long long blocks = (rows + 7) / 8;  // 8 warps of 256 threads, one row each
  if (blocks > 148LL * 32) blocks = 148LL * 32;
  if (blocks < 1) blocks = 1;
  const dim3 grid((unsigned)blocks);
  if (dtype == DCELL_F64) {
    if (is2d)
      launch_one<double, 2>(grid, b, (const double *)global, gd, gdof, first, (double *)vel, st);
    else
      launch_one<double, 3>(grid, b, (const double *)global, gd, gdof, first, (double *)vel, st);
  } else {
    if (is2d)
      launch_one<float, 2>(grid, b, (const float *)global, gd, gdof, first, (float *)vel, st);
    else
      launch_one<float, 3>(grid, b, (const float *)global, gd, gdof, first, (float *)vel, st);
  }
  return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
}

int launch_velocity_boxes(const dcell_box *boxes, int nboxes, int dim, int dtype, const void *global,
                          const int gdims[3], int gdof, int first, long long max_points, void *vel, cudaStream_t st) {
  if (nboxes <= 0) return DCELL_OK;
  const int gd[3] = {gdims[0], gdims[1], dim == 2 ? 1 : gdims[2]};
  long long bx = (max_points + 8 * 32 - 1) / (8 * 32);  // ~8 rows of >= 32 points per block
  if (bx > 64) bx = 64;  // per box; the warps stride over the rows of larger boxes
  if (bx < 1) bx = 1;
  const dim3 grid((unsigned)bx, (unsigned)nboxes);
  if (dtype == DCELL_F64) {
    if (dim == 2)
      launch_many<double, 2>(grid, boxes, (const double *)global, gd, gdof, first, (double *)vel, st);
    else
      launch_many<double, 3>(grid, boxes, (const double *)global, gd, gdof, first, (double *)vel, st);
  } else {
    if (dim == 2)
      launch_many<float, 2>(grid, boxes, (const float *)global, gd, gdof, first, (float *)vel, st);
    else
      launch_many<float, 3>(grid, boxes, (const float *)global, gd, gdof, first, (float *)vel, st);
  }
  return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
}

// max |v[c]| over n points of a dof-component field, as the bits of a
// non-negative FP32 (monotone as integers) combined with atomicMax into *out
__global__ void __launch_bounds__(256) max_abs_component_kernel(const float *__restrict__ v, long long n, int dof,
                                                                int comp, int *out) {
  float m = 0.f;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    m = fmaxf(m, fabsf(__ldg(v + i * dof + comp)));
#pragma unroll
  for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_int(m));
}

int launch_max_abs_component(const float *v, long long n, int dof, int comp, int *out, cudaStream_t st) {
  if (n <= 0) return DCELL_OK;
  long long blocks = (n + 255) / 256;
  if (blocks > 148LL * 8) blocks = 148LL * 8;
  max_abs_component_kernel<<<(int)blocks, 256, 0, st>>>(v, n, dof, comp, out);
  return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
}
