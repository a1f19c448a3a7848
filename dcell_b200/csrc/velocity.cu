// Velocity acquisition: the velocity grid of a level set's box from the
// fluid's global MAC field -- LevelSetGetVelocity (LevelSetMethod/Advect.c:
// 145-192).  The reference resizes the velocity grid to the phi box (which
// zeroes it, Common/Grid.c:146) and NGA_Gets the part of the box inside the
// Global Array [z][y][x][c] (components U_FACE.. of the cell, CELL_CENTER
// first).  Here the global field is a device array and the copy is a kernel:
// one thread per (point, component) of the box, x fastest so the global reads
// and the box writes coalesce; zero outside the field.  The batched form
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

template <typename T, int DIM>
__device__ __forceinline__ void copy_box(const VBox &b, const T *__restrict__ global, int gx, int gy, int gz, int gdof,
                                         int first, T *__restrict__ out, long long start, long long stride) {
  const long long total = (long long)b.nx * b.ny * b.nz * DIM;
  for (long long e = start; e < total; e += stride) {
    const int c = (int)(e % DIM);
    const long long q = e / DIM;
    const int x = (int)(q % b.nx), y = (int)((q / b.nx) % b.ny), z = (int)(q / ((long long)b.nx * b.ny));
    const int X = b.px + x, Y = b.py + y, Z = DIM == 3 ? b.pz + z : 0;
    T v = T(0);
    if (X >= 0 && X < gx && Y >= 0 && Y < gy && Z >= 0 && Z < gz)
      v = global[(((long long)Z * gy + Y) * gx + X) * gdof + first + c];
    out[b.offset * DIM + e] = v;
  }
}

template <typename T, int DIM>
__global__ void __launch_bounds__(256) velocity_box_kernel(VBox b, const T *__restrict__ global, int gx, int gy,
                                                           int gz, int gdof, int first, T *__restrict__ out) {
  copy_box<T, DIM>(b, global, gx, gy, gz, gdof, first, out, blockIdx.x * (long long)blockDim.x + threadIdx.x,
                   (long long)gridDim.x * blockDim.x);
}

template <typename T, int DIM>
__global__ void __launch_bounds__(256) velocity_boxes_kernel(const dcell_box *__restrict__ boxes,
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
  copy_box<T, DIM>(b, global, gx, gy, gz, gdof, first, out, blockIdx.x * (long long)blockDim.x + threadIdx.x,
                   (long long)gridDim.x * blockDim.x);
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
  const long long total = (long long)g.nx * g.ny * g.nz * (is2d ? 2 : 3);
  long long blocks = (total + 255) / 256;
  if (blocks > 148LL * 32) blocks = 148LL * 32;
  if (blocks < 1) blocks = 1;
  if (dtype == DCELL_F64) {
    if (is2d)
      velocity_box_kernel<double, 2><<<(int)blocks, 256, 0, st>>>(b, (const double *)global, gdims[0], gdims[1], 1,
                                                                  gdof, first, (double *)vel);
    else
      velocity_box_kernel<double, 3><<<(int)blocks, 256, 0, st>>>(b, (const double *)global, gdims[0], gdims[1],
                                                                  gdims[2], gdof, first, (double *)vel);
  } else {
    if (is2d)
      velocity_box_kernel<float, 2><<<(int)blocks, 256, 0, st>>>(b, (const float *)global, gdims[0], gdims[1], 1, gdof,
                                                                 first, (float *)vel);
    else
      velocity_box_kernel<float, 3><<<(int)blocks, 256, 0, st>>>(b, (const float *)global, gdims[0], gdims[1],
                                                                 gdims[2], gdof, first, (float *)vel);
  }
  return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
}

int launch_velocity_boxes(const dcell_box *boxes, int nboxes, int dim, int dtype, const void *global,
                          const int gdims[3], int gdof, int first, long long max_points, void *vel, cudaStream_t st) {
  if (nboxes <= 0) return DCELL_OK;
  long long bx = (max_points * dim + 255) / 256;
  if (bx > 64) bx = 64;  // per box; the blocks stride over larger boxes
  if (bx < 1) bx = 1;
  const dim3 grid((unsigned)bx, (unsigned)nboxes);
  if (dtype == DCELL_F64) {
    if (dim == 2)
      velocity_boxes_kernel<double, 2><<<grid, 256, 0, st>>>(boxes, (const double *)global, gdims[0], gdims[1], 1,
                                                             gdof, first, (double *)vel);
    else
      velocity_boxes_kernel<double, 3><<<grid, 256, 0, st>>>(boxes, (const double *)global, gdims[0], gdims[1],
                                                             gdims[2], gdof, first, (double *)vel);
  } else {
    if (dim == 2)
      velocity_boxes_kernel<float, 2><<<grid, 256, 0, st>>>(boxes, (const float *)global, gdims[0], gdims[1], 1, gdof,
                                                            first, (float *)vel);
    else
      velocity_boxes_kernel<float, 3><<<grid, 256, 0, st>>>(boxes, (const float *)global, gdims[0], gdims[1],
                                                            gdims[2], gdof, first, (float *)vel);
  }
  return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
}
