// Brick staging shared by the dense split-BF16 tensor-core stepper
// (sl_tc.cu) and the brick-staged CUDA-core steps (sl_cubic.cu): brick
// geometry, the two TMA boxes a brick reads (phi or its split words, and the
// interleaved MAC velocity), their edge replication, and the departures of a
// thread's points from the staged boxes.
//
// A CTA walks bricks of 32 x 4 x 4P arrival points, P = points each thread
// carries per step along z (2).  For each brick two tiled TMA loads stage
// the 32-bit phi words of the box [x0-4, x0+36) x [y0-2, y0+6) x [z0-2,
// z0+4P+2) and the interleaved velocity of [x0-4, x0+36) x [y0-1, y0+5) x
// [z0-1, z0+4P+1) in shared memory, completion tracked by an mbarrier's
// transaction count.  TMA x coordinates are multiples of 4 elements (16-byte
// rule); nothing starts a store at a negative coordinate.  Points whose
// departure (or midpoint) leaves the box -- per-component CFL >= 1 -- take the
// global-memory path.
#pragma once

#include "dcell_common.cuh"
#include "dcell_tma.cuh"
#include "sl_device.cuh"

namespace dcell {

struct BrickGrid {
  int nbx, nby, nbz;  // bricks of this launch per axis
  int bz0;            // z brick index of the launch's first brick (z-slab launches)
};

// Geometry of a brick and its two staged boxes (P points per thread along z).
template <int P>
struct BrickBox {
  static constexpr int BX = 32, BY = 4, BZ = 4 * P;          // 4 steps of P points
  static constexpr int PX = BX + 8, PY = BY + 4, PZ = BZ + 4;  // phi box (halo 4 | 2 | 2)
  static constexpr int VX = BX + 8, VY = BY + 2, VZ = BZ + 2;  // velocity box (halo 4 | 1 | 1)
  static constexpr int PhiBytes = PX * PY * PZ * 4;
  static constexpr int VelBytes = 3 * VX * VY * VZ * 4;
  static constexpr int BufBytes = PhiBytes + VelBytes;
  static_assert(PhiBytes % 128 == 0 && BufBytes % 128 == 0, "TMA destinations must stay 128-byte aligned");
  static_assert(3 * VX <= 256 && PX <= 256 && PY <= 256 && PZ <= 256, "TMA box dimensions are at most 256");
};

// Bricks are numbered z fastest, x slowest: a persistent CTA striding by the
// grid size then visits every x position (the x faces, where boxes need edge
// replication, are shared out evenly), and the bricks in flight at one time
// are z/y neighbours that share halo rows in L2.
template <class S>
__device__ __forceinline__ void brick_origin(const BrickGrid &bg, int b, int &x0, int &y0, int &z0) {
  const int bz = bg.bz0 + b % bg.nbz, r = b / bg.nbz;
  z0 = bz * S::BZ;
  y0 = (r % bg.nby) * S::BY;
  x0 = (r / bg.nby) * S::BX;
}

// one thread: both boxes of brick b into buffer `buf` (whose previous
// contents every thread has finished reading: order those generic-proxy reads
// before the async-proxy writes)
template <class S>
__device__ __forceinline__ void issue_brick(const BrickGrid &bg, int b, uint8_t *buf, const CUtensorMap *tm_phi,
                                            const CUtensorMap *tm_vel, uint64_t *bar) {
  int x0, y0, z0;
  brick_origin<S>(bg, b, x0, y0, z0);
  fence_proxy_async();
  mbar_expect_tx(bar, (uint32_t)S::BufBytes);
  tma_load_3d(buf, tm_phi, x0 - 4, y0 - 2, z0 - 2, bar);
  tma_load_3d(buf + S::PhiBytes, tm_vel, 3 * (x0 - 4), y0 - 1, z0 - 1, bar);
}

// Edge replication of a staged box.  TMA zero-fills the parts of a box that
// lie outside the grid; afterwards each of them holds the value of the
// nearest in-grid cell along each axis -- exactly what the reference's
// clamped interpolation indices read (Common/InterpolateVelocity.c and
// Common/LevelSetMethod.c clamp i, j, k to the grid independently).  A
// box-local read at an unclamped index then equals a global read at the
// clamped index, so the per-point code needs no clamping.  One pass per axis
// (x, y, z in that order, a CTA barrier between passes, each reading what the
// one before wrote), which replicates edges and corners like per-axis
// clamping.  The box is [DZ][DY][DX][C] 32-bit words whose cell (0,0,0) sits
// at grid point o[0..2]; in-grid cells of each axis are a non-empty range
// because the brick's own points are in the grid.  Run by threads 0 ..
// nthreads-1, together.  Returns whether the pass had anything to do (uniform
// over those threads).
template <int DX, int DY, int DZ, int C>
__device__ __forceinline__ bool replicate_pass(uint32_t *box, int axis, const int o[3], const int n[3],
                                               int nthreads) {
  constexpr int D[3] = {DX, DY, DZ};
  const int dim = D[axis];
  const int lo = min(max(-o[axis], 0), dim), hi = min(max(n[axis] - o[axis], 0), dim);  // in-grid [lo, hi)
  const int out = lo + (dim - hi);
  if (!out) return false;
  // a "line" is the stride-1 run of words inside one unit of this axis: C
  // words for x, one row (DX*C) for y, one plane (DY*DX*C) for z; "lines"
  // repeats over the slower axes
  const int inner = axis == 0 ? C : axis == 1 ? DX * C : DY * DX * C;
  const int lines = axis == 0 ? DY * DZ : axis == 1 ? DZ : 1;
  const int total = out * inner * lines;
  for (int i = threadIdx.x; i < total; i += nthreads) {
    const int w = i % inner, r = i / inner, j = r % out, line = r / out;
    const int dst = j < lo ? j : hi + (j - lo), src = j < lo ? lo : hi - 1;
    const int base = line * dim * inner + w;
    box[base + dst * inner] = box[base + src * inner];
  }
  return true;
}


// Front half of a thread's P points from the staged, edge-replicated boxes:
// node velocity, midpoint velocity, departure cell and fraction, and the box
// offset of each stencil's first word.  Point 0 sits at velocity-box cell
// (vx, vy, vz) / phi-box cell (px, py, pz), point p p planes above it.
// Consecutive points share the w face between them, and when all P midpoint
// cells have the same floors (checked over the warp) the trilinear stencils of
// one velocity component stack into P+1 layers: 4(P+1) corner loads instead
// of 8P.  hdth = -dt/(2h) per axis, so dl = U * hdth rounds exactly like
// (-U/2) * dt/h.  Returns false when a midpoint or a stencil leaves the box
// (per-component CFL >= 1): the warp then takes the global path.  The
// arithmetic is the clamped global path's, operation for operation (explicit
// roundings), so both give the same bits.
template <int BT, class S, int P>
__device__ __forceinline__ bool brick_depart(const float *__restrict__ vbox, int vx, int vy, int vz, int px, int py,
                                             int pz, const float dth[3], const float hdth[3], float f[P][3],
                                             int soff[P]) {
  constexpr int SX = 3, SY = 3 * S::VX, SZ = 3 * S::VX * S::VY;
  constexpr int ST[3] = {SX, SY, SZ};
  const float *v0 = vbox + (vz * S::VY + vy) * (3 * S::VX) + 3 * vx;  // point p's node is v0 + p SZ
  float wf[P + 1];
#pragma unroll
  for (int q = 0; q <= P; ++q) wf[q] = v0[q * SZ + 2];
  float U[P][3];
#pragma unroll
  for (int p = 0; p < P; ++p) {
    const float *v = v0 + p * SZ;
    U[p][0] = face_mean(v[0], v[SX]);
    U[p][1] = face_mean(v[1], v[SY + 1]);
    U[p][2] = face_mean(wf[p], wf[p + 1]);
  }
  bool near = true;
  if (BT == DCELL_MIDPOINT) {
    float sn[P][3], sp[P][3];
    int on[P][3];
#pragma unroll
    for (int p = 0; p < P; ++p)
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const float dl = rmul(U[p][a], hdth[a]);
        near = near && fabsf(dl) < 0.5f;
        // Along a component's own (staggered) axis the midpoint lies in
        // [X, X+1): floor 0, fraction t.  Across the other two axes the
        // node-centred fraction and floor serve both other components.
        // Where the result is used (|dl| < 0.5: `near`) floor(t) is -1 or 0,
        // so a sign test gives the floor and t - floor(t) is t + 1 or t.
        const float t = dl + 0.f;
        const bool ng = t < 0.f;
        sn[p][a] = ng ? t + 1.f : t;
        on[p][a] = ng ? -ST[a] : 0;
        sp[p][a] = dl + 0.5f;
      }
    bool same = true;
#pragma unroll
    for (int p = 1; p < P; ++p) same = same && on[p][0] == on[0][0] && on[p][1] == on[0][1] && on[p][2] == on[0][2];
    if (__all_sync(0xffffffffu, same)) {
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const float *q = v0 + d + (d == 0 ? 0 : on[0][0]) + (d == 1 ? 0 : on[0][1]) + (d == 2 ? 0 : on[0][2]);
        float L[P + 1][4];  // layer l: the 4 corners one z plane up per l
#pragma unroll
        for (int l = 0; l <= P; ++l) {
          L[l][0] = q[l * SZ];
          L[l][1] = q[l * SZ + SX];
          L[l][2] = q[l * SZ + SY];
          L[l][3] = q[l * SZ + SY + SX];
        }
#pragma unroll
        for (int p = 0; p < P; ++p) {
          const float s3[3] = {d == 0 ? sp[p][0] : sn[p][0], d == 1 ? sp[p][1] : sn[p][1],
                               d == 2 ? sp[p][2] : sn[p][2]};
          U[p][d] = trilerp(L[p][0], L[p][1], L[p][2], L[p][3], L[p + 1][0], L[p + 1][1], L[p + 1][2], L[p + 1][3],
                            s3);
        }
      }
    } else {
#pragma unroll
      for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int p = 0; p < P; ++p) {
          const float s3[3] = {d == 0 ? sp[p][0] : sn[p][0], d == 1 ? sp[p][1] : sn[p][1],
                               d == 2 ? sp[p][2] : sn[p][2]};
          const float *q = v0 + p * SZ + d + (d == 0 ? 0 : on[p][0]) + (d == 1 ? 0 : on[p][1]) +
                           (d == 2 ? 0 : on[p][2]);
          U[p][d] = trilerp(q[0], q[SX], q[SY], q[SY + SX], q[SZ], q[SZ + SX], q[SZ + SY], q[SZ + SY + SX], s3);
        }
    }
  }
  bool in = near;
#pragma unroll
  for (int p = 0; p < P; ++p) {
    int cl[3];
    const int Pc[3] = {px, py, pz + p};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float t = rmul(-U[p][a], dth[a]);
      const float fl = floorf(t);
      cl[a] = Pc[a] + (int)fl - 1;  // first stencil cell, box-local
      f[p][a] = t - fl;
    }
    soff[p] = (cl[2] * S::PY + cl[1]) * S::PX + cl[0];
    in = in && (unsigned)cl[0] <= (unsigned)(S::PX - 4) && (unsigned)cl[1] <= (unsigned)(S::PY - 4) &&
         (unsigned)cl[2] <= (unsigned)(S::PZ - 4);
  }
  return in;
}

}  // namespace dcell
