// Production FP32 trilinear semi-Lagrangian step: the reference's own
// LevelSetAdvectSL_2D / _3D mode (LevelSetMethod/AdvectSL.c:23-89) -- MAC
// velocity at the arrival node (Common/InterpolateVelocity.c:7-67), departure
// S = X - V dt / h, bi/trilinear phi0 at S (Common/Grid.c:190-212,
// Grid3D.c:4-31) -- plus the midpoint backtrace.
//
// This unit is compiled with FMA contraction.  The bit-exact FP64 path stays
// the reference-order kernel of sl_exact.cu; this one is the fast FP32 form:
// dt / h is formed once on the host, the departure is carried as an integer
// cell plus an FP32 fraction (S = X + t, cell = X + floor(t), frac = t -
// floor(t): exact to the precision of the displacement, not of the absolute
// coordinate), interpolation is nested lerps (one subtraction and one FMA
// each), and index math is 32-bit.  Every rounding is explicit
// (__fmul_rn / __fmaf_rn / __fsub_rn / __fadd_rn), so the staged and the
// global-memory paths below give the same bits.
//
// Dense 3-D grids (nx % 4 == 0) march z-columns through a plane ring staged
// by TMA: a CTA owns a 32 x TY tile (TY = 8 for Euler, 16 for the midpoint)
// of every plane of a z-run, each consumer warp two of its rows, and keeps
// planes z-2 .. z+5 of phi0 (40 x (TY+4) floats, halo 4 | 2) and of the
// interleaved velocity in an 8-slot ring; each plane is loaded once as it
// enters the window, three planes ahead of its first use.  Per point: 6
// (Euler) or 6 + 24 (midpoint) velocity and 8 phi0 values from shared memory,
// one coalesced store.  Bands, 2-D grids and other shapes run the
// global-gather kernel with the same arithmetic.
#include <math.h>

#include <stdlib.h>

#include <algorithm>

#include "dcell_common.cuh"
#include "dcell_kernels.h"
#include "dcell_tma.cuh"
#include "sl_device.cuh"

namespace dcell {
namespace lin {

constexpr int TX = 32;                     // points of a tile row (one warp)
constexpr int HX = 4, HY = 2;              // phi box halo (x: 4 keeps TMA x coordinates 16-byte aligned)
constexpr int PW = TX + 2 * HX;            // 40 phi values per box row
constexpr int kRing = 8;                   // ring slots: planes z-2 .. z+2 in use, up to three ahead

// A tile of TX x TY points per plane: TY / RW consumer warps (RW adjacent
// tile rows each) and one producer warp.  The phi box is [x0-4, x0+36) x
// [y0-2, y0+TY+2).
// The velocity box holds what the backtrace reads: the faces around the
// nodes for Euler, [x0, x0+36) x [y0, y0+TY+1) (36 points keep the row a
// multiple of 16 bytes), and the midpoint's trilinear corners within one
// cell of the nodes as well, [x0-4, x0+36) x [y0-1, y0+TY+2).  Planes start
// on 128-byte boundaries.
template <int TY_, int BT, int RW_>
struct MarchShape {
  static constexpr int TY = TY_;
  static constexpr int RW = RW_;      // tile rows per consumer warp
  static constexpr int Warps = TY / RW;  // consumer warps
  static constexpr int PH = TY + 2 * HY;
  static constexpr int VX0 = BT == DCELL_MIDPOINT ? -4 : 0;   // velocity box x origin - x0
  static constexpr int VY0 = BT == DCELL_MIDPOINT ? -1 : 0;   // velocity box y origin - y0
  static constexpr int VXN = BT == DCELL_MIDPOINT ? 40 : 36;  // velocity box points per row
  static constexpr int VH = BT == DCELL_MIDPOINT ? TY + 3 : TY + 1;
  static constexpr int VW = 3 * VXN;                            // velocity floats per box row
  static constexpr int PlanePhi = PW * PH;                      // floats of one staged phi plane
  static constexpr int PlaneVel = (VW * VH + 31) / 32 * 32;     // floats of one staged velocity plane (padded)
  static constexpr int VelBoxBytes = 4 * VW * VH;               // bytes a velocity load writes
  static constexpr int PlaneBytes = 4 * PlanePhi + VelBoxBytes;  // transaction bytes per plane
  static constexpr int Threads = 32 * (Warps + 1);
  static constexpr int Smem = kRing * 4 * (PlanePhi + PlaneVel) + 2 * kRing * 8;  // + full / empty mbarriers
  static constexpr int CtasPerSm = (228 * 1024) / (Smem + 1024) < 4 ? (228 * 1024) / (Smem + 1024) : 4;
  static_assert((4 * PlanePhi) % 128 == 0 && (4 * PlaneVel) % 128 == 0, "staged planes stay 128-byte aligned");
  static_assert((4 * VW) % 16 == 0 && (4 * PW) % 16 == 0, "box rows are multiples of 16 bytes");
  static_assert(CtasPerSm >= 1, "ring too large for one CTA");
  static_assert(TY % RW == 0, "whole rows per consumer warp");
};
static_assert((kRing & (kRing - 1)) == 0 && kRing >= 8, "ring slot of plane p is (p + kRing) & (kRing - 1)");

// phi0 / velocity through global memory, indices clamped into the grid (the
// reference's per-axis clamping).
template <int DIM>
struct GlobalAcc {
  const float *__restrict__ phi0;
  const float *__restrict__ vel;
  int nx, ny, nz;
  __device__ __forceinline__ int at(int i, int j, int k) const {
    i = clampi(i, 0, nx - 1);
    j = clampi(j, 0, ny - 1);
    k = DIM == 3 ? clampi(k, 0, nz - 1) : 0;
    return (k * ny + j) * nx + i;
  }
  __device__ __forceinline__ float phi(int i, int j, int k) const { return __ldg(phi0 + at(i, j, k)); }
  __device__ __forceinline__ float v(int i, int j, int k, int d) const { return __ldg(vel + DIM * at(i, j, k) + d); }
};

// The staged ring: box origin (bx, by) = (x0 - 4, y0 - 2) of the tile; plane
// p of the grid sits in slot (p + kRing) & (kRing - 1) and holds plane
// clamp(p, 0, nz - 1) (the z clamping is done by the load).  CLAMP (tiles
// whose box crosses the grid's x or y edge): columns and rows are clamped
// into the grid and into the box in one step, so a read at any index stays
// in the ring and equals the global clamped read wherever the grid-clamped
// position lies in the box.  Without CLAMP (the box inside the grid) indices
// map straight into the box: lin_points reads only indices it has checked to
// lie in the box.
template <class S, bool CLAMP>
struct BoxAcc {
  const float *phis;  // ring of phi planes
  const float *vels;  // ring of velocity planes
  int bx, by;         // phi box origin (grid coordinates)
  int vbx, vby;       // velocity box origin
  int clo, chi;       // phi box columns that hold grid columns: [max(-bx, 0), min(nx - 1 - bx, PW - 1)]
  int rlo, rhi;       // phi box rows that hold grid rows
  int vclo, vchi, vrlo, vrhi;  // the same for the velocity box
  __device__ __forceinline__ BoxAcc(const float *p, const float *v, int x0, int y0, int nx, int ny)
      : phis(p), vels(v), bx(x0 - HX), by(y0 - HY), vbx(x0 + S::VX0), vby(y0 + S::VY0),
        clo(max(HX - x0, 0)), chi(min(nx - 1 - (x0 - HX), PW - 1)), rlo(max(HY - y0, 0)),
        rhi(min(ny - 1 - (y0 - HY), S::PH - 1)), vclo(max(-(x0 + S::VX0), 0)),
        vchi(min(nx - 1 - (x0 + S::VX0), S::VXN - 1)), vrlo(max(-(y0 + S::VY0), 0)),
        vrhi(min(ny - 1 - (y0 + S::VY0), S::VH - 1)) {}
  __device__ __forceinline__ int col(int i) const { return CLAMP ? clampi(i - bx, clo, chi) : i - bx; }
  __device__ __forceinline__ int row(int j) const { return CLAMP ? clampi(j - by, rlo, rhi) : j - by; }
  __device__ __forceinline__ int vcol(int i) const { return CLAMP ? clampi(i - vbx, vclo, vchi) : i - vbx; }
  __device__ __forceinline__ int vrow(int j) const { return CLAMP ? clampi(j - vby, vrlo, vrhi) : j - vby; }
  __device__ __forceinline__ static int slot(int k) { return (k + kRing) & (kRing - 1); }
  __device__ __forceinline__ float phi(int i, int j, int k) const {
    return phis[slot(k) * S::PlanePhi + row(j) * PW + col(i)];
  }
  __device__ __forceinline__ float v(int i, int j, int k, int d) const {
    return vels[slot(k) * S::PlaneVel + vrow(j) * S::VW + 3 * vcol(i) + d];
  }
};

// Paired FP32 (fma.rn.f32x2 / add / mul): two points of one thread advance
// together, each lane rounding exactly as the scalar helpers of
// sl_device.cuh do (explicit round-to-nearest, no contraction), so a pair
// gives the bits of two scalar evaluations.
__device__ __forceinline__ float2 pair(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 lerp2(float2 a, float2 b, float2 s) {  // a + s (b - a)
  return __ffma2_rn(s, __fadd2_rn(b, make_float2(-a.x, -a.y)), a);
}
__device__ __forceinline__ float2 trilerp2(float2 v000, float2 v100, float2 v010, float2 v110, float2 v001,
                                           float2 v101, float2 v011, float2 v111, const float2 s[3]) {
  return lerp2(lerp2(lerp2(v000, v100, s[0]), lerp2(v010, v110, s[0]), s[1]),
               lerp2(lerp2(v001, v101, s[0]), lerp2(v011, v111, s[0]), s[1]), s[2]);
}
__device__ __forceinline__ float2 face_mean2(float2 a, float2 b) {  // 0.5 a + (0.5 b), as face_mean
  return __ffma2_rn(pair(0.5f, 0.5f), a, __fmul2_rn(pair(0.5f, 0.5f), b));
}

// lin_points for two points of one thread on a 3-D grid (rows y[0], y[1]):
// the same operations in the same order, the two points' floating-point
// steps paired.
template <int BT, bool VOTE, class A>
__device__ __forceinline__ bool lin_points_pair(const A &acc, int x, const int y[2], int z, const float dth[3],
                                                const float hdth[3], float out[2], int c[2][3], float f[2][3]) {
  const int y0 = y[0], y1 = y[1];
  float2 U[3];
  U[0] = face_mean2(pair(acc.v(x, y0, z, 0), acc.v(x, y1, z, 0)), pair(acc.v(x + 1, y0, z, 0), acc.v(x + 1, y1, z, 0)));
  U[1] = face_mean2(pair(acc.v(x, y0, z, 1), acc.v(x, y1, z, 1)), pair(acc.v(x, y0 + 1, z, 1), acc.v(x, y1 + 1, z, 1)));
  U[2] = face_mean2(pair(acc.v(x, y0, z, 2), acc.v(x, y1, z, 2)), pair(acc.v(x, y0, z + 1, 2), acc.v(x, y1, z + 1, 2)));
  const int X0[3] = {x, y0, z}, X1[3] = {x, y1, z};
  if (BT == DCELL_MIDPOINT) {
    float2 dl[3];
    bool near = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      dl[a] = __fmul2_rn(U[a], pair(hdth[a], hdth[a]));
      near = near && fabsf(dl[a].x) < 1.f && fabsf(dl[a].y) < 1.f;
    }
    if (VOTE && !__all_sync(0xffffffffu, near)) return false;
    float2 V[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      int b0[3], b1[3];
      float2 s[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) {  // the component's own axis carries the half-cell stagger
        const float2 t = a == d ? __fadd2_rn(dl[a], pair(0.5f, 0.5f)) : dl[a];
        const float fl0 = floorf(t.x), fl1 = floorf(t.y);
        b0[a] = X0[a] + (int)fl0;
        b1[a] = X1[a] + (int)fl1;
        s[a] = __fadd2_rn(t, pair(-fl0, -fl1));
      }
      V[d] = trilerp2(pair(acc.v(b0[0], b0[1], b0[2], d), acc.v(b1[0], b1[1], b1[2], d)),
                      pair(acc.v(b0[0] + 1, b0[1], b0[2], d), acc.v(b1[0] + 1, b1[1], b1[2], d)),
                      pair(acc.v(b0[0], b0[1] + 1, b0[2], d), acc.v(b1[0], b1[1] + 1, b1[2], d)),
                      pair(acc.v(b0[0] + 1, b0[1] + 1, b0[2], d), acc.v(b1[0] + 1, b1[1] + 1, b1[2], d)),
                      pair(acc.v(b0[0], b0[1], b0[2] + 1, d), acc.v(b1[0], b1[1], b1[2] + 1, d)),
                      pair(acc.v(b0[0] + 1, b0[1], b0[2] + 1, d), acc.v(b1[0] + 1, b1[1], b1[2] + 1, d)),
                      pair(acc.v(b0[0], b0[1] + 1, b0[2] + 1, d), acc.v(b1[0], b1[1] + 1, b1[2] + 1, d)),
                      pair(acc.v(b0[0] + 1, b0[1] + 1, b0[2] + 1, d), acc.v(b1[0] + 1, b1[1] + 1, b1[2] + 1, d)), s);
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) U[a] = V[a];
  }
  bool in = true;
  float2 fr[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float2 t = __fmul2_rn(pair(-U[a].x, -U[a].y), pair(dth[a], dth[a]));
    in = in && t.x >= -2.f && t.x < 2.f && t.y >= -2.f && t.y < 2.f;
    const float fl0 = floorf(t.x), fl1 = floorf(t.y);
    c[0][a] = X0[a] + (int)fl0;
    c[1][a] = X1[a] + (int)fl1;
    fr[a] = __fadd2_rn(t, pair(-fl0, -fl1));
    f[0][a] = fr[a].x;
    f[1][a] = fr[a].y;
  }
  if (VOTE && !__all_sync(0xffffffffu, in)) return false;
  const int *C0 = c[0], *C1 = c[1];
  const float2 v = trilerp2(pair(acc.phi(C0[0], C0[1], C0[2]), acc.phi(C1[0], C1[1], C1[2])),
                            pair(acc.phi(C0[0] + 1, C0[1], C0[2]), acc.phi(C1[0] + 1, C1[1], C1[2])),
                            pair(acc.phi(C0[0], C0[1] + 1, C0[2]), acc.phi(C1[0], C1[1] + 1, C1[2])),
                            pair(acc.phi(C0[0] + 1, C0[1] + 1, C0[2]), acc.phi(C1[0] + 1, C1[1] + 1, C1[2])),
                            pair(acc.phi(C0[0], C0[1], C0[2] + 1), acc.phi(C1[0], C1[1], C1[2] + 1)),
                            pair(acc.phi(C0[0] + 1, C0[1], C0[2] + 1), acc.phi(C1[0] + 1, C1[1], C1[2] + 1)),
                            pair(acc.phi(C0[0], C0[1] + 1, C0[2] + 1), acc.phi(C1[0], C1[1] + 1, C1[2] + 1)),
                            pair(acc.phi(C0[0] + 1, C0[1] + 1, C0[2] + 1), acc.phi(C1[0] + 1, C1[1] + 1, C1[2] + 1)),
                            fr);
  out[0] = v.x;
  out[1] = v.y;
  return true;
}

// R arrival points of one thread (local indices x, y[r], z): node velocity,
// optional midpoint velocity, departure, bi/trilinear phi0, into out[r]; c,
// f: the departure cells (local) and fractions.  dth = dt / h per axis,
// hdth = -dt / (2 h).  Each phase runs over all R points before the next, so
// their loads overlap.  VOTE (staged boxes; called by whole warps): before
// the midpoint velocity and before phi0 are read, the warp checks that every
// lane's reads of all R points stay in the staged box (|midpoint offset| <
// 1, departure offset in [-2, 2) per axis) and returns false, with nothing
// read, where one does not; the node velocity always lies in the box.  The
// arithmetic is the same either way, so a warp redone through global memory
// gives the same bits.
template <int BT, int DIM, bool VOTE, int R, class A>
__device__ __forceinline__ bool lin_points(const A &acc, int x, const int y[R], int z, const float dth[3],
                                           const float hdth[3], float out[R], int c[R][3], float f[R][3]) {
  float U[R][3];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    U[r][0] = face_mean(acc.v(x, y[r], z, 0), acc.v(x + 1, y[r], z, 0));
    U[r][1] = face_mean(acc.v(x, y[r], z, 1), acc.v(x, y[r] + 1, z, 1));
    U[r][2] = DIM == 3 ? face_mean(acc.v(x, y[r], z, 2), acc.v(x, y[r], z + 1, 2)) : 0.f;
  }
  if (BT == DCELL_MIDPOINT) {
    float dl[R][3];
    bool near = true;
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        dl[r][a] = rmul(U[r][a], hdth[a]);
        near = near && fabsf(dl[r][a]) < 1.f;
      }
    if (VOTE && !__all_sync(0xffffffffu, near)) return false;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int X[3] = {x, y[r], z};
      float V[3] = {0.f, 0.f, 0.f};
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        int b[3] = {0, 0, z};
        float s[3] = {0.f, 0.f, 0.f};
#pragma unroll
        for (int a = 0; a < DIM; ++a) {  // the component's own axis carries the half-cell stagger
          const float t = a == d ? __fadd_rn(dl[r][a], 0.5f) : dl[r][a];
          const float fl = floorf(t);
          b[a] = X[a] + (int)fl;
          s[a] = __fsub_rn(t, fl);
        }
        if (DIM == 3)
          V[d] = trilerp(acc.v(b[0], b[1], b[2], d), acc.v(b[0] + 1, b[1], b[2], d), acc.v(b[0], b[1] + 1, b[2], d),
                         acc.v(b[0] + 1, b[1] + 1, b[2], d), acc.v(b[0], b[1], b[2] + 1, d),
                         acc.v(b[0] + 1, b[1], b[2] + 1, d), acc.v(b[0], b[1] + 1, b[2] + 1, d),
                         acc.v(b[0] + 1, b[1] + 1, b[2] + 1, d), s);
        else
          V[d] = bilerp(acc.v(b[0], b[1], 0, d), acc.v(b[0] + 1, b[1], 0, d), acc.v(b[0], b[1] + 1, 0, d),
                        acc.v(b[0] + 1, b[1] + 1, 0, d), s[0], s[1]);
      }
#pragma unroll
      for (int a = 0; a < DIM; ++a) U[r][a] = V[a];
    }
  }
  bool in = true;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int X[3] = {x, y[r], z};
    c[r][2] = z;
    f[r][2] = 0.f;
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
      const float t = rmul(-U[r][a], dth[a]);
      in = in && t >= -2.f && t < 2.f;
      const float fl = floorf(t);
      c[r][a] = X[a] + (int)fl;
      f[r][a] = __fsub_rn(t, fl);
    }
  }
  if (VOTE && !__all_sync(0xffffffffu, in)) return false;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int *C = c[r];
    if (DIM == 3)
      out[r] = trilerp(acc.phi(C[0], C[1], C[2]), acc.phi(C[0] + 1, C[1], C[2]), acc.phi(C[0], C[1] + 1, C[2]),
                       acc.phi(C[0] + 1, C[1] + 1, C[2]), acc.phi(C[0], C[1], C[2] + 1),
                       acc.phi(C[0] + 1, C[1], C[2] + 1), acc.phi(C[0], C[1] + 1, C[2] + 1),
                       acc.phi(C[0] + 1, C[1] + 1, C[2] + 1), f[r]);
    else
      out[r] = bilerp(acc.phi(C[0], C[1], 0), acc.phi(C[0] + 1, C[1], 0), acc.phi(C[0], C[1] + 1, 0),
                      acc.phi(C[0] + 1, C[1] + 1, 0), f[r][0], f[r][1]);
  }
  return true;
}

// Global-gather form: one thread per arrival point of the band (or of the
// dense grid when band is null).  Band entries outside the grid are skipped
// and flagged; on bands, a departure outside the grid (clamped) is flagged.
template <int BT, int DIM>
__global__ void __launch_bounds__(256) sl_lin_gather_kernel(Geom g, const float *__restrict__ phi0,
                                                            const float *__restrict__ vel, float dth0, float dth1,
                                                            float dth2, const int *__restrict__ band, int npts,
                                                            float *__restrict__ phi, int *flags) {
  const float dth[3] = {dth0, dth1, dth2};
  const float hdth[3] = {-0.5f * dth0, -0.5f * dth1, -0.5f * dth2};
  const GlobalAcc<DIM> acc{phi0, vel, g.nx, g.ny, g.nz};
  const int n[3] = {g.nx, g.ny, g.nz};
  bool bad = false, clamped = false;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < npts; q += gridDim.x * blockDim.x) {
    int x, y, z;
    if (!arrival_local(g, band, q, x, y, z)) {
      bad = true;
      continue;
    }
    int c[1][3];
    float f[1][3];
    float v[1];
    const int yy[1] = {y};
    lin_points<BT, DIM, false, 1>(acc, x, yy, z, dth, hdth, v, c, f);
    phi[(z * g.ny + y) * g.nx + x] = v[0];
#pragma unroll
    for (int a = 0; a < DIM; ++a) clamped |= c[0][a] < 0 || c[0][a] + (f[0][a] > 0.f ? 1 : 0) > n[a] - 1;
  }
  if (bad) raise_flag(flags, FLAG_BAD_BAND);
  if (clamped && band) raise_flag(flags, FLAG_DEPARTURE_CLAMPED);  // dense grids: the edge is the domain boundary
}

struct MarchGrid {
  int ncx;     // tiles per row of tiles (x)
  int ntiles;  // tiles per plane
  int seglen;  // planes per z-segment
  int units;   // segments x tiles: unit u = segment (u / ntiles) of tile (u % ntiles)
};

// One z-run of a tile on the consumer side: planes [zs, ze) of the tile at
// (x0, y0), the staged ring read through accessor A (clamped at the grid's x
// / y edges, or not); warps whose reads would leave the box redo the plane
// through global memory.  Returns false when a wait gave up.
template <int BT, class S, class A>
__device__ __forceinline__ bool march_run(const A &bacc, const GlobalAcc<3> &gacc, const Geom &g, int x0, int y0,
                                          int zs, int ze, int lane, int warp, const float dth[3], const float hdth[3],
                                          uint64_t *full, uint64_t *empty, uint32_t &fpar, float *__restrict__ phi) {
  const int x = min(x0 + lane, g.nx - 1);
  int y[S::RW];
  bool store[S::RW];
#pragma unroll
  for (int r = 0; r < S::RW; ++r) {  // the warp's rows: y0 + RW * warp + r
    const int yr = y0 + S::RW * warp + r;
    y[r] = min(yr, g.ny - 1);
    store[r] = x0 + lane < g.nx && yr < g.ny;
  }
  int waited = zs - 2;
  for (int z = zs; z < ze; ++z) {
    for (; waited <= z + 2; ++waited) {  // planes up to z + 2 present
      const int s = BoxAcc<S, false>::slot(waited);
      const bool ok = mbar_wait_sleep(&full[s], (fpar >> s) & 1u);
      if (!__all_sync(0xffffffffu, ok)) return false;
      fpar ^= 1u << s;
    }
    int c[S::RW][3];
    float f[S::RW][3];
    float v[S::RW];
    if constexpr (S::RW == 2) {  // two rows per warp: the points' arithmetic in f32x2 pairs
      if (!lin_points_pair<BT, true>(bacc, x, y, z, dth, hdth, v, c, f))
        lin_points_pair<BT, false>(gacc, x, y, z, dth, hdth, v, c, f);
    } else {
      if (!lin_points<BT, 3, true, S::RW>(bacc, x, y, z, dth, hdth, v, c, f))
        lin_points<BT, 3, false, S::RW>(gacc, x, y, z, dth, hdth, v, c, f);
    }
#pragma unroll
    for (int r = 0; r < S::RW; ++r)
      if (store[r]) phi[(z * g.ny + y[r]) * g.nx + x] = v[r];
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[BoxAcc<S, false>::slot(z - 2)]);  // plane z - 2 read for the last time
  }
  __syncwarp();
  if (lane == 0)
    for (int p = max(ze - 2, zs - 2); p <= ze + 1; ++p) mbar_arrive(&empty[BoxAcc<S, false>::slot(p)]);
  return true;
}

// Dense 3-D march (see the head of the file).  Work units are z-segments of
// `seglen` planes of one tile, numbered segment-major (all tiles of a
// segment, then the next segment), and CTA b takes units b, b + G, b + 2G,
// ...: the CTAs in flight work on neighbouring tiles of the same segment at
// the same time, so the halo rows their boxes share come from L2, and a
// segment's boundary planes, reloaded by the next segment's unit one round
// later, too.  Per unit a producer warp loads every plane the unit reads
// (zs-2 .. ze+1) into the ring, each one once the slot's previous plane is
// released; the TY / RW consumer warps wait on a slot's `full` mbarrier
// before a plane's first use, compute their rows of the plane, release plane z-2
// on its `empty` mbarrier after plane z (the unit's last planes at its end).
// No CTA barrier in the loop: warps drift up to a few planes apart.  Warps
// whose points read outside the staged box (per-axis displacement >= 2, or a
// midpoint offset >= 1) take the global path for that plane.  Every wait is
// bounded; a warp that gives up raises FLAG_WAIT_TIMEOUT and leaves (the
// others then give up at their next wait), and the producer waits (bounded)
// for its last load per slot before the CTA ends.
template <int BT, int TY, int RW>
__global__ void __launch_bounds__(MarchShape<TY, BT, RW>::Threads, MarchShape<TY, BT, RW>::CtasPerSm)
    sl_lin_march_kernel(const __grid_constant__ CUtensorMap tm_phi, const __grid_constant__ CUtensorMap tm_vel,
                        Geom g, MarchGrid mg, const float *__restrict__ phi0, const float *__restrict__ vel, float dth0,
                        float dth1, float dth2, float *__restrict__ phi, int *flags) {
  using S = MarchShape<TY, BT, RW>;
  extern __shared__ __align__(1024) uint8_t smem[];
  float *const phis = reinterpret_cast<float *>(smem);
  float *const vels = phis + kRing * S::PlanePhi;
  uint64_t *const full = reinterpret_cast<uint64_t *>(smem + kRing * 4 * (S::PlanePhi + S::PlaneVel));
  uint64_t *const empty = full + kRing;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0)
    for (int s = 0; s < kRing; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], S::Warps);
    }
  __syncthreads();

  if (warp == S::Warps) {  // ---------------- producer ----------------
    if (lane == 0) {
      uint32_t used = 0, epar = 0, lastpar = 0;  // per slot: loaded once, next empty phase, phase of the last load
      bool err = false;
      for (int u = blockIdx.x; u < mg.units && !err; u += gridDim.x) {
        const int seg = u / mg.ntiles, tile = u - seg * mg.ntiles;
        const int zs = seg * mg.seglen, ze = min(g.nz, zs + mg.seglen);
        const int x0 = (tile % mg.ncx) * TX, y0 = (tile / mg.ncx) * TY;
        for (int p = zs - 2; p <= ze + 1; ++p) {
          const int s = BoxAcc<S, false>::slot(p), pz = clampi(p, 0, g.nz - 1);
          const uint32_t bit = 1u << s;
          if (used & bit) {  // suspend-hinted: a polling producer would take issue slots from the consumers
            if (!mbar_wait_sleep(&empty[s], (epar & bit) ? 1u : 0u)) {
              err = true;
              break;
            }
            epar ^= bit;
            lastpar ^= bit;
          }
          used |= bit;
          fence_proxy_async();  // the consumers' reads of the slot before these writes
          mbar_expect_tx(&full[s], (uint32_t)S::PlaneBytes);
          tma_load_3d(phis + s * S::PlanePhi, &tm_phi, x0 - HX, y0 - HY, pz, &full[s]);
          tma_load_3d(vels + s * S::PlaneVel, &tm_vel, 3 * (x0 + S::VX0), y0 + S::VY0, pz, &full[s]);
        }
      }
      // nothing may still be in flight when the CTA's shared memory goes away
      bool ok = true;
      for (int s = 0; s < kRing; ++s)
        if (used & (1u << s)) ok &= mbar_wait(&full[s], (lastpar >> s) & 1u);
      if (err || !ok) raise_flag(flags, FLAG_WAIT_TIMEOUT);
    }
    return;
  }
  // ---------------- consumers: warp w = tile rows RW w .. RW w + RW - 1 ----------------
  const float dth[3] = {dth0, dth1, dth2};
  const float hdth[3] = {-0.5f * dth0, -0.5f * dth1, -0.5f * dth2};
  const GlobalAcc<3> gacc{phi0, vel, g.nx, g.ny, g.nz};
  uint32_t fpar = 0;  // bit s: phase of slot s's next full completion
  bool ok = true;
  for (int u = blockIdx.x; u < mg.units && ok; u += gridDim.x) {
    const int seg = u / mg.ntiles, tile = u - seg * mg.ntiles;
    const int zs = seg * mg.seglen, ze = min(g.nz, zs + mg.seglen);
    const int x0 = (tile % mg.ncx) * TX, y0 = (tile / mg.ncx) * TY;
    if (x0 >= HX && x0 - HX + PW <= g.nx && y0 >= HY && y0 - HY + S::PH <= g.ny && x0 + S::VX0 >= 0 &&
        x0 + S::VX0 + S::VXN <= g.nx && y0 + S::VY0 >= 0 && y0 + S::VY0 + S::VH <= g.ny)
      ok = march_run<BT, S>(BoxAcc<S, false>(phis, vels, x0, y0, g.nx, g.ny), gacc, g, x0, y0, zs, ze, lane, warp, dth,
                            hdth, full, empty, fpar, phi);
    else
      ok = march_run<BT, S>(BoxAcc<S, true>(phis, vels, x0, y0, g.nx, g.ny), gacc, g, x0, y0, zs, ze, lane, warp, dth,
                            hdth, full, empty, fpar, phi);
  }
  if (!ok && lane == 0) raise_flag(flags, FLAG_WAIT_TIMEOUT);
}

}  // namespace lin
}  // namespace dcell

using namespace dcell;

// The z-march applies to dense 3-D grids with nx % 4 == 0 (16-byte rows),
// 16-byte aligned bases and planes at least one box wide.
static bool lin_march_applicable(const Geom &g, const void *phi0, const void *vel) {
  return g.nz > 1 && g.nx % 4 == 0 && g.nx >= 8 && g.ny >= 4 && ((uintptr_t)phi0 % 16) == 0 &&
         ((uintptr_t)vel % 16) == 0;
}

// Tile rows of the z-march: 8 for Euler, 16 for the midpoint backtrace (the
// faster of the two at 256^3); DCELL_LIN_TILE_ROWS (8 or 16) overrides both.
static int lin_tile_rows(bool mid) {
  if (const char *e = getenv("DCELL_LIN_TILE_ROWS")) return atoi(e) == 16 ? 16 : 8;
  return mid ? 16 : 8;
}

// Tile rows per consumer warp: 2; DCELL_LIN_ROWS_PER_WARP (1, 2 or 4)
// overrides it.
static int lin_rows_per_warp() {
  if (const char *e = getenv("DCELL_LIN_ROWS_PER_WARP")) {
    const int r = atoi(e);
    return r == 1 || r == 4 ? r : 2;
  }
  return 2;
}

// Planes per z-segment (work unit) of the march: 16; DCELL_LIN_SEGMENT
// overrides it (4 .. 256).
static int lin_segment_planes() {
  static int planes = 0;
  if (!planes) {
    planes = 16;
    if (const char *e = getenv("DCELL_LIN_SEGMENT")) planes = std::max(4, std::min(256, atoi(e)));
  }
  return planes;
}

// The march with backtrace BT; false when no tensor maps could be made.
template <int TY, int RW, int BT>
static bool launch_march_bt(const Geom &g, const float *phi0, const float *vel, float dth0, float dth1, float dth2,
                            float *phi, int *flags, cudaStream_t st) {
  using S = lin::MarchShape<TY, BT, RW>;
  static bool configured = false;
  if (!configured) {
    if (cudaFuncSetAttribute(lin::sl_lin_march_kernel<BT, TY, RW>, cudaFuncAttributeMaxDynamicSharedMemorySize, S::Smem) !=
        cudaSuccess)
      return false;
    configured = true;
  }
  CUtensorMap tm_phi, tm_vel;
  if (!make_tensor_map_3d(&tm_phi, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, phi0, (uint64_t)g.nx, (uint64_t)g.ny,
                          (uint64_t)g.nz, lin::PW, S::PH, 1, 4) ||
      !make_tensor_map_3d(&tm_vel, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, vel, 3ull * g.nx, (uint64_t)g.ny, (uint64_t)g.nz,
                          S::VW, S::VH, 1, 4))
    return false;
  lin::MarchGrid mg;
  mg.ncx = (g.nx + lin::TX - 1) / lin::TX;
  mg.ntiles = mg.ncx * ((g.ny + TY - 1) / TY);
  mg.seglen = std::min(lin_segment_planes(), g.nz);
  mg.units = mg.ntiles * ((g.nz + mg.seglen - 1) / mg.seglen);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // rounds of at most one resident wave; the grid evens the units over them
  const int slots = S::CtasPerSm * sms, rounds = (mg.units + slots - 1) / slots;
  const int grid = (mg.units + rounds - 1) / rounds;
  lin::sl_lin_march_kernel<BT, TY, RW><<<grid, S::Threads, S::Smem, st>>>(tm_phi, tm_vel, g, mg, phi0, vel, dth0,
                                                                           dth1, dth2, phi, flags);
  return true;
}

// Launches the march; false when no tensor maps could be made.
template <int TY, int RW>
static bool launch_march(const Geom &g, const float *phi0, const float *vel, float dth0, float dth1, float dth2,
                         bool mid, float *phi, int *flags, cudaStream_t st) {
  return mid ? launch_march_bt<TY, RW, DCELL_MIDPOINT>(g, phi0, vel, dth0, dth1, dth2, phi, flags, st)
             : launch_march_bt<TY, RW, DCELL_EULER>(g, phi0, vel, dth0, dth1, dth2, phi, flags, st);
}

template <int TY>
static bool launch_march_rows(const Geom &g, const float *phi0, const float *vel, float dth0, float dth1, float dth2,
                              bool mid, float *phi, int *flags, cudaStream_t st) {
  switch (lin_rows_per_warp()) {
    case 1: return launch_march<TY, 1>(g, phi0, vel, dth0, dth1, dth2, mid, phi, flags, st);
    case 4: return launch_march<TY, 4>(g, phi0, vel, dth0, dth1, dth2, mid, phi, flags, st);
    default: return launch_march<TY, 2>(g, phi0, vel, dth0, dth1, dth2, mid, phi, flags, st);
  }
}

int launch_sl_lin_f32(const Geom &g, const float *phi0, const float *vel, double dt, const int *band, long long npts,
                      int backtrace, float *phi, int *flags, cudaStream_t st, bool gather) {
  const float dth0 = (float)(dt / g.hx), dth1 = (float)(dt / g.hy), dth2 = (float)(dt / g.hz);
  const bool mid = backtrace == DCELL_MIDPOINT;
  if (!band && !gather && lin_march_applicable(g, phi0, vel)) {
    if (lin_tile_rows(mid) == 16 ? launch_march_rows<16>(g, phi0, vel, dth0, dth1, dth2, mid, phi, flags, st)
                              : launch_march_rows<8>(g, phi0, vel, dth0, dth1, dth2, mid, phi, flags, st))
      return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
    // no tensor maps (driver entry point unavailable): the gather form below
  }
  const int n = (int)npts;
  int blocks = (n + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (blocks < 1) blocks = 1;
  if (g.nz == 1) {
    if (mid) lin::sl_lin_gather_kernel<DCELL_MIDPOINT, 2><<<blocks, 256, 0, st>>>(g, phi0, vel, dth0, dth1, dth2, band, n, phi, flags);
    else lin::sl_lin_gather_kernel<DCELL_EULER, 2><<<blocks, 256, 0, st>>>(g, phi0, vel, dth0, dth1, dth2, band, n, phi, flags);
  } else {
    if (mid) lin::sl_lin_gather_kernel<DCELL_MIDPOINT, 3><<<blocks, 256, 0, st>>>(g, phi0, vel, dth0, dth1, dth2, band, n, phi, flags);
    else lin::sl_lin_gather_kernel<DCELL_EULER, 3><<<blocks, 256, 0, st>>>(g, phi0, vel, dth0, dth1, dth2, band, n, phi, flags);
  }
  return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
}
