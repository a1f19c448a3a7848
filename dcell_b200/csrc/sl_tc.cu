// Split-BF16 tensor-core tricubic semi-Lagrangian step (sm_100a, tcgen05).
//
// Per departure point the 64 Catmull-Rom coefficients are a = M s, with s the
// 4^3 stencil of phi0 around the departure cell and M the fixed 64x64
// operator of the reference's TricubicInverse.h (= C (x) C (x) C, every entry
// exact in BF16).  The kernel batches that contraction over 128 points per
// MMA:
//
//     D[128 points x 64 coefs] = A[128 x 128] * B[128 x 64]
//       A row p = [ bf16_hi(s_p - r_p) | bf16_lo(s_p - r_p) ]   (K = 64 + 64)
//       B       = [ M^T ; M^T ]                                  (BF16, exact)
//       D       = FP32 accumulator in tensor memory
//
// r_p = phi0 at the departure cell (stencil entry (1,1,1)); subtracting it
// shrinks the dynamic range before the split and is exact algebraically
// (M maps the constant stencil to the constant monomial).  hi + lo carry
// ~16 significant bits of each stencil difference.
//
// Data path per CTA (128 threads = 4 warps, thread t <-> TMEM lane t):
//   1. each thread backtraces its point (integer cell + FP32 fraction),
//      gathers its 64 stencil values, splits them and writes its A row into
//      TMEM with tcgen05.st (A is the MMA's TMEM operand, no shared-memory
//      staging of the gathered stencils);
//   2. one thread issues 8 tcgen05.mma (M=128, N=64, K=16; 4 K-steps for hi,
//      4 for lo, B from shared memory) and a tcgen05.commit to an mbarrier;
//   3. every thread waits (bounded) on the mbarrier, reads its 64
//      coefficients with tcgen05.ld, evaluates the tricubic polynomial at its
//      fraction (Horner) and adds r back.
// Several CTAs per SM (128 TMEM columns each) overlap one CTA's gathers with
// another's MMA.  Band structure and backtrace follow LevelSetAdvectSL_3D
// (LevelSetMethod/AdvectSL.c:56-89).
#include <cuda.h>
#include <cuda_bf16.h>

#include "dcell_common.cuh"
#include "dcell_kernels.h"
#include "sl_device.cuh"

namespace dcell {
namespace tc {

constexpr int kTile = 128;       // points per MMA (M)
constexpr int kCoef = 64;        // coefficients (N)
constexpr int kK = 128;          // K: stencil entry j contributes hi_j at K = 2j and lo_j at K = 2j + 1
constexpr int kTmemCols = 128;   // A: 64 columns (one packed hi|lo word per stencil entry), D: 64 columns
constexpr int kBBytes = kCoef * kK * 2;  // B: 64 rows x 128 K of bf16, B[n][2j] = B[n][2j+1] = M[n][j]
constexpr int kDynSmem = 56 * 1024;      // caps residency at 4 CTAs/SM = 512 TMEM columns
constexpr unsigned kWaitLimit = 1u << 20;  // bounded mbarrier polls (a normal MMA completes in microseconds)

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor, K-major, no swizzle: 8-row x 16-byte core
// matrices; LBO = byte stride between K-adjacent core matrices, SBO = byte
// stride between 8-row groups; version 1 (sm_100) in bits 46-47.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: D F32, A/B BF16, both K-major, N, M.
__host__ __device__ constexpr uint32_t instr_desc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// Byte offset of element (row n, k) of a K-major no-swizzle operand with K = 128.
__device__ __forceinline__ int b_offset(int n, int k) {
  return (((n >> 3) * (kK / 8) + (k >> 3)) * 128) + (n & 7) * 16 + (k & 7) * 2;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

// Bounded wait for phase `parity` of the mbarrier; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (unsigned it = 0; it < kWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t *dst_smem, int ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, int ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

#define DCELL_R8(b) "r"(v[b + 0]), "r"(v[b + 1]), "r"(v[b + 2]), "r"(v[b + 3]), "r"(v[b + 4]), "r"(v[b + 5]), \
                    "r"(v[b + 6]), "r"(v[b + 7])
// 32 consecutive 32-bit columns of this thread's lane <- v[0..31]
__device__ __forceinline__ void tmem_st32(uint32_t taddr, const uint32_t *v) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32};" ::"r"(taddr),
      DCELL_R8(0), DCELL_R8(8), DCELL_R8(16), DCELL_R8(24)
      : "memory");
}
#undef DCELL_R8

#define DCELL_W8(b) "=r"(v[b + 0]), "=r"(v[b + 1]), "=r"(v[b + 2]), "=r"(v[b + 3]), "=r"(v[b + 4]), "=r"(v[b + 5]), \
                    "=r"(v[b + 6]), "=r"(v[b + 7])
// v[0..31] <- 32 consecutive 32-bit columns of this thread's lane
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t *v) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : DCELL_W8(0), DCELL_W8(8), DCELL_W8(16), DCELL_W8(24)
      : "r"(taddr)
      : "memory");
}
#undef DCELL_W8

__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint32_t a_tmem, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d_tmem),
      "r"(a_tmem), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// Shared state and one-time set-up of a CTA: B operand, mbarrier, TMEM.
struct Ctx {
  uint32_t tmem;      // base TMEM address (lane 0, first column)
  uint32_t lane_off;  // this warp's lane quarter, in TMEM address units
  uint64_t bdesc;     // descriptor of B at K-step 0
};

__device__ __forceinline__ void setup(uint8_t *sB, uint64_t *bar, uint32_t *tmem_slot, Ctx &c) {
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int e = tid; e < kCoef * kK; e += blockDim.x) {
    const int n = e / kK, k = e % kK, j = k >> 1;  // B[n][k] = M[n][j]: coefficient n from stencil entry j
    const float w = cr_coef(n >> 4, j >> 4) * cr_coef((n >> 2) & 3, (j >> 2) & 3) * cr_coef(n & 3, j & 3);
    *reinterpret_cast<__nv_bfloat16 *>(sB + b_offset(n, k)) = __float2bfloat16_rn(w);
  }
  if (tid == 0) mbar_init(bar, 1);
  if (warp == 0) tmem_alloc(tmem_slot, kTmemCols);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  fence_before();
  __syncthreads();
  fence_after();
  c.tmem = *tmem_slot;
  c.lane_off = (uint32_t)(warp * 32) << 16;
  c.bdesc = smem_desc(smem_u32(sB), 128, (kK / 8) * 128);
}

// Packed split word of v: bf16 hi = RN_bf16(v) in the low half, bf16
// lo = RN_bf16(v - hi) in the high half (= TMEM column layout of one stencil
// entry: K = 2j low half, K = 2j + 1 high half).
__device__ __forceinline__ uint32_t pack_split(float v) {
  const __nv_bfloat16 h = __float2bfloat16_rn(v);
  const __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));
  return (uint32_t)__bfloat16_as_ushort(h) | ((uint32_t)__bfloat16_as_ushort(l) << 16);
}

// A (this lane: 64 packed words) -> TMEM, barrier, MMA by thread 0, bounded
// wait, D -> regs.  Returns false (CTA-uniformly) when the wait timed out.
__device__ __forceinline__ bool mma_tile(const Ctx &c, uint64_t *bar, uint32_t parity, const uint32_t *w,
                                         float *coef) {
  tmem_st32(c.tmem + c.lane_off + 0, w);
  tmem_st32(c.tmem + c.lane_off + 32, w + 32);
  tmem_wait_st();
  fence_before();
  __syncthreads();
  if (threadIdx.x == 0) {
    fence_after();
    constexpr uint32_t idesc = instr_desc_bf16(kTile, kCoef);
#pragma unroll
    for (int kk = 0; kk < kK / 16; ++kk) {
      const uint32_t a_tmem = c.tmem + (uint32_t)(kk * 8);          // 8 columns = 16 bf16 of K
      const uint64_t bdesc = c.bdesc + (uint64_t)((kk * 256) >> 4);  // K-step of B (2 core matrices)
      mma_bf16(c.tmem + 64, a_tmem, bdesc, idesc, kk > 0 ? 1u : 0u);
    }
    mma_commit(bar);
  }
  // only the issuing thread polls the mbarrier; the others sleep in the barrier
  const bool ok = threadIdx.x == 0 ? mbar_wait(bar, parity) : true;
  const int all_ok = __syncthreads_and(ok ? 1 : 0);
  if (!all_ok) return false;
  fence_after();
  uint32_t *u = reinterpret_cast<uint32_t *>(coef);
  tmem_ld32(c.tmem + c.lane_off + 64, u);
  tmem_ld32(c.tmem + c.lane_off + 96, u + 32);
  tmem_wait_ld();
  fence_before();
  return true;
}

__device__ __forceinline__ float horner3(const float *a, const float f[3]) {
  float pz = 0.f;
#pragma unroll
  for (int k = 3; k >= 0; --k) {
    float py = 0.f;
#pragma unroll
    for (int j = 3; j >= 0; --j) {
      const float *r = a + 4 * j + 16 * k;
      const float px = fmaf(fmaf(fmaf(r[3], f[0], r[2]), f[0], r[1]), f[0], r[0]);
      py = fmaf(py, f[1], px);
    }
    pz = fmaf(pz, f[2], py);
  }
  return pz;
}

// Per-point front half: backtrace, stencil gather, centring, hi/lo split.
// Invalid lanes contribute a zero A row.
__device__ __forceinline__ void tc_prepare(const Geom &g, const float *__restrict__ phi0,
                                           const float *__restrict__ vel, const float dth[3], int backtrace,
                                           bool valid, int x, int y, int z, float f[3], float &r, uint32_t *w,
                                           bool &clamped) {
  if (valid) {
    int cc[3];
    float s[64];
    clamped |= departure_cell<float, 3>(g, vel, dth, backtrace, x, y, z, cc, f);
    gather_stencil<float, 3>(g, phi0, cc, s);
    r = s[21];
#pragma unroll
    for (int e = 0; e < 64; ++e) w[e] = pack_split(s[e] - r);
  } else {
#pragma unroll
    for (int e = 0; e < 64; ++e) w[e] = 0u;
  }
}

__global__ void __launch_bounds__(kTile, 4) sl_tc_kernel(Geom g, const float *__restrict__ phi0,
                                                         const float *__restrict__ vel, float dt,
                                                         const int *__restrict__ band, long long npts, int backtrace,
                                                         float *__restrict__ phi, int *flags) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t *sB = smem;
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + kBBytes);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + kBBytes + 8);
  Ctx c;
  setup(sB, bar, tmem_slot, c);

  const float dth[3] = {dt / (float)g.hx, dt / (float)g.hy, dt / (float)g.hz};
  const long long ntiles = (npts + kTile - 1) / kTile;
  uint32_t parity = 0;
  bool clamped = false, timeout = false, bad = false;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long q = tile * kTile + threadIdx.x;
    int x = 0, y = 0, z = 0;
    bool valid = q < npts;
    if (valid && !arrival_local(g, band, q, x, y, z)) {
      valid = false;
      bad = true;
    }
    float f[3] = {0.f, 0.f, 0.f}, r = 0.f;
    uint32_t w[64];
    tc_prepare(g, phi0, vel, dth, backtrace, valid, x, y, z, f, r, w, clamped);
    float a[64];
    if (!mma_tile(c, bar, parity, w, a)) {
      timeout = true;
      break;
    }
    parity ^= 1u;
    if (valid) phi[(z * g.ny + y) * g.nx + x] = horner3(a, f) + r;
  }
  if (clamped && band) raise_flag(flags, FLAG_DEPARTURE_CLAMPED);  // dense grids: the edge is the domain boundary
  if (bad) raise_flag(flags, FLAG_BAD_BAND);
  if (timeout && threadIdx.x == 0) raise_flag(flags, FLAG_WAIT_TIMEOUT);
  fence_before();
  __syncthreads();
  fence_after();
  if ((threadIdx.x >> 5) == 0) tmem_dealloc(c.tmem, kTmemCols);
}

// ---------------------------------------------------------------------------
// Split-state variant.  The level set is carried as FP32 *and* as its packed
// BF16 split (one 32-bit word per point: hi = RN_bf16(phi) in the low half,
// lo = RN_bf16(phi - hi) in the high half), written by the step that produces
// phi.  A step then gathers the 64 packed words of each stencil and forms the
// A row's TMEM columns with one byte-permute per column -- no per-entry
// subtraction or conversion: with the interleaved K order the gathered words
// are the A row.  M (hi + lo) = M phi to ~2^-17 relative.
__global__ void __launch_bounds__(256) split_kernel(const float *__restrict__ phi, uint32_t *__restrict__ out,
                                                    long long n) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    out[q] = pack_split(phi[q]);
}

__device__ __forceinline__ void tc_prepare_split(const Geom &g, const uint32_t *__restrict__ words,
                                                 const float *__restrict__ vel, const float dth[3], int backtrace,
                                                 bool valid, int x, int y, int z, float f[3], uint32_t *w,
                                                 bool &clamped) {
  if (valid) {
    int cc[3];
    clamped |= departure_cell<float, 3>(g, vel, dth, backtrace, x, y, z, cc, f);
    gather_stencil<uint32_t, 3>(g, words, cc, w);  // the packed words are the A row as they stand
  } else {
#pragma unroll
    for (int e = 0; e < 64; ++e) w[e] = 0u;
  }
}

__global__ void __launch_bounds__(kTile, 4) sl_tc_split_kernel(Geom g, const uint32_t *__restrict__ phi0s,
                                                               const float *__restrict__ vel, float dt,
                                                               const int *__restrict__ band, long long npts,
                                                               int backtrace, float *__restrict__ phi,
                                                               uint32_t *__restrict__ phis, int *flags) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t *sB = smem;
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + kBBytes);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + kBBytes + 8);
  Ctx c;
  setup(sB, bar, tmem_slot, c);

  const float dth[3] = {dt / (float)g.hx, dt / (float)g.hy, dt / (float)g.hz};
  const long long ntiles = (npts + kTile - 1) / kTile;
  uint32_t parity = 0;
  bool clamped = false, timeout = false, bad = false;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long q = tile * kTile + threadIdx.x;
    int x = 0, y = 0, z = 0;
    bool valid = q < npts;
    if (valid && !arrival_local(g, band, q, x, y, z)) {
      valid = false;
      bad = true;
    }
    float f[3] = {0.f, 0.f, 0.f};
    uint32_t w[64];
    tc_prepare_split(g, phi0s, vel, dth, backtrace, valid, x, y, z, f, w, clamped);
    float a[64];
    if (!mma_tile(c, bar, parity, w, a)) {
      timeout = true;
      break;
    }
    parity ^= 1u;
    if (valid) {
      const int p = (z * g.ny + y) * g.nx + x;
      const float v = horner3(a, f);
      phi[p] = v;
      if (phis) phis[p] = pack_split(v);
    }
  }
  if (clamped && band) raise_flag(flags, FLAG_DEPARTURE_CLAMPED);  // dense grids: the edge is the domain boundary
  if (bad) raise_flag(flags, FLAG_BAD_BAND);
  if (timeout && threadIdx.x == 0) raise_flag(flags, FLAG_WAIT_TIMEOUT);
  fence_before();
  __syncthreads();
  fence_after();
  if ((threadIdx.x >> 5) == 0) tmem_dealloc(c.tmem, kTmemCols);
}

// ---------------------------------------------------------------------------
// TMA-staged brick variant of the split-state step (dense grids, nx % 4 == 0).
//
// A CTA walks bricks of 32 x 2 x 4 arrival points (two 128-point MMA tiles).
// For each brick, thread 0 issues two tiled TMA loads into shared memory --
// the phi-split words of the box [x0-4, x0+36) x [y0-2, y0+4) x [z0-2, z0+6)
// and the interleaved velocity of [x0-4, x0+36) x [y0-1, y0+3) x [z0-1, z0+5)
// -- one brick ahead, double-buffered, completion tracked by an mbarrier's
// transaction count.  Gathers then read shared memory with 32-bit offsets.
// Out-of-grid parts of a box are zero-filled by TMA but never read: indices
// are clamped to the grid before they are made box-local.  Points whose
// departure (or midpoint) leaves the box -- per-component CFL >= 1 -- take
// the global-memory path.  TMA x coordinates are multiples of 4 elements
// (16-byte rule); nothing starts a store at a negative coordinate.
constexpr int kBX = 32, kBY = 2, kBZ = 4;               // brick = 256 points = 2 MMA tiles
constexpr int kPX = kBX + 8, kPY = kBY + 4, kPZ = kBZ + 4;  // phi box (halo 4 | 2 | 2)
constexpr int kVX = kBX + 8, kVY = kBY + 2, kVZ = kBZ + 2;  // velocity box (halo 4 | 1 | 1)
constexpr int kPhiBoxBytes = kPX * kPY * kPZ * 4;
constexpr int kVelBoxBytes = 3 * kVX * kVY * kVZ * 4;
constexpr int kBufBytes = kPhiBoxBytes + kVelBoxBytes;
constexpr int kBrickSmem = kBBytes + 2 * kBufBytes + 64;
static_assert(kBrickSmem <= kDynSmem, "brick buffers exceed the CTA's shared memory budget");
static_assert(kPhiBoxBytes % 128 == 0 && kBufBytes % 128 == 0, "TMA destinations must stay 128-byte aligned");

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *tm, int c0, int c1, int c2,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}

struct BrickGrid {
  int nbx, nby, nbz;
};

// Bricks are numbered z fastest, x slowest: a persistent CTA striding by the
// grid size then visits every x position (the x faces, where boxes need edge
// replication, are shared out evenly), and the bricks in flight at one time
// are z/y neighbours that share halo rows in L2.
__device__ __forceinline__ void brick_origin(const BrickGrid &bg, int b, int &x0, int &y0, int &z0) {
  const int bz = b % bg.nbz, r = b / bg.nbz;
  z0 = bz * kBZ;
  y0 = (r % bg.nby) * kBY;
  x0 = (r / bg.nby) * kBX;
}

// thread 0: both boxes of brick b into buffer `buf` (whose previous contents
// every thread has finished reading: order those generic-proxy reads before
// the async-proxy writes)
__device__ __forceinline__ void issue_brick(const BrickGrid &bg, int b, uint8_t *buf, const CUtensorMap *tm_phi,
                                            const CUtensorMap *tm_vel, uint64_t *bar) {
  int x0, y0, z0;
  brick_origin(bg, b, x0, y0, z0);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  mbar_expect_tx(bar, (uint32_t)kBufBytes);
  tma_load_3d(buf, tm_phi, x0 - 4, y0 - 2, z0 - 2, bar);
  tma_load_3d(buf + kPhiBoxBytes, tm_vel, 3 * (x0 - 4), y0 - 1, z0 - 1, bar);
}

// Edge replication of a staged box.  TMA zero-fills the parts of a box that
// lie outside the grid; afterwards each of them holds the value of the
// nearest in-grid cell along each axis -- exactly what the reference's
// clamped interpolation indices read (Common/InterpolateVelocity.c and
// Common/LevelSetMethod.c clamp i, j, k to the grid independently).  A
// box-local read at an unclamped index then equals a global read at the
// clamped index, so the per-point code needs no clamping.  Passes run x, y, z,
// each reading what the one before wrote, which replicates edges and corners
// like per-axis clamping.  The box is [DZ][DY][DX][C] 32-bit words whose cell
// (0,0,0) sits at grid point (gx0, gy0, gz0); in-grid cells of each axis are a
// non-empty range because the brick's own points are in the grid.  Only
// CTA-uniform branches; every thread takes part.
template <int DX, int DY, int DZ, int C>
__device__ __forceinline__ void replicate_box_edges(uint32_t *box, int gx0, int gy0, int gz0, int nx, int ny,
                                                    int nz) {
  const int xl = min(max(-gx0, 0), DX), xh = min(max(nx - gx0, 0), DX);  // in-grid columns [xl, xh)
  const int yl = min(max(-gy0, 0), DY), yh = min(max(ny - gy0, 0), DY);
  const int zl = min(max(-gz0, 0), DZ), zh = min(max(nz - gz0, 0), DZ);
  const int ox = xl + (DX - xh), oy = yl + (DY - yh), oz = zl + (DZ - zh);  // out-of-grid counts
  if (ox) {
    const int total = ox * DY * DZ * C;
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
      const int k = i % C, r = i / C, j = r % ox, row = r / ox;
      const int col = j < xl ? j : xh + (j - xl), src = j < xl ? xl : xh - 1;
      box[(row * DX + col) * C + k] = box[(row * DX + src) * C + k];
    }
    __syncthreads();
  }
  if (oy) {
    constexpr int W = DX * C;
    const int total = oy * DZ * W;
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
      const int w = i % W, r = i / W, j = r % oy, plane = r / oy;
      const int row = j < yl ? j : yh + (j - yl), src = j < yl ? yl : yh - 1;
      box[(plane * DY + row) * W + w] = box[(plane * DY + src) * W + w];
    }
    __syncthreads();
  }
  if (oz) {
    constexpr int P = DY * DX * C;
    const int total = oz * P;
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
      const int w = i % P, j = i / P;
      const int plane = j < zl ? j : zh + (j - zl), src = j < zl ? zl : zh - 1;
      box[plane * P + w] = box[src * P + w];
    }
  }
  if (ox | oy | oz) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // before TMA refills the buffer
}

// Front half of one point from the staged, edge-replicated boxes: node
// velocity, midpoint velocity, departure cell and fraction, and the box offset
// of the stencil's first word.  (vx, vy, vz) is the point's cell in the
// velocity box, (px, py, pz) in the phi box.  Returns false when the midpoint
// or the stencil leaves the box (per-component CFL >= 1): the warp then takes
// the global path.  The arithmetic is the clamped global path's, operation for
// operation (explicit roundings), so both give the same bits.
__device__ __forceinline__ bool brick_depart(const float *__restrict__ vbox, int vx, int vy, int vz, int px, int py,
                                             int pz, const float dth[3], int backtrace, float f[3], int &soff) {
  constexpr int SX = 3, SY = 3 * kVX, SZ = 3 * kVX * kVY;
  const float *vb = vbox + (vz * kVY + vy) * (3 * kVX) + 3 * vx;
  float U[3] = {face_mean(vb[0], vb[SX]), face_mean(vb[1], vb[SY + 1]), face_mean(vb[2], vb[SZ + 2])};
  if (backtrace == DCELL_MIDPOINT) {
    const float dl[3] = {rmul(rmul(-0.5f, U[0]), dth[0]), rmul(rmul(-0.5f, U[1]), dth[1]),
                         rmul(rmul(-0.5f, U[2]), dth[2])};
    if (fabsf(dl[0]) >= 0.5f || fabsf(dl[1]) >= 0.5f || fabsf(dl[2]) >= 0.5f) return false;
    // Along a component's own (staggered) axis the midpoint lies in [X, X+1):
    // floor 0, fraction t.  Across the other two axes the node-centred
    // fraction and floor are shared by both components.
    float sn[3], sp[3];
    int on[3];
    constexpr int S[3] = {SX, SY, SZ};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float t = dl[a] + 0.f;
      const float fl = floorf(t);
      sn[a] = t - fl;
      on[a] = (int)fl * S[a];
      sp[a] = dl[a] + 0.5f;
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const float s3[3] = {d == 0 ? sp[0] : sn[0], d == 1 ? sp[1] : sn[1], d == 2 ? sp[2] : sn[2]};
      const float *q = vb + d + (d == 0 ? 0 : on[0]) + (d == 1 ? 0 : on[1]) + (d == 2 ? 0 : on[2]);
      U[d] = trilerp(q[0], q[SX], q[SY], q[SY + SX], q[SZ], q[SZ + SX], q[SZ + SY], q[SZ + SY + SX], s3);
    }
  }
  int cl[3];
  const int P[3] = {px, py, pz};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float t = rmul(-U[a], dth[a]);
    const float fl = floorf(t);
    cl[a] = P[a] + (int)fl - 1;  // first stencil cell, box-local
    f[a] = t - fl;
  }
  soff = (cl[2] * kPY + cl[1]) * kPX + cl[0];
  return (unsigned)cl[0] <= (unsigned)(kPX - 4) && (unsigned)cl[1] <= (unsigned)(kPY - 4) &&
         (unsigned)cl[2] <= (unsigned)(kPZ - 4);
}

__global__ void __launch_bounds__(kTile, 4) sl_tc_brick_kernel(const __grid_constant__ CUtensorMap tm_phi,
                                                               const __grid_constant__ CUtensorMap tm_vel, Geom g,
                                                               BrickGrid bg, const uint32_t *__restrict__ phi0s,
                                                               const float *__restrict__ vel, float dt,
                                                               int backtrace, float *__restrict__ phi,
                                                               uint32_t *__restrict__ phis, int *flags) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t *sB = smem;
  uint8_t *const buf0 = smem + kBBytes, *const buf1 = smem + kBBytes + kBufBytes;
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + kBBytes + 2 * kBufBytes);
  uint64_t *tbar = bar + 1;  // two TMA barriers
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bar + 3);
  if (threadIdx.x == 0) {
    mbar_init(&tbar[0], 1);
    mbar_init(&tbar[1], 1);
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tm_phi)) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tm_vel)) : "memory");
  }
  Ctx c;
  setup(sB, bar, tmem_slot, c);  // B operand, MMA barrier, TMEM; ends with a CTA barrier

  const float dth[3] = {dt / (float)g.hx, dt / (float)g.hy, dt / (float)g.hz};
  const int nbricks = bg.nbx * bg.nby * bg.nbz;
  const int lx = threadIdx.x & (kBX - 1), ly = (threadIdx.x >> 5) & 1, lzt = threadIdx.x >> 6;  // tile: 32x2x2
  uint32_t parity = 0;
  uint32_t uses0 = 0u, uses1 = 0u;  // completed phases per TMA buffer
  bool pending0 = false, pending1 = false;
  bool timeout = false;
  int it = 0;
  if (threadIdx.x == 0 && (int)blockIdx.x < nbricks) issue_brick(bg, blockIdx.x, buf0, &tm_phi, &tm_vel, &tbar[0]);
  pending0 = (int)blockIdx.x < nbricks;
  for (int b = blockIdx.x; b < nbricks; b += gridDim.x, ++it) {
    const bool odd = it & 1;
    uint8_t *const cbuf = odd ? buf1 : buf0;
    const int nb = b + gridDim.x;
    if (threadIdx.x == 0 && nb < nbricks)
      issue_brick(bg, nb, odd ? buf0 : buf1, &tm_phi, &tm_vel, odd ? &tbar[0] : &tbar[1]);
    if (odd) pending0 = nb < nbricks; else pending1 = nb < nbricks;
    const bool ok = mbar_wait(odd ? &tbar[1] : &tbar[0], (odd ? uses1 : uses0) & 1u);
    if (!__syncthreads_and(ok ? 1 : 0)) {
      timeout = true;
      break;
    }
    if (odd) { pending1 = false; ++uses1; } else { pending0 = false; ++uses0; }
    int x0, y0, z0;
    brick_origin(bg, b, x0, y0, z0);
    uint32_t *pbox = reinterpret_cast<uint32_t *>(cbuf);
    const float *vbox = reinterpret_cast<const float *>(cbuf + kPhiBoxBytes);
    if (x0 < 4 || x0 + kPX - 4 > g.nx || y0 < 2 || y0 + kPY - 2 > g.ny || z0 < 2 || z0 + kPZ - 2 > g.nz) {
      replicate_box_edges<kPX, kPY, kPZ, 1>(pbox, x0 - 4, y0 - 2, z0 - 2, g.nx, g.ny, g.nz);
      replicate_box_edges<kVX, kVY, kVZ, 3>(reinterpret_cast<uint32_t *>(cbuf + kPhiBoxBytes), x0 - 4, y0 - 1,
                                            z0 - 1, g.nx, g.ny, g.nz);
      __syncthreads();
    }
#pragma unroll 1
    for (int t = 0; t < 2; ++t) {
      // lanes past the grid's end (partial bricks) compute a copy of the last
      // in-grid point and store nothing
      const int xr = x0 + lx, yr = y0 + ly, zr = z0 + 2 * t + lzt;
      const bool valid = xr < g.nx && yr < g.ny && zr < g.nz;
      const int x = min(xr, g.nx - 1), y = min(yr, g.ny - 1), z = min(zr, g.nz - 1);
      float f[3];
      uint32_t w[64];
      int soff;
      const bool inbox = brick_depart(vbox, x - x0 + 4, y - y0 + 1, z - z0 + 1, x - x0 + 4, y - y0 + 2, z - z0 + 2,
                                      dth, backtrace, f, soff);
      if (__all_sync(0xffffffffu, inbox)) {
        const uint32_t *q = pbox + soff;
#pragma unroll
        for (int zz = 0; zz < 4; ++zz)
#pragma unroll
          for (int yy = 0; yy < 4; ++yy)
#pragma unroll
            for (int xx = 0; xx < 4; ++xx) w[xx + 4 * yy + 16 * zz] = q[(zz * kPY + yy) * kPX + xx];
      } else {  // the whole warp recomputes from global memory with clamped indices
        bool clamped = false;
        tc_prepare_split(g, phi0s, vel, dth, backtrace, true, x, y, z, f, w, clamped);
      }
      float a[64];
      if (!mma_tile(c, bar, parity, w, a)) {
        timeout = true;
        break;
      }
      parity ^= 1u;
      if (valid) {
        const int p = (z * g.ny + y) * g.nx + x;
        const float v = horner3(a, f);
        phi[p] = v;
        if (phis) phis[p] = pack_split(v);
      }
    }
    if (timeout) break;
    __syncthreads();  // everyone is done with buf[cur] before it is refilled
  }
  if (timeout && threadIdx.x == 0) {
    raise_flag(flags, FLAG_WAIT_TIMEOUT);
    // let every TMA still in flight land before the CTA's shared memory goes away (bounded waits)
    if (pending0) mbar_wait(&tbar[0], uses0 & 1u);
    if (pending1) mbar_wait(&tbar[1], uses1 & 1u);
  }
  fence_before();
  __syncthreads();
  fence_after();
  if ((threadIdx.x >> 5) == 0) tmem_dealloc(c.tmem, kTmemCols);
}

// Batched cells: a persistent CTA walks a packed queue of 128-point tiles
// (tx x ty x tz boxes of one cell's grid) over many uneven cell grids.
__global__ void __launch_bounds__(kTile, 4) batch_tc_kernel(const dcell_cell *__restrict__ cells,
                                                            const dcell_tile *__restrict__ tiles, int ntiles, int tx,
                                                            int ty, const float *__restrict__ phi0,
                                                            const float *__restrict__ vel, int backtrace,
                                                            float *__restrict__ phi, int *flags) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t *sB = smem;
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + kBBytes);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + kBBytes + 8);
  Ctx c;
  setup(sB, bar, tmem_slot, c);
  const int lx = threadIdx.x % tx, ly = (threadIdx.x / tx) % ty, lz = threadIdx.x / (tx * ty);
  uint32_t parity = 0;
  bool clamped = false, timeout = false;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const dcell_tile T = tiles[t];
    const dcell_cell C = cells[T.cell];
    Geom g;
    g.nx = C.n[0]; g.ny = C.n[1]; g.nz = C.n[2];
    g.px = g.py = g.pz = 0;
    g.hx = C.h[0]; g.hy = C.h[1]; g.hz = C.h[2];
    const float dtf = (float)C.dt;  // same rounding as the single-grid kernels
    const float dth[3] = {dtf / (float)C.h[0], dtf / (float)C.h[1], dtf / (float)C.h[2]};
    const int x = T.x0 + lx, y = T.y0 + ly, z = T.z0 + lz;
    const bool valid = x < g.nx && y < g.ny && z < g.nz;
    float f[3] = {0.f, 0.f, 0.f}, r = 0.f;
    uint32_t w[64];
    tc_prepare(g, phi0 + C.offset, vel + 3 * C.offset, dth, backtrace, valid, x, y, z, f, r, w, clamped);
    float a[64];
    if (!mma_tile(c, bar, parity, w, a)) {
      timeout = true;
      break;
    }
    parity ^= 1u;
    if (valid) phi[C.offset + (z * g.ny + y) * g.nx + x] = horner3(a, f) + r;
  }
  (void)clamped;  // dense cells: the grid edge is the cell's domain boundary
  if (timeout && threadIdx.x == 0) raise_flag(flags, FLAG_WAIT_TIMEOUT);
  fence_before();
  __syncthreads();
  fence_after();
  if ((threadIdx.x >> 5) == 0) tmem_dealloc(c.tmem, kTmemCols);
}

// D = bf16(A) * M^T on the same tensor-core path (hi half only): a check of
// the operand layouts against a host GEMM.  A: 128 x 64 row-major, D: 128 x 64.
__global__ void __launch_bounds__(kTile, 1) tc_gemm_check_kernel(const float *__restrict__ A, float *__restrict__ D,
                                                                 int *flags) {
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t *sB = smem;
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + kBBytes);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + kBBytes + 8);
  Ctx c;
  setup(sB, bar, tmem_slot, c);
  uint32_t w[64];
  for (int e = 0; e < 64; ++e)  // hi only (lo half zero): D = bf16(A) M^T
    w[e] = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(A[threadIdx.x * 64 + e]));
  float a[64];
  if (mma_tile(c, bar, 0, w, a)) {
    for (int e = 0; e < 64; ++e) D[threadIdx.x * 64 + e] = a[e];
  } else if (threadIdx.x == 0) {
    raise_flag(flags, FLAG_WAIT_TIMEOUT);
  }
  fence_before();
  __syncthreads();
  fence_after();
  if ((threadIdx.x >> 5) == 0) tmem_dealloc(c.tmem, kTmemCols);
}

}  // namespace tc
}  // namespace dcell

using namespace dcell;

static int tc_grid(long long npts) {
  static int num_sms = 0;
  if (!num_sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (num_sms <= 0) num_sms = 148;
  }
  const long long ntiles = (npts + tc::kTile - 1) / tc::kTile;
  long long grid = 4LL * num_sms;
  if (grid > ntiles) grid = ntiles;
  return (int)(grid < 1 ? 1 : grid);
}

int launch_sl_tc(const Geom &g, const float *phi0, const float *vel, double dt, const int *band, long long npts,
                 int backtrace, float *phi, int *flags, cudaStream_t st) {
  static bool configured = false;
  if (!configured) {
    DCELL_CUDA_CHECK(
        cudaFuncSetAttribute(tc::sl_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kDynSmem));
    DCELL_CUDA_CHECK(
        cudaFuncSetAttribute(tc::tc_gemm_check_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kDynSmem));
    configured = true;
  }
  if (npts <= 0) return DCELL_OK;
  tc::sl_tc_kernel<<<tc_grid(npts), tc::kTile, tc::kDynSmem, st>>>(g, phi0, vel, (float)dt, band, npts, backtrace,
                                                                   phi, flags);
  return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
}

int launch_batch_tc(const dcell_cell *cells, const dcell_tile *tiles, int ntiles, int tx, int ty, int ctas_per_sm,
                    const float *phi0, const float *vel, int backtrace, float *phi, int *flags, cudaStream_t st) {
  static bool configured = false;
  if (!configured) {
    DCELL_CUDA_CHECK(
        cudaFuncSetAttribute(tc::batch_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kDynSmem));
    configured = true;
  }
  if (ntiles <= 0) return DCELL_OK;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int per = ctas_per_sm < 1 ? 1 : (ctas_per_sm > 4 ? 4 : ctas_per_sm);
  const int grid = per * sms < ntiles ? per * sms : ntiles;
  tc::batch_tc_kernel<<<grid, tc::kTile, tc::kDynSmem, st>>>(cells, tiles, ntiles, tx, ty, phi0, vel, backtrace, phi,
                                                            flags);
  return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
}

int launch_split_bf16(const float *phi, uint32_t *out, long long n, cudaStream_t st) {
  long long blocks = (n + 255) / 256;
  if (blocks > 148LL * 32) blocks = 148LL * 32;
  if (n > 0) tc::split_kernel<<<(int)(blocks < 1 ? 1 : blocks), 256, 0, st>>>(phi, out, n);
  return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
}

bool tc_brick_applicable(const Geom &g, const void *phi0s, const void *vel);
int launch_sl_tc_brick(const Geom &g, const uint32_t *phi0s, const float *vel, double dt, int backtrace, float *phi,
                       uint32_t *phis, int *flags, cudaStream_t st);

int launch_sl_tc_split(const Geom &g, const uint32_t *phi0s, const float *vel, double dt, const int *band,
                       long long npts, int backtrace, float *phi, uint32_t *phis, int *flags, cudaStream_t st) {
  if (!band && tc_brick_applicable(g, phi0s, vel))
    return launch_sl_tc_brick(g, phi0s, vel, dt, backtrace, phi, phis, flags, st);
  static bool configured = false;
  if (!configured) {
    DCELL_CUDA_CHECK(
        cudaFuncSetAttribute(tc::sl_tc_split_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kDynSmem));
    configured = true;
  }
  if (npts <= 0) return DCELL_OK;
  tc::sl_tc_split_kernel<<<tc_grid(npts), tc::kTile, tc::kDynSmem, st>>>(g, phi0s, vel, (float)dt, band, npts,
                                                                         backtrace, phi, phis, flags);
  return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
    cudaGetLastError();
  }
  return fn;
}

// 3-D tiled map over a row-major array (x fastest) of `elem` bytes per value.
static bool make_map(CUtensorMap *m, CUtensorMapDataType type, const void *base, uint64_t dx, uint64_t dy,
                     uint64_t dz, uint32_t bx, uint32_t by, uint32_t bz, uint32_t elem) {
  EncodeTiledFn fn = encode_tiled();
  if (!fn) return false;
  const cuuint64_t dims[3] = {dx, dy, dz};
  const cuuint64_t strides[2] = {dx * elem, dx * dy * elem};
  const cuuint32_t box[3] = {bx, by, bz};
  const cuuint32_t es[3] = {1, 1, 1};
  return fn(m, type, 3, const_cast<void *>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The TMA brick path applies to dense 3D grids with nx % 4 == 0 (16-byte row strides) and 16-byte aligned bases.
bool tc_brick_applicable(const Geom &g, const void *phi0s, const void *vel) {
  return g.nz >= tc::kPZ && g.ny >= tc::kPY && g.nx >= tc::kPX && g.nx % 4 == 0 && ((uintptr_t)phi0s % 16) == 0 &&
         ((uintptr_t)vel % 16) == 0 && encode_tiled() != nullptr;
}

int launch_sl_tc_brick(const Geom &g, const uint32_t *phi0s, const float *vel, double dt, int backtrace, float *phi,
                       uint32_t *phis, int *flags, cudaStream_t st) {
  static bool configured = false;
  if (!configured) {
    DCELL_CUDA_CHECK(
        cudaFuncSetAttribute(tc::sl_tc_brick_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kDynSmem));
    configured = true;
  }
  CUtensorMap tm_phi, tm_vel;
  if (!make_map(&tm_phi, CU_TENSOR_MAP_DATA_TYPE_UINT32, phi0s, (uint64_t)g.nx, (uint64_t)g.ny, (uint64_t)g.nz,
                tc::kPX, tc::kPY, tc::kPZ, 4) ||
      !make_map(&tm_vel, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, vel, 3ull * g.nx, (uint64_t)g.ny, (uint64_t)g.nz,
                3 * tc::kVX, tc::kVY, tc::kVZ, 4)) {
    dcell_set_error(DCELL_ERR_CUDA, "cuTensorMapEncodeTiled failed for the TMA brick path");
    return DCELL_ERR_CUDA;
  }
  tc::BrickGrid bg;
  bg.nbx = (g.nx + tc::kBX - 1) / tc::kBX;
  bg.nby = (g.ny + tc::kBY - 1) / tc::kBY;
  bg.nbz = (g.nz + tc::kBZ - 1) / tc::kBZ;
  const long long nbricks = (long long)bg.nbx * bg.nby * bg.nbz;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  long long grid = 4LL * sms;
  if (grid > nbricks) grid = nbricks;
  tc::sl_tc_brick_kernel<<<(int)grid, tc::kTile, tc::kDynSmem, st>>>(tm_phi, tm_vel, g, bg, phi0s, vel, (float)dt,
                                                                       backtrace, phi, phis, flags);
  return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
}

int launch_tc_gemm_check(const float *A, float *D, int *flags, cudaStream_t st) {
  DCELL_CUDA_CHECK(
      cudaFuncSetAttribute(tc::tc_gemm_check_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kDynSmem));
  tc::tc_gemm_check_kernel<<<1, tc::kTile, tc::kDynSmem, st>>>(A, D, flags);
  return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
}
