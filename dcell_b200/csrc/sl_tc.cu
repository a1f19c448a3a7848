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
#include <cstdlib>
#include <cuda.h>
#include <cuda_bf16.h>

#include "dcell_common.cuh"
#include "dcell_tma.cuh"
#include "brick_stage.cuh"
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
// 16 consecutive 32-bit columns of this thread's lane <- v[0..15]
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t *v) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16};" ::"r"(taddr),
      DCELL_R8(0), DCELL_R8(8)
      : "memory");
}
#undef DCELL_R8

#define DCELL_F8(b) "=f"(v[b + 0]), "=f"(v[b + 1]), "=f"(v[b + 2]), "=f"(v[b + 3]), "=f"(v[b + 4]), "=f"(v[b + 5]), \
                    "=f"(v[b + 6]), "=f"(v[b + 7])
// FP32 coefficients v[0..31] <- 32 consecutive columns of this thread's lane,
// written straight into the float registers that a tied tcgen05.wait::ld
// (tmem_wait_ld_tied) then completes: no copy of them sits between the load
// and its wait
__device__ __forceinline__ void tmem_ld32f(uint32_t taddr, float *v) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : DCELL_F8(0), DCELL_F8(8), DCELL_F8(16), DCELL_F8(24)
      : "r"(taddr)
      : "memory");
}
#undef DCELL_F8

// wait::ld that also ties the 64 registers it completes (a[0..32), b[0..32))
// to the wait, so that no use of them is scheduled before it
__device__ __forceinline__ void tmem_wait_ld_tied(float *a, float *b) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               :
                 "+f"(a[0]), "+f"(a[1]), "+f"(a[2]), "+f"(a[3]), "+f"(a[4]), "+f"(a[5]), "+f"(a[6]), "+f"(a[7]),
                 "+f"(a[8]), "+f"(a[9]), "+f"(a[10]), "+f"(a[11]), "+f"(a[12]), "+f"(a[13]), "+f"(a[14]), "+f"(a[15]),
                 "+f"(a[16]), "+f"(a[17]), "+f"(a[18]), "+f"(a[19]), "+f"(a[20]), "+f"(a[21]), "+f"(a[22]), "+f"(a[23]),
                 "+f"(a[24]), "+f"(a[25]), "+f"(a[26]), "+f"(a[27]), "+f"(a[28]), "+f"(a[29]), "+f"(a[30]), "+f"(a[31]),
                 "+f"(b[0]), "+f"(b[1]), "+f"(b[2]), "+f"(b[3]), "+f"(b[4]), "+f"(b[5]), "+f"(b[6]), "+f"(b[7]),
                 "+f"(b[8]), "+f"(b[9]), "+f"(b[10]), "+f"(b[11]), "+f"(b[12]), "+f"(b[13]), "+f"(b[14]), "+f"(b[15]),
                 "+f"(b[16]), "+f"(b[17]), "+f"(b[18]), "+f"(b[19]), "+f"(b[20]), "+f"(b[21]), "+f"(b[22]), "+f"(b[23]),
                 "+f"(b[24]), "+f"(b[25]), "+f"(b[26]), "+f"(b[27]), "+f"(b[28]), "+f"(b[29]), "+f"(b[30]), "+f"(b[31])
               :
               : "memory");
}

__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

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

__device__ __forceinline__ void setup(uint8_t *sB, uint64_t *bar, uint32_t *tmem_slot, Ctx &c,
                                      int tmem_cols = kTmemCols) {
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int e = tid; e < kCoef * kK; e += blockDim.x) {
    const int n = e / kK, k = e % kK, j = k >> 1;  // B[n][k] = M[n][j]: coefficient n from stencil entry j
    const float w = cr_coef(n >> 4, j >> 4) * cr_coef((n >> 2) & 3, (j >> 2) & 3) * cr_coef(n & 3, j & 3);
    *reinterpret_cast<__nv_bfloat16 *>(sB + b_offset(n, k)) = __float2bfloat16_rn(w);
  }
  if (tid == 0) mbar_init(bar, 1);
  if (warp == 0) tmem_alloc(tmem_slot, tmem_cols);
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
  const float r = v - __bfloat162float(h);
  uint32_t w;  // one paired conversion: RN_bf16(r) to the high half, RN_bf16(v) = h to the low half
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(w) : "f"(r), "f"(v));
  return w;
}

// A (this lane: 64 packed words) -> TMEM, barrier, MMA by thread 0 with its
// completion signalled on `bar`.  Every thread of the CTA takes part.
__device__ __forceinline__ void mma_issue(const Ctx &c, uint64_t *bar, const uint32_t *w) {
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
}

// Bounded wait for the MMA issued last, then D -> regs.  Only the issuing
// thread polls the mbarrier; the others sleep in the barrier.  Returns false
// (CTA-uniformly) when the wait timed out.
__device__ __forceinline__ bool mma_finish(const Ctx &c, uint64_t *bar, uint32_t parity, float *coef) {
  const bool ok = threadIdx.x == 0 ? mbar_wait(bar, parity) : true;
  const int all_ok = __syncthreads_and(ok ? 1 : 0);
  if (!all_ok) return false;
  fence_after();
  tmem_ld32f(c.tmem + c.lane_off + 64, coef);
  tmem_ld32f(c.tmem + c.lane_off + 96, coef + 32);
  tmem_wait_ld_tied(coef, coef + 32);
  fence_before();
  return true;
}

__device__ __forceinline__ bool mma_tile(const Ctx &c, uint64_t *bar, uint32_t parity, const uint32_t *w,
                                         float *coef) {
  mma_issue(c, bar, w);
  return mma_finish(c, bar, parity, coef);
}

// One z-slice of horner3: the y/x polynomial of coefficients r[4j + i].
__device__ __forceinline__ float horner_slice(const float *r, const float f[3]) {
  float py = 0.f;
#pragma unroll
  for (int j = 3; j >= 0; --j) {
    const float *q = r + 4 * j;
    const float px = fmaf(fmaf(fmaf(q[3], f[0], q[2]), f[0], q[1]), f[0], q[0]);
    py = fmaf(py, f[1], px);
  }
  return py;
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
// TMA-staged brick variant of the split-state step (dense grids, nx % 4 == 0):
// bricks and boxes of brick_stage.cuh, the phi box holding split words,
// double-buffered; P TMEM stages of A | D per CTA.
template <int P>
struct BrickShape : BrickBox<P> {
  using Box = BrickBox<P>;
  static constexpr int TmemCols = 128 * P;                    // P stages of A | D
  static constexpr int CtasPerSm = 512 / TmemCols;
  static constexpr int Smem = kBBytes + 2 * Box::BufBytes + 64;  // + 6 mbarriers and the TMEM slot
  // shared memory sized so that exactly CtasPerSm CTAs fit on an SM: no CTA
  // ever waits in tcgen05.alloc
  static constexpr int DynSmem = CtasPerSm == 2 ? 105 * 1024 : ((Smem + 1023) / 1024) * 1024;
  static_assert(Smem <= DynSmem && (CtasPerSm + 1) * (DynSmem + 1024) > 228 * 1024 &&
                    CtasPerSm * (DynSmem + 1024) <= 228 * 1024,
                "brick shared memory must admit exactly CtasPerSm CTAs per SM");
};

// The global-memory path for one point of a brick warp that left its boxes:
// departure and clamped gathers from global memory (tc_prepare_split), A row
// straight to the TMEM columns at `taddr`; returns the fraction.  Out of line,
// so the brick loop keeps its registers and code small; called by whole warps.
__device__ __noinline__ float3 brick_rows_global(Geom g, const uint32_t *__restrict__ phi0s,
                                                 const float *__restrict__ vel, float dth0, float dth1, float dth2,
                                                 int backtrace, int x, int y, int z, uint32_t taddr) {
  const float dth[3] = {dth0, dth1, dth2};
  float f[3];
  uint32_t w[64];
  bool clamped = false;
  tc_prepare_split(g, phi0s, vel, dth, backtrace, true, x, y, z, f, w, clamped);
  __syncwarp();
  tmem_st32(taddr, w);
  tmem_st32(taddr + 32, w + 32);
  return make_float3(f[0], f[1], f[2]);
}



// Dense-grid stepper over TMA-staged bricks.
//
// Each CTA owns bricks blockIdx.x, blockIdx.x + gridDim.x, ... (32 x 4 x 4P
// points, P = 2, 4 steps each); their boxes are double-buffered with the next
// brick in flight.  Four compute warps carry P points per thread and step --
// the same (x, y) in P consecutive z planes -- held in P TMEM stages (A | D,
// 128 columns each); a fifth warp only issues the MMAs and the TMA loads.
// Warps are decoupled by mbarriers, not CTA barriers:
//
//   compute warp, step j (step j+1's departures are known from step j-1):
//     1. wait dfull: step j's MMAs are done
//     2. A rows of step j+1's points -> the stages (step j's rows are read)
//     3. step j's coefficients -> registers, then arrive on afull (step j+1)
//     4. step j's values evaluated and stored
//     5. departures of step j+2's points (overlaps step j+1's MMAs)
//   issuer, step j: wait afull (all four warps), every stage's MMAs, commit to
//     dfull; after a brick's last step, refill that brick's buffer with the
//     brick two ahead.
//
// When every lane's P stencils are stacked one plane apart (the usual case:
// the points depart from vertically adjacent cells) the warp gathers their
// 4 x 4 x (P+3) union once.  A stage's A columns are rewritten only after the
// writing warp saw the MMAs that read them complete (1); D columns are
// overwritten only after every warp has read them and arrived for the next
// step (3).  A buffer is refilled only after afull of its brick's last step:
// every warp has then gathered from it for the last time (its departures were
// computed before).  Every wait is bounded; a
// warp that gives up raises FLAG_WAIT_TIMEOUT and leaves, and the others then
// give up at their next wait.  Before the CTA ends, the issuer waits for its
// last TMA load per buffer and its last commit.  SPLIT: also write the
// stepped values as packed split words (the next step's input).
constexpr int kBrickThreads = kTile + 32;

template <int BT, int P, bool SPLIT>
__global__ void __launch_bounds__(kBrickThreads, BrickShape<P>::CtasPerSm)
    sl_tc_brick_kernel(const __grid_constant__ CUtensorMap tm_phi, const __grid_constant__ CUtensorMap tm_vel, Geom g,
                       BrickGrid bg, const uint32_t *__restrict__ phi0s, const float *__restrict__ vel, float dt,
                       float *__restrict__ phi, uint32_t *__restrict__ phis, int *flags, const int *gate_maxw,
                       float gate_limit) {
  using S = BrickShape<P>;
  static_assert(P == 2, "the step loop holds two points' coefficients per thread");
  // z-slab launches: run only if the staged planes bound every departure
  // (max |w| dt / h_z over them within gate_limit); otherwise leave the slab
  // to a full-grid step once all planes are present
  if (gate_maxw && __int_as_float(*gate_maxw) * (dt / (float)g.hz) > gate_limit) {
    if (threadIdx.x == 0) raise_flag(flags, FLAG_PIPELINE_REDO);
    return;
  }
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t *sB = smem;
  uint8_t *const buf0 = smem + kBBytes, *const buf1 = smem + kBBytes + S::BufBytes;
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + kBBytes + 2 * S::BufBytes);
  uint64_t *const unused = bars + 0;  // setup() initialises one MMA barrier; this kernel uses its own
  uint64_t *const afull = bars + 1, *const dfull = bars + 2, *const tbar = bars + 3, *const fixbar = bars + 5;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 6);
  if (threadIdx.x == 0) {
    mbar_init(afull, 4);
    mbar_init(dfull, 1);
    mbar_init(&tbar[0], 1);
    mbar_init(&tbar[1], 1);
    mbar_init(fixbar, kTile);
  }
  Ctx c;
  setup(sB, unused, tmem_slot, c, S::TmemCols);  // B operand, TMEM; ends with a CTA barrier

  const int nbricks = bg.nbx * bg.nby * bg.nbz;
  const int nmine = (int)blockIdx.x < nbricks ? (nbricks - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  const int nsteps = 4 * nmine;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  bool err = false;

  if (warp == 4) {  // ---------------- issuer ----------------
    if (lane == 0) {
      int tma_issued[2] = {0, 0}, mma_issued = 0;
      if (nmine > 0) {
        issue_brick<S>(bg, blockIdx.x, buf0, &tm_phi, &tm_vel, &tbar[0]);
        tma_issued[0] = 1;
      }
      if (nmine > 1) {
        issue_brick<S>(bg, blockIdx.x + gridDim.x, buf1, &tm_phi, &tm_vel, &tbar[1]);
        tma_issued[1] = 1;
      }
      constexpr uint32_t idesc = instr_desc_bf16(kTile, kCoef);
      for (int j = 0; j < nsteps && !err; ++j) {
        // the issuer polls without a suspend hint: it reacts a little sooner
        // to the fourth arrival (measured ~1% on the 256^3 step)
        if (!mbar_wait(afull, (uint32_t)j & 1u)) { err = true; break; }
        fence_after();
#pragma unroll
        for (int st = 0; st < P; ++st)
#pragma unroll
          for (int kk = 0; kk < kK / 16; ++kk)
            mma_bf16(c.tmem + 128 * st + 64, c.tmem + 128 * st + (uint32_t)(kk * 8),
                     c.bdesc + (uint64_t)((kk * 256) >> 4), idesc, kk > 0 ? 1u : 0u);
        mma_commit(dfull);
        ++mma_issued;
        const int k = j >> 2;
        if ((j & 3) == 3 && k + 2 < nmine) {  // brick k read for the last time: refill with brick k+2
          issue_brick<S>(bg, (int)blockIdx.x + (k + 2) * (int)gridDim.x, k & 1 ? buf1 : buf0, &tm_phi, &tm_vel,
                         k & 1 ? &tbar[1] : &tbar[0]);
          ++tma_issued[k & 1];
        }
      }
      // nothing of this CTA may still be in flight when its TMEM and shared memory go away
      bool ok = true;
#pragma unroll
      for (int b = 0; b < 2; ++b)
        if (tma_issued[b]) ok &= mbar_wait(&tbar[b], (uint32_t)(tma_issued[b] - 1) & 1u);
      if (mma_issued) ok &= mbar_wait(dfull, (uint32_t)(mma_issued - 1) & 1u);
      if (err || !ok) raise_flag(flags, FLAG_WAIT_TIMEOUT);
    }
  } else {  // ---------------- compute warps ----------------
    const float dth[3] = {dt / (float)g.hx, dt / (float)g.hy, dt / (float)g.hz};
    const float hdth[3] = {-0.5f * dth[0], -0.5f * dth[1], -0.5f * dth[2]};
    const int lx = lane, ly = warp;  // a tile: 32 x 4 points of one z plane
    const int plane = g.nx * g.ny;
    const int nn[3] = {g.nx, g.ny, g.nz};
    uint32_t fixphase = 0;

    // Boxes of brick k staged (and edge-replicated where they cross the grid).
    auto open_brick = [&](int k, int &x0, int &y0, int &z0) -> bool {
      const bool odd = k & 1;
      if (!mbar_wait_sleep(odd ? &tbar[1] : &tbar[0], (uint32_t)(k >> 1) & 1u)) return false;
      brick_origin<S>(bg, (int)blockIdx.x + k * (int)gridDim.x, x0, y0, z0);
      if (x0 < 4 || x0 + S::PX - 4 > g.nx || y0 < 2 || y0 + S::PY - 2 > g.ny || z0 < 2 || z0 + S::PZ - 2 > g.nz) {
        uint8_t *cbuf = odd ? buf1 : buf0;
        const int op[3] = {x0 - 4, y0 - 2, z0 - 2}, ov[3] = {x0 - 4, y0 - 1, z0 - 1};
        for (int axis = 0; axis < 3; ++axis) {
          const bool a =
              replicate_pass<S::PX, S::PY, S::PZ, 1>(reinterpret_cast<uint32_t *>(cbuf), axis, op, nn, kTile);
          const bool b = replicate_pass<S::VX, S::VY, S::VZ, 3>(reinterpret_cast<uint32_t *>(cbuf + S::PhiBytes),
                                                                axis, ov, nn, kTile);
          if (!(a || b)) continue;
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic writes before a later TMA refill
          mbar_arrive(fixbar);
          const bool ok = mbar_wait_sleep(fixbar, fixphase);
          fixphase ^= 1u;
          if (!ok) return false;
        }
      }
      return true;
    };
    // Departures of step j's P points from brick (x0, y0, z0)'s boxes; lanes
    // past the grid's end (partial bricks) compute a copy of the last in-grid
    // column and store nothing; points past the grid's last plane are
    // computed from edge-replicated box cells and not stored.  Returns
    // whether the whole warp stays in the boxes.
    auto depart = [&](int j, int x0, int y0, int z0, float f[P][3], int soff[P]) -> bool {
      const float *vbox = reinterpret_cast<const float *>(((j >> 2) & 1 ? buf1 : buf0) + S::PhiBytes);
      const int x = min(x0 + lx, g.nx - 1), y = min(y0 + ly, g.ny - 1);
      const int zl = P * (j & 3);  // brick-local plane of point 0
      const bool in = brick_depart<BT, S, P>(vbox, x - x0 + 4, y - y0 + 1, zl + 1, x - x0 + 4, y - y0 + 2, zl + 2,
                                             dth, hdth, f, soff);
      return __all_sync(0xffffffffu, in);
    };
    // A rows of one point -> TMEM stage `st` (gathered from the box, or the
    // whole warp's global path).
    auto stage_rows = [&](int j, int x0, int y0, int z0, bool boxed, int soff, float f[3], int st) {
      if (boxed) {
        uint32_t w[64];
        const uint32_t *q = reinterpret_cast<const uint32_t *>((j >> 2) & 1 ? buf1 : buf0) + soff;
#pragma unroll
        for (int e = 0; e < 64; ++e) w[e] = q[((e >> 4) * S::PY + ((e >> 2) & 3)) * S::PX + (e & 3)];
        __syncwarp();  // the TMEM store is warp-collective
        tmem_st32(c.tmem + c.lane_off + 128 * st, w);
        tmem_st32(c.tmem + c.lane_off + 128 * st + 32, w + 32);
      } else {
        const int x = min(x0 + lx, g.nx - 1), y = min(y0 + ly, g.ny - 1);
        const int z = min(z0 + P * (j & 3) + st, g.nz - 1);
        const float3 r = brick_rows_global(g, phi0s, vel, dth[0], dth[1], dth[2], BT, x, y, z,
                                           c.tmem + c.lane_off + 128 * st);
        f[0] = r.x;
        f[1] = r.y;
        f[2] = r.z;
      }
    };

    // A rows of step s (points of brick (bx, by, bz), departures ff / so)
    // into their stages; the warp's 4 x 4 x (P+3) union is gathered once
    // when its stencils are stacked plane over plane (the usual case)
    auto stage_step = [&](int s, int bx, int by, int bz, bool bxd, int so[P], float ff[P][3]) {
      bool stacked = bxd;
#pragma unroll
      for (int p = 1; p < P; ++p) stacked = stacked && so[p] == so[0] + p * S::PX * S::PY;
      if (__all_sync(0xffffffffu, stacked)) {
        const uint32_t *q = reinterpret_cast<const uint32_t *>((s >> 2) & 1 ? buf1 : buf0) + so[0];
        uint32_t v[16 * (P + 3)];
#pragma unroll
        for (int e = 0; e < 16 * (P + 3); ++e) v[e] = q[((e >> 4) * S::PY + ((e >> 2) & 3)) * S::PX + (e & 3)];
#pragma unroll
        for (int p = 0; p < P; ++p)
#pragma unroll
          for (int q16 = 0; q16 < 4; ++q16)  // point p's z-slice q16 is plane p + q16 of the union
            tmem_st16(c.tmem + c.lane_off + 128 * p + 16 * q16, v + 16 * (p + q16));
      } else {
#pragma unroll
        for (int p = 0; p < P; ++p) stage_rows(s, bx, by, bz, bxd, so[p], ff[p], p);
      }
    };

    // Step j's points (brick origin x0.., departures f / soff) and step
    // j+1's (x1.., f1 / soff1): step j+1's A rows go in as soon as step j's
    // MMAs are done, so its MMAs run while step j is evaluated and step
    // j+2's departures are computed.
    int x0 = 0, y0 = 0, z0 = 0, x1 = 0, y1 = 0, z1 = 0;
    float f[P][3], f1[P][3];
    int soff[P], soff1[P];
    bool boxed = true, boxed1 = true;
    if (nsteps > 0) {
      err = !open_brick(0, x0, y0, z0);
      if (__any_sync(0xffffffffu, err)) err = true;
      else boxed = depart(0, x0, y0, z0, f, soff);
    }
    if (nsteps > 0 && !err) {
      stage_step(0, x0, y0, z0, boxed, soff, f);
      tmem_wait_st();
      fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(afull);
      x1 = x0; y1 = y0; z1 = z0;
      if (nsteps > 1) boxed1 = depart(1, x1, y1, z1, f1, soff1);  // step 1 lies in brick 0
    }
    for (int j = 0; j < nsteps && !err; ++j) {
      const int x = min(x0 + lx, g.nx - 1), y = min(y0 + ly, g.ny - 1);
      const bool xy_valid = x0 + lx < g.nx && y0 + ly < g.ny;
      const int zr = z0 + P * (j & 3);
      const int p0 = (min(zr, g.nz - 1) * g.ny + y) * g.nx + x;
      // polled, not suspend-hinted: the warp resumes as the MMAs complete
      const bool ok = mbar_wait(dfull, (uint32_t)j & 1u);
      if (__any_sync(0xffffffffu, !ok)) { err = true; break; }
      fence_after();
      // step j's MMAs have read their A rows: step j+1's replace them
      const bool more = j + 1 < nsteps;
      if (more) stage_step(j + 1, x1, y1, z1, boxed1, soff1, f1);
      // step j's coefficients into registers before step j+1's MMAs overwrite them
      float ca[64], cb[64];
      tmem_ld32f(c.tmem + c.lane_off + 96, ca + 32);
      tmem_ld32f(c.tmem + c.lane_off + 128 + 96, cb + 32);
      tmem_ld32f(c.tmem + c.lane_off + 64, ca);
      tmem_ld32f(c.tmem + c.lane_off + 128 + 64, cb);
      tmem_wait_ld_tied(ca + 32, cb + 32);
      tmem_wait_ld_tied(ca, cb);  // (the first wait completed all four loads; this one ties the rest)
      if (more) {
        tmem_wait_st();
        fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(afull);
      }
      // step j's values (horner3 order: slices k = 3 .. 0)
      float va = 0.f, vb = 0.f;
#pragma unroll
      for (int kz = 3; kz >= 0; --kz) {
        va = fmaf(va, f[0][2], horner_slice(ca + 16 * kz, f[0]));
        vb = fmaf(vb, f[1][2], horner_slice(cb + 16 * kz, f[1]));
      }
      if (xy_valid && zr < g.nz) {
        phi[p0] = va;
        if (SPLIT) phis[p0] = pack_split(va);
      }
      if (xy_valid && zr + 1 < g.nz) {
        phi[p0 + plane] = vb;
        if (SPLIT) phis[p0 + plane] = pack_split(vb);
      }
      // step j+2's departures while step j+1's MMAs run
      int x2 = x1, y2 = y1, z2 = z1;
      float f2[P][3];
      int soff2[P];
      bool boxed2 = true;
      if (j + 2 < nsteps) {
        if (((j + 2) & 3) == 0) err = !open_brick((j + 2) >> 2, x2, y2, z2);
        if (__any_sync(0xffffffffu, err)) err = true;
        else boxed2 = depart(j + 2, x2, y2, z2, f2, soff2);
      }
      x0 = x1; y0 = y1; z0 = z1;
      x1 = x2; y1 = y2; z1 = z2;
#pragma unroll
      for (int p = 0; p < P; ++p) {
        f[p][0] = f1[p][0]; f[p][1] = f1[p][1]; f[p][2] = f1[p][2];
        soff[p] = soff1[p];
        f1[p][0] = f2[p][0]; f1[p][1] = f2[p][1]; f1[p][2] = f2[p][2];
        soff1[p] = soff2[p];
      }
      boxed = boxed1;
      boxed1 = boxed2;
    }
    if (err) raise_flag(flags, FLAG_WAIT_TIMEOUT);
  }
  __syncwarp();  // the issuer warp's other lanes wait here for lane 0
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 0) tmem_dealloc(c.tmem, S::TmemCols);
}

// Batched split-state stepper over the bricks of many cells (cells of uneven
// sizes in one persistent launch).  Same bricks, step loop and arithmetic as
// sl_tc_brick_kernel, hence per cell the bits of dcell_sl_step_tc_split.
// The cells' rows have arbitrary lengths and offsets in the packed arrays,
// which TMA's 16-byte strides do not admit, so the compute warps stage the
// boxes themselves with 4-byte cp.async copies from source indices clamped to
// the cell: the edge replication that zero fill + replicate_pass gives the
// dense kernel.  Double-buffered as there: brick m lands in buffer m & 1;
// its copies are issued when brick m-2 has been read for the last time and
// complete on staged[m & 1] (each thread's copies arrive with
// cp.async.mbarrier.arrive.noinc), which the first departure of brick m waits
// for; freed[m & 1] collects the compute threads after brick m's last step.
// The issuer warp only issues MMAs.  Every wait is bounded.
__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_arrive(uint64_t *bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// one brick of a cell and the cell's grid
struct CellBrick {
  Geom g;         // the cell's grid, origin 0
  long long off;  // the cell's first point in the packed arrays
  float dth[3], hdth[3];
  int x0, y0, z0;
};

__device__ __forceinline__ CellBrick cell_brick(const dcell_cell *__restrict__ cells,
                                                const dcell_tile *__restrict__ bricks, int b) {
  const dcell_tile T = bricks[b];
  const dcell_cell C = cells[T.cell];
  CellBrick r;
  r.g.nx = C.n[0];
  r.g.ny = C.n[1];
  r.g.nz = C.n[2];
  r.g.px = r.g.py = r.g.pz = 0;
  r.g.hx = C.h[0];
  r.g.hy = C.h[1];
  r.g.hz = C.h[2];
  r.off = C.offset;
  const float dt = (float)C.dt;  // the rounding of the single-grid launch
  r.dth[0] = dt / (float)C.h[0];
  r.dth[1] = dt / (float)C.h[1];
  r.dth[2] = dt / (float)C.h[2];
#pragma unroll
  for (int a = 0; a < 3; ++a) r.hdth[a] = -0.5f * r.dth[a];
  r.x0 = T.x0;
  r.y0 = T.y0;
  r.z0 = T.z0;
  return r;
}

// A compute thread's share of brick B's two boxes into buf (rows spread over
// the four compute warps, lanes along a row), then its arrival on `bar` once
// its copies have landed.
template <class S>
__device__ __forceinline__ void stage_brick(uint8_t *buf, const CellBrick &B, const uint32_t *__restrict__ phi0s,
                                            const float *__restrict__ vel, int warp, int lane, uint64_t *bar) {
  const int nx = B.g.nx, ny = B.g.ny, nz = B.g.nz;
  const uint32_t *ps = phi0s + B.off;
  const float *vs = vel + 3 * B.off;
  uint32_t *pb = reinterpret_cast<uint32_t *>(buf);
  float *vb = reinterpret_cast<float *>(buf + S::PhiBytes);
  for (int r = warp; r < S::PY * S::PZ; r += 4) {
    const int gy = min(max(B.y0 - 2 + r % S::PY, 0), ny - 1), gz = min(max(B.z0 - 2 + r / S::PY, 0), nz - 1);
    const uint32_t *src = ps + ((long long)gz * ny + gy) * nx;
    for (int x = lane; x < S::PX; x += 32) cp_async4(pb + r * S::PX + x, src + min(max(B.x0 - 4 + x, 0), nx - 1));
  }
  for (int r = warp; r < S::VY * S::VZ; r += 4) {
    const int gy = min(max(B.y0 - 1 + r % S::VY, 0), ny - 1), gz = min(max(B.z0 - 1 + r / S::VY, 0), nz - 1);
    const float *src = vs + ((long long)gz * ny + gy) * nx * 3;
    for (int c = lane; c < 3 * S::VX; c += 32) {
      const int x = c / 3;
      cp_async4(vb + r * 3 * S::VX + c, src + 3 * min(max(B.x0 - 4 + x, 0), nx - 1) + (c - 3 * x));
    }
  }
  cp_async_arrive(bar);
}

template <int BT>
__global__ void __launch_bounds__(kBrickThreads, BrickShape<2>::CtasPerSm)
    batch_brick_kernel(const dcell_cell *__restrict__ cells, const dcell_tile *__restrict__ bricks, int nbricks,
                       const uint32_t *__restrict__ phi0s, const float *__restrict__ vel, float *__restrict__ phi,
                       uint32_t *__restrict__ phis, int *flags) {
  constexpr int P = 2;
  using S = BrickShape<P>;
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t *sB = smem;
  uint8_t *const buf0 = smem + kBBytes, *const buf1 = smem + kBBytes + S::BufBytes;
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + kBBytes + 2 * S::BufBytes);
  uint64_t *const unused = bars + 0;  // setup() initialises one MMA barrier; this kernel uses its own
  uint64_t *const afull = bars + 1, *const dfull = bars + 2, *const staged = bars + 3, *const freed = bars + 5;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 7);
  if (threadIdx.x == 0) {
    mbar_init(afull, 4);
    mbar_init(dfull, 1);
    for (int b = 0; b < 2; ++b) {
      mbar_init(&staged[b], kTile);
      mbar_init(&freed[b], kTile);
    }
  }
  Ctx c;
  setup(sB, unused, tmem_slot, c, S::TmemCols);  // B operand, TMEM; ends with a CTA barrier

  const int nmine = (int)blockIdx.x < nbricks ? (nbricks - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  const int nsteps = 4 * nmine;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  bool err = false;

  if (warp == 4) {  // ---------------- issuer ----------------
    if (lane == 0) {
      int mma_issued = 0;
      constexpr uint32_t idesc = instr_desc_bf16(kTile, kCoef);
      for (int j = 0; j < nsteps && !err; ++j) {
        if (!mbar_wait(afull, (uint32_t)j & 1u)) { err = true; break; }
        fence_after();
#pragma unroll
        for (int st = 0; st < P; ++st)
#pragma unroll
          for (int kk = 0; kk < kK / 16; ++kk)
            mma_bf16(c.tmem + 128 * st + 64, c.tmem + 128 * st + (uint32_t)(kk * 8),
                     c.bdesc + (uint64_t)((kk * 256) >> 4), idesc, kk > 0 ? 1u : 0u);
        mma_commit(dfull);
        ++mma_issued;
      }
      bool ok = true;
      if (mma_issued) ok &= mbar_wait(dfull, (uint32_t)(mma_issued - 1) & 1u);
      if (err || !ok) raise_flag(flags, FLAG_WAIT_TIMEOUT);
    }
  } else {  // ---------------- compute warps ----------------
    const int lx = lane, ly = warp;
    auto brick = [&](int k) { return cell_brick(cells, bricks, (int)blockIdx.x + k * (int)gridDim.x); };
    auto buffer = [&](int k) { return k & 1 ? buf1 : buf0; };
    // brick k staged (bounded wait)
    auto landed = [&](int k) -> bool { return mbar_wait_sleep(&staged[k & 1], (uint32_t)(k >> 1) & 1u); };
    auto depart = [&](int j, const CellBrick &B, float f[P][3], int soff[P]) -> bool {
      const float *vbox = reinterpret_cast<const float *>(buffer(j >> 2) + S::PhiBytes);
      const int x = min(B.x0 + lx, B.g.nx - 1), y = min(B.y0 + ly, B.g.ny - 1);
      const int zl = P * (j & 3);
      const bool in = brick_depart<BT, S, P>(vbox, x - B.x0 + 4, y - B.y0 + 1, zl + 1, x - B.x0 + 4, y - B.y0 + 2,
                                             zl + 2, B.dth, B.hdth, f, soff);
      return __all_sync(0xffffffffu, in);
    };
    if (nmine > 0) stage_brick<S>(buf0, brick(0), phi0s, vel, warp, lane, &staged[0]);
    if (nmine > 1) stage_brick<S>(buf1, brick(1), phi0s, vel, warp, lane, &staged[1]);
    CellBrick B;
    float f[P][3];
    int soff[P];
    bool boxed = true;
    if (nsteps > 0) {
      B = brick(0);
      if (!landed(0)) err = true;
      if (__any_sync(0xffffffffu, err)) err = true;
      else boxed = depart(0, B, f, soff);
    }
    for (int j = 0; j < nsteps && !err; ++j) {
      const int k = j >> 2;
      const uint32_t *ps = phi0s + B.off;
      const float *vs = vel + 3 * B.off;
      // a: A rows of the P points into their stages, then this warp's arrival
      bool stacked = boxed;
#pragma unroll
      for (int p = 1; p < P; ++p) stacked = stacked && soff[p] == soff[0] + p * S::PX * S::PY;
      if (__all_sync(0xffffffffu, stacked)) {
        const uint32_t *q = reinterpret_cast<const uint32_t *>(buffer(k)) + soff[0];
        uint32_t v[16 * (P + 3)];
#pragma unroll
        for (int e = 0; e < 16 * (P + 3); ++e) v[e] = q[((e >> 4) * S::PY + ((e >> 2) & 3)) * S::PX + (e & 3)];
#pragma unroll
        for (int p = 0; p < P; ++p)
#pragma unroll
          for (int q16 = 0; q16 < 4; ++q16) tmem_st16(c.tmem + c.lane_off + 128 * p + 16 * q16, v + 16 * (p + q16));
      } else {
#pragma unroll
        for (int p = 0; p < P; ++p) {
          if (boxed) {
            uint32_t w[64];
            const uint32_t *q = reinterpret_cast<const uint32_t *>(buffer(k)) + soff[p];
#pragma unroll
            for (int e = 0; e < 64; ++e) w[e] = q[((e >> 4) * S::PY + ((e >> 2) & 3)) * S::PX + (e & 3)];
            __syncwarp();
            tmem_st32(c.tmem + c.lane_off + 128 * p, w);
            tmem_st32(c.tmem + c.lane_off + 128 * p + 32, w + 32);
          } else {  // the warp left its boxes: departure and gathers from global memory
            const int x = min(B.x0 + lx, B.g.nx - 1), y = min(B.y0 + ly, B.g.ny - 1);
            const int z = min(B.z0 + P * (j & 3) + p, B.g.nz - 1);
            const float3 r = brick_rows_global(B.g, ps, vs, B.dth[0], B.dth[1], B.dth[2], BT, x, y, z,
                                               c.tmem + c.lane_off + 128 * p);
            f[p][0] = r.x;
            f[p][1] = r.y;
            f[p][2] = r.z;
          }
        }
      }
      tmem_wait_st();
      fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(afull);
      // b: next step's departures while the tensor core works
      CellBrick Bn = B;
      float fn[P][3];
      int soffn[P];
      bool boxedn = true;
      if (j + 1 < nsteps) {
        if (((j + 1) & 3) == 0) {  // brick k+1: staged?
          Bn = brick(k + 1);
          if (!landed(k + 1)) err = true;
        }
        if (__any_sync(0xffffffffu, err)) err = true;
        else boxedn = depart(j + 1, Bn, fn, soffn);
      }
      // c: coefficients -> values, two points at a time
      const int x = min(B.x0 + lx, B.g.nx - 1), y = min(B.y0 + ly, B.g.ny - 1);
      const bool xy_valid = B.x0 + lx < B.g.nx && B.y0 + ly < B.g.ny;
      const int zr = B.z0 + P * (j & 3);
      const int plane = B.g.nx * B.g.ny;
      const long long p0 = B.off + ((long long)min(zr, B.g.nz - 1) * B.g.ny + y) * B.g.nx + x;
      const bool ok = mbar_wait_sleep(dfull, (uint32_t)j & 1u);
      if (__any_sync(0xffffffffu, !ok)) { err = true; break; }
      fence_after();
      {
        float ca[64], cb[64];
        tmem_ld32f(c.tmem + c.lane_off + 64, ca);
        tmem_ld32f(c.tmem + c.lane_off + 128 + 64, cb);
        tmem_ld32f(c.tmem + c.lane_off + 96, ca + 32);
        tmem_ld32f(c.tmem + c.lane_off + 128 + 96, cb + 32);
        tmem_wait_ld_tied(ca, cb);
        tmem_wait_ld_tied(ca + 32, cb + 32);  // completes nothing more: ties the other halves
        float va = 0.f, vb = 0.f;  // horner3 order: slices k = 3 .. 0
#pragma unroll
        for (int kz = 3; kz >= 0; --kz) {
          va = fmaf(va, f[0][2], horner_slice(ca + 16 * kz, f[0]));
          vb = fmaf(vb, f[1][2], horner_slice(cb + 16 * kz, f[1]));
        }
        if (xy_valid && zr < B.g.nz) {
          phi[p0] = va;
          phis[p0] = pack_split(va);
        }
        if (xy_valid && zr + 1 < B.g.nz) {
          phi[p0 + plane] = vb;
          phis[p0 + plane] = pack_split(vb);
        }
      }
      fence_before();
      if ((j & 3) == 3) {  // brick k read for the last time: its buffer takes brick k+2
        mbar_arrive(&freed[k & 1]);
        if (k + 2 < nmine) {
          if (!mbar_wait_sleep(&freed[k & 1], (uint32_t)(k >> 1) & 1u)) err = true;
          if (__any_sync(0xffffffffu, err)) { err = true; break; }
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // the reads above before the copies
          stage_brick<S>(buffer(k), brick(k + 2), phi0s, vel, warp, lane, &staged[k & 1]);
        }
      }
      B = Bn;
#pragma unroll
      for (int p = 0; p < P; ++p) {
        f[p][0] = fn[p][0]; f[p][1] = fn[p][1]; f[p][2] = fn[p][2];
        soff[p] = soffn[p];
      }
      boxed = boxedn;
    }
    asm volatile("cp.async.wait_all;" ::: "memory");  // no copy may land after the CTA is gone
    if (err) raise_flag(flags, FLAG_WAIT_TIMEOUT);
  }
  __syncwarp();  // the issuer warp's other lanes wait here for lane 0
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 0) tmem_dealloc(c.tmem, S::TmemCols);
}

// Batched split-state stepper over the bricks of many cells, the boxes
// staged by TMA as in sl_tc_brick_kernel.  The cells are packed with padded
// rows (dcell_cell.pad = the row length in points, a multiple of 4; cell
// offsets multiples of 4 points) whose pad columns hold copies of the cell's
// last column, so every cell is a dense grid of its padded width whose extra
// columns read as the clamped edge: a TMA map per cell (maps[2 c] the split
// words, maps[2 c + 1] the velocity, built by dcell_batch_tma_maps), the
// dense kernel's boxes, edge replication and departures, and the clamped
// global path all see the cell's own values.  Arrival points are clamped to
// the cell's columns; lanes over the pad columns store the stepped last
// column there, which keeps the pads copies.  Per cell the real points get
// the bits of dcell_sl_step_tc_split on the unpadded cell.
struct CellBrickP {
  CellBrick b;  // geometry: g.nx = the padded row length
  int nxl;      // the cell's columns
};

__device__ __forceinline__ CellBrickP cell_brick_padded(const dcell_cell *__restrict__ cells,
                                                        const dcell_tile *__restrict__ bricks, int b) {
  CellBrickP r;
  r.b = cell_brick(cells, bricks, b);
  const dcell_cell C = cells[bricks[b].cell];
  r.nxl = C.n[0];
  if (C.pad > C.n[0]) r.b.g.nx = C.pad;
  return r;
}

template <int BT>
__global__ void __launch_bounds__(kBrickThreads, BrickShape<2>::CtasPerSm)
    batch_brick_tma_kernel(const dcell_cell *__restrict__ cells, const dcell_tile *__restrict__ bricks, int nbricks,
                           const CUtensorMap *__restrict__ maps, const uint32_t *__restrict__ phi0s,
                           const float *__restrict__ vel, float *__restrict__ phi, uint32_t *__restrict__ phis,
                           int *flags) {
  constexpr int P = 2;
  using S = BrickShape<P>;
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t *sB = smem;
  uint8_t *const buf0 = smem + kBBytes, *const buf1 = smem + kBBytes + S::BufBytes;
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + kBBytes + 2 * S::BufBytes);
  uint64_t *const unused = bars + 0;  // setup() initialises one MMA barrier; this kernel uses its own
  uint64_t *const afull = bars + 1, *const dfull = bars + 2, *const tbar = bars + 3, *const fixbar = bars + 5;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 6);
  if (threadIdx.x == 0) {
    mbar_init(afull, 4);
    mbar_init(dfull, 1);
    mbar_init(&tbar[0], 1);
    mbar_init(&tbar[1], 1);
    mbar_init(fixbar, kTile);
  }
  Ctx c;
  setup(sB, unused, tmem_slot, c, S::TmemCols);  // B operand, TMEM; ends with a CTA barrier

  const int nmine = (int)blockIdx.x < nbricks ? (nbricks - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  const int nsteps = 4 * nmine;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  bool err = false;
  // both boxes of the k-th brick of this CTA into `buf` (one thread)
  auto issue = [&](int k, uint8_t *buf, uint64_t *bar) {
    const dcell_tile T = bricks[(int)blockIdx.x + k * (int)gridDim.x];
    fence_proxy_async();
    mbar_expect_tx(bar, (uint32_t)S::BufBytes);
    tma_load_3d(buf, maps + 2 * T.cell, T.x0 - 4, T.y0 - 2, T.z0 - 2, bar);
    tma_load_3d(buf + S::PhiBytes, maps + 2 * T.cell + 1, 3 * (T.x0 - 4), T.y0 - 1, T.z0 - 1, bar);
  };

  if (warp == 4) {  // ---------------- issuer ----------------
    if (lane == 0) {
      int tma_issued[2] = {0, 0}, mma_issued = 0;
      if (nmine > 0) {
        issue(0, buf0, &tbar[0]);
        tma_issued[0] = 1;
      }
      if (nmine > 1) {
        issue(1, buf1, &tbar[1]);
        tma_issued[1] = 1;
      }
      constexpr uint32_t idesc = instr_desc_bf16(kTile, kCoef);
      for (int j = 0; j < nsteps && !err; ++j) {
        if (!mbar_wait(afull, (uint32_t)j & 1u)) { err = true; break; }
        fence_after();
#pragma unroll
        for (int st = 0; st < P; ++st)
#pragma unroll
          for (int kk = 0; kk < kK / 16; ++kk)
            mma_bf16(c.tmem + 128 * st + 64, c.tmem + 128 * st + (uint32_t)(kk * 8),
                     c.bdesc + (uint64_t)((kk * 256) >> 4), idesc, kk > 0 ? 1u : 0u);
        mma_commit(dfull);
        ++mma_issued;
        const int k = j >> 2;
        if ((j & 3) == 3 && k + 2 < nmine) {  // brick k read for the last time: refill with brick k+2
          issue(k + 2, k & 1 ? buf1 : buf0, k & 1 ? &tbar[1] : &tbar[0]);
          ++tma_issued[k & 1];
        }
      }
      bool ok = true;
#pragma unroll
      for (int b = 0; b < 2; ++b)
        if (tma_issued[b]) ok &= mbar_wait(&tbar[b], (uint32_t)(tma_issued[b] - 1) & 1u);
      if (mma_issued) ok &= mbar_wait(dfull, (uint32_t)(mma_issued - 1) & 1u);
      if (err || !ok) raise_flag(flags, FLAG_WAIT_TIMEOUT);
    }
  } else {  // ---------------- compute warps ----------------
    const int lx = lane, ly = warp;
    uint32_t fixphase = 0;
    // Boxes of brick k staged (and edge-replicated where they cross the cell's padded grid).
    auto open_brick = [&](int k, CellBrickP &B) -> bool {
      const bool odd = k & 1;
      if (!mbar_wait_sleep(odd ? &tbar[1] : &tbar[0], (uint32_t)(k >> 1) & 1u)) return false;
      B = cell_brick_padded(cells, bricks, (int)blockIdx.x + k * (int)gridDim.x);
      const Geom &g = B.b.g;
      const int x0 = B.b.x0, y0 = B.b.y0, z0 = B.b.z0;
      if (x0 < 4 || x0 + S::PX - 4 > g.nx || y0 < 2 || y0 + S::PY - 2 > g.ny || z0 < 2 || z0 + S::PZ - 2 > g.nz) {
        uint8_t *cbuf = odd ? buf1 : buf0;
        const int op[3] = {x0 - 4, y0 - 2, z0 - 2}, ov[3] = {x0 - 4, y0 - 1, z0 - 1};
        const int nn[3] = {g.nx, g.ny, g.nz};
        for (int axis = 0; axis < 3; ++axis) {
          const bool a =
              replicate_pass<S::PX, S::PY, S::PZ, 1>(reinterpret_cast<uint32_t *>(cbuf), axis, op, nn, kTile);
          const bool b = replicate_pass<S::VX, S::VY, S::VZ, 3>(reinterpret_cast<uint32_t *>(cbuf + S::PhiBytes),
                                                                axis, ov, nn, kTile);
          if (!(a || b)) continue;
          fence_proxy_async();  // generic writes before a later TMA refill
          mbar_arrive(fixbar);
          const bool ok = mbar_wait_sleep(fixbar, fixphase);
          fixphase ^= 1u;
          if (!ok) return false;
        }
      }
      return true;
    };
    // Departures of step j's P points; lanes over the cell's pad columns (and
    // past its last column) compute the last column
    auto depart = [&](int j, const CellBrickP &B, float f[P][3], int soff[P]) -> bool {
      const float *vbox = reinterpret_cast<const float *>(((j >> 2) & 1 ? buf1 : buf0) + S::PhiBytes);
      const int x = min(B.b.x0 + lx, B.nxl - 1), y = min(B.b.y0 + ly, B.b.g.ny - 1);
      const int zl = P * (j & 3);
      const bool in = brick_depart<BT, S, P>(vbox, x - B.b.x0 + 4, y - B.b.y0 + 1, zl + 1, x - B.b.x0 + 4,
                                             y - B.b.y0 + 2, zl + 2, B.b.dth, B.b.hdth, f, soff);
      return __all_sync(0xffffffffu, in);
    };

    CellBrickP B;
    float f[P][3];
    int soff[P];
    bool boxed = true;
    if (nsteps > 0) {
      err = !open_brick(0, B);
      if (__any_sync(0xffffffffu, err)) err = true;
      else boxed = depart(0, B, f, soff);
    }
    for (int j = 0; j < nsteps && !err; ++j) {
      const int k = j >> 2;
      const uint32_t *ps = phi0s + B.b.off;
      const float *vs = vel + 3 * B.b.off;
      // a: A rows of the P points into their stages, then this warp's arrival
      bool stacked = boxed;
#pragma unroll
      for (int p = 1; p < P; ++p) stacked = stacked && soff[p] == soff[0] + p * S::PX * S::PY;
      if (__all_sync(0xffffffffu, stacked)) {
        const uint32_t *q = reinterpret_cast<const uint32_t *>(k & 1 ? buf1 : buf0) + soff[0];
        uint32_t v[16 * (P + 3)];
#pragma unroll
        for (int e = 0; e < 16 * (P + 3); ++e) v[e] = q[((e >> 4) * S::PY + ((e >> 2) & 3)) * S::PX + (e & 3)];
#pragma unroll
        for (int p = 0; p < P; ++p)
#pragma unroll
          for (int q16 = 0; q16 < 4; ++q16) tmem_st16(c.tmem + c.lane_off + 128 * p + 16 * q16, v + 16 * (p + q16));
      } else {
#pragma unroll
        for (int p = 0; p < P; ++p) {
          if (boxed) {
            uint32_t w[64];
            const uint32_t *q = reinterpret_cast<const uint32_t *>(k & 1 ? buf1 : buf0) + soff[p];
#pragma unroll
            for (int e = 0; e < 64; ++e) w[e] = q[((e >> 4) * S::PY + ((e >> 2) & 3)) * S::PX + (e & 3)];
            __syncwarp();
            tmem_st32(c.tmem + c.lane_off + 128 * p, w);
            tmem_st32(c.tmem + c.lane_off + 128 * p + 32, w + 32);
          } else {  // the warp left its boxes: departure and gathers from global memory
            const int x = min(B.b.x0 + lx, B.nxl - 1), y = min(B.b.y0 + ly, B.b.g.ny - 1);
            const int z = min(B.b.z0 + P * (j & 3) + p, B.b.g.nz - 1);
            const float3 r = brick_rows_global(B.b.g, ps, vs, B.b.dth[0], B.b.dth[1], B.b.dth[2], BT, x, y, z,
                                               c.tmem + c.lane_off + 128 * p);
            f[p][0] = r.x;
            f[p][1] = r.y;
            f[p][2] = r.z;
          }
        }
      }
      tmem_wait_st();
      fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(afull);
      // b: next step's departures while the tensor core works
      CellBrickP Bn = B;
      float fn[P][3];
      int soffn[P];
      bool boxedn = true;
      if (j + 1 < nsteps) {
        if (((j + 1) & 3) == 0) err = !open_brick(k + 1, Bn);
        if (__any_sync(0xffffffffu, err)) err = true;
        else boxedn = depart(j + 1, Bn, fn, soffn);
      }
      // c: coefficients -> values, two points at a time
      const Geom &g = B.b.g;
      const int y = min(B.b.y0 + ly, g.ny - 1);
      const int xs = B.b.x0 + lx;  // the column stored: pad columns take the last column's value
      const bool xy_valid = xs < g.nx && B.b.y0 + ly < g.ny;
      const int zr = B.b.z0 + P * (j & 3);
      const int plane = g.nx * g.ny;
      const long long p0 = B.b.off + ((long long)min(zr, g.nz - 1) * g.ny + y) * g.nx + min(xs, g.nx - 1);
      const bool ok = mbar_wait_sleep(dfull, (uint32_t)j & 1u);
      if (__any_sync(0xffffffffu, !ok)) { err = true; break; }
      fence_after();
      {
        float ca[64], cb[64];
        tmem_ld32f(c.tmem + c.lane_off + 64, ca);
        tmem_ld32f(c.tmem + c.lane_off + 128 + 64, cb);
        tmem_ld32f(c.tmem + c.lane_off + 96, ca + 32);
        tmem_ld32f(c.tmem + c.lane_off + 128 + 96, cb + 32);
        tmem_wait_ld_tied(ca, cb);
        tmem_wait_ld_tied(ca + 32, cb + 32);  // completes nothing more: ties the other halves
        float va = 0.f, vb = 0.f;  // horner3 order: slices k = 3 .. 0
#pragma unroll
        for (int kz = 3; kz >= 0; --kz) {
          va = fmaf(va, f[0][2], horner_slice(ca + 16 * kz, f[0]));
          vb = fmaf(vb, f[1][2], horner_slice(cb + 16 * kz, f[1]));
        }
        if (xy_valid && zr < g.nz) {
          phi[p0] = va;
          phis[p0] = pack_split(va);
        }
        if (xy_valid && zr + 1 < g.nz) {
          phi[p0 + plane] = vb;
          phis[p0 + plane] = pack_split(vb);
        }
      }
      fence_before();
      B = Bn;
#pragma unroll
      for (int p = 0; p < P; ++p) {
        f[p][0] = fn[p][0]; f[p][1] = fn[p][1]; f[p][2] = fn[p][2];
        soff[p] = soffn[p];
      }
      boxed = boxedn;
    }
    if (err) raise_flag(flags, FLAG_WAIT_TIMEOUT);
  }
  __syncwarp();  // the issuer warp's other lanes wait here for lane 0
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 0) tmem_dealloc(c.tmem, S::TmemCols);
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

// The give-up path of the kernels' bounded waits: one thread waits on phase 0
// of an mbarrier that expects one arrival nobody makes, first with the
// polling wait (the MMA issuer's), then with the suspending wait (the compute
// warps'); result = 1 if the first gave up, + 2 if the second did.
__global__ void wait_timeout_check_kernel(int *result) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    const bool a = mbar_wait(&bar, 0u);
    const bool b = mbar_wait_sleep(&bar, 0u);
    *result = (a ? 0 : 1) | (b ? 0 : 2);
  }
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

int launch_batch_brick(const dcell_cell *cells, const dcell_tile *bricks, int nbricks, const uint32_t *phi0s,
                       const float *vel, int backtrace, float *phi, uint32_t *phis, int *flags, cudaStream_t st) {
  using S = tc::BrickShape<2>;
  static bool configured = false;
  if (!configured) {
    DCELL_CUDA_CHECK(cudaFuncSetAttribute(tc::batch_brick_kernel<DCELL_EULER>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, S::DynSmem));
    DCELL_CUDA_CHECK(cudaFuncSetAttribute(tc::batch_brick_kernel<DCELL_MIDPOINT>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, S::DynSmem));
    configured = true;
  }
  if (nbricks <= 0) return DCELL_OK;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = S::CtasPerSm * sms < nbricks ? S::CtasPerSm * sms : nbricks;
  auto kern = backtrace == DCELL_MIDPOINT ? tc::batch_brick_kernel<DCELL_MIDPOINT> : tc::batch_brick_kernel<DCELL_EULER>;
  kern<<<grid, tc::kBrickThreads, S::DynSmem, st>>>(cells, bricks, nbricks, phi0s, vel, phi, phis, flags);
  return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
}

int launch_batch_brick_tma(const dcell_cell *cells, const dcell_tile *bricks, int nbricks, const void *maps,
                           const uint32_t *phi0s, const float *vel, int backtrace, float *phi, uint32_t *phis,
                           int *flags, cudaStream_t st) {
  using S = tc::BrickShape<2>;
  static bool configured = false;
  if (!configured) {
    DCELL_CUDA_CHECK(cudaFuncSetAttribute(tc::batch_brick_tma_kernel<DCELL_EULER>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, S::DynSmem));
    DCELL_CUDA_CHECK(cudaFuncSetAttribute(tc::batch_brick_tma_kernel<DCELL_MIDPOINT>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, S::DynSmem));
    configured = true;
  }
  if (nbricks <= 0) return DCELL_OK;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = S::CtasPerSm * sms < nbricks ? S::CtasPerSm * sms : nbricks;
  auto kern = backtrace == DCELL_MIDPOINT ? tc::batch_brick_tma_kernel<DCELL_MIDPOINT>
                                          : tc::batch_brick_tma_kernel<DCELL_EULER>;
  kern<<<grid, tc::kBrickThreads, S::DynSmem, st>>>(cells, bricks, nbricks, (const CUtensorMap *)maps, phi0s, vel,
                                                      phi, phis, flags);
  return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
}

int batch_tma_maps_host(const dcell_cell *cells, int ncells, const uint32_t *phi0s, const float *vel, void *out) {
  using S = tc::BrickShape<2>;
  CUtensorMap *m = (CUtensorMap *)out;
  for (int c = 0; c < ncells; ++c) {
    const dcell_cell &C = cells[c];
    const int sx = C.pad > C.n[0] ? C.pad : C.n[0];
    if (sx % 4 || C.offset % 4 || C.n[1] < 1 || C.n[2] < 2) {
      dcell_set_error(DCELL_ERR_ARG, "cell %d: rows of %d points at offset %lld: TMA needs rows and offsets that are "
                                     "multiples of 4 points, and a 3D cell", c, sx, C.offset);
      return DCELL_ERR_ARG;
    }
    if (!make_tensor_map_3d(&m[2 * c], CU_TENSOR_MAP_DATA_TYPE_UINT32, phi0s + C.offset, (uint64_t)sx,
                            (uint64_t)C.n[1], (uint64_t)C.n[2], S::PX, S::PY, S::PZ, 4) ||
        !make_tensor_map_3d(&m[2 * c + 1], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, vel + 3 * C.offset, 3ull * sx,
                            (uint64_t)C.n[1], (uint64_t)C.n[2], 3 * S::VX, S::VY, S::VZ, 4)) {
      dcell_set_error(DCELL_ERR_CUDA, "cuTensorMapEncodeTiled failed for cell %d", c);
      return DCELL_ERR_CUDA;
    }
  }
  return DCELL_OK;
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
bool make_tensor_map_3d(CUtensorMap *m, CUtensorMapDataType type, const void *base, uint64_t dx, uint64_t dy,
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

// The TMA brick path applies to dense 3D grids with nx % 4 == 0 (16-byte row
// strides), 16-byte aligned bases and at least one box per axis.
bool tc_brick_applicable(const Geom &g, const void *phi0s, const void *vel) {
  using S = tc::BrickShape<2>;
  return g.nz >= S::PZ && g.ny >= S::PY && g.nx >= S::PX && g.nx % 4 == 0 && ((uintptr_t)phi0s % 16) == 0 &&
         ((uintptr_t)vel % 16) == 0 && encode_tiled() != nullptr;
}

template <int P>
static int launch_brick(const Geom &g, const uint32_t *phi0s, const float *vel, double dt, int backtrace, float *phi,
                        uint32_t *phis, int *flags, cudaStream_t st, const TcSlab *slab) {
  using S = tc::BrickShape<P>;
  static bool configured = false;
  if (!configured) {
    DCELL_CUDA_CHECK(cudaFuncSetAttribute(tc::sl_tc_brick_kernel<DCELL_EULER, P, true>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, S::DynSmem));
    DCELL_CUDA_CHECK(cudaFuncSetAttribute(tc::sl_tc_brick_kernel<DCELL_MIDPOINT, P, true>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, S::DynSmem));
    DCELL_CUDA_CHECK(cudaFuncSetAttribute(tc::sl_tc_brick_kernel<DCELL_EULER, P, false>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, S::DynSmem));
    DCELL_CUDA_CHECK(cudaFuncSetAttribute(tc::sl_tc_brick_kernel<DCELL_MIDPOINT, P, false>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, S::DynSmem));
    configured = true;
  }
  CUtensorMap tm_phi, tm_vel;
  if (!make_tensor_map_3d(&tm_phi, CU_TENSOR_MAP_DATA_TYPE_UINT32, phi0s, (uint64_t)g.nx, (uint64_t)g.ny, (uint64_t)g.nz,
                S::PX, S::PY, S::PZ, 4) ||
      !make_tensor_map_3d(&tm_vel, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, vel, 3ull * g.nx, (uint64_t)g.ny, (uint64_t)g.nz,
                3 * S::VX, S::VY, S::VZ, 4)) {
    dcell_set_error(DCELL_ERR_CUDA, "cuTensorMapEncodeTiled failed for the TMA brick path");
    return DCELL_ERR_CUDA;
  }
  BrickGrid bg;
  bg.nbx = (g.nx + S::BX - 1) / S::BX;
  bg.nby = (g.ny + S::BY - 1) / S::BY;
  bg.nbz = (g.nz + S::BZ - 1) / S::BZ;
  bg.bz0 = 0;
  if (slab) {  // z bricks [bz0, bz0 + nbz) only
    bg.bz0 = slab->bz0;
    bg.nbz = slab->nbz;
  }
  const long long nbricks = (long long)bg.nbx * bg.nby * bg.nbz;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  long long grid = (long long)S::CtasPerSm * sms;
  if (grid > nbricks) grid = nbricks;
  const bool mid = backtrace == DCELL_MIDPOINT, split = phis != nullptr;
  auto kern = mid ? (split ? tc::sl_tc_brick_kernel<DCELL_MIDPOINT, P, true> : tc::sl_tc_brick_kernel<DCELL_MIDPOINT, P, false>)
                  : (split ? tc::sl_tc_brick_kernel<DCELL_EULER, P, true> : tc::sl_tc_brick_kernel<DCELL_EULER, P, false>);
  kern<<<(int)grid, tc::kBrickThreads, S::DynSmem, st>>>(tm_phi, tm_vel, g, bg, phi0s, vel, (float)dt, phi, phis,
                                                          flags, slab ? slab->gate_maxw : nullptr,
                                                          slab ? slab->gate_limit : 0.f);
  return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
}

int launch_sl_tc_brick(const Geom &g, const uint32_t *phi0s, const float *vel, double dt, int backtrace, float *phi,
                       uint32_t *phis, int *flags, cudaStream_t st) {
  return launch_brick<2>(g, phi0s, vel, dt, backtrace, phi, phis, flags, st, nullptr);
}

int tc_slab_planes() { return tc::BrickShape<2>::BZ; }

int launch_sl_tc_slab(const Geom &g, const uint32_t *phi0s, const float *vel, double dt, int backtrace, float *phi,
                      uint32_t *phis, int *flags, cudaStream_t st, const TcSlab &slab) {
  return launch_brick<2>(g, phi0s, vel, dt, backtrace, phi, phis, flags, st, &slab);
}

int launch_sl_tc_split_planes(const Geom &g, const uint32_t *phi0s, const float *vel, double dt, int backtrace,
                              float *phi, uint32_t *phis, int *flags, cudaStream_t st, int bz0, int nbz) {
  const TcSlab slab{bz0, nbz, nullptr, 0.f};
  return launch_brick<2>(g, phi0s, vel, dt, backtrace, phi, phis, flags, st, &slab);
}

int launch_wait_timeout_check(int *result, cudaStream_t st) {
  tc::wait_timeout_check_kernel<<<1, 32, 0, st>>>(result);
  return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
}

int launch_tc_gemm_check(const float *A, float *D, int *flags, cudaStream_t st) {
  DCELL_CUDA_CHECK(
      cudaFuncSetAttribute(tc::tc_gemm_check_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kDynSmem));
  tc::tc_gemm_check_kernel<<<1, tc::kTile, tc::kDynSmem, st>>>(A, D, flags);
  return cudaGetLastError() == cudaSuccess ? DCELL_OK : DCELL_ERR_CUDA;
}
