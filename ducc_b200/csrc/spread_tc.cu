// Split-precision tensor-core spreader (type 1, 2D, complex64 data).
//
// For one tile of the oversampled grid the spread is a dense contraction
//     subgrid[u][v] = sum_p ku_p[u - ou_p] * c_p * kv_p[v - ov_p]
//                   = (Ku^T diag(c) Kv)[u][v]
// over the points p of the tile.  It runs on the 5th-generation tensor cores
// (tcgen05.mma, kind::f16, FP32 accumulation in tensor memory) with every
// operand split into FP16 hi + lo parts, x = hi + lo, so that
//     A.B = Ahi.Bhi + Ahi.Blo + Alo.Bhi + Alo.Blo
// keeps ~22 significant bits of each operand.  One MMA does all four products and both
// complex parts at once:
//     A (M=128 x K=16 points) rows: hi block 0..47, row 2u + c = hi part of
//                             c-th component (Re, Im) of Re/Im(c) ku[u]; lo
//                             block 48..95 the same for the lo parts (rows
//                             96..127 stay zero)
//     B (K=16 x N=48)         column 2v + h: part h (hi, lo) of kv[v]
//     D (128 x 48, FP32, TMEM):  Re at window (u, v) = D[2u, 2v] + D[2u, 2v+1]
//                                 + D[48+2u, 2v] + D[48+2u, 2v+1] (Im: rows 2u+1)
// (the Alo.Blo block costs nothing extra: the MMA computes it anyway).
// Interleaving the parts puts each tap of a point in one 32-bit word of its
// operand column (Re and Im of A, hi and lo of B), so a point's taps land at a
// whole-word offset and are placed with word selects only.  A 32x32 tile (DUCC's 2D
// single-precision tile) is split into four 16x16 quadrants with their own
// accumulators, so a point's <= 8 taps always fit the 24 rows/columns of its
// quadrant window.  Points arrive sorted by (tile, quadrant); the plan cuts
// them into K-blocks of <= 16 points of one quadrant of one chunk.
//
// The kernel is persistent (one CTA per SM, a contiguous range of K-blocks
// per CTA, balanced at chunk boundaries) and warp-specialised, every hand-off
// an mbarrier:
//   loader warps (4)   : K-block records, permutation, value gathers (L2-only
//                        loads) and cp.async of the coordinates of one round
//                        (8 K-blocks) into a 16-slot ring;
//   builder warps (8)  : 2 threads per point (A column: Re(c)ku and Im(c)ku, B
//                        row: kv): fold, Horner weights, FP16 hi/lo split,
//                        placement; MN-major operand tiles in 3 stages;
//   MMA warp (1)       : one thread issues the MMAs of a round into the
//                        accumulator of each K-block's quadrant and commits;
//   epilogue warps (4) : read finished accumulators from tensor memory and add
//                        them into FP32 shared-memory planes (no atomics);
//   flusher warps (4)  : add a finished sub-chunk's planes (double-buffered)
//                        to the grid with float2 atomics and zero them.
// Tensor memory holds two accumulator sets (2 x 4 quadrants x 64 columns), so
// the MMA thread continues with the next chunk while the epilogue drains the
// previous one.  An accumulator is also handed to the epilogue once any of its
// quadrants has taken DRAIN_AT MMAs, which bounds each tensor-core
// accumulation chain and with it the accumulation error.
//
// Values are scaled by a global power of two (largest |Re|,|Im| -> 2^14) so
// FP16 neither overflows nor loses the small kernel tails to underflow; the
// scale is removed exactly in the epilogue.
//
// Every wait is bounded (wall clock) and on expiry sets the device error word
// and a shared abort flag that ends every role's loop; the host turns the
// word into DNUFFT_ERR_TIMEOUT.
#include <cuda_fp16.h>

#include "common.cuh"
#include "kernels.h"
#include "spread_impl.cuh"

namespace dnufft {

namespace tc {

constexpr int KB = 16;             // points per MMA (K)
constexpr int ROUND = 8;           // K-blocks per round (one operand stage)
constexpr int NST = 3;             // operand stages
// point-data ring slots (rounds): fewer for float64 coordinates (larger slots)
template <typename Tc> constexpr int npre() { return sizeof(Tc) == 8 ? 12 : 16; }
constexpr int A_BYTES = 4096;      // 128 x 16 fp16, MN-major, no swizzle
constexpr int B_BYTES = 1536;      // 48 x 16 fp16, MN-major, no swizzle
constexpr int A_LBO = 2048;        // between the two K-groups of 8 points
constexpr int B_LBO = 768;
constexpr int SBO = 128;           // between consecutive 8-element MN chunks
constexpr int PART = 3;            // 8-element chunks per operand part (24 rows / columns)
constexpr int M = 128, N = 48;
constexpr int STAGE_BYTES = ROUND * (A_BYTES + B_BYTES);   // 45056
constexpr int TMEM_COLS = 512;     // quadrant q, buffer b at column 128*q + 64*b
constexpr int PL = 40, PP = 41;    // FP32 plane rows, odd pitch
constexpr int PLANE_FLOATS = PL * PP;
#ifndef DNUFFT_TC_DRAIN_AT
#define DNUFFT_TC_DRAIN_AT 24
#endif
constexpr int DRAIN_AT = DNUFFT_TC_DRAIN_AT;   // K-blocks per quadrant per sub-chunk (chain bound)
constexpr uint32_t FLUSH_COST = 16;  // CTA balancing: one sub-chunk flush ~ this many records

// warp roles
constexpr int EPI_W0 = 0, N_EPI = 4;     // warps 0..3: tensor-memory lane quarters 0..3
constexpr int MMA_W0 = 4, N_MMA = 4;     // warp 4+q issues the MMAs of quadrant q
constexpr int LOAD_W0 = 8, N_LOAD = 4;
constexpr int FLUSH_W0 = 12, N_FLUSH = 4;   // planes -> grid
constexpr int BUILD_W0 = 16, N_BUILD = 8;
constexpr int WARPS = BUILD_W0 + N_BUILD;   // 24
constexpr int THREADS = 32 * WARPS;         // 768
constexpr int BUILDERS = 32 * N_BUILD;      // 256 = 2 groups x 128 point slots

// K-block record in global memory: {first sorted point index, meta}
//   meta bits 0-4 points (0..16), 5-6 quadrant, 7 last record of its quadrant
//   in its sub-chunk, 8-31 tile id.  Every sub-chunk has at least one record per
//   quadrant (an empty one, 0 points, if the quadrant has no points there);
//   padding records at the end of a CTA's range are all zero.
constexpr uint32_t META_LAST = 1u << 7;
constexpr int TILE_SHIFT_META = 8;
constexpr uint32_t MAX_TILES = 1u << 24;

// decoded record in the point-data ring
struct KRec {
  uint32_t start;   // first sorted point index
  uint32_t meta;    // as above
  int b0u, b0v;     // grid origin of the quadrant window
};

constexpr unsigned long long WAIT_NS = 2000000000ull;   // 2 s per wait

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= uint64_t((saddr & 0x3FFFFu) >> 4);
  d |= uint64_t((lbo >> 4) & 0x3FFFu) << 16;
  d |= uint64_t((sbo >> 4) & 0x3FFFu) << 32;
  d |= uint64_t(1) << 46;   // descriptor version for sm_100
  return d;                 // base offset 0, relative LBO, no swizzle
}

// kind::f16 instruction descriptor: F32 accumulate, F16 A/B, both MN-major
constexpr uint32_t IDESC = (1u << 4) | (0u << 7) | (0u << 10) | (1u << 15) | (1u << 16) |
                           (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// one potentially blocking test: the thread may be suspended (without taking
// issue slots) for up to the hint while the phase is incomplete
__device__ __forceinline__ bool mbar_try(uint32_t addr, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(addr), "r"(parity), "r"(1000u)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait for the phase with the given parity.  Gives up (returning
// false) when another role has raised the abort flag, or after WAIT_NS, in
// which case it raises the flag and the device error word itself.
__device__ __forceinline__ bool mbar_wait_for(uint64_t *bar, uint32_t parity,
                                              volatile int *abort_flag, int *err,
                                              unsigned long long limit_ns) {
  const uint32_t addr = smem_u32(bar);
  if (mbar_try(addr, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (uint32_t it = 1;; ++it) {
    if (mbar_try(addr, parity)) return true;
    if ((it & 3u) == 0) {
      if (*abort_flag) return false;
      if (global_ns() - t0 > limit_ns) {
        *abort_flag = 1;
        atomicExch(err, 1);
        return false;
      }
    }
  }
}

__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, volatile int *abort_flag,
                                          int *err) {
  return mbar_wait_for(bar, parity, abort_flag, err, WAIT_NS);
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void mma_f16(uint32_t dtmem, uint64_t adesc, uint64_t bdesc,
                                        uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(dtmem), "l"(adesc), "l"(bdesc), "r"(IDESC), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void named_bar(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// named barrier that also returns whether any participating thread passed true
__device__ __forceinline__ bool named_bar_or(int id, int nthreads, bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "barrier.cta.red.or.pred q, %2, %3, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"(v ? 1u : 0u), "r"(id), "r"(nthreads)
      : "memory");
  return r != 0;
}

__device__ __forceinline__ void cp_async(void *dst, const void *src, int bytes) {
  const uint32_t d = smem_u32(dst);
  if (bytes == 16)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
  else if (bytes == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}

__device__ __forceinline__ void cp_async_arrive(uint64_t *bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// hi = RN_fp16(x), lo = RN_fp16(x - hi) for a pair, packed as half2 words
__device__ __forceinline__ void split2(float a, float b, uint32_t &hi, uint32_t &lo) {
  const __half2 h = __floats2half2_rn(a, b);
  const float2 hf = __half22float2(h);
  const __half2 l = __floats2half2_rn(a - hf.x, b - hf.y);
  hi = *reinterpret_cast<const uint32_t *>(&h);
  lo = *reinterpret_cast<const uint32_t *>(&l);
}

// hi = RN_fp16(x) in the low half, lo = RN_fp16(x - hi) in the high half
__device__ __forceinline__ uint32_t split1(float x) {
  const __half h = __float2half_rn(x);
  const __half l = __float2half_rn(x - __half2float(h));
  return uint32_t(__half_as_ushort(h)) | (uint32_t(__half_as_ushort(l)) << 16);
}

// Words d[0..7] of a point's operand column at word offset off (0..16) of a
// 24-word (6-chunk) part: y = the words shifted up by off & 3, written to
// chunks off/4 .. off/4 + 2, zeros to the other three (chunk indices taken
// mod 6, so the six stores cover the part once; for off = 16 the third of
// them is a zero chunk that wraps to chunk 0)
__device__ __forceinline__ void place24(const uint32_t (&d)[8], int off, uint32_t base);

__device__ __forceinline__ void st_v4(uint32_t saddr, uint32_t a, uint32_t b, uint32_t c,
                                      uint32_t d) {
  asm volatile("st.shared.v4.b32 [%0], {%1,%2,%3,%4};" ::"r"(saddr), "r"(a), "r"(b), "r"(c),
               "r"(d)
               : "memory");
}

__device__ __forceinline__ void place24(const uint32_t (&d)[8], int off, uint32_t base) {
  const int r = off & 3, c0 = off >> 2;
  uint32_t x[10], y[12];
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    const uint32_t a = (i < 8) ? d[i] : 0u;
    const uint32_t b = (i >= 2) ? d[i - 2] : 0u;
    x[i] = (r & 2) ? b : a;
  }
#pragma unroll
  for (int i = 0; i < 12; ++i) {
    const uint32_t a = (i < 10) ? x[i] : 0u;
    const uint32_t b = (i >= 1) ? x[i - 1] : 0u;
    y[i] = (r & 1) ? b : a;
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    int c = c0 + k;
    c = (c >= 6) ? c - 6 : c;
    if (k < 3)
      st_v4(base + uint32_t(c) * SBO, y[4 * k], y[4 * k + 1], y[4 * k + 2], y[4 * k + 3]);
    else
      st_v4(base + uint32_t(c) * SBO, 0u, 0u, 0u, 0u);
  }
}

// per-slot layout of the point-data ring
template <typename Tc> struct PreLayout {
  static constexpr int REC = 0;                                     // 8 KRec
  static constexpr int PLAN = ROUND * int(sizeof(KRec));            // 4 x u32 issue plans
  static constexpr int COORD = PLAN + 16;                           // 128 x 2 Tc
  static constexpr int VAL = COORD + ROUND * KB * 2 * int(sizeof(Tc));   // 128 float2
  static constexpr int BYTES = VAL + ROUND * KB * 8;
};

// two sets of the four planes: the epilogue fills one while the flusher warps
// add the other to the grid
constexpr int PLANE_SET_BYTES = 4 * PLANE_FLOATS * 4;
template <typename Tc> constexpr int smem_bytes() {
  return NST * STAGE_BYTES + 2 * PLANE_SET_BYTES + npre<Tc>() * PreLayout<Tc>::BYTES;
}

}  // namespace tc

// Largest |Re|, |Im| over the values (for the power-of-two operand scale).
__global__ void k_absmax(const float2 *__restrict__ values, int64_t vs, uint32_t n,
                         unsigned *__restrict__ out) {
  float m = 0.f;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float2 v = values[int64_t(i) * vs];
    m = fmaxf(m, fmaxf(fabsf(v.x), fabsf(v.y)));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m > 0.f) atomicMax(out, __float_as_uint(m));
}

template <typename Tc, int W>
__global__ void __launch_bounds__(tc::THREADS, 1)
    k_spread_tc(PointsDesc pts, const uint2 *__restrict__ kblk,
                const uint32_t *__restrict__ kb_range, Geometry g, KernelPoly<float> kp,
                const float2 *__restrict__ values, int64_t vs,
                const unsigned *__restrict__ absmax, float2 *__restrict__ grid,
                int *__restrict__ err) {
  using namespace tc;
  static_assert(W <= 8, "tensor-core spreader handles supports up to 8");
  using PL_ = PreLayout<Tc>;
  constexpr int NPRE = npre<Tc>();
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  __shared__ uint64_t full_bar[NST], empty_bar[NST];
  __shared__ uint64_t pre_full[NPRE], pre_empty[NPRE];
  __shared__ uint64_t acc_full[4][2], acc_empty[4][2], done_bar;
  __shared__ uint64_t pl_full[2], pl_empty[2];   // plane sets: epilogue <-> flusher
  __shared__ uint2 pl_info[2];                   // {tile, dirty quadrants | exit bit 8}
  __shared__ uint2 acc_info[4][2];   // {flags (1 dirty, 2 exit), tile}
  __shared__ uint32_t s_tmem;
  __shared__ int s_abort;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t kb0 = kb_range[blockIdx.x], kb1 = kb_range[blockIdx.x + 1];
  const int nrounds = int((kb1 - kb0 + ROUND - 1) / ROUND);
  const float maxc = __uint_as_float(*absmax);
  // nothing to add (no K-blocks, or all values zero): uniform early exit
  if (nrounds == 0 || maxc == 0.f) return;
  int e2 = 0;
  if (isfinite(maxc)) frexpf(maxc, &e2);
  const float sA = ldexpf(1.f, 14 - e2), sB = 16384.f;
  const float unscale = ldexpf(1.f, e2 - 28);

  unsigned char *stages = tc_smem;
  float *planes = reinterpret_cast<float *>(tc_smem + NST * STAGE_BYTES);   // 2 sets
  unsigned char *pre = tc_smem + NST * STAGE_BYTES + 2 * PLANE_SET_BYTES;

  if (warp == MMA_W0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"(smem_u32(&s_tmem)), "r"(uint32_t(TMEM_COLS)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int s = 0; s < NST; ++s) {
      mbar_init(&full_bar[s], BUILDERS);
      mbar_init(&empty_bar[s], N_MMA);
    }
    for (int s = 0; s < NPRE; ++s) {
      mbar_init(&pre_full[s], 33);                  // 32 cp.async arrivals + 1 record arrival
      mbar_init(&pre_empty[s], BUILDERS + N_MMA);   // builders + MMA threads
    }
    for (int q = 0; q < 4; ++q)
      for (int b = 0; b < 2; ++b) {
        mbar_init(&acc_full[q][b], 2);              // MMA commit + MMA thread (info)
        mbar_init(&acc_empty[q][b], 32 * N_EPI);
      }
    mbar_init(&done_bar, N_MMA);
    for (int b = 0; b < 2; ++b) {
      mbar_init(&pl_full[b], 1);
      mbar_init(&pl_empty[b], 32 * N_FLUSH);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_abort = 0;
  }
  // zero the operand stages (A rows 96..127 are never written again) and planes
  {
    const uint32_t zb = smem_u32(tc_smem);
    const int nvec = (NST * STAGE_BYTES + 2 * PLANE_SET_BYTES) / 16;
    for (int i = tid; i < nvec; i += THREADS) st_v4(zb + uint32_t(i) * 16u, 0u, 0u, 0u, 0u);
  }
  fence_proxy_async();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  volatile int *abortp = &s_abort;
  const int ntv = int(g.ntiles[1]);

  if (warp >= LOAD_W0 && warp < LOAD_W0 + N_LOAD) {
    // ------------------------------------------------------------ loaders
    const int lw = warp - LOAD_W0;
    const Tc *crd = static_cast<const Tc *>(pts.coord);
    auto load_rec = [&](int r) -> uint2 {
      uint2 v = make_uint2(0u, 0u);
      if (r < nrounds && lane < ROUND) {
        const uint32_t k = kb0 + uint32_t(r) * ROUND + uint32_t(lane);
        if (k < kb1) v = kblk[k];
      }
      return v;
    };
    uint2 rec_next = load_rec(lw);
    for (int r = lw; r < nrounds; r += N_LOAD) {
      const uint2 rec = rec_next;
      rec_next = load_rec(r + N_LOAD);   // in flight during this round
      uint32_t idx[4], pj[4];
      bool ok[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int p = lane + 32 * j, kbl = p >> 4, e = p & 15;
        const uint32_t st = __shfl_sync(0xffffffffu, rec.x, kbl);
        const uint32_t np = __shfl_sync(0xffffffffu, rec.y, kbl) & 31u;
        ok[j] = uint32_t(e) < np;
        idx[j] = st + uint32_t(e);
        pj[j] = ok[j] ? pts.perm[idx[j]] : 0u;
      }
      // values: gathered through the permutation with loads cached in L2
      // only (a miss brings one 32-byte sector, not a whole L1 line), in
      // flight while the loader waits for its ring slot
      float2 vv[4];
#pragma unroll
      for (int j = 0; j < 4; ++j)
        vv[j] = ok[j] ? __ldcg(values + int64_t(pj[j]) * vs) : make_float2(0.f, 0.f);
      const int slot = r % NPRE;
      if (r >= NPRE && !mbar_wait(&pre_empty[slot], uint32_t((r / NPRE - 1) & 1), abortp, err))
        break;
      unsigned char *sl = pre + slot * PL_::BYTES;
      if (lane < ROUND) {
        KRec kr;
        kr.start = rec.x;
        kr.meta = rec.y;
        const int tile = int(rec.y >> TILE_SHIFT_META), q = int((rec.y >> 5) & 3u);
        const int tu = tile / ntv, tv = tile - tu * ntv;
        kr.b0u = (tu << 5) - g.nsafe + ((q & 2) ? 16 : 0);
        kr.b0v = (tv << 5) - g.nsafe + ((q & 1) ? 16 : 0);
        reinterpret_cast<KRec *>(sl + PL_::REC)[lane] = kr;
      }
      {
        // per quadrant: slots with points (bits 0-7) and slots closing the
        // quadrant's sub-chunk event (bits 8-15)
        const uint32_t meta = rec.y;
        const int rq = int((meta >> 5) & 3u);
        const bool has = lane < ROUND && (meta & 31u) != 0u;
        const bool cls = lane < ROUND && (meta & META_LAST) != 0u;
        uint32_t plan[4];
#pragma unroll
        for (int q = 0; q < 4; ++q)
          plan[q] = (__ballot_sync(0xffffffffu, has && rq == q) & 0xFFu) |
                    ((__ballot_sync(0xffffffffu, cls && rq == q) & 0xFFu) << 8);
        if (lane == 0)
          *reinterpret_cast<uint4 *>(sl + PL_::PLAN) = make_uint4(plan[0], plan[1], plan[2], plan[3]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        if (!ok[j]) continue;
        const int p = lane + 32 * j;
        Tc *cdst = reinterpret_cast<Tc *>(sl + PL_::COORD) + 2 * p;
        if (pts.sorted) {
          cp_async(cdst, crd + uint64_t(idx[j]) * 2, 2 * int(sizeof(Tc)));
        } else {
          cp_async(cdst, crd + int64_t(pj[j]) * pts.cs0, int(sizeof(Tc)));
          cp_async(cdst + 1, crd + int64_t(pj[j]) * pts.cs0 + pts.cs1, int(sizeof(Tc)));
        }
        reinterpret_cast<float2 *>(sl + PL_::VAL)[p] = vv[j];
      }
      // the value stores are ordered before lane 0's arrival (release) by
      // this warp barrier
      __syncwarp();
      if (lane == 0) mbar_arrive(&pre_full[slot]);
      cp_async_arrive(&pre_full[slot]);
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
  } else if (warp >= BUILD_W0) {
    // ------------------------------------------------------------ builders
    // Two threads per point: group 0 builds the point's A column (ku times
    // Re(c) and Im(c), hi and lo: four parts), group 1 its B row (kv, hi and lo).
    const int bt = tid - BUILD_W0 * 32;
    const int grp = bt >> 7;   // 0: A column, 1: B row
    const int slot = bt & 127, kbl = slot >> 4, e = slot & 15;
    const int d = grp;
    for (int r = 0; r < nrounds; ++r) {
      const int ps = r % NPRE;
      if (!mbar_wait(&pre_full[ps], uint32_t((r / NPRE) & 1), abortp, err)) break;
      const unsigned char *sl = pre + ps * PL_::BYTES;
      const KRec kr = reinterpret_cast<const KRec *>(sl + PL_::REC)[kbl];
      const int np = int(kr.meta & 31u);
      const bool valid = e < np;
      Tc x = Tc(0);
      float s0 = 0.f, s1 = 0.f;
      if (valid) {
        x = reinterpret_cast<const Tc *>(sl + PL_::COORD)[2 * slot + d];
        if (grp == 0) {
          const float2 v = reinterpret_cast<const float2 *>(sl + PL_::VAL)[slot];
          s0 = v.x * sA;
          s1 = v.y * sA;
        } else {
          s0 = sB;
        }
      }
      mbar_arrive(&pre_empty[ps]);
      // one word per tap: A: (Re, Im) hi in wh, (Re, Im) lo in wl; B: (hi, lo)
      // in wh
      uint32_t wh[8], wl[8];
#pragma unroll
      for (int t = 0; t < 8; ++t) wh[t] = wl[t] = 0u;
      int off = 0;
      if (valid) {
        int i0;
        double fr;
        fold<Tc>(x, g.coordfct[d], int(g.nover[d]), g.shift[d], g.maxi0[d], i0, fr);
        off = i0 - (d ? kr.b0v : kr.b0u);
        float k[W];
        kernel_weights<float, W>(kp, float(double(W - 1) - 2.0 * fr), k);
        if (grp == 0) {
#pragma unroll
          for (int t = 0; t < W; ++t) split2(k[t] * s0, k[t] * s1, wh[t], wl[t]);
        } else {
#pragma unroll
          for (int t = 0; t < W; ++t) wh[t] = split1(k[t] * s0);
        }
      }
      const int s = r % NST;
      if (r >= NST &&
          !mbar_wait(&empty_bar[s], uint32_t((r / NST - 1) & 1), abortp, err))
        break;
      if (np > 0) {
        unsigned char *stA = stages + s * STAGE_BYTES;
        // A column of point e: hi block at rows 0..47 (chunks 0..5), lo block at
        // rows 48..95 (chunks 6..11); B row of point e: columns 0..47
        const uint32_t base =
            grp == 0 ? smem_u32(stA + kbl * A_BYTES) + (e & 7) * 16 + (e >> 3) * A_LBO
                     : smem_u32(stA + ROUND * A_BYTES + kbl * B_BYTES) + (e & 7) * 16 +
                           (e >> 3) * B_LBO;
        if (valid) {
          place24(wh, off, base);
          if (grp == 0) place24(wl, off, base + uint32_t(2 * PART) * SBO);
        } else {
          const int nchunk = grp == 0 ? 4 * PART : 2 * PART;
#pragma unroll
          for (int c = 0; c < 4 * PART; ++c)
            if (c < nchunk) st_v4(base + uint32_t(c) * SBO, 0u, 0u, 0u, 0u);
        }
      }
      fence_proxy_async();
      mbar_arrive(&full_bar[s]);
    }
  } else if (warp >= MMA_W0 && warp < MMA_W0 + N_MMA) {
    // ------------------------------------------------------------ MMA issue
    // Warp 4+q issues every MMA into quadrant q's accumulators (so MMAs into
    // one accumulator keep their order), four issuers in parallel.  Event k of
    // quadrant q (one per sub-chunk) uses tensor-memory buffer k & 1.
    const int q = warp - MMA_W0;
    if (lane == 0) {
      uint32_t k = 0;          // events sent
      bool waited = true;      // buffer k & 1 released by the epilogue
      bool fresh = true, dirty = false;
      bool failed = false;
      auto acquire = [&]() -> bool {
        if (waited) return true;
        if (!mbar_wait(&acc_empty[q][k & 1], ((k >> 1) - 1) & 1u, abortp, err)) return false;
        tc_fence_after();
        waited = true;
        return true;
      };
      for (int r = 0; r < nrounds && !failed; ++r) {
        // the builders waited for the point-data slot before completing
        // full_bar, so its records are visible once full_bar is
        const int ps = r % NPRE;
        const KRec *src = reinterpret_cast<const KRec *>(pre + ps * PL_::BYTES + PL_::REC);
        const int s = r % NST;
        if (!mbar_wait(&full_bar[s], uint32_t((r / NST) & 1), abortp, err)) break;
        tc_fence_after();
        const uint32_t sA_ = smem_u32(stages + s * STAGE_BYTES);
        const uint32_t plan =
            reinterpret_cast<const uint32_t *>(pre + ps * PL_::BYTES + PL_::PLAN)[q];
        uint32_t todo = (plan | (plan >> 8)) & 0xFFu;
        while (todo) {
          const int b = __ffs(todo) - 1;
          todo &= todo - 1;
          if (!acquire()) {
            failed = true;
            break;
          }
          const uint32_t buf = k & 1;
          if ((plan >> b) & 1u) {
            const uint64_t ad = make_desc(sA_ + uint32_t(b * A_BYTES), A_LBO, SBO);
            const uint64_t bd =
                make_desc(sA_ + uint32_t(ROUND * A_BYTES + b * B_BYTES), B_LBO, SBO);
            mma_f16(tmem + uint32_t(128 * q + 64 * buf), ad, bd, fresh ? 0u : 1u);
            fresh = false;
            dirty = true;
          }
          if ((plan >> (8 + b)) & 1u) {
            acc_info[q][buf] = make_uint2(dirty ? 1u : 0u, src[b].meta >> TILE_SHIFT_META);
            mma_commit(&acc_full[q][buf]);
            mbar_arrive(&acc_full[q][buf]);
            ++k;
            waited = (k < 2);
            fresh = true;
            dirty = false;
          }
        }
        mma_commit(&empty_bar[s]);
        mbar_arrive(&pre_empty[ps]);   // records read: release the point-data slot
      }
      // exit record (after the epilogue released the buffer)
      if (*abortp || acquire()) {
        acc_info[q][k & 1] = make_uint2(2u, 0u);
        mma_commit(&acc_full[q][k & 1]);
        mbar_arrive(&acc_full[q][k & 1]);
      }
      // every MMA of this CTA has completed before tensor memory is released
      mma_commit(&done_bar);
      mbar_wait(&done_bar, 0u, abortp, err);
    }
    __syncwarp();
  } else if (warp < EPI_W0 + N_EPI) {
    // ------------------------------------------------------------ epilogue
    // One event per quadrant per sub-chunk, taken in quadrant order: the
    // accumulators are added into the FP32 planes of the current plane set
    // (part p of tensor-memory lane L = 24p + u is row u of plane p).
    // Consecutive sub-chunks of the same tile keep adding into the same set
    // (sub-chunks bound the tensor-memory accumulation chains, not the FP32
    // planes); when the tile changes, the set goes to the flusher warps and the
    // epilogue continues in the other one.  Hand-off h uses set h & 1.
    const int L = tid;                   // tensor-memory lane 0..127
    // lane 48 b + 2 u + c: window row u of part p = 2 b + c (0 Re hi, 1 Im hi,
    // 2 Re lo, 3 Im lo); lanes 96..127 hold nothing
    const int p = (L < 96) ? 2 * (L / 48) + (L & 1) : 4, u = (L % 48) >> 1;
    uint32_t h = 0;                      // plane sets handed to the flusher so far
    bool have = false;                   // set h & 1 holds data of tile cur_tile
    uint32_t cur_tile = 0, cur_dq = 0;   // cur_dq: dirty quadrants of the set
    for (uint32_t k = 0;; ++k) {
      const uint32_t buf = k & 1, par = (k >> 1) & 1;   // tensor-memory buffer of sub-chunk k
      // 'stop' (a failed wait or the exit record) is uniform in a warp, and
      // made uniform across the four warps at each named barrier; the
      // hand-off decisions depend only on acc_info, the same for all warps
      bool stop = false;
#pragma unroll 1
      for (int q = 0; q < 4; ++q) {
        // rows 16..23 are shared by both halves of the quadrants
        if (q == 2 && named_bar_or(1, 32 * N_EPI, stop)) stop = true;
        if (stop) continue;
        const bool ok = __all_sync(0xffffffffu, mbar_wait(&acc_full[q][buf], par, abortp, err));
        if (!ok) {
          stop = true;
          continue;
        }
        tc_fence_after();
        const uint2 info = acc_info[q][buf];
        if (info.x & 2u) {
          stop = true;
          continue;
        }
        if (q == 0 && have && info.y != cur_tile) {
          // a new tile: every warp finished adding into the current set at the
          // previous sub-chunk's barrier; hand it over and move to the other
          // set once the flusher has released it (hand-off h - 2)
          if (L == 0) {
            pl_info[h & 1] = make_uint2(cur_tile, cur_dq);
            mbar_arrive(&pl_full[h & 1]);
          }
          ++h;
          have = false;
          cur_dq = 0;
          if (h >= 2 &&
              !__all_sync(0xffffffffu, mbar_wait(&pl_empty[h & 1], ((h >> 1) - 1) & 1u, abortp, err))) {
            stop = true;
            continue;
          }
        }
        cur_tile = info.y;
        have = true;
        cur_dq |= (info.x & 1u) << q;
        if (info.x & 1u) {
          float *plane = planes + (h & 1) * (4 * PLANE_FLOATS) + (p < 4 ? p : 0) * PLANE_FLOATS;
          uint32_t d0[16], d1[16], d2[16];
          const uint32_t ta = tmem + (uint32_t(32 * warp) << 16) + uint32_t(128 * q + 64 * buf);
          tmem_ld16(ta, d0);
          tmem_ld16(ta + 16, d1);
          tmem_ld16(ta + 32, d2);
          tmem_wait_ld();
          if (p < 4) {
            float *dst = plane + (u + ((q & 2) ? 16 : 0)) * PP + ((q & 1) ? 16 : 0);
#pragma unroll
            for (int v = 0; v < 24; ++v) {
              // columns 2v (kv hi) and 2v + 1 (kv lo): hi.hi + hi.lo in the
              // hi rows, lo.hi + lo.lo in the lo rows
              const int a = 2 * v, b = 2 * v + 1;
              const float val = __uint_as_float(a < 16 ? d0[a] : (a < 32 ? d1[a - 16] : d2[a - 32])) +
                                __uint_as_float(b < 16 ? d0[b] : (b < 32 ? d1[b - 16] : d2[b - 32]));
              dst[v] += val;
            }
          }
        }
        tc_fence_before();
        mbar_arrive(&acc_empty[q][buf]);
      }
      const bool fin = named_bar_or(1, 32 * N_EPI, stop);
      if (fin) {
        // hand over the last data, then tell the flusher to stop (in a set it
        // has released)
        if (have) {
          if (L == 0) {
            pl_info[h & 1] = make_uint2(cur_tile, cur_dq);
            mbar_arrive(&pl_full[h & 1]);
          }
          ++h;
          if (h >= 2) mbar_wait(&pl_empty[h & 1], ((h >> 1) - 1) & 1u, abortp, err);
        }
        if (L == 0) {
          pl_info[h & 1] = make_uint2(0u, 0x100u);
          mbar_arrive(&pl_full[h & 1]);
        }
        break;
      }
    }
  }
  if (warp >= FLUSH_W0 && warp < FLUSH_W0 + N_FLUSH) {
    // ------------------------------------------------------------ flusher
    // Hand-off k's planes (set k & 1) -> grid with float2 atomics, zeroing
    // them for hand-off k + 2.  Only the dirty quadrants' windows hold data.
    const int L = tid - FLUSH_W0 * 32;
    const int S = 32 + W;
    const int nu = int(g.nover[0]), nv = int(g.nover[1]);
    for (uint32_t k = 0;; ++k) {
      const uint32_t buf = k & 1;
      if (!mbar_wait(&pl_full[buf], (k >> 1) & 1u, abortp, err)) break;
      const uint2 info = pl_info[buf];
      if (info.y & 0x100u) break;
      const uint32_t dq = info.y;
      const float *pls = planes + buf * (4 * PLANE_FLOATS);
      float *plw = planes + buf * (4 * PLANE_FLOATS);
      const int tu = int(info.x) / ntv, tv = int(info.x) - tu * ntv;
      const int b0u = (tu << 5) - g.nsafe, b0v = (tv << 5) - g.nsafe;
      const int r0 = (dq & 3u) ? 0 : 16, r1 = min((dq & 12u) ? 40 : 24, S);
      const int c0 = (dq & 5u) ? 0 : 16, c1 = min((dq & 10u) ? 40 : 24, S);
      // thread -> one column of the box and every nph-th row: the column's
      // wrapped index once, rows wrapped incrementally, no divisions per cell
      const int bw = c1 - c0, nph = (32 * N_FLUSH) / bw;
      if (dq != 0 && L < nph * bw) {
        const int col = c0 + L % bw;
        const int gv = wrapi(b0v + col, nv);
        int a = r0 + L / bw;
        int gu = wrapi(b0u + a, nu);
#pragma unroll 4
        for (; a < r1; a += nph) {
          const int o = a * PP + col;
          const float re = pls[o] + pls[2 * PLANE_FLOATS + o];
          const float im = pls[PLANE_FLOATS + o] + pls[3 * PLANE_FLOATS + o];
          plw[o] = 0.f;
          plw[PLANE_FLOATS + o] = 0.f;
          plw[2 * PLANE_FLOATS + o] = 0.f;
          plw[3 * PLANE_FLOATS + o] = 0.f;
          if (re != 0.f || im != 0.f)
            atomicAdd(grid + int64_t(gu) * nv + gv, make_float2(re * unscale, im * unscale));
          gu += nph;
          gu -= (gu >= nu) ? nu : 0;
        }
      }
      mbar_arrive(&pl_empty[buf]);
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == MMA_W0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(uint32_t(TMEM_COLS)));
  }
}

// ---------------------------------------------------------------- K-block lists
// A chunk (consecutive sorted points of one tile, ordered by quadrant and, in
// each quadrant, by cell in Morton order) is cut
// into sub-chunks with at most DRAIN_AT K-blocks per quadrant, which bounds
// every tensor-core accumulation chain; a sub-chunk is one accumulator event
// per quadrant and one flush of the tile planes.  Inside a sub-chunk the
// records take the quadrants in turn, so the four MMA issuers share each round.
__device__ __forceinline__ void tc_chunk_bounds(const uint32_t *__restrict__ skeys, const Chunk &ch,
                                                int cell_bits, uint32_t (&b)[5]) {
  b[0] = ch.start;
  b[4] = ch.start + ch.count;
  for (uint32_t q = 1; q < 4; ++q) {
    uint32_t lo = b[q - 1], hi = b[4];
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (((skeys[mid] >> cell_bits) & 3u) < q) lo = mid + 1;
      else hi = mid;
    }
    b[q] = lo;
  }
}

__device__ __forceinline__ uint32_t tc_subchunks(const uint32_t (&kq)[4]) {
  uint32_t m = 0;
  for (int q = 0; q < 4; ++q) m = max(m, (kq[q] + tc::DRAIN_AT - 1) / tc::DRAIN_AT);
  return max(m, 1u);
}

// Per chunk: the first sorted index of quadrants 1..3 (binary search on the
// quadrant bits of the sorted keys) and the number of records.
__global__ void k_tc_count(const uint32_t *__restrict__ skeys, const Chunk *__restrict__ chunks,
                           uint32_t nch, int cell_bits, uint4 *__restrict__ qb,
                           uint32_t *__restrict__ nrec, uint32_t *__restrict__ cost) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nch) return;
  const Chunk ch = chunks[c];
  uint32_t b[5];
  tc_chunk_bounds(skeys, ch, cell_bits, b);
  uint32_t kq[4];
  for (int q = 0; q < 4; ++q) kq[q] = (b[q + 1] - b[q] + tc::KB - 1) / tc::KB;
  const uint32_t S = tc_subchunks(kq);
  uint32_t n = 0;
  for (uint32_t j = 0; j < S; ++j)
    for (int q = 0; q < 4; ++q) {
      const uint32_t done = j * tc::DRAIN_AT;
      const uint32_t m = kq[q] > done ? min(kq[q] - done, uint32_t(tc::DRAIN_AT)) : 0u;
      n += max(m, 1u);
    }
  qb[c] = make_uint4(b[1], b[2], b[3], b[4]);
  nrec[c] = n;
  cost[c] = n + tc::FLUSH_COST * S;
}

__global__ void k_tc_emit(const Chunk *__restrict__ chunks, const uint4 *__restrict__ qb,
                          const uint32_t *__restrict__ kbpos, uint32_t nch,
                          uint2 *__restrict__ kblk) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nch) return;
  const Chunk ch = chunks[c];
  const uint4 q4 = qb[c];
  const uint32_t b[5] = {ch.start, q4.x, q4.y, q4.z, q4.w};
  uint32_t kq[4];
  for (int q = 0; q < 4; ++q) kq[q] = (b[q + 1] - b[q] + tc::KB - 1) / tc::KB;
  const uint32_t S = tc_subchunks(kq);
  const uint32_t tbits = ch.tile << tc::TILE_SHIFT_META;
  uint32_t k = kbpos[c];
  for (uint32_t j = 0; j < S; ++j) {
    uint32_t m[4], cnt[4], mx = 0;
    for (int q = 0; q < 4; ++q) {
      const uint32_t done = j * tc::DRAIN_AT;
      m[q] = kq[q] > done ? min(kq[q] - done, uint32_t(tc::DRAIN_AT)) : 0u;
      cnt[q] = max(m[q], 1u);
      mx = max(mx, cnt[q]);
    }
    for (uint32_t i = 0; i < mx; ++i)
      for (uint32_t q = 0; q < 4; ++q) {
        if (i >= cnt[q]) continue;
        const uint32_t last = (i + 1 == cnt[q]) ? tc::META_LAST : 0u;
        if (m[q] == 0) {
          kblk[k++] = make_uint2(0u, (q << 5) | last | tbits);   // empty quadrant
        } else {
          const uint32_t st = b[q] + (j * tc::DRAIN_AT + i) * tc::KB;
          const uint32_t np = min(uint32_t(tc::KB), b[q + 1] - st);
          kblk[k++] = make_uint2(st, np | (q << 5) | last | tbits);
        }
      }
  }
}

// CTA b takes records [range[b], range[b+1]), cut at chunk starts so that the
// CTAs get about equal estimated cost (records + FLUSH_COST per sub-chunk).
__global__ void k_tc_ranges(const uint32_t *__restrict__ kbpos, const uint32_t *__restrict__ cpos,
                            uint32_t nch, uint32_t total, uint32_t ctotal, uint32_t groups,
                            uint32_t *__restrict__ range) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b > groups) return;
  if (b == groups || b == 0) {
    range[b] = (b == 0) ? 0u : total;
    return;
  }
  const uint32_t target = uint32_t((uint64_t(b) * ctotal) / groups);
  uint32_t lo = 0, hi = nch;   // first chunk with cost prefix >= target
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (cpos[mid] < target) lo = mid + 1;
    else hi = mid;
  }
  range[b] = (lo < nch) ? kbpos[lo] : total;
}

size_t tc_kblock_workspace_bytes(uint32_t nch) {
  return size_t(nch) * (sizeof(uint4) + 4 * sizeof(uint32_t)) + scan_workspace_bytes(nch) + 1024;
}

uint32_t tc_kblock_upper_bound(uint32_t npts, uint32_t nch) {
  // per chunk of n points: K-blocks <= n/16 + 4, sub-chunks S <= (n/16 + 1)/24 + 1,
  // and at most 4 empty records per sub-chunk
  return npts / tc::KB + npts / (tc::KB * tc::DRAIN_AT) * 4 + 9 * nch + 16;
}

uint32_t build_tc_kblocks(const uint32_t *skeys, const ChunkList &cl, uint32_t groups, void *ws,
                          uint2 *kblk, uint32_t *range, uint32_t *d_total, int cell_bits,
                          cudaStream_t st) {
  const uint32_t nch = cl.nchunks;
  DN_REQUIRE(nch > 0, ST_INTERNAL, "no chunks");
  uint4 *qb = static_cast<uint4 *>(ws);
  uint32_t *nrec = reinterpret_cast<uint32_t *>(qb + nch);
  uint32_t *pos = nrec + nch;
  uint32_t *cost = pos + nch;
  uint32_t *cpos = cost + nch;
  uint32_t *sws = reinterpret_cast<uint32_t *>(
      (reinterpret_cast<uintptr_t>(cpos + nch) + 255) & ~uintptr_t(255));
  const unsigned gb = (nch + 255) / 256;
  k_tc_count<<<gb, 256, 0, st>>>(skeys, cl.chunks, nch, cell_bits, qb, nrec, cost);
  DN_LAUNCHED();
  exclusive_scan(nrec, pos, nch, sws, st);
  exclusive_scan(cost, cpos, nch, sws, st);
  k_tc_emit<<<gb, 256, 0, st>>>(cl.chunks, qb, pos, nch, kblk);
  DN_LAUNCHED();
  uint32_t h[4] = {0u, 0u, 0u, 0u};
  const uint32_t *src[4] = {pos + nch - 1, nrec + nch - 1, cpos + nch - 1, cost + nch - 1};
  read_words(src, 4, h, st);
  const uint32_t total = h[0] + h[1], ctotal = h[2] + h[3];
  k_tc_ranges<<<(groups + 1 + 255) / 256, 256, 0, st>>>(pos, cpos, nch, total, ctotal, groups,
                                                         range);
  DN_LAUNCHED();
  (void)d_total;
  return total;
}

// Self-test of the failure path of the bounded waits: one warp waits, with the
// spreader's wait routine and a short limit, on an mbarrier that nothing
// arrives at; the routine gives up, raises the abort flag and sets the error
// word, which the host turns into DNUFFT_ERR_TIMEOUT.  No fault, no hang.
__global__ void k_wait_selftest(int *err, unsigned long long limit_ns) {
  __shared__ uint64_t bar;
  __shared__ int abort_flag;
  if (threadIdx.x == 0) {
    tc::mbar_init(&bar, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  tc::mbar_wait_for(&bar, 0u, &abort_flag, err, limit_ns);
}

void launch_wait_selftest(int *err, unsigned long long limit_ns, cudaStream_t st) {
  k_wait_selftest<<<1, 32, 0, st>>>(err, limit_ns);
  DN_LAUNCHED();
}

bool spread_tc_supported(const Geometry &g, bool calc_f64) {
  return !calc_f64 && g.ndim == 2 && g.log2tile == 5 && g.W <= 8 &&
         uint64_t(g.ntiles[0]) * uint64_t(g.ntiles[1]) < uint64_t(tc::MAX_TILES);
}

void launch_spread_tc(const PointsDesc &pts, const TcBlocks &tb, const Geometry &g,
                      const KernelPoly<float> &kp, const void *values, int64_t vs, void *grid,
                      unsigned *absmax, int *err, cudaStream_t st) {
  if (tb.groups == 0 || tb.total == 0) return;
  DN_REQUIRE(spread_tc_supported(g, false), ST_UNSUPPORTED,
             "tensor-core spreader: 2D single precision with support <= 8 only");
  DN_CUDA(cudaMemsetAsync(absmax, 0, sizeof(unsigned), st));
  {
    unsigned nb = unsigned(std::min<uint64_t>((uint64_t(pts.npts) + 255) / 256, 148 * 8));
    k_absmax<<<nb, 256, 0, st>>>(static_cast<const float2 *>(values), vs, pts.npts, absmax);
    DN_LAUNCHED();
  }
#define DN_TC(TC, WW)                                                                           \
  {                                                                                             \
    auto kern = k_spread_tc<TC, WW>;                                                            \
    constexpr int smem = tc::smem_bytes<TC>();                                                  \
    DN_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));     \
    kern<<<tb.groups, tc::THREADS, smem, st>>>(pts, tb.kblk, tb.range, g, kp,                   \
                                               static_cast<const float2 *>(values), vs, absmax, \
                                               static_cast<float2 *>(grid), err);               \
    DN_LAUNCHED();                                                                              \
    return;                                                                                     \
  }
  if (pts.coord_f64) {
    switch (g.W) {
      case 4: DN_TC(double, 4) case 5: DN_TC(double, 5) case 6: DN_TC(double, 6)
      case 7: DN_TC(double, 7) case 8: DN_TC(double, 8)
    }
  } else {
    switch (g.W) {
      case 4: DN_TC(float, 4) case 5: DN_TC(float, 5) case 6: DN_TC(float, 6)
      case 7: DN_TC(float, 7) case 8: DN_TC(float, 8)
    }
  }
#undef DN_TC
  throw Error(ST_UNSUPPORTED, "tensor-core spreader: unsupported kernel support");
}

}  // namespace dnufft
