// Split-precision tensor-core spreader (type 1, 2D, complex64 data).
//
// For one tile of the oversampled grid the spread is a dense contraction
//     subgrid[u][v] = sum_p ku_p[u - ou_p] * c_p * kv_p[v - ov_p]
//                   = (Ku^T diag(c) Kv)[u][v]
// over the points p of the tile.  It runs on the 5th-generation tensor cores
// (tcgen05.mma, kind::f16, FP32 accumulation in tensor memory) with every
// operand split into FP16 hi + lo parts, x = hi + lo, so that
//     A.B ~= Ahi.Bhi + Ahi.Blo + Alo.Bhi
// keeps ~22 significant bits.  One MMA does all three products and both
// complex parts at once:
//     A (M=128 x K=16 points) rows = [Re(c)ku hi | Im(c)ku hi | Re(c)ku lo | Im(c)ku lo] x 32
//     B (K=16 x N=48)         cols = [kv hi | kv lo] x 24
//     D (128 x 48, FP32, TMEM):  Re = D[0:24, 0:24] + D[0:24, 24:48] + D[64:88, 0:24]
//                                Im = D[32:56, 0:24] + D[32:56, 24:48] + D[96:120, 0:24]
// (the Alo.Blo block is computed and ignored).  A 32x32 tile (DUCC's 2D
// single-precision tile) is split into four 16x16 quadrants, each with its own
// accumulator, so a point's 8 taps always fit the 24 rows/columns of a quadrant.
// Operands are built per point in registers (Horner weights, FP16 hi/lo split,
// funnel-shift placement at the point's row offset) and stored MN-major into
// shared memory; two operand stages let the CUDA cores build one round of
// K-blocks while the tensor cores consume the previous one.  Results are
// combined in shared memory and added to the grid with vector atomics.
//
// Values are scaled by a power of two per chunk (largest |Re|,|Im| -> 2^14)
// so FP16 neither overflows nor loses the small kernel tails to underflow; the
// scale is removed exactly in the epilogue.
#include <cuda_fp16.h>

#include "common.cuh"
#include "kernels.h"
#include "spread_impl.cuh"

namespace dnufft {

namespace tc {

constexpr int THREADS = 128;       // one warpgroup: TMEM lanes 0..127
constexpr int KB = 16;             // points per MMA (K)
constexpr int ROUND = 8;           // K-blocks per round (one operand stage)
constexpr int A_BYTES = 4096;      // 128 x 16 fp16, MN-major, no swizzle
constexpr int B_BYTES = 1536;      // 48 x 16 fp16, MN-major, no swizzle
constexpr int A_LBO = 2048;        // between the two K-groups of 8 points
constexpr int B_LBO = 768;
constexpr int SBO = 128;           // between consecutive 8-element MN chunks
constexpr int M = 128, N = 48;
constexpr int TMEM_COLS = 256;     // quadrant q accumulates at column 64*q
constexpr int MAXCHUNK = 1024;
constexpr int STAGE_BYTES = ROUND * (A_BYTES + B_BYTES);   // 45056
// shared memory: 2 operand stages (each descriptor reads only its own 4 KB /
// 1.5 KB block: 16 resp. 6 chunks of 128 B at SBO, 2 K-groups at LBO)
constexpr int OPER_BYTES = 2 * STAGE_BYTES;
// + the FP32 combine planes (re, im), 2 x 40 x 41 floats
constexpr int SMEM_BYTES = OPER_BYTES + 2 * 40 * 41 * 4;
constexpr uint32_t SPIN_LIMIT = 1u << 26;

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

// bounded wait for the phase with the given parity; returns false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  uint32_t addr = smem_u32(bar);
  for (uint32_t it = 0; it < SPIN_LIMIT; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(addr), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
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

__device__ __forceinline__ uint32_t pack_half2(float a, float b) {
  __half2 h = __floats2half2_rn(a, b);
  return *reinterpret_cast<uint32_t *>(&h);
}

// x = hi + lo in FP16
__device__ __forceinline__ void split(float x, float &hi, float &lo) {
  hi = __half2float(__float2half_rn(x));
  lo = x - hi;
}

// 8 halves (4 words) shifted up by r halves (0..7) across two 8-half chunks:
// z[0..3] = low chunk, z[4..7] = high chunk
__device__ __forceinline__ void place8(const uint32_t (&h)[4], int r, uint32_t (&z)[8]) {
  const uint32_t bs = (r & 1) ? 16u : 0u;
  uint32_t x[5];
  x[0] = __funnelshift_l(0u, h[0], bs);
  x[1] = __funnelshift_l(h[0], h[1], bs);
  x[2] = __funnelshift_l(h[1], h[2], bs);
  x[3] = __funnelshift_l(h[2], h[3], bs);
  x[4] = __funnelshift_l(h[3], 0u, bs);
  const int ws = r >> 1;
  uint32_t y[8];
  // shift by two words if ws&2
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    uint32_t a = (j < 5) ? x[j] : 0u;
    uint32_t b = (j >= 2 && j - 2 < 5) ? x[j - 2] : 0u;
    y[j] = (ws & 2) ? b : a;
  }
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    uint32_t b = (j >= 1) ? y[j - 1] : 0u;
    z[j] = (ws & 1) ? b : y[j];
  }
}

__device__ __forceinline__ void st_v4(uint32_t saddr, uint32_t a, uint32_t b, uint32_t c,
                                      uint32_t d) {
  asm volatile("st.shared.v4.b32 [%0], {%1,%2,%3,%4};" ::"r"(saddr), "r"(a), "r"(b), "r"(c),
               "r"(d)
               : "memory");
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

// 384 threads in three builder groups of 128, one point slot each:
//   group 0: A rows of Re(c)*ku (hi and lo parts), group 1: A rows of
//   Im(c)*ku, group 2: the B row kv (hi and lo) - balanced work per thread.
// The points of a chunk arrive ordered by tile quadrant (the sort key carries
// the quadrant in its two low bits), so every K-block of 16 consecutive points
// of one quadrant feeds one MMA into that quadrant's accumulator.  The
// tensor-memory accumulators are added into FP32 shared-memory planes and
// restarted once one of them has taken DRAIN_AT
// MMAs, which bounds the length of each tensor-core accumulation chain (and
// with it the accumulation error); typical chunks never need a drain.
constexpr int TC_GROUPS = 3;
constexpr int DRAIN_AT = 24;   // drain when an accumulator has taken this many MMAs

template <int W>
__device__ __forceinline__ void tc_drain(uint32_t tmem, int warp, int lane, const int *s_dirty,
                                         float *tre, float *tim, int P, float unscale) {
  constexpr int S = 32 + W;
  for (int q = 0; q < 4; ++q) {
    if (!s_dirty[q]) continue;
    uint32_t d0[16], d1[16], d2[16];
    const uint32_t ta = tmem + (uint32_t(32 * warp) << 16) + uint32_t(64 * q);
    tc::tmem_ld16(ta, d0);
    tc::tmem_ld16(ta + 16, d1);
    tc::tmem_ld16(ta + 32, d2);
    tc::tmem_wait_ld();
    const int u = lane;
    const int tu = u + ((q & 2) ? 16 : 0);
    const int tv0 = (q & 1) ? 16 : 0;
    if (u < 24 && tu < S) {
      float *dst = ((warp & 1) ? tim : tre) + tu * P + tv0;
#pragma unroll
      for (int v = 0; v < 24; ++v) {
        float val = __uint_as_float(v < 16 ? d0[v] : d1[v - 16]);
        if (warp < 2) val += __uint_as_float(v + 24 < 32 ? d1[v + 8] : d2[v - 8]);
        if (tv0 + v < S) atomicAdd(dst + v, val * unscale);
      }
    }
  }
}

template <typename Tc, int W>
__global__ void __launch_bounds__(TC_GROUPS * tc::THREADS, 2)
    k_spread_tc(PointsDesc pts, const uint32_t *__restrict__ skeys, const Chunk *__restrict__ chunks,
                Geometry g, KernelPoly<float> kp, const float2 *__restrict__ values, int64_t vs,
                const unsigned *__restrict__ absmax, float2 *__restrict__ grid,
                int *__restrict__ err) {
  using namespace tc;
  static_assert(W <= 8, "tensor-core spreader handles supports up to 8");
  constexpr int NT = TC_GROUPS * THREADS;
  constexpr int S = 32 + W;   // tile buffer side (rows 0..32+W-2 used)
  constexpr int P = S | 1;    // odd pitch of the FP32 planes (conflict-free rows)
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  __shared__ uint64_t bars[2];
  __shared__ uint32_t s_tmem;
  __shared__ int s_first[5], s_cnt[4], s_blk[5];
  __shared__ int s_dirty[4];
  __shared__ int s_fail;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int grp = tid / THREADS;            // 0: Re A, 1: Im A, 2: B
  const int slot = tid - grp * THREADS;
  const Chunk ch = chunks[blockIdx.x];
  const int cnt = int(ch.count);
  int b0[2];
  {
    const int ntv = int(g.ntiles[1]);
    const int tile = int(ch.tile);
    b0[0] = ((tile / ntv) << g.log2tile) - g.nsafe;
    b0[1] = ((tile % ntv) << g.log2tile) - g.nsafe;
  }
  unsigned char *oper = tc_smem;
  float *tre = reinterpret_cast<float *>(tc_smem + OPER_BYTES);
  float *tim = tre + S * P;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"(smem_u32(&s_tmem)), "r"(uint32_t(TMEM_COLS)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_fail = 0;
  }
  if (tid < 5) s_first[tid] = cnt;
  if (tid < 4) s_dirty[tid] = 0;
  for (int c = tid; c < 2 * S * P; c += NT) tre[c] = 0.f;
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;

  // ---- quadrant segments of the (quadrant-sorted) chunk
  for (int i = tid; i < cnt; i += NT) {
    const int q = int(skeys[ch.start + uint32_t(i)] & 3u);
    if (i == 0 || int(skeys[ch.start + uint32_t(i) - 1] & 3u) != q) s_first[q] = i;
  }
  __syncthreads();
  if (tid == 0) {
    for (int q = 3; q >= 0; --q)
      if (s_first[q] == cnt) s_first[q] = s_first[q + 1];
    int acc = 0;
    for (int q = 0; q < 4; ++q) {
      s_cnt[q] = s_first[q + 1] - s_first[q];
      s_blk[q] = acc;
      acc += (s_cnt[q] + KB - 1) / KB;
    }
    s_blk[4] = acc;
  }
  __syncthreads();
  const float maxc = __uint_as_float(*absmax);
  const int NB = s_blk[4];
  const int nrounds = (NB + ROUND - 1) / ROUND;
  bool active = (maxc > 0.f) && isfinite(maxc) && NB > 0;
  int e2 = 0;
  if (active) frexpf(maxc, &e2);
  const float sA = ldexpf(1.f, 14 - e2), sB = 16384.f;
  const float unscale = ldexpf(1.f, e2 - 28);
  const Tc *crd = static_cast<const Tc *>(pts.coord);
  unsigned fresh = 0xFu;   // quadrants whose next MMA overwrites (issuing thread only)
  const int d = (grp == 2) ? 1 : 0;
  const int kbl = slot / KB, e = slot % KB;

  // point data of this thread's slot in round rr (loads only; used one round later)
  auto fetch = [&](int rr, Tc &x, float &sc, int &q, bool &valid) {
    const int kb = rr * ROUND + kbl;
    q = 0;
    valid = false;
    x = Tc(0);
    sc = 0.f;
    if (kb >= NB) return;
#pragma unroll
    for (int qq = 1; qq < 4; ++qq)
      if (kb >= s_blk[qq]) q = qq;
    const int j = (kb - s_blk[q]) * KB + e;
    if (j >= s_cnt[q]) return;
    valid = true;
    const uint32_t i = ch.start + uint32_t(s_first[q] + j);
    const uint32_t pi = pts.perm[i];
    x = pts.sorted ? crd[uint64_t(i) * 2 + d] : crd[int64_t(pi) * pts.cs0 + int64_t(d) * pts.cs1];
    if (grp < 2) {
      const float2 v = values[int64_t(pi) * vs];
      sc = (grp == 0 ? v.x : v.y) * sA;
    } else {
      sc = sB;
    }
  };
  Tc xc = Tc(0);
  float scc = 0.f;
  int qc = 0;
  bool vc = false;
  if (active) fetch(0, xc, scc, qc, vc);
  uint32_t chains = 0;   // MMAs per accumulator since its last drain, 8 bits each (uniform)

  for (int r = 0; active && r < nrounds; ++r) {
    const int s = r & 1;
    bool timed_out = false;
    if (r >= 2) timed_out = !mbar_wait(&bars[s], uint32_t(((r - 2) >> 1) & 1));
    // prefetch the next round's point data
    Tc xn;
    float scn;
    int qn;
    bool vn;
    fetch(r + 1, xn, scn, qn, vn);
    unsigned char *stA = oper + s * STAGE_BYTES;
    unsigned char *stB = stA + ROUND * A_BYTES;
    const int kb = r * ROUND + kbl;
    if (kb < NB) {
      uint32_t hw[2][4];
#pragma unroll
      for (int p = 0; p < 2; ++p)
#pragma unroll
        for (int w = 0; w < 4; ++w) hw[p][w] = 0u;
      int off = 0;
      if (vc) {
        double fr;
        fold<Tc>(xc, g.coordfct[d], int(g.nover[d]), g.shift[d], g.maxi0[d], off, fr);
        off -= b0[d] + (((grp == 2) ? (qc & 1) : (qc & 2)) ? 16 : 0);
        float k[W];
        kernel_weights<float, W>(kp, float(double(W - 1) - 2.0 * fr), k);
        float hv[8], lv[8];
#pragma unroll
        for (int t = 0; t < 8; ++t) split((t < W) ? k[t] * scc : 0.f, hv[t], lv[t]);
#pragma unroll
        for (int w = 0; w < 4; ++w) {
          hw[0][w] = pack_half2(hv[2 * w], hv[2 * w + 1]);
          hw[1][w] = pack_half2(lv[2 * w], lv[2 * w + 1]);
        }
      }
      const int c0 = off >> 3;
      if (grp < 2) {
        // A column of point e: part p rows p*32 + off + a; group g owns
        // parts g (hi) and g+2 (lo)
        const uint32_t base = smem_u32(stA + kbl * A_BYTES) + (e & 7) * 16 + (e >> 3) * A_LBO;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          uint32_t z[8];
          place8(hw[h], off & 7, z);
          const uint32_t pb = base + uint32_t((grp + 2 * h) * 4) * SBO;
          st_v4(pb + uint32_t(c0) * SBO, z[0], z[1], z[2], z[3]);
          st_v4(pb + uint32_t(c0 + 1) * SBO, z[4], z[5], z[6], z[7]);
          st_v4(pb + uint32_t(c0 == 0 ? 2 : 0) * SBO, 0u, 0u, 0u, 0u);
          st_v4(pb + 3u * SBO, 0u, 0u, 0u, 0u);
        }
      } else {
        // B row of point e: part h columns h*24 + off + b
        const uint32_t base = smem_u32(stB + kbl * B_BYTES) + (e & 7) * 16 + (e >> 3) * B_LBO;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          uint32_t z[8];
          place8(hw[h], off & 7, z);
          const uint32_t pb = base + uint32_t(h * 3) * SBO;
          st_v4(pb + uint32_t(c0) * SBO, z[0], z[1], z[2], z[3]);
          st_v4(pb + uint32_t(c0 + 1) * SBO, z[4], z[5], z[6], z[7]);
          st_v4(pb + uint32_t(c0 == 0 ? 2 : 0) * SBO, 0u, 0u, 0u, 0u);
        }
      }
    }
    fence_proxy_async();
    tc_fence_before();
    if (__syncthreads_or(timed_out ? 1 : 0)) {
      if (tid == 0) atomicExch(err, 1);
      s_fail = 1;
      active = false;
      break;
    }
    // this round's K-blocks per accumulator (computed identically by all threads)
    int maxchain = 0;
    for (int bb = 0; bb < ROUND; ++bb) {
      const int k = r * ROUND + bb;
      if (k >= NB) break;
      int q = 0;
      for (int qq = 1; qq < 4; ++qq)
        if (k >= s_blk[qq]) q = qq;
      if (tid == 0) {
        if (bb == 0) tc_fence_after();
        const uint64_t ad = make_desc(smem_u32(stA + bb * A_BYTES), A_LBO, SBO);
        const uint64_t bd = make_desc(smem_u32(stB + bb * B_BYTES), B_LBO, SBO);
        mma_f16(tmem + uint32_t(64 * q), ad, bd, ((fresh >> q) & 1u) ? 0u : 1u);
        fresh &= ~(1u << q);
        s_dirty[q] = 1;
      }
      chains += 1u << (8 * q);
      maxchain = max(maxchain, int((chains >> (8 * q)) & 0xFFu));
    }
    if (tid == 0) mma_commit(&bars[s]);
    // bound the tensor-core accumulation chains: drain into the FP32 planes
    if (maxchain >= DRAIN_AT && r != nrounds - 1) {
      const bool to2 = !mbar_wait(&bars[s], uint32_t((r >> 1) & 1));
      tc_fence_before();
      if (__syncthreads_or(to2 ? 1 : 0)) {
        if (tid == 0) atomicExch(err, 1);
        s_fail = 1;
        active = false;
        break;
      }
      tc_fence_after();
      if (warp < 4) tc_drain<W>(tmem, warp, lane, s_dirty, tre, tim, P, unscale);
      tc_fence_before();
      __syncthreads();
      if (tid == 0) {
        fresh = 0xFu;
        for (int q = 0; q < 4; ++q) s_dirty[q] = 0;
      }
      chains = 0;
    }
    xc = xn;
    scc = scn;
    qc = qn;
    vc = vn;
  }

  // ---- wait for the last round's MMAs (a commit covers all earlier ones)
  if (active) {
    const int last = nrounds - 1;
    if (!mbar_wait(&bars[last & 1], uint32_t((last >> 1) & 1))) {
      atomicExch(err, 1);
      s_fail = 1;
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (s_fail) active = false;

  // ---- epilogue: remaining accumulators into the planes, then the grid
  if (active) {
    if (warp < 4) tc_drain<W>(tmem, warp, lane, s_dirty, tre, tim, P, unscale);
    __syncthreads();
    const int nu = int(g.nover[0]), nv = int(g.nover[1]);
    for (int c = tid; c < S * S; c += NT) {
      const int a = c / S, bcol = c - (c / S) * S;
      const float2 v = make_float2(tre[a * P + bcol], tim[a * P + bcol]);
      if (v.x == 0.f && v.y == 0.f) continue;
      int gu = b0[0] + a, gv = b0[1] + bcol;
      gu += (gu < 0) ? nu : ((gu >= nu) ? -nu : 0);
      gv += (gv < 0) ? nv : ((gv >= nv) ? -nv : 0);
      atomicAdd(grid + int64_t(gu) * nv + gv, v);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(uint32_t(TMEM_COLS)));
  }
}

bool spread_tc_supported(const Geometry &g, bool calc_f64) {
  return !calc_f64 && g.ndim == 2 && g.log2tile == 5 && g.W <= 8;
}

void launch_spread_tc(const PointsDesc &pts, const uint32_t *skeys, const ChunkList &cl,
                      const Geometry &g, const KernelPoly<float> &kp, const void *values,
                      int64_t vs, void *grid, unsigned *absmax, int *err, cudaStream_t st) {
  if (cl.nchunks == 0) return;
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
    DN_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,             \
                                 tc::SMEM_BYTES));                                              \
    kern<<<cl.nchunks, TC_GROUPS * tc::THREADS, tc::SMEM_BYTES, st>>>(                                  \
        pts, skeys, cl.chunks, g, kp, static_cast<const float2 *>(values), vs, absmax,          \
        static_cast<float2 *>(grid), err);                                                      \
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
