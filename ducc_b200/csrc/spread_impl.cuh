// Plain spreading (type 1) and interpolation (type 2) kernels.
//
// One CTA per chunk of tile-sorted points (at most CHUNK points of one tile).
// Spreading: every warp takes 32 points at a time, each lane folds its point
// and evaluates the W weights per axis by Horner in registers, stages them in
// shared memory, then the warp walks the 32 points and its lanes cover the
// W^d footprint of one point together (no two lanes touch the same cell), adding
// into a shared-memory copy of the tile plus halo with shared-memory atomics
// (the per-point FP32/FP64 atomics of the plain form).  The tile buffer is
// flushed once with vectorised global atomics at wrapped grid positions.
// Interpolation: the tile plus halo is staged in shared memory and every thread
// evaluates one point (weights in registers, W^d multiply-adds), writing the
// result through the tile permutation.  In 2D a tile that lies inside the grid
// (no periodic wrap) arrives by one TMA tensor copy (cp.async.bulk.tensor.2d,
// issued by one thread, completion on an mbarrier) while the CTA folds and
// orders its first batch of points; tiles at the grid edges are loaded by all
// threads with the wrap.
//
// Mirrors HelperNu2u / spreading_helper and HelperU2nu / interpolation_helper
// (src/ducc0/nufft/nufft.h:917-1272 for 2D, :1391-1729 for 3D, :526-834 for 1D).
#pragma once

#include <cuda.h>   // CUtensorMap (the map is encoded through the runtime's driver entry point)

#include "common.cuh"
#include "kernels.h"

namespace dnufft {

constexpr int SP_THREADS = 256;
constexpr int SP_WARPS = SP_THREADS / 32;

template <int NDIM>
__device__ __forceinline__ void tile_origin(uint32_t tile, const Geometry &g, int (&b0)[NDIM]) {
  const int L = g.log2tile;
  if constexpr (NDIM == 1) {
    b0[0] = (int(tile) << L) - g.nsafe;
  } else if constexpr (NDIM == 2) {
    int ntv = int(g.ntiles[1]);
    b0[0] = ((int(tile) / ntv) << L) - g.nsafe;
    b0[1] = ((int(tile) % ntv) << L) - g.nsafe;
  } else {
    int ntv = int(g.ntiles[1]), ntw = int(g.ntiles[2]);
    int tu = int(tile) / (ntv * ntw), r = int(tile) % (ntv * ntw);
    b0[0] = (tu << L) - g.nsafe;
    b0[1] = ((r / ntw) << L) - g.nsafe;
    b0[2] = ((r % ntw) << L) - g.nsafe;
  }
}

template <typename Tc, int NDIM>
__device__ __forceinline__ uint32_t load_point(const PointsDesc &pts, uint32_t i, Tc (&x)[NDIM]) {
  uint32_t j = pts.perm[i];
  const Tc *c = static_cast<const Tc *>(pts.coord);
  if (pts.sorted) {
#pragma unroll
    for (int d = 0; d < NDIM; ++d) x[d] = c[uint64_t(i) * NDIM + d];
  } else {
#pragma unroll
    for (int d = 0; d < NDIM; ++d) x[d] = c[int64_t(j) * pts.cs0 + int64_t(d) * pts.cs1];
  }
  return j;
}

// per-lane stride of the staged weights: odd, so that the 32 lanes writing
// their own weights hit 32 different banks; even entry count keeps the
// following complex values aligned
template <int NDIM, int W> constexpr int stage_stride() {
  return ((NDIM * W) % 2 == 0) ? NDIM * W + 1 : NDIM * W;
}

template <typename T> struct BufferLayout {
  // does the tile buffer live in shared memory for this (precision, ndim)?
  static constexpr bool smem(int ndim) { return !(ndim == 3 && sizeof(T) == 8); }
};

template <typename T>
__device__ __forceinline__ void global_add(cplx<T> *p, T re, T im) {
  if constexpr (sizeof(T) == 4) {
    atomicAdd(reinterpret_cast<float2 *>(p), make_float2(re, im));
  } else {
    atomicAdd(&p->x, re);
    atomicAdd(&p->y, im);
  }
}

// Periodic wrap without a division is valid where every axis is at least 2S
// long: a tile origin lies in [-W/2, n + W), so its cells' indices stay in
// [-n, 2n).
template <int NDIM> __device__ __forceinline__ bool fast_wrap_ok(const Geometry &g, int S) {
  bool ok = true;
#pragma unroll
  for (int d = 0; d < NDIM; ++d) ok = ok && int(g.nover[d]) >= 2 * S;
  return ok;
}

// grid index of tile cell c (row-major in S^NDIM, c * S < 2^32; mS =
// fastdiv_magic(S)) for the tile at origin b0, wrapped periodically
template <int NDIM>
__device__ __forceinline__ int64_t cell_index(int c, int S, uint32_t mS, bool fastwrap,
                                              const int (&b0)[NDIM], const Geometry &g) {
  int gi[NDIM];
  uint32_t rem = uint32_t(c);
#pragma unroll
  for (int d = NDIM - 1; d >= 0; --d) {
    const uint32_t qd = fastdiv(rem, mS);
    gi[d] = int(rem - qd * uint32_t(S));
    rem = qd;
  }
  int64_t gidx = 0;
#pragma unroll
  for (int d = 0; d < NDIM; ++d) {
    const int nd = int(g.nover[d]);
    gidx = gidx * nd + (fastwrap ? wrap1(b0[d] + gi[d], nd) : wrapi(b0[d] + gi[d], nd));
  }
  return gidx;
}

// One chunk of one transform (the body of k_spread; also used by the
// multi-instance kernel of batched transforms).
template <typename T, typename Tc, int NDIM, int W>
__device__ __forceinline__ void spread_chunk(const PointsDesc &pts, const Chunk ch, const Geometry &g,
                                             const KernelPoly<T> &kp,
                                             const cplx<T> *__restrict__ values, int64_t vs,
                                             cplx<T> *__restrict__ grid, unsigned char *smraw) {
  constexpr bool SMEM = BufferLayout<T>::smem(NDIM);
  constexpr int FP = (NDIM == 1) ? W : (NDIM == 2 ? W * W : W * W * W);
  constexpr int NIT = (FP + 31) / 32;
  constexpr int UNR = NIT <= 8 ? NIT : 4;
  const int S = (1 << g.log2tile) + W;
  int ncell = S;
  if (NDIM >= 2) ncell *= S;
  if (NDIM >= 3) ncell *= S;
  int b0[NDIM];
  tile_origin<NDIM>(ch.tile, g, b0);
  const uint32_t mS = fastdiv_magic(uint32_t(S));
  const bool fastwrap = fast_wrap_ok<NDIM>(g, S);
  cplx<T> *buf = reinterpret_cast<cplx<T> *>(smraw);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned char *stage = smraw + (SMEM ? size_t(ncell) * sizeof(cplx<T>) : 0);
  constexpr int WS = stage_stride<NDIM, W>();   // per-lane weight stride (odd)
  T *stw = reinterpret_cast<T *>(stage) + warp * 32 * WS;
  cplx<T> *stv = reinterpret_cast<cplx<T> *>(reinterpret_cast<T *>(stage) + SP_WARPS * 32 * WS) +
                 warp * 32;
  int *sto = reinterpret_cast<int *>(reinterpret_cast<cplx<T> *>(reinterpret_cast<T *>(stage) +
                                                                 SP_WARPS * 32 * WS) +
                                     SP_WARPS * 32) +
             warp * 32 * NDIM;
  if constexpr (SMEM) {
    for (int c = threadIdx.x; c < ncell; c += SP_THREADS) buf[c] = mkc<T>(T(0), T(0));
    __syncthreads();
  }
  const uint32_t end = ch.start + ch.count;
  // points per warp and round: 32, or fewer for a chunk of fewer than
  // 32 * SP_WARPS points, so that every warp takes a share of a small chunk
  // (each warp walks its points one by one)
  const int pw = min(32, max(1, int((ch.count + SP_WARPS - 1) / SP_WARPS)));
  for (uint32_t base = ch.start + uint32_t(warp * pw); base < end; base += SP_WARPS * pw) {
    uint32_t i = base + lane;
    if (lane < pw && i < end) {
      Tc x[NDIM];
      uint32_t j = load_point<Tc, NDIM>(pts, i, x);
      // a gather through the permutation: cached in L2 only, so a miss
      // brings one 32-byte sector instead of a whole L1 line
      cplx<T> v = __ldcg(values + int64_t(j) * vs);
#pragma unroll
      for (int d = 0; d < NDIM; ++d) {
        int i0;
        double frac;
        fold<Tc>(x[d], g.coordfct[d], int(g.nover[d]), g.shift[d], g.maxi0[d], i0, frac);
        T w[W];
        kernel_weights<T, W>(kp, T(double(W - 1) - 2.0 * frac), w);
#pragma unroll
        for (int a = 0; a < W; ++a) stw[lane * WS + d * W + a] = w[a];
        sto[lane * NDIM + d] = i0 - b0[d];
      }
      stv[lane] = v;
    }
    __syncwarp();
    int np = min(pw, int(end - base));
    for (int p = 0; p < np; ++p) {
      const cplx<T> v = stv[p];
      const T *wp = stw + p * WS;
      int o[NDIM];
#pragma unroll
      for (int d = 0; d < NDIM; ++d) o[d] = sto[p * NDIM + d];
#pragma unroll UNR
      for (int c0 = 0; c0 < FP; c0 += 32) {
        int c = c0 + lane;
        if (FP % 32 == 0 || c < FP) {
          T wt;
          int cell;
          if constexpr (NDIM == 1) {
            wt = wp[c];
            cell = o[0] + c;
          } else if constexpr (NDIM == 2) {
            int a = c / W, b = c - (c / W) * W;
            wt = wp[a] * wp[W + b];
            cell = (o[0] + a) * S + (o[1] + b);
          } else {
            int a = c / (W * W), r = c - a * (W * W), b = r / W, e = r - b * W;
            wt = wp[a] * wp[W + b] * wp[2 * W + e];
            cell = ((o[0] + a) * S + (o[1] + b)) * S + (o[2] + e);
          }
          T re = wt * v.x, im = wt * v.y;
          if constexpr (SMEM) {
            atomicAdd(&buf[cell].x, re);
            atomicAdd(&buf[cell].y, im);
          } else {
            // direct global accumulation at wrapped positions
            global_add<T>(grid + cell_index<NDIM>(cell, S, mS, fastwrap, b0, g), re, im);
          }
        }
      }
    }
    __syncwarp();
  }
  if constexpr (SMEM) {
    __syncthreads();
    for (int c = threadIdx.x; c < ncell; c += SP_THREADS) {
      cplx<T> v = buf[c];
      if (v.x == T(0) && v.y == T(0)) continue;
      global_add<T>(grid + cell_index<NDIM>(c, S, mS, fastwrap, b0, g), v.x, v.y);
    }
  }
}

// four CTAs per SM for single-precision values at float64 coordinates (whose
// exact fold takes many registers): sparse tiles, where the CTAs are short,
// need the warps
template <typename T, typename Tc> constexpr int spread_min_ctas() {
  return (sizeof(T) == 4 && sizeof(Tc) == 8) ? 4 : 1;
}

template <typename T, typename Tc, int NDIM, int W>
__global__ void __launch_bounds__(SP_THREADS, spread_min_ctas<T, Tc>())
    k_spread(PointsDesc pts, const Chunk *__restrict__ chunks, Geometry g, KernelPoly<T> kp,
             const cplx<T> *__restrict__ values, int64_t vs, int64_t vtrans,
             cplx<T> *__restrict__ grid, int64_t gtrans) {
  extern __shared__ __align__(16) unsigned char smraw[];
  spread_chunk<T, Tc, NDIM, W>(pts, chunks[blockIdx.x], g, kp,
                               values + int64_t(blockIdx.y) * vtrans, vs,
                               grid + int64_t(blockIdx.y) * gtrans, smraw);
}

// One chunk of one transform (the body of k_interp; also used by the
// multi-instance kernel of batched transforms).
// scratch of the bank-balanced interpolation order (after the tile buffer)
template <typename T> struct InterpOrder {
  static constexpr int NSLOT = 128 / int(sizeof(cplx<T>));   // 8-/16-byte bank slots
  static constexpr int IB = 512;                             // points per sorted batch
  // slot counters, then per-point records: output index, first cell, kernel
  // argument per axis
  static constexpr size_t bytes(int ndim) { return NSLOT * 4 + IB * (8 + ndim * sizeof(T)); }
};

// Row pitch (cells) of a 2D tile staged by a TMA copy: the copy starts at an
// even grid column (16-byte aligned for complex64), one column before the tile
// when the halo width nsafe is odd, and spans an even number of columns.
__host__ __device__ constexpr int tma_tile_pitch(int S, int nsafe) {
  return (S + (nsafe & 1) + 1) & ~1;
}

__device__ __forceinline__ bool tile_bar_wait(uint64_t *bar, uint32_t parity) {
  const uint32_t addr = static_cast<uint32_t>(__cvta_generic_to_shared(bar));
  unsigned long long t0 = 0;
  for (uint32_t it = 0;; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(addr), "r"(parity), "r"(1000u)
        : "memory");
    if (ok) return true;
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    if (it == 0) t0 = t;
    else if (t - t0 > 1000000000ull) return false;   // one second
  }
}

// One chunk of one transform (the body of k_interp; also used by the
// multi-instance kernel of batched transforms, which passes no tensor map).
// tmap: 2D tensor map of the grid (rows x 2*columns scalars) with box
// (2*tpitch, S); tbar: an mbarrier in shared memory; err: device error word.
template <typename T, typename Tc, int NDIM, int W>
__device__ __forceinline__ void interp_chunk(const PointsDesc &pts, const Chunk ch, const Geometry &g,
                                             const KernelPoly<T> &kp,
                                             const cplx<T> *__restrict__ grid,
                                             cplx<T> *__restrict__ out, int64_t os,
                                             unsigned char *smraw,
                                             const CUtensorMap *tmap = nullptr, int tpitch = 0,
                                             uint64_t *tbar = nullptr, int *err = nullptr) {
  constexpr bool SMEM = BufferLayout<T>::smem(NDIM);
  const int S = (1 << g.log2tile) + W;
  int ncell = S;
  if (NDIM >= 2) ncell *= S;
  if (NDIM >= 3) ncell *= S;
  int b0[NDIM];
  tile_origin<NDIM>(ch.tile, g, b0);
  cplx<T> *buf = reinterpret_cast<cplx<T> *>(smraw);
  // staged tile: row pitch (cells) and column of the tile's first cell
  int pitch = S, sh = 0;
  bool tma = false;
  size_t tile_bytes = size_t(ncell) * sizeof(cplx<T>);
  if constexpr (NDIM == 2 && SMEM) {
    if (tmap) {
      tile_bytes = size_t(tpitch) * size_t(S) * sizeof(cplx<T>);
      const int v0 = b0[1] & ~1;   // even start column (also for negative origins)
      tma = b0[0] >= 0 && b0[0] + S <= int(g.nover[0]) && v0 >= 0 &&
            v0 + tpitch <= int(g.nover[1]);
      if (tma) {
        pitch = tpitch;
        sh = b0[1] - v0;
        if (threadIdx.x == 0) {
          const uint32_t bar = static_cast<uint32_t>(__cvta_generic_to_shared(tbar));
          asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar));
          asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncthreads();
        if (threadIdx.x == 0) {
          const uint32_t bar = static_cast<uint32_t>(__cvta_generic_to_shared(tbar));
          asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                       "r"(uint32_t(tile_bytes))
                       : "memory");
          asm volatile(
              "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
              " [%0], [%1, {%2, %3}], [%4];"
              ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(buf))),
                "l"(reinterpret_cast<uint64_t>(tmap)), "r"(2 * v0), "r"(b0[0]), "r"(bar)
              : "memory");
        }
      }
    }
  }
  if (SMEM && !tma) {
    // tile + halo, LB loads in flight per thread before their stores
    // cell -> grid index by multiply-high division and division-free wrap
    constexpr int LB = 8;
    const uint32_t mS = fastdiv_magic(uint32_t(S));
    const bool fastwrap = fast_wrap_ok<NDIM>(g, S);
    auto cell = [&](int c) -> cplx<T> { return grid[cell_index<NDIM>(c, S, mS, fastwrap, b0, g)]; };
    for (int c0 = threadIdx.x; c0 < ncell; c0 += LB * SP_THREADS) {
      cplx<T> v[LB];
#pragma unroll
      for (int u = 0; u < LB; ++u) {
        const int c = c0 + u * SP_THREADS;
        v[u] = c < ncell ? cell(c) : mkc<T>(T(0), T(0));
      }
#pragma unroll
      for (int u = 0; u < LB; ++u) {
        const int c = c0 + u * SP_THREADS;
        if (c < ncell) buf[c] = v[u];
      }
    }
    __syncthreads();
  }
  auto point = [&](uint32_t i) {
    Tc x[NDIM];
    uint32_t j = load_point<Tc, NDIM>(pts, i, x);
    T w[NDIM][W];
    int o[NDIM];
#pragma unroll
    for (int d = 0; d < NDIM; ++d) {
      int i0;
      double frac;
      fold<Tc>(x[d], g.coordfct[d], int(g.nover[d]), g.shift[d], g.maxi0[d], i0, frac);
      kernel_weights<T, W>(kp, T(double(W - 1) - 2.0 * frac), w[d]);
      o[d] = i0 - b0[d];
    }
    T ar = 0, ai = 0;
    if constexpr (NDIM == 1) {
#pragma unroll
      for (int a = 0; a < W; ++a) {
        cplx<T> gv = buf[o[0] + a];
        ar += w[0][a] * gv.x;
        ai += w[0][a] * gv.y;
      }
    } else if constexpr (NDIM == 2) {
#pragma unroll
      for (int a = 0; a < W; ++a) {
        const cplx<T> *row = buf + (o[0] + a) * S + o[1];
        T rr = 0, ri = 0;
#pragma unroll
        for (int b = 0; b < W; ++b) {
          cplx<T> gv = row[b];
          rr += w[1][b] * gv.x;
          ri += w[1][b] * gv.y;
        }
        ar += w[0][a] * rr;
        ai += w[0][a] * ri;
      }
    } else {
      if constexpr (SMEM) {
#pragma unroll 1
        for (int a = 0; a < W; ++a) {
          T pr = 0, pi = 0;
#pragma unroll
          for (int b = 0; b < W; ++b) {
            const cplx<T> *row = buf + ((o[0] + a) * S + (o[1] + b)) * S + o[2];
            T rr = 0, ri = 0;
#pragma unroll
            for (int e = 0; e < W; ++e) {
              cplx<T> gv = row[e];
              rr += w[2][e] * gv.x;
              ri += w[2][e] * gv.y;
            }
            pr += w[1][b] * rr;
            pi += w[1][b] * ri;
          }
          ar += w[0][a] * pr;
          ai += w[0][a] * pi;
        }
      } else {
        const int nu = int(g.nover[0]), nv = int(g.nover[1]), nw = int(g.nover[2]);
        // indices stay in [-n, 2n) where every axis is at least 2S long
        const bool fw = nu >= 2 * S && nv >= 2 * S && nw >= 2 * S;
        auto wr = [fw](int i, int n) { return fw ? wrap1(i, n) : wrapi(i, n); };
        int iw[W];
#pragma unroll
        for (int e = 0; e < W; ++e) iw[e] = wr(b0[2] + o[2] + e, nw);
#pragma unroll 1
        for (int a = 0; a < W; ++a) {
          int iu = wr(b0[0] + o[0] + a, nu);
          T pr = 0, pi = 0;
#pragma unroll
          for (int b = 0; b < W; ++b) {
            int iv = wr(b0[1] + o[1] + b, nv);
            const cplx<T> *row = grid + (int64_t(iu) * nv + iv) * nw;
            T rr = 0, ri = 0;
#pragma unroll
            for (int e = 0; e < W; ++e) {
              cplx<T> gv = __ldg(row + iw[e]);
              rr += w[2][e] * gv.x;
              ri += w[2][e] * gv.y;
            }
            pr += w[1][b] * rr;
            pi += w[1][b] * ri;
          }
          ar += w[0][a] * pr;
          ai += w[0][a] * pi;
        }
      }
    }
    out[int64_t(j) * os] = mkc<T>(ar, ai);
  };
  const uint32_t end = ch.start + ch.count;
  if constexpr (!SMEM) {
    for (uint32_t i = ch.start + threadIdx.x; i < end; i += SP_THREADS) point(i);
  } else {
    // Bank-balanced order.  At a given step of the footprint loop all lanes of
    // a warp read at the same offset from their point's first cell, so the
    // bank conflicts of that read depend only on the first cells' banks.  Each
    // batch of IB points is folded once (coalesced coordinate reads), its
    // records (output index, first cell, kernel arguments) kept in registers,
    // counting-sorted by bank slot of the first cell (cell index mod 128 bytes
    // / cell size, NSLOT slots) and written to shared memory so that, at step
    // r, lane NSLOT*h + l of a warp takes sorted entry p*q + r with
    // p = l*(32/NSLOT) + h (q = ceil(n/32)) from word r*32 + p: the NSLOT lanes
    // of one 128-byte wavefront group (a half-warp for 8-byte cells, a
    // quarter-warp for 16-byte ones) take entries spread over the whole sorted
    // list, one per slot for uniformly spread points, and all lanes read their
    // records without conflicts.  Every point is still computed by one thread
    // in a fixed order, so results do not depend on the assignment.
    using IO = InterpOrder<T>;
    constexpr int NSLOT = IO::NSLOT, IB = IO::IB, PER = IB / SP_THREADS;
    int *s_cnt = reinterpret_cast<int *>(smraw + tile_bytes);
    uint32_t *r_j = reinterpret_cast<uint32_t *>(s_cnt + NSLOT);
    int *r_base = reinterpret_cast<int *>(r_j + IB);
    T *r_t = reinterpret_cast<T *>(r_base + IB);   // [NDIM][IB]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t s0 = ch.start; s0 < end; s0 += IB) {
      const int nb = int(min(uint32_t(IB), end - s0));
      const int q = (nb + 31) >> 5;
      const uint32_t mq = q > 1 ? fastdiv_magic(uint32_t(q)) : 0u;
      if (threadIdx.x < NSLOT) s_cnt[threadIdx.x] = 0;
      __syncthreads();
      uint32_t pj[PER];
      int pb[PER];
      T pt[PER][NDIM];
#pragma unroll
      for (int k = 0; k < PER; ++k) {
        const int li = k * SP_THREADS + int(threadIdx.x);
        pb[k] = -1;
        if (li < nb) {
          Tc x[NDIM];
          pj[k] = load_point<Tc, NDIM>(pts, s0 + uint32_t(li), x);
          int base = 0;
#pragma unroll
          for (int d = 0; d < NDIM; ++d) {
            int i0;
            double frac;
            fold<Tc>(x[d], g.coordfct[d], int(g.nover[d]), g.shift[d], g.maxi0[d], i0, frac);
            pt[k][d] = T(double(W - 1) - 2.0 * frac);
            base = (d == NDIM - 1) ? base * pitch + (i0 - b0[d] + sh) : base * S + (i0 - b0[d]);
          }
          pb[k] = base;
          atomicAdd(&s_cnt[base & (NSLOT - 1)], 1);
        }
      }
      __syncthreads();
      if (warp == 0) {   // exclusive prefix over the slots
        const int c = lane < NSLOT ? s_cnt[lane] : 0;
        int incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int v = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += v;
        }
        __syncwarp();
        if (lane < NSLOT) s_cnt[lane] = incl - c;
      }
      __syncthreads();
#pragma unroll
      for (int k = 0; k < PER; ++k) {
        if (pb[k] >= 0) {
          const int e = atomicAdd(&s_cnt[pb[k] & (NSLOT - 1)], 1);
          const int eq = q > 1 ? int(fastdiv(uint32_t(e), mq)) : e;   // e / q (e < IB)
          const int w = (e - eq * q) * 32 + eq;
          r_j[w] = pj[k];
          r_base[w] = pb[k];
#pragma unroll
          for (int d = 0; d < NDIM; ++d) r_t[d * IB + w] = pt[k][d];
        }
      }
      __syncthreads();
      if (tma && s0 == ch.start) {
        // the tile copy has been in flight while the first batch was ordered
        const bool ok = tile_bar_wait(tbar, 0u);
        if (__syncthreads_or(ok ? 0 : 1)) {
          if (threadIdx.x == 0 && err) atomicExch(err, 1);
          return;
        }
      }
      const int pl = (lane % NSLOT) * (32 / NSLOT) + lane / NSLOT;
      for (int r = warp; r < q; r += SP_WARPS) {
        if (pl * q + r >= nb) continue;
        const int w = r * 32 + pl;
        const uint32_t j = r_j[w];
        const cplx<T> *p0 = buf + r_base[w];
        T wt[NDIM][W];
#pragma unroll
        for (int d = 0; d < NDIM; ++d) kernel_weights<T, W>(kp, r_t[d * IB + w], wt[d]);
        T ar = 0, ai = 0;
        if constexpr (NDIM == 1) {
#pragma unroll
          for (int a = 0; a < W; ++a) {
            cplx<T> gv = p0[a];
            ar += wt[0][a] * gv.x;
            ai += wt[0][a] * gv.y;
          }
        } else if constexpr (NDIM == 2) {
#pragma unroll
          for (int a = 0; a < W; ++a) {
            const cplx<T> *row = p0 + a * pitch;
            T rr = 0, ri = 0;
#pragma unroll
            for (int b = 0; b < W; ++b) {
              cplx<T> gv = row[b];
              rr += wt[1][b] * gv.x;
              ri += wt[1][b] * gv.y;
            }
            ar += wt[0][a] * rr;
            ai += wt[0][a] * ri;
          }
        } else {
#pragma unroll 1
          for (int a = 0; a < W; ++a) {
            T pr = 0, pi = 0;
#pragma unroll
            for (int b = 0; b < W; ++b) {
              const cplx<T> *row = p0 + (a * S + b) * S;
              T rr = 0, ri = 0;
#pragma unroll
              for (int e = 0; e < W; ++e) {
                cplx<T> gv = row[e];
                rr += wt[2][e] * gv.x;
                ri += wt[2][e] * gv.y;
              }
              pr += wt[1][b] * rr;
              pi += wt[1][b] * ri;
            }
            ar += wt[0][a] * pr;
            ai += wt[0][a] * pi;
          }
        }
        out[int64_t(j) * os] = mkc<T>(ar, ai);
      }
      __syncthreads();
    }
  }
}

// six CTAs per SM for single-precision 1D/2D (fits 40 registers)
template <typename T, int NDIM> constexpr int interp_min_ctas() {
  return (sizeof(T) == 4 && NDIM < 3) ? 6 : 1;
}

// tpitch > 0: 2D tiles inside the grid are staged by TMA through tmap (one
// transform); err: device error word for a tile copy that never completes
template <typename T, typename Tc, int NDIM, int W>
__global__ void __launch_bounds__(SP_THREADS, interp_min_ctas<T, NDIM>())
    k_interp(PointsDesc pts, const Chunk *__restrict__ chunks, Geometry g, KernelPoly<T> kp,
             const cplx<T> *__restrict__ grid, int64_t gtrans, cplx<T> *__restrict__ out,
             int64_t os, int64_t otrans, const __grid_constant__ CUtensorMap tmap, int tpitch,
             int *err) {
  extern __shared__ __align__(128) unsigned char smraw_tile[];
  __shared__ uint64_t tbar;
  interp_chunk<T, Tc, NDIM, W>(pts, chunks[blockIdx.x], g, kp, grid + int64_t(blockIdx.y) * gtrans,
                               out + int64_t(blockIdx.y) * otrans, os, smraw_tile,
                               tpitch > 0 ? &tmap : nullptr, tpitch, &tbar, err);
}

template <typename T, int NDIM, int W>
size_t spread_smem_bytes(const Geometry &g) {
  int S = (1 << g.log2tile) + W;
  size_t ncell = size_t(S);
  for (int d = 1; d < NDIM; ++d) ncell *= size_t(S);
  size_t buf = BufferLayout<T>::smem(NDIM) ? ncell * sizeof(cplx<T>) : 0;
  constexpr int WS = stage_stride<NDIM, W>();
  size_t wbytes = (size_t(SP_WARPS) * 32 * WS * sizeof(T) + 15) / 16 * 16;
  size_t stage = wbytes + size_t(SP_WARPS) * 32 * (sizeof(cplx<T>) + NDIM * sizeof(int));
  return buf + stage;
}

// tpitch > 0: the staged 2D tile has that row pitch (TMA staging)
template <typename T, int NDIM, int W>
size_t interp_smem_bytes(const Geometry &g, int tpitch = 0) {
  int S = (1 << g.log2tile) + W;
  size_t ncell = size_t(S);
  for (int d = 1; d < NDIM; ++d) ncell *= size_t(S);
  if (NDIM == 2 && tpitch > 0) ncell = size_t(tpitch) * size_t(S);
  return BufferLayout<T>::smem(NDIM) ? ncell * sizeof(cplx<T>) + InterpOrder<T>::bytes(NDIM) : 0;
}

// 2D tensor map of a contiguous complex grid (nover[0] rows of nover[1]
// cells) as rows of 2*nover[1] scalars, box (2*tpitch, S); false where the
// encoder is unavailable or the grid does not meet the copy's alignment rules
// (16-byte base address and row pitch)
bool encode_tile_map(CUtensorMap *map, const void *grid, bool f64, int64_t n0, int64_t n1,
                     int tpitch, int S);

template <typename T, typename Tc, int NDIM, int W>
void spread_w(const PointsDesc &pts, const ChunkList &cl, const Geometry &g,
              const KernelPoly<T> &kp, const void *values, int64_t vs, int64_t vtrans,
              void *grid, int64_t gtrans, int ntrans, cudaStream_t st) {
  size_t sm = spread_smem_bytes<T, NDIM, W>(g);
  auto kern = k_spread<T, Tc, NDIM, W>;
  DN_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
  dim3 grd(cl.nchunks, ntrans);
  kern<<<grd, SP_THREADS, sm, st>>>(pts, cl.chunks, g, kp, static_cast<const cplx<T> *>(values), vs,
                                    vtrans, static_cast<cplx<T> *>(grid), gtrans);
  DN_LAUNCHED();
}

template <typename T, typename Tc, int NDIM, int W>
void interp_w(const PointsDesc &pts, const ChunkList &cl, const Geometry &g,
              const KernelPoly<T> &kp, const void *grid, int64_t gtrans, void *out, int64_t os,
              int64_t otrans, int ntrans, cudaStream_t st, int *err) {
  CUtensorMap map;
  memset(&map, 0, sizeof(map));
  int tpitch = 0;
  if constexpr (NDIM == 2 && BufferLayout<T>::smem(NDIM)) {
    const int S = (1 << g.log2tile) + W;
    const int tp = tma_tile_pitch(S, g.nsafe);
    if (err && ntrans == 1 &&
        encode_tile_map(&map, grid, sizeof(T) == 8, g.nover[0], g.nover[1], tp, S))
      tpitch = tp;
  }
  size_t sm = interp_smem_bytes<T, NDIM, W>(g, tpitch);
  auto kern = k_interp<T, Tc, NDIM, W>;
  DN_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
  dim3 grd(cl.nchunks, ntrans);
  kern<<<grd, SP_THREADS, sm, st>>>(pts, cl.chunks, g, kp, static_cast<const cplx<T> *>(grid),
                                    gtrans, static_cast<cplx<T> *>(out), os, otrans, map, tpitch,
                                    err);
  DN_LAUNCHED();
}

// W dispatch: float supports W 4..8, double 4..16 (the kernel table's ranges)
#define DN_FOR_W_FLOAT(M) M(4) M(5) M(6) M(7) M(8)
#define DN_FOR_W_DOUBLE(M) \
  M(4) M(5) M(6) M(7) M(8) M(9) M(10) M(11) M(12) M(13) M(14) M(15) M(16)

template <typename T, typename Tc, int NDIM>
void spread_dispatch(const PointsDesc &pts, const ChunkList &cl, const Geometry &g,
                     const KernelPoly<T> &kp, const void *values, int64_t vs, int64_t vtrans,
                     void *grid, int64_t gtrans, int ntrans, cudaStream_t st) {
#define DN_CASE(WW) \
  case WW: spread_w<T, Tc, NDIM, WW>(pts, cl, g, kp, values, vs, vtrans, grid, gtrans, ntrans, st); return;
  if constexpr (sizeof(T) == 4) {
    switch (g.W) { DN_FOR_W_FLOAT(DN_CASE) }
  } else {
    switch (g.W) { DN_FOR_W_DOUBLE(DN_CASE) }
  }
#undef DN_CASE
  throw Error(ST_UNSUPPORTED, "kernel support not supported by this build");
}

template <typename T, typename Tc, int NDIM>
void interp_dispatch(const PointsDesc &pts, const ChunkList &cl, const Geometry &g,
                     const KernelPoly<T> &kp, const void *grid, int64_t gtrans, void *out,
                     int64_t os, int64_t otrans, int ntrans, cudaStream_t st, int *err) {
#define DN_CASE(WW) \
  case WW: interp_w<T, Tc, NDIM, WW>(pts, cl, g, kp, grid, gtrans, out, os, otrans, ntrans, st, err); return;
  if constexpr (sizeof(T) == 4) {
    switch (g.W) { DN_FOR_W_FLOAT(DN_CASE) }
  } else {
    switch (g.W) { DN_FOR_W_DOUBLE(DN_CASE) }
  }
#undef DN_CASE
  throw Error(ST_UNSUPPORTED, "kernel support not supported by this build");
}

template <typename T>
void launch_spread_impl(const PointsDesc &pts, const ChunkList &cl, const Geometry &g,
                        const KernelPoly<T> &kp, const void *values, int64_t vs,
                        int64_t vtrans, void *grid, int64_t gtrans, int ntrans,
                        cudaStream_t st) {
  if (cl.nchunks == 0 || ntrans == 0) return;
#define DN_SD(TC, ND) spread_dispatch<T, TC, ND>(pts, cl, g, kp, values, vs, vtrans, grid, gtrans, ntrans, st)
  if (pts.coord_f64) {
    if (g.ndim == 1) DN_SD(double, 1); else if (g.ndim == 2) DN_SD(double, 2); else DN_SD(double, 3);
  } else {
    if (g.ndim == 1) DN_SD(float, 1); else if (g.ndim == 2) DN_SD(float, 2); else DN_SD(float, 3);
  }
#undef DN_SD
}

template <typename T>
void launch_interp_impl(const PointsDesc &pts, const ChunkList &cl, const Geometry &g,
                        const KernelPoly<T> &kp, const void *grid, int64_t gtrans, void *out,
                        int64_t os, int64_t otrans, int ntrans, cudaStream_t st, int *err) {
  if (cl.nchunks == 0 || ntrans == 0) return;
#define DN_ID(TC, ND) interp_dispatch<T, TC, ND>(pts, cl, g, kp, grid, gtrans, out, os, otrans, ntrans, st, err)
  if (pts.coord_f64) {
    if (g.ndim == 1) DN_ID(double, 1); else if (g.ndim == 2) DN_ID(double, 2); else DN_ID(double, 3);
  } else {
    if (g.ndim == 1) DN_ID(float, 1); else if (g.ndim == 2) DN_ID(float, 2); else DN_ID(float, 3);
  }
#undef DN_ID
}

}  // namespace dnufft
