// Coordinate binning and the stable tile sort.
//
//  k_fold_keys   - per point: fold every axis (bit-exact getpix) and form DUCC's
//                  tile key (src/ducc0/nufft/nufft.h:892-907, :1364-1381,
//                  :1862-1892).
//  radix sort    - stable LSD radix sort of (key, index) pairs, up to 11 bits per
//                  pass: per-block digit histograms, one device-wide exclusive
//                  scan, and a scatter whose in-block ranks come from warp-level
//                  __match_any_sync, so equal keys keep their input order.  A
//                  stable sort by key reproduces DUCC's coord_idx exactly
//                  (bucket_sort2, src/ducc0/infra/bucket_sort.h:170-354).
//  chunking      - sorted points are cut into chunks of at most CHUNK points
//                  that lie in one tile; each chunk is one CTA of the spreading
//                  / interpolation kernels.
#include "common.cuh"
#include "kernels.h"

#include <algorithm>

namespace dnufft {

// ---------------------------------------------------------------- keys
template <typename Tc, int NDIM>
__global__ void k_fold_keys(const Tc *__restrict__ coord, int64_t cs0, int64_t cs1,
                            uint32_t npts, Geometry g, uint32_t *__restrict__ keys,
                            uint32_t *__restrict__ idx, bool qbits) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npts) return;
  int t[NDIM];
#pragma unroll
  for (int d = 0; d < NDIM; ++d) {
    int i0;
    double frac;
    fold<Tc>(coord[int64_t(i) * cs0 + int64_t(d) * cs1], g.coordfct[d], int(g.nover[d]),
             g.shift[d], g.maxi0[d], i0, frac);
    t[d] = i0 + g.nsafe;
  }
  uint32_t key;
  if constexpr (NDIM == 1) {
    key = uint32_t(t[0] >> g.log2tile);
  } else if constexpr (NDIM == 2) {
    key = uint32_t(t[0] >> g.log2tile) * uint32_t(g.ntiles[1]) + uint32_t(t[1] >> g.log2tile);
    if (qbits) {
      // quadrant, then the cell inside it in Morton order: consecutive points
      // (one K-block of the tensor-core spreader) lie close together, so each
      // accumulator cell receives contributions from fewer K-blocks
      const int lh = g.log2tile - 1, half = 1 << lh, m = (1 << g.log2tile) - 1;
      const uint32_t du = uint32_t(t[0] & (half - 1)), dv = uint32_t(t[1] & (half - 1));
      uint32_t mort = 0;
      for (int b = 0; b < lh; ++b)
        mort |= (((du >> b) & 1u) << (2 * b + 1)) | (((dv >> b) & 1u) << (2 * b));
      key = (key << 2) | (((t[0] & m) >= half) ? 2u : 0u) | (((t[1] & m) >= half) ? 1u : 0u);
      key = (key << (2 * lh)) | mort;
    }
  } else {
    uint32_t ss = uint32_t(g.ssmall), ms = (1u << ss) - 1u;
    uint32_t a = uint32_t(t[0] >> g.lsq2), b = uint32_t(t[1] >> g.lsq2),
             c = uint32_t(t[2] >> g.lsq2);
    uint32_t low = ((a & ms) << (2 * ss)) | ((b & ms) << ss) | (c & ms);
    uint32_t hi = (a >> ss) * uint32_t(g.ntiles[1] * g.ntiles[2]) +
                  (b >> ss) * uint32_t(g.ntiles[2]) + (c >> ss);
    key = (hi << (3 * ss)) | low;
  }
  keys[i] = key;
  idx[i] = i;
}

void launch_fold_keys(bool coord_f64, const void *coord, int64_t cs0, int64_t cs1,
                      uint32_t npts, const Geometry &g, uint32_t *keys, uint32_t *idx,
                      cudaStream_t st, bool quadrant_bits) {
  if (npts == 0) return;
  dim3 block(256), grid((npts + 255) / 256);
#define FK(TC, ND) \
  k_fold_keys<TC, ND><<<grid, block, 0, st>>>((const TC *)coord, cs0, cs1, npts, g, keys, idx, \
                                               quadrant_bits)
  if (coord_f64) {
    if (g.ndim == 1) FK(double, 1); else if (g.ndim == 2) FK(double, 2); else FK(double, 3);
  } else {
    if (g.ndim == 1) FK(float, 1); else if (g.ndim == 2) FK(float, 2); else FK(float, 3);
  }
#undef FK
  DN_LAUNCHED();
}

// ---------------------------------------------------------------- scan
// exclusive prefix sum of uint32, three phases with recursion on block sums
constexpr int SCAN_THREADS = 512;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t *warp_sums,
                                                    uint32_t *total) {
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int nw = blockDim.x >> 5;
    uint32_t s = lane < nw ? warp_sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < nw) warp_sums[lane] = s;
  }
  __syncthreads();
  uint32_t base = wid > 0 ? warp_sums[wid - 1] : 0;
  if (total) *total = warp_sums[(blockDim.x >> 5) - 1];
  return base + x - v;
}

__global__ void k_scan_tiles(const uint32_t *__restrict__ in, uint32_t *__restrict__ out,
                             uint64_t n, uint32_t *__restrict__ block_sums) {
  __shared__ uint32_t ws[32];
  uint64_t base = uint64_t(blockIdx.x) * SCAN_TILE + uint64_t(threadIdx.x) * SCAN_ITEMS;
  uint32_t v[SCAN_ITEMS];
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    v[k] = (base + k < n) ? in[base + k] : 0u;
    s += v[k];
  }
  uint32_t tot;
  uint32_t run = block_excl_scan(s, ws, &tot);
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    if (base + k < n) out[base + k] = run;
    run += v[k];
  }
  if (threadIdx.x == 0 && block_sums) block_sums[blockIdx.x] = tot;
}

__global__ void k_scan_add(uint32_t *__restrict__ out, uint64_t n,
                           const uint32_t *__restrict__ block_offs) {
  uint64_t base = uint64_t(blockIdx.x) * SCAN_TILE + uint64_t(threadIdx.x) * SCAN_ITEMS;
  uint32_t add = block_offs[blockIdx.x];
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k)
    if (base + k < n) out[base + k] += add;
}

size_t scan_workspace_bytes(uint64_t n) {
  size_t b = 0;
  while (n > uint64_t(SCAN_TILE)) {
    n = (n + SCAN_TILE - 1) / SCAN_TILE;
    b += ((n + 63) / 64) * 64 * sizeof(uint32_t) * 2;
  }
  return b + 256;
}

void exclusive_scan(const uint32_t *in, uint32_t *out, uint64_t n, uint32_t *ws,
                    cudaStream_t st) {
  if (n == 0) return;
  uint64_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
  if (nb == 1) {
    k_scan_tiles<<<1, SCAN_THREADS, 0, st>>>(in, out, n, nullptr);
    DN_LAUNCHED();
    return;
  }
  uint32_t *sums = ws;
  uint32_t *offs = ws + ((nb + 63) / 64) * 64;
  uint32_t *rest = offs + ((nb + 63) / 64) * 64;
  k_scan_tiles<<<unsigned(nb), SCAN_THREADS, 0, st>>>(in, out, n, sums);
  DN_LAUNCHED();
  exclusive_scan(sums, offs, nb, rest, st);
  k_scan_add<<<unsigned(nb), SCAN_THREADS, 0, st>>>(out, n, offs);
  DN_LAUNCHED();
}

// ---------------------------------------------------------------- radix sort
constexpr int RS_WARPS = 8;
constexpr int RS_ROUNDS = 8;                                   // 32-item rounds per warp
constexpr int RS_TILE = RS_WARPS * RS_ROUNDS * 32;             // 2048 items per block

__global__ void k_radix_hist(const uint32_t *__restrict__ keys, uint32_t n, int shift,
                             int nbits, uint32_t *__restrict__ hist, uint32_t nblocks) {
  extern __shared__ uint32_t sh[];
  int nb = 1 << nbits;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  uint32_t mask = uint32_t(nb - 1);
  uint64_t base = uint64_t(blockIdx.x) * RS_TILE;
  for (int k = threadIdx.x; k < RS_TILE; k += blockDim.x) {
    uint64_t i = base + k;
    if (i < n) atomicAdd(&sh[(keys[i] >> shift) & mask], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nb; i += blockDim.x)
    hist[uint64_t(i) * nblocks + blockIdx.x] = sh[i];
}

__global__ void k_radix_scatter(const uint32_t *__restrict__ kin, const uint32_t *__restrict__ vin,
                                uint32_t *__restrict__ kout, uint32_t *__restrict__ vout,
                                uint32_t n, int shift, int nbits,
                                const uint32_t *__restrict__ offs, uint32_t nblocks) {
  extern __shared__ uint32_t sh[];
  const int nb = 1 << nbits;
  uint32_t *whist = sh;                        // [RS_WARPS][nb] counts, then offsets
  const uint32_t mask = uint32_t(nb - 1);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < RS_WARPS * nb; i += blockDim.x) whist[i] = 0;
  __syncthreads();
  uint64_t wbase = uint64_t(blockIdx.x) * RS_TILE + uint64_t(w) * RS_ROUNDS * 32;
  uint32_t dig[RS_ROUNDS], loc[RS_ROUNDS];
  const unsigned lt = (1u << lane) - 1u;
#pragma unroll
  for (int r = 0; r < RS_ROUNDS; ++r) {
    uint64_t i = wbase + uint64_t(r) * 32 + lane;
    bool valid = i < n;
    uint32_t d = valid ? ((kin[i] >> shift) & mask) : uint32_t(nb);   // sentinel
    unsigned grp = __match_any_sync(0xffffffffu, d);
    int leader = __ffs(grp) - 1;
    uint32_t cnt = (valid ? whist[w * nb + d] : 0u);
    loc[r] = cnt + uint32_t(__popc(grp & lt));
    dig[r] = d;
    __syncwarp();
    if (valid && lane == leader) whist[w * nb + d] = cnt + uint32_t(__popc(grp));
    __syncwarp();
  }
  __syncthreads();
  // per digit: global offset of this block + counts of earlier warps
  for (int d = threadIdx.x; d < nb; d += blockDim.x) {
    uint32_t run = offs[uint64_t(d) * nblocks + blockIdx.x];
#pragma unroll
    for (int ww = 0; ww < RS_WARPS; ++ww) {
      uint32_t c = whist[ww * nb + d];
      whist[ww * nb + d] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < RS_ROUNDS; ++r) {
    uint64_t i = wbase + uint64_t(r) * 32 + lane;
    if (i < n) {
      uint32_t dst = whist[w * nb + dig[r]] + loc[r];
      kout[dst] = kin[i];
      vout[dst] = vin[i];
    }
  }
}

size_t radix_workspace_bytes(uint32_t n, int keybits) {
  int passes = (keybits + 10) / 11;
  if (passes < 1) passes = 1;
  int nbits = (keybits + passes - 1) / passes;
  uint64_t nblocks = (uint64_t(n) + RS_TILE - 1) / RS_TILE;
  uint64_t hn = (uint64_t(1) << nbits) * nblocks;
  return 2 * size_t(n) * sizeof(uint32_t)       // ping-pong keys/values
         + 2 * hn * sizeof(uint32_t)            // histogram + offsets
         + scan_workspace_bytes(hn) + 1024;
}

// element-wise copy of the sorted pairs back (the ping-pong halves of the
// workspace are only 4-byte aligned)
__global__ void k_copy_pairs(const uint32_t *__restrict__ ka, const uint32_t *__restrict__ va,
                             uint32_t *__restrict__ kb, uint32_t *__restrict__ vb, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    kb[i] = ka[i];
    vb[i] = va[i];
  }
}

// Sorts (keys, vals) in place by the low 'keybits' bits of keys, stably.
void radix_sort_pairs(uint32_t *keys, uint32_t *vals, uint32_t n, int keybits, void *ws,
                      cudaStream_t st) {
  if (n <= 1 || keybits <= 0) return;
  int passes = (keybits + 10) / 11;
  int nbits = (keybits + passes - 1) / passes;
  uint32_t nblocks = uint32_t((uint64_t(n) + RS_TILE - 1) / RS_TILE);
  uint64_t hn = (uint64_t(1) << nbits) * nblocks;
  char *p = static_cast<char *>(ws);
  uint32_t *k2 = reinterpret_cast<uint32_t *>(p);
  p += size_t(n) * 4;
  uint32_t *v2 = reinterpret_cast<uint32_t *>(p);
  p += size_t(n) * 4;
  uint32_t *hist = reinterpret_cast<uint32_t *>(p);
  p += hn * 4;
  uint32_t *offs = reinterpret_cast<uint32_t *>(p);
  p += hn * 4;
  uint32_t *sws = reinterpret_cast<uint32_t *>((reinterpret_cast<uintptr_t>(p) + 255) & ~uintptr_t(255));
  uint32_t *ka = keys, *va = vals, *kb = k2, *vb = v2;
  size_t hsm = sizeof(uint32_t) << nbits;
  size_t ssm = size_t(RS_WARPS) * hsm;
  static bool attr_set = false;
  if (!attr_set) {
    DN_CUDA(cudaFuncSetAttribute(k_radix_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 RS_WARPS * (4 << 11)));
    attr_set = true;
  }
  for (int pass = 0; pass < passes; ++pass) {
    int shift = pass * nbits;
    int bits = (keybits - shift < nbits) ? keybits - shift : nbits;
    if (bits <= 0) break;
    uint64_t hn_pass = (uint64_t(1) << bits) * nblocks;
    k_radix_hist<<<nblocks, 256, hsm, st>>>(ka, n, shift, bits, hist, nblocks);
    DN_LAUNCHED();
    exclusive_scan(hist, offs, hn_pass, sws, st);
    k_radix_scatter<<<nblocks, RS_WARPS * 32, ssm, st>>>(ka, va, kb, vb, n, shift, bits, offs,
                                                         nblocks);
    DN_LAUNCHED();
    std::swap(ka, kb);
    std::swap(va, vb);
  }
  if (ka != keys) {
    // a kernel, not a device-to-device memcpy: a copy engine may be busy with a
    // host transfer of the same call on another stream
    const unsigned nb = unsigned(std::min<uint64_t>((uint64_t(n) + 255) / 256, 148 * 16));
    k_copy_pairs<<<nb, 256, 0, st>>>(ka, va, keys, vals, n);
    DN_LAUNCHED();
  }
}

// ---------------------------------------------------------------- chunking
// A chunk starts where the tile changes or every 'chunk' points inside a run
// of equal tiles.  Tile = key >> tile_shift (3D: drop the sub-tile bits).
__global__ void k_chunk_flags(const uint32_t *__restrict__ skeys, uint32_t n, int tile_shift,
                              uint32_t chunk, uint32_t *__restrict__ flags) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t t = skeys[i] >> tile_shift;
  bool f = (i == 0) || (t != (skeys[i - 1] >> tile_shift)) || (i % chunk == 0);
  flags[i] = f ? 1u : 0u;
}

__global__ void k_chunk_fill(const uint32_t *__restrict__ skeys, const uint32_t *__restrict__ flags,
                             const uint32_t *__restrict__ pos, uint32_t n, int tile_shift,
                             Chunk *__restrict__ chunks) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !flags[i]) return;
  Chunk c;
  c.start = i;
  c.count = 0;
  c.tile = skeys[i] >> tile_shift;
  c.pad = 0;
  chunks[pos[i]] = c;
}

__global__ void k_chunk_counts(Chunk *__restrict__ chunks, const uint32_t *__restrict__ nchunks_p,
                               uint32_t n) {
  uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t nc = *nchunks_p;
  if (c >= nc) return;
  uint32_t end = (c + 1 < nc) ? chunks[c + 1].start : n;
  chunks[c].count = end - chunks[c].start;
}

__global__ void k_count_total(const uint32_t *__restrict__ flags, const uint32_t *__restrict__ pos,
                              uint32_t n, uint32_t *__restrict__ total) {
  *total = pos[n - 1] + flags[n - 1];
}

size_t chunk_workspace_bytes(uint32_t n) {
  return 2 * size_t(n) * sizeof(uint32_t) + scan_workspace_bytes(n) + 1024;
}

// ---------------------------------------------------------------- small read-backs
// A few 32-bit device words are read back by a one-warp kernel that stores
// them into mapped pinned host memory, then the stream is synchronised.  A
// device->host memcpy of the same words would queue on the device->host copy
// engine behind large result copies that other streams issued earlier (the
// pipelined host calls copy 100 MB result ranges back while the next groups
// are sorted), and the sort would wait for them; a kernel's stores to host
// memory do not.
struct WordSrcs {
  const uint32_t *p[8];
};

__global__ void k_read_words(WordSrcs s, int n, volatile uint32_t *dst) {
  const int i = threadIdx.x;
  if (i < n) dst[i] = *s.p[i];
  __threadfence_system();
}

void read_words(const uint32_t *const *src, int n, uint32_t *out, cudaStream_t st) {
  DN_REQUIRE(n >= 1 && n <= 8, ST_INTERNAL, "read_words: 1 to 8 words");
  // one mapped buffer per host thread and device (calls of one thread are
  // sequential; calls from several threads use separate buffers)
  static thread_local uint32_t *host[64] = {nullptr};
  static thread_local uint32_t *mapped[64] = {nullptr};
  int dev = 0;
  DN_CUDA(cudaGetDevice(&dev));
  DN_REQUIRE(dev >= 0 && dev < 64, ST_INTERNAL, "device index out of range");
  if (!host[dev]) {
    void *h = nullptr;
    DN_CUDA(cudaHostAlloc(&h, 8 * sizeof(uint32_t), cudaHostAllocMapped | cudaHostAllocPortable));
    void *d = nullptr;
    DN_CUDA(cudaHostGetDevicePointer(&d, h, 0));
    host[dev] = static_cast<uint32_t *>(h);
    mapped[dev] = static_cast<uint32_t *>(d);
  }
  WordSrcs s{};
  for (int i = 0; i < n; ++i) s.p[i] = src[i];
  k_read_words<<<1, 32, 0, st>>>(s, n, mapped[dev]);
  DN_LAUNCHED();
  DN_CUDA(cudaStreamSynchronize(st));
  const volatile uint32_t *h = host[dev];
  for (int i = 0; i < n; ++i) out[i] = h[i];
}

// Builds the chunk list from sorted keys; returns the number of chunks (the
// count is read back to the host, which synchronises the stream once: through
// mapped host memory, or with zero_copy false, which allocates nothing, by a
// device->host copy).
uint32_t build_chunks(const uint32_t *skeys, uint32_t n, int tile_shift, uint32_t chunk,
                      Chunk *chunks, uint32_t *d_count, void *ws, cudaStream_t st,
                      bool zero_copy) {
  if (n == 0) return 0;
  uint32_t *flags = static_cast<uint32_t *>(ws);
  uint32_t *pos = flags + n;
  uint32_t *sws = reinterpret_cast<uint32_t *>(
      (reinterpret_cast<uintptr_t>(pos + n) + 255) & ~uintptr_t(255));
  unsigned g = (n + 255) / 256;
  k_chunk_flags<<<g, 256, 0, st>>>(skeys, n, tile_shift, chunk, flags);
  DN_LAUNCHED();
  exclusive_scan(flags, pos, n, sws, st);
  k_chunk_fill<<<g, 256, 0, st>>>(skeys, flags, pos, n, tile_shift, chunks);
  DN_LAUNCHED();
  k_count_total<<<1, 1, 0, st>>>(flags, pos, n, d_count);
  DN_LAUNCHED();
  k_chunk_counts<<<g, 256, 0, st>>>(chunks, d_count, n);
  DN_LAUNCHED();
  uint32_t h = 0;
  if (zero_copy) {
    const uint32_t *src[1] = {d_count};
    read_words(src, 1, &h, st);
  } else {
    DN_CUDA(cudaMemcpyAsync(&h, d_count, 4, cudaMemcpyDeviceToHost, st));
    DN_CUDA(cudaStreamSynchronize(st));
  }
  return h;
}

// ---------------------------------------------------------------- gathers
template <typename Tc>
__global__ void k_gather_coords(const Tc *__restrict__ coord, int64_t cs0, int64_t cs1,
                                int ndim, const uint32_t *__restrict__ perm, uint32_t n,
                                Tc *__restrict__ out) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t j = perm[i];
  for (int d = 0; d < ndim; ++d) out[uint64_t(i) * ndim + d] = coord[int64_t(j) * cs0 + d * cs1];
}

void launch_gather_coords(bool coord_f64, const void *coord, int64_t cs0, int64_t cs1, int ndim,
                          const uint32_t *perm, uint32_t n, void *out, cudaStream_t st) {
  if (n == 0) return;
  unsigned g = (n + 255) / 256;
  if (coord_f64)
    k_gather_coords<double><<<g, 256, 0, st>>>((const double *)coord, cs0, cs1, ndim, perm, n,
                                               (double *)out);
  else
    k_gather_coords<float><<<g, 256, 0, st>>>((const float *)coord, cs0, cs1, ndim, perm, n,
                                              (float *)out);
  DN_LAUNCHED();
}

// inverse of the gather: out[perm[i]] = sorted[i]
template <typename Tc>
__global__ void k_scatter_coords(const Tc *__restrict__ sorted, int ndim,
                                 const uint32_t *__restrict__ perm, uint32_t n, Tc *__restrict__ out) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t j = perm[i];
  for (int d = 0; d < ndim; ++d) out[uint64_t(j) * ndim + d] = sorted[uint64_t(i) * ndim + d];
}

void launch_scatter_coords(bool coord_f64, const void *sorted, int ndim, const uint32_t *perm,
                           uint32_t n, void *out, cudaStream_t st) {
  if (n == 0) return;
  unsigned g = (n + 255) / 256;
  if (coord_f64)
    k_scatter_coords<double><<<g, 256, 0, st>>>((const double *)sorted, ndim, perm, n, (double *)out);
  else
    k_scatter_coords<float><<<g, 256, 0, st>>>((const float *)sorted, ndim, perm, n, (float *)out);
  DN_LAUNCHED();
}

}  // namespace dnufft

namespace dnufft {

// ---------------------------------------------------------------- grouped index
// keys[i] = (keys[i] << gbits) | group[i]: points sorted by (tile, group)
__global__ void k_group_keys(uint32_t *__restrict__ keys, const uint32_t *__restrict__ group,
                             uint32_t n, int gbits) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    keys[i] = (keys[i] << gbits) | group[i];
}

// start[k] = first i with v[i] >= k, k = 0..nk, for ascending v: a binary
// search per k (the key space may hold long gaps, e.g. past the last tile)
__global__ void k_key_starts(const uint32_t *__restrict__ v, uint32_t n, uint32_t nk,
                             uint32_t *__restrict__ start) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k <= nk; k += gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
      const uint32_t mid = lo + (hi - lo) / 2;
      if (v[mid] < k) lo = mid + 1;
      else hi = mid;
    }
    start[k] = lo;
  }
}

// chunks of the points of groups [g0, g1) of every tile (at most `chunk`
// points each): counts, then (after a scan into pos) the records
__global__ void k_gchunk_count(const uint32_t *__restrict__ start, uint32_t ntiles, int gbits,
                               uint32_t g0, uint32_t g1, uint32_t chunk,
                               uint32_t *__restrict__ cnt) {
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t <= ntiles;
       t += gridDim.x * blockDim.x) {
    if (t == ntiles) {
      cnt[t] = 0;
      continue;
    }
    const uint32_t s = start[(uint64_t(t) << gbits) + g0], e = start[(uint64_t(t) << gbits) + g1];
    cnt[t] = (e - s + chunk - 1) / chunk;
  }
}

__global__ void k_gchunk_fill(const uint32_t *__restrict__ start,
                              const uint32_t *__restrict__ cnt, const uint32_t *__restrict__ pos,
                              uint32_t ntiles, int gbits, uint32_t g0, uint32_t g1,
                              uint32_t chunk, Chunk *__restrict__ chunks) {
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < ntiles;
       t += gridDim.x * blockDim.x) {
    const uint32_t s = start[(uint64_t(t) << gbits) + g0], e = start[(uint64_t(t) << gbits) + g1];
    for (uint32_t k = 0; k < cnt[t]; ++k) {
      Chunk c;
      c.start = s + k * chunk;
      c.count = min(chunk, e - c.start);
      c.tile = t;
      c.pad = 0;
      chunks[pos[t] + k] = c;
    }
  }
}

static unsigned grid_of(uint64_t n) {
  uint64_t b = (n + 255) / 256;
  return unsigned(b < 1 ? 1 : (b > 4096 ? 4096 : b));
}

void launch_group_keys(uint32_t *keys, const uint32_t *group, uint32_t n, int gbits,
                       cudaStream_t st) {
  if (n == 0) return;
  k_group_keys<<<grid_of(n), 256, 0, st>>>(keys, group, n, gbits);
  DN_LAUNCHED();
}

void launch_key_starts(const uint32_t *skeys, uint32_t n, uint32_t nkeys, uint32_t *start,
                       cudaStream_t st) {
  k_key_starts<<<grid_of(uint64_t(nkeys) + 1), 256, 0, st>>>(skeys, n, nkeys, start);
  DN_LAUNCHED();
}

size_t group_chunk_workspace_bytes(uint32_t ntiles) {
  return size_t(2) * (ntiles + 1) * 4 + 256 + scan_workspace_bytes(uint64_t(ntiles) + 1);
}

uint32_t build_group_chunks(const uint32_t *start, uint32_t ntiles, int gbits, uint32_t g0,
                            uint32_t g1, uint32_t chunk, Chunk *chunks, void *ws,
                            cudaStream_t st) {
  uint32_t *cnt = static_cast<uint32_t *>(ws);
  uint32_t *pos = cnt + (ntiles + 1);
  uint32_t *sws = reinterpret_cast<uint32_t *>(
      (reinterpret_cast<uintptr_t>(pos + ntiles + 1) + 255) & ~uintptr_t(255));
  k_gchunk_count<<<grid_of(uint64_t(ntiles) + 1), 256, 0, st>>>(start, ntiles, gbits, g0, g1,
                                                                chunk, cnt);
  DN_LAUNCHED();
  exclusive_scan(cnt, pos, uint64_t(ntiles) + 1, sws, st);
  k_gchunk_fill<<<grid_of(ntiles), 256, 0, st>>>(start, cnt, pos, ntiles, gbits, g0, g1, chunk,
                                                 chunks);
  DN_LAUNCHED();
  const uint32_t *src[1] = {pos + ntiles};
  uint32_t h = 0;
  read_words(src, 1, &h, st);
  return h;
}

}  // namespace dnufft
