// Multi-instance spreading and interpolation for batched transforms: one
// launch covers the chunks of every instance of a batch (x) and every
// transform of an instance (y).  CTA x finds its instance by binary search over
// the first-chunk prefix, copies the instance's descriptor (geometry, kernel
// polynomial, point arrays) into shared memory and runs the same per-chunk body
// as the single-transform kernels, dispatching on the instance's coordinate
// type and kernel support at run time.  The point arrays of a call come from a
// per-call device table, so a captured graph replays on new arrays.
#include "spread_impl.cuh"

namespace dnufft {

template <typename T>
__device__ __forceinline__ int find_instance(const SpreadInst<T> *__restrict__ insts, int ninst,
                                             uint32_t b) {
  int lo = 0, hi = ninst - 1;   // last instance with chunk0 <= b
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (insts[mid].chunk0 <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

template <typename T>
__device__ __forceinline__ void load_instance(const SpreadInst<T> *__restrict__ insts, int ninst,
                                              SpreadInst<T> &si) {
  __shared__ int s_i;
  if (threadIdx.x == 0) s_i = find_instance(insts, ninst, blockIdx.x);
  __syncthreads();
  const uint32_t *src = reinterpret_cast<const uint32_t *>(insts + s_i);
  for (int i = threadIdx.x; i < int(sizeof(SpreadInst<T>) / 4); i += blockDim.x)
    reinterpret_cast<uint32_t *>(&si)[i] = src[i];
  __syncthreads();
}

#define DN_W_SWITCH_F(X) \
  switch (W) { case 4: X(4) break; case 5: X(5) break; case 6: X(6) break; case 7: X(7) break; \
               case 8: X(8) break; default: break; }
#define DN_W_SWITCH_D(X)                                                                       \
  switch (W) { case 4: X(4) break; case 5: X(5) break; case 6: X(6) break; case 7: X(7) break; \
               case 8: X(8) break; case 9: X(9) break; case 10: X(10) break;                  \
               case 11: X(11) break; case 12: X(12) break; case 13: X(13) break;              \
               case 14: X(14) break; case 15: X(15) break; case 16: X(16) break;              \
               default: break; }

// CTAs per SM the register allocation must allow: the kernels hold every
// support and both coordinate types, and without a bound the largest case sets
// the register count for all (110 for single precision: two CTAs per SM,
// too few warps for the short CTAs of small instances)
template <typename T> constexpr int multi_spread_min_ctas() { return sizeof(T) == 4 ? 4 : 1; }
template <typename T> constexpr int multi_interp_min_ctas() { return sizeof(T) == 4 ? 6 : 1; }

template <typename T>
__global__ void __launch_bounds__(SP_THREADS, multi_spread_min_ctas<T>())
    k_spread_multi(const SpreadInst<T> *__restrict__ insts, int ninst,
                   const BatchArray *__restrict__ vals) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ SpreadInst<T> si;
  load_instance(insts, ninst, si);
  const int t = blockIdx.y;
  if (t >= si.ntrans) return;
  const BatchArray a = vals[find_instance(insts, ninst, blockIdx.x)];
  const cplx<T> *values = static_cast<const cplx<T> *>(a.ptr) + int64_t(t) * a.stride[0];
  cplx<T> *grid = static_cast<cplx<T> *>(si.grid) +
                  int64_t(t) * si.g.nover[0] * si.g.nover[1];
  const Chunk ch = si.chunks[blockIdx.x - si.chunk0];
  const int W = si.g.W;
#define DN_SC(WW)                                                                            \
  if (si.pts.coord_f64)                                                                      \
    spread_chunk<T, double, 2, WW>(si.pts, ch, si.g, si.kp, values, a.stride[1], grid, smraw); \
  else                                                                                       \
    spread_chunk<T, float, 2, WW>(si.pts, ch, si.g, si.kp, values, a.stride[1], grid, smraw);
  if constexpr (sizeof(T) == 4) {
    DN_W_SWITCH_F(DN_SC)
  } else {
    DN_W_SWITCH_D(DN_SC)
  }
#undef DN_SC
}

template <typename T>
__global__ void __launch_bounds__(SP_THREADS, multi_interp_min_ctas<T>())
    k_interp_multi(const SpreadInst<T> *__restrict__ insts, int ninst,
                   const BatchArray *__restrict__ outs) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ SpreadInst<T> si;
  load_instance(insts, ninst, si);
  const int t = blockIdx.y;
  if (t >= si.ntrans) return;
  const BatchArray a = outs[find_instance(insts, ninst, blockIdx.x)];
  cplx<T> *out = static_cast<cplx<T> *>(a.ptr) + int64_t(t) * a.stride[0];
  const cplx<T> *grid = static_cast<const cplx<T> *>(si.grid) +
                        int64_t(t) * si.g.nover[0] * si.g.nover[1];
  const Chunk ch = si.chunks[blockIdx.x - si.chunk0];
  const int W = si.g.W;
#define DN_IC(WW)                                                                          \
  if (si.pts.coord_f64)                                                                    \
    interp_chunk<T, double, 2, WW>(si.pts, ch, si.g, si.kp, grid, out, a.stride[1], smraw); \
  else                                                                                     \
    interp_chunk<T, float, 2, WW>(si.pts, ch, si.g, si.kp, grid, out, a.stride[1], smraw);
  if constexpr (sizeof(T) == 4) {
    DN_W_SWITCH_F(DN_IC)
  } else {
    DN_W_SWITCH_D(DN_IC)
  }
#undef DN_IC
}

template <typename T> size_t spread_multi_smem(const Geometry &g) {
  size_t r = 0;
#define DN_SM(WW) r = spread_smem_bytes<T, 2, WW>(g);
  const int W = g.W;
  if constexpr (sizeof(T) == 4) {
    DN_W_SWITCH_F(DN_SM)
  } else {
    DN_W_SWITCH_D(DN_SM)
  }
#undef DN_SM
  return r;
}

template <typename T> size_t interp_multi_smem(const Geometry &g) {
  size_t r = 0;
#define DN_SM(WW) r = interp_smem_bytes<T, 2, WW>(g);
  const int W = g.W;
  if constexpr (sizeof(T) == 4) {
    DN_W_SWITCH_F(DN_SM)
  } else {
    DN_W_SWITCH_D(DN_SM)
  }
#undef DN_SM
  return r;
}

template <typename T>
void launch_spread_multi(const SpreadInst<T> *insts, int ninst, uint32_t nchunks, int max_ntrans,
                         size_t smem, const BatchArray *vals, cudaStream_t st) {
  if (nchunks == 0) return;
  DN_CUDA(cudaFuncSetAttribute(k_spread_multi<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(smem)));
  k_spread_multi<T><<<dim3(nchunks, max_ntrans), SP_THREADS, smem, st>>>(insts, ninst, vals);
  DN_LAUNCHED();
}

template <typename T>
void launch_interp_multi(const SpreadInst<T> *insts, int ninst, uint32_t nchunks, int max_ntrans,
                         size_t smem, const BatchArray *outs, cudaStream_t st) {
  if (nchunks == 0) return;
  DN_CUDA(cudaFuncSetAttribute(k_interp_multi<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(smem)));
  k_interp_multi<T><<<dim3(nchunks, max_ntrans), SP_THREADS, smem, st>>>(insts, ninst, outs);
  DN_LAUNCHED();
}

template void launch_spread_multi<float>(const SpreadInst<float> *, int, uint32_t, int, size_t,
                                         const BatchArray *, cudaStream_t);
template void launch_spread_multi<double>(const SpreadInst<double> *, int, uint32_t, int, size_t,
                                          const BatchArray *, cudaStream_t);
template void launch_interp_multi<float>(const SpreadInst<float> *, int, uint32_t, int, size_t,
                                         const BatchArray *, cudaStream_t);
template void launch_interp_multi<double>(const SpreadInst<double> *, int, uint32_t, int, size_t,
                                          const BatchArray *, cudaStream_t);
template size_t spread_multi_smem<float>(const Geometry &);
template size_t spread_multi_smem<double>(const Geometry &);
template size_t interp_multi_smem<float>(const Geometry &);
template size_t interp_multi_smem<double>(const Geometry &);

}  // namespace dnufft
