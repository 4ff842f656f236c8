// Plain spreading / interpolation kernels, single precision (complex64 data).
#include "spread_impl.cuh"

namespace dnufft {

template <typename T>
void launch_spread(const PointsDesc &pts, const ChunkList &cl, const Geometry &g,
                   const KernelPoly<T> &kp, const void *values, int64_t vs, int64_t vtrans,
                   void *grid, int64_t gtrans, int ntrans, cudaStream_t st) {
  launch_spread_impl<T>(pts, cl, g, kp, values, vs, vtrans, grid, gtrans, ntrans, st);
}

template <typename T>
void launch_interp(const PointsDesc &pts, const ChunkList &cl, const Geometry &g,
                   const KernelPoly<T> &kp, const void *grid, int64_t gtrans, void *out,
                   int64_t os, int64_t otrans, int ntrans, cudaStream_t st, int *err) {
  launch_interp_impl<T>(pts, cl, g, kp, grid, gtrans, out, os, otrans, ntrans, st, err);
}

template void launch_spread<float>(const PointsDesc &, const ChunkList &, const Geometry &,
                                   const KernelPoly<float> &, const void *, int64_t, int64_t,
                                   void *, int64_t, int, cudaStream_t);
template void launch_interp<float>(const PointsDesc &, const ChunkList &, const Geometry &,
                                   const KernelPoly<float> &, const void *, int64_t, void *,
                                   int64_t, int64_t, int, cudaStream_t, int *);

}  // namespace dnufft

// ---- tensor map of a 2D grid for the TMA-staged interpolation tiles
#include <cudaTypedefs.h>

namespace dnufft {

bool encode_tile_map(CUtensorMap *map, const void *grid, bool f64, int64_t n0, int64_t n1,
                     int tpitch, int S) {
  static const PFN_cuTensorMapEncodeTiled_v12000 encode = [] {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault,
                                         &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      (void)cudaGetLastError();
      fn = nullptr;
    }
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }();
  if (!encode) return false;
  // the copy's rules: 16-byte base and row pitch, an even number of complex64
  // columns per box (16-byte inner extent), box sides up to 256 elements
  if ((reinterpret_cast<uintptr_t>(grid) & 15u) != 0 || (n1 & 1) != 0 || tpitch <= 0 ||
      (tpitch & 1) != 0 || 2 * tpitch > 256 || S > 256 || n0 < S || n1 < tpitch)
    return false;
  const cuuint64_t es = f64 ? 8 : 4;
  const cuuint64_t dims[2] = {cuuint64_t(2 * n1), cuuint64_t(n0)};
  const cuuint64_t strides[1] = {cuuint64_t(2 * n1) * es};
  const cuuint32_t box[2] = {cuuint32_t(2 * tpitch), cuuint32_t(S)};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r =
      encode(map, f64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
             const_cast<void *>(grid), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

}  // namespace dnufft
