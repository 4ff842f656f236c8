// Plain spreading / interpolation kernels, double precision (complex128 data).
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

template void launch_spread<double>(const PointsDesc &, const ChunkList &, const Geometry &,
                                   const KernelPoly<double> &, const void *, int64_t, int64_t,
                                   void *, int64_t, int, cudaStream_t);
template void launch_interp<double>(const PointsDesc &, const ChunkList &, const Geometry &,
                                   const KernelPoly<double> &, const void *, int64_t, void *,
                                   int64_t, int64_t, int, cudaStream_t, int *);

}  // namespace dnufft
