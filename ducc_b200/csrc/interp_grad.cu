// Coordinate gradients of the type-2 transform: interpolation with the
// derivative of the kernel.
//
// For points x_j and the type-2 result f(x_j) = sum_cells phi(x_j - cell) G[cell]
// (G the deconvolved, zero-padded, FFT-ed oversampled grid), this kernel
// returns, per point and axis,
//     grad[j][d] = Re( conj(w_j) * d f(x_j) / d x_{j,d} ),
// i.e. the vector-Jacobian product of the transform's coordinate dependence
// with the cotangent w (type 2: w = dL/df; type 1: the transform of the
// cotangent grid with the opposite sign, contracted with the values).  The
// kernel weights of tap k are phi_k(x) at x = W-1-2*frac with
// frac = r - i0 and r = (t/period - floor(t/period)) * n, so
//     d weight_k / d t = -2 * (n/period) * phi_k'(x).
// The staging is the interpolation kernel's (tile plus halo in shared memory,
// one thread per point); all NDIM derivatives come from one pass over the
// W^NDIM footprint.
#include "spread_impl.cuh"

namespace dnufft {

template <typename T, typename Tc, int NDIM, int W>
__global__ void __launch_bounds__(SP_THREADS)
    k_interp_dcoord(PointsDesc pts, const Chunk *__restrict__ chunks, Geometry g,
                    KernelPoly<T> kp, const cplx<T> *__restrict__ grid,
                    const cplx<T> *__restrict__ wts, int64_t ws, Tc *__restrict__ grad,
                    int64_t gs0, int64_t gs1) {
  constexpr bool SMEM = BufferLayout<T>::smem(NDIM);
  extern __shared__ __align__(16) unsigned char smraw[];
  const Chunk ch = chunks[blockIdx.x];
  const int S = (1 << g.log2tile) + W;
  int ncell = S;
  if (NDIM >= 2) ncell *= S;
  if (NDIM >= 3) ncell *= S;
  int b0[NDIM];
  tile_origin<NDIM>(ch.tile, g, b0);
  cplx<T> *buf = reinterpret_cast<cplx<T> *>(smraw);
  const uint32_t mS = fastdiv_magic(uint32_t(S));
  const bool fastwrap = fast_wrap_ok<NDIM>(g, S);
  if constexpr (SMEM) {
    for (int c = threadIdx.x; c < ncell; c += SP_THREADS)
      buf[c] = grid[cell_index<NDIM>(c, S, mS, fastwrap, b0, g)];
    __syncthreads();
  }
  T dscale[NDIM];
#pragma unroll
  for (int d = 0; d < NDIM; ++d) dscale[d] = T(-2.0 * double(g.nover[d]) * g.coordfct[d]);
  const uint32_t end = ch.start + ch.count;
  for (uint32_t i = ch.start + threadIdx.x; i < end; i += SP_THREADS) {
    Tc x[NDIM];
    uint32_t j = load_point<Tc, NDIM>(pts, i, x);
    T w[NDIM][W], dw[NDIM][W];
    int o[NDIM];
#pragma unroll
    for (int d = 0; d < NDIM; ++d) {
      int i0;
      double frac;
      fold<Tc>(x[d], g.coordfct[d], int(g.nover[d]), g.shift[d], g.maxi0[d], i0, frac);
      kernel_weights_deriv<T, W>(kp, T(double(W - 1) - 2.0 * frac), w[d], dw[d]);
      o[d] = i0 - b0[d];
    }
    cplx<T> D[NDIM];
#pragma unroll
    for (int d = 0; d < NDIM; ++d) D[d] = mkc<T>(T(0), T(0));
    if constexpr (NDIM == 1) {
#pragma unroll
      for (int a = 0; a < W; ++a) {
        cplx<T> gv = buf[o[0] + a];
        D[0].x += dw[0][a] * gv.x;
        D[0].y += dw[0][a] * gv.y;
      }
    } else if constexpr (NDIM == 2) {
#pragma unroll
      for (int a = 0; a < W; ++a) {
        const cplx<T> *row = buf + (o[0] + a) * S + o[1];
        T rr = 0, ri = 0, dr = 0, di = 0;
#pragma unroll
        for (int b = 0; b < W; ++b) {
          cplx<T> gv = row[b];
          rr += w[1][b] * gv.x;
          ri += w[1][b] * gv.y;
          dr += dw[1][b] * gv.x;
          di += dw[1][b] * gv.y;
        }
        D[0].x += dw[0][a] * rr;
        D[0].y += dw[0][a] * ri;
        D[1].x += w[0][a] * dr;
        D[1].y += w[0][a] * di;
      }
    } else {
      const int nu = int(g.nover[0]), nv = int(g.nover[1]), nw = int(g.nover[2]);
#pragma unroll 1
      for (int a = 0; a < W; ++a) {
        T pr = 0, pi = 0, p1r = 0, p1i = 0, p2r = 0, p2i = 0;
#pragma unroll 2
        for (int b = 0; b < W; ++b) {
          const cplx<T> *row;
          if constexpr (SMEM) {
            row = buf + ((o[0] + a) * S + (o[1] + b)) * S + o[2];
          } else {
            const int iu = fastwrap ? wrap1(b0[0] + o[0] + a, nu) : wrapi(b0[0] + o[0] + a, nu);
            const int iv = fastwrap ? wrap1(b0[1] + o[1] + b, nv) : wrapi(b0[1] + o[1] + b, nv);
            row = grid + (int64_t(iu) * nv + iv) * nw;
          }
          T rr = 0, ri = 0, dr = 0, di = 0;
#pragma unroll
          for (int e = 0; e < W; ++e) {
            cplx<T> gv;
            if constexpr (SMEM) gv = row[e];
            else gv = __ldg(row + (fastwrap ? wrap1(b0[2] + o[2] + e, nw) : wrapi(b0[2] + o[2] + e, nw)));
            rr += w[2][e] * gv.x;
            ri += w[2][e] * gv.y;
            dr += dw[2][e] * gv.x;
            di += dw[2][e] * gv.y;
          }
          pr += w[1][b] * rr;
          pi += w[1][b] * ri;
          p1r += dw[1][b] * rr;
          p1i += dw[1][b] * ri;
          p2r += w[1][b] * dr;
          p2i += w[1][b] * di;
        }
        D[0].x += dw[0][a] * pr;
        D[0].y += dw[0][a] * pi;
        D[1].x += w[0][a] * p1r;
        D[1].y += w[0][a] * p1i;
        D[2].x += w[0][a] * p2r;
        D[2].y += w[0][a] * p2i;
      }
    }
    const cplx<T> c = wts[int64_t(j) * ws];
#pragma unroll
    for (int d = 0; d < NDIM; ++d)
      grad[int64_t(j) * gs0 + int64_t(d) * gs1] = Tc((c.x * D[d].x + c.y * D[d].y) * dscale[d]);
  }
}

template <typename T, typename Tc, int NDIM, int W>
static void dcoord_w(const PointsDesc &pts, const ChunkList &cl, const Geometry &g,
                     const KernelPoly<T> &kp, const void *grid, const void *wts, int64_t ws,
                     void *grad, int64_t gs0, int64_t gs1, cudaStream_t st) {
  size_t sm = interp_smem_bytes<T, NDIM, W>(g);
  auto kern = k_interp_dcoord<T, Tc, NDIM, W>;
  DN_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
  kern<<<cl.nchunks, SP_THREADS, sm, st>>>(pts, cl.chunks, g, kp,
                                          static_cast<const cplx<T> *>(grid),
                                          static_cast<const cplx<T> *>(wts), ws,
                                          static_cast<Tc *>(grad), gs0, gs1);
  DN_LAUNCHED();
}

template <typename T, typename Tc, int NDIM>
static void dcoord_dispatch(const PointsDesc &pts, const ChunkList &cl, const Geometry &g,
                            const KernelPoly<T> &kp, const void *grid, const void *wts,
                            int64_t ws, void *grad, int64_t gs0, int64_t gs1, cudaStream_t st) {
#define DN_CASE(WW) \
  case WW: dcoord_w<T, Tc, NDIM, WW>(pts, cl, g, kp, grid, wts, ws, grad, gs0, gs1, st); return;
  if constexpr (sizeof(T) == 4) {
    switch (g.W) { DN_FOR_W_FLOAT(DN_CASE) }
  } else {
    switch (g.W) { DN_FOR_W_DOUBLE(DN_CASE) }
  }
#undef DN_CASE
  throw Error(ST_UNSUPPORTED, "kernel support not supported by this build");
}

template <typename T>
void launch_interp_dcoord(const PointsDesc &pts, const ChunkList &cl, const Geometry &g,
                          const KernelPoly<T> &kp, const void *grid, const void *wts,
                          int64_t ws, void *grad, int64_t gs0, int64_t gs1, cudaStream_t st) {
  if (cl.nchunks == 0) return;
#define DN_DC(TC, ND) dcoord_dispatch<T, TC, ND>(pts, cl, g, kp, grid, wts, ws, grad, gs0, gs1, st)
  if (pts.coord_f64) {
    if (g.ndim == 1) DN_DC(double, 1); else if (g.ndim == 2) DN_DC(double, 2); else DN_DC(double, 3);
  } else {
    if (g.ndim == 1) DN_DC(float, 1); else if (g.ndim == 2) DN_DC(float, 2); else DN_DC(float, 3);
  }
#undef DN_DC
}

template void launch_interp_dcoord<float>(const PointsDesc &, const ChunkList &, const Geometry &,
                                          const KernelPoly<float> &, const void *, const void *,
                                          int64_t, void *, int64_t, int64_t, cudaStream_t);
template void launch_interp_dcoord<double>(const PointsDesc &, const ChunkList &,
                                           const Geometry &, const KernelPoly<double> &,
                                           const void *, const void *, int64_t, void *, int64_t,
                                           int64_t, cudaStream_t);

}  // namespace dnufft
