// Host-callable launchers of the CUDA kernels (defined in the .cu files).
#pragma once

#include "dnufft_internal.h"

namespace dnufft {

// ---- binning / sorting (binsort.cu)
// quadrant_bits: append the point's quadrant within its 2D tile as two extra
// key bits and, below them, the Morton code of its cell within the quadrant
// (2 * (log2tile - 1) bits): the tensor-core spreader's processing order
void launch_fold_keys(bool coord_f64, const void *coord, int64_t cs0, int64_t cs1,
                      uint32_t npts, const Geometry &g, uint32_t *keys, uint32_t *idx,
                      cudaStream_t st, bool quadrant_bits = false);
// bits of the within-quadrant cell order in a tensor-core sort key
inline int tc_cell_bits(const Geometry &g) { return 2 * (g.log2tile - 1); }
size_t scan_workspace_bytes(uint64_t n);
void exclusive_scan(const uint32_t *in, uint32_t *out, uint64_t n, uint32_t *ws,
                    cudaStream_t st);
size_t radix_workspace_bytes(uint32_t n, int keybits);
void radix_sort_pairs(uint32_t *keys, uint32_t *vals, uint32_t n, int keybits, void *ws,
                      cudaStream_t st);
size_t chunk_workspace_bytes(uint32_t n);
uint32_t build_chunks(const uint32_t *skeys, uint32_t n, int tile_shift, uint32_t chunk,
                      Chunk *chunks, uint32_t *d_count, void *ws, cudaStream_t st,
                      bool zero_copy = true);
// reads n (1..8) device words into out through mapped host memory; synchronises st
void read_words(const uint32_t *const *src, int n, uint32_t *out, cudaStream_t st);
void launch_gather_coords(bool coord_f64, const void *coord, int64_t cs0, int64_t cs1,
                          int ndim, const uint32_t *perm, uint32_t n, void *out,
                          cudaStream_t st);

// grouped index (points sorted by (tile, group)): keys = keys << gbits | group;
// start[k] (k = 0..nkeys) = first sorted point whose key is >= k; the chunks
// (at most `chunk` points) of groups [g0, g1) of every tile, their number
// returned (read back: synchronises st)
void launch_group_keys(uint32_t *keys, const uint32_t *group, uint32_t n, int gbits,
                       cudaStream_t st);
void launch_key_starts(const uint32_t *skeys, uint32_t n, uint32_t nkeys, uint32_t *start,
                       cudaStream_t st);
size_t group_chunk_workspace_bytes(uint32_t ntiles);
uint32_t build_group_chunks(const uint32_t *start, uint32_t ntiles, int gbits, uint32_t g0,
                            uint32_t g1, uint32_t chunk, Chunk *chunks, void *ws,
                            cudaStream_t st);

void launch_scatter_coords(bool coord_f64, const void *sorted, int ndim, const uint32_t *perm,
                           uint32_t n, void *out, cudaStream_t st);

// ---- spreading / interpolation (spread_*.cu)
struct PointsDesc {
  const void *coord;      // sorted==true: contiguous (npts, ndim) in tile order
  int64_t cs0, cs1;       //   else the caller's array, addressed through perm
  bool sorted;
  bool coord_f64;
  const uint32_t *perm;   // tile order -> caller's point index
  uint32_t npts;
};

struct ChunkList {
  const Chunk *chunks;
  uint32_t nchunks;
};

// grid: contiguous oversampled grid (nover[0] x ... ), complex<T>
// values: caller's point values, complex<T>, element stride vs; ntrans
// transforms, values of transform t at values + t*vtrans, grids at grid + t*gtrans
template <typename T>
void launch_spread(const PointsDesc &pts, const ChunkList &cl, const Geometry &g,
                   const KernelPoly<T> &kp, const void *values, int64_t vs,
                   int64_t vtrans, void *grid, int64_t gtrans, int ntrans,
                   cudaStream_t st);

// err: device error word; with it, 2D single-transform tiles inside the grid
// are staged by TMA (a copy that never completes sets the word)
template <typename T>
void launch_interp(const PointsDesc &pts, const ChunkList &cl, const Geometry &g,
                   const KernelPoly<T> &kp, const void *grid, int64_t gtrans,
                   void *out, int64_t os, int64_t otrans, int ntrans, cudaStream_t st,
                   int *err = nullptr);

// grad[j*gs0 + d*gs1] = Re(conj(wts[j*ws]) * d/dx_{j,d} interp(grid)(x_j)), in
// the coordinates' dtype (interp_grad.cu)
template <typename T>
void launch_interp_dcoord(const PointsDesc &pts, const ChunkList &cl, const Geometry &g,
                          const KernelPoly<T> &kp, const void *grid, const void *wts,
                          int64_t ws, void *grad, int64_t gs0, int64_t gs1, cudaStream_t st);

// ---- split-precision tensor-core spreader (spread_tc.cu): 2D, complex64
// failure-path self-test of the bounded device waits (sets word *err)
void launch_wait_selftest(int *err, unsigned long long limit_ns, cudaStream_t st);
bool spread_tc_supported(const Geometry &g, bool calc_f64);
// K-block list of a (tile, quadrant)-sorted point set: records {first sorted
// point, meta} of <= 16 points of one quadrant of one chunk, and the K-block
// range [range[b], range[b+1]) of each of 'groups' persistent CTAs
struct TcBlocks {
  const uint2 *kblk;
  const uint32_t *range;
  uint32_t groups;
  uint32_t total;
};
size_t tc_kblock_workspace_bytes(uint32_t nchunks);
uint32_t tc_kblock_upper_bound(uint32_t npts, uint32_t nchunks);
// returns the number of K-blocks (reads it back: synchronises the stream)
// (cell_bits: the key bits below the quadrant bits, tc_cell_bits)
uint32_t build_tc_kblocks(const uint32_t *skeys, const ChunkList &cl, uint32_t groups, void *ws,
                          uint2 *kblk, uint32_t *range, uint32_t *d_total, int cell_bits,
                          cudaStream_t st);
void launch_spread_tc(const PointsDesc &pts, const TcBlocks &tb, const Geometry &g,
                      const KernelPoly<float> &kp, const void *values, int64_t vs, void *grid,
                      unsigned *absmax, int *err, cudaStream_t st);

// ---- FFT and correction (fft.cu)
struct FFTAxisPlan {
  int n;
  int nfac;
  int fac[24];
  const void *tw;   // device table of n twiddles exp(-2 pi i k/n) (float2/double2)
};

// Type 1 tail: FFTs over the oversampled grid with output pruning, then
// deconvolution + crop into the caller's uniform array (arbitrary strides).
// work: n0 x N1 scratch for the four-step column passes of 2D grids
// (fft_work_bytes; may be null: the single-pass column kernel is used); err:
// device error word for the bounded waits of the persistent row kernel (null:
// the row kernel is not used)
template <typename T>
void fft_nu2u_tail(void *grid, const Geometry &g, const FFTAxisPlan *ax, bool forward,
                   const double *const corfac[3], bool fft_order, void *out,
                   const int64_t *ostride, cudaStream_t st, void *work = nullptr,
                   int *err = nullptr);

// The two halves of the 2D type-1 tail: row FFTs (axis 1, kept columns written
// in place) over nrows consecutive rows of the oversampled grid, and column
// FFTs of the kept columns with correction and crop into out.
template <typename T>
void fft_nu2u_rows(void *rows, int nrows, const Geometry &g, const FFTAxisPlan *ax, bool forward,
                   cudaStream_t st, int *err);
template <typename T>
void fft_nu2u_cols(void *grid, const Geometry &g, const FFTAxisPlan *ax, bool forward,
                   const double *const corfac[3], bool fft_order, void *out,
                   const int64_t *ostride, cudaStream_t st, void *work);
// The same for kept columns col0 .. col0 + ncols - 1 only, packed in (n0, ncols)
// cols, into an (N0, ncols) out (column x: kept column col0 + x); false when the
// four-step column passes do not apply (n0 < 1024 or no pencil plan)
template <typename T>
bool fft_nu2u_cols_range(void *cols, int ncols, int col0, const Geometry &g,
                         const FFTAxisPlan *ax, bool forward, const double *const corfac[3],
                         bool fft_order, void *out, const int64_t *ostride, cudaStream_t st,
                         void *work);

// Type 2 halves for a split transform (2D): the column pass of a block of kept
// columns from the uniform array into an (n0, ncols) array (false when the
// four-step column passes do not apply), and the row FFTs of a slab of rows
// whose kept columns are set (whole rows out, in place)
template <typename T>
bool fft_u2nu_cols_range(const void *uni, const int64_t *istride, const Geometry &g,
                         const FFTAxisPlan *ax, bool forward, const double *const corfac[3],
                         bool fft_order, void *cols, int ncols, int col0, cudaStream_t st,
                         void *work);
template <typename T>
void fft_u2nu_rows(void *rows, int nrows, const Geometry &g, const FFTAxisPlan *ax, bool forward,
                   cudaStream_t st, int *err);

// Type 2 head: deconvolution + zero-pad of the caller's uniform array into the
// oversampled grid, then FFTs with input pruning.
template <typename T>
void fft_u2nu_head(const void *uni, const int64_t *istride, const Geometry &g,
                   const FFTAxisPlan *ax, bool forward, const double *const corfac[3],
                   bool fft_order, void *grid, cudaStream_t st, void *work = nullptr,
                   int *err = nullptr);
size_t fft_work_bytes(const Geometry &g, size_t esize);

void zero_strided(void *ptr, int ndim, const int64_t *shape, const int64_t *stride, size_t esize,
                  cudaStream_t st);

// ---- batched transforms (batch.cu, fft.cu)
// caller's array of one instance in a per-call device table: stride[0] between
// transforms, stride[1..] per axis (elements)
struct BatchArray {
  void *ptr;
  int64_t stride[4];
};

struct FFTBatchInst {
  Geometry g;
  const FFTAxisPlan *ax;      // host copies (twiddle pointers are device memory)
  const double *corfac[3];    // device
  void *grid;                 // ntrans oversampled grids, back to back
  int ntrans;
  bool fft_order;
};
// line passes of all instances, one launch per pass; type 0 = type 1 tail
// (rows, then kept columns with correction into the uniform arrays), type 1 =
// type 2 head (columns from the uniform arrays, then rows)
template <typename T>
void *fft_batch_create(const std::vector<FFTBatchInst> &insts, cudaStream_t st);
template <typename T>
void fft_batch_run(void *h, int type, const BatchArray *uni, bool fwd, cudaStream_t st);
void fft_batch_destroy(void *h);

template <typename T> struct SpreadInst {
  PointsDesc pts;
  const Chunk *chunks;
  Geometry g;
  KernelPoly<T> kp;
  void *grid;        // ntrans grids back to back
  int ntrans;
  uint32_t chunk0;   // first chunk of this instance in the launch
};
// one launch over the chunks of all instances (x) and their transforms (y);
// vals: per-call table of the point arrays (type 1 input, type 2 output)
template <typename T>
void launch_spread_multi(const SpreadInst<T> *insts, int ninst, uint32_t nchunks, int max_ntrans,
                         size_t smem, const BatchArray *vals, cudaStream_t st);
template <typename T>
void launch_interp_multi(const SpreadInst<T> *insts, int ninst, uint32_t nchunks, int max_ntrans,
                         size_t smem, const BatchArray *vals, cudaStream_t st);
template <typename T> size_t spread_multi_smem(const Geometry &g);
template <typename T> size_t interp_multi_smem(const Geometry &g);

}  // namespace dnufft
