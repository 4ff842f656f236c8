/*
 * ducc_b200.h - C-ABI of the B200 (sm_100a) NUFFT library.
 *
 * A drop-in for DUCC's type-1 / type-2 non-uniform FFT: the entry points below
 * are the ones a binding of DUCC's NUFFT module binds (Python: python/nufft_pymod.cc,
 * Julia: julia/ducc_julia.cc), with plain pointers, sizes and status codes.
 * No C++ or torch types cross this boundary.
 *
 * Arrays are described by dnufft_array (modelled on DUCC's ArrayDescriptor,
 * src/ducc0/bindings/array_descriptor.h:35-45).  Data may live in device memory
 * (used in place, zero-copy) or in host memory (staged through the device inside
 * the call; host arrays must be C-contiguous).
 *
 * Every function returns 0 on success and a DNUFFT_ERR_* code otherwise; the
 * message of the last failure on the calling thread is dnufft_last_error().
 * Argument errors are detected before any kernel is launched.
 */
#ifndef DUCC_B200_H
#define DUCC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define DNUFFT_OK 0
#define DNUFFT_ERR_BADARG 1       /* shape / dtype / stride / size mismatch        */
#define DNUFFT_ERR_EPSILON 2      /* no kernel reaches the requested epsilon       */
#define DNUFFT_ERR_OOM 3          /* device allocation failed                      */
#define DNUFFT_ERR_CUDA 4         /* CUDA runtime error                            */
#define DNUFFT_ERR_TIMEOUT 5      /* a bounded device-side wait gave up            */
#define DNUFFT_ERR_UNSUPPORTED 6  /* valid request outside what this build handles */
#define DNUFFT_ERR_INTERNAL 7

/* dtype codes */
#define DNUFFT_F32 1
#define DNUFFT_F64 2
#define DNUFFT_C64 3
#define DNUFFT_C128 4
#define DNUFFT_U8 5    /* masks of the w-gridder                                 */

/* spreader selection (type 1) */
/* AUTO: the tensor-core form for 2D complex64 type 1 with at least 0.5 points
   per uniform mode (where it is measured faster), else plain */
#define DNUFFT_SPREAD_AUTO 0
#define DNUFFT_SPREAD_PLAIN 1  /* per-point FP32/FP64 atomics in shared memory   */
#define DNUFFT_SPREAD_TC 2     /* split-precision FP16 tcgen05 tile contraction  */

typedef struct dnufft_array {
  void *data;          /* first element                                       */
  int32_t dtype;       /* DNUFFT_F32 / F64 / C64 / C128                        */
  int32_t ndim;        /* 1..4                                                 */
  int64_t shape[4];
  int64_t stride[4];   /* in elements (not bytes); may be any non-zero value   */
} dnufft_array;

typedef struct dnufft_opts {
  size_t nthreads;        /* as in DUCC; only feeds DUCC's parameter cost model  */
  double sigma_min;       /* minimum / maximum oversampling factor               */
  double sigma_max;
  double periodicity[3];  /* per axis                                            */
  int32_t fft_order;      /* 0: most negative mode first, 1: zero mode first     */
  int32_t verbosity;      /* 1: print sizes and a CUDA-event stage profile       */
  int32_t spreader;       /* DNUFFT_SPREAD_*                                     */
  int32_t simd_lanes;     /* SIMD width DUCC's cost model assumes (default 8)    */
  int32_t force_kernel;   /* >=0: use this kernel-table row instead of choosing  */
  int32_t log2tile;       /* 0: DUCC's tile size; 2D/3D: 4 or 5, 1D: 9 (tuning) */
  int64_t force_nover[3]; /* with force_kernel: oversampled sizes                */
} dnufft_opts;

typedef struct dnufft_plan dnufft_plan;

typedef struct dnufft_plan_info {
  int32_t ndim;
  int32_t supp;           /* kernel support W                                    */
  int32_t kernel_index;   /* row of the kernel table                             */
  int32_t log2tile;
  int64_t nuni[3];
  int64_t nover[3];
  double ofactor;
  double beta;            /* beta (already multiplied by W) and exponent e0      */
  double e0;
  int64_t npoints;
  int32_t coord_f64;
  int32_t calc_f64;
  int64_t nchunks;        /* tile chunks of the sorted points                    */
  int64_t tc_records;     /* tensor-core plans: K-block records (<= 1 MMA each)  */
} dnufft_plan_info;

/* Fill *opts with the defaults of DUCC's functions (for_plan=0:
 * nthreads=1, sigma 1.2..2.51) or of its plan class (for_plan=1:
 * nthreads=0, sigma 1.1..2.6); periodicity 2*pi, fft_order 0.
 * Replaces the keyword defaults of python/nufft_pymod.cc:445-471. */
void dnufft_default_opts(dnufft_opts *opts, int for_plan);

/* Smallest epsilon reachable for ndim / precision / sigma range.
 * Replaces ducc0.nufft.bestEpsilon (python/nufft_pymod.cc:458-459,
 * src/ducc0/math/gridding_kernel.cc:1562-1576; Julia nufft_best_epsilon,
 * julia/ducc_julia.cc:176-186). */
int dnufft_best_epsilon(size_t ndim, int singleprec, double sigma_min, double sigma_max,
                        double *out);

/* Type 1: out[k] = sum_j points[j] exp(-+ i 2pi k.coord_j / period).
 * points: (M,) C64|C128; coord: (M, ndim) F32|F64; out: ndim-D grid of the
 * points' dtype (its shape defines the grid).  forward!=0 means exponent -1.
 * Replaces ducc0.nufft.nu2u (python/nufft_pymod.cc:113-137 ->
 * src/ducc0/nufft/nufft.h:1897-1927; Julia nufft_nu2u, julia/ducc_julia.cc:247-312). */
int dnufft_nu2u(const dnufft_array *points, const dnufft_array *coord, int forward,
                double epsilon, dnufft_array *out, const dnufft_opts *opts, void *stream);

/* Type 2: out[j] = sum_k grid[k] exp(-+ i 2pi k.coord_j / period).
 * Replaces ducc0.nufft.u2nu (python/nufft_pymod.cc:52-94 ->
 * src/ducc0/nufft/nufft.h:1928-1958; Julia nufft_u2nu, julia/ducc_julia.cc:188-245). */
int dnufft_u2nu(const dnufft_array *grid, const dnufft_array *coord, int forward,
                double epsilon, dnufft_array *out, const dnufft_opts *opts, void *stream);

/* Plan for repeated transforms with fixed coordinates: the points are binned,
 * sorted and their coordinates copied in tile order once.  Coordinate dtype
 * fixes the precision (F32 coords -> C64 data, F64 coords -> C128 data).
 * Replaces ducc0.nufft.plan.__init__ (python/nufft_pymod.cc:200-237 ->
 * src/ducc0/nufft/nufft.h:452-462; Julia nufft_make_plan, julia/ducc_julia.cc:314-370). */
int dnufft_plan_create(int nu2u, const dnufft_array *coord, const int64_t *grid_shape,
                       int ndim, double epsilon, const dnufft_opts *opts, void *stream,
                       dnufft_plan **plan);

/* Replaces plan.nu2u (python/nufft_pymod.cc:240-249, :170-183;
 * Julia nufft_nu2u_planned, julia/ducc_julia.cc:394-457).  Extension: with a
 * leading axis of ntrans on both arrays, points (ntrans, M) and out
 * (ntrans, N...), the call runs ntrans transforms over the plan's points
 * (the same for dnufft_plan_u2nu, grid (ntrans, N...) and out (ntrans, M)). */
int dnufft_plan_nu2u(dnufft_plan *plan, int forward, int verbosity,
                     const dnufft_array *points, dnufft_array *out, void *stream);

/* Replaces plan.u2nu (python/nufft_pymod.cc:250-259, :184-197;
 * Julia nufft_u2nu_planned, julia/ducc_julia.cc:459-522). */
int dnufft_plan_u2nu(dnufft_plan *plan, int forward, int verbosity,
                     const dnufft_array *grid, dnufft_array *out, void *stream);

/* Coordinate gradient of a type-2 transform (no counterpart in DUCC; it serves
 * differentiation with respect to the points):
 *   grad[j][d] = Re( conj(weights[j]) * d/dcoord[j][d] u2nu(grid, coord, forward)[j] )
 * computed by interpolating the transformed grid with the derivative of the
 * kernel.  weights: (M,) of the grid's dtype; grad: (M, ndim) real, the dtype
 * of the coordinates.  With weights = dL/d(u2nu result) this is the
 * coordinate part of the type-2 vector-Jacobian product; the type-1 one is
 * grad[j][d] = Re(conj(points[j]) * d/dcoord u2nu(cotangent, coord, !forward)[j]),
 * i.e. this call with grid = the cotangent and weights = the points. */
int dnufft_u2nu_dcoord(const dnufft_array *grid, const dnufft_array *coord, int forward,
                       double epsilon, const dnufft_array *weights, dnufft_array *grad,
                       const dnufft_opts *opts, void *stream);
int dnufft_plan_u2nu_dcoord(dnufft_plan *plan, int forward, const dnufft_array *grid,
                            const dnufft_array *weights, dnufft_array *grad, void *stream);

/* Type 1 in two halves, for one transform whose points are split over several
 * GPUs (no counterpart in DUCC, whose transforms run on one node's threads):
 * each process makes a plan of its own points (with the kernel and
 * oversampled sizes of the whole transform, see dnufft_find_parameters),
 * dnufft_plan_spread writes the spread of its points into an oversampled grid
 * (zeroed first), the caller sums these grids over the processes (one
 * all-reduce), and dnufft_plan_grid_to_uniform runs the FFT and the
 * correction of the summed grid (which it overwrites) into out.  Spreading is
 * linear in the values, so the result is the type 1 of all points.  grid: a
 * C-contiguous device array of the plan's data type with the plan's
 * oversampled shape (dnufft_plan_info.nover).  The two halves are
 * src/ducc0/nufft/nufft.h:1279-1285 (zeroing and spreading) and :1286-1312
 * (FFT and correction) of DUCC's 2D nonuni2uni (1D and 3D alike). */
int dnufft_plan_spread(dnufft_plan *plan, const dnufft_array *points, dnufft_array *grid,
                       void *stream);
int dnufft_plan_grid_to_uniform(dnufft_plan *plan, int forward, dnufft_array *grid,
                                dnufft_array *out, void *stream);

/* The FFT half of a 2D type 1 split once more, for an exchange that moves
 * fewer bytes than summing whole grids: each process sums one slab of rows of
 * the spread grids (a reduce-scatter), dnufft_plan_rows_fft transforms those
 * rows along axis 1 in place (rows: a C-contiguous device array of (r,
 * nover[1]) cells, any r <= nover[0]; only the nuni[1] kept columns, the first
 * (nuni[1]+1)/2 and the last nuni[1]/2, are written), the processes gather
 * the kept columns of all rows, and dnufft_plan_cols_to_uniform runs the
 * column FFTs, the correction and the crop into out.  Its grid is either the
 * whole oversampled grid with the kept columns in place (other columns are
 * not read) or the kept columns packed, a C-contiguous (nover[0], nuni[1])
 * array (the first (nuni[1]+1)/2 and the last nuni[1]/2 of every row side by
 * side); it is overwritten.
 * src/ducc0/nufft/nufft.h:1290 (rows) and :1291-1312 (columns, correction). */
int dnufft_plan_rows_fft(dnufft_plan *plan, int forward, dnufft_array *rows, void *stream);
int dnufft_plan_cols_to_uniform(dnufft_plan *plan, int forward, dnufft_array *grid,
                                dnufft_array *out, void *stream);

/* The column half for one block of the kept columns, so that the column pass
 * is split over the processes too: cols is a C-contiguous device array of
 * (nover[0], ncols) cells, the kept columns col0 .. col0 + ncols - 1 (kept
 * column x is grid column x for x < (nuni[1]+1)/2, else nover[1] - nuni[1] +
 * x) of every row, already transformed along axis 1 (dnufft_plan_rows_fft);
 * it is overwritten.  out: an (nuni[0], ncols) device array that receives the
 * corrected uniform column of each: column x of out is uniform column
 * (col0 + x + s) mod nuni[1], with s = nuni[1]/2 in DUCC's default mode order
 * and s = 0 with fft_order.  Needs nover[0] >= 1024 (DNUFFT_ERR_UNSUPPORTED
 * otherwise).  src/ducc0/nufft/nufft.h:1291-1312 over a range of columns. */
int dnufft_plan_cols_to_uniform_range(dnufft_plan *plan, int forward, dnufft_array *cols,
                                      int64_t col0, dnufft_array *out, void *stream);

/* The type-2 counterparts, for a type 2 split over processes by row slabs
 * (2D): dnufft_plan_uniform_to_cols_range runs the correction, zero padding
 * and column FFTs of one block of kept columns of the uniform array grid
 * (device, (nuni[0], nuni[1])) into cols, an (nover[0], ncols) C-contiguous
 * device array (column x: kept column col0 + x; needs nover[0] >= 1024);
 * dnufft_plan_rows_fft_kept_in transforms rows (C-contiguous device (r,
 * nover[1])) along axis 1 in place, reading only their kept columns (the
 * first (nuni[1]+1)/2 and the last nuni[1]/2) and writing whole rows;
 * dnufft_plan_interp interpolates the plan's points from a C-contiguous
 * device oversampled grid (the rows their footprints reach must be set) into
 * out (device, (M,)).  src/ducc0/nufft/nufft.h:1317-1362 (uni2nonuni) in its
 * three stages. */
int dnufft_plan_uniform_to_cols_range(dnufft_plan *plan, int forward, const dnufft_array *grid,
                                      int64_t col0, dnufft_array *cols, void *stream);
int dnufft_plan_rows_fft_kept_in(dnufft_plan *plan, int forward, dnufft_array *rows,
                                 void *stream);
int dnufft_plan_interp(dnufft_plan *plan, const dnufft_array *grid, dnufft_array *out,
                       void *stream);

/* Kernel-table row and oversampled sizes (nover[0..2], 1 beyond ndim) that
 * DUCC's parameter choice gives for a transform of npoints points; its cost
 * model depends on npoints and opts->nthreads, so processes sharing one
 * transform pass the global count and plan with force_kernel / force_nover.
 * opts: plan defaults when NULL.  Replaces findNufftParameters
 * (src/ducc0/nufft/nufft.h:155-216). */
int dnufft_find_parameters(int nu2u, int ndim, const int64_t *grid_shape, uint64_t npoints,
                           double epsilon, int calc_f64, int coord_f64, const dnufft_opts *opts,
                           int32_t *kernel_index, int64_t *nover);

/* Replaces plan destruction (Julia nufft_delete_plan, julia/ducc_julia.cc:372-392). */
int dnufft_plan_destroy(dnufft_plan *plan);

/* Sizes and kernel parameters of a plan (DUCC prints these under verbosity,
 * src/ducc0/nufft/nufft.h:371-380). */
int dnufft_plan_get_info(const dnufft_plan *plan, dnufft_plan_info *info);

/* Tile-order permutation of the points (DUCC's coord_idx, nufft.h:266,
 * produced by build_index + bucket_sort2) copied to a device or host buffer
 * of npoints uint32. */
int dnufft_plan_get_permutation(const dnufft_plan *plan, uint32_t *out, void *stream);

/* Type 1 like dnufft_nu2u, for callers that cannot allocate device memory
 * while they run it: plugins inside a framework that owns the whole device
 * memory pool, and services with a fixed memory budget.  It has no counterpart
 * in the reference (DUCC allocates its temporaries on the host heap).  Every
 * temporary comes from one area of dnufft_noalloc_scratch_bytes() bytes
 * (32 MiB) compiled into the library and held by every GPU that loads it until
 * the process exits; problems that need more are rejected with
 * DNUFFT_ERR_BADARG before any launch.  All arrays must be device arrays.
 * The first call on a device looks up the area's address and keeps it for the
 * life of the process, so make that first call before any stream capture, and
 * do not call this entry point on a device after resetting it.  The call waits
 * on its stream once, part-way through, to read the number of point chunks
 * back to the host.  All calls share the one area and it keeps the previous
 * call's contents: calls that can overlap on the GPU (other streams, other
 * host threads) race, so serialise them.  Plain spreader only; 2D rows run in
 * the line FFT kernel. */
int dnufft_nu2u_noalloc(const dnufft_array *points, const dnufft_array *coord, int forward,
                        double epsilon, dnufft_array *out, const dnufft_opts *opts,
                        void *stream);
size_t dnufft_noalloc_scratch_bytes(void);

/* Batched transforms (no counterpart in DUCC): 2D plans of one precision,
 * each with its own grid size, points, epsilon (kernel) and ntrans[i]
 * transforms over its coordinates, executed together - one multi-instance
 * launch per stage (grid zeroing, spreading or interpolation, the two FFT line
 * passes with the correction), captured into a CUDA graph on the first call of
 * each direction and sign and replayed afterwards.  The plans must outlive the
 * batch.  Per call, points[i] is (ntrans[i], M_i) (or (M_i,) when ntrans[i] is
 * 1) and the uniform array (ntrans[i], N0, N1) (or (N0, N1)); device arrays
 * only, any strides.  Calls on one batch are serialised (each waits until the
 * previous one has consumed its argument table). */
typedef struct dnufft_batch dnufft_batch;
int dnufft_batch_create(int nplans, dnufft_plan *const *plans, const int32_t *ntrans, void *stream,
                        dnufft_batch **batch);
int dnufft_batch_nu2u(dnufft_batch *batch, int forward, const dnufft_array *points,
                      dnufft_array *out, void *stream);
int dnufft_batch_u2nu(dnufft_batch *batch, int forward, const dnufft_array *grids,
                      dnufft_array *out, void *stream);
int dnufft_batch_destroy(dnufft_batch *batch);

/* Candidate (kernel, oversampled size) pairs for an autotuner: for every
 * kernel support W, the smallest oversampling factor in [sigma_min, sigma_max]
 * whose kernel reaches epsilon (DUCC's getAvailableKernels,
 * src/ducc0/math/gridding_kernel.h:420-444) and the oversampled sizes DUCC's
 * findNufftParameters would use with it (nufft.h:177-178).  Writes up to max
 * entries (nover: 3 per entry) and their number to *count.  Feed the choice
 * back through dnufft_opts.force_kernel / force_nover. */
int dnufft_kernel_candidates(int ndim, const int64_t *shape, int singleprec, double epsilon,
                             double sigma_min, double sigma_max, int max, int32_t *kernel_index,
                             int32_t *supp, double *ofactor, int64_t *nover, int *count);

/* ------------------------------------------------------------ w-gridder
 * Radio-interferometric gridding with w-stacking on top of the 2D transforms,
 * the counterpart of ducc0.wgridder (python/wgridder_pymod.cc:612-656:
 * vis2dirty / dirty2vis, and ms2dirty / dirty2ms, which are these with the
 * default options).  Definitions (src/ducc0/wgridder/wgridder.h): for pixel
 * (i, j), x = center_x + (i - nx/2) pixsize_x, y = center_y + (j - ny/2)
 * pixsize_y, n = sqrt(1 - x^2 - y^2), and visibility k at (u, v, w) = uvw *
 * freq / c (flipped per axis on request):
 *   vis2dirty: dirty(i,j) = sum_k Re(vis_k wgt_k e^{2 pi i (x u + y v - w (n-1))}) / n
 *   dirty2vis: vis_k = wgt_k sum_ij dirty(i,j) / n e^{-2 pi i (x u + y v - w (n-1))}
 * (the w term and the division by n with do_wgridding only; division by n on
 * request), to the requested epsilon.  A visibility takes part where
 * |vis|^2 * wgt * mask != 0 (vis2dirty) or wgt * mask != 0 (dirty2vis; the
 * others are set to zero).  Every array is a device array: uvw (nrows, 3) f64,
 * freq (nchan) f64, vis (nrows, nchan) c64/c128, wgt (nrows, nchan) real of
 * the same precision or NULL, mask (nrows, nchan) DNUFFT_U8 or NULL, dirty
 * (nx, ny) real (nx, ny even).  Error behaviour as in the rest of this header
 * (DUCC raises the same conditions as exceptions). */
typedef struct dnufft_wgrid_opts {
  size_t nthreads;        /* as in DUCC; only feeds its parameter cost model      */
  double sigma_min;       /* oversampling factor range (DUCC: 1.1 .. 2.6)        */
  double sigma_max;
  double center_x;        /* image centre relative to the phase centre           */
  double center_y;
  int32_t do_wgridding;   /* 1: w-stacking with the w term; 0: w taken as zero   */
  int32_t flip_u, flip_v, flip_w;
  int32_t divide_by_n;    /* DUCC's default 1                                    */
  int32_t allow_nshift;   /* DUCC's default 1: centre the w-screen phases        */
  int32_t double_precision_accumulation;   /* single-precision data, double grids */
  int32_t verbosity;      /* 1: print the chosen parameters                      */
  /* Only w planes [plane_begin, plane_begin + plane_count) of the call's
   * planes (plane_count 0: all), for a split over processes: the results of
   * calls over a partition of the planes sum to the whole result (without
   * w-stacking the one plane is plane 0).  No DUCC counterpart. */
  int32_t plane_begin;
  int32_t plane_count;
} dnufft_wgrid_opts;

/* DUCC's keyword defaults of vis2dirty / dirty2vis. */
void dnufft_wgrid_default_opts(dnufft_wgrid_opts *opts);

int dnufft_vis2dirty(const dnufft_array *uvw, const dnufft_array *freq, const dnufft_array *vis,
                     const dnufft_array *wgt, const dnufft_array *mask, double pixsize_x,
                     double pixsize_y, double epsilon, const dnufft_wgrid_opts *opts,
                     dnufft_array *dirty, void *stream);
int dnufft_dirty2vis(const dnufft_array *uvw, const dnufft_array *freq, const dnufft_array *dirty,
                     const dnufft_array *wgt, const dnufft_array *mask, double pixsize_x,
                     double pixsize_y, double epsilon, const dnufft_wgrid_opts *opts,
                     dnufft_array *vis, void *stream);

/* The parameters the two calls above choose for these inputs (DUCC's
 * getNuNv / countRanges, wgridder.h:1499-1579, :675-692): kernel table row,
 * support, oversampled grid, w planes (count, spacing, first plane's w), the
 * w-screen shift and the number of visibilities taking part.  gridding: 1 for
 * vis2dirty (vis is read), 0 for dirty2vis (vis may be NULL). */
typedef struct dnufft_wgrid_info {
  int32_t kernel_index;
  int32_t supp;
  int64_t nu, nv;
  int64_t nplanes;
  double dw, wmin, nshift;
  int64_t nvis;
} dnufft_wgrid_info;
int dnufft_wgrid_params(const dnufft_array *uvw, const dnufft_array *freq, const dnufft_array *vis,
                        const dnufft_array *wgt, const dnufft_array *mask, int64_t nx, int64_t ny,
                        double pixsize_x, double pixsize_y, double epsilon, int gridding,
                        const dnufft_wgrid_opts *opts, dnufft_wgrid_info *info, void *stream);

/* Message of the last failed call on this thread ("" if none). */
const char *dnufft_last_error(void);

/* Number of CUDA kernels this library has launched in this process (a
 * diagnostic without a counterpart in DUCC, which has no GPU path). */
uint64_t dnufft_kernel_launches(void);

/* Stage profiler (no counterpart in DUCC, whose verbosity report prints CPU
 * stage times): while enabled, every transform records CUDA events between its
 * stages and accumulates the elapsed time per stage.  Enabling clears the
 * totals.  dnufft_profile_json() returns {"<transform>/<stage>": [ms, calls]}. */
/* Test hook for the failure path of the bounded device-side waits: runs the
   tensor-core spreader's wait routine, with the given limit, on a barrier that
   nothing arrives at.  Returns DNUFFT_ERR_TIMEOUT (the context stays usable).
   No DUCC counterpart. */
int dnufft_selftest_wait_timeout(int64_t limit_ns, void *stream);

void dnufft_profile_enable(int enable);
const char *dnufft_profile_json(void);

#ifdef __cplusplus
}
#endif

#endif /* DUCC_B200_H */
