// Internal declarations shared by the host planner, the C-ABI layer and the
// CUDA kernels of the B200 NUFFT library.  Nothing here is part of the public
// interface (that is include/ducc_b200.h).
#pragma once

#include <cstdint>
#include <cstddef>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

struct dnufft_opts;   // include/ducc_b200.h

namespace dnufft {

// ---------------------------------------------------------------- errors
enum Status : int {
  ST_OK = 0,
  ST_BADARG = 1,
  ST_EPSILON = 2,
  ST_OOM = 3,
  ST_CUDA = 4,
  ST_TIMEOUT = 5,
  ST_UNSUPPORTED = 6,
  ST_INTERNAL = 7,
};

struct Error : public std::runtime_error {
  int code;
  Error(int c, const std::string &msg) : std::runtime_error(msg), code(c) {}
};

#define DN_REQUIRE(cond, code, msg) \
  do { if (!(cond)) throw ::dnufft::Error((code), (msg)); } while (0)

void cuda_check(cudaError_t e, const char *what);
// the message dnufft_last_error() returns on this host thread
void set_last_error(const char *msg);
#define DN_CUDA(call) ::dnufft::cuda_check((call), #call)

// number of kernels this library launched (diagnostics)
void note_launch(uint64_t n = 1);
uint64_t launch_count();
// check a launch and count it
#define DN_LAUNCHED() do { ::dnufft::cuda_check(cudaGetLastError(), "kernel launch"); ::dnufft::note_launch(); } while (0)

// Starts a named sub-stage of the transform running on this host thread (one
// NVTX range, and one CUDA event in the stage profile when that is on); used
// between the launches of a multi-kernel stage such as the 2D FFT so that
// each kernel gets its own time.  No effect outside a transform.
void stage_mark(const char *name);

// ---------------------------------------------------------------- planner
struct KernelShape {
  int W;
  double ofactor, epsilon, beta, e0;
  int ndim;
  bool singleprec;
};
const std::vector<KernelShape> &kernel_db();

size_t good_size_complex(size_t n);
std::vector<size_t> available_kernels(double epsilon, size_t ndim, bool singleprec,
                                      double ofactor_min, double ofactor_max);
double best_epsilon(size_t ndim, bool singleprec, double ofactor_min, double ofactor_max);
// returns kernel row, fills nover
size_t find_parameters(double epsilon, double sigma_min, double sigma_max,
                       const std::vector<size_t> &dims, size_t npoints, bool gridding,
                       size_t nthreads, bool singleprec, size_t vlen,
                       std::vector<size_t> &nover);
size_t effective_threads(size_t nthreads);
std::vector<double> kernel_coeffs(int W, double beta_scaled, double e0);
std::vector<double> correction_factors(size_t n, double dx, int W, double beta_scaled,
                                       double e0);
// the quadrature of the correction function 1 / sum_k wpsi[k] cos(pi W x[k] v)
// (positive Gauss-Legendre nodes x, weights times the kernel, doubled)
void correction_nodes(int W, double beta_scaled, double e0, std::vector<double> &x,
                      std::vector<double> &wpsi);
std::vector<int> fft_factors(int n);

// ---------------------------------------------------------------- device params
constexpr int MAXW = 16;
constexpr int MAXD = MAXW + 4;   // D'+1 coefficient rows, D' = W+3+(W&1)
constexpr int MAXH = (MAXW + 1) / 2;

// piecewise-polynomial kernel: c[j][k], j = 0 (highest power) .. D', k < ceil(W/2)
template <typename T> struct KernelPoly {
  T c[MAXD][MAXH];
};

// geometry of the oversampled grid and the folding constants
struct Geometry {
  int ndim;
  int W, nsafe, log2tile;
  int64_t nuni[3];
  int64_t nover[3];
  double coordfct[3];
  double shift[3];
  int maxi0[3];
  int64_t ntiles[3];   // (nover>>log2tile)+3
  // 3D sub-tile key parameters
  int lsq2, ssmall;
};

// one tile-chunk of sorted points: points [start, start+count) share a tile
struct Chunk {
  uint32_t start;
  uint32_t count;
  uint32_t tile;   // tile id (2D: tu*ntv+tv; 3D: hikey; 1D: tu)
  uint32_t pad;
};

// A 2D index over points in groups, sorted once by (tile, group) (capi.cpp);
// the w-gridder's w planes are runs of groups [g0, g1), each transformed
// without a sort.  create returns null where the (tile, group) table would be
// too large.  perm_out (device, M words): sorted position -> the caller's
// point index.  Values and results are in the caller's order; the uniform
// arrays are contiguous (nuni[0], nuni[1]); the transforms return false
// (writing nothing) for a run without points.
struct GroupedPlan;
GroupedPlan *grouped_plan_create(const double *coord, uint32_t M, const uint32_t *group,
                                 uint32_t ngroups, const int64_t *shape, double eps,
                                 bool calc_f64, const ::dnufft_opts &opts,
                                 cudaStream_t st, uint32_t *perm_out);
void grouped_plan_destroy(GroupedPlan *gp, cudaStream_t st);
const uint32_t *grouped_plan_perm(const GroupedPlan *gp);
bool grouped_nu2u(GroupedPlan *gp, uint32_t g0, uint32_t g1, const void *values, void *out,
                  bool forward, cudaStream_t st);
bool grouped_u2nu(GroupedPlan *gp, uint32_t g0, uint32_t g1, const void *uni, void *out,
                  bool forward, cudaStream_t st);

}  // namespace dnufft
