// Host-side NUFFT planner: kernel shape choice, oversampled grid sizes, the
// piecewise-polynomial kernel fit and the deconvolution (correction) factors.
//
// Behaviour follows DUCC so that, for the same arguments, the same kernel row,
// support W and oversampled size n are chosen (which makes the tile keys and
// the point permutation bit-identical to DUCC's):
//   good_size_complex   src/ducc0/fft/fft.h:93-118   (smallest 11-smooth >= n)
//   available_kernels   src/ducc0/math/gridding_kernel.h:420-444
//   best_epsilon        src/ducc0/math/gridding_kernel.cc:1562-1576
//   find_parameters     src/ducc0/nufft/nufft.h:155-208 (cost model constants)
//   kernel_coeffs       src/ducc0/math/gridding_kernel.cc:28-76 (Chebyshev fit,
//                       degree W+3, converted to monomials per sub-interval)
//   correction_factors  src/ducc0/math/gridding_kernel.h:77-129 (Gauss-Legendre
//                       quadrature of the kernel's Fourier transform)
#include "dnufft_internal.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <thread>
#include <sched.h>
#include <atomic>

namespace dnufft {

static const std::vector<KernelShape> kDB = {
#include "kernel_db.inc"
};

const std::vector<KernelShape> &kernel_db() { return kDB; }

static bool smooth11(size_t m) {
  for (size_t p : {2u, 3u, 5u, 7u, 11u})
    while (m % p == 0) m /= p;
  return m == 1;
}

size_t good_size_complex(size_t n) {
  if (n <= 12) return n;
  // enumerate 11-smooth numbers: for every 3,5,7,11 part, scale by powers of 2
  size_t best = 2 * n;
  for (size_t a = 1; a < best; a *= 11)
    for (size_t b = a; b < best; b *= 7)
      for (size_t c = b; c < best; c *= 5)
        for (size_t d = c; d < best; d *= 3) {
          size_t x = d;
          while (x < n) x *= 2;
          if (x < best) best = x;
        }
  return best;
}

std::vector<size_t> available_kernels(double epsilon, size_t ndim, bool singleprec,
                                      double ofactor_min, double ofactor_max) {
  std::vector<double> ofc(20, ofactor_max);
  std::vector<size_t> idx(20, kDB.size());
  size_t wlim = singleprec ? 8 : 16;
  for (size_t i = 0; i < kDB.size(); ++i) {
    const auto &k = kDB[i];
    size_t W = size_t(k.W);
    if (size_t(k.ndim) == ndim && k.singleprec == singleprec && W <= wlim &&
        k.epsilon <= epsilon && k.ofactor <= ofc[W] && k.ofactor >= ofactor_min) {
      ofc[W] = k.ofactor;
      idx[W] = i;
    }
  }
  std::vector<size_t> res;
  for (auto v : idx)
    if (v < kDB.size()) res.push_back(v);
  DN_REQUIRE(!res.empty(), ST_EPSILON, "no appropriate kernel found");
  return res;
}

double best_epsilon(size_t ndim, bool singleprec, double ofactor_min, double ofactor_max) {
  DN_REQUIRE(ndim >= 1 && ndim <= 3, ST_BADARG, "bad dimensionality");
  double res = 1000.;
  for (const auto &k : kDB)
    if (size_t(k.ndim) == ndim && k.singleprec == singleprec && k.epsilon <= res &&
        k.ofactor <= ofactor_max && k.ofactor >= ofactor_min)
      res = k.epsilon;
  DN_REQUIRE(res < 1000., ST_EPSILON, "no appropriate kernel found");
  return res;
}

// Threads the CPU cost model assumes: 0 means all hardware threads (honouring
// DUCC0_NUM_THREADS / OMP_NUM_THREADS); larger requests are capped there.
size_t effective_threads(size_t nthreads) {
  static const size_t hw = []() {
    size_t res = 0;
    cpu_set_t set;
    if (sched_getaffinity(0, sizeof(set), &set) == 0) res = size_t(CPU_COUNT(&set));
    if (res == 0) res = std::max<size_t>(1, std::thread::hardware_concurrency());
    const char *ev = std::getenv("DUCC0_NUM_THREADS");
    if (!ev) ev = std::getenv("OMP_NUM_THREADS");
    if (ev) {
      long v = std::strtol(ev, nullptr, 10);
      if (v > 0) res = std::min<size_t>(res, size_t(v));
    }
    return res;
  }();
  if (nthreads == 0) return hw;
  return std::min(hw, nthreads);
}

size_t find_parameters(double epsilon, double sigma_min, double sigma_max,
                       const std::vector<size_t> &dims, size_t npoints, bool gridding,
                       size_t nthreads, bool singleprec, size_t vlen,
                       std::vector<size_t> &nover) {
  (void)gridding;  // DUCC scales by sizeof(Tacc)/sizeof(Tcalc), which is 1 here
  size_t ndim = dims.size();
  auto idx = available_kernels(epsilon, ndim, singleprec, sigma_min, sigma_max);
  const double nref_fft = 2048, costref_fft = 0.0693;
  double mincost = 1e300;
  size_t minidx = kDB.size();
  double nt = double(nthreads);
  for (size_t i : idx) {
    size_t W = size_t(kDB[i].W);
    double of = kDB[i].ofactor;
    size_t nvec = (W + vlen - 1) / vlen;
    std::vector<size_t> big(ndim);
    double gridsize = 1;
    for (size_t d = 0; d < ndim; ++d) {
      big[d] = std::max<size_t>(2 * good_size_complex(size_t(dims[d] * of * 0.5) + 1), 16);
      gridsize *= double(big[d]);
    }
    double logterm = std::log(gridsize) / std::log(nref_fft * nref_fft);
    double fftcost = gridsize / (nref_fft * nref_fft) * logterm * costref_fft;
    size_t kernelpoints = nvec * vlen;
    for (size_t d = 0; d + 1 < ndim; ++d) kernelpoints *= W;
    double gridcost =
        2.2e-10 * double(npoints) * double(kernelpoints + ndim * nvec * (W + 3) * vlen);
    gridcost /= nt;
    double x2 = nt - 1, m2 = 6. - 1;
    double sig = 1. + x2 / std::pow(1. + std::pow(x2 / m2, 2.), 1. / 2.);
    fftcost /= sig;
    double cost = fftcost + gridcost;
    if (cost < mincost) {
      mincost = cost;
      nover = big;
      minidx = i;
    }
  }
  return minidx;
}

static double es_kernel(double v, double beta, double e0) {
  double t = (1 - v) * (1 + v);
  if (t < 0) return 0.;
  return std::exp(beta * (std::pow(t, e0) - 1));
}

std::vector<double> kernel_coeffs(int W, double beta, double e0) {
  const int D = W + 3;
  std::vector<double> coeff(size_t(W) * (D + 1));
  std::vector<double> node(D + 1), y(D + 1), cheb(D + 1), mono(D + 1);
  for (int i = 0; i <= D; ++i) node[i] = std::cos((2 * i + 1.) * M_PI / (2 * D + 2));
  // T_j(x) = sum_k C[j][k] x^k
  std::vector<double> C(size_t(D + 1) * (D + 1), 0.);
  C[0] = 1.;
  if (D >= 1) C[(D + 1) + 1] = 1.;
  for (int j = 2; j <= D; ++j) {
    C[size_t(j) * (D + 1)] = -C[size_t(j - 2) * (D + 1)];
    for (int k = 1; k <= j; ++k)
      C[size_t(j) * (D + 1) + k] =
          2 * C[size_t(j - 1) * (D + 1) + k - 1] - C[size_t(j - 2) * (D + 1) + k];
  }
  for (int i = 0; i < W; ++i) {
    double l = -1 + 2. * i / W, r = -1 + 2. * (i + 1) / W;
    double avg = 0;
    for (int j = 0; j <= D; ++j) {
      y[j] = es_kernel(node[j] * (r - l) * 0.5 + (r + l) * 0.5, beta, e0);
      avg += y[j];
    }
    avg /= (D + 1);
    for (int j = 0; j <= D; ++j) y[j] -= avg;
    for (int j = 0; j <= D; ++j) {
      double s = 0;
      for (int k = 0; k <= D; ++k) s += y[k] * std::cos(j * (2 * k + 1) * M_PI / (2 * D + 2));
      cheb[j] = 2. / (D + 1) * s;
    }
    cheb[0] *= 0.5;
    std::fill(mono.begin(), mono.end(), 0.);
    for (int j = 0; j <= D; ++j)
      for (int k = 0; k <= D; ++k) mono[k] += C[size_t(j) * (D + 1) + k] * cheb[j];
    mono[0] += avg;
    for (int j = 0; j <= D; ++j) coeff[size_t(j) * W + i] = mono[D - j];
  }
  return coeff;
}

// Gauss-Legendre nodes (x>=0) and weights on [-1,1] by Newton iteration on P_m.
static void gauss_legendre_half(int m, std::vector<double> &x, std::vector<double> &w) {
  x.clear();
  w.clear();
  for (int i = 1; i <= m / 2 + (m & 1); ++i) {
    double z = std::cos(M_PI * (i - 0.25) / (m + 0.5));
    double dp = 0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1, p1 = z;
      for (int k = 2; k <= m; ++k) {
        double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      dp = m * (z * p1 - p0) / (z * z - 1);
      double dz = p1 / dp;
      z -= dz;
      if (std::abs(dz) < 1e-16) {
        // one more evaluation at the converged node for the weight
        p0 = 1; p1 = z;
        for (int k = 2; k <= m; ++k) {
          double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
          p0 = p1;
          p1 = p2;
        }
        dp = m * (z * p1 - p0) / (z * z - 1);
        break;
      }
    }
    x.push_back(z);
    w.push_back(2. / ((1 - z * z) * dp * dp));
  }
}

void correction_nodes(int W, double beta, double e0, std::vector<double> &x,
                      std::vector<double> &wpsi) {
  int p = int(1.5 * W) + 2;
  std::vector<double> w;
  gauss_legendre_half(2 * p, x, w);   // 2p nodes: p positive ones
  wpsi.resize(x.size());
  for (size_t i = 0; i < x.size(); ++i) wpsi[i] = 2 * w[i] * es_kernel(x[i], beta, e0) * W * 0.5;
}

std::vector<double> correction_factors(size_t n, double dx, int W, double beta, double e0) {
  std::vector<double> x, wpsi;
  correction_nodes(W, beta, e0, x, wpsi);
  std::vector<double> res(n);
  for (size_t i = 0; i < n; ++i) {
    double v = double(i) * dx, s = 0;
    for (size_t k = 0; k < x.size(); ++k) s += wpsi[k] * std::cos((M_PI * W * x[k]) * v);
    res[i] = 1. / s;
  }
  return res;
}

// radix sequence for the Stockham FFT: 8s first, then 4, 2, 3, 5, 7, 11, others
std::vector<int> fft_factors(int n) {
  std::vector<int> f;
  int m = n;
  while (m % 8 == 0) { f.push_back(8); m /= 8; }
  while (m % 4 == 0) { f.push_back(4); m /= 4; }
  while (m % 2 == 0) { f.push_back(2); m /= 2; }
  for (int p : {3, 5, 7, 11})
    while (m % p == 0) { f.push_back(p); m /= p; }
  for (int p = 13; p * p <= m; p += 2)
    while (m % p == 0) { f.push_back(p); m /= p; }
  if (m > 1) f.push_back(m);
  if (f.empty()) f.push_back(1);
  return f;
}

static std::atomic<uint64_t> g_launches{0};
void note_launch(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
uint64_t launch_count() { return g_launches.load(std::memory_order_relaxed); }

void cuda_check(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return;
  int code = (e == cudaErrorMemoryAllocation) ? ST_OOM : ST_CUDA;
  throw Error(code, std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}

}  // namespace dnufft
