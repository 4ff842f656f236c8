// C-ABI of the B200 NUFFT library and the host orchestration behind it.
//
// Mirrors DUCC's control flow for one transform (src/ducc0/nufft/nufft.h):
//   parameter choice + kernel fit + correction factors   (Nufft_ancestor ctor, :392-433)
//   build_index: fold, tile keys, stable sort            (:1364-1381 and friends)
//   type 1: zero grid, spread, pruned FFT, correct+crop  (nonuni2uni, :1274-1315)
//   type 2: correct+pad, pruned FFT, interpolate         (uni2nonuni, :1317-1362)
// and its argument checks (nufft.h:335-361, :400-424, python/nufft_pymod.cc).
// Errors become a status code plus dnufft_last_error() (the convention of DUCC's
// C interface, julia/ducc_julia.cc:58-59); argument errors never launch kernels.
#include "../../include/ducc_b200.h"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "dnufft_internal.h"
#include "kernels.h"

static thread_local std::string g_last_error;

#include <map>
#include <mutex>
namespace {
// per-stage CUDA-event times accumulated while profiling is enabled
std::mutex g_prof_mu;
bool g_prof_on = false;
std::map<std::string, std::pair<double, long>> g_prof;   // name -> (ms, calls)
std::string g_prof_json;
}  // namespace

namespace dnufft {

constexpr uint32_t CHUNK = 1024;       // points per chunk (one CTA)
constexpr uint32_t CHUNK_TC = 4096;    // tensor-core plans: fewer, longer chunks
constexpr double TC_AUTO_DENSITY = 0.5;   // points per uniform mode from which 'auto' picks TC

// ---------------------------------------------------------------- device buffers
// Keep memory freed with cudaFreeAsync in the device's default pool instead of
// returning it to the driver at every synchronisation, so repeated transforms
// do not pay for mapping fresh pages.
static void keep_pool_memory() {
  static thread_local int done_for = -1;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev == done_for) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t thr = ~uint64_t(0);
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  done_for = dev;
}

struct DevBuf {
  void *p = nullptr;
  cudaStream_t st = nullptr;
  DevBuf() = default;
  DevBuf(size_t bytes, cudaStream_t s) : st(s) {
    keep_pool_memory();
    if (bytes) DN_CUDA(cudaMallocAsync(&p, bytes, s));
  }
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  DevBuf(DevBuf &&o) noexcept : p(o.p), st(o.st) { o.p = nullptr; }
  DevBuf &operator=(DevBuf &&o) noexcept {
    release();
    p = o.p;
    st = o.st;
    o.p = nullptr;
    return *this;
  }
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
  }
  template <typename X> X *as() const { return static_cast<X *>(p); }
};

// ---------------------------------------------------------------- device error word
// Kernels with bounded waits set this word instead of hanging; it is read back
// after such a kernel (outside stream capture) and turned into ST_TIMEOUT.
static int *device_error_word() {
  static thread_local int dev_cached = -1;
  static int *words[64] = {nullptr};
  int dev = 0;
  DN_CUDA(cudaGetDevice(&dev));
  DN_REQUIRE(dev >= 0 && dev < 64, ST_INTERNAL, "device index out of range");
  if (!words[dev]) {
    // word 0: error flag; word 1: scratch for the operand-scale reduction
    DN_CUDA(cudaMalloc(&words[dev], 4 * sizeof(int)));
    DN_CUDA(cudaMemset(words[dev], 0, 4 * sizeof(int)));
  }
  dev_cached = dev;
  return words[dev];
}

static void check_device_error(int *word, cudaStream_t st) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  DN_CUDA(cudaStreamIsCapturing(st, &cs));
  if (cs != cudaStreamCaptureStatusNone) return;
  uint32_t h = 0;
  const uint32_t *src[1] = {reinterpret_cast<const uint32_t *>(word)};
  read_words(src, 1, &h, st);
  if (h != 0) {
    DN_CUDA(cudaMemsetAsync(word, 0, sizeof(int), st));
    throw Error(ST_TIMEOUT, "a bounded device-side wait gave up (tensor-core spreader or FFT)");
  }
}

// ---------------------------------------------------------------- stage timers
// CUDA-event stage profile printed under verbosity>0 (the counterpart of DUCC's
// TimerHierarchy report, src/ducc0/infra/timers.h:69-266), with one NVTX range
// per stage.
struct StageTimer {
  bool on;
  bool print;
  cudaStream_t st;
  std::vector<std::pair<std::string, cudaEvent_t>> marks;
  bool range_open = false;   // an NVTX range named after the current stage
  StageTimer *outer;         // the timer this one hides (nested transforms)
  StageTimer(bool on_, cudaStream_t s) : on(on_ || g_prof_on), print(on_), st(s) {
    outer = current();
    current() = this;
  }
  // the innermost timer alive on this host thread (target of stage_mark)
  static StageTimer *&current() {
    static thread_local StageTimer *cur = nullptr;
    return cur;
  }
  // Starts stage `name`: closes the previous stage's NVTX range and opens one
  // for this stage (host-side ranges around the launches of each stage, for
  // a timeline tool; without one attached they cost a function call), and
  // records a CUDA event when timing is on.
  void mark(const char *name) {
    if (range_open) nvtxRangePop();
    nvtxRangePushA(name);
    range_open = true;
    if (!on) return;
    cudaEvent_t e;
    DN_CUDA(cudaEventCreate(&e));
    DN_CUDA(cudaEventRecord(e, st));
    marks.emplace_back(name, e);
  }
  void report(const char *title) {
    if (!on || marks.size() < 2) return;
    DN_CUDA(cudaEventSynchronize(marks.back().second));
    float total = 0;
    DN_CUDA(cudaEventElapsedTime(&total, marks.front().second, marks.back().second));
    if (print) std::printf("%s (GPU, CUDA events): %.4f ms total\n", title, total);
    for (size_t i = 0; i + 1 < marks.size(); ++i) {
      float ms = 0;
      DN_CUDA(cudaEventElapsedTime(&ms, marks[i].second, marks[i + 1].second));
      if (print)
        std::printf("  %-22s %10.4f ms  %5.1f%%\n", marks[i].first.c_str(), ms,
                    total > 0 ? 100. * ms / total : 0.);
      if (g_prof_on) {
        std::lock_guard<std::mutex> lk(g_prof_mu);
        auto &e = g_prof[std::string(title) + "/" + marks[i].first];
        e.first += ms;
        e.second += 1;
      }
    }
    if (print) std::fflush(stdout);
  }
  ~StageTimer() {
    current() = outer;
    if (range_open) nvtxRangePop();
    for (auto &m : marks) cudaEventDestroy(m.second);
  }
};

void stage_mark(const char *name) {
  if (StageTimer *t = StageTimer::current()) t->mark(name);
}

// ---------------------------------------------------------------- array views
struct View {
  void *data;
  int dtype;
  int ndim;
  int64_t shape[4];
  int64_t stride[4];
  bool host;
};

static size_t dtype_size(int dt) {
  switch (dt) {
    case DNUFFT_F32: return 4;
    case DNUFFT_F64: return 8;
    case DNUFFT_C64: return 8;
    case DNUFFT_C128: return 16;
  }
  return 0;
}

static bool is_host_pointer(const void *p) {
  cudaPointerAttributes at;
  cudaError_t e = cudaPointerGetAttributes(&at, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return true;
  }
  return at.type == cudaMemoryTypeUnregistered || at.type == cudaMemoryTypeHost;
}

static View view_of(const dnufft_array *a, const char *what) {
  DN_REQUIRE(a != nullptr, ST_BADARG, std::string(what) + ": null array");
  View v;
  v.data = a->data;
  v.dtype = a->dtype;
  v.ndim = a->ndim;
  DN_REQUIRE(v.ndim >= 1 && v.ndim <= 4, ST_BADARG, std::string(what) + ": bad ndim");
  DN_REQUIRE(dtype_size(v.dtype) != 0, ST_BADARG, std::string(what) + ": bad dtype");
  int64_t size = 1;
  for (int d = 0; d < v.ndim; ++d) {
    v.shape[d] = a->shape[d];
    v.stride[d] = a->stride[d];
    DN_REQUIRE(v.shape[d] >= 0, ST_BADARG, std::string(what) + ": negative extent");
    size *= v.shape[d];
  }
  DN_REQUIRE(size == 0 || v.data != nullptr, ST_BADARG, std::string(what) + ": null data");
  if (size > 0)
    for (int d = 0; d < v.ndim; ++d)
      DN_REQUIRE(v.shape[d] <= 1 || v.stride[d] != 0, ST_BADARG,
                 std::string(what) + ": zero stride");
  v.host = (size > 0) ? is_host_pointer(v.data) : false;
  if (v.host) {
    int64_t s = 1;
    for (int d = v.ndim - 1; d >= 0; --d) {
      DN_REQUIRE(v.shape[d] <= 1 || v.stride[d] == s, ST_BADARG,
                 std::string(what) + ": host arrays must be C-contiguous");
      s *= v.shape[d];
    }
  }
  return v;
}

static int64_t nelem(const View &v) {
  int64_t s = 1;
  for (int d = 0; d < v.ndim; ++d) s *= v.shape[d];
  return s;
}

// A second stream of an unplanned call on host arrays: host->device copies
// (and work that needs only them) run there while the caller's stream builds
// the index, forked from and joined back into the caller's stream by events.
// Created only for calls with host arrays (device-array calls, e.g. recorded
// into a stream capture, keep to the caller's stream); inactive otherwise.
struct SideStream {
  cudaStream_t main, s = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  SideStream(cudaStream_t m, bool use) : main(m) {
    if (!use) return;
    DN_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    DN_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    DN_CUDA(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
  }
  bool active() const { return s != nullptr; }
  // the side stream continues after everything queued on the main stream so far
  void start() {
    if (!s) return;
    DN_CUDA(cudaEventRecord(fork, main));
    DN_CUDA(cudaStreamWaitEvent(s, fork, 0));
  }
  // the main stream continues after everything queued on the side stream so far
  void merge() {
    if (!s) return;
    DN_CUDA(cudaEventRecord(join, s));
    DN_CUDA(cudaStreamWaitEvent(main, join, 0));
  }
  ~SideStream() {
    if (s) {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
    if (fork) cudaEventDestroy(fork);
    if (join) cudaEventDestroy(join);
  }
};

// Device-side copy of a host array (inputs copied in, outputs copied back).
// The buffer is allocated on the caller's stream; with a side stream, the
// input copy runs there (after the caller's stream's work so far).
struct Staged {
  View dev;
  DevBuf buf;
  const View *orig = nullptr;
  bool is_output = false;
  cudaStream_t st;
  cudaStream_t side = nullptr;
  Staged(const View &v, bool input, bool output, cudaStream_t s, SideStream *ss = nullptr)
      : st(s) {
    dev = v;
    orig = &v;
    is_output = output && v.host;
    if (!v.host) return;
    size_t bytes = size_t(nelem(v)) * dtype_size(v.dtype);
    buf = DevBuf(bytes, s);
    dev.data = buf.p;
    dev.host = false;
    if (!input || !bytes) return;
    if (ss && ss->active()) {
      ss->start();
      side = ss->s;
      DN_CUDA(cudaMemcpyAsync(buf.p, v.data, bytes, cudaMemcpyHostToDevice, side));
    } else {
      DN_CUDA(cudaMemcpyAsync(buf.p, v.data, bytes, cudaMemcpyHostToDevice, s));
    }
  }
  ~Staged() {
    // an exception may leave a side-stream copy in flight: finish it before
    // the buffer returns to the caller's stream's pool
    if (side) cudaStreamSynchronize(side);
  }
  void finish() {
    if (!is_output) return;
    size_t bytes = size_t(nelem(*orig)) * dtype_size(orig->dtype);
    if (bytes) DN_CUDA(cudaMemcpyAsync(orig->data, buf.p, bytes, cudaMemcpyDeviceToHost, st));
    DN_CUDA(cudaStreamSynchronize(st));
  }
};

// ---------------------------------------------------------------- setup
struct Setup {
  Geometry g;
  bool calc_f64 = false, coord_f64 = false;
  uint32_t npoints = 0;
  int kidx = 0;
  double ofactor = 0, beta = 0, e0 = 0, epsilon = 0;
  KernelPoly<float> kpf;
  KernelPoly<double> kpd;
  std::vector<double> corfac[3];
  std::vector<int> factors[3];
  int spreader = DNUFFT_SPREAD_AUTO;
  bool qbits = false;   // sort key carries the 2D tile quadrant and cell (tensor-core order)
  int keybits = 1;
  int tile_shift = 0;
  uint64_t max_tiles = 0;
  uint32_t chunk = CHUNK;   // largest chunk (consecutive sorted points of one tile)
};

static void fill_poly(Setup &s, const std::vector<double> &coeff) {
  const int W = s.g.W;
  const int D = W + 3;
  const int Dp = W + 3 + (W & 1);
  const int ofs = Dp - D;
  const int H = (W + 1) / 2;
  std::memset(&s.kpf, 0, sizeof(s.kpf));
  std::memset(&s.kpd, 0, sizeof(s.kpd));
  for (int j = 0; j <= D; ++j)
    for (int k = 0; k < H; ++k) {
      double c = coeff[size_t(j) * W + k];
      s.kpd.c[j + ofs][k] = c;
      s.kpf.c[j + ofs][k] = float(c);
    }
}

static int bitlen64(uint64_t v) {
  int b = 0;
  while (v) {
    ++b;
    v >>= 1;
  }
  return b;
}

static Setup make_setup(int ndim, const int64_t *nuni, uint64_t npoints, double epsilon,
                        bool gridding, bool calc_f64, bool coord_f64, const dnufft_opts &o) {
  DN_REQUIRE(ndim >= 1 && ndim <= 3, ST_BADARG, "transform must be 1D/2D/3D");
  DN_REQUIRE(npoints <= 0xffffffffull, ST_BADARG, "too many nonuniform points");
  DN_REQUIRE(epsilon > 0, ST_BADARG, "epsilon must be positive");
  Setup s;
  s.calc_f64 = calc_f64;
  s.coord_f64 = coord_f64;
  DN_REQUIRE(o.spreader >= DNUFFT_SPREAD_AUTO && o.spreader <= DNUFFT_SPREAD_TC, ST_BADARG,
             "unknown spreader");
  s.spreader = o.spreader;
  s.npoints = uint32_t(npoints);
  s.epsilon = epsilon;
  Geometry &g = s.g;
  std::memset(&g, 0, sizeof(g));
  g.ndim = ndim;
  std::vector<size_t> dims(ndim), nover;
  for (int d = 0; d < ndim; ++d) {
    DN_REQUIRE(nuni[d] >= 1, ST_BADARG, "uniform grid dimensions must be positive");
    dims[d] = size_t(nuni[d]);
    g.nuni[d] = nuni[d];
  }
  if (o.force_kernel >= 0) {
    DN_REQUIRE(size_t(o.force_kernel) < kernel_db().size(), ST_BADARG, "bad forced kernel");
    s.kidx = o.force_kernel;
    for (int d = 0; d < ndim; ++d) nover.push_back(size_t(o.force_nover[d]));
  } else {
    size_t vlen = calc_f64 ? size_t(o.simd_lanes > 0 ? o.simd_lanes : 8) : 8;
    s.kidx = int(find_parameters(epsilon, o.sigma_min, o.sigma_max, dims, npoints, gridding,
                                 effective_threads(o.nthreads), !calc_f64, vlen, nover));
  }
  const KernelShape &ks = kernel_db()[size_t(s.kidx)];
  DN_REQUIRE(ks.singleprec == !calc_f64 || o.force_kernel >= 0, ST_EPSILON,
             "no appropriate kernel found");
  g.W = ks.W;
  g.nsafe = (g.W + 1) / 2;
  g.log2tile = (ndim == 1) ? 9 : (ndim == 2 ? (calc_f64 ? 4 : 5) : 4);
  if (o.log2tile != 0) {
    DN_REQUIRE(ndim == 1 ? o.log2tile == 9
                         : (ndim == 2 ? (o.log2tile == 4 || o.log2tile == 5) : o.log2tile == 4),
               ST_BADARG, "log2tile must be 9 (1D), 4 or 5 (2D), 4 (3D)");
    g.log2tile = o.log2tile;
  }
  s.ofactor = ks.ofactor;
  s.beta = ks.beta * ks.W;
  s.e0 = ks.e0;
  const uint64_t max_ntile = ndim == 1 ? 0xffffffffull - 10 : (ndim == 2 ? (1u << 16) - 10 : (1u << 10) - 10);
  for (int d = 0; d < ndim; ++d) {
    int64_t n = int64_t(nover[d]);
    DN_REQUIRE(n >= 2 * g.nsafe, ST_BADARG, "oversampled length too small");
    DN_REQUIRE((n & 1) == 0, ST_BADARG, "oversampled dimensions must be even");
    DN_REQUIRE(uint64_t(n >> g.log2tile) <= max_ntile, ST_BADARG, "oversampled grid too large");
    DN_REQUIRE(n < (int64_t(1) << 30), ST_BADARG, "oversampled grid too large");
    g.nover[d] = n;
    g.shift[d] = g.W * (-0.5) + 1 + double(n);
    g.maxi0[d] = int((n + g.nsafe) - g.W);
    g.ntiles[d] = (n >> g.log2tile) + 3;
    double per = o.periodicity[d];
    DN_REQUIRE(per > 0 && std::isfinite(per), ST_BADARG, "periodicity must be positive");
    g.coordfct[d] = 1. / per;
    DN_REQUIRE(g.nuni[d] <= n, ST_BADARG, "oversampled grid smaller than uniform grid");
    auto f = fft_factors(int(n));
    for (int r : f)
      DN_REQUIRE(r <= 11, ST_UNSUPPORTED, "oversampled size must be 11-smooth");
    DN_REQUIRE(f.size() <= 24, ST_UNSUPPORTED, "too many FFT factors");
    s.factors[d] = f;
  }
  // tile keys (DUCC build_index)
  uint64_t maxkey;
  if (ndim == 1) {
    maxkey = uint64_t(g.ntiles[0]);
    s.tile_shift = 0;
    s.max_tiles = maxkey;
  } else if (ndim == 2) {
    maxkey = uint64_t(g.ntiles[0]) * uint64_t(g.ntiles[1]);
    s.tile_shift = 0;
    s.max_tiles = maxkey;
  } else {
    uint64_t prod = uint64_t(g.ntiles[0]) * g.ntiles[1] * g.ntiles[2];
    int lsq2 = g.log2tile;
    while (lsq2 >= 1 && (prod << (3 * (g.log2tile - lsq2))) < (uint64_t(1) << 28)) --lsq2;
    g.lsq2 = lsq2;
    g.ssmall = g.log2tile - lsq2;
    maxkey = prod << (3 * g.ssmall);
    s.tile_shift = 3 * g.ssmall;
    s.max_tiles = prod;
  }
  // automatic choice for type 1: the tensor-core spreader where it is the
  // faster one (measured on B200 from 256^2 to 4096^2 grids, uniform and
  // clustered points: from about half a point per uniform mode up; below that
  // its per-tile set-up and flush cost more than the plain atomics)
  if (s.spreader == DNUFFT_SPREAD_AUTO && gridding && ndim == 2 && !calc_f64 &&
      spread_tc_supported(g, calc_f64) &&
      double(npoints) >= TC_AUTO_DENSITY * double(nuni[0]) * double(nuni[1]))
    s.spreader = DNUFFT_SPREAD_TC;
  if (s.spreader == DNUFFT_SPREAD_TC && spread_tc_supported(g, calc_f64)) {
    s.qbits = true;
    maxkey <<= 2 + tc_cell_bits(g);
    s.tile_shift = 2 + tc_cell_bits(g);
    // per-chunk set-up and flush of the tensor-core spreader cost more than
    // the plain one's: amortise them over longer chunks
    s.chunk = CHUNK_TC;
  }
  DN_REQUIRE(maxkey < (uint64_t(1) << 32), ST_UNSUPPORTED, "tile key space too large");
  s.keybits = std::max(1, bitlen64(maxkey));
  if (s.spreader == DNUFFT_SPREAD_TC)
    DN_REQUIRE(spread_tc_supported(g, calc_f64), ST_UNSUPPORTED,
               "tensor-core spreader: 2D single precision (complex64) with support <= 8 only");
  auto coeff = kernel_coeffs(g.W, s.beta, s.e0);
  fill_poly(s, coeff);
  for (int d = 0; d < ndim; ++d)
    s.corfac[d] = correction_factors(size_t(g.nuni[d] / 2 + 1), 1. / double(g.nover[d]), g.W,
                                     s.beta, s.e0);
  return s;
}

// device-resident per-transform constants: correction factors and twiddles
struct DevConst {
  DevBuf corfac[3];
  DevBuf tw[3];
  FFTAxisPlan ax[3];
  const double *cf[3] = {nullptr, nullptr, nullptr};
};

static void upload_consts(const Setup &s, DevConst &dc, cudaStream_t st) {
  for (int d = 0; d < s.g.ndim; ++d) {
    size_t nb = s.corfac[d].size() * sizeof(double);
    dc.corfac[d] = DevBuf(nb, st);
    DN_CUDA(cudaMemcpyAsync(dc.corfac[d].p, s.corfac[d].data(), nb, cudaMemcpyHostToDevice, st));
    dc.cf[d] = dc.corfac[d].as<double>();
    int n = int(s.g.nover[d]);
    size_t esz = s.calc_f64 ? 16 : 8;
    dc.tw[d] = DevBuf(size_t(n) * esz, st);
    if (s.calc_f64) {
      std::vector<double> t(2 * size_t(n));
      for (int k = 0; k < n; ++k) {
        double a = -2.0 * M_PI * double(k) / double(n);
        t[2 * k] = std::cos(a);
        t[2 * k + 1] = std::sin(a);
      }
      DN_CUDA(cudaMemcpyAsync(dc.tw[d].p, t.data(), t.size() * 8, cudaMemcpyHostToDevice, st));
    } else {
      std::vector<float> t(2 * size_t(n));
      for (int k = 0; k < n; ++k) {
        double a = -2.0 * M_PI * double(k) / double(n);
        t[2 * k] = float(std::cos(a));
        t[2 * k + 1] = float(std::sin(a));
      }
      DN_CUDA(cudaMemcpyAsync(dc.tw[d].p, t.data(), t.size() * 4, cudaMemcpyHostToDevice, st));
    }
    FFTAxisPlan &p = dc.ax[d];
    p.n = n;
    p.nfac = int(s.factors[d].size());
    for (int i = 0; i < p.nfac; ++i) p.fac[i] = s.factors[d][i];
    p.tw = dc.tw[d].p;
  }
  // host vectors must stay alive until the copies ran
  DN_CUDA(cudaStreamSynchronize(st));
}

// Constants of an unplanned call, shared by later unplanned calls with the same
// geometry on the same device: the upload (host twiddles, pageable copies and
// a stream synchronisation) then happens once instead of on every call.  Up to
// MAX_SHARED geometries per process are kept (about the size of their
// twiddle tables each) for the life of the process; beyond that a call uploads
// into the caller's `local` as before.  An entry is complete (its stream was
// synchronised) before it is published, so any stream may read it.
static const DevConst &consts_for(const Setup &s, DevConst &local, cudaStream_t st) {
  constexpr size_t MAX_SHARED = 32;
  struct Key {
    int dev, ndim, f64, W;
    double beta, e0;
    int64_t nover[3], nuni[3];
    bool operator<(const Key &o) const {
      return std::memcmp(this, &o, sizeof(Key)) < 0;
    }
  };
  Key k;
  std::memset(&k, 0, sizeof(k));   // padding bytes take part in the comparison
  DN_CUDA(cudaGetDevice(&k.dev));
  k.ndim = s.g.ndim;
  k.f64 = s.calc_f64 ? 1 : 0;
  k.W = s.g.W;
  k.beta = s.beta;
  k.e0 = s.e0;
  for (int d = 0; d < s.g.ndim; ++d) {
    k.nover[d] = s.g.nover[d];
    k.nuni[d] = s.g.nuni[d];
  }
  static std::mutex mu;
  static std::map<Key, DevConst *> *cache = new std::map<Key, DevConst *>();   // never freed
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache->find(k);
  if (it != cache->end()) return *it->second;
  if (cache->size() >= MAX_SHARED) {
    upload_consts(s, local, st);
    return local;
  }
  DevConst *dc = new DevConst();   // kept until exit (not destroyed: no frees at teardown)
  upload_consts(s, *dc, st);
  (*cache)[k] = dc;
  return *dc;
}

// index: tile permutation, sorted keys and chunk list
struct Index {
  DevBuf perm, keys, chunks, count;
  uint32_t nchunks = 0;
  // tensor-core order only: K-block list and per-CTA ranges
  DevBuf kblk, kbrange;
  uint32_t nkblk = 0, groups = 0;
  TcBlocks tc() const { return TcBlocks{kblk.as<uint2>(), kbrange.as<uint32_t>(), groups, nkblk}; }
};

static uint32_t sm_count() {
  int dev = 0, n = 0;
  DN_CUDA(cudaGetDevice(&dev));
  DN_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
  return uint32_t(n > 0 ? n : 1);
}

static void build_index(const Setup &s, const View &coord, Index &ix, cudaStream_t st) {
  uint32_t M = s.npoints;
  ix.perm = DevBuf(size_t(M) * 4, st);
  ix.keys = DevBuf(size_t(M) * 4, st);
  launch_fold_keys(s.coord_f64, coord.data, coord.stride[0], coord.stride[1], M, s.g,
                   ix.keys.as<uint32_t>(), ix.perm.as<uint32_t>(), st, s.qbits);
  {
    DevBuf ws(radix_workspace_bytes(M, s.keybits), st);
    radix_sort_pairs(ix.keys.as<uint32_t>(), ix.perm.as<uint32_t>(), M, s.keybits, ws.p, st);
  }
  uint64_t maxchunks = std::min<uint64_t>(M, s.max_tiles) + M / s.chunk + 2;
  ix.chunks = DevBuf(size_t(maxchunks) * sizeof(Chunk), st);
  ix.count = DevBuf(16, st);
  DevBuf ws(chunk_workspace_bytes(M), st);
  ix.nchunks = build_chunks(ix.keys.as<uint32_t>(), M, s.tile_shift, s.chunk, ix.chunks.as<Chunk>(),
                            ix.count.as<uint32_t>(), ws.p, st);
  if (s.qbits && ix.nchunks > 0) {
    ix.groups = sm_count();
    ix.kblk = DevBuf(size_t(tc_kblock_upper_bound(M, ix.nchunks)) * sizeof(uint2), st);
    ix.kbrange = DevBuf(size_t(ix.groups + 1) * sizeof(uint32_t), st);
    DevBuf kws(tc_kblock_workspace_bytes(ix.nchunks), st);
    ChunkList cl{ix.chunks.as<Chunk>(), ix.nchunks};
    ix.nkblk = build_tc_kblocks(ix.keys.as<uint32_t>(), cl, ix.groups, kws.p, ix.kblk.as<uint2>(),
                                ix.kbrange.as<uint32_t>(), ix.count.as<uint32_t>(),
                                tc_cell_bits(s.g), st);
  }
}

static size_t grid_cells(const Geometry &g) {
  size_t c = 1;
  for (int d = 0; d < g.ndim; ++d) c *= size_t(g.nover[d]);
  return c;
}

static void report_sizes(const Setup &s, bool gridding) {
  const Geometry &g = s.g;
  std::printf("%s\n  device=B200 (CUDA), grid=(", gridding ? "Nu2u:" : "U2nu:");
  for (int d = 0; d < g.ndim; ++d) std::printf(d ? "x%lld" : "%lld", (long long)g.nuni[d]);
  std::printf("), oversampled grid=(");
  for (int d = 0; d < g.ndim; ++d) std::printf(d ? "x%lld" : "%lld", (long long)g.nover[d]);
  std::printf("), supp=%d, eps=%g\n  npoints=%u\n  memory overhead: %gGB (index) + %gGB "
              "(oversampled grid)\n",
              g.W, s.epsilon, s.npoints, s.npoints * 4.0 / double(1 << 30),
              double(grid_cells(g)) * (s.calc_f64 ? 16 : 8) / double(1 << 30));
  std::fflush(stdout);
}

// ---------------------------------------------------------------- transforms
// Spreading of the points of pts (values at `values` with stride vs) into the
// oversampled grid: the tensor-core spreader where the setup chose it, else
// the plain one.
template <typename T>
static void spread_points(const Setup &s, const PointsDesc &pts, const ChunkList &cl,
                          const TcBlocks *tb, const void *values, int64_t vs, void *grid, int *err,
                          cudaStream_t st) {
  const KernelPoly<T> &kp = *reinterpret_cast<const KernelPoly<T> *>(
      sizeof(T) == 4 ? static_cast<const void *>(&s.kpf) : static_cast<const void *>(&s.kpd));
  bool use_tc = false;
  if constexpr (sizeof(T) == 4) {
    bool ok = spread_tc_supported(s.g, s.calc_f64);
    DN_REQUIRE(s.spreader != DNUFFT_SPREAD_TC || ok, ST_UNSUPPORTED,
               "tensor-core spreader: 2D single precision with support <= 8 only");
    use_tc = ok && s.qbits && tb != nullptr;
  } else {
    DN_REQUIRE(s.spreader != DNUFFT_SPREAD_TC, ST_UNSUPPORTED,
               "tensor-core spreader: single precision (complex64) only");
  }
  if (use_tc) {
    launch_spread_tc(pts, *tb, s.g, s.kpf, values, vs, grid, reinterpret_cast<unsigned *>(err + 1),
                     err, st);
  } else {
    launch_spread<T>(pts, cl, s.g, kp, values, vs, 0, grid, 0, 1, st);
  }
}

template <typename T>
static void do_spread_fft(const Setup &s, const DevConst &dc, const PointsDesc &pts,
                          const ChunkList &cl, const TcBlocks *tb, const View &points,
                          const View &out, bool forward, bool fft_order, StageTimer &tm,
                          cudaStream_t st, DevBuf *ws = nullptr, DevBuf *wk = nullptr) {
  size_t cells = grid_cells(s.g);
  tm.mark("zeroing grid");
  DevBuf local;
  DevBuf &grid = ws ? *ws : local;
  if (!grid.p) grid = DevBuf(cells * sizeof(T) * 2, st);
  DN_CUDA(cudaMemsetAsync(grid.p, 0, cells * sizeof(T) * 2, st));
  tm.mark("spreading");
  int *err = device_error_word();
  spread_points<T>(s, pts, cl, tb, points.data, points.stride[0], grid.p, err, st);
  tm.mark("FFT + correction");
  DevBuf localw;
  DevBuf &work = wk ? *wk : localw;
  const size_t wb = fft_work_bytes(s.g, sizeof(T) * 2);
  if (wb && !work.p) work = DevBuf(wb, st);
  fft_nu2u_tail<T>(grid.p, s.g, dc.ax, forward, dc.cf, fft_order, out.data, out.stride, st,
                   work.p, err);
  tm.mark("output copy");   // last mark of a planned call; an unplanned call copies out next
  check_device_error(err, st);
}

// With a side stream, the FFT pass runs there and st waits for it before the
// interpolation; the caller provides the grid and work buffers, allocated on
// st before the side stream was last started (so the FFT does not wait for
// whatever st queued after that, e.g. the index build).
template <typename T>
static void do_fft_interp(const Setup &s, const DevConst &dc, const PointsDesc &pts,
                          const ChunkList &cl, const View &uni, const View &out, bool forward,
                          bool fft_order, StageTimer &tm, cudaStream_t st, DevBuf *ws = nullptr,
                          DevBuf *wk = nullptr, SideStream *side = nullptr) {
  size_t cells = grid_cells(s.g);
  DevBuf local;
  DevBuf &grid = ws ? *ws : local;
  if (!grid.p) grid = DevBuf(cells * sizeof(T) * 2, st);
  DevBuf localw;
  DevBuf &work = wk ? *wk : localw;
  const size_t wb = fft_work_bytes(s.g, sizeof(T) * 2);
  if (wb && !work.p) work = DevBuf(wb, st);
  int *err = device_error_word();
  tm.mark("correction + FFT");
  if (side) {
    DN_REQUIRE(ws && wk, ST_INTERNAL, "side-stream FFT without preallocated buffers");
    fft_u2nu_head<T>(uni.data, uni.stride, s.g, dc.ax, forward, dc.cf, fft_order, grid.p,
                     side->s, work.p, err);
    side->merge();
  } else {
    fft_u2nu_head<T>(uni.data, uni.stride, s.g, dc.ax, forward, dc.cf, fft_order, grid.p, st,
                     work.p, err);
  }
  tm.mark("interpolation");
  const KernelPoly<T> &kp = *reinterpret_cast<const KernelPoly<T> *>(
      sizeof(T) == 4 ? static_cast<const void *>(&s.kpf) : static_cast<const void *>(&s.kpd));
  launch_interp<T>(pts, cl, s.g, kp, grid.p, 0, out.data, out.stride[0], 0, 1, st, err);
  tm.mark("output copy");
  check_device_error(err, st);
}

template <typename T>
static void do_fft_dcoord(const Setup &s, const DevConst &dc, const PointsDesc &pts,
                          const ChunkList &cl, const View &uni, const View &wts,
                          const View &grad, bool forward, bool fft_order, StageTimer &tm,
                          cudaStream_t st, DevBuf *ws = nullptr, DevBuf *wk = nullptr) {
  size_t cells = grid_cells(s.g);
  DevBuf local;
  DevBuf &grid = ws ? *ws : local;
  if (!grid.p) grid = DevBuf(cells * sizeof(T) * 2, st);
  DevBuf localw;
  DevBuf &work = wk ? *wk : localw;
  const size_t wb = fft_work_bytes(s.g, sizeof(T) * 2);
  if (wb && !work.p) work = DevBuf(wb, st);
  int *err = device_error_word();
  tm.mark("correction + FFT");
  fft_u2nu_head<T>(uni.data, uni.stride, s.g, dc.ax, forward, dc.cf, fft_order, grid.p, st,
                   work.p, err);
  tm.mark("derivative interpolation");
  const KernelPoly<T> &kp = *reinterpret_cast<const KernelPoly<T> *>(
      sizeof(T) == 4 ? static_cast<const void *>(&s.kpf) : static_cast<const void *>(&s.kpd));
  launch_interp_dcoord<T>(pts, cl, s.g, kp, grid.p, wts.data, wts.stride[0], grad.data,
                          grad.stride[0], grad.stride[1], st);
  tm.mark("end");
  check_device_error(err, st);
}

static void check_dcoord_args(const View &wts, const View &grad, int cdt, int coord_dt,
                              uint64_t npoints, int ndim) {
  DN_REQUIRE(wts.ndim == 1 && uint64_t(wts.shape[0]) == npoints, ST_BADARG,
             "weights: number of points mismatch");
  DN_REQUIRE(wts.dtype == cdt, ST_BADARG, "weights must have the grid's dtype");
  DN_REQUIRE(grad.ndim == 2 && uint64_t(grad.shape[0]) == npoints && grad.shape[1] == ndim,
             ST_BADARG, "grad must be (npoints, ndim)");
  DN_REQUIRE(grad.dtype == coord_dt, ST_BADARG, "grad must have the coordinates' dtype");
}

static void zero_view(const View &v, cudaStream_t st) {
  DN_REQUIRE(v.ndim <= 3, ST_BADARG, "bad output rank");
  zero_strided(v.data, v.ndim, v.shape, v.stride, dtype_size(v.dtype), st);
}

static void check_coord(const View &coord, int ndim) {
  DN_REQUIRE(coord.ndim == 2, ST_BADARG, "coord must be a 2D array (npoints, ndim)");
  DN_REQUIRE(coord.dtype == DNUFFT_F32 || coord.dtype == DNUFFT_F64, ST_BADARG,
             "coord must be float32 or float64");
  DN_REQUIRE(coord.shape[1] == ndim, ST_BADARG, "dimensionality mismatch");
}

static dnufft_opts resolved(const dnufft_opts *o, bool for_plan) {
  dnufft_opts r;
  if (o) {
    r = *o;
  } else {
    dnufft_default_opts(&r, for_plan ? 1 : 0);
  }
  return r;
}

// ---------------------------------------------------------------- pipelined host calls
// Unplanned calls whose points come from host memory are bound by the PCIe
// transfers (about 55 GB/s each way).  Large ones are cut into groups of
// consecutive points (in the caller's order).  Every group is sorted and spread
// on its own (type 1: spreading adds into one grid) or sorted and interpolated
// on its own (type 2: its results are one contiguous range), so the
// host->device copy of the next groups, and for type 2 the device->host copy of
// the finished groups' results, overlap the work on the current one.  Kernel,
// oversampled grid and FFT are those of the whole problem.
constexpr uint32_t PIPE_MIN_POINTS = 1u << 22;     // pipelined from 4M points
constexpr uint32_t PIPE_GROUP_POINTS = 8500000u;   // about this many per group

static int pipe_groups(uint32_t M) {
  if (M < PIPE_MIN_POINTS) return 1;
  const int G = int((uint64_t(M) + PIPE_GROUP_POINTS - 1) / PIPE_GROUP_POINTS);
  return std::max(2, std::min(8, G));
}

struct EventSet {
  std::vector<cudaEvent_t> ev;
  explicit EventSet(int n) : ev(size_t(n), nullptr) {
    for (auto &e : ev) DN_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  ~EventSet() {
    for (auto e : ev)
      if (e) cudaEventDestroy(e);
  }
};

// first point of group gi of G over M points
static uint64_t group_start(uint32_t M, int G, int gi) { return uint64_t(M) * uint64_t(gi) / uint64_t(G); }

// coordinates (C-contiguous (M, d) device copy) of points [a, b)
static View coord_range(const View &coord, void *dev, uint64_t a, uint64_t b, size_t cb) {
  View v = coord;
  v.data = static_cast<char *>(dev) + a * size_t(coord.shape[1]) * cb;
  v.shape[0] = int64_t(b - a);
  v.host = false;
  return v;
}

template <typename T>
static void nu2u_pipelined(const Setup &s, const View &points, const View &coord, const View &out,
                           bool forward, bool fft_order, StageTimer &tm, cudaStream_t st) {
  const uint32_t M = s.npoints;
  const size_t nd = size_t(coord.shape[1]);
  const size_t cb = s.coord_f64 ? 8 : 4, vb = sizeof(T) * 2;
  const int G = pipe_groups(M);
  tm.mark("upload constants");
  DevConst dcl;
  const DevConst &dc = consts_for(s, dcl, st);
  DevBuf dcoord(size_t(M) * nd * cb, st), dvals(size_t(M) * vb, st);
  const size_t cells = grid_cells(s.g);
  DevBuf grid(cells * vb, st), work;
  const size_t wb = fft_work_bytes(s.g, vb);
  if (wb) work = DevBuf(wb, st);
  Staged so(out, false, true, st);
  EventSet copied(G);
  // declared after the buffers: destroyed (after synchronising) before them
  SideStream up(st, true);
  up.start();
  // zeroed on the caller's stream while the first groups are copied in
  DN_CUDA(cudaMemsetAsync(grid.p, 0, cells * vb, st));
  for (int gi = 0; gi < G; ++gi) {
    const uint64_t a = group_start(M, G, gi), b = group_start(M, G, gi + 1);
    DN_CUDA(cudaMemcpyAsync(static_cast<char *>(dcoord.p) + a * nd * cb,
                            static_cast<const char *>(coord.data) + a * nd * cb, (b - a) * nd * cb,
                            cudaMemcpyHostToDevice, up.s));
    DN_CUDA(cudaMemcpyAsync(static_cast<char *>(dvals.p) + a * vb,
                            static_cast<const char *>(points.data) + a * vb, (b - a) * vb,
                            cudaMemcpyHostToDevice, up.s));
    DN_CUDA(cudaEventRecord(copied.ev[gi], up.s));
  }
  tm.mark("groups: index + spreading");
  int *err = device_error_word();
  for (int gi = 0; gi < G; ++gi) {
    const uint64_t a = group_start(M, G, gi), b = group_start(M, G, gi + 1);
    DN_CUDA(cudaStreamWaitEvent(st, copied.ev[gi], 0));
    Setup sg = s;
    sg.npoints = uint32_t(b - a);
    const View cv = coord_range(coord, dcoord.p, a, b, cb);
    Index ix;
    build_index(sg, cv, ix, st);
    PointsDesc pts{cv.data, cv.stride[0], cv.stride[1], false, s.coord_f64,
                   ix.perm.as<uint32_t>(), sg.npoints};
    ChunkList cl{ix.chunks.as<Chunk>(), ix.nchunks};
    const TcBlocks tb = ix.tc();
    spread_points<T>(sg, pts, cl, &tb, static_cast<char *>(dvals.p) + a * vb, 1, grid.p, err, st);
  }
  tm.mark("FFT + correction");
  fft_nu2u_tail<T>(grid.p, s.g, dc.ax, forward, dc.cf, fft_order, so.dev.data, so.dev.stride, st,
                   work.p, err);
  tm.mark("output copy");
  check_device_error(err, st);
  so.finish();
}

template <typename T>
static void u2nu_pipelined(const Setup &s, const View &uni, const View &coord, const View &out,
                           bool forward, bool fft_order, StageTimer &tm, cudaStream_t st) {
  const uint32_t M = s.npoints;
  const size_t nd = size_t(coord.shape[1]);
  const size_t cb = s.coord_f64 ? 8 : 4, vb = sizeof(T) * 2;
  const int G = pipe_groups(M);
  tm.mark("upload constants");
  DevConst dcl;
  const DevConst &dc = consts_for(s, dcl, st);
  DevBuf dcoord(size_t(M) * nd * cb, st), duni, dout;
  const size_t ubytes = size_t(nelem(uni)) * vb;
  if (uni.host) duni = DevBuf(ubytes, st);
  if (out.host) dout = DevBuf(size_t(M) * vb, st);
  DevBuf grid(grid_cells(s.g) * vb, st), work;
  const size_t wb = fft_work_bytes(s.g, vb);
  if (wb) work = DevBuf(wb, st);
  View uv = uni, ov = out;
  if (uni.host) {
    uv.data = duni.p;
    uv.host = false;
  }
  if (out.host) {
    ov.data = dout.p;
    ov.host = false;
  }
  EventSet copied(G + 1), done(G);
  // declared after the buffers: destroyed (after synchronising) before them
  SideStream up(st, true), down(st, out.host);
  up.start();
  down.start();
  // the uniform grid first, then the coordinates group by group
  if (uni.host) DN_CUDA(cudaMemcpyAsync(duni.p, uni.data, ubytes, cudaMemcpyHostToDevice, up.s));
  DN_CUDA(cudaEventRecord(copied.ev[G], up.s));
  for (int gi = 0; gi < G; ++gi) {
    const uint64_t a = group_start(M, G, gi), b = group_start(M, G, gi + 1);
    DN_CUDA(cudaMemcpyAsync(static_cast<char *>(dcoord.p) + a * nd * cb,
                            static_cast<const char *>(coord.data) + a * nd * cb, (b - a) * nd * cb,
                            cudaMemcpyHostToDevice, up.s));
    DN_CUDA(cudaEventRecord(copied.ev[gi], up.s));
  }
  int *err = device_error_word();
  tm.mark("correction + FFT");
  DN_CUDA(cudaStreamWaitEvent(st, copied.ev[G], 0));
  fft_u2nu_head<T>(uv.data, uv.stride, s.g, dc.ax, forward, dc.cf, fft_order, grid.p, st, work.p,
                   err);
  tm.mark("groups: index + interpolation");
  const KernelPoly<T> &kp = *reinterpret_cast<const KernelPoly<T> *>(
      sizeof(T) == 4 ? static_cast<const void *>(&s.kpf) : static_cast<const void *>(&s.kpd));
  for (int gi = 0; gi < G; ++gi) {
    const uint64_t a = group_start(M, G, gi), b = group_start(M, G, gi + 1);
    DN_CUDA(cudaStreamWaitEvent(st, copied.ev[gi], 0));
    Setup sg = s;
    sg.npoints = uint32_t(b - a);
    const View cv = coord_range(coord, dcoord.p, a, b, cb);
    Index ix;
    build_index(sg, cv, ix, st);
    PointsDesc pts{cv.data, cv.stride[0], cv.stride[1], false, s.coord_f64,
                   ix.perm.as<uint32_t>(), sg.npoints};
    ChunkList cl{ix.chunks.as<Chunk>(), ix.nchunks};
    launch_interp<T>(pts, cl, s.g, kp, grid.p, 0,
                     static_cast<char *>(ov.data) + a * size_t(ov.stride[0]) * vb, ov.stride[0], 0,
                     1, st, err);
    if (out.host) {
      // the finished range goes back while the next groups are interpolated
      DN_CUDA(cudaEventRecord(done.ev[gi], st));
      DN_CUDA(cudaStreamWaitEvent(down.s, done.ev[gi], 0));
      DN_CUDA(cudaMemcpyAsync(static_cast<char *>(out.data) + a * vb,
                              static_cast<const char *>(dout.p) + a * vb, (b - a) * vb,
                              cudaMemcpyDeviceToHost, down.s));
    }
  }
  tm.mark("output copy");
  down.merge();
  check_device_error(err, st);
  DN_CUDA(cudaStreamSynchronize(st));
}

static void nu2u_impl(const dnufft_array *points_, const dnufft_array *coord_, int forward,
                      double eps, dnufft_array *out_, const dnufft_opts *opts_, cudaStream_t st) {
  dnufft_opts o = resolved(opts_, false);
  View points = view_of(points_, "points"), coord = view_of(coord_, "coord"),
       out = view_of(out_, "out");
  int ndim = out.ndim;
  DN_REQUIRE(ndim >= 1 && ndim <= 3, ST_BADARG, "transform must be 1D/2D/3D");
  check_coord(coord, ndim);
  DN_REQUIRE(points.ndim == 1, ST_BADARG, "points must be 1D");
  DN_REQUIRE(points.shape[0] == coord.shape[0], ST_BADARG, "number of points mismatch");
  DN_REQUIRE(points.dtype == DNUFFT_C64 || points.dtype == DNUFFT_C128, ST_BADARG,
             "points must be complex64 or complex128");
  DN_REQUIRE(out.dtype == points.dtype, ST_BADARG, "out must have the dtype of points");
  bool f64 = points.dtype == DNUFFT_C128;
  Setup s = make_setup(ndim, out.shape, uint64_t(points.shape[0]), eps, true, f64,
                       coord.dtype == DNUFFT_F64, o);
  StageTimer tm(o.verbosity > 0, st);
  if (o.verbosity > 0) report_sizes(s, true);
  if (points.host && coord.host && pipe_groups(s.npoints) > 1) {
    if (f64)
      nu2u_pipelined<double>(s, points, coord, out, forward != 0, o.fft_order != 0, tm, st);
    else
      nu2u_pipelined<float>(s, points, coord, out, forward != 0, o.fft_order != 0, tm, st);
    tm.mark("end");
    tm.report("nu2u");
    return;
  }
  // constants first (small pageable copies, which would otherwise queue behind
  // the large transfers on the copy engine)
  tm.mark("upload constants");
  DevConst dcl;
  const DevConst &dc = s.npoints ? consts_for(s, dcl, st) : dcl;
  tm.mark("coordinates host->device");
  // host arrays: the coordinates next; the point values follow on a side
  // stream while this stream builds the index
  SideStream side(st, points.host);
  Staged sc(coord, true, false, st);
  Staged sp(points, true, false, st, &side), so(out, false, true, st);
  if (s.npoints == 0) {
    side.merge();
    zero_view(so.dev, st);
    so.finish();
    return;
  }
  tm.mark("building index");
  Index ix;
  build_index(s, sc.dev, ix, st);
  tm.mark("wait for values copy");
  side.merge();
  PointsDesc pts{sc.dev.data, sc.dev.stride[0], sc.dev.stride[1], false, s.coord_f64,
                 ix.perm.as<uint32_t>(), s.npoints};
  ChunkList cl{ix.chunks.as<Chunk>(), ix.nchunks};
  const TcBlocks tb = ix.tc();
  if (f64)
    do_spread_fft<double>(s, dc, pts, cl, &tb, sp.dev, so.dev, forward != 0,
                          o.fft_order != 0, tm, st);
  else
    do_spread_fft<float>(s, dc, pts, cl, &tb, sp.dev, so.dev, forward != 0,
                         o.fft_order != 0, tm, st);
  so.finish();
  tm.mark("end");
  tm.report("nu2u");
}

static void u2nu_impl(const dnufft_array *grid_, const dnufft_array *coord_, int forward,
                      double eps, dnufft_array *out_, const dnufft_opts *opts_, cudaStream_t st) {
  dnufft_opts o = resolved(opts_, false);
  View uni = view_of(grid_, "grid"), coord = view_of(coord_, "coord"), out = view_of(out_, "out");
  int ndim = uni.ndim;
  DN_REQUIRE(ndim >= 1 && ndim <= 3, ST_BADARG, "transform must be 1D/2D/3D");
  check_coord(coord, ndim);
  DN_REQUIRE(out.ndim == 1 && out.shape[0] == coord.shape[0], ST_BADARG,
             "number of points mismatch");
  DN_REQUIRE(uni.dtype == DNUFFT_C64 || uni.dtype == DNUFFT_C128, ST_BADARG,
             "grid must be complex64 or complex128");
  DN_REQUIRE(out.dtype == uni.dtype, ST_BADARG, "out must have the dtype of grid");
  bool f64 = uni.dtype == DNUFFT_C128;
  Setup s = make_setup(ndim, uni.shape, uint64_t(coord.shape[0]), eps, false, f64,
                       coord.dtype == DNUFFT_F64, o);
  StageTimer tm(o.verbosity > 0, st);
  if (o.verbosity > 0) report_sizes(s, false);
  if (s.npoints == 0) return;
  if (coord.host && pipe_groups(s.npoints) > 1) {
    if (f64)
      u2nu_pipelined<double>(s, uni, coord, out, forward != 0, o.fft_order != 0, tm, st);
    else
      u2nu_pipelined<float>(s, uni, coord, out, forward != 0, o.fft_order != 0, tm, st);
    tm.mark("end");
    tm.report("u2nu");
    return;
  }
  tm.mark("upload constants");
  DevConst dcl;
  const DevConst &dc = consts_for(s, dcl, st);
  tm.mark("coordinates host->device");
  // host arrays: the coordinates first; the uniform grid follows on a side
  // stream, which also runs the FFT pass, while this stream builds the index
  SideStream side(st, uni.host);
  Staged sc(coord, true, false, st), so(out, false, true, st);
  Staged su(uni, true, false, st, &side);
  const size_t esz = f64 ? 16 : 8;
  DevBuf grid(grid_cells(s.g) * esz, st), work;
  const size_t wb = fft_work_bytes(s.g, esz);
  if (wb) work = DevBuf(wb, st);
  side.start();   // the FFT pass may use the buffers from here on
  tm.mark("building index");
  Index ix;
  build_index(s, sc.dev, ix, st);
  PointsDesc pts{sc.dev.data, sc.dev.stride[0], sc.dev.stride[1], false, s.coord_f64,
                 ix.perm.as<uint32_t>(), s.npoints};
  ChunkList cl{ix.chunks.as<Chunk>(), ix.nchunks};
  if (f64)
    do_fft_interp<double>(s, dc, pts, cl, su.dev, so.dev, forward != 0, o.fft_order != 0, tm, st,
                          &grid, &work, side.active() ? &side : nullptr);
  else
    do_fft_interp<float>(s, dc, pts, cl, su.dev, so.dev, forward != 0, o.fft_order != 0, tm, st,
                         &grid, &work, side.active() ? &side : nullptr);
  so.finish();
  tm.mark("end");
  tm.report("u2nu");
}

static void u2nu_dcoord_impl(const dnufft_array *grid_, const dnufft_array *coord_, int forward,
                             double eps, const dnufft_array *wts_, dnufft_array *grad_,
                             const dnufft_opts *opts_, cudaStream_t st) {
  dnufft_opts o = resolved(opts_, false);
  View uni = view_of(grid_, "grid"), coord = view_of(coord_, "coord");
  View wts = view_of(wts_, "weights"), grad = view_of(grad_, "grad");
  int ndim = uni.ndim;
  DN_REQUIRE(ndim >= 1 && ndim <= 3, ST_BADARG, "transform must be 1D/2D/3D");
  check_coord(coord, ndim);
  DN_REQUIRE(uni.dtype == DNUFFT_C64 || uni.dtype == DNUFFT_C128, ST_BADARG,
             "grid must be complex64 or complex128");
  check_dcoord_args(wts, grad, uni.dtype, coord.dtype, uint64_t(coord.shape[0]), ndim);
  bool f64 = uni.dtype == DNUFFT_C128;
  Setup s = make_setup(ndim, uni.shape, uint64_t(coord.shape[0]), eps, false, f64,
                       coord.dtype == DNUFFT_F64, o);
  StageTimer tm(o.verbosity > 0, st);
  if (s.npoints == 0) return;
  Staged su(uni, true, false, st), sc(coord, true, false, st), sw(wts, true, false, st),
      sg(grad, false, true, st);
  tm.mark("upload constants");
  DevConst dcl;
  const DevConst &dc = consts_for(s, dcl, st);
  tm.mark("building index");
  Index ix;
  build_index(s, sc.dev, ix, st);
  PointsDesc pts{sc.dev.data, sc.dev.stride[0], sc.dev.stride[1], false, s.coord_f64,
                 ix.perm.as<uint32_t>(), s.npoints};
  ChunkList cl{ix.chunks.as<Chunk>(), ix.nchunks};
  if (f64)
    do_fft_dcoord<double>(s, dc, pts, cl, su.dev, sw.dev, sg.dev, forward != 0, o.fft_order != 0,
                          tm, st);
  else
    do_fft_dcoord<float>(s, dc, pts, cl, su.dev, sw.dev, sg.dev, forward != 0, o.fft_order != 0,
                         tm, st);
  tm.report("u2nu_dcoord");
  sg.finish();
}

}  // namespace dnufft

// ---------------------------------------------------------------- plans
namespace dnufft {
// One group of a plan's points, split by input order: points [a, b) with
// their own index and sorted coordinates.  A plan made from host coordinates
// with many points keeps these beside its whole-plan index, so that calls on
// host arrays copy one group's values in (type 1) or its results out (type 2)
// while other groups are spread or interpolated.
struct PlanGroup {
  uint64_t a = 0, b = 0;
  Index ix;
  DevBuf sorted_coord;
};
}  // namespace dnufft

struct dnufft_plan {
  dnufft::Setup s;
  dnufft::DevConst dc;
  dnufft::Index ix;
  dnufft::DevBuf sorted_coord;
  dnufft::DevBuf grid;   // oversampled grid, allocated on first execution
  dnufft::DevBuf work;   // FFT column-pass scratch (2D), allocated on first execution
  std::vector<dnufft::PlanGroup> groups;   // host-coordinate plans with many points
  dnufft_opts o;
  int device = 0;
};

namespace dnufft {

static void plan_create_impl(int nu2u, const dnufft_array *coord_, const int64_t *shape, int ndim,
                             double eps, const dnufft_opts *opts_, cudaStream_t st,
                             dnufft_plan **out) {
  DN_REQUIRE(out != nullptr, ST_BADARG, "null plan pointer");
  DN_REQUIRE(shape != nullptr, ST_BADARG, "null grid shape");
  dnufft_opts o = resolved(opts_, true);
  View coord = view_of(coord_, "coord");
  DN_REQUIRE(ndim >= 1 && ndim <= 3, ST_BADARG, "unsupported dimensionality");
  check_coord(coord, ndim);
  bool f64 = coord.dtype == DNUFFT_F64;
  auto p = std::make_unique<dnufft_plan>();
  p->o = o;
  p->s = make_setup(ndim, shape, uint64_t(coord.shape[0]), eps, nu2u != 0, f64, f64, o);
  DN_CUDA(cudaGetDevice(&p->device));
  upload_consts(p->s, p->dc, st);
  if (p->s.npoints > 0) {
    Staged sc(coord, true, false, st);
    build_index(p->s, sc.dev, p->ix, st);
    p->sorted_coord = DevBuf(size_t(p->s.npoints) * ndim * (f64 ? 8 : 4), st);
    launch_gather_coords(f64, sc.dev.data, sc.dev.stride[0], sc.dev.stride[1], ndim,
                         p->ix.perm.as<uint32_t>(), p->s.npoints, p->sorted_coord.p, st);
    // the plan keeps the sorted coordinates (and, for the tensor-core
    // spreader, the K-block list); the sorted keys are no longer needed
    p->ix.keys.release();
    // coordinates from the host: the caller will likely pass host arrays,
    // whose copies the per-group index lets overlap with the work
    const int G = pipe_groups(p->s.npoints);
    if (coord.host && G > 1) {
      const size_t cb = f64 ? 8 : 4;
      p->groups.resize(size_t(G));
      for (int gi = 0; gi < G; ++gi) {
        PlanGroup &pg = p->groups[size_t(gi)];
        pg.a = group_start(p->s.npoints, G, gi);
        pg.b = group_start(p->s.npoints, G, gi + 1);
        Setup sg = p->s;
        sg.npoints = uint32_t(pg.b - pg.a);
        const View cv = coord_range(coord, sc.dev.data, pg.a, pg.b, cb);
        build_index(sg, cv, pg.ix, st);
        pg.sorted_coord = DevBuf(size_t(sg.npoints) * ndim * cb, st);
        launch_gather_coords(f64, cv.data, cv.stride[0], cv.stride[1], ndim,
                             pg.ix.perm.as<uint32_t>(), sg.npoints, pg.sorted_coord.p, st);
        pg.ix.keys.release();
      }
    }
  }
  DN_CUDA(cudaStreamSynchronize(st));
  *out = p.release();
}

static void plan_buffers(dnufft_plan *p, cudaStream_t st) {
  if (p->grid.p) return;
  // allocated once, on first use, and made visible to every stream
  const size_t vb = p->s.calc_f64 ? 16 : 8;
  p->grid = DevBuf(grid_cells(p->s.g) * vb, st);
  const size_t wb = fft_work_bytes(p->s.g, vb);
  if (wb) p->work = DevBuf(wb, st);
  DN_CUDA(cudaStreamSynchronize(st));
}

static PointsDesc group_points(const dnufft_plan *p, const PlanGroup &pg) {
  return PointsDesc{pg.sorted_coord.p, int64_t(p->s.g.ndim), 1, true, p->s.coord_f64,
                    pg.ix.perm.as<uint32_t>(), uint32_t(pg.b - pg.a)};
}

// Planned type 1 on host values, group by group: the values of later groups
// are copied in (side stream) while earlier groups are spread.
template <typename T>
static void plan_nu2u_groups(dnufft_plan *p, const View &points, const View &out, bool forward,
                             StageTimer &tm, cudaStream_t st) {
  const Setup &s = p->s;
  const size_t vb = sizeof(T) * 2;
  const int G = int(p->groups.size());
  Staged so(out, false, true, st);
  DevBuf dvals(size_t(s.npoints) * vb, st);
  EventSet copied(G);
  // declared after the buffers: destroyed (after synchronising) before them
  SideStream up(st, true);
  up.start();
  for (int gi = 0; gi < G; ++gi) {
    const PlanGroup &pg = p->groups[size_t(gi)];
    DN_CUDA(cudaMemcpyAsync(static_cast<char *>(dvals.p) + pg.a * vb,
                            static_cast<const char *>(points.data) + pg.a * vb,
                            (pg.b - pg.a) * vb, cudaMemcpyHostToDevice, up.s));
    DN_CUDA(cudaEventRecord(copied.ev[size_t(gi)], up.s));
  }
  tm.mark("zeroing grid");
  DN_CUDA(cudaMemsetAsync(p->grid.p, 0, grid_cells(s.g) * vb, st));
  tm.mark("groups: spreading");
  int *err = device_error_word();
  for (int gi = 0; gi < G; ++gi) {
    const PlanGroup &pg = p->groups[size_t(gi)];
    DN_CUDA(cudaStreamWaitEvent(st, copied.ev[size_t(gi)], 0));
    Setup sg = s;
    sg.npoints = uint32_t(pg.b - pg.a);
    const ChunkList cl{pg.ix.chunks.as<Chunk>(), pg.ix.nchunks};
    const TcBlocks tb = pg.ix.tc();
    spread_points<T>(sg, group_points(p, pg), cl, s.qbits ? &tb : nullptr,
                     static_cast<char *>(dvals.p) + pg.a * vb, 1, p->grid.p, err, st);
  }
  tm.mark("FFT + correction");
  fft_nu2u_tail<T>(p->grid.p, s.g, p->dc.ax, forward, p->dc.cf, p->o.fft_order != 0,
                   so.dev.data, so.dev.stride, st, p->work.p, err);
  tm.mark("output copy");
  check_device_error(err, st);
  up.merge();
  so.finish();
}

// Planned type 2 into a host array, group by group: each group's results go
// back (side stream) while the next groups are interpolated.
template <typename T>
static void plan_u2nu_groups(dnufft_plan *p, const View &uni, const View &out, bool forward,
                             StageTimer &tm, cudaStream_t st) {
  const Setup &s = p->s;
  const size_t vb = sizeof(T) * 2;
  const int G = int(p->groups.size());
  Staged su(uni, true, false, st);
  DevBuf dout(size_t(s.npoints) * vb, st);
  EventSet done(G);
  // declared after the buffers: destroyed (after synchronising) before them
  SideStream down(st, true);
  down.start();
  int *err = device_error_word();
  tm.mark("correction + FFT");
  fft_u2nu_head<T>(su.dev.data, su.dev.stride, s.g, p->dc.ax, forward, p->dc.cf,
                   p->o.fft_order != 0, p->grid.p, st, p->work.p, err);
  tm.mark("groups: interpolation");
  const KernelPoly<T> &kp = *reinterpret_cast<const KernelPoly<T> *>(
      sizeof(T) == 4 ? static_cast<const void *>(&s.kpf) : static_cast<const void *>(&s.kpd));
  for (int gi = 0; gi < G; ++gi) {
    const PlanGroup &pg = p->groups[size_t(gi)];
    const ChunkList cl{pg.ix.chunks.as<Chunk>(), pg.ix.nchunks};
    launch_interp<T>(group_points(p, pg), cl, s.g, kp, p->grid.p, 0,
                     static_cast<char *>(dout.p) + pg.a * vb, 1, 0, 1, st, err);
    DN_CUDA(cudaEventRecord(done.ev[size_t(gi)], st));
    DN_CUDA(cudaStreamWaitEvent(down.s, done.ev[size_t(gi)], 0));
    DN_CUDA(cudaMemcpyAsync(static_cast<char *>(out.data) + pg.a * vb,
                            static_cast<const char *>(dout.p) + pg.a * vb, (pg.b - pg.a) * vb,
                            cudaMemcpyDeviceToHost, down.s));
  }
  tm.mark("output copy");
  down.merge();
  check_device_error(err, st);
  DN_CUDA(cudaStreamSynchronize(st));
}

static void plan_exec_one(dnufft_plan *p, bool type1, int forward, int verbosity, const View &in,
                          const View &out, cudaStream_t st);

// The array without its leading (transform) axis, at transform t.
static View slice0(const View &v, int64_t t) {
  View r = v;
  r.data = static_cast<char *>(v.data) + t * v.stride[0] * int64_t(dtype_size(v.dtype));
  r.ndim = v.ndim - 1;
  for (int d = 0; d < r.ndim; ++d) {
    r.shape[d] = v.shape[d + 1];
    r.stride[d] = v.stride[d + 1];
  }
  return r;
}

static void plan_exec_impl(dnufft_plan *p, bool type1, int forward, int verbosity,
                           const dnufft_array *in_, dnufft_array *out_, cudaStream_t st) {
  DN_REQUIRE(p != nullptr, ST_BADARG, "null plan");
  View in = view_of(in_, type1 ? "points" : "grid");
  View out = view_of(out_, "out");
  // several transforms over the plan's points: a leading axis of ntrans on
  // both the point array (ntrans, M) and the uniform array (ntrans, N...)
  const View &pv = type1 ? in : out;
  if (pv.ndim == 2) {
    const View &uv = type1 ? out : in;
    DN_REQUIRE(uv.ndim == p->s.g.ndim + 1 && uv.shape[0] == pv.shape[0], ST_BADARG,
               "several transforms: the point array (ntrans, M) and the uniform array "
               "(ntrans, N...) must have the same leading extent");
    for (int64_t t = 0; t < pv.shape[0]; ++t)
      plan_exec_one(p, type1, forward, verbosity, slice0(in, t), slice0(out, t), st);
    return;
  }
  plan_exec_one(p, type1, forward, verbosity, in, out, st);
}

static void plan_exec_one(dnufft_plan *p, bool type1, int forward, int verbosity, const View &in,
                          const View &out, cudaStream_t st) {
  const Setup &s = p->s;
  bool f64 = s.calc_f64;
  int cdt = f64 ? DNUFFT_C128 : DNUFFT_C64;
  DN_REQUIRE(in.dtype == cdt && out.dtype == cdt, ST_BADARG,
             f64 ? "a float64-coordinate plan needs complex128 data"
                 : "a float32-coordinate plan needs complex64 data");
  const View &pv = type1 ? in : out;
  const View &uv = type1 ? out : in;
  DN_REQUIRE(pv.ndim == 1 && uint64_t(pv.shape[0]) == s.npoints, ST_BADARG,
             "number of points mismatch");
  DN_REQUIRE(uv.ndim == s.g.ndim, ST_BADARG, "uniform grid dimensions mismatch");
  for (int d = 0; d < s.g.ndim; ++d)
    DN_REQUIRE(uv.shape[d] == s.g.nuni[d], ST_BADARG, "uniform grid dimensions mismatch");
  StageTimer tm(verbosity > 0, st);
  if (verbosity > 0) report_sizes(s, type1);
  if (!p->groups.empty() && (type1 ? in.host : out.host)) {
    plan_buffers(p, st);
    if (type1) {
      if (f64) plan_nu2u_groups<double>(p, in, out, forward != 0, tm, st);
      else plan_nu2u_groups<float>(p, in, out, forward != 0, tm, st);
      tm.report("nu2u (planned, host values)");
    } else {
      if (f64) plan_u2nu_groups<double>(p, in, out, forward != 0, tm, st);
      else plan_u2nu_groups<float>(p, in, out, forward != 0, tm, st);
      tm.report("u2nu (planned, host output)");
    }
    return;
  }
  Staged si(in, true, false, st), so(out, false, true, st);
  if (s.npoints == 0) {
    if (type1) zero_view(so.dev, st);
    so.finish();
    return;
  }
  plan_buffers(p, st);
  PointsDesc pts{p->sorted_coord.p, int64_t(s.g.ndim), 1, true, s.coord_f64,
                 p->ix.perm.as<uint32_t>(), s.npoints};
  ChunkList cl{p->ix.chunks.as<Chunk>(), p->ix.nchunks};
  bool fo = p->o.fft_order != 0;
  if (type1) {
    const TcBlocks tb = p->ix.tc();
    const TcBlocks *sk = s.qbits ? &tb : nullptr;
    if (f64) do_spread_fft<double>(s, p->dc, pts, cl, sk, si.dev, so.dev, forward != 0, fo, tm, st, &p->grid, &p->work);
    else do_spread_fft<float>(s, p->dc, pts, cl, sk, si.dev, so.dev, forward != 0, fo, tm, st, &p->grid, &p->work);
    tm.report("nu2u (planned)");
  } else {
    if (f64) do_fft_interp<double>(s, p->dc, pts, cl, si.dev, so.dev, forward != 0, fo, tm, st, &p->grid, &p->work);
    else do_fft_interp<float>(s, p->dc, pts, cl, si.dev, so.dev, forward != 0, fo, tm, st, &p->grid, &p->work);
    tm.report("u2nu (planned)");
  }
  so.finish();
}

static void plan_dcoord_impl(dnufft_plan *p, int forward, const dnufft_array *grid_,
                             const dnufft_array *wts_, dnufft_array *grad_, cudaStream_t st) {
  DN_REQUIRE(p != nullptr, ST_BADARG, "null plan");
  const Setup &s = p->s;
  bool f64 = s.calc_f64;
  int cdt = f64 ? DNUFFT_C128 : DNUFFT_C64;
  View uni = view_of(grid_, "grid"), wts = view_of(wts_, "weights"), grad = view_of(grad_, "grad");
  DN_REQUIRE(uni.dtype == cdt, ST_BADARG,
             f64 ? "a float64-coordinate plan needs complex128 data"
                 : "a float32-coordinate plan needs complex64 data");
  DN_REQUIRE(uni.ndim == s.g.ndim, ST_BADARG, "uniform grid dimensions mismatch");
  for (int d = 0; d < s.g.ndim; ++d)
    DN_REQUIRE(uni.shape[d] == s.g.nuni[d], ST_BADARG, "uniform grid dimensions mismatch");
  check_dcoord_args(wts, grad, cdt, s.coord_f64 ? DNUFFT_F64 : DNUFFT_F32, s.npoints, s.g.ndim);
  if (s.npoints == 0) return;
  StageTimer tm(false, st);
  Staged su(uni, true, false, st), sw(wts, true, false, st), sg(grad, false, true, st);
  if (!p->grid.p) {
    p->grid = DevBuf(grid_cells(s.g) * (f64 ? 16 : 8), st);
    const size_t wb = fft_work_bytes(s.g, f64 ? 16 : 8);
    if (wb) p->work = DevBuf(wb, st);
    DN_CUDA(cudaStreamSynchronize(st));
  }
  PointsDesc pts{p->sorted_coord.p, int64_t(s.g.ndim), 1, true, s.coord_f64,
                 p->ix.perm.as<uint32_t>(), s.npoints};
  ChunkList cl{p->ix.chunks.as<Chunk>(), p->ix.nchunks};
  bool fo = p->o.fft_order != 0;
  if (f64) do_fft_dcoord<double>(s, p->dc, pts, cl, su.dev, sw.dev, sg.dev, forward != 0, fo, tm, st, &p->grid, &p->work);
  else do_fft_dcoord<float>(s, p->dc, pts, cl, su.dev, sw.dev, sg.dev, forward != 0, fo, tm, st, &p->grid, &p->work);
  tm.report("u2nu_dcoord (planned)");
  sg.finish();
}

// ---------------------------------------------------------------- split type 1
// A type-1 transform whose points are split over several GPUs (one process
// each): every rank spreads its own points into a full oversampled grid
// (plan_spread), the caller sums the grids over the ranks (one all-reduce),
// and the sum goes through the FFT and the correction (plan_grid_to_uniform).
// Spreading is linear in the values, so the summed grid is the grid of all
// points.  The oversampled grid is a C-contiguous device array of the plan's
// data type and oversampled shape.
static View over_grid_view(const dnufft_plan *p, const dnufft_array *grid_) {
  const Setup &s = p->s;
  View g = view_of(grid_, "grid");
  DN_REQUIRE(!g.host, ST_BADARG, "the oversampled grid must be a device array");
  DN_REQUIRE(g.dtype == (s.calc_f64 ? DNUFFT_C128 : DNUFFT_C64), ST_BADARG,
             "the oversampled grid must have the plan's data type");
  DN_REQUIRE(g.ndim == s.g.ndim, ST_BADARG, "oversampled grid dimensions mismatch");
  int64_t cs = 1;
  for (int d = s.g.ndim - 1; d >= 0; --d) {
    DN_REQUIRE(g.shape[d] == int64_t(s.g.nover[d]), ST_BADARG,
               "the oversampled grid must have the plan's oversampled sizes");
    DN_REQUIRE(g.stride[d] == cs, ST_BADARG, "the oversampled grid must be C-contiguous");
    cs *= g.shape[d];
  }
  return g;
}

static void plan_spread_impl(dnufft_plan *p, const dnufft_array *points_, dnufft_array *grid_,
                             cudaStream_t st) {
  DN_REQUIRE(p != nullptr, ST_BADARG, "null plan");
  const Setup &s = p->s;
  const bool f64 = s.calc_f64;
  View points = view_of(points_, "points");
  DN_REQUIRE(points.dtype == (f64 ? DNUFFT_C128 : DNUFFT_C64), ST_BADARG,
             f64 ? "a float64-coordinate plan needs complex128 data"
                 : "a float32-coordinate plan needs complex64 data");
  DN_REQUIRE(points.ndim == 1 && uint64_t(points.shape[0]) == s.npoints, ST_BADARG,
             "number of points mismatch");
  const View grid = over_grid_view(p, grid_);
  DN_CUDA(cudaMemsetAsync(grid.data, 0, grid_cells(s.g) * (f64 ? 16 : 8), st));
  if (s.npoints > 0) {
    Staged sp(points, true, false, st);
    PointsDesc pts{p->sorted_coord.p, int64_t(s.g.ndim), 1, true, s.coord_f64,
                   p->ix.perm.as<uint32_t>(), s.npoints};
    ChunkList cl{p->ix.chunks.as<Chunk>(), p->ix.nchunks};
    const TcBlocks tb = p->ix.tc();
    const TcBlocks *sk = s.qbits ? &tb : nullptr;
    int *err = device_error_word();
    if (f64) spread_points<double>(s, pts, cl, sk, sp.dev.data, sp.dev.stride[0], grid.data, err, st);
    else spread_points<float>(s, pts, cl, sk, sp.dev.data, sp.dev.stride[0], grid.data, err, st);
    check_device_error(err, st);
  }
}

static void plan_grid_to_uniform_impl(dnufft_plan *p, int forward, dnufft_array *grid_,
                                      dnufft_array *out_, cudaStream_t st) {
  DN_REQUIRE(p != nullptr, ST_BADARG, "null plan");
  const Setup &s = p->s;
  const bool f64 = s.calc_f64;
  const View grid = over_grid_view(p, grid_);
  View out = view_of(out_, "out");
  DN_REQUIRE(out.dtype == grid.dtype, ST_BADARG, "out must have the plan's data type");
  DN_REQUIRE(out.ndim == s.g.ndim, ST_BADARG, "uniform grid dimensions mismatch");
  for (int d = 0; d < s.g.ndim; ++d)
    DN_REQUIRE(out.shape[d] == s.g.nuni[d], ST_BADARG, "uniform grid dimensions mismatch");
  Staged so(out, false, true, st);
  const size_t wb = fft_work_bytes(s.g, f64 ? 16 : 8);
  if (wb && !p->work.p) {
    p->work = DevBuf(wb, st);
    DN_CUDA(cudaStreamSynchronize(st));
  }
  int *err = device_error_word();
  const bool fo = p->o.fft_order != 0;
  if (f64)
    fft_nu2u_tail<double>(grid.data, s.g, p->dc.ax, forward != 0, p->dc.cf, fo, so.dev.data,
                          so.dev.stride, st, p->work.p, err);
  else
    fft_nu2u_tail<float>(grid.data, s.g, p->dc.ax, forward != 0, p->dc.cf, fo, so.dev.data,
                         so.dev.stride, st, p->work.p, err);
  check_device_error(err, st);
  so.finish();
}

// The 2D type-1 FFT in two halves, for the exchange in which every rank sums
// one slab of rows of the spread grids (a reduce-scatter), transforms those
// rows, and the ranks gather the kept columns for the column pass.
static View rows_view(const dnufft_plan *p, const dnufft_array *rows_) {
  const Setup &s = p->s;
  DN_REQUIRE(s.g.ndim == 2, ST_UNSUPPORTED, "row and column halves: 2D plans only");
  View r = view_of(rows_, "rows");
  DN_REQUIRE(!r.host, ST_BADARG, "the rows must be a device array");
  DN_REQUIRE(r.dtype == (s.calc_f64 ? DNUFFT_C128 : DNUFFT_C64), ST_BADARG,
             "the rows must have the plan's data type");
  DN_REQUIRE(r.ndim == 2 && r.shape[1] == int64_t(s.g.nover[1]) &&
                 r.shape[0] <= int64_t(s.g.nover[0]),
             ST_BADARG, "rows: (at most nover[0], nover[1]) cells expected");
  DN_REQUIRE(r.shape[0] <= 1 || r.stride[0] == r.shape[1], ST_BADARG,
             "the rows must be C-contiguous");
  DN_REQUIRE(r.stride[1] == 1, ST_BADARG, "the rows must be C-contiguous");
  return r;
}

static void plan_rows_fft_impl(dnufft_plan *p, int forward, dnufft_array *rows_, cudaStream_t st) {
  DN_REQUIRE(p != nullptr, ST_BADARG, "null plan");
  const View r = rows_view(p, rows_);
  if (r.shape[0] == 0) return;
  int *err = device_error_word();
  if (p->s.calc_f64)
    fft_nu2u_rows<double>(r.data, int(r.shape[0]), p->s.g, p->dc.ax, forward != 0, st, err);
  else
    fft_nu2u_rows<float>(r.data, int(r.shape[0]), p->s.g, p->dc.ax, forward != 0, st, err);
  check_device_error(err, st);
}

static void plan_rows_fft_kept_in_impl(dnufft_plan *p, int forward, dnufft_array *rows_,
                                       cudaStream_t st) {
  DN_REQUIRE(p != nullptr, ST_BADARG, "null plan");
  const View r = rows_view(p, rows_);
  if (r.shape[0] == 0) return;
  int *err = device_error_word();
  if (p->s.calc_f64)
    fft_u2nu_rows<double>(r.data, int(r.shape[0]), p->s.g, p->dc.ax, forward != 0, st, err);
  else
    fft_u2nu_rows<float>(r.data, int(r.shape[0]), p->s.g, p->dc.ax, forward != 0, st, err);
  check_device_error(err, st);
}

static void plan_uniform_to_cols_impl(dnufft_plan *p, int forward, const dnufft_array *uni_,
                                      int64_t col0, dnufft_array *cols_, cudaStream_t st) {
  DN_REQUIRE(p != nullptr, ST_BADARG, "null plan");
  const Setup &s = p->s;
  DN_REQUIRE(s.g.ndim == 2, ST_UNSUPPORTED, "row and column halves: 2D plans only");
  const bool f64 = s.calc_f64;
  const int dt = f64 ? DNUFFT_C128 : DNUFFT_C64;
  View uni = view_of(uni_, "grid"), cols = view_of(cols_, "cols");
  DN_REQUIRE(!uni.host && !cols.host, ST_BADARG, "column blocks: device arrays only");
  DN_REQUIRE(uni.dtype == dt && cols.dtype == dt, ST_BADARG,
             "column blocks must have the plan's data type");
  DN_REQUIRE(uni.ndim == 2 && uni.shape[0] == s.g.nuni[0] && uni.shape[1] == s.g.nuni[1],
             ST_BADARG, "uniform grid dimensions mismatch");
  DN_REQUIRE(cols.ndim == 2 && cols.shape[0] == s.g.nover[0], ST_BADARG,
             "cols must be (nover[0], ncols)");
  const int64_t nc = cols.shape[1];
  DN_REQUIRE(nc >= 1 && col0 >= 0 && col0 + nc <= s.g.nuni[1], ST_BADARG,
             "column block outside the kept columns");
  DN_REQUIRE(cols.stride[1] == 1 && cols.stride[0] == nc, ST_BADARG,
             "cols must be C-contiguous");
  const size_t wb = fft_work_bytes(s.g, f64 ? 16 : 8);
  if (wb && !p->work.p) {
    p->work = DevBuf(wb, st);
    DN_CUDA(cudaStreamSynchronize(st));
  }
  const bool fo = p->o.fft_order != 0;
  const bool ok =
      f64 ? fft_u2nu_cols_range<double>(uni.data, uni.stride, s.g, p->dc.ax, forward != 0,
                                        p->dc.cf, fo, cols.data, int(nc), int(col0), st,
                                        p->work.p)
          : fft_u2nu_cols_range<float>(uni.data, uni.stride, s.g, p->dc.ax, forward != 0,
                                       p->dc.cf, fo, cols.data, int(nc), int(col0), st,
                                       p->work.p);
  DN_REQUIRE(ok, ST_UNSUPPORTED,
             "column blocks need the four-step column passes (oversampled rows >= 1024)");
}

static void plan_interp_impl(dnufft_plan *p, const dnufft_array *grid_, dnufft_array *out_,
                             cudaStream_t st) {
  DN_REQUIRE(p != nullptr, ST_BADARG, "null plan");
  const Setup &s = p->s;
  View grid = over_grid_view(p, grid_);
  View out = view_of(out_, "out");
  DN_REQUIRE(!out.host, ST_BADARG, "out must be a device array");
  DN_REQUIRE(out.dtype == grid.dtype, ST_BADARG, "out must have the plan's data type");
  DN_REQUIRE(out.ndim == 1 && uint64_t(out.shape[0]) == s.npoints, ST_BADARG,
             "number of points mismatch");
  if (s.npoints == 0) return;
  PointsDesc pts{p->sorted_coord.p, int64_t(s.g.ndim), 1, true, s.coord_f64,
                 p->ix.perm.as<uint32_t>(), s.npoints};
  ChunkList cl{p->ix.chunks.as<Chunk>(), p->ix.nchunks};
  if (s.calc_f64)
    launch_interp<double>(pts, cl, s.g, s.kpd, grid.data, 0, out.data, out.stride[0], 0, 1, st);
  else
    launch_interp<float>(pts, cl, s.g, s.kpf, grid.data, 0, out.data, out.stride[0], 0, 1, st);
}

static void plan_cols_to_uniform_impl(dnufft_plan *p, int forward, dnufft_array *grid_,
                                      dnufft_array *out_, cudaStream_t st) {
  DN_REQUIRE(p != nullptr, ST_BADARG, "null plan");
  const Setup &s = p->s;
  DN_REQUIRE(s.g.ndim == 2, ST_UNSUPPORTED, "row and column halves: 2D plans only");
  const bool f64 = s.calc_f64;
  // the whole oversampled grid, or its kept columns packed ((n0, N1): the
  // column pass then sees a grid of row length N1, whose kept columns are all
  // of its columns, with the same output and correction indices)
  Geometry gc = s.g;
  View grid = view_of(grid_, "grid");
  if (grid.ndim == 2 && grid.shape[0] == int64_t(s.g.nover[0]) &&
      grid.shape[1] == int64_t(s.g.nuni[1]) && s.g.nuni[1] != s.g.nover[1]) {
    DN_REQUIRE(!grid.host, ST_BADARG, "the oversampled grid must be a device array");
    DN_REQUIRE(grid.dtype == (f64 ? DNUFFT_C128 : DNUFFT_C64), ST_BADARG,
               "the oversampled grid must have the plan's data type");
    DN_REQUIRE(grid.stride[1] == 1 && grid.stride[0] == grid.shape[1], ST_BADARG,
               "the oversampled grid must be C-contiguous");
    gc.nover[1] = s.g.nuni[1];
  } else {
    grid = over_grid_view(p, grid_);
  }
  View out = view_of(out_, "out");
  DN_REQUIRE(out.dtype == grid.dtype, ST_BADARG, "out must have the plan's data type");
  DN_REQUIRE(out.ndim == 2 && out.shape[0] == s.g.nuni[0] && out.shape[1] == s.g.nuni[1],
             ST_BADARG, "uniform grid dimensions mismatch");
  Staged so(out, false, true, st);
  const size_t wb = fft_work_bytes(s.g, f64 ? 16 : 8);
  if (wb && !p->work.p) {
    p->work = DevBuf(wb, st);
    DN_CUDA(cudaStreamSynchronize(st));
  }
  const bool fo = p->o.fft_order != 0;
  if (f64)
    fft_nu2u_cols<double>(grid.data, gc, p->dc.ax, forward != 0, p->dc.cf, fo, so.dev.data,
                          so.dev.stride, st, p->work.p);
  else
    fft_nu2u_cols<float>(grid.data, gc, p->dc.ax, forward != 0, p->dc.cf, fo, so.dev.data,
                         so.dev.stride, st, p->work.p);
  so.finish();
}

static void plan_cols_range_impl(dnufft_plan *p, int forward, dnufft_array *cols_, int64_t col0,
                                 dnufft_array *out_, cudaStream_t st) {
  DN_REQUIRE(p != nullptr, ST_BADARG, "null plan");
  const Setup &s = p->s;
  DN_REQUIRE(s.g.ndim == 2, ST_UNSUPPORTED, "row and column halves: 2D plans only");
  const bool f64 = s.calc_f64;
  const int dt = f64 ? DNUFFT_C128 : DNUFFT_C64;
  View cols = view_of(cols_, "cols"), out = view_of(out_, "out");
  DN_REQUIRE(!cols.host && !out.host, ST_BADARG, "column blocks: device arrays only");
  DN_REQUIRE(cols.dtype == dt && out.dtype == dt, ST_BADARG,
             "column blocks must have the plan's data type");
  DN_REQUIRE(cols.ndim == 2 && cols.shape[0] == s.g.nover[0], ST_BADARG,
             "cols must be (nover[0], ncols)");
  const int64_t nc = cols.shape[1];
  DN_REQUIRE(nc >= 1 && col0 >= 0 && col0 + nc <= s.g.nuni[1], ST_BADARG,
             "column block outside the kept columns");
  DN_REQUIRE(cols.stride[1] == 1 && cols.stride[0] == nc, ST_BADARG,
             "cols must be C-contiguous");
  DN_REQUIRE(out.ndim == 2 && out.shape[0] == s.g.nuni[0] && out.shape[1] == nc, ST_BADARG,
             "out must be (nuni[0], ncols)");
  const size_t wb = fft_work_bytes(s.g, f64 ? 16 : 8);
  if (wb && !p->work.p) {
    p->work = DevBuf(wb, st);
    DN_CUDA(cudaStreamSynchronize(st));
  }
  const bool fo = p->o.fft_order != 0;
  const bool ok =
      f64 ? fft_nu2u_cols_range<double>(cols.data, int(nc), int(col0), s.g, p->dc.ax,
                                        forward != 0, p->dc.cf, fo, out.data, out.stride, st,
                                        p->work.p)
          : fft_nu2u_cols_range<float>(cols.data, int(nc), int(col0), s.g, p->dc.ax,
                                       forward != 0, p->dc.cf, fo, out.data, out.stride, st,
                                       p->work.p);
  DN_REQUIRE(ok, ST_UNSUPPORTED,
             "column blocks need the four-step column passes (oversampled rows >= 1024)");
}

static void find_parameters_impl(int nu2u, int ndim, const int64_t *shape, uint64_t npoints,
                                 double eps, int calc_f64, int coord_f64, const dnufft_opts *opts_,
                                 int32_t *kidx, int64_t *nover) {
  DN_REQUIRE(shape != nullptr && kidx != nullptr && nover != nullptr, ST_BADARG,
             "null argument");
  DN_REQUIRE(ndim >= 1 && ndim <= 3, ST_BADARG, "unsupported dimensionality");
  const dnufft_opts o = resolved(opts_, true);
  const Setup s = make_setup(ndim, shape, npoints, eps, nu2u != 0, calc_f64 != 0, coord_f64 != 0, o);
  *kidx = s.kidx;
  for (int d = 0; d < 3; ++d) nover[d] = d < ndim ? int64_t(s.g.nover[d]) : 1;
}

// ---------------------------------------------------------------- scratch-only type 1
// A type-1 transform whose every temporary (correction factors, twiddles,
// tile keys and permutation, sort / chunk workspaces, chunk list, oversampled
// grid) is carved from a device region the caller owns, so nothing is
// allocated.  Device arrays only; the plain spreader.
struct Carver {
  char *base;
  size_t cap, used = 0;
  Carver(void *b, size_t c) : base(static_cast<char *>(b)), cap(c) {}
  void *take(size_t bytes) {
    size_t off = (used + 255) & ~size_t(255);
    if (off + bytes > cap) return nullptr;
    used = off + bytes;
    return base + off;
  }
};

template <typename T>
static void nu2u_scratch_typed(const Setup &s, const View &points, const View &coord,
                               const View &out, bool forward, bool fft_order, void *scratch,
                               size_t cap, cudaStream_t st) {
  const Geometry &g = s.g;
  const uint32_t M = s.npoints;
  const size_t csz = sizeof(T) * 2;
  uint64_t maxchunks = std::min<uint64_t>(M, s.max_tiles) + M / s.chunk + 2;
  Carver cv(scratch, cap);
  double *cf[3] = {nullptr, nullptr, nullptr};
  void *tw[3] = {nullptr, nullptr, nullptr};
  for (int d = 0; d < g.ndim; ++d) {
    cf[d] = static_cast<double *>(cv.take(s.corfac[d].size() * sizeof(double)));
    tw[d] = cv.take(size_t(g.nover[d]) * csz);
  }
  uint32_t *keys = static_cast<uint32_t *>(cv.take(size_t(M) * 4));
  uint32_t *perm = static_cast<uint32_t *>(cv.take(size_t(M) * 4));
  void *rws = cv.take(radix_workspace_bytes(M, s.keybits));
  void *cws = cv.take(chunk_workspace_bytes(M));
  Chunk *chunks = static_cast<Chunk *>(cv.take(size_t(maxchunks) * sizeof(Chunk)));
  uint32_t *count = static_cast<uint32_t *>(cv.take(16));
  void *grid = cv.take(grid_cells(g) * csz);
  bool fits = grid != nullptr;
  for (int d = 0; d < g.ndim; ++d) fits = fits && cf[d] && tw[d];
  fits = fits && keys && perm && rws && cws && chunks && count;
  if (!fits) {
    // measure what would have been needed for the message
    Carver probe(nullptr, ~size_t(0));
    for (int d = 0; d < g.ndim; ++d) {
      probe.take(s.corfac[d].size() * sizeof(double));
      probe.take(size_t(g.nover[d]) * csz);
    }
    probe.take(size_t(M) * 4);
    probe.take(size_t(M) * 4);
    probe.take(radix_workspace_bytes(M, s.keybits));
    probe.take(chunk_workspace_bytes(M));
    probe.take(size_t(maxchunks) * sizeof(Chunk));
    probe.take(16);
    probe.take(grid_cells(g) * csz);
    throw Error(ST_BADARG, "problem needs " + std::to_string(probe.used) +
                               " bytes of scratch, more than the " + std::to_string(cap) +
                               " bytes of the no-allocation scratch area");
  }
  // constants: correction factors and FP64-accurate twiddles
  FFTAxisPlan ax[3];
  std::vector<std::vector<double>> hd(g.ndim);
  std::vector<std::vector<float>> hf(g.ndim);
  for (int d = 0; d < g.ndim; ++d) {
    DN_CUDA(cudaMemcpyAsync(cf[d], s.corfac[d].data(), s.corfac[d].size() * sizeof(double),
                            cudaMemcpyHostToDevice, st));
    const int n = int(g.nover[d]);
    if (sizeof(T) == 8) {
      hd[d].resize(2 * size_t(n));
      for (int k = 0; k < n; ++k) {
        double a = -2.0 * M_PI * double(k) / double(n);
        hd[d][2 * k] = std::cos(a);
        hd[d][2 * k + 1] = std::sin(a);
      }
      DN_CUDA(cudaMemcpyAsync(tw[d], hd[d].data(), hd[d].size() * 8, cudaMemcpyHostToDevice, st));
    } else {
      hf[d].resize(2 * size_t(n));
      for (int k = 0; k < n; ++k) {
        double a = -2.0 * M_PI * double(k) / double(n);
        hf[d][2 * k] = float(std::cos(a));
        hf[d][2 * k + 1] = float(std::sin(a));
      }
      DN_CUDA(cudaMemcpyAsync(tw[d], hf[d].data(), hf[d].size() * 4, cudaMemcpyHostToDevice, st));
    }
    ax[d].n = n;
    ax[d].nfac = int(s.factors[d].size());
    for (int i = 0; i < ax[d].nfac; ++i) ax[d].fac[i] = s.factors[d][i];
    ax[d].tw = tw[d];
  }
  // index: fold + stable sort + chunks (the chunk count read-back synchronises
  // the stream, after which the host constant buffers may be released)
  launch_fold_keys(s.coord_f64, coord.data, coord.stride[0], coord.stride[1], M, g, keys, perm, st);
  radix_sort_pairs(keys, perm, M, s.keybits, rws, st);
  uint32_t nch = build_chunks(keys, M, s.tile_shift, s.chunk, chunks, count, cws, st,
                              /*zero_copy=*/false);
  PointsDesc pts{coord.data, coord.stride[0], coord.stride[1], false, s.coord_f64, perm, M};
  ChunkList cl{chunks, nch};
  // the scratch keeps the previous call's contents: the grid must start at zero
  DN_CUDA(cudaMemsetAsync(grid, 0, grid_cells(g) * csz, st));
  const KernelPoly<T> &kp = *reinterpret_cast<const KernelPoly<T> *>(
      sizeof(T) == 4 ? static_cast<const void *>(&s.kpf) : static_cast<const void *>(&s.kpd));
  launch_spread<T>(pts, cl, g, kp, points.data, points.stride[0], 0, grid, 0, 1, st);
  const double *cfc[3] = {cf[0], cf[1], cf[2]};
  fft_nu2u_tail<T>(grid, g, ax, forward, cfc, fft_order, out.data, out.stride, st);
}

static void nu2u_scratch_impl(const dnufft_array *points_, const dnufft_array *coord_, int forward,
                              double eps, dnufft_array *out_, const dnufft_opts *opts_,
                              cudaStream_t st, void *scratch, size_t cap) {
  dnufft_opts o = resolved(opts_, false);
  DN_REQUIRE(o.spreader != DNUFFT_SPREAD_TC, ST_UNSUPPORTED,
             "the no-allocation entry point uses the plain spreader only");
  // plain keys and chunks below (no tensor-core quadrant bits): 'auto' must
  // not resolve to the tensor-core setup here
  o.spreader = DNUFFT_SPREAD_PLAIN;
  View points = view_of(points_, "points"), coord = view_of(coord_, "coord"),
       out = view_of(out_, "out");
  DN_REQUIRE(!points.host && !coord.host && !out.host, ST_BADARG,
             "the no-allocation entry point needs device arrays");
  int ndim = out.ndim;
  DN_REQUIRE(ndim >= 1 && ndim <= 3, ST_BADARG, "transform must be 1D/2D/3D");
  check_coord(coord, ndim);
  DN_REQUIRE(points.ndim == 1, ST_BADARG, "points must be 1D");
  DN_REQUIRE(points.shape[0] == coord.shape[0], ST_BADARG, "number of points mismatch");
  DN_REQUIRE(points.dtype == DNUFFT_C64 || points.dtype == DNUFFT_C128, ST_BADARG,
             "points must be complex64 or complex128");
  DN_REQUIRE(out.dtype == points.dtype, ST_BADARG, "out must have the dtype of points");
  bool f64 = points.dtype == DNUFFT_C128;
  Setup s = make_setup(ndim, out.shape, uint64_t(points.shape[0]), eps, true, f64,
                       coord.dtype == DNUFFT_F64, o);
  if (s.npoints == 0) {
    zero_view(out, st);
    return;
  }
  if (f64)
    nu2u_scratch_typed<double>(s, points, coord, out, forward != 0, o.fft_order != 0, scratch, cap,
                               st);
  else
    nu2u_scratch_typed<float>(s, points, coord, out, forward != 0, o.fft_order != 0, scratch, cap,
                              st);
}

int nu2u_in_scratch(const dnufft_array *points, const dnufft_array *coord, int forward,
                    double epsilon, dnufft_array *out, const dnufft_opts *opts, void *stream,
                    void *scratch, size_t scratch_bytes) {
  try {
    nu2u_scratch_impl(points, coord, forward, epsilon, out, opts, static_cast<cudaStream_t>(stream),
                      scratch, scratch_bytes);
    g_last_error.clear();
    return DNUFFT_OK;
  } catch (const Error &e) {
    g_last_error = e.what();
    return e.code;
  } catch (const std::exception &e) {
    g_last_error = e.what();
    return DNUFFT_ERR_INTERNAL;
  }
}

// ---------------------------------------------------------------- grouped index
// A 2D index over points that belong to groups (the w-gridder's first w
// plane): sorted once by (tile, group), so that within every tile the points
// of any run of groups are one contiguous range, and a type 1 or type 2
// transform over such a run needs only a chunk list (one chunk per tile and
// at most CHUNK points, so a tile is still flushed once), not a sort of its
// own.  Plain spreader; kernel and grid as forced in the options.
struct GroupedPlan {
  Setup s;
  DevConst dcl;
  const DevConst *dc = nullptr;
  DevBuf sorted_coord, perm, start, chunks, cws, grid, work;
  uint32_t ntiles = 0, ngroups = 0, nchunks = 0, g0 = 0, g1 = 0;
  int gbits = 0;
};

static int bits_for(uint64_t v) {   // bits to hold 0..v
  int b = 0;
  while (b < 64 && (uint64_t(1) << b) <= v) ++b;
  return b;
}

GroupedPlan *grouped_plan_create(const double *coord, uint32_t M, const uint32_t *group,
                                 uint32_t ngroups, const int64_t *shape, double eps,
                                 bool calc_f64, const dnufft_opts &opts, cudaStream_t st,
                                 uint32_t *perm_out) {
  dnufft_opts o = opts;
  o.spreader = DNUFFT_SPREAD_PLAIN;
  auto gp = std::make_unique<GroupedPlan>();
  gp->s = make_setup(2, shape, M, eps, true, calc_f64, true, o);
  Setup &s = gp->s;
  DN_REQUIRE(!s.qbits, ST_INTERNAL, "grouped index with a tensor-core key");
  const int tilebits = s.keybits;
  gp->gbits = bits_for(ngroups);
  // keys (tile << gbits | group) in 32 bits, and a start table of
  // ntiles * 2^gbits + 1 entries of at most 512 MB
  const uint64_t ntiles = uint64_t(s.g.ntiles[0]) * uint64_t(s.g.ntiles[1]);
  if (tilebits + gp->gbits > 32 || (ntiles << gp->gbits) > (uint64_t(1) << 27) || M == 0 ||
      ngroups == 0)
    return nullptr;
  gp->ngroups = ngroups;
  gp->ntiles = uint32_t(ntiles);
  gp->dc = &consts_for(s, gp->dcl, st);
  DevBuf keys(size_t(M) * 4, st);
  gp->perm = DevBuf(size_t(M) * 4, st);
  launch_fold_keys(true, coord, 2, 1, M, s.g, keys.as<uint32_t>(), gp->perm.as<uint32_t>(), st,
                   false);
  launch_group_keys(keys.as<uint32_t>(), group, M, gp->gbits, st);
  const int total = tilebits + gp->gbits;
  {
    DevBuf ws(radix_workspace_bytes(M, total), st);
    radix_sort_pairs(keys.as<uint32_t>(), gp->perm.as<uint32_t>(), M, total, ws.p, st);
  }
  const uint32_t nkeys = gp->ntiles << gp->gbits;
  gp->start = DevBuf(size_t(nkeys + 1) * 4, st);
  launch_key_starts(keys.as<uint32_t>(), M, nkeys, gp->start.as<uint32_t>(), st);
  gp->sorted_coord = DevBuf(size_t(M) * 16, st);
  launch_gather_coords(true, coord, 2, 1, 2, gp->perm.as<uint32_t>(), M, gp->sorted_coord.p, st);
  gp->chunks = DevBuf((size_t(gp->ntiles) + M / s.chunk + 2) * sizeof(Chunk), st);
  gp->cws = DevBuf(group_chunk_workspace_bytes(gp->ntiles), st);
  if (perm_out)
    DN_CUDA(cudaMemcpyAsync(perm_out, gp->perm.p, size_t(M) * 4, cudaMemcpyDeviceToDevice, st));
  const size_t vb = calc_f64 ? 16 : 8;
  gp->grid = DevBuf(grid_cells(s.g) * vb, st);
  const size_t wb = fft_work_bytes(s.g, vb);
  if (wb) gp->work = DevBuf(wb, st);
  DN_CUDA(cudaStreamSynchronize(st));
  return gp.release();
}

void grouped_plan_destroy(GroupedPlan *gp, cudaStream_t st) {
  if (!gp) return;
  // buffers go back to the pool in the order of the stream that last used them
  for (DevBuf *b : {&gp->sorted_coord, &gp->perm, &gp->start, &gp->chunks, &gp->cws, &gp->grid,
                    &gp->work})
    b->st = st;
  delete gp;
}

const uint32_t *grouped_plan_perm(const GroupedPlan *gp) { return gp->perm.as<uint32_t>(); }

// chunk list of groups [g0, g1), kept for the next call with the same run;
// false: no point in the run
static bool grouped_chunks(GroupedPlan *gp, uint32_t g0, uint32_t g1, cudaStream_t st) {
  if (gp->g1 == 0 || gp->g0 != g0 || gp->g1 != g1) {
    gp->nchunks = build_group_chunks(gp->start.as<uint32_t>(), gp->ntiles, gp->gbits, g0, g1,
                                     gp->s.chunk, gp->chunks.as<Chunk>(), gp->cws.p, st);
    gp->g0 = g0;
    gp->g1 = g1;
  }
  return gp->nchunks > 0;
}

static View plain_view(void *data, int dtype, int ndim, int64_t s0, int64_t s1 = 0) {
  View v;
  std::memset(&v, 0, sizeof(v));
  v.data = data;
  v.dtype = dtype;
  v.ndim = ndim;
  v.shape[0] = s0;
  v.shape[1] = s1;
  v.stride[0] = ndim == 1 ? 1 : s1;
  v.stride[1] = 1;
  v.host = false;
  return v;
}

// type 1 over the points of groups [g0, g1): values in the caller's order
// (index = position before sorting), result into out (N0 x N1, contiguous);
// false (nothing written) where the run has no point
bool grouped_nu2u(GroupedPlan *gp, uint32_t g0, uint32_t g1, const void *values, void *out,
                  bool forward, cudaStream_t st) {
  const Setup &s = gp->s;
  if (!grouped_chunks(gp, g0, g1, st)) return false;
  const ChunkList cl{gp->chunks.as<Chunk>(), gp->nchunks};
  const PointsDesc pts{gp->sorted_coord.p, 2, 1, true, true, gp->perm.as<uint32_t>(),
                       s.npoints};
  const int dt = s.calc_f64 ? DNUFFT_C128 : DNUFFT_C64;
  const View vv = plain_view(const_cast<void *>(values), dt, 1, s.npoints);
  const View ov = plain_view(out, dt, 2, s.g.nuni[0], s.g.nuni[1]);
  StageTimer tm(false, st);
  if (s.calc_f64)
    do_spread_fft<double>(s, *gp->dc, pts, cl, nullptr, vv, ov, forward, false, tm, st,
                          &gp->grid, &gp->work);
  else
    do_spread_fft<float>(s, *gp->dc, pts, cl, nullptr, vv, ov, forward, false, tm, st,
                         &gp->grid, &gp->work);
  return true;
}

// type 2 at the points of groups [g0, g1): results into out at the caller's
// positions (other entries untouched); false where the run has no point
bool grouped_u2nu(GroupedPlan *gp, uint32_t g0, uint32_t g1, const void *uni, void *out,
                  bool forward, cudaStream_t st) {
  const Setup &s = gp->s;
  if (!grouped_chunks(gp, g0, g1, st)) return false;
  const ChunkList cl{gp->chunks.as<Chunk>(), gp->nchunks};
  const PointsDesc pts{gp->sorted_coord.p, 2, 1, true, true, gp->perm.as<uint32_t>(),
                       s.npoints};
  const int dt = s.calc_f64 ? DNUFFT_C128 : DNUFFT_C64;
  const View uv = plain_view(const_cast<void *>(uni), dt, 2, s.g.nuni[0], s.g.nuni[1]);
  const View ov = plain_view(out, dt, 1, s.npoints);
  StageTimer tm(false, st);
  if (s.calc_f64)
    do_fft_interp<double>(s, *gp->dc, pts, cl, uv, ov, forward, false, tm, st, &gp->grid,
                          &gp->work);
  else
    do_fft_interp<float>(s, *gp->dc, pts, cl, uv, ov, forward, false, tm, st, &gp->grid,
                         &gp->work);
  return true;
}

void set_last_error(const char *msg) { g_last_error = msg; }

}  // namespace dnufft

// ---------------------------------------------------------------- C-ABI
#define DN_GUARD(body)                                   \
  try {                                                  \
    body;                                                \
    g_last_error.clear();                                \
    return DNUFFT_OK;                                    \
  } catch (const dnufft::Error &e) {                     \
    g_last_error = e.what();                             \
    return e.code;                                       \
  } catch (const std::bad_alloc &) {                     \
    g_last_error = "host allocation failed";             \
    return DNUFFT_ERR_OOM;                               \
  } catch (const std::exception &e) {                    \
    g_last_error = e.what();                             \
    return DNUFFT_ERR_INTERNAL;                          \
  }

extern "C" {

void dnufft_default_opts(dnufft_opts *o, int for_plan) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->nthreads = for_plan ? 0 : 1;
  o->sigma_min = for_plan ? 1.1 : 1.2;
  o->sigma_max = for_plan ? 2.6 : 2.51;
  for (int d = 0; d < 3; ++d) o->periodicity[d] = 2 * M_PI;
  o->fft_order = 0;
  o->verbosity = 0;
  o->spreader = DNUFFT_SPREAD_AUTO;
  o->simd_lanes = 8;
  o->force_kernel = -1;
}

int dnufft_best_epsilon(size_t ndim, int singleprec, double sigma_min, double sigma_max,
                        double *out) {
  DN_GUARD({
    DN_REQUIRE(out != nullptr, dnufft::ST_BADARG, "null output");
    *out = dnufft::best_epsilon(ndim, singleprec != 0, sigma_min, sigma_max);
  })
}

int dnufft_kernel_candidates(int ndim, const int64_t *shape, int singleprec, double epsilon,
                             double sigma_min, double sigma_max, int max, int32_t *kernel_index,
                             int32_t *supp, double *ofactor, int64_t *nover, int *count) {
  DN_GUARD({
    DN_REQUIRE(ndim >= 1 && ndim <= 3 && shape && count && max >= 0, dnufft::ST_BADARG,
               "bad arguments");
    auto idx = dnufft::available_kernels(epsilon, size_t(ndim), singleprec != 0, sigma_min,
                                         sigma_max);
    int c = 0;
    for (size_t i : idx) {
      if (c >= max) break;
      const auto &k = dnufft::kernel_db()[i];
      if (kernel_index) kernel_index[c] = int32_t(i);
      if (supp) supp[c] = k.W;
      if (ofactor) ofactor[c] = k.ofactor;
      if (nover)
        for (int d = 0; d < 3; ++d)
          nover[3 * c + d] =
              d < ndim ? int64_t(std::max<size_t>(
                             2 * dnufft::good_size_complex(size_t(double(shape[d]) * k.ofactor * 0.5) + 1),
                             16))
                       : 1;
      ++c;
    }
    *count = c;
  })
}

int dnufft_nu2u(const dnufft_array *points, const dnufft_array *coord, int forward, double epsilon,
                dnufft_array *out, const dnufft_opts *opts, void *stream) {
  DN_GUARD(dnufft::nu2u_impl(points, coord, forward, epsilon, out, opts,
                             static_cast<cudaStream_t>(stream)))
}

int dnufft_u2nu(const dnufft_array *grid, const dnufft_array *coord, int forward, double epsilon,
                dnufft_array *out, const dnufft_opts *opts, void *stream) {
  DN_GUARD(dnufft::u2nu_impl(grid, coord, forward, epsilon, out, opts,
                             static_cast<cudaStream_t>(stream)))
}

int dnufft_plan_create(int nu2u, const dnufft_array *coord, const int64_t *grid_shape, int ndim,
                       double epsilon, const dnufft_opts *opts, void *stream, dnufft_plan **plan) {
  DN_GUARD(dnufft::plan_create_impl(nu2u, coord, grid_shape, ndim, epsilon, opts,
                                    static_cast<cudaStream_t>(stream), plan))
}

int dnufft_plan_nu2u(dnufft_plan *plan, int forward, int verbosity, const dnufft_array *points,
                     dnufft_array *out, void *stream) {
  DN_GUARD(dnufft::plan_exec_impl(plan, true, forward, verbosity, points, out,
                                  static_cast<cudaStream_t>(stream)))
}

int dnufft_plan_u2nu(dnufft_plan *plan, int forward, int verbosity, const dnufft_array *grid,
                     dnufft_array *out, void *stream) {
  DN_GUARD(dnufft::plan_exec_impl(plan, false, forward, verbosity, grid, out,
                                  static_cast<cudaStream_t>(stream)))
}

int dnufft_u2nu_dcoord(const dnufft_array *grid, const dnufft_array *coord, int forward,
                       double epsilon, const dnufft_array *weights, dnufft_array *grad,
                       const dnufft_opts *opts, void *stream) {
  DN_GUARD(dnufft::u2nu_dcoord_impl(grid, coord, forward, epsilon, weights, grad, opts,
                                    static_cast<cudaStream_t>(stream)))
}

int dnufft_plan_u2nu_dcoord(dnufft_plan *plan, int forward, const dnufft_array *grid,
                            const dnufft_array *weights, dnufft_array *grad, void *stream) {
  DN_GUARD(dnufft::plan_dcoord_impl(plan, forward, grid, weights, grad,
                                    static_cast<cudaStream_t>(stream)))
}

int dnufft_plan_spread(dnufft_plan *plan, const dnufft_array *points, dnufft_array *grid,
                       void *stream) {
  DN_GUARD(dnufft::plan_spread_impl(plan, points, grid, static_cast<cudaStream_t>(stream)))
}

int dnufft_plan_grid_to_uniform(dnufft_plan *plan, int forward, dnufft_array *grid,
                                dnufft_array *out, void *stream) {
  DN_GUARD(dnufft::plan_grid_to_uniform_impl(plan, forward, grid, out,
                                             static_cast<cudaStream_t>(stream)))
}

int dnufft_plan_rows_fft(dnufft_plan *plan, int forward, dnufft_array *rows, void *stream) {
  DN_GUARD(dnufft::plan_rows_fft_impl(plan, forward, rows, static_cast<cudaStream_t>(stream)))
}

int dnufft_plan_cols_to_uniform(dnufft_plan *plan, int forward, dnufft_array *grid,
                                dnufft_array *out, void *stream) {
  DN_GUARD(dnufft::plan_cols_to_uniform_impl(plan, forward, grid, out,
                                             static_cast<cudaStream_t>(stream)))
}

int dnufft_plan_cols_to_uniform_range(dnufft_plan *plan, int forward, dnufft_array *cols,
                                      int64_t col0, dnufft_array *out, void *stream) {
  DN_GUARD(dnufft::plan_cols_range_impl(plan, forward, cols, col0, out,
                                        static_cast<cudaStream_t>(stream)))
}

int dnufft_plan_uniform_to_cols_range(dnufft_plan *plan, int forward, const dnufft_array *grid,
                                      int64_t col0, dnufft_array *cols, void *stream) {
  DN_GUARD(dnufft::plan_uniform_to_cols_impl(plan, forward, grid, col0, cols,
                                             static_cast<cudaStream_t>(stream)))
}

int dnufft_plan_rows_fft_kept_in(dnufft_plan *plan, int forward, dnufft_array *rows,
                                 void *stream) {
  DN_GUARD(dnufft::plan_rows_fft_kept_in_impl(plan, forward, rows,
                                              static_cast<cudaStream_t>(stream)))
}

int dnufft_plan_interp(dnufft_plan *plan, const dnufft_array *grid, dnufft_array *out,
                       void *stream) {
  DN_GUARD(dnufft::plan_interp_impl(plan, grid, out, static_cast<cudaStream_t>(stream)))
}

int dnufft_find_parameters(int nu2u, int ndim, const int64_t *grid_shape, uint64_t npoints,
                           double epsilon, int calc_f64, int coord_f64, const dnufft_opts *opts,
                           int32_t *kernel_index, int64_t *nover) {
  DN_GUARD(dnufft::find_parameters_impl(nu2u, ndim, grid_shape, npoints, epsilon, calc_f64,
                                        coord_f64, opts, kernel_index, nover))
}

int dnufft_plan_destroy(dnufft_plan *plan) {
  DN_GUARD({
    if (plan) {
      cudaStream_t st = nullptr;
      plan->ix.perm.st = plan->ix.chunks.st = plan->ix.count.st = plan->ix.keys.st = st;
      plan->ix.kblk.st = plan->ix.kbrange.st = st;
      plan->sorted_coord.st = st;
      plan->grid.st = st;
      plan->work.st = st;
      for (int d = 0; d < 3; ++d) plan->dc.corfac[d].st = plan->dc.tw[d].st = st;
      for (auto &pg : plan->groups) {
        pg.ix.perm.st = pg.ix.chunks.st = pg.ix.count.st = pg.ix.keys.st = st;
        pg.ix.kblk.st = pg.ix.kbrange.st = st;
        pg.sorted_coord.st = st;
      }
      delete plan;
      DN_CUDA(cudaDeviceSynchronize());
    }
  })
}

int dnufft_plan_get_info(const dnufft_plan *p, dnufft_plan_info *info) {
  DN_GUARD({
    DN_REQUIRE(p && info, dnufft::ST_BADARG, "null argument");
    std::memset(info, 0, sizeof(*info));
    info->ndim = p->s.g.ndim;
    info->supp = p->s.g.W;
    info->kernel_index = p->s.kidx;
    info->log2tile = p->s.g.log2tile;
    for (int d = 0; d < p->s.g.ndim; ++d) {
      info->nuni[d] = p->s.g.nuni[d];
      info->nover[d] = p->s.g.nover[d];
    }
    info->ofactor = p->s.ofactor;
    info->beta = p->s.beta;
    info->e0 = p->s.e0;
    info->npoints = p->s.npoints;
    info->coord_f64 = p->s.coord_f64;
    info->calc_f64 = p->s.calc_f64;
    info->nchunks = p->ix.nchunks;
    info->tc_records = p->ix.nkblk;
  })
}

int dnufft_plan_get_permutation(const dnufft_plan *p, uint32_t *out, void *stream) {
  DN_GUARD({
    DN_REQUIRE(p && out, dnufft::ST_BADARG, "null argument");
    if (p->s.npoints == 0) return DNUFFT_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!p->s.qbits) {
      DN_CUDA(cudaMemcpyAsync(out, p->ix.perm.p, size_t(p->s.npoints) * 4, cudaMemcpyDefault, st));
    } else {
      // the plan processes points in (tile, quadrant, cell) order; DUCC's
      // permutation is the stable order by tile alone: re-sort the original
      // coordinates
      dnufft::Setup s2 = p->s;
      s2.qbits = false;
      s2.keybits -= 2 + dnufft::tc_cell_bits(s2.g);
      s2.tile_shift = 0;
      s2.chunk = dnufft::CHUNK;
      const uint32_t M = s2.npoints;
      const int nd = s2.g.ndim;
      // sorted coordinates in original order: scatter back through perm
      dnufft::Index ix2;
      ix2.perm = dnufft::DevBuf(size_t(M) * 4, st);
      ix2.keys = dnufft::DevBuf(size_t(M) * 4, st);
      dnufft::DevBuf orig(size_t(M) * nd * (s2.coord_f64 ? 8 : 4), st);
      dnufft::launch_scatter_coords(s2.coord_f64, p->sorted_coord.p, nd, p->ix.perm.as<uint32_t>(),
                                    M, orig.p, st);
      dnufft::launch_fold_keys(s2.coord_f64, orig.p, nd, 1, M, s2.g, ix2.keys.as<uint32_t>(),
                               ix2.perm.as<uint32_t>(), st, false);
      dnufft::DevBuf ws(dnufft::radix_workspace_bytes(M, s2.keybits), st);
      dnufft::radix_sort_pairs(ix2.keys.as<uint32_t>(), ix2.perm.as<uint32_t>(), M, s2.keybits,
                               ws.p, st);
      DN_CUDA(cudaMemcpyAsync(out, ix2.perm.p, size_t(M) * 4, cudaMemcpyDefault, st));
    }
    DN_CUDA(cudaStreamSynchronize(st));
  })
}

const char *dnufft_last_error(void) { return g_last_error.c_str(); }

uint64_t dnufft_kernel_launches(void) { return dnufft::launch_count(); }

int dnufft_selftest_wait_timeout(int64_t limit_ns, void *stream) {
  DN_GUARD({
    DN_REQUIRE(limit_ns > 0 && limit_ns <= 1000000000, dnufft::ST_BADARG,
               "limit must be in (0, 1 s]");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int *err = dnufft::device_error_word();
    dnufft::launch_wait_selftest(err, (unsigned long long)limit_ns, st);
    dnufft::check_device_error(err, st);
  })
}

void dnufft_profile_enable(int enable) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  g_prof_on = enable != 0;
  if (g_prof_on) g_prof.clear();
}

const char *dnufft_profile_json(void) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  std::string js = "{";
  bool first = true;
  for (auto &kv : g_prof) {
    char buf[512];
    std::snprintf(buf, sizeof(buf), "%s\"%s\": [%.6f, %ld]", first ? "" : ", ", kv.first.c_str(),
                  kv.second.first, kv.second.second);
    js += buf;
    first = false;
  }
  js += "}";
  g_prof_json = js;
  return g_prof_json.c_str();
}

}  // extern "C"

// ---------------------------------------------------------------- batches
struct dnufft_batch {
  std::vector<dnufft_plan *> plans;
  std::vector<int> ntrans;
  bool f64 = false;
  int device = 0;
  int max_ntrans = 1;
  uint32_t nchunks = 0;
  size_t sm_spread = 0, sm_interp = 0;
  dnufft::DevBuf grids, insts, tab;
  void *fftb = nullptr;
  dnufft::BatchArray *htab = nullptr;    // pinned: [points | uniform] x nplans
  cudaStream_t cap = nullptr;            // capture stream
  cudaEvent_t done = nullptr;
  cudaGraphExec_t exec[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};   // [type][forward]
  ~dnufft_batch() {
    for (auto &e : exec)
      for (auto &x : e)
        if (x) cudaGraphExecDestroy(x);
    if (done) {
      cudaEventSynchronize(done);
      cudaEventDestroy(done);
    }
    if (fftb) dnufft::fft_batch_destroy(fftb);
    if (htab) cudaFreeHost(htab);
    if (cap) cudaStreamDestroy(cap);
    grids.st = insts.st = tab.st = nullptr;
  }
};

namespace dnufft {

template <typename T>
static void batch_build(dnufft_batch *b, cudaStream_t st) {
  const int n = int(b->plans.size());
  const size_t nn = static_cast<size_t>(n);
  std::vector<SpreadInst<T>> si(nn);
  std::vector<FFTBatchInst> fi(nn);
  size_t total = 0;
  std::vector<size_t> off(nn);
  for (int i = 0; i < n; ++i) {
    const dnufft_plan *p = b->plans[size_t(i)];
    off[size_t(i)] = total;
    total += grid_cells(p->s.g) * size_t(b->ntrans[size_t(i)]) * sizeof(T) * 2;
  }
  b->grids = DevBuf(total, st);
  uint32_t c0 = 0;
  for (int i = 0; i < n; ++i) {
    const dnufft_plan *p = b->plans[size_t(i)];
    SpreadInst<T> &s = si[size_t(i)];
    std::memset(&s, 0, sizeof(s));
    s.pts = PointsDesc{p->sorted_coord.p, int64_t(2), 1, true, p->s.coord_f64,
                       p->ix.perm.as<uint32_t>(), p->s.npoints};
    s.chunks = p->ix.chunks.as<Chunk>();
    s.g = p->s.g;
    s.kp = *reinterpret_cast<const KernelPoly<T> *>(
        sizeof(T) == 4 ? static_cast<const void *>(&p->s.kpf) : static_cast<const void *>(&p->s.kpd));
    s.grid = static_cast<unsigned char *>(b->grids.p) + off[size_t(i)];
    s.ntrans = b->ntrans[size_t(i)];
    s.chunk0 = c0;
    c0 += p->ix.nchunks;
    b->sm_spread = std::max(b->sm_spread, spread_multi_smem<T>(p->s.g));
    b->sm_interp = std::max(b->sm_interp, interp_multi_smem<T>(p->s.g));
    FFTBatchInst &f = fi[size_t(i)];
    f.g = p->s.g;
    f.ax = p->dc.ax;
    for (int d = 0; d < 3; ++d) f.corfac[d] = p->dc.cf[d];
    f.grid = s.grid;
    f.ntrans = s.ntrans;
    f.fft_order = p->o.fft_order != 0;
  }
  b->nchunks = c0;
  b->insts = DevBuf(si.size() * sizeof(SpreadInst<T>), st);
  DN_CUDA(cudaMemcpyAsync(b->insts.p, si.data(), si.size() * sizeof(SpreadInst<T>),
                          cudaMemcpyHostToDevice, st));
  b->fftb = fft_batch_create<T>(fi, st);
  DN_CUDA(cudaStreamSynchronize(st));
}

static void batch_create_impl(int nplans, dnufft_plan *const *plans, const int32_t *ntrans,
                              cudaStream_t st, dnufft_batch **out) {
  DN_REQUIRE(out && plans && nplans > 0, ST_BADARG, "batch: bad arguments");
  auto b = std::make_unique<dnufft_batch>();
  DN_CUDA(cudaGetDevice(&b->device));
  for (int i = 0; i < nplans; ++i) {
    dnufft_plan *p = plans[i];
    DN_REQUIRE(p != nullptr, ST_BADARG, "batch: null plan");
    DN_REQUIRE(p->s.g.ndim == 2, ST_UNSUPPORTED, "batch: 2D plans only");
    DN_REQUIRE(p->s.npoints > 0, ST_BADARG, "batch: plans need at least one point");
    DN_REQUIRE(p->device == b->device, ST_BADARG, "batch: plans of another device");
    if (i == 0) b->f64 = p->s.calc_f64;
    DN_REQUIRE(p->s.calc_f64 == b->f64, ST_BADARG, "batch: plans of one precision only");
    const int nt = ntrans ? ntrans[i] : 1;
    DN_REQUIRE(nt >= 1 && nt <= 65535, ST_BADARG, "batch: ntrans out of range");
    b->plans.push_back(p);
    b->ntrans.push_back(nt);
    b->max_ntrans = std::max(b->max_ntrans, nt);
  }
  if (b->f64) batch_build<double>(b.get(), st);
  else batch_build<float>(b.get(), st);
  b->tab = DevBuf(size_t(2 * nplans) * sizeof(BatchArray), st);
  DN_CUDA(cudaMallocHost(reinterpret_cast<void **>(&b->htab), size_t(2 * nplans) * sizeof(BatchArray)));
  DN_CUDA(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking));
  DN_CUDA(cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming));
  DN_CUDA(cudaEventRecord(b->done, st));
  DN_CUDA(cudaStreamSynchronize(st));
  *out = b.release();
}

// describe instance i's arrays in the table: points (ntrans, M) and uniform (ntrans, N0, N1)
static void batch_fill(dnufft_batch *b, bool type1, const dnufft_array *pts_,
                       const dnufft_array *uni_) {
  const int n = int(b->plans.size());
  const int cdt = b->f64 ? DNUFFT_C128 : DNUFFT_C64;
  for (int i = 0; i < n; ++i) {
    const dnufft_plan *p = b->plans[size_t(i)];
    const int nt = b->ntrans[size_t(i)];
    View pv = view_of(pts_ + i, "points"), uv = view_of(uni_ + i, "uniform");
    DN_REQUIRE(!pv.host && !uv.host, ST_BADARG, "batch: device arrays only");
    DN_REQUIRE(pv.dtype == cdt && uv.dtype == cdt, ST_BADARG, "batch: dtype mismatch");
    BatchArray &a = b->htab[i];
    BatchArray &u = b->htab[n + i];
    std::memset(&a, 0, sizeof(a));
    std::memset(&u, 0, sizeof(u));
    if (pv.ndim == 1) {
      DN_REQUIRE(nt == 1 && uint64_t(pv.shape[0]) == p->s.npoints, ST_BADARG,
                 "batch: points shape mismatch");
      a.stride[1] = pv.stride[0];
    } else {
      DN_REQUIRE(pv.ndim == 2 && pv.shape[0] == nt && uint64_t(pv.shape[1]) == p->s.npoints,
                 ST_BADARG, "batch: points shape mismatch");
      a.stride[0] = pv.stride[0];
      a.stride[1] = pv.stride[1];
    }
    a.ptr = pv.data;
    const int base = (uv.ndim == 3) ? 1 : 0;
    DN_REQUIRE((uv.ndim == 2 && nt == 1) || (uv.ndim == 3 && uv.shape[0] == nt), ST_BADARG,
               "batch: uniform array shape mismatch");
    DN_REQUIRE(uv.shape[base] == p->s.g.nuni[0] && uv.shape[base + 1] == p->s.g.nuni[1],
               ST_BADARG, "batch: uniform array shape mismatch");
    u.ptr = uv.data;
    u.stride[0] = base ? uv.stride[0] : 0;
    u.stride[1] = uv.stride[base];
    u.stride[2] = uv.stride[base + 1];
    (void)type1;
  }
}

template <typename T>
static void batch_record(dnufft_batch *b, int type, bool fwd, cudaStream_t cs) {
  const int n = int(b->plans.size());
  BatchArray *tab = b->tab.as<BatchArray>();
  DN_CUDA(cudaMemcpyAsync(tab, b->htab, size_t(2 * n) * sizeof(BatchArray),
                          cudaMemcpyHostToDevice, cs));
  const SpreadInst<T> *insts = b->insts.as<const SpreadInst<T>>();
  if (type == 0) {
    size_t bytes = 0;
    for (int i = 0; i < n; ++i)
      bytes += grid_cells(b->plans[size_t(i)]->s.g) * size_t(b->ntrans[size_t(i)]) * sizeof(T) * 2;
    DN_CUDA(cudaMemsetAsync(b->grids.p, 0, bytes, cs));
    launch_spread_multi<T>(insts, n, b->nchunks, b->max_ntrans, b->sm_spread, tab, cs);
    fft_batch_run<T>(b->fftb, 0, tab + n, fwd, cs);
  } else {
    fft_batch_run<T>(b->fftb, 1, tab + n, fwd, cs);
    launch_interp_multi<T>(insts, n, b->nchunks, b->max_ntrans, b->sm_interp, tab, cs);
  }
}

static void batch_exec_impl(dnufft_batch *b, bool type1, int forward, const dnufft_array *in,
                            dnufft_array *out, cudaStream_t st) {
  DN_REQUIRE(b && in && out, ST_BADARG, "batch: null argument");
  int dev = 0;
  DN_CUDA(cudaGetDevice(&dev));
  DN_REQUIRE(dev == b->device, ST_BADARG, "batch: wrong current device");
  // the previous call must have copied its argument table before it is reused
  DN_CUDA(cudaEventSynchronize(b->done));
  if (type1) batch_fill(b, true, in, out);
  else batch_fill(b, false, out, in);
  const int type = type1 ? 0 : 1, f = forward ? 1 : 0;
  if (!b->exec[type][f]) {
    cudaGraph_t graph = nullptr;
    DN_CUDA(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
    try {
      if (b->f64) batch_record<double>(b, type, forward != 0, b->cap);
      else batch_record<float>(b, type, forward != 0, b->cap);
    } catch (...) {
      cudaStreamEndCapture(b->cap, &graph);
      if (graph) cudaGraphDestroy(graph);
      throw;
    }
    DN_CUDA(cudaStreamEndCapture(b->cap, &graph));
    cudaGraphExec_t ex = nullptr;
    cudaError_t e = cudaGraphInstantiate(&ex, graph, 0);
    cudaGraphDestroy(graph);
    DN_CUDA(e);
    b->exec[type][f] = ex;
  }
  DN_CUDA(cudaGraphLaunch(b->exec[type][f], st));
  note_launch(type1 ? 4 : 3);
  DN_CUDA(cudaEventRecord(b->done, st));
}

}  // namespace dnufft

extern "C" {

int dnufft_batch_create(int nplans, dnufft_plan *const *plans, const int32_t *ntrans, void *stream,
                        dnufft_batch **batch) {
  DN_GUARD(dnufft::batch_create_impl(nplans, plans, ntrans, static_cast<cudaStream_t>(stream),
                                     batch))
}

int dnufft_batch_nu2u(dnufft_batch *batch, int forward, const dnufft_array *points,
                      dnufft_array *out, void *stream) {
  DN_GUARD(dnufft::batch_exec_impl(batch, true, forward, points, out,
                                   static_cast<cudaStream_t>(stream)))
}

int dnufft_batch_u2nu(dnufft_batch *batch, int forward, const dnufft_array *grids,
                      dnufft_array *out, void *stream) {
  DN_GUARD(dnufft::batch_exec_impl(batch, false, forward, grids, out,
                                   static_cast<cudaStream_t>(stream)))
}

int dnufft_batch_destroy(dnufft_batch *batch) {
  DN_GUARD({ delete batch; })
}

}  // extern "C"
