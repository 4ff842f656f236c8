// w-gridder: radio-interferometric gridding / degridding with w-stacking, the
// counterpart of ducc0.wgridder (src/ducc0/wgridder/wgridder.h,
// python/wgridder_pymod.cc).
//
// The 2D part of every w plane is this library's type-1 / type-2 transform
// (dnufft_nu2u / dnufft_u2nu on device arrays), so the spreading,
// interpolation, FFT and u/v correction kernels are the ones of the NUFFT
// path.  The w-gridder adds:
//   * visibility preparation (k_wg_flags, k_wg_compact): active visibilities
//     (|vis|^2 * wgt * mask != 0 for gridding, wgt * mask != 0 for
//     degridding) compacted into (u, v) coordinates in wavelengths, w, a value
//     and the (row, channel) index; with w-stacking a visibility with w < 0 is
//     replaced by its Hermitian mirror (-u, -v, -w, conjugate value), which
//     leaves every real image sum unchanged and halves the w range
//     (wgridder.h:256-270, :1170-1172);
//   * the phase of an image centre off the phase centre and of the w-screen
//     shift, e^{2 pi i (u l0 + v m0 + w nshift)}, folded into the values
//     (wgridder.h:1121-1135);
//   * w planes (wgridder.h:675-692): planes at w_p = wmin + p dw, a visibility
//     contributes to the supp planes from floor((w - wmin)/dw + 1 - supp/2) on
//     with the weights of the same kernel as in u and v; the visibilities are
//     sorted by that first plane, so the ones of plane p are one contiguous
//     range;
//   * per plane (wgridder.h:1426-1460): values times the plane's w weight ->
//     2D type 1 -> dirty += Re(image e^{-2 pi i w_p (n - 1 + nshift)})
//     (k_wg_screen_add); degridding mirrors it with the 2D type 2 and
//     accumulates the weighted results per visibility (k_wg_degrid_acc);
//   * the global correction (wgridder.h:1343-1396): the w kernel's correction
//     function at (n - 1 + nshift) dw and the division by n (k_wg_correct).
// The parameter choice (kernel, oversampled grid, plane spacing) follows
// DUCC's cost model (wgridder.h:1499-1579), so both pick the same kernel.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "ducc_b200.h"
#include "kernels.h"

namespace dnufft {
namespace wg {

constexpr double SPEED_OF_LIGHT = 299792458.;
constexpr int MAXNODES = 32;   // Gauss-Legendre nodes of the correction function

// ---------------------------------------------------------------- helpers
struct Arr {
  void *p = nullptr;
  int dtype = 0;
  int ndim = 0;
  int64_t shape[2] = {0, 0};
  int64_t stride[2] = {0, 0};
};

static Arr arr_of(const dnufft_array *a, const char *what, int ndim, bool optional = false) {
  Arr r;
  if (a == nullptr) {
    DN_REQUIRE(optional, ST_BADARG, std::string(what) + ": null array");
    return r;
  }
  DN_REQUIRE(a->ndim == ndim, ST_BADARG, std::string(what) + ": wrong number of dimensions");
  r.p = a->data;
  r.dtype = a->dtype;
  r.ndim = ndim;
  int64_t size = 1;
  for (int d = 0; d < ndim; ++d) {
    r.shape[d] = a->shape[d];
    r.stride[d] = a->stride[d];
    DN_REQUIRE(r.shape[d] >= 0, ST_BADARG, std::string(what) + ": negative extent");
    size *= r.shape[d];
  }
  if (size > 0) {
    DN_REQUIRE(r.p != nullptr, ST_BADARG, std::string(what) + ": null data");
    cudaPointerAttributes at;
    cudaError_t e = cudaPointerGetAttributes(&at, r.p);
    if (e != cudaSuccess) cudaGetLastError();
    DN_REQUIRE(e == cudaSuccess && (at.type == cudaMemoryTypeDevice ||
                                    at.type == cudaMemoryTypeManaged),
               ST_BADARG, std::string(what) + ": must be a device array");
  }
  return r;
}

struct Buf {
  void *p = nullptr;
  cudaStream_t st = nullptr;
  Buf() = default;
  Buf(size_t bytes, cudaStream_t s) : st(s) {
    if (bytes) {
      cudaError_t e = cudaMallocAsync(&p, bytes, s);
      if (e != cudaSuccess) {
        cudaGetLastError();
        throw Error(ST_OOM, "device allocation failed (w-gridder)");
      }
    }
  }
  Buf(const Buf &) = delete;
  Buf &operator=(const Buf &) = delete;
  Buf(Buf &&o) noexcept : p(o.p), st(o.st) { o.p = nullptr; }
  Buf &operator=(Buf &&o) noexcept {
    if (this != &o) {
      if (p) cudaFreeAsync(p, st);
      p = o.p;
      st = o.st;
      o.p = nullptr;
    }
    return *this;
  }
  ~Buf() {
    if (p) cudaFreeAsync(p, st);
  }
};

template <typename X> static X *ptr(const Buf &b) { return static_cast<X *>(b.p); }

static dnufft_array dev_array(void *p, int dtype, int ndim, int64_t s0, int64_t s1 = 0) {
  dnufft_array a;
  std::memset(&a, 0, sizeof(a));
  a.data = p;
  a.dtype = dtype;
  a.ndim = ndim;
  a.shape[0] = s0;
  a.shape[1] = s1;
  if (ndim == 1) {
    a.stride[0] = 1;
  } else {
    a.stride[0] = s1;
    a.stride[1] = 1;
  }
  return a;
}

static void check_nufft(int status) {
  if (status != 0) throw Error(status, std::string("w-gridder: ") + dnufft_last_error());
}

// n - 1 for an image pixel, in the form DUCC uses near n = 1
// (wgridder.h:385-388) and beyond the horizon
__host__ __device__ inline double nm1_of(double x, double y) {
  const double xsq = x * x, ysq = y * y, tmp = 1. - xsq - ysq;
  return (tmp >= 0) ? (-xsq - ysq) / (sqrt(tmp) + 1.) : -sqrt(-tmp) - 1.;
}

// e^{2 pi i t} with t reduced to [0, 1) first
__device__ inline void cis2pi(double t, double &c, double &s) {
  t -= floor(t);
  sincospi(2. * t, &s, &c);
}

// tap nth (0..W-1) of the kernel weights at argument x (common.cuh's
// kernel_weights for a run-time support)
template <typename C>
__device__ inline C kernel_tap(const KernelPoly<C> &kp, int W, C x, int nth) {
  const int D = W + 3 + (W & 1);
  const int k = nth < W - 1 - nth ? nth : W - 1 - nth;
  const C x2 = x * x;
  C e = kp.c[0][k], o = kp.c[1][k];
  for (int j = 2; j < D; j += 2) {
    e = e * x2 + kp.c[j][k];
    o = o * x2 + kp.c[j + 1][k];
  }
  return (nth == k) ? e * x + o : o - e * x;
}

struct CorrNodes {
  int n, W;
  double x[MAXNODES], wpsi[MAXNODES];
};

__device__ inline double corfunc(const CorrNodes &cn, double v) {
  double s = 0;
  for (int k = 0; k < cn.n; ++k) s += cn.wpsi[k] * cos((M_PI * cn.W * cn.x[k]) * v);
  return 1. / s;
}

struct Common {
  int64_t nrows, nchan;
  const double *uvw;
  int64_t us0, us1;     // uvw strides (elements)
  const double *freq;
  int64_t fs;
  const void *wgt;      // real, T; nullptr: 1
  int64_t ws0, ws1;
  const uint8_t *mask;  // nullptr: 1
  int64_t ms0, ms1;
  double ufac, vfac, wfac;
  int do_w;
};

template <typename T>
__device__ inline T wgt_at(const Common &c, int64_t r, int64_t ch) {
  return c.wgt ? static_cast<const T *>(c.wgt)[r * c.ws0 + ch * c.ws1] : T(1);
}

__device__ inline bool mask_at(const Common &c, int64_t r, int64_t ch) {
  return c.mask ? c.mask[r * c.ms0 + ch * c.ms1] != 0 : true;
}

// ---------------------------------------------------------------- kernels
// flag[e] = 1 where visibility e = row * nchan + chan takes part
template <typename T>
__global__ void k_wg_flags(Common c, const cplx<T> *__restrict__ vis, int64_t vs0, int64_t vs1,
                           uint32_t *__restrict__ flag) {
  const int64_t n = c.nrows * c.nchan;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t r = e / c.nchan, ch = e - r * c.nchan;
    T f = wgt_at<T>(c, r, ch) * T(mask_at(c, r, ch) ? 1 : 0);
    if (vis) {
      const cplx<T> v = vis[r * vs0 + ch * vs1];
      f *= v.x * v.x + v.y * v.y;
    }
    flag[e] = (f != T(0)) ? 1u : 0u;
  }
}

// compacted visibility pos = scan[e]: coordinates (u, v), w, index e with the
// mirror flag in bit 31, and (gridding) the value with weight and phases;
// also the largest and smallest w (non-negative with w-stacking: the bit
// patterns order like the values)
template <typename T, typename C>
__global__ void k_wg_compact(Common c, const cplx<T> *__restrict__ vis, int64_t vs0,
                             int64_t vs1, const uint32_t *__restrict__ flag,
                             const uint32_t *__restrict__ scan, double l0, double m0,
                             double nshift, double *__restrict__ coord, double *__restrict__ wv,
                             uint32_t *__restrict__ idx, cplx<C> *__restrict__ val,
                             unsigned long long *__restrict__ wrange) {
  const int64_t n = c.nrows * c.nchan;
  unsigned long long wlo = ~0ull, whi = 0ull;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n;
       e += int64_t(gridDim.x) * blockDim.x) {
    if (!flag[e]) continue;
    const int64_t r = e / c.nchan, ch = e - r * c.nchan;
    const double foc = c.freq[ch * c.fs] / SPEED_OF_LIGHT;
    double u = c.ufac * c.uvw[r * c.us0] * foc;
    double v = c.vfac * c.uvw[r * c.us0 + c.us1] * foc;
    double w = c.wfac * c.uvw[r * c.us0 + 2 * c.us1] * foc;
    const uint32_t pos = scan[e];
    // value with the centre / w-screen shift phase at the original coordinates
    double vr = 0, vi = 0;
    if (val) {
      const cplx<T> x = vis[r * vs0 + ch * vs1];
      const double wt = double(wgt_at<T>(c, r, ch));
      double cs, sn;
      cis2pi(u * l0 + v * m0 + w * nshift, cs, sn);
      vr = wt * (double(x.x) * cs - double(x.y) * sn);
      vi = wt * (double(x.x) * sn + double(x.y) * cs);
    }
    uint32_t fl = 0;
    if (c.do_w && w < 0) {
      u = -u;
      v = -v;
      w = -w;
      vi = -vi;
      fl = 1u << 31;
    }
    coord[2 * int64_t(pos)] = u;
    coord[2 * int64_t(pos) + 1] = v;
    wv[pos] = w;
    idx[pos] = uint32_t(e) | fl;
    if (val) val[pos] = mkc<C>(C(vr), C(vi));
    if (c.do_w) {
      const unsigned long long b = __double_as_longlong(w);
      wlo = b < wlo ? b : wlo;
      whi = b > whi ? b : whi;
    }
  }
  if (c.do_w) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long a = __shfl_xor_sync(0xffffffffu, wlo, o);
      const unsigned long long b = __shfl_xor_sync(0xffffffffu, whi, o);
      wlo = a < wlo ? a : wlo;
      whi = b > whi ? b : whi;
    }
    if ((threadIdx.x & 31) == 0) {
      atomicMin(&wrange[0], wlo);
      atomicMax(&wrange[1], whi);
    }
  }
}

__global__ void k_wg_count(const uint32_t *__restrict__ flag, const uint32_t *__restrict__ scan,
                           int64_t n, uint32_t *__restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) out[0] = n > 0 ? scan[n - 1] + flag[n - 1] : 0u;
}

// first plane of every compacted visibility (the sort key)
__global__ void k_wg_minplane(const double *__restrict__ wv, uint32_t nvis, double wmin,
                              double xdw, int W, uint32_t *__restrict__ key,
                              uint32_t *__restrict__ ord) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nvis; i += gridDim.x * blockDim.x) {
    // DUCC: max(0, int((w + wshift) * xdw)), wshift = dw - W dw / 2 - wmin
    const double t = (wv[i] - wmin) * xdw + 1. - 0.5 * W;
    const uint32_t p = t > 0 ? uint32_t(t) : 0u;
    key[i] = p;
    ord[i] = i;
  }
}

// start[p] = first sorted visibility whose first plane is >= p (p = 0..np),
// from the sorted keys: position i writes the planes in (key[i-1], key[i]]
__global__ void k_wg_plane_starts(const uint32_t *__restrict__ key, uint32_t n, uint32_t np,
                                  uint32_t *__restrict__ start) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += gridDim.x * blockDim.x) {
    const int64_t lo = i > 0 ? int64_t(key[i - 1]) : -1;
    const int64_t hi = i < n ? int64_t(min(key[i], np)) : int64_t(np);
    for (int64_t p = lo + 1; p <= hi; ++p) start[p] = i;
  }
}

// compacted arrays in plane order
template <typename C>
__global__ void k_wg_gather(const uint32_t *__restrict__ ord, uint32_t nvis,
                            const double *__restrict__ coord, const double *__restrict__ wv,
                            const uint32_t *__restrict__ idx, const cplx<C> *__restrict__ val,
                            double *__restrict__ coord2, double *__restrict__ wv2,
                            uint32_t *__restrict__ idx2, cplx<C> *__restrict__ val2) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nvis; i += gridDim.x * blockDim.x) {
    const uint32_t j = ord[i];
    coord2[2 * int64_t(i)] = coord[2 * int64_t(j)];
    coord2[2 * int64_t(i) + 1] = coord[2 * int64_t(j) + 1];
    wv2[i] = wv[j];
    idx2[i] = idx[j];
    if (val) val2[i] = val[j];
  }
}

// weight of plane p for visibility i (0 outside its supp planes)
template <typename C>
__device__ inline C plane_weight(const KernelPoly<C> &kp, int W, double wi, uint32_t key, int p,
                                 double wmin, double xdw) {
  const int nth = p - int(key);
  if (nth < 0 || nth >= W) return C(0);
  // frac = (w - w_first) / dw, kernel argument W - 1 - 2 frac (wgridder.h:1001-1012,
  // gridding_kernel.h:240-248)
  const double frac = (wi - wmin) * xdw - double(key);
  return kernel_tap<C>(kp, W, C(double(W - 1) - 2. * frac), nth);
}

template <typename C>
__global__ void k_wg_plane_vals(const cplx<C> *__restrict__ val, const double *__restrict__ wv,
                                const uint32_t *__restrict__ key, uint32_t lo, uint32_t cnt,
                                KernelPoly<C> kp, int W, int p, double wmin, double xdw,
                                cplx<C> *__restrict__ out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
    const uint32_t j = lo + i;
    const C f = plane_weight<C>(kp, W, wv[j], key[j], p, wmin, xdw);
    const cplx<C> v = val[j];
    out[i] = mkc<C>(v.x * f, v.y * f);
  }
}

struct ImgGeom {
  int64_t nx, ny;
  double x0, y0, psx, psy;   // pixel (i, j) at (x0 + i psx, y0 + j psy)
  double nshift;
};

// pm(i, j) = n - 1 + nshift of every pixel, once per call for the w screens
__global__ void k_wg_pixel_nm1(ImgGeom g, double *__restrict__ pm) {
  const int64_t n = g.nx * g.ny;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = e / g.ny, j = e - i * g.ny;
    pm[e] = nm1_of(g.x0 + i * g.psx, g.y0 + j * g.psy) + g.nshift;
  }
}

// e^{2 pi i t}: the product is formed and reduced to [0, 1) in double, the
// sine and cosine taken in the compute precision C (as DUCC does for single
// precision, wgridder.h:392-394)
template <typename C> __device__ inline void cis2pi_c(double t, C &c, C &s) {
  t -= floor(t);
  if constexpr (sizeof(C) == 4) {
    sincospif(float(2. * t), &s, &c);
  } else {
    sincospi(2. * t, &s, &c);
  }
}

// dirty(i, j) += Re(img(i, j) e^{-2 pi i w_p (n - 1 + nshift)})
template <typename C, typename T>
__global__ void k_wg_screen_add(const cplx<C> *__restrict__ img, const double *__restrict__ pm,
                                ImgGeom g, double wp, T *__restrict__ dirty, int64_t ds0,
                                int64_t ds1) {
  const int64_t n = g.nx * g.ny;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = e / g.ny, j = e - i * g.ny;
    C cs, sn;
    cis2pi_c<C>(-wp * pm[e], cs, sn);
    const cplx<C> a = img[e];
    T &d = dirty[i * ds0 + j * ds1];
    d += T(a.x * cs - a.y * sn);
  }
}

// dirty(i, j) = Re(img(i, j)) (no w term)
template <typename C, typename T>
__global__ void k_wg_real(const cplx<C> *__restrict__ img, int64_t nx, int64_t ny,
                          T *__restrict__ dirty, int64_t ds0, int64_t ds1) {
  const int64_t n = nx * ny;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = e / ny, j = e - i * ny;
    dirty[i * ds0 + j * ds1] = T(img[e].x);
  }
}

// w correction and division by n (wgridder.h:1343-1396); the u/v correction
// is applied by the 2D transforms
__device__ inline double global_corr(const CorrNodes &cn, double nm1, double nshift, double dw,
                                     bool divide_by_n) {
  if (nm1 > -1.) {
    // inside the horizon (1 - x^2 - y^2 >= 0 gives n - 1 >= -1)
    double f = corfunc(cn, (nm1 + nshift) * dw);
    return divide_by_n ? f / (nm1 + 1.) : f;
  }
  return divide_by_n ? 0. : corfunc(cn, (nm1 + nshift) * dw);
}

template <typename T>
__global__ void k_wg_correct(T *__restrict__ dirty, int64_t ds0, int64_t ds1, ImgGeom g,
                             CorrNodes cn, double dw, int divide_by_n) {
  const int64_t n = g.nx * g.ny;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = e / g.ny, j = e - i * g.ny;
    const double x = g.x0 + i * g.psx, y = g.y0 + j * g.psy;
    const double nm1 = nm1_of(x, y);
    const bool inside = 1. - x * x - y * y >= 0;
    double f;
    if (inside) {
      f = corfunc(cn, (nm1 + g.nshift) * dw);
      if (divide_by_n) f /= nm1 + 1.;
    } else {
      f = divide_by_n ? 0. : corfunc(cn, (nm1 + g.nshift) * dw);
    }
    T &d = dirty[i * ds0 + j * ds1];
    d = T(double(d) * f);
  }
}

// degridding input: img0(i, j) = dirty(i, j) times the global correction (w
// term) or as it is (no w term), as a complex image
template <typename T, typename C>
__global__ void k_wg_dirty_in(const T *__restrict__ dirty, int64_t ds0, int64_t ds1, ImgGeom g,
                              CorrNodes cn, double dw, int with_w, int divide_by_n,
                              C *__restrict__ img0) {
  const int64_t n = g.nx * g.ny;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = e / g.ny, j = e - i * g.ny;
    double f = 1.;
    if (with_w) {
      const double x = g.x0 + i * g.psx, y = g.y0 + j * g.psy;
      const double nm1 = nm1_of(x, y);
      if (1. - x * x - y * y >= 0) {
        f = corfunc(cn, (nm1 + g.nshift) * dw);
        if (divide_by_n) f /= nm1 + 1.;
      } else {
        f = divide_by_n ? 0. : corfunc(cn, (nm1 + g.nshift) * dw);
      }
    }
    img0[e] = C(double(dirty[i * ds0 + j * ds1]) * f);
  }
}

// plane image for degridding: img0 e^{+2 pi i w_p (n - 1 + nshift)}
template <typename C>
__global__ void k_wg_screen_apply(const C *__restrict__ img0, const double *__restrict__ pm,
                                  int64_t n, double wp, cplx<C> *__restrict__ img) {
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n;
       e += int64_t(gridDim.x) * blockDim.x) {
    C cs, sn;
    cis2pi_c<C>(wp * pm[e], cs, sn);
    const C a = img0[e];
    img[e] = mkc<C>(a * cs, a * sn);
  }
}

template <typename C>
__global__ void k_wg_real_to_complex(const C *__restrict__ img0, int64_t n,
                                     cplx<C> *__restrict__ img) {
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n;
       e += int64_t(gridDim.x) * blockDim.x)
    img[e] = mkc<C>(img0[e], C(0));
}

// acc[lo + i] += w_p(vis) * res[i]
template <typename C>
__global__ void k_wg_degrid_acc(const cplx<C> *__restrict__ res, const double *__restrict__ wv,
                                const uint32_t *__restrict__ key, uint32_t lo, uint32_t cnt,
                                KernelPoly<C> kp, int W, int p, double wmin, double xdw,
                                cplx<C> *__restrict__ acc) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
    const uint32_t j = lo + i;
    const C f = plane_weight<C>(kp, W, wv[j], key[j], p, wmin, xdw);
    const cplx<C> r = res[i];
    cplx<C> a = acc[j];
    a.x += f * r.x;
    a.y += f * r.y;
    acc[j] = a;
  }
}

// the degridding accumulation over all compacted visibilities (a grouped
// index leaves the results of those outside plane p untouched: they are
// skipped, not weighted by zero)
template <typename C>
__global__ void k_wg_degrid_acc_all(const cplx<C> *__restrict__ res,
                                    const double *__restrict__ wv,
                                    const uint32_t *__restrict__ key, uint32_t n,
                                    KernelPoly<C> kp, int W, int p, double wmin, double xdw,
                                    cplx<C> *__restrict__ acc) {
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const int nth = p - int(key[j]);
    if (nth < 0 || nth >= W) continue;
    const C f = plane_weight<C>(kp, W, wv[j], key[j], p, wmin, xdw);
    const cplx<C> r = res[j];
    cplx<C> a = acc[j];
    a.x += f * r.x;
    a.y += f * r.y;
    acc[j] = a;
  }
}

// vis(row, chan) = wgt * S (S conjugated for a mirrored visibility), S = the
// accumulated sum times e^{-2 pi i (u l0 + v m0 + w nshift)} at the (mirrored)
// coordinates
template <typename T, typename C>
__global__ void k_wg_scatter(const cplx<C> *__restrict__ acc, const double *__restrict__ coord,
                             const double *__restrict__ wv, const uint32_t *__restrict__ idx,
                             uint32_t nvis, Common c, double l0, double m0, double nshift,
                             cplx<T> *__restrict__ vis, int64_t vs0, int64_t vs1) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nvis; i += gridDim.x * blockDim.x) {
    const uint32_t id = idx[i];
    const int64_t e = int64_t(id & 0x7fffffffu);
    const int64_t r = e / c.nchan, ch = e - r * c.nchan;
    const double u = coord[2 * int64_t(i)], v = coord[2 * int64_t(i) + 1];
    const double w = c.do_w ? wv[i] : 0.;
    double cs, sn;
    cis2pi(-(u * l0 + v * m0 + w * nshift), cs, sn);
    const cplx<C> a = acc[i];
    double sr = double(a.x) * cs - double(a.y) * sn;
    double si = double(a.x) * sn + double(a.y) * cs;
    if (id >> 31) si = -si;
    const double wt = double(wgt_at<T>(c, r, ch));
    vis[r * vs0 + ch * vs1] = mkc<T>(T(wt * sr), T(wt * si));
  }
}

template <typename T>
__global__ void k_wg_zero_vis(Common c, cplx<T> *__restrict__ vis, int64_t vs0, int64_t vs1) {
  const int64_t n = c.nrows * c.nchan;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t r = e / c.nchan, ch = e - r * c.nchan;
    vis[r * vs0 + ch * vs1] = mkc<T>(T(0), T(0));
  }
}

template <typename T>
__global__ void k_wg_zero_dirty(T *__restrict__ dirty, int64_t nx, int64_t ny, int64_t ds0,
                                int64_t ds1) {
  const int64_t n = nx * ny;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = e / ny, j = e - i * ny;
    dirty[i * ds0 + j * ds1] = T(0);
  }
}

static unsigned grid_for(int64_t n, int threads = 256) {
  int64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > 148 * 16) b = 148 * 16;
  return unsigned(b);
}

// ---------------------------------------------------------------- host side
struct Params {
  int kidx = -1, W = 0;
  int64_t nu = 0, nv = 0;
  double ofactor = 0, beta = 0, e0 = 0;
  double nm1min = 0, nm1max = 0, nshift = 0;
  double dw = 0, xdw = 0, wmin = 0;
  int64_t nplanes = 0;
  double lshift = 0, mshift = 0;
};

// DUCC's getNuNv and countRanges (wgridder.h:1499-1579, :675-692)
static Params choose(int64_t nx, int64_t ny, double psx, double psy, double epsilon,
                     bool singleprec, const dnufft_wgrid_opts &o, int64_t nvis, double wmin_d,
                     double wmax_d) {
  Params P;
  P.lshift = o.flip_u ? -o.center_x : o.center_x;
  P.mshift = o.flip_v ? -o.center_y : o.center_y;
  const double xmin = P.lshift - 0.5 * nx * psx, xmax = xmin + (nx - 1) * psx;
  const double ymin = P.mshift - 0.5 * ny * psy, ymax = ymin + (ny - 1) * psy;
  std::vector<double> xext{xmin, xmax}, yext{ymin, ymax};
  if (xmin * xmax < 0) xext.push_back(0);
  if (ymin * ymax < 0) yext.push_back(0);
  P.nm1min = 1e300;
  P.nm1max = -1e300;
  for (double xc : xext)
    for (double yc : yext) {
      const double t = xc * xc + yc * yc;
      const double nv_ = (t <= 1.) ? (std::sqrt(1. - t) - 1.) : (-std::sqrt(t - 1.) - 1.);
      P.nm1min = std::min(P.nm1min, nv_);
      P.nm1max = std::max(P.nm1max, nv_);
    }
  const bool do_w = o.do_wgridding != 0;
  P.nshift = (!o.allow_nshift || !do_w) ? 0. : -0.5 * (P.nm1max + P.nm1min);
  auto idx = available_kernels(epsilon, do_w ? 3 : 2, singleprec, o.sigma_min, o.sigma_max);
  const double nref_fft = 2048, costref_fft = 0.0693;
  // DUCC's SIMD width in this model is min(8, native lanes): 8 for float, and
  // 8 for double on an AVX-512 build (4 on AVX2); the NUFFT planner's
  // default assumes the same build
  const size_t vlen = 8;
  const double nt = double(effective_threads(o.nthreads));
  double mincost = 1e300;
  for (size_t i : idx) {
    const auto &k = kernel_db()[i];
    const size_t W = size_t(k.W);
    const size_t nvec = (W + vlen - 1) / vlen;
    const double of = k.ofactor;
    int64_t nu = std::max<int64_t>(2 * int64_t(good_size_complex(size_t(nx * of * 0.5) + 1)), 16);
    int64_t nv = std::max<int64_t>(2 * int64_t(good_size_complex(size_t(ny * of * 0.5) + 1)), 16);
    const double logterm = std::log(double(nu) * double(nv)) / std::log(nref_fft * nref_fft);
    double fftcost = double(nu) / nref_fft * double(nv) / nref_fft * logterm * costref_fft;
    double gridcost = 2.2e-10 * double(nvis) *
                      double(W * nvec * vlen + ((2 * nvec + 1) * (W + 3) * vlen));
    if (do_w) {
      const double dw =
          0.5 / of / std::max(std::abs(P.nm1max + P.nshift), std::abs(P.nm1min + P.nshift));
      const double np_ = double(size_t((wmax_d - wmin_d) / dw + double(W)));
      fftcost *= np_;
      gridcost *= double(W);
    }
    gridcost /= nt;
    const double x2 = nt - 1, m2 = 6. - 1;
    fftcost /= 1. + x2 / std::pow(1. + std::pow(x2 / m2, 2.), 0.5);
    const double cost = fftcost + gridcost;
    if (cost < mincost) {
      mincost = cost;
      P.kidx = int(i);
      P.nu = nu;
      P.nv = nv;
    }
  }
  const auto &k = kernel_db()[size_t(P.kidx)];
  P.W = k.W;
  P.beta = k.beta * k.W;
  P.e0 = k.e0;
  P.ofactor = std::min(double(P.nu) / double(nx), double(P.nv) / double(ny));
  if (do_w) {
    P.dw = 0.5 / P.ofactor /
           std::max(std::abs(P.nm1max + P.nshift), std::abs(P.nm1min + P.nshift));
    P.xdw = 1. / P.dw;
    P.nplanes = int64_t(size_t((wmax_d - wmin_d) / P.dw + double(P.W)));
    DN_REQUIRE(P.nplanes < (int64_t(1) << 16), ST_UNSUPPORTED, "too many w planes");
    P.wmin = (wmin_d + wmax_d) * 0.5 - 0.5 * double(P.nplanes - 1) * P.dw;
  }
  DN_REQUIRE(P.nu >= 2 * ((P.W + 1) / 2) && P.nv >= 2 * ((P.W + 1) / 2), ST_BADARG,
             "oversampled grid too small");
  return P;
}

template <typename C> static KernelPoly<C> make_poly(int W, double beta, double e0) {
  KernelPoly<C> kp;
  std::memset(&kp, 0, sizeof(kp));
  const auto coeff = kernel_coeffs(W, beta, e0);
  const int D = W + 3, Dp = W + 3 + (W & 1), ofs = Dp - D, H = (W + 1) / 2;
  for (int j = 0; j <= D; ++j)
    for (int k = 0; k < H; ++k) kp.c[j + ofs][k] = C(coeff[size_t(j) * W + k]);
  return kp;
}

static CorrNodes make_nodes(int W, double beta, double e0) {
  CorrNodes cn;
  std::memset(&cn, 0, sizeof(cn));
  std::vector<double> x, wpsi;
  correction_nodes(W, beta, e0, x, wpsi);
  DN_REQUIRE(int(x.size()) <= MAXNODES, ST_INTERNAL, "too many quadrature nodes");
  cn.n = int(x.size());
  cn.W = W;
  for (int k = 0; k < cn.n; ++k) {
    cn.x[k] = x[size_t(k)];
    cn.wpsi[k] = wpsi[size_t(k)];
  }
  return cn;
}

// inputs common to both directions
struct Inputs {
  Common c;
  Arr uvw, freq, vis, wgt, mask;
  bool f64 = false;     // data precision
  int64_t nx = 0, ny = 0;
};

static Inputs parse(const dnufft_array *uvw_, const dnufft_array *freq_,
                    const dnufft_array *vis_, bool vis_needed, const dnufft_array *wgt_,
                    const dnufft_array *mask_, const dnufft_wgrid_opts &o) {
  Inputs in;
  in.uvw = arr_of(uvw_, "uvw", 2);
  in.freq = arr_of(freq_, "freq", 1);
  in.vis = arr_of(vis_, "vis", 2, !vis_needed);
  in.wgt = arr_of(wgt_, "wgt", 2, true);
  in.mask = arr_of(mask_, "mask", 2, true);
  DN_REQUIRE(in.uvw.dtype == DNUFFT_F64 && in.uvw.shape[1] == 3, ST_BADARG,
             "uvw must be float64 of shape (nrows, 3)");
  DN_REQUIRE(in.freq.dtype == DNUFFT_F64, ST_BADARG, "freq must be float64");
  const int64_t nrows = in.uvw.shape[0], nchan = in.freq.shape[0];
  DN_REQUIRE(nrows * nchan < (int64_t(1) << 31), ST_UNSUPPORTED,
             "more than 2^31 visibilities");
  if (in.vis.p || vis_needed) {
    DN_REQUIRE(in.vis.shape[0] == nrows && in.vis.shape[1] == nchan, ST_BADARG,
               "vis must have shape (nrows, nchan)");
    DN_REQUIRE(in.vis.dtype == DNUFFT_C64 || in.vis.dtype == DNUFFT_C128, ST_BADARG,
               "vis must be complex64 or complex128");
  }
  in.c.nrows = nrows;
  in.c.nchan = nchan;
  in.c.uvw = static_cast<const double *>(in.uvw.p);
  in.c.us0 = in.uvw.stride[0];
  in.c.us1 = in.uvw.stride[1];
  in.c.freq = static_cast<const double *>(in.freq.p);
  in.c.fs = in.freq.stride[0];
  in.c.wgt = in.wgt.p;
  in.c.ws0 = in.wgt.stride[0];
  in.c.ws1 = in.wgt.stride[1];
  in.c.mask = static_cast<const uint8_t *>(in.mask.p);
  in.c.ms0 = in.mask.stride[0];
  in.c.ms1 = in.mask.stride[1];
  in.c.ufac = o.flip_u ? -1. : 1.;
  in.c.vfac = o.flip_v ? -1. : 1.;
  in.c.wfac = o.flip_w ? -1. : 1.;
  in.c.do_w = o.do_wgridding ? 1 : 0;
  if (in.mask.p) {
    DN_REQUIRE(in.mask.dtype == DNUFFT_U8 && in.mask.shape[0] == nrows &&
                   in.mask.shape[1] == nchan,
               ST_BADARG, "mask must be uint8 of shape (nrows, nchan)");
  }
  return in;
}

// frequencies positive and ascending (DUCC's Baselines, wgridder.h:285-296)
static void check_freq(const Inputs &in, cudaStream_t st) {
  const int64_t nchan = in.freq.shape[0];
  if (nchan == 0) return;
  std::vector<double> f(static_cast<size_t>(nchan), 0.);
  if (in.freq.stride[0] == 1) {
    DN_CUDA(cudaMemcpyAsync(f.data(), in.freq.p, size_t(nchan) * 8, cudaMemcpyDeviceToHost, st));
  } else {
    DN_CUDA(cudaMemcpy2DAsync(f.data(), 8, in.freq.p, size_t(in.freq.stride[0]) * 8, 8,
                              size_t(nchan), cudaMemcpyDeviceToHost, st));
  }
  DN_CUDA(cudaStreamSynchronize(st));
  for (int64_t i = 0; i < nchan; ++i) {
    DN_REQUIRE(f[size_t(i)] > 0, ST_BADARG, "negative channel frequency encountered");
    if (i > 0)
      DN_REQUIRE(f[size_t(i)] >= f[size_t(i - 1)], ST_BADARG,
                 "channel frequencies must be sorted in ascending order");
  }
}

// active visibilities, compacted (in input order), and their w range
template <typename T, typename C> struct Compacted {
  uint32_t nvis = 0;
  double wmin = 0, wmax = 0;
  Buf coord, wv, idx, val;
};

template <typename T, typename C>
static void compact(const Inputs &in, bool gridding, const Params *shift,
                    Compacted<T, C> &out, cudaStream_t st) {
  const int64_t n = in.c.nrows * in.c.nchan;
  if (n == 0) return;
  const cplx<T> *vis = gridding ? static_cast<const cplx<T> *>(in.vis.p) : nullptr;
  Buf flag(size_t(n) * 4, st), scan(size_t(n) * 4, st);
  Buf sws(scan_workspace_bytes(uint64_t(n)), st);
  Buf words(32, st);
  k_wg_flags<T><<<grid_for(n), 256, 0, st>>>(in.c, vis, in.vis.stride[0], in.vis.stride[1],
                                             ptr<uint32_t>(flag));
  DN_LAUNCHED();
  exclusive_scan(ptr<uint32_t>(flag), ptr<uint32_t>(scan), uint64_t(n), ptr<uint32_t>(sws), st);
  k_wg_count<<<1, 32, 0, st>>>(ptr<uint32_t>(flag), ptr<uint32_t>(scan), n, ptr<uint32_t>(words));
  DN_LAUNCHED();
  uint32_t cnt = 0;
  DN_CUDA(cudaMemcpyAsync(&cnt, words.p, 4, cudaMemcpyDeviceToHost, st));
  DN_CUDA(cudaStreamSynchronize(st));
  out.nvis = cnt;
  if (cnt == 0) return;
  out.coord = Buf(size_t(cnt) * 16, st);
  out.wv = Buf(size_t(cnt) * 8, st);
  out.idx = Buf(size_t(cnt) * 4, st);
  if (gridding) out.val = Buf(size_t(cnt) * sizeof(cplx<C>), st);
  unsigned long long init[2] = {~0ull, 0ull};
  unsigned long long *wr = reinterpret_cast<unsigned long long *>(ptr<char>(words) + 16);
  DN_CUDA(cudaMemcpyAsync(wr, init, 16, cudaMemcpyHostToDevice, st));
  k_wg_compact<T, C><<<grid_for(n), 256, 0, st>>>(
      in.c, vis, in.vis.stride[0], in.vis.stride[1], ptr<uint32_t>(flag), ptr<uint32_t>(scan),
      shift ? shift->lshift : 0., shift ? shift->mshift : 0., shift ? shift->nshift : 0.,
      ptr<double>(out.coord), ptr<double>(out.wv), ptr<uint32_t>(out.idx),
      gridding ? ptr<cplx<C>>(out.val) : nullptr, wr);
  DN_LAUNCHED();
  if (in.c.do_w) {
    unsigned long long got[2];
    DN_CUDA(cudaMemcpyAsync(got, wr, 16, cudaMemcpyDeviceToHost, st));
    DN_CUDA(cudaStreamSynchronize(st));
    std::memcpy(&out.wmin, &got[0], 8);
    std::memcpy(&out.wmax, &got[1], 8);
  }
}

// w range over the active visibilities, before the centre phases are known
// (the parameter choice needs it): a compaction without values
template <typename T>
static void scan_w(const Inputs &in, bool gridding, uint32_t &nvis, double &wmin, double &wmax,
                   cudaStream_t st) {
  Compacted<T, T> c;
  compact<T, T>(in, gridding, nullptr, c, st);
  nvis = c.nvis;
  wmin = c.wmin;
  wmax = c.wmax;
}

// plane order: visibilities sorted by first plane; start[p] = first of plane p
template <typename C> struct PlaneOrder {
  Buf coord, wv, idx, val, key;
  std::vector<uint32_t> start;   // nplanes + 1
};

template <typename T, typename C>
static void plane_order(Compacted<T, C> &cv, const Params &P, bool gridding,
                        PlaneOrder<C> &po, cudaStream_t st) {
  const uint32_t n = cv.nvis;
  const int64_t np = P.nplanes;
  Buf key(size_t(n) * 4, st), ord(size_t(n) * 4, st), starts(size_t(np + 1) * 4, st);
  k_wg_minplane<<<grid_for(n), 256, 0, st>>>(ptr<double>(cv.wv), n, P.wmin, P.xdw, P.W,
                                             ptr<uint32_t>(key), ptr<uint32_t>(ord));
  DN_LAUNCHED();
  int keybits = 1;
  while ((int64_t(1) << keybits) <= np) ++keybits;
  Buf rws(radix_workspace_bytes(n, keybits), st);
  radix_sort_pairs(ptr<uint32_t>(key), ptr<uint32_t>(ord), n, keybits, rws.p, st);
  k_wg_plane_starts<<<grid_for(int64_t(n) + 1), 256, 0, st>>>(ptr<uint32_t>(key), n,
                                                               uint32_t(np), ptr<uint32_t>(starts));
  DN_LAUNCHED();
  po.coord = Buf(size_t(n) * 16, st);
  po.wv = Buf(size_t(n) * 8, st);
  po.idx = Buf(size_t(n) * 4, st);
  if (gridding) po.val = Buf(size_t(n) * sizeof(cplx<C>), st);
  k_wg_gather<C><<<grid_for(n), 256, 0, st>>>(
      ptr<uint32_t>(ord), n, ptr<double>(cv.coord), ptr<double>(cv.wv), ptr<uint32_t>(cv.idx),
      gridding ? ptr<cplx<C>>(cv.val) : nullptr, ptr<double>(po.coord), ptr<double>(po.wv),
      ptr<uint32_t>(po.idx), gridding ? ptr<cplx<C>>(po.val) : nullptr);
  DN_LAUNCHED();
  po.key = std::move(key);
  po.start.assign(size_t(np + 1), 0u);
  DN_CUDA(cudaMemcpyAsync(po.start.data(), starts.p, size_t(np + 1) * 4,
                          cudaMemcpyDeviceToHost, st));
  DN_CUDA(cudaStreamSynchronize(st));
}

// planes [p0, p1) of this call (the caller's share of a split)
static void plane_range(const Params &P, const dnufft_wgrid_opts &o, int64_t &p0, int64_t &p1) {
  p0 = std::max<int64_t>(0, o.plane_begin);
  p1 = o.plane_count > 0 ? std::min<int64_t>(P.nplanes, p0 + o.plane_count) : P.nplanes;
}

static dnufft_opts nufft_opts(const Params &P, double psx, double psy, const dnufft_wgrid_opts &o) {
  dnufft_opts no;
  dnufft_default_opts(&no, 0);
  no.nthreads = o.nthreads;
  no.sigma_min = o.sigma_min;
  no.sigma_max = o.sigma_max;
  no.periodicity[0] = 1. / psx;
  no.periodicity[1] = 1. / psy;
  no.force_kernel = P.kidx;
  no.force_nover[0] = P.nu;
  no.force_nover[1] = P.nv;
  return no;
}

static ImgGeom img_geom(const Params &P, int64_t nx, int64_t ny, double psx, double psy) {
  ImgGeom g;
  g.nx = nx;
  g.ny = ny;
  g.x0 = P.lshift - 0.5 * double(nx) * psx;
  g.y0 = P.mshift - 0.5 * double(ny) * psy;
  g.psx = psx;
  g.psy = psy;
  g.nshift = P.nshift;
  return g;
}

static void report(const Params &P, const char *what, int64_t nx, int64_t ny, uint32_t nvis,
                   bool do_w) {
  std::printf("%s: dirty %lld x %lld, grid %lld x %lld", what, (long long)nx, (long long)ny,
              (long long)P.nu, (long long)P.nv);
  if (do_w) std::printf(" x %lld planes", (long long)P.nplanes);
  std::printf(", supp %d, ofactor %.3f, nvis %u", P.W, P.ofactor, nvis);
  if (do_w) std::printf(", dw %.6g, wmin %.6g, nshift %.6g", P.dw, P.wmin, P.nshift);
  std::printf("\n");
}

// The visibilities indexed once by (first w plane, tile), so that no plane
// sorts its own (null where the keys do not fit 32 bits: then every plane's
// transform sorts its range).  key: the first plane of every compacted
// visibility.
struct Grouped {
  GroupedPlan *gp = nullptr;
  cudaStream_t st = nullptr;
  Grouped(const double *coord, uint32_t n, const uint32_t *key, const Params &P, int64_t nx,
          int64_t ny, double eps, bool f64, const dnufft_opts &no, cudaStream_t s)
      : st(s) {
    const int64_t shape[2] = {nx, ny};
    gp = grouped_plan_create(coord, n, key, uint32_t(P.nplanes), shape, eps, f64, no, s,
                             nullptr);
  }
  Grouped(const Grouped &) = delete;
  Grouped &operator=(const Grouped &) = delete;
  ~Grouped() { grouped_plan_destroy(gp, st); }
};

static void plane_keys(const double *wv, uint32_t n, const Params &P, Buf &key, cudaStream_t st) {
  Buf ord(size_t(n) * 4, st);
  key = Buf(size_t(n) * 4, st);
  k_wg_minplane<<<grid_for(n), 256, 0, st>>>(wv, n, P.wmin, P.xdw, P.W, ptr<uint32_t>(key),
                                             ptr<uint32_t>(ord));
  DN_LAUNCHED();
}

// ---- vis2dirty
template <typename T, typename C>
static void vis2dirty_t(const Inputs &in, double psx, double psy, double eps,
                        const dnufft_wgrid_opts &o, const Arr &dirty, cudaStream_t st) {
  const int64_t nx = dirty.shape[0], ny = dirty.shape[1];
  T *dp = static_cast<T *>(dirty.p);
  const bool do_w = o.do_wgridding != 0;
  uint32_t nvis;
  double wmin_d, wmax_d;
  scan_w<T>(in, true, nvis, wmin_d, wmax_d, st);
  k_wg_zero_dirty<T><<<grid_for(nx * ny), 256, 0, st>>>(dp, nx, ny, dirty.stride[0],
                                                        dirty.stride[1]);
  DN_LAUNCHED();
  if (nvis == 0) return;
  const Params P = choose(nx, ny, psx, psy, eps, sizeof(T) == 4, o, nvis, wmin_d, wmax_d);
  if (o.verbosity > 0) report(P, "vis2dirty", nx, ny, nvis, do_w);
  int64_t pl0, pl1;
  plane_range(P, o, pl0, pl1);
  if (do_w ? pl1 <= pl0 : pl0 > 0) return;   // no plane of this share
  Compacted<T, C> cv;
  compact<T, C>(in, true, &P, cv, st);
  const dnufft_opts no = nufft_opts(P, psx, psy, o);
  const int cdt = sizeof(C) == 4 ? DNUFFT_C64 : DNUFFT_C128;
  Buf img(size_t(nx * ny) * sizeof(cplx<C>), st);
  dnufft_array a_img = dev_array(img.p, cdt, 2, nx, ny);
  if (!do_w) {
    dnufft_array a_v = dev_array(cv.val.p, cdt, 1, cv.nvis);
    dnufft_array a_c = dev_array(cv.coord.p, DNUFFT_F64, 2, cv.nvis, 2);
    check_nufft(dnufft_nu2u(&a_v, &a_c, 0, eps, &a_img, &no, st));
    k_wg_real<C, T><<<grid_for(nx * ny), 256, 0, st>>>(ptr<cplx<C>>(img), nx, ny, dp,
                                                       dirty.stride[0], dirty.stride[1]);
    DN_LAUNCHED();
    return;
  }
  Buf pm(size_t(nx * ny) * 8, st);
  k_wg_pixel_nm1<<<grid_for(nx * ny), 256, 0, st>>>(img_geom(P, nx, ny, psx, psy),
                                                    ptr<double>(pm));
  DN_LAUNCHED();
  const KernelPoly<C> kp = make_poly<C>(P.W, P.beta, P.e0);
  const ImgGeom g = img_geom(P, nx, ny, psx, psy);
  Buf pv(size_t(cv.nvis) * sizeof(cplx<C>), st);
  Buf key;
  plane_keys(ptr<double>(cv.wv), cv.nvis, P, key, st);
  Grouped gr(ptr<double>(cv.coord), cv.nvis, ptr<uint32_t>(key), P, nx, ny, eps, sizeof(C) == 8,
             no, st);
  const CorrNodes cn = make_nodes(P.W, P.beta, P.e0);
  if (gr.gp) {
    for (int64_t p = pl0; p < pl1; ++p) {
      const uint32_t g0 = uint32_t(std::max<int64_t>(0, p - P.W + 1)), g1 = uint32_t(p + 1);
      // values of every visibility for plane p (zero outside its planes; the
      // chunk list of the run reads only the plane's own)
      k_wg_plane_vals<C><<<grid_for(cv.nvis), 256, 0, st>>>(
          ptr<cplx<C>>(cv.val), ptr<double>(cv.wv), ptr<uint32_t>(key), 0, cv.nvis, kp, P.W,
          int(p), P.wmin, P.xdw, ptr<cplx<C>>(pv));
      DN_LAUNCHED();
      if (!grouped_nu2u(gr.gp, g0, g1, pv.p, img.p, false, st)) continue;
      k_wg_screen_add<C, T><<<grid_for(nx * ny), 256, 0, st>>>(
          ptr<cplx<C>>(img), ptr<double>(pm), g, P.wmin + double(p) * P.dw, dp, dirty.stride[0],
          dirty.stride[1]);
      DN_LAUNCHED();
    }
    k_wg_correct<T><<<grid_for(nx * ny), 256, 0, st>>>(dp, dirty.stride[0], dirty.stride[1], g,
                                                       cn, P.dw, o.divide_by_n);
    DN_LAUNCHED();
    return;
  }
  PlaneOrder<C> po;
  plane_order<T, C>(cv, P, true, po, st);
  for (int64_t p = pl0; p < pl1; ++p) {
    const uint32_t lo = po.start[size_t(std::max<int64_t>(0, p - P.W + 1))];
    const uint32_t hi = po.start[size_t(p + 1)];
    if (hi <= lo) continue;
    const uint32_t cnt = hi - lo;
    k_wg_plane_vals<C><<<grid_for(cnt), 256, 0, st>>>(ptr<cplx<C>>(po.val), ptr<double>(po.wv),
                                                      ptr<uint32_t>(po.key), lo, cnt, kp, P.W,
                                                      int(p), P.wmin, P.xdw, ptr<cplx<C>>(pv));
    DN_LAUNCHED();
    dnufft_array a_v = dev_array(pv.p, cdt, 1, cnt);
    dnufft_array a_c = dev_array(ptr<double>(po.coord) + 2 * size_t(lo), DNUFFT_F64, 2, cnt, 2);
    check_nufft(dnufft_nu2u(&a_v, &a_c, 0, eps, &a_img, &no, st));
    k_wg_screen_add<C, T><<<grid_for(nx * ny), 256, 0, st>>>(
        ptr<cplx<C>>(img), ptr<double>(pm), g, P.wmin + double(p) * P.dw, dp, dirty.stride[0],
        dirty.stride[1]);
    DN_LAUNCHED();
  }
  k_wg_correct<T><<<grid_for(nx * ny), 256, 0, st>>>(dp, dirty.stride[0], dirty.stride[1], g, cn,
                                                     P.dw, o.divide_by_n);
  DN_LAUNCHED();
}

// ---- dirty2vis
template <typename T, typename C>
static void dirty2vis_t(const Inputs &in, const Arr &dirty, double psx, double psy, double eps,
                        const dnufft_wgrid_opts &o, const Arr &vis, cudaStream_t st) {
  const int64_t nx = dirty.shape[0], ny = dirty.shape[1];
  const T *dp = static_cast<const T *>(dirty.p);
  cplx<T> *vp = static_cast<cplx<T> *>(vis.p);
  const bool do_w = o.do_wgridding != 0;
  uint32_t nvis;
  double wmin_d, wmax_d;
  scan_w<T>(in, false, nvis, wmin_d, wmax_d, st);
  if (in.c.nrows * in.c.nchan > 0) {
    k_wg_zero_vis<T><<<grid_for(in.c.nrows * in.c.nchan), 256, 0, st>>>(in.c, vp, vis.stride[0],
                                                                        vis.stride[1]);
    DN_LAUNCHED();
  }
  if (nvis == 0) return;
  const Params P = choose(nx, ny, psx, psy, eps, sizeof(T) == 4, o, nvis, wmin_d, wmax_d);
  if (o.verbosity > 0) report(P, "dirty2vis", nx, ny, nvis, do_w);
  int64_t pl0, pl1;
  plane_range(P, o, pl0, pl1);
  if (do_w ? pl1 <= pl0 : pl0 > 0) return;   // no plane of this share: zeros
  Compacted<T, C> cv;
  compact<T, C>(in, false, &P, cv, st);
  const dnufft_opts no = nufft_opts(P, psx, psy, o);
  const int cdt = sizeof(C) == 4 ? DNUFFT_C64 : DNUFFT_C128;
  const ImgGeom g = img_geom(P, nx, ny, psx, psy);
  const CorrNodes cn = make_nodes(P.W, P.beta, P.e0);
  Buf img0(size_t(nx * ny) * sizeof(C), st), img(size_t(nx * ny) * sizeof(cplx<C>), st);
  k_wg_dirty_in<T, C><<<grid_for(nx * ny), 256, 0, st>>>(dp, dirty.stride[0], dirty.stride[1], g,
                                                         cn, P.dw, do_w ? 1 : 0,
                                                         o.divide_by_n, ptr<C>(img0));
  DN_LAUNCHED();
  dnufft_array a_img = dev_array(img.p, cdt, 2, nx, ny);
  Buf acc(size_t(cv.nvis) * sizeof(cplx<C>), st);
  if (!do_w) {
    k_wg_real_to_complex<C><<<grid_for(nx * ny), 256, 0, st>>>(ptr<C>(img0), nx * ny,
                                                               ptr<cplx<C>>(img));
    DN_LAUNCHED();
    dnufft_array a_c = dev_array(cv.coord.p, DNUFFT_F64, 2, cv.nvis, 2);
    dnufft_array a_o = dev_array(acc.p, cdt, 1, cv.nvis);
    check_nufft(dnufft_u2nu(&a_img, &a_c, 1, eps, &a_o, &no, st));
    k_wg_scatter<T, C><<<grid_for(cv.nvis), 256, 0, st>>>(
        ptr<cplx<C>>(acc), ptr<double>(cv.coord), ptr<double>(cv.wv), ptr<uint32_t>(cv.idx),
        cv.nvis, in.c, P.lshift, P.mshift, 0., vp, vis.stride[0], vis.stride[1]);
    DN_LAUNCHED();
    return;
  }
  Buf pm(size_t(nx * ny) * 8, st);
  k_wg_pixel_nm1<<<grid_for(nx * ny), 256, 0, st>>>(g, ptr<double>(pm));
  DN_LAUNCHED();
  const KernelPoly<C> kp = make_poly<C>(P.W, P.beta, P.e0);
  DN_CUDA(cudaMemsetAsync(acc.p, 0, size_t(cv.nvis) * sizeof(cplx<C>), st));
  Buf res(size_t(cv.nvis) * sizeof(cplx<C>), st);
  Buf key;
  plane_keys(ptr<double>(cv.wv), cv.nvis, P, key, st);
  Grouped gr(ptr<double>(cv.coord), cv.nvis, ptr<uint32_t>(key), P, nx, ny, eps, sizeof(C) == 8,
             no, st);
  if (gr.gp) {
    for (int64_t p = pl0; p < pl1; ++p) {
      const uint32_t g0 = uint32_t(std::max<int64_t>(0, p - P.W + 1)), g1 = uint32_t(p + 1);
      k_wg_screen_apply<C><<<grid_for(nx * ny), 256, 0, st>>>(
          ptr<C>(img0), ptr<double>(pm), nx * ny, P.wmin + double(p) * P.dw, ptr<cplx<C>>(img));
      DN_LAUNCHED();
      if (!grouped_u2nu(gr.gp, g0, g1, img.p, res.p, true, st)) continue;
      k_wg_degrid_acc_all<C><<<grid_for(cv.nvis), 256, 0, st>>>(
          ptr<cplx<C>>(res), ptr<double>(cv.wv), ptr<uint32_t>(key), cv.nvis, kp, P.W, int(p),
          P.wmin, P.xdw, ptr<cplx<C>>(acc));
      DN_LAUNCHED();
    }
    k_wg_scatter<T, C><<<grid_for(cv.nvis), 256, 0, st>>>(
        ptr<cplx<C>>(acc), ptr<double>(cv.coord), ptr<double>(cv.wv), ptr<uint32_t>(cv.idx),
        cv.nvis, in.c, P.lshift, P.mshift, P.nshift, vp, vis.stride[0], vis.stride[1]);
    DN_LAUNCHED();
    return;
  }
  PlaneOrder<C> po;
  plane_order<T, C>(cv, P, false, po, st);
  for (int64_t p = pl0; p < pl1; ++p) {
    const uint32_t lo = po.start[size_t(std::max<int64_t>(0, p - P.W + 1))];
    const uint32_t hi = po.start[size_t(p + 1)];
    if (hi <= lo) continue;
    const uint32_t cnt = hi - lo;
    k_wg_screen_apply<C><<<grid_for(nx * ny), 256, 0, st>>>(
        ptr<C>(img0), ptr<double>(pm), nx * ny, P.wmin + double(p) * P.dw, ptr<cplx<C>>(img));
    DN_LAUNCHED();
    dnufft_array a_c = dev_array(ptr<double>(po.coord) + 2 * size_t(lo), DNUFFT_F64, 2, cnt, 2);
    dnufft_array a_o = dev_array(res.p, cdt, 1, cnt);
    check_nufft(dnufft_u2nu(&a_img, &a_c, 1, eps, &a_o, &no, st));
    k_wg_degrid_acc<C><<<grid_for(cnt), 256, 0, st>>>(ptr<cplx<C>>(res), ptr<double>(po.wv),
                                                      ptr<uint32_t>(po.key), lo, cnt, kp, P.W,
                                                      int(p), P.wmin, P.xdw, ptr<cplx<C>>(acc));
    DN_LAUNCHED();
  }
  k_wg_scatter<T, C><<<grid_for(cv.nvis), 256, 0, st>>>(
      ptr<cplx<C>>(acc), ptr<double>(po.coord), ptr<double>(po.wv), ptr<uint32_t>(po.idx),
      cv.nvis, in.c, P.lshift, P.mshift, P.nshift, vp, vis.stride[0], vis.stride[1]);
  DN_LAUNCHED();
}

static void check_common(double psx, double psy, double eps, const dnufft_wgrid_opts *o) {
  DN_REQUIRE(o != nullptr, ST_BADARG, "null options");
  DN_REQUIRE(eps > 0, ST_BADARG, "epsilon must be positive");
  DN_REQUIRE(psx > 0, ST_BADARG, "pixsize_x must be positive");
  DN_REQUIRE(psy > 0, ST_BADARG, "pixsize_y must be positive");
}

static void check_dirty(const Arr &d, bool f64) {
  DN_REQUIRE(d.dtype == (f64 ? DNUFFT_F64 : DNUFFT_F32), ST_BADARG,
             "dirty must be real of the visibilities' precision");
  DN_REQUIRE((d.shape[0] & 1) == 0 && (d.shape[1] & 1) == 0, ST_BADARG,
             "nx_dirty and ny_dirty must be even");
}

static void check_wgt(const Inputs &in, bool f64) {
  if (!in.wgt.p) return;
  DN_REQUIRE(in.wgt.dtype == (f64 ? DNUFFT_F64 : DNUFFT_F32), ST_BADARG,
             "wgt must be real of the visibilities' precision");
  DN_REQUIRE(in.wgt.shape[0] == in.c.nrows && in.wgt.shape[1] == in.c.nchan, ST_BADARG,
             "wgt must have shape (nrows, nchan)");
}

static void vis2dirty_impl(const dnufft_array *uvw, const dnufft_array *freq,
                           const dnufft_array *vis, const dnufft_array *wgt,
                           const dnufft_array *mask, double psx, double psy, double eps,
                           const dnufft_wgrid_opts *o, dnufft_array *dirty_, cudaStream_t st) {
  check_common(psx, psy, eps, o);
  Inputs in = parse(uvw, freq, vis, true, wgt, mask, *o);
  const bool f64 = in.vis.dtype == DNUFFT_C128;
  check_wgt(in, f64);
  Arr dirty = arr_of(dirty_, "dirty", 2);
  check_dirty(dirty, f64);
  check_freq(in, st);
  if (f64)
    vis2dirty_t<double, double>(in, psx, psy, eps, *o, dirty, st);
  else if (o->double_precision_accumulation)
    vis2dirty_t<float, double>(in, psx, psy, eps, *o, dirty, st);
  else
    vis2dirty_t<float, float>(in, psx, psy, eps, *o, dirty, st);
}

static void dirty2vis_impl(const dnufft_array *uvw, const dnufft_array *freq,
                           const dnufft_array *dirty_, const dnufft_array *wgt,
                           const dnufft_array *mask, double psx, double psy, double eps,
                           const dnufft_wgrid_opts *o, dnufft_array *vis_, cudaStream_t st) {
  check_common(psx, psy, eps, o);
  Inputs in = parse(uvw, freq, vis_, true, wgt, mask, *o);
  const bool f64 = in.vis.dtype == DNUFFT_C128;
  check_wgt(in, f64);
  Arr dirty = arr_of(dirty_, "dirty", 2);
  check_dirty(dirty, f64);
  check_freq(in, st);
  if (f64)
    dirty2vis_t<double, double>(in, dirty, psx, psy, eps, *o, in.vis, st);
  else
    dirty2vis_t<float, float>(in, dirty, psx, psy, eps, *o, in.vis, st);
}

static void params_impl(const dnufft_array *uvw, const dnufft_array *freq,
                        const dnufft_array *vis, const dnufft_array *wgt,
                        const dnufft_array *mask, int64_t nx, int64_t ny, double psx, double psy,
                        double eps, int gridding, const dnufft_wgrid_opts *o,
                        dnufft_wgrid_info *info, cudaStream_t st) {
  check_common(psx, psy, eps, o);
  DN_REQUIRE(info != nullptr, ST_BADARG, "null info");
  Inputs in = parse(uvw, freq, vis, gridding != 0, wgt, mask, *o);
  // precision: the visibilities' (gridding) or the weights' (else double)
  bool f64 = true;
  if (in.vis.p) f64 = in.vis.dtype == DNUFFT_C128;
  else if (in.wgt.p) f64 = in.wgt.dtype == DNUFFT_F64;
  check_wgt(in, f64);
  check_freq(in, st);
  uint32_t nvis;
  double wmin_d, wmax_d;
  if (f64)
    scan_w<double>(in, gridding != 0, nvis, wmin_d, wmax_d, st);
  else
    scan_w<float>(in, gridding != 0, nvis, wmin_d, wmax_d, st);
  std::memset(info, 0, sizeof(*info));
  info->nvis = nvis;
  if (nvis == 0) return;
  const Params P = choose(nx, ny, psx, psy, eps, !f64, *o, nvis, wmin_d, wmax_d);
  info->kernel_index = P.kidx;
  info->supp = P.W;
  info->nu = P.nu;
  info->nv = P.nv;
  info->nplanes = P.nplanes;
  info->dw = P.dw;
  info->wmin = P.wmin;
  info->nshift = P.nshift;
}

#define DN_WG_GUARD(body)                                        \
  try {                                                          \
    body;                                                        \
    dnufft::set_last_error("");                                  \
    return DNUFFT_OK;                                            \
  } catch (const dnufft::Error &e) {                             \
    dnufft::set_last_error(e.what());                            \
    return e.code;                                               \
  } catch (const std::bad_alloc &) {                             \
    dnufft::set_last_error("host allocation failed");            \
    return DNUFFT_ERR_OOM;                                       \
  } catch (const std::exception &e) {                            \
    dnufft::set_last_error(e.what());                            \
    return DNUFFT_ERR_INTERNAL;                                  \
  }

extern "C" {

void dnufft_wgrid_default_opts(dnufft_wgrid_opts *o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->nthreads = 1;
  o->sigma_min = 1.1;
  o->sigma_max = 2.6;
  o->divide_by_n = 1;
  o->allow_nshift = 1;
}

int dnufft_vis2dirty(const dnufft_array *uvw, const dnufft_array *freq, const dnufft_array *vis,
                     const dnufft_array *wgt, const dnufft_array *mask, double pixsize_x,
                     double pixsize_y, double epsilon, const dnufft_wgrid_opts *opts,
                     dnufft_array *dirty, void *stream) {
  DN_WG_GUARD(dnufft::wg::vis2dirty_impl(uvw, freq, vis, wgt, mask, pixsize_x, pixsize_y, epsilon,
                                         opts, dirty, static_cast<cudaStream_t>(stream)))
}

int dnufft_dirty2vis(const dnufft_array *uvw, const dnufft_array *freq, const dnufft_array *dirty,
                     const dnufft_array *wgt, const dnufft_array *mask, double pixsize_x,
                     double pixsize_y, double epsilon, const dnufft_wgrid_opts *opts,
                     dnufft_array *vis, void *stream) {
  DN_WG_GUARD(dnufft::wg::dirty2vis_impl(uvw, freq, dirty, wgt, mask, pixsize_x, pixsize_y, epsilon,
                                         opts, vis, static_cast<cudaStream_t>(stream)))
}

int dnufft_wgrid_params(const dnufft_array *uvw, const dnufft_array *freq, const dnufft_array *vis,
                        const dnufft_array *wgt, const dnufft_array *mask, int64_t nx, int64_t ny,
                        double pixsize_x, double pixsize_y, double epsilon, int gridding,
                        const dnufft_wgrid_opts *opts, dnufft_wgrid_info *info, void *stream) {
  DN_WG_GUARD(dnufft::wg::params_impl(uvw, freq, vis, wgt, mask, nx, ny, pixsize_x, pixsize_y,
                                      epsilon, gridding, opts, info,
                                      static_cast<cudaStream_t>(stream)))
}

}  // extern "C"

}  // namespace wg
}  // namespace dnufft
