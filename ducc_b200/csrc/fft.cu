// Oversampled-grid FFTs and the grid correction (deconvolution + crop / pad).
//
// Each CTA transforms 'nl' lines of length n held in shared memory (element k of
// line l at s[k*nl+l]) with a mixed-radix Stockham FFT (radices 2,3,4,5,7,8,11;
// DUCC's oversampled sizes are 2*good_size_complex(...), always 11-smooth).
// Every stage is done in place: each thread first gathers its butterflies into
// registers, the block synchronises, then it writes the outputs.  Twiddles come
// from an FP64-accurate table of n entries.
//
// The NUFFT needs only the N kept frequencies of every axis, so (as DUCC does,
// src/ducc0/nufft/nufft.h:1287-1298, :1345-1356, :1743-1773, :1824-1854) the
// second and third axes are transformed only on kept index ranges.  In addition
//  - type 1: the last pass multiplies by the correction factors and writes
//    straight into the caller's uniform array in DUCC's output order
//    (comp_indices, nufft.h:142-151), so no separate correction pass is run;
//  - type 2: the first pass gathers the caller's uniform array, multiplies by
//    the correction factors and zero-pads in shared memory, so the oversampled
//    grid is never zeroed or written before the first FFT.
#include "common.cuh"
#include "fft_pencil_plan.h"
#include "kernels.h"

#include <algorithm>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>

namespace dnufft {

constexpr int FFT_MAXE = 16;   // elements per thread per stage

struct AxisMap {
  int N, n;   // kept count, full length
};

// kept index x in [0,N) -> grid index: low half first, then high half
__device__ __forceinline__ int kept_to_grid(int x, int N, int n) {
  int lo = (N + 1) / 2;
  return x < lo ? x : x + n - N;
}
// grid index -> uniform index along an axis and the correction-factor index
// (inverse of comp_indices' i2 = (n - N/2 + i) mod n)
__device__ __forceinline__ void grid_to_uni(int c, int N, int n, bool fft_order, int &iuni,
                                            int &icf) {
  int j = c + N / 2;
  if (j >= n) j -= n;
  icf = abs(N / 2 - j);
  int i1 = fft_order ? N - N / 2 + j : j;
  if (i1 >= N) i1 -= N;
  iuni = i1;
}

enum { IO_FULL = 0, IO_KEPT = 1, IO_UNI = 2 };

// element d of a 3-array held in a by-value kernel parameter, without dynamic
// indexing (which would force a local-memory copy of the whole parameter)
template <typename X> __device__ __forceinline__ X sel3(const X (&a)[3], int d) {
  return d == 0 ? a[0] : (d == 1 ? a[1] : a[2]);
}

struct LineSpec {
  int n;            // transform length
  int ax;           // transformed grid axis
  int64_t es;       // element stride in the grid
  int nlines;
  int cntb;         // line index L = a*cntb + b
  int64_t sa, sb;   // grid strides of a and b
  int axa, axb;     // grid axes of a and b (-1: unused)
  int kepta, keptb; // a / b enumerate kept indices of their axis
  int in_mode, out_mode;
  int nl;           // lines per CTA
};

struct UniSpec {
  void *ptr;
  int64_t stride[3];
  const double *corfac[3];
  int N[3];
  int n[3];
  bool fft_order;
};

template <typename T>
__device__ __forceinline__ cplx<T> twiddle(const cplx<T> *__restrict__ tw, int t, bool fwd) {
  cplx<T> w = __ldg(tw + t);
  if (!fwd) w.y = -w.y;
  return w;
}

// y = DFT_R(a) with sign from fwd; generic direct form for odd radices
template <typename T, int R>
__device__ __forceinline__ void dft_small(cplx<T> (&a)[R], const cplx<T> *__restrict__ tw, int n,
                                          bool fwd) {
  if constexpr (R == 2) {
    cplx<T> t = a[1];
    a[1] = csub<T>(a[0], t);
    a[0] = cadd<T>(a[0], t);
  } else if constexpr (R == 4) {
    cplx<T> s02 = cadd<T>(a[0], a[2]), d02 = csub<T>(a[0], a[2]);
    cplx<T> s13 = cadd<T>(a[1], a[3]), d13 = csub<T>(a[1], a[3]);
    // multiply d13 by -i (forward) or +i (backward)
    cplx<T> r = fwd ? mkc<T>(d13.y, -d13.x) : mkc<T>(-d13.y, d13.x);
    a[0] = cadd<T>(s02, s13);
    a[2] = csub<T>(s02, s13);
    a[1] = cadd<T>(d02, r);
    a[3] = csub<T>(d02, r);
  } else if constexpr (R == 8) {
    cplx<T> e[4] = {a[0], a[2], a[4], a[6]};
    cplx<T> o[4] = {a[1], a[3], a[5], a[7]};
    dft_small<T, 4>(e, tw, n, fwd);
    dft_small<T, 4>(o, tw, n, fwd);
    const T h = T(0.70710678118654752440084436210485);
    const T s = fwd ? T(-1) : T(1);
    // W8^1 = h(1 + s i), W8^2 = s i, W8^3 = h(-1 + s i)
    cplx<T> o1 = mkc<T>(h * (o[1].x - s * o[1].y), h * (o[1].y + s * o[1].x));
    cplx<T> o2 = mkc<T>(-s * o[2].y, s * o[2].x);
    cplx<T> o3 = mkc<T>(h * (-o[3].x - s * o[3].y), h * (-o[3].y + s * o[3].x));
    a[0] = cadd<T>(e[0], o[0]);
    a[4] = csub<T>(e[0], o[0]);
    a[1] = cadd<T>(e[1], o1);
    a[5] = csub<T>(e[1], o1);
    a[2] = cadd<T>(e[2], o2);
    a[6] = csub<T>(e[2], o2);
    a[3] = cadd<T>(e[3], o3);
    a[7] = csub<T>(e[3], o3);
  } else {
    const int step = n / R;
    cplx<T> w[R];
#pragma unroll
    for (int m = 0; m < R; ++m) w[m] = twiddle<T>(tw, m * step, fwd);
    cplx<T> y[R];
#pragma unroll
    for (int q = 0; q < R; ++q) {
      cplx<T> acc = a[0];
#pragma unroll
      for (int m = 1; m < R; ++m) {
        cplx<T> t = cmul<T>(a[m], w[(m * q) % R]);
        acc = cadd<T>(acc, t);
      }
      y[q] = acc;
    }
#pragma unroll
    for (int q = 0; q < R; ++q) a[q] = y[q];
  }
}

template <typename T, int R>
__device__ __forceinline__ void stockham_stage(cplx<T> *s, int n, int nl, int Ns,
                                               const cplx<T> *__restrict__ tw, bool fwd) {
  constexpr int QM = FFT_MAXE / R + 1;
  const int B = (n / R) * nl;
  const int NT = blockDim.x;
  const int tstep = n / (Ns * R);
  cplx<T> v[QM][R];
#pragma unroll
  for (int q = 0; q < QM; ++q) {
    int b = threadIdx.x + q * NT;
    if (b < B) {
      int l = b % nl, j = b / nl;
      int k = j % Ns;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        cplx<T> x = s[(j + r * (n / R)) * nl + l];
        if (r > 0 && k > 0) x = cmul<T>(x, twiddle<T>(tw, k * r * tstep, fwd));
        v[q][r] = x;
      }
      dft_small<T, R>(v[q], tw, n, fwd);
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < QM; ++q) {
    int b = threadIdx.x + q * NT;
    if (b < B) {
      int l = b % nl, j = b / nl;
      int k = j % Ns;
      int base = (j - k) * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) s[(base + r * Ns) * nl + l] = v[q][r];
    }
  }
  __syncthreads();
}

template <typename T>
__device__ void fft_lines(cplx<T> *s, int n, int nl, const FFTAxisPlan &p, bool fwd) {
  const cplx<T> *tw = static_cast<const cplx<T> *>(p.tw);
  int Ns = 1;
  for (int f = 0; f < p.nfac; ++f) {
    int R = p.fac[f];
    switch (R) {
      case 2: stockham_stage<T, 2>(s, n, nl, Ns, tw, fwd); break;
      case 3: stockham_stage<T, 3>(s, n, nl, Ns, tw, fwd); break;
      case 4: stockham_stage<T, 4>(s, n, nl, Ns, tw, fwd); break;
      case 5: stockham_stage<T, 5>(s, n, nl, Ns, tw, fwd); break;
      case 7: stockham_stage<T, 7>(s, n, nl, Ns, tw, fwd); break;
      case 8: stockham_stage<T, 8>(s, n, nl, Ns, tw, fwd); break;
      case 11: stockham_stage<T, 11>(s, n, nl, Ns, tw, fwd); break;
      default: break;   // excluded on the host
    }
    Ns *= R;
  }
}

__device__ __forceinline__ int64_t line_base(const LineSpec &ls, const int (&Nk)[3],
                                             const int (&nk)[3], int L, int &ia, int &ib) {
  int a = L / ls.cntb, b = L - (L / ls.cntb) * ls.cntb;
  ia = (ls.axa >= 0 && ls.kepta) ? kept_to_grid(a, sel3(Nk, ls.axa), sel3(nk, ls.axa)) : a;
  ib = (ls.axb >= 0 && ls.keptb) ? kept_to_grid(b, sel3(Nk, ls.axb), sel3(nk, ls.axb)) : b;
  return int64_t(ia) * ls.sa + int64_t(ib) * ls.sb;
}

// factor and uniform offset for the fixed (non-transformed) coordinates of a line
__device__ __forceinline__ void line_uni(const LineSpec &ls, const UniSpec &u, int ia, int ib,
                                         double &fac, int64_t &uoff) {
  fac = 1.0;
  uoff = 0;
  if (ls.axa >= 0) {
    int iu, icf;
    grid_to_uni(ia, sel3(u.N, ls.axa), sel3(u.n, ls.axa), u.fft_order, iu, icf);
    fac *= sel3(u.corfac, ls.axa)[icf];
    uoff += int64_t(iu) * sel3(u.stride, ls.axa);
  }
  if (ls.axb >= 0) {
    int iu, icf;
    grid_to_uni(ib, sel3(u.N, ls.axb), sel3(u.n, ls.axb), u.fft_order, iu, icf);
    fac *= sel3(u.corfac, ls.axb)[icf];
    uoff += int64_t(iu) * sel3(u.stride, ls.axb);
  }
}

template <typename T> constexpr int fft_max_threads() { return sizeof(T) == 4 ? 1024 : 512; }

template <typename T>
__global__ void __launch_bounds__(fft_max_threads<T>())
    k_fft_lines(cplx<T> *__restrict__ grid, LineSpec ls, FFTAxisPlan plan, UniSpec u, bool fwd) {
  extern __shared__ __align__(16) unsigned char smraw[];
  cplx<T> *s = reinterpret_cast<cplx<T> *>(smraw);
  const int n = ls.n, nl = ls.nl;
  const int L0 = blockIdx.x * nl;
  const int nloc = min(nl, ls.nlines - L0);
  const int N = sel3(u.N, ls.ax);
  const int total = n * nl;
  // ---------------- load
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    int l, k;
    if (ls.es == 1) {
      l = idx / n;
      k = idx - l * n;
    } else {
      k = idx / nl;
      l = idx - k * nl;
    }
    cplx<T> v = mkc<T>(T(0), T(0));
    if (l < nloc) {
      int ia, ib;
      int64_t base = line_base(ls, u.N, u.n, L0 + l, ia, ib);
      if (ls.in_mode == IO_FULL) {
        v = grid[base + int64_t(k) * ls.es];
      } else {
        int lo = (N + 1) / 2;
        bool kept = (k < lo) || (k >= n - N / 2);
        if (kept) {
          if (ls.in_mode == IO_KEPT) {
            v = grid[base + int64_t(k) * ls.es];
          } else {   // IO_UNI: gather caller's uniform array with correction
            double fac;
            int64_t uoff;
            line_uni(ls, u, ia, ib, fac, uoff);
            int iu, icf;
            grid_to_uni(k, N, n, u.fft_order, iu, icf);
            fac *= sel3(u.corfac, ls.ax)[icf];
            const cplx<T> *up = static_cast<const cplx<T> *>(u.ptr);
            cplx<T> x = up[uoff + int64_t(iu) * sel3(u.stride, ls.ax)];
            T f = T(fac);
            v = mkc<T>(x.x * f, x.y * f);
          }
        }
      }
    }
    s[k * nl + l] = v;
  }
  __syncthreads();
  fft_lines<T>(s, n, nl, plan, fwd);
  // ---------------- store
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    int l, k;
    if (ls.es == 1) {
      l = idx / n;
      k = idx - l * n;
    } else {
      k = idx / nl;
      l = idx - k * nl;
    }
    if (l >= nloc) continue;
    int ia, ib;
    int64_t base = line_base(ls, u.N, u.n, L0 + l, ia, ib);
    if (ls.out_mode == IO_FULL) {
      grid[base + int64_t(k) * ls.es] = s[k * nl + l];
    } else {
      int lo = (N + 1) / 2;
      bool kept = (k < lo) || (k >= n - N / 2);
      if (!kept) continue;
      if (ls.out_mode == IO_KEPT) {
        grid[base + int64_t(k) * ls.es] = s[k * nl + l];
      } else {   // IO_UNI: correction + crop into the caller's array
        double fac;
        int64_t uoff;
        line_uni(ls, u, ia, ib, fac, uoff);
        int iu, icf;
        grid_to_uni(k, N, n, u.fft_order, iu, icf);
        fac *= sel3(u.corfac, ls.ax)[icf];
        cplx<T> x = s[k * nl + l];
        T f = T(fac);
        cplx<T> *up = static_cast<cplx<T> *>(u.ptr);
        up[uoff + int64_t(iu) * sel3(u.stride, ls.ax)] = mkc<T>(x.x * f, x.y * f);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// FFT v2: one or more lines per CTA, stages in place with register staging,
// no runtime integer division in the butterfly indexing (lines per CTA is a
// power of two, the Stockham group index comes from a precomputed reciprocal),
// twiddles from a two-level table in shared memory (tw[t] = hi[t>>6]*lo[t&63]),
// and constant-folded butterflies for radices 2, 3, 4, 5, 7, 8, 11.
// ---------------------------------------------------------------------------
struct StageInfo {
  int nst;
  int R[24];
  int Ns[24];
  int tstep[24];
  uint32_t mul[24];   // ceil(2^32 / Ns)
  PencilPlan pen;     // pencil passes of the line kernels (pen.L == 0: the stages above)
};

// cos / sin of 2*pi*k/R, k < R, for the odd radices 3, 5, 7, 11 (rows 0..3)
__constant__ double kcos_d[4][11] = {
  {1.0, -0.5, -0.5, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0},
  {1.0, 0.30901699437494745, -0.8090169943749473, -0.8090169943749476, 0.30901699437494723, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0},
  {1.0, 0.6234898018587336, -0.22252093395631434, -0.900968867902419, -0.9009688679024191, -0.2225209339563146, 0.6234898018587334, 0.0, 0.0, 0.0, 0.0},
  {1.0, 0.8412535328311812, 0.41541501300188644, -0.142314838273285, -0.654860733945285, -0.9594929736144974, -0.9594929736144975, -0.6548607339452852, -0.14231483827328523, 0.41541501300188605, 0.8412535328311812}};
__constant__ double ksin_d[4][11] = {
  {0.0, 0.8660254037844387, -0.8660254037844384, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0},
  {0.0, 0.9510565162951535, 0.5877852522924732, -0.587785252292473, -0.9510565162951536, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0},
  {0.0, 0.7818314824680298, 0.9749279121818236, 0.43388373911755823, -0.433883739117558, -0.9749279121818236, -0.7818314824680299, 0.0, 0.0, 0.0, 0.0},
  {0.0, 0.5406408174555976, 0.9096319953545183, 0.9898214418809328, 0.7557495743542583, 0.28173255684142967, -0.2817325568414294, -0.7557495743542582, -0.9898214418809327, -0.9096319953545186, -0.5406408174555974}};
__constant__ float kcos_f[4][11] = {
  {1.0f, -0.5f, -0.5f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f},
  {1.0f, 0.30901699437494745f, -0.8090169943749473f, -0.8090169943749476f, 0.30901699437494723f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f},
  {1.0f, 0.6234898018587336f, -0.22252093395631434f, -0.900968867902419f, -0.9009688679024191f, -0.2225209339563146f, 0.6234898018587334f, 0.0f, 0.0f, 0.0f, 0.0f},
  {1.0f, 0.8412535328311812f, 0.41541501300188644f, -0.142314838273285f, -0.654860733945285f, -0.9594929736144974f, -0.9594929736144975f, -0.6548607339452852f, -0.14231483827328523f, 0.41541501300188605f, 0.8412535328311812f}};
__constant__ float ksin_f[4][11] = {
  {0.0f, 0.8660254037844387f, -0.8660254037844384f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f},
  {0.0f, 0.9510565162951535f, 0.5877852522924732f, -0.587785252292473f, -0.9510565162951536f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f},
  {0.0f, 0.7818314824680298f, 0.9749279121818236f, 0.43388373911755823f, -0.433883739117558f, -0.9749279121818236f, -0.7818314824680299f, 0.0f, 0.0f, 0.0f, 0.0f},
  {0.0f, 0.5406408174555976f, 0.9096319953545183f, 0.9898214418809328f, 0.7557495743542583f, 0.28173255684142967f, -0.2817325568414294f, -0.7557495743542582f, -0.9898214418809327f, -0.9096319953545186f, -0.5406408174555974f}};

template <int R> constexpr int radix_row() { return R == 3 ? 0 : R == 5 ? 1 : R == 7 ? 2 : 3; }
template <typename T, int R> __device__ __forceinline__ T trig_cos(int k) {
  if constexpr (sizeof(T) == 4) return kcos_f[radix_row<R>()][k]; else return kcos_d[radix_row<R>()][k];
}
template <typename T, int R> __device__ __forceinline__ T trig_sin(int k) {
  if constexpr (sizeof(T) == 4) return ksin_f[radix_row<R>()][k]; else return ksin_d[radix_row<R>()][k];
}

template <typename T, int R>
__device__ __forceinline__ void dft_const(cplx<T> (&a)[R], bool fwd) {
  if constexpr (R == 2 || R == 4 || R == 8) {
    dft_small<T, R>(a, nullptr, 0, fwd);
  } else {
    constexpr int H = (R - 1) / 2;
    cplx<T> sp[H + 1], sm[H + 1];
#pragma unroll
    for (int m = 1; m <= H; ++m) {
      sp[m] = cadd<T>(a[m], a[R - m]);
      sm[m] = csub<T>(a[m], a[R - m]);
    }
    cplx<T> y0 = a[0];
#pragma unroll
    for (int m = 1; m <= H; ++m) y0 = cadd<T>(y0, sp[m]);
    const T sg = fwd ? T(-1) : T(1);
#pragma unroll
    for (int q = 1; q <= H; ++q) {
      cplx<T> re = a[0];
      cplx<T> im = mkc<T>(T(0), T(0));
#pragma unroll
      for (int m = 1; m <= H; ++m) {
        const T c = trig_cos<T, R>((m * q) % R), sn = trig_sin<T, R>((m * q) % R);
        re.x += sp[m].x * c;
        re.y += sp[m].y * c;
        im.x += sm[m].x * sn;
        im.y += sm[m].y * sn;
      }
      // y_q = re + sg*i*im, y_{R-q} = re - sg*i*im
      a[q] = mkc<T>(re.x - sg * im.y, re.y + sg * im.x);
      a[R - q] = mkc<T>(re.x + sg * im.y, re.y - sg * im.x);
    }
    a[0] = y0;
  }
}

}  // namespace dnufft

#include "fft_pencil.cuh"

namespace dnufft {

template <typename T>
__device__ __forceinline__ cplx<T> tw2(const cplx<T> *twh, const cplx<T> *twl, int t, bool fwd) {
  cplx<T> w = cmul<T>(twh[t >> 6], twl[t & 63]);
  if (!fwd) w.y = -w.y;
  return w;
}

template <typename T, int R>
__device__ __forceinline__ void stage2(const cplx<T> *__restrict__ src, cplx<T> *__restrict__ dst,
                                       int n, int lnl, int Ns, uint32_t mul, int tstep,
                                       const cplx<T> *twh, const cplx<T> *twl, bool fwd) {
  const int nR = n / R;
  const int B = nR << lnl;
  const int lmask = (1 << lnl) - 1;
  for (int b = threadIdx.x; b < B; b += blockDim.x) {
    const int l = b & lmask, j = b >> lnl;
    const int g = (Ns == 1) ? j : int(__umulhi(uint32_t(j), mul));
    const int k = j - g * Ns;
    cplx<T> v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      cplx<T> x = src[((j + r * nR) << lnl) + l];
      if (r > 0 && k > 0) x = cmul<T>(x, tw2<T>(twh, twl, k * r * tstep, fwd));
      v[r] = x;
    }
    dft_const<T, R>(v, fwd);
    const int ob = ((g * Ns * R + k) << lnl) + l;
#pragma unroll
    for (int r = 0; r < R; ++r) dst[ob + ((r * Ns) << lnl)] = v[r];
  }
  __syncthreads();
}

template <typename T> constexpr int fft2_max_threads() { return sizeof(T) == 4 ? 1024 : 512; }
// largest pencil radix of the line kernels (64 / 128 registers at 1024 / 512
// threads)
template <typename T> constexpr int lines_maxr() { return sizeof(T) == 4 ? 12 : 16; }
constexpr int FFT2_MAXE = 12;   // elements per CTA <= FFT2_MAXE * threads

// One block of lines (the body of k_fft_lines2, also run by the multi-job
// kernel of batched transforms): lines blk*2^ls.nl ... of the pass ls.
template <typename T>
__device__ __forceinline__ void fft_lines_block(cplx<T> *__restrict__ grid, const LineSpec &ls,
                                                const StageInfo &si,
                                                const cplx<T> *__restrict__ tw, const UniSpec &u,
                                                bool fwd, int blk, unsigned char *smraw) {
  const int n = ls.n;
  const int lnl = ls.nl;   // log2 of lines per CTA
  const int nl = 1 << lnl;
  const int nh = (n + 63) / 64 + 1;
  cplx<T> *s = reinterpret_cast<cplx<T> *>(smraw);
  cplx<T> *s2 = s + (n << lnl);
  cplx<T> *twl = s2 + (n << lnl);
  cplx<T> *twh = twl + 64;
  int64_t *lbase = reinterpret_cast<int64_t *>(twh + nh);
  int64_t *luoff = lbase + nl;
  double *lfac = reinterpret_cast<double *>(luoff + nl);
  __shared__ int stR[24], stNs[24], stT[24];
  __shared__ uint32_t stM[24];
  __shared__ PencilPlan spen;
  if (threadIdx.x < 24) {
    stR[threadIdx.x] = si.R[threadIdx.x];
    stNs[threadIdx.x] = si.Ns[threadIdx.x];
    stT[threadIdx.x] = si.tstep[threadIdx.x];
    stM[threadIdx.x] = si.mul[threadIdx.x];
  }
  if (threadIdx.x == 0) spen = si.pen;
  const int L0 = blk << lnl;
  const int nloc = min(nl, ls.nlines - L0);
  const int N = sel3(u.N, ls.ax);
  const int lo = (N + 1) / 2, hi0 = n - N / 2;
  for (int i = threadIdx.x; i < 64; i += blockDim.x) twl[i] = (i < n) ? tw[i] : mkc<T>(T(1), T(0));
  for (int i = threadIdx.x; i < nh; i += blockDim.x) twh[i] = (64 * i < n) ? tw[64 * i] : mkc<T>(T(1), T(0));
  for (int l = threadIdx.x; l < nl; l += blockDim.x) {
    int ia = 0, ib = 0;
    lbase[l] = (l < nloc) ? line_base(ls, u.N, u.n, L0 + l, ia, ib) : 0;
    double fac = 1.0;
    int64_t uoff = 0;
    if (l < nloc && (ls.in_mode == IO_UNI || ls.out_mode == IO_UNI)) line_uni(ls, u, ia, ib, fac, uoff);
    lfac[l] = fac;
    luoff[l] = uoff;
  }
  __syncthreads();
  const cplx<T> *uin = static_cast<const cplx<T> *>(u.ptr);
  const int64_t ust = sel3(u.stride, ls.ax);
  const double *cfa = sel3(u.corfac, ls.ax);
  auto load_elem = [&](int l, int k) -> cplx<T> {
    cplx<T> v = mkc<T>(T(0), T(0));
    if (l >= nloc) return v;
    if (ls.in_mode == IO_FULL) return grid[lbase[l] + int64_t(k) * ls.es];
    if (k >= lo && k < hi0) return v;
    if (ls.in_mode == IO_KEPT) return grid[lbase[l] + int64_t(k) * ls.es];
    int iu, icf;
    grid_to_uni(k, N, n, u.fft_order, iu, icf);
    cplx<T> x = uin[luoff[l] + int64_t(iu) * ust];
    T f = T(lfac[l] * cfa[icf]);
    return mkc<T>(x.x * f, x.y * f);
  };
  auto store_elem = [&](int l, int k, cplx<T> x) {
    if (l >= nloc) return;
    if (ls.out_mode == IO_FULL) {
      grid[lbase[l] + int64_t(k) * ls.es] = x;
      return;
    }
    if (k >= lo && k < hi0) return;
    if (ls.out_mode == IO_KEPT) {
      grid[lbase[l] + int64_t(k) * ls.es] = x;
      return;
    }
    int iu, icf;
    grid_to_uni(k, N, n, u.fft_order, iu, icf);
    T f = T(lfac[l] * cfa[icf]);
    static_cast<cplx<T> *>(u.ptr)[luoff[l] + int64_t(iu) * ust] = mkc<T>(x.x * f, x.y * f);
  };
  {
    // LB loads in flight per thread before their shared-memory stores;
    // contiguous lines walk each line with consecutive threads (coalesced).
    // Each thread keeps its (line, element) position and steps it by the
    // block size (no division per element).
    constexpr int LB = 8;
    const int tot = n << lnl;
    const int nt = int(blockDim.x);
    int fl, fk;   // position of flat index f = threadIdx.x (+ multiples of nt)
    if (ls.es == 1) {
      fl = int(threadIdx.x) / n;
      fk = int(threadIdx.x) - fl * n;
    } else {
      fl = int(threadIdx.x) & (nl - 1);
      fk = int(threadIdx.x) >> lnl;
    }
    const int dl = ls.es == 1 ? nt / n : (nt & (nl - 1));
    const int dk = ls.es == 1 ? nt - (nt / n) * n : (nt >> lnl);
    for (int b0 = threadIdx.x; b0 < tot; b0 += LB * nt) {
      cplx<T> v[LB];
      int dst[LB];
#pragma unroll
      for (int u2 = 0; u2 < LB; ++u2) {
        const bool in = b0 + u2 * nt < tot;
        dst[u2] = (fk << lnl) + fl;
        v[u2] = in ? load_elem(fl, fk) : mkc<T>(T(0), T(0));
        // advance by nt in the flat order
        if (ls.es == 1) {
          fk += dk;
          fl += dl;
          if (fk >= n) {
            fk -= n;
            ++fl;
          }
        } else {
          fl += dl;
          fk += dk;
          if (fl >= nl) {
            fl -= nl;
            ++fk;
          }
        }
      }
#pragma unroll
      for (int u2 = 0; u2 < LB; ++u2)
        if (b0 + u2 * nt < tot) s[dst[u2]] = v[u2];
    }
  }
  __syncthreads();
  if (spen.L > 0) {
    // pencil passes (result in s2)
    if (fwd)
      pencil_fft<T, true, lines_maxr<T>()>(s, s2, nl, lnl, spen, twh, twl);
    else
      pencil_fft<T, false, lines_maxr<T>()>(s, s2, nl, lnl, spen, twh, twl);
    s = s2;
  } else {
  cplx<T> *src = s, *dst = s2;
  for (int f = 0; f < si.nst; ++f) {
    const int R = stR[f], Ns = stNs[f], ts = stT[f];
    const uint32_t mul = stM[f];
    switch (R) {
      case 2: stage2<T, 2>(src, dst, n, lnl, Ns, mul, ts, twh, twl, fwd); break;
      case 3: stage2<T, 3>(src, dst, n, lnl, Ns, mul, ts, twh, twl, fwd); break;
      case 4: stage2<T, 4>(src, dst, n, lnl, Ns, mul, ts, twh, twl, fwd); break;
      case 5: stage2<T, 5>(src, dst, n, lnl, Ns, mul, ts, twh, twl, fwd); break;
      case 7: stage2<T, 7>(src, dst, n, lnl, Ns, mul, ts, twh, twl, fwd); break;
      case 8: stage2<T, 8>(src, dst, n, lnl, Ns, mul, ts, twh, twl, fwd); break;
      case 11: stage2<T, 11>(src, dst, n, lnl, Ns, mul, ts, twh, twl, fwd); break;
      default: break;
    }
    cplx<T> *t = src;
    src = dst;
    dst = t;
  }
  s = src;
  }
  if (ls.es == 1) {
    for (int l = 0; l < nl; ++l)
      for (int k = threadIdx.x; k < n; k += blockDim.x) store_elem(l, k, s[(k << lnl) + l]);
  } else {
    const int tot = n << lnl;
    for (int idx = threadIdx.x; idx < tot; idx += blockDim.x)
      store_elem(idx & (nl - 1), idx >> lnl, s[idx]);
  }
}

template <typename T>
__global__ void __launch_bounds__(fft2_max_threads<T>())
    k_fft_lines2(cplx<T> *__restrict__ grid, LineSpec ls, StageInfo si, const cplx<T> *__restrict__ tw,
                 UniSpec u, bool fwd) {
  extern __shared__ __align__(16) unsigned char smraw[];
  fft_lines_block<T>(grid, ls, si, tw, u, fwd, blockIdx.x, smraw);
}

static bool make_pencil(int n, int maxr, int maxlast, PencilPlan &pp);

// Radix-by-radix stage table of an axis, plus the pencil passes with radices up
// to pen_maxr where such a plan exists (pen_maxr == 0: none).
static StageInfo make_stages(const FFTAxisPlan &p, int pen_maxr) {
  StageInfo si;
  std::memset(&si, 0, sizeof(si));
  if (pen_maxr > 0 && !make_pencil(p.n, pen_maxr, 1 << 30, si.pen)) si.pen.L = 0;
  si.nst = p.nfac;
  int Ns = 1;
  for (int f = 0; f < p.nfac; ++f) {
    si.R[f] = p.fac[f];
    si.Ns[f] = Ns;
    si.tstep[f] = p.n / (Ns * p.fac[f]);
    si.mul[f] = Ns == 1 ? 0u : uint32_t(((uint64_t(1) << 32) + uint64_t(Ns) - 1) / uint64_t(Ns));
    Ns *= p.fac[f];
  }
  return si;
}

// v2 launch if the line fits its register / shared-memory budget; false otherwise
template <typename T>
static bool run_lines2(cplx<T> *grid, LineSpec ls, const FFTAxisPlan &p, const UniSpec &u,
                       bool fwd, cudaStream_t st) {
  const int n = ls.n;
  const int maxnt = fft2_max_threads<T>();
  const size_t maxsm = 200 * 1024;
  if (n > FFT2_MAXE * maxnt || n >= (1 << 16)) return false;
  int lnl = 0;
  const int want = (ls.es == 1) ? 2048 : 8192;   // elements per CTA to aim for
  if (size_t(2 * n) * sizeof(cplx<T>) > maxsm - 8192) return false;
  while ((n << (lnl + 1)) <= want && (1 << (lnl + 1)) <= 16 && (1 << lnl) < ls.nlines &&
         size_t(n << (lnl + 2)) * sizeof(cplx<T>) <= maxsm / 2 &&
         (n << (lnl + 1)) <= FFT2_MAXE * maxnt)
    ++lnl;
  const int total = n << lnl;
  int nt = 32 * ((total + FFT2_MAXE - 1) / FFT2_MAXE / 32 + 1);
  nt = std::max(64, std::min(maxnt, nt));
  if (total > FFT2_MAXE * nt) return false;
  const int nh = (n + 63) / 64 + 1;
  size_t sm = size_t(2 * total + 64 + nh) * sizeof(cplx<T>) + size_t(1 << lnl) * 24;
  if (sm > maxsm) return false;
  ls.nl = lnl;
  StageInfo si = make_stages(p, lines_maxr<T>());
  DN_CUDA(cudaFuncSetAttribute(k_fft_lines2<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
  unsigned nb = unsigned((ls.nlines + (1 << lnl) - 1) >> lnl);
  k_fft_lines2<T><<<nb, nt, sm, st>>>(grid, ls, si, static_cast<const cplx<T> *>(p.tw), u, fwd);
  DN_LAUNCHED();
  return true;
}

// ---------------------------------------------------------------------------
// FFT v3 for 2D grids.
//
// Rows (the contiguous axis): a persistent kernel, one CTA per SM, walks its
// rows with three shared-memory line buffers: the next row is fetched by a TMA
// bulk copy (cp.async.bulk, completion on an mbarrier) while the current one
// runs its Stockham stages (ping-pong between the other two buffers), and the
// result is written back by bulk stores.  Kept ranges (type 1 output, type 2
// input) are copied as two ranges; 16-byte alignment is kept by moving ragged
// end elements with ordinary loads and stores.
//
// Columns (the strided axis, length n = P*Q): the four-step method, as two
// passes over blocks of C adjacent kept columns (C*8 or C*16 contiguous bytes
// per row, so every access is coalesced):
//   pass A: for each q < Q, the P-point DFTs over rows q + Q*p, times the
//           twiddle w_n^(q*k1), into a compact work array (row q + Q*k1);
//   pass B: for each k1 < P, the Q-point DFTs over the Q contiguous work rows
//           Q*k1 + q; output element k = k1 + P*k2 (natural order), either the
//           corrected, cropped uniform array (type 1) or the grid (type 2).
// The small DFTs are the Stockham stages above on a [len][C] tile.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t fft_smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void fft_bar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(fft_smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void fft_bar_expect(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fft_smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// bounded wait (a second of wall clock); false if the phase did not complete
__device__ __forceinline__ bool fft_bar_wait(uint64_t *bar, uint32_t parity) {
  const uint32_t addr = fft_smem_u32(bar);
  unsigned long long t0 = 0;
  for (uint32_t it = 0;; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(addr), "r"(parity), "r"(1000u)
        : "memory");
    if (ok) return true;
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    if (it == 0) t0 = t;
    else if (t - t0 > 1000000000ull) return false;
  }
}

__device__ __forceinline__ void fft_bulk_load(void *sdst, const void *gsrc, uint32_t bytes,
                                              uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(fft_smem_u32(sdst)), "l"(gsrc), "r"(bytes), "r"(fft_smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void fft_bulk_store(void *gdst, const void *ssrc, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gdst),
               "r"(fft_smem_u32(ssrc)), "r"(bytes)
               : "memory");
}

// 16-byte aligned part [a2, b2) of an element range [a, b) (esz = element bytes)
__device__ __forceinline__ void fft_aligned(int a, int b, int esz, int &a2, int &b2) {
  const int per = 16 / esz;   // elements per 16 bytes (2 for complex64, 1 for complex128)
  a2 = (a + per - 1) / per * per;
  b2 = b / per * per;
  if (b2 < a2) b2 = a2;
}

#ifndef ROWS_MAXR_F
#define ROWS_MAXR_F 25
#define ROWS_MAXR_D 16
#define COLS_MAXR_F 12
#define COLS_MAXR_D 11
#endif
// every prime factor the planner allows (up to 11) must fit one pass
static_assert(ROWS_MAXR_F >= 11 && ROWS_MAXR_D >= 11 && COLS_MAXR_F >= 11 && COLS_MAXR_D >= 11,
              "pencil radix bound below the largest prime factor");

// largest pencil radix of the row and column passes (register budgets of their
// CTAs: 512 / 256 threads per SM for rows, several 256-thread CTAs for columns)
template <typename T> constexpr int rows_maxr() { return sizeof(T) == 4 ? ROWS_MAXR_F : ROWS_MAXR_D; }
template <typename T> constexpr int cols_maxr() { return sizeof(T) == 4 ? COLS_MAXR_F : COLS_MAXR_D; }
// column CTAs per SM the register allocation must allow (64 / 80 registers)
template <typename T> constexpr int cols_min_ctas() { return sizeof(T) == 4 ? 4 : 3; }
template <typename T> constexpr int rows_threads() { return 512; }

// One row = line of n contiguous elements at grid + row*rs.  Ranges: the whole
// line, or the kept ranges [0, lo) and [hi0, n) (zeros in between on input).
// Two row buffers: the current row is transformed in place while the next one
// arrives by TMA bulk copy into the other; the result is written back by bulk
// stores from the current buffer, which becomes the prefetch target of the
// row after next once those stores have read it.
template <typename T, bool FWD>
__global__ void __launch_bounds__(rows_threads<T>(), 1)
    k_fft_rows(cplx<T> *__restrict__ grid, int64_t rs, int n, int nlines, int lo, int hi0,
               int in_kept, int out_kept, PencilPlan pp, const cplx<T> *__restrict__ tw,
               int full_tw, int *__restrict__ err) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ uint64_t bars[2];
  __shared__ PencilPlan spp;
  __shared__ int s_fail;
  constexpr int ES = int(sizeof(cplx<T>));
  cplx<T> *bufs = reinterpret_cast<cplx<T> *>(smraw);
  // twiddles: the full table of n roots after the buffers where it fits
  // (full_tw), else the two-level one
  const int nh = (n + 63) / 64 + 1;
  cplx<T> *twl = bufs + 2 * n;
  cplx<T> *twh = full_tw ? nullptr : twl + 64;
  const int tid = threadIdx.x;
  if (tid == 0) spp = pp;
  if (full_tw) {
    for (int i = tid; i < n; i += blockDim.x) twl[i] = tw[i];
  } else {
    for (int i = tid; i < 64; i += blockDim.x) twl[i] = (i < n) ? tw[i] : mkc<T>(T(1), T(0));
    for (int i = tid; i < nh; i += blockDim.x)
      twh[i] = (64 * i < n) ? tw[64 * i] : mkc<T>(T(1), T(0));
  }
  if (tid == 0) {
    for (int b = 0; b < 2; ++b) fft_bar_init(&bars[b], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_fail = 0;
  }
  __syncthreads();
  const int nr = in_kept ? 2 : 1;
  // issue the bulk part of row L into buffer b (thread 0)
  auto issue_load = [&](int L, int b) {
    const cplx<T> *src = grid + int64_t(L) * rs;
    cplx<T> *dst = bufs + b * n;
    uint32_t bytes = 0;
    int a2[2], b2[2];
    for (int r = 0; r < nr; ++r) {
      const int ra = in_kept ? (r == 0 ? 0 : hi0) : 0;
      const int rb = in_kept ? (r == 0 ? lo : n) : n;
      fft_aligned(ra, rb, ES, a2[r], b2[r]);
      bytes += uint32_t(b2[r] - a2[r]) * ES;
    }
    fft_bar_expect(&bars[b], bytes);
    for (int r = 0; r < nr; ++r)
      if (b2[r] > a2[r])
        fft_bulk_load(dst + a2[r], src + a2[r], uint32_t(b2[r] - a2[r]) * ES, &bars[b]);
  };
  int bi = 0, bf = 1;
  uint32_t ph = 0;   // bit b: parity of the next completion of bars[b]
  if (tid == 0 && int(blockIdx.x) < nlines) issue_load(blockIdx.x, bi);
  for (int L = blockIdx.x; L < nlines; L += gridDim.x) {
    const int Ln = L + gridDim.x;
    cplx<T> *in = bufs + bi * n;
    const cplx<T> *src = grid + int64_t(L) * rs;
    // ragged ends of the ranges and the zero middle (disjoint from the bulk part)
    for (int r = 0; r < nr; ++r) {
      const int ra = in_kept ? (r == 0 ? 0 : hi0) : 0;
      const int rb = in_kept ? (r == 0 ? lo : n) : n;
      int a2, b2;
      fft_aligned(ra, rb, ES, a2, b2);
      for (int k = ra + tid; k < a2; k += blockDim.x) in[k] = src[k];
      for (int k = b2 + tid; k < rb; k += blockDim.x) in[k] = src[k];
    }
    if (in_kept)
      for (int k = lo + tid; k < hi0; k += blockDim.x) in[k] = mkc<T>(T(0), T(0));
    const bool ok = fft_bar_wait(&bars[bi], (ph >> bi) & 1u);
    ph ^= 1u << bi;
    if (__syncthreads_or(ok ? 0 : 1)) {
      if (tid == 0) atomicExch(err, 1);
      break;
    }
    // every thread has finished the previous row (its ragged output copies
    // read buffer bf): prefetch the next row there once the previous row's
    // bulk stores have read it
    if (tid == 0 && Ln < nlines) {
      asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
      issue_load(Ln, bf);
    }
    // all passes in place in the input buffer (each thread fences its
    // shared-memory writes for the bulk stores before the final barrier)
    pencil_fft_inplace<T, FWD, rows_maxr<T>()>(in, spp, twh, twl);
    const cplx<T> *sa = in;
    // result in sa; write it back (bulk part by thread 0, ragged ends by all)
    cplx<T> *dst = grid + int64_t(L) * rs;
    const int nro = out_kept ? 2 : 1;
    if (tid == 0) {
      for (int r = 0; r < nro; ++r) {
        const int ra = out_kept ? (r == 0 ? 0 : hi0) : 0;
        const int rb = out_kept ? (r == 0 ? lo : n) : n;
        int a2, b2;
        fft_aligned(ra, rb, ES, a2, b2);
        if (b2 > a2) fft_bulk_store(dst + a2, sa + a2, uint32_t(b2 - a2) * ES);
      }
      asm volatile("cp.async.bulk.commit_group;" ::: "memory");
    }
    for (int r = 0; r < nro; ++r) {
      const int ra = out_kept ? (r == 0 ? 0 : hi0) : 0;
      const int rb = out_kept ? (r == 0 ? lo : n) : n;
      int a2, b2;
      fft_aligned(ra, rb, ES, a2, b2);
      for (int k = ra + tid; k < a2; k += blockDim.x) dst[k] = sa[k];
      for (int k = b2 + tid; k < rb; k += blockDim.x) dst[k] = sa[k];
    }
    // the prefetched buffer is next; this one is busy storing
    const int t = bi;
    bi = bf;
    bf = t;
  }
  if (tid == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
  __syncthreads();
}


// Four-step column pass.  PASS 0 = A, 1 = B.  Columns: x in [0, N1) kept
// columns (grid column kept_to_grid(x)); C = 1 << lc columns per CTA.
struct ColSpec {
  int n;        // column length (n0)
  int P, Q;     // n = P*Q
  int N1, n1;   // kept columns / row length of the grid
  int lc;       // log2 columns per CTA
  int in_mode;  // pass A: 0 grid, 1 uniform array (type 2); pass B: work
  int out_mode; // pass A: work; pass B: 0 grid (natural order), 1 uniform array (type 1)
  // column x of this pass is column x0 + x of a transform with N1t kept of
  // n1t grid columns (uniform index and correction factor); with packed_out
  // the uniform result of column x goes to column x of out (x0 = 0, N1t = N1,
  // n1t = n1 and packed_out = 0 for a whole transform)
  int x0, N1t, n1t, packed_out;
};

template <typename T, int PASS, bool FWD>
__global__ void __launch_bounds__(256, cols_min_ctas<T>())
    k_fft_colstep(cplx<T> *__restrict__ grid, cplx<T> *__restrict__ work, ColSpec cs,
                  PencilPlan pp, const cplx<T> *__restrict__ tw, UniSpec u) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int C = 1 << cs.lc;
  const int len = PASS == 0 ? cs.P : cs.Q;    // DFT length of this pass
  const int tstr = PASS == 0 ? cs.Q : cs.P;   // sub-table stride into tw (length n)
  cplx<T> *s = reinterpret_cast<cplx<T> *>(smraw);
  cplx<T> *s2 = s + len * C;
  cplx<T> *twl = s2 + len * C;   // the len roots of this pass (every tstr-th of tw)
  const cplx<T> *twh = nullptr;
  __shared__ PencilPlan spp;
  const int tid = threadIdx.x;
  if (tid == 0) spp = pp;
  for (int i = tid; i < len; i += blockDim.x) twl[i] = tw[i * tstr];
  const int nblk = (cs.N1 + C - 1) >> cs.lc;
  const int cb = blockIdx.x % nblk;      // column block
  const int g = blockIdx.x / nblk;       // q (pass A) or k1 (pass B)
  const int x0 = cb << cs.lc;
  const int N0 = sel3(u.N, 0);
  const int lo0 = (N0 + 1) / 2, hi00 = cs.n - N0 / 2;
  // ---- load the [len][C] tile (element m of column c at s[m*C + c]).  Every
  // thread keeps one column c (blockDim is a multiple of C) and walks rows
  // m = m0, m0 + mstep, ...: the column's grid index, row pointers and the
  // column part of the uniform index are computed once.
  const int c = tid & (C - 1), m0 = tid >> cs.lc, mstep = int(blockDim.x) >> cs.lc;
  const int x = x0 + c;
  const bool colok = x < cs.N1;
  const int gx = colok ? kept_to_grid(x, cs.N1, cs.n1) : 0;
  const cplx<T> *uptr = static_cast<const cplx<T> *>(u.ptr);
  int iu1 = 0, icf1 = 0;
  double cf1 = 0.0;
  if (colok && ((PASS == 0 && cs.in_mode != 0) || (PASS == 1 && cs.out_mode != 0))) {
    grid_to_uni(cs.x0 + gx, cs.N1t, cs.n1t, u.fft_order, iu1, icf1);
    cf1 = u.corfac[1][icf1];
    if (cs.packed_out) iu1 = x;
  }
  auto load_m = [&](int m) -> cplx<T> {
    cplx<T> v = mkc<T>(T(0), T(0));
    if (!colok) return v;
    if (PASS == 0) {
      const int row = g + cs.Q * m;   // q + Q*p
      if (cs.in_mode == 0) {
        v = grid[int64_t(row) * cs.n1 + gx];
      } else if (row < lo0 || row >= hi00) {
        // gather the caller's uniform array with the correction factors
        int iu0, icf0;
        grid_to_uni(row, N0, cs.n, u.fft_order, iu0, icf0);
        const cplx<T> xv = uptr[int64_t(iu0) * u.stride[0] + int64_t(iu1) * u.stride[1]];
        const T f = T(u.corfac[0][icf0] * cf1);
        v = mkc<T>(xv.x * f, xv.y * f);
      }
    } else {
      v = work[int64_t(g * cs.Q + m) * cs.N1 + x];   // row Q*k1 + q
    }
    return v;
  };
  {
    constexpr int LB = 8;   // loads in flight per thread
    for (int mb = m0; mb < len; mb += LB * mstep) {
      cplx<T> v[LB];
#pragma unroll
      for (int u2 = 0; u2 < LB; ++u2) {
        const int m = mb + u2 * mstep;
        v[u2] = m < len ? load_m(m) : mkc<T>(T(0), T(0));
      }
#pragma unroll
      for (int u2 = 0; u2 < LB; ++u2) {
        const int m = mb + u2 * mstep;
        if (m < len) s[m * C + c] = v[u2];
      }
    }
  }
  __syncthreads();
  pencil_fft<T, FWD, cols_maxr<T>()>(s, s2, C, cs.lc, spp, twh, twl);
  const cplx<T> *sa = s2;
  // ---- store (same column per thread)
  if (colok) {
    for (int m = m0; m < len; m += mstep) {
      cplx<T> v = sa[m * C + c];
      if (PASS == 0) {
        // twiddle w_n^(q*k1) (q*k1 < Q*P = n), then work row q + Q*k1
        cplx<T> w = tw[g * m];
        if (!FWD) w.y = -w.y;
        v = cmul<T>(v, w);
        work[int64_t(g + cs.Q * m) * cs.N1 + x] = v;
      } else {
        const int k = g + cs.P * m;   // k1 + P*k2
        if (cs.out_mode == 0) {
          grid[int64_t(k) * cs.n1 + gx] = v;
        } else if (k < lo0 || k >= hi00) {
          int iu0, icf0;
          grid_to_uni(k, N0, cs.n, u.fft_order, iu0, icf0);
          const T f = T(u.corfac[0][icf0] * cf1);
          static_cast<cplx<T> *>(u.ptr)[int64_t(iu0) * u.stride[0] + int64_t(iu1) * u.stride[1]] =
              mkc<T>(v.x * f, v.y * f);
        }
      }
    }
  }
}

// n = P*Q with P, Q as close to sqrt(n) as the factors allow (both >= 8)
static bool split_pq(int n, int &P, int &Q) {
  int best = -1;
  for (int p = 8; p * p <= n; ++p) {
    if (n % p) continue;
    const int q = n / p;
    if (q < 8) continue;
    best = p;   // largest p <= sqrt(n)
  }
  if (best < 0) return false;
  P = best;
  Q = n / best;
  return P <= 1024 && Q <= 1024;
}

// Radix sequence of the pencil passes for a line of length n: the fewest
// passes with radices of a register DFT up to maxr; among those, an odd last
// radix and an odd product of the radices before the last two (the strides of
// the last pass's shared-memory reads and writes of rows, conflict-free when
// odd), then the smallest largest radix.  maxlast bounds the groups of the
// last pass (n / R_L), which the in-place row transform gives one thread each.
// Cached per (n, maxr, maxlast).
static bool make_pencil(int n, int maxr, int maxlast, PencilPlan &pp) {
  static std::mutex mu;
  static std::map<std::tuple<int, int, int>, std::pair<bool, PencilPlan>> cache;
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find({n, maxr, maxlast});
    if (it != cache.end()) {
      pp = it->second.second;
      return it->second.first;
    }
  }
  static const int rad[] = {2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 14,
                            15, 16, 18, 20, 21, 22, 24, 25, 27, 28, 30, 32};
  std::vector<int> cur, best;
  long best_score = -1;
  std::function<void(int)> rec = [&](int rem) {
    if (rem == 1) {
      const int L = int(cur.size());
      if (n / cur[L - 1] > maxlast) return;
      int mx = 0, pre = 1;
      for (int i = 0; i < L; ++i) mx = std::max(mx, cur[i]);
      for (int i = 0; i + 2 < L; ++i) pre *= cur[i];
      const int conflicts = (cur[L - 1] % 2 == 0) + (pre % 2 == 0);
      const long score = long(L) * 1000000 + conflicts * 10000 + mx * 10 + (cur[0] % 2 == 0);
      if (best_score < 0 || score < best_score) {
        best_score = score;
        best = cur;
      }
      return;
    }
    if (int(cur.size()) == PEN_MAXL) return;
    for (int r : rad) {
      if (r > maxr || rem % r) continue;
      cur.push_back(r);
      rec(rem / r);
      cur.pop_back();
    }
  };
  if (n >= 2) rec(n);
  std::memset(&pp, 0, sizeof(pp));
  const bool ok = !best.empty();
  if (ok) {
    pp.n = n;
    pp.L = int(best.size());
    int m = n, P = 1;
    for (int i = 0; i < pp.L; ++i) {
      pp.R[i] = best[i];
      m /= best[i];
      pp.m[i] = m;
      pp.P[i] = P;
      pp.mmul[i] = m <= 1 ? 0u : uint32_t(((uint64_t(1) << 32) + uint64_t(m) - 1) / uint64_t(m));
      P *= best[i];
    }
  }
  std::lock_guard<std::mutex> lk(mu);
  cache[{n, maxr, maxlast}] = {ok, pp};
  return ok;
}

static int sm_count_dev() {
  int dev = 0, nsm = 0;
  DN_CUDA(cudaGetDevice(&dev));
  DN_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  return nsm > 0 ? nsm : 1;
}

// persistent row FFTs; false if this size is not handled (the caller falls back)
template <typename T>
static bool run_rows_v3(cplx<T> *grid, int n, int nlines, int64_t rs, int Nk, bool in_kept,
                        bool out_kept, const FFTAxisPlan &p, bool fwd, int *err,
                        cudaStream_t st) {
  if (err == nullptr || nlines <= 0) return false;
  const int nh = (n + 63) / 64 + 1;
  const size_t smfull = size_t(3 * n) * sizeof(cplx<T>);
  const int full_tw = smfull <= 224 * 1024 ? 1 : 0;
  const size_t sm = full_tw ? smfull : size_t(2 * n + 64 + nh) * sizeof(cplx<T>);
  if (sm > 224 * 1024 || n < 1024) return false;
  PencilPlan pp;
  if (!make_pencil(n, rows_maxr<T>(), rows_threads<T>(), pp)) return false;
  const int lo = (Nk + 1) / 2, hi0 = n - Nk / 2;
  auto kern = fwd ? k_fft_rows<T, true> : k_fft_rows<T, false>;
  DN_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
  const int nb = std::min(nlines, sm_count_dev());
  stage_mark(out_kept ? "FFT rows (k_fft_rows)" : "FFT rows, kept columns in (k_fft_rows)");
  kern<<<nb, rows_threads<T>(), sm, st>>>(grid, rs, n, nlines, lo, hi0, in_kept ? 1 : 0,
                                          out_kept ? 1 : 0, pp, static_cast<const cplx<T> *>(p.tw),
                                          full_tw, err);
  DN_LAUNCHED();
  return true;
}

// four-step column FFTs over the N1 kept columns of an n0 x n1 grid
template <typename T>
static bool run_cols_v3(cplx<T> *grid, cplx<T> *work, int n0, int n1, int N1,
                        const FFTAxisPlan &p, const UniSpec &u, bool type1, bool fwd,
                        cudaStream_t st, int x0 = 0, int N1t = -1, int n1t = -1,
                        bool packed_out = false) {
  if (work == nullptr || n0 < 1024) return false;
  int P, Q;
  if (!split_pq(n0, P, Q)) return false;
  PencilPlan ppP, ppQ;
  if (!make_pencil(P, cols_maxr<T>(), 1 << 30, ppP) || !make_pencil(Q, cols_maxr<T>(), 1 << 30, ppQ))
    return false;
  const int lc = sizeof(T) == 4 ? 5 : 4;   // 32 (complex64) or 16 (complex128) columns
  const int C = 1 << lc;
  ColSpec cs;
  cs.n = n0;
  cs.P = P;
  cs.Q = Q;
  cs.N1 = N1;
  cs.n1 = n1;
  cs.lc = lc;
  cs.x0 = x0;
  cs.N1t = N1t < 0 ? N1 : N1t;
  cs.n1t = n1t < 0 ? n1 : n1t;
  cs.packed_out = packed_out ? 1 : 0;
  const cplx<T> *tw = static_cast<const cplx<T> *>(p.tw);
  const int nblk = (N1 + C - 1) / C;
  for (int pass = 0; pass < 2; ++pass) {
    const int len = pass == 0 ? P : Q;
    const size_t sm = size_t(2 * len * C + len) * sizeof(cplx<T>);
    if (sm > 200 * 1024) return false;
  }
  cs.in_mode = type1 ? 0 : 1;
  cs.out_mode = type1 ? 1 : 0;
  {
    const size_t sm = size_t(2 * P * C + P) * sizeof(cplx<T>);
    auto kern = fwd ? k_fft_colstep<T, 0, true> : k_fft_colstep<T, 0, false>;
    DN_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
    stage_mark(type1 ? "FFT columns A (k_fft_colstep)"
                     : "FFT columns A, correction + pad (k_fft_colstep)");
    kern<<<unsigned(nblk) * unsigned(Q), 256, sm, st>>>(grid, work, cs, ppP, tw, u);
    DN_LAUNCHED();
  }
  {
    const size_t sm = size_t(2 * Q * C + Q) * sizeof(cplx<T>);
    auto kern = fwd ? k_fft_colstep<T, 1, true> : k_fft_colstep<T, 1, false>;
    DN_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
    stage_mark(type1 ? "FFT columns B, correction + crop (k_fft_colstep)"
                     : "FFT columns B (k_fft_colstep)");
    kern<<<unsigned(nblk) * unsigned(P), 256, sm, st>>>(grid, work, cs, ppQ, tw, u);
    DN_LAUNCHED();
  }
  return true;
}

template <typename T>
static void run_lines(cplx<T> *grid, LineSpec ls, const FFTAxisPlan &p, const UniSpec &u,
                      bool fwd, cudaStream_t st) {
  if (ls.nlines <= 0) return;
  if (run_lines2<T>(grid, ls, p, u, fwd, st)) return;
  const int n = ls.n;
  const size_t maxsm = 200 * 1024;
  int nl;
  if (ls.es == 1) {
    nl = std::max(1, std::min(32, 4096 / n));
  } else {
    nl = std::max(1, std::min(16, 16384 / n));
  }
  const int maxnt = fft_max_threads<T>();
  while (nl > 1 && (size_t(n) * nl * sizeof(cplx<T>) > maxsm || n * nl > FFT_MAXE * maxnt)) --nl;
  nl = std::min(nl, ls.nlines);
  DN_REQUIRE(size_t(n) * sizeof(cplx<T>) <= maxsm && n <= FFT_MAXE * maxnt, ST_UNSUPPORTED,
             "oversampled axis too long for the single-CTA FFT of this build");
  ls.nl = nl;
  int total = n * nl;
  int nt = 32 * ((total / 8 + 31) / 32);
  nt = std::max(64, std::min(maxnt, nt));
  while (total > FFT_MAXE * nt) nt += 32;
  size_t sm = size_t(total) * sizeof(cplx<T>);
  DN_CUDA(cudaFuncSetAttribute(k_fft_lines<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(sm)));
  unsigned nb = unsigned((ls.nlines + nl - 1) / nl);
  k_fft_lines<T><<<nb, nt, sm, st>>>(grid, ls, p, u, fwd);
  DN_LAUNCHED();
}

static LineSpec mk_spec(int n, int ax, int64_t es, int cnta, int cntb, int64_t sa, int64_t sb,
                        int axa, int axb, int kepta, int keptb, int in_mode, int out_mode) {
  LineSpec ls;
  ls.n = n;
  ls.ax = ax;
  ls.es = es;
  ls.nlines = cnta * cntb;
  ls.cntb = cntb;
  ls.sa = sa;
  ls.sb = sb;
  ls.axa = axa;
  ls.axb = axb;
  ls.kepta = kepta;
  ls.keptb = keptb;
  ls.in_mode = in_mode;
  ls.out_mode = out_mode;
  ls.nl = 1;
  return ls;
}

static UniSpec mk_uni(void *ptr, const int64_t *stride, const Geometry &g,
                      const double *const corfac[3], bool fft_order) {
  UniSpec u;
  u.ptr = ptr;
  for (int d = 0; d < 3; ++d) {
    u.stride[d] = d < g.ndim ? stride[d] : 0;
    u.corfac[d] = d < g.ndim ? corfac[d] : nullptr;
    u.N[d] = d < g.ndim ? int(g.nuni[d]) : 1;
    u.n[d] = d < g.ndim ? int(g.nover[d]) : 1;
  }
  u.fft_order = fft_order;
  return u;
}

// 2D type 1, first half: FFTs along axis 1 of nrows consecutive rows (any
// rows of the oversampled grid: they are independent), writing only the N1
// kept columns, in place.
template <typename T>
void fft_nu2u_rows(void *rowsv, int nrows, const Geometry &g, const FFTAxisPlan *ax, bool fwd,
                   cudaStream_t st, int *err) {
  cplx<T> *rows = static_cast<cplx<T> *>(rowsv);
  const int n1 = int(g.nover[1]);
  const int N1 = int(g.nuni[1]);
  if (nrows <= 0) return;
  if (!run_rows_v3<T>(rows, n1, nrows, n1, N1, false, true, ax[1], fwd, err, st)) {
    static const int64_t zs[3] = {0, 0, 0};
    const double *const nocf[3] = {nullptr, nullptr, nullptr};
    const UniSpec u = mk_uni(nullptr, zs, g, nocf, false);
    run_lines<T>(rows, mk_spec(n1, 1, 1, nrows, 1, n1, 0, -1, -1, 0, 0, IO_FULL, IO_KEPT), ax[1],
                 u, fwd, st);
  }
}

// 2D type 1, second half: FFTs along axis 0 of the N1 kept columns (every row
// already transformed along axis 1), correction and crop into out.
template <typename T>
void fft_nu2u_cols(void *gridv, const Geometry &g, const FFTAxisPlan *ax, bool fwd,
                   const double *const corfac[3], bool fft_order, void *out,
                   const int64_t *ostride, cudaStream_t st, void *workv) {
  cplx<T> *grid = static_cast<cplx<T> *>(gridv);
  cplx<T> *work = static_cast<cplx<T> *>(workv);
  const UniSpec u = mk_uni(out, ostride, g, corfac, fft_order);
  const int n0 = int(g.nover[0]), n1 = int(g.nover[1]);
  const int N1 = int(g.nuni[1]);
  if (!run_cols_v3<T>(grid, work, n0, n1, N1, ax[0], u, true, fwd, st))
    run_lines<T>(grid, mk_spec(n0, 0, n1, 1, N1, 0, 1, -1, 1, 0, 1, IO_FULL, IO_UNI), ax[0], u,
                 fwd, st);
}

// 2D type 1, second half for a block of kept columns: cols is (n0, ncols),
// the kept columns col0 .. col0 + ncols - 1 (of N1) packed, already
// transformed along axis 1; column FFTs, correction and crop into out, an
// (N0, ncols) array whose column x is the uniform column of kept column
// col0 + x.  Four-step column passes only (n0 >= 1024): false otherwise.
template <typename T>
bool fft_nu2u_cols_range(void *colsv, int ncols, int col0, const Geometry &g,
                         const FFTAxisPlan *ax, bool fwd, const double *const corfac[3],
                         bool fft_order, void *out, const int64_t *ostride, cudaStream_t st,
                         void *workv) {
  cplx<T> *cols = static_cast<cplx<T> *>(colsv);
  cplx<T> *work = static_cast<cplx<T> *>(workv);
  const UniSpec u = mk_uni(out, ostride, g, corfac, fft_order);
  const int n0 = int(g.nover[0]);
  const int N1 = int(g.nuni[1]);
  return run_cols_v3<T>(cols, work, n0, ncols, ncols, ax[0], u, true, fwd, st, col0, N1, N1,
                        true);
}

// 2D type 2, first half for a block of kept columns: the uniform columns of
// kept columns col0 .. col0 + ncols - 1 (with the correction factors and the
// zero padding) are transformed along axis 0 into cols, an (n0, ncols) array
// (column x: kept column col0 + x).  Four-step column passes only.
template <typename T>
bool fft_u2nu_cols_range(const void *uni, const int64_t *istride, const Geometry &g,
                         const FFTAxisPlan *ax, bool fwd, const double *const corfac[3],
                         bool fft_order, void *colsv, int ncols, int col0, cudaStream_t st,
                         void *workv) {
  cplx<T> *cols = static_cast<cplx<T> *>(colsv);
  cplx<T> *work = static_cast<cplx<T> *>(workv);
  const UniSpec u = mk_uni(const_cast<void *>(uni), istride, g, corfac, fft_order);
  const int n0 = int(g.nover[0]);
  const int N1 = int(g.nuni[1]);
  return run_cols_v3<T>(cols, work, n0, ncols, ncols, ax[0], u, false, fwd, st, col0, N1, N1,
                        false);
}

// 2D type 2, rows of a slab: nrows rows of n1 cells with only the kept
// columns set on input (the middle is not read), transformed along axis 1
// into whole rows, in place.
template <typename T>
void fft_u2nu_rows(void *rowsv, int nrows, const Geometry &g, const FFTAxisPlan *ax, bool fwd,
                   cudaStream_t st, int *err) {
  cplx<T> *rows = static_cast<cplx<T> *>(rowsv);
  const int n1 = int(g.nover[1]);
  const int N1 = int(g.nuni[1]);
  if (nrows <= 0) return;
  if (!run_rows_v3<T>(rows, n1, nrows, n1, N1, true, false, ax[1], fwd, err, st)) {
    static const int64_t zs[3] = {0, 0, 0};
    const double *const nocf[3] = {nullptr, nullptr, nullptr};
    const UniSpec u = mk_uni(nullptr, zs, g, nocf, false);
    run_lines<T>(rows, mk_spec(n1, 1, 1, nrows, 1, n1, 0, -1, -1, 0, 0, IO_KEPT, IO_FULL), ax[1],
                 u, fwd, st);
  }
}

template <typename T>
void fft_nu2u_tail(void *gridv, const Geometry &g, const FFTAxisPlan *ax, bool fwd,
                   const double *const corfac[3], bool fft_order, void *out,
                   const int64_t *ostride, cudaStream_t st, void *workv, int *err) {
  cplx<T> *grid = static_cast<cplx<T> *>(gridv);
  cplx<T> *work = static_cast<cplx<T> *>(workv);
  UniSpec u = mk_uni(out, ostride, g, corfac, fft_order);
  const int n0 = int(g.nover[0]);
  if (g.ndim == 1) {
    run_lines<T>(grid, mk_spec(n0, 0, 1, 1, 1, 0, 0, -1, -1, 0, 0, IO_FULL, IO_UNI), ax[0], u, fwd, st);
  } else if (g.ndim == 2) {
    // rows (axis 1), all n0 rows, keep N1 columns; then the kept columns
    // (axis 0), correction + crop
    fft_nu2u_rows<T>(grid, n0, g, ax, fwd, st, err);
    fft_nu2u_cols<T>(grid, g, ax, fwd, corfac, fft_order, out, ostride, st, work);
  } else {
    const int n1 = int(g.nover[1]), n2 = int(g.nover[2]);
    const int N1 = int(g.nuni[1]), N2 = int(g.nuni[2]);
    // axis 2: all n0*n1 lines, keep N2
    run_lines<T>(grid, mk_spec(n2, 2, 1, n0 * n1, 1, n2, 0, -1, -1, 0, 0, IO_FULL, IO_KEPT), ax[2],
                 u, fwd, st);
    // axis 1: lines (i0, k) for kept k, keep N1
    run_lines<T>(grid, mk_spec(n1, 1, n2, n0, N2, int64_t(n1) * n2, 1, -1, 2, 0, 1, IO_FULL,
                               IO_KEPT), ax[1], u, fwd, st);
    // axis 0: lines (j, k) kept x kept, correction + crop
    run_lines<T>(grid, mk_spec(n0, 0, int64_t(n1) * n2, N1, N2, n2, 1, 1, 2, 1, 1, IO_FULL, IO_UNI),
                 ax[0], u, fwd, st);
  }
}

template <typename T>
void fft_u2nu_head(const void *uni, const int64_t *istride, const Geometry &g,
                   const FFTAxisPlan *ax, bool fwd, const double *const corfac[3],
                   bool fft_order, void *gridv, cudaStream_t st, void *workv, int *err) {
  cplx<T> *grid = static_cast<cplx<T> *>(gridv);
  cplx<T> *work = static_cast<cplx<T> *>(workv);
  UniSpec u = mk_uni(const_cast<void *>(uni), istride, g, corfac, fft_order);
  const int n0 = int(g.nover[0]);
  if (g.ndim == 1) {
    run_lines<T>(grid, mk_spec(n0, 0, 1, 1, 1, 0, 0, -1, -1, 0, 0, IO_UNI, IO_FULL), ax[0], u, fwd, st);
  } else if (g.ndim == 2) {
    const int n1 = int(g.nover[1]);
    const int N1 = int(g.nuni[1]);
    // columns (axis 0) of the kept columns: gather + correction + pad
    if (!run_cols_v3<T>(grid, work, n0, n1, N1, ax[0], u, false, fwd, st))
      run_lines<T>(grid, mk_spec(n0, 0, n1, 1, N1, 0, 1, -1, 1, 0, 1, IO_UNI, IO_FULL), ax[0],
                   u, fwd, st);
    // rows (axis 1): only kept columns are non-zero
    if (!run_rows_v3<T>(grid, n1, n0, n1, N1, true, false, ax[1], fwd, err, st))
      run_lines<T>(grid, mk_spec(n1, 1, 1, n0, 1, n1, 0, -1, -1, 0, 0, IO_KEPT, IO_FULL), ax[1],
                   u, fwd, st);
  } else {
    const int n1 = int(g.nover[1]), n2 = int(g.nover[2]);
    const int N1 = int(g.nuni[1]), N2 = int(g.nuni[2]);
    run_lines<T>(grid, mk_spec(n0, 0, int64_t(n1) * n2, N1, N2, n2, 1, 1, 2, 1, 1, IO_UNI, IO_FULL),
                 ax[0], u, fwd, st);
    run_lines<T>(grid, mk_spec(n1, 1, n2, n0, N2, int64_t(n1) * n2, 1, -1, 2, 0, 1, IO_KEPT,
                               IO_FULL), ax[1], u, fwd, st);
    run_lines<T>(grid, mk_spec(n2, 2, 1, n0 * n1, 1, n2, 0, -1, -1, 0, 0, IO_KEPT, IO_FULL), ax[2],
                 u, fwd, st);
  }
}

// ---------------------------------------------------------------------------
// Batched FFT passes: the line passes of many transforms (instances of
// different sizes, several transforms each) in one launch.  A job is one pass
// over the lines of one transform; CTA b runs block b - blk0[j] of job j (found
// by binary search over the prefix of block counts).  The uniform array of a
// job comes from the per-call table (pointer and strides of its instance, plus
// the transform's offset), so a captured graph can be replayed on new arrays.
// ---------------------------------------------------------------------------
static bool lines2_config(int n, int64_t es, int nlines, size_t esz, int maxnt, int &lnl, int &nt,
                          size_t &sm) {
  const size_t maxsm = 200 * 1024;
  if (n > FFT2_MAXE * maxnt || n >= (1 << 16)) return false;
  lnl = 0;
  const int want = (es == 1) ? 2048 : 8192;
  if (size_t(2 * n) * esz > maxsm - 8192) return false;
  while ((n << (lnl + 1)) <= want && (1 << (lnl + 1)) <= 16 && (1 << lnl) < nlines &&
         size_t(n << (lnl + 2)) * esz <= maxsm / 2 && (n << (lnl + 1)) <= FFT2_MAXE * maxnt)
    ++lnl;
  const int total = n << lnl;
  nt = 32 * ((total + FFT2_MAXE - 1) / FFT2_MAXE / 32 + 1);
  nt = std::max(64, std::min(maxnt, nt));
  if (total > FFT2_MAXE * nt) return false;
  const int nh = (n + 63) / 64 + 1;
  sm = size_t(2 * total + 64 + nh) * esz + size_t(1 << lnl) * 24;
  return sm <= maxsm;
}

struct FFTJob {
  LineSpec ls;
  StageInfo si;
  UniSpec u;          // ptr / stride[] filled from the per-call table at run time
  const void *tw;
  void *grid;         // this transform's oversampled grid
  int inst;           // instance (row of the per-call table)
  int t;              // transform of the instance
};

template <typename T>
__global__ void __launch_bounds__(fft2_max_threads<T>())
    k_fft_lines_multi(const FFTJob *__restrict__ jobs, const uint32_t *__restrict__ blk0, int njobs,
                      const BatchArray *__restrict__ uni, bool fwd) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ FFTJob job;
  __shared__ int s_j;
  if (threadIdx.x == 0) {
    int lo = 0, hi = njobs - 1;   // last job with blk0 <= blockIdx.x
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (blk0[mid] <= blockIdx.x) lo = mid;
      else hi = mid - 1;
    }
    s_j = lo;
  }
  __syncthreads();
  const int j = s_j;
  for (int i = threadIdx.x; i < int(sizeof(FFTJob) / 4); i += blockDim.x)
    reinterpret_cast<uint32_t *>(&job)[i] = reinterpret_cast<const uint32_t *>(jobs + j)[i];
  __syncthreads();
  if (threadIdx.x == 0) {
    const BatchArray a = uni[job.inst];
    job.u.ptr = static_cast<cplx<T> *>(a.ptr) + int64_t(job.t) * a.stride[0];
    for (int d = 0; d < 3; ++d) job.u.stride[d] = a.stride[d + 1];
  }
  __syncthreads();
  fft_lines_block<T>(static_cast<cplx<T> *>(job.grid), job.ls, job.si,
                     static_cast<const cplx<T> *>(job.tw), job.u, fwd, int(blockIdx.x - blk0[j]),
                     smraw);
}

// device buffer owned by a batch (synchronous allocation at batch creation)
struct DevBufRaw {
  void *p = nullptr;
  DevBufRaw() = default;
  DevBufRaw(const DevBufRaw &) = delete;
  DevBufRaw &operator=(const DevBufRaw &) = delete;
  void alloc(size_t bytes) {
    if (p) cudaFree(p);
    p = nullptr;
    if (bytes) DN_CUDA(cudaMalloc(&p, bytes));
  }
  ~DevBufRaw() {
    if (p) cudaFree(p);
  }
};

struct FFTBatchPass {
  DevBufRaw jobs, blk0;
  int njobs = 0;
  uint32_t nblocks = 0;
  int nt = 64;
  size_t sm = 0;
};

struct FFTBatchImpl {
  bool f64 = false;
  FFTBatchPass pass[2][2];   // [type 1 / type 2][first / second pass]
};

static void batch_pass_upload(FFTBatchPass &bp, const std::vector<FFTJob> &jobs,
                              const std::vector<uint32_t> &blk0, cudaStream_t st) {
  bp.njobs = int(jobs.size());
  bp.jobs.alloc(jobs.size() * sizeof(FFTJob));
  bp.blk0.alloc(blk0.size() * sizeof(uint32_t));
  DN_CUDA(cudaMemcpyAsync(bp.jobs.p, jobs.data(), jobs.size() * sizeof(FFTJob),
                          cudaMemcpyHostToDevice, st));
  DN_CUDA(cudaMemcpyAsync(bp.blk0.p, blk0.data(), blk0.size() * sizeof(uint32_t),
                          cudaMemcpyHostToDevice, st));
}

template <typename T>
void *fft_batch_create(const std::vector<FFTBatchInst> &insts, cudaStream_t st) {
  DN_REQUIRE(!insts.empty(), ST_BADARG, "empty batch");
  auto impl = std::make_unique<FFTBatchImpl>();
  impl->f64 = sizeof(T) == 8;
  const int maxnt = fft2_max_threads<T>();
  for (int type = 0; type < 2; ++type)
    for (int ps = 0; ps < 2; ++ps) {
      std::vector<FFTJob> jobs;
      std::vector<uint32_t> blk0;
      FFTBatchPass &bp = impl->pass[type][ps];
      uint32_t nb = 0;
      for (size_t i = 0; i < insts.size(); ++i) {
        const FFTBatchInst &in = insts[i];
        const Geometry &g = in.g;
        DN_REQUIRE(g.ndim == 2, ST_UNSUPPORTED, "batched transforms: 2D only");
        const int n0 = int(g.nover[0]), n1 = int(g.nover[1]), N1 = int(g.nuni[1]);
        // type 1: rows (full -> kept), then kept columns (-> uniform)
        // type 2: kept columns (uniform -> full), then rows (kept -> full)
        const bool rows = (type == 0) == (ps == 0);
        LineSpec ls = rows ? mk_spec(n1, 1, 1, n0, 1, n1, 0, -1, -1, 0, 0,
                                     type == 0 ? IO_FULL : IO_KEPT, type == 0 ? IO_KEPT : IO_FULL)
                           : mk_spec(n0, 0, n1, 1, N1, 0, 1, -1, 1, 0, 1,
                                     type == 0 ? IO_FULL : IO_UNI, type == 0 ? IO_UNI : IO_FULL);
        const FFTAxisPlan &ax = in.ax[rows ? 1 : 0];
        int lnl, nt;
        size_t sm;
        DN_REQUIRE(lines2_config(ls.n, ls.es, ls.nlines, sizeof(cplx<T>), maxnt, lnl, nt, sm),
                   ST_UNSUPPORTED, "batched transforms: oversampled grid too large");
        ls.nl = lnl;
        bp.nt = std::max(bp.nt, nt);
        bp.sm = std::max(bp.sm, sm);
        const uint32_t blocks = uint32_t((ls.nlines + (1 << lnl) - 1) >> lnl);
        for (int t = 0; t < in.ntrans; ++t) {
          FFTJob jb;
          std::memset(&jb, 0, sizeof(jb));
          jb.ls = ls;
          jb.si = make_stages(ax, lines_maxr<T>());
          const int64_t zero[3] = {0, 0, 0};
          jb.u = mk_uni(nullptr, zero, g, in.corfac, in.fft_order);
          jb.tw = ax.tw;
          jb.grid = static_cast<cplx<T> *>(in.grid) + int64_t(t) * n0 * n1;
          jb.inst = int(i);
          jb.t = t;
          jobs.push_back(jb);
          blk0.push_back(nb);
          nb += blocks;
        }
      }
      bp.nblocks = nb;
      batch_pass_upload(bp, jobs, blk0, st);
    }
  DN_CUDA(cudaStreamSynchronize(st));
  return impl.release();
}

void fft_batch_destroy(void *h) { delete static_cast<FFTBatchImpl *>(h); }

template <typename T>
void fft_batch_run(void *h, int type, const BatchArray *uni, bool fwd, cudaStream_t st) {
  FFTBatchImpl *impl = static_cast<FFTBatchImpl *>(h);
  for (int ps = 0; ps < 2; ++ps) {
    FFTBatchPass &bp = impl->pass[type][ps];
    if (bp.nblocks == 0) continue;
    DN_CUDA(cudaFuncSetAttribute(k_fft_lines_multi<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(bp.sm)));
    k_fft_lines_multi<T><<<bp.nblocks, bp.nt, bp.sm, st>>>(
        static_cast<const FFTJob *>(bp.jobs.p), static_cast<const uint32_t *>(bp.blk0.p),
        bp.njobs, uni, fwd);
    DN_LAUNCHED();
  }
}

template void *fft_batch_create<float>(const std::vector<FFTBatchInst> &, cudaStream_t);
template void *fft_batch_create<double>(const std::vector<FFTBatchInst> &, cudaStream_t);
template void fft_batch_run<float>(void *, int, const BatchArray *, bool, cudaStream_t);
template void fft_batch_run<double>(void *, int, const BatchArray *, bool, cudaStream_t);

// zero a strided array of up to 3 dimensions (element size 8 or 16 bytes)
template <typename E>
__global__ void k_zero_strided(E *p, int64_t n0, int64_t n1, int64_t n2, int64_t s0, int64_t s1,
                               int64_t s2) {
  int64_t tot = n0 * n1 * n2;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < tot;
       i += int64_t(gridDim.x) * blockDim.x) {
    int64_t c = i % n2, r = i / n2, b = r % n1, a = r / n1;
    E z;
    memset(&z, 0, sizeof(E));
    p[a * s0 + b * s1 + c * s2] = z;
  }
}

void zero_strided(void *ptr, int ndim, const int64_t *shape, const int64_t *stride, size_t esize,
                  cudaStream_t st) {
  int64_t n[3] = {1, 1, 1}, s[3] = {0, 0, 0};
  for (int d = 0; d < ndim; ++d) {
    n[3 - ndim + d] = shape[d];
    s[3 - ndim + d] = stride[d];
  }
  int64_t tot = n[0] * n[1] * n[2];
  if (tot == 0) return;
  unsigned blocks = unsigned(std::min<int64_t>((tot + 255) / 256, 4096));
  if (esize == 8)
    k_zero_strided<float2><<<blocks, 256, 0, st>>>((float2 *)ptr, n[0], n[1], n[2], s[0], s[1], s[2]);
  else
    k_zero_strided<double2><<<blocks, 256, 0, st>>>((double2 *)ptr, n[0], n[1], n[2], s[0], s[1],
                                                    s[2]);
  DN_LAUNCHED();
}

template void fft_nu2u_tail<float>(void *, const Geometry &, const FFTAxisPlan *, bool,
                                   const double *const[3], bool, void *, const int64_t *,
                                   cudaStream_t, void *, int *);
template void fft_nu2u_tail<double>(void *, const Geometry &, const FFTAxisPlan *, bool,
                                    const double *const[3], bool, void *, const int64_t *,
                                    cudaStream_t, void *, int *);
template void fft_nu2u_rows<float>(void *, int, const Geometry &, const FFTAxisPlan *, bool,
                                   cudaStream_t, int *);
template void fft_nu2u_rows<double>(void *, int, const Geometry &, const FFTAxisPlan *, bool,
                                    cudaStream_t, int *);
template bool fft_u2nu_cols_range<float>(const void *, const int64_t *, const Geometry &,
                                         const FFTAxisPlan *, bool, const double *const[3], bool,
                                         void *, int, int, cudaStream_t, void *);
template bool fft_u2nu_cols_range<double>(const void *, const int64_t *, const Geometry &,
                                          const FFTAxisPlan *, bool, const double *const[3], bool,
                                          void *, int, int, cudaStream_t, void *);
template void fft_u2nu_rows<float>(void *, int, const Geometry &, const FFTAxisPlan *, bool,
                                   cudaStream_t, int *);
template void fft_u2nu_rows<double>(void *, int, const Geometry &, const FFTAxisPlan *, bool,
                                    cudaStream_t, int *);
template bool fft_nu2u_cols_range<float>(void *, int, int, const Geometry &, const FFTAxisPlan *,
                                         bool, const double *const[3], bool, void *,
                                         const int64_t *, cudaStream_t, void *);
template bool fft_nu2u_cols_range<double>(void *, int, int, const Geometry &,
                                          const FFTAxisPlan *, bool, const double *const[3],
                                          bool, void *, const int64_t *, cudaStream_t, void *);
template void fft_nu2u_cols<float>(void *, const Geometry &, const FFTAxisPlan *, bool,
                                   const double *const[3], bool, void *, const int64_t *,
                                   cudaStream_t, void *);
template void fft_nu2u_cols<double>(void *, const Geometry &, const FFTAxisPlan *, bool,
                                    const double *const[3], bool, void *, const int64_t *,
                                    cudaStream_t, void *);
template void fft_u2nu_head<float>(const void *, const int64_t *, const Geometry &,
                                   const FFTAxisPlan *, bool, const double *const[3], bool,
                                   void *, cudaStream_t, void *, int *);
template void fft_u2nu_head<double>(const void *, const int64_t *, const Geometry &,
                                    const FFTAxisPlan *, bool, const double *const[3], bool,
                                    void *, cudaStream_t, void *, int *);

size_t fft_work_bytes(const Geometry &g, size_t esize) {
  if (g.ndim != 2) return 0;
  return size_t(g.nover[0]) * size_t(g.nuni[1]) * esize;
}

}  // namespace dnufft
