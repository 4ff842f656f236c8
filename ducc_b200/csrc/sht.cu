// Spherical-harmonic synthesis at arbitrary points and its adjoint: the
// counterparts of ducc0.sht.synthesis_general / adjoint_synthesis_general
// (src/ducc0/sht/sht.cc:2926-2994, python/sht_pymod.cc:805-885), spin 0 and
// spin > 0 (modes STANDARD, GRAD_ONLY, DERIV1).
//
// DUCC evaluates the expansion on an equiangular grid (alm2leg), resamples
// the rings in theta, transforms them in phi and interpolates the resulting
// "doubled sphere" grid at the points with its gridding kernel
// (src/ducc0/sht/sphere_interpol.h:418-540).  Here the same idea is arranged
// around this library's transforms:
//
//   F_m(theta) = sum_l a_lm lambda_lm(theta), continued past the pole by
//   F_m(2 pi - theta) = (-1)^m F_m(theta), is a trigonometric polynomial of
//   degree lmax in theta, so with N >= 2 lmax + 2 rings theta_j = 2 pi j / N
//     c_km = (w_m / N) sum_j F_m(theta_j) e^{-i k theta_j},  |k| <= lmax
//   (w_0 = 1, w_m = 2) and the real map is
//     map(theta, phi) = Re sum_{k, 0 <= m <= mmax} c_km e^{i (k theta + m phi)}.
//
//   1. k_alm2leg: F_m on rings 0 .. N/2 by the three-term recurrence of the
//      normalised associated Legendre functions in FP64, one ring pair
//      (theta, pi - theta) per thread (lambda_lm(pi - theta) =
//      (-1)^{l+m} lambda_lm(theta)), with an exponent carried beside each
//      value so that sin^m theta does not underflow; written for all N rings
//      with the weights w_m / N;
//   2. c_km: the DFT along the rings in FP64, by a radix-2 transform in shared
//      memory per m (k_ring_fft, N the power of two from 2 lmax + 2, up to
//      8192 rings: lmax <= 4095);
//   3. the map: a 2D type-2 transform of this library at (theta_i, phi_i)
//      over the modes (k, m - s), s = (mmax + 1) / 2, in the data precision,
//      and Re(z_i e^{i s phi_i}) (k_points_out).
//
// Spin s > 0 (the spin section below): Q + iU is one complex field, the sum
// over -mmax <= m <= mmax of F_m(theta) e^{i m phi} with F_m from the
// Wigner-d recurrence (k_alm2leg_spin, rows m and -m from one recurrence),
// continued by F_m(2 pi - theta) = (-1)^(m+s) F_m(theta); the 2D transform
// runs over (2 lmax + 1) x (2 mmax + 1) modes and its complex result is (Q, U).
//
// The adjoint runs the transposed steps: values map_i e^{-i s phi_i}
// (k_points_in) -> 2D type 1 -> inverse DFT back to the rings -> the rings
// folded onto 0 .. N/2 and k_leg2alm, the transposed recurrence, whose sums
// over the rings of a thread block are reduced per l through shared memory
// and over blocks in a fixed order (no atomics: the result does not depend on
// the launch).
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ducc_b200.h"
#include "ducc_b200_sht.h"
#include "dnufft_internal.h"

namespace dnufft {
namespace sht {

constexpr int LCHUNK = 64;        // l values staged in shared memory per step
constexpr int THREADS = 128;      // threads of the Legendre kernels
constexpr int PAIRS = 2;          // ring pairs per thread (synthesis)
constexpr int PAIRS_ADJ = 4;      // ring pairs per thread (adjoint: its per-l sums cost more)
constexpr int SCALE_EXP = 600;    // a value is v * 2^(SCALE_EXP * scale)
constexpr double RESCALE_ABOVE = 0x1p300;
constexpr double RESCALE_BY = 0x1p-600;

// ---------------------------------------------------------------- helpers
struct Arr {
  void *p = nullptr;
  int dtype = 0;
  int64_t shape[2] = {0, 0};
  int64_t stride[2] = {0, 0};
};

static Arr arr_of(const dnufft_array *a, const char *what) {
  DN_REQUIRE(a != nullptr, ST_BADARG, std::string(what) + ": null array");
  DN_REQUIRE(a->ndim == 2, ST_BADARG, std::string(what) + ": must be a 2D array");
  Arr r;
  r.p = a->data;
  r.dtype = a->dtype;
  int64_t size = 1;
  for (int d = 0; d < 2; ++d) {
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
        throw Error(ST_OOM, "device allocation failed (synthesis_general)");
      }
    }
  }
  Buf(const Buf &) = delete;
  Buf &operator=(const Buf &) = delete;
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

static dnufft_array dev_array(void *p, int dtype, int64_t s0, int64_t s1, int64_t st0,
                              int64_t st1) {
  dnufft_array a;
  std::memset(&a, 0, sizeof(a));
  a.data = p;
  a.dtype = dtype;
  a.ndim = 2;
  a.shape[0] = s0;
  a.shape[1] = s1;
  a.stride[0] = st0;
  a.stride[1] = st1;
  return a;
}

static void check_nufft(int status, const char *what) {
  if (status != 0) throw Error(status, std::string(what) + ": " + dnufft_last_error());
}

static unsigned grid_for(int64_t n, int threads = 256) {
  int64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > 148 * 16) b = 148 * 16;
  return unsigned(b);
}

// n_m = sqrt((2m+1)/(4 pi) prod_{k=1..m} (2k-1)/(2k)) as mantissa * 2^exponent
// (the magnitude of lambda_mm / sin^m theta; DUCC's mfac, sht.cc:133-136),
// accumulated in long double so that the product over m factors keeps FP64
// accuracy.
static void mnorm_table(int mmax, std::vector<double> &mant, std::vector<int> &ex) {
  mant.resize(mmax + 1);
  ex.resize(mmax + 1);
  long double acc = 1.0L;
  long accexp = 0;
  const long double inv4pi = 1.0L / (4.0L * 3.141592653589793238462643383279502884L);
  for (int m = 0; m <= mmax; ++m) {
    if (m > 0) {
      acc *= (long double)(2 * m - 1) / (long double)(2 * m);
      int t;
      acc = frexpl(acc, &t);
      accexp += t;
    }
    int t;
    long double v = frexpl((long double)(2 * m + 1) * inv4pi * acc, &t);
    long e = accexp + t;
    if (e & 1) {
      v *= 2.0L;
      e -= 1;
    }
    mant[m] = double(sqrtl(v));
    ex[m] = int(e / 2);
  }
}

// ---------------------------------------------------------------- Legendre kernels
// lambda_mm(theta) = (-1)^m n_m sin^m theta as value * 2^(SCALE_EXP * scale),
// scale <= 0, |value| < 2^300.  sin^m by binary powering on (mantissa,
// exponent) pairs, so nothing underflows.
__device__ inline void start_value(double s, int m, double nmant, int nexp, double &lam,
                                   int &scale) {
  scale = 0;
  if (m == 0) {
    lam = ldexp(nmant, nexp);
    return;
  }
  if (s <= 0.) {
    lam = 0.;
    return;
  }
  int be;
  double bm = frexp(s, &be);
  double rm = 1.;
  long long re = 0;
  int k = m;
  while (true) {
    int t;
    if (k & 1) {
      rm = frexp(rm * bm, &t);
      re += be + t;
    }
    k >>= 1;
    if (!k) break;
    bm = frexp(bm * bm, &t);
    be = 2 * be + t;
  }
  const long long E = re + nexp;
  // scale = floor((E + 300) / 600)
  long long q = E + SCALE_EXP / 2;
  long long sc = q >= 0 ? q / SCALE_EXP : -((-q + SCALE_EXP - 1) / SCALE_EXP);
  const int rem = int(E - SCALE_EXP * sc);
  lam = ldexp(((m & 1) ? -rm : rm) * nmant, rem);
  scale = int(sc);
}

// recurrence coefficients of lambda_l = alpha_l (x lambda_{l-1} - beta_l lambda_{l-2})
__device__ inline void rec_coeffs(int l, int m, double &alpha, double &beta) {
  const double dl = l, dm = m;
  alpha = sqrt(((2. * dl - 1.) * (2. * dl + 1.)) / ((dl - dm) * (dl + dm)));
  beta = sqrt(((dl - 1. - dm) * (dl - 1. + dm)) / ((2. * dl - 3.) * (2. * dl - 1.)));
}

template <typename C> __device__ inline double2 load_c(const C *p);
template <> __device__ inline double2 load_c<float2>(const float2 *p) {
  const float2 v = *p;
  return make_double2(v.x, v.y);
}
template <> __device__ inline double2 load_c<double2>(const double2 *p) { return *p; }

// ring positions: theta_j = 2 pi j / nring; pair p = (p, nring/2 - p)
__device__ inline void ring_sc(int j, int nring, double &s, double &c) {
  sincospi(2. * double(j) / double(nring), &s, &c);
}

// Recurrence data of the l values l0 .. l0+n-1 (n <= LCHUNK = 64) of one m,
// staged in shared memory by the whole block (two __syncthreads inside):
//   al, be   alpha_l, beta_l of lambda_l = alpha_l (x lambda_{l-1} - beta_l lambda_{l-2})
//   q        Q_l = prod_{k=l0..l} alpha_k
//   gm       gamma_l0 = beta_l0, gamma_l = beta_l / alpha_{l-1} (l > l0)
// With mu_l = lambda_l / Q_l (mu_{l0-1} = lambda_{l0-1}, and lambda_{l0-2} in
// the place of mu_{l0-2}) the recurrence is mu_l = x mu_{l-1} - gamma_l mu_{l-2}:
// two FP64 operations per step instead of three, the factors Q_l going into
// the coefficients (synthesis) or into the per-l sums (adjoint).  Q_l grows
// by about 2 per l (far more just above l = m), so the chunk length bounds it.
__device__ inline void stage_rec(int l0, int n, int m, double *s_al, double *s_be, double *s_q,
                                 double *s_g) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) rec_coeffs(l0 + i, m, s_al[i], s_be[i]);
  __syncthreads();
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    double p0 = lane < n ? s_al[lane] : 1., p1 = lane + 32 < n ? s_al[lane + 32] : 1.;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const double t0 = __shfl_up_sync(0xffffffffu, p0, off);
      const double t1 = __shfl_up_sync(0xffffffffu, p1, off);
      if (lane >= off) {
        p0 *= t0;
        p1 *= t1;
      }
    }
    p1 *= __shfl_sync(0xffffffffu, p0, 31);
    if (lane < n) {
      s_q[lane] = p0;
      s_g[lane] = lane == 0 ? s_be[0] : s_be[lane] / s_al[lane - 1];
    }
    if (lane + 32 < n) {
      s_q[lane + 32] = p1;
      s_g[lane + 32] = s_be[lane + 32] / s_al[lane + 31];
    }
  }
  __syncthreads();
}

// one step of the plain recurrence with the underflow guard
template <int NP>
__device__ inline void step_guarded(double al, double be, const double (&x)[NP], double (&l1)[NP],
                                    double (&l2)[NP], int (&sc)[NP]) {
#pragma unroll
  for (int r = 0; r < NP; ++r) {
    const double ln = al * fma(x[r], l1[r], -be * l2[r]);
    l2[r] = l1[r];
    l1[r] = ln;
    if (sc[r] < 0 && fabs(ln) > RESCALE_ABOVE) {
      l1[r] *= RESCALE_BY;
      l2[r] *= RESCALE_BY;
      ++sc[r];
    }
  }
}

// For m > 0 the pole pair (ring 0 and ring nring/2) is zero (lambda_lm has a
// factor sin^m theta): those rows start at pair 1, and their blocks over the
// pairs number active_blocks(m).
__host__ __device__ inline int pair_offset(int m) { return m > 0 ? 1 : 0; }
__host__ __device__ inline int active_blocks(int m, int npairs, int per_block) {
  return (npairs - pair_offset(m) + per_block - 1) / per_block;
}

// F_m on every ring: V[m][j] = w_m / nring * sum_l a_lm lambda_lm(theta_j),
// rings past the south pole by F_m(2 pi - theta) = (-1)^m F_m(theta).
// grid (mmax + 1, ceil(npairs / (THREADS * PAIRS))), THREADS threads.  A warp
// whose values are all in the double range (scale 0) runs a chunk in the
// rescaled form without the guard; the others step lambda with it.
template <typename C>
__global__ void __launch_bounds__(THREADS) k_alm2leg(
    const C *__restrict__ alm, int64_t astride, const int64_t *__restrict__ mstart,
    int64_t lstride, int lmax, int nring, int npairs, const double *__restrict__ nmant,
    const int *__restrict__ nexp, double2 *__restrict__ V) {
  __shared__ double2 s_a[LCHUNK], s_aq[LCHUNK];
  __shared__ double s_al[LCHUNK], s_be[LCHUNK], s_q[LCHUNK], s_g[LCHUNK];
  const int m = blockIdx.x;
  const int pofs = pair_offset(m);
  if (m > 0 && blockIdx.y == 0 && threadIdx.x == 0) {
    V[int64_t(m) * nring] = make_double2(0., 0.);
    V[int64_t(m) * nring + nring / 2] = make_double2(0., 0.);
  }
  if (int(blockIdx.y) >= active_blocks(m, npairs, THREADS * PAIRS)) return;
  const int64_t m0 = mstart[m];
  double x[PAIRS], l1[PAIRS], l2[PAIRS];
  int sc[PAIRS];
  double2 E[PAIRS], O[PAIRS];
  int jp[PAIRS];
  const double nm = nmant[m];
  const int ne = nexp[m];
  const double2 amm = load_c(alm + (m0 + int64_t(m) * lstride) * astride);
#pragma unroll
  for (int r = 0; r < PAIRS; ++r) {
    jp[r] = pofs + (blockIdx.y * PAIRS + r) * THREADS + threadIdx.x;
    double s = 0., c = 0.;
    if (jp[r] < npairs) ring_sc(jp[r], nring, s, c);
    x[r] = c;
    start_value(s, m, nm, ne, l1[r], sc[r]);
    if (jp[r] >= npairs) l1[r] = 0.;
    l2[r] = 0.;
    const double v = sc[r] == 0 ? l1[r] : 0.;
    E[r] = make_double2(amm.x * v, amm.y * v);
    O[r] = make_double2(0., 0.);
  }
  // chunks start at l0 = m + 1 + 64 k: l0 - m is odd, so even i add to O
  for (int l0 = m + 1; l0 <= lmax; l0 += LCHUNK) {
    const int n = min(LCHUNK, lmax - l0 + 1);
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += THREADS)
      s_a[i] = load_c(alm + (m0 + int64_t(l0 + i) * lstride) * astride);
    stage_rec(l0, n, m, s_al, s_be, s_q, s_g);
    for (int i = threadIdx.x; i < n; i += THREADS)
      s_aq[i] = make_double2(s_a[i].x * s_q[i], s_a[i].y * s_q[i]);
    __syncthreads();
    bool inrange = true;
#pragma unroll
    for (int r = 0; r < PAIRS; ++r) inrange &= sc[r] == 0;
    if (__all_sync(0xffffffffu, inrange)) {
      // mu form: u1 = mu_{l-1}, u2 = mu_{l-2}
      double u1[PAIRS], u2[PAIRS];
#pragma unroll
      for (int r = 0; r < PAIRS; ++r) {
        u1[r] = l1[r];
        u2[r] = l2[r];
      }
      int i = 0;
      for (; i + 1 < n; i += 2) {
        const double g0 = s_g[i], g1 = s_g[i + 1];
        const double2 a0 = s_aq[i], a1 = s_aq[i + 1];
#pragma unroll
        for (int r = 0; r < PAIRS; ++r) {
          const double t0 = fma(x[r], u1[r], -g0 * u2[r]);
          O[r].x = fma(a0.x, t0, O[r].x);
          O[r].y = fma(a0.y, t0, O[r].y);
          const double t1 = fma(x[r], t0, -g1 * u1[r]);
          E[r].x = fma(a1.x, t1, E[r].x);
          E[r].y = fma(a1.y, t1, E[r].y);
          u2[r] = t0;
          u1[r] = t1;
        }
      }
      if (i < n) {
        const double g0 = s_g[i];
        const double2 a0 = s_aq[i];
#pragma unroll
        for (int r = 0; r < PAIRS; ++r) {
          const double t0 = fma(x[r], u1[r], -g0 * u2[r]);
          O[r].x = fma(a0.x, t0, O[r].x);
          O[r].y = fma(a0.y, t0, O[r].y);
          u2[r] = u1[r];
          u1[r] = t0;
        }
      }
      const double q1 = s_q[n - 1], q2 = n >= 2 ? s_q[n - 2] : 1.;
#pragma unroll
      for (int r = 0; r < PAIRS; ++r) {
        l1[r] = u1[r] * q1;
        l2[r] = u2[r] * q2;
      }
    } else {
      for (int i = 0; i < n; ++i) {
        const double2 a = s_a[i];
        step_guarded(s_al[i], s_be[i], x, l1, l2, sc);
#pragma unroll
        for (int r = 0; r < PAIRS; ++r) {
          const double v = sc[r] == 0 ? l1[r] : 0.;
          if ((i & 1) == 0) {
            O[r].x = fma(a.x, v, O[r].x);
            O[r].y = fma(a.y, v, O[r].y);
          } else {
            E[r].x = fma(a.x, v, E[r].x);
            E[r].y = fma(a.y, v, E[r].y);
          }
        }
      }
    }
  }
  const double w = (m == 0 ? 1. : 2.) / double(nring);
  const double sg = (m & 1) ? -w : w;
  const int half = nring / 2;
  double2 *row = V + int64_t(m) * nring;
#pragma unroll
  for (int r = 0; r < PAIRS; ++r) {
    const int j = jp[r];
    if (j >= npairs) continue;
    const double2 vn = make_double2(E[r].x + O[r].x, E[r].y + O[r].y);
    const double2 vs = make_double2(E[r].x - O[r].x, E[r].y - O[r].y);
    row[j] = make_double2(w * vn.x, w * vn.y);
    if (j > 0 && j < half) row[nring - j] = make_double2(sg * vn.x, sg * vn.y);
    const int js = half - j;
    if (js != j) {
      row[js] = make_double2(w * vs.x, w * vs.y);
      if (js > 0 && js < half) row[nring - js] = make_double2(sg * vs.x, sg * vs.y);
    }
  }
}

// Transposed: part[b][mofs[m] + l] = sum over the ring pairs of block b of
// lambda_lm(theta_j) G_m(theta_j), G the ring values g[m][*] folded onto
// rings 0 .. nring/2 (g(theta_j) + (-1)^m g(2 pi - theta_j)).  Per thread the
// contributions of its pairs are summed in registers, per warp through a
// shared-memory transpose of 8 l values at a time, per block over its warps.
// grid (mmax + 1, nblk), THREADS threads.  Chunks after the first run in the
// rescaled form for warps whose values are all in the double range (the
// warp's per-l sums then take the factor Q_l).
__global__ void __launch_bounds__(THREADS) k_leg2alm(
    const double2 *__restrict__ g, int lmax, int nring, int npairs,
    const double *__restrict__ nmant, const int *__restrict__ nexp,
    const int64_t *__restrict__ mofs, int64_t nalm_dense, double2 *__restrict__ part) {
  constexpr int NW = THREADS / 32;
  __shared__ double s_al[LCHUNK], s_be[LCHUNK], s_q[LCHUNK], s_g[LCHUNK];
  __shared__ double2 s_tr[NW][8][33];
  __shared__ double2 s_blk[LCHUNK][NW];
  const int m = blockIdx.x;
  if (int(blockIdx.y) >= active_blocks(m, npairs, THREADS * PAIRS_ADJ)) return;
  const int pofs = pair_offset(m);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int half = nring / 2;
  const double2 *row = g + int64_t(m) * nring;
  const double sgn = (m & 1) ? -1. : 1.;
  double x[PAIRS_ADJ], l1[PAIRS_ADJ], l2[PAIRS_ADJ];
  int sc[PAIRS_ADJ];
  double2 P[PAIRS_ADJ], Q[PAIRS_ADJ];
#pragma unroll
  for (int r = 0; r < PAIRS_ADJ; ++r) {
    const int j = pofs + (blockIdx.y * PAIRS_ADJ + r) * THREADS + threadIdx.x;
    double s = 0., c = 0.;
    double2 gn = make_double2(0., 0.), gs = make_double2(0., 0.);
    if (j < npairs) {
      ring_sc(j, nring, s, c);
      gn = row[j];
      if (j > 0 && j < half) {
        const double2 t = row[nring - j];
        gn.x += sgn * t.x;
        gn.y += sgn * t.y;
      }
      const int js = half - j;
      if (js != j) {
        gs = row[js];
        if (js > 0 && js < half) {
          const double2 t = row[nring - js];
          gs.x += sgn * t.x;
          gs.y += sgn * t.y;
        }
      }
    }
    x[r] = c;
    start_value(s, m, nmant[m], nexp[m], l1[r], sc[r]);
    if (j >= npairs) l1[r] = 0.;
    l2[r] = 0.;
    P[r] = make_double2(gn.x + gs.x, gn.y + gs.y);
    Q[r] = make_double2(gn.x - gs.x, gn.y - gs.y);
  }
  const int li = lane & 7, part8 = lane >> 3;
  // chunks start at l0 = m + 64 k: l0 - m is even, so odd i take Q
  for (int l0 = m; l0 <= lmax; l0 += LCHUNK) {
    const int n = min(LCHUNK, lmax - l0 + 1);
    __syncthreads();
    stage_rec(l0, n, m, s_al, s_be, s_q, s_g);
    bool inrange = true;
#pragma unroll
    for (int r = 0; r < PAIRS_ADJ; ++r) inrange &= sc[r] == 0;
    const bool fast = l0 > m && __all_sync(0xffffffffu, inrange);
    double u1[PAIRS_ADJ], u2[PAIRS_ADJ];
#pragma unroll
    for (int r = 0; r < PAIRS_ADJ; ++r) {
      u1[r] = l1[r];
      u2[r] = l2[r];
    }
    for (int i8 = 0; i8 < n; i8 += 8) {
      if (fast) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const int i = i8 + k;
          double2 c = make_double2(0., 0.);
          if (i < n) {
            const double gi = s_g[i];
#pragma unroll
            for (int r = 0; r < PAIRS_ADJ; ++r) {
              const double t = fma(x[r], u1[r], -gi * u2[r]);
              u2[r] = u1[r];
              u1[r] = t;
              const double2 f = (k & 1) ? Q[r] : P[r];
              c.x = fma(t, f.x, c.x);
              c.y = fma(t, f.y, c.y);
            }
          }
          s_tr[warp][k][lane] = c;
        }
      } else {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const int i = i8 + k;
          const int l = l0 + i;
          double2 c = make_double2(0., 0.);
          if (i < n) {
            if (l > m) step_guarded(s_al[i], s_be[i], x, l1, l2, sc);
#pragma unroll
            for (int r = 0; r < PAIRS_ADJ; ++r) {
              const double v = sc[r] == 0 ? l1[r] : 0.;
              const double2 f = (k & 1) ? Q[r] : P[r];
              c.x = fma(v, f.x, c.x);
              c.y = fma(v, f.y, c.y);
            }
          }
          s_tr[warp][k][lane] = c;
        }
      }
      __syncwarp();
      double2 t = make_double2(0., 0.);
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const double2 u = s_tr[warp][li][part8 * 8 + k];
        t.x += u.x;
        t.y += u.y;
      }
      t.x += __shfl_xor_sync(0xffffffffu, t.x, 8);
      t.y += __shfl_xor_sync(0xffffffffu, t.y, 8);
      t.x += __shfl_xor_sync(0xffffffffu, t.x, 16);
      t.y += __shfl_xor_sync(0xffffffffu, t.y, 16);
      if (part8 == 0) {
        if (fast && i8 + li < n) {
          const double q = s_q[i8 + li];
          t.x *= q;
          t.y *= q;
        }
        s_blk[i8 + li][warp] = t;
      }
      __syncwarp();
    }
    if (fast) {
      const double q1 = s_q[n - 1], q2 = n >= 2 ? s_q[n - 2] : 1.;
#pragma unroll
      for (int r = 0; r < PAIRS_ADJ; ++r) {
        l1[r] = u1[r] * q1;
        l2[r] = u2[r] * q2;
      }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += THREADS) {
      double2 t = s_blk[i][0];
#pragma unroll
      for (int w = 1; w < NW; ++w) {
        t.x += s_blk[i][w].x;
        t.y += s_blk[i][w].y;
      }
      part[int64_t(blockIdx.y) * nalm_dense + mofs[m] + (l0 + i)] = t;
    }
  }
}

// alm[(mstart[m] + l lstride) astride] = sum_b part[b][mofs[m] + l] / nring,
// in the order of b (the active blocks of m); imaginary part 0 for m = 0 (a_l0 of a real map is real).
template <typename C>
__global__ void k_alm_out(const double2 *__restrict__ part, int npairs, int64_t nalm_dense,
                          const int64_t *__restrict__ mofs, const int64_t *__restrict__ mstart,
                          int64_t lstride, int64_t astride, int lmax, int nm, double scale,
                          C *__restrict__ alm) {
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < nalm_dense;
       e += int64_t(gridDim.x) * blockDim.x) {
    // m of dense index e: mofs[m] + m <= e < mofs[m+1] + m + 1 (binary search)
    int lo = 0, hi = nm - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (mofs[mid] + mid <= e) lo = mid;
      else hi = mid - 1;
    }
    const int m = lo;
    const int64_t l = e - mofs[m];
    double2 t = make_double2(0., 0.);
    const int nblk = active_blocks(m, npairs, THREADS * PAIRS_ADJ);
    for (int b = 0; b < nblk; ++b) {
      const double2 u = part[int64_t(b) * nalm_dense + e];
      t.x += u.x;
      t.y += u.y;
    }
    t.x *= scale;
    t.y = m == 0 ? 0. : t.y * scale;
    C o;
    o.x = decltype(o.x)(t.x);
    o.y = decltype(o.y)(t.y);
    alm[(mstart[m] + l * lstride) * astride] = o;
    (void)lmax;
  }
}

// ---------------------------------------------------------------- point kernels
// map_i = Re(z_i e^{i s phi_i})
template <typename C, typename T>
__global__ void k_points_out(const C *__restrict__ z, const double *__restrict__ loc,
                             int64_t ls0, int64_t ls1, int64_t n, double s, T *__restrict__ map,
                             int64_t ms) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    double sn, cs;
    sincos(s * loc[i * ls0 + ls1], &sn, &cs);
    const C v = z[i];
    map[i * ms] = T(double(v.x) * cs - double(v.y) * sn);
  }
}

// z_i = map_i e^{-i s phi_i}
template <typename C, typename T>
__global__ void k_points_in(const T *__restrict__ map, int64_t ms, const double *__restrict__ loc,
                            int64_t ls0, int64_t ls1, int64_t n, double s, C *__restrict__ z) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    double sn, cs;
    sincos(s * loc[i * ls0 + ls1], &sn, &cs);
    const double f = double(map[i * ms]);
    C v;
    v.x = decltype(v.x)(f * cs);
    v.y = decltype(v.y)(-f * sn);
    z[i] = v;
  }
}

template <typename A, typename B>
__global__ void k_convert(const A *__restrict__ in, int64_t n, B *__restrict__ out) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    const A v = in[i];
    B o;
    o.x = decltype(o.x)(v.x);
    o.y = decltype(o.y)(v.y);
    out[i] = o;
  }
}

// ---------------------------------------------------------------- spin > 0
template <typename B> __device__ inline B from_d2b(const double2 &v) {
  B o;
  o.x = decltype(o.x)(v.x);
  o.y = decltype(o.y)(v.y);
  return o;
}

// D_lm(theta) = sqrt((2l+1)/(4 pi)) d^l_{m,-s}(theta) for l >= l0 = max(|m|, s):
// the three-term recurrence of the Wigner d functions in l,
//   D_l = alpha_l (x - beta_l) D_{l-1} - gamma_l D_{l-2},
//   alpha_l = l sqrt((2l+1)(2l-1)) / sqrt((l^2-m^2)(l^2-s^2)),
//   beta_l  = -m s / (l (l-1)),
//   gamma_l = l/(l-1) sqrt((2l+1)/(2l-3)) sqrt(((l-1)^2-m^2)((l-1)^2-s^2)/((l^2-m^2)(l^2-s^2))),
// started from D_l0 = N_m cos(theta/2)^pc sin(theta/2)^ps (the single term
// of Wigner's sum at l = l0; N_m with its sign from the host table).
struct SpinStart {
  int l0, pc, ps;
  double mant;   // N_m = mant * 2^ex
  int ex;
};

__device__ inline void spin_coeffs(int l, int m, int sp, double &al, double &be, double &ga) {
  const double dl = l, dm = m, ds = sp;
  const double den = sqrt((dl * dl - dm * dm) * (dl * dl - ds * ds));
  al = dl * sqrt((2. * dl + 1.) * (2. * dl - 1.)) / den;
  be = -dm * ds / (dl * (dl - 1.));
  const double l1 = dl - 1.;
  ga = dl / l1 * sqrt((2. * dl + 1.) / (2. * dl - 3.)) *
       sqrt(fmax((l1 * l1 - dm * dm) * (l1 * l1 - ds * ds), 0.)) / den;
}

// c^pc sn^ps * mant * 2^ex as value * 2^(SCALE_EXP * scale)
__device__ inline void spin_start(double c, double sn, const SpinStart &S, double &v, int &scale) {
  scale = 0;
  if ((c <= 0. && S.pc > 0) || (sn <= 0. && S.ps > 0)) {
    v = 0.;
    return;
  }
  double rm = S.mant;
  long long re = S.ex;
  const double bases[2] = {c, sn};
  const int pw[2] = {S.pc, S.ps};
#pragma unroll
  for (int b = 0; b < 2; ++b) {
    int k = pw[b];
    if (k == 0) continue;
    int be;
    double bm = frexp(bases[b], &be);
    while (true) {
      int t;
      if (k & 1) {
        rm = frexp(rm * bm, &t);
        re += be + t;
      }
      k >>= 1;
      if (!k) break;
      bm = frexp(bm * bm, &t);
      be = 2 * be + t;
    }
  }
  int t;
  rm = frexp(rm, &t);
  re += t;
  long long q = re + SCALE_EXP / 2;
  long long sc = q >= 0 ? q / SCALE_EXP : -((-q + SCALE_EXP - 1) / SCALE_EXP);
  v = ldexp(rm, int(re - SCALE_EXP * sc));
  scale = int(sc);
}

// the coefficient of D_lm in Q + iU: sigma (E + iB) for m >= 0,
// sigma (-1)^m (conj E + i conj B) for m < 0 (E_{l,-m} = (-1)^m conj E_lm);
// sigma = (-1)^(s+1); DERIV1: E sqrt(l (l+1)), no B
template <typename C>
__device__ inline double2 spin_coef(const C *alm, int64_t cstride, int64_t astride, int64_t idx,
                                    int m, int l, int mode, double sigma) {
  double2 e = load_c(alm + idx * astride);
  double2 b = make_double2(0., 0.);
  if (mode == DNUFFT_SHT_STANDARD) b = load_c(alm + cstride + idx * astride);
  if (mode == DNUFFT_SHT_DERIV1) {
    const double f = sqrt(double(l) * double(l + 1));
    e.x *= f;
    e.y *= f;
  }
  if (m >= 0) return make_double2(sigma * (e.x - b.y), sigma * (e.y + b.x));
  const double sg = (m & 1) ? -sigma : sigma;
  return make_double2(sg * (e.x + b.y), sg * (b.x - e.y));
}

// F_m on the rings: V[mmax + m][j] = sum_l A_lm D_lm(theta_j) / nring, continued
// by V[row][nring - j] = (-1)^(m+s) V[row][j].  One block row per m >= 0: since
// D_{l,-m}(theta) = (-1)^(l+s) D_lm(pi - theta), the recurrence of D_lm at ring j
// also gives row -m at ring nring/2 - j (its coefficient staged with the sign).
// RINGS rings per thread; grid (mmax + 1, blocks over rings 0 .. nring/2).
// Chunks of warps whose values are all in the double range run without the
// underflow guard.
constexpr int RINGS = 2;
template <typename C>
__global__ void __launch_bounds__(THREADS) k_alm2leg_spin(
    const C *__restrict__ alm, int64_t cstride, int64_t astride,
    const int64_t *__restrict__ mstart, int64_t lstride, int lmax, int mmax, int sp, int mode,
    int nring, const SpinStart *__restrict__ starts, double2 *__restrict__ V) {
  __shared__ double2 s_ap[LCHUNK], s_an[LCHUNK];
  __shared__ double s_al[LCHUNK], s_be[LCHUNK], s_ga[LCHUNK];
  const int m = blockIdx.x;
  const bool neg = m > 0;   // row -m handled too
  const SpinStart S = starts[mmax + m];
  const int half = nring / 2;
  const double sigma = (sp & 1) ? 1. : -1.;
  const int64_t m0 = mstart[m];
  double x[RINGS], d1[RINGS], d2[RINGS];
  int sc[RINGS], jr[RINGS];
  double2 Fp[RINGS], Fn[RINGS];
  const int64_t i0 = m0 + int64_t(S.l0) * lstride;
  const double2 a0 = spin_coef(alm, cstride, astride, i0, m, S.l0, mode, sigma);
  double2 b0 = make_double2(0., 0.);
  if (neg) {
    b0 = spin_coef(alm, cstride, astride, i0, -m, S.l0, mode, sigma);
    if ((S.l0 + sp) & 1) b0 = make_double2(-b0.x, -b0.y);
  }
#pragma unroll
  for (int r = 0; r < RINGS; ++r) {
    jr[r] = (blockIdx.y * RINGS + r) * THREADS + threadIdx.x;
    double c = 1., sn = 0.;
    x[r] = 1.;
    if (jr[r] <= half) {
      sincospi(double(jr[r]) / double(nring), &sn, &c);
      x[r] = cospi(2. * double(jr[r]) / double(nring));
    }
    spin_start(c, sn, S, d1[r], sc[r]);
    if (jr[r] > half) d1[r] = 0.;
    d2[r] = 0.;
    const double v = sc[r] == 0 ? d1[r] : 0.;
    Fp[r] = make_double2(a0.x * v, a0.y * v);
    Fn[r] = make_double2(b0.x * v, b0.y * v);
  }
  for (int l0 = S.l0 + 1; l0 <= lmax; l0 += LCHUNK) {
    const int n = min(LCHUNK, lmax - l0 + 1);
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += THREADS) {
      const int l = l0 + i;
      const int64_t idx = m0 + int64_t(l) * lstride;
      s_ap[i] = spin_coef(alm, cstride, astride, idx, m, l, mode, sigma);
      double2 b = make_double2(0., 0.);
      if (neg) {
        b = spin_coef(alm, cstride, astride, idx, -m, l, mode, sigma);
        if ((l + sp) & 1) b = make_double2(-b.x, -b.y);
      }
      s_an[i] = b;
      spin_coeffs(l, m, sp, s_al[i], s_be[i], s_ga[i]);
    }
    __syncthreads();
    bool inrange = true;
#pragma unroll
    for (int r = 0; r < RINGS; ++r) inrange &= sc[r] == 0;
    if (__all_sync(0xffffffffu, inrange)) {
      for (int i = 0; i < n; ++i) {
        const double al = s_al[i], be = s_be[i], ga = s_ga[i];
        const double2 a = s_ap[i], b = s_an[i];
#pragma unroll
        for (int r = 0; r < RINGS; ++r) {
          const double dn = fma(al * (x[r] - be), d1[r], -ga * d2[r]);
          d2[r] = d1[r];
          d1[r] = dn;
          Fp[r].x = fma(a.x, dn, Fp[r].x);
          Fp[r].y = fma(a.y, dn, Fp[r].y);
          Fn[r].x = fma(b.x, dn, Fn[r].x);
          Fn[r].y = fma(b.y, dn, Fn[r].y);
        }
      }
    } else {
      for (int i = 0; i < n; ++i) {
        const double al = s_al[i], be = s_be[i], ga = s_ga[i];
        const double2 a = s_ap[i], b = s_an[i];
#pragma unroll
        for (int r = 0; r < RINGS; ++r) {
          const double dn = fma(al * (x[r] - be), d1[r], -ga * d2[r]);
          d2[r] = d1[r];
          d1[r] = dn;
          if (sc[r] < 0 && fabs(dn) > RESCALE_ABOVE) {
            d1[r] *= RESCALE_BY;
            d2[r] *= RESCALE_BY;
            ++sc[r];
          }
          const double v = sc[r] == 0 ? d1[r] : 0.;
          Fp[r].x = fma(a.x, v, Fp[r].x);
          Fp[r].y = fma(a.y, v, Fp[r].y);
          Fn[r].x = fma(b.x, v, Fn[r].x);
          Fn[r].y = fma(b.y, v, Fn[r].y);
        }
      }
    }
  }
  const double w = 1. / double(nring);
  const double sg = ((m + sp) & 1) ? -w : w;   // (-1)^(m+s) = (-1)^(-m+s)
  double2 *op = V + int64_t(mmax + m) * nring;
  double2 *on = V + int64_t(mmax - m) * nring;
#pragma unroll
  for (int r = 0; r < RINGS; ++r) {
    const int j = jr[r];
    if (j > half) continue;
    op[j] = make_double2(w * Fp[r].x, w * Fp[r].y);
    if (j > 0 && j < half) op[nring - j] = make_double2(sg * Fp[r].x, sg * Fp[r].y);
    if (neg) {
      const int jn = half - j;
      on[jn] = make_double2(w * Fn[r].x, w * Fn[r].y);
      if (jn > 0 && jn < half) on[nring - jn] = make_double2(sg * Fn[r].x, sg * Fn[r].y);
    }
  }
}

// Transposed: part[b][mmax + m][l] = sum over the rings of block b of
// D_lm(theta_j) G_m(theta_j) and part[b][mmax - m][l] =
// (-1)^(l+s) sum_j D_lm(theta_j) G_-m(theta_{nring/2 - j}) (the same recurrence,
// D_{l,-m}(theta) = (-1)^(l+s) D_lm(pi - theta)), G = g[row][j] +
// (-1)^(m+s) g[row][nring - j] (0 < j < nring/2), for l0 <= l <= lmax; sums per
// warp through the shared-memory transpose of 8 l values, per block over its
// warps.
__global__ void __launch_bounds__(THREADS) k_leg2alm_spin(
    const double2 *__restrict__ g, int lmax, int mmax, int sp, int nring,
    const SpinStart *__restrict__ starts, double2 *__restrict__ part) {
  constexpr int NW = THREADS / 32;
  __shared__ double s_al[LCHUNK], s_be[LCHUNK], s_ga[LCHUNK];
  __shared__ double2 s_tr[2][NW][8][33];
  __shared__ double2 s_blk[2][LCHUNK][NW];
  const int m = blockIdx.x;
  const bool neg = m > 0;
  const SpinStart S = starts[mmax + m];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int half = nring / 2;
  const double2 *inp = g + int64_t(mmax + m) * nring;
  const double2 *inn = g + int64_t(mmax - m) * nring;
  const double sgn = ((m + sp) & 1) ? -1. : 1.;
  double x[RINGS], d1[RINGS], d2[RINGS];
  int sc[RINGS];
  double2 Gp[RINGS], Gn[RINGS];
#pragma unroll
  for (int r = 0; r < RINGS; ++r) {
    const int j = (blockIdx.y * RINGS + r) * THREADS + threadIdx.x;
    double c = 1., sn = 0.;
    x[r] = 1.;
    Gp[r] = make_double2(0., 0.);
    Gn[r] = make_double2(0., 0.);
    if (j <= half) {
      sincospi(double(j) / double(nring), &sn, &c);
      x[r] = cospi(2. * double(j) / double(nring));
      Gp[r] = inp[j];
      if (j > 0 && j < half) {
        const double2 t = inp[nring - j];
        Gp[r].x += sgn * t.x;
        Gp[r].y += sgn * t.y;
      }
      if (neg) {
        const int jn = half - j;
        Gn[r] = inn[jn];
        if (jn > 0 && jn < half) {
          const double2 t = inn[nring - jn];
          Gn[r].x += sgn * t.x;
          Gn[r].y += sgn * t.y;
        }
      }
    }
    spin_start(c, sn, S, d1[r], sc[r]);
    if (j > half) d1[r] = 0.;
    d2[r] = 0.;
  }
  const int li = lane & 7, part8 = lane >> 3;
  const int64_t rowlen = lmax + 1;
  const int64_t bofs = int64_t(blockIdx.y) * (2 * mmax + 1) * rowlen;
  for (int l0 = S.l0; l0 <= lmax; l0 += LCHUNK) {
    const int n = min(LCHUNK, lmax - l0 + 1);
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += THREADS) {
      const int l = l0 + i;
      if (l > S.l0) {
        spin_coeffs(l, m, sp, s_al[i], s_be[i], s_ga[i]);
      } else {
        s_al[i] = 0.;
        s_be[i] = 0.;
        s_ga[i] = 0.;
      }
    }
    __syncthreads();
    bool inrange = true;
#pragma unroll
    for (int r = 0; r < RINGS; ++r) inrange &= sc[r] == 0;
    const bool fast = l0 > S.l0 && __all_sync(0xffffffffu, inrange);
    for (int i8 = 0; i8 < n; i8 += 8) {
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int i = i8 + k;
        double2 cp = make_double2(0., 0.), cn = make_double2(0., 0.);
        if (i < n) {
          if (l0 + i > S.l0) {
            const double al = s_al[i], be = s_be[i], ga = s_ga[i];
#pragma unroll
            for (int r = 0; r < RINGS; ++r) {
              const double dn = fma(al * (x[r] - be), d1[r], -ga * d2[r]);
              d2[r] = d1[r];
              d1[r] = dn;
              if (!fast && sc[r] < 0 && fabs(dn) > RESCALE_ABOVE) {
                d1[r] *= RESCALE_BY;
                d2[r] *= RESCALE_BY;
                ++sc[r];
              }
            }
          }
#pragma unroll
          for (int r = 0; r < RINGS; ++r) {
            const double v = (fast || sc[r] == 0) ? d1[r] : 0.;
            cp.x = fma(v, Gp[r].x, cp.x);
            cp.y = fma(v, Gp[r].y, cp.y);
            cn.x = fma(v, Gn[r].x, cn.x);
            cn.y = fma(v, Gn[r].y, cn.y);
          }
        }
        s_tr[0][warp][k][lane] = cp;
        s_tr[1][warp][k][lane] = cn;
      }
      __syncwarp();
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        double2 t = make_double2(0., 0.);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const double2 u = s_tr[h][warp][li][part8 * 8 + k];
          t.x += u.x;
          t.y += u.y;
        }
        t.x += __shfl_xor_sync(0xffffffffu, t.x, 8);
        t.y += __shfl_xor_sync(0xffffffffu, t.y, 8);
        t.x += __shfl_xor_sync(0xffffffffu, t.x, 16);
        t.y += __shfl_xor_sync(0xffffffffu, t.y, 16);
        if (part8 == 0) s_blk[h][i8 + li][warp] = t;
      }
      __syncwarp();
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += THREADS) {
      double2 tp = s_blk[0][i][0], tn = s_blk[1][i][0];
#pragma unroll
      for (int w = 1; w < NW; ++w) {
        tp.x += s_blk[0][i][w].x;
        tp.y += s_blk[0][i][w].y;
        tn.x += s_blk[1][i][w].x;
        tn.y += s_blk[1][i][w].y;
      }
      const int l = l0 + i;
      part[bofs + (mmax + m) * rowlen + l] = tp;
      if (neg) {
        const double f = ((l + sp) & 1) ? -1. : 1.;
        part[bofs + (mmax - m) * rowlen + l] = make_double2(f * tn.x, f * tn.y);
      }
    }
  }
}

// E' = sigma (W_m + (-1)^m conj W_-m) / 2, B' = -i sigma (W_m - (-1)^m conj W_-m) / 2
// with W summed over the blocks in order and divided by nring; DERIV1: E'
// times sqrt(l (l+1)); zero for l < s.  One thread per (m >= 0, l) of the
// dense layout.
template <typename C>
__global__ void k_alm_out_spin(const double2 *__restrict__ part, int nblk, int64_t nalm_dense,
                               const int64_t *__restrict__ mofs,
                               const int64_t *__restrict__ mstart, int64_t lstride,
                               int64_t cstride, int64_t astride, int lmax, int mmax, int sp,
                               int mode, double scale, C *__restrict__ alm) {
  const int nm = mmax + 1;
  const int64_t rowlen = lmax + 1, blkstride = int64_t(2 * mmax + 1) * rowlen;
  const double sigma = (sp & 1) ? 1. : -1.;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < nalm_dense;
       e += int64_t(gridDim.x) * blockDim.x) {
    int lo = 0, hi = nm - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (mofs[mid] + mid <= e) lo = mid;
      else hi = mid - 1;
    }
    const int m = lo;
    const int l = int(e - mofs[m]);
    double2 E = make_double2(0., 0.), B = make_double2(0., 0.);
    if (l >= sp) {
      double2 wp = make_double2(0., 0.), wn = make_double2(0., 0.);
      for (int b = 0; b < nblk; ++b) {
        const double2 u = part[b * blkstride + (mmax + m) * rowlen + l];
        const double2 v = part[b * blkstride + (mmax - m) * rowlen + l];
        wp.x += u.x;
        wp.y += u.y;
        wn.x += v.x;
        wn.y += v.y;
      }
      const double f = (m & 1) ? -1. : 1.;
      const double h = 0.5 * sigma * scale;
      // conj(wn) = (wn.x, -wn.y)
      E = make_double2(h * (wp.x + f * wn.x), h * (wp.y - f * wn.y));
      // -i (a + i b) = b - i a with (a + i b) = wp - f conj(wn)
      const double ar = wp.x - f * wn.x, ai = wp.y + f * wn.y;
      B = make_double2(h * ai, -h * ar);
      if (mode == DNUFFT_SHT_DERIV1) {
        const double d = sqrt(double(l) * double(l + 1));
        E.x *= d;
        E.y *= d;
      }
    }
    const int64_t idx = (mstart[m] + int64_t(l) * lstride) * astride;
    alm[idx] = from_d2b<C>(E);
    if (mode == DNUFFT_SHT_STANDARD) alm[cstride + idx] = from_d2b<C>(B);
  }
}

// Q_i + i U_i = z_i (synthesis) and z_i = Q_i + i U_i (adjoint)
template <typename C, typename T>
__global__ void k_points_out_spin(const C *__restrict__ z, int64_t n, T *__restrict__ map,
                                  int64_t rs, int64_t ms) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    const C v = z[i];
    map[i * ms] = T(v.x);
    map[rs + i * ms] = T(v.y);
  }
}
template <typename C, typename T>
__global__ void k_points_in_spin(const T *__restrict__ map, int64_t rs, int64_t ms, int64_t n,
                                 C *__restrict__ z) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    C v;
    v.x = map[i * ms];
    v.y = map[rs + i * ms];
    z[i] = v;
  }
}

// The DFT along the rings (a power of two of them, up to FFT_MAX): one CTA
// per m, an in-place radix-2 transform in shared memory
// (bit-reversed load, log2 N butterfly stages, twiddles from a table made by
// the CTA).  Forward (synthesis): c[k + lmax][m] = sum_j V[m][j] e^{-2 pi i jk/N}
// for |k| <= lmax, written in the data precision as the 2D transform's
// (nk, nm) uniform array.  Inverse (adjoint): g[m][j] = sum_k H[k + lmax][m]
// e^{2 pi i jk/N}, H the 2D type-1 result (nk, nm).
constexpr int FFT_MAX = 8192;
constexpr int FFT_THREADS = 512;

template <typename A> __device__ inline double2 to_d2(const A &v) {
  return make_double2(double(v.x), double(v.y));
}
template <typename B> __device__ inline B from_d2(const double2 &v) {
  B o;
  o.x = decltype(o.x)(v.x);
  o.y = decltype(o.y)(v.y);
  return o;
}

template <typename Cin, typename Cout, bool INVERSE>
__global__ void __launch_bounds__(FFT_THREADS) k_ring_fft(const Cin *__restrict__ in,
                                                          Cout *__restrict__ out, int log2n,
                                                          int lmax, int nm) {
  extern __shared__ double2 sm[];
  const int n = 1 << log2n;
  double2 *data = sm;
  double2 *tw = sm + n;
  const int m = blockIdx.x;
  const int nk = 2 * lmax + 1;
  for (int i = threadIdx.x; i < n / 2; i += blockDim.x) {
    double sn, cs;
    sincospi(2. * double(i) / double(n), &sn, &cs);
    tw[i] = make_double2(cs, INVERSE ? sn : -sn);
  }
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    double2 v;
    if (!INVERSE) {
      v = to_d2(in[int64_t(m) * n + j]);
    } else {
      const int k = j <= lmax ? j : (j >= n - lmax ? j - n : INT_MIN);
      v = k == INT_MIN ? make_double2(0., 0.) : to_d2(in[int64_t(k + lmax) * nm + m]);
    }
    data[__brev(unsigned(j)) >> (32 - log2n)] = v;
  }
  __syncthreads();
  for (int s = 1; s <= log2n; ++s) {
    const int half = 1 << (s - 1);
    const int tstep = n >> s;   // twiddle stride
    for (int b = threadIdx.x; b < n / 2; b += blockDim.x) {
      const int pos = b & (half - 1);
      const int i0 = ((b >> (s - 1)) << s) + pos;
      const double2 w = tw[pos * tstep];
      const double2 u = data[i0], v = data[i0 + half];
      const double2 t = make_double2(w.x * v.x - w.y * v.y, w.x * v.y + w.y * v.x);
      data[i0] = make_double2(u.x + t.x, u.y + t.y);
      data[i0 + half] = make_double2(u.x - t.x, u.y - t.y);
    }
    __syncthreads();
  }
  if (!INVERSE) {
    for (int i = threadIdx.x; i < nk; i += blockDim.x) {
      const int k = i - lmax;
      out[int64_t(i) * nm + m] = from_d2<Cout>(data[k < 0 ? k + n : k]);
    }
  } else {
    for (int j = threadIdx.x; j < n; j += blockDim.x)
      out[int64_t(m) * n + j] = from_d2<Cout>(data[j]);
  }
}

// ---------------------------------------------------------------- host side
struct Problem {
  int lmax = 0, mmax = 0;
  int spin = 0, mode = 0;
  int rows = 0;            // transforms along the rings: mmax + 1 (spin 0), 2 mmax + 1
  int nblk_spin = 0;       // blocks over the rings 0 .. nring/2 (spin > 0)
  int log2n = 0;           // nring = 2^log2n rings (the ring DFT's length)
  int nring = 0, npairs = 0, nk = 0, nblk = 0, nblk_adj = 0;
  int64_t npts = 0;
  int64_t nalm_dense = 0;
  double s = 0;            // phi mode shift (mmax + 1) / 2
  double eps2 = 0;
  bool f64 = false;
  dnufft_opts po2;         // point transforms, parameters forced
};

struct Tables {
  Buf mstart, mofs, nmant, nexp;
};

static void upload(Buf &b, const void *src, size_t bytes, cudaStream_t st) {
  DN_CUDA(cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyHostToDevice, st));
}

// The kernel and oversampled sizes of the ring transforms and of the point
// transforms are chosen once (DUCC's cost model, as for gridding, the choice
// DUCC's SphereInterpol makes for both directions, sphere_interpol.h:425-426)
// and forced on every transform of either direction, so that the synthesis
// and its adjoint are adjoint to rounding.
static void forced(dnufft_opts &po, int nu2u, int ndim, const int64_t *shape, uint64_t npoints,
                   double eps, bool calc_f64) {
  int32_t kidx = -1;
  int64_t nover[3] = {1, 1, 1};
  check_nufft(dnufft_find_parameters(nu2u, ndim, shape, npoints, eps, calc_f64 ? 1 : 0, 1, &po,
                                     &kidx, nover),
              "synthesis_general (parameters)");
  po.force_kernel = kidx;
  for (int d = 0; d < 3; ++d) po.force_nover[d] = nover[d];
}

static Problem setup(size_t spin, int mode, size_t lmax, size_t nm, const int64_t *mstart,
                     int64_t lstride, const Arr &alm, const Arr &map, const Arr &loc,
                     double epsilon, const dnufft_sht_opts *o, bool adjoint) {
  DN_REQUIRE(o != nullptr, ST_BADARG, "null options");
  DN_REQUIRE(mode == DNUFFT_SHT_STANDARD || mode == DNUFFT_SHT_GRAD_ONLY ||
                 mode == DNUFFT_SHT_DERIV1,
             ST_BADARG, "unknown SHT mode");
  DN_REQUIRE(spin > 0 || mode == DNUFFT_SHT_STANDARD, ST_BADARG,
             "spin must be positive for grad-only SHTs");
  DN_REQUIRE(mode != DNUFFT_SHT_DERIV1 || spin == 1, ST_BADARG,
             "DERIV1 needs spin 1");
  DN_REQUIRE(spin <= lmax, ST_BADARG, "incorrect l_max: must be >= spin");
  DN_REQUIRE(spin <= 1024, ST_UNSUPPORTED, "spin above 1024");
  DN_REQUIRE(nm >= 1, ST_BADARG, "need at least m=0");
  DN_REQUIRE(nm <= lmax + 1, ST_BADARG, "mmax>lmax");
  DN_REQUIRE(lmax <= 65535, ST_UNSUPPORTED, "lmax above 65535");
  DN_REQUIRE(mstart != nullptr, ST_BADARG, "null mstart");
  DN_REQUIRE(std::isfinite(epsilon) && epsilon > 0, ST_BADARG, "epsilon must be positive");
  DN_REQUIRE(o->sigma_min > 1. && o->sigma_max >= o->sigma_min, ST_BADARG,
             "bad oversampling factor range");
  DN_REQUIRE(alm.dtype == DNUFFT_C64 || alm.dtype == DNUFFT_C128, ST_BADARG,
             "alm must be complex64 or complex128");
  const bool f64 = alm.dtype == DNUFFT_C128;
  DN_REQUIRE(map.dtype == (f64 ? DNUFFT_F64 : DNUFFT_F32), ST_BADARG,
             "map must be real with the precision of alm");
  DN_REQUIRE(loc.dtype == DNUFFT_F64, ST_BADARG, "loc must be float64");
  DN_REQUIRE(loc.shape[1] == 2, ST_BADARG, "last dimension of loc must have size 2");
  const int64_t nalm_c = (spin == 0 || mode != DNUFFT_SHT_STANDARD) ? 1 : 2;
  const int64_t nmaps = spin == 0 ? 1 : 2;
  DN_REQUIRE(alm.shape[0] == nalm_c, ST_BADARG, "number of components mismatch in alm");
  DN_REQUIRE(map.shape[0] == nmaps, ST_BADARG, "number of components mismatch in map");
  DN_REQUIRE(map.shape[1] == loc.shape[0], ST_BADARG, "map and loc disagree on the points");
  // DUCC's min_almdim (python/sht_pymod.cc:153-176)
  int64_t need = 0;
  for (size_t m = 0; m < nm; ++m) {
    const int64_t first = mstart[m] + int64_t(m) * lstride;
    const int64_t last = mstart[m] + int64_t(lmax) * lstride;
    DN_REQUIRE(first >= 0 && last >= 0, ST_BADARG, "impossible a_lm memory layout");
    need = std::max(need, std::max(first, last));
  }
  DN_REQUIRE(alm.shape[1] >= need + 1, ST_BADARG, "alm array too small for lmax / mstart");
  Problem P;
  P.lmax = int(lmax);
  P.mmax = int(nm) - 1;
  P.spin = int(spin);
  P.mode = mode;
  P.rows = spin == 0 ? P.mmax + 1 : 2 * P.mmax + 1;
  // rings: the power of two from 2 lmax + 2 (the DFT along the rings runs in
  // shared memory, up to FFT_MAX rings)
  P.nring = 2 * P.lmax + 2;
  P.log2n = 0;
  while ((1 << P.log2n) < P.nring) ++P.log2n;
  P.nring = 1 << P.log2n;
  DN_REQUIRE(P.nring <= FFT_MAX, ST_UNSUPPORTED,
             "lmax above 4095 is not supported by this build (the ring DFT runs in shared "
             "memory, up to 8192 rings)");
  P.npairs = (P.nring / 2) / 2 + 1;
  P.nk = 2 * P.lmax + 1;
  P.nblk = (P.npairs + THREADS * PAIRS - 1) / (THREADS * PAIRS);
  P.nblk_adj = (P.npairs + THREADS * PAIRS_ADJ - 1) / (THREADS * PAIRS_ADJ);
  P.nblk_spin = (P.nring / 2 + 1 + THREADS * RINGS - 1) / (THREADS * RINGS);
  P.npts = loc.shape[0];
  P.s = spin == 0 ? double(nm / 2) : 0.;
  P.f64 = f64;
  P.eps2 = epsilon;
  P.nalm_dense = 0;
  for (int m = 0; m <= P.mmax; ++m) P.nalm_dense += P.lmax + 1 - m;
  (void)adjoint;
  // parameters of the point transforms, chosen (and checked) before any launch
  dnufft_default_opts(&P.po2, 0);
  P.po2.nthreads = o->nthreads;
  P.po2.sigma_min = o->sigma_min;
  P.po2.sigma_max = o->sigma_max;
  const int64_t shape2[2] = {P.nk, P.rows};
  forced(P.po2, 1, 2, shape2, uint64_t(P.npts), P.eps2, P.f64);
  return P;
}

static void fft_smem_optin() {
  const int bytes = (FFT_MAX + FFT_MAX / 2) * int(sizeof(double2));
  DN_CUDA(cudaFuncSetAttribute(k_ring_fft<double2, float2, false>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  DN_CUDA(cudaFuncSetAttribute(k_ring_fft<double2, double2, false>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  DN_CUDA(cudaFuncSetAttribute(k_ring_fft<float2, double2, true>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  DN_CUDA(cudaFuncSetAttribute(k_ring_fft<double2, double2, true>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
}

static void make_tables(const Problem &P, const int64_t *mstart, cudaStream_t st, Tables &t) {
  const int nm = P.mmax + 1;
  std::vector<double> mant;
  std::vector<int> ex;
  mnorm_table(P.mmax, mant, ex);
  std::vector<int64_t> ms(mstart, mstart + nm), mofs(nm);
  int64_t idx = 0;
  for (int m = 0; m < nm; ++m) {
    mofs[m] = idx - m;   // dense index of (l, m) = mofs[m] + l
    idx += P.lmax + 1 - m;
  }
  fft_smem_optin();
  t.mstart = Buf(nm * sizeof(int64_t), st);
  t.mofs = Buf(nm * sizeof(int64_t), st);
  t.nmant = Buf(nm * sizeof(double), st);
  t.nexp = Buf(nm * sizeof(int), st);
  upload(t.mstart, ms.data(), nm * sizeof(int64_t), st);
  upload(t.mofs, mofs.data(), nm * sizeof(int64_t), st);
  upload(t.nmant, mant.data(), nm * sizeof(double), st);
  upload(t.nexp, ex.data(), nm * sizeof(int), st);
  // (copies from pageable host memory are staged before cudaMemcpyAsync
  // returns, so the vectors may end with this function)
}

static void report(const Problem &P, const char *what) {
  std::fprintf(stderr,
               "%s: lmax %d, mmax %d, spin %d, %lld points; %d rings, 2D modes %d x %d "
               "(epsilon %.3g)\n",
               what, P.lmax, P.mmax, P.spin, (long long)P.npts, P.nring, P.nk, P.rows, P.eps2);
}


// the DFT along the rings of `rows` transforms: V (rows, nring) FP64 -> c
// (nk, rows) in the data precision (forward), or h (nk, rows) in the data
// precision -> g (rows, nring) FP64 (inverse), one CTA per row
template <typename C>
static void rings_forward(const Problem &P, const Buf &V, Buf &cdat, cudaStream_t st) {
  const size_t smem = size_t(P.nring + P.nring / 2) * sizeof(double2);
  k_ring_fft<double2, C, false><<<P.rows, FFT_THREADS, smem, st>>>(
      ptr<double2>(V), ptr<C>(cdat), P.log2n, P.lmax, P.rows);
  DN_LAUNCHED();
}

template <typename C>
static void rings_inverse(const Problem &P, const Buf &hdat, Buf &gr, cudaStream_t st) {
  const size_t smem = size_t(P.nring + P.nring / 2) * sizeof(double2);
  k_ring_fft<C, double2, true><<<P.rows, FFT_THREADS, smem, st>>>(
      ptr<C>(hdat), ptr<double2>(gr), P.log2n, P.lmax, P.rows);
  DN_LAUNCHED();
}

// N_m of D_l0 per row (m = row - mmax), with its sign, and the powers of
// cos(theta/2), sin(theta/2): the single term of Wigner's sum at l0 =
// max(|m|, s); the binomial C(2 l0, l0 - s) accumulated over |m| in long
// double (its ratio between consecutive |m| is a product of four integers).
static std::vector<SpinStart> spin_starts(int mmax, int sp) {
  std::vector<SpinStart> res(2 * mmax + 1);
  const long double inv4pi = 1.0L / (4.0L * 3.141592653589793238462643383279502884L);
  std::vector<long double> bm(mmax + 1, 0.L);   // C(2 mu, mu - s) as mantissa * 2^be
  std::vector<long> be(mmax + 1, 0);
  long double b = 1.L;
  long e = 0;
  for (int mu = sp; mu <= mmax; ++mu) {
    if (mu > sp) {
      b *= (long double)(2 * mu) * (long double)(2 * mu - 1) /
           ((long double)(mu - sp) * (long double)(mu + sp));
      int t;
      b = frexpl(b, &t);
      e += t;
    }
    bm[mu] = b;
    be[mu] = e;
  }
  for (int row = 0; row <= 2 * mmax; ++row) {
    const int m = row - mmax, mu = m < 0 ? -m : m;
    SpinStart S;
    long double bin;
    long bexp;
    int sign = ((m + sp) & 1) ? -1 : 1;
    if (mu >= sp) {
      S.l0 = mu;
      bin = bm[mu];
      bexp = be[mu];
      if (m >= 0) {
        S.pc = mu - sp;
        S.ps = mu + sp;
      } else {
        S.pc = mu + sp;
        S.ps = mu - sp;
        if ((mu - sp) & 1) sign = -sign;
      }
    } else {
      S.l0 = sp;
      const int k = sp - m;   // C(2s, s - m), 1 <= k <= 2s - 1
      long double bb = 1.L;
      long ee = 0;
      for (int i = 1; i <= k; ++i) {
        bb *= (long double)(2 * sp - k + i) / (long double)i;
        int t;
        bb = frexpl(bb, &t);
        ee += t;
      }
      bin = bb;
      bexp = ee;
      S.pc = sp - m;
      S.ps = sp + m;
    }
    // N = sign sqrt((2 l0 + 1)/(4 pi) bin 2^bexp)
    int t;
    long double v = frexpl((long double)(2 * S.l0 + 1) * inv4pi * bin, &t);
    long ex = bexp + t;
    if (ex & 1) {
      v *= 2.L;
      ex -= 1;
    }
    S.mant = double(sign * sqrtl(v));
    S.ex = int(ex / 2);
    res[row] = S;
  }
  return res;
}

template <typename T, typename C>
static void synthesis_spin_t(const Problem &P, const Arr &alm, const int64_t *mstart,
                             int64_t lstride, const Arr &loc, const dnufft_sht_opts &o,
                             const Arr &map, cudaStream_t st) {
  if (o.verbosity) report(P, "synthesis_general");
  if (P.npts == 0) return;
  Tables tb;
  make_tables(P, mstart, st, tb);
  const std::vector<SpinStart> ss = spin_starts(P.mmax, P.spin);
  Buf dstarts(ss.size() * sizeof(SpinStart), st);
  upload(dstarts, ss.data(), ss.size() * sizeof(SpinStart), st);
  Buf V(size_t(P.rows) * P.nring * sizeof(double2), st);
  k_alm2leg_spin<C><<<dim3(P.mmax + 1, P.nblk_spin), THREADS, 0, st>>>(
      static_cast<const C *>(alm.p), alm.stride[0], alm.stride[1], ptr<int64_t>(tb.mstart),
      lstride, P.lmax, P.mmax, P.spin, P.mode, P.nring, ptr<SpinStart>(dstarts),
      ptr<double2>(V));
  DN_LAUNCHED();
  Buf cdat(size_t(P.rows) * P.nk * sizeof(C), st);
  rings_forward<C>(P, V, cdat, st);
  const int cdt = P.f64 ? DNUFFT_C128 : DNUFFT_C64;
  Buf z(size_t(P.npts) * sizeof(C), st);
  {
    dnufft_array a_u = dev_array(cdat.p, cdt, P.nk, P.rows, P.rows, 1);
    dnufft_array a_l = dev_array(loc.p, DNUFFT_F64, P.npts, 2, loc.stride[0], loc.stride[1]);
    dnufft_array a_z = dev_array(z.p, cdt, P.npts, 1, 1, 1);
    a_z.ndim = 1;
    check_nufft(dnufft_u2nu(&a_u, &a_l, 0, P.eps2, &a_z, &P.po2, st),
                "synthesis_general (points)");
  }
  k_points_out_spin<C, T><<<grid_for(P.npts), 256, 0, st>>>(
      ptr<C>(z), P.npts, static_cast<T *>(map.p), map.stride[0], map.stride[1]);
  DN_LAUNCHED();
}

template <typename T, typename C>
static void adjoint_spin_t(const Problem &P, const Arr &map, const int64_t *mstart,
                           int64_t lstride, const Arr &loc, const dnufft_sht_opts &o,
                           const Arr &alm, cudaStream_t st) {
  if (o.verbosity) report(P, "adjoint_synthesis_general");
  Tables tb;
  make_tables(P, mstart, st, tb);
  const std::vector<SpinStart> ss = spin_starts(P.mmax, P.spin);
  Buf dstarts(ss.size() * sizeof(SpinStart), st);
  upload(dstarts, ss.data(), ss.size() * sizeof(SpinStart), st);
  const int cdt = P.f64 ? DNUFFT_C128 : DNUFFT_C64;
  Buf hdat(size_t(P.rows) * P.nk * sizeof(C), st);
  {
    Buf z(size_t(std::max<int64_t>(P.npts, 1)) * sizeof(C), st);
    if (P.npts > 0) {
      k_points_in_spin<C, T><<<grid_for(P.npts), 256, 0, st>>>(
          static_cast<const T *>(map.p), map.stride[0], map.stride[1], P.npts, ptr<C>(z));
      DN_LAUNCHED();
    }
    dnufft_array a_z = dev_array(z.p, cdt, P.npts, 1, 1, 1);
    a_z.ndim = 1;
    dnufft_array a_l = dev_array(loc.p, DNUFFT_F64, P.npts, 2, loc.stride[0], loc.stride[1]);
    dnufft_array a_h = dev_array(hdat.p, cdt, P.nk, P.rows, P.rows, 1);
    check_nufft(dnufft_nu2u(&a_z, &a_l, 1, P.eps2, &a_h, &P.po2, st),
                "adjoint_synthesis_general (points)");
  }
  Buf gr(size_t(P.rows) * P.nring * sizeof(double2), st);
  rings_inverse<C>(P, hdat, gr, st);
  Buf part(size_t(P.nblk_spin) * P.rows * (P.lmax + 1) * sizeof(double2), st);
  k_leg2alm_spin<<<dim3(P.mmax + 1, P.nblk_spin), THREADS, 0, st>>>(
      ptr<double2>(gr), P.lmax, P.mmax, P.spin, P.nring, ptr<SpinStart>(dstarts),
      ptr<double2>(part));
  DN_LAUNCHED();
  k_alm_out_spin<C><<<grid_for(P.nalm_dense), 256, 0, st>>>(
      ptr<double2>(part), P.nblk_spin, P.nalm_dense, ptr<int64_t>(tb.mofs),
      ptr<int64_t>(tb.mstart), lstride, alm.stride[0], alm.stride[1], P.lmax, P.mmax, P.spin,
      P.mode, 1. / double(P.nring), static_cast<C *>(alm.p));
  DN_LAUNCHED();
}

template <typename T, typename C>
static void synthesis_t(const Problem &P, const Arr &alm, const int64_t *mstart, int64_t lstride,
                        const Arr &loc, const dnufft_sht_opts &o, const Arr &map,
                        cudaStream_t st) {
  const int nm = P.mmax + 1;
  if (o.verbosity) report(P, "synthesis_general");
  if (P.npts == 0) return;
  Tables tb;
  make_tables(P, mstart, st, tb);
  // 1. F_m on the rings (FP64)
  Buf V(size_t(nm) * P.nring * sizeof(double2), st);
  k_alm2leg<C><<<dim3(nm, P.nblk), THREADS, 0, st>>>(
      static_cast<const C *>(alm.p), alm.stride[1], ptr<int64_t>(tb.mstart), lstride, P.lmax,
      P.nring, P.npairs, ptr<double>(tb.nmant), ptr<int>(tb.nexp), ptr<double2>(V));
  DN_LAUNCHED();
  // 2. c_km, written [k][m] (row-major (nk, nm)) in the data precision
  Buf cdat(size_t(nm) * P.nk * sizeof(C), st);
  rings_forward<C>(P, V, cdat, st);
  // 3. the 2D type 2 at the points, in the data precision
  const void *uni = cdat.p;
  const int cdt = P.f64 ? DNUFFT_C128 : DNUFFT_C64;
  Buf z(size_t(P.npts) * sizeof(C), st);
  {
    const dnufft_opts &po = P.po2;
    dnufft_array a_u = dev_array(const_cast<void *>(uni), cdt, P.nk, nm, nm, 1);
    dnufft_array a_l = dev_array(loc.p, DNUFFT_F64, P.npts, 2, loc.stride[0], loc.stride[1]);
    dnufft_array a_z = dev_array(z.p, cdt, P.npts, 1, 1, 1);
    a_z.ndim = 1;
    check_nufft(dnufft_u2nu(&a_u, &a_l, 0, P.eps2, &a_z, &po, st), "synthesis_general (points)");
  }
  k_points_out<C, T><<<grid_for(P.npts), 256, 0, st>>>(
      ptr<C>(z), static_cast<const double *>(loc.p), loc.stride[0], loc.stride[1], P.npts, P.s,
      static_cast<T *>(map.p), map.stride[1]);
  DN_LAUNCHED();
}

template <typename T, typename C>
static void adjoint_t(const Problem &P, const Arr &map, const int64_t *mstart, int64_t lstride,
                      const Arr &loc, const dnufft_sht_opts &o, const Arr &alm, cudaStream_t st) {
  const int nm = P.mmax + 1;
  if (o.verbosity) report(P, "adjoint_synthesis_general");
  Tables tb;
  make_tables(P, mstart, st, tb);
  const int cdt = P.f64 ? DNUFFT_C128 : DNUFFT_C64;
  // 1. values map_i e^{-i s phi_i} -> 2D type 1, modes [k][m - s] (row-major (nk, nm))
  Buf hdat(size_t(nm) * P.nk * sizeof(C), st);
  {
    Buf z(size_t(std::max<int64_t>(P.npts, 1)) * sizeof(C), st);
    if (P.npts > 0) {
      k_points_in<C, T><<<grid_for(P.npts), 256, 0, st>>>(
          static_cast<const T *>(map.p), map.stride[1], static_cast<const double *>(loc.p),
          loc.stride[0], loc.stride[1], P.npts, P.s, ptr<C>(z));
      DN_LAUNCHED();
    }
    const dnufft_opts &po = P.po2;
    dnufft_array a_z = dev_array(z.p, cdt, P.npts, 1, 1, 1);
    a_z.ndim = 1;
    dnufft_array a_l = dev_array(loc.p, DNUFFT_F64, P.npts, 2, loc.stride[0], loc.stride[1]);
    dnufft_array a_h = dev_array(hdat.p, cdt, P.nk, nm, nm, 1);
    check_nufft(dnufft_nu2u(&a_z, &a_l, 1, P.eps2, &a_h, &po, st), "adjoint_synthesis_general (points)");
  }
  // 2. back to the rings (FP64)
  Buf gr(size_t(nm) * P.nring * sizeof(double2), st);
  rings_inverse<C>(P, hdat, gr, st);
  // 3. the transposed recurrence, per-block partial sums, summed in block order
  Buf part(size_t(P.nblk_adj) * P.nalm_dense * sizeof(double2), st);
  k_leg2alm<<<dim3(nm, P.nblk_adj), THREADS, 0, st>>>(
      ptr<double2>(gr), P.lmax, P.nring, P.npairs, ptr<double>(tb.nmant), ptr<int>(tb.nexp),
      ptr<int64_t>(tb.mofs), P.nalm_dense, ptr<double2>(part));
  DN_LAUNCHED();
  k_alm_out<C><<<grid_for(P.nalm_dense), 256, 0, st>>>(
      ptr<double2>(part), P.npairs, P.nalm_dense, ptr<int64_t>(tb.mofs), ptr<int64_t>(tb.mstart),
      lstride, alm.stride[1], P.lmax, nm, 1. / double(P.nring), static_cast<C *>(alm.p));
  DN_LAUNCHED();
}

static void synthesis_impl(const dnufft_array *alm_, size_t spin, int mode, size_t lmax,
                           const int64_t *mstart, size_t nm, int64_t lstride,
                           const dnufft_array *loc_, double epsilon, const dnufft_sht_opts *o,
                           dnufft_array *map_, cudaStream_t st) {
  const Arr alm = arr_of(alm_, "alm"), map = arr_of(map_, "map"), loc = arr_of(loc_, "loc");
  const Problem P =
      setup(spin, mode, lmax, nm, mstart, lstride, alm, map, loc, epsilon, o, false);
  if (P.spin > 0) {
    if (P.f64)
      synthesis_spin_t<double, double2>(P, alm, mstart, lstride, loc, *o, map, st);
    else
      synthesis_spin_t<float, float2>(P, alm, mstart, lstride, loc, *o, map, st);
    return;
  }
  if (P.f64)
    synthesis_t<double, double2>(P, alm, mstart, lstride, loc, *o, map, st);
  else
    synthesis_t<float, float2>(P, alm, mstart, lstride, loc, *o, map, st);
}

static void adjoint_impl(const dnufft_array *map_, size_t spin, int mode, size_t lmax,
                         const int64_t *mstart, size_t nm, int64_t lstride,
                         const dnufft_array *loc_, double epsilon, const dnufft_sht_opts *o,
                         dnufft_array *alm_, cudaStream_t st) {
  const Arr alm = arr_of(alm_, "alm"), map = arr_of(map_, "map"), loc = arr_of(loc_, "loc");
  const Problem P =
      setup(spin, mode, lmax, nm, mstart, lstride, alm, map, loc, epsilon, o, true);
  if (P.spin > 0) {
    if (P.f64)
      adjoint_spin_t<double, double2>(P, map, mstart, lstride, loc, *o, alm, st);
    else
      adjoint_spin_t<float, float2>(P, map, mstart, lstride, loc, *o, alm, st);
    return;
  }
  if (P.f64)
    adjoint_t<double, double2>(P, map, mstart, lstride, loc, *o, alm, st);
  else
    adjoint_t<float, float2>(P, map, mstart, lstride, loc, *o, alm, st);
}

#define DN_SHT_GUARD(body)                                       \
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

void dnufft_sht_default_opts(dnufft_sht_opts *o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->nthreads = 1;
  o->sigma_min = 1.1;
  o->sigma_max = 2.6;
}

int dnufft_synthesis_general(const dnufft_array *alm, size_t spin, int mode, size_t lmax,
                             const int64_t *mstart, size_t nm, int64_t lstride,
                             const dnufft_array *loc, double epsilon, const dnufft_sht_opts *opts,
                             dnufft_array *map, void *stream) {
  DN_SHT_GUARD(dnufft::sht::synthesis_impl(alm, spin, mode, lmax, mstart, nm, lstride, loc,
                                           epsilon, opts, map,
                                           static_cast<cudaStream_t>(stream)))
}

int dnufft_adjoint_synthesis_general(const dnufft_array *map, size_t spin, int mode,
                                     size_t lmax, const int64_t *mstart, size_t nm,
                                     int64_t lstride, const dnufft_array *loc, double epsilon,
                                     const dnufft_sht_opts *opts, dnufft_array *alm,
                                     void *stream) {
  DN_SHT_GUARD(dnufft::sht::adjoint_impl(map, spin, mode, lmax, mstart, nm, lstride, loc,
                                         epsilon, opts, alm, static_cast<cudaStream_t>(stream)))
}

}  // extern "C"

}  // namespace sht
}  // namespace dnufft
