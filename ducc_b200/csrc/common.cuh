// Device helpers shared by the NUFFT kernels: complex types, the coordinate
// fold (DUCC's getpix, bit-exact), tile keys and the ES-kernel polynomial
// evaluation.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "dnufft_internal.h"

namespace dnufft {

template <typename T> struct CplxOf;
template <> struct CplxOf<float> { using type = float2; };
template <> struct CplxOf<double> { using type = double2; };
template <typename T> using cplx = typename CplxOf<T>::type;

template <typename T> __host__ __device__ __forceinline__ cplx<T> mkc(T r, T i) {
  cplx<T> c;
  c.x = r;
  c.y = i;
  return c;
}
template <typename T>
__device__ __forceinline__ cplx<T> cmul(cplx<T> a, cplx<T> b) {
  return mkc<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename T>
__device__ __forceinline__ cplx<T> cadd(cplx<T> a, cplx<T> b) {
  return mkc<T>(a.x + b.x, a.y + b.y);
}
template <typename T>
__device__ __forceinline__ cplx<T> csub(cplx<T> a, cplx<T> b) {
  return mkc<T>(a.x - b.x, a.y - b.y);
}

// ---------------------------------------------------------------------------
// Coordinate fold: DUCC's Nufft_ancestor::getpix (src/ducc0/nufft/nufft.h:285-298)
//   tmp  = x * (1/period);  f = tmp - floor(tmp)
//   tmp2 = f * n            (long double for float64 coords, double otherwise)
//   i0   = min(int(tmp2 + shift) - n, maxi0)
//   frac = tmp2 - i0
// For float32 coordinates DUCC's optimised build evaluates frac as one fused
// multiply-add, fma(f, n, -i0); that is reproduced here.  For float64
// coordinates the x87 80-bit arithmetic (64-bit significand, round to nearest
// even) is emulated exactly with 128-bit integers.
// ---------------------------------------------------------------------------

__device__ __forceinline__ void fold_f32(double x, double coordfct, int n, double shift,
                                         int maxi0, int &i0, double &frac) {
  double tmp = __dmul_rn(x, coordfct);
  double f = tmp - floor(tmp);
  double tmp2 = __dmul_rn(f, double(n));
  int s = int(__dadd_rn(tmp2, shift));
  i0 = min(s - n, maxi0);
  frac = __fma_rn(f, double(n), -double(i0));
}

typedef unsigned __int128 u128;

__device__ __forceinline__ int bitlen128(u128 v) {
  uint64_t hi = uint64_t(v >> 64), lo = uint64_t(v);
  if (hi) return 128 - __clzll((long long)hi);
  if (lo) return 64 - __clzll((long long)lo);
  return 0;
}

// Round v (whose true value may exceed v by less than one unit in the last
// place when 'sticky' is set) to 'keep' significant bits, round-to-nearest-even.
// Returns the rounded integer and the number of dropped bits in *drop.
__device__ __forceinline__ u128 round_sig(u128 v, bool sticky, int keep, int *drop) {
  int bl = bitlen128(v);
  if (bl <= keep) {
    *drop = 0;
    return v;   // exact (sticky bits below would not change a RNE result here)
  }
  int d = bl - keep;
  u128 rem = v & ((u128(1) << d) - 1);
  u128 half = u128(1) << (d - 1);
  u128 r = v >> d;
  bool up = (rem > half) || (rem == half && (sticky || (r & 1)));
  r += up ? 1 : 0;
  if (bitlen128(r) > keep) {   // carry into a new bit
    r >>= 1;
    d += 1;
  }
  *drop = d;
  return r;
}

__device__ __forceinline__ void fold_f64(double x, double coordfct, int n, double shift,
                                         int maxi0, int &i0, double &frac) {
  double tmp = __dmul_rn(x, coordfct);
  double f = tmp - floor(tmp);
  // exact f = mant * 2^e
  uint64_t bits = uint64_t(__double_as_longlong(f));
  int ex = int((bits >> 52) & 0x7ff);
  uint64_t mant = bits & ((uint64_t(1) << 52) - 1);
  int e;
  if (ex == 0) {
    e = -1074;
  } else {
    mant |= uint64_t(1) << 52;
    e = ex - 1075;
  }
  // tmp2 = RN64(mant * n * 2^e) = P * 2^e2
  int drop;
  u128 P = round_sig(u128(mant) * u128(uint32_t(n)), false, 64, &drop);
  int e2 = e + drop;
  // fixed point Q = tmp2 * 2^64 (plus sticky for bits below 2^-64)
  int sh = e2 + 64;
  u128 Q;
  bool sticky = false;
  if (P == 0) {
    Q = 0;
  } else if (sh >= 0) {
    Q = P << sh;   // tmp2 < 2^31, so Q < 2^95
  } else if (sh > -128) {
    sticky = (P & ((u128(1) << (-sh)) - 1)) != 0;
    Q = P >> (-sh);
  } else {
    sticky = true;
    Q = 0;
  }
  // tmp2 + shift, shift a multiple of 1/2, rounded to 64 significant bits
  uint64_t twoshift = uint64_t(shift * 2.0);
  u128 S = Q + (u128(twoshift) << 63);
  u128 Sr = round_sig(S, sticky, 64, &drop);
  int s = int((Sr << drop) >> 64);
  i0 = min(s - n, maxi0);
  // frac = RN53(RN64(tmp2 - i0)); tmp2 - i0 > 0 always
  u128 I = u128(uint64_t(int64_t(i0) < 0 ? -int64_t(i0) : int64_t(i0))) << 64;
  u128 Dv = (i0 < 0) ? Q + I : Q - I;
  u128 D64 = round_sig(Dv, sticky, 64, &drop);
  int drop2;
  u128 D53 = round_sig(D64, false, 53, &drop2);
  frac = ldexp(double(uint64_t(D53)), drop + drop2 - 64);
}

template <typename Tc>
__device__ __forceinline__ void fold(Tc x, double coordfct, int n, double shift, int maxi0,
                                     int &i0, double &frac) {
  if constexpr (sizeof(Tc) == 4)
    fold_f32(double(x), coordfct, n, shift, maxi0, i0, frac);
  else
    fold_f64(double(x), coordfct, n, shift, maxi0, i0, frac);
}

// ---------------------------------------------------------------------------
// ES kernel weights for one axis: W piecewise polynomials of degree D'=W+3+(W&1)
// evaluated at x = W-1-2*frac, using the mirror symmetry poly_{W-1-k}(x) =
// poly_k(-x) and an even/odd split in x^2 (the evaluation scheme of DUCC's
// TemplateKernel, src/ducc0/math/gridding_kernel.h:178-382).
// ---------------------------------------------------------------------------
template <typename T, int W>
__device__ __forceinline__ void kernel_weights(const KernelPoly<T> &kp, T x, T (&w)[W]) {
  constexpr int D = W + 3 + (W & 1);
  constexpr int H = (W + 1) / 2;
  T x2 = x * x;
#pragma unroll
  for (int k = 0; k < H; ++k) {
    T e = kp.c[0][k], o = kp.c[1][k];
#pragma unroll
    for (int j = 2; j < D; j += 2) {
      e = e * x2 + kp.c[j][k];
      o = o * x2 + kp.c[j + 1][k];
    }
    w[k] = e * x + o;
    if (W - 1 - k != k) w[W - 1 - k] = o - e * x;
  }
}

// Derivative d/dx of the weights above (for coordinate gradients).
template <typename T, int W>
__device__ __forceinline__ void kernel_weights_deriv(const KernelPoly<T> &kp, T x,
                                                     T (&w)[W], T (&dw)[W]) {
  constexpr int D = W + 3 + (W & 1);
  constexpr int H = (W + 1) / 2;
  T x2 = x * x;
#pragma unroll
  for (int k = 0; k < H; ++k) {
    // p(x) = sum_j c[j] x^(D-j)
    T p = kp.c[0][k], dp = T(0);
#pragma unroll
    for (int j = 1; j <= D; ++j) {
      dp = dp * x + p;
      p = p * x + kp.c[j][k];
    }
    // mirror: q(x) = p(-x), q'(x) = -p'(-x)
    T pm = kp.c[0][k], dpm = T(0), xm = -x;
#pragma unroll
    for (int j = 1; j <= D; ++j) {
      dpm = dpm * xm + pm;
      pm = pm * xm + kp.c[j][k];
    }
    w[k] = p;
    dw[k] = dp;
    if (W - 1 - k != k) {
      w[W - 1 - k] = pm;
      dw[W - 1 - k] = -dpm;
    }
  }
  (void)x2;
}

// positive modulo for wrap-around indexing
__device__ __forceinline__ int wrapi(int i, int n) {
  i %= n;
  return i < 0 ? i + n : i;
}

// periodic wrap of i in [-n, 2n) without a division
__device__ __forceinline__ int wrap1(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// floor(x / d) for d >= 2 and x * d < 2^32 by a multiply-high with m = ceil(2^32 / d)
__host__ __device__ __forceinline__ uint32_t fastdiv_magic(uint32_t d) {
  return uint32_t(((uint64_t(1) << 32) + d - 1) / d);
}
__device__ __forceinline__ uint32_t fastdiv(uint32_t x, uint32_t m) { return __umulhi(x, m); }

}  // namespace dnufft
