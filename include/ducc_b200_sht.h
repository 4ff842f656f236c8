/*
 * ducc_b200_sht.h - C-ABI of the spherical-harmonic consumers of the B200
 * NUFFT library: synthesis of a spherical-harmonic expansion at arbitrary
 * points on the sphere and its adjoint, the counterparts of
 * ducc0.sht.synthesis_general / adjoint_synthesis_general (the third of
 * DUCC's functions, pseudo_analysis_general, is the least-squares solver
 * over these two in ducc_b200/sht.py).
 *
 * Conventions (DUCC's, src/ducc0/sht/sht.cc:60-171): a_lm for 0 <= m <= mmax,
 * m <= l <= lmax, at element mstart[m] + l * lstride of each a_lm row (DUCC's
 * layout; mstart is a host array of mmax + 1 entries).
 * Spin 0: orthonormal Y_lm with the Condon-Shortley phase, one real map
 *   map(theta, phi) = sum_l a_l0 Y_l0 + 2 Re sum_{m>0} sum_l a_lm Y_lm(theta, phi)
 * and the adjoint a_lm = sum_i map_i conj(Y_lm(theta_i, phi_i)) for every m.
 * Spin s > 0: two a_lm rows (E, B; one row, E, with GRAD_ONLY and DERIV1)
 * and two maps (Q, U) with
 *   Q + i U = (-1)^(s+1) sum_{l, |m| <= mmax} (E_lm + i B_lm) D_lm(theta) e^{i m phi},
 *   D_lm = sqrt((2l+1)/(4 pi)) d^l_{m,-s}(theta) (Wigner d), l >= max(|m|, s),
 *   E_{l,-m} = (-1)^m conj(E_lm) (the same for B);
 * DERIV1 (spin 1) is GRAD_ONLY with E_lm * sqrt(l (l+1)); the adjoints are the
 * transposes for DUCC's inner product (m > 0 counted twice), a_lm with l < s
 * written as zero.
 *
 * Arrays are dnufft_array descriptors (include/ducc_b200.h) of DEVICE memory:
 *   alm (ncomp, nalm) C64 | C128, map (nmaps, npoints) F32 | F64 of the same
 *   precision, loc (npoints, 2) F64 holding (theta, phi) per point.
 * Points outside [0, pi] x [0, 2 pi] are evaluated on the periodic
 * continuation of the expansion (DUCC rejects them).
 * Every function returns 0 on success and a DNUFFT_ERR_* code otherwise
 * (message: dnufft_last_error()); argument errors are detected before any
 * kernel is launched.  DERIV1 needs spin 1 (DUCC accepts other spins there
 * and computes the spin-1 recurrence with that spin's pole parity).  Limits
 * of this build: lmax <= 4095 (the DFT along the rings runs in shared memory,
 * up to 8192 rings) and the 2D transform's row limits (in double precision
 * mmax up to about 4095 for spin 0, 2047 for spin > 0); beyond them
 * DNUFFT_ERR_UNSUPPORTED.
 */
#ifndef DUCC_B200_SHT_H
#define DUCC_B200_SHT_H

#include "ducc_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* mode (DUCC's SHT_mode) */
#define DNUFFT_SHT_STANDARD 0   /* spin 0: one row; spin > 0: E and B      */
#define DNUFFT_SHT_GRAD_ONLY 1  /* spin > 0, E only (B = 0)                */
#define DNUFFT_SHT_DERIV1 2     /* spin 1, first derivatives of a spin-0 a_lm */

typedef struct dnufft_sht_opts {
  size_t nthreads;     /* as in DUCC; only feeds the NUFFT's parameter cost model */
  double sigma_min;    /* oversampling factor range of the 2D transform           */
  double sigma_max;    /* (DUCC: 1.1 .. 2.6)                                      */
  int32_t verbosity;   /* 1: print the sizes chosen                                */
} dnufft_sht_opts;

/* DUCC's keyword defaults of synthesis_general (python/sht_pymod.cc:2299). */
void dnufft_sht_default_opts(dnufft_sht_opts *opts);

/* map = synthesis of alm at the points loc, to the requested epsilon.
 * Replaces ducc0.sht.synthesis_general (python/sht_pymod.cc:805-845 ->
 * src/ducc0/sht/sht.cc:2926-2961). */
int dnufft_synthesis_general(const dnufft_array *alm, size_t spin, int mode, size_t lmax,
                             const int64_t *mstart, size_t nm, int64_t lstride,
                             const dnufft_array *loc, double epsilon,
                             const dnufft_sht_opts *opts, dnufft_array *map, void *stream);

/* alm = adjoint synthesis of map at the points loc (every a_lm with
 * m <= l <= lmax is written).  Replaces ducc0.sht.adjoint_synthesis_general
 * (python/sht_pymod.cc:847-885 -> src/ducc0/sht/sht.cc:2965-2994). */
int dnufft_adjoint_synthesis_general(const dnufft_array *map, size_t spin, int mode, size_t lmax,
                                     const int64_t *mstart, size_t nm, int64_t lstride,
                                     const dnufft_array *loc, double epsilon,
                                     const dnufft_sht_opts *opts, dnufft_array *alm,
                                     void *stream);

#ifdef __cplusplus
}
#endif

#endif /* DUCC_B200_SHT_H */
