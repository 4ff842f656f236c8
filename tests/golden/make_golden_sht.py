"""Generate the spherical-harmonic golden fixtures in this directory from DUCC.

Runs DUCC's own ``synthesis_general`` / ``adjoint_synthesis_general`` (its sht
module, compiled from the reference sources by oracle/Makefile into
oracle/_ref) on small seeded problems at a tight epsilon and stores
inputs and outputs (spin 0, and spin 1-3 in the modes STANDARD, GRAD_ONLY and
DERIV1), so that the direct-sum oracle (oracle/sht_oracle.py) and
the CUDA path can be checked against DUCC where the reference is not
available.

Usage:  python tests/golden/make_golden_sht.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))
from oracle import ref  # noqa: E402
from oracle import sht_oracle as O  # noqa: E402

# name, lmax, mmax, npoints, precision, epsilon, spin, mode
CASES = [
    ("sht_l10_m8_f64", 10, 8, 200, np.complex128, 1e-13, 0, "STANDARD"),
    ("sht_l40_m40_f64", 40, 40, 500, np.complex128, 1e-13, 0, "STANDARD"),
    ("sht_l100_m70_f64", 100, 70, 300, np.complex128, 1e-12, 0, "STANDARD"),
    ("sht_l32_m32_f32", 32, 32, 400, np.complex64, 1e-6, 0, "STANDARD"),
    ("sht_s1_l20_m17_f64", 20, 17, 300, np.complex128, 1e-13, 1, "STANDARD"),
    ("sht_s2_l30_m30_f64", 30, 30, 300, np.complex128, 1e-13, 2, "STANDARD"),
    ("sht_s3_l25_m12_f64_grad", 25, 12, 200, np.complex128, 1e-13, 3, "GRAD_ONLY"),
    ("sht_s1_l24_m24_f64_deriv1", 24, 24, 200, np.complex128, 1e-13, 1, "DERIV1"),
    ("sht_s2_l30_m20_f32", 30, 20, 300, np.complex64, 1e-6, 2, "STANDARD"),
]


def main():
    R = ref.load()
    rng = np.random.default_rng(20261204)
    for name, lmax, mmax, npts, cdt, eps, spin, mode in CASES:
        ncomp = 1 if (spin == 0 or mode != "STANDARD") else 2
        alm = O.random_alm_spin(lmax, mmax, spin, ncomp, rng).astype(cdt)
        loc = np.stack([rng.uniform(0., np.pi, npts), rng.uniform(0., 2 * np.pi, npts)], 1)
        rdt = np.float64 if cdt == np.complex128 else np.float32
        mp = rng.uniform(-0.5, 0.5, (1 if spin == 0 else 2, npts)).astype(rdt)
        synth = R.sht.synthesis_general(alm=alm, spin=spin, lmax=lmax, mmax=mmax, loc=loc,
                                        epsilon=eps, nthreads=1, mode=mode)
        adj = R.sht.adjoint_synthesis_general(map=mp, spin=spin, lmax=lmax, mmax=mmax, loc=loc,
                                              epsilon=eps, nthreads=1, mode=mode)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), lmax=lmax, mmax=mmax, eps=eps,
                            spin=spin, mode=mode, alm=alm, loc=loc, map_in=mp, synthesis=synth,
                            adjoint=adj)
        print(name, synth.shape, adj.shape)


if __name__ == "__main__":
    main()
