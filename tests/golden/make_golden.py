"""Generate the golden fixtures in this directory from DUCC itself.

Runs DUCC's own NUFFT (compiled from the reference sources by oracle/Makefile
into oracle/_ref) on small seeded problems and stores inputs, outputs and DUCC's
internal index data (getpix start indices, tile permutation, chosen kernel and
oversampled sizes).  The fixtures let the oracle and the CUDA path be checked
against DUCC on machines where the reference is not available.

Usage:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))
from oracle import ref  # noqa: E402

CASES = [
    # name, shape, M, coord dtype, singleprec, eps, forward, periodicity, fft_order, spread
    ("g1d_f32", (100,), 300, np.float32, True, 1e-4, True, 2 * np.pi, False, 1.0),
    ("g1d_f64", (101,), 300, np.float64, False, 1e-9, False, 1.0, True, 3.0),
    ("g2d_f32", (64, 48), 600, np.float32, True, 1e-5, True, 2 * np.pi, False, 1.0),
    ("g2d_f32_eps6", (96, 80), 800, np.float32, True, 1e-6, False, 2 * np.pi, True, 2.0),
    ("g2d_f64", (33, 40), 500, np.float64, False, 1e-10, False, [1.0, 3.0], True, 5.0),
    ("g2d_mixed", (40, 41), 300, np.float64, True, 1e-5, True, 2 * np.pi, False, 1.0),
    ("g2d_cfg1_small", (256, 256), 2000, np.float64, False, 1e-6, True, 2 * np.pi, False, 1.0),
    ("g3d_f32", (12, 14, 16), 300, np.float32, True, 1e-5, True, 2 * np.pi, False, 1.0),
    ("g3d_f64", (10, 12, 9), 200, np.float64, False, 1e-11, False, [1.0, np.pi, 7.0], True, 2.0),
]


def make(R, case, rng):
    name, shape, M, cdt, sp, eps, fwd, per, fftord, spread = case
    ndim = len(shape)
    pers = [per] * ndim if np.ndim(per) == 0 else list(per)
    coord = ((rng.random((M, ndim)) - 0.5) * np.array(pers) * spread).astype(cdt)
    vdt = np.complex64 if sp else np.complex128
    values = (rng.standard_normal(M) + 1j * rng.standard_normal(M)).astype(vdt)
    grid_in = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(vdt)
    out1 = np.zeros(shape, dtype=vdt)
    R.nufft.nu2u(points=values, coord=coord, forward=fwd, epsilon=eps, nthreads=1,
                 out=out1, periodicity=per, fft_order=fftord)
    out2 = R.nufft.u2nu(grid=grid_in, coord=coord, forward=fwd, epsilon=eps, nthreads=1,
                        periodicity=per, fft_order=fftord)
    pr1 = R.index_probe(coord=coord, shape=list(shape), epsilon=eps, singleprec=sp,
                        gridding=True, nthreads=1, sigma_min=1.2, sigma_max=2.51,
                        periodicity=[float(p) for p in pers], fft_order=fftord)
    pr2 = R.index_probe(coord=coord, shape=list(shape), epsilon=eps, singleprec=sp,
                        gridding=False, nthreads=1, sigma_min=1.2, sigma_max=2.51,
                        periodicity=[float(p) for p in pers], fft_order=fftord)
    np.savez_compressed(
        os.path.join(HERE, name + ".npz"),
        shape=np.array(shape), coord=coord, values=values, grid_in=grid_in,
        nu2u=out1, u2nu=out2, eps=eps, forward=fwd, periodicity=np.array(pers),
        fft_order=fftord, singleprec=sp,
        W1=pr1["W"], nover1=np.array(pr1["nover"]), kidx1=pr1["kernel_index"],
        i0_1=pr1["i0"], perm1=pr1["coord_idx"],
        W2=pr2["W"], nover2=np.array(pr2["nover"]), kidx2=pr2["kernel_index"],
        perm2=pr2["coord_idx"])
    print("wrote", name)


def main():
    R = ref.load()
    if R is None:
        raise SystemExit("reference module not built: run make -C oracle")
    rng = np.random.default_rng(20241203)
    for case in CASES:
        make(R, case, rng)
    db = np.array([tuple(r)[:6] + (float(r[6]),) for r in R.kernel_db()], dtype=np.float64)
    np.savez_compressed(os.path.join(HERE, "kernel_db.npz"), rows=db)
    print("wrote kernel_db")


if __name__ == "__main__":
    main()
