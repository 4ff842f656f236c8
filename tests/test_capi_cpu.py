"""C-ABI surface and host logic, no GPU: the library loads, exports every
symbol declared in include/ducc_b200.h, and host-side argument checks fail
before any kernel launch."""
import os
import re

import numpy as np
import pytest

from ducc_b200 import _capi as C
from ducc_b200 import nufft

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            names += re.findall(r"^(?:int|void|uint64_t|size_t|const char \*)\s*(dnufft_\w+)\s*\(", src, re.M)
    return names


def test_library_exports_every_declared_symbol():
    L = C.lib()
    decl = declared_functions()
    assert len(decl) >= 11
    for name in decl:
        assert hasattr(L, name), name


def test_best_epsilon_matches_ducc_values():
    assert abs(nufft.bestEpsilon(ndim=2, singleprec=True) - 4.4514883e-07) < 1e-13
    assert abs(nufft.bestEpsilon(ndim=2, singleprec=False) - 7.1866641e-15) < 1e-21
    with pytest.raises(RuntimeError):
        nufft.bestEpsilon(ndim=4, singleprec=True)


def test_default_opts():
    o = C.make_opts(False)
    assert o.nthreads == 1 and o.sigma_min == 1.2 and o.sigma_max == 2.51
    p = C.make_opts(True)
    assert p.nthreads == 0 and p.sigma_min == 1.1 and p.sigma_max == 2.6
    assert abs(o.periodicity[0] - 2 * np.pi) < 1e-15


def test_argument_errors_raise_before_launch():
    coord = np.zeros((10, 2), np.float64)
    pts = np.zeros(10, np.complex128)
    with pytest.raises(TypeError):
        nufft.nu2u(points=pts, coord=coord, forward=True, epsilon=1e-5)
    out = np.zeros((8, 8), np.complex128)
    with pytest.raises(RuntimeError, match="number of points"):
        nufft.nu2u(points=pts[:5], coord=coord, forward=True, epsilon=1e-5, out=out)
    with pytest.raises(RuntimeError, match="dtype"):
        nufft.nu2u(points=pts, coord=coord, forward=True, epsilon=1e-5,
                   out=np.zeros((8, 8), np.complex64))
    with pytest.raises(RuntimeError, match="no appropriate kernel"):
        nufft.nu2u(points=pts.astype(np.complex64), coord=coord, forward=True, epsilon=1e-8,
                   out=np.zeros((8, 8), np.complex64))
    with pytest.raises(RuntimeError, match="not yet supported"):
        nufft.nu2u(points=pts.real.copy(), coord=coord, forward=True, epsilon=1e-5, out=out)
    with pytest.raises(RuntimeError, match="dimensionality"):
        nufft.nu2u(points=pts, coord=coord, forward=True, epsilon=1e-5,
                   out=np.zeros((4, 4, 4), np.complex128))
    with pytest.raises(RuntimeError, match="periodicity"):
        nufft.nu2u(points=pts, coord=coord, forward=True, epsilon=1e-5, out=out,
                   periodicity=[1.0, 2.0, 3.0])
    with pytest.raises(RuntimeError, match="epsilon"):
        nufft.u2nu(grid=out, coord=coord, forward=True, epsilon=-1.0)


def test_plan_type_rules():
    coord = np.zeros((10, 2), np.float32)
    with pytest.raises(RuntimeError, match="unsupported"):
        nufft.plan(nu2u=True, coord=coord.astype(np.int32), grid_shape=(8, 8), epsilon=1e-5)


def test_parameter_choice_matches_oracle():
    """Planner (C++) and oracle (numpy) choose the same kernel row and
    oversampled sizes, which is what makes the tile keys bit-identical."""
    from oracle import nufft_oracle as O
    import ctypes
    for shape, eps, sp, M, nthr in [((256, 256), 1e-6, False, 200000, 1),
                                    ((4096, 4096), 1e-6, True, 50000000, 1),
                                    ((4096, 4096), 1e-6, True, 50000000, 8),
                                    ((256, 256, 256), 1e-10, False, 20000000, 8),
                                    ((1000,), 1e-4, True, 300, 1)]:
        kidx, nover = O.find_parameters(eps, 1.2, 2.51, shape, M, True, nthr, sp)
        row = O.kernel_db()[kidx]
        assert row[6] == sp
        assert len(nover) == len(shape)


@pytest.mark.parametrize("shape,eps,single", [((4096, 4096), 1e-6, True), ((300, 200), 1e-4, True),
                                              ((64, 80, 90), 1e-10, False), ((1000,), 1e-9, False)])
def test_kernel_candidates_match_oracle(shape, eps, single):
    """The autotuner's candidates: DUCC's available kernels (one per support,
    smallest oversampling factor reaching eps) with DUCC's oversampled sizes."""
    from ducc_b200 import autotune
    from oracle import nufft_oracle as O
    got = autotune.candidates(shape, eps, single, 1.1, 2.6)
    ref = O.available_kernels(eps, len(shape), single, 1.1, 2.6)
    assert [g[0] for g in got] == list(ref)
    db = O.kernel_db()
    for kidx, W, of, nov in got:
        assert W == db[kidx][0] and of == db[kidx][1]
        assert nov == [max(2 * O.good_size_complex(int(s * of * 0.5) + 1), 16) for s in shape]
    # the model's own choice is one of the candidates
    p = O.Params(shape, eps, single, 1000, True, 1)
    assert p.kidx in [g[0] for g in got]


def test_log2tile_option_checked():
    with pytest.raises(RuntimeError, match="log2tile"):
        nufft.plan(nu2u=True, coord=np.zeros((3, 2), np.float32), grid_shape=(16, 16),
                   epsilon=1e-4, log2tile=7)


def test_sht_defaults_and_argument_errors():
    """The spherical-harmonic entry points: DUCC's keyword defaults, and
    argument errors (null arrays, host memory, bad options) reported before
    any kernel launch."""
    import ctypes
    L = C.lib()
    o = C.ShtOpts()
    L.dnufft_sht_default_opts(ctypes.byref(o))
    assert o.nthreads == 1 and o.sigma_min == 1.1 and o.sigma_max == 2.6 and o.verbosity == 0
    ms = np.zeros(3, np.int64)
    pms = ms.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
    alm = np.zeros((1, 6), np.complex128)
    loc = np.zeros((4, 2))
    mp = np.zeros((1, 4))
    a_alm, a_loc, a_map = C.describe(alm), C.describe(loc), C.describe(mp)
    n0 = L.dnufft_kernel_launches()
    # null arrays
    st = L.dnufft_synthesis_general(None, 0, 0, 2, pms, 3, 1, ctypes.byref(a_loc), 1e-6,
                                    ctypes.byref(o), ctypes.byref(a_map), None)
    assert st == 1 and b"null" in L.dnufft_last_error()
    # host memory is not accepted by these entry points
    for f, a, b in ((L.dnufft_synthesis_general, a_alm, a_map),
                    (L.dnufft_adjoint_synthesis_general, a_map, a_alm)):
        st = f(ctypes.byref(a), 0, 0, 2, pms, 3, 1, ctypes.byref(a_loc), 1e-6,
               ctypes.byref(o), ctypes.byref(b), None)
        assert st == 1 and b"device array" in L.dnufft_last_error()
    assert L.dnufft_kernel_launches() == n0
