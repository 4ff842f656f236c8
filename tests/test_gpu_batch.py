"""Batched transforms (ducc_b200.batch) and the autotuner (ducc_b200.autotune).

A batch of 2D instances with different grid sizes, point counts, epsilons and
numbers of transforms is run through the multi-instance launches (replayed
from a CUDA graph) and checked, instance by instance and transform by
transform, against the oracle (FP64 restatement of DUCC's algorithm with the
same kernel and oversampled sizes) and against the instance's own plan.  Two
calls with different arrays check that the replayed graph reads the new
arguments.
"""
import numpy as np
import pytest

from ducc_b200 import autotune, batch, nufft
from oracle import nufft_oracle as O

pytestmark = pytest.mark.gpu

INSTANCES = [
    # shape, npoints, eps, ntrans
    ((64, 64), 1000, 1e-4, 1),
    ((96, 130), 5000, 1e-6, 3),
    ((250, 180), 20000, 1e-4, 1),
    ((300, 300), 3000, 1e-6, 2),
    ((70, 512), 12000, 1e-5, 1),
    ((128, 66), 800, 1e-6, 4),
]


def make(single, seed):
    import torch
    rng = np.random.default_rng(seed)
    cdt, ct = (np.float32, np.complex64) if single else (np.float64, np.complex128)
    insts = []
    for shape, M, eps, nt in INSTANCES:
        if not single:
            eps = eps * 1e-4
        coord = rng.uniform(-np.pi, np.pi, (M, 2)).astype(cdt)
        vals = (rng.standard_normal((nt, M)) + 1j * rng.standard_normal((nt, M))).astype(ct)
        grid = (rng.standard_normal((nt,) + shape) + 1j * rng.standard_normal((nt,) + shape)).astype(ct)
        p = nufft.plan(nu2u=True, coord=torch.from_numpy(coord).cuda(), grid_shape=shape,
                       epsilon=eps, nthreads=1, sigma_min=1.2, sigma_max=2.51)
        insts.append(dict(shape=shape, M=M, eps=eps, nt=nt, coord=coord, vals=vals, grid=grid,
                          plan=p))
    return insts


def dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


@pytest.mark.parametrize("single", [True, False])
def test_batch_type1_matches_oracle_and_plans(single):
    import torch
    insts = make(single, 1)
    b = batch.Batch([it["plan"] for it in insts], ntrans=[it["nt"] for it in insts])
    for rep in range(2):   # second call: replayed graph, new arrays
        pts, outs = [], []
        for it in insts:
            v = it["vals"] if rep == 0 else it["vals"][::-1].copy()
            it["cur"] = v
            pts.append(dev(v) if it["nt"] > 1 else dev(v[0]))
            shp = ((it["nt"],) if it["nt"] > 1 else ()) + it["shape"]
            outs.append(torch.full(shp, float("nan"), dtype=pts[-1].dtype, device="cuda"))
        b.nu2u(points=pts, out=outs, forward=True)
        torch.cuda.synchronize()
        for it, o in zip(insts, outs):
            got = o.cpu().numpy().reshape((it["nt"],) + it["shape"])
            p = O.Params(it["shape"], it["eps"], single, it["M"], True, 1)
            for t in range(it["nt"]):
                ref = O.nu2u(p, it["coord"], it["cur"][t], True)
                assert O.l2error(got[t], ref) < max(it["eps"], 3e-7 if single else 1e-13)
                own = it["plan"].nu2u(points=dev(it["cur"][t]), forward=True).cpu().numpy()
                assert O.l2error(got[t], own) < (1e-6 if single else 1e-12)


@pytest.mark.parametrize("single", [True, False])
def test_batch_type2_matches_oracle(single):
    import torch
    insts = make(single, 2)
    b = batch.Batch([it["plan"] for it in insts], ntrans=[it["nt"] for it in insts])
    for fwd in (False, True):
        grids, outs = [], []
        for it in insts:
            g = it["grid"]
            grids.append(dev(g) if it["nt"] > 1 else dev(g[0]))
            shp = (it["nt"], it["M"]) if it["nt"] > 1 else (it["M"],)
            outs.append(torch.full(shp, float("nan"), dtype=grids[-1].dtype, device="cuda"))
        b.u2nu(grids=grids, out=outs, forward=fwd)
        torch.cuda.synchronize()
        for it, o in zip(insts, outs):
            got = o.cpu().numpy().reshape(it["nt"], it["M"])
            p = O.Params(it["shape"], it["eps"], single, it["M"], True, 1)
            for t in range(it["nt"]):
                ref = O.u2nu(p, it["grid"][t], it["coord"], fwd)
                assert O.l2error(got[t], ref) < max(it["eps"], 3e-7 if single else 1e-13)


def test_batch_rejects_bad_arguments():
    import torch
    insts = make(True, 3)
    b = batch.Batch([insts[0]["plan"], insts[2]["plan"]])
    with pytest.raises(RuntimeError):
        # host arrays are not accepted by the batch
        b.nu2u(points=[insts[0]["vals"][0], insts[2]["vals"][0]],
               out=[np.zeros(insts[0]["shape"], np.complex64),
                    np.zeros(insts[2]["shape"], np.complex64)], forward=True)
    with pytest.raises(RuntimeError):
        b.nu2u(points=[dev(insts[0]["vals"][0]), dev(insts[2]["vals"][0])],
               out=[torch.zeros((5, 5), dtype=torch.complex64, device="cuda"),
                    torch.zeros(insts[2]["shape"], dtype=torch.complex64, device="cuda")],
               forward=True)
    c = torch.from_numpy(np.zeros((10, 2))).cuda()
    p64 = nufft.plan(nu2u=True, coord=c, grid_shape=(32, 32), epsilon=1e-9)
    with pytest.raises(RuntimeError, match="precision"):
        batch.Batch([insts[0]["plan"], p64])


def test_autotune_choice_is_accurate():
    import torch
    rng = np.random.default_rng(4)
    shape, M, eps = (200, 160), 30000, 1e-5
    coord = rng.uniform(-np.pi, np.pi, (M, 2)).astype(np.float32)
    vals = (rng.standard_normal(M) + 1j * rng.standard_normal(M)).astype(np.complex64)
    res = autotune.tune(dev(coord), shape, eps, ntrans=2, reps=2)
    assert len(res["table"]) >= 2 and res["ms"] > 0
    p = nufft.plan(nu2u=True, coord=dev(coord), grid_shape=shape, epsilon=eps,
                   **autotune.plan_kwargs(res))
    assert p.info()["supp"] == res["supp"] and p.info()["nover"] == res["nover"]
    got = p.nu2u(points=dev(vals), forward=True).cpu().numpy()
    ref = O.direct_nu2u(coord, vals, shape, True)
    assert O.l2error(got, ref) < 2 * 2 * eps
    assert autotune.tune(dev(coord), shape, eps, ntrans=2) is res   # cached
