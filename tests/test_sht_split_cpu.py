"""The split of synthesis_general / adjoint_synthesis_general over processes
(ducc_b200.distributed.synthesis_general_split / adjoint_synthesis_general_split)
on the CPU with two and three `gloo` ranks: every rank evaluates its
consecutive share of the points, the all-gather assembles the map and the
all-reduce sums the partial a_lm.  Without a GPU the rank's computation is the
direct sum of oracle/sht_oracle.py on its share, so the assembled results must
equal the direct sums over all points; tests/test_gpu_sht.py checks that the
library's results on shares add up the same way."""
import json
import os
import socket

import numpy as np
import pytest

from oracle import sht_oracle as O

LMAX, NPTS = 12, 47


def _free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _problem(spin):
    rng = np.random.default_rng(5 + spin)
    ncomp = 1 if spin == 0 else 2
    alm = O.random_alm_spin(LMAX, LMAX, spin, ncomp, rng)
    loc = np.stack([rng.uniform(0, np.pi, NPTS), rng.uniform(0, 2 * np.pi, NPTS)], 1)
    mp = rng.uniform(-1, 1, (ncomp, NPTS))
    return alm, loc, mp


def _synth(alm, spin, loc, **_):
    if spin == 0:
        return O.synthesis(alm[0], LMAX, LMAX, loc)[None]
    return O.synthesis_spin(alm, spin, LMAX, LMAX, loc)


def _adj(map, spin, loc, **_):
    if spin == 0:
        return O.adjoint_synthesis(map[0], LMAX, LMAX, loc)[None]
    return O.adjoint_synthesis_spin(map, spin, LMAX, LMAX, loc)


def _worker(rank, world, port, outdir):
    import datetime

    import torch.distributed as td

    from ducc_b200 import distributed as D
    td.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                          world_size=world, timeout=datetime.timedelta(seconds=60))
    errs = []
    try:
        for spin in (0, 2):
            alm, loc, mp = _problem(spin)
            seen = []

            def synth(loc, **kw):
                seen.append(loc.shape[0])
                return _synth(loc=loc, **kw)

            m = D.synthesis_general_split(_run=synth, alm=alm, spin=spin, lmax=LMAX, loc=loc,
                                          epsilon=1e-10)
            a = D.adjoint_synthesis_general_split(_run=_adj, map=mp, spin=spin, lmax=LMAX,
                                                  loc=loc, epsilon=1e-10)
            ref_m = _synth(alm=alm, spin=spin, loc=loc)
            ref_a = _adj(map=mp, spin=spin, loc=loc)
            errs.append([float(np.abs(m - ref_m).max()), float(np.abs(a - ref_a).max()),
                         seen[0]])
        td.barrier()
    finally:
        td.destroy_process_group()
    with open(os.path.join(outdir, "rank%d.json" % rank), "w") as f:
        json.dump(errs, f)


@pytest.mark.parametrize("world", [2, 3])
def test_point_split_over_gloo_ranks(tmp_path, world):
    import torch.multiprocessing as mp
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    shares = [0, 0]
    for r in range(world):
        res = json.load(open(tmp_path / ("rank%d.json" % r)))
        for i, (em, ea, n) in enumerate(res):
            assert em < 1e-12 and ea < 1e-12
            shares[i] += n
    assert shares == [NPTS, NPTS]
