"""Benchmark: 2D NUFFT at eps=1e-6 on a B200 (type 1 then type 2).

Workload (one "step"): on a 4096x4096 grid, M=5e7 points drawn from a mixture
of 16 Gaussians (sigma 0.3 rad, centres uniform in [-pi,pi)^2, wrapped),
float32 coordinates, complex64 values N(0,1): a planned nu2u followed by a
planned u2nu with the same plan (DUCC's ``plan.nu2u`` / ``plan.u2nu``; the
plan, which bins and sorts the fixed coordinates, is built before the timed
region in both arms).  Throughput = points x transforms / time, in Mpts/s.
The headline line uses the split-precision tensor-core spreader; the plain
FP32 atomic spreader is timed on the same inputs and reported beside it
(``alt_plain``), and both are checked against DUCC's FP64 transforms
(``errors``).

Arms
  default            this library on N GPUs (one process per GPU under
                     torchrun; each rank runs its own seeded instance: weak
                     scaling, no collective on the data path)
  --impl reference   DUCC's own CPU NUFFT (built from source into oracle/_ref)
                     on the host cores, rank 0 only, same plan-based step

Both arms print the same ``config`` and feed the same ``nthreads`` value to
DUCC's parameter cost model (``--param-threads``, default: the host's thread
count, which is also the thread count of the reference arm), so they choose
the same kernel support and oversampled grid.

Prints one JSON line (rank 0).
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_SIDE = 4096
M_POINTS = 50_000_000
EPS = 1e-6
ERR_SUBSET = 100_000      # type-2 error: DUCC FP64 evaluated on this many points
METRIC = "NUFFT Mpts/s 2D eps=1e-6: TC split-prec vs plain FP32 spreader, same B200"

# Counter-based figures of the dominant launches, from the ncu summaries under
# profiles/ (named there), for the workload they were captured on.  They are
# attached to the line only when the run's workload is that one.
PROFILED = {
    "workload": (4096, 50_000_000),
    # dram__bytes_read.sum + dram__bytes_write.sum of one spreading launch
    # (profiles/launches_bench_4096sq_M5e7.md, one-pass metrics, full workload)
    "spread_dram_bytes": {"tc": 6460321536.0 + 528613120.0,
                          "plain": 6345106944.0 + 451456000.0},
    # shared-memory wavefronts of one launch (l1tex__data_pipe_lsu_wavefronts_
    # mem_shared_op_atom.sum for the plain spreader, ..._op_ld.sum for the
    # interpolation), captured at 2048^2 / M=1.25e7 (profiles/k_spread_plain_
    # 2048sq_M12.5M.md, profiles/k_interp_2048sq_M12.5M.md) and scaled by 4:
    # the points and the grid cells both grow by 4 at the same points per tile
    "smem_wavefronts": {"plain_spread": 4 * 210563619.0, "interp": 4 * 86883694.0},
}


def clustered_coords(rng, m, ncl=16, sigma=0.3):
    centres = rng.uniform(-np.pi, np.pi, (ncl, 2))
    which = rng.integers(0, ncl, m)
    x = centres[which] + sigma * rng.standard_normal((m, 2))
    x = np.mod(x + np.pi, 2 * np.pi) - np.pi
    return x.astype(np.float32)


def make_inputs(seed, m, n):
    rng = np.random.default_rng(seed)
    coord = clustered_coords(rng, m)
    vals = (rng.standard_normal(m, dtype=np.float32)
            + 1j * rng.standard_normal(m, dtype=np.float32)).astype(np.complex64)
    grid = (rng.standard_normal((n, n), dtype=np.float32)
            + 1j * rng.standard_normal((n, n), dtype=np.float32)).astype(np.complex64)
    return coord, vals, grid


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p["hbm_gbs"], p["bf16_tflops"], "measured"
    except Exception:
        return 6650.0, 1590.0, "fallback"


# ---------------------------------------------------------------- shared by both arms
def bench_config(args):
    """The workload description; identical in both arms' lines."""
    return {"workload": "2D type-1 + type-2 NUFFT, 4096x4096 grid, M=5e7 clustered points "
                        "(16 Gaussians, sigma 0.3), f32 coords, c64, eps=1e-6",
            "grid": [args.n, args.n], "npoints": args.m, "eps": EPS,
            "coord_dtype": "float32", "value_dtype": "complex64",
            "step": "plan.nu2u(forward=True) + plan.u2nu(forward=False), one plan built "
                    "before the timed region",
            "param_threads": args.param_threads,
            "l2": "inputs and oversampled grid larger than L2 (no flush needed)"}


# ---------------------------------------------------------------- reference arm
def run_reference(args, rank):
    if rank != 0:
        return
    from oracle import ref
    R = ref.load()
    if R is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          "DUCC module not built in oracle/_ref (make -C oracle)"}))
        return
    m, n = args.m, args.n
    coord, vals, grid = make_inputs(1234, m, n)
    nthr = args.param_threads
    choice = R.params_probe(shape=[n, n], npoints=m, epsilon=EPS, singleprec=True,
                            gridding=True, nthreads=nthr, sigma_min=1.1, sigma_max=2.6)
    out = np.empty((n, n), np.complex64)
    pts = np.empty(m, np.complex64)
    t0 = time.perf_counter()
    plan = R.nufft.plan(nu2u=True, coord=coord, grid_shape=(n, n), epsilon=EPS, nthreads=nthr)
    plan_s = time.perf_counter() - t0

    def step():
        plan.nu2u(points=vals, forward=True, out=out)
        plan.u2nu(grid=grid, forward=False, out=pts)

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = (time.perf_counter() - t0) / args.steps
    v = 2 * m / dt / 1e6
    # DUCC's functions without a plan (each call bins and sorts), for reference
    t0 = time.perf_counter()
    R.nufft.nu2u(points=vals, coord=coord, forward=True, epsilon=EPS, nthreads=nthr, out=out)
    R.nufft.u2nu(grid=grid, coord=coord, forward=False, epsilon=EPS, nthreads=nthr, out=pts)
    du = time.perf_counter() - t0
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "Mpts/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c64 (f32 arithmetic)", "data": "synthetic",
        "config": bench_config(args),
        "parallelism": "%d host threads" % nthr,
        "call": "ducc0.nufft.plan(nu2u=True, coord, grid_shape, epsilon, nthreads) "
                ".nu2u + .u2nu (DUCC's own CPU NUFFT, built from source)",
        "ducc_choice": {"kernel_index": choice["kernel_index"], "supp": choice["W"],
                        "ofactor": choice["ofactor"], "nover": choice["nover"]},
        "plan_create_s": plan_s,
        "unplanned": {"value": 2 * m / du / 1e6, "ms_per_step": du * 1e3,
                      "call": "ducc0.nufft.nu2u + u2nu", "steps": 1},
        "cpu_baseline": {"value": v, "unit": "Mpts/s", "cores": nthr, "kind": "reference",
                         "sample": "the full workload, %d planned step(s)" % args.steps},
        "e2e": {"value": v, "unit": "Mpts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


# ---------------------------------------------------------------- other workloads
# Reported beside the headline (same JSON line, "workloads"): the batched,
# differentiable and 3D double-precision transforms, each timed with CUDA
# events on the current stream after warm-up.
def _events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def workload_batched(dev, steps=5, warmup=2, ninst=64, seed=7):
    """64 uneven 2D instances: side log-uniform in [64, 1024] (even), M
    log-uniform in [1e3, 1e6] uniform points, ntrans in {1, 4}, eps in
    {1e-4, 1e-6}, complex64; autotuned per instance; one batch (multi-instance
    launches replayed from a CUDA graph) against the same plans run one by one."""
    import torch
    from ducc_b200 import autotune, batch, nufft
    rng = np.random.default_rng(seed)
    t0 = time.perf_counter()
    plans, nts, pts, outs, grids, pouts, total = [], [], [], [], [], [], 0
    for _ in range(ninst):
        side = int(round(np.exp(rng.uniform(np.log(64), np.log(1024))) / 2)) * 2
        M = int(np.exp(rng.uniform(np.log(1e3), np.log(1e6))))
        nt = int(rng.choice([1, 4]))
        eps = float(rng.choice([1e-4, 1e-6]))
        coord = torch.from_numpy(rng.uniform(-np.pi, np.pi, (M, 2)).astype(np.float32)).to(dev)
        choice = autotune.tune(coord, (side, side), eps, ntrans=nt, reps=1)
        plans.append(nufft.plan(nu2u=True, coord=coord, grid_shape=(side, side), epsilon=eps,
                                **autotune.plan_kwargs(choice)))
        nts.append(nt)
        v = torch.randn((nt, M), dtype=torch.complex64, device=dev)
        g = torch.randn((nt, side, side), dtype=torch.complex64, device=dev)
        pts.append(v)
        grids.append(g)
        outs.append(torch.empty((nt, side, side), dtype=torch.complex64, device=dev))
        pouts.append(torch.empty((nt, M), dtype=torch.complex64, device=dev))
        total += M * nt
    tune_s = time.perf_counter() - t0
    b = batch.Batch(plans, ntrans=nts)

    def batched():
        b.nu2u(points=pts, out=outs, forward=True)
        b.u2nu(grids=grids, out=pouts, forward=False)

    def one_by_one():
        for p, nt, v, o, g, po in zip(plans, nts, pts, outs, grids, pouts):
            for t in range(nt):
                p.nu2u(points=v[t], forward=True, out=o[t])
                p.u2nu(grid=g[t], forward=False, out=po[t])

    res = {}
    for name, fn in (("batched", batched), ("one_by_one", one_by_one)):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize(dev)
        e0, e1 = _events()
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize(dev)
        res[name] = e0.elapsed_time(e1) / steps
    return {"metric": "Mpts/s (points x transforms x 2 / time)",
            "value": 2 * total / (res["batched"] * 1e-3) / 1e6,
            "ms_per_step": res["batched"], "one_by_one_ms": res["one_by_one"],
            "one_by_one_value": 2 * total / (res["one_by_one"] * 1e-3) / 1e6,
            "instances": ninst, "points_x_ntrans": total, "autotune_s": tune_s,
            "config": "64 uneven 2D instances (side 64..1024, M 1e3..1e6, ntrans 1/4, "
                      "eps 1e-4/1e-6), complex64, step = batched nu2u + u2nu"}


def workload_autograd(dev, steps=5, warmup=2, seed=8):
    """1024^2 complex64 image, radial trajectory 2048 spokes x 2048 samples,
    float32 coordinates, eps 1e-6: forward u2nu + backward (image and
    coordinate gradients) of L = ||u2nu(img) - y||^2."""
    import torch
    from ducc_b200 import autograd as AG
    rng = np.random.default_rng(seed)
    N, ns = 1024, 2048
    ang = np.pi * np.arange(ns) / ns
    rad = np.linspace(-np.pi, np.pi, ns, endpoint=False)
    x = np.stack([np.outer(np.cos(ang), rad).ravel(), np.outer(np.sin(ang), rad).ravel()], 1)
    coord = torch.from_numpy(x.astype(np.float32)).to(dev).requires_grad_()
    img = torch.randn((N, N), dtype=torch.complex64, device=dev).requires_grad_()
    with torch.no_grad():
        y = AG.u2nu(img + 0.3 * torch.randn_like(img), coord, epsilon=1e-6)

    def step():
        img.grad = None
        coord.grad = None
        loss = (AG.u2nu(img, coord, epsilon=1e-6) - y).abs().pow(2).sum()
        loss.backward()

    for _ in range(warmup):
        step()
    torch.cuda.synchronize(dev)
    e0, e1 = _events()
    e0.record()
    for _ in range(steps):
        step()
    e1.record()
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / steps
    return {"metric": "ms per forward + backward", "value": ms,
            "mpts_per_s": ns * ns / (ms * 1e-3) / 1e6,
            "config": "1024^2 c64 image, 2048x2048 radial f32 coords, eps 1e-6; step = plan + "
                      "u2nu + adjoint nu2u + derivative-kernel coordinate gradient"}


def workload_3d(dev, steps=3, warmup=1, seed=9):
    """3D type 2 on a 256^3 grid, M = 2e7 uniform points: float64 coordinates
    and complex128 modes at eps 1e-10, and float32 / complex64 at eps 1e-5."""
    import torch
    from ducc_b200 import nufft
    rng = np.random.default_rng(seed)
    N, M = 256, 20_000_000
    out = {}
    for name, cdt, ct, eps in (("fp64_eps1e-10", np.float64, torch.complex128, 1e-10),
                               ("fp32_eps1e-5", np.float32, torch.complex64, 1e-5)):
        coord = torch.from_numpy(rng.uniform(-np.pi, np.pi, (M, 3)).astype(cdt)).to(dev)
        grid = torch.randn((N, N, N), dtype=ct, device=dev)
        pts = torch.empty(M, dtype=ct, device=dev)
        p = nufft.plan(nu2u=False, coord=coord, grid_shape=(N, N, N), epsilon=eps, nthreads=8)
        for _ in range(warmup):
            p.u2nu(grid=grid, forward=True, out=pts)
        torch.cuda.synchronize(dev)
        e0, e1 = _events()
        e0.record()
        for _ in range(steps):
            p.u2nu(grid=grid, forward=True, out=pts)
        e1.record()
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1) / steps
        out[name] = {"ms": ms, "mpts_per_s": M / (ms * 1e-3) / 1e6, "supp": p.info()["supp"],
                     "nover": p.info()["nover"]}
        del p, coord, grid, pts
        torch.cuda.empty_cache()
    out["config"] = "3D type 2, 256^3 modes, M=2e7 uniform points, planned u2nu"
    return out


WG_NPIX, WG_NROW, WG_NCHAN, WG_EPS = 4096, 500_000, 16, 1e-5


def wgridder_inputs(seed=11, nrow=WG_NROW, npix=WG_NPIX):
    """Synthetic measurement set for the w-gridder workload: 500k rows x 16
    channels (8e6 visibilities, 1.0-1.45 GHz), baselines filling the uv plane of
    a 4096^2 image at 2 degrees field of view (|u|, |v| up to ~0.45 / pixel size
    at the top channel), w up to a third of that; complex64 visibilities,
    float32 weights, a 4096^2 float32 image for the degridding direction."""
    rng = np.random.default_rng(seed)
    ps = 2.0 * np.pi / 180 / npix
    freq = 1.0e9 + np.arange(WG_NCHAN) * (0.45e9 / WG_NCHAN)
    umax = 0.45 / ps * 299792458. / freq[-1]
    r = umax * np.sqrt(rng.random(nrow))
    phi = rng.uniform(0, 2 * np.pi, nrow)
    uvw = np.stack([r * np.cos(phi), r * np.sin(phi), rng.uniform(-umax / 3, umax / 3, nrow)], 1)
    vis = (rng.standard_normal((nrow, WG_NCHAN))
           + 1j * rng.standard_normal((nrow, WG_NCHAN))).astype(np.complex64)
    wgt = rng.uniform(0.5, 1.5, (nrow, WG_NCHAN)).astype(np.float32)
    dirty = rng.standard_normal((npix, npix)).astype(np.float32)
    return ps, freq, uvw, vis, wgt, dirty


def workload_wgridder(dev, steps=5, warmup=2, nrow=WG_NROW, npix=WG_NPIX):
    """w-gridder (ducc0.wgridder counterpart): vis2dirty and dirty2vis with
    w-stacking at eps 1e-5 on the synthetic set above, device-resident."""
    import torch
    from ducc_b200 import wgridder as WG
    ps, freq, uvw, vis, wgt, dirty = wgridder_inputs(nrow=nrow, npix=npix)
    d_uvw = torch.from_numpy(uvw).to(dev)
    d_freq = torch.from_numpy(freq).to(dev)
    d_vis = torch.from_numpy(vis).to(dev)
    d_wgt = torch.from_numpy(wgt).to(dev)
    d_dirty = torch.from_numpy(dirty).to(dev)
    out_dirty = torch.empty((npix, npix), dtype=torch.float32, device=dev)
    out_vis = torch.empty((nrow, WG_NCHAN), dtype=torch.complex64, device=dev)
    kw = dict(uvw=d_uvw, freq=d_freq, wgt=d_wgt, pixsize_x=ps, pixsize_y=ps, epsilon=WG_EPS,
              do_wgridding=True, nthreads=16)
    out = {}
    for name, call in (
            ("vis2dirty", lambda: WG.vis2dirty(vis=d_vis, dirty=out_dirty, **kw)),
            ("dirty2vis", lambda: WG.dirty2vis(dirty=d_dirty, vis=out_vis, **kw))):
        for _ in range(warmup):
            call()
        torch.cuda.synchronize(dev)
        e0, e1 = _events()
        e0.record()
        for _ in range(steps):
            call()
        e1.record()
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1) / steps
        out[name] = {"ms": ms, "mvis_per_s": nrow * WG_NCHAN / (ms * 1e-3) / 1e6}
    prm = WG.wgrid_params(uvw=d_uvw, freq=d_freq, vis=d_vis, wgt=d_wgt, npix_x=npix,
                          npix_y=npix, pixsize_x=ps, pixsize_y=ps, epsilon=WG_EPS,
                          do_wgridding=True, nthreads=16)
    out["parameters"] = {k: prm[k] for k in ("supp", "nu", "nv", "nplanes")}
    out["config"] = ("w-gridder, %d rows x %d channels (complex64), %d^2 image at 2 deg, "
                     "w-stacking, eps %g; device-resident vis2dirty / dirty2vis"
                     % (nrow, WG_NCHAN, npix, WG_EPS))
    return out


def cpu_baseline_wgridder(nthreads):
    """DUCC's own w-gridder on the host cores, one call of each direction on the
    w-gridder workload's inputs."""
    from oracle import ref
    R = ref.load()
    if R is None or not hasattr(R, "wgridder"):
        return None
    ps, freq, uvw, vis, wgt, dirty = wgridder_inputs()
    kw = dict(uvw=uvw, freq=freq, wgt=wgt, pixsize_x=ps, pixsize_y=ps, epsilon=WG_EPS,
              do_wgridding=True, nthreads=nthreads)
    res = {"cores": nthreads, "kind": "reference", "sample": "one call of each direction"}
    t0 = time.perf_counter()
    R.wgridder.vis2dirty(vis=vis, npix_x=WG_NPIX, npix_y=WG_NPIX, **kw)
    res["vis2dirty_ms"] = (time.perf_counter() - t0) * 1e3
    t0 = time.perf_counter()
    R.wgridder.dirty2vis(dirty=dirty, **kw)
    res["dirty2vis_ms"] = (time.perf_counter() - t0) * 1e3
    return res


SH_LMAX, SH_NPTS, SH_EPS = 2047, 10_000_000, 1e-5


def sphere_inputs(seed=12, lmax=SH_LMAX, npts=SH_NPTS):
    """Synthetic inputs of the sphere workload: a spin-0 expansion to
    lmax = mmax = 2047 with coefficients uniform in [-1, 1) (a_l0 real, as
    DUCC's test_sht.py random_alm), complex64; 1e7 points uniform on the
    sphere (theta = arccos U[-1, 1], phi = U[0, 2 pi)) in float64; map values
    uniform in [-0.5, 0.5) as float32 for the adjoint direction."""
    rng = np.random.default_rng(seed)
    nalm = ((lmax + 1) * (lmax + 2)) // 2
    alm = (rng.uniform(-1, 1, nalm) + 1j * rng.uniform(-1, 1, nalm)).astype(np.complex64)
    alm[:lmax + 1] = alm[:lmax + 1].real
    loc = np.stack([np.arccos(rng.uniform(-1, 1, npts)), rng.uniform(0, 2 * np.pi, npts)], 1)
    mp = rng.uniform(-0.5, 0.5, (1, npts)).astype(np.float32)
    return alm[None, :], loc, mp


def workload_sphere(dev, steps=5, warmup=2, lmax=SH_LMAX, npts=SH_NPTS, with_outputs=False):
    """Spin-0 synthesis at arbitrary points and its adjoint
    (ducc0.sht.synthesis_general / adjoint_synthesis_general counterparts) at
    eps 1e-5 in single precision, device-resident, each call timed with CUDA
    events (median, min and max over the calls)."""
    import torch
    from ducc_b200 import _capi as C
    from ducc_b200 import sht as SH
    alm, loc, mp = sphere_inputs(lmax=lmax, npts=npts)
    d_alm = torch.from_numpy(alm).to(dev)
    d_loc = torch.from_numpy(loc).to(dev)
    d_mp = torch.from_numpy(mp).to(dev)
    out_map = torch.empty((1, npts), dtype=torch.float32, device=dev)
    out_alm = torch.empty_like(d_alm)
    kw = dict(spin=0, lmax=lmax, mmax=lmax, loc=d_loc, epsilon=SH_EPS, nthreads=16)
    # spin 2 (E and B rows -> Q and U) on the same points
    d_alm2 = torch.cat([d_alm, d_alm.flip(1)]).contiguous()
    d_alm2[:, :lmax + 1] = d_alm2[:, :lmax + 1].real.to(d_alm2.dtype)
    d_alm2[:, 0:2] = 0
    d_alm2[:, lmax + 1] = 0
    d_mp2 = torch.cat([d_mp, d_mp.flip(1)]).contiguous()
    out_map2 = torch.empty((2, npts), dtype=torch.float32, device=dev)
    out_alm2 = torch.empty_like(d_alm2)
    kw2 = dict(kw, spin=2)
    out = {}
    for name, call in (
            ("synthesis_general", lambda: SH.synthesis_general(alm=d_alm, map=out_map, **kw)),
            ("adjoint_synthesis_general",
             lambda: SH.adjoint_synthesis_general(map=d_mp, alm=out_alm, **kw)),
            ("synthesis_general_spin2",
             lambda: SH.synthesis_general(alm=d_alm2, map=out_map2, **kw2)),
            ("adjoint_synthesis_general_spin2",
             lambda: SH.adjoint_synthesis_general(map=d_mp2, alm=out_alm2, **kw2))):
        for _ in range(warmup):
            call()
        torch.cuda.synchronize(dev)
        n0 = C.lib().dnufft_kernel_launches()
        per = []
        for _ in range(steps):
            e0, e1 = _events()
            e0.record()
            call()
            e1.record()
            torch.cuda.synchronize(dev)
            per.append(e0.elapsed_time(e1))
        ms = float(np.median(per))
        out[name] = {"ms": ms, "ms_min": float(min(per)), "ms_max": float(max(per)),
                     "mpts_per_s": npts / (ms * 1e-3) / 1e6,
                     "gpu_launches_per_call": (C.lib().dnufft_kernel_launches() - n0) / steps}
    out["config"] = ("synthesis_general / adjoint, spin 0 and spin 2, lmax = mmax = %d "
                     "(complex64 a_lm), %d points uniform on the sphere (float64 theta, phi), "
                     "eps %g; device-resident" % (lmax, npts, SH_EPS))
    if with_outputs:
        out["_map"] = out_map.cpu().numpy()
        out["_alm"] = out_alm.cpu().numpy()
        out["_spin2"] = (d_alm2.cpu().numpy(), d_mp2.cpu().numpy(), out_map2.cpu().numpy(),
                         out_alm2.cpu().numpy())
    return out


def cpu_baseline_sphere(nthreads, ours_map=None, ours_alm=None, spin2=None):
    """DUCC's own synthesis_general / adjoint_synthesis_general on the host
    cores, one call of each direction on the sphere workload's inputs, and the
    relative L2 error of our outputs against DUCC's at eps 1e-5."""
    from oracle import ref
    R = ref.load()
    if R is None or not hasattr(R, "sht"):
        return None
    alm, loc, mp = sphere_inputs()
    kw = dict(spin=0, lmax=SH_LMAX, mmax=SH_LMAX, loc=loc, epsilon=SH_EPS, nthreads=nthreads)
    res = {"cores": nthreads, "kind": "reference", "sample": "one call of each direction"}
    t0 = time.perf_counter()
    m2 = R.sht.synthesis_general(alm=alm, **kw)
    res["synthesis_general_ms"] = (time.perf_counter() - t0) * 1e3
    t0 = time.perf_counter()
    a2 = R.sht.adjoint_synthesis_general(map=mp, **kw)
    res["adjoint_synthesis_general_ms"] = (time.perf_counter() - t0) * 1e3

    def l2(a, b):
        a, b = np.asarray(a, np.complex128).ravel(), np.asarray(b, np.complex128).ravel()
        return float(np.sqrt(np.sum(np.abs(a - b) ** 2) / np.sum(np.abs(b) ** 2)))
    if ours_map is not None:
        res["l2_vs_ducc_synthesis"] = l2(ours_map, m2)
    if ours_alm is not None:
        res["l2_vs_ducc_adjoint"] = l2(ours_alm, a2)
    if spin2 is not None:
        alm2, mp2, om2, oa2 = spin2
        kw2 = dict(kw, spin=2)
        t0 = time.perf_counter()
        m2 = R.sht.synthesis_general(alm=alm2, **kw2)
        res["synthesis_general_spin2_ms"] = (time.perf_counter() - t0) * 1e3
        t0 = time.perf_counter()
        a2 = R.sht.adjoint_synthesis_general(map=mp2, **kw2)
        res["adjoint_synthesis_general_spin2_ms"] = (time.perf_counter() - t0) * 1e3
        res["l2_vs_ducc_synthesis_spin2"] = l2(om2, m2)
        res["l2_vs_ducc_adjoint_spin2"] = l2(oa2, a2)
    return res


# ---------------------------------------------------------------- our arm
def cpu_baseline_leg(args, coord, vals, grid, budget_s=20.0):
    """DUCC's CPU NUFFT on the host cores (same planned step, same inputs),
    bounded to about budget_s seconds.  Returns the baseline entry and DUCC's
    own single-precision outputs (kept for the error report)."""
    from oracle import ref
    R = ref.load()
    if R is None:
        return None, None
    m, n, nthr = args.m, args.n, args.param_threads
    out = np.empty((n, n), np.complex64)
    pts = np.empty(m, np.complex64)
    plan = R.nufft.plan(nu2u=True, coord=coord, grid_shape=(n, n), epsilon=EPS, nthreads=nthr)
    t0 = time.perf_counter()
    plan.nu2u(points=vals, forward=True, out=out)
    plan.u2nu(grid=grid, forward=False, out=pts)
    first = time.perf_counter() - t0
    reps = max(1, min(3, int(budget_s / max(first, 1e-3)) - 1))
    t0 = time.perf_counter()
    for _ in range(reps):
        plan.nu2u(points=vals, forward=True, out=out)
        plan.u2nu(grid=grid, forward=False, out=pts)
    dt = (time.perf_counter() - t0) / reps
    return ({"value": 2 * m / dt / 1e6, "unit": "Mpts/s", "cores": nthr, "kind": "reference",
             "sample": "the full workload (plan.nu2u + plan.u2nu, M=%d), 1 warm-up + %d timed"
                       % (m, reps)},
            (out, pts))


def error_report(args, coord, vals, grid, err_idx, ours, ducc_f32):
    """Relative L2 errors (DUCC's l2error) of the type-1 outputs over the whole
    grid and of the type-2 outputs at err_idx, against DUCC's FP64 transforms
    (float64 coordinates, complex128 data, eps=1e-13) of the same inputs."""
    from oracle import ref
    from oracle.nufft_oracle import l2error
    R = ref.load()
    if R is None:
        return None
    n, nthr = args.n, args.param_threads
    t0 = time.perf_counter()
    c64 = coord.astype(np.float64)
    ref1 = np.empty((n, n), np.complex128)
    R.nufft.nu2u(points=vals.astype(np.complex128), coord=c64, forward=True, epsilon=1e-13,
                 nthreads=nthr, out=ref1)
    ref2 = R.nufft.u2nu(grid=grid.astype(np.complex128), coord=c64[err_idx], forward=False,
                        epsilon=1e-13, nthreads=nthr)
    del c64
    rep = {"reference": "DUCC FP64 nu2u / u2nu (float64 coords, complex128, eps=1e-13)",
           "type1_points": args.m, "type2_points": int(len(err_idx)),
           "type1": {}, "type2": {}}
    for sp, (g, p) in ours.items():
        rep["type1"][sp] = l2error(g, ref1)
        rep["type2"][sp] = l2error(p, ref2)
    if ducc_f32 is not None:
        rep["type1"]["ducc_f32"] = l2error(ducc_f32[0], ref1)
        rep["type2"]["ducc_f32"] = l2error(ducc_f32[1][err_idx], ref2)
    if "tc" in ours and "plain" in ours:
        rep["type1_tc_over_plain"] = rep["type1"]["tc"] / rep["type1"]["plain"]
    if "tc" in ours and "plain_matched" in ours:
        rep["type1_tc_over_plain_matched"] = rep["type1"]["tc"] / rep["type1"]["plain_matched"]
    rep["seconds"] = time.perf_counter() - t0
    return rep


def max_over_ranks(value, dev, dist):
    """The largest of every rank's value (the job's time is its slowest rank)."""
    if not dist:
        return value
    import torch
    import torch.distributed as td
    t = torch.tensor([float(value)], device=dev)
    td.all_reduce(t, op=td.ReduceOp.MAX)
    return float(t.item())


def _stage_ms(prof):
    return {k: v[0] / max(v[1], 1) for k, v in prof.items()}


def kernel_rooflines(stages, spreader, info, m, n, recs, hbm, bf16, sm_mhz, peak_src):
    """One entry per kernel of the step: its bound resource, the achieved rate
    from its CUDA-event time inside the timed region and the fraction of that
    resource's peak.  Algorithmic bytes assume complex64 values (8 B), float32
    coordinates (4 B per axis) and a uint32 permutation."""
    n0, n1 = info["nover"]
    N0, N1 = n, n
    cells, kept = n0 * n1, n0 * N1
    out = {}

    def hbm_entry(key, nbytes, bound="hbm"):
        ms = stages.get(key)
        if not ms:
            return None
        ach = nbytes / (ms * 1e-3) / 1e9
        return {"bound": bound, "avg_launch_ms": ms, "algorithmic_bytes": nbytes,
                "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                "peak_source": peak_src}

    pts_bytes = m * (8 + 8 + 4)   # sorted coords, values (gathered), permutation
    out["zeroing grid (memset)"] = hbm_entry("nu2u (planned)/zeroing grid", cells * 8)
    sp = stages.get("nu2u (planned)/spreading")
    if sp:
        if spreader == "tc":
            fl = recs * 2 * 128 * 48 * 16
            ach = fl / (sp * 1e-3) / 1e12
            e = {"bound": "tensor", "avg_launch_ms": sp, "executed_flops": fl,
                 "achieved": ach, "peak": bf16, "unit": "TFLOP/s", "frac": ach / bf16,
                 "peak_source": peak_src,
                 "note": "one 128x48x16 FP16 MMA per K-block record (<= 16 points)"}
        else:
            wf = PROFILED["smem_wavefronts"]["plain_spread"]
            e = {"bound": "smem", "avg_launch_ms": sp}
            if (n, m) == PROFILED["workload"] and sm_mhz:
                ach = wf / (sp * 1e-3)
                pk = 148 * sm_mhz * 1e6
                e.update({"achieved": ach, "peak": pk, "unit": "wavefronts/s",
                          "frac": ach / pk, "wavefronts_per_launch": wf,
                          "note": "shared-memory atomic wavefronts (ncu count, profiles/); "
                                  "peak one wavefront per SM per clock at the sampled clock"})
        h = pts_bytes + cells * 8
        e["hbm_view"] = {"algorithmic_bytes": h,
                         "achieved_gbs": h / (sp * 1e-3) / 1e9,
                         "frac": h / (sp * 1e-3) / 1e9 / hbm}
        out["k_spread_tc" if spreader == "tc" else "k_spread"] = e
    for key, nb in (("nu2u (planned)/FFT rows (k_fft_rows)", (cells + kept) * 8),
                    ("nu2u (planned)/FFT columns A (k_fft_colstep)", 2 * kept * 8),
                    ("nu2u (planned)/FFT columns B, correction + crop (k_fft_colstep)",
                     (kept + N0 * N1) * 8),
                    ("u2nu (planned)/FFT columns A, correction + pad (k_fft_colstep)",
                     (N0 * N1 + kept) * 8),
                    ("u2nu (planned)/FFT columns B (k_fft_colstep)", 2 * kept * 8),
                    ("u2nu (planned)/FFT rows, kept columns in (k_fft_rows)",
                     (kept + cells) * 8)):
        e = hbm_entry(key, nb)
        if e:
            out[key] = e
    ip = stages.get("u2nu (planned)/interpolation")
    if ip:
        h = pts_bytes + cells * 8
        e = {"bound": "smem", "avg_launch_ms": ip,
             "hbm_view": {"algorithmic_bytes": h, "achieved_gbs": h / (ip * 1e-3) / 1e9,
                          "frac": h / (ip * 1e-3) / 1e9 / hbm}}
        if (n, m) == PROFILED["workload"] and sm_mhz:
            wf = PROFILED["smem_wavefronts"]["interp"]
            pk = 148 * sm_mhz * 1e6
            e.update({"achieved": wf / (ip * 1e-3), "peak": pk, "unit": "wavefronts/s",
                      "frac": wf / (ip * 1e-3) / pk, "wavefronts_per_launch": wf,
                      "note": "shared-memory load wavefronts (ncu count, profiles/); peak "
                              "one wavefront per SM per clock at the sampled clock"})
        out["k_interp"] = e
    return out


def run_ours(args, rank, world, local_rank):
    import torch
    from ducc_b200 import nufft
    from ducc_b200 import _capi as C

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = world > 1
    if dist:
        import torch.distributed as td
    m, n = args.m, args.n
    coord, vals, grid = make_inputs(1234 + rank, m, n)
    err_idx = np.sort(np.random.default_rng(99).choice(m, min(ERR_SUBSET, m), replace=False))
    d_err_idx = torch.from_numpy(err_idx.astype(np.int64)).to(dev)
    d_coord = torch.from_numpy(coord).to(dev)
    d_vals = torch.from_numpy(vals).to(dev)
    d_grid = torch.from_numpy(grid).to(dev)
    d_out_grid = torch.empty((n, n), dtype=torch.complex64, device=dev)
    d_out_pts = torch.empty(m, dtype=torch.complex64, device=dev)
    stream = torch.cuda.current_stream(dev)

    def barrier():
        if dist:
            td.barrier()
        torch.cuda.synchronize(dev)

    results, kept = {}, {}
    # the arms: each spreader at the requested epsilon, and the plain spreader
    # at a looser epsilon whose error is not below the tensor-core spreader's
    # at the requested one (the comparison at equal or lower error)
    arms = [(sp, sp, EPS) for sp in args.spreaders]
    if args.matched_eps > 0 and "tc" in args.spreaders:
        arms.append(("plain_matched", "plain", args.matched_eps))
    for spreader, kind, eps in arms:
        t0 = time.perf_counter()
        plan = nufft.plan(nu2u=True, coord=d_coord, grid_shape=(n, n), epsilon=eps,
                          nthreads=args.param_threads, spreader=kind)
        torch.cuda.synchronize(dev)
        plan_s = time.perf_counter() - t0

        def step():
            plan.nu2u(points=d_vals, forward=True, out=d_out_grid)
            plan.u2nu(grid=d_grid, forward=False, out=d_out_pts)

        for _ in range(args.warmup):
            step()
        barrier()
        clk = ClockSampler(local_rank)
        clk.start()
        time.sleep(0.3)
        C.lib().dnufft_profile_enable(1)
        l0 = C.lib().dnufft_kernel_launches()
        barrier()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        barrier()
        launches = C.lib().dnufft_kernel_launches() - l0
        prof = json.loads(C.lib().dnufft_profile_json().decode())
        C.lib().dnufft_profile_enable(0)
        clocks = clk.stop()
        ms = max_over_ranks(ev0.elapsed_time(ev1) / args.steps, dev, dist)
        results[spreader] = {"ms": ms, "plan_s": plan_s, "prof": prof, "clocks": clocks,
                             "launches": launches, "info": plan.info()}
        # this arm's outputs of the last timed step, for the error report
        kept[spreader] = (d_out_grid.cpu().numpy(), d_out_pts[d_err_idx].cpu().numpy())
        del plan

    head = args.spreaders[0]
    e2e = e2e_unplanned = e2e_concurrent = None
    if not args.no_e2e:
        h_coord = torch.from_numpy(coord).pin_memory().numpy()
        h_vals = torch.from_numpy(vals).pin_memory().numpy()
        h_grid = torch.from_numpy(grid).pin_memory().numpy()
        h_out = torch.empty((n, n), dtype=torch.complex64).pin_memory().numpy()
        h_pts = torch.empty(m, dtype=torch.complex64).pin_memory().numpy()
        k = max(1, min(args.steps, 5))

        # the same planned step through the public API on pinned host arrays:
        # every step copies its values / uniform grid in and its results out
        hplan = nufft.plan(nu2u=True, coord=h_coord, grid_shape=(n, n), epsilon=EPS,
                           nthreads=args.param_threads, spreader=head)

        def e2e_step():
            hplan.nu2u(points=h_vals, forward=True, out=h_out)
            hplan.u2nu(grid=h_grid, forward=False, out=h_pts)

        e2e_step()
        barrier()
        t0 = time.perf_counter()
        for _ in range(k):
            e2e_step()
        barrier()
        et = max_over_ranks((time.perf_counter() - t0) / k, dev, dist)
        e2e = {"value": world * 2 * m / et / 1e6, "unit": "Mpts/s",
               "h2d_bytes_per_step": int(vals.nbytes + grid.nbytes),
               "d2h_bytes_per_step": int(n * n * 8 + m * 8),
               "call": "ducc_b200.nufft.plan(coord on the host).nu2u + .u2nu on pinned host "
                       "numpy arrays (plan built before the timed region)",
               "ms_per_step": et * 1e3}

        # the step's two transforms are independent (u2nu reads its own grid):
        # a caller with both can issue them from two host threads on two
        # streams with a plan each, so that the uploads of one overlap the
        # downloads of the other (PCIe is full duplex)
        hplan2 = nufft.plan(nu2u=False, coord=h_coord, grid_shape=(n, n), epsilon=EPS,
                            nthreads=args.param_threads, spreader=head)
        s1, s2 = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
        errs = []

        def type2_call():
            try:
                hplan2.u2nu(grid=h_grid, forward=False, out=h_pts, stream=s2.cuda_stream)
            except Exception as e:   # re-raised on the main thread
                errs.append(e)

        def e2e_concurrent_step():
            th = threading.Thread(target=type2_call)
            th.start()
            hplan.nu2u(points=h_vals, forward=True, out=h_out, stream=s1.cuda_stream)
            th.join()
            if errs:
                raise errs[0]

        e2e_concurrent_step()
        barrier()
        t0 = time.perf_counter()
        for _ in range(k):
            e2e_concurrent_step()
        barrier()
        et = max_over_ranks((time.perf_counter() - t0) / k, dev, dist)
        del hplan, hplan2
        e2e_concurrent = {"value": world * 2 * m / et / 1e6, "unit": "Mpts/s",
                          "h2d_bytes_per_step": int(vals.nbytes + grid.nbytes),
                          "d2h_bytes_per_step": int(n * n * 8 + m * 8),
                          "call": "the same two planned calls on pinned host numpy arrays, "
                                  "issued from two host threads on two streams (one plan "
                                  "each)", "ms_per_step": et * 1e3}

        # unplanned functions (each call uploads and sorts the coordinates)
        def e2e_unplanned_step():
            nufft.nu2u(points=h_vals, coord=h_coord, forward=True, epsilon=EPS,
                       nthreads=args.param_threads, out=h_out)
            nufft.u2nu(grid=h_grid, coord=h_coord, forward=False, epsilon=EPS,
                       nthreads=args.param_threads, out=h_pts)

        e2e_unplanned_step()
        barrier()
        t0 = time.perf_counter()
        for _ in range(k):
            e2e_unplanned_step()
        barrier()
        et = max_over_ranks((time.perf_counter() - t0) / k, dev, dist)
        e2e_unplanned = {"value": world * 2 * m / et / 1e6, "unit": "Mpts/s",
                         "h2d_bytes_per_step": int(2 * coord.nbytes + vals.nbytes + grid.nbytes),
                         "d2h_bytes_per_step": int(n * n * 8 + m * 8),
                         "call": "ducc_b200.nufft.nu2u + u2nu (unplanned) on pinned host "
                                 "numpy arrays", "ms_per_step": et * 1e3}

    if rank != 0:
        return
    hbm, bf16, src = peaks()
    r = results[head]
    ms = r["ms"]
    stages = _stage_ms(r["prof"])
    sm_mhz = r["clocks"].get("sm_mhz")
    recs = r["info"].get("tc_records", 0)
    rl = kernel_rooflines(stages, head, r["info"], m, n, recs, hbm, bf16, sm_mhz, src)
    for other in args.spreaders[1:]:
        o = results[other]
        rl.update({k: v for k, v in kernel_rooflines(
            _stage_ms(o["prof"]), other, o["info"], m, n, o["info"].get("tc_records", 0),
            hbm, bf16, o["clocks"].get("sm_mhz"), src).items() if k.startswith("k_spread")})
    # the headline roofline: the dominant kernel, the spreader of the head arm
    sp_key = "k_spread_tc" if head == "tc" else "k_spread"
    spr = rl.get(sp_key, {})
    roofline = {k: spr.get(k) for k in ("bound", "achieved", "peak", "unit", "frac")}
    roofline.update({"kernel": sp_key, "avg_launch_ms": spr.get("avg_launch_ms"),
                     "peak_source": src, "hbm_view": spr.get("hbm_view")})
    # DRAM bytes of one launch from ncu (PROFILED), only for the profiled workload
    roofline["traffic"] = (PROFILED["spread_dram_bytes"].get(head)
                           if (n, m) == PROFILED["workload"] else None)
    roofline["traffic_source"] = "profiles/launches_bench_4096sq_M5e7.md"

    cpu, ducc_out = (None, None) if args.no_cpu else cpu_baseline_leg(args, coord, vals, grid)
    errors = None if args.no_errors else error_report(args, coord, vals, grid, err_idx, kept,
                                                      ducc_out)
    workloads = None
    if not args.no_extra and world == 1:
        del d_coord, d_vals, d_grid, d_out_grid, d_out_pts
        torch.cuda.empty_cache()
        workloads = {}
        for name, fn in (("batched_uneven_2d", workload_batched),
                         ("radial_autograd_2d", workload_autograd),
                         ("type2_3d_256", workload_3d),
                         ("wgridder", workload_wgridder),
                         ("sphere_synthesis", lambda d: workload_sphere(d, with_outputs=True))):
            try:
                workloads[name] = fn(dev)
            except Exception as e:   # reported, never fatal for the headline line
                workloads[name] = {"error": str(e)[:200]}
        if not args.no_cpu and "error" not in workloads["wgridder"]:
            try:
                workloads["wgridder"]["cpu_baseline"] = cpu_baseline_wgridder(args.param_threads)
            except Exception as e:
                workloads["wgridder"]["cpu_baseline"] = {"error": str(e)[:200]}
        sph = workloads["sphere_synthesis"]
        om, oa, s2 = sph.pop("_map", None), sph.pop("_alm", None), sph.pop("_spin2", None)
        if not args.no_cpu and "error" not in sph:
            try:
                sph["cpu_baseline"] = cpu_baseline_sphere(args.param_threads, om, oa, s2)
            except Exception as e:
                sph["cpu_baseline"] = {"error": str(e)[:200]}
    line = {
        "metric": METRIC,
        "value": world * 2 * m / (ms * 1e-3) / 1e6,
        "unit": "Mpts/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c64 (f32 arithmetic)", "data": "synthetic",
        "config": bench_config(args),
        "parallelism": "replicas" if world > 1 else "1 GPU",
        "spreader": head, "kernel_support": r["info"]["supp"], "oversampled": r["info"]["nover"],
        "roofline": roofline,
        "kernels": rl,
        "stages_ms": stages,
        "plan_create_s": r["plan_s"],
        "clocks": r["clocks"],
        "gpu_launches": int(r["launches"]),
        "e2e": e2e,
        "e2e_unplanned": e2e_unplanned,
        "e2e_concurrent": e2e_concurrent,
        "cpu_baseline": cpu,
        "errors": errors,
        "workloads": workloads,
    }
    for other in [k for k in results if k != head]:
        o = results[other]
        line["alt_" + other] = {"value": world * 2 * m / (o["ms"] * 1e-3) / 1e6,
                                "ms_per_step": o["ms"], "stages_ms": _stage_ms(o["prof"]),
                                "clocks": o["clocks"]}
        if other == "plain_matched":
            line["alt_" + other]["eps"] = args.matched_eps
            line["alt_" + other]["kernel_support"] = o["info"]["supp"]
            line["alt_" + other]["oversampled"] = o["info"]["nover"]
    print(json.dumps(line))


def run_sharded(args, rank, world, local_rank):
    """One transform split over the ranks (strong scaling): every rank holds
    1/world of the bench workload's points, ShardedPlan with the row-slab
    partition (2D) does the type 1 and type 2 of all of them."""
    import torch
    import torch.distributed as td
    from ducc_b200 import distributed as D

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    m, n = args.m, args.n
    coord, vals, grid = make_inputs(1234, m, n)
    a, b = m * rank // world, m * (rank + 1) // world
    d_coord = torch.from_numpy(coord[a:b]).to(dev)
    d_vals = torch.from_numpy(vals[a:b]).to(dev)
    d_grid = torch.from_numpy(grid).to(dev)
    del coord, vals, grid
    t0 = time.perf_counter()
    sp = D.ShardedPlan(nu2u=True, coord=d_coord, grid_shape=(n, n), epsilon=EPS,
                       nthreads=args.param_threads, spreader=args.spreaders[0],
                       partition="rows")
    torch.cuda.synchronize(dev)
    plan_s = time.perf_counter() - t0
    out = torch.empty((n, n), dtype=torch.complex64, device=dev)

    def step():
        sp.nu2u(forward=True, points=d_vals, out=out)
        sp.u2nu(forward=False, grid=d_grid)

    for _ in range(args.warmup):
        step()
    td.barrier()
    torch.cuda.synchronize(dev)
    clk = ClockSampler(local_rank)
    clk.start()
    time.sleep(0.3)
    stream = torch.cuda.current_stream(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    td.barrier()
    torch.cuda.synchronize(dev)
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    td.barrier()
    torch.cuda.synchronize(dev)
    clocks = clk.stop()
    ms = max_over_ranks(ev0.elapsed_time(ev1) / args.steps, dev, True)
    if rank != 0:
        return
    cfg = bench_config(args)
    cfg["parallelism"] = "one transform over %d GPUs: row-slab partition" % world
    print(json.dumps({
        "metric": METRIC, "value": 2 * m / (ms * 1e-3) / 1e6, "unit": "Mpts/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "c64 (f32 arithmetic)", "data": "synthetic", "config": cfg,
        "partition": sp.partition, "plan_create_s": plan_s, "clocks": clocks,
        "step": "ShardedPlan.nu2u (all points, result on every rank) + ShardedPlan.u2nu"}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--m", type=int, default=M_POINTS)
    ap.add_argument("--n", type=int, default=N_SIDE)
    ap.add_argument("--spreaders", default="tc,plain")
    ap.add_argument("--param-threads", type=int, default=os.cpu_count(),
                    help="nthreads fed to DUCC's parameter cost model in both arms (and the "
                         "reference arm's thread count)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-errors", action="store_true",
                    help="skip the FP64 error report (DUCC on the host)")
    ap.add_argument("--matched-eps", type=float, default=3e-6,
                    help="also time the plain spreader at this epsilon (its error at the bench "
                         "workload is not below the tensor-core spreader's at 1e-6); 0: skip")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the batched / autograd / 3D workloads")
    ap.add_argument("--sharded", action="store_true",
                    help="one transform split over the ranks (strong scaling) instead of one "
                         "independent transform per rank")
    ap.add_argument("--workload", default=None,
                    choices=["batched_uneven_2d", "radial_autograd_2d", "type2_3d_256",
                             "wgridder", "sphere_synthesis"],
                    help="run one of the extra workloads alone and print its result (for "
                         "profiling); the w-gridder one takes --wg-rows / --wg-npix")
    ap.add_argument("--wg-rows", type=int, default=WG_NROW)
    ap.add_argument("--wg-npix", type=int, default=WG_NPIX)
    ap.add_argument("--sh-lmax", type=int, default=SH_LMAX)
    ap.add_argument("--sh-npts", type=int, default=SH_NPTS)
    args = ap.parse_args()
    args.spreaders = args.spreaders.split(",")
    if args.workload:
        import torch
        dev = torch.device("cuda", 0)
        fn = {"batched_uneven_2d": workload_batched, "radial_autograd_2d": workload_autograd,
              "type2_3d_256": workload_3d}.get(args.workload)
        if args.workload == "sphere_synthesis":
            res = workload_sphere(dev, lmax=args.sh_lmax, npts=args.sh_npts,
                                  with_outputs=not args.no_cpu)
            om, oa, s2 = res.pop("_map", None), res.pop("_alm", None), res.pop("_spin2", None)
            if (not args.no_cpu and args.sh_lmax == SH_LMAX and args.sh_npts == SH_NPTS):
                res["cpu_baseline"] = cpu_baseline_sphere(args.param_threads, om, oa, s2)
        else:
            res = (fn(dev) if fn else
                   workload_wgridder(dev, nrow=args.wg_rows, npix=args.wg_npix))
        print(json.dumps({"workload": args.workload, **res}))
        return
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if world > 1 or args.sharded:
        import datetime
        import torch
        import torch.distributed as td
        torch.cuda.set_device(local_rank)
        if world == 1:
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            os.environ.setdefault("MASTER_PORT", "29531")
            os.environ.setdefault("RANK", "0")
            os.environ.setdefault("WORLD_SIZE", "1")
        # what the communicator set-up prints (NCCL's version line) goes to
        # stderr, so that stdout carries the one JSON line only
        sys.stdout.flush()
        saved = os.dup(1)
        os.dup2(2, 1)
        try:
            td.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                  device_id=torch.device("cuda", local_rank))
            td.barrier()
        finally:
            sys.stdout.flush()
            os.dup2(saved, 1)
            os.close(saved)
    try:
        if args.sharded:
            run_sharded(args, rank, world, local_rank)
        else:
            run_ours(args, rank, world, local_rank)
    finally:
        if world > 1 or args.sharded:
            import torch.distributed as td
            td.destroy_process_group()


if __name__ == "__main__":
    main()
