"""Benchmark: 2D NUFFT at eps=1e-6 on a B200 (type 1 then type 2).

Workload (one "step"): on a 4096x4096 grid, M=5e7 points drawn from a mixture
of 16 Gaussians (sigma 0.3 rad, centres uniform in [-pi,pi)^2, wrapped),
float32 coordinates, complex64 values N(0,1): a planned nu2u followed by a
planned u2nu with the same plan (DUCC's ``plan.nu2u`` / ``plan.u2nu``).
Throughput = points x transforms / time, in Mpts/s.  The headline line uses
the split-precision tensor-core spreader; the plain FP32 atomic spreader is
timed on the same inputs and reported beside it (``alt_plain``).

Arms
  default            this library on N GPUs (one process per GPU under
                     torchrun; each rank runs its own seeded instance: weak
                     scaling, no collective on the data path)
  --impl reference   DUCC's own CPU NUFFT (built from source into oracle/_ref)
                     on the host cores, rank 0 only

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
METRIC = "NUFFT Mpts/s 2D eps=1e-6: TC split-prec vs plain FP32 spreader, same B200"
KERNEL_NAMES = {"tc": "k_spread_tc (split-precision tensor-core spreader)",
                "plain": "k_spread (plain FP32 atomic spreader)",
                "auto": "k_spread (plain FP32 atomic spreader)"}
# DRAM bytes per spreading launch at the full workload: ncu dram__bytes_read.sum
# + dram__bytes_write.sum (a one-pass metric set) of launches of this bench's
# default command (profiles/launches_bench_4096sq_M5e7.md)
TRAFFIC_PER_LAUNCH = {"tc": 6460321536.0 + 528613120.0,
                      "plain": 6345106944.0 + 451456000.0}


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
    nthr = os.cpu_count()
    out = np.empty((n, n), np.complex64)

    def step():
        R.nufft.nu2u(points=vals, coord=coord, forward=True, epsilon=EPS, nthreads=nthr, out=out)
        R.nufft.u2nu(grid=grid, coord=coord, forward=False, epsilon=EPS, nthreads=nthr)

    plan_t0 = time.perf_counter()
    del plan_t0
    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = (time.perf_counter() - t0) / args.steps
    v = 2 * m / dt / 1e6
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "Mpts/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c64", "data": "synthetic",
        "config": {"workload": "2D type-1 + type-2 NUFFT, 4096x4096 grid, M=5e7 clustered "
                               "points (16 Gaussians, sigma 0.3), f32 coords, c64, eps=1e-6",
                   "grid": [n, n], "npoints": m, "call": "ducc0.nufft.nu2u + u2nu (unplanned)"},
        "cpu_baseline": {"value": v, "unit": "Mpts/s", "cores": nthr, "kind": "reference",
                         "sample": "full workload, %d step(s)" % args.steps},
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


# ---------------------------------------------------------------- our arm
def cpu_baseline_leg(m, n, coord, vals, grid, budget_s=30.0):
    """DUCC's CPU NUFFT on the host cores, bounded to ~budget_s seconds."""
    from oracle import ref
    R = ref.load()
    if R is None:
        return None
    nthr = os.cpu_count()
    out = np.empty((n, n), np.complex64)
    t0 = time.perf_counter()
    R.nufft.nu2u(points=vals, coord=coord, forward=True, epsilon=EPS, nthreads=nthr, out=out)
    R.nufft.u2nu(grid=grid, coord=coord, forward=False, epsilon=EPS, nthreads=nthr)
    first = time.perf_counter() - t0
    reps = max(1, min(3, int(budget_s / max(first, 1e-3)) - 1))
    t0 = time.perf_counter()
    for _ in range(reps):
        R.nufft.nu2u(points=vals, coord=coord, forward=True, epsilon=EPS, nthreads=nthr, out=out)
        R.nufft.u2nu(grid=grid, coord=coord, forward=False, epsilon=EPS, nthreads=nthr)
    dt = (time.perf_counter() - t0) / reps
    return {"value": 2 * m / dt / 1e6, "unit": "Mpts/s", "cores": nthr, "kind": "reference",
            "sample": "the full workload (nu2u + u2nu, unplanned, M=%d), 1 warm-up + %d timed"
                      % (m, reps)}


def max_over_ranks(value, dev, dist):
    """The largest of every rank's value (the job's time is its slowest rank)."""
    if not dist:
        return value
    import torch
    import torch.distributed as td
    t = torch.tensor([float(value)], device=dev)
    td.all_reduce(t, op=td.ReduceOp.MAX)
    return float(t.item())


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

    results = {}
    for spreader in args.spreaders:
        t0 = time.perf_counter()
        plan = nufft.plan(nu2u=True, coord=d_coord, grid_shape=(n, n), epsilon=EPS,
                          nthreads=args.param_threads, spreader=spreader)
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
        del plan

    # end-to-end through the public API with host (pinned) buffers: unplanned
    # nu2u + u2nu, host->device and device->host copies inside the timed region
    e2e = None
    if not args.no_e2e:
        h_coord = torch.from_numpy(coord).pin_memory().numpy()
        h_vals = torch.from_numpy(vals).pin_memory().numpy()
        h_grid = torch.from_numpy(grid).pin_memory().numpy()
        h_out = torch.empty((n, n), dtype=torch.complex64).pin_memory().numpy()
        h_pts = torch.empty(m, dtype=torch.complex64).pin_memory().numpy()

        def e2e_step():
            nufft.nu2u(points=h_vals, coord=h_coord, forward=True, epsilon=EPS,
                       nthreads=args.param_threads, out=h_out)
            nufft.u2nu(grid=h_grid, coord=h_coord, forward=False, epsilon=EPS,
                       nthreads=args.param_threads, out=h_pts)

        e2e_step()
        barrier()
        t0 = time.perf_counter()
        k = max(1, min(args.steps, 5))
        for _ in range(k):
            e2e_step()
        barrier()
        et = max_over_ranks((time.perf_counter() - t0) / k, dev, dist)
        e2e = {"value": world * 2 * m / et / 1e6, "unit": "Mpts/s",
               "h2d_bytes_per_step": int(2 * coord.nbytes + vals.nbytes + grid.nbytes),
               "d2h_bytes_per_step": int(n * n * 8 + m * 8),
               "call": "ducc_b200.nufft.nu2u + u2nu (unplanned) on pinned host numpy arrays",
               "ms_per_step": et * 1e3}

    if rank != 0:
        return
    hbm, bf16, src = peaks()
    head = args.spreaders[0]
    r = results[head]
    ms = r["ms"]
    # dominant kernel: the spreader of the planned type-1 transform
    sp = r["prof"].get("nu2u (planned)/spreading", [0.0, 0])
    ip = r["prof"].get("u2nu (planned)/interpolation", [0.0, 0])
    sp_ms = sp[0] / max(sp[1], 1)
    ip_ms = ip[0] / max(ip[1], 1)
    W = r["info"]["supp"]
    nov = r["info"]["nover"]
    # algorithmic bytes of one spreading launch: sorted coords (8 B) + values
    # (8 B) + permutation (4 B) per point, plus one write of the oversampled grid
    spread_bytes = m * (8 + 8 + 4) + nov[0] * nov[1] * 8
    achieved = spread_bytes / (sp_ms * 1e-3) / 1e9 if sp_ms > 0 else None
    # DRAM bytes of one spreading launch from ncu (dram__bytes_read.sum +
    # dram__bytes_write.sum), measured on the same kernel at a quarter of the
    # workload (2048^2 grid, 1.25e7 points: same points per tile) and scaled
    # by 4, since points and grid cells both scale by 4 (profiles/)
    traffic = TRAFFIC_PER_LAUNCH.get(head)
    # tensor pipe: each K-block record is at most one 128x48x16 MMA
    recs = r["info"].get("tc_records", 0)
    tc_flops = recs * 2 * 128 * 48 * 16
    cpu = None if args.no_cpu else cpu_baseline_leg(m, n, coord, vals, grid)
    workloads = None
    if not args.no_extra and world == 1:
        del d_coord, d_vals, d_grid, d_out_grid, d_out_pts
        torch.cuda.empty_cache()
        workloads = {}
        for name, fn in (("batched_uneven_2d", workload_batched),
                         ("radial_autograd_2d", workload_autograd),
                         ("type2_3d_256", workload_3d)):
            try:
                workloads[name] = fn(dev)
            except Exception as e:   # reported, never fatal for the headline line
                workloads[name] = {"error": str(e)[:200]}
    line = {
        "metric": METRIC,
        "value": world * 2 * m / (ms * 1e-3) / 1e6,
        "unit": "Mpts/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c64 (f32 arithmetic)", "data": "synthetic",
        "config": {"workload": "2D type-1 + type-2 NUFFT, 4096x4096 grid, M=5e7 clustered "
                               "points (16 Gaussians, sigma 0.3), f32 coords, c64, eps=1e-6",
                   "grid": [n, n], "npoints": m, "eps": EPS, "spreader": head,
                   "kernel_support": W, "oversampled": nov,
                   "step": "plan.nu2u + plan.u2nu, inputs resident in HBM",
                   "l2": "inputs and oversampled grid larger than L2 (no flush needed)",
                   "parallelism": "replicas" if world > 1 else "1 GPU"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": (achieved / hbm) if achieved else None, "traffic": traffic,
                     "kernel": KERNEL_NAMES[head], "peak_source": src,
                     "algorithmic_bytes_per_launch": spread_bytes,
                     "avg_launch_ms": sp_ms,
                     "tensor": None if not recs else {
                         "executed_tflops": tc_flops / (sp_ms * 1e-3) / 1e12,
                         "peak_tflops": bf16, "frac": tc_flops / (sp_ms * 1e-3) / 1e12 / bf16,
                         "mma_per_launch": recs}},
        "stages_ms": {k: v[0] / max(v[1], 1) for k, v in r["prof"].items()},
        "plan_create_s": r["plan_s"],
        "interp_avg_ms": ip_ms,
        "clocks": r["clocks"],
        "gpu_launches": int(r["launches"]),
        "e2e": e2e,
        "cpu_baseline": cpu,
        "workloads": workloads,
    }
    for other in args.spreaders[1:]:
        o = results[other]
        line["alt_" + other] = {"value": world * 2 * m / (o["ms"] * 1e-3) / 1e6,
                                "ms_per_step": o["ms"],
                                "stages_ms": {k: v[0] / max(v[1], 1) for k, v in o["prof"].items()}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--m", type=int, default=M_POINTS)
    ap.add_argument("--n", type=int, default=N_SIDE)
    ap.add_argument("--spreaders", default="tc,plain")
    ap.add_argument("--param-threads", type=int, default=8,
                    help="nthreads fed to DUCC's parameter cost model (fixes W / sigma)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the batched / autograd / 3D workloads")
    args = ap.parse_args()
    args.spreaders = args.spreaders.split(",")
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as td
        torch.cuda.set_device(local_rank)
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as td
            td.destroy_process_group()


if __name__ == "__main__":
    main()
