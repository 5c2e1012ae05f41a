#!/usr/bin/env python
"""Benchmark of the B200-native TOP3D_XL engine: OC iterations per second.

Workload (default): GLOBAL compliance minimisation on a 128x256x128 cuboid with
the reference's built-in BCs (4,194,304 hex elements, 12.8M DOFs), V0=0.12,
rMin=sqrt(3) -- TOP3D_XL(true(128,256,128),'GLOBAL',0.12,50,sqrt(3)).  One
"step" is one optimisation iteration (SIMP, coarse-operator assembly + coarse
factorisation, multigrid PCG, compliance, PDE sensitivity filter, OC update),
with all state resident in HBM.

`value` is the FP64 engine (the reference's own precision).  The mixed-precision
engine (FP64 Krylov iteration, operator and filter, FP32 multigrid preconditioner)
is measured beside it, with its per-iteration relative compliance
error against FP64.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl native|reference]

Multi-GPU: the path does not shard (one design job per GPU); N ranks run N
independent replicas and `value` is their total throughput.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "cuboid128": dict(shape=(128, 256, 128), cons="GLOBAL", V0=0.12, rMin=math.sqrt(3), rHat=0.0, nLoop=50),
    "cuboid50": dict(shape=(50, 100, 50), cons="GLOBAL", V0=0.12, rMin=math.sqrt(3), rHat=0.0, nLoop=50),
    "cuboid50_local": dict(shape=(50, 100, 50), cons="LOCAL", V0=0.5, rMin=math.sqrt(3), rHat=6.0, nLoop=300),
    "cuboid25": dict(shape=(25, 50, 25), cons="GLOBAL", V0=0.12, rMin=math.sqrt(3), rHat=0.0, nLoop=50),
    # generated irregular domain (top3d_xl_b200/workloads.py, seed 8) read from a .TopVoxel file
    "irregular4": dict(topvoxel="IRREGULAR_FULL", cons="LOCAL", V0=0.5, rMin=math.sqrt(3), rHat=6.0, nLoop=300),
}
_TOPVOXEL = {}


def workload_source(wl):
    """A voxel array (cuboids) or the path of the generated .TopVoxel file (written once)."""
    if "topvoxel" not in wl:
        return np.ones(wl["shape"], bool)
    key = wl["topvoxel"]
    if key not in _TOPVOXEL:
        import tempfile

        from top3d_xl_b200 import workloads as W
        path = os.path.join(tempfile.mkdtemp(prefix="topx_"), key + ".TopVoxel")
        W.write_topvoxel(path, *W.irregular_domain(**getattr(W, key)))
        _TOPVOXEL[key] = path
    return _TOPVOXEL[key]


def load_workload(ctx, wl):
    src = workload_source(wl)
    if isinstance(src, str):
        ctx.load_topvoxel(src)
    else:
        ctx.load_voxels(src)
METRIC = "OC iterations/s (GLOBAL, FP64; mixed precision beside it)"
# DRAM bytes (read + write) per grid node of one K*u launch in PCG mode (tile kernel + last-row
# kernel), from an ncu capture of the 128x256x128 cuboid: dram__bytes_read.sum +
# dram__bytes_write.sum of the tile kernel (637.2 MB) and the last-row kernel (52.9 MB) over
# 4,276,737 nodes; the traffic of a launch scales with its node count.
KU_TRAFFIC_PER_NODE = 690.1e6 / 4276737
# Nominal FP64 rate of a B200 on CUDA cores: 148 SMs x 64 FMA/clk x 2 flop x 1.965 GHz.
FP64_NOMINAL_TFLOPS = 148 * 64 * 2 * 1.965e9 / 1e12


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks, utilisation and throttle reasons.  As a context manager it
    samples the enclosed block; run_native starts and stops it around the warm-up and timed
    iterations only.  sm_mhz is the median over the samples taken while a kernel was running
    (utilisation >= 50 %), so idle host-side gaps do not read as low clocks."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,utilization.gpu")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines += [l for l in out.splitlines() if l.strip()]
            self.proc = None

    def __enter__(self):
        self.start()
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        self.stop()

    def summary(self):
        sm, busy, mx, reasons = [], [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 10:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
                if float(f[9]) >= 50:
                    busy.append(float(f[1]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(busy or sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "samples_under_load": len(busy)}


def run_native(wl, precision, steps, warmup, device, profile_steps=0, keep=False, clk=None):
    """Run `warmup` then `steps` timed OC iterations (device time via CUDA events on the
    engine stream); then, if asked, `profile_steps` more iterations with per-section
    event timing (direct launches instead of CUDA graphs, outside the timed region).
    `clk` (a Clocks) samples the warm-up and timed iterations."""
    from top3d_xl_b200 import Context
    ctx = Context(precision, device=device)
    load_workload(ctx, wl)
    ctx.begin(wl["cons"], wl["V0"], wl["nLoop"], wl["rMin"], wl["rHat"])
    hist = []
    if clk:
        clk.start()
    for _ in range(warmup):
        hist.append(ctx.step())
    launches0 = ctx.launch_count()
    ctx.timer_start()
    t0 = time.perf_counter()
    for _ in range(steps):
        hist.append(ctx.step())
    ms = ctx.timer_stop()
    wall = time.perf_counter() - t0
    if clk:
        clk.stop()
    launches = ctx.launch_count() - launches0
    prof = None
    if profile_steps:
        ctx.set_profiling(True)
        for _ in range(profile_steps):
            if ctx.step() is None:
                break
        prof = ctx.profile()
        prof["steps"] = profile_steps
        ctx.set_profiling(False)
    out = dict(ms=ms, wall=wall, hist=hist, prof=prof, launches=launches, launches_before=launches0, ne=ctx.numElements, ndof=ctx.numDOFs,
               nnodes=int(ctx.info.numNodes))
    if keep:
        out["ctx"] = ctx
    else:
        ctx.close()
    return out


def run_e2e(wl, precision, steps, warmup, device):
    """Same metric through the public API with host buffers: per step the host density
    (page-locked host memory) goes to the device, one iteration runs, and the new density
    comes back into the same host buffer."""
    import torch
    from top3d_xl_b200 import Context
    ctx = Context(precision, device=device)
    load_workload(ctx, wl)
    ctx.begin(wl["cons"], wl["V0"], wl["nLoop"], wl["rMin"], wl["rHat"])
    x = torch.empty(ctx.numElements, dtype=torch.float64, pin_memory=True).numpy()
    ctx.density(out=x)
    for _ in range(warmup):
        ctx.set_density(x)
        ctx.step()
        ctx.density(out=x)
    t0 = time.perf_counter()
    for _ in range(steps):
        ctx.set_density(x)
        ctx.step()
        ctx.density(out=x)
    wall = time.perf_counter() - t0
    ne = ctx.numElements
    ctx.close()
    return dict(value=steps / wall, h2d=8 * ne, d2h=8 * ne)


def profile_one_step(wl, precision, device, coop=True):
    """One warm-up OC iteration, then one OC iteration bracketed by cudaProfilerStart/Stop, so that
    `ncu --profile-from-start off` captures exactly the kernels of one iteration."""
    import ctypes
    from top3d_xl_b200 import Context
    rt = ctypes.CDLL("libcudart.so")
    with Context(precision, device=device, **({} if coop else dict(coarse_coop=0))) as ctx:
        load_workload(ctx, wl)
        ctx.begin(wl["cons"], wl["V0"], wl["nLoop"], wl["rMin"], wl["rHat"])
        ctx.step()
        rt.cudaDeviceSynchronize()
        rt.cudaProfilerStart()
        r = ctx.step()
        rt.cudaDeviceSynchronize()
        rt.cudaProfilerStop()
    print(json.dumps({"profiled_step": r["loop"], "pcg_its": r["its"], "c": r["c"]}), flush=True)
    return 0


def cpu_sample(wl, its_per_oc, filter_its_per_oc, budget_s=30.0):
    """Time the FP64 oracle (CPU restatement of TOP3D_XL.m) on a bounded sample of the
    workload and extrapolate one OC iteration from the GPU's measured iteration counts."""
    import threadpoolctl  # noqa: F401
    from oracle import top3dxl_oracle as O
    cores = os.cpu_count() or 1
    m = O.build_model(workload_source(wl))
    sol = O.Solver(m)
    Ne = m.levels[0].numElements
    S = m.S
    E = S.modulusMin + wl["V0"] ** S.SIMPpenalty * (S.modulus - S.modulusMin) * np.ones(Ne)
    t = time.perf_counter()
    sol.assemble(E)
    t_asm = time.perf_counter() - t
    u = np.random.default_rng(0).standard_normal(m.levels[0].numDOFs)
    t = time.perf_counter()
    y = sol.ku(u)
    z = sol.vcycle(y)
    _ = (z @ y, np.linalg.norm(y))
    t_it = time.perf_counter() - t
    flt = O.PDEFilter(m, wl["rMin"], S)
    un = np.random.default_rng(1).standard_normal(m.levels[0].numNodes)
    t = time.perf_counter()
    flt.matvec(un)
    t_fit = time.perf_counter() - t
    U = u.reshape(-1, 1)
    t = time.perf_counter()
    ce = O.unit_compliance(m, U)
    t_ce = time.perf_counter() - t
    # one OC update (the full bisection, ~60 passes over the elements) on the same element count
    x = np.full(Ne, wl["V0"])
    dc = -np.abs(ce) - 1e-9
    t = time.perf_counter()
    O.oc_update(x, dc, np.ones(Ne), 0.0, np.zeros(0, np.int64))
    t_ocu = time.perf_counter() - t
    t_oc = t_asm + its_per_oc * t_it + filter_its_per_oc * t_fit + t_ce + t_ocu
    what = ("%dx%dx%d cuboid" % wl["shape"]) if "shape" in wl else ("generated %s domain" % wl["topvoxel"])
    sample = ("bounded sample, extrapolated: oracle FP64 (numpy/scipy, BLAS on all cores, elementwise passes "
              "on one) on the same %s: 1 stencil assembly (%.1fs), 1 PCG iteration (K*u + V-cycle, %.2fs), "
              "1 filter matvec (%.2fs), 1 compliance (%.2fs), 1 OC bisection (%.2fs); OC iteration = assembly + "
              "%.1f PCG its + %.1f filter its + compliance + OC (counts measured in the GPU run)"
              % (what, t_asm, t_it, t_fit, t_ce, t_ocu, its_per_oc, filter_its_per_oc))
    return dict(value=1.0 / t_oc, unit="OC iterations/s", cores=cores, kind="port", sample=sample,
                sec_per_oc=t_oc)


def cpu_whole_iterations(wl, max_steps, budget_s):
    """Time whole OC iterations of the FP64 oracle (the CPU restatement of TOP3D_XL.m, BLAS on all
    host cores) on the workload itself.  Model set-up and the solid solve (cSolid) run untimed;
    then iterations run until `max_steps` are done or `budget_s` is spent (at least one), and
    every one of them is timed whole: assembly, PCG to tol 1e-3, compliance, filter, OC."""
    from oracle import top3dxl_oracle as O
    marks = []

    def hook(loop):
        marks.append(time.perf_counter())
        n = len(marks) - 1
        return n >= max_steps or (n >= 1 and marks[-1] - marks[0] >= budget_s)
    t0 = time.perf_counter()
    src = workload_source(wl)
    if wl["cons"] == "GLOBAL":
        h = O.run_global(src, wl["V0"], wl["nLoop"], wl["rMin"], hook=hook)
    else:
        h = O.run_local(src, wl["V0"], wl["nLoop"], wl["rMin"], wl["rHat"], hook=hook)
    n = len(marks) - 1
    secs = marks[-1] - marks[0]
    nlc = max(1, len(h["its"]) // max(1, n))
    return dict(value=n / secs, steps=n, seconds=secs, setup_s=marks[0] - t0, its=[int(k) for k in h["its"]],
                load_cases=nlc, cores=os.cpu_count() or 1)


def serve_stream(n_jobs, seed=5, mean_gap=0.05):
    """The served workload: n_jobs solid cuboids with Poisson arrivals (mean gap 50 ms),
    dimensions (16, 32, 16) x s with one common scale s log-uniform in [1, 6] (rounded), 70 %
    GLOBAL (V0 uniform 0.08-0.2, 50 iterations) and 30 % LOCAL (V0 0.5, 100 iterations, local
    radius 6), rMin sqrt(3).  Seeded numpy.random.default_rng."""
    rng = np.random.default_rng(seed)
    jobs, t = [], 0.0
    for _ in range(n_jobs):
        t += rng.exponential(mean_gap)
        s = math.exp(rng.uniform(0.0, math.log(6.0)))
        shape = (max(3, round(16 * s)), max(3, round(32 * s)), max(3, round(16 * s)))
        if rng.uniform() < 0.7:
            jobs.append(dict(at=t, shape=shape, cons="GLOBAL", V0=float(rng.uniform(0.08, 0.2)), nLoop=50, rHat=0.0))
        else:
            jobs.append(dict(at=t, shape=shape, cons="LOCAL", V0=0.5, nLoop=100, rHat=6.0))
    return jobs


def run_served(jobs, precision, slots, device):
    """Submit `jobs` to a Server on their arrival schedule and wait for all; per-job latency is
    completion minus submission on the server clock."""
    from top3d_xl_b200 import Server
    with Server(slots=slots, precision=precision, device=device) as srv:
        t0 = time.perf_counter()
        ids = []
        for j in jobs:
            delay = j["at"] - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            ids.append(srv.submit(j["shape"], j["cons"], j["V0"], j["nLoop"], math.sqrt(3), j["rHat"]))
        res = [srv.wait(i) for i in ids]
        stats = srv.stats()
        err = srv.last_error()
    ok = [r for r in res if r["status"] == 0]
    lat = np.array([r["t_end"] - r["t_submit"] for r in ok])
    span = max(r["t_end"] for r in res) - min(r["t_submit"] for r in res)
    its = sum(r["loops"] for r in ok)
    return dict(jobs=len(jobs), ok=len(ok), failed=len(res) - len(ok), error=err if len(ok) < len(res) else "",
                p50_s=float(np.percentile(lat, 50)) if len(lat) else None,
                p99_s=float(np.percentile(lat, 99)) if len(lat) else None,
                oc_its=its, span_s=span, oc_its_per_s=its / span if span > 0 else None,
                max_running=stats["max_running"], peak_bytes=stats["peak_bytes"])


def run_sequential(jobs, precision, device):
    """The same jobs one after another (one slot): busy time per job and OC iterations/s."""
    from top3d_xl_b200 import Server
    with Server(slots=1, precision=precision, device=device) as srv:
        res = [srv.wait(srv.submit(j["shape"], j["cons"], j["V0"], j["nLoop"], math.sqrt(3), j["rHat"])) for j in jobs]
    busy = sum(r["t_end"] - r["t_submit"] for r in res)
    its = sum(r["loops"] for r in res if r["status"] == 0)
    return dict(jobs=len(jobs), oc_its=its, busy_s=busy, oc_its_per_s=its / busy if busy > 0 else None)


def max_over_ranks(ms_local, dist, torch, device):
    """The job's time: the slowest rank's device time (one all-reduce of a scalar), then a
    barrier so no rank leaves the timed phase early.  Identity without a process group."""
    if not dist:
        return ms_local
    t = torch.tensor([ms_local], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.barrier()
    return float(t.item())


def replicas_value(world_size, steps, ms_max):
    """Whole-job throughput of N independent replicas: all ranks' OC iterations / slowest time."""
    return world_size * steps / (ms_max / 1000.0)


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        return ws, rank, local, dist, torch
    return 1, 0, 0, None, None


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="native", choices=["native", "reference"])
    ap.add_argument("--workload", default="cuboid128", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline sample")
    ap.add_argument("--serve", action="store_true",
                    help="run only the served stream (continuous batching) and print its line")
    ap.add_argument("--serve-jobs", type=int, default=256)
    ap.add_argument("--serve-precision", choices=["mixed", "mixed32", "fp64"], default="mixed")
    ap.add_argument("--serve-slots", type=int, default=8)
    ap.add_argument("--serve-seq-jobs", type=int, default=32,
                    help="jobs of the stream also run one at a time in FP64 for the baseline")
    ap.add_argument("--ref-budget-s", type=float, default=240.0,
                    help="reference arm: time spent on timed whole OC iterations (at least one runs)")
    ap.add_argument("--mixed", choices=["mixed", "mixed32"], default="mixed",
                    help="precision of the mixed arm: FP32 preconditioner (mixed), also FP32 filter (mixed32)")
    ap.add_argument("--profile-one-step", action="store_true",
                    help="profiling pass: one warm-up OC iteration, then one OC iteration between "
                         "cudaProfilerStart/Stop (for ncu --profile-from-start off); prints its PCG counts")
    ap.add_argument("--coarse-levels", action="store_true",
                    help="with --profile-one-step: run the coarsest solve level by level, not as one persistent launch")
    ap.add_argument("--only", choices=["mixed", "mixed32", "fp64"], default=None,
                    help="run one precision arm only (profiling); prints its timing and exits")
    a = ap.parse_args(argv)
    wl = WORKLOADS[a.workload]
    ws, rank, local, dist, torch = dist_setup()
    if "shape" in wl:
        call = "TOP3D_XL(true(%d,%d,%d),'%s',%g,%d,sqrt(3)%s)" % (*wl["shape"], wl["cons"], wl["V0"], wl["nLoop"],
                                                             ",%g" % wl["rHat"] if wl["cons"] == "LOCAL" else "")
    else:
        call = "TOP3D_XL('<generated %s>.TopVoxel','%s',%g,%d,sqrt(3),%g)" % (wl["topvoxel"], wl["cons"], wl["V0"],
                                                                           wl["nLoop"], wl["rHat"])
    cfg = {"workload": "%s %s V0=%g rMin=sqrt(3): %s" % (a.workload, wl["cons"], wl["V0"], call),
           "elements": int(np.prod(wl["shape"])) if "shape" in wl else None, "consType": wl["cons"],
           "l2": "inputs larger than L2 (state > 126 MB per job)", "parallelism": "replicas only"}

    if a.impl == "reference":
        if rank != 0:
            return 0
        # The reference is MATLAB and cannot run here; its CPU restatement (the oracle) runs whole
        # OC iterations on the host cores, as many of the requested steps as fit the time budget.
        t0 = time.perf_counter()
        cw = cpu_whole_iterations(wl, a.steps, a.ref_budget_s)
        sample = ("whole OC iterations of the oracle FP64 (numpy/scipy CPU restatement of TOP3D_XL.m; BLAS on "
                  "all %d cores, elementwise passes on one) on the workload itself: %d timed in %.1f s after "
                  "%.1f s of untimed set-up and solid solve; PCG iterations per solve %s"
                  % (cw["cores"], cw["steps"], cw["seconds"], cw["setup_s"], cw["its"]))
        line = {"impl": "reference", "metric": METRIC, "value": cw["value"], "unit": "OC iterations/s",
                "n_gpus": a.gpus, "steps": cw["steps"], "warmup": 0, "steps_requested": a.steps,
                "warmup_requested": a.warmup, "ms_per_step": 1000.0 * cw["seconds"] / cw["steps"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (built-in cuboid BCs)" if "shape" in wl else "synthetic (generated .TopVoxel)",
                "config": cfg,
                "cpu_baseline": {"value": cw["value"], "unit": "OC iterations/s", "cores": cw["cores"],
                                 "kind": "port", "sample": sample},
                "e2e": {"value": cw["value"], "unit": "OC iterations/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0},
                "wall_s": time.perf_counter() - t0}
        print(json.dumps(line), flush=True)
        return 0

    device = local
    if a.serve:
        if rank != 0:
            return 0
        jobs = serve_stream(a.serve_jobs)
        with Clocks(device) as clk:
            served = run_served(jobs, a.serve_precision, a.serve_slots, device)
        seq = run_sequential(jobs[:a.serve_seq_jobs], "fp64", device)
        seq_mixed_slots = run_served(jobs[:a.serve_seq_jobs], a.serve_precision, a.serve_slots, device)
        line = {"metric": "served design latency p50/p99 and OC iterations/s (continuous batching)",
                "value": served["oc_its_per_s"], "unit": "OC iterations/s", "n_gpus": 1,
                "higher_is_better": True, "dtype": "f64 Krylov/operator, f32 preconditioner (mixed)",
                "data": "synthetic served stream (seeded Poisson arrivals, solid cuboids, built-in BCs)",
                "config": {"workload": "%d jobs, mean gap 50 ms, dims (16,32,16)*s, s log-uniform [1,6], "
                                       "70%% GLOBAL 50 its / 30%% LOCAL 100 its" % a.serve_jobs,
                           "slots": a.serve_slots},
                "p50_latency_s": served["p50_s"], "p99_latency_s": served["p99_s"], "served": served,
                "sequential_fp64": seq, "same_jobs_served": seq_mixed_slots,
                "served_vs_sequential_fp64": (seq_mixed_slots["oc_its_per_s"] / seq["oc_its_per_s"])
                if seq["oc_its_per_s"] and seq_mixed_slots["oc_its_per_s"] else None,
                "clocks": clk.summary()}
        print(json.dumps(line), flush=True)
        return 0
    if a.profile_one_step:
        return profile_one_step(wl, a.only or "fp64", device, coop=not a.coarse_levels)
    if a.only:
        r = run_native(wl, a.only, a.steps, a.warmup, device, profile_steps=1)
        print(json.dumps({"only": a.only, "ms_per_step": r["ms"] / max(1, a.steps),
                          "launches_before_timed": r["launches_before"], "launches_timed": r["launches"],
                          "pcg_its": [k for h in r["hist"] for k in h["its"]],
                          "ku_ms_per_launch": r["prof"]["ku_ms"] / max(1, r["prof"]["ku_launches"]),
                          "sections_ms_per_profiled_step": {k: v[0] for k, v in r["prof"]["sections"].items()}}),
              flush=True)
        return 0
    if dist:
        dist.barrier()
    clk = Clocks(device)
    fp64 = run_native(wl, "fp64", a.steps, a.warmup, device, profile_steps=2, clk=clk)
    ms_local = fp64["ms"]
    ms_max = max_over_ranks(ms_local, dist, torch, "cuda")
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return 0
    mixed = run_native(wl, a.mixed, a.steps, a.warmup, device)
    value = replicas_value(ws, a.steps, ms_max)
    cm = np.array([h["c"] for h in mixed["hist"]])
    cd = np.array([h["c"] for h in fp64["hist"]])
    n = min(len(cm), len(cd))
    relerrs = np.abs(cm[:n] - cd[:n]) / np.abs(cd[:n])
    relerr = float(np.max(relerrs))
    # roofline of the dominant kernel: level-1 K*u in PCG mode (FP64 in both arms; the tile
    # kernel and its last-row kernel).  Per launch it reads p_old and z and writes q and the new
    # direction p, and reads and writes the solution y for the previous iteration's step (3
    # doubles per node each), reads the moduli (1 double per element) and the free-DOF bits (1
    # byte per node): 145 B/node + 8 B/element; per node 8 hexes x 3 rows x 24 DOFs + 24
    # scalings = 600 FMA.
    prof = fp64["prof"]
    nn = fp64["nnodes"]
    alg_bytes = 145 * nn + 8 * fp64["ne"]
    flop = 2 * 600 * nn
    ku_ms = prof["ku_ms"] / max(1, prof["ku_launches"])
    achieved = alg_bytes / (ku_ms * 1e-3) / 1e9
    tflops = flop / (ku_ms * 1e-3) / 1e12
    peak, kind = peaks()
    its64 = [k for h in fp64["hist"][a.warmup:] for k in h["its"]]
    its_mixed = [k for h in mixed["hist"][a.warmup:] for k in h["its"]]
    fits = [h["filter_its"] for h in fp64["hist"][a.warmup:]]
    e2e = run_e2e(wl, "fp64", a.steps, a.warmup, device)  # the same OC iterations as the device-timed run

    def phases(run):
        hs = run["hist"][a.warmup:]
        return {k: 1000.0 * float(np.mean([h[k] for h in hs])) for k in ("t_assemble", "t_cg", "t_filter", "t_opt")}
    line = {"metric": METRIC, "value": value, "unit": "OC iterations/s", "n_gpus": ws, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms_max / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (built-in cuboid BCs)", "config": cfg,
            "mixed": {"value": a.steps / (mixed["ms"] / 1000.0), "ms_per_step": mixed["ms"] / a.steps,
                      "dtype": "f64 Krylov iteration, operator, dots, compliance, OC%s; f32 multigrid "
                               "preconditioner%s" % ((", filter", "") if a.mixed == "mixed" else ("", " and filter")),
                      "precision": a.mixed,
                      "pcg_its_per_step": float(np.mean(its_mixed)),
                      "max_rel_compliance_err_vs_fp64": relerr, "iterations_compared": n,
                      "rel_compliance_err_per_iteration": [float("%.3g" % e) for e in relerrs]},
            "pcg_its_per_step": float(np.mean(its64)), "filter_its_per_step": float(np.mean(fits)),
            "phases_ms": {"fp64": phases(fp64), "mixed": phases(mixed)},
            "sections_ms_per_step": {k: round(v[0] / prof["steps"], 3) for k, v in prof["sections"].items()},
            "section_groups_per_step": {k: round(v[1] / prof["steps"], 1) for k, v in prof["sections"].items()},
            "gpu_launches": fp64["launches"],
            "roofline": {"kernel": "k_ku_l1<double, KU_P_UPDATE> (level-1 K*u, PCG mode)", "bound": "hbm",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": kind, "algorithmic_bytes_per_launch": alg_bytes,
                         "ms_per_launch": ku_ms, "traffic": KU_TRAFFIC_PER_NODE * nn if KU_TRAFFIC_PER_NODE else None,
                         "fp64_pipe": {"flop_per_launch": flop, "achieved_tflops": tflops,
                                       "nominal_peak_tflops": FP64_NOMINAL_TFLOPS,
                                       "frac_of_nominal": tflops / FP64_NOMINAL_TFLOPS}},
            "e2e": {"value": e2e["value"], "unit": "OC iterations/s", "h2d_bytes_per_step": e2e["h2d"],
                    "d2h_bytes_per_step": e2e["d2h"]},
            "clocks": clk.summary()}
    if not a.no_cpu and ws == 1:
        cb = cpu_sample(wl, float(np.mean(its64)), float(np.mean(fits)))
        line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
