#!/usr/bin/env python
"""Benchmark: FP64 point-substeps per second of the channel-flow RK3 substep.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the large single instance, sized for one B200): order-4 chanfast4
substep, grid nx = 512 (streamwise) x ny = 512 (spanwise) x nz = 384
(wall-normal, cosine-stretched), box 2pi x pi x 2, Re_b = 20000 (nu = 1/20000,
U_b = 1), dt = 2.5e-4, passive scalar Pr = 0.71, constant flow rate and scalar
mean; initial state laminar Poiseuille + divergence-projected seeded
perturbation (amplitude 0.05 U_cl, scalar noise 0.01), generated on the device.
Synthetic data: there is no dataset.

A bench step is one RK3 time step = 3 substeps; value = interior points x 3 x K
(summed over ranks) / device time of the K steps (CUDA events on the instance
stream, max over ranks).  With N > 1 every rank runs an independent replica
(weak scaling, no collective on the data path).  Every field is 805 MB, far
above the 126 MB L2, so no flush is needed between steps.

--impl reference times the reference's own CPU implementation (the unmodified
sources compiled by oracle/Makefile) on a bounded sample of the same workload
on this host's cores; only rank 0 works.
"""
from __future__ import annotations

import argparse
import csv
import importlib
import io
import json
import math
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # the large single instance (headline)
    "config2": dict(name="chanfast4 512x512x384 Re_b=20000", order=4, nx=512, ny=512, nz=384,
                    lx=2 * math.pi, ly=math.pi, lz=2.0, dt=2.5e-4, nu=1.0 / 20000.0, prandtl=0.71,
                    seed=2, amp=0.05, c_amp=0.01, run_steps=50),
    # mid size, used for profiling captures
    "config1": dict(name="chanfast4 256x256x192 Re_b=10000", order=4, nx=256, ny=256, nz=192,
                    lx=2 * math.pi, ly=math.pi, lz=2.0, dt=5e-4, nu=1.0 / 10000.0, prandtl=0.71,
                    seed=1, amp=0.1, c_amp=0.01, run_steps=200),
    # the benchmark grid cut to a quarter of the planes, for profiling captures
    # of the kernels whose parallelism follows the x-y size (the band solves:
    # the same 66k column pairs as config2) in a quarter of the memory
    "config2z96": dict(name="chanfast4 512x512x96 Re_b=20000", order=4, nx=512, ny=512, nz=96,
                       lx=2 * math.pi, ly=math.pi, lz=2.0, dt=2.5e-4, nu=1.0 / 20000.0, prandtl=0.71,
                       seed=2, amp=0.05, c_amp=0.01, run_steps=50),
    # the reference's own CPU-runnable case
    "config0": dict(name="chanfast2 64x64x64 Re_b=2800", order=2, nx=64, ny=64, nz=64,
                    lx=4 * math.pi, ly=4 * math.pi / 3, lz=2.0, dt=1e-3, nu=1.0 / 2800.0, prandtl=1.0,
                    seed=0, amp=0.1, c_amp=0.0, run_steps=100),
    # the fully implicit scheme (channel4) on the headline grid
    "channel4": dict(name="channel4 512x512x384 Re_b=20000", order=4, nx=512, ny=512, nz=384,
                     lx=2 * math.pi, ly=math.pi, lz=2.0, dt=2.5e-4, nu=1.0 / 20000.0, prandtl=0.71,
                     seed=2, amp=0.05, c_amp=0.01, run_steps=20, scheme="channel", b_alg=496.0),
}
WORKLOAD = WORKLOADS["config2"]
B_ALG = 240.0            # algorithmic HBM bytes per point-substep (whole substep)
# The fully implicit scheme adds, per field, the x and y transforms there and
# back and the spectral solve over the half spectrum (8 B/pt each way per
# pass: 5 passes x 16 B x 4 fields) and drops the back substitution (64 B):
# 240 + 320 - 64 = 496 B/pt (the workload's "b_alg").
METRIC = "FP64 Mpt-substeps/s"
# Minimal bytes per interior point of each kernel group (own inputs + outputs):
# rhs = RHS + forward sweeps (read u,v,w,c,g x4; write f x4, s x4), solve = back
# substitution (read s x4, write x x4)
KERNEL_BYTES = {"rhs": 128.0, "solve": 64.0,
                "div_fftx": 32.0, "ffty_fwd": 16.0, "poisson": 16.0, "ffty_bwd": 16.0,
                "fftx_c2r": 16.0, "project": 72.0}
# CPU-baseline sample: same order / nz / dt / viscosity, fewer x-y points per
# process; REPEATS timed repeats of `substeps` substeps after one warm-up
CPU_SAMPLE = dict(nx=128, ny=128, substeps=1, repeats=5)
# the oracle's build of the reference sources (oracle/Makefile)
REF_CFLAGS = "-O3 -funroll-loops -ffp-contract=off"


def cpu_sample_grid():
    """x-y size of one CPU-sample instance: the workload's own grid when it
    is no larger than the sample, else the sample (same nz)."""
    return min(WORKLOAD["nx"], CPU_SAMPLE["nx"]), min(WORKLOAD["ny"], CPU_SAMPLE["ny"])


def host_info():
    """CPU model, physical and logical cores, compiler, and whether an MPI
    compiler and FFTW 3 exist on this host (they decide how the reference
    can be built here: with neither, the oracle's single-rank shims)."""
    info = {"cpu_model": None, "physical_cores": None, "logical_cpus": os.cpu_count()}
    try:
        cores, model = set(), None
        phys = core = None
        with open("/proc/cpuinfo") as f:
            for line in f:
                k, _, v = line.partition(":")
                k, v = k.strip(), v.strip()
                if k == "model name" and model is None:
                    model = v
                elif k == "physical id":
                    phys = v
                elif k == "core id":
                    core = v
                elif not k and phys is not None:
                    cores.add((phys, core))
                    phys = core = None
        if phys is not None:
            cores.add((phys, core))
        info["cpu_model"] = model
        info["physical_cores"] = len(cores) or None
    except OSError:
        pass
    import shutil

    def first_line(cmd):
        try:
            r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, timeout=20)
            return r.stdout.strip().splitlines()[0] if r.returncode == 0 and r.stdout.strip() else None
        except (OSError, subprocess.SubprocessError):
            return None
    info["compiler"] = first_line([os.environ.get("CC", "gcc"), "--version"])
    info["cflags"] = REF_CFLAGS
    info["mpicc"] = first_line(["mpicc", "--version"]) if shutil.which("mpicc") else "not found"
    info["fftw3"] = first_line(["pkg-config", "--modversion", "fftw3"]) or "not found (pkg-config)"
    return info


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------------ clocks

class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-i", str(self.gpu), "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        self.out = ""
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self):
        rows = [r for r in csv.reader(io.StringIO(getattr(self, "out", ""))) if len(r) >= 9]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        smax = max(float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for n, v in zip(names, r[5:9]):
                if v.strip() == "Active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "samples": len(rows), "reasons": sorted(reasons)}


# ------------------------------------------------------------ CPU reference

def _ref_worker(args):
    """One single-rank reference instance (oracle/_ref) on a sample grid:
    `warm` untimed substeps, then `reps` timed runs of `nsub` substeps."""
    wname, nx, ny, nsub, warm, reps, seed = args
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import chanfast_np as cn
    import ic
    import ref
    w = WORKLOADS[wname]
    prm = cn.Params(order=w["order"], nx=nx, ny=ny, nz=w["nz"], lx=w["lx"], ly=w["ly"], lz=w["lz"],
                    dt=w["dt"], nu=w["nu"], prandtl=w["prandtl"])
    g = cn.Grid(prm)
    R = ref.RefInstance(prm)
    u, v, wf, c = ic.raw_state(prm, g.dz, seed, w["amp"], w["c_amp"])
    for nm, a in zip("uvwc", (u, v, wf, c)):
        R.set(nm, a)
    R.project(1.0)
    scheme = w.get("scheme", "chanfast")
    if warm:
        R.substeps(warm, scheme)
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        R.substeps(nsub, scheme)
        times.append(time.perf_counter() - t0)
    R.close()
    return times


def cpu_reference(nsub, warm, reps, nproc=None):
    """Aggregate reference throughput on `nproc` independent single-rank
    processes (one per core), Mpt-substeps/s: the median over `reps` timed
    repeats (each the sum over processes of that repeat's rate), with the
    spread.  Returns (median, nproc, sample, per-repeat slowest time,
    [min, max])."""
    if nproc is None:
        ncpu = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
        try:
            mem_gb = os.sysconf("SC_PAGE_SIZE") * os.sysconf("SC_PHYS_PAGES") / 2 ** 30
        except (ValueError, OSError):
            mem_gb = 16.0
        nproc = max(1, min(ncpu, int(mem_gb // 3), 64))
    nx, ny = cpu_sample_grid()
    ctx = mp.get_context("spawn")
    with ctx.Pool(nproc) as pool:
        wname = next(k for k, v in WORKLOADS.items() if v is WORKLOAD)
        times = pool.map(_ref_worker, [(wname, nx, ny, nsub, warm, reps, 100 + r) for r in range(nproc)])
    pts = nx * ny * WORKLOAD["nz"]
    per_rep = [sum(pts * nsub / t[r] for t in times) / 1e6 for r in range(reps)]
    slowest = statistics.median(max(t[r] for t in times) for r in range(reps))
    sample = (f"unmodified reference {WORKLOAD.get('scheme', 'chanfast')}{WORKLOAD['order']} substep "
              f"(oracle/_ref, single-rank MPI/FFTW shims, "
              f"gcc {REF_CFLAGS}) on {nproc} independent {nx}x{ny}x{WORKLOAD['nz']} instances, one per core; "
              f"median of {reps} timed repeats of {nsub} substep(s) each after {warm} warm-up")
    return statistics.median(per_rep), nproc, sample, slowest, [min(per_rep), max(per_rep)]


def ensure_reference():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref
    if not ref.available():
        if os.path.isdir(ref.REFERENCE_SRC):
            ref.build()
        else:
            return False
    return True


# ---------------------------------------------------------------- GPU arm

def max_over_ranks(x, dist, device="cuda"):
    """The largest x over all ranks: a multi-GPU run takes as long as its
    slowest replica."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(pts, substeps, world, seconds):
    """Whole-job throughput in Mpt-substeps/s: every replica advances its
    own `pts`-point instance by `substeps` in the job's time."""
    return pts * substeps * world / seconds / 1e6


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_ours(args):
    import torch
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    cf = importlib.import_module("ubiquitous-spoon_b200")
    w = WORKLOAD
    cfg = cf.Config.make(order=w["order"], nx=w["nx"], ny=w["ny"], nz=w["nz"], lx=w["lx"], ly=w["ly"],
                         lz=w["lz"], dt=w["dt"], nu=w["nu"], prandtl=w["prandtl"],
                         scheme=w.get("scheme", "chanfast"))
    b_alg = w.get("b_alg", B_ALG)
    stream = torch.cuda.Stream()
    inst = cf.Instance(cfg, stream=ctypes_stream(stream))
    if args.launch_shape:
        inst.set_launch_shape(tuple(int(x) for x in args.launch_shape.split(",")))
    lshape = list(inst.launch_shape())
    inst.init_fields(w["seed"] + rank, w["amp"], w["c_amp"])
    inst.step_graph(args.warmup)
    inst.sync()

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        barrier()
        start.record(stream)
        inst.step_graph(args.steps)
        end.record(stream)
        end.synchronize()
        barrier()
    ms = max_over_ranks(start.elapsed_time(end), dist)
    pts = w["nx"] * w["ny"] * w["nz"]
    substeps = 3 * args.steps
    value = job_value(pts, substeps, world, ms * 1e-3)
    ms_per_step = ms / args.steps

    # per-kernel device times (CUDA events between the launch groups)
    prof = inst.profile(3)
    sub_ms = sum(prof.values()) / 3.0
    peak, peak_kind = measured_peaks()
    kernels = {}
    fused = inst.pressure_fused()
    for name, t in prof.items():
        t1 = t / 3.0
        nb = KERNEL_BYTES.get(name) if "scheme" not in w else None
        if fused and name in ("ffty_fwd", "ffty_bwd"):
            kernels[name] = {"ms": round(t1, 4), "fused_into": "poisson"}
            continue
        gbs = nb * pts / (t1 * 1e-3) / 1e9 if nb and t1 > 0 else None
        kernels[name] = {"ms": round(t1, 4), "alg_bytes_per_pt": nb,
                         "gbs": round(gbs, 1) if gbs else None,
                         "frac": round(gbs / peak, 3) if gbs else None}
        if fused and name == "poisson":
            kernels[name]["kernel"] = "k_poisson_fft: y transform, Poisson solve, inverse y transform"
    substep_ms = ms_per_step / 3.0
    achieved = b_alg * pts / (substep_ms * 1e-3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic_per_substep.json")
    if os.path.exists(tpath) and "scheme" not in w:   # measured for the headline workload
        with open(tpath) as f:
            traffic = json.load(f).get("dram_bytes_per_substep_full_size")
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": traffic,
                "kernel": f"whole RK3 substep (CUDA graph of {inst.launches_per_substep()} launches)",
                "alg_bytes_per_unit": b_alg, "unit_desc": "interior point-substep",
                "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                "kernels": kernels, "profiled_substep_ms": round(sub_ms, 4)}

    # end to end through the C ABI with host buffers: restart-style run of
    # run_steps time steps, fields in and out in the reference layout
    e2e = None
    if not args.no_e2e:
        shape = cfg.padded_shape()
        host = {nm: torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy() for nm in "uvwc"}
        for nm in "uvwc":
            inst.get_field(nm, out=host[nm])
        nrun = w["run_steps"]
        inst2 = cf.Instance(cfg, stream=ctypes_stream(stream))
        barrier()
        t0 = time.perf_counter()
        for nm in "uvwc":
            inst2.set_field(nm, host[nm])
        inst2.step_graph(nrun)
        for nm in "uvwc":
            inst2.get_field(nm, out=host[nm])
        barrier()
        t_e2e = max_over_ranks(time.perf_counter() - t0, dist)
        nbytes = 4 * host["u"].nbytes
        e2e = {"value": round(job_value(pts, 3 * nrun, world, t_e2e), 1), "unit": METRIC,
               "h2d_bytes_per_step": nbytes // nrun, "d2h_bytes_per_step": nbytes // nrun,
               "run_steps": nrun,
               "how": "cf_set_field x4 (pinned host, reference padded layout) + cf_step_graph(run_steps) "
                      "+ cf_get_field x4, wall clock, max over ranks"}
        inst2.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu and ensure_reference():
        v, nproc, sample, _, spread = cpu_reference(CPU_SAMPLE["substeps"], 1, CPU_SAMPLE["repeats"])
        cpu = {"value": round(v, 3), "unit": METRIC, "cores": nproc, "kind": "reference", "sample": sample,
               "spread": [round(x, 3) for x in spread], "host": host_info()}

    div = inst.max_divergence()
    launches = inst.launches_per_substep() * substeps
    inst.close()
    result = {
        "metric": METRIC, "value": round(value, 1), "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": w["name"], "order": w["order"], "nx": w["nx"], "ny": w["ny"], "nz": w["nz"],
                   "box": "2pi x pi x 2", "dt": w["dt"], "nu": w["nu"], "prandtl": w["prandtl"],
                   "step": "one RK3 time step = 3 substeps",
                   "l2": f"inputs larger than L2 ({pts * (w['nz'] + 6) // w['nz'] * 8 / 1e6:.0f} MB per field, "
                         "4 fields read per kernel vs 126 MB L2); no flush",
                   "parallelism": f"replicas x{world}" if world > 1 else "single instance",
                   "launch_shape": {"solve_threads": lshape[0], "poisson_threads": lshape[1],
                                    "project_block": lshape[2:]}},
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
        "clocks": clk.summary(), "max_divergence": div,
    }
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result), flush=True)


# ------------------------------------------------------------- ensemble

ENSEMBLE_GRIDS = [(64, 64, 64), (96, 96, 64), (128, 128, 96), (192, 192, 128)]   # (nx, ny, nz)


def ensemble_members(n=64):
    """The 64-instance ensemble: per seed s a grid from ENSEMBLE_GRIDS and
    Re_b ~ U[2800, 10000], order 2, box 4pi x 4pi/3 x 2, dt 1e-3."""
    import numpy as np
    out = []
    for s in range(n):
        rng = np.random.default_rng(s)
        nx, ny, nz = ENSEMBLE_GRIDS[int(rng.integers(len(ENSEMBLE_GRIDS)))]
        out.append(dict(seed=s, nx=nx, ny=ny, nz=nz, re=float(rng.uniform(2800.0, 10000.0))))
    return out


def run_ensemble(args):
    """Solves/hour of the ensemble batched (cf_batch: one launch per stage
    for all 64 instances, replayed as a CUDA graph) against the same
    instances one after another through the plain path (cf_step_graph), both
    on device time; a solve is 500 RK3 steps, timed over args.steps.  Both
    arms start from the same seeded states and run the same steps, so every
    member is then compared with its plain-path run (relative L2 of u, v, w,
    c; the batched kernels are other instantiations of the same bodies and
    may contract multiply-adds differently)."""
    import numpy as np
    import torch
    cf = importlib.import_module("ubiquitous-spoon_b200")
    torch.cuda.set_device(0)
    members = ensemble_members()

    def create():
        insts = []
        for m in members:
            cfg = cf.Config.make(order=2, nx=m["nx"], ny=m["ny"], nz=m["nz"], lx=4 * math.pi,
                                 ly=4 * math.pi / 3, lz=2.0, dt=1e-3, nu=1.0 / m["re"], prandtl=1.0)
            inst = cf.Instance(cfg)
            inst.init_fields(m["seed"], 0.1, 0.0)
            insts.append(inst)
        for inst in insts:
            inst.sync()
        return insts

    pts = sum(m["nx"] * m["ny"] * m["nz"] for m in members)
    # batched
    insts = create()
    t0 = time.perf_counter()
    B = cf.Batch(insts)   # records the cycle and tunes the batched launch shapes
    t_create = time.perf_counter() - t0
    batch_shape = list(B.launch_shape())
    B.run(args.warmup)
    B.sync()
    with ClockSampler(0) as clk:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        B.run(args.steps)
        B.sync()
        t_batch = time.perf_counter() - t0
    launches = B.launches_per_substep()
    div = max(inst.max_divergence() for inst in insts)
    batched = [{nm: inst.get_field(nm, layout=cf.LAYOUT_INTERIOR) for nm in "uvwc"} for inst in insts]
    B.close()
    for inst in insts:
        inst.close()
    # one after another, plain path
    insts = create()
    t_seq = 0.0
    worst = {nm: 0.0 for nm in "uvwc"}
    for m, inst in enumerate(insts):
        inst.step_graph(args.warmup)
        inst.sync()
        t0 = time.perf_counter()
        inst.step_graph(args.steps)
        inst.sync()
        t_seq += time.perf_counter() - t0
        for nm in "uvwc":
            a, b = batched[m][nm], inst.get_field(nm, layout=cf.LAYOUT_INTERIOR)
            worst[nm] = max(worst[nm], float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)))
        inst.close()
    solve_steps = 500
    per_h = lambda t: len(members) / (t * solve_steps / args.steps) * 3600.0
    result = {
        "metric": "ensemble solves/h", "value": round(per_h(t_batch), 1), "unit": "solves/h",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
        "sequential_plain_path": round(per_h(t_seq), 1), "speedup_vs_sequential": round(t_seq / t_batch, 2),
        "batch_launch_shape": {"solve_threads": batch_shape[0], "poisson_threads": batch_shape[1],
                               "project_block": batch_shape[2:]},
        "batch_create_s": round(t_create, 3),
        "mpt_substeps_per_s": round(pts * 3 * args.steps / t_batch / 1e6, 1),
        "ms_per_step_all_members": round(t_batch / args.steps * 1e3, 3),
        "batched_launches_per_substep": launches, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "64-instance ensemble, order 2, grids per seed from "
                               + ", ".join("x".join(map(str, g)) for g in ENSEMBLE_GRIDS)
                               + ", Re_b ~ U[2800, 10000], dt 1e-3",
                   "solve": f"{solve_steps} RK3 steps (timed over {args.steps}, scaled)",
                   "points": pts, "timing": "wall clock around stream-synchronised runs"},
        "max_divergence": div, "clocks": clk.summary(),
        "members_vs_plain_path": {"members": len(members), "max_rel_l2": {k: float(f"{v:.3e}") for k, v in worst.items()},
                                  "within_1e-13": all(v <= 1e-13 for v in worst.values())},
    }
    print(json.dumps(result), flush=True)


# -------------------------------------------------------------- serving

SERVE_GRIDS = ENSEMBLE_GRIDS + [(256, 256, 192)]


def serve_trace(n, rate, step_scale, seed=0):
    """Poisson arrivals at `rate` per second; per request a grid from
    SERVE_GRIDS, Re_b log-uniform in [2800, 20000], order 2 or 4, and
    U[200, 2000] RK3 steps times step_scale."""
    import numpy as np
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for q in range(n):
        t += rng.exponential(1.0 / rate)
        nx, ny, nz = SERVE_GRIDS[int(rng.integers(len(SERVE_GRIDS)))]
        re = float(math.exp(rng.uniform(math.log(2800.0), math.log(20000.0))))
        order = int(rng.choice([2, 4]))
        steps = max(1, int(round(int(rng.integers(200, 2001)) * step_scale)))
        out.append(dict(arrival_s=t, nx=nx, ny=ny, nz=nz, re=re, order=order, nsteps=steps, seed=q))
    return out


def run_serve(args):
    """p50 / p99 completion latency and solves/hour of the serving loop
    (cf_serve: admission by a 150 GB budget, continuous batching, one
    batched step per round) on a Poisson trace; with --serve-baseline also
    the same trace served one solve at a time (max_active = 1)."""
    import numpy as np
    import torch
    cf = importlib.import_module("ubiquitous-spoon_b200")
    torch.cuda.set_device(0)
    trace = serve_trace(args.serve_requests, 4.0, args.serve_step_scale)
    reqs = []
    for r in trace:
        # the ensemble's box and time step (4pi x 4pi/3 x 2, dt 1e-3)
        cfg = cf.Config.make(order=r["order"], nx=r["nx"], ny=r["ny"], nz=r["nz"], lx=4 * math.pi,
                             ly=4 * math.pi / 3, lz=2.0, dt=1e-3, nu=1.0 / r["re"], prandtl=0.71)
        reqs.append(dict(cfg=cfg, seed=r["seed"], amp=0.05, c_amp=0.01, nsteps=r["nsteps"],
                         arrival_s=r["arrival_s"]))

    def measure(max_active):
        t0 = time.perf_counter()
        res = cf.serve(reqs, hbm_budget_bytes=150e9, max_active=max_active, quantum=args.serve_quantum)
        wall = time.perf_counter() - t0
        lat = np.array([x["finish_s"] - r["arrival_s"] for x, r in zip(res, reqs)])
        ok = sum(1 for x in res if x["status"] == 0)
        work = sum(r["nx"] * r["ny"] * r["nz"] * 3 * r["nsteps"] for r in trace)
        return {"p50_latency_s": round(float(np.percentile(lat, 50)), 3),
                "p99_latency_s": round(float(np.percentile(lat, 99)), 3),
                "solves_per_h": round(ok / wall * 3600.0, 1), "completed": ok, "wall_s": round(wall, 2),
                "mpt_substeps_per_s": round(work / wall / 1e6, 1)}

    with ClockSampler(0) as clk:
        served = measure(64)
    result = {"metric": "serving p50/p99 completion latency, solves/h", "value": served["solves_per_h"],
              "unit": "solves/h", "n_gpus": 1, "higher_is_better": True, "served": served,
              "dtype": "f64", "data": "synthetic",
              "config": {"workload": f"{len(reqs)} requests, Poisson arrivals 4/s (seed 0), grids "
                                     + ", ".join("x".join(map(str, g)) for g in SERVE_GRIDS)
                                     + ", Re_b log-U[2800, 20000], order 2 or 4",
                         "steps": f"U[200, 2000] x {args.serve_step_scale} RK3 steps per request",
                         "box": "4pi x 4pi/3 x 2, dt 1e-3",
                         "admission": "150 GB budget by cf_instance_bytes, at most 64 resident",
                         "rounds": f"{args.serve_quantum} RK3 step(s) of every resident solve per batched call"},
              "clocks": clk.summary()}
    if args.serve_baseline:
        result["one_at_a_time"] = measure(1)
    print(json.dumps(result), flush=True)


def ctypes_stream(torch_stream):
    import ctypes
    return ctypes.c_void_p(torch_stream.cuda_stream)


def run_reference(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return
    if not ensure_reference():
        print(json.dumps({"impl": "reference", "unavailable": "reference sources absent and oracle/_ref not built"}))
        return
    # a step: one substep on every process; the median over the K steps
    v, nproc, sample, tstep, spread = cpu_reference(1, args.warmup, args.steps)
    nx, ny = cpu_sample_grid()
    ms_per_step = tstep * 1e3
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": METRIC, "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD["name"], "order": WORKLOAD["order"], "nx": WORKLOAD["nx"], "ny": WORKLOAD["ny"],
                   "nz": WORKLOAD["nz"], "step": f"one substep on each of {nproc} {nx}x{ny}x{WORKLOAD['nz']} "
                   "sample instances in parallel"},
        "cpu_baseline": {"value": round(v, 3), "unit": METRIC, "cores": nproc, "kind": "reference",
                         "sample": sample, "spread": [round(x, 3) for x in spread], "host": host_info()},
        "e2e": {"value": round(v, 3), "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--ensemble", action="store_true",
                    help="the 64-instance batched ensemble against running its members one after another")
    ap.add_argument("--serve", action="store_true", help="the serving loop on a Poisson request trace")
    ap.add_argument("--serve-requests", type=int, default=100)
    ap.add_argument("--serve-step-scale", type=float, default=0.1,
                    help="scale of the U[200, 2000] step counts (1.0 = the full trace)")
    ap.add_argument("--serve-baseline", action="store_true", help="also serve the trace one solve at a time")
    ap.add_argument("--serve-quantum", type=int, default=1, help="RK3 steps per serving round")
    ap.add_argument("--launch-shape", default="",
                    help="force the tuned kernels' launch shape: solve,poisson,proj_bx,proj_by")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="config2",
                    help="config2 (default) is the benchmark; the others serve profiling and checks")
    args = ap.parse_args()
    global WORKLOAD
    WORKLOAD = WORKLOADS[args.workload]
    if args.warmup < 3 and args.impl == "ours":
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    if args.ensemble:
        run_ensemble(args)
    elif args.serve:
        run_serve(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
