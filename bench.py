#!/usr/bin/env python
"""Benchmark of the fused LBM time step on B200.

Workload (the configuration the headline metric is quoted on): D3Q15 MRT
porous medium, 256^3 nodes, FP32 population storage, overlapping spheres
(radius 6) at solid fraction 0.30 with full-way bounceback, Zou-He pressure
faces rho = 1.001 / 0.999 on x, periodic y/z, tau = 0.7, s_e = s_eps = 1.19,
s_q = s_m = 1.2, s_nu = 1/tau.  Inputs are seeded synthetic arrays of that
shape; populations (1 GB) exceed the 126 MB L2, so no flush is needed
between steps.

One bench step = one LBM time step over the whole domain (one launch of the
fused step kernel).  value = lattice updates per second (GLUPS) over all
ranks, timed with CUDA events on the engine's stream, max over ranks.
e2e = the same metric through the C ABI with host buffers: lbmc_init from
host arrays (host->device copies), E2E_STEPS time steps, lbmc_fetch of rho
and u (device->host) into host arrays that exist before the job, per e2e
step; lbmc_destroy follows outside the timer (LBM-C's program exits without
freeing) and is reported beside it.

--impl reference times the reference's own step (host-compiled from its
sources, oracle/_ref) on the host cores with all threads, on a z-crop of the
same workload.  Multi-GPU: independent replicas (the reference is one GPU,
one domain), so scaling is weak and there is no collective in the data path.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "lbm-c_b200"))
sys.path.insert(0, ROOT)

UNIT = "GLUPS"
E2E_STEPS = 500
REF_ARM_SECONDS = 90.0  # bound of one --impl reference run (warm-up + steps)
STORAGE_BYTES = {"f32": 4, "f16": 2, "f16sr": 2, "bf16": 2, "f64": 8}


def algorithmic_bytes_per_lup(q: int, storage: str) -> int:
    """One read and one write of every population plus the class byte."""
    return 2 * q * STORAGE_BYTES[storage] + 1


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(kernel_tag: str):
    """dram read+write bytes per launch from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", f"{kernel_tag}.md")
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                value = line.split(":", 1)[1].split()[0]
                # "null": no per-launch DRAM figure (a state that stays in L2)
                return None if value == "null" else float(value)
    except OSError:
        pass
    return None


class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region.

    NVML (the library nvidia-smi reads) is polled every 2 ms from a thread,
    so that a region of a few milliseconds still holds samples; nvidia-smi's
    100 ms loop is the fallback when NVML cannot be loaded."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, device_index: int, period_s: float = 0.002):
        self.dev = device_index
        self.period = period_s
        self.proc = None
        self.nvml = None
        self.lines = []
        self.samples = []  # (sm_mhz, max_mhz, reasons)
        self.stop = threading.Event()
        self.source = None

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.dev).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(("GPU-" + uuid).encode())
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.dev)

    def _sample(self):
        nv, h = self.nvml
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        try:
            mhz = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
            r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
            self.samples.append((float(mhz), float(self.max_mhz), {k for k, b in bits.items() if r & b}))
        except Exception:
            pass

    def _poll(self):
        while not self.stop.is_set():
            self._sample()
            self.stop.wait(self.period)

    def __enter__(self):
        try:
            self.nvml = self._nvml_handle()
            nv, h = self.nvml
            self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            self.source = "nvml 2 ms"
            self._sample()  # one sample at the start, however short the region
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.source = "nvidia-smi 100 ms"
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.strip().split(",")]
            if len(parts) < 9:
                continue
            try:
                self.samples.append((float(parts[1]), float(parts[2]),
                                     {n for n, f in zip(self.REASONS, parts[5:9]) if f.lower() == "active"}))
            except ValueError:
                continue

    def __exit__(self, *exc):
        self.stop.set()
        if self.nvml is not None:
            self.thread.join(timeout=5)
            self._sample()  # and one at the end
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0,
                    "source": self.source}
        reasons = set().union(*(r for _, _, r in self.samples))
        return {"sm_mhz": statistics.median(m for m, _, _ in self.samples),
                "sm_max_mhz": max(x for _, x, _ in self.samples),
                "reasons": sorted(reasons), "samples": len(self.samples), "source": self.source}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        backend = "nccl" if args.impl == "ours" else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def dist_max(value: float, world: int, device=None) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_sum(value: float, world: int, device=None) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def aggregate_rate(units_local: float, seconds_local: float, world: int, device=None):
    """Whole-job throughput of independent replicas: all ranks' units over the
    slowest rank's time.  Returns (units per second, max seconds)."""
    t_max = dist_max(seconds_local, world, device)
    units = dist_sum(units_local, world, device)
    return units / t_max, t_max


def dist_barrier(world: int, device=None):
    if world > 1:
        import torch.distributed as dist
        if device is not None:
            dist.barrier(device_ids=[device.index])
        else:
            dist.barrier()


WORKLOAD_METRIC = {
    "batch": "aggregate GLUPS ({n} D2Q9 domains, persistent batched launch, to steady state)",
    "porous": "GLUPS (D3Q15 MRT porous {n}^3 fused step)",
    "tgv": "GLUPS (D3Q15 BGK+Smagorinsky Taylor-Green {n}^3 fused step)",
    "poiseuille": "GLUPS (D2Q9 BGK+Guo Poiseuille 128x64 fused step)",
    "closure": "GLUPS (D3Q15 BGK+Guo {n}^3 step with the learned subgrid closure)",
}


def build_workload(args):
    import workloads
    if args.workload == "tgv":
        return workloads.taylor_green(args.size)
    if args.workload == "poiseuille":
        return workloads.poiseuille_channel()
    if args.workload == "closure":
        return workloads.forced_box(args.size)
    L = (args.size, args.size, args.size)
    return workloads.porous_spheres(L)


def metric_name(args):
    if args.workload == "batch":
        return WORKLOAD_METRIC["batch"].format(n=args.domains)
    return WORKLOAD_METRIC[args.workload].format(n=args.size)


def run_batch(args, world, rank, local):
    """Batched sweep: independent D2Q9 NTPOR+Guo domains (IMB circles), one
    persistent launch replayed from a CUDA graph until every domain's
    max |u(t) - u(t-C)| < tol (C = check interval).  Per-domain latency =
    device time from the run's start to the domain's convergence; the
    comparison runs a seeded sample of domains alone through
    lbmc_init/lbmc_iterate (one launch per step) with the same criterion.

    FP16 storage floors max|u(t) - u(t-C)| at ~1e-8..1e-6 (quantisation of
    f - w), above the 1e-9 tolerance, in both paths; so the FP16 run is
    bounded by --batch-cap and reports throughput and the floor, and the
    time-to-steady / latency figures come from the FP32 run, which converges."""
    import torch

    import lbmc
    import workloads
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    tau, g, tol, check = BATCH_TAU, BATCH_G, 1e-9, 100
    geoms = workloads.batch_sweep(args.domains, seed=5 + rank, tau=tau)
    nodes = np.array([x.size for x in geoms])
    with lbmc.Batch(geoms[:8], tau=tau, force=(g, 0.0), storage=args.storage) as wb:
        wb.run(max(1, args.warmup) * check, 0.0, check)

    def batched(storage, cap):
        torch.cuda.synchronize(dev)
        b = lbmc.Batch(geoms, tau=tau, force=(g, 0.0), storage=storage, wide_below=args.wide_below,
                       wide_min_nodes=args.wide_min_nodes)
        t1 = time.perf_counter()
        res = b.run(cap, tol, check)
        torch.cuda.synchronize(dev)
        t_run = time.perf_counter() - t1
        info = b.info()
        b.close()
        steps = np.array([r.steps for r in res])
        conv = np.array([r.converged for r in res], bool)
        lat = np.array([r.elapsed_ms for r in res])
        du = np.array([r.delta_u for r in res])
        rate, t_max = aggregate_rate(float((steps * nodes).sum()), t_run, world, dev)
        out = {"storage": storage, "glups": rate / 1e9, "run_s": t_max, "step_cap": cap,
               "max_steps": int(steps.max()), "converged": int(conv.sum()),
               "unconverged": int((~conv).sum()), "threads": info["threads"],
               "steps_per_launch": info["steps_per_launch"],
               "resident_domains": info["resident_domains"]}
        if conv.any():
            out["time_to_steady_s"] = float(lat[conv].max() / 1e3)
            out["latency_p50_ms"] = float(np.percentile(lat[conv], 50))
            out["latency_p99_ms"] = float(np.percentile(lat[conv], 99))
        if (~conv).any():
            out["unconverged_delta_u"] = {"min": float(du[~conv].min()),
                                          "median": float(np.median(du[~conv])),
                                          "max": float(du[~conv].max())}
        return out, lat, conv

    with ClockSampler(local) as clk:
        main, _, _ = batched(args.storage, args.batch_cap)
    f32, lat32, conv32 = batched("f32", 400000) if args.storage != "f32" else (main, None, None)
    if lat32 is None:
        f32, lat32, conv32 = batched("f32", 400000)

    # alone: a seeded sample of domains, each through the single-domain engine (FP32)
    rng = np.random.default_rng(11)
    sample = rng.choice(len(geoms), size=min(args.alone_sample, len(geoms)), replace=False)
    alone, alone_conv = [], []
    for d in sample:
        ly, lx = geoms[d].shape
        n = lx * ly
        force = np.zeros((2, n))
        force[0] = g
        cfg = lbmc.make_config("d2q9", (lx, ly, 1), tau=tau, collision_type=lbmc.NTPOR,
                               forcing=True, storage="f32", device=local)
        dom, keep = lbmc.make_domain(n, 2, 9, geoms[d].reshape(n), force)
        torch.cuda.synchronize(dev)
        ta = time.perf_counter()
        ok = False
        with lbmc.Engine(cfg, dom) as e:
            prev, done = None, 0
            while done < 400000:
                e.iterate(check - 1, 0)
                e.iterate(1, lbmc.STORE_MACROS)
                done += check
                u = e.u()
                if prev is not None and np.abs(u - prev).max() < tol:
                    ok = True
                    break
                prev = u
        alone.append((time.perf_counter() - ta) * 1e3)
        alone_conv.append(ok)
        del keep
    both = [i for i, d in enumerate(sample) if conv32[d] and alone_conv[i]]
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        rate, desc = reference_batch_rate(geoms, batch_sample(len(geoms)), 200, threads)
        cpu = {"value": rate / 1e9, "unit": UNIT, "cores": threads, "kind": "reference", "sample": desc}
    # HBM roofline of the whole run: one read and one write of every
    # population plus the class byte per lattice update, as for a single
    # domain; domains held in shared memory read and write HBM once per
    # launch of K steps, so the run can sit above it.
    bpl = algorithmic_bytes_per_lup(9, args.storage)
    peak, peak_kind = measured_peak()
    achieved = main["glups"] * bpl
    if rank == 0:
        line = {
            "metric": metric_name(args), "value": main["glups"], "unit": UNIT, "n_gpus": world,
            "steps": main["max_steps"], "warmup": args.warmup, "ms_per_step": None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": args.storage, "data": "synthetic (seeded circles, IMB edges)",
            "config": {"workload": "batch_d2q9_ntpor_guo_circles", "domains": args.domains,
                       "total_nodes": int(nodes.sum()), "tau": tau, "g": g, "tol": tol,
                       "criterion": "max|u(t) - u(t-C)|, C = check_every",
                       "check_every": check, "sides": "log-uniform [32, 512] per axis",
                       "parallelism": f"replicas{world}"},
            "run": main, "fp32_run": f32,
            "latency_vs_alone_fp32": {
                "sample": len(sample), "both_converged": len(both),
                "batched_p50_ms": float(np.percentile(lat32[sample[both]], 50)) if both else None,
                "batched_p99_ms": float(np.percentile(lat32[sample[both]], 99)) if both else None,
                "alone_p50_ms": float(np.percentile(np.array(alone)[both], 50)) if both else None,
                "alone_p99_ms": float(np.percentile(np.array(alone)[both], 99)) if both else None,
                "alone_sequential_total_ms": float(np.sum(alone))},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": profiled_traffic(f"batch_kernel_sweep16_{args.storage}"),
                         "peak_source": peak_kind, "bytes_per_lup": bpl,
                         "kernel": "batch_kernel (persistent, domains from an atomic queue; small domains "
                                   "K steps per load in shared memory) + batch_wide_kernel (tail phase)"},
            "cpu_baseline": cpu,
            "gpu_launches": None,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)


class ReferenceTimer:
    """The host-compiled reference step on a crop (z, or y for 2-D) of the
    workload."""

    def __init__(self, w, nz: int, threads: int):
        from oracle.oracle import Case, Reference
        lx, ly, lz = w.length
        if w.dim == 2:
            ly_c, lz_c = ly, 1
        else:
            ly_c, lz_c = ly, (lz if nz <= 0 else max(1, min(nz, lz)))
        n = lx * ly_c * lz_c
        a = w.arrays

        def crop(x, comp=False):
            if x is None:
                return None
            return x[:, :n] if comp else x[:n]
        f0 = None
        if w.init_type == 1:  # f_eq(rho, u), as lbmc_init does
            from oracle.oracle import Restatement
            tmp = Case(lattice=w.lattice, length=(lx, ly_c, lz_c))
            f0 = Restatement(tmp).equilibrium(crop(a["rho"]), crop(a["u"], True))
        case = Case(lattice=w.lattice, length=(lx, ly_c, lz_c), tau=w.tau, tau_mrt=w.tau_mrt,
                    c_smag=w.c_smag, collision_type=w.collision_type, forcing=w.forcing,
                    macro_bc=w.macro_bc, micro_bc=w.micro_bc,
                    geometry=crop(a.get("geometry")), force=crop(a.get("force"), True),
                    macro=crop(a.get("macro")), micro=crop(a.get("micro")),
                    rho=crop(a.get("rho")), u=crop(a.get("u"), True), f0=f0)
        variant = "patched" if (w.lattice == "d3q15" or w.c_smag > 0) else "asis"
        self.ref = Reference(case, variant, nthreads=threads)
        self.n, self.threads = n, threads
        shape = f"{lx}x{ly_c}" if w.dim == 2 else f"{lx}x{ly_c}x{lz_c}"
        whole = (lx, ly_c, lz_c)[:w.dim] == tuple(w.length[:w.dim])
        self.sample = (f"the whole {shape} workload" if whole else f"{shape} crop of the workload") + \
            f", FP64, {variant} reference step"

    def rate(self, steps: int) -> float:
        """Lattice updates per second over `steps` reference steps."""
        t = time.perf_counter()
        self.ref.run(steps)
        return self.n * steps / (time.perf_counter() - t)

    def close(self):
        self.ref.close()


def cpu_reference_rate(w, nz: int, budget_s: float, threads: int):
    """Reference steps on the crop until about budget_s seconds of CPU work."""
    timer = ReferenceTimer(w, nz, threads)
    timer.rate(1)  # page-in
    steps, t_total = 0, 0.0
    while t_total < budget_s and steps < 1000:
        t = time.perf_counter()
        timer.ref.run(1)
        t_total += time.perf_counter() - t
        steps += 1
    timer.close()
    return timer.n * steps / t_total, f"{timer.sample}, {steps} steps ({t_total:.1f} s)"


BATCH_TAU, BATCH_G = 1.0, 1e-6


def _reference_domain(job):
    """One sweep domain through the host-compiled reference step (a worker
    process: the reference keeps its DomainConstant in a file-scope global,
    so one process runs one domain at a time, as LBM-C does)."""
    geometry, steps = job
    from oracle.oracle import Case, Reference
    ly, lx = geometry.shape
    n = lx * ly
    if steps == 0:
        Reference(Case(lattice="d2q9", length=(4, 4, 1)), "asis", nthreads=1).close()
        return 0
    force = np.zeros((2, n))
    force[0] = BATCH_G
    case = Case(lattice="d2q9", length=(lx, ly, 1), tau=BATCH_TAU, collision_type=1, forcing=True,
                geometry=geometry.reshape(n), force=force)
    ref = Reference(case, "asis", nthreads=1)
    ref.run(steps)
    ref.close()
    return n * steps


def reference_batch_rate(geoms, sample, steps, threads):
    """The host-compiled reference step (D2Q9 NTPOR + Guo, FP64) on a sample
    of the sweep's domains, one domain per worker process and one process
    per host thread: total lattice updates per second and a description.
    The pool is spawned (never forked after CUDA use) and warmed up before
    the timer starts."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor

    with ProcessPoolExecutor(max_workers=threads, mp_context=mp.get_context("spawn")) as pool:
        list(pool.map(_reference_domain, [(geoms[0], 0)] * threads))
        t = time.perf_counter()
        lups = sum(pool.map(_reference_domain, [(geoms[d], steps) for d in sample]))
        secs = time.perf_counter() - t
    nodes = int(sum(geoms[d].size for d in sample))
    return lups / secs, (f"{len(sample)} seeded domains of the sweep ({nodes} nodes), {steps} steps each, "
                         f"one domain per process on {threads} host threads, FP64 reference step "
                         f"({secs:.1f} s)")


def batch_sample(ndomains, size=64):
    return np.random.default_rng(17).choice(ndomains, size=min(size, ndomains), replace=False)


def run_reference_arm(args, world, rank):
    if rank != 0:
        return
    if args.workload == "batch":
        import workloads
        geoms = workloads.batch_sweep(args.domains, seed=5, tau=BATCH_TAU)
        threads = os.cpu_count() or 1
        sample = batch_sample(len(geoms))
        rate, desc = reference_batch_rate(geoms, sample, max(1, args.steps), threads)
        value = rate / 1e9
        line = {"metric": metric_name(args), "value": value, "unit": UNIT, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": None,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded circles, IMB edges)", "impl": "reference",
                "config": {"workload": "batch_d2q9_ntpor_guo_circles", "domains": args.domains,
                           "sample": desc, "threads": threads},
                "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                                 "sample": desc},
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    w = build_workload(args)
    threads = os.cpu_count() or 1
    timer = ReferenceTimer(w, args.ref_nz, threads)
    # Each step is a bounded sample: a z-crop sized from one timed step so
    # that warm-up and K steps end within REF_ARM_SECONDS.
    timer.ref.run(1)  # page-in and thread start
    t = time.perf_counter()
    timer.ref.run(1)
    total = (args.steps + max(1, args.warmup)) * (time.perf_counter() - t)
    lz_now = timer.n // (w.length[0] * w.length[1]) if w.dim == 3 else 1
    if w.dim == 3 and total > REF_ARM_SECONDS and lz_now > 1:
        timer.close()
        timer = ReferenceTimer(w, max(1, int(lz_now * REF_ARM_SECONDS / total)), threads)
    timer.rate(max(1, args.warmup))
    t_total, steps = 0.0, 0
    for _ in range(args.steps):
        t = time.perf_counter()
        timer.ref.run(1)
        t_total += time.perf_counter() - t
        steps += 1
    timer.close()
    value = timer.n * steps / t_total / 1e9
    line = {
        "metric": metric_name(args), "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_total / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)", "impl": "reference",
        "config": {"workload": w.name, "length": list(w.length), "nodes": w.n, "sample": timer.sample,
                   "storage": "f64", "threads": threads,
                   # the sampled crop's FP64 populations against the host's caches
                   "l2": ("sample larger than the host's last-level cache"
                          if timer.n * w.q * 8 > 64e6 else "sample may fit the host's caches")},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"{timer.sample}, {steps} steps"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------- GPU arm

def run_ours(args, world, rank, local):
    import torch

    import lbmc
    import workloads
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    w = build_workload(args)
    q = w.q
    stream = torch.cuda.Stream(device)
    kernel = {"auto": lbmc.KERNEL_AUTO, "direct": lbmc.KERNEL_DIRECT,
              "pipelined": lbmc.KERNEL_PIPELINED}[args.kernel]
    streaming = lbmc.STREAM_AA if args.streaming == "aa" else lbmc.STREAM_SHIFT
    eng = workloads.engine_for(lbmc, w, args.storage, device=local, kernel=kernel, streaming=streaming)
    lbmc.check(lbmc.library().lbmc_set_stream(eng.h, stream.cuda_stream))
    mlp = None
    if args.workload == "closure" and args.closure_passes > 0:
        # The network's cost does not depend on its weights: seeded hidden
        # layers with an open input range, so every node evaluates the
        # whole network, and an output layer (W3 = 0, b3 = 1) that gives
        # nu_t = 2e-3 everywhere, so the under-resolved box stays stable
        # for any number of steps.  (--closure-passes 0: the same box with
        # Smagorinsky alone.)
        mlp = lbmc.Mlp(seed=1, device=local)
        params = mlp.params()
        params[1280:1312] = 0.0  # W3
        params[1312] = 1.0       # b3
        mlp.set_params(params)
        mlp.set_normalization(np.zeros(6), np.full(6, 10.0), target_scale=2e-3)
        mlp.attach(eng, iterations=args.closure_passes)
    # warm-up
    eng.iterate(args.warmup, lbmc.SYNC)
    dist_barrier(world, device)
    torch.cuda.synchronize(device)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        start.record(stream)
        eng.iterate(args.steps, 0)
        stop.record(stream)
        stop.synchronize()
    torch.cuda.synchronize(device)
    dist_barrier(world, device)
    ms = start.elapsed_time(stop)
    rate, t_max = aggregate_rate(w.n * args.steps, ms / 1e3, world, device)
    ms_max = t_max * 1e3
    value = rate / 1e9
    eng.iterate(1, lbmc.REDUCE_DIAG | lbmc.SYNC)
    diag = eng.diag()
    eng.close()

    # Roofline of the dominant kernel (the fused step): algorithmic bytes per
    # launch over the average launch time in the timed region.
    bpl = algorithmic_bytes_per_lup(q, args.storage)
    per_launch_s = (ms / 1e3) / args.steps
    achieved = w.n * bpl / per_launch_s / 1e9
    peak, peak_kind = measured_peak()
    tag = f"step_kernel_{args.workload}{args.size}_{args.storage}"
    if args.kernel == "pipelined":
        tag = f"step_pipelined_kernel_{args.workload}{args.size}_{args.storage}"
    elif args.streaming == "aa":
        # AA runs over 64-node tiles when Lx is a multiple of 64.
        tag += "_aa" if w.length[0] % 64 == 0 else "_aa_untiled"
    traffic = profiled_traffic(tag)
    layout_name = args.streaming
    if args.streaming == "aa":
        layout_name = "tiled aa" if w.length[0] % 64 == 0 else "aa"

    # End to end through the C ABI with host buffers.
    e2e = None
    if not args.no_e2e:
        times, phases = [], []
        h2d = w.host_bytes()
        d2h = w.n * 8 * (1 + w.dim)

        # Inputs and outputs in pinned host memory: the workload's arrays
        # are copied into page-locked buffers once, before any job, and the
        # outputs exist before the job too (LBM-C fills the host Domain
        # arrays that set-up allocated, index.cu:196-216).
        def pinned(a):
            t = torch.empty(a.shape, dtype=torch.from_numpy(a[:0]).dtype, pin_memory=True)
            out = t.numpy()
            out[...] = a
            keep_pinned.append(t)
            return out
        keep_pinned = []
        w = dataclasses.replace(w, arrays={k: (None if v is None else pinned(np.ascontiguousarray(v)))
                                           for k, v in w.arrays.items()})
        rho_out = pinned(np.zeros(w.n))
        u_out = pinned(np.zeros((w.dim, w.n)))
        for k in range(args.e2e_reps + 1):
            torch.cuda.synchronize(device)
            t = time.perf_counter()
            e = workloads.engine_for(lbmc, w, args.storage, device=local, kernel=kernel,
                                     streaming=streaming)
            if mlp is not None:
                mlp.attach(e, iterations=args.closure_passes)
            t1 = time.perf_counter()
            e.iterate(E2E_STEPS, lbmc.STORE_MACROS | lbmc.SYNC)
            t2 = time.perf_counter()
            e.rho(out=rho_out)
            e.u(out=u_out)
            t3 = time.perf_counter()
            # LBM-C's program ends without freeing (index.cu:61-153), so the
            # job ends at the fetch; lbmc_destroy is timed and reported on
            # its own (the driver's cudaFree of ~1.5 GB takes 0.005 s, now
            # and then 0.1-0.5 s).
            e.close()
            t4 = time.perf_counter()
            if k > 0:  # the first job pays for context and module loading
                times.append(t3 - t)
                phases.append({"init": round(t1 - t, 4), "steps": round(t2 - t1, 4),
                               "fetch": round(t3 - t2, 4), "destroy_untimed": round(t4 - t3, 4)})
        # The median job counts (the list is reported): now and then the
        # driver's cudaMalloc / cudaFree of the ~1.5 GB a handle holds takes
        # 0.1-0.5 s instead of milliseconds, in one job of a run.
        e2e_rate, _ = aggregate_rate(w.n * E2E_STEPS, float(np.median(times)), world, device)
        # Each job moves its inputs in once and its result out once; per step
        # that is the job's bytes over its steps.
        e2e = {"value": e2e_rate / 1e9, "unit": UNIT, "host_memory": "pinned (page-locked) input and output arrays",
               "h2d_bytes_per_step": int(round(h2d / E2E_STEPS)),
               "d2h_bytes_per_step": int(round(d2h / E2E_STEPS)),
               "h2d_bytes_per_job": int(h2d), "d2h_bytes_per_job": int(d2h),
               "steps_per_job": E2E_STEPS,
               "job": f"lbmc_init from host arrays + {E2E_STEPS} steps + fetch rho,u into host arrays"
                      " allocated before the job (lbmc_destroy after the timer, as LBM-C exits without"
                      " freeing); median of the timed jobs",
               "seconds_per_job": [round(x, 4) for x in times], "phases": phases}

    # Reduced-precision storage: the velocity error of this storage against
    # an FP64-storage run of the same workload and step count (outside the
    # timed region).
    accuracy = None
    if rank == 0 and STORAGE_BYTES[args.storage] == 2 and args.accuracy_steps > 0 and mlp is None:
        fields = {}
        for st in ("f64", args.storage):
            e = workloads.engine_for(lbmc, w, st, device=local, kernel=kernel, streaming=streaming)
            e.iterate(args.accuracy_steps, lbmc.STORE_MACROS | lbmc.SYNC)
            fields[st] = e.u()
            e.close()
        u64, u2 = fields["f64"], fields[args.storage]
        accuracy = {"steps": args.accuracy_steps, "reference": "f64 storage, same engine and workload",
                    "u_rel_l2": float(np.linalg.norm(u2 - u64) / np.linalg.norm(u64)),
                    "u_rel_max": float(np.abs(u2 - u64).max() / np.abs(u64).max())}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        rate, sample = cpu_reference_rate(w, args.ref_nz, args.cpu_seconds, threads)
        cpu = {"value": rate / 1e9, "unit": UNIT, "cores": threads, "kind": "reference",
               "sample": sample}

    if rank == 0:
        line = {
            "metric": metric_name(args), "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": args.storage, "data": "synthetic (seeded)",
            "config": {"workload": w.name, "length": list(w.length), "nodes": w.n,
                       "storage": args.storage, "streaming": args.streaming,
                       "compute": "f32" if args.storage != "f64" else "f64",
                       "params": {k: (round(v, 6) if isinstance(v, float) else v)
                                  for k, v in w.params.items()},
                       "parallelism": f"replicas{world}",
                       "l2": ("inputs larger than L2 (no flush)" if w.n * w.q * 2 > 126e6
                              else "inputs fit in L2: steady-state in-cache rate")},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_source": peak_kind,
                         "bytes_per_lup": bpl,
                         "kernel": ("step_pipelined_kernel (bulk-copy row pipeline, fused stream+BC+collide)"
                                    if args.kernel == "pipelined" else
                                    f"step_kernel (direct loads, fused stream+BC+collide, {layout_name} layout)"
                                    + (f", learned closure {args.closure_passes} pass(es) on the tensor cores:"
                                       " SFU/issue-bound, not HBM-bound" if mlp is not None else ""))},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": args.steps,
            "clocks": clk.summary(),
            "accuracy_vs_f64": accuracy,
            "diag": {"mass": diag.mass, "kinetic_energy": diag.kinetic_energy,
                     "nonfinite": diag.nonfinite},
        }
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    # 10000 steps of the default workload take about 3 s: long enough for
    # the clock record to hold tens of samples, short of a minute.
    ap.add_argument("--steps", type=int, default=10000)
    ap.add_argument("--warmup", type=int, default=50)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--storage", choices=list(STORAGE_BYTES), default="f32")
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--kernel", choices=["auto", "direct", "pipelined"], default="auto")
    ap.add_argument("--streaming", choices=["shift", "aa"], default="aa")
    ap.add_argument("--closure-passes", type=int, default=1)
    ap.add_argument("--workload", choices=list(WORKLOAD_METRIC), default="porous")
    ap.add_argument("--domains", type=int, default=4096)
    ap.add_argument("--batch-cap", type=int, default=20000)
    ap.add_argument("--wide-min-nodes", type=int, default=0,
                    help="batched sweep: HBM domains of at least this many nodes are stepped over "
                         "every SM, the others one block per domain (0 = the storage's default)")
    ap.add_argument("--wide-below", type=int, default=0,
                    help="batched sweep: the one-block-per-domain HBM domains join the wide path "
                         "once fewer than this many run (0 = half the SMs, -1 = never)")
    ap.add_argument("--alone-sample", type=int, default=32)
    ap.add_argument("--e2e-reps", type=int, default=5)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--ref-nz", type=int, default=0,
                    help="reference step on the first NZ planes of a 3-D workload (0 = all; the "
                         "reference arm still crops if its run would pass %d s)" % REF_ARM_SECONDS)
    ap.add_argument("--accuracy-steps", type=int, default=5000,
                    help="2-byte storages: steps of the FP64 comparison run reported in the line "
                         "(0 = none)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    world, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference_arm(args, world, rank)
        elif args.workload == "batch":
            run_batch(args, world, rank, local)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
