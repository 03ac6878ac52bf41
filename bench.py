#!/usr/bin/env python3
"""Throughput of the 2-body + 3-body path: dimers+trimers/s with forces, 2048 H2O.

One step = one Get2B + one Get3B of the 2048-water box (cubic 39.44 A, 2b
cutoff 9 A, 3b cutoff 7 A, seed 0): FixMonomerCoordinates, the n-mer search,
every evaluator with energies, gradients and virial, both terms in one call
(mbx_energy_2b3b: the two terms side by side on the GPU).  Units = listed
n-mers (dimers within 9 A + trimers by the reference's AddClusters rule within
7 A), the reference's unit of work.

* value: device-resident (coordinates and gradients in HBM), CUDA events on
  the library's stream, L2 flushed between steps (inputs are far smaller than
  the 126 MB L2), FP64 path;
* e2e: the same through the public API (mbx_b200.system.System,
  TwoAndThreeBodyEnergy) with pinned host buffers, host<->device copies
  inside, wall clock per step;
* mixed: MB-pol 3b on the tensor cores (the shifted-basis polynomial as a
  quadratic form, FP16 split operands, FP32 accumulation; variables, chain
  rule and sums FP64), its throughput and its energy and force errors
  against the FP64 path;
* roofline: the MB-pol 3b evaluation kernel launched alone (3b-only calls,
  L2 flushed), algorithmic flops counted from the reference's gradient
  program (mbx_b200/data/flops.json) over its CUDA-event duration, against
  the measured FP64 FMA peak of this GPU;
* cpu_baseline: the reference's own CPU path (oracle/_ref, built from the
  reference sources) on the host's cores, bounded sample.

``--impl reference`` times the reference CPU implementation alone on the same
workload.  With torchrun (N>1) every rank runs an independent replica (the
path needs no exchange between replicas); value = all ranks' units / max time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "dimers+trimers/s with forces, 2048 H2O; FP32-mixed vs FP64 GPU at <=1e-6 rel E"
CUT2, CUT3 = 9.0, 7.0


def workload():
    from mbx_b200 import workloads
    ids, xyz, box = workloads.water_2048(0)
    return ids, xyz, box


def config(n):
    return {"workload": "2048 H2O periodic box 39.44 A (1.0 g/cm3), cutoffs 9/7 A, seed 0",
            "monomers": 2048, "cutoff2b": CUT2, "cutoff3b": CUT3, "l2": "flushed between steps (256 MiB write)",
            "parallelism": "replicas" if n > 1 else "single"}


class Clocks:
    """Samples nvidia-smi during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []          # (arrival time, csv line)
        self.window = None       # (t0, t1) of the timed region, time.monotonic()

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            # line-buffered (stdbuf), so that a sample's arrival time is its time
            self.proc = subprocess.Popen(["stdbuf", "-oL", "nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))

    def wait_first(self, work, limit=10.0):
        """Runs work() until the sampler has produced a line (or limit s)."""
        t0 = time.monotonic()
        while self.proc and not self.lines and time.monotonic() - t0 < limit:
            work()

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for t, line in self.lines:
            if self.window and not (self.window[0] <= t <= self.window[1]):
                continue
            p = [x.strip() for x in line.split(",")]
            if len(p) < 7:
                continue
            try:
                sm.append(float(p[0]))
                mx.append(float(p[1]))
            except ValueError:
                continue
            for k, name in enumerate(names):
                if p[3 + k].lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def ref_cpu(ids, xyz, box, seconds=12.0, threads=None, label="2048 H2O"):
    """The reference CPU path (oracle/_ref) on this host: (units/s, cores, sample)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import mbx_oracle as mo
    if not mo.RefSystem.available():
        return None
    threads = threads or os.cpu_count()
    mo.RefSystem.set_threads(threads)
    r = mo.RefSystem(ids, xyz, box, CUT2, CUT3)
    nd = len(r.pair_list(2, CUT2))
    nt = len(r.pair_list(3, CUT3))
    e2 = r.energy(2)
    e3 = r.energy(3)
    t0 = time.perf_counter()
    steps = 0
    while True:
        r.energy(2)
        r.energy(3)
        steps += 1
        if time.perf_counter() - t0 > seconds:
            break
    dt = (time.perf_counter() - t0) / steps
    return {"value": (nd + nt) / dt, "unit": "n-mers/s", "cores": threads, "kind": "reference",
            "sample": "%d full steps (TwoBodyEnergy(true)+ThreeBodyEnergy(true), %s), %.2f s/step, "
                      "OMP_NUM_THREADS=%d" % (steps, label, dt, threads), "ms_per_step": dt * 1e3,
            "energies": {"E2B": e2, "E3B": e3}}


def run_reference(args, rank):
    if rank != 0:
        return 0
    ids, xyz, box = workload()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import mbx_oracle as mo
    if not mo.RefSystem.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libmbx_ref.so not built"}))
        return 0
    threads = os.cpu_count()
    mo.RefSystem.set_threads(threads)
    r = mo.RefSystem(ids, xyz, box, CUT2, CUT3)
    units = len(r.pair_list(2, CUT2)) + len(r.pair_list(3, CUT3))
    # one reference step takes ~0.4 s on 16 cores: the sample is bounded so
    # that the run ends within a minute or two whatever --steps is
    nwarm = min(args.warmup, 2)
    nsteps = max(1, min(args.steps, 20))
    for _ in range(nwarm):
        r.energy(2)
        r.energy(3)
    times = []
    for _ in range(nsteps):
        t0 = time.perf_counter()
        r.energy(2)
        r.energy(3)
        times.append(time.perf_counter() - t0)
    dt = sum(times) / len(times)
    v = units / dt
    out = {"metric": METRIC, "value": v, "unit": "n-mers/s", "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config(1), "impl": "reference",
           "cpu_baseline": {"value": v, "unit": "n-mers/s", "cores": threads, "kind": "reference",
                            "sample": "%d timed steps (after %d warm-up) of TwoBodyEnergy(true)+ThreeBodyEnergy(true) "
                                      "of the compiled reference, OMP_NUM_THREADS=%d" % (nsteps, nwarm, threads)},
           "e2e": {"value": v, "unit": "n-mers/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


def batched_leg(args, local, flush, fp64_value, dist=None, world=1):
    """32 beads of the 2048-water box (sigma 0.05 A) + 64 gas-phase clusters of
    8-512 molecules: mixed precision, builder shapes autotuned, the whole 2b+3b
    device sequence replayed from CUDA graphs; errors against the FP64
    evaluation of the same batch."""
    import torch
    from mbx_b200 import workloads
    from mbx_b200.batch import Batch
    from mbx_b200 import capi
    cfgs = workloads.batch_beads_clusters(32, 64, seed=0)
    stream = torch.cuda.current_stream()
    bctx = capi.Context(local, stream.cuda_stream)
    b = Batch(cfgs, CUT2, CUT3, device=local, context=bctx)
    tuned = {}
    for nb in (2, 3):
        knobs, ms = b.tune(nb, mixed=True)
        tuned[str(nb)] = dict(knobs, ms=ms)
    e64 = sum(b.energy_2b3b(graph=False))
    for _ in range(max(args.warmup, 3)):
        b.grad.zero_()
        b.energy_2b3b(mixed=True)
    listed2, eval2 = b.ctx.counts(2)
    listed3, eval3 = b.ctx.counts(3)
    times = []
    emx = None
    steps = max(3, min(args.steps, 20))
    for _ in range(steps):
        flush.zero_()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        z = torch.cuda.Event(enable_timing=True)
        # an NVTX range per timed step, so that a profiler can select the
        # step's launches (ncu --nvtx --nvtx-include "mbx_batched_step/")
        torch.cuda.nvtx.range_push("mbx_batched_step")
        a.record(stream)
        b.grad.zero_()
        t0, t1 = b.energy_2b3b(mixed=True)   # replays the graph on the same stream
        z.record(stream)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        times.append(a.elapsed_time(z))
        emx = t0 + t1
    bctx.close()
    from mbx_b200 import replicas
    ms, = replicas.max_over_ranks([sum(times) / len(times)], dist, "cuda")
    units = listed2 + listed3
    rel = np.abs(emx - e64) / np.abs(e64)
    return {"workload": "32 beads of the 2048-H2O box (Gaussian sigma 0.05 A per atom) + 64 gas-phase water "
                        "clusters of 8-512 molecules at 0.0334 /A^3, seed 0; cutoffs 9/7 A",
            "configurations": len(cfgs), "molecules": int(sum(len(c[0]) for c in cfgs)),
            "value": replicas.throughput(units, ms, world), "unit": "n-mers/s", "ms_per_step": ms,
            "units_per_step": {"dimers": listed2, "trimers": listed3, "evaluated_dimers": eval2,
                               "evaluated_trimers": eval3},
            "dtype": "mixed (3b: quadratic form over a shifted basis on the tensor cores, FP16 split operands, "
                     "FP32 accumulation; 2b f64)", "cuda_graph": True,
            "timing": "CUDA events on the bench's stream around the gradient reset and the graph replay of "
                      "both terms (the library runs on that stream), L2 flushed before each step",
            "autotuned": tuned,
            "max_rel_err_E_per_configuration": float(rel.max()),
            "speedup_vs_fp64_plain": replicas.throughput(units, ms, world) / fp64_value}


def salt_leg(args, local, flush, cpu=True):
    """A 1 M NaCl solution at the headline size: the 2048-site lattice box with
    32 Na+ and 32 Cl- in place of waters, FP64 through mbx_energy_2b3b
    (MB-pol water, the Na+/Cl- - water 2b and 3b, Na+-Na+, Cl--Cl-, Na+-Cl-
    2b); energies against the compiled reference on the same box."""
    import torch
    from mbx_b200 import capi, system as msys, workloads
    ids, xyz, box = workloads.ion_water_box(["na+", "cl-"] * 32, n_side=14, n_mol=2048, L=39.44, seed=0)
    stream = torch.cuda.current_stream()
    ctx = capi.Context(local, stream.cuda_stream)
    s = msys.from_arrays(ids, xyz, box, CUT2, CUT3, context=ctx)
    sites = torch.tensor(s.sites, dtype=torch.float64, device="cuda")
    grad = torch.zeros_like(sites)
    vir = np.zeros(9)
    for _ in range(max(args.warmup, 3)):
        grad.zero_()
        e2, e3 = ctx.energy_2b3b(sites, grad, vir)
    listed2, eval2 = ctx.counts(2)
    listed3, eval3 = ctx.counts(3)
    times = []
    for _ in range(max(3, min(args.steps, 50))):
        flush.zero_()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        grad.zero_()
        e2, e3 = ctx.energy_2b3b(sites, grad, vir)
        b.record(stream)
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
    ctx.close()
    ms = sum(times) / len(times)
    units = listed2 + listed3
    out = {"workload": "1 M NaCl: 1984 H2O + 32 Na+ + 32 Cl- on the 2048-site lattice box 39.44 A, seed 0; "
                       "cutoffs 9/7 A",
           "value": units / (ms * 1e-3), "unit": "n-mers/s", "ms_per_step": ms, "dtype": "f64",
           "units_per_step": {"dimers": listed2, "trimers": listed3, "evaluated_dimers": eval2,
                              "evaluated_trimers": eval3},
           "energies": {"E2B": e2, "E3B": e3}}
    if cpu:
        cb = ref_cpu(ids, xyz, box, seconds=8.0, label="1 M NaCl, 2048 sites")
        if cb:
            out["cpu_reference"] = {k: cb[k] for k in ("value", "unit", "cores", "sample", "ms_per_step")}
            out["rel_err_E2B_vs_reference"] = abs(e2 - cb["energies"]["E2B"]) / abs(cb["energies"]["E2B"])
            out["rel_err_E3B_vs_reference"] = abs(e3 - cb["energies"]["E3B"]) / abs(cb["energies"]["E3B"])
            out["speedup_vs_reference_cpu"] = cb["ms_per_step"] / ms
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision leg")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-configurations leg")
    ap.add_argument("--no-salt", action="store_true", help="skip the NaCl-solution leg")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank)

    import torch
    from mbx_b200 import capi, replicas, system as msys
    from mbx_b200.tables import load_fit  # noqa: F401

    torch.cuda.set_device(local)
    # a stream of our own: the library's kernels and the bench's CUDA events
    # on the same (non-default) stream
    torch.cuda.set_stream(torch.cuda.Stream(local))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    ids, xyz, box = workload()
    stream = torch.cuda.current_stream()
    ctx = capi.Context(local, stream.cuda_stream)
    peaks = capi.fma_peaks(local)
    flops = json.load(open(os.path.join(ROOT, "mbx_b200", "data", "flops.json")))

    # ---------------- device-resident steps
    sys_d = msys.from_arrays(ids, xyz, box, CUT2, CUT3, context=ctx)
    sites = torch.tensor(sys_d.sites, dtype=torch.float64, device="cuda")
    grad = torch.zeros_like(sites)
    vir = np.zeros(9)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")

    def step(mixed=False):
        # Get2B + Get3B: both terms in one call, side by side on the GPU
        grad.zero_()
        e2, e3 = ctx.energy_2b3b(sites, grad, vir, mixed=mixed)
        return e2, e3, ctx.timing()

    for _ in range(max(args.warmup, 3)):
        step()
    listed2, eval2 = ctx.counts(2)
    listed3, eval3 = ctx.counts(3)
    units = listed2 + listed3

    def timed(mixed):
        times, launches, energies = [], 0, None
        for _ in range(args.steps):
            flush.zero_()
            if dist:
                dist.barrier()
            torch.cuda.synchronize()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            e2, e3, tm = step(mixed)
            b.record(stream)
            torch.cuda.synchronize()
            times.append(a.elapsed_time(b))
            launches += tm[2]
            energies = (e2, e3)
        return times, launches, energies

    def kernel_3b(mixed, steps):
        """Duration of the 3b evaluation kernel launched alone (CUDA events
        on the library's stream), L2 flushed before each call."""
        evs = []
        for _ in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            grad.zero_()
            ctx.energy(3, sites, grad, vir, mixed=mixed)
            evs.append(ctx.timing()[1])
        return evs

    clk = Clocks(local).__enter__()
    clk.wait_first(step)
    t_begin = time.monotonic()
    t64, launches, (e2_64, e3_64) = timed(False)
    g64 = grad.cpu().numpy()
    ev64 = kernel_3b(False, max(3, min(args.steps, 20)))
    if not args.no_mixed:
        for _ in range(max(args.warmup, 3)):
            step(True)
        tmx, launches_mx, (e2_mx, e3_mx) = timed(True)
        grad.zero_()
        ctx.energy_2b3b(sites, grad, vir, mixed=True)
        gmx = grad.cpu().numpy()
        evmx = kernel_3b(True, max(3, min(args.steps, 20)))
        # per-term forces of the two paths (2b and 3b gradients separately)
        grad.zero_()
        ctx.energy(2, sites, grad, vir)
        g2_64 = grad.cpu().numpy()
        grad.zero_()
        ctx.energy(2, sites, grad, vir, mixed=True)
        g2_mx = grad.cpu().numpy()
    else:
        tmx = list(t64)

    ms = sum(t64) / len(t64)
    ms_mx = sum(tmx) / len(tmx)
    ms, ms_mx = replicas.max_over_ranks([ms, ms_mx], dist, "cuda")
    value = replicas.throughput(units, ms, world)

    # ---------------- end to end through the public API (host buffers)
    sys_h = msys.from_arrays(ids, xyz, box, CUT2, CUT3, context=ctx)
    pinned_sites = torch.tensor(sys_h.sites, dtype=torch.float64).pin_memory()
    pinned_grad = torch.zeros_like(pinned_sites).pin_memory()
    sys_h.sites = pinned_sites.numpy()
    sys_h.grad = pinned_grad.numpy()
    for _ in range(max(args.warmup, 3)):
        sys_h.TwoAndThreeBodyEnergy(True)
    e2e_t = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sys_h.TwoAndThreeBodyEnergy(True)
        g23 = sys_h.GetRealGrads()
        e2e_t.append(time.perf_counter() - t0)
    e2e_ms = 1e3 * sum(e2e_t) / len(e2e_t)
    e2e_ms, = replicas.max_over_ranks([e2e_ms], dist, "cuda")
    nbytes = 8 * sys_h.sites.size
    h2d = nbytes                     # the coordinates, once per step
    d2h = 2 * nbytes + 2 * 8 * 8     # wrapped coordinates + gradient; both terms' results

    # ---------------- roofline of the MB-pol 3b evaluation kernel
    kern_ms = sum(ev64) / len(ev64)
    achieved = eval3 * flops["mbpol3b"]["flops"] / (kern_ms * 1e-3) / 1e12
    roofline = {"bound": "fp64-fma", "kernel": "holder_lock_kernel<mbpol3b_T, mbpol3b_CC, HM_GRAD_FP64>",
                "achieved": achieved,
                "peak": peaks["fp64_tflops"], "unit": "TFLOP/s", "frac": achieved / peaks["fp64_tflops"],
                "traffic": None,
                "traffic_note": "DRAM bytes are not measured inside this run (no profiler here); the kernel's "
                                "inputs (0.2 MB of coordinates, 0.2 MB of n-mer records) are L2-resident",
                "note": "algorithmic flops = evaluated trimers x %d (reference gradient program, "
                        "mbx_b200/data/flops.json); peak = FP64 FMA pipe measured on this GPU by "
                        "mbx_fma_peaks (MEASURED_PEAKS.json has no FP64 figure)" % flops["mbpol3b"]["flops"],
                "fp32_peak": peaks["fp32_tflops"], "kernel_ms": kern_ms, "evaluated_trimers": eval3}

    out = {"metric": METRIC, "value": value, "unit": "n-mers/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config(world),
           "units_per_step": {"dimers": listed2, "trimers": listed3, "evaluated_dimers": eval2,
                              "evaluated_trimers": eval3},
           "energies": {"E2B": e2_64, "E3B": e3_64},
           "e2e": {"value": world * units / (e2e_ms * 1e-3), "unit": "n-mers/s", "h2d_bytes_per_step": h2d,
                   "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms,
                   "api": "mbx_b200.system.System.TwoAndThreeBodyEnergy (mbx_energy_2b3b, host arrays)"},
           "gpu_launches": launches, "roofline": roofline,
           "fma_peaks_tflops": peaks}
    if not args.no_mixed:
        g3_64, g3_mx = g64 - g2_64, gmx - g2_mx
        out["mixed"] = {"value": world * units / (ms_mx * 1e-3), "ms_per_step": ms_mx,
                        "dtype": "3b: quadratic form over a shifted FP32 basis on the tensor cores (tcgen05, FP16 "
                                 "split operands, FP32 accumulation), f64 variables, switch, chain rule "
                                 "and sums; 2b: f64",
                        "error_vs": "FP64 path of the same run (within 1e-10 of the reference)",
                        "rel_err_E2B": abs(e2_mx - e2_64) / abs(e2_64), "rel_err_E3B": abs(e3_mx - e3_64) / abs(e3_64),
                        "rel_err_E": abs((e2_mx + e3_mx) - (e2_64 + e3_64)) / abs(e2_64 + e3_64),
                        "max_abs_force_err_2b": float(np.abs(g2_mx - g2_64).max()),
                        "max_abs_force_err_3b": float(np.abs(g3_mx - g3_64).max()),
                        "rms_force_err": float(np.sqrt(((gmx - g64) ** 2).mean())),
                        "max_abs_force": float(np.abs(g64).max()), "force_unit": "kcal/mol/A",
                        "speedup_vs_fp64": ms / ms_mx}
        kmx = sum(evmx) / len(evmx)
        amx = eval3 * flops["mbpol3b"]["flops"] / (kmx * 1e-3) / 1e12
        out["mixed"]["roofline_3b"] = {"kernel": "pair_vars_kernel + qf_eval_kernel<mbpol3b_T, mbpol3b_Q> + "
                                                 "pair_finish_kernel (one evaluation, events around all three)",
                                       "kernel_ms": kmx,
                                       "achieved": amx, "unit": "TFLOP/s (reference flops)",
                                       "peak": peaks["fp32_tflops"], "frac": amx / peaks["fp32_tflops"],
                                       "bound": "fp32-fma"}
    if not args.no_batch:
        out["batched"] = batched_leg(args, local, flush, value, dist, world)
    # clocks sampled over the timed legs (FP64, mixed, batched)
    clk.window = (t_begin, time.monotonic())
    clk.__exit__()
    out["clocks"] = clk.summary()
    out["clocks"]["window"] = "FP64, mixed and batched timed legs"
    if not args.no_salt and rank == 0 and world == 1:
        out["salt"] = salt_leg(args, local, flush, cpu=not args.no_cpu_baseline)
    if rank == 0 and not args.no_cpu_baseline:
        cb = ref_cpu(ids, xyz, box)
        if cb:
            out["cpu_baseline"] = cb
    if rank == 0:
        print(json.dumps(out))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    ctx.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
