#!/usr/bin/env python
"""Benchmark of the four-phonon scattering-rate path on B200.

Workload (one GPU): the 16x16x16 diamond solve -- 2-atom cell, fcc a=5.43 A,
masses 28.085 amu, seeded Born-von Karman springs and N(0,5)/N(0,2) cubic and
quartic clusters (3rd-neighbour / 1st-neighbour cutoffs), T in {300, 700} K,
scalebroad 1.  One step is one RTA_driver_4ph pass over all 870 irreducible
modes with both temperatures fused (the matrix elements are contracted once
and weighted for both).  Synthetic inputs generated from a fixed seed.

Metric: four-phonon processes/s (surviving processes of the energy filter,
counted as the reference's N_plusplus+N_plusminus+N_minusminus).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N>1 runs one rank per GPU (torchrun); each rank solves the same cell at its
own pair of temperatures (300+10r, 700+10r K): per-GPU work is fixed
(weak scaling) and there is no collective on the data path.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT,):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "4ph processes/s"
UNIT = "processes/s"
WORKLOAD = "diamond 2-atom fcc a=5.43A, 16x16x16 q-grid, 3ph+4ph, 4ph RTA at T={300,700}K fused, scalebroad=1"

# The workloads: 1 is the benchmarked one (the default); 0, 2 and 3 are the
# other cells of the task, timed the same way when asked for with --config.
CONFIGS = {
    0: dict(kind="diamond", grid=6, temps=(300.0,),
            workload="diamond 2-atom fcc a=5.43A, 6x6x6 q-grid, 4ph RTA at T=300K, scalebroad=1"),
    1: dict(kind="diamond", grid=16, temps=(300.0, 700.0), workload=WORKLOAD),
    2: dict(kind="layered", grid=12, temps=(300.0,),
            workload="R-3m 4-atom layered cell (masses 6.94/58.93/16/16, a=2.82A, c/a=5), 12 branches, 12x12x12, "
                     "4th-order cutoff at the 2nd shell, 4ph RTA at T=300K"),
    3: dict(kind="zincblende", grid=24, temps=(100.0, 300.0, 500.0, 1000.0),
            workload="zincblende 2-atom a=4.78A masses 10.81/74.92, 24x24x24, 4ph RTA at T={100,300,500,1000}K "
                     "in one launch; full enumeration, and 2e6 sampled processes per mode and channel"),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", type=int, default=1, choices=sorted(CONFIGS),
                    help="workload (1 = the benchmarked 16^3 diamond solve)")
    ap.add_argument("--grid", type=int, default=None, help="override the q-grid edge of the workload")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--no-sampled", action="store_true")
    ap.add_argument("--mixed-modes", default="mixed,mixed_simt",
                    help="mixed precisions timed beside FP64: mixed (tensor cores), mixed_simt (CUDA cores)")
    ap.add_argument("--precision", choices=["fp64", "mixed", "mixed_simt"], default="fp64",
                    help="precision of the timed arm (fp64 = the plain drop-in, the benchmarked path)")
    ap.add_argument("--serve-budget", type=float, default=90.0,
                    help="estimated serial seconds of the served prefix of the request stream")
    ap.add_argument("--no-bte", action="store_true")
    return ap.parse_args()


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---------------------------------------------------------------------------- workload


def config_of(args):
    c = dict(CONFIGS[args.config])
    if args.grid:
        c["grid"] = args.grid
        c["workload"] = c["workload"] + f" (grid overridden: {args.grid}^3)"
    return c


def workload(cfg, rank=0):
    from fourphonon_b200 import system as S

    g = cfg["grid"]
    base = S.cached_solve(cfg["kind"], (g, g, g), temperatures=tuple(cfg["temps"]))
    if rank:
        import copy

        s = copy.copy(base)
        s.temperatures = [t + 10.0 * rank for t in cfg["temps"]]
        return s
    return base


def ref_flops_per_process(s):
    """The reference formulation's per-process work: 644*Ntri4 + 40 real flops
    (the 81-term Vp_pp/pm/mm contraction per cluster plus the weights)."""
    return 644.0 * s.ifc4.ntri + 40.0


def executed_flops(s, counters, npi):
    """FP64 operations the main kernel executes, from its work counters: 27 per
    broadening evaluation, 3 per window test, 27+25+12*nT+116*classes per
    contracted process and nb*9*Ntri*98 per reciprocal cluster table build."""
    nproc, ncontr, nsig, ncand, nz = counters[:5]
    nT = len(s.temperatures)
    f_sigma = 27.0
    f_test = 3.0
    f_proc = 27.0 + 25.0 + 12.0 * nT + 116.0 * npi
    f_z = s.nb * 9.0 * s.ifc4.ntri * 98.0  # per table build (one branch i, all j)
    return nsig * f_sigma + ncand * f_test + ncontr * f_proc + nz * f_z


def filter_stage(counters, kernel_ms, phase_a_frac, peak):
    """Phase A alone (enumeration and the energy-conservation filter): candidates
    tested per second and its FP64 work (27 per broadening evaluation, 3 per window
    test) over phase A's share of the kernel time, against the FP64 peak."""
    if not phase_a_frac or kernel_ms <= 0:
        return None
    t = kernel_ms / 1e3 * phase_a_frac
    nsig, ncand = float(counters[2]), float(counters[3])
    tf = (27.0 * nsig + 3.0 * ncand) / t / 1e12
    return {"candidates_per_s": nsig / t, "window_tests_per_s": ncand / t, "fp64_tflops": tf,
            "frac_of_fp64_peak": tf / peak if peak else None, "seconds": t,
            "note": "phase A time = the event-timed kernel duration x phase A's share of the CTA cycles; "
                    "candidates = broadening evaluations (q'', k, l kept by the channel's restrictions)"}


def npi_of(s):
    f = s.ifc4
    keys = set()
    for c in range(f.ntri):
        keys.add((tuple(f.cells[1, c] - f.cells[2, c]), int(f.atoms[2, c]), int(f.atoms[3, c])))
    return len(keys)


# ---------------------------------------------------------------------------- clocks


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        sm = []
        mx = None
        reasons = set()
        for s in self.samples:
            try:
                sm.append(float(s[1]))
                mx = float(s[2])
            except (ValueError, IndexError):
                continue
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for n, v in zip(names, s[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        load = [x for x in sm if mx and x > 0.3 * mx] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------- distributed plumbing


def dist_setup(n):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def all_max(world, x):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], device="cuda", dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def all_sum(world, x):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], device="cuda", dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


# ---------------------------------------------------------------------------- CPU baseline (oracle)


def cpu_sample(s, target_s=15.0, full=False):
    """Time the oracle (the C restatement of RTA_driver_4ph, OpenMP over modes
    and q' points) on the workload.  full=True times the whole driver (every
    mode, all three channels, first temperature).  Otherwise a bounded sample
    spread over the whole workload: (mode, q') pairs drawn uniformly at random,
    as many as take about target_s; processes/s of the sample stand for the
    whole."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    lib = O.lib()
    threads = lib.fp4o_num_threads()
    o = O.Oracle(s, T=s.temperatures[0])
    nm = s.nmodes
    if full:
        t0 = time.perf_counter()
        o.rta4()
        dt = time.perf_counter() - t0
        n = int(sum(x.sum() for x in O.Oracle(s).np4()[0]))
        return {"value": n / dt, "unit": UNIT, "cores": threads, "kind": "port",
                "sample": f"full oracle RTA_driver_4ph restatement: all {nm} modes, all q' points, three channels, "
                          f"T={s.temperatures[0]:.0f} K: {n} processes in {dt:.1f} s", "processes": n, "seconds": dt}
    # uniformly drawn (mode, q') pairs of the whole workload; a probe sizes the sample
    rng = np.random.default_rng(20240607)
    probe = 4 * max(threads, 1)
    t0 = time.perf_counter()
    o.rta4_pairs(rng.integers(0, nm, probe), rng.integers(0, s.nptk, probe))
    per_pair = max(time.perf_counter() - t0, 1e-3) / probe
    npairs = int(max(probe, min(nm * s.nptk, target_s / per_pair)))
    modes, qps = rng.integers(0, nm, npairs), rng.integers(0, s.nptk, npairs)
    t0 = time.perf_counter()
    n = o.rta4_pairs(modes, qps)
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"oracle RTA_driver_4ph restatement at {npairs} (mode, q') pairs drawn uniformly from the "
                      f"{nm} x {s.nptk} of the workload (seeded), three channels each, T={s.temperatures[0]:.0f} K: "
                      f"{n} processes in {dt:.1f} s; processes/s of the sample stand for the whole",
            "processes": n, "seconds": dt}


def run_reference(args):
    # rank 0 alone times the CPU oracle; the other ranks have no work and need no process group
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        # torchrun sets OMP_NUM_THREADS=1 for every rank; the one rank that works here takes
        # every host thread (read when the oracle's OpenMP runtime loads, below)
        os.environ["OMP_NUM_THREADS"] = str(len(os.sched_getaffinity(0)))
    cfg = config_of(args)
    s = workload(cfg)
    full = args.config == 0
    vals = []
    for w in range(args.warmup):
        cpu_sample(s, target_s=2.0, full=False)
    samples = []
    for k in range(args.steps):
        r = cpu_sample(s, target_s=10.0, full=full)
        samples.append(r)
        vals.append(r["value"])
    v = float(np.mean(vals))
    total_s = sum(r["seconds"] for r in samples)
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * total_s / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)", "impl": "reference",
            "config": {"workload": cfg["workload"], "sample": samples[-1]["sample"]},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": samples[-1]["cores"], "kind": "port",
                             "sample": samples[-1]["sample"]},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------- our arm


def fp64_dgemm_peak(torch):
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(3):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    return 2.0 * n ** 3 / best / 1e12


def time_steps(torch, ctx, s, steps, flush):
    """Run `steps` RTA_driver_4ph calls on torch's current stream; returns per-step
    device ms (CUDA events), main-kernel ms, processes, contracted and counters."""
    out = []
    for _ in range(steps):
        flush.zero_()  # write a buffer larger than L2 between steps
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        r = ctx.rta_driver_4ph(s)
        e1.record()
        torch.cuda.synchronize()
        nproc, ncontr, call_ms, kms, launches = ctx.stats()
        cyc = ctx.phase_cycles(full=True)
        item, phb = cyc[0], cyc[1]
        phases = {"phase_a_frac": (item - phb) / item if item else None, "phase_b_frac": phb / item if item else None}
        if cyc[2] or cyc[3]:  # the tensor-core contraction's own split, as fractions of phase B
            phases.update({"tc_tables_frac_of_b": cyc[2] / phb, "tc_gather_frac_of_b": cyc[3] / phb / 2,
                           "tc_product_weights_frac_of_b": cyc[4] / phb / 2, "tc_epilogue_frac_of_b": cyc[5] / phb / 2})
        out.append(dict(ms=e0.elapsed_time(e1), kms=kms, nproc=nproc, ncontr=ncontr, launches=launches,
                        counters=ctx.counters(), rates=r, phases=phases))
    return out


def pinned_copy(torch, s):
    """A shallow copy of the solve whose arrays live in pinned host memory."""
    import copy

    def pin(a, order):
        t = torch.empty(a.size * a.itemsize, dtype=torch.uint8, pin_memory=True)
        v = t.numpy().view(a.dtype)
        if order == "F":
            v = v.reshape(a.shape, order="F")
            v[...] = a
        else:
            v = v.reshape(a.shape)
            v[...] = a
        return v, t

    p = copy.copy(s)
    keep = []
    p.energy, t1 = pin(np.asfortranarray(s.energy), "F")
    p.velocity, t2 = pin(np.asfortranarray(s.velocity), "F")
    p.eig, t3 = pin(np.asfortranarray(s.eig), "F")
    ifc = copy.copy(s.ifc4)
    ifc.phi, t4 = pin(np.ascontiguousarray(s.ifc4.phi), "C")
    ifc.R, t5 = pin(np.ascontiguousarray(s.ifc4.R), "C")
    ifc.atoms, t6 = pin(np.ascontiguousarray(s.ifc4.atoms), "C")
    p.ifc4 = ifc
    keep += [t1, t2, t3, t4, t5, t6]
    p._pinned = keep
    h2d = sum(x.numel() for x in keep) + s.nlist * 4 + s.nptk * 12 + 8 * len(s.temperatures)
    return p, h2d


def rta_kappa(ctx, s, rate_total, t):
    """kappa_RTA = trace/3 of sum over branches, from per-mode total rates (device BTE kernels)."""
    tau = np.zeros_like(rate_total)
    nz = rate_total != 0
    tau[nz] = 1.0 / rate_total[nz]
    F = ctx.iteration0(s, tau)
    k = ctx.tconduct(s, F, T=s.temperatures[t]).reshape(3, 3, s.nb).sum(axis=2)
    return float(np.trace(k) / 3.0)


def bf16_peak():
    """Measured dense bf16 peak (burst) in TFLOP/s and where it came from."""
    fn = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(fn):
        try:
            d = json.load(open(fn))
            for k in ("bf16_tflops", "bf16_dense_tflops"):
                if k in d:
                    return float(d[k]), "measured (MEASURED_PEAKS.json bf16 burst)"
        except (ValueError, OSError):
            pass
    return 1590.0, "fallback 1.59 PFLOP/s (no MEASURED_PEAKS.json on this box)"


def run_mixed(torch, world, dev, stream, s, args, flush, precision, ref_last, ref_value, ctx64):
    """The same workload in one of the mixed precisions: throughput, its speed-up
    over FP64, the per-mode rate and kappa errors against the FP64 driver."""
    from fourphonon_b200 import abi

    cmx = abi.Context(dev, precision)
    cmx.set_stream(stream.cuda_stream)
    for _ in range(max(1, args.warmup)):
        cmx.rta_driver_4ph(s)
    torch.cuda.synchronize()
    barrier(world)
    rmx = time_steps(torch, cmx, s, args.steps, flush)
    barrier(world)
    tmx = all_max(world, sum(r["ms"] for r in rmx) / 1e3)
    vmx = all_sum(world, sum(r["nproc"] for r in rmx)) / tmx
    cnt = rmx[-1]["counters"]
    cmx.close()
    r3 = ctx64.rta_driver(s)["rate"]
    kerr, rate_err = [], []
    for t in range(len(s.temperatures)):
        r64 = ref_last["rates"]["rate_4ph"][t]
        rm = rmx[-1]["rates"]["rate_4ph"][t]
        k64 = rta_kappa(ctx64, s, r3 + r64, t)
        kmx = rta_kappa(ctx64, s, r3 + rm, t)
        k64_4 = rta_kappa(ctx64, s, r64, t)
        kmx_4 = rta_kappa(ctx64, s, rm, t)
        kerr.append(max(abs(kmx - k64) / abs(k64), abs(kmx_4 - k64_4) / abs(k64_4)))
        m = r64 > 1e-6 * r64.max()
        rate_err.append(float(np.max(np.abs(rm[m] - r64[m]) / r64[m])))
    kms = float(np.mean([r["kms"] for r in rmx]))
    out = {"value": vmx, "unit": UNIT, "speedup_vs_fp64": vmx / ref_value, "kappa_rel_err": max(kerr),
           "rate_rel_err_max": max(rate_err), "kernel_ms": kms, "tensor_cores": bool(cnt[7])}
    if cnt[7]:
        tflops = cnt[6] * 65536.0 / (kms / 1e3) / 1e12
        peak, note = bf16_peak()
        out["dtype"] = "split-bf16 (hi*hi+hi*lo+lo*hi) tcgen05 products, FP32 accumulation in TMEM; FP64 filter/weights/sums"
        out["roofline"] = {"bound": "tensor", "achieved": tflops, "peak": peak, "unit": "TFLOP/s",
                           "frac": tflops / peak, "kernel": "k4_work_tc", "peak_note": note,
                           "achieved_note": "tensor-core flops issued (work counter 6 x 65536) / event-timed kernel "
                                            "duration; the kernel is bound by its FP64 filter, not by the products"}
    else:
        out["dtype"] = "FP32 contraction on the CUDA cores; FP64 filter/weights/sums"
    out["phase_split"] = rmx[-1]["phases"]
    return out


def run_ours(args):
    world, rank, local = dist_setup(args.gpus)
    import torch

    from fourphonon_b200 import abi

    cfg = config_of(args)
    torch.cuda.set_device(local)
    dev = torch.cuda.current_device()
    # rank 0 builds (and caches) the synthetic solve first
    if rank == 0:
        s = workload(cfg, rank)
    barrier(world)
    if rank != 0:
        s = workload(cfg, rank)
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    prec = {"fp64": abi.FP4_PREC_FP64, "mixed": abi.FP4_PREC_MIXED, "mixed_simt": abi.FP4_PREC_MIXED_SIMT}
    ctx = abi.Context(dev, prec[args.precision])
    ctx.set_stream(stream.cuda_stream)
    npi = npi_of(s)

    for _ in range(args.warmup):
        ctx.rta_driver_4ph(s)
    torch.cuda.synchronize()
    barrier(world)
    clocks = Clocks(int(os.environ.get("CUDA_VISIBLE_DEVICES", str(dev)).split(",")[0]) if world == 1 else dev)
    clocks.start()
    torch.cuda.synchronize()
    barrier(world)
    res = time_steps(torch, ctx, s, args.steps, flush)
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    t_local = sum(r["ms"] for r in res) / 1e3
    t_max = all_max(world, t_local)
    nproc_local = sum(r["nproc"] for r in res)
    nproc_all = all_sum(world, nproc_local)
    value = nproc_all / t_max
    kms = float(np.mean([r["kms"] for r in res]))
    last = res[-1]
    cnt = last["counters"]
    fl = executed_flops(s, cnt, npi)
    achieved = fl / (kms / 1e3) / 1e12
    launches = sum(r["launches"] for r in res)

    out = {}
    log(f"fp64: {value:.4g} processes/s, {1000.0 * t_max / args.steps:.0f} ms/step")
    if not args.no_mixed:
        modes = args.mixed_modes.split(",")
        if "mixed" in modes:
            out["mixed"] = run_mixed(torch, world, dev, stream, s, args, flush, abi.FP4_PREC_MIXED, last, value, ctx)
        if "mixed_simt" in modes:
            out["mixed_simt"] = run_mixed(torch, world, dev, stream, s, args, flush, abi.FP4_PREC_MIXED_SIMT, last,
                                          value, ctx)

    log("mixed done" if not args.no_mixed else "mixed skipped")
    # end to end through the public API with host buffers (no upload cache)
    if not args.no_e2e:
        ce = abi.Context(dev, abi.FP4_PREC_FP64)
        ce.set_stream(stream.cuda_stream)
        ce.set_upload_cache(False)
        ps, h2d = pinned_copy(torch, s)
        d2h = 6 * s.nmodes * len(s.temperatures) * 8
        ce.rta_driver_4ph(ps)
        torch.cuda.synchronize()
        barrier(world)
        t0 = time.perf_counter()
        n_e = 0
        for _ in range(args.steps):
            ce.rta_driver_4ph(ps)
            n_e += ce.stats()[0]
        torch.cuda.synchronize()
        te = all_max(world, time.perf_counter() - t0)
        barrier(world)
        out["e2e"] = {"value": all_sum(world, n_e) / te, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                      "d2h_bytes_per_step": int(d2h)}
        ce.close()

    if args.config == 3 and not args.no_sampled:
        out["sampled"] = run_sampled(torch, ctx, s, last, flush, 1000.0 * t_max / args.steps)
    if rank == 0 and world == 1 and not args.no_bte and args.config == 1 and args.precision == "fp64":
        log("bte ...")
        out["bte"] = run_bte(ctx, s, last["rates"]["rate_4ph"][0], s.temperatures[0])
    if rank == 0 and world == 1 and not args.no_serve and args.config == 1:
        log("serving ...")
        out["serving"] = run_serving(args)
        log("serving done")
    peak = fp64_dgemm_peak(torch) if rank == 0 else None
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_sample(s, target_s=15.0, full=(args.config == 0))
    ctx.close()
    if rank != 0:
        barrier(world)
        import torch.distributed as dist

        dist.destroy_process_group()
        return 0
    traffic = None
    tf = os.path.join(ROOT, "profiles", "k4_work_diamond16.txt")
    if os.path.exists(tf) and args.config == 1:
        for line in open(tf):
            if line.startswith("traffic_bytes_per_launch:"):
                traffic = float(line.split(":")[1])
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * t_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f64 filter/weights/sums, " + args.precision + " contraction",
        "data": "synthetic (seeded)",
        "config": {"workload": cfg["workload"], "config_index": args.config, "precision": args.precision, "grid": [cfg["grid"]] * 3,
                   "temperatures_K": s.temperatures, "nmodes": s.nmodes, "nbands": s.nb,
                   "ntri4": s.ifc4.ntri, "displacement_classes": npi, "processes_per_step": last["nproc"],
                   "contracted_per_step": last["ncontr"],
                   "work_counters": {"sigma_evals": int(cnt[2]), "window_tests": int(cnt[3]),
                                     "table_builds": int(cnt[4])},
                   "phase_split": last["phases"],
                   "l2": "256 MiB buffer written between timed steps",
                   "parallelism": f"{world} rank(s), independent solves"},
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak if peak else None, "traffic": traffic,
                     "kernel": "k4_work", "kernel_ms": kms,
                     "peak_note": "FP64: cuBLAS DGEMM 8192^3 measured in this run (no FP64 figure in "
                                  "MEASURED_PEAKS)",
                     "achieved_note": "executed FP64 flops of k4_work from its work counters / event-timed duration",
                     "ref_equivalent_tflops": last["nproc"] * ref_flops_per_process(s) / (kms / 1e3) / 1e12},
        "filter_stage": filter_stage(cnt, kms, last["phases"].get("phase_a_frac"), peak),
        "clocks": clk, "gpu_launches": launches,
        "cpu_baseline": ({k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")} if cpu else None),
    }
    line.update(out)
    print(json.dumps(line), flush=True)
    barrier(world)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


def run_sampled(torch, ctx, s, full, flush, full_ms, nsamples=2_000_000, seed=20240605):
    """The sampled estimator of the same workload, in FP64 and in mixed precision
    (FP32 V(4) sums): its time and the error of its rates against the full FP64
    enumeration, summed over modes and per mode; and mixed against FP64 on the
    same draws."""
    from fourphonon_b200 import abi

    out = {"nsamples_per_mode_channel": nsamples}
    rates = {}
    for name, prec in (("fp64", abi.FP4_PREC_FP64), ("mixed", abi.FP4_PREC_MIXED)):
        c = abi.Context(torch.cuda.current_device(), prec)
        c.set_stream(torch.cuda.current_stream().cuda_stream)
        c.rta_driver_4ph_sample(s, 1000, seed)  # allocations
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        r = c.rta_driver_4ph_sample(s, nsamples, seed)
        e1.record()
        torch.cuda.synchronize()
        c.close()
        ms = e0.elapsed_time(e1)
        errs = {}
        for t, T in enumerate(s.temperatures):
            f = full["rates"]["rate_4ph"][t]
            g = r["rate_plusplus"][t] + r["rate_plusminus"][t] + r["rate_minusminus"][t]
            m = f > 1e-6 * f.max()
            rel = np.abs(g[m] - f[m]) / f[m]
            errs[f"{T:.0f}K"] = {"sum_rel_err": float(abs(g.sum() - f.sum()) / f.sum()),
                                 "per_mode_median": float(np.median(rel)),
                                 "per_mode_p90": float(np.percentile(rel, 90))}
        rates[name] = r
        out[name] = {"ms": ms, "speedup_vs_full_fp64": full_ms / ms, "errors_vs_full_fp64": errs}
    worst = 0.0
    for t in range(len(s.temperatures)):
        a = sum(rates["fp64"]["rate_" + ch][t] for ch in ("plusplus", "plusminus", "minusminus"))
        b = sum(rates["mixed"]["rate_" + ch][t] for ch in ("plusplus", "plusminus", "minusminus"))
        m = a > 1e-6 * a.max()
        worst = max(worst, float(np.max(np.abs(b[m] - a[m]) / a[m])))
    out["mixed"]["rate_rel_err_vs_fp64_same_draws"] = worst
    return out


# ---------------------------------------------------------------------------- serving stream


def serial_fp64_solve(ctx, s, T):
    """One request solved alone through the plain FP64 drivers: 3ph and 4ph RTA
    rates, tau, iteration0, TConduct and the symmetrised kappa tensor."""
    r3 = ctx.rta_driver(s, T=T)
    n = ctx.stats()[0]
    r4 = ctx.rta_driver_4ph(s, temperatures=[T])
    n += ctx.stats()[0]
    rate = r3["rate_plus"] + r3["rate_minus"] + (r4["rate_plusplus"][0] + r4["rate_plusminus"][0]) + \
        r4["rate_minusminus"][0]
    tau = np.zeros_like(rate)
    tau[rate != 0] = 1.0 / rate[rate != 0]
    F = ctx.iteration0(s, tau)
    kap = ctx.tconduct(s, F, T=T).reshape(3, 3, s.nb).sum(axis=2).T
    R = s.sym.crotations
    return sum(R[r] @ kap @ R[r].T for r in range(len(R))) / len(R), n


def run_serving(args, precision=None, tick_ms=25.0, max_slots=16):
    """The serving workload: the seeded 512-request stream of random 2-8 atom cells
    on grids {6,8,10,12,14}^3 at T~U[100,1000] K (system.config4_stream), 3ph+4ph
    RTA + kappa per request, through the serving path (continuous batching, mixed
    precision), against the same requests solved one at a time through the plain
    FP64 drivers.  The whole stream is hours of GPU work (its 8-atom 14^3 requests
    take minutes each), so a prefix of it is served: the longest one whose
    estimated serial time fits --serve-budget seconds; the line states it."""
    from fourphonon_b200 import abi, serve
    from fourphonon_b200 import system as S

    stream = S.config4_stream(512)
    est = [S.request_seconds(na, g) for (na, g, T, sd) in stream]
    full_hours = sum(est) / 3600.0
    npre, acc = 0, 0.0
    while npre < len(stream) and acc + est[npre] <= args.serve_budget:
        acc += est[npre]
        npre += 1
    npre = max(npre, 1)
    specs = stream[:npre]
    solves = [S.cached_solve(f"random{na}", (g, g, g), (T,), seed=sd) for (na, g, T, sd) in specs]
    ctx = abi.Context(0, abi.FP4_PREC_FP64)
    serial_solve = lambda s, T: serial_fp64_solve(ctx, s, T)  # noqa: E731
    serial_solve(S.cached_solve("random2", (4, 4, 4), (300.0,), seed=7), 300.0)  # library and allocation warm-up
    k64, times, nserial = [], [], 0
    for s, (na, g, T, sd) in zip(solves, specs):
        t0 = time.perf_counter()
        k, n = serial_solve(s, T)
        times.append(time.perf_counter() - t0)
        k64.append(k)
        nserial += n
    ctx.close()
    t_serial = float(np.mean(times))
    rng = np.random.default_rng(20240606)
    arrivals = np.cumsum(rng.exponential(t_serial / 2.0, size=npre))  # Poisson, twice the serial FP64 rate
    reqs = [serve.Request(float(arrivals[i]), solves[i], specs[i][2], tag=i) for i in range(npre)]
    precision = abi.FP4_PREC_MIXED if precision is None else precision
    maxb = max(s.nb for s in solves)
    srv = serve.Server(0, precision, max_slots=max_slots, max_bands=max(12, maxb), hbm_budget=48 << 30)
    warm = [serve.Request(0.0, S.cached_solve("random2", (4, 4, 4), (300.0,), seed=7), 300.0)]
    serve.run_stream(srv, warm, tick_items=1 << 16, target_tick_ms=tick_ms)
    done, summ = serve.run_stream(srv, reqs, tick_items=1 << 16, target_tick_ms=tick_ms)
    srv.close()
    kerr = 0.0
    for r in done:  # relative error of the kappa trace, served mixed against serial FP64
        ref = float(np.trace(k64[r.tag]))
        if ref != 0.0:
            kerr = max(kerr, abs(float(np.trace(r.result["kappa"])) - ref) / abs(ref))
    return {"kappa_traces_fp64": [float(np.trace(k)) for k in k64], "requests": npre, "of_stream": len(stream), "solves_per_s": summ["solves_per_s"],
            "p50_ms": summ["p50_ms"], "p99_ms": summ["p99_ms"], "mean_ms": summ["mean_ms"],
            "processes_per_s": summ["processes_per_s"], "ticks": summ["ticks"],
            "serial_fp64_solves_per_s": npre / sum(times), "vs_serial_fp64": summ["solves_per_s"] * sum(times) / npre,
            "serial_fp64_processes_per_s": nserial / sum(times), "kappa_rel_err_max": kerr,
            "precision": "mixed" if precision == abi.FP4_PREC_MIXED else "fp64", "max_slots": max_slots,
            "tick_ms_target": tick_ms, "host_s": summ["host_s"], "wall_s": summ["wall_s"],
            "arrivals": "Poisson at twice the serial FP64 rate of the prefix",
            "prefix": [{"natoms": na, "grid": g, "T": round(T, 1)} for (na, g, T, sd) in specs],
            "full_stream_estimate_gpu_hours": full_hours, "prefix_estimate_serial_s": acc,
            "estimate_note": "system.request_seconds leaves out the growth of the contraction with the number "
                             "of displacement classes and underestimates many-atom cells (compare "
                             "prefix_estimate_serial_s with the measured serial time of the prefix)",
            "prefix_serial_fp64_s": sum(times),
            "workload": "seeded stream of 512 random 2-8 atom cells (masses U[6,120] amu, BvK + Gaussian IFCs), "
                        "grids {6,8,10,12,14}^3, T~U[100,1000] K, 3ph+4ph RTA + kappa; the first `requests` of it"}


def run_bte(ctx, s, rate4, T, maxiter=200):
    """The iterative three-phonon BTE of the benchmarked workload at one temperature:
    Ind_driver (per-process Gamma and lists), tau from the 3ph+4ph RTA rates,
    iteration0, then Gauss-Seidel sweeps (iteration, symmetrisation, TConduct)
    until the relative change of kappa is below 1e-5 (ShengBTE.f90:1271-1306)."""
    eps = float(np.float32(1e-5))
    t0 = time.perf_counter()
    n3 = ctx.np_driver(s)
    lists = ctx.ind_driver(s, n3[0], n3[1], T=T)
    ind_ms = ctx.stats()[3]
    rate = lists["rate_plus"] + lists["rate_minus"] + rate4
    tau = np.zeros_like(rate)
    tau[rate != 0] = 1.0 / rate[rate != 0]
    F = ctx.iteration0(s, tau)
    k = ctx.tconduct(s, F, T=T).reshape(3, 3, s.nb).sum(axis=2)
    k_rta = float(np.trace(k) / 3.0)
    t1 = time.perf_counter()
    sweep_ms, it = [], 0
    for it in range(1, maxiter + 1):
        kold = k
        F = ctx.iteration(s, F, tau, n3[0], n3[1], lists)
        sweep_ms.append(ctx.stats()[3])
        F = ctx.symmetrize_fn(s, F)
        k = ctx.tconduct(s, F, T=T).reshape(3, 3, s.nb).sum(axis=2)
        if np.linalg.norm(k - kold) / np.linalg.norm(kold) < eps:
            break
    t2 = time.perf_counter()
    k_gs = float(np.trace(k) / 3.0)
    # the Jacobi form of the same sweep, from the same iteration0 start
    F = ctx.iteration0(s, tau)
    k = ctx.tconduct(s, F, T=T).reshape(3, 3, s.nb).sum(axis=2)
    t3 = time.perf_counter()
    jac_ms, itj = [], 0
    for itj in range(1, maxiter + 1):
        kold = k
        F = ctx.iteration_jacobi(s, F, tau, n3[0], n3[1], lists)
        jac_ms.append(ctx.stats()[3])
        k = ctx.tconduct(s, F, T=T).reshape(3, 3, s.nb).sum(axis=2)
        if np.linalg.norm(k - kold) / np.linalg.norm(kold) < eps:
            break
    t4 = time.perf_counter()
    k_j = float(np.trace(k) / 3.0)
    return {"T_K": T, "processes_3ph": int(n3[0].sum() + n3[1].sum()), "ind_driver_kernel_ms": ind_ms,
            "iterations": it, "sweep_kernel_ms_mean": float(np.mean(sweep_ms)),
            "sweep_wall_s_mean": (t2 - t1) / it, "to_convergence_wall_s": t2 - t0,
            "kappa_rta": k_rta, "kappa_converged": k_gs,
            "jacobi": {"iterations": itj, "sweep_kernel_ms_mean": float(np.mean(jac_ms)),
                       "sweep_wall_s_mean": (t4 - t3) / itj, "loop_wall_s": t4 - t3, "kappa_converged": k_j,
                       "kappa_rel_diff_vs_gauss_seidel": abs(k_j - k_gs) / abs(k_gs)},
            "note": "Gauss-Seidel: one CTA runs each sweep in the reference's order; Jacobi: every step of a "
                    "sweep at once (fp4_iteration_jacobi); wall times include the host calls that pass the lists"}


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
