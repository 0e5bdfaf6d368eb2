#!/usr/bin/env python
"""Benchmark of the explicit species / electron-energy update (cell-updates/s).

Workload (default ``precision3d``): one 3-D box of 128^3 cells, a 24-species /
150-reaction mechanism (seeded Arrhenius rates), densities log-uniform 1e8-1e22,
Te 0.3-10 eV, WENO-Z drift fluxes, Joule heating, one explicit step
n += dt*(-div F + S) per "step".  The state (134^3 x 34 comps, 654 MB) and the six
face fields are larger than the 126 MB L2, so every step streams them from HBM.

One JSON line on rank 0:
  value        cell-updates/s of the plain FP64 fused update (inputs resident), the
               same arithmetic as the reference's CPU code
  e2e          the same through the C ABI with each step's inputs copied from
               pinned host memory and its updated densities copied back, inside the
               timing (double-buffered copy streams)
  roofline     dominant kernel: algorithmic bytes / average launch time vs the
               measured HBM copy bandwidth; roofline_compute: its issue and pipe
               fractions from the committed ncu summaries
  cpu_baseline the reference's own hot-path code (oracle/_ref) on all host cores
               and on one core, on a bounded slab of the same workload
  summary      compact figures of every path (mixed, batched, serving, large)
  mixed        the mixed-precision path on the same inputs, with its error against
               FP64 per species at the end of the line
Multi-GPU: one process per GPU, each updating its own box (independent boxes, as
AMReX distributes boxes over ranks; no data-path collective); value sums the
cells of all ranks over the slowest rank's time.

``--impl reference`` times the reference's own CPU code instead (rank 0 only).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOADS = {
    "precision3d": "3-D 128^3 box, 24 species / 150 reactions, WENO-Z, one explicit step",
    "argon2d": "2-D 256^2 box, E/Ar+/Ar*/Ar, 10 reactions, WENO-Z, one explicit step",
    "batched": "64 independent 2-D cases, sides log-uniform 64-512, 8 species / 40 reactions, "
               "WENO-Z, 20 explicit steps per case per solve",
    "serving": "Poisson stream at 500 req/s of 1-D/2-D discharge cases, sides log-uniform 256-1024, "
               "0.5-5 kV, 0.1-10 bar, 50-2000 explicit steps, 8 species / 40 reactions, fixed HBM budget",
    "large": "3-D 384^3 single box, 12 species / 60 reactions, WENO-Z, potential solve (multigrid) + explicit "
             "step every step, 100 steps",
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="precision3d", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU time of the baseline sample")
    ap.add_argument("--only-update", action="store_true",
                    help="run W+K mixed-precision updates and nothing else (the command ncu profiles)")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"],
                    help="precision of the --only-update run")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched-workload measurement added to the default line")
    ap.add_argument("--no-serving", action="store_true",
                    help="skip the serving-workload measurement added to the default line")
    ap.add_argument("--requests", type=int, default=48, help="requests of the serving stream")
    ap.add_argument("--budget-gb", type=float, default=8.0, help="HBM budget of the serving loop")
    ap.add_argument("--large-n", type=int, default=384, help="cells per side of the large workload")
    ap.add_argument("--no-large", action="store_true",
                    help="skip the large-case measurement added to the default line")
    return ap.parse_args()


def make_case(workload: str, rank: int = 0):
    from vidyut_b200 import inputs as vin
    seed = vin.BASE_SEED + 1000 * rank
    if workload == "precision3d":
        return vin.config_precision3d(seed=seed) if rank else vin.config_precision3d()
    return vin.config_argon2d(seed=seed) if rank else vin.config_argon2d()


def box_config(case, workload: str, world: int) -> dict:
    """The config object of a one-box workload line (both arms print the same)."""
    return {"workload": WORKLOADS[workload], "cells_per_gpu": case.ncell, "species": case.mech.ns,
            "reactions": len(case.mech.reactions), "dim": case.dim, "hyp_order": 5, "weno_scheme": 3,
            "precision": "fp64", "l2": "inputs larger than L2 (state + faces stream from HBM every step)",
            "parallelism": f"{world} independent boxes (one per GPU)"}


def ref_case_name(case) -> str:
    return case.mech.name


def algorithmic_bytes_per_cell(case) -> dict:
    """Algorithmic bytes of one cell-update (FP64 storage).  Reads: NS densities,
    the electron energy, Te and D field components of the state plus 2*D face
    values (E on faces, grad ne on faces); writes: NS+1 updated densities/energy
    minus the background species that only carry over.  The transport kernel moves
    all of them; the prep kernel reads the NS densities and Te."""
    ns, d = case.mech.ns, case.dim
    reads = ns + 2 + d + 2 * d
    writes = ns + 1
    return {"step": 8 * (reads + writes), "k_transport": 8 * (reads + writes), "k_prep": 8 * (ns + 1),
            "k_prep_spec": 8 * (ns + 1)}


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, power, throttle reasons)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev: int):
        self.dev = dev
        self.proc = None
        self.f = None

    def start(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", delete=False, suffix=".csv")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.dev)], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self) -> dict | None:
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.flush()
        rows = [r.split(",") for r in Path(self.f.name).read_text().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for i, nm in enumerate(names):
                    if r[5 + i].strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
def cpu_reference_rate(case, target_s: float, threads: int | None = None, warm: bool = True):
    """Cell-updates/s of the reference's own code (oracle/_ref) or, if that was not
    built, the C restatement, on a slab of the case sized for about target_s."""
    import oracle
    kind = "reference"
    try:
        lib = oracle.RefLib(ref_case_name(case), case.dim)
    except FileNotFoundError:
        lib = oracle.Port(case.mech)
        kind = "port"
    prm = case.vd_params()
    ax = case.dim - 1  # slab along the slowest swept direction
    n_ax = case.n[ax]

    def run(nplanes):
        hi = list(case.hi)
        hi[ax] = nplanes - 1
        t0 = time.perf_counter()
        lib.update_all(case, prm, lo=case.lo, hi=tuple(hi))
        return time.perf_counter() - t0

    probe = 1 if case.dim == 3 else max(1, n_ax // 64)
    if warm:
        run(probe)
    t = run(probe)
    per_plane = t / probe
    nplanes = int(max(1, min(n_ax, math.ceil(target_s / max(per_plane, 1e-6)))))
    cells_per_plane = case.ncell // n_ax
    return lib, kind, run, nplanes, cells_per_plane


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(threads)
    if args.workload == "batched":
        return run_reference_batched(args, threads)
    if args.workload == "serving":
        return run_reference_serving(args, threads)
    case = make_case(args.workload)
    lib, kind, run, nplanes, cpp = cpu_reference_rate(case, max(1.0, args.cpu_seconds / max(1, args.steps)))
    for _ in range(args.warmup):
        run(nplanes)
    ts = [run(nplanes) for _ in range(args.steps)]
    cells = nplanes * cpp
    t = sum(ts)
    value = cells * args.steps / t
    sample = f"{nplanes} of {case.n[case.dim - 1]} planes ({cells} cells) per step"
    line = {"metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": box_config(case, args.workload, args.gpus),
            "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": threads, "kind": kind,
                             "sample": sample},
            "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_reference_batched(args, threads: int):
    """The reference's own code on the batched workload: each step updates a
    bounded sample of the cases (smallest first) by one explicit step."""
    import oracle
    from vidyut_b200 import inputs
    mech, cases = inputs.config_batched()
    try:
        lib, kind = oracle.RefLib(mech.name, 2), "reference"
    except FileNotFoundError:
        lib, kind = oracle.Port(mech), "port"
    budget = max(1.0, args.cpu_seconds / max(1, args.steps))
    order = sorted(cases, key=lambda c: c.ncell)
    sample, t = [], 0.0
    for c in order:  # choose the sample once, by timing one step of each
        t0 = time.perf_counter()
        lib.update_all(c, c.vd_params())
        t += time.perf_counter() - t0
        sample.append(c)
        if t >= budget:
            break
    for _ in range(args.warmup):
        for c in sample:
            lib.update_all(c, c.vd_params())
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for c in sample:
            lib.update_all(c, c.vd_params())
    t = time.perf_counter() - t0
    cells = sum(c.ncell for c in sample)
    value = cells * args.steps / t
    line = {"metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": WORKLOADS["batched"], "cases": len(cases),
                       "cells": sum(c.ncell for c in cases)},
            "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": threads, "kind": kind,
                             "sample": f"one explicit step of {len(sample)} of {len(cases)} cases "
                                       f"({cells} cells) per step"},
            "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_reference_serving(args, threads: int):
    """The reference's own code on the serving stream, one request at a time (the
    reference runs one case per process): each step of the bench times one
    explicit step of every request of a bounded sample and extrapolates each
    request's service time to its step count; solves/s = requests / total service."""
    import oracle
    from vidyut_b200 import inputs
    mech, reqs = inputs.config_serving(n_requests=args.requests)
    try:
        lib, kind = oracle.RefLib(mech.name, 2), "reference"
        lib1 = oracle.RefLib(mech.name, 1)
    except FileNotFoundError:
        lib = lib1 = oracle.Port(mech)
        kind = "port"
    budget = max(1.0, args.cpu_seconds / max(1, args.steps))
    sample, t = [], 0.0
    for _, c, n in reqs:  # choose the sample once, in arrival order
        t0 = time.perf_counter()
        (lib if c.dim == 2 else lib1).update_all(c, c.vd_params())
        t += time.perf_counter() - t0
        sample.append((c, n))
        if t >= budget:
            break
    for _ in range(args.warmup):
        for c, _ in sample:
            (lib if c.dim == 2 else lib1).update_all(c, c.vd_params())
    service = 0.0
    t_all = time.perf_counter()
    for _ in range(args.steps):
        for c, n in sample:
            t0 = time.perf_counter()
            (lib if c.dim == 2 else lib1).update_all(c, c.vd_params())
            service += (time.perf_counter() - t0) * n
    t_all = time.perf_counter() - t_all
    service /= args.steps
    value = len(sample) / service
    line = {"metric": "solves/s", "value": value, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_all / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": WORKLOADS["serving"], "requests": len(reqs)},
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": kind,
                             "sample": f"one timed explicit step of each of the first {len(sample)} of {len(reqs)} "
                                       "requests, times its step count"},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
def read_profile_traffic(kernel: str, workload: str):
    """DRAM bytes per launch from the committed ncu summary (profiles/), if any."""
    p = ROOT / "profiles" / f"{kernel}_{workload}.md"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.strip().startswith("dram_bytes_per_launch_full:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


def read_profile_metrics(kernel: str, workload: str) -> dict | None:
    """Pipe and issue fractions of one kernel from the committed ncu summary
    (profiles/<kernel>_<workload>.md, lines ``metric_<name>: value``), if any."""
    p = ROOT / "profiles" / f"{kernel}_{workload}.md"
    if not p.exists():
        return None
    out = {}
    for line in p.read_text().splitlines():
        line = line.strip()
        if line.startswith("metric_") and ":" in line:
            k, v = line.split(":", 1)
            try:
                out[k[len("metric_"):].strip()] = float(v.split()[0])
            except (ValueError, IndexError):
                continue
    if not out:
        return None
    out["source"] = f"profiles/{p.name}"
    return out


def hbm_peak():
    peaks = {}
    pk = ROOT / "MEASURED_PEAKS.json"
    if pk.exists():
        peaks = json.loads(pk.read_text())
    hbm = peaks.get("hbm_gbs")
    return (hbm, "measured") if hbm else (6650.0, "fallback")


def e2e_pipelined(case, prm, nsteps: int, world: int, barrier, max_over_ranks) -> dict:
    """cell-updates/s through vd_explicit_update_all with host buffers: every step
    copies its inputs from pinned host memory (the components the update reads:
    species, EEN and Te, the D cell field components, the 2D face arrays) and its
    result (the NS+1 updated densities and energy) back to pinned host memory.
    Double-buffered on three streams, so that step k+1's upload and step k-1's
    download overlap step k's update; the timed region runs from the first upload
    to the last download."""
    import torch

    from vidyut_b200 import _abi as abi
    from vidyut_b200 import api

    ns, dim = case.mech.ns, case.dim
    efx = abi.EFX(ns)
    h_state = torch.from_numpy(case.state).pin_memory()
    h_ef = [torch.from_numpy(a).pin_memory() for a in case.efield[:dim]]
    h_gn = [torch.from_numpy(a).pin_memory() for a in case.gradne[:dim]]
    dcs = [api.upload(case), api.upload(case)]
    phis = [dcs[0].new_outputs()[0], dcs[1].new_outputs()[0]]
    h_out = [torch.empty((ns + 1,) + tuple(phis[0].shape[1:]), dtype=torch.float64).pin_memory() for _ in range(2)]
    need_ef = prm.elecenergy_solve and not prm.cs_technique
    need_gn = prm.elecenergy_solve and not prm.gradne_from_state
    h2d = 8 * (h_state[:ns + 2].numel() + h_state[efx:efx + dim].numel()
               + (sum(a.numel() for a in h_ef) if need_ef else 0) + (sum(a.numel() for a in h_gn) if need_gn else 0))
    d2h = 8 * h_out[0].numel()
    comp = torch.cuda.current_stream()
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
    ev = {k: [torch.cuda.Event(), torch.cuda.Event()] for k in ("h2d", "comp", "d2h")}
    for k in ev:
        for e in ev[k]:
            e.record(comp)

    def step(k):
        b = k & 1
        dc = dcs[b]
        s_in.wait_event(ev["comp"][b])          # step k-2 has finished reading buffer b
        with torch.cuda.stream(s_in):
            dc.state[:ns + 2].copy_(h_state[:ns + 2], non_blocking=True)
            dc.state[efx:efx + dim].copy_(h_state[efx:efx + dim], non_blocking=True)
            for d in range(dim):
                if need_ef:
                    dc.efield[d].copy_(h_ef[d], non_blocking=True)
                if need_gn:
                    dc.gradne[d].copy_(h_gn[d], non_blocking=True)
        ev["h2d"][b].record(s_in)
        comp.wait_event(ev["h2d"][b])
        comp.wait_event(ev["d2h"][b])           # step k-2's result has left phis[b]
        api.explicit_update_all(dc, prm, phis[b], stream=comp)
        ev["comp"][b].record(comp)
        s_out.wait_event(ev["comp"][b])
        with torch.cuda.stream(s_out):
            h_out[b].copy_(phis[b][:ns + 1], non_blocking=True)
        ev["d2h"][b].record(s_out)

    for k in range(3):
        step(k)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s_in)
    for k in range(nsteps):
        step(k)
    e1.record(s_out)
    torch.cuda.synchronize()
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1)) / nsteps
    del dcs, phis
    return {"value": world * case.ncell / (ms * 1e-3), "unit": "cell-updates/s", "ms_per_step": ms,
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "path": "vd_explicit_update_all; per step the inputs it reads from pinned host memory and its "
                    "updated densities back, double-buffered on copy streams, inside the timing"}


def cpu_baselines(case, seconds: float) -> dict:
    """The reference build on all host cores, and on one core, each on a bounded
    slab of the same workload."""
    threads = os.cpu_count() or 1
    lib, kind, run, nplanes, cpp = cpu_reference_rate(case, seconds)
    t = run(nplanes)
    cpu = {"value": nplanes * cpp / t, "unit": "cell-updates/s", "cores": threads, "kind": kind,
           "sample": f"{nplanes} of {case.n[case.dim - 1]} planes ({nplanes * cpp} cells), one step, {t:.1f} s"}
    import ctypes
    try:
        gomp = ctypes.CDLL("libgomp.so.1")
        gomp.omp_set_num_threads(1)
        _, _, run1, np1, cpp1 = cpu_reference_rate(case, seconds / 2, warm=False)
        t1 = run1(np1)
        gomp.omp_set_num_threads(threads)
        cpu["one_core"] = {"value": np1 * cpp1 / t1, "unit": "cell-updates/s", "cores": 1, "kind": kind,
                           "sample": f"{np1} planes ({np1 * cpp1} cells), one step, {t1:.1f} s"}
    except OSError:
        cpu["one_core"] = None
    return cpu


def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    from vidyut_b200 import _abi as abi
    from vidyut_b200 import api

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    L = abi.lib()
    case = make_case(args.workload, rank)
    ns = case.mech.ns
    api.mech_init(case.mech)
    dc = api.upload(case)
    phi_new, _, _ = dc.new_outputs()
    stream = torch.cuda.current_stream()
    prm_mixed = case.vd_params(precision=abi.PREC_MIXED)
    prm_fp64 = case.vd_params(precision=abi.PREC_FP64)

    def timed(prm, steps, warmup):
        for _ in range(warmup):
            api.explicit_update_all(dc, prm, phi_new)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n0 = L.vd_launch_count()
        e0.record(stream)
        for _ in range(steps):
            api.explicit_update_all(dc, prm, phi_new)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ms = e0.elapsed_time(e1)
        return max_over_ranks(ms) / steps, L.vd_launch_count() - n0

    def kernel_profile(prm, steps):
        L.vd_profile_enable(1)
        for _ in range(steps):
            api.explicit_update_all(dc, prm, phi_new)
        torch.cuda.synchronize()
        prof = abi.profile_read()
        L.vd_profile_enable(0)
        return prof

    if args.only_update:
        prm = prm_mixed if args.precision == "mixed" else prm_fp64
        ms, launches = timed(prm, args.steps, args.warmup)
        if rank == 0:
            print(json.dumps({"only_update": True, "precision": args.precision, "ms_per_step": ms,
                              "cells": case.ncell, "gpu_launches": int(launches)}), flush=True)
        if world > 1:
            dist.destroy_process_group()
        return 0

    # headline: the plain FP64 path (the reference's own arithmetic)
    clock = ClockSampler(local)
    clock.start()
    ms_fp64, launches = timed(prm_fp64, args.steps, args.warmup)
    clocks = clock.stop()
    cells = case.ncell
    value = world * cells / (ms_fp64 * 1e-3)
    prof64 = kernel_profile(prm_fp64, args.steps)

    # the mixed-precision path on the same inputs
    ms_mixed, launches_mixed = timed(prm_mixed, args.steps, args.warmup)
    prof_mixed = kernel_profile(prm_mixed, args.steps)

    # per-species error of the mixed result against the FP64 result (which matches
    # the CPU oracle to 1e-12, tests/test_gpu_parity.py)
    dsdt64 = torch.zeros((ns + 1,) + tuple(phi_new.shape[1:]), dtype=torch.float64, device="cuda")
    api.explicit_update_all(dc, prm_fp64, phi_new, dsdt64)
    ref64 = phi_new[:ns + 1].clone()
    api.explicit_update_all(dc, prm_mixed, phi_new)
    mix = phi_new[:ns + 1]
    g = case.gvec
    n_old = dc.state[:ns + 1, g[2]:g[2] + case.n[2], g[1]:g[1] + case.n[1], g[0]:g[0] + case.n[0]]
    diff = (mix - ref64).abs()
    rel = (diff / ref64.abs().clamp_min(1e-300)).reshape(ns + 1, -1)
    srel = (diff / (n_old.abs() + prm_fp64.dt * dsdt64.abs()).clamp_min(1e-300)).reshape(ns + 1, -1)
    err_max = rel.max(dim=1).values.cpu().numpy()
    err_scaled = srel.max(dim=1).values.cpu().numpy()
    err_l2 = ((diff ** 2).reshape(ns + 1, -1).sum(1).sqrt() /
              (ref64 ** 2).reshape(ns + 1, -1).sum(1).sqrt()).cpu().numpy()
    del dsdt64, ref64, diff, rel, srel

    # end to end through the C ABI with host buffers, both precisions
    e2e = e2e_mixed = None
    if not args.no_e2e:
        dc = phi_new = None
        torch.cuda.empty_cache()
        n_e2e = max(4, args.steps // 2)
        e2e = e2e_pipelined(case, prm_fp64, n_e2e, world, barrier, max_over_ranks)
        e2e_mixed = e2e_pipelined(case, prm_mixed, n_e2e, world, barrier, max_over_ranks)
        torch.cuda.empty_cache()

    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return 0

    # roofline of the dominant kernel of each path
    hbm, peak_src = hbm_peak()
    alg = algorithmic_bytes_per_cell(case)

    def roof(prof, ms_step, workload_tag):
        kname, (kcount, kms) = max(prof.items(), key=lambda kv: kv[1][1])
        per_launch_ms = kms / kcount
        achieved = alg.get(kname, alg["step"]) * cells / (per_launch_ms * 1e-3) / 1e9
        return {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                "traffic": read_profile_traffic(kname, workload_tag), "kernel": kname, "peak_source": peak_src,
                "kernel_ms": per_launch_ms, "kernel_share": kms / sum(v[1] for v in prof.values()),
                "alg_bytes_per_cell": alg.get(kname, alg["step"]),
                "step_achieved_gbs": alg["step"] * cells / (ms_step * 1e-3) / 1e9}

    roofline = roof(prof64, ms_fp64, f"{args.workload}_fp64")
    roofline_mixed = roof(prof_mixed, ms_mixed, args.workload)
    roofline_compute = {}
    for k, tag in (("k_transport", f"{args.workload}_fp64"), ("k_prep_spec", f"{args.workload}_fp64"),
                   ("k_transport", args.workload), ("k_prep_spec", args.workload)):
        m = read_profile_metrics(k, tag)
        if m:
            roofline_compute[f"{k}_{'fp64' if tag.endswith('fp64') else 'mixed'}"] = m

    batched = serving = large = None
    if world == 1 and args.workload == "precision3d":
        dc = phi_new = None
        torch.cuda.empty_cache()
        if not args.no_batched:
            r = measure_batched(args.steps, args.warmup, e2e=not args.no_e2e)
            api.mech_init(case.mech)
            batched = {k: r[k] for k in ("speedup_vs_plain_fp64", "value", "ms_per_solve", "solves_per_s", "cases",
                                         "cells", "steps_per_solve", "plain_fp64", "batched_fp64",
                                         "mixed_vs_fp64_max_rel", "roofline", "tile_2d", "gpu_launches", "e2e",
                                         "kernels_ms_per_launch") if k in r}
            batched["unit"] = "cell-updates/s"
            batched["workload"] = WORKLOADS["batched"]
            torch.cuda.empty_cache()
        if not args.no_serving:
            serving = measure_serving(args.requests, args.budget_gb)
            serving.pop("clocks", None)
            serving["workload"] = WORKLOADS["serving"]
            api.mech_init(case.mech)
            torch.cuda.empty_cache()
        if not args.no_large:
            large = measure_large(100, 3, n=args.large_n)
            large.pop("clocks", None)
            large["workload"] = WORKLOADS["large"].replace("384^3", f"{args.large_n}^3")
            torch.cuda.empty_cache()
            api.mech_init(case.mech)

    cpu = None
    if not args.no_cpu_baseline and world == 1:
        cpu = cpu_baselines(case, args.cpu_seconds)

    # compact figures first (a reader of a truncated line keeps them), long arrays last
    summary = {
        "fp64_ms_per_step": ms_fp64, "mixed_ms_per_step": ms_mixed, "mixed_speedup_vs_fp64": ms_fp64 / ms_mixed,
        "mixed_max_rel_vs_fp64": float(np.max(err_max)),
        "e2e_fp64_ms_per_step": e2e["ms_per_step"] if e2e else None,
        "e2e_mixed_ms_per_step": e2e_mixed["ms_per_step"] if e2e_mixed else None,
        "cpu_cores_value": cpu["value"] if cpu else None,
        "cpu_one_core_value": (cpu.get("one_core") or {}).get("value") if cpu else None,
    }
    if batched:
        summary.update({"batched_mixed_speedup_vs_plain_fp64": batched.get("speedup_vs_plain_fp64"),
                        "batched_ms_per_solve": batched.get("ms_per_solve"),
                        "batched_max_rel_vs_fp64": batched.get("mixed_vs_fp64_max_rel", {}).get("max")})
    if serving:
        summary.update({"serving_solves_per_s": serving.get("solves_per_s"), "serving_p50_ms": serving.get("p50_ms"),
                        "serving_p99_ms": serving.get("p99_ms"),
                        "serving_speedup_vs_plain_fp64": serving.get("speedup_solves_vs_plain_fp64")})
    if large:
        summary.update({"large_ms_per_step": large.get("ms_per_step"),
                        "large_max_rel_vs_fp64": (large.get("mixed_vs_fp64_max_rel") or {}).get("max")})

    line = {
        "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_fp64, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": box_config(case, args.workload, world),
        "e2e": e2e,
        "roofline": roofline,
        "roofline_compute": roofline_compute or None,
        "cpu_baseline": cpu,
        "gpu_launches": int(launches),
        "clocks": clocks,
        "summary": summary,
        "mixed": {"value": world * cells / (ms_mixed * 1e-3), "ms_per_step": ms_mixed,
                  "speedup_vs_fp64": ms_fp64 / ms_mixed, "e2e": e2e_mixed, "roofline": roofline_mixed,
                  "gpu_launches": int(launches_mixed),
                  "dtype": "f32/f64 (FP32 WENO, rates, flux arithmetic; FP64 accumulate)",
                  "max_rel_vs_fp64": float(np.max(err_max)),
                  "max_rel_to_step_scale": float(np.max(err_scaled))},
        "kernels_ms_fp64": {k: v[1] / v[0] for k, v in prof64.items()},
        "kernels_ms_mixed": {k: v[1] / v[0] for k, v in prof_mixed.items()},
        "batched": batched,
        "serving": serving,
        "large": large,
        "mixed_vs_fp64_error": {"against": "FP64 GPU result (matches the CPU oracle to 1e-12)",
                                "max_rel_per_species": [float(x) for x in err_max],
                                "l2_rel_per_species": [float(x) for x in err_l2],
                                "max_rel_to_step_scale_per_species": [float(x) for x in err_scaled]},
    }
    print(json.dumps(line), flush=True)
    return 0


BATCH_STEPS = 20  # explicit steps per case in one batched solve


def measure_batched(steps: int, warmup: int, *, cpu_seconds: float = 0.0, e2e: bool = True,
                    plain_fp64: bool = True) -> dict:
    """The batched workload on one GPU.  One bench step = one solve of every case:
    its state is re-loaded from a device-resident copy of its initial state and the
    batch takes BATCH_STEPS steps (one graph replay).  Returns the measurements."""
    import numpy as np
    import torch

    from vidyut_b200 import _abi as abi
    from vidyut_b200 import api, inputs

    L = abi.lib()
    mech, cases = inputs.config_batched()
    api.mech_init(mech)
    stream = torch.cuda.current_stream()
    cells = sum(c.ncell for c in cases)
    H = 3
    init_host = [torch.from_numpy(api.trim_ghosts(c, c.state, H)).pin_memory() for c in cases]
    init_dev = [h.cuda() for h in init_host]

    def make_batch(prec):
        need = sum(api.Batch.case_bytes(c, c.vd_params(precision=prec)) for c in cases)
        b = api.Batch(prec, budget_bytes=int(need * 1.05) + (64 << 20), max_cases=len(cases))
        ids = [b.add(c, c.vd_params(precision=prec), nsteps=BATCH_STEPS) for c in cases]
        return b, ids

    def solve(b, ids, src):
        for i, cid in enumerate(ids):
            b.load(cid, src[i], nsteps=BATCH_STEPS)
        b.step(BATCH_STEPS)

    def timed(fn, k, w):
        for _ in range(w):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n0 = L.vd_launch_count()
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / k, L.vd_launch_count() - n0

    out = {"cases": len(cases), "cells": cells, "steps_per_solve": BATCH_STEPS,
           "sides": [list(c.n[:2]) for c in cases]}
    bm, idm = make_batch(abi.PREC_MIXED)
    tune_ms = bm.tune(trials=3)
    out["tuner_ms"] = {f"{d}d_v{v}": round(ms, 4) for (d, v), ms in tune_ms.items()}
    out["tile_variant_2d"] = bm.stats()["tile_variant"][2]
    shp, _, minb = api.batch_tile_shape(2, out["tile_variant_2d"])
    out["tile_2d"] = list(shp[:2]) + [f"{minb} CTAs/SM"]
    clock = ClockSampler(torch.cuda.current_device())
    clock.start()
    ms, launches = timed(lambda: solve(bm, idm, init_dev), steps, warmup)
    out["clocks"] = clock.stop()
    out["ms_per_solve"] = ms
    out["value"] = cells * BATCH_STEPS / (ms * 1e-3)
    out["solves_per_s"] = len(cases) / (ms * 1e-3)
    out["gpu_launches"] = int(launches)
    out["graph_builds"] = bm.stats()["graph_builds"]

    # per-kernel device time (direct launches so that every launch has its events)
    bm.set_graph(False)
    L.vd_profile_enable(1)
    solve(bm, idm, init_dev)
    torch.cuda.synchronize()
    prof = abi.profile_read()
    L.vd_profile_enable(0)
    bm.set_graph(True)
    out["kernels_ms_per_launch"] = {k: v[1] / v[0] for k, v in prof.items()}
    out["kernels_launches"] = {k: v[0] for k, v in prof.items()}
    mixed_final = [bm.read(i, out=torch.empty_like(init_dev[n])) for n, i in enumerate(idm)]

    # the same batch machinery in FP64, and the mixed result's error against it
    b64, id64 = make_batch(abi.PREC_FP64)
    ms64, _ = timed(lambda: solve(b64, id64, init_dev), max(2, steps // 2), 1)
    out["batched_fp64"] = {"ms_per_solve": ms64, "value": cells * BATCH_STEPS / (ms64 * 1e-3)}
    solve(b64, id64, init_dev)
    solve(bm, idm, init_dev)
    ns = mech.ns
    comps = list(range(ns)) + [abi.EEN(ns), abi.ETEMP(ns)]
    errs = np.zeros(len(comps))
    for n, (i64, im) in enumerate(zip(id64, idm)):
        c = cases[n]
        a = bm.read(im, out=torch.empty_like(init_dev[n]))
        r = b64.read(i64, out=torch.empty_like(init_dev[n]))
        sl = (comps, slice(None), slice(H, H + c.n[1]), slice(H, H + c.n[0]))
        e = ((a[sl] - r[sl]).abs() / r[sl].abs().clamp_min(1e-300)).reshape(len(comps), -1).max(1).values
        errs = np.maximum(errs, e.cpu().numpy())
    out["mixed_vs_fp64_max_rel"] = {"per_component": [float(x) for x in errs], "max": float(errs.max()),
                                    "components": "species 0..NS-1, EEN, ETEMP; all cells of all cases "
                                                  f"after {BATCH_STEPS} steps"}
    b64.close()
    del mixed_final

    # plain FP64 per-box path, case by case (vd_explicit_update_all + vd_fill_ghosts)
    if plain_fp64:
        dcs = [api.upload(c) for c in cases]
        outs = [dc.new_outputs()[0] for dc in dcs]
        init_full = [dc.state.clone() for dc in dcs]
        g = H

        def plain_solve():
            for dc, pn, st0, c in zip(dcs, outs, init_full, cases):
                dc.state.copy_(st0, non_blocking=True)
                prm = c.vd_params(precision=abi.PREC_FP64)
                v = dc.state[:, :, g:g + c.n[1], g:g + c.n[0]]
                for _ in range(BATCH_STEPS):
                    api.explicit_update_all(dc, prm, pn)
                    v.copy_(pn)
                    api.fill_ghosts(dc.state, c, H, comps, c.periodic)

        msp, _ = timed(plain_solve, 2, 1)
        out["plain_fp64"] = {"ms_per_solve": msp, "value": cells * BATCH_STEPS / (msp * 1e-3),
                             "path": "per case: 20 x (vd_explicit_update_all FP64 + vd_fill_ghosts)"}
        out["speedup_vs_plain_fp64"] = msp / ms
        del dcs, outs, init_full

    # end to end: states from pinned host memory, results back to pinned host memory
    if e2e:
        res_host = [torch.empty_like(h).pin_memory() for h in init_host]

        def e2e_solve():
            solve(bm, idm, init_host)
            for n, i in enumerate(idm):
                bm.read(i, out=res_host[n])

        mse, _ = timed(e2e_solve, max(3, steps // 2), 1)
        nbytes = sum(h.numel() * 8 for h in init_host)
        out["e2e"] = {"value": cells * BATCH_STEPS / (mse * 1e-3), "unit": "cell-updates/s", "ms_per_solve": mse,
                      "h2d_bytes_per_step": int(nbytes), "d2h_bytes_per_step": int(nbytes),
                      "path": "vd_batch_load_case from pinned host, vd_batch_step, vd_batch_read_case "
                              "to pinned host, inside the timing"}
    bm.close()

    # roofline of the dominant batched kernel: algorithmic bytes per cell-update
    dom = max(prof.items(), key=lambda kv: kv[1][1])
    kname, (kcount, kms) = dom
    per_launch = kms / kcount
    alg = algorithmic_bytes_per_cell(cases[0])
    abytes = {"k_transport_batch": alg["step"], "k_prep_batch": alg["k_prep"],
              "k_prep_batch_spec": alg["k_prep"]}.get(kname, alg["step"])
    achieved = abytes * cells / (per_launch * 1e-3) / 1e9
    out["roofline"] = {"kernel": kname, "achieved": achieved, "unit": "GB/s", "kernel_ms": per_launch,
                       "kernel_share": kms / sum(v[1] for v in prof.values()),
                       "alg_bytes_per_cell": abytes}

    if cpu_seconds > 0:
        import oracle
        name = mech.name
        threads = os.cpu_count() or 1
        try:
            lib = oracle.RefLib(name, 2)
            kind = "reference"
        except FileNotFoundError:
            lib = oracle.Port(mech)
            kind = "port"
        done_cells, t = 0, 0.0
        for c in sorted(cases, key=lambda c: c.ncell):
            t0 = time.perf_counter()
            lib.update_all(c, c.vd_params())
            t += time.perf_counter() - t0
            done_cells += c.ncell
            if t >= cpu_seconds:
                break
        out["cpu_baseline"] = {"value": done_cells / t, "unit": "cell-updates/s", "cores": threads, "kind": kind,
                               "sample": f"one step of {done_cells} cells (smallest cases first), {t:.1f} s"}
    return out


def measure_serving(n_requests: int = 48, budget_gb: float = 8.0, quantum: int = 25, plain_fp64: bool = True,
                    warmup: bool = True) -> dict:
    """The serving workload on one GPU: the seeded Poisson stream is submitted to
    the continuous-batching server at its arrival times (host inputs in, final
    states back to host memory), then every result is collected.  The baseline is
    the same stream served first-come-first-served one case at a time on the plain
    FP64 per-box path (a queue alone): each request's service time is measured on
    the GPU and its latency follows from the queue, finish_i = max(arrival_i,
    finish_(i-1)) + service_i."""
    import threading

    import torch

    from vidyut_b200 import _abi as abi
    from vidyut_b200 import api, inputs

    L = abi.lib()
    mech, reqs = inputs.config_serving(n_requests=n_requests)
    api.mech_init(mech)
    budget = int(budget_gb * (1 << 30))
    if warmup:  # graph capture paths, NVRTC module load, pinned pools
        with api.Server(abi.PREC_MIXED, budget_bytes=budget, max_cases=256, quantum_steps=quantum) as s:
            ids = [s.submit(c, c.vd_params(precision=abi.PREC_MIXED), 30) for _, c, _ in reqs[:4]]
            for i in ids:
                s.wait(i)
    clock = ClockSampler(torch.cuda.current_device())
    n0 = L.vd_launch_count()
    clock.start()
    with api.Server(abi.PREC_MIXED, budget_bytes=budget, max_cases=256, quantum_steps=quantum) as s:
        ids = [None] * len(reqs)

        def feeder():
            t0 = time.perf_counter()
            for k, (t_arr, c, n) in enumerate(reqs):
                dt = t_arr - (time.perf_counter() - t0)
                if dt > 0:
                    time.sleep(dt)
                ids[k] = s.submit(c, c.vd_params(precision=abi.PREC_MIXED), n)

        th = threading.Thread(target=feeder)
        t_start = time.perf_counter()
        th.start()
        th.join()
        # a request whose state met a NaN or infinity comes back failed (the
        # reference aborts such a run); it is counted, and left out of the latencies
        lat, failed = [], 0
        for i in ids:
            try:
                lat.append(s.wait(i)[1])
            except abi.VidyutError as e:
                if e.status != abi.ERR_NONFINITE:
                    raise
                failed += 1
        wall = time.perf_counter() - t_start
        st = s.stats()
    clocks = clock.stop()
    launches = L.vd_launch_count() - n0
    cells_steps = sum(c.ncell * n for _, c, n in reqs)
    nbytes = sum(c.state.nbytes for _, c, _ in reqs)
    out = {"requests": len(reqs), "offered_rate_per_s": len(reqs) / reqs[-1][0], "n_2d": sum(c.dim == 2 for _, c, _ in reqs),
           "cell_updates": cells_steps, "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "max_ms": st["max_ms"],
           "solves_per_s": st["solves_per_s"], "cell_updates_per_s": st["cell_updates_per_s"], "span_s": st["span_s"],
           "wall_s": wall, "peak_bytes_used": st["peak_bytes_used"], "budget_bytes": budget, "quanta": st["quanta"],
           "graph_builds": st["graph_builds"], "quantum_steps": quantum, "gpu_launches": int(launches),
           "h2d_bytes": int(nbytes), "d2h_bytes": int(nbytes), "clocks": clocks,
           "lat_mean_ms": float(sum(lat) / len(lat)) if lat else None, "failed_nonfinite": failed}
    if plain_fp64:
        import numpy as np
        service, ok = [], []
        for t_arr, c, n in reqs:
            ns = c.mech.ns
            comps = list(range(ns)) + [abi.EEN(ns), abi.ETEMP(ns)]
            prm = c.vd_params(precision=abi.PREC_FP64)
            # every quantum-th step checks for NaN / infinity, as the server does
            # once per quantum; a request that meets one stops there, failed
            prm_chk = c.vd_params(precision=abi.PREC_FP64, check_finite=1)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            dc = api.upload(c)
            pn, _, _ = dc.new_outputs()
            g = c.gvec
            v = dc.state[:, g[2]:g[2] + c.n[2], g[1]:g[1] + c.n[1], g[0]:g[0] + c.n[0]]
            good = True
            for k in range(n):
                try:
                    api.explicit_update_all(dc, prm_chk if k % quantum == quantum - 1 else prm, pn)
                except abi.VidyutError as e:
                    if e.status != abi.ERR_NONFINITE:
                        raise
                    good = False
                    break
                v.copy_(pn)
                api.fill_ghosts(dc.state, c, c.ghost, comps, c.periodic)
            res = dc.state.cpu()
            torch.cuda.synchronize()
            service.append(time.perf_counter() - t0)
            ok.append(good)
            del dc, pn, res
        fin, lats = 0.0, []
        for (t_arr, _, _), sv, good in zip(reqs, service, ok):
            fin = max(t_arr, fin) + sv
            if good:
                lats.append(1e3 * (fin - t_arr))
        span = fin - reqs[0][0]
        out["plain_fp64_fifo"] = {"p50_ms": float(np.percentile(lats, 50)), "p99_ms": float(np.percentile(lats, 99)),
                                  "solves_per_s": sum(ok) / span, "cell_updates_per_s": cells_steps / span,
                                  "service_s_total": float(sum(service)), "failed_nonfinite": len(ok) - sum(ok),
                                  "path": "one request at a time: upload, n x (vd_explicit_update_all FP64 + "
                                          "vd_fill_ghosts, a NaN check every quantum), result to host"}
        out["speedup_solves_vs_plain_fp64"] = out["solves_per_s"] / out["plain_fp64_fifo"]["solves_per_s"]
        out["p99_ratio_vs_plain_fp64"] = out["plain_fp64_fifo"]["p99_ms"] / max(out["p99_ms"], 1e-9)
    return out


def measure_large(steps: int = 100, warmup: int = 3, n: int = 384, fp64_compare: bool = True) -> dict:
    """The large single case: every step solves the potential (multigrid, warm
    started, to 1e-8 relative residual) and takes one explicit step (prep +
    transport), then refills the ghosts.  Mixed precision timed; the same steps in
    FP64 from the same initial state give the error of the mixed run."""
    import ctypes as C

    import torch

    from vidyut_b200 import _abi as abi
    from vidyut_b200 import api, inputs

    L = abi.lib()
    mech, case, st_init = inputs.config_large_device(n=(n, n, n))
    api.mech_init(mech)
    ns = mech.ns
    cells = case.ncell
    ef = [torch.zeros((1, n + (d == 2), n + (d == 1), n + (d == 0)), dtype=torch.float64, device="cuda")
          for d in range(3)]
    gn = [torch.zeros((1, 1, 1, 1), dtype=torch.float64, device="cuda") for _ in range(3)]  # not read
    comps = list(range(ns)) + [abi.EEN(ns), abi.ETEMP(ns)]
    stream = torch.cuda.current_stream()
    pp = api.poisson_params(3, 1000.0, 0.0, max_vcycles=40, tol_rel=1e-8)
    box = abi.make_box(case.lo, case.hi, 3)
    null = abi.null_array4()
    cyc = []

    def run(prec, nsteps, bufs, profile=False):
        prm = case.vd_params(precision=prec)
        cur, nxt = bufs
        dc = api.DeviceCase(case, cur, ef, gn)
        for _ in range(nsteps):
            dc.state = cur
            nv, _ = api.poisson_solve(dc, prm, pp)
            cyc.append(nv)
            # next step's initial guess: 2 phi_n - phi_(n-1) (nxt still holds phi_(n-1))
            pot = abi.POT(ns)
            nxt[pot].mul_(-1.0).add_(cur[pot], alpha=2.0)
            rc = L.vd_explicit_update_all(C.byref(box), api.t_a4(cur, case.state_begin()), dc.face_a4s("efield"),
                                          dc.face_a4s("gradne"), api.t_a4(nxt, case.state_begin()), null, null,
                                          C.byref(prm), stream.cuda_stream)
            abi.check(rc, "vd_explicit_update_all")
            api.fill_ghosts(nxt, case, case.ghost, comps)
            cur, nxt = nxt, cur
        return cur, nxt

    # mixed precision
    a, b = st_init.clone(), st_init.clone()
    a, b = run(abi.PREC_MIXED, warmup, (a, b))
    a.copy_(st_init)
    b.copy_(st_init)
    cyc.clear()
    torch.cuda.synchronize()
    clock = ClockSampler(torch.cuda.current_device())
    clock.start()
    n0 = L.vd_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    fin_mixed, spare = run(abi.PREC_MIXED, steps, (a, b))
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = clock.stop()
    ms = e0.elapsed_time(e1) / steps
    launches = L.vd_launch_count() - n0
    vcycles = sum(cyc) / max(1, len(cyc))
    # per-kernel device time of a few more steps (from the final state)
    L.vd_profile_enable(1)
    run(abi.PREC_MIXED, 2, (fin_mixed, spare))
    torch.cuda.synchronize()
    prof = abi.profile_read()
    L.vd_profile_enable(0)
    kms = {k: v[1] / v[0] for k, v in prof.items()}
    update_ms = kms.get("k_transport", 0.0) + kms.get("k_prep_spec", kms.get("k_prep", 0.0)) + \
        kms.get("k_joule_pre", 0.0) + 2 * kms.get("k_ghost", 0.0)
    out = {"cells": cells, "steps": steps, "ms_per_step": ms, "value": cells / (ms * 1e-3),
           "update_ms_per_step": update_ms, "potential_ms_per_step": ms - update_ms,
           "vcycles_per_step": vcycles, "gpu_launches": int(launches), "clocks": clocks,
           "kernels_ms_per_launch": {k: v[1] / v[0] for k, v in prof.items()},
           "kernels_launches_2_steps": {k: v[0] for k, v in prof.items()}}
    del spare
    if fp64_compare:
        # the mixed final state was advanced 2 more profiled steps: redo it cleanly
        fin_mixed = spare = None
        torch.cuda.empty_cache()
        a, b = st_init.clone(), st_init.clone()
        fm, other = run(abi.PREC_MIXED, steps, (a, b))
        del a, b, other
        torch.cuda.empty_cache()
        c64, d64 = st_init.clone(), st_init
        torch.cuda.synchronize()
        e0.record(stream)
        fin64, _ = run(abi.PREC_FP64, steps, (c64, d64))
        e1.record(stream)
        torch.cuda.synchronize()
        ms64 = e0.elapsed_time(e1) / steps
        g = case.ghost
        errs = []
        for q in comps:
            x = fm[q, g:g + n, g:g + n, g:g + n]
            r = fin64[q, g:g + n, g:g + n, g:g + n]
            errs.append(float(((x - r).abs() / r.abs().clamp_min(1e-300)).max()))
        out["fp64"] = {"ms_per_step": ms64, "value": cells / (ms64 * 1e-3), "mixed_speedup": ms64 / ms}
        out["mixed_vs_fp64_max_rel"] = {"per_component": errs, "max": max(errs),
                                        "components": f"species 0..{ns - 1}, EEN, ETEMP after {steps} steps"}
        # the trajectory's own sensitivity: FP64 again from the same initial state
        # with every density scaled by (1 + 1e-15), against the FP64 run above
        keep = fin64
        del fm, c64, d64, st_init, fin64
        torch.cuda.empty_cache()
        a = inputs.config_large_device(n=(n, n, n))[2]
        a[:ns] *= 1.0 + 1e-15
        b = a.clone()
        finp, _ = run(abi.PREC_FP64, steps, (a, b))
        errs_p = []
        for q in comps:
            x = finp[q, g:g + n, g:g + n, g:g + n]
            r = keep[q, g:g + n, g:g + n, g:g + n]
            errs_p.append(float(((x - r).abs() / r.abs().clamp_min(1e-300)).max()))
        out["fp64_vs_fp64_perturbed_1e-15"] = {"per_component": errs_p, "max": max(errs_p)}
    return out


def run_large_line(args):
    import torch
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1 and int(os.environ.get("RANK", "0")) != 0:
        return 0  # one resident domain on one GPU
    steps = args.steps if args.steps != 10 else 100
    r = measure_large(steps, max(3, args.warmup), n=args.large_n)
    peaks = {}
    pk = ROOT / "MEASURED_PEAKS.json"
    if pk.exists():
        peaks = json.loads(pk.read_text())
    hbm = peaks.get("hbm_gbs") or 6650.0
    kt = r["kernels_ms_per_launch"].get("k_transport")
    alg = 8 * (12 + 2 + 3 + 6 + 12 + 1)  # reads NS+2+D+2D, writes NS+1 (FP64)
    roof = None
    if kt:
        ach = alg * r["cells"] / (kt * 1e-3) / 1e9
        roof = {"bound": "hbm", "kernel": "k_transport", "achieved": ach, "peak": hbm, "unit": "GB/s",
                "frac": ach / hbm, "traffic": read_profile_traffic("k_transport", "large"), "kernel_ms": kt,
                "alg_bytes_per_cell": alg, "peak_source": "measured" if peaks.get("hbm_gbs") else "fallback"}
    line = {"metric": "cell-updates/s", "value": r["value"], "unit": "cell-updates/s", "n_gpus": 1,
            "steps": r["steps"], "warmup": max(3, args.warmup), "ms_per_step": r["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32/f64 (mixed: FP32 WENO, rates, fluxes; FP64 accumulate; FP64 potential solve)",
            "data": "synthetic",
            "config": {"workload": WORKLOADS["large"].replace("384^3", f"{args.large_n}^3"), "cells": r["cells"],
                       "species": 12, "reactions": 60,
                       "l2": "inputs larger than L2 (10.4 GB state per copy)"},
            "roofline": roof, "cpu_baseline": None, "e2e": None, "gpu_launches": r["gpu_launches"],
            "clocks": r["clocks"], "large": r}
    print(json.dumps(line), flush=True)
    return 0


def run_serving_line(args):
    import torch
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1 and int(os.environ.get("RANK", "0")) != 0:
        return 0  # replicas only: the serving workload is measured on one GPU
    r = measure_serving(args.requests, args.budget_gb)
    line = {"metric": "solves/s", "value": r["solves_per_s"], "unit": "solves/s", "n_gpus": 1,
            "steps": r["requests"], "warmup": 4, "ms_per_step": 1e3 * r["span_s"] / max(1, r["requests"]),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32/f64 (mixed: FP32 WENO, rates, fluxes; FP64 accumulate)", "data": "synthetic",
            "config": {"workload": WORKLOADS["serving"], "requests": r["requests"],
                       "budget_bytes": r["budget_bytes"], "quantum_steps": r["quantum_steps"],
                       "l2": "inputs larger than L2 (resident cases of up to 1M cells x 18 comps, two copies)"},
            "p50_ms": r["p50_ms"], "p99_ms": r["p99_ms"], "max_ms": r["max_ms"],
            "cell_updates_per_s": r["cell_updates_per_s"],
            "e2e": {"value": r["solves_per_s"], "unit": "solves/s", "h2d_bytes_per_step": r["h2d_bytes"] // r["requests"],
                    "d2h_bytes_per_step": r["d2h_bytes"] // r["requests"],
                    "path": "vd_server_submit with host inputs .. vd_server_wait with host results; every "
                            "request's copies are inside its latency"},
            "roofline": None, "cpu_baseline": None, "gpu_launches": r["gpu_launches"], "clocks": r["clocks"],
            "serving": r}
    print(json.dumps(line), flush=True)
    return 0


def run_batched_line(args):
    import torch
    from vidyut_b200 import _abi as abi
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1 and int(os.environ.get("RANK", "0")) != 0:
        return 0  # replicas only: the batched workload is measured on one GPU
    r = measure_batched(args.steps, args.warmup, cpu_seconds=0.0 if args.no_cpu_baseline else args.cpu_seconds,
                        e2e=not args.no_e2e)
    peaks = {}
    pk = ROOT / "MEASURED_PEAKS.json"
    if pk.exists():
        peaks = json.loads(pk.read_text())
    hbm = peaks.get("hbm_gbs") or 6650.0
    roof = dict(r["roofline"])
    roof.update({"bound": "hbm", "peak": hbm, "frac": roof["achieved"] / hbm,
                 "peak_source": "measured" if peaks.get("hbm_gbs") else "fallback",
                 "traffic": read_profile_traffic(roof["kernel"], "batched")})
    line = {"metric": "cell-updates/s", "value": r["value"], "unit": "cell-updates/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_solve"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32/f64 (mixed: FP32 WENO, rates, fluxes; FP64 accumulate)", "data": "synthetic",
            "config": {"workload": WORKLOADS["batched"], "cases": r["cases"], "cells": r["cells"],
                       "steps_per_solve": BATCH_STEPS, "species": 8, "reactions": 40,
                       "l2": "inputs larger than L2 (two state copies of 3M cells x 18 comps)"},
            "roofline": roof, "cpu_baseline": r.get("cpu_baseline"), "e2e": r.get("e2e"),
            "gpu_launches": r["gpu_launches"], "clocks": r["clocks"],
            "solves_per_s": r["solves_per_s"], "speedup_vs_plain_fp64": r.get("speedup_vs_plain_fp64"),
            "plain_fp64": r.get("plain_fp64"), "batched_fp64": r["batched_fp64"],
            "mixed_vs_fp64_max_rel": r["mixed_vs_fp64_max_rel"], "tuner_ms": r["tuner_ms"],
            "tile_2d": r["tile_2d"], "kernels_ms_per_launch": r["kernels_ms_per_launch"]}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batched":
        if args.only_update:
            return run_batched_only(args)
        return run_batched_line(args)
    if args.workload == "serving":
        return run_serving_line(args)
    if args.workload == "large":
        return run_large_line(args)
    return run_ours(args)


def run_batched_only(args):
    """W + K batched solves and nothing else (the command ncu profiles); graph
    replay off so that every kernel is a separate launch."""
    import torch
    from vidyut_b200 import _abi as abi
    from vidyut_b200 import api, inputs
    mech, cases = inputs.config_batched()
    api.mech_init(mech)
    prec = abi.PREC_MIXED if args.precision == "mixed" else abi.PREC_FP64
    need = sum(api.Batch.case_bytes(c, c.vd_params(precision=prec)) for c in cases)
    with api.Batch(prec, budget_bytes=int(need * 1.05) + (64 << 20), max_cases=len(cases)) as b:
        b.set_graph(False)
        ids = [b.add(c, c.vd_params(precision=prec), nsteps=-1) for c in cases]
        for _ in range(args.warmup):
            b.step(1)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            b.step(1)
        e1.record()
        torch.cuda.synchronize()
        print(json.dumps({"only_update": True, "workload": "batched", "precision": args.precision,
                          "ms_per_batch_step": e0.elapsed_time(e1) / max(1, args.steps),
                          "cells": sum(c.ncell for c in cases), "cases": len(ids)}), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
