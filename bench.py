"""Benchmark of the leapfrog time-stepping path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload fit512|fit64]

A step is one leapfrog step (E half, sources, probe export, H half) over the
whole workload.  Default workload `fit512`: the 512^3-cell Cartesian FIT cavity
with 200 seeded lossy dielectric spheres over vacuum, PEC on surfaces 2-6 and
the H-wave source on surface 1, FP32 field state (807,667,200 edge+face dofs;
the field arrays, 3.3 GB, are far larger than the 126 MB L2, so no flush is
needed between steps).  `value` is device-timed dof-steps/s (CUDA events on the
library's stream); `e2e` is the same metric through the stepwise C-ABI call
tf_step_io with host buffers (this step's carrier values H2D from pinned
memory, the exported probe sample D2H).  Multi-GPU runs are independent
replicas (the path has no exchange step on one mesh per GPU): weak scaling.

`--impl reference` times the FP64 CPU restatement of the reference (the
reference itself cannot be built here) with all host threads on a bounded
sample of the same scene (a 96^3 grid, same spheres and sources).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0

WORKLOADS = {
    # name: (cells per axis, spheres, precision, steps in the script)
    "fit512": (512, 200, "fp32", 5000),
    "fit64": (64, 0, "fp64", 2000),
    "fit256": (256, 200, "fp32", 2000),   # profiling size: state 400 MB > L2
}


def hbm_peak():
    try:
        with open(MEASURED_PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 9:
                rows.append(p)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for r in rows for q in range(4) if r[5 + q].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def make_case(workdir: str, workload: str, n_override: int | None = None):
    from tetfit_b200.cases import FitCase, random_spheres, write_fit_cavity
    n, nsph, prec, steps = WORKLOADS[workload]
    spheres = random_spheres(nsph, seed=2026) if nsph else []
    case = FitCase(n=n, steps=steps, spheres=spheres)
    if n_override:
        # same scene and time step, coarser grid (bounded CPU sample)
        case = FitCase(n=n_override, steps=steps, spheres=spheres, step=case.dt())
    return write_fit_cavity(workdir, case), prec, case


def fit_bytes(info: dict, es: int):
    """Algorithmic bytes of one E and one H launch (FIT byte model):
    E reads U and F and writes U; H reads F and U and writes F; plus 1 B of
    material index per cell each."""
    nE, nF, nc = info["n_edges"], info["n_faces"], info["n_cells"]
    e_bytes = es * (2 * nE + nF) + nc
    h_bytes = es * (2 * nF + nE) + nc
    return e_bytes, h_bytes


def run_ours(args, rank, world, local_rank):
    import tetfit_b200 as tb
    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist_
        dist = dist_
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    work = tempfile.mkdtemp(prefix=f"tfbench{rank}_")
    script, prec, case = make_case(work, args.workload)
    d = tb.Discretization(script)
    t0 = time.time()
    info = d.prepare(1, precision=prec, device=local_rank, graph_steps=1 if case.n >= 256 else 0)
    setup_s = time.time() - t0
    K, W = args.steps, args.warmup
    need = W + K + min(K, 50) + 20
    if info["n_steps"] < need:
        raise SystemExit(f"workload has {info['n_steps']} steps, bench needs {need}")
    d.step(W)
    # per-phase timing (events between kernels) for the roofline; untimed
    ms5, nph = d.phase_times(min(K, 20))

    def barrier():
        if dist:
            import torch
            torch.cuda.synchronize()
            dist.barrier()

    barrier()
    with ClockSampler(local_rank) as clk:
        d.step(K)
        dev_ms = d.last_step_ms()
    barrier()
    # e2e: tf_step_io with host buffers, K' steps
    n_src = info["n_sources"]
    K2 = min(K, 50)
    carrier = np.zeros(max(n_src, 1))
    probe = np.zeros(max(info["n_probes"], 1) * 6)
    barrier()
    t0 = time.perf_counter()
    s0 = d.info()["step_index"]
    for i in range(K2):
        s = s0 + i
        carrier[:] = np.sin(2 * np.pi * case.frequency * (s * info["dt"] - 0.5 * info["dt"]))
        d.step_io(carrier, probe)
    e2e_s = time.perf_counter() - t0
    barrier()
    dofs = info["n_edges"] + info["n_faces"]
    max_ms = dev_ms
    max_e2e = e2e_s
    if dist:
        import torch
        t = torch.tensor([dev_ms, e2e_s], dtype=torch.float64, device=f"cuda:{local_rank}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        max_ms, max_e2e = float(t[0]), float(t[1])
    kps = info["kernels_per_step"]
    result = None
    if rank == 0:
        es = 4 if prec == "fp32" else 8
        e_bytes, h_bytes = fit_bytes(info, es)
        e_ms, h_ms = ms5[1] / nph, ms5[4] / nph
        dom = "fit_e_kernel" if e_ms >= h_ms else "fit_h_kernel"
        dom_bytes, dom_ms = (e_bytes, e_ms) if dom == "fit_e_kernel" else (h_bytes, h_ms)
        peak, peak_kind = hbm_peak()
        achieved = dom_bytes / (dom_ms * 1e-3) / 1e9
        value = world * dofs * K / (max_ms * 1e-3)
        result = {
            "metric": "dof-steps/s", "value": value, "unit": "dof-steps/s", "n_gpus": world, "steps": K,
            "warmup": W, "ms_per_step": max_ms / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if prec == "fp32" else "f64", "data": "synthetic",
            "config": {"workload": f"{args.workload}: FIT cavity {case.n}^3 cells, {len(case.spheres)} lossy "
                                   f"spheres, PEC surfaces 2-6, H-wave source on surface 1, "
                                   f"{prec} state, 156 probes every step",
                       "dofs": dofs, "cells": info["n_cells"], "parallelism": f"replicas x{world}",
                       "l2": "state 6 arrays >> 126 MB L2 (no flush needed)", "setup_s": round(setup_s, 2)},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind, "traffic": None,
                         "algorithmic_bytes": dom_bytes, "launch_ms": dom_ms},
            "phases_ms_per_step": {k: v / nph for k, v in
                                   zip(["sources_bc", "e_update", "scatter_flux", "probes", "h_update"], ms5)},
            "e2e": {"value": world * dofs * K2 / max_e2e, "unit": "dof-steps/s",
                    "h2d_bytes_per_step": 8 * n_src, "d2h_bytes_per_step": 8 * 6 * info["n_probes"],
                    "api": "tf_step_io"},
            "gpu_launches": kps * K,
            "clocks": clk.summary(),
        }
        if world == 1 and not args.no_cpu_baseline:
            result["cpu_baseline"] = cpu_baseline(args, seconds=args.cpu_seconds)
    d.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return result


def cpu_baseline(args, seconds=15.0, threads=None):
    """FP64 CPU restatement of the reference on a bounded sample of the scene."""
    import oracle
    work = tempfile.mkdtemp(prefix="tfcpu_")
    n_sample = 96 if args.workload == "fit512" else WORKLOADS[args.workload][0]
    script, _, _ = make_case(work, args.workload, n_override=n_sample)
    if threads:
        os.environ["OMP_NUM_THREADS"] = str(threads)
    os.environ["TF_ORACLE_SKIP_DT"] = "1"  # the step is pinned; skip the setup-only eigen-estimate
    o = oracle.FitOracle(script, omp=True)
    dofs = o.nE + o.nF
    o.step(2)
    t0 = time.perf_counter()
    n = 0
    while time.perf_counter() - t0 < seconds and n + 10 <= o.n_steps - 2:
        n += o.step(10)
    el = time.perf_counter() - t0
    o.close()
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": dofs * n / el, "unit": "dof-steps/s", "cores": cores, "kind": "port",
            "sample": f"{n_sample}^3 grid of the same scene (FP64), {n} steps, {el:.1f} s, "
                      f"OpenMP threads={cores}", "cpu": _cpu_model()}


def _cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return None


def run_reference(args, rank):
    if rank != 0:
        return None
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    import oracle
    work = tempfile.mkdtemp(prefix="tfref_")
    n_sample = 96 if args.workload == "fit512" else WORKLOADS[args.workload][0]
    script, _, _ = make_case(work, args.workload, n_override=n_sample)
    os.environ["TF_ORACLE_SKIP_DT"] = "1"  # the step is pinned; skip the setup-only eigen-estimate
    o = oracle.FitOracle(script, omp=True)
    dofs = o.nE + o.nF
    o.step(args.warmup)
    t0 = time.perf_counter()
    o.step(args.steps)
    el = time.perf_counter() - t0
    o.close()
    v = dofs * args.steps / el
    cores = int(os.environ["OMP_NUM_THREADS"])
    sample = (f"{n_sample}^3 grid of the {args.workload} scene, FP64 C++ restatement of the reference "
              f"(reference needs Eigen/Spectra/GSL/Silo, not buildable here), {args.steps} steps")
    return {"impl": "reference", "metric": "dof-steps/s", "value": v, "unit": "dof-steps/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": el * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": f"{args.workload} (bounded CPU sample {n_sample}^3)"},
            "cpu_baseline": {"value": v, "unit": "dof-steps/s", "cores": cores, "kind": "port",
                             "sample": sample, "cpu": _cpu_model()},
            "e2e": {"value": v, "unit": "dof-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="fit512", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        out = run_reference(args, rank)
    else:
        out = run_ours(args, rank, world, local_rank)
    if rank == 0 and out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
