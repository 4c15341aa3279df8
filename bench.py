"""Benchmark of the leapfrog time-stepping path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload batch128|fit512|gfdtd24|...]

A step is one leapfrog step (E half, sources, probe export, H half) over the
whole workload.  Default workload `batch128`: 128 independent gfdtd
simulations (Kuhn meshes of 8^3..48^3 cubes, own materials, sources and time
steps) advanced together in one device image, FP32 fields with FP64 CG
reductions, CG to ||r|| <= 1e-8 ||b||; the JSON line also carries the plain
FP64 arm (the same members one at a time, previous-solution guess) and the
probe error of small members against the FP64 CPU oracle.  Workload `fit512`:
the 512^3-cell Cartesian FIT cavity
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
    # Cartesian FIT cavities: 64^3 FP64 vacuum cavity, 512^3 FP32 with 200 random spheres
    "fit512": dict(kind="fit", n=512, spheres=200, prec="fp32", steps=5000),
    "fit64": dict(kind="fit", n=64, spheres=0, prec="fp64", steps=2000),
    "fit256": dict(kind="fit", n=256, spheres=200, prec="fp32", steps=2000),  # profiling size, state > L2
    # tetrahedral 1 m box, jittered Kuhn mesh of 24^3 or 96^3 cubes (96^3: GRF eps_r)
    "gfdtd24": dict(kind="tet", method="gfdtd", n=24, prec="fp64", steps=1200, cpu_n=24),
    "dga24": dict(kind="tet", method="dga", n=24, prec="fp64", steps=1200, cpu_n=24),
    "gfdtd96": dict(kind="tet", method="gfdtd", n=96, prec="fp32", steps=5000, grf=True, cpu_n=24),
    "gfdtd96_fp64": dict(kind="tet", method="gfdtd", n=96, prec="fp64", steps=5000, grf=True, cpu_n=24),
    # batched gfdtd: 128 members, n ~ U{8..48}, FP32 fields, FP64 CG reductions, CG to
    # ||r|| <= 1e-8 ||b||; the plain arm runs the same members one at a time in FP64 with the
    # reference's previous-solution guess
    "batch128": dict(kind="batch", members=128, n_lo=8, n_hi=48, steps=1000, seed=31337, prec="fp32",
                     warm="learned", learn_steps=300, crit="rhs", plain_steps=10),
    # the same scene at profiling size: 16 members n ~ U{8..32} (1.5 M CG rows, state > L2)
    "batch16": dict(kind="batch", members=16, n_lo=8, n_hi=32, steps=1000, seed=31337, prec="fp32",
                    warm="learned", learn_steps=40, crit="rhs", plain_steps=5),
    # DRAM-traffic capture size: 32 members n ~ U{8..48} (A about 0.7 GB, far above L2; about 2 GB held)
    "batch32": dict(kind="batch", members=32, n_lo=8, n_hi=48, steps=1000, seed=31337, prec="fp32",
                    warm="learned", learn_steps=40, crit="rhs", plain_steps=5),
    # learned warm start on one 96^3 Kuhn box (5.3 M tets), GRF eps_r
    "learned96": dict(kind="batch", members=1, n_lo=96, n_hi=96, steps=5000, seed=4242, prec="fp32",
                      warm="learned", learn_steps=500, crit="rhs", plain_steps=5, grf=True),
}


def max_over_ranks(values, dist=None, device="cpu"):
    """Element-wise maximum of per-rank timings over all ranks (the job's time
    is its slowest rank's); identity without a process group."""
    if dist is None:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t]


def replica_seed(base: int, rank: int) -> int:
    """Each rank of a multi-GPU run advances its own independent replica."""
    return base + rank


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

    def _lines(self):
        try:
            with open(self.path) as f:
                return sum(1 for _ in f)
        except OSError:
            return 0

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
            # the timed region opens once the sampler is live (its start-up
            # would otherwise swallow a short region)
            t0 = time.time()
            while self._lines() == 0 and time.time() - t0 < 3.0 and self.proc.poll() is None:
                time.sleep(0.01)
            self.n0 = self._lines()
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            # one more sample at the end of a region shorter than the period
            t0 = time.time()
            while self._lines() <= self.n0 and time.time() - t0 < 0.5 and self.proc.poll() is None:
                time.sleep(0.01)
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
    """Write the workload's script (and solids file or netgen mesh); return
    (script path, precision, case object)."""
    w = WORKLOADS[workload]
    if w["kind"] == "fit":
        from tetfit_b200.cases import FitCase, random_spheres, write_fit_cavity
        spheres = random_spheres(w["spheres"], seed=2026) if w["spheres"] else []
        case = FitCase(n=w["n"], steps=w["steps"], spheres=spheres)
        if n_override:
            # same scene and time step, coarser grid (bounded CPU sample)
            case = FitCase(n=n_override, steps=w["steps"], spheres=spheres, step=case.dt())
        return write_fit_cavity(workdir, case), w["prec"], case
    from tetfit_b200.cases import TetCase, grf_materials, write_tet_case
    kw = {}
    if w.get("grf"):
        mat, table, _ = grf_materials()
        kw = dict(mat_field=mat, eps=table)
    case = TetCase(n=w["n"], method=w["method"], steps=w["steps"], **kw)
    if n_override:
        case = TetCase(n=n_override, method=w["method"], steps=w["steps"], step=case.dt(), **kw)
    return write_tet_case(workdir, case), w["prec"], case


def fit_bytes(info: dict, es: int):
    """Algorithmic bytes of one E and one H launch (FIT byte model):
    E reads U and F and writes U; H reads F and U and writes F; plus 1 B of
    material index per cell each."""
    nE, nF, nc = info["n_edges"], info["n_faces"], info["n_cells"]
    e_bytes = es * (2 * nE + nF) + nc
    h_bytes = es * (2 * nF + nE) + nc
    return e_bytes, h_bytes


def phase_names(info):
    if info["method"] == "fdtd":
        return ["sources_bc", "e_update", "scatter_flux", "probes", "h_update"]
    if info["method"] == "dga":
        return ["sources", "e_update", "flux", "h_update", "probes"]
    return ["h_update_probes", "sources_rhs", "cg_solve", "scatter", "step_end"]


def describe(name, case, prec, info):
    if WORKLOADS[name]["kind"] == "fit":
        return (f"{name}: FIT cavity {case.n}^3 cells, {len(case.spheres)} lossy spheres, PEC surfaces 2-6, "
                f"H-wave source on surface 1, {prec} state, {info['n_probes']} probes every step")
    mats = "GRF eps_r in [1,12], 24 levels" if WORKLOADS[name].get("grf") else "vacuum"
    extra = f", CG tol {case.tolerance:g} (reference criterion), previous-solution guess" \
        if case.method == "gfdtd" else ""
    return (f"{name}: {case.method} on a jittered Kuhn box {case.n}^3 x 6 = {info['n_cells']} tets, {mats}, "
            f"PEC surfaces 2-6, H-wave source on surface 1, {prec} state{extra}")


def l2_note(info, es):
    state = (info["n_edges"] + 2 * info["n_faces"]) * es + info.get("nnz_operators", 0) * (4 + es) \
        + info.get("nnz_system", 0) * (4 + es)
    if state > 126e6:
        return f"state + operators {state / 1e6:.0f} MB > 126 MB L2 (no flush needed)"
    return f"state + operators {state / 1e6:.1f} MB fit in the 126 MB L2 (L2-resident workload, no flush)"


def roofline_kernel(d, info, es, ms5, nph):
    """(kernel name, algorithmic bytes per launch, launch ms, extra config)."""
    if info["method"] == "fdtd":
        e_bytes, h_bytes = fit_bytes(info, es)
        # the per-dof coefficient variant streams M_h, M_q (E) and M_nu, M_mu (H)
        # kernel variant = e + 8 h: 0 node slot, 1/2 z-march (4/16 planes),
        # 3 per-dof coefficients, 4 TMA-staged z-march, 5 coefficient classes
        ev, hv = info.get("cg_variant", 0) % 8, info.get("cg_variant", 0) // 8
        if ev == 3:
            e_bytes += 2 * es * info["n_edges"] - info["n_cells"]
        if hv == 3:
            h_bytes += 2 * es * info["n_faces"] - info["n_cells"]
        if ev == 5:  # a 2-byte class per edge instead of a material byte per cell
            e_bytes += 2 * info["n_edges"] - info["n_cells"]
        if hv == 5:
            h_bytes += 2 * info["n_faces"] - info["n_cells"]
        e_ms, h_ms = ms5[1] / nph, ms5[4] / nph
        names = {0: "fit_{}_kernel", 1: "fit_{}_march", 2: "fit_{}_march", 3: "fit_{}_coef", 4: "fit_{}_tma",
                 5: "fit_{}_class"}
        extra = {"e_variant": ev, "h_variant": hv}
        if e_ms >= h_ms:
            return names[ev].format("e"), e_bytes, e_ms, extra
        return names[hv].format("h"), h_bytes, h_ms, extra
    if info["method"] == "dga":
        # tet_curl_f + tet_h_update: C^T F gather and the H SpMV
        # bytes: C^T F gather (int32 per entry, F once, cb, I, cf written),
        # then the H SpMV (int32 + value per entry, cf once, U read/write)
        nE, nF = info["n_edges"], info["n_faces"]
        nnz_ct, nnz_h = 3 * nF, info["nnz_operators"]
        b = (nnz_ct * 4 + nE * 8 + nF * es + nE * 3 * es) + (nnz_h * (4 + es) + nE * (8 + 3 * es))
        return "tet_curl_f+tet_h_update", b, ms5[1] / nph, {}
    it, _ = d.solver_stats()
    its = it[-nph:]
    n, nnz = info["n_free"], info["nnz_system"]
    per_iter = nnz * (4 + es) + n * (13 * es + 8)
    setup = nnz * (4 + es) + n * (8 + 4 * es)
    b = float(its.mean()) * per_iter + setup
    return "tet_cg", b, ms5[2] / nph, {"cg_iterations_mean": float(its.mean()), "n_free": n, "nnz_A": nnz}


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
    info = d.prepare(1, precision=prec, device=local_rank,
                     graph_steps=1 if WORKLOADS[args.workload]["kind"] == "fit" and case.n >= 256 else 0)
    setup_s = time.time() - t0
    K, W = args.steps, args.warmup
    # FIT grids of >= 2 M cells time each kernel variant twice (at most 6
    # variants) in their first steps before settling: keep those steps in
    # the warm-up so the timed steps run the chosen kernels
    tune = 12 if info["method"] == "fdtd" and info["n_cells"] >= 2000000 else 0
    need = W + tune + K + min(K, 50) + 20
    if info["n_steps"] < need:
        raise SystemExit(f"workload has {info['n_steps']} steps, bench needs {need}")
    d.step(W + tune)
    info = {**info, **{k: v for k, v in d.info().items() if k == "cg_variant"}}
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
    # the script's own waveform for these steps, supplied from the host
    tshift = 0.5 if WORKLOADS[args.workload]["kind"] == "fit" else -0.5
    for i in range(K2):
        s = s0 + i + (0 if tshift > 0 else 1)
        carrier[:] = np.sin(2 * np.pi * case.frequency * (s * info["dt"] - 0.5 * info["dt"]))
        d.step_io(carrier, probe)
    e2e_s = time.perf_counter() - t0
    barrier()
    dofs = info["n_edges"] + info["n_faces"]
    max_ms, max_e2e = max_over_ranks([dev_ms, e2e_s], dist, f"cuda:{local_rank}")
    kps = info["kernels_per_step"]
    result = None
    if rank == 0:
        es = 4 if prec == "fp32" else 8
        dom, dom_bytes, dom_ms, extra = roofline_kernel(d, info, es, ms5, nph)
        peak, peak_kind = hbm_peak()
        achieved = dom_bytes / (dom_ms * 1e-3) / 1e9
        value = world * dofs * K / (max_ms * 1e-3)
        result = {
            "metric": "dof-steps/s", "value": value, "unit": "dof-steps/s", "n_gpus": world, "steps": K,
            "warmup": W, "ms_per_step": max_ms / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if prec == "fp32" else "f64", "data": "synthetic",
            "config": {"workload": describe(args.workload, case, prec, info),
                       "dofs": dofs, "cells": info["n_cells"], "parallelism": f"replicas x{world}",
                       "l2": l2_note(info, es), "setup_s": round(setup_s, 2), "autotune_steps": tune, **extra},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind,
                         "traffic": fit_traffic_estimate(dom, es, dom_bytes),
                         "traffic_note": FIT_TRAFFIC_NOTE if fit_traffic_estimate(dom, es, dom_bytes) else None,
                         "algorithmic_bytes": dom_bytes, "launch_ms": dom_ms},
            "phases_ms_per_step": {k: v / nph for k, v in zip(phase_names(info), ms5)},
            "e2e": {"value": world * dofs * K2 / max_e2e, "unit": "dof-steps/s",
                    "h2d_bytes_per_step": 8 * n_src, "d2h_bytes_per_step": 8 * 6 * info["n_probes"],
                    "api": "tf_step_io"},
            "gpu_launches": kps * K,
            "clocks": clk.summary(),
        }
        if world == 1 and not args.no_cpu_baseline:
            result["cpu_baseline"] = cpu_baseline(args, seconds=args.cpu_seconds)
    d.close()
    if rank == 0 and prec == "fp32" and WORKLOADS[args.workload]["kind"] == "fit" and not args.no_arms:
        result["precision_vs_fp64_gpu"] = precision_report(script, local_rank, steps=400, every=100)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return result


def precision_report(script, device, steps=400, every=100):
    """The same scene run from rest in FP32 and in FP64 on the GPU for a
    bounded number of steps: relative L2 of the FP32 probe series against the
    FP64 one, and the relative difference of the field energy (FP64
    accumulation on the GPU, tf_energy) at every `every` steps."""
    import tetfit_b200 as tb
    runs = {}
    for prec in ("fp64", "fp32"):
        with tb.Discretization(script) as d:
            d.prepare(1, precision=prec, device=device)
            en = []
            for _ in range(steps // every):
                d.step(every)
                en.append(d.energy())
            runs[prec] = (d.probes(), en)
    (t64, v64), e64 = runs["fp64"]
    (t32, v32), e32 = runs["fp32"]
    k = min(len(t32), len(t64))
    return {
        "steps": steps, "reference_run": "FP64 GPU run of the same scene (bitwise equal to the FP64 oracle at "
                                         "64^3 x 2000 steps)",
        "probe_rel_l2": _rel(v32[:k], v64[:k]),
        "energy": [{"step": every * (q + 1), "fp64": a, "fp32": b, "rel_diff": abs(b - a) / max(abs(a), 1e-300)}
                   for q, (a, b) in enumerate(zip(e64, e32))],
    }


# DRAM traffic of the FIT class kernels measured by ncu (one launch each of
# the 256^3 scene, state 607 MB > L2, 32 x 4 blocks): fit_e_class 689.7 MB
# against 709.4 MB algorithmic, fit_h_class 697.6 MB against 708.2 MB.  The ratio is per byte
# (one plane per block, the same re-use at every size), reported for the
# dominant kernel as ratio x its algorithmic bytes.
FIT_DRAM_OVER_ALGORITHMIC = {("fit_e_class", 4): 0.972, ("fit_h_class", 4): 0.985}
FIT_TRAFFIC_NOTE = "ncu DRAM bytes / algorithmic bytes of the kernel at 256^3, times this launch's algorithmic bytes"


def fit_traffic_estimate(kernel, es, nbytes):
    r = FIT_DRAM_OVER_ALGORITHMIC.get((kernel, es))
    return None if r is None else r * nbytes


def cg_bytes_per_launch(infos, its, es, dual=False):
    """Algorithmic bytes of one grp_cg launch: per member and iteration the
    entries of A (int32 column + value) and 11 row-vector accesses
    (p-update/SpMV phase: z, p_old, x read, x, p_new, q written; residual
    phase: r, q, pre read, r, z written), plus the initial residual (A once;
    b, pre read, r, z written; with the learned warm start's dual start also
    the second guess's residual read and its z written) and the final x
    update (x, p read, x written)."""
    total = 0.0
    for info, it in zip(infos, its):
        nnz, n = info["nnz_system"], info["n_free"]
        start = nnz * (4 + es) + 5 * es * n
        total += it * (nnz * (4 + es) + 11 * es * n) + start + (3 * es * n if dual else 0) + 3 * es * n
    return total


def member_carriers(infos, cases, steps_done):
    """The scripts' own H-wave carrier values (sin, source amplitude applied
    on the device) for each member's next step: t = (i + 1) dt - dt / 2."""
    out = []
    for info, case, i in zip(infos, cases, steps_done):
        t = (i + 1) * info["dt"] - 0.5 * info["dt"]
        out += [np.sin(2 * np.pi * case.frequency * t)] * info["n_sources"]
    return np.asarray(out if out else [0.0])


def batch_description(workload, cases):
    """The `config.workload` text of a batch workload (both bench arms)."""
    w = WORKLOADS[workload]
    learn = w.get("learn_steps", 0) if w["warm"] == "learned" else 0
    ns = sorted(c.n for c in cases)
    if w.get("grf"):
        scene = (f"{workload}: gfdtd on a {w['n_lo']}^3 x 6 jittered Kuhn box, eps_r from a seeded "
                 f"Gaussian random field (corr. 0.1 m) mapped to [1,12] in 24 levels, PEC box, H-wave source")
    else:
        scene = (f"{workload}: {w['members']} gfdtd members in one group, Kuhn meshes "
                 f"n ~ U{{{w['n_lo']}..{w['n_hi']}}} (min {ns[0]}, median {ns[len(ns) // 2]}, max {ns[-1]}) "
                 f"x 6 tets, eps_r ~ U[1,4] per x-half, f ~ U[1e8,4e8] Hz")
    return (scene + f", {w['prec']} fields, FP64 CG reductions, CG tol 1e-8 (||r|| <= tol ||b||), "
            f"{w['warm']} warm start" + (f" (network trained on the first {learn} steps, untimed)" if learn else ""))


def _sample_members(cases):
    """Members whose probe series are checked: the smallest, the quartiles,
    the median and the largest mesh (ties: the first in member order)."""
    order = sorted(range(len(cases)), key=lambda m: (cases[m].n, m))
    picks = [order[0], order[len(order) // 4], order[len(order) // 2], order[(3 * len(order)) // 4], order[-1]]
    return sorted(set(picks))


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def run_batch(args, rank, world, local_rank):
    import tetfit_b200 as tb
    from tetfit_b200.cases import batch_cases, write_batch
    w = WORKLOADS[args.workload]
    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist_
        dist = dist_
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))

    def barrier():
        if dist:
            import torch
            torch.cuda.synchronize()
            dist.barrier()

    # every rank runs its own batch of members (independent replicas)
    if w.get("grf"):
        from tetfit_b200.cases import TetCase, grf_materials
        mat, table, _ = grf_materials(seed=w["seed"])
        cases = [TetCase(n=w["n_lo"], method="gfdtd", steps=w["steps"], mat_field=mat, eps=table,
                         seed=replica_seed(0x7E7F17, rank))]
    else:
        cases = batch_cases(w["members"], w["n_lo"], w["n_hi"], steps=w["steps"], seed=replica_seed(w["seed"], rank))
    work = tempfile.mkdtemp(prefix=f"tfbatch{rank}_")
    t0 = time.time()
    members = write_batch(work, cases)
    write_s = time.time() - t0
    es = 4 if w["prec"] == "fp32" else 8
    t0 = time.time()
    learn = w.get("learn_steps", 0) if w["warm"] == "learned" else 0
    b = tb.Batch(members, precision=w["prec"], cg_criterion=w["crit"], warm_start=w["warm"], device=local_rank,
                 learn_steps=learn)
    setup_s = time.time() - t0
    infos = [b.info(m) for m in range(b.size)]
    dofs = sum(i["n_edges"] + i["n_faces"] for i in infos)
    K, W = args.steps, args.warmup
    nph = min(K, 10)
    K2 = min(K, 20)
    Kd = min(K, w.get("arm_steps", 10))
    need = learn + W + nph + K + K2
    if need > w["steps"]:
        raise SystemExit(f"batch members have {w['steps']} steps, bench needs {need}")
    # the learned warm start trains on its first steps (untimed), then W warm-up steps
    t0 = time.time()
    if learn:
        b.step(learn)
    train_s = time.time() - t0
    W = learn + W
    b.step(W - learn)
    ms5, _ = b.phase_times(nph)
    its_ph = [b.solver_stats(m)[0][W:W + nph].mean() for m in range(b.size)]
    cg_bytes = cg_bytes_per_launch(infos, its_ph, es, dual=bool(learn))
    cg_ms = ms5[2] / nph
    win0 = W + nph            # first step of the timed window
    barrier()
    with ClockSampler(local_rank) as clk:
        b.step(K)
        dev_ms = b.last_step_ms()
    barrier()
    stats = [b.solver_stats(m)[0] for m in range(b.size)]
    it_timed = float(np.mean([s_[win0:win0 + K].mean() for s_ in stats]))
    it_arm_window = float(np.mean([s_[win0:win0 + Kd].mean() for s_ in stats]))
    learned_info = None
    if learn:
        kept = np.concatenate([b.guess_stats(m)[win0:win0 + K] for m in range(b.size)])
        loss = b.training_loss()
        nz = loss[loss > 0]
        tenth = max(1, len(nz) // 10)
        learned_info = {"training_steps": learn, "training_s": round(train_s, 1), "adam_steps": int(len(loss)),
                        "loss_first": float(loss[0]) if len(loss) else None,
                        "loss_first_nonzero": float(nz[0]) if len(nz) else None,
                        "loss_mean_first_tenth": float(nz[:tenth].mean()) if len(nz) else None,
                        "loss_mean_last_tenth": float(nz[-tenth:].mean()) if len(nz) else None,
                        "loss_last": float(loss[-1]) if len(loss) else None,
                        "loss_note": "training loss of each Adam step on that step's new samples; the first "
                                     "steps' targets are zero (fields still zero), so the tenths use non-zero "
                                     "losses",
                        "network_guess_kept_frac": float(kept.mean())}
    # e2e: tf_batch_step_io, every member's carrier values H2D and probe samples D2H each step
    n_src = sum(i["n_sources"] for i in infos)
    n_probe_vals = 6 * sum(i["n_probes"] for i in infos)
    probes = np.zeros(max(n_probe_vals, 1))
    done = [win0 + K] * b.size
    barrier()
    t0 = time.perf_counter()
    for k in range(K2):
        b.step_io(member_carriers(infos, cases, [d_ + k for d_ in done]), probes)
    e2e_s = time.perf_counter() - t0
    barrier()
    # the CPU oracle steps members of up to 24^3 cubes within the bench's time
    smallest = [q for q in sorted(range(len(cases)), key=lambda q: (cases[q].n, q))[:3] if cases[q].n <= 24]
    check = sorted(set(_sample_members(cases)) | set(smallest)) if rank == 0 else []
    fp32_probes = {m: b.probes(m) for m in check}
    kps = infos[0]["kernels_per_step"]
    b.close()

    # Decomposition of the speed-up: the same members over the same window
    # [win0, win0 + Kd), batched in FP64 and FP32 with the reference's
    # previous-solution guess, batched FP32 with quadratic extrapolation, and
    # the plain FP64 form (members one at a time, previous-solution guess).
    arms = {}
    fp64_probes = {}

    def run_arm(name, **kw):
        t0_ = time.time()
        a = tb.Batch(members, cg_criterion=w["crit"], device=local_rank, **kw)
        su = time.time() - t0_
        a.step(win0)
        barrier()
        a.step(Kd)
        ms = a.last_step_ms()
        barrier()
        it = float(np.mean([a.solver_stats(m)[0][win0:win0 + Kd].mean() for m in range(a.size)]))
        if name == "batched_fp64_previous":
            for m in check:
                fp64_probes[m] = a.probes(m)
        a.close()
        arms[name] = {"ms_per_step": ms, "cg_iterations_mean": it, "setup_s": round(su, 1), **{
            k: v for k, v in kw.items() if k in ("precision", "warm_start", "batch_mode")}}

    if args.no_arms:
        # profiling runs: the headline arm only (the other arms' lines read null)
        arms = {k: {"ms_per_step": float("nan"), "cg_iterations_mean": float("nan")}
                for k in ("batched_fp64_previous", "batched_fp32_previous", "batched_fp32_extrapolate",
                          "plain_fp64")}
        fp64_probes = fp32_probes
    else:
        run_arm("batched_fp64_previous", precision="fp64", warm_start="previous")
        run_arm("batched_fp32_previous", precision="fp32", warm_start="previous")
        run_arm("batched_fp32_extrapolate", precision="fp32", warm_start="extrapolate")
        run_arm("plain_fp64", precision="fp64", warm_start="previous", batch_mode="serial")
    arm_names = list(arms)
    arm_ms = max_over_ranks([arms[k]["ms_per_step"] for k in arm_names], dist, f"cuda:{local_rank}")
    for k, v in zip(arm_names, arm_ms):
        arms[k]["ms_per_step"] = v / Kd
        arms[k]["value"] = world * dofs / (v / Kd * 1e-3)
    compare = None
    if args.compare_warm:
        compare = {"window": [win0, win0 + Kd], "learned": it_arm_window,
                   "previous": arms["batched_fp32_previous"]["cg_iterations_mean"],
                   "extrapolate": arms["batched_fp32_extrapolate"]["cg_iterations_mean"]}
        c = tb.Batch(members, precision=w["prec"], cg_criterion=w["crit"], warm_start="zero", device=local_rank)
        c.step(win0 + Kd)
        compare["zero"] = float(np.mean([c.solver_stats(m)[0][win0:win0 + Kd].mean() for m in range(c.size)]))
        c.close()
    # probe error of the FP32 learned run: against the batched FP64 run of the
    # same members (stratified sample incl. the largest mesh) over the steps
    # both took, and against the FP64 CPU oracle for the three smallest members
    perr, perr_oracle = {}, {}
    if rank == 0:
        for m in check:
            t32, v32 = fp32_probes[m]
            t64, v64 = fp64_probes[m]
            k = min(len(t32), len(t64))
            perr[m] = _rel(v32[:k], v64[:k])
        import oracle
        for m in ([] if args.no_arms else smallest):
            if m not in fp32_probes:
                continue
            t32, v32 = fp32_probes[m]
            o = oracle.TetOracle(members[m][0])
            o.step(len(t32))
            vo = o.probes()[1]
            o.close()
            perr_oracle[m] = _rel(v32, vo)
    max_ms, max_e2e = max_over_ranks([dev_ms, e2e_s], dist, f"cuda:{local_rank}")
    result = None
    if rank == 0:
        peak, peak_kind = hbm_peak()
        achieved = cg_bytes / (cg_ms * 1e-3) / 1e9
        value = world * dofs * K / (max_ms * 1e-3)
        desc = batch_description(args.workload, cases)
        plain = arms["plain_fp64"]
        decomposition = {
            "window_steps": [win0, win0 + Kd],
            "arms": arms,
            "learned_fp32_batched": {"value": value, "ms_per_step": max_ms / K, "cg_iterations_mean": it_timed,
                                     "cg_iterations_mean_arm_window": it_arm_window},
            "factors": {
                "batching (batched fp64 previous / plain fp64)":
                    arms["batched_fp64_previous"]["value"] / plain["value"],
                "precision (batched fp32 previous / batched fp64 previous)":
                    arms["batched_fp32_previous"]["value"] / arms["batched_fp64_previous"]["value"],
                "extrapolation (batched fp32 extrapolate / batched fp32 previous)":
                    arms["batched_fp32_extrapolate"]["value"] / arms["batched_fp32_previous"]["value"],
                "learned (learned fp32 batched / batched fp32 extrapolate)":
                    value / arms["batched_fp32_extrapolate"]["value"]},
            "criterion": "every GPU arm: ||r|| <= 1e-8 ||b||",
        }
        result = {
            "metric": "dof-steps/s", "value": value, "unit": "dof-steps/s", "n_gpus": world, "steps": K,
            "warmup": args.warmup, "ms_per_step": max_ms / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if es == 4 else "f64", "data": "synthetic",
            "config": {"workload": desc,
                       "members": w["members"], "dofs": dofs, "parallelism": f"replicas x{world}",
                       "l2": f"CG working set {cg_bytes / max(it_timed, 1) / 1e6:.0f} MB per iteration > 126 MB L2 "
                             f"(no flush needed)",
                       "setup_s": round(setup_s, 1), "mesh_write_s": round(write_s, 1),
                       "cg_iterations_mean": it_timed, "cg_variant": infos[0]["cg_variant"],
                       "cg_blocks": infos[0]["cg_blocks"]},
            "roofline": {"bound": "hbm", "kernel": "grp_cg", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind,
                         "traffic": cg_traffic_estimate(cg_bytes, es),
                         "traffic_note": CG_TRAFFIC_NOTE,
                         "algorithmic_bytes": cg_bytes, "launch_ms": cg_ms},
            "phases_ms_per_step": {k: v / nph for k, v in zip(
                ["h_update_probes", "sources_rhs", "cg_solve", "scatter", "step_end"], ms5)},
            "plain_fp64": {"value": plain["value"], "unit": "dof-steps/s", "ms_per_step": plain["ms_per_step"],
                           "steps": Kd, "window_steps": [win0, win0 + Kd],
                           "cg_iterations_mean": plain["cg_iterations_mean"],
                           "mode": "members one at a time, FP64, previous-solution guess, same CG tolerance",
                           "speedup": value / plain["value"]},
            "speedup_decomposition": decomposition,
            "probe_error_vs_fp64": {
                "reference_run": "batched FP64 GPU run of the same members (previous-solution guess, same "
                                 "tolerance), over the steps both took",
                "members": [{"member": m, "n": cases[m].n, "rel_l2": perr[m]} for m in sorted(perr)],
                "max_rel_l2": max(perr.values()) if perr else None},
            "probe_error_vs_fp64_oracle": {"members": [{"member": m, "n": cases[m].n, "rel_l2": v}
                                                       for m, v in sorted(perr_oracle.items())],
                                           "max_rel_l2": max(perr_oracle.values()) if perr_oracle else None},
            "learned_warm_start": learned_info,
            "cg_iterations_by_warm_start": compare or {
                "window": [win0, win0 + Kd], "learned": it_arm_window,
                "previous": arms["batched_fp32_previous"]["cg_iterations_mean"],
                "extrapolate": arms["batched_fp32_extrapolate"]["cg_iterations_mean"],
                "previous_fp64": arms["batched_fp64_previous"]["cg_iterations_mean"]},
            "e2e": {"value": world * dofs * K2 / max_e2e, "unit": "dof-steps/s",
                    "h2d_bytes_per_step": 8 * n_src, "d2h_bytes_per_step": 8 * n_probe_vals,
                    "api": "tf_batch_step_io"},
            "gpu_launches": kps * K,
            "clocks": clk.summary(),
        }
        if world == 1 and not args.no_cpu_baseline:
            result["cpu_baseline"] = batch_cpu_baseline(cases, members, seconds=args.cpu_seconds)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return result


# DRAM traffic of grp_cg measured by ncu (dram__bytes_read.sum +
# dram__bytes_write.sum) on two launches of the 32-member batch (n ~ U{8..48},
# FP32 state, A about 0.7 GB, far above L2): 13.05 GB read + 2.41 GB write
# per launch against 15.08 GB of algorithmic bytes, a ratio of 1.025.  The
# traffic reported for a launch is that ratio times its algorithmic bytes
# (traffic grows with the row-iterations, as the algorithmic bytes do).
CG_DRAM_OVER_ALGORITHMIC = {4: 1.025}
CG_TRAFFIC_NOTE = ("ncu DRAM bytes of captured grp_cg launches (32-member FP32 batch) / their algorithmic "
                   "bytes = 1.025, times this launch's algorithmic bytes")


def cg_traffic_estimate(cg_bytes, es):
    r = CG_DRAM_OVER_ALGORITHMIC.get(es)
    return None if r is None else r * cg_bytes


def batch_cpu_baseline(cases, members, seconds=15.0):
    """FP64 CPU restatement, single thread, stepping members in order for a
    bounded time (the reference runs a script's simulations one by one);
    beside it the same with one member per host thread (all cores)."""
    import oracle
    os.environ["TF_ORACLE_SKIP_DT"] = "1"
    t_all, dofs_steps, used = 0.0, 0.0, 0
    order = sorted(range(len(cases)), key=lambda m: (cases[m].n, m))
    # a stratified sample: members across the size range, smallest first
    pick = [order[int(q * (len(order) - 1) / 7)] for q in range(8)] if len(order) >= 8 else order
    for m in pick:
        if t_all >= seconds:
            break
        o = oracle.TetOracle(members[m][0])
        dofs = o.nE + o.nF
        o.step(1)
        t0 = time.perf_counter()
        k = 0
        while time.perf_counter() - t0 < max(seconds - t_all, 0.5) / 2 and k < 200:
            k += o.step(1)
        el = time.perf_counter() - t0
        o.close()
        t_all += el
        dofs_steps += dofs * k
        used += 1
    out = {"value": dofs_steps / t_all, "unit": "dof-steps/s", "cores": 1, "kind": "port",
           "sample": f"{used} batch members across the size range (n = "
                     f"{', '.join(str(cases[m].n) for m in pick[:used])}) stepped one after another (FP64, the "
                     f"reference's criterion and previous-solution guess), {t_all:.1f} s",
           "cpu": _cpu_model()}
    allc = _reference_pool([members[m][0] for m in pick], warm=1, steps=3)
    out["all_cores"] = {"value": allc["value"], "unit": "dof-steps/s", "cores": allc["cores"],
                        "sample": f"the same {len(pick)} members, one per host process, 3 steps each"}
    return out


def cpu_baseline(args, seconds=15.0, threads=None):
    """FP64 CPU restatement of the reference on a bounded sample of the scene."""
    import oracle
    work = tempfile.mkdtemp(prefix="tfcpu_")
    n_sample = sample_size(args.workload)
    script, _, _ = make_case(work, args.workload, n_override=n_sample)
    if threads:
        os.environ["OMP_NUM_THREADS"] = str(threads)
    os.environ["TF_ORACLE_SKIP_DT"] = "1"  # the step is pinned; skip the setup-only eigen-estimate
    o = open_oracle(args.workload, script)
    dofs = o.nE + o.nF
    o.step(2)
    t0 = time.perf_counter()
    n = 0
    while time.perf_counter() - t0 < seconds and n + 10 <= o.n_steps - 2:
        n += o.step(10)
    el = time.perf_counter() - t0
    o.close()
    cores = oracle_threads(args.workload)
    return {"value": dofs * n / el, "unit": "dof-steps/s", "cores": cores, "kind": "port",
            "sample": f"{n_sample}^3 grid of the same scene (FP64), {n} steps, {el:.1f} s, "
                      f"threads={cores}", "cpu": _cpu_model()}


def sample_size(workload):
    w = WORKLOADS[workload]
    if w["kind"] == "fit":
        return 96 if w["n"] > 96 else w["n"]
    return w.get("cpu_n", w["n"])


def open_oracle(workload, script):
    import oracle
    if WORKLOADS[workload]["kind"] == "fit":
        return oracle.FitOracle(script, omp=True)
    return oracle.TetOracle(script, omp=True)


def oracle_threads(workload):
    # the tetrahedral restatement is single-threaded, as the reference
    if WORKLOADS[workload]["kind"] != "fit":
        return 1
    return int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))


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
    n_sample = sample_size(args.workload)
    script, _, _ = make_case(work, args.workload, n_override=n_sample)
    os.environ["TF_ORACLE_SKIP_DT"] = "1"  # the step is pinned; skip the setup-only eigen-estimate
    o = open_oracle(args.workload, script)
    dofs = o.nE + o.nF
    o.step(args.warmup)
    t0 = time.perf_counter()
    o.step(args.steps)
    el = time.perf_counter() - t0
    o.close()
    v = dofs * args.steps / el
    cores = oracle_threads(args.workload)
    sample = (f"{n_sample}^3 grid of the {args.workload} scene, FP64 C++ restatement of the reference "
              f"(reference needs Eigen/Spectra/GSL/Silo, not buildable here), {args.steps} steps")
    return {"impl": "reference", "metric": "dof-steps/s", "value": v, "unit": "dof-steps/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": el * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": f"{args.workload} (bounded CPU sample {n_sample}^3)"},
            "cpu_baseline": {"value": v, "unit": "dof-steps/s", "cores": cores, "kind": "port",
                             "sample": sample, "cpu": _cpu_model()},
            "e2e": {"value": v, "unit": "dof-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def _ref_member(arg):
    """Worker: the FP64 restatement of the reference on one batch member
    (its own criterion ||r||/||r0|| <= tol and previous-solution guess)."""
    script, warm, steps = arg
    os.environ["TF_ORACLE_SKIP_DT"] = "1"
    os.environ["OMP_NUM_THREADS"] = "1"
    import oracle
    o = oracle.TetOracle(script)
    dofs = o.nE + o.nF
    o.step(warm)
    t0 = time.perf_counter()
    k = o.step(steps)
    el = time.perf_counter() - t0
    o.close()
    return dofs, el, k


def _reference_pool(scripts, warm, steps):
    """The reference's CPU path on independent members with every host core:
    one member per worker process, largest meshes first.  Throughput = the
    members' dof-steps over their summed timed seconds, times the number of
    workers (all workers run side by side until the queue drains)."""
    import multiprocessing as mp
    workers = max(1, min(os.cpu_count() or 1, len(scripts)))
    sizes = [os.path.getsize(os.path.join(os.path.dirname(sc), "box.mesh"))
             if os.path.exists(os.path.join(os.path.dirname(sc), "box.mesh")) else 0 for sc in scripts]
    order = sorted(range(len(scripts)), key=lambda q: -sizes[q])
    with mp.get_context("spawn").Pool(workers) as pool:
        res = pool.map(_ref_member, [(scripts[q], warm, steps) for q in order], chunksize=1)
    work = sum(r[0] * r[2] for r in res)
    secs = sum(r[1] for r in res)
    return {"value": work / secs * workers, "cores": workers, "members": len(scripts),
            "dof_steps": work, "core_seconds": secs}


def run_batch_reference(args, rank):
    """The reference's CPU path on the whole batch: every member (the same
    members, meshes, materials, sources and time steps as the GPU arm), one
    member per host core, each advanced a few warm-up steps and then a few
    timed steps with the reference's own CG criterion and initial guess."""
    if rank != 0:
        return None
    from tetfit_b200.cases import batch_cases, write_batch
    w = WORKLOADS[args.workload]
    if w.get("grf"):
        return {"impl": "reference", "unavailable": "reference arm defined for the uneven-member batches only"}
    cases = batch_cases(w["members"], w["n_lo"], w["n_hi"], steps=w["steps"], seed=w["seed"])
    work = tempfile.mkdtemp(prefix="tfbref_")
    members = write_batch(work, cases)
    warm, steps = min(args.warmup, 2), min(args.steps, 5)
    r = _reference_pool([m[0] for m in members], warm, steps)
    v = r["value"]
    sample = (f"all {r['members']} batch members, one per host process ({r['cores']} processes), FP64 C++ "
              f"restatement of the reference (the reference needs Eigen/Spectra/GSL/Silo, not buildable here), "
              f"{warm} warm-up + {steps} timed steps each; throughput = member dof-steps / summed timed "
              f"seconds x processes")
    return {"impl": "reference", "metric": "dof-steps/s", "value": v, "unit": "dof-steps/s", "n_gpus": 1,
            "steps": steps, "warmup": warm, "ms_per_step": 1e3 * (r["dof_steps"] / steps) / v,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": batch_description(args.workload, cases), "members": w["members"],
                       "parallelism": "host processes", "cpu_sample": "every member",
                       "cg": "reference criterion ||r||/||r0|| <= 1e-8, previous-solution guess, FP64"},
            "cpu_baseline": {"value": v, "unit": "dof-steps/s", "cores": r["cores"], "kind": "port",
                             "sample": sample, "cpu": _cpu_model()},
            "e2e": {"value": v, "unit": "dof-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batch128", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-arms", action="store_true",
                    help="batch workloads: skip the speed-up decomposition arms and the probe checks (profiling)")
    ap.add_argument("--compare-warm", action="store_true",
                    help="batch workloads: also run the zero, previous and extrapolation warm starts and report "
                         "their CG iterations per step over the timed window")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        out = run_reference(args, rank) if WORKLOADS[args.workload]["kind"] != "batch" \
            else run_batch_reference(args, rank)
    elif WORKLOADS[args.workload]["kind"] == "batch":
        out = run_batch(args, rank, world, local_rank)
    else:
        out = run_ours(args, rank, world, local_rank)
    if rank == 0 and out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
