"""Benchmark of the force-evaluation path on B200 (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME]
                    [--impl b200|reference]

Workloads (seeded synthetic inputs with the shapes of the measured configs):
  bh-collision-2m          two disc galaxies, 2,000,000 particles, Barnes-Hut
                           theta 0.5 with quadrupoles, leaf 32, eps 0.02, FP32
                           force / FP64 state, velocity Verlet dt 5e-4; a step
                           is one VV step (Morton order, tree, walk, kicks).
                           Metric: BH ms/step at 2M (lower is better).
  bh-collision-500k        the same scenario at 500,000 particles (profiling size).
  direct-plummer-4096      Plummer sphere N=4096, eps 0.01, FP32 direct, VV
                           dt 1e-3. Metric: direct Gint/s, N(N-1) per step.
  direct-plummer-262144-fp32  Plummer N=262,144, FP32 direct, VV dt 1e-3: the
                           plain kernel at a size that fills the GPU.
  batched-512              512 independent Plummer clusters, N log-uniform in
                           [256, 16384], scale radius U[0.5, 2], eps = 0.01 x
                           radius, split precision, all systems in one
                           persistent launch, Yoshida-4 dt 1e-3 as one graph.
  serving                  a seeded Poisson stream of jobs at 20 jobs/s (70% direct
                           Plummer N 1k..64k x 200..2000 Yoshida-4 steps, 30%
                           Barnes-Hut collisions N 100k..4M x 100..500 VV steps)
                           fed in real time for --window seconds to the serving
                           loop and, separately, to the plain drop-in run
                           serially; completed jobs/s and latencies of both.
  direct-plummer-262144    the same at N=262,144 with the split-precision
                           kernel and Yoshida-4 dt 1e-3 (3 evaluations/step).

Timing: W untimed warm-up steps, then exactly K steps bracketed by a barrier
and torch.cuda.synchronize() on both sides, timed with CUDA events on the
stream the work runs on, max over ranks. One step is a replayed CUDA graph.
Per-phase device times inside the timed region come from event nodes in the
graph (DeviceSystem.profile). Under torchrun every rank runs an independent
replica on its own GPU (the path has no exchange step: replicas only).
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
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

L2_BYTES = 126 * 1024 * 1024


# ---------------------------------------------------------------------------
# Workloads
# ---------------------------------------------------------------------------

WORKLOADS = {
    "bh-collision-2m": dict(kind="tree", n=2_000_000, eps=0.02, dt=5e-4, integrator="vv",
                            theta=0.5, leaf=32, quadrupole=True, precision="fp32",
                            metric="BH ms/step at 2M", unit="ms/step", higher=False,
                            generator="collision"),
    # The parity mode: forces bit-identical to the reference's FP64
    # BarnesHutSolver (scalar leaf kernel).
    "bh-collision-2m-fp64": dict(kind="tree", n=2_000_000, eps=0.02, dt=5e-4, integrator="vv",
                                 theta=0.5, leaf=32, quadrupole=True, precision="fp64",
                                 metric="BH ms/step at 2M (FP64 parity)", unit="ms/step",
                                 higher=False, generator="collision"),
    # The same scenario at a quarter of the size, for profiler captures.
    "bh-collision-500k": dict(kind="tree", n=500_000, eps=0.02, dt=5e-4, integrator="vv",
                              theta=0.5, leaf=32, quadrupole=True, precision="fp32",
                              metric="BH ms/step at 500k", unit="ms/step", higher=False,
                              generator="collision"),
    "direct-plummer-4096": dict(kind="direct", n=4096, eps=0.01, dt=1e-3, integrator="vv",
                                precision="fp32", metric="direct Gint/s", unit="Gint/s",
                                higher=True, generator="plummer"),
    "direct-plummer-262144-fp32": dict(kind="direct", n=262_144, eps=0.01, dt=1e-3,
                                       integrator="vv", precision="fp32",
                                       metric="direct Gint/s", unit="Gint/s", higher=True,
                                       generator="plummer"),
    "batched-512": dict(kind="batch", n=512, eps=0.01, dt=1e-3, integrator="yoshida4",
                        precision="split", metric="batched Gint/s", unit="Gint/s", higher=True,
                        generator="clusters"),
    "serving": dict(kind="serving", n=0, eps=0.01, dt=1e-3, integrator="yoshida4",
                    precision="split", metric="served jobs/s", unit="jobs/s", higher=True,
                    generator="stream"),
    "direct-plummer-262144": dict(kind="direct", n=262_144, eps=0.01, dt=1e-3,
                                  integrator="yoshida4", precision="split",
                                  metric="direct Gint/s", unit="Gint/s", higher=True,
                                  generator="plummer"),
    # Run output of the 2M collision: trajectory frames (positions and
    # velocities) every `stride` steps and checkpoints, in the reference's
    # formats.
    "run-output-2m": dict(kind="output", n=2_000_000, eps=0.02, dt=5e-4, integrator="vv",
                          theta=0.5, leaf=32, quadrupole=True, precision="fp32",
                          metric="run time per trajectory frame at 2M", unit="ms/frame",
                          higher=False, generator="collision", stride=5),
}
DEFAULT_WORKLOAD = "bh-collision-2m"


def make_clusters(count, seed=20260813):
    """512-cluster batch: sizes log-uniform in [256, 16384], radii U[0.5, 2]."""
    from orrery_b200 import initial_conditions as ic

    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(256), np.log(16384), count)).astype(np.int64)
    radii = rng.uniform(0.5, 2.0, count)
    systems = [ic.plummer_sphere(int(n), scale_radius=float(a), seed=seed + 1 + k)
               for k, (n, a) in enumerate(zip(sizes, radii))]
    return sizes, radii, systems


def make_inputs(w, seed=20260811):
    from orrery_b200 import initial_conditions as ic

    if w["generator"] == "clusters":
        return make_clusters(w["n"])
    if w["generator"] == "plummer":
        return ic.plummer_sphere(w["n"], seed=seed)
    return ic.galaxy_collision(w["n"], softening=w["eps"], seed=seed)


def evaluations_per_step(w):
    return 3 if w["integrator"] == "yoshida4" else 1


def step_units(w):
    """Units of the metric one step processes (interactions, or one step)."""
    if w["kind"] == "direct":
        return evaluations_per_step(w) * w["n"] * (w["n"] - 1)
    return 1


def dtype_of(w):
    """The arithmetic the force path computes in."""
    return {"fp32": "f32", "split": "f32-split (hi/lo FP32 pair math, FP64 sums)",
            "fp64": "f64"}[w["precision"]]


def relative_errors(got, exact):
    """Per-particle |a - a_ref| / |a_ref| over particles with a nonzero a_ref."""
    mag = np.linalg.norm(exact, axis=1)
    ok = mag > 0
    return np.linalg.norm(got - exact, axis=1)[ok] / mag[ok]


def error_summary(err, against):
    return {"median": float(np.median(err)), "max": float(np.max(err)),
            "rms": float(np.sqrt(np.mean(err ** 2))), "particles": int(err.size),
            "against": against}


def direct_fp64_sampled(torch, device, st, m, eps, targets, chunk=1 << 14):
    """FP64 direct sum sum_j m_j d / (|d|^2 + eps^2)^(3/2) at the sampled
    targets over every source, on the device (torch FP64; a measurement of the
    error, not the product path). The target's own term is exactly zero under
    softening, as the reference's skip makes it."""
    pos = torch.tensor(np.stack([st["x"], st["y"], st["z"]], axis=1), dtype=torch.float64,
                       device=device)
    mass = torch.tensor(m, dtype=torch.float64, device=device)
    tgt = pos[torch.as_tensor(targets, device=device)]
    acc = torch.zeros_like(tgt)
    for start in range(0, pos.shape[0], chunk):
        d = pos[start:start + chunk][None, :, :] - tgt[:, None, :]
        r2 = (d * d).sum(-1) + eps * eps
        w = mass[start:start + chunk][None, :] / (r2 * torch.sqrt(r2))
        acc += (w[:, :, None] * d).sum(1)
    return acc.cpu().numpy()


# ---------------------------------------------------------------------------
# Clocks during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    """nvidia-smi sampling every 200 ms while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device = device_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200", "-f", self.path],
                stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        rows = []
        if self.path and os.path.exists(self.path):
            with open(self.path) as fh:
                for line in fh:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) >= 9:
                        rows.append(parts)
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4)
                          if r[5 + k].lower().startswith("active")})
        load = [v for v in sm if mx and v > 0.5 * max(mx)] or sm
        return {"sm_mhz": statistics.median(load) if load else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


# ---------------------------------------------------------------------------
# Distributed plumbing
# ---------------------------------------------------------------------------

def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def init_dist(world, backend):
    import datetime

    import torch.distributed as dist

    if world > 1 and not dist.is_initialized():
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
    return dist if world > 1 else None


def reduce_max(dist, value, device):
    if dist is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


# ---------------------------------------------------------------------------
# CPU baseline: the reference's own CPU solvers on this host's cores
# ---------------------------------------------------------------------------

def cpu_baseline(w, data, budget_s=20.0):
    """Times the reference's CPU implementation (oracle/_ref) on a bounded
    sample of the workload; returns the cpu_baseline object."""
    import oracle

    if not oracle.Reference.available():
        r = oracle.Restatement()
        kind = "port"
        cores = 1
        n = min(w["n"], 2048)
        sub = {k: np.ascontiguousarray(v[:n]) for k, v in data.items()}
        t0 = time.perf_counter()
        if w["kind"] == "direct":
            r.direct(sub["x"], sub["y"], sub["z"], sub["m"], w["eps"])
            sec = time.perf_counter() - t0
            value = n * (n - 1) / sec / 1e9
            return dict(value=value, unit="Gint/s", cores=cores, kind=kind,
                        sample=f"one scalar direct evaluation of {n} particles")
        r.barnes_hut(sub["x"], sub["y"], sub["z"], sub["m"], w["eps"], w["theta"], w["leaf"],
                     w["quadrupole"])
        sec = time.perf_counter() - t0
        return dict(value=sec * 1e3, unit="ms/step", cores=cores, kind=kind,
                    sample=f"one scalar Barnes-Hut evaluation of {n} particles (not 2M)")
    ref = oracle.Reference()
    threads = ref.worker_count()
    x, y, z, m = (np.ascontiguousarray(data[k]) for k in ("x", "y", "z", "m"))
    if w["kind"] == "direct":
        n = len(m)
        # One evaluation first to size the sample to the budget.
        one = ref.direct_seconds(x, y, z, m, w["eps"], threads, repeats=1)
        reps = max(1, min(int(budget_s / max(one, 1e-6)),
                          100 * evaluations_per_step(w)))
        sec = ref.direct_seconds(x, y, z, m, w["eps"], threads, repeats=reps)
        value = n * (n - 1) / sec / 1e9
        return dict(value=value, unit="Gint/s", cores=threads, kind="reference",
                    evaluations_timed=reps,
                    steps_timed=reps / evaluations_per_step(w),
                    sample=f"{reps} DirectSolver evaluations (AVX2, {threads} threads) "
                           f"of the full {n}-particle input")
    one = ref.barnes_hut_seconds(x, y, z, m, w["eps"], w["theta"], w["leaf"], w["quadrupole"],
                                 threads, repeats=1)
    reps = max(1, min(int(budget_s / max(one, 1e-6)) - 1, 10))
    sec = one
    if reps > 1:
        sec = ref.barnes_hut_seconds(x, y, z, m, w["eps"], w["theta"], w["leaf"],
                                     w["quadrupole"], threads, repeats=reps)
    return dict(value=sec * 1e3 * evaluations_per_step(w), unit="ms/step", cores=threads,
                kind="reference", evaluations_timed=reps,
                steps_timed=reps / evaluations_per_step(w),
                sample=f"{reps} BarnesHutSolver evaluation(s) (AVX2 leaves, {threads} threads) "
                       f"of the full {len(m)}-particle input, after one untimed; one "
                       "evaluation is one VV step's force work (the O(N) kicks are not "
                       "timed: under 0.1 % of the step)")


def cpu_baseline_batch(w, sizes, radii, systems, budget_s=15.0):
    """The reference's DirectSolver (AVX2, all host threads, one solver per
    system with its own softening) on the clusters in order until the budget
    is spent; the rate over the systems done stands for the batch."""
    import oracle

    ref = oracle.Reference()
    threads = ref.worker_count()
    done_pairs, spent, count = 0, 0.0, 0
    for k, d in enumerate(systems):
        sec = ref.direct_seconds(d["x"], d["y"], d["z"], d["m"], w["eps"] * radii[k], threads,
                                 repeats=1)
        n = int(sizes[k])
        done_pairs += n * (n - 1)
        spent += sec
        count += 1
        if spent > budget_s:
            break
    return dict(value=done_pairs / spent / 1e9, unit="Gint/s", cores=threads, kind="reference",
                sample=f"one DirectSolver evaluation (AVX2, {threads} threads) of each of the "
                       f"first {count} of {len(systems)} clusters")


def cpu_baseline_serving(w, budget_s):
    """The reference's CPU solvers (all host threads) on the serving stream in
    arrival order: one timed force evaluation per job until the budget is
    spent, each job's time taken as that evaluation times its evaluation count
    (its own steps x evaluations per step, plus the initial one)."""
    import oracle

    ref = oracle.Reference()
    threads = ref.worker_count()
    jobs = make_stream(3.0)
    states = job_states(jobs)
    projected, spent, done = 0.0, 0.0, 0
    for job, st in zip(jobs, states):
        p = JOB_PARAMS[job["kind"]]
        if job["kind"] == "direct":
            sec = ref.direct_seconds(st["x"], st["y"], st["z"], st["m"], p["softening"], threads,
                                     repeats=1)
            evals = 1 + 3 * job["steps"]
        else:
            sec = ref.barnes_hut_seconds(st["x"], st["y"], st["z"], st["m"], p["softening"],
                                         p["theta"], p["leaf"], True, threads, repeats=1)
            evals = 1 + job["steps"]
        projected += sec * evals
        spent += sec
        done += 1
        if spent > budget_s:
            break
    return dict(value=done / projected, unit="jobs/s", cores=threads, kind="reference",
                sample=f"one timed force evaluation of each of the stream's first {done} jobs "
                       f"(of {len(jobs)}), scaled by each job's evaluation count; jobs run "
                       "serially")


def reference_gpu_serving(budget_s):
    """The reference's own CUDA solvers on the serving stream in arrival order:
    one timed host-buffer evaluation per job (after one warm-up evaluation)
    until the budget is spent, each job's time taken as that evaluation times
    its evaluation count; jobs serial. None without the library or a device."""
    import oracle

    if not oracle.ReferenceCuda.built():
        return None
    try:
        ref = oracle.ReferenceCuda()
        if not ref.available():
            return None
        threads = oracle.Reference().worker_count() if oracle.Reference.available() else 1
        jobs = make_stream(3.0)
        states = job_states(jobs)
        projected, spent, done = 0.0, 0.0, 0
        for job, st in zip(jobs, states):
            p = JOB_PARAMS[job["kind"]]
            if job["kind"] == "direct":
                wall, _, _ = ref.direct_timed(st["x"], st["y"], st["z"], st["m"], p["softening"],
                                              repeats=1)
                evals = 1 + 3 * job["steps"]
            else:
                wall, _, _, _ = ref.tree_timed(st["x"], st["y"], st["z"], st["m"], p["softening"],
                                               p["theta"], p["leaf"], True, threads, repeats=1)
                evals = 1 + job["steps"]
            projected += wall * evals
            spent += 2 * wall
            done += 1
            if spent > budget_s:
                break
        return {"solvers": "CudaDirectSolver (FP64) and CudaTreeSolver (host build on "
                           f"{threads} threads), the reference's own GPU path",
                "value": done / projected, "unit": "jobs/s",
                "sample": f"one timed evaluation of each of the stream's first {done} jobs "
                          f"(of {len(jobs)}), scaled by each job's evaluation count; jobs "
                          "run serially"}
    except (OSError, RuntimeError) as err:
        return {"unavailable": str(err)}


def reference_gpu(w, data):
    """The reference's own CUDA solvers (its .cu kernels built for sm_100a by
    oracle/Makefile) on the same input and device, when built and a device is
    present: per-evaluation wall time of its host-buffer evaluate and its
    kernel time."""
    import oracle

    if w["kind"] not in ("direct", "tree") or not oracle.ReferenceCuda.built():
        return None
    try:
        ref = oracle.ReferenceCuda()
        if not ref.available():
            return None
        x, y, z, m = (np.ascontiguousarray(data[k]) for k in ("x", "y", "z", "m"))
        n = len(m)
        builds = [("f64", ref)]
        if oracle.ReferenceCuda.built(single=True):
            builds.append(("f32", oracle.ReferenceCuda(single=True)))
        out = {}
        threads = oracle.Reference().worker_count() if oracle.Reference.available() else 1
        for real, r in builds:
            if w["kind"] == "direct":
                wall, kern, _ = r.direct_timed(x, y, z, m, w["eps"], repeats=3)
                out[real] = {"solver": f"CudaDirectSolver ({real} Real build, the reference's "
                                       "direct_kernel)",
                             "kernel_gint_s": n * (n - 1) / kern / 1e9,
                             "evaluate_gint_s": n * (n - 1) / wall / 1e9,
                             "kernel_ms": kern * 1e3, "evaluate_ms": wall * 1e3}
            else:
                wall, kern, _, counts = r.tree_timed(x, y, z, m, w["eps"], w["theta"], w["leaf"],
                                                     w["quadrupole"], threads, repeats=1)
                out[real] = {"solver": f"CudaTreeSolver ({real} Real build; host sort and "
                                       f"build on {threads} threads, coherent traversal on "
                                       "the device)",
                             "evaluate_ms": wall * 1e3, "kernel_ms": kern * 1e3,
                             "pairs": counts[0], "cells": counts[1]}
        # The double-precision build's figures stay at the top level.
        line = dict(out["f64"])
        if "f32" in out:
            line["single_precision_build"] = out["f32"]
        return line
    except (OSError, RuntimeError) as err:
        return {"unavailable": str(err)}


def run_reference(args, w):
    world, rank, local = dist_env()
    dist = init_dist(world, "gloo")
    if rank != 0:
        barrier(dist)
        return
    steps = max(1, args.steps)
    if w["kind"] == "serving":
        base = cpu_baseline_serving(w, budget_s=min(60.0, 10.0 * steps))
        line = {"impl": "reference", "metric": w["metric"], "value": base["value"],
                "unit": "jobs/s", "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup,
                "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": args.workload, "arrival_window_s": 3.0},
                "cpu_baseline": base,
                "e2e": {"value": base["value"], "unit": "jobs/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        gpu = reference_gpu_serving(budget_s=min(120.0, 20.0 * steps))
        if gpu is not None:
            line["reference_gpu"] = gpu
        print(json.dumps(line), flush=True)
        barrier(dist)
        return
    if w["kind"] == "output":
        import tempfile

        directory = tempfile.mkdtemp(prefix="orrery_output_ref_")
        base = cpu_baseline_output(w, make_inputs(w), directory)
        os.rmdir(directory)
        line = {"impl": "reference", "metric": w["metric"], "value": base.get("value"),
                "unit": "ms/frame", "n_gpus": args.gpus, "steps": steps,
                "warmup": args.warmup, "ms_per_step": None, "higher_is_better": False,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": args.workload, "n": w["n"], "stride": w["stride"]},
                "cpu_baseline": base,
                "e2e": {"value": base.get("value"), "unit": "ms/frame", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        if "unavailable" in base:
            line = {"impl": "reference", "unavailable": base["unavailable"]}
        print(json.dumps(line), flush=True)
        barrier(dist)
        return
    data = make_inputs(w)
    if w["kind"] == "batch":
        base = cpu_baseline_batch(w, *data, budget_s=min(60.0, 10.0 * steps))
    else:
        base = cpu_baseline(w, data, budget_s=min(60.0, 10.0 * steps))
    value = base["value"]
    if w["kind"] == "batch":
        pairs = sum(int(n) * (int(n) - 1) for n in data[0])
        ms_per_step = pairs * evaluations_per_step(w) / (value * 1e9) * 1e3
    else:
        ms_per_step = value if w["unit"] == "ms/step" else \
            step_units(w) / (value * 1e9) * 1e3
    # `steps`: the steps' worth of work actually timed (a bounded sample: the
    # CPU takes seconds per 2M evaluation), not the requested K.
    timed = base.get("steps_timed", steps)
    line = {
        "impl": "reference", "metric": w["metric"], "value": value, "unit": w["unit"],
        "n_gpus": args.gpus, "steps": timed, "steps_requested": steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": w["higher"],
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "sampled": f"value measured on {base.get('evaluations_timed', '?')} evaluation(s) of "
                   "the full input and stated per step",
        "config": config_of(args, w), "cpu_baseline": base,
        "e2e": {"value": value, "unit": w["unit"], "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    gpu = reference_gpu(w, data) if w["kind"] != "batch" else None
    if gpu is not None:
        line["reference_gpu"] = gpu
    print(json.dumps(line), flush=True)
    barrier(dist)


def config_of(args, w):
    if w["kind"] == "batch":
        return {"workload": args.workload, "systems": w["n"], "precision": w["precision"],
                "integrator": w["integrator"], "dt": w["dt"], "replicas": args.gpus}
    c = {"workload": args.workload, "n": w["n"], "solver": w["kind"],
         "precision": w["precision"], "softening": w["eps"], "dt": w["dt"],
         "integrator": w["integrator"], "replicas": args.gpus,
         "l2": "inputs larger than L2" if w["n"] * 80 > L2_BYTES else
               "L2 flushed between timed steps"}
    if w["kind"] == "tree":
        c.update(theta=w["theta"], leaf_capacity=w["leaf"], quadrupole=w["quadrupole"],
                 morton_bits=63)
    return c


# ---------------------------------------------------------------------------
# The B200 arm
# ---------------------------------------------------------------------------

# DRAM bytes (read + write) per launch of each dominant kernel, from one ncu
# capture each, scaled to the workload by the units one launch processes
# (the captures and commands are in profiles/):
#   walk: 31.34 MB for 500,000 targets (L2-resident case; lower bound at 2M);
#   direct FP32 / split at 262,144: 8.47 MB / 17.20 MB, reads of the packed
#   sources through L2, proportional to N;
#   batch: 258.9 MB for 1.742e10 pairs (sources re-read per target tile).
TRAFFIC_BYTES = {
    ("walk", "fp32"): lambda n: 31.34e6 * n / 500_000,
    ("direct", "fp32"): lambda n: 8.47e6 * n / 262_144,
    ("direct", "split"): lambda n: 17.20e6 * n / 262_144,
    ("batch", "split"): lambda pairs: 258.9e6 * pairs / 1.7416705824e10,
}


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            p = json.load(fh)
        return p.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def output_state(data):
    """The ten arrays of a checkpoint for the collision inputs (accelerations
    zero: the writers only move bytes)."""
    st = {k: np.ascontiguousarray(data[k]) for k in ("m", "x", "y", "z", "vx", "vy", "vz")}
    for k in ("ax", "ay", "az"):
        st[k] = np.zeros(len(st["m"]))
    return st


def cpu_baseline_output(w, data, directory):
    """The reference's own writers (sim::TrajectoryWriter, sim::write_checkpoint,
    oracle/_ref) on the same 2M state: the run time a frame costs the
    reference's run loop, which writes it synchronously."""
    import oracle

    if not oracle.Reference.available():
        return {"unavailable": "the reference library (oracle/_ref) is not built"}
    ref = oracle.Reference()
    st = output_state(data)
    frame = {k: st[k] for k in ("x", "y", "z", "vx", "vy", "vz")}
    path = os.path.join(directory, "reference.tj")
    frames = 3
    t0 = time.perf_counter()
    ref.write_trajectory(path, st["m"], w["dt"], [(k, k * w["dt"], frame)
                                                  for k in range(frames)], True)
    traj_s = time.perf_counter() - t0
    os.remove(path)
    path = os.path.join(directory, "reference.ck")
    t0 = time.perf_counter()
    ref.write_checkpoint(path, 1, st)
    ck_s = time.perf_counter() - t0
    size = os.path.getsize(path)
    os.remove(path)
    header = 8 + 4 + 4 + 8 + 8 * len(st["m"])
    per_frame = traj_s / frames  # the header (masses, a sixth of a frame) included
    return {"value": per_frame * 1e3, "unit": "ms/frame", "cores": 1, "kind": "reference",
            "sample": f"sim::TrajectoryWriter: header ({header / 1e6:.0f} MB) and {frames} frames "
                      "of positions and velocities of the 2M state; sim::write_checkpoint of it",
            "checkpoint_s": ck_s, "checkpoint_bytes": size}


def run_output(args, w):
    """Trajectory frames and checkpoints of the 2M collision as it steps."""
    import tempfile

    import torch

    import orrery_b200 as ob

    world, rank, local = dist_env()
    dist = init_dist(world, "nccl")
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    ob.load_library()
    data = make_inputs(w)
    n, dt, stride = w["n"], w["dt"], w["stride"]
    system = ob.DeviceSystem(n, w["eps"], kind=ob.SOLVER_TREE, precision="fp32",
                             opening_angle=w["theta"], leaf_capacity=w["leaf"],
                             quadrupole=w["quadrupole"])
    system.set_state(data["x"], data["y"], data["z"], data["vx"], data["vy"], data["vz"],
                     data["m"])
    system.step(dt, max(args.warmup, 3), w["integrator"])
    kernels_per_step = system.step_kernels(dt, w["integrator"])
    K = max(args.steps, 12 * stride)  # enough frames for the writers' steady state
    directory = tempfile.mkdtemp(prefix="orrery_output_")
    frame_bytes = 6 * 8 * n

    def steps_with_frames(every, path):
        """Wall seconds of K steps with a frame every `every` steps (none when
        0), up to the last step's completion, and the further seconds until
        every frame is in the file."""
        t = ob.Trajectory(path, dt, system=system, with_velocities=True) if every else None
        system.synchronize()
        t0 = time.perf_counter()
        for k in range(1, K + 1):
            system.step_async(dt, 1, w["integrator"])
            if every and k % every == 0:
                t.write_frame(k, k * dt)
        system.synchronize()
        stepped = time.perf_counter() - t0
        if t is not None:
            t.close()
        drained = time.perf_counter() - t0 - stepped
        if every:
            os.remove(path)
        return stepped, drained

    sampler = ClockSampler(local)
    barrier(dist)
    sampler.start()
    time.sleep(0.3)
    base, _ = steps_with_frames(0, None)
    strided, strided_drain = steps_with_frames(stride, os.path.join(directory, f"rank{rank}_s.tj"))
    every, every_drain = steps_with_frames(1, os.path.join(directory, f"rank{rank}_1.tj"))
    # The snapshot on the device: two device-to-device copies of 3n doubles,
    # timed on the system's stream.
    stream = torch.cuda.ExternalStream(system.stream(), device=device)
    t = ob.Trajectory(os.path.join(directory, f"rank{rank}_copy.tj"), dt, system=system,
                      with_velocities=True)
    reps = 4
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(reps):
        t.write_frame(k, k * dt)
    e1.record(stream)
    e1.synchronize()
    snapshot_ms = e0.elapsed_time(e1) / reps
    t.close()
    os.remove(os.path.join(directory, f"rank{rank}_copy.tj"))
    # Checkpoint write and restore.
    ck = os.path.join(directory, f"rank{rank}.ck")
    t0 = time.perf_counter()
    system.write_checkpoint(ck, K, "")
    write_s = time.perf_counter() - t0
    ck_bytes = os.path.getsize(ck)
    t0 = time.perf_counter()
    system.read_checkpoint(ck)
    read_s = time.perf_counter() - t0
    os.remove(ck)
    clocks = sampler.stop()
    barrier(dist)
    per_frame_ms = (strided - base) / (K // stride) * 1e3
    per_frame_every_ms = (every - base) / K * 1e3
    step_ms = base / K * 1e3
    peak, src = load_peaks()
    copy_gbs = 2 * frame_bytes / (snapshot_ms * 1e-3) / 1e9
    if rank == 0:
        line = {
            "metric": w["metric"], "value": max(per_frame_ms, 0.0), "unit": "ms/frame",
            "n_gpus": world, "steps": K, "warmup": max(args.warmup, 3),
            "ms_per_step": step_ms, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "n": n, "stride": stride,
                       "frame": "positions and velocities (ORRERYTJ v1)",
                       "frame_bytes": frame_bytes + 24, "checkpoint": "ORRERYCK v1",
                       "l2": "state 160 MB, larger than L2"},
            "stepping": {"ms_per_step_without_output": step_ms,
                         f"ms_per_step_frame_every_{stride}": strided / K * 1e3,
                         f"drain_after_last_step_s_every_{stride}": strided_drain,
                         "ms_per_step_frame_every_step": every / K * 1e3,
                         "drain_after_last_step_s_every_step": every_drain,
                         "run_time_per_frame_every_step_ms": per_frame_every_ms,
                         "frames_per_s_written_every_step": K / (every + every_drain)},
            "checkpoint": {"write_s": write_s, "read_s": read_s, "bytes": ck_bytes,
                           "write_gb_s": ck_bytes / write_s / 1e9,
                           "read_gb_s": ck_bytes / read_s / 1e9},
            "roofline": {"bound": "hbm", "kernel": "snapshot copy (device to device)",
                         "achieved": copy_gbs, "peak": peak, "unit": "GB/s",
                         "frac": copy_gbs / peak, "traffic": 2 * frame_bytes,
                         "ms_per_snapshot": snapshot_ms,
                         "peak_source": f"{src} (MEASURED_PEAKS.json hbm_gbs)"},
            "e2e": {"value": K / (every + every_drain), "unit": "frames/s",
                    "h2d_bytes_per_step": 0, "d2h_bytes_per_step": frame_bytes,
                    "path": "ob_trajectory_write_system_frame each step of the stepping 2M "
                            "collision, frames in the file when the clock stops"},
            "gpu_launches": 3 * K * kernels_per_step, "clocks": clocks,
        }
        base_line = cpu_baseline_output(w, data, directory)
        line["cpu_baseline"] = base_line
        print(json.dumps(line), flush=True)
    try:
        os.rmdir(directory)
    except OSError:
        pass
    barrier(dist)
    if dist is not None:
        dist.destroy_process_group()


def e2e_integrator_plugin(system, w, data, steps, torch):
    """The step as a B200 Integrator::step over host-resident particle data:
    every step uploads x y z v a m from pinned host memory, advances one step
    on the device and downloads x y z v a (ob_system_step_host)."""
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    host = {k: pin(v) for k, v in system.state().items()}
    host["m"] = pin(data["m"])
    system.step_host(host, w["dt"], 1, w["integrator"])
    t0 = time.perf_counter()
    for _ in range(steps):
        system.step_host(host, w["dt"], 1, w["integrator"])
    sec = (time.perf_counter() - t0) / steps
    n = w["n"]
    return sec, 10 * 8 * n, 9 * 8 * n


def e2e_drop_in(ob, w, data, steps, torch):
    """The drop-in path: the reference's host integrator arithmetic on FP64
    arrays in pinned host memory, with the B200 solver's host-buffer evaluate
    (H2D positions + masses, device pipeline, D2H accelerations) per step."""
    n = w["n"]
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    x, y, z, m = (pin(data[k]) for k in ("x", "y", "z", "m"))
    vx, vy, vz = (pin(data[k]) for k in ("vx", "vy", "vz"))
    ax, ay, az = (pin(np.zeros(n)) for _ in range(3))
    if w["kind"] == "direct":
        solver = ob.B200DirectSolver(w["eps"], w["precision"])
    else:
        solver = ob.B200TreeSolver(w["eps"], w["theta"], w["leaf"], w["quadrupole"],
                                   w["precision"])
    solver.evaluate((x, y, z), m, (ax, ay, az))
    weights = [w["dt"]]
    if w["integrator"] == "yoshida4":
        c = 1.2599210498948731647672106
        outer, inner = 1.0 / (2.0 - c), -c / (2.0 - c)
        weights = [outer * w["dt"], inner * w["dt"], outer * w["dt"]]

    tmp = np.empty(n)
    clock = {"host": 0.0, "evaluate": 0.0, "transfer_in": 0.0, "transfer_out": 0.0,
             "device": 0.0}

    def kick(half):
        # v += (dt/2) a in place, as the reference's kick (no temporaries).
        for v, a in ((vx, ax), (vy, ay), (vz, az)):
            np.multiply(a, half, out=tmp)
            v += tmp

    def step():
        for h in weights:
            half = h / 2.0
            t = time.perf_counter()
            kick(half)
            for p, v in ((x, vx), (y, vy), (z, vz)):
                np.multiply(v, h, out=tmp)
                p += tmp
            t1 = time.perf_counter()
            solver.evaluate((x, y, z), m, (ax, ay, az))
            t2 = time.perf_counter()
            kick(half)
            t3 = time.perf_counter()
            clock["host"] += (t1 - t) + (t3 - t2)
            clock["evaluate"] += t2 - t1
            tm = solver.timings()
            clock["transfer_in"] += tm["transfer_in_ms"] * 1e-3
            clock["transfer_out"] += tm["transfer_out_ms"] * 1e-3
            clock["device"] += (tm["ordering_ms"] + tm["construction_ms"] +
                                tm["traversal_ms"]) * 1e-3

    step()
    for k in clock:
        clock[k] = 0.0
    t0 = time.perf_counter()
    for _ in range(steps):
        step()
    sec = (time.perf_counter() - t0) / steps
    evals = len(weights)
    breakdown = {f"{k}_ms": v / steps * 1e3 for k, v in clock.items()}
    breakdown["note"] = ("per step: host = the integrator's NumPy kick/drift arithmetic; "
                         "evaluate = ob_solver_evaluate's wall time, of which transfer_in / "
                         "transfer_out are its host<->device copies and device its kernels "
                         "(CUDA events)")
    return sec, evals * 4 * 8 * n, evals * 3 * 8 * n, solver, breakdown


def run_batch(args, w):
    """The batched form: every cluster stepped by one replayed graph."""
    import torch

    import orrery_b200 as ob

    world, rank, local = dist_env()
    dist = init_dist(world, "nccl")
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    sizes, radii, systems = make_inputs(w)
    batch = ob.DeviceBatch(sizes, w["eps"] * radii)
    for k, d in enumerate(systems):
        batch.set_state(k, d["x"], d["y"], d["z"], d["vx"], d["vy"], d["vz"], d["m"])
    batch.refresh()
    shape, tuned_ms = batch.autotune()
    batch.step(w["dt"], max(args.warmup, 3), w["integrator"])
    pairs, _, items = batch.stats()
    evals = evaluations_per_step(w)
    stream = torch.cuda.ExternalStream(batch.stream(), device=device)
    K = args.steps
    sampler = ClockSampler(local)
    barrier(dist)
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    batch.step_async(w["dt"], K, w["integrator"])
    end.record(stream)
    end.synchronize()
    total_ms = start.elapsed_time(end)
    batch.synchronize()
    barrier(dist)
    clocks = sampler.stop()
    total_ms = reduce_max(dist, total_ms, device)
    value = pairs * evals * K * world / (total_ms * 1e-3) / 1e9
    if rank == 0:
        ffma, rsq = ob.probe_fp32()
        peak = min(ffma / 31.0, rsq) / 1e9
        achieved = pairs * evals / (tuned_ms * 1e-3 * evals) / 1e9
        # e2e through the public API with host buffers: each step uploads every
        # system's state from pinned memory and downloads it again.
        pinned = [{k: torch.from_numpy(np.ascontiguousarray(d[k])).pin_memory().numpy()
                   for k in ("x", "y", "z", "vx", "vy", "vz", "m")} for d in systems]
        e2e_steps = max(2, min(K, 5))
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            for k, d in enumerate(pinned):
                batch.set_state(k, d["x"], d["y"], d["z"], d["vx"], d["vy"], d["vz"], d["m"])
            batch.step(w["dt"], 1, w["integrator"])
            for k in range(len(pinned)):
                batch.state(k)
        sec = (time.perf_counter() - t0) / e2e_steps
        total_n = int(sizes.sum())
        line = {
            "metric": w["metric"], "value": value, "unit": w["unit"], "n_gpus": world,
            "steps": K, "warmup": max(args.warmup, 3), "ms_per_step": total_ms / K,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": dtype_of(w), "state_dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "systems": len(sizes),
                       "particles": total_n, "pairs_per_evaluation": pairs,
                       "precision": "split", "integrator": "yoshida4", "dt": w["dt"],
                       "softening": "0.01 x scale radius", "work_items": items,
                       "autotuned_shape": {"threads": shape[0], "targets_per_thread": shape[1],
                                           "chunk_tiles": shape[2], "groups": shape[3]},
                       "l2": "inputs larger than L2"},
            "roofline": {"bound": "fp32-fma-pipe", "achieved": achieved, "peak": peak,
                         "unit": "Gint/s", "frac": achieved / peak,
                         "traffic": TRAFFIC_BYTES[("batch", "split")](pairs),
                         "kernel_ms": tuned_ms,
                         "peak_source": "measured FFMA lane rate / 31 FP32 operations per "
                                        "interaction of the split arithmetic"},
            "e2e": {"value": pairs * evals / sec / 1e9, "unit": w["unit"],
                    "h2d_bytes_per_step": total_n * 7 * 8, "d2h_bytes_per_step": total_n * 9 * 8,
                    "path": "ob_batch_set_state for every system, one step, ob_batch_get_state"},
            # Per substep: kick-drift, pack, batched forces, (partial-sum
            # reduction when sources are chunked), kick.
            "gpu_launches": K * evals * (5 if shape[2] else 4),
            "clocks": clocks,
        }
        if world == 1:
            line["cpu_baseline"] = cpu_baseline_batch(w, sizes, radii, systems)
        print(json.dumps(line), flush=True)
    barrier(dist)
    del batch
    if dist is not None:
        dist.destroy_process_group()


def make_stream(window, rate=20.0, seed=20260814):
    """Arrival times and parameters of the serving workload's jobs: a Poisson
    stream at `rate` jobs/s over `window` seconds; 70% direct Plummer jobs (N
    log-uniform in 1k..64k, 200..2000 Yoshida-4 steps, eps 0.01, dt 1e-3) and
    30% Barnes-Hut collision jobs (N log-uniform in 100k..4M, 100..500 VV
    steps, theta 0.5, quadrupoles, eps 0.02, dt 5e-4)."""
    rng = np.random.default_rng(seed)
    jobs, t = [], 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= window:
            break
        if rng.uniform() < 0.7:
            n = int(np.exp(rng.uniform(np.log(1000), np.log(64000))))
            jobs.append(dict(t=t, kind="direct", n=n, steps=int(rng.integers(200, 2001)),
                             offset=int(rng.integers(0, 1 << 30))))
        else:
            n = int(np.exp(rng.uniform(np.log(100_000), np.log(4_000_000))))
            jobs.append(dict(t=t, kind="tree", n=n, steps=int(rng.integers(100, 501)),
                             offset=int(rng.integers(0, 1 << 30))))
    return jobs


def job_states(jobs):
    """Every job's initial state, cut from two templates: a 65,536-particle
    Plummer sphere and a 4,000,000-particle two-disc collision. A job of N
    particles takes N consecutive entries of a fixed random permutation of its
    template, from a per-job offset, with masses rescaled to total 1."""
    from orrery_b200 import initial_conditions as ic

    rng = np.random.default_rng(7)
    kinds = {j["kind"] for j in jobs}
    templates = {}
    if "direct" in kinds:
        templates["direct"] = ic.plummer_sphere(65536, seed=20260815)
    if "tree" in kinds:
        templates["tree"] = ic.galaxy_collision(4_000_000, softening=0.02, seed=20260816)
    perms = {"direct": rng.permutation(65536), "tree": rng.permutation(4_000_000)}
    out = []
    for job in jobs:
        src, perm = templates[job["kind"]], perms[job["kind"]]
        idx = perm[(job["offset"] + np.arange(job["n"])) % len(perm)]
        st = {k: np.ascontiguousarray(src[k][idx]) for k in ("x", "y", "z", "vx", "vy", "vz")}
        st["m"] = np.full(job["n"], 1.0 / job["n"])
        out.append(st)
    return out


JOB_PARAMS = {"direct": dict(dt=1e-3, softening=0.01, integrator="yoshida4"),
              "tree": dict(dt=5e-4, softening=0.02, integrator="vv", theta=0.5, leaf=32)}


def served_arm(ob, jobs, states, sample):
    """The serving loop fed in real time (each job submitted at its arrival
    offset) and then drained. Returns per-job (arrival, finish) in seconds from
    the start of the stream, the loop's latency statistics and the final states
    of the `sample` jobs."""
    import threading

    server = ob.Server(hbm_budget_bytes=150 << 30, direct_pairs_cap=1 << 34, max_tree_jobs=2)
    ids = [None] * len(jobs)
    origin = {}

    def feed():
        origin["t"] = time.perf_counter()
        for k, job in enumerate(jobs):
            delay = job["t"] - (time.perf_counter() - origin["t"])
            if delay > 0:
                time.sleep(delay)
            p = JOB_PARAMS[job["kind"]]
            if job["kind"] == "direct":
                ids[k] = server.submit(states[k], steps=job["steps"], dt=p["dt"],
                                       softening=p["softening"])
            else:
                ids[k] = server.submit(states[k], steps=job["steps"], dt=p["dt"],
                                       softening=p["softening"], kind="tree", integrator="vv",
                                       opening_angle=p["theta"], leaf_capacity=p["leaf"],
                                       quadrupole=True)

    t_query = time.perf_counter()
    server_clock0 = server.stats()["elapsed_s"]
    feeder = threading.Thread(target=feed)
    feeder.start()
    feeder.join()
    server.drain(timeout=3600)
    # Server clock -> stream clock.
    shift = server_clock0 + (origin["t"] - t_query)
    finishes, finals = [], {}
    for k, job in enumerate(jobs):
        report, final = server.wait(ids[k], timeout=60, outputs=k in sample)
        assert report["status"] == ob.JOB_DONE, report
        finishes.append(report["finished_s"] - shift)
        if k in sample:
            finals[k] = final
    stats = server.stats()
    server.close()
    return finishes, stats, finals


def plain_arm(ob, torch, jobs, states, precision, sample, horizon):
    """The plain drop-in on the same stream, one job at a time in arrival
    order, as the reference's Simulation drives a ForceSolver: host integrator
    arithmetic on FP64 arrays in pinned memory and ob_solver_evaluate (host
    buffers in, accelerations out) per force evaluation. Stops early once the
    stream clock passes `horizon` seconds when one is given (the line then
    reports the arm as undrained); by default every job runs."""
    c = 1.2599210498948731647672106
    weights = {"yoshida4": [1.0 / (2.0 - c), -c / (2.0 - c), 1.0 / (2.0 - c)], "vv": [1.0]}
    solvers = {"direct": ob.B200DirectSolver(0.01, precision),
               "tree": ob.B200TreeSolver(0.02, 0.5, 32, True)}
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    finishes, step_times, finals = [], [], {}
    start = time.perf_counter()
    for k, job in enumerate(jobs):
        now = time.perf_counter() - start
        if horizon and now > horizon:
            break
        if job["t"] > now:
            time.sleep(job["t"] - now)
        p, st = JOB_PARAMS[job["kind"]], states[k]
        solver = solvers[job["kind"]]
        x, y, z, m = (pin(st[q]) for q in ("x", "y", "z", "m"))
        vx, vy, vz = (pin(st[q]) for q in ("vx", "vy", "vz"))
        ax, ay, az = (pin(np.zeros(job["n"])) for _ in range(3))
        tmp = np.empty(job["n"])
        solver.evaluate((x, y, z), m, (ax, ay, az))
        for _ in range(job["steps"]):
            t0 = time.perf_counter()
            for wgt in weights[p["integrator"]]:
                h = wgt * p["dt"]
                half = h / 2.0
                # In place, as the reference's kick and drift (no temporaries).
                for v, a in ((vx, ax), (vy, ay), (vz, az)):
                    np.multiply(a, half, out=tmp)
                    v += tmp
                for q, v in ((x, vx), (y, vy), (z, vz)):
                    np.multiply(v, h, out=tmp)
                    q += tmp
                solver.evaluate((x, y, z), m, (ax, ay, az))
                for v, a in ((vx, ax), (vy, ay), (vz, az)):
                    np.multiply(a, half, out=tmp)
                    v += tmp
            step_times.append(time.perf_counter() - t0)
        finishes.append(time.perf_counter() - start)
        if k in sample:
            finals[k] = {"x": x.copy(), "y": y.copy(), "z": z.copy(), "ax": ax.copy(),
                         "ay": ay.copy(), "az": az.copy()}
    return finishes, step_times, finals


def force_errors(ob, jobs, states, finals):
    """Per-particle relative force error of the returned accelerations against
    the FP64 direct solver (bit-identical to the reference's) at the returned
    positions: median and max over the sampled direct jobs' particles."""
    errs = []
    for k, fin in finals.items():
        exact = ob.B200DirectSolver(JOB_PARAMS["direct"]["softening"], "fp64")
        n = jobs[k]["n"]
        ex, ey, ez = (np.zeros(n) for _ in range(3))
        exact.evaluate((fin["x"], fin["y"], fin["z"]), states[k]["m"], (ex, ey, ez))
        num = np.sqrt((fin["ax"] - ex) ** 2 + (fin["ay"] - ey) ** 2 + (fin["az"] - ez) ** 2)
        errs.append(num / np.sqrt(ex ** 2 + ey ** 2 + ez ** 2))
    e = np.concatenate(errs) if errs else np.zeros(1)
    return {"median": float(np.median(e)), "max": float(np.max(e)), "jobs": len(finals),
            "particles": int(e.size)}


def latency_summary(jobs, finishes):
    done = len(finishes)
    lat = [finishes[k] - jobs[k]["t"] for k in range(done)]
    makespan = max(finishes) if finishes else float("inf")
    pct = lambda v, q: float(np.percentile(v, q)) if v else None  # noqa: E731
    return {"completed": done, "drained": done == len(jobs), "makespan_s": makespan,
            "jobs_per_s": done / makespan,
            "job_latency_p50_s": pct(lat, 50), "job_latency_p99_s": pct(lat, 99)}


def run_serving(args, w):
    """The serving form against the plain drop-in on the same job stream."""
    import torch

    import orrery_b200 as ob

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    ob.load_library()
    jobs = make_stream(args.window)
    states = job_states(jobs)
    direct_ids = [k for k, j in enumerate(jobs) if j["kind"] == "direct"]
    sample = set(sorted(direct_ids, key=lambda k: jobs[k]["n"])[:3])
    sampler = ClockSampler(local)
    sampler.start()
    fin_s, stats, finals_s = served_arm(ob, jobs, states, sample)
    served = latency_summary(jobs, fin_s)
    served.update(step_latency_p50_ms=stats["step_latency_p50_ms"],
                  step_latency_p99_ms=stats["step_latency_p99_ms"], hbm_peak=stats["hbm_peak"],
                  force_error=force_errors(ob, jobs, states, finals_s),
                  direct_arithmetic="split hi/lo FP32, Kahan, FP64 tile sums")
    plains = {}
    for precision in args.plain_precision.split(","):
        horizon = args.plain_horizon_factor * served["makespan_s"]
        fin_p, steps_p, finals_p = plain_arm(ob, torch, jobs, states, precision, sample, horizon)
        p = latency_summary(jobs, fin_p)
        pct = lambda v, q: float(np.percentile(v, q)) * 1e3 if v else None  # noqa: E731
        p.update(step_latency_p50_ms=pct(steps_p, 50), step_latency_p99_ms=pct(steps_p, 99),
                 force_error=force_errors(ob, jobs, states, finals_p),
                 direct_arithmetic=precision)
        if p["completed"] < len(jobs):
            p["note"] = (f"stopped after {p['completed']} of {len(jobs)} jobs once the stream "
                         f"clock passed {horizon:.0f} s; jobs/s is completed / makespan")
        plains[precision] = p
    clocks = sampler.stop()
    if rank == 0:
        kinds = [j["kind"] for j in jobs]
        first = plains[args.plain_precision.split(",")[0]]
        line = {
            "metric": w["metric"], "value": served["jobs_per_s"], "unit": "jobs/s",
            "n_gpus": world, "steps": len(jobs), "warmup": 0,
            "ms_per_step": served["step_latency_p50_ms"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": dtype_of(w), "state_dtype": "f64",
            "data": "synthetic",
            "config": {"workload": args.workload, "arrival_window_s": args.window,
                       "arrival_rate_per_s": 20.0, "jobs": len(jobs),
                       "direct_jobs": kinds.count("direct"), "tree_jobs": kinds.count("tree"),
                       "direct_particles": sum(j["n"] for j in jobs if j["kind"] == "direct"),
                       "tree_particles": sum(j["n"] for j in jobs if j["kind"] == "tree"),
                       "hbm_budget_gb": 150, "max_tree_jobs": 2, "direct_pairs_cap": 1 << 34,
                       "jobs_per_s": "jobs / (last completion - stream start); an arm "
                                     "that did not drain the stream says so (drained)"},
            "served": served,
            "plain": plains,
            "served_over_plain": {k: served["jobs_per_s"] / v["jobs_per_s"]
                                  for k, v in plains.items()},
            "e2e": {"value": served["jobs_per_s"], "unit": "jobs/s",
                    "h2d_bytes_per_step": 56 * sum(j["n"] for j in jobs) // len(jobs),
                    "d2h_bytes_per_step": 72 * sum(j["n"] for j in jobs) // len(jobs),
                    "step": "one job (its state in, its final state out)",
                    "path": "ob_server_submit (host state in) .. ob_server_wait (host state out)"},
            "vs_plain_" + args.plain_precision.split(",")[0]:
                served["jobs_per_s"] / first["jobs_per_s"],
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)


def run_b200(args, w):
    import torch

    import orrery_b200 as ob

    world, rank, local = dist_env()
    dist = init_dist(world, "nccl")
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    ob.load_library()

    data = make_inputs(w)
    n = w["n"]
    kind = ob.SOLVER_DIRECT if w["kind"] == "direct" else ob.SOLVER_TREE
    system = ob.DeviceSystem(n, w["eps"], kind=kind, precision=w["precision"],
                             opening_angle=w.get("theta", 0.5), leaf_capacity=w.get("leaf", 32),
                             quadrupole=w.get("quadrupole", False))
    system.set_state(data["x"], data["y"], data["z"], data["vx"], data["vy"], data["vz"],
                     data["m"])
    # Direct workloads state their energy drift from t = 0 (FP64 energies on
    # the device, outside the timed region); at 2M the O(N^2) FP64 potential
    # takes about a minute, so tree workloads give it only with --energy.
    track_energy = w["kind"] == "direct" or args.energy
    energy0 = sum(system.energy()) if track_energy else None
    tuned = None
    if w["kind"] == "direct" and w["precision"] != "fp64":
        tuned = system.autotune()
    system.step(w["dt"], max(args.warmup, 3), w["integrator"])
    kernels_per_step = system.step_kernels(w["dt"], w["integrator"])
    stream = torch.cuda.ExternalStream(system.stream(), device=device)
    flush = None
    if n * 80 <= L2_BYTES:
        flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=device)

    def run_steps(count):
        """`count` steps on the system's stream; device milliseconds summed
        over the steps (L2 flushed before each when the state fits in L2)."""
        if flush is None:
            start = torch.cuda.Event(enable_timing=True)
            end = torch.cuda.Event(enable_timing=True)
            start.record(stream)
            system.step_async(w["dt"], count, w["integrator"])
            end.record(stream)
            end.synchronize()
            return start.elapsed_time(end)
        pairs = []
        for _ in range(count):
            with torch.cuda.stream(stream):
                flush.add_(1.0)
            s = torch.cuda.Event(enable_timing=True)
            e = torch.cuda.Event(enable_timing=True)
            s.record(stream)
            system.step_async(w["dt"], 1, w["integrator"])
            e.record(stream)
            pairs.append((s, e))
        pairs[-1][1].synchronize()
        return sum(s.elapsed_time(e) for s, e in pairs)

    K = args.steps
    counts_start = system.interaction_count()
    sampler = ClockSampler(local)
    barrier(dist)
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)
    total_ms = run_steps(K)
    system.synchronize()
    torch.cuda.synchronize()
    barrier(dist)
    clocks = sampler.stop()
    total_ms = reduce_max(dist, total_ms, device)
    counts_end = system.interaction_count()
    # Phase times (and the force kernel's time for the roofline) from K more
    # steps of the step graph with event nodes between the phases, outside
    # the timed region.
    system.profile(K)
    run_steps(K)
    system.synchronize()
    phases, evals = system.phase_times()
    interactions = (counts_end.particle_particle + counts_end.particle_cell -
                    counts_start.particle_particle - counts_start.particle_cell)
    pair_count = counts_end.particle_particle - counts_start.particle_particle
    cell_count = counts_end.particle_cell - counts_start.particle_cell

    ms_per_step = total_ms / K
    # Stated error of the result, outside the timed region: the final state's
    # accelerations against FP64 solvers on the same positions.
    taken = max(args.warmup, 3) + 2 * K  # warm-up, timed and profiled steps
    extra = max(0, args.accuracy_steps - taken)
    if extra:
        system.step(w["dt"], extra, w["integrator"])
    st = system.state()
    got = np.stack([st["ax"], st["ay"], st["az"]], axis=1)
    accuracy = {"steps": taken + extra}
    if energy0 is not None:
        energy1 = sum(system.energy())
        accuracy["relative_energy_drift"] = (energy1 - energy0) / abs(energy0)
    if w["kind"] == "direct":
        exact = ob.B200DirectSolver(w["eps"], "fp64").evaluate((st["x"], st["y"], st["z"]),
                                                               data["m"])
        accuracy["force_error_vs_fp64"] = error_summary(
            relative_errors(got, exact),
            "the final state's accelerations against the FP64 direct solver (bit-identical "
            "to the reference's DirectSolver)")
    else:
        if w["precision"] != "fp64":
            tree64 = ob.B200TreeSolver(w["eps"], w["theta"], w["leaf"], w["quadrupole"],
                                       precision="fp64")
            exact = tree64.evaluate((st["x"], st["y"], st["z"]), data["m"])
            del tree64
            accuracy["force_error_vs_fp64_tree"] = error_summary(
                relative_errors(got, exact),
                f"every particle against the FP64 tree at the same theta {w['theta']} (the "
                "reference's BarnesHutSolver, bit-identical), same positions")
        rng = np.random.default_rng(20261203)
        targets = np.sort(rng.choice(n, size=min(n, 4096), replace=False))
        direct = direct_fp64_sampled(torch, device, st, data["m"], w["eps"], targets)
        accuracy["force_error_vs_fp64_direct"] = error_summary(
            relative_errors(got[targets], direct),
            f"{len(targets)} sampled particles against the FP64 direct sum over all "
            f"{n} sources (the tree's own theta {w['theta']} approximation included)")
    if w["unit"] == "ms/step":
        value = ms_per_step / world  # whole-job time per 2M step across replicas
    else:
        value = step_units(w) * K * world / (total_ms * 1e-3) / 1e9

    # Roofline of the dominant kernel (the force kernel: walk or direct sum).
    kernel_ms = phases["traversal_ms"]
    if w["kind"] == "direct":
        ffma, rsq = ob.probe_fp32()
        # FP32 interaction peak: the FMA pipe carries 12 lane operations per
        # interaction in FP32 (3 sub, 3 fma for r^2, 3 mul, 3 fma) and 31 in
        # the split arithmetic (9 hi/lo differences, 3 r^2, 4 Newton, 3 m y^3,
        # 12 Kahan); the SFU one rsqrt either way.
        ops = 31.0 if w["precision"] == "split" else 12.0
        peak_gint = min(ffma / ops, rsq) / 1e9
        achieved = n * (n - 1) / (kernel_ms * 1e-3) / 1e9
        roofline = {"bound": "fp32-fma-pipe", "achieved": achieved, "peak": peak_gint,
                    "unit": "Gint/s", "frac": achieved / peak_gint,
                    "traffic": TRAFFIC_BYTES.get(("direct", w["precision"]), lambda n: None)(n),
                    "peak_source": f"measured FFMA lane rate / {ops:.0f} FP32 operations per "
                                   f"interaction (FFMA {ffma / 1e12:.2f} T lane-op/s, SFU "
                                   f"rsqrt {rsq / 1e12:.2f} T/s) on this GPU",
                    "fp32_interaction_peak_gint_s": min(ffma / 12.0, rsq) / 1e9,
                    "kernel_ms": kernel_ms}
    else:
        # The walk keeps its nodes and leaf sources in L2 and is bound by the
        # FP32 pipe and instruction issue: its roofline counts the FP32
        # operations of the reference's arithmetic, 12 per particle-particle
        # term and 16 (monopole) or 39 (with quadrupole) per particle-cell
        # term, against the measured FFMA lane rate. Its HBM figures are
        # reported beside it.
        hbm, src = load_peaks()
        evals_done = max(1, K * evaluations_per_step(w))
        if w["precision"] == "fp64":
            # The parity walk's FP64 operations by the reference's arithmetic
            # (square root and divide counted as one each): 20 per pair term,
            # 20 per monopole and 41 more per quadrupole cell term, against
            # the measured DFMA lane rate.
            peak = ob.probe_fp64()
            ops = (20 * pair_count + (61 if w["quadrupole"] else 20) * cell_count) / evals_done
            bound, unit, src_peak = ("fp64-pipe", "T FP64 op/s",
                                     "measured DFMA lane rate on this GPU (ob_probe_fp64)")
        else:
            peak, _ = ob.probe_fp32()
            ops = (12 * pair_count + (39 if w["quadrupole"] else 16) * cell_count) / evals_done
            bound, unit, src_peak = ("fp32-fma-pipe", "T FP32 op/s",
                                     "measured FFMA lane rate on this GPU (ob_probe_fp32)")
        achieved_t = ops / (kernel_ms * 1e-3) / 1e12
        roofline = {"bound": bound, "achieved": achieved_t, "peak": peak / 1e12,
                    "unit": unit, "frac": achieved_t / (peak / 1e12),
                    "peak_source": src_peak,
                    "algorithmic_ops": ops, "kernel_ms": kernel_ms,
                    "traffic": TRAFFIC_BYTES[("walk", "fp32")](n) if w["precision"] == "fp32"
                    else None,
                    "hbm": {"peak": hbm, "unit": "GB/s",
                            "peak_source": f"{src} (MEASURED_PEAKS.json hbm_gbs, a copy "
                                           "kernel)"}}
    line = None
    if rank == 0:
        e2e_steps = max(2, min(K, 10 if w["kind"] == "tree" else 50))
        sec, h2d, d2h = e2e_integrator_plugin(system, w, data, e2e_steps, torch)
        sec_solver, h2d_solver, d2h_solver, solver, split = e2e_drop_in(ob, w, data, e2e_steps,
                                                                         torch)
        if w["kind"] == "tree":
            nodes, leaves, depth = solver.tree_stats()
            # Algorithmic bytes of one walk launch: each target's FP64 position
            # (24 B) and permutation entry (4 B) read and FP64 acceleration
            # (24 B) written, every leaf-relative source (16 B) and every node
            # (64 B) and FP32 quadrupole (32 B) read once.
            quad_bytes = 32 if w["quadrupole"] else 0
            algorithmic = n * (24 + 4 + 24 + 16) + nodes * (64 + quad_bytes)
            achieved = algorithmic / (kernel_ms * 1e-3) / 1e9
            per_eval = interactions / max(1, K * evaluations_per_step(w))
            roofline["hbm"].update({"achieved": achieved,
                                    "frac": achieved / roofline["hbm"]["peak"],
                                    "algorithmic_bytes": algorithmic})
            roofline.update({"nodes": nodes, "leaves": leaves, "depth": depth,
                             "interactions_per_walk": per_eval,
                             "pairs_per_walk": pair_count / max(1, K * evaluations_per_step(w)),
                             "cells_per_walk": cell_count / max(1, K * evaluations_per_step(w)),
                             "interaction_rate_gint_s": per_eval / (kernel_ms * 1e-3) / 1e9})
        if w["unit"] == "ms/step":
            e2e_value, e2e_solver = sec * 1e3, sec_solver * 1e3
        else:
            e2e_value = step_units(w) / sec / 1e9
            e2e_solver = step_units(w) / sec_solver / 1e9
        base = cpu_baseline(w, data) if world == 1 else None
        line = {
            "metric": w["metric"], "value": value, "unit": w["unit"], "n_gpus": world,
            "steps": K, "warmup": max(args.warmup, 3), "ms_per_step": ms_per_step,
            "higher_is_better": w["higher"], "scaling": "weak", "vs_baseline": None,
            "dtype": dtype_of(w), "state_dtype": "f64", "data": "synthetic",
            "config": config_of(args, w),
            "phases_ms": {k: phases[k] for k in ("ordering_ms", "construction_ms",
                                                  "traversal_ms")},
            "profiled_evaluations": evals,
            "autotuned_shape": None if tuned is None else
            {"threads": tuned[0][0], "targets_per_thread": tuned[0][1], "split": tuned[0][2],
             "groups": tuned[0][3]},
            "roofline": roofline,
            "accuracy": accuracy,
            "e2e": {"value": e2e_value, "unit": w["unit"], "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "path": "ob_system_step_host: Integrator::step over pinned host particle "
                            "data (upload x v a m, one device step, download x v a)"},
            "e2e_solver_plugin": {"value": e2e_solver, "unit": w["unit"],
                                  "h2d_bytes_per_step": h2d_solver,
                                  "d2h_bytes_per_step": d2h_solver,
                                  "path": "the reference's host integrator arithmetic (NumPy) "
                                          "around ob_solver_evaluate (ForceSolver::evaluate) "
                                          "on pinned host buffers",
                                  "breakdown": split},
            "gpu_launches": kernels_per_step * K,
            "clocks": clocks,
        }
        if base is not None:
            line["cpu_baseline"] = base
        print(json.dumps(line), flush=True)
    barrier(dist)
    del system
    if dist is not None:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default=DEFAULT_WORKLOAD)
    ap.add_argument("--window", type=float, default=3.0,
                    help="serving: seconds of Poisson arrivals (every arm drains them all)")
    ap.add_argument("--accuracy-steps", type=int, default=0,
                    help="total steps after which the energy drift and force error are "
                         "stated (default: the warm-up, timed and profiled steps)")
    ap.add_argument("--energy", action="store_true",
                    help="tree workloads: also state the FP64 energy drift (the O(N^2) "
                         "potential at 2M takes about a minute of device time)")
    ap.add_argument("--plain-precision", default="fp32",
                    help="serving: comma-separated direct precisions of the plain arms")
    ap.add_argument("--plain-horizon-factor", type=float, default=0.0,
                    help="serving: a plain arm stops once its clock passes this multiple "
                         "of the served makespan and is reported undrained (0: every arm "
                         "drains the whole stream)")
    args = ap.parse_args()
    w = WORKLOADS[args.workload]
    if args.impl == "reference":
        run_reference(args, w)
    elif w["kind"] == "batch":
        run_batch(args, w)
    elif w["kind"] == "serving":
        run_serving(args, w)
    elif w["kind"] == "output":
        run_output(args, w)
    else:
        run_b200(args, w)


if __name__ == "__main__":
    main()
