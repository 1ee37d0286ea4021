#!/usr/bin/env python
"""Time steps/s of the SCoPI time step on B200 at 1M spheres.

Workload (N=1): 1,000,000 spheres on a jittered 100^3 lattice in the unit box with six
plane walls, inward desired velocity 0.1 (vap_fixed), NoFriction, dmax 0.0018,
dt 1e-3, APGD tol 1e-6 / max_ite 40000 (scopi_b200.configs.spheres_1m).  A step is one
full ScopiSolver time step: obstacle motion, contact detection, assembly, APGD,
velocity and position/quaternion update.  The headline arm is the mixed form (FP32
APGD iterations + FP64 outer correction to violation <= 1e-6); the plain FP64 form is
timed on the same steps from the same state and reported beside it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N>1 runs under torchrun, one independent replica per GPU (every APGD iteration needs
global reductions over the scene, so the solve has no data-path exchange to shard), timed
on the device and reduced as the max over ranks.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "time steps/s at 1M spheres (mixed FP32-APGD + FP64 correction, violation <= 1e-6)"
UNIT = "steps/s"
WORKLOAD = "spheres_1m"


def env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


def roofline_bytes_per_iter(C, N, s, dim=3, torque_free=False):
    """Algorithmic bytes of one APGD iteration (accepted step, no backtracks).

    Rows of B: 3 passes over B (values + 2 int32 indices per contact), 6 contact vector
    streams, 4 particle vector streams.  Full rows carry 9 values per contact in 3D
    (n, R_i^T(r_i x n), R_j^T(r_j x n)) and 6N particle slots (4 values and 3N slots in
    2D): this is the figure `roofline.achieved` uses.  For normal-only problems on
    sphere/plane/segment contacts the rotational values are identically zero, so the
    torque-free kernel streams a row as the normal alone (3 values in 3D, 2 in 2D) with
    N*dim translational particle slots (`torque_free=True`, reported beside it).
    """
    if torque_free:
        return 3 * C * (dim * s + 8) + 6 * C * s + 4 * (dim * N) * s
    if dim == 3:
        return 3 * C * (9 * s + 8) + 6 * C * s + 4 * (6 * N) * s
    return 3 * C * (4 * s + 8) + 6 * C * s + 4 * (3 * N) * s


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons, power = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
                power.append(float(parts[3]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "power_w_max": max(power) if power else None}


# ----------------------------------------------------------------------------- ranks
class Ranks:
    def __init__(self, n_gpus):
        self.world = env_int("WORLD_SIZE", 1)
        self.rank = env_int("RANK", 0)
        self.local = env_int("LOCAL_RANK", 0)
        self.n_gpus = n_gpus
        self.pg = False
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            backend = "nccl" if torch.cuda.is_available() else "gloo"
            if torch.cuda.is_available():
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
            self.pg = True

    def barrier(self):
        if self.pg:
            import torch.distributed as dist
            dist.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        import torch.distributed as dist
        dev = "cuda" if torch.cuda.is_available() else "cpu"
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            import torch.distributed as dist
            dist.destroy_process_group()


# ----------------------------------------------------------------------------- GPU arm
def solver_kwargs():
    from scopi_b200 import configs
    st = configs.SETTINGS[WORKLOAD]
    return dict(dmax=st["dmax"], tolerance=st["tolerance"], max_ite=st["max_ite"], vap=st["vap"]), st["dt"]


def time_path(pa, precision, steps, warmup, ranks, sampler=None, solver=None, **extra):
    import torch

    from scopi_b200 import ScopiSolver
    kw, dt = solver if solver else solver_kwargs()
    s = ScopiSolver(pa, precision=precision, mixed_violation_tol=1e-6, device=ranks.local, **kw, **extra)
    s.step(dt, warmup)
    stream = torch.cuda.ExternalStream(s.stream_handle(), device=ranks.local)
    torch.cuda.synchronize()
    ranks.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    l0 = s.kernel_launches()
    if sampler:
        sampler.start()
    per = []
    e0.record(stream)
    for _ in range(steps):
        s.step(dt, 1)
        per.append(s.stats())
    e1.record(stream)
    e1.synchronize()
    clocks = sampler.stop() if sampler else None
    torch.cuda.synchronize()
    ranks.barrier()
    ms = e0.elapsed_time(e1)
    launches = s.kernel_launches() - l0
    s.close()
    return {"ms": ms, "per_step": per, "launches": launches, "clocks": clocks}


def time_e2e(pa, precision, steps, warmup, ranks, full_upload=False):
    """Same steps through the C ABI with host buffers: upload, step, download every step.

    The upload is the state a step updates (pos, q, v, omega: scopi_gpu_set_state), or with
    full_upload the whole container (scopi_gpu_set_particles: shapes, masses, forces and
    desired velocities too, and the container's checks)."""
    import numpy as np
    import torch

    from scopi_b200 import ScopiSolver
    kw, dt = solver_kwargs()

    def pinned(a):
        t = torch.empty(a.shape, dtype=torch.float64 if a.dtype == np.float64 else torch.int32, pin_memory=True)
        out = t.numpy()
        out[...] = a
        return out, t

    keep = []
    host = pa.copy()
    for k in ("shape", "worm", "pos", "q", "v", "omega", "vd", "omega_d", "f", "m", "j", "radius", "length"):
        arr, t = pinned(getattr(host, k))
        keep.append(t)
        setattr(host, k, arr)
    s = ScopiSolver(host, precision=precision, mixed_violation_tol=1e-6, device=ranks.local, **kw)
    s.step(dt, warmup)
    s.download(host)
    stream = torch.cuda.ExternalStream(s.stream_handle(), device=ranks.local)
    torch.cuda.synchronize()
    ranks.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    upload = s.upload if full_upload else s.upload_state
    for _ in range(steps):
        upload(host)
        s.step(dt, 1)
        s.download(host)
    e1.record(stream)
    e1.synchronize()
    ranks.barrier()
    ms = e0.elapsed_time(e1)
    n = host.n
    if full_upload:
        h2d = 4 * n + 4 * n + 8 * n * (3 + 4 + 3 + 3 + 3 + 3 + 3 + 1 + 3 + 1 + 1)  # shape, worm, 11 FP64 fields
    else:
        h2d = 8 * n * (3 + 4 + 3 + 3)  # pos, q, v, omega
    d2h = 8 * n * (3 + 4 + 3 + 3)
    s.close()
    return ms, h2d, d2h


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# DRAM bytes (read + write) per FP32 APGD iteration per contact of k_apgd_sph on the
# 1M-sphere workload, from one ncu capture of a whole launch at time step 2 (19 iterations,
# the curvature pre-pass and one backtrack included): 5.930 GB / (19 x 3,000,279).  The
# line's roofline.traffic scales it by the run's contacts and iterations per launch.
TRAFFIC_FP32_PER_CONTACT_ITERATION = 104.0
TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one k_apgd_sph<float,3,0> launch at "
                  "time step 2 (104 B per FP32 contact-iteration), scaled by this run's contacts and FP32 "
                  "iterations per launch")


# ----------------------------------------------------------------------------- CPU legs
def cpu_sample(pa, iterations_per_step, threads, solver=None, caps=(1, 3)):
    """Oracle (CPU restatement of the reference path) on the full workload.

    Two time steps from the same state with the APGD loop capped at caps[0] and caps[1]
    iterations: t_per_iteration = the solve's time difference / the iteration difference;
    everything else (detection, problem build, the solve's set-up, velocity recovery,
    update) is t_fixed; steps/s is rebuilt as 1 / (t_fixed + t_per_iteration *
    iterations_per_step)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import py_oracle as orc
    kw, dt = solver if solver else solver_kwargs()
    out = {}
    t0 = time.perf_counter()
    for cap in caps:
        o = orc.OracleSolver(pa, **dict(kw, max_ite=cap, num_threads=threads))
        o.run(dt, 1)
        out[cap] = o.stats()
        del o
    wall = time.perf_counter() - t0
    if len(caps) == 1:
        # one capped step: the solve's time per iteration includes its set-up (an upper bound)
        c = caps[0]
        out[1] = out[3] = out[c]
        t_iter = max(1e-9, out[c]["seconds_solve"] / max(1, out[c]["iterations"]))
        t_fixed = out[c]["seconds_contacts"] + out[c]["seconds_other"]
        est = 1.0 / (t_fixed + t_iter * iterations_per_step)
        return {"value": est, "t_per_iteration_s": t_iter, "t_outside_apgd_s": t_fixed, "wall_s": wall,
                "contacts": out[c]["contacts"], "iterations_timed": out[c]["iterations"]}
    lo, hi = caps
    d_it = max(1, out[hi]["iterations"] - out[lo]["iterations"])
    t_iter = max(1e-9, (out[hi]["seconds_solve"] - out[lo]["seconds_solve"]) / d_it)
    t_fixed = (out[lo]["seconds_contacts"] + out[lo]["seconds_other"] +
               max(0.0, out[lo]["seconds_solve"] - t_iter * out[lo]["iterations"]))
    est = 1.0 / (t_fixed + t_iter * iterations_per_step)
    return {"value": est, "t_per_iteration_s": t_iter, "t_outside_apgd_s": t_fixed, "wall_s": wall,
            "contacts": out[hi]["contacts"], "iterations_timed": out[lo]["iterations"] + out[hi]["iterations"]}


def reference_arm(args, ranks):
    """--impl reference: the CPU restatement of the reference path on the host cores."""
    if ranks.rank != 0:
        return 0
    from scopi_b200 import configs
    threads = os.cpu_count() or 1
    pa = configs.spheres_1m()
    iters, iters_src = reference_iterations(args.warmup + 1, args.warmup + args.steps)
    samples = []
    for k in range(args.warmup + args.steps):
        r = cpu_sample(pa, iters, threads)
        if k >= args.warmup:
            samples.append(r)
    value = statistics.median(r["value"] for r in samples)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / value, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD + ": 1,000,000 spheres, NoFriction, vap_fixed, dmax 0.0018, dt 1e-3, tol 1e-6"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "extrapolated": True,
                         "cpu_model": cpu_model(),
                         "sample": (f"oracle (C++ restatement of the reference path, OpenMP on the loops the reference "
                                    f"parallelises, serial APGD) on the full 1M-sphere step, APGD capped at 1 and 3 "
                                    f"iterations; steps/s = 1/(t_outside_apgd + t_per_iteration * {iters:.1f}), "
                                    f"{iters:.1f} = mean FP64 APGD iterations per step of the timed steps ({iters_src})")},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "samples": samples,
    }
    print(json.dumps(line), flush=True)
    return 0


# FP64 APGD iterations of every step of the 100-step spheres_1m run, measured on B200 with
# the FP64 path (the reference's iterate rule, cold start and tolerance); the file holds
# the command that measured them.  The CPU legs take the mean over the steps they stand for.
ITERATIONS_FILE = os.path.join(ROOT, "scopi_b200", "data", "spheres_1m_fp64_iterations.json")
REF_APGD_ITERATIONS_DEFAULT = 497


def reference_iterations(first, last):
    """Mean FP64 iterations per step over steps first..last (1-based) and where it came from."""
    try:
        with open(ITERATIONS_FILE) as fh:
            d = json.load(fh)
        its = d["iterations"][first - 1:last]
        if its:
            return statistics.mean(its), f"measured per step on B200 ({d['command']}), steps {first}..{last}"
    except (OSError, KeyError, ValueError):
        pass
    return REF_APGD_ITERATIONS_DEFAULT, "constant (first two steps measured on B200)"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--side", type=int, default=100)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-viscous", action="store_true")
    ap.add_argument("--no-errors", action="store_true")
    ap.add_argument("--workload", default="spheres_1m",
                    choices=["spheres_1m", "piles", "se_pile", "disks_2d", "box_3d"],
                    help="spheres_1m: the headline line; piles: 256 pile scenes stepped as one batch; "
                         "se_pile: 50k superellipsoids with friction; disks_2d: 1024 disks in FP64; "
                         "box_3d: 100k spheres in a box under gravity")
    ap.add_argument("--cpu-budget", type=float, default=120.0,
                    help="disks_2d / box_3d: seconds of oracle steps in the CPU baseline (all threads)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 0)
    if args.steps is None:
        # the workloads' own run lengths: 100 steps (1M spheres), 1000 steps (piles); the
        # superellipsoid pile (300 steps, ~1 s each) is timed on 20
        args.steps = {"spheres_1m": 100, "piles": 1000, "se_pile": 20 + args.warmup, "disks_2d": 200,
                      "box_3d": 500}[args.workload] - args.warmup
    ranks = Ranks(args.gpus)
    try:
        if args.impl == "reference":
            return reference_arm(args, ranks)
        if args.workload == "piles":
            return piles(args, ranks)
        if args.workload == "se_pile":
            return se_pile(args, ranks)
        if args.workload in ("disks_2d", "box_3d"):
            return config_line(args, ranks)
        return ours(args, ranks)
    finally:
        ranks.close()


def piles(args, ranks):
    """256 independent 2D pile scenes (200-5000 disks each, log-uniform) on a segment, all
    stepped by one batch handle: one CUDA graph replay and one persistent APGD launch per
    time step.  Steps 1..W warm up (graph capture), the next K are timed; with the
    defaults that is the whole 1000-step run."""
    import torch
    from scopi_b200 import FP64, MIXED, ScopiBatch, configs
    from scopi_b200.build import build
    build()
    st = configs.SETTINGS["pile_scenes"]
    scenes = configs.pile_scenes(256)
    kw = dict(dmax=st["dmax"], tolerance=st["tolerance"], max_ite=st["max_ite"])
    n_disks = sum(s.n - s.nb_inactive for s in scenes)

    def run(precision, sampler=None, steps=None, **extra):
        steps = steps or args.steps
        b = ScopiBatch(scenes, vap=st["vap"], precision=precision, device=ranks.local, mixed_violation_tol=1e-6,
                       **kw, **extra)
        b.run(st["dt"], args.warmup)
        stream = torch.cuda.ExternalStream(b.stream_handle(), device=ranks.local)
        torch.cuda.synchronize()
        ranks.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        l0 = b.kernel_launches()
        if sampler:
            sampler.start()
        viol, iters, contacts, conv = 0.0, [], [], True
        e0.record(stream)
        for _ in range(steps):
            b.run(st["dt"], 1)
            s = b.stats()
            viol = max(viol, s["violation"])
            iters.append(s["iterations"])
            contacts.append(s["contacts"])
            conv = conv and bool(s["converged"])
        e1.record(stream)
        e1.synchronize()
        clocks = sampler.stop() if sampler else None
        torch.cuda.synchronize()
        ranks.barrier()
        out = {"ms": ranks.max(e0.elapsed_time(e1)), "launches": b.kernel_launches() - l0, "clocks": clocks,
               "violation_max": viol, "longest_scene_iterations_mean": statistics.mean(iters),
               "contacts_mean": statistics.mean(contacts), "converged_all": conv, "block_threads": b.block_threads(),
               "tile": b.tile()}
        b.close()
        return out

    sampler = ClockSampler(ranks.local)
    mixed = run(MIXED, sampler)
    f64 = None if args.no_fp64 else run(FP64)
    abl = {}
    if not args.no_fp64:
        for name, prec, init in (("mixed_reference_start", MIXED, 0), ("fp64_curvature_start", FP64, 1)):
            r = run(prec, initial_step=init)
            abl[name] = {"value": ranks.world * args.steps * 1000.0 / r["ms"], "unit": UNIT,
                         "violation_max": r["violation_max"],
                         "longest_scene_iterations_mean": r["longest_scene_iterations_mean"]}
    # the same scenes with friction (mu 0.3; FP64, the 6-dof rows solved per scene), the first
    # 200 steps after the warm-up
    fr = None
    if not args.no_fp64:
        from scopi_b200 import FRICTION
        fsteps = min(args.steps, 200)
        r = run(FP64, steps=fsteps, problem=FRICTION, mu=0.3)
        fr = {"value": ranks.world * fsteps * 1000.0 / r["ms"], "unit": UNIT, "problem": "Friction, mu 0.3",
              "precision": "fp64", "steps": fsteps, "violation_max": r["violation_max"],
              "longest_scene_iterations_mean": r["longest_scene_iterations_mean"],
              "contacts_mean": r["contacts_mean"], "converged_all": r["converged_all"]}
    value = ranks.world * args.steps * 1000.0 / mixed["ms"]
    # the FP64 leg with the reference's first step stops its landing solves at violations
    # above 1e-6 (the reference's stopping rule); the FP64 leg that meets the bar is the one
    # with the curvature first step
    equal = None
    if abl.get("fp64_curvature_start"):
        fc = abl["fp64_curvature_start"]
        equal = {"fp64_leg": "fp64_curvature_start", "fp64_violation_max": fc["violation_max"],
                 "mixed_violation_max": mixed["violation_max"], "mixed_over_fp64": value / fc["value"]}
    line = {
        "metric": "time steps/s of 256 independent 2D pile scenes (one batch, violation <= 1e-6)",
        "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": mixed["ms"] / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 APGD iterations, f64 correction/geometry/integration", "data": "synthetic",
        "config": {"workload": (f"pile_scenes: 256 scenes, {n_disks:,} disks in all (N_s = round(exp(U[ln 200, "
                                f"ln 5000]))), r U[0.008,0.012], segment floor, gravity, NoFriction, vap_fpd, dmax "
                                f"0.009, dt 1e-3, per-scene APGD tol 1e-6, steps {args.warmup + 1}.."
                                f"{args.warmup + args.steps} of the run timed"),
                   "precision": "mixed", "l2": "working set L2-resident; latency-bound (one CTA per scene)",
                   "parallelism": f"replicas x{ranks.world}" if ranks.world > 1 else "single GPU"},
        "fp64": ({"value": ranks.world * args.steps * 1000.0 / f64["ms"], "unit": UNIT,
                  "mixed_over_fp64": f64["ms"] / mixed["ms"], "violation_max": f64["violation_max"],
                  "longest_scene_iterations_mean": f64["longest_scene_iterations_mean"],
                  "block_threads": f64["block_threads"]} if f64 else None),
        "ablation": abl or None,
        "at_equal_violation": equal,
        "friction": fr,
        "solver": {k: mixed[k] for k in ("violation_max", "longest_scene_iterations_mean", "contacts_mean",
                                        "converged_all", "block_threads", "tile")},
        "clocks": mixed["clocks"], "gpu_launches": mixed["launches"],
    }
    if ranks.rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def se_pile(args, ranks):
    """50,000 3D superellipsoids (semi-axes U[0.004, 0.008], squareness U[0.6, 1.4], random
    orientations) on a lattice above a floor, with friction (mu 0.3): the contact search
    keeps the pairs whose bounding spheres come within dmax, each pair's closest points are
    solved on the GPU (start grid + hybrid method), then the 6-dof friction problem."""
    import torch
    from scopi_b200 import FP64, FRICTION, MIXED, configs
    from scopi_b200.build import build
    build()
    st = configs.SETTINGS["se_pile"]
    pa = configs.se_pile(count=50_000)
    kd = configs.se_kd_radius(pa, st["dmax"])
    solver = (dict(dmax=st["dmax"], tolerance=st["tolerance"], max_ite=st["max_ite"], vap=st["vap"], mu=st["mu"],
                   problem=FRICTION, kd_tree_radius=kd), st["dt"])
    sampler = ClockSampler(ranks.local)
    mixed = time_path(pa, MIXED, args.steps, args.warmup, ranks, sampler, solver=solver)
    f64 = None if args.no_fp64 else time_path(pa, FP64, args.steps, args.warmup, ranks, solver=solver)
    value = ranks.world * args.steps * 1000.0 / ranks.max(mixed["ms"])
    per = mixed["per_step"]
    cpu = None
    if not args.no_cpu_baseline and ranks.rank == 0:
        threads = os.cpu_count() or 1
        its = statistics.mean(p["iterations"] for p in (f64["per_step"] if f64 else per))
        r = cpu_sample(pa, its, threads, solver=solver, caps=(3,))
        cpu = {"value": r["value"], "unit": UNIT, "cores": threads, "kind": "port",
               "sample": (f"oracle on one step of the 50k pile with APGD capped at 3 iterations ({r['wall_s']:.1f} s "
                          f"wall; contacts and closest points {r['t_outside_apgd_s']:.1f} s); steps/s = "
                          f"1/(t_outside_apgd + t_per_iteration * {its:.0f} FP64 iterations per step on the GPU)")}
    line = {
        "metric": "time steps/s, 50k superellipsoids with friction (mixed FP32-APGD + FP64 correction)",
        "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ranks.max(mixed["ms"]) / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 APGD iterations, f64 closest points/correction/integration",
        "data": "synthetic",
        "config": {"workload": ("se_pile: 50,000 superellipsoids, semi-axes U[0.004,0.008], e, n U[0.6,1.4], random "
                                "orientation, 37^3 lattice spacing 0.018 above a floor, gravity, Friction mu 0.3, "
                                f"dmax 0.004, dt 5e-4, steps {args.warmup + 1}..{args.warmup + args.steps} timed"),
                   "precision": "mixed", "parallelism": "single GPU"},
        "fp64": ({"value": ranks.world * args.steps * 1000.0 / ranks.max(f64["ms"]), "unit": UNIT,
                  "violation_max": max(p["violation"] for p in f64["per_step"]),
                  "iterations_per_step": statistics.mean(p["iterations"] for p in f64["per_step"])} if f64 else None),
        "solver": {"contacts": statistics.mean(p["contacts"] for p in per),
                   "violation_max": max(p["violation"] for p in per),
                   "fp32_iterations_per_step": statistics.mean(p["fp32_iterations"] for p in per),
                   "corrections_per_step": statistics.mean(p["corrections"] for p in per),
                   "converged_all": all(p["converged"] for p in per)},
        "cpu_baseline": cpu, "clocks": mixed["clocks"], "gpu_launches": mixed["launches"],
    }
    if ranks.rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def error_samples(pa, args, ranks):
    """Error of the mixed form against FP64 on the same step: at 3 sampled steps k of the
    timed window, the mixed trajectory's state before step k is solved once in FP64 and once
    in the mixed form; errors in lambda, velocities and gaps (d + dt n.(v_i - v_j))."""
    from scopi_b200 import FP64, MIXED, ScopiSolver
    from scopi_b200.errors import solve_errors
    kw, dt = solver_kwargs()
    nin = pa.nb_inactive
    steps = sorted({args.warmup + 1, args.warmup + max(1, args.steps // 2), args.warmup + args.steps})
    walker = ScopiSolver(pa, precision=MIXED, mixed_violation_tol=1e-6, device=ranks.local, **kw)
    done, out = 0, []
    for k in steps:
        if k - 1 > done:
            walker.step(dt, k - 1 - done)
            done = k - 1
        state = walker.sync().copy()
        recs = []
        for prec in (FP64, MIXED):
            s = ScopiSolver(state, precision=prec, mixed_violation_tol=1e-6, device=ranks.local, **kw).run(dt, 1)
            recs.append({"contacts": s.current_contacts(), "lambda": s.lagrange_multiplier(),
                         "v": s.particles.v.copy()})
            s.close()
        out.append({"step": k, **solve_errors(recs[0], recs[1], dt, nin)})
    walker.close()
    keys = ("lambda_rel", "lambda_max_abs", "v_rel", "v_max_abs", "gap_max_abs", "violation_ref", "violation_other")
    return {"steps": steps, **{k + "_max": max(o[k] for o in out) for k in keys},
            "definition": "same state, one FP64 and one mixed solve; gap = d + dt n.(v_i - v_j); rel = 2-norm",
            "samples": out}


def cpu_full_steps(pa, solver, threads, budget_s, max_steps):
    """The oracle stepped from the workload's initial state with the full APGD (no cap),
    one step at a time, until `budget_s` seconds of host time or `max_steps` steps."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import py_oracle as orc
    kw, dt = solver
    o = orc.OracleSolver(pa, **dict(kw, num_threads=threads))
    per, t0 = [], time.perf_counter()
    while len(per) < max_steps and time.perf_counter() - t0 < budget_s:
        t = time.perf_counter()
        o.run(dt, 1)
        per.append(time.perf_counter() - t)
    st = o.stats()
    del o
    return {"steps": len(per), "seconds": sum(per), "value": len(per) / sum(per), "per_step_s": per,
            "last_step_iterations": st["iterations"]}


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def gpu_steps_from_start(pa, precision, steps, solver, ranks):
    """Device time of steps 1..steps from the initial state (per-step CUDA events of the
    engine), to compare with a CPU sample over the same steps."""
    from scopi_b200 import ScopiSolver
    kw, dt = solver
    s = ScopiSolver(pa, precision=precision, mixed_violation_tol=1e-6, device=ranks.local, **kw)
    ms = 0.0
    for _ in range(steps):
        s.step(dt, 1)
        ms += s.stats()["ms_step"]
    s.close()
    return ms


def config_line(args, ranks):
    """Lines of the smaller configurations: disks_2d (1024 disks, 2D, 200 steps, plain FP64 is
    the configuration's own form) and box_3d (100,000 spheres in a box with 6 walls, gravity,
    vap_fpd, 500 steps, FP64 vs mixed).  The CPU baseline is the oracle's full steps (no APGD
    cap) from the initial state, on all host threads and on one, for as many steps as fit a
    time budget; the GPU is timed over the same steps beside it."""
    import torch  # noqa: F401
    from scopi_b200 import FP64, MIXED, configs
    from scopi_b200.build import build
    build()
    name = args.workload
    st = configs.SETTINGS[name]
    pa = configs.disks_2d() if name == "disks_2d" else configs.box_3d()
    solver = (dict(dmax=st["dmax"], tolerance=st["tolerance"], max_ite=st["max_ite"], vap=st["vap"]), st["dt"])
    n_active = pa.n - pa.nb_inactive
    sampler = ClockSampler(ranks.local)
    head_prec = FP64 if name == "disks_2d" else MIXED
    head = time_path(pa, head_prec, args.steps, args.warmup, ranks, sampler, solver=solver)
    other = None if args.no_fp64 else time_path(pa, MIXED if head_prec == FP64 else FP64, args.steps, args.warmup,
                                                  ranks, solver=solver)
    value = ranks.world * args.steps * 1000.0 / ranks.max(head["ms"])
    per = head["per_step"]
    cpu = None
    if not args.no_cpu_baseline and ranks.rank == 0:
        threads = os.cpu_count() or 1
        budget = args.cpu_budget
        full = cpu_full_steps(pa, solver, threads, budget, st["steps"])
        # the one-thread leg, unless a single step already takes more than 30 s (the APGD loop
        # is serial in the oracle as in the reference, so it costs the same again)
        one = (cpu_full_steps(pa, solver, 1, budget / 2, full["steps"]) if full["per_step_s"][0] <= 30.0
               else None)
        k = full["steps"]
        gpu_ms = {nm: gpu_steps_from_start(pa, prec, k, solver, ranks) for nm, prec in (("fp64", FP64),
                                                                                     ("mixed", MIXED))}
        cpu = {"value": full["value"], "unit": UNIT, "cores": threads, "kind": "port", "cpu_model": cpu_model(),
               "sample": (f"oracle (C++ restatement of the reference path: OpenMP where the reference has pragmas, "
                          f"serial APGD), full steps 1..{k} of the run from the initial state, no APGD cap, "
                          f"{full['seconds']:.1f} s on {threads} threads"),
               "one_thread": ({"value": one["value"], "steps": one["steps"], "seconds": one["seconds"]} if one
                              else "skipped: the first step alone takes more than 30 s"),
               "gpu_same_steps": {nm: k * 1000.0 / v for nm, v in gpu_ms.items()},
               "per_step_s": [round(x, 4) for x in full["per_step_s"]]}
    desc = {"disks_2d": ("disks_2d: 1024 disks (32x32 jittered grid, spacing 0.025, r U[0.008,0.012]), inward "
                         "desired velocity -0.25 (x-c)/|x-c|, NoFriction, vap_fixed, dmax 0.01, dt 0.005, APGD tol "
                         "1e-6, max_ite 40000"),
            "box_3d": ("box_3d: 100,000 spheres (47^3 jittered lattice, spacing 0.0115, r U[0.9,1.1]*0.005) + 6 "
                       "plane walls, gravity, NoFriction, vap_fpd, dmax 0.0045, dt 1e-3, APGD tol 1e-6")}[name]
    line = {
        "metric": f"time steps/s, {name} ({'plain FP64' if head_prec == FP64 else 'mixed FP32-APGD + FP64 correction'})",
        "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ranks.max(head["ms"]) / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if head_prec == FP64 else "f32 APGD iterations, f64 elsewhere",
        "data": "synthetic",
        "config": {"workload": desc + f", steps {args.warmup + 1}..{args.warmup + args.steps} timed",
                   "precision": "fp64" if head_prec == FP64 else "mixed", "bodies": n_active,
                   "parallelism": "single GPU", "l2": "working set L2-resident" if name == "disks_2d" else
                   "contact arrays ~50 MB per step (L2-resident between kernels)"},
        ("mixed" if head_prec == FP64 else "fp64"): ({
            "value": ranks.world * args.steps * 1000.0 / ranks.max(other["ms"]), "unit": UNIT,
            "violation_max": max(p["violation"] for p in other["per_step"]),
            "iterations_per_step": statistics.mean(p["iterations"] for p in other["per_step"])} if other else None),
        "solver": {"contacts": statistics.mean(p["contacts"] for p in per),
                   "violation_max": max(p["violation"] for p in per),
                   "iterations_per_step": statistics.mean(p["iterations"] for p in per),
                   "converged_all": all(p["converged"] for p in per)},
        "cpu_baseline": cpu, "clocks": head["clocks"], "gpu_launches": head["launches"],
    }
    if ranks.rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def ours(args, ranks):
    import torch
    if not torch.cuda.is_available():
        print(json.dumps({"error": "no CUDA device"}))
        return 1
    from scopi_b200 import FP64, MIXED, VISCOUS, configs
    from scopi_b200.build import build
    build()
    pa = configs.spheres_1m(side=args.side)
    n_active = pa.n - pa.nb_inactive
    sampler = ClockSampler(ranks.local)
    mixed = time_path(pa, MIXED, args.steps, args.warmup, ranks, sampler)
    f64 = None if args.no_fp64 else time_path(pa, FP64, args.steps, args.warmup, ranks)
    # ablation: the two changes of the mixed form taken one at a time (FP32 iterations with
    # the reference's first step; the curvature first step alone in FP64)
    abl = {}
    if not args.no_fp64:
        for name, prec, init in (("mixed_reference_start", MIXED, 0), ("fp64_curvature_start", FP64, 1)):
            r = time_path(pa, prec, args.steps, args.warmup, ranks, initial_step=init)
            its = [p["fp32_iterations"] if prec == MIXED else p["iterations"] for p in r["per_step"]]
            abl[name] = {"value": ranks.world * args.steps * 1000.0 / ranks.max(r["ms"]), "unit": UNIT,
                         "iterations_per_step": statistics.mean(its),
                         "violation_max": max(p["violation"] for p in r["per_step"])}
    e2e_ms, h2d, d2h = time_e2e(pa, MIXED, args.steps, args.warmup, ranks)
    e2e_full_ms, h2d_full, _ = time_e2e(pa, MIXED, args.steps, args.warmup, ranks, full_upload=True)
    # ViscousWithoutFriction on the same workload (gamma defaults 0 / -2 / 1e-6)
    visc = None
    if not args.no_viscous:
        vm = time_path(pa, MIXED, args.steps, args.warmup, ranks, problem=VISCOUS)
        vf = None if args.no_fp64 else time_path(pa, FP64, args.steps, args.warmup, ranks, problem=VISCOUS)
        vm_val = ranks.world * args.steps * 1000.0 / ranks.max(vm["ms"])
        visc = {"value": vm_val, "unit": UNIT, "problem": "ViscousWithoutFriction",
                "violation_max": max(p["violation"] for p in vm["per_step"]),
                "fp32_iterations_per_step": statistics.mean(p["fp32_iterations"] for p in vm["per_step"]),
                "fp64": ({"value": ranks.world * args.steps * 1000.0 / ranks.max(vf["ms"]), "unit": UNIT,
                          "violation_max": max(p["violation"] for p in vf["per_step"]),
                          "iterations_per_step": statistics.mean(p["iterations"] for p in vf["per_step"])}
                         if vf else None)}
        if vf:
            visc["mixed_over_fp64"] = vm_val / visc["fp64"]["value"]
    errs = None if (args.no_fp64 or args.no_errors) else error_samples(pa, args, ranks)

    ms = ranks.max(mixed["ms"])
    value = args.gpus * args.steps * 1000.0 / ms if ranks.world > 1 else args.steps * 1000.0 / ms
    e2e_ms = ranks.max(e2e_ms)
    e2e_val = (ranks.world * args.steps * 1000.0 / e2e_ms)
    e2e_full_val = (ranks.world * args.steps * 1000.0 / ranks.max(e2e_full_ms))
    f64_val = None
    if f64:
        f64_ms = ranks.max(f64["ms"])
        f64_val = ranks.world * args.steps * 1000.0 / f64_ms

    # roofline of the dominant kernel: the persistent APGD launches (FP32 in the mixed form)
    per = mixed["per_step"]
    C = statistics.mean(p["contacts"] for p in per)
    it32 = sum(p["fp32_iterations"] for p in per)
    ms_apgd = sum(p["ms_apgd_kernel"] for p in per)
    # headline bytes: what the torque-free iteration must move (normal only, translational
    # slots); the full-row formula (9 values per contact, 6N slots, a third pass over B)
    # counts six identically zero values per row and a pass the fused iteration never makes
    b_iter32 = roofline_bytes_per_iter(C, n_active, 4, torque_free=True)
    b_iter32_full = roofline_bytes_per_iter(C, n_active, 4)
    achieved = (it32 * b_iter32) / (ms_apgd * 1e-3) / 1e9 if ms_apgd > 0 else None
    achieved_full = (it32 * b_iter32_full) / (ms_apgd * 1e-3) / 1e9 if ms_apgd > 0 else None
    peak, peak_kind = measured_peaks()
    # DRAM bytes of one APGD launch (one whole solve): ncu dram__bytes_read.sum +
    # dram__bytes_write.sum per FP32 iteration per contact, times this run's contacts and
    # iterations per launch
    traffic = (TRAFFIC_FP32_PER_CONTACT_ITERATION * C * it32 / max(1, len(per))
               if it32 and TRAFFIC_FP32_PER_CONTACT_ITERATION else None)
    f64_roof = None
    if f64:
        p64 = f64["per_step"]
        it64 = sum(p["iterations"] for p in p64)
        ms64 = sum(p["ms_apgd_kernel"] for p in p64)
        a64 = ((it64 * roofline_bytes_per_iter(C, n_active, 8, torque_free=True)) / (ms64 * 1e-3) / 1e9
               if ms64 > 0 else None)
        a64_full = (it64 * roofline_bytes_per_iter(C, n_active, 8)) / (ms64 * 1e-3) / 1e9 if ms64 > 0 else None
        f64_roof = {"achieved": a64, "peak": peak, "unit": "GB/s", "frac": (a64 / peak) if a64 else None,
                    "achieved_formula_full_rows": a64_full,
                    "frac_formula_full_rows": (a64_full / peak) if a64_full else None,
                    "iterations_per_step": it64 / len(p64), "ms_apgd_per_step": ms64 / len(p64),
                    "violation_max": max(p["violation"] for p in p64)}

    cpu = None
    if not args.no_cpu_baseline and ranks.rank == 0 and args.side == 100:
        iters = (f64_roof["iterations_per_step"] if f64_roof else
                 reference_iterations(args.warmup + 1, args.warmup + args.steps)[0])
        threads = os.cpu_count() or 1
        # caps 1 and 20: the 19-iteration difference gives the steady-state cost of an iteration
        # (a full uncapped oracle step of 471 iterations measured 1.521 s per iteration on an
        # 8-core host where the 1-to-20 difference gave 1.521 s and the 1-to-3 difference 1.58-1.70 s)
        r = cpu_sample(pa, iters, threads, caps=(1, 20))
        cpu = {"value": r["value"], "unit": UNIT, "cores": threads, "kind": "port", "extrapolated": True,
               "cpu_model": cpu_model(),
               "sample": (f"oracle on the full 1M-sphere step, APGD capped at 1 and 20 iterations "
                          f"({r['wall_s']:.1f} s wall); steps/s = 1/(t_outside_apgd "
                          f"{r['t_outside_apgd_s']:.2f} s + t_per_iteration {r['t_per_iteration_s']:.3f} s * "
                          f"{iters:.0f} FP64 iterations per step measured on the GPU)"),
               "t_per_iteration_s": r["t_per_iteration_s"], "t_outside_apgd_s": r["t_outside_apgd_s"]}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 APGD iterations, f64 correction/geometry/integration",
        "data": "synthetic",
        "config": {"workload": (f"{WORKLOAD}: {n_active:,} spheres ({args.side}^3 jittered lattice, spacing 0.0045, "
                                f"r U[0.9,1.1]*0.002) + 6 plane walls, NoFriction, vap_fixed, dmax 0.0018, dt 1e-3, "
                                f"APGD tol 1e-6, mixed violation target 1e-6"),
                   "precision": "mixed", "l2": "inputs larger than L2 (contact arrays > 1 GB per step)",
                   "parallelism": f"replicas x{ranks.world}" if ranks.world > 1 else "single GPU"},
        "fp64": {"value": f64_val, "unit": UNIT, "mixed_over_fp64": (value / f64_val) if f64_val else None,
                 "roofline": f64_roof},
        "ablation": abl or None,
        "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "upload": "scopi_gpu_set_state (pos, q, v, omega), step, scopi_gpu_get_particles",
                "full_container": {"value": e2e_full_val, "unit": UNIT, "h2d_bytes_per_step": h2d_full,
                                   "d2h_bytes_per_step": d2h,
                                   "upload": "scopi_gpu_set_particles (all 13 fields), step, "
                                             "scopi_gpu_get_particles"}},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                     "peak_source": f"{peak_kind} hbm_gbs",
                     "kernel": "k_apgd_sph<float,3,NoFriction> (persistent, torque-free rows)",
                     "bytes_per_iteration": b_iter32,
                     "bytes_definition": "3C(3s+8) + 6Cs + 4(3N)s: normal-only rows, translational slots",
                     "achieved_formula_full_rows": achieved_full,
                     "frac_formula_full_rows": (achieved_full / peak) if achieved_full else None,
                     "bytes_per_iteration_formula_full_rows": b_iter32_full,
                     "traffic_source": TRAFFIC_SOURCE,
                     "traffic_per_iteration": (traffic / (it32 / len(per))) if traffic else None,
                     "iterations_per_step": it32 / len(per),
                     "ms_apgd_per_step": ms_apgd / len(per)},
        "cpu_baseline": cpu,
        "viscous": visc,
        "error_vs_fp64": errs,
        "clocks": mixed["clocks"],
        "gpu_launches": mixed["launches"],
        "solver": {"contacts": C, "violation_max": max(p["violation"] for p in per),
                   "corrections_per_step": sum(p["corrections"] for p in per) / len(per),
                   "converged_all": all(p["converged"] for p in per)},
    }
    if ranks.rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
