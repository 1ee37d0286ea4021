"""Run time steps of a synthetic workload on the GPU and print per-step solver statistics.

    python -m scopi_b200.run_steps --workload spheres --side 60 --precision fp64 --steps 2

Workloads: spheres (jittered cubic lattice, scopi_b200.configs.spheres_1m with `side`^3
spheres), box (configs.box_3d with `count` spheres), disks (configs.disks_2d), piles
(`scenes` pile scenes of configs.pile_scenes stepped as one batch; `vmax` > 0 starts the
disks with random velocities so the first steps have active constraints).  Used as the
driver of the ncu captures summarised under profiles/.
"""
from __future__ import annotations

import argparse
import json

from . import FP64, FRICTION, MIXED, NOFRICTION, VISCOUS, ScopiBatch, ScopiSolver, configs


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="spheres", choices=["spheres", "box", "disks", "piles", "se"])
    ap.add_argument("--scenes", type=int, default=256)
    ap.add_argument("--vmax", type=float, default=0.0)
    ap.add_argument("--block-threads", type=int, default=0)
    ap.add_argument("--initial-step", type=int, default=-1, choices=[-1, 0, 1])
    ap.add_argument("--side", type=int, default=100)
    ap.add_argument("--count", type=int, default=100_000)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--problem", default="nofriction", choices=["nofriction", "viscous"])
    ap.add_argument("--steps", type=int, default=2)
    a = ap.parse_args(argv)
    if a.workload == "piles":
        st = configs.SETTINGS["pile_scenes"]
        b = ScopiBatch(configs.pile_scenes(a.scenes, vmax=a.vmax), vap=st["vap"],
                       precision=FP64 if a.precision == "fp64" else MIXED, block_threads=a.block_threads,
                       initial_step=a.initial_step, dmax=st["dmax"], tolerance=st["tolerance"], max_ite=st["max_ite"])
        for k in range(a.steps):
            b.run(st["dt"], 1)
            print(json.dumps({"step": k, "block_threads": b.block_threads(), **b.stats()}), flush=True)
        b.close()
        return
    extra = {}
    if a.workload == "se":
        # superellipsoid pile with friction (configs.se_pile with `count` bodies)
        pa, st = configs.se_pile(count=a.count), configs.SETTINGS["se_pile"]
        extra = dict(mu=st["mu"], kd_tree_radius=configs.se_kd_radius(pa, st["dmax"]))
    elif a.workload == "spheres":
        pa, st = configs.spheres_1m(side=a.side), configs.SETTINGS["spheres_1m"]
    elif a.workload == "box":
        pa, st = configs.box_3d(count=a.count), configs.SETTINGS["box_3d"]
    else:
        pa, st = configs.disks_2d(side=a.side if a.side != 100 else 32), configs.SETTINGS["disks_2d"]
    problem = VISCOUS if a.problem == "viscous" else NOFRICTION
    if a.workload == "se":
        problem = FRICTION
    s = ScopiSolver(pa, precision=FP64 if a.precision == "fp64" else MIXED, problem=problem, **extra,
                    initial_step=a.initial_step, dmax=st["dmax"], tolerance=st["tolerance"], max_ite=st["max_ite"],
                    vap=st["vap"])
    for k in range(a.steps):
        s.step(st["dt"], 1)
        print(json.dumps({"step": k, **s.stats()}), flush=True)
    s.close()


if __name__ == "__main__":
    main()
