"""Run time steps of a synthetic workload on the GPU and print per-step solver statistics.

    python -m scopi_b200.run_steps --workload spheres --side 60 --precision fp64 --steps 2

Workloads: spheres (jittered cubic lattice, scopi_b200.configs.spheres_1m with `side`^3
spheres), box (configs.box_3d with `count` spheres), disks (configs.disks_2d).  Used as
the driver of the ncu captures summarised under profiles/.
"""
from __future__ import annotations

import argparse
import json

from . import FP64, MIXED, VISCOUS, NOFRICTION, ScopiSolver, configs


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="spheres", choices=["spheres", "box", "disks"])
    ap.add_argument("--side", type=int, default=100)
    ap.add_argument("--count", type=int, default=100_000)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--problem", default="nofriction", choices=["nofriction", "viscous"])
    ap.add_argument("--steps", type=int, default=2)
    a = ap.parse_args(argv)
    if a.workload == "spheres":
        pa, st = configs.spheres_1m(side=a.side), configs.SETTINGS["spheres_1m"]
    elif a.workload == "box":
        pa, st = configs.box_3d(count=a.count), configs.SETTINGS["box_3d"]
    else:
        pa, st = configs.disks_2d(side=a.side if a.side != 100 else 32), configs.SETTINGS["disks_2d"]
    s = ScopiSolver(pa, precision=FP64 if a.precision == "fp64" else MIXED,
                    problem=VISCOUS if a.problem == "viscous" else NOFRICTION,
                    dmax=st["dmax"], tolerance=st["tolerance"], max_ite=st["max_ite"], vap=st["vap"])
    for k in range(a.steps):
        s.step(st["dt"], 1)
        print(json.dumps({"step": k, **s.stats()}), flush=True)
    s.close()


if __name__ == "__main__":
    main()
