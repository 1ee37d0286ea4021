"""Host-side error statements (scopi_b200.errors) checked against the oracle's own solves.

normal_kkt must find the oracle's FP64 NoFriction solve optimal: v = U + dt M^-1 B^T lambda to
rounding, lambda >= 0, no negative gap beyond the solver's accuracy, zero gap on the
contacts that carry force.  solve_errors of a solve against itself is zero, and against a
perturbed copy reports the perturbation.
"""
import numpy as np
import pytest

import py_oracle as orc
from scopi_b200 import configs
from scopi_b200.errors import normal_kkt, solve_errors, step_gaps


@pytest.mark.parametrize("name", ["spheres_1m", "box_3d"])
def test_normal_kkt_of_oracle_solve(name):
    pa = configs.spheres_1m(side=10) if name == "spheres_1m" else configs.box_3d(count=2000)
    st = configs.SETTINGS[name]
    kw = dict(dmax=st["dmax"], tolerance=st["tolerance"], max_ite=st["max_ite"], vap=st["vap"])
    o = orc.OracleSolver(pa, **kw).run(st["dt"], 1)
    nin = pa.nb_inactive
    U = pa.vd.copy() if st["vap"] == 0 else pa.v + st["dt"] * pa.f / pa.m[:, None]
    k = normal_kkt(o.contacts(), o.lagrange_multiplier(), o.pa.v, U, 1.0 / pa.m[nin:], st["dt"], nin)
    assert k["active"] > 0
    assert k["v_consistency"] <= 1e-14, k
    assert k["lambda_min"] >= 0.0
    assert k["violation"] <= 1e-9 and k["stationarity"] <= 1e-9, k
    # the violation agrees with the oracle's own report
    assert abs(k["violation"] - o.stats()["violation"]) <= 1e-12
    rec = {"contacts": o.contacts(), "lambda": o.lagrange_multiplier(), "v": o.pa.v.copy()}
    assert solve_errors(rec, rec, st["dt"], nin)["gap_max_abs"] == 0.0
    pert = dict(rec, v=rec["v"].copy())
    pert["v"][nin:] += 1e-3
    e = solve_errors(rec, pert, st["dt"], nin)
    assert e["v_max_abs"] == pytest.approx(1e-3, rel=1e-9)
    g = step_gaps(rec["contacts"], rec["v"], st["dt"], nin)
    assert np.all(np.isfinite(g))
