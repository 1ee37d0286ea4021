"""Parity at the workloads' full sizes: 1,000,000 spheres in the unit box and the
100,000-sphere box under gravity (vap_fpd).

* Contact lists: GPU and oracle bit for bit (pairs in (i, j) order, dij, nij, pi, pj), on the
  initial state and on the state the GPU reaches after a few steps (fed to both).
* Solves: at these sizes the oracle's serial APGD takes minutes per step, so the FP64 GPU
  multipliers are checked by the optimality conditions of the contact QP, evaluated in
  FP64 on the host from the step's own contact list (a size-independent property):
  lambda >= 0, no gap below zero, zero gap wherever lambda > 0, and v = U + dt M^-1 B^T lambda.
  The 100k box's later steps (one-iteration solves) run on both engines from the GPU's state.
* Mixed precision: its error against the FP64 solve of the same step, in lambda, velocities
  and gaps, stated and bounded; its violation at most the 1e-6 target.
* Viscous at 1M: FP64 and mixed trajectories agree and meet the violation target.
"""
import numpy as np
import pytest

from gpu_helpers import gpu_solver, oracle_solver, rel_err, same_contacts
from scopi_b200 import configs
from scopi_b200.errors import normal_kkt, solve_errors

pytestmark = pytest.mark.gpu

MIXED, FP64, VISCOUS = 1, 0, 2


def _kw(name):
    st = configs.SETTINGS[name]
    return dict(dmax=st["dmax"], tolerance=st["tolerance"], max_ite=st["max_ite"], vap=st["vap"]), st["dt"]


def _solve_record(s):
    return {"contacts": s.current_contacts(), "lambda": s.lagrange_multiplier(), "v": s.particles.v.copy()}


@pytest.fixture(scope="module")
def spheres_1m():
    return configs.spheres_1m()


@pytest.fixture(scope="module")
def box_100k():
    return configs.box_3d()


def _detect_pair(pa, kw):
    g = gpu_solver(pa, **kw)
    gc = g.detect()
    g.close()
    oc = oracle_solver(pa, **kw).detect()
    return gc, oc


def test_contacts_bitexact_spheres_1m(spheres_1m):
    kw, dt = _kw("spheres_1m")
    gc, oc = _detect_pair(spheres_1m, kw)
    assert len(oc["i"]) > 2_500_000
    same_contacts(gc, oc)
    # after three steps of the mixed form (the benchmarked one), from the GPU's state
    g = gpu_solver(spheres_1m, precision=MIXED, mixed_violation_tol=1e-6, **kw).run(dt, 3)
    state = g.particles.copy()
    g.close()
    gc, oc = _detect_pair(state, kw)
    same_contacts(gc, oc)


def test_contacts_bitexact_box_100k(box_100k):
    kw, dt = _kw("box_3d")
    gc, oc = _detect_pair(box_100k, kw)
    assert len(oc["i"]) > 250_000
    same_contacts(gc, oc)
    g = gpu_solver(box_100k, **kw).run(dt, 3)
    state = g.particles.copy()
    g.close()
    gc, oc = _detect_pair(state, kw)
    same_contacts(gc, oc)


def test_fp64_solve_optimal_and_mixed_error_spheres_1m(spheres_1m):
    """The FP64 step meets the QP's optimality conditions; the mixed step's error against it."""
    kw, dt = _kw("spheres_1m")
    pa = spheres_1m
    nin = pa.nb_inactive
    f64 = gpu_solver(pa, **kw).run(dt, 1)
    ref = _solve_record(f64)
    U = pa.vd.copy()  # vap_fixed: the a-priori velocity is the desired one
    kkt = normal_kkt(ref["contacts"], ref["lambda"], ref["v"], U, 1.0 / pa.m[nin:], dt, nin)
    print("FP64 optimality at 1M:", kkt)
    assert kkt["v_consistency"] <= 1e-12, kkt
    assert kkt["lambda_min"] >= 0.0, kkt
    assert kkt["violation"] <= 1e-8, kkt
    assert kkt["stationarity"] <= 1e-8, kkt
    f64.close()
    mix = gpu_solver(pa, precision=MIXED, mixed_violation_tol=1e-6, **kw).run(dt, 1)
    err = solve_errors(ref, _solve_record(mix), dt, nin)
    print("mixed vs FP64 at 1M:", err)
    assert err["violation_other"] <= 1e-6, err
    assert err["gap_max_abs"] <= 2e-6, err
    assert err["v_rel"] <= 1e-5, err
    mix.close()


def test_fp64_box_100k_optimal_then_steps_match_oracle(box_100k):
    """First step: optimality of the FP64 multipliers (the oracle's serial APGD needs minutes
    here).  Next two steps: GPU and oracle stepped from the GPU's state agree."""
    kw, dt = _kw("box_3d")
    pa = box_100k
    nin = pa.nb_inactive
    g = gpu_solver(pa, **kw).run(dt, 1)
    rec = _solve_record(g)
    U = pa.v + dt * pa.f / pa.m[:, None]  # vap_fpd on spheres (no rotation)
    kkt = normal_kkt(rec["contacts"], rec["lambda"], rec["v"], U, 1.0 / pa.m[nin:], dt, nin)
    print("FP64 optimality at 100k:", kkt)
    assert kkt["v_consistency"] <= 1e-12, kkt
    assert kkt["lambda_min"] >= 0.0, kkt
    assert kkt["violation"] <= 1e-8, kkt
    assert kkt["stationarity"] <= 1e-8, kkt
    state = g.particles.copy()
    g.close()
    g = gpu_solver(state, **kw)
    o = oracle_solver(state, **kw)
    for k in range(2):
        g.run(dt, 1)
        o.run(dt, 1)
        gc, oc = g.current_contacts(), o.contacts()
        assert np.array_equal(gc["i"], oc["i"]) and np.array_equal(gc["j"], oc["j"]), k
        assert rel_err(g.particles.pos, o.pa.pos) <= 1e-9, k
        assert rel_err(g.particles.v, o.pa.v) <= 1e-7, k
        assert rel_err(g.lagrange_multiplier(), o.lagrange_multiplier()) <= 1e-6, k
    g.close()


def test_viscous_spheres_1m_mixed_and_fp64(spheres_1m):
    """ViscousWithoutFriction at 1M (gamma defaults 0 / -2 / 1e-6): three steps in FP64 and in
    the mixed form from the same state; both meet the violation target, the contact lists
    agree pair for pair and the trajectories within 1e-7."""
    kw, dt = _kw("spheres_1m")
    f64 = gpu_solver(spheres_1m, problem=VISCOUS, **kw)
    mix = gpu_solver(spheres_1m, problem=VISCOUS, precision=MIXED, mixed_violation_tol=1e-6, **kw)
    viscous_rows = 0
    for k in range(3):
        f64.run(dt, 1)
        mix.run(dt, 1)
        sf, sm = f64.stats(), mix.stats()
        assert sf["violation"] <= 1e-6 and sm["violation"] <= 1e-6, (k, sf, sm)
        cf, cm = f64.current_contacts(), mix.current_contacts()
        assert np.array_equal(cf["i"], cm["i"]) and np.array_equal(cf["j"], cm["j"]), k
        viscous_rows = len(f64.lagrange_multiplier()) - len(cf["i"])
    assert viscous_rows > 0  # some contacts carry the second (viscous) multiplier by step 3
    assert rel_err(mix.particles.pos, f64.particles.pos) <= 1e-7
    assert rel_err(mix.particles.v, f64.particles.v) <= 1e-4
    f64.close()
    mix.close()
